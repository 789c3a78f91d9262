// Pipeline construction and per-launch preparation.
#include "ml_pipeline.hpp"
#include "ml_jit.hpp"

#include <algorithm>
#include <cstring>

namespace mlg {

uint32_t StringIntern::id(const std::string& s) {
    auto it = ids.find(s);
    if (it != ids.end()) return it->second;
    uint32_t v = (uint32_t)strs.size();
    ids.emplace(s, v);
    strs.push_back(s);
    return v;
}

static int key_width(int t) {
    switch (t) {
        case ML_TYPE_BOOL: return 8;
        case ML_TYPE_INT32:
        case ML_TYPE_DATE:
        case ML_TYPE_UTF8: return 32;
        default: return 64;
    }
}

// Field placement depends only on the key types, so a join's build and probe sides
// (whose key types are equal) always produce identical normalized keys.
static void place_fields(KeyLayout& L, const std::vector<int>& types) {
    int word = 0, used = 0;
    for (size_t k = 0; k < types.size(); k++) {
        int w = key_width(types[k]);
        if (used + w > 64) {
            word++;
            used = 0;
        }
        if (word >= kKeyWords) raise(ML_ERR_UNSUPPORTED, "key tuple wider than 128 bits on the GPU");
        L.f[k].word = (int8_t)word;
        L.f[k].shift = (int8_t)used;
        L.f[k].width = (int8_t)w;
        L.f[k].type = (int8_t)types[k];
        L.f[k].strid = types[k] == ML_TYPE_UTF8;
        used += w;
    }
    L.nkeys = (int)types.size();
    L.nwords = word + 1;
}

KeyLayout Pipeline::key_layout(const ml_expr* exprs, int n, const Schema& schema, bool group, std::vector<KeyDecode>* dec) {
    if (n > kMaxKeys) raise(ML_ERR_UNSUPPORTED, "more than 4 key expressions on the GPU");
    KeyLayout L{};
    std::vector<int> types;
    for (int k = 0; k < n; k++) types.push_back(exprs[k].dtype);
    place_fields(L, types);
    for (int k = 0; k < n; k++) {
        ExprNode e = parse_expr(exprs[k]);
        KeyDecode d;
        d.type = types[k];
        if (types[k] == ML_TYPE_UTF8) {
            int slot;
            L.prog[k] = C.compile_string_key(e, schema, &slot);
            d.slot = slot;
            const SlotInfo& si = C.slots[slot];
            // join keys compare the context's global string ids, which the source's columns carry
            // (a build side's strings carry canonical build rows instead)
            if (!group && si.src != 0)
                raise(ML_ERR_UNSUPPORTED, "a string join key read from an earlier join's build side on the GPU");
            if (si.src == 0) {
                d.str_kind = 1;
            } else {
                d.str_kind = 2;
                d.build = si.src - 1;
                d.build_col = si.index;
            }
        } else {
            L.prog[k] = C.compile_value(e, schema, types[k]);
        }
        if (dec) dec->push_back(d);
    }
    return L;
}

DevBuf Pipeline::intern_plain_strings(const DevColumn& col, cudaStream_t s) {
    const int64_t n = col.n;
    DevBuf ids(ctx, std::max<size_t>((size_t)n * 4, 4), nullptr);
    if (n == 0) return ids;
    // canonical rows: equal strings of the batch share one row (a device hash table of strings)
    const uint64_t cap = std::max<uint64_t>(16, 1ull << (64 - __builtin_clzll((uint64_t)n * 2)));
    DevBuf tslots(ctx, cap * 16, nullptr), canon(ctx, (size_t)n * 4, nullptr), err(ctx, 8, nullptr);
    CK(cudaMemsetAsync(tslots.get(), 0, cap * 16, s));
    CK(cudaMemsetAsync(err.get(), 0, 4, s));
    TableView tv{tslots.get<uint64_t>(), cap - 1, 1, 2};
    launch_strid(col.optr(), (const uint8_t*)col.dptr(), col.vptr(), n, tv, canon.get<uint32_t>(), err.get<uint32_t>(), s);
    ctx->count_launch();
    std::vector<uint32_t> canon_h(n), off(n + 1), ids_h(n, 0);
    uint32_t err_h = 0;
    CK(cudaMemcpyAsync(canon_h.data(), canon.get(), (size_t)n * 4, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(off.data(), col.optr(), (size_t)(n + 1) * 4, cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&err_h, err.get(), 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (err_h) raise(ML_ERR_TIMEOUT, "a bounded wait ran out while hashing a string key column");
    std::vector<uint8_t> bytes(off[n] - off[0]);
    if (!bytes.empty())
        CK(cudaMemcpyAsync(bytes.data(), (const uint8_t*)col.dptr() + off[0], bytes.size(), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    {
        std::lock_guard<std::mutex> g(intern.mu);
        for (int64_t r = 0; r < n; r++)
            if (canon_h[r] == (uint32_t)r)
                ids_h[r] = intern.id(std::string((const char*)bytes.data() + (off[r] - off[0]), off[r + 1] - off[r]));
    }
    for (int64_t r = 0; r < n; r++) ids_h[r] = ids_h[canon_h[r] < (uint64_t)n ? canon_h[r] : r];
    CK(cudaMemcpyAsync(ids.get(), ids_h.data(), (size_t)n * 4, cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));  // the host vector goes out of scope
    return ids;
}

void Pipeline::build(const ml_pipe_op* ops, int nops, const int32_t* types, int ntypes) {
    if (ntypes < 0 || (ntypes > 0 && !types)) raise(ML_ERR_INVALID, "bad input types");
    input_types.assign(types, types + ntypes);
    out.clear();
    for (int i = 0; i < ntypes; i++) {
        if (types[i] < 0 || types[i] > ML_TYPE_UTF8) raise(ML_ERR_INVALID, "bad input type");
        ColRef r;
        r.kind = 0;
        r.src = 0;
        r.index = i;
        r.dtype = types[i];
        out.push_back(r);
    }
    if (nops < 0 || (nops > 0 && !ops)) raise(ML_ERR_INVALID, "bad prologue");
    for (int o = 0; o < nops; o++) {
        const ml_pipe_op& op = ops[o];
        if (op.nexprs < 0 || (op.nexprs > 0 && !op.exprs)) raise(ML_ERR_INVALID, "operator without expressions");
        switch (op.kind) {
            case ML_PIPE_FILTER: {  // filter.rs:19-25
                if (op.nexprs != 1) raise(ML_ERR_INVALID, "filter takes one predicate");
                if ((int)filters.size() >= kMaxFilters || nstages >= kMaxFilters + kMaxProbes)
                    raise(ML_ERR_UNSUPPORTED, "too many filters in one pipeline");
                filters.push_back(C.compile_value(parse_expr(op.exprs[0]), out, ML_TYPE_BOOL));
                stages[nstages++] = Stage{0, (int8_t)(filters.size() - 1)};
                break;
            }
            case ML_PIPE_PROJECT: {  // projection.rs:21-32: expressions over the input
                auto env = std::make_shared<Schema>(out);
                Schema next;
                for (int k = 0; k < op.nexprs; k++) {
                    auto e = std::make_shared<ExprNode>(parse_expr(op.exprs[k]));
                    if (e->kind == ML_EXPR_COLUMN) {
                        if (e->index < 0 || (size_t)e->index >= env->size()) raise(ML_ERR_INVALID, "projection column missing");
                        ColRef r = (*env)[e->index];
                        if (r.dtype != op.exprs[k].dtype && r.kind != 2) {
                            ColRef c;
                            c.kind = 2;
                            c.dtype = op.exprs[k].dtype;
                            c.expr = std::make_shared<ExprNode>();
                            c.expr->kind = ML_EXPR_CAST;
                            c.expr->dtype = op.exprs[k].dtype;
                            c.expr->kids.push_back(*e);
                            c.env = env;
                            next.push_back(c);
                        } else {
                            next.push_back(r);
                        }
                        continue;
                    }
                    ColRef c;
                    c.kind = 2;
                    c.dtype = op.exprs[k].dtype;
                    if (op.exprs[k].dtype != ML_TYPE_UTF8) {  // evaluate_to_column's cast to the output type
                        c.expr = std::make_shared<ExprNode>();
                        c.expr->kind = ML_EXPR_CAST;
                        c.expr->dtype = op.exprs[k].dtype;
                        c.expr->kids.push_back(*e);
                    } else {
                        c.expr = e;
                    }
                    c.env = env;
                    next.push_back(c);
                }
                out = next;
                break;
            }
            case ML_PIPE_PROBE: {  // join.rs:263-337
                if ((int)probes.size() >= kMaxProbes) raise(ML_ERR_UNSUPPORTED, "more than 4 probes in one pipeline");
                if (!op.join) raise(ML_ERR_INVALID, "probe without a join table");
                ml_join_table* jt = op.join;
                if ((int)jt->key_types.size() != op.nexprs) raise(ML_ERR_INVALID, "probe key count differs from the build");
                for (int k = 0; k < op.nexprs; k++)
                    if (op.exprs[k].dtype != jt->key_types[k]) raise(ML_ERR_INVALID, "probe key type differs from the build");
                ProbeInfo pi;
                pi.jt = jt;
                pi.keys = key_layout(op.exprs, op.nexprs, out, false, nullptr);
                probes.push_back(pi);
                int p = (int)probes.size() - 1;
                stages[nstages++] = Stage{1, (int8_t)p};
                Schema bcols;
                for (size_t j = 0; j < jt->batch.cols.size(); j++) {
                    ColRef r;
                    r.kind = 1;
                    r.src = p + 1;
                    r.index = (int)j;
                    r.dtype = jt->batch.cols[j]->dtype;
                    bcols.push_back(r);
                }
                Schema next;
                if (op.build_is_left) {
                    next = bcols;
                    next.insert(next.end(), out.begin(), out.end());
                } else {
                    next = out;
                    next.insert(next.end(), bcols.begin(), bcols.end());
                }
                out = next;
                break;
            }
            default: raise(ML_ERR_INVALID, "bad pipeline operator");
        }
    }
}

void Pipeline::upload() {
    const size_t pb = (std::max<size_t>(C.code.size() * sizeof(Instr), 32) + 255) & ~(size_t)255;
    const size_t ab = std::max<size_t>(C.arena.size(), 16);
    std::vector<uint8_t> host(pb + ab, 0);
    if (!C.code.empty()) memcpy(host.data(), C.code.data(), C.code.size() * sizeof(Instr));
    if (!C.arena.empty()) memcpy(host.data() + pb, C.arena.data(), C.arena.size());
    d_code = DevBuf(ctx, pb + ab, nullptr);
    d_prog = d_code.get<Instr>();
    d_arena = d_code.get<uint8_t>() + pb;
    h2d_now(d_code.get(), host.data(), host.size());
}

static bool dict_pred(const LutSpec& L, const std::string& s) {  // per-entry predicate
    bool r;
    if (L.what == SW_CMP) {
        int c = s.compare(L.lit);
        c = c < 0 ? -1 : (c > 0);
        switch (L.op) {
            case ML_BIN_EQ: r = c == 0; break;
            case ML_BIN_NOTEQ: r = c != 0; break;
            case ML_BIN_LT: r = c < 0; break;
            case ML_BIN_LTEQ: r = c <= 0; break;
            case ML_BIN_GT: r = c > 0; break;
            default: r = c >= 0; break;
        }
    } else if (L.what == SW_LIKE) {
        r = like_match_host(s, L.lit, L.shape);
    } else {
        r = std::find(L.list.begin(), L.list.end(), s) != L.list.end();
    }
    return r != L.negated;
}

void Pipeline::prepare(Launch& L, const ml_column* cols, int ncols, int64_t nrows, const uint32_t* sel, int64_t nsel,
                       cudaStream_t s, Staging& st, Reservation* res, uint8_t* tables_dst, size_t tables_cap) {
    if (ncols != (int)input_types.size())
        raise(ML_ERR_INVALID, "batch has " + std::to_string(ncols) + " columns, the pipeline expects " +
                                  std::to_string(input_types.size()));
    if (nrows < 0 || nrows > 0xFFFFFFFFll) raise(ML_ERR_INVALID, "batch row count out of range");
    if (ncols > 0 && !cols) raise(ML_ERR_INVALID, "null column array");
    L.src.clear();
    for (int c = 0; c < ncols; c++) {
        if (cols[c].dtype != input_types[c])
            raise(ML_ERR_INVALID, "column " + std::to_string(c) + " has type " + std::to_string(cols[c].dtype) +
                                      ", the pipeline expects " + std::to_string(input_types[c]));
        L.src.push_back(stage_column(ctx, cols[c], nrows, s, st, res));
    }
    PipeArgs& P = L.P;
    P = PipeArgs{};
    P.n = sel ? nsel : nrows;
    P.sel = sel;
    P.nsrc = nrows;
    P.prog = d_prog;
    P.arena = d_arena;
    P.nstages = nstages;
    P.nprobes = (int)probes.size();
    P.head_probe = -1;
    for (int i = 0; i < nstages; i++) P.stages[i] = stages[i];
    for (size_t i = 0; i < filters.size(); i++) P.filters[i] = filters[i];
    P.has_chains = 0;
    for (size_t p = 0; p < probes.size(); p++) {
        ml_join_table* jt = probes[p].jt;
        P.probes[p].t = jt->view();
        P.probes[p].next = jt->has_dups ? jt->next.get<uint32_t>() : nullptr;
        P.probes[p].keys = probes[p].keys;
        P.probes[p].dense = jt->dense ? jt->dense.get<uint32_t>() : nullptr;
        P.probes[p].dmin = jt->dmin;
        P.probes[p].drange = jt->drange;
        P.has_chains |= jt->has_dups ? 1 : 0;
    }
    // scratch: dictionary id maps and predicate tables for this batch
    std::vector<uint8_t> scratch;
    std::vector<std::pair<int, size_t>> gid_at;   // slot -> offset
    std::vector<std::pair<int, size_t>> lut_at;   // lut -> offset
    std::vector<std::pair<int, size_t>> dict_at, dbytes_at;  // slot -> dictionary offsets / bytes
    auto put = [&](const void* p, size_t n) {  // n bytes (at least one, zeroed) at a 16-byte offset
        size_t o = (scratch.size() + 15) & ~(size_t)15;
        scratch.resize(o + std::max<size_t>(n, 1), 0);
        if (n && p) memcpy(scratch.data() + o, p, n);
        return o;
    };
    L.col_valid.assign(C.slots.size(), 0);
    L.gid_range.assign(C.slots.size(), {1u, 0u});
    for (size_t i = 0; i < C.slots.size(); i++) {
        const SlotInfo& si = C.slots[i];
        DCol& d = P.cols[i];
        const DevColumn* col;
        if (si.src == 0) {
            if (si.index < 0 || si.index >= (int)L.src.size()) raise(ML_ERR_INVALID, "column slot out of range");
            col = L.src[si.index].get();
        } else {
            ml_join_table* jt = probes[si.src - 1].jt;
            col = jt->batch.cols[si.index].get();
            d.gid = col->strid ? col->strid.get<uint32_t>() : nullptr;
        }
        d.dt = col->dtype;
        d.kind = col->kind;
        d.src = si.src;
        d.data = col->dptr();
        d.off = col->optr();
        d.valid = col->vptr();
        d.n = col->n;
        L.col_valid[i] = d.valid != nullptr;
        if (col->kind == CK_DICT) {
            const HostDict& hd = *col->dict;
            std::vector<uint32_t> g(hd.len() + 1, 0);
            {
                std::lock_guard<std::mutex> lk(intern.mu);
                for (size_t e = 0; e < hd.len(); e++) g[e] = intern.id(hd.get(e));
                g[hd.len()] = intern.id(std::string());  // spare entry for clamped codes
            }
            d.dict_len = (uint32_t)hd.len();
            if (si.src == 0) L.gid_range[i] = {*std::min_element(g.begin(), g.end()), *std::max_element(g.begin(), g.end())};
            gid_at.push_back({(int)i, put(g.data(), g.size() * 4)});
            std::vector<uint32_t> doff(hd.off);
            doff.push_back(hd.off.back());  // the spare entry is the empty string
            dict_at.push_back({(int)i, put(doff.data(), doff.size() * 4)});
            dbytes_at.push_back({(int)i, put(hd.bytes.data(), hd.bytes.size())});
        }
    }
    // plain strings read as keys: per-row global string ids (equal strings, equal ids)
    L.strids.clear();
    for (int slot : C.string_key_slots) {
        const SlotInfo& si = C.slots[slot];
        if (si.src != 0 || si.index < 0 || si.index >= (int)L.src.size()) continue;
        const DevColumn& col = *L.src[si.index];
        if (col.kind != CK_UTF8) continue;
        L.strids.push_back(intern_plain_strings(col, s));
        P.cols[slot].gid = L.strids.back().get<uint32_t>();
    }
    for (size_t l = 0; l < C.luts.size(); l++) {
        const LutSpec& spec = C.luts[l];
        const DevColumn* col = spec.slot < (int)C.slots.size() && C.slots[spec.slot].src == 0
                                   ? L.src[C.slots[spec.slot].index].get()
                                   : nullptr;
        if (!col || col->kind != CK_DICT) continue;
        std::vector<uint8_t> t(col->dict->len() + 1, 0);
        for (size_t e = 0; e < col->dict->len(); e++) t[e] = dict_pred(spec, col->dict->get(e));
        lut_at.push_back({(int)l, put(t.data(), t.size())});
    }
    if (!scratch.empty()) {
        uint8_t* base;
        if (tables_dst) {
            if (scratch.size() > tables_cap)
                raise(ML_ERR_INVALID, "dictionary tables of this batch need " + std::to_string(scratch.size()) +
                                          " bytes, more than the " + std::to_string(tables_cap) + " the call provides");
            CK(cudaMemcpyAsync(tables_dst, scratch.data(), scratch.size(), cudaMemcpyHostToDevice, s));
            base = tables_dst;
        } else {
            L.scratch = DevBuf(ctx, scratch.size(), nullptr);
            void* h = st.get(scratch.size());
            CK(cudaStreamSynchronize(s));  // the staging buffer may still feed an earlier copy
            memcpy(h, scratch.data(), scratch.size());
            CK(cudaMemcpyAsync(L.scratch.get(), h, scratch.size(), cudaMemcpyHostToDevice, s));
            base = L.scratch.get<uint8_t>();
        }
        for (auto& g : gid_at) P.cols[g.first].gid = (const uint32_t*)(base + g.second);
        for (auto& g : dict_at) P.cols[g.first].off = (const uint32_t*)(base + g.second);
        for (auto& g : dbytes_at) P.cols[g.first].dbytes = base + g.second;
        for (auto& t : lut_at) P.luts[t.first] = base + t.second;
    }
}

bool Pipeline::reads_nullable(const Prog& p, const Launch& L) const {
    for (int i = 0; i < p.len; i++) {
        const Instr& in = C.code[p.start + i];
        if ((in.op == I_COL || in.op == I_STRPRED) && L.col_valid[in.a]) return true;
        if (in.op == I_STRCMP_COL && (L.col_valid[in.a] || L.col_valid[in.b])) return true;
    }
    return false;
}

uint64_t scan_counts(Ctx* ctx, const uint32_t* counts, int64_t n, DevBuf& offsets, cudaStream_t s, Reservation* res) {
    offsets = DevBuf(ctx, (size_t)(n + 1) * 8, res);
    DevBuf scratch(ctx, scan_scratch_words(n) * 8, res);
    launch_scan_u32(counts, offsets.get<uint64_t>(), n, scratch.get<uint64_t>(), s);
    ctx->count_launch(3);
    uint64_t total = 0;
    CK(cudaMemcpyAsync(&total, offsets.get<uint64_t>() + n, 8, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return total;
}

int64_t run_select(Ctx* ctx, const Pipeline& pipe, const PipeArgs& P, DevBuf& out, cudaStream_t s, Reservation* res) {
    int nb = select_blocks(P.n);
    DevBuf bits(ctx, std::max<size_t>((size_t)(P.n + 31) / 32 * 4, 4), res);
    DevBuf counts(ctx, std::max<size_t>((size_t)nb * 4, 4), res);
    {
        void* jit = jit_select_kernel(ctx, pipe, P);
        KernelTimer kt(ctx, s, "select");
        if (jit) {
            if (nb) {
                uint32_t* b = bits.get<uint32_t>();
                uint32_t* c = counts.get<uint32_t>();
                CK(cudaMemsetAsync(c, 0, (size_t)nb * 4, s));
                void* args[] = {(void*)&P, &b, &c};
                const int grid = std::min<int64_t>(nb, (int64_t)jit_resident_blocks(jit, kPipelineThreads, 0) * num_sms());
                jit_launch(jit, grid, kPipelineThreads, 0, s, args);
            }
            ctx->add_profile("jit_launch", 0);
        } else {
            launch_select_flags(P, bits.get<uint32_t>(), counts.get<uint32_t>(), s);
        }
        kt.stop();
    }
    ctx->count_launch();
    DevBuf offs;
    uint64_t total = scan_counts(ctx, counts.get<uint32_t>(), nb, offs, s, res);
    out = DevBuf(ctx, std::max<size_t>(total * 4, 4), res);
    {
        KernelTimer kt(ctx, s, "select_write");
        launch_select_write(P, bits.get<uint32_t>(), offs.get<uint64_t>(), out.get<uint32_t>(), s);
        kt.stop();
    }
    ctx->count_launch();
    CK(cudaStreamSynchronize(s));
    return (int64_t)total;
}

void gather_utf8(Ctx* ctx, const uint32_t* off, const uint8_t* bytes, const uint32_t* idx, int64_t k, DevColumn& out,
                 cudaStream_t s, Reservation* res) {
    DevBuf lens(ctx, std::max<size_t>((size_t)k * 4, 4), nullptr);
    launch_utf8_lengths(off, idx, k, lens.get<uint32_t>(), s);
    DevBuf offs64;
    uint64_t total = scan_counts(ctx, lens.get<uint32_t>(), k, offs64, s);
    if (total > 0xFFFFFFFFull) raise(ML_ERR_UNSUPPORTED, "string column larger than 4 GiB");
    out.kind = CK_UTF8;
    out.dtype = ML_TYPE_UTF8;
    out.n = k;
    out.offsets = DevBuf(ctx, (size_t)(k + 1) * 4, res);
    launch_u64_to_u32(offs64.get<uint64_t>(), out.offsets.get<uint32_t>(), k + 1, s);
    out.data = DevBuf(ctx, std::max<size_t>(total, 1), res);
    launch_utf8_copy(off, bytes, idx, k, offs64.get<uint64_t>(), out.data.get<uint8_t>(), s);
    ctx->count_launch(3);
}

}  // namespace mlg
