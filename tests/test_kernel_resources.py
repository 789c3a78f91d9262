"""Stack frames and spills of the kernels as ptxas reports them for sm_100a (CPU only: the build's
report kept beside each object, and the runtime-specialized kernels compiled here through NVRTC).
A stack frame in a hot kernel means per-thread state in local memory; the top-N scan lost a third
of its speed to one (208 bytes behind a sorting network that was not inlined)."""
import os
import pathlib
import re
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BUILD = os.path.join(ROOT, "minilake_b200", "_build")

# kernels allowed a stack frame (bytes) or spills: the interpreter form of the aggregate (the
# runtime-specialized kernels replace it on every measured path) and the serial Snappy pass
ALLOWED = {"k_agg": 64, "k_pq_snappy_serial": 16}
ALLOWED_SPILLS = {"k_agg"}
# runtime-specialized kernels allowed a frame: the GROUP BY forms with per-thread accumulators
ALLOWED_JIT = {"aggregate_groups_contig": 64, "aggregate_groups_strided": 64}


def _kernel_name(mangled: str) -> str:
    """The kernel's own identifier in an Itanium-mangled name (<length><identifier> pieces)."""
    if not mangled.startswith("_Z"):
        return mangled  # extern "C"
    i = 3 if mangled.startswith("_ZN") else 2
    while i < len(mangled):
        m = re.match(r"\d+", mangled[i:])
        if not m:
            break
        n, i = int(m.group()), i + len(m.group())
        ident, i = mangled[i:i + n], i + n
        if ident.startswith(("k_", "ml_")):
            return ident
    return mangled


def _frames(text: str):
    """(kernel, stack bytes, spill store bytes, spill load bytes) per compiled entry function."""
    out, name = [], None
    for line in text.splitlines():
        m = re.search(r"Compiling entry function '([^']+)'", line)
        if m:
            name = _kernel_name(m.group(1))
            continue
        m = re.search(r"(\d+) bytes stack frame, (\d+) bytes spill stores, (\d+) bytes spill loads", line)
        if m and name:
            out.append((name, int(m.group(1)), int(m.group(2)), int(m.group(3))))
            name = None
    return out


@pytest.mark.parametrize("unit", ["ml_kernels", "ml_parquet", "ml_card"])
def test_library_kernels_keep_their_state_in_registers(unit):
    path = os.path.join(BUILD, unit + ".ptxas.txt")
    if not os.path.exists(path):
        pytest.skip("no ptxas report: build the library (__graft_entry__.build())")
    frames = _frames(open(path).read())
    assert frames, "the report lists no kernels"
    bad = [(k, st, ss, sl) for k, st, ss, sl in frames
           if st > ALLOWED.get(k, 0) or ((ss or sl) and k not in ALLOWED_SPILLS)]
    assert not bad, bad
    if unit == "ml_kernels":
        assert any(k == "k_topn_warp" for k, *_ in frames)


def test_specialized_kernels_keep_their_state_in_registers():
    import test_jit_codegen as T
    nvrtc = T._nvrtc()
    sources = T._generated_sources(pathlib.Path(tempfile.mkdtemp()))
    names, texts = T._header_set()
    opts = [b"--gpu-architecture=sm_100a", b"-std=c++17", b"--fmad=false", b"-Xptxas=-v"]
    bad = {}
    for name, src in sorted(sources.items()):
        err, prog = nvrtc.nvrtcCreateProgram(src.encode(), name.encode() + b".cu", len(names), texts, names)
        assert err == nvrtc.nvrtcResult.NVRTC_SUCCESS
        (res,) = nvrtc.nvrtcCompileProgram(prog, len(opts), opts)
        _, n = nvrtc.nvrtcGetProgramLogSize(prog)
        log = b" " * n
        nvrtc.nvrtcGetProgramLog(prog, log)
        nvrtc.nvrtcDestroyProgram(prog)
        assert res == nvrtc.nvrtcResult.NVRTC_SUCCESS, log.decode()[:2000]
        m = re.search(r"(\d+) bytes stack frame, (\d+) bytes spill stores", log.decode())
        assert m, (name, log.decode()[:500])
        if int(m.group(1)) > ALLOWED_JIT.get(name, 0):
            bad[name] = m.group(0)
    assert not bad, bad
