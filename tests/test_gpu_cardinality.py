"""The learned cardinality estimator: HyperLogLog features bit-exact against a Python
restatement of the kernel on the oracle's key hash, the FP32 MLP's training step against a
PyTorch fp32 reference, and learned sizing never changing a query result."""
import numpy as np
import pytest

from minilake_b200 import abi
from minilake_b200.abi import INT64, Col
from minilake_b200.columns import fixed
from oracle import orc

pytestmark = pytest.mark.gpu
M64 = (1 << 64) - 1


def fmix64(k):
    k ^= k >> 33
    k = (k * 0xFF51AFD7ED558CCD) & M64
    k ^= k >> 33
    k = (k * 0xC4CEB9FE1A85EC53) & M64
    return k ^ (k >> 33)


def reference_registers(keys, valid):
    """HLL registers of int64 keys: idx = top 14 bits, rank = leading zeros of the rest + 1."""
    regs = np.zeros(1 << 14, dtype=np.int64)
    null_hash = orc.LIB.orc_hash_u64(0 ^ (1 << 56))  # key_hash of an all-NULL key: nm = 1 in bits 56..
    for v, ok in zip(keys.tolist(), valid.tolist()):
        h = fmix64(orc.LIB.orc_hash_u64(v & M64) if ok else null_hash)
        idx = h >> 50
        rest = ((h << 14) & M64) | (1 << 13)
        rank = 64 - rest.bit_length() + 1
        regs[idx] = max(regs[idx], rank)
    return regs


@pytest.fixture(scope="module")
def ctx():
    from minilake_b200.gpu import Context
    c = Context(0)
    yield c
    c.close()


def test_hll_features_match_reference(ctx):
    from minilake_b200.gpu import card_features
    rng = np.random.default_rng(51)
    n = 20_000
    keys = rng.integers(-(1 << 40), 1 << 40, n).astype(np.int64) // 7
    valid = rng.random(n) > 0.05
    f, est = card_features(ctx, [fixed(INT64, keys, valid)], [(Col(0), INT64)])
    regs = reference_registers(keys, valid)
    hist = np.bincount(regs, minlength=64)[:64] / float(1 << 14)
    assert np.array_equal(f[:64], hist.astype(np.float32))
    kv = keys[valid].view(np.uint64)
    span = float(kv.max() - kv.min()) + 1.0
    assert f[65] == np.float32(np.log2(span + 1.0) / 64.0)
    assert f[66] == np.float32((~valid).sum() / n)
    assert f[71] == 1.0
    true = len(np.unique(keys[valid])) + 1
    assert abs(est - true) / true < 0.05


@pytest.mark.parametrize("distinct", [1, 100, 10_000, 1_000_000])
def test_hll_estimate_accuracy(ctx, distinct):
    from minilake_b200.gpu import card_features
    rng = np.random.default_rng(52)
    keys = rng.permutation(np.arange(distinct, dtype=np.int64) * 3 + 11)
    keys = np.concatenate([keys, rng.choice(keys, 200_000)])
    _, est = card_features(ctx, [fixed(INT64, keys)], [(Col(0), INT64)])
    assert abs(est - distinct) / distinct < 0.05, (est, distinct)


def test_mlp_training_matches_torch_fp32(ctx):
    """Five Adam steps of the library's kernels against torch.optim.Adam on the same
    parameters and batches (fp32; tolerance rtol 1e-4, atol 1e-5 for summation order).  The
    prediction adds 32 * feature 67 (the sketch's log2 estimate) to the network's output."""
    import torch
    from minilake_b200.gpu import CardinalityModel
    model = CardinalityModel(ctx, seed=7)
    p0 = model.params
    layers = [torch.nn.Linear(72, 64), torch.nn.Linear(64, 64), torch.nn.Linear(64, 64), torch.nn.Linear(64, 1)]
    off = 0
    with torch.no_grad():
        for lin in layers:
            w = lin.weight.numel()
            lin.weight.copy_(torch.from_numpy(p0[off:off + w].reshape(lin.weight.shape)))
            off += w
            lin.bias.copy_(torch.from_numpy(p0[off:off + lin.bias.numel()]))
            off += lin.bias.numel()
    net = torch.nn.Sequential(layers[0], torch.nn.ReLU(), layers[1], torch.nn.ReLU(), layers[2], torch.nn.ReLU(),
                              layers[3]).double().float()
    opt = torch.optim.Adam(net.parameters(), lr=1e-3, betas=(0.9, 0.999), eps=1e-8)
    rng = np.random.default_rng(53)
    for _ in range(5):
        x = rng.random((32, 72), dtype=np.float32)
        y = (rng.random(32, dtype=np.float32) * 20).astype(np.float32)
        loss = model.step(x, y, lr=1e-3)
        opt.zero_grad()
        xt = torch.from_numpy(x)
        out = net(xt).squeeze(1) + 32.0 * xt[:, 67]  # skip connection from log2(HLL estimate + 1) / 32
        ref_loss = torch.mean((out - torch.from_numpy(y)) ** 2)
        ref_loss.backward()
        opt.step()
        assert abs(loss - ref_loss.item()) <= 1e-4 * max(1.0, abs(ref_loss.item()))
    ref = torch.cat([t.detach().reshape(-1) for lin in layers for t in (lin.weight, lin.bias)]).numpy()
    np.testing.assert_allclose(model.params, ref, rtol=1e-4, atol=1e-5)
    x = rng.random((100, 72), dtype=np.float32)
    xt = torch.from_numpy(x)
    np.testing.assert_allclose(model.predict(x), (net(xt).squeeze(1) + 32.0 * xt[:, 67]).detach().numpy(),
                               rtol=1e-4, atol=1e-4)
    model.close()


def test_learned_sizing_keeps_results_identical():
    """A small sweep: the engine's group counts match torch.unique, and the four arms
    (resize-on-overflow, the planner's rows / 10, HyperLogLog- and MLP-presized) give identical
    results, the presized arms with no more resizes than the plain one."""
    from minilake_b200 import cardinality
    from minilake_b200.gpu import Context
    res = cardinality.run(instances=24, train=16, seed=46, min_rows=10_000, max_rows=400_000, epochs=60,
                          log=lambda *a: None)
    assert res["identical_results"]
    assert res["resizes_mean"]["learned"] <= res["resizes_mean"]["plain"]
    assert res["resizes_mean"]["hll"] <= res["resizes_mean"]["plain"]
    assert set(res["total_ms"]) == {"plain", "planner", "hll", "learned"}
    ctx = Context(0)
    for inst in cardinality.make_instances(6, seed=47, min_rows=10_000, max_rows=200_000):
        di = cardinality.DeviceInstance(inst)
        assert cardinality.aggregate(ctx, di, 0, fetch=False)[1] == di.unique_groups()
    ctx.close()
