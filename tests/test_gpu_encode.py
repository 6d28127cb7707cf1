"""GPU parity of the GF(2^16) multiply-accumulate (K1) through the C ABI
against the oracle, bit-exact.

Mirrors par2-rs's own strategy tests (src/galois/tests.rs:482-553: every
strategy against the scalar path at sizes {7, 8, 15, 16, 31, 32, 100, 1024}
x scalars {0, 1, 2, 12345, 65535}) and its fixture check
(src/parser.rs:957-1021, here for all 60 QuickPar recovery slices).
"""
import numpy as np
import pytest

from oracle import oracle
from tests import quickpar

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import par2gpu

    c = par2gpu.Context(0)
    yield c
    c.close()


def test_strategy_available():
    import par2gpu

    name, prio, avail = par2gpu.strategy_info()
    assert (name, prio, avail) == ("CUDA-sm100a", 40, True)


SIZES = [7, 8, 15, 16, 31, 32, 100, 1024]
SCALARS = [0, 1, 2, 12345, 65535]


@pytest.mark.parametrize("size", SIZES)
def test_mul_slice_and_muladd_sweep(ctx, size):
    for scalar in SCALARS:
        data = ((np.arange(size) * 97 + 1) & 0xFFFF).astype(np.uint16)
        want = np.array([oracle.gf_mul(int(v), scalar) for v in data], np.uint16)
        got = data.copy()
        ctx.mul_slice(scalar, got)
        assert np.array_equal(got, want), (size, scalar)

        src = ((np.arange(size) * 13 + 7) & 0xFFFF).astype(np.uint16)
        dst = ((np.arange(size) * 17 + 3) & 0xFFFF).astype(np.uint16)
        want = dst ^ np.array([oracle.gf_mul(int(v), scalar) for v in src], np.uint16)
        ctx.muladd(dst, src, scalar)
        assert np.array_equal(dst, want), (size, scalar)


def test_quickpar_recovery_slices(ctx):
    qp = quickpar.load()
    src, _ = qp.slices()
    got = ctx.encode_array(src, np.arange(60, dtype=np.uint32))
    for e in range(60):
        assert np.array_equal(got[e], qp.recovery[e]), f"exponent {e}"


@pytest.mark.parametrize("k,S,r", [
    (1, 2, 1), (3, 6, 2), (5, 64, 3), (17, 2050, 5), (40, 4096, 13), (256, 65536 // 8, 13),
    (64, 2048 * 3 + 34, 37), (33, 8192, 104), (20, 4096, 105), (12, 2048, 210),
])
def test_encode_matches_oracle(ctx, k, S, r):
    rng = np.random.default_rng(k * 1000 + r)
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    exps = np.arange(r, dtype=np.uint32)
    got = ctx.encode_array(src, exps)
    want = oracle.encode(src, exps)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("k,S,r", [(128, 65536, 9), (300, 65536 + 2050, 7), (200, 131072 + 4, 30)])
def test_host_pipeline_groups_and_tail_slabs(ctx, k, S, r):
    """Host buffers with k >= 128: inputs go up in groups while earlier groups
    are accumulated (slices this narrow fill under 1.5 waves, so the outputs
    are read back whole at the end)."""
    rng = np.random.default_rng(k + S)
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    exps = np.arange(r, dtype=np.uint32)
    want = oracle.encode(src, exps)
    assert np.array_equal(ctx.encode_array(src, exps), want)
    # separately allocated rows (no common stride): one copy per slice
    rows = [np.ascontiguousarray(src[i]) for i in range(k)]
    outs = [np.zeros(S, np.uint8) for _ in range(r)]
    ctx.encode(rows, S, exps, outs)
    assert np.array_equal(np.stack(outs), want)


@pytest.mark.parametrize("k,S,r", [(256, (1 << 20) + 6, 205), (320, 600 * 1024 + 2050, 110)])
def test_host_pipeline_wave_sized_slabs(ctx, k, S, r):
    """Slices wide enough that the tail runs as several wave-sized column
    slabs (7 for 1 MiB x 205 outputs, 4 for 600 KiB x 110, ragged last
    tile): the host pipeline equals the device-resident single launch over
    the whole width, and the oracle on column windows (encoding is
    column-independent) at the start, in the middle and at the end."""
    import torch

    rng = np.random.default_rng(S)
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    exps = np.arange(r, dtype=np.uint32)
    got = ctx.encode_array(src, exps)
    d_src = torch.from_numpy(src).cuda()
    d_out = torch.zeros((r, S), dtype=torch.uint8, device="cuda")
    ctx.encode(d_src, S, exps, d_out, device=True)
    torch.cuda.synchronize()
    assert np.array_equal(got, d_out.cpu().numpy())
    tiles = (S + 2047) // 2048
    cut = tiles // 2 * 2048  # a slab boundary for an even slab count
    for c0, c1 in ((0, 4096), (cut - 2048, cut + 2048), (S - 4098, S)):
        assert np.array_equal(got[:, c0:c1], oracle.encode(np.ascontiguousarray(src[:, c0:c1]), exps))


def test_encode_sparse_exponents_and_zero_slices(ctx):
    rng = np.random.default_rng(5)
    src = rng.integers(0, 256, (30, 4096), dtype=np.uint8)
    src[3] = 0
    src[7, :100] = 0
    exps = np.array([0, 5, 17, 65534, 1000, 2], np.uint32)
    assert np.array_equal(ctx.encode_array(src, exps), oracle.encode(src, exps))


def test_muladd_region_offsets(ctx):
    rng = np.random.default_rng(11)
    n = 5000
    srcs = [rng.integers(0, 65536, n, dtype=np.uint16) for _ in range(9)]
    dsts = [rng.integers(0, 65536, n, dtype=np.uint16) for _ in range(6)]
    coeffs = rng.integers(0, 65536, (6, 9), dtype=np.uint16)
    coeffs[2, 4] = 0
    coeffs[5, :] = 0
    want = [d.copy() for d in dsts]
    oracle.muladd_region(want, srcs, coeffs, 129, 3001)
    got = [d.copy() for d in dsts]
    ctx.muladd_region(got, srcs, coeffs, 129, 3001)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def test_device_pointers_aligned_and_misaligned(ctx):
    import torch

    rng = np.random.default_rng(21)
    k, S, r = 19, 6144, 7
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    exps = np.arange(r, dtype=np.uint32)
    want = oracle.encode(src, exps)
    d_src = torch.from_numpy(src).cuda()
    d_out = torch.zeros((r, S), dtype=torch.uint8, device="cuda")
    ctx.encode([d_src[i] for i in range(k)], S, exps, [d_out[e] for e in range(r)], device=True)
    assert np.array_equal(d_out.cpu().numpy(), want)
    # 2-byte aligned device slices are staged internally
    big = torch.zeros(k * (S + 2) + 2, dtype=torch.uint8, device="cuda")
    views = [big[2 + i * (S + 2): 2 + i * (S + 2) + S] for i in range(k)]
    for i in range(k):
        views[i].copy_(d_src[i])
    outbig = torch.zeros(r * (S + 2) + 2, dtype=torch.uint8, device="cuda")
    oviews = [outbig[2 + e * (S + 2): 2 + e * (S + 2) + S] for e in range(r)]
    ctx.encode(views, S, exps, oviews, device=True)
    for e in range(r):
        assert np.array_equal(oviews[e].cpu().numpy(), want[e])


def test_bad_arguments_report_errors(ctx):
    import par2gpu

    src = np.zeros((2, 7), np.uint8)
    with pytest.raises(par2gpu.Par2GpuError) as ei:
        ctx.encode([src[0], src[1]], 7, [0], [np.zeros(7, np.uint8)])
    assert ei.value.code == par2gpu.EINVAL
    assert "even" in par2gpu.last_error()


VARIANTS = [(8, e, 1) for e in range(1, 14)] + [(12, e, 1) for e in (4, 6, 7, 8)] + \
    [(16, e, 1) for e in (2, 3, 4, 5)] + [(16, e, 2) for e in (8, 10, 12)]


def test_every_tile_shape_matches_oracle(ctx):
    """Each compiled (warps, outputs per warp) shape, with and without input
    splits, gives the oracle's recovery slices."""
    rng = np.random.default_rng(31)
    k, S, r = 40, 2048 * 5 + 64, 50
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    exps = np.arange(r, dtype=np.uint32)
    want = oracle.encode(src, exps)
    for W, E, P in VARIANTS:
        G = W // P
        nblk = -(-r // (G * E))
        if (nblk - 1) * G * E >= r:
            continue
        for ns in (1, 3):
            ctx.set_plan(k, r, S, W, E, nblk, ns, P)
            got = ctx.encode_array(src, exps)
            assert np.array_equal(got, want), (W, E, P, nblk, ns)


PAIRED = [(8, e, 1) for e in range(7, 14)] + [(12, 8, 1)] + \
    [(8, e, 2) for e in (7, 9, 11, 13)] + [(12, 8, 2)]


@pytest.mark.parametrize("r", [25, 105, 151, 205, 209])
def test_every_paired_shape_matches_oracle(ctx, r):
    """The paired form (512-symbol tiles, half a warp per output): every
    compiled shape, one or two inputs per barrier, that covers r in at most
    three output blocks, with and without input splits (odd and even input
    counts per split), on a ragged last tile (an odd number of 512-symbol
    tiles, the last one partial) and an odd output count (the last pair of a
    block half empty), gives the oracle's recovery slices."""
    rng = np.random.default_rng(500 + r)
    k, S = 41, 1024 * 4 + 68
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    exps = rng.choice(3000, r, replace=False).astype(np.uint32)
    want = oracle.encode(src, exps)
    ran = 0
    for W, E, G in PAIRED:
        per = W * E * 2
        for nblk in (-(-r // per), -(-r // per) + 1):
            if (nblk - 1) * per >= r or nblk > 3:
                continue
            for ns in (1, 3):
                ctx.set_plan(k, r, S, W, 2 * E, nblk, ns, 1, tile_symbols=512,
                             inputs_per_stage=G)
                assert np.array_equal(ctx.encode_array(src, exps), want), (W, E, G, nblk, ns)
                ran += 1
    assert ran > 0


def test_paired_form_in_accumulating_groups_and_repair(ctx):
    """The heuristic picks the paired form above 104 outputs: 300 host inputs
    go up in groups whose later passes accumulate into the outputs; a 150-slice
    repair runs both of its passes (store, then accumulate) on it."""
    rng = np.random.default_rng(77)
    k, S, r = 300, 4096 + 1024, 205
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    exps = np.arange(r, dtype=np.uint32)
    rec = ctx.encode_array(src, exps)
    assert np.array_equal(rec, oracle.encode(src, exps))
    m = 150
    missing = np.sort(rng.choice(k, m, replace=False))
    data = src.copy()
    data[missing] = 0
    got = ctx.repair_array(data, missing, exps[:m], rec[:m])
    assert np.array_equal(got, src[missing])


def test_set_plan_rejects_bad_paired_shapes(ctx):
    import par2gpu

    for bad in [dict(outputs_per_group=13, tile_symbols=512),   # odd: not whole pairs
                dict(outputs_per_group=26, tile_symbols=256),   # no such tile
                dict(outputs_per_group=30, tile_symbols=512),   # not compiled
                dict(outputs_per_group=20, tile_symbols=512, inputs_per_stage=2),  # not compiled
                dict(outputs_per_group=13, tile_symbols=1024, inputs_per_stage=2)]:
        with pytest.raises(par2gpu.Par2GpuError) as ei:
            ctx.set_plan(40, 150 if bad["tile_symbols"] != 1024 else 100, 4096, 8,
                         bad["outputs_per_group"], 1, 1, 1, tile_symbols=bad["tile_symbols"],
                         inputs_per_stage=bad.get("inputs_per_stage", 1))
        assert ei.value.code == par2gpu.EINVAL


@pytest.mark.parametrize("r", [1, 5, 8, 9, 16, 17, 24, 25])
def test_small_output_tables_match_oracle(ctx, r):
    """Up to 24 outputs the kernel uses the 6 + 5 + 5 tables (24-word
    records); 25 is the first problem on the 8 + 8 tables.  Every compiled
    small shape (8 warps x 1-3 outputs) that covers r, with and without input
    splits, in store mode and (through the host pipeline's groups) in
    accumulate mode, gives the oracle's slices; a ragged last tile included."""
    rng = np.random.default_rng(400 + r)
    k, S = 48, 2048 * 3 + 36
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    exps = rng.choice(5000, r, replace=False).astype(np.uint32)
    want = oracle.encode(src, exps)
    assert np.array_equal(ctx.encode_array(src, exps), want)
    if r <= 24:
        for E in (1, 2, 3):
            if 8 * E < r:
                continue
            for ns in (1, 3, 6):
                ctx.set_plan(k, r, S, 8, E, 1, ns)
                assert np.array_equal(ctx.encode_array(src, exps), want), (E, ns)
    # 256 inputs from host buffers: 4 groups, the later ones accumulated
    big = rng.integers(0, 256, (256, 4096), dtype=np.uint8)
    assert np.array_equal(ctx.encode_array(big, exps), oracle.encode(big, exps))


def test_autotune_picks_a_correct_plan(ctx):
    rng = np.random.default_rng(32)
    k, S, r = 300, 16384, 37
    plan = ctx.autotune(k, r, S)
    assert plan.warps in (8, 12, 16) and plan.ms > 0
    assert plan.output_blocks * plan.warps // plan.warps_per_group * plan.outputs_per_group >= r
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    exps = np.arange(r, dtype=np.uint32)
    assert np.array_equal(ctx.encode_array(src, exps), oracle.encode(src, exps))


def test_set_plan_rejects_uncompiled_shapes(ctx):
    import par2gpu

    with pytest.raises(par2gpu.Par2GpuError) as ei:
        ctx.set_plan(10, 20, 4096, 16, 9, 1, 1)
    assert ei.value.code == par2gpu.EINVAL


def test_caller_default_stream_is_ordered(ctx):
    """Work on torch's default stream (handle 0) must be ordered with the
    context's work once the context runs on that stream."""
    import torch

    k, S, r = 64, 65536, 5
    src = torch.randint(0, 256, (k, S), dtype=torch.uint8, device="cuda")  # queued, not waited
    out = torch.zeros((r, S), dtype=torch.uint8, device="cuda")
    exps = np.arange(r, dtype=np.uint32)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    try:
        ctx.encode([src[i] for i in range(k)], S, exps, [out[e] for e in range(r)], device=True)
    finally:
        ctx.set_stream(None)
    assert np.array_equal(out.cpu().numpy(), oracle.encode(src.cpu().numpy(), exps))
