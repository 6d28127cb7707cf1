"""GPU parity of the batch executor (p2g_batch_*): many independent create,
repair and verify jobs of uneven shapes in one persistent-kernel execution
must give, job by job, exactly what the oracle gives for that job alone."""
import numpy as np
import pytest

from oracle import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    import par2gpu

    c = par2gpu.Context(0)
    yield c
    c.close()


def dev(a):
    """Device copy of [n, S] bytes whose rows start 16-byte aligned (rows
    padded to a multiple of 16 bytes); returns the row views."""
    import torch

    a = np.ascontiguousarray(a)
    n, S = a.shape
    pad = (S + 15) // 16 * 16
    t = torch.zeros((n, pad), dtype=torch.uint8, device="cuda")
    t[:, :S] = torch.from_numpy(a).cuda()
    return t[:, :S]


def zeros(n, S):
    import torch

    pad = (S + 15) // 16 * 16
    return torch.zeros((n, pad), dtype=torch.uint8, device="cuda")[:, :S]


def make_set(rng, k, S, r):
    src = rng.integers(0, 256, (k, S), dtype=np.uint8)
    exps = np.arange(r, dtype=np.uint32)
    return src, exps, oracle.encode(src, exps)


def test_mixed_batch_matches_oracle(ctx):
    """Default forms: small tables for 1-24 outputs, the 8 + 8 tables for
    25-104, the paired form above 104 -- all three in one persistent run."""
    ctx.batch_set_forms(None)
    mixed_batch_roundtrip(ctx, 41)


# Forms pinned per class (classes 0-1: 1-24 outputs, 2-3: 25-104, 4-5: 105-208,
# 6-7: more); every valid form runs every problem of the mixed batch.
FORM_MAPS = {
    "wide": [0] * 8,
    "paired": [2] * 8,
    "small_then_paired": [1, 1, 2, 2, 2, 2, 2, 2],
    "small_then_wide": [1, 1, 0, 0, 0, 0, 0, 0],
    "by_slice_size": [1, 0, 0, 2, 2, 0, 0, 2],
}


@pytest.mark.parametrize("name", sorted(FORM_MAPS))
def test_mixed_batch_in_pinned_forms(ctx, name):
    ctx.batch_set_forms(FORM_MAPS[name])
    try:
        mixed_batch_roundtrip(ctx, 43)
    finally:
        ctx.batch_set_forms(None)


def test_batch_autotune_picks_valid_forms_and_keeps_parity(ctx):
    import par2gpu

    forms, ms = ctx.batch_autotune(reps=1)
    assert len(forms) == par2gpu.BATCH_CLASSES
    for c, f in enumerate(forms):
        assert f in (par2gpu.FORM_WIDE, par2gpu.FORM_PAIRED) or (f == par2gpu.FORM_SMALL and c < 2)
        assert 0 < ms[c] < 1e4
    try:
        mixed_batch_roundtrip(ctx, 44)
    finally:
        ctx.batch_set_forms(None)


def test_set_forms_rejects_small_form_above_24_outputs(ctx):
    import par2gpu

    with pytest.raises(par2gpu.Par2GpuError):
        ctx.batch_set_forms([1] * 8)
    with pytest.raises(ValueError):
        ctx.batch_set_forms([0] * 7)
    ctx.batch_set_forms(None)


def mixed_batch_roundtrip(ctx, seed):
    """Creates of 1-110 outputs, repairs (single-CTA, blocked and host
    inverses) and a verify in one batch; every job equals the oracle's."""
    import par2gpu

    rng = np.random.default_rng(seed)
    shapes = [(5, 4096, 1), (60, 6144 + 64, 13), (300, 2048, 3), (17, 16384, 40),
              (200, 8192, 110), (1, 64, 1), (33, 2050, 7)]
    jobs, checks = [], []
    keep = []
    for k, S, r in shapes:
        src, exps, want = make_set(rng, k, S, r)
        d_src = dev(src)
        out = zeros(r, S)
        keep += [d_src, out]
        jobs.append({"kind": par2gpu.JOB_CREATE, "k": k, "slice_bytes": S,
                     "src": [d_src[i] for i in range(k)], "exps": exps,
                     "out": [out[e] for e in range(r)]})
        checks.append(("create", out, want))
    # repairs: one small (single-CTA inverse), one blocked, one with a host inverse
    for k, S, m, host_inv in [(40, 4096, 5, False), (300, 4096, 130, False), (80, 6144, 9, True)]:
        src, exps, rec = make_set(rng, k, S, m)
        missing = np.sort(rng.choice(k, m, replace=False))
        mset = set(missing.tolist())
        d_src, d_rec = dev(src), dev(rec)
        out = zeros(m, S)
        keep += [d_src, d_rec, out]
        job = {"kind": par2gpu.JOB_REPAIR, "k": k, "slice_bytes": S,
               "src": [d_src[i] for i in range(k) if i not in mset], "missing": missing,
               "exps": exps, "recovery": [d_rec[j] for j in range(m)],
               "out": [out[j] for j in range(m)]}
        if host_inv:
            job["inverse"] = ctx.reconstruction_matrix(k, missing, exps)
        jobs.append(job)
        checks.append(("repair", out, src[missing]))
    # verify
    vsrc = rng.integers(0, 256, (50, 5376), dtype=np.uint8)
    d_v = dev(vsrc)
    keep.append(d_v)
    jobs.append({"kind": par2gpu.JOB_VERIFY, "k": 50, "slice_bytes": 5376,
                 "src": [d_v[i] for i in range(50)]})
    b = par2gpu.Batch(ctx, jobs)
    st = b.run()
    assert all(s == 0 for s in st), st
    for kind, out, want in checks:
        assert np.array_equal(out.cpu().numpy(), want), kind
    md5, crc = oracle.hash_slices(vsrc)
    assert np.array_equal(b.results[-1]["md5"], md5)
    assert np.array_equal(b.results[-1]["crc"], crc)
    b.close()


def test_graph_replay_and_column_ranges(ctx):
    import torch

    import par2gpu

    rng = np.random.default_rng(42)
    k, S, r = 120, 2048 * 12, 30
    src, exps, want = make_set(rng, k, S, r)
    d_src = dev(src)
    out = torch.zeros((r, S), dtype=torch.uint8, device="cuda")
    # the same set as two column ranges in one batch
    jobs = [{"kind": par2gpu.JOB_CREATE, "k": k, "slice_bytes": S, "col_begin": 0,
             "col_end": 2048 * 5, "src": [d_src[i] for i in range(k)], "exps": exps,
             "out": [out[e] for e in range(r)]},
            {"kind": par2gpu.JOB_CREATE, "k": k, "slice_bytes": S, "col_begin": 2048 * 5,
             "src": [d_src[i] for i in range(k)], "exps": exps,
             "out": [out[e] for e in range(r)]}]
    b = par2gpu.Batch(ctx, jobs, graph=True)
    for _ in range(2):
        out.fill_(0x5A)
        assert b.run() == [0, 0]
        assert np.array_equal(out.cpu().numpy(), want)
    b.close()


def test_singular_job_does_not_spoil_the_batch(ctx):
    import torch

    import par2gpu

    rng = np.random.default_rng(43)
    k, S = 30, 4096
    src, exps, rec = make_set(rng, k, S, 4)
    d_src, d_rec = dev(src), dev(rec)
    out_bad = torch.zeros((2, S), dtype=torch.uint8, device="cuda")
    out_ok = torch.zeros((2, S), dtype=torch.uint8, device="cuda")
    missing = [3, 9]
    present = [d_src[i] for i in range(k) if i not in (3, 9)]
    bad = {"kind": par2gpu.JOB_REPAIR, "k": k, "slice_bytes": S, "src": present,
           "missing": missing, "exps": np.array([1, 1], np.uint32),   # equal rows: singular
           "recovery": [d_rec[1], d_rec[1]], "out": [out_bad[0], out_bad[1]]}
    ok = {"kind": par2gpu.JOB_REPAIR, "k": k, "slice_bytes": S, "src": present,
          "missing": missing, "exps": np.array([0, 1], np.uint32),
          "recovery": [d_rec[0], d_rec[1]], "out": [out_ok[0], out_ok[1]]}
    b = par2gpu.Batch(ctx, [bad, ok])
    st = b.run()
    assert st == [par2gpu.ESINGULAR, 0]
    assert np.array_equal(out_ok.cpu().numpy(), src[missing])
    b.close()


def test_unaligned_pointers_rejected(ctx):
    import torch

    import par2gpu

    buf = torch.zeros(4096 + 16, dtype=torch.uint8, device="cuda")
    job = {"kind": par2gpu.JOB_CREATE, "k": 1, "slice_bytes": 2048, "src": [buf.data_ptr() + 2],
           "exps": [0], "out": [buf.data_ptr() + 2048]}
    with pytest.raises(par2gpu.Par2GpuError) as ei:
        par2gpu.Batch(ctx, [job])
    assert ei.value.code == par2gpu.EINVAL


def test_cancel_stops_the_batch_and_the_context_stays_usable(ctx):
    """p2g_batch_cancel while the persistent kernel runs: it takes no further
    item, the batch ends early with P2G_ECANCELED, and the same context then
    runs a batch correctly."""
    import time

    import torch

    import par2gpu

    rng = np.random.default_rng(44)
    k, S, r = 2048, 1 << 20, 205        # ~35 ms of work per job
    src = torch.randint(0, 256, (k, S), dtype=torch.uint8, device="cuda")
    outs = [torch.zeros((r, S), dtype=torch.uint8, device="cuda") for _ in range(6)]
    jobs = [{"kind": par2gpu.JOB_CREATE, "k": k, "slice_bytes": S,
             "src": [src[i] for i in range(k)], "exps": np.arange(r),
             "out": [o[e] for e in range(r)]} for o in outs]
    b = par2gpu.Batch(ctx, jobs)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    b.launch()
    time.sleep(0.02)
    b.cancel()
    with pytest.raises(par2gpu.Par2GpuError) as ei:
        b.wait()
    took = time.perf_counter() - t0
    assert ei.value.code == par2gpu.ECANCELED
    assert b.statuses() == [par2gpu.ECANCELED] * len(jobs)
    assert took < 0.15, took            # well short of the ~210 ms the batch needs
    # relaunching clears the flag: the full batch completes and is correct
    assert b.run() == [0] * len(jobs)
    small = src[:64, :8192].cpu().numpy()
    want = oracle.encode(small, np.arange(3, dtype=np.uint32))
    b.close()
    o = torch.zeros((3, 8192), dtype=torch.uint8, device="cuda")
    b2 = par2gpu.Batch(ctx, [{"kind": par2gpu.JOB_CREATE, "k": 64, "slice_bytes": 8192,
                              "src": [src[i] for i in range(64)], "exps": np.arange(3),
                              "out": [o[e] for e in range(3)]}])
    assert b2.run() == [0]
    assert np.array_equal(o.cpu().numpy(), want)
    b2.close()
