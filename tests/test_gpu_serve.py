"""The serving loop (continuous batching) returns, for every job, exactly
what the job gives when run alone with the plain per-job calls."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_each_job_same_alone_and_in_the_mix():
    import torch

    import par2gpu
    from par2gpu.serve import ServedJob, serve_continuous, serve_one_at_a_time

    rng = np.random.default_rng(5)
    ctxs = [par2gpu.Context(0), par2gpu.Context(0), par2gpu.Context(0)]
    shapes = [(40, 8192, 5), (300, 4096, 30), (8, 65536, 2), (120, 2048 * 9, 12)]
    data = []
    for k, S, r in shapes:
        src = torch.from_numpy(rng.integers(0, 256, (k, S), dtype=np.uint8)).cuda()
        m = max(1, r // 2)
        miss = np.sort(rng.choice(k, m, replace=False))
        rec = torch.zeros((m, S), dtype=torch.uint8, device="cuda")
        ctxs[0].encode([src[i] for i in range(k)], S, np.arange(m), [rec[q] for q in range(m)],
                       device=True)
        data.append((src, r, miss, rec))

    def jobs():
        out = []
        for jid in range(24):
            src, r, miss, rec = data[jid % len(data)]
            kind = ("create", "verify", "repair")[jid % 3]
            if kind == "create":
                out.append(ServedJob(jid, kind, src, r=r))
            elif kind == "verify":
                out.append(ServedJob(jid, kind, src))
            else:
                out.append(ServedJob(jid, kind, src, missing=miss, rec=rec))
        return out

    arrivals = np.cumsum(rng.exponential(1 / 500.0, 24))
    a, b = jobs(), jobs()
    # small iteration budget: big jobs are split over several iterations
    serve_continuous(ctxs, a, arrivals, iter_macs=2e8)
    serve_one_at_a_time(ctxs[0], b, arrivals)
    for ja, jb in zip(a, b):
        if ja.kind == "verify":
            assert np.array_equal(ja.md5, jb.md5) and np.array_equal(ja.crc, jb.crc)
        else:
            assert torch.equal(ja.out, jb.out), ja.jid
    # repairs give back the original slices
    for j in a:
        if j.kind == "repair":
            assert torch.equal(j.out, j.src[torch.from_numpy(j.missing).cuda()])
    for c in ctxs:
        c.close()
