"""A request loop for create / verify / repair jobs on one GPU.

Two servers over the same arrival stream:

* ``serve_continuous`` -- continuous batching.  Arrived jobs are admitted in
  arrival order while their scratch fits an HBM budget and the device's free
  memory (a job is always admitted when nothing else runs); every admitted job is
  cut into work units (column ranges of create / repair jobs, slice groups of
  verify jobs, each bounded in work); each iteration gives the oldest admitted
  job up to half of an iteration work budget, fills the rest with units taken
  round-robin from all admitted jobs and runs them as one
  batch (``Batch``: one persistent kernel per phase).  The next batch is
  prepared on a second context while the current one runs, so jobs that
  arrive while others are on the GPU join at the next iteration and their
  work overlaps on the device with the others'.
* ``serve_one_at_a_time`` -- the same jobs, first come first served, each
  with the plain per-job calls.

Both return per-job latencies (arrival to completion) and the outputs, so a
test can check that every job's result is the same alone and in the mix.
Device data stays resident: the caller hands in jobs whose slices already
live on the device.
"""
import collections
import time

import numpy as np

from . import JOB_CREATE, JOB_REPAIR, JOB_VERIFY, Batch

TILE = 2048


class ServedJob:
    """One request.  kind: "create" | "verify" | "repair".
    src: device tensor [k, S] (repair: erased rows are ignored);
    create: r recovery slices; repair: missing (sorted), exps, rec tensor [m, S]."""

    def __init__(self, jid, kind, src, r=0, missing=None, rec=None):
        self.jid = jid
        self.kind = kind
        self.src = src
        self.k, self.S = int(src.shape[0]), int(src.shape[1])
        self.r = r
        self.missing = None if missing is None else np.asarray(missing, np.int64)
        self.rec = rec
        self.m = 0 if missing is None else len(self.missing)
        self.inverse = None
        self.out = None
        self.md5 = None
        self.crc = None

    @property
    def n(self):
        return self.r if self.kind == "create" else self.m

    def macs(self, cols=None):
        cols = self.S if cols is None else cols
        if self.kind == "verify":
            return self.k * cols * 8  # hashing: count bytes x 8 as its work
        return self.k * self.n * cols // 2

    def scratch_bytes(self):
        """What admission reserves: outputs, bit planes (whole 2 KiB tiles),
        coefficient records (96 bytes per pair up to 24 outputs, else 32)
        and, for a repair, the right-hand sides of its first pass."""
        if self.kind == "verify":
            return self.k * 20
        planes = self.k * (-(-self.S // 2048) * 2048)
        records = self.k * self.n * (96 if self.n <= 24 else 32)
        rhs = self.n * self.S if self.kind == "repair" else 0
        return self.n * self.S + planes + records + rhs


class _DeviceRoom:
    """Real free device memory for admission (the budget counts estimates):
    the driver's free memory plus what torch's caching allocator holds
    unused, read at most every `every` seconds, less the scratch of the jobs
    admitted since the reading."""

    def __init__(self, every=0.05, margin=256 << 20):
        self.every, self.margin = every, margin
        self.free, self.t, self.since = None, -1.0, 0

    def fits(self, job, t):
        import torch

        if self.free is None or t - self.t > self.every:
            dev = job.src.device
            cached = torch.cuda.memory_reserved(dev) - torch.cuda.memory_allocated(dev)
            self.free = torch.cuda.mem_get_info(dev)[0] + cached
            self.t, self.since = t, 0
        return job.scratch_bytes() + self.margin <= self.free - self.since

    def admitted(self, job):
        self.since += job.scratch_bytes()


def _alloc_outputs(job):
    import torch

    if job.kind == "verify":
        job.md5 = np.zeros((job.k, 16), np.uint8)
        job.crc = np.zeros(job.k, np.uint32)
    else:
        job.out = torch.empty((job.n, job.S), dtype=torch.uint8, device=job.src.device)


def _units(job, unit_macs):
    """Work units of a job: (kind, a, b) column ranges or slice ranges."""
    if job.kind == "verify":
        per = max(1, int(unit_macs // max(1, job.S * 8)))
        return [("slices", a, min(job.k, a + per)) for a in range(0, job.k, per)]
    tiles = (job.S + TILE - 1) // TILE
    per_tile = job.macs(TILE)
    tpu = max(1, int(unit_macs // max(1, per_tile)))
    out = []
    for t in range(0, tiles, tpu):
        a, b = t * TILE, min(job.S, (t + tpu) * TILE)
        out.append(("cols", a, b))
    return out


def _unit_work(job, unit):
    kind, a, b = unit
    if kind == "slices":
        return (b - a) * job.S * 8
    return job.k * job.n * (b - a) // 2


def _rows(t, idx=None):
    """Addresses of the rows of a [n, S] device tensor as a uint64 array."""
    n, S = int(t.shape[0]), int(t.stride(0))
    i = np.arange(n, dtype=np.uint64) if idx is None else np.asarray(idx, np.uint64)
    return np.uint64(t.data_ptr()) + i * np.uint64(S)


def _job_spec(job, unit):
    kind, a, b = unit
    S = job.S
    if job.kind == "verify":
        return {"kind": JOB_VERIFY, "k": b - a, "slice_bytes": S,
                "src": _rows(job.src, np.arange(a, b))}
    spec = {"k": job.k, "slice_bytes": S, "col_begin": a, "col_end": b if b < S else 0,
            "out": _rows(job.out)}
    if job.kind == "create":
        spec.update(kind=JOB_CREATE, src=_rows(job.src), exps=np.arange(job.r))
    else:
        present = np.delete(np.arange(job.k), job.missing)
        spec.update(kind=JOB_REPAIR, src=_rows(job.src, present), missing=job.missing,
                    exps=np.arange(job.m), recovery=_rows(job.rec), inverse=job.inverse)
    return spec


def serve_continuous(ctxs, jobs, arrivals, budget_bytes=120 << 30, iter_macs=4e10,
                     unit_macs=None):
    """Continuous batching over `jobs` arriving at `arrivals` (seconds from
    start).  ctxs: par2gpu.Context objects: the first two alternate (one
    batch runs while the next is prepared), a third, when given, forms the
    decode matrices of admitted repair jobs.  Returns (latencies in s, wall
    seconds)."""
    aux = ctxs[2] if len(ctxs) > 2 else ctxs[0]
    unit_macs = unit_macs or iter_macs / 4
    n = len(jobs)
    order = np.argsort(arrivals, kind="stable")
    lat = np.zeros(n)
    queue = collections.deque()
    active = collections.deque()       # [job, pending units deque, outstanding count, admission no.]
    state = {}
    used = 0
    nxt = 0
    done = 0
    inflight = None                    # (batch, [(jid, unit)...], ctx index)
    prepared = None
    room = _DeviceRoom()
    admitted = 0
    ci = 0
    t0 = time.perf_counter()

    def now():
        return time.perf_counter() - t0

    def build(ctx):
        """Pick units up to the iteration budget -- the oldest job with work
        left first, up to half of it, then round-robin from all admitted
        jobs -- and merge each job's contiguous units into one spec so that
        its coefficient records are built once per batch.  A job alone with
        nothing queued gets 16 budgets: cutting it finer only rebuilds its
        records, and a job that arrives meanwhile waits for at most that."""
        picked, work = [], 0.0
        alone = sum(1 for e in active if e[1]) == 1 and not queue
        budget = iter_macs * (16 if alone else 1)
        # the oldest job with work left takes up to half the budget first
        # (the longest-running jobs make the latency tail), then every job
        # takes units in turn
        oldest = min((e for e in active if e[1]), key=lambda e: e[3], default=None)
        while oldest is not None and oldest[1] and work < budget / 2:
            u = oldest[1].popleft()
            picked.append((oldest[0], u))
            work += _unit_work(oldest[0], u)
        progress = True
        while progress and work < budget:
            progress = False
            for _ in range(len(active)):
                ent = active[0]
                active.rotate(-1)
                job, pend = ent[0], ent[1]
                if not pend:
                    continue
                u = pend.popleft()
                picked.append((job, u))
                work += _unit_work(job, u)
                progress = True
                if work >= budget:
                    break
        if not picked:
            return None
        merged = []  # [job, (kind, a, b), units merged]
        for job, u in sorted(picked, key=lambda p: (p[0].jid, p[1][1])):
            if merged and merged[-1][0] is job and merged[-1][1][2] == u[1]:
                last = merged[-1]
                last[1] = (u[0], last[1][1], u[2])
                last[2] += 1
            else:
                merged.append([job, u, 1])
        b = Batch(ctx, [_job_spec(j, u) for j, u, _ in merged])
        return (b, merged)

    while done < n:
        t = now()
        while nxt < n and arrivals[order[nxt]] <= t:
            queue.append(jobs[order[nxt]])
            nxt += 1
        while queue and used + queue[0].scratch_bytes() <= budget_bytes and \
                (not active or room.fits(queue[0], t)):
            job = queue.popleft()
            used += job.scratch_bytes()
            room.admitted(job)
            _alloc_outputs(job)
            if job.kind == "repair":
                job.inverse = aux.reconstruction_matrix(job.k, job.missing, np.arange(job.m))
            units = collections.deque(_units(job, unit_macs))
            ent = [job, units, len(units), admitted]
            admitted += 1
            state[job.jid] = ent
            active.append(ent)
        if inflight is not None and inflight[0].poll():
            b, picked = inflight[0], inflight[1]
            b.wait()
            t = now()
            for pos, (job, u, cnt) in enumerate(picked):
                if job.kind == "verify":
                    res = b.results[pos]
                    a, c = u[1], u[2]
                    job.md5[a:c] = res["md5"]
                    job.crc[a:c] = res["crc"]
                ent = state[job.jid]
                ent[2] -= cnt
                if ent[2] == 0:
                    lat[job.jid] = t - arrivals[job.jid]
                    done += 1
                    used -= job.scratch_bytes()
                    active.remove(ent)
            b.close()
            inflight = None
        if prepared is None and active:
            prepared = build(ctxs[ci])
            if prepared is not None:
                ci ^= 1
        if inflight is None and prepared is not None:
            prepared[0].launch()
            inflight = prepared
            prepared = None
        elif inflight is None and prepared is None and nxt < n and not queue and not active:
            time.sleep(max(0.0, min(0.002, arrivals[order[nxt]] - now())))
    return lat, now()


def serve_one_at_a_time(ctx, jobs, arrivals):
    """First come first served, one job at a time, plain per-job calls."""
    n = len(jobs)
    order = np.argsort(arrivals, kind="stable")
    lat = np.zeros(n)
    t0 = time.perf_counter()
    for idx in order:
        job = jobs[idx]
        wait = arrivals[idx] - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        _alloc_outputs(job)
        S = job.S
        # slice tables as address arrays (what a caller holds; no per-slice
        # Python objects)
        if job.kind == "create":
            ctx.encode(_rows(job.src), S, np.arange(job.r), _rows(job.out), device=True)
        elif job.kind == "verify":
            job.md5, job.crc = ctx.hash_slices(_rows(job.src), S, device=True)
        else:
            present = np.setdiff1d(np.arange(job.k), job.missing)
            ctx.repair(job.k, S, job.missing, _rows(job.src, present), np.arange(job.m),
                       _rows(job.rec), _rows(job.out), device=True)
        lat[idx] = (time.perf_counter() - t0) - arrivals[idx]
    return lat, time.perf_counter() - t0


def latency_stats(lat, wall):
    return {"jobs": int(len(lat)), "jobs_per_s": len(lat) / wall,
            "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p95_ms": float(np.percentile(lat, 95) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3)}
