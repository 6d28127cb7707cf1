"""Benchmark of the sm_100a GF(2^16) erasure-coding path.

Default workload (one GPU): the large-encode configuration -- 4 files x
512 MiB of seeded uniform random bytes, 1 MiB slices -> k = 2048 source
slices, r = 205 recovery slices (10 %), recovery data computed by the region
multiply-accumulate.  One "step" is one full encode of that set.

  value   source GB/s with the slices resident in HBM (device pointers through
          the C ABI, CUDA events on the launching stream, max over ranks)
  e2e     the same through the C ABI with pinned HOST buffers: the 2 GiB H2D
          copy of the sources and the D2H copy of the 205 recovery slices are
          inside the timed region
  roofline  the multiply-accumulate kernel's integer-issue roofline: 2 LOP3
          per symbol multiply-accumulate against the LOP3 rate measured on
          this device, plus its HBM side
  cpu_baseline  the reference's CPU strategy (par2-rs AVX2-Shuffle restated
          in C, all host threads) on the whole set, its recovery slices
          compared with the GPU's byte for byte (gpu_matches_full)
  repair / batched / serving  the metric's other parts, on the high-slice-
          count verify + repair set, 256 heterogeneous sets, and Poisson
          arrivals at 100 / 1000 / 2000 jobs/s (omitted with --no-legs)

``--impl reference`` times that CPU strategy alone (rank 0) and prints the
reference line.  Multi-GPU (torchrun): every rank encodes its own set
(independent recovery sets, weak scaling, no data-path collective).
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, os.path.join(ROOT, "par2-rs_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

# the headline metric of the benchmark contract
METRIC = "encode/repair GB/s,%roofline; served jobs/s+p99 vs per-job plain, bit-exact"
WORKLOADS = {
    # the configuration the headline metric is quoted on
    "large_encode": (2048, 1 << 20, 205,
                     "large_encode: 4 files x 512 MiB seeded uniform random, 1 MiB slices, "
                     "k=2048, r=205 (10%)"),
    # the same shape with 128 KiB slices (256 MB of sources): small enough
    # for an ncu --set full capture
    "profile_encode": (2048, 128 << 10, 205,
                       "profile_encode: k=2048 x 128 KiB seeded uniform random, r=205"),
    # a small-output problem (13 outputs: the 6 + 5 + 5 tables) at the
    # profile size, for ncu
    "profile_small": (2048, 128 << 10, 13,
                      "profile_small: k=2048 x 128 KiB seeded uniform random, r=13"),
    # the CPU-runnable plain configuration: 16 MiB, 64 KiB slices, 5 %
    "plain": (256, 64 << 10, 13, "plain: 1 file x 16 MiB, 64 KiB slices, k=256, r=13 (5%)"),
}
K_SRC, SLICE, R_REC, WORKLOAD = WORKLOADS["large_encode"]
SEED = 20261203


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def probe_int_peak(device):
    lib = ctypes.CDLL(os.path.join(ROOT, "par2-rs_b200", "lib", "libp2g_probe.so"))
    ops = ctypes.c_double()
    ms = ctypes.c_double()
    sms = ctypes.c_int()
    rc = lib.p2g_probe_lop3(device, ctypes.byref(ops), ctypes.byref(ms), ctypes.byref(sms))
    if rc != 0:
        return None, None
    return ops.value, sms.value


def cpu_model():
    """The host CPU's model name (from /proc/cpuinfo; None elsewhere)."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
            return
        # running (first sample written) before the caller's timed region
        for _ in range(100):
            if os.path.getsize(self.f.name) > 0 or self.proc.poll() is not None:
                break
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def gen_sources(k, S, seed):
    rng = np.random.default_rng(seed)
    return rng.integers(0, 256, (k, S), dtype=np.uint8)


def cpu_encode_rate(src_host, r, threads):
    """The restated par2-rs AVX2 strategy on the whole set (every slice, every
    column): returns (source GB/s, seconds, recovery slices)."""
    from oracle import oracle

    t0 = time.perf_counter()
    rec = oracle.cpu_encode(src_host, r, threads)
    dt = time.perf_counter() - t0
    return src_host.nbytes / dt / 1e9, dt, rec


def traffic_from_profile():
    path = os.path.join(ROOT, "profiles", "muladd_large_encode_traffic.json")
    if os.path.exists(path):
        try:
            return json.load(open(path)).get("dram_bytes_per_launch")
        except ValueError:
            return None
    return None


def run_reference(args, rank):
    if rank != 0:
        return
    k, S, r = K_SRC, SLICE, R_REC
    threads = os.cpu_count() or 1
    src = gen_sources(k, S, SEED)
    from oracle import oracle

    for _ in range(args.warmup):
        oracle.cpu_encode(src, r, threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle.cpu_encode(src, r, threads)
        times.append(time.perf_counter() - t0)
    dt = sum(times) / len(times)
    gbs = src.nbytes / dt / 1e9
    sample = f"the whole set per step: all {k} slices x {S} bytes, r={r}"
    line = {
        "impl": "reference", "metric": METRIC, "value": gbs, "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u16 (GF(2^16))", "data": "synthetic (seeded uniform bytes)",
        "config": {"workload": WORKLOAD, "k": k, "r": r, "slice_bytes": S, "sample": sample},
        "cpu_baseline": {"value": gbs, "unit": "GB/s", "cores": threads,
                         "cpu_model": cpu_model(), "kind": "port",
                         "sample": sample,
                         "what": "par2-rs AVX2-Shuffle strategy restated in C (Rust reference "
                                 "not buildable here), reference threading"},
        "e2e": {"value": gbs, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world):
    import torch
    import torch.distributed as dist

    import par2gpu

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    k, S, r = K_SRC, SLICE, R_REC
    exps = np.arange(r, dtype=np.uint32)

    src_host_np = gen_sources(k, S, SEED + rank)
    src_pinned = torch.from_numpy(src_host_np).pin_memory()
    out_pinned = torch.zeros((r, S), dtype=torch.uint8).pin_memory()
    src_dev = src_pinned.to(dev)
    out_dev = torch.zeros((r, S), dtype=torch.uint8, device=dev)

    ctx = par2gpu.Context(local)
    stream = torch.cuda.current_stream(dev)
    ctx.set_stream(stream.cuda_stream)
    # [k, S] / [r, S] tensors: one pointer per row from base + i * stride
    def step_dev():
        ctx.encode(src_dev, S, exps, out_dev, device=True)

    plan = None
    if not args.no_autotune:
        plan = ctx.autotune(k, r, S).as_dict()

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v):
        from par2gpu.shard import max_over_ranks as mx

        return mx(v, device=dev)

    # ---- device-resident timed region (value) ----
    # A set larger than L2 (126 MB) streams from HBM on every step; a smaller
    # one is evicted between steps by writing a 256 MiB buffer, outside the
    # per-step events.
    big = (k + r) * S > (256 << 20)
    flush = None if big else torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    clocks = ClockSampler(local)
    clocks.start()  # sampling from the warm-up on, through the timed steps
    for _ in range(args.warmup):
        step_dev()
    ctx.set_timing(True)
    barrier()
    torch.cuda.synchronize(dev)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    mul_ms, launches = [], 0
    for a, b in evs:
        if flush is not None:
            flush.fill_(1)
        a.record(stream)
        step_dev()
        b.record(stream)
        t = ctx.last_timing()
        mul_ms.append(t.ms_kernel)
        launches += t.launches
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    barrier()
    ms_step = max_over_ranks(sum(a.elapsed_time(b) for a, b in evs) / args.steps)
    ctx.set_timing(False)
    value = world * k * S / (ms_step * 1e-3) / 1e9

    if args.quick:
        ctx.close()
        if rank == 0:
            print(json.dumps({"workload": WORKLOAD, "plan": plan, "ms_per_step": ms_step,
                              "value": value,
                              "unit": "GB/s", "kernel_ms": sum(mul_ms) / len(mul_ms),
                              "gpu_launches": launches, "clocks": clk}), flush=True)
        return

    # ---- end to end through the C ABI with pinned host buffers (e2e) ----
    # [k, S] / [r, S] host arrays: the binding passes one pointer per row
    # (base + i * stride), as a C caller passes its slice table
    host_src = src_pinned.numpy()
    host_out = out_pinned.numpy()
    e2e_steps = max(1, args.steps)
    ctx.encode(host_src, S, exps, host_out)  # warm the staging buffers
    barrier()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        ctx.encode(host_src, S, exps, host_out)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / e2e_steps)
    e2e_value = world * k * S / (e2e_ms * 1e-3) / 1e9
    # the repair of the same set from the same pinned host buffers (host_out
    # now holds its r recovery slices)
    repair_host = repair_e2e_part(ctx, host_src, host_out, stream) if world == 1 else None

    # ---- roofline of the multiply-accumulate kernel ----
    int_peak, sms = probe_int_peak(local)
    hbm_peak, peak_kind = peaks()
    t_kernel = sum(mul_ms) / len(mul_ms) * 1e-3
    macs = k * r * (S // 2)
    int_ops = 2.0 * macs
    alg_bytes = (k + r) * S
    # the heuristic plan takes the paired form above 104 outputs
    paired = (plan["tile_symbols"] == 512) if plan else r > 104
    roofline = {
        "bound": "int",
        "kernel": "muladd_paired" if paired else "muladd_bitsliced",
        "achieved": int_ops / t_kernel / 1e12,
        "peak": (int_peak or 0) / 1e12,
        "unit": "Tops/s (2 LOP3 per GF(2^16) symbol MAC)",
        "frac": (int_ops / t_kernel) / int_peak if int_peak else None,
        "peak_source": f"LOP3 issue rate measured on this device ({sms} SMs)",
        "kernel_ms": t_kernel * 1e3,
        "alg_bytes": alg_bytes,
        "hbm": {"achieved": alg_bytes / t_kernel / 1e9, "peak": hbm_peak, "unit": "GB/s",
                "frac": alg_bytes / t_kernel / 1e9 / hbm_peak, "peak_source": peak_kind},
        # ncu DRAM bytes per launch, profiled for the large-encode shape only
        "traffic": traffic_from_profile() if WORKLOAD == WORKLOADS["large_encode"][3] else None,
    }

    # ---- CPU baseline + bit-exact cross-check of the whole recovery output ----
    cpu = None
    if rank == 0 and world == 1:
        threads = os.cpu_count() or 1
        gbs, dt, rec_cpu = cpu_encode_rate(src_host_np, r, threads)
        cpu = {"value": gbs, "unit": "GB/s", "cores": threads, "cpu_model": cpu_model(),
               "kind": "port",
               "sample": f"the whole set: all {k} slices x {S} bytes, r={r}",
               "seconds": dt,
               "what": "par2-rs AVX2-Shuffle strategy restated in C, reference threading",
               "gpu_matches_full": bool(np.array_equal(out_dev.cpu().numpy(), rec_cpu))}
        del rec_cpu

    # ---- the drop-in through the unchanged callers: par2-rs's streaming
    # encoder (batches of 16-128 blocks, recovery batches of 4-8, one strategy
    # call per pair from worker threads) over the CUDA strategy's shuffle2x
    # hooks, host buffers in and out ----
    trait = None
    if rank == 0 and world == 1 and not args.no_legs and WORKLOAD == WORKLOADS["large_encode"][3]:
        try:
            trait = trait_path_leg(src_host_np, r, out_dev.cpu().numpy(), steps=2)
        except Exception as exc:  # the headline line must still print
            trait = {"error": f"{type(exc).__name__}: {exc}"}

    # ---- the plain configuration's repair leg: r seeded slices zeroed and
    # rebuilt from the r recovery slices just made (device-resident) ----
    repair_leg = None
    if WORKLOAD == WORKLOADS["plain"][3]:
        rng = np.random.default_rng(SEED + 2)
        miss = np.sort(rng.choice(k, r, replace=False))
        d_miss = torch.from_numpy(miss).to(dev)
        damaged = src_dev.clone()
        damaged[d_miss] = 0
        keep = np.ones(k, bool)
        keep[miss] = False
        present = np.uint64(damaged.data_ptr()) + \
            np.flatnonzero(keep).astype(np.uint64) * np.uint64(damaged.stride(0))
        fixed = torch.zeros((r, S), dtype=torch.uint8, device=dev)

        def step_rep():
            ctx.repair(k, S, miss, present, exps, out_dev, fixed, device=True)

        for _ in range(args.warmup):
            step_rep()
        torch.cuda.synchronize(dev)
        rms = []
        for _ in range(max(1, args.steps)):
            if flush is not None:
                flush.fill_(1)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step_rep()
            b.record(stream)
            torch.cuda.synchronize(dev)
            rms.append(a.elapsed_time(b))
        rep_ms = sum(rms) / len(rms)
        repair_leg = {"ms_per_step": rep_ms, "missing": int(r),
                      "source_gbs": k * S / (rep_ms * 1e-3) / 1e9,
                      "bit_exact": bool(torch.equal(fixed, src_dev[d_miss])),
                      "what": f"{r} seeded slices zeroed, rebuilt from the {r} recovery slices "
                              "(decode matrix + multiply-accumulate), L2 flushed between steps"}
    ctx.close()

    # ---- the metric's other parts: repair at the high-slice-count size,
    # batched sets and served jobs, each bit-exact against its own check ----
    legs = {}
    if rank == 0 and world == 1 and not args.no_legs and WORKLOAD == WORKLOADS["large_encode"][3]:
        del src_dev, out_dev, src_pinned, out_pinned, host_src, host_out
        if flush is not None:
            del flush
        torch.cuda.empty_cache()
        for key, fn in (("repair", lambda: verify_repair_leg(autotune=False)),
                        ("batched", batched_leg),
                        ("serving", lambda: serving_leg((100, 1000, 2000)))):
            t0 = time.perf_counter()
            try:
                legs[key] = fn()
            except Exception as exc:  # the headline line must still print
                legs[key] = {"error": f"{type(exc).__name__}: {exc}"}
            legs[key]["leg_wall_s"] = time.perf_counter() - t0

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u16 (GF(2^16))", "data": "synthetic (seeded uniform bytes)",
            "config": {"workload": WORKLOAD, "k": k, "r": r, "slice_bytes": S,
                       "plan": plan if plan else "heuristic",
                       "parallelism": f"{world} independent sets" if world > 1 else "1 set",
                       "l2": (f"inputs {(k + r) * S / 2**20:.0f} MiB per step > 126 MB L2; no flush"
                              if big else "L2 flushed between steps (256 MiB write, untimed)")},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "GB/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": k * S, "d2h_bytes_per_step": r * S},
            "gpu_launches": launches,
            "clocks": clk,
        }
        if repair_host is not None:
            line["repair_e2e"] = repair_host
        if repair_leg is not None:
            line["repair"] = repair_leg
        if trait is not None:
            line["trait_path"] = trait
        line.update(legs)
        print(json.dumps(line), flush=True)


def repair_e2e_part(ctx, src_host, rec_host, stream, steps=3):
    """Repair of r erased slices of the large-encode set through the C ABI
    from pinned host buffers (present slices, recovery slices and outputs in
    host memory, both copy directions inside the timed region): best of
    `steps` after one warm-up, and equality with the erased slices."""
    import torch

    k, S = src_host.shape
    r = rec_host.shape[0]
    rng = np.random.default_rng(SEED + 11)
    missing = np.sort(rng.choice(k, r, replace=False))
    keep = np.ones(k, bool)
    keep[missing] = False

    def rows(a):
        return np.uint64(a.ctypes.data) + np.arange(a.shape[0], dtype=np.uint64) * \
            np.uint64(a.strides[0])

    present = rows(src_host)[keep]
    out = torch.zeros((r, S), dtype=torch.uint8).pin_memory().numpy()
    exps = np.arange(r, dtype=np.uint32)

    def run():
        ctx.repair(k, S, missing, present, exps, rows(rec_host), rows(out))

    run()
    times = []
    for _ in range(steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run()
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = min(times)
    return {"workload": f"repair of {r} erased slices of the same set (random, seeded) from "
                        f"pinned host buffers", "ms": ms,
            "source_gbs": k * S / (ms * 1e-3) / 1e9,
            "h2d_bytes": k * S, "d2h_bytes": r * S,
            "bit_exact": bool(np.array_equal(out, src_host[missing]))}


def trait_path_leg(src_host, r, want, steps=2):
    """The encode through par2-rs's unchanged streaming-encoder call sequence
    (p2f_streaming_encode: par2_rs.rs:687-902 restated over the selected
    strategy, all host threads) from host buffers; wall time of whole calls,
    best of `steps` after one warm-up, and equality with `want`."""
    from par2gpu import format as fmt

    threads = os.cpu_count() or 1
    k, S = src_host.shape
    got = fmt.streaming_encode(src_host, r, threads=threads)   # warm-up
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        got = fmt.streaming_encode(src_host, r, threads=threads)
        times.append(time.perf_counter() - t0)
    dt = min(times)
    return {"source_gbs": k * S / dt / 1e9, "seconds": dt, "threads": threads,
            "bit_exact": bool(np.array_equal(got, want)),
            "what": "StreamingEncoder process_block x k + finalize over the CUDA strategy's "
                    "shuffle2x hooks (host u16 buffers, batches of 16-128 data blocks x "
                    "recovery batches of 4-8 from worker threads); wall time of the whole "
                    "call, copies included"}


def run_verify_repair(args):
    print(json.dumps(verify_repair_leg(autotune=not args.no_autotune)), flush=True)


def verify_repair_leg(autotune=True):
    """The high-slice-count verify + repair configuration: 32000 source slices
    of 64 KiB (~2 GiB, 8 files' worth) with 1600 recovery slices; 1600 slices
    damaged (800 zeroed, 800 with 1-64 flipped bytes); per-slice MD5/CRC32
    verification of all 32000, the 1600 x 1600 inversion and the repair, all
    checked bit-exact against the pristine slices.  Returns the results."""
    import torch

    import par2gpu

    dev = torch.device("cuda", 0)
    k, S, m = 32000, 64 << 10, 1600
    g = torch.Generator(device=dev)
    g.manual_seed(SEED)
    src = torch.randint(0, 256, (k, S), dtype=torch.uint8, device=dev, generator=g)
    rec = torch.zeros((m, S), dtype=torch.uint8, device=dev)
    exps = np.arange(m, dtype=np.uint32)
    base, rbase = src.data_ptr(), rec.data_ptr()
    sptr = [base + i * S for i in range(k)]
    rptr = [rbase + j * S for j in range(m)]
    ctx = par2gpu.Context(0)
    ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    ctx.set_timing(True)
    out = {"workload": "verify_repair: 32000 x 64 KiB seeded uniform random, 1600 recovery "
                       "slices, 1600 damaged (800 zeroed, 800 with 1-64 byte flips)"}

    def timed(fn, reps=2):
        best = None
        for _ in range(reps):
            fn()
            t = ctx.last_timing()
            if best is None or t.ms_total < best[0]:
                best = (t.ms_total, t.ms_kernel)
        return best

    if autotune:
        # the encode shape and the two repair passes (present -> RHS, RHS -> missing)
        out["plans"] = {f"{a}x{b}": ctx.autotune(a, b, S).as_dict()
                        for a, b in ((k, m), (k - m, m), (m, m))}
    # create: recovery slices of the pristine set
    tot, ker = timed(lambda: ctx.encode(sptr, S, exps, rptr, device=True))
    out["encode"] = {"ms": tot, "kernel_ms": ker, "source_gbs": k * S / tot / 1e6}
    # IFSC checksums of the pristine slices
    tot, ker = timed(lambda: ctx.hash_slices(sptr, S, device=True))
    md5, crc = ctx.hash_slices(sptr, S, device=True)
    out["hash"] = {"ms": tot, "kernel_ms": ker, "gbs": k * S / tot / 1e6}
    # damage
    rng = np.random.default_rng(SEED + 1)
    dmg = np.sort(rng.choice(k, m, replace=False))
    pristine = src[torch.from_numpy(dmg).to(dev)].clone()
    zeroed, flipped = dmg[: m // 2], dmg[m // 2:]
    src[torch.from_numpy(zeroed).to(dev)] = 0
    for i in flipped:
        nflip = int(rng.integers(1, 65))
        offs = torch.from_numpy(rng.choice(S, nflip, replace=False)).to(dev)
        vals = torch.from_numpy(rng.integers(1, 256, nflip, dtype=np.uint8)).to(dev)
        src[int(i)].index_put_((offs,), src[int(i)][offs] ^ vals)
    # verify all slices (CRC then MD5 verdict)
    tot, ker = timed(lambda: ctx.verify_slices(sptr, S, md5, crc, device=True))
    ok = ctx.verify_slices(sptr, S, md5, crc, device=True)
    found = np.flatnonzero(~ok)
    out["verify"] = {"ms": tot, "kernel_ms": ker, "gbs": k * S / tot / 1e6,
                     "damaged_found": int(len(found)),
                     "damage_detected_exactly": bool(np.array_equal(found, dmg))}
    # inversion alone
    inv_ms = []
    for _ in range(2):
        ctx.reconstruction_matrix(k, dmg, exps)
        inv_ms.append(ctx.last_timing().ms_total)
    out["invert"] = {"m": m, "ms": min(inv_ms), "method": "closed-form Vandermonde inverse "
                     "(exponents 0..m-1)"}
    # the same inversion when one recovery slice of the run is missing
    gapped = np.concatenate([np.arange(m - 1), [m + 4]]).astype(np.uint32)
    inv_ms = []
    for _ in range(2):
        ctx.reconstruction_matrix(k, dmg, gapped)
        inv_ms.append(ctx.last_timing().ms_total)
    out["invert_gapped"] = {"m": m, "ms": min(inv_ms),
                            "method": "Woodbury correction of the Vandermonde inverse "
                                      "(one exponent outside the run)"}
    # repair
    fixed = torch.zeros((m, S), dtype=torch.uint8, device=dev)
    fbase = fixed.data_ptr()
    dset = set(dmg.tolist())
    present = [sptr[i] for i in range(k) if i not in dset]
    tot, ker = timed(lambda: ctx.repair(k, S, dmg, present, exps, rptr,
                                        [fbase + j * S for j in range(m)], device=True))
    torch.cuda.synchronize(dev)
    int_peak, _ = probe_int_peak(0)
    macs = m * k * (S // 2)
    out["repair"] = {"ms": tot, "last_muladd_kernel_ms": ker,
                     "source_gbs": k * S / tot / 1e6,
                     "bit_exact": bool(torch.equal(fixed, pristine)),
                     "int_roofline_frac": (2.0 * macs / (tot * 1e-3)) / int_peak if int_peak else None}
    ctx.close()
    del src, rec, fixed, pristine
    torch.cuda.empty_cache()
    return out


HASH_WORKLOADS = {
    # the IFSC checksums of the verify configuration
    "hash": (32000, 64 << 10, "hash: MD5+CRC32 of 32000 x 64 KiB seeded uniform slices"),
    # the same occupancy (256 slices on each of 148 SMs) at 310 MB, for ncu
    "profile_hash": (37888, 8 << 10, "profile_hash: MD5+CRC32 of 37888 x 8 KiB seeded uniform "
                                     "slices"),
}


def run_hash(args):
    """Per-slice MD5 + CRC32 of device-resident slices; roofline in integer
    ops (MD5: 64 steps x 5 ops per 64-byte block; CRC32 counted as bytes)."""
    import torch

    import par2gpu

    n, S, name = HASH_WORKLOADS[args.workload]
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev)
    g.manual_seed(SEED)
    d = torch.randint(0, 256, (n, S), dtype=torch.uint8, device=dev, generator=g)
    ptrs = [d.data_ptr() + i * S for i in range(n)]
    ctx = par2gpu.Context(0)
    ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
    for _ in range(args.warmup):
        ctx.hash_slices(ptrs, S, device=True)
    ctx.set_timing(True)
    ker, tot = [], []
    for _ in range(max(1, args.steps)):
        md5, crc = ctx.hash_slices(ptrs, S, device=True)
        t = ctx.last_timing()
        ker.append(t.ms_kernel)
        tot.append(t.ms_total)
    ctx.close()
    # the first and last slices against Python's hashlib / zlib
    import hashlib
    import zlib

    ok = True
    for i in (0, n - 1):
        row = d[i].cpu().numpy().tobytes()
        ok = ok and md5[i].tobytes() == hashlib.md5(row).digest() and int(crc[i]) == zlib.crc32(row)
    ok = bool(ok)
    int_peak, sms = probe_int_peak(0)
    kms = statistics.median(ker)
    ops = n * S / 64 * 64 * 5
    print(json.dumps({"workload": name, "slices": n, "slice_bytes": S, "steps": args.steps,
                      "kernel_ms": kms, "call_ms": statistics.median(tot),
                      "gbs": n * S / kms / 1e6,
                      "roofline": {"bound": "int", "achieved": ops / kms / 1e9,
                                   "peak": (int_peak or 0) / 1e12, "unit": "Tops/s (MD5 5 ops/step)",
                                   "frac": ops / (kms * 1e-3) / int_peak if int_peak else None},
                      "matches_hashlib": ok}), flush=True)


class _GF:
    """GF(2^16) (poly 0x1100B) log/antilog tables for result checks."""

    def __init__(self):
        self.exp = np.zeros(2 * 65535, np.int64)
        self.log = np.zeros(65536, np.int64)
        b = 1
        for i in range(65535):
            self.exp[i] = self.exp[i + 65535] = b
            self.log[b] = i
            b <<= 1
            if b & 0x10000:
                b ^= 0x1100B

    def mul(self, a, v):
        """scalar a times the uint16 vector v"""
        v = v.astype(np.int64)
        if a == 0:
            return np.zeros(len(v), np.uint16)
        r = self.exp[self.log[a] + self.log[v]]
        return np.where(v == 0, 0, r).astype(np.uint16)

    def pow(self, a, e):
        return int(self.exp[(int(self.log[a]) * int(e)) % 65535]) if a else int(e == 0)


def run_invert(args):
    """The 1600 x 1600 decode matrix of the verify configuration (32000 slices):
    consecutive exponents (closed-form Vandermonde inverse) and exponents with
    a gap (Woodbury correction of that inverse), time per call, each checked
    through A * A^-1 = I on sampled rows."""
    import par2gpu

    k, m = 32000, 1600
    rng = np.random.default_rng(SEED + 5)
    missing = np.sort(rng.choice(k, m, replace=False))
    gf = _GF()
    c = par2gpu.par2_constants(k)
    ctx = par2gpu.Context(0)
    ctx.set_timing(True)
    out = {"workload": f"invert: decode matrix m={m} of k={k} slices", "m": m, "k": k}
    for name, exps in (("consecutive", np.arange(m)),
                       ("gapped", np.concatenate([np.arange(m - 1), [m + 4]]))):
        for _ in range(args.warmup):
            ctx.reconstruction_matrix(k, missing, exps)
        ms = []
        for _ in range(max(1, args.steps)):
            inv = ctx.reconstruction_matrix(k, missing, exps)
            ms.append(ctx.last_timing().ms_total)
        ok = True
        for r in rng.choice(m, 4, replace=False):
            acc = np.zeros(m, np.uint16)
            for j, cj in enumerate(c[missing]):
                acc ^= gf.mul(gf.pow(int(cj), exps[r]), inv[j])
            ok = ok and acc[r] == 1 and np.count_nonzero(acc) == 1
        out[name] = {"ms": statistics.median(ms), "identity_rows_ok": bool(ok)}
    ctx.close()
    print(json.dumps(out), flush=True)


def run_create_files(args):
    """Create and repair from files (p2f_create / p2f_repair): the large-encode
    set as 4 files x 512 MiB on tmpfs (page cache), 1 MiB slices, 10 %
    redundancy; then 200 slices of one file zeroed and repaired.  Beside it
    the reference's CPU create path restated: whole-file MD5s of the files in
    parallel, IFSC checksums slice by slice, the AVX2 encode (timed on the
    48 KiB column sample of every slice and scaled to the slice size)."""
    import shutil
    import tempfile
    from concurrent.futures import ThreadPoolExecutor

    from par2gpu import format as fmt

    nfiles, fsize, bs, pct = 4, 512 << 20, 1 << 20, 10.0
    base = "/dev/shm" if os.path.isdir("/dev/shm") and \
        shutil.disk_usage("/dev/shm").free > 3 * nfiles * fsize else None
    d = tempfile.mkdtemp(prefix="p2f_", dir=base)
    try:
        rng = np.random.default_rng(SEED + 9)
        files = []
        for i in range(nfiles):
            p = os.path.join(d, f"file{i}.bin")
            rng.integers(0, 256, fsize, dtype=np.uint8).tofile(p)
            files.append(p)
        # warm-up on a small set of as many files (device context, kernels,
        # one reader thread per file, the pooled pinned chunks they use)
        warm = []
        for i in range(nfiles):
            wp = os.path.join(d, f"warm{i}.bin")
            rng.integers(0, 256, 8 << 20, dtype=np.uint8).tofile(wp)
            warm.append(wp)
        for _ in range(max(1, args.warmup)):
            fmt.create(warm, os.path.join(d, "warm.par2"), block_size=bs, redundancy=pct)
        out = os.path.join(d, "set.par2")
        total = nfiles * fsize
        steps = max(1, args.steps)

        def phases(st):  # total / ingest / gpu / write ms of one run
            return [round(v, 1) for v in (st.ms_total, st.ms_ingest, st.ms_gpu, st.ms_write)]

        def median_run(runs):
            runs = sorted(runs, key=lambda x: x[0].ms_total)
            return runs[len(runs) // 2]

        creates = []
        for _ in range(steps):
            for f in os.listdir(d):
                if f.startswith("set."):
                    os.remove(os.path.join(d, f))
            creates.append((fmt.create(files, out, block_size=bs, redundancy=pct), None))
        st = median_run(creates)[0]
        repairs = []
        for _ in range(steps):
            # damage: 200 slices of file 1 zeroed
            with open(files[1], "r+b") as f:
                f.write(bytes(200 * bs))
            n, rst_i = fmt.repair(out, d)
            repairs.append((rst_i, n))
        rst, n = median_run(repairs)
        res = {"workload": f"create_files: {nfiles} files x {fsize >> 20} MiB (tmpfs: "
                           f"{base is not None}), {bs >> 20} MiB slices, {pct:g}% recovery; repair "
                           f"of 200 zeroed slices; median of {steps} runs each",
               "create": dict(st.as_dict(), gbs=total / (st.ms_total * 1e-3) / 1e9,
                              runs_ms=[phases(x[0]) for x in creates]),
               "repair": dict(rst.as_dict(), rebuilt=n, gbs=total / (rst.ms_total * 1e-3) / 1e9,
                              runs_ms=[phases(x[0]) for x in repairs])}
        # the reference's CPU create path (restated; oracle = OpenSSL MD5, zlib CRC32)
        from oracle import oracle

        threads = os.cpu_count() or 1
        t0 = time.perf_counter()
        data = [np.fromfile(p, np.uint8) for p in files]
        t_read = time.perf_counter() - t0
        t0 = time.perf_counter()
        with ThreadPoolExecutor(nfiles) as ex:
            list(ex.map(oracle.md5, data))
        t_md5 = time.perf_counter() - t0
        slices = np.concatenate(data).reshape(-1, bs)
        t0 = time.perf_counter()
        oracle.hash_slices(slices)
        t_ifsc = time.perf_counter() - t0
        r = int(st.recovery_blocks)
        _, t_enc, _ = cpu_encode_rate(slices, r, threads)
        t_cpu = t_read + t_md5 + t_ifsc + t_enc
        res["cpu_baseline"] = {
            "value": total / t_cpu / 1e9, "unit": "GB/s", "cores": threads, "kind": "port",
            "sample": "whole files: MD5, IFSC and the encode of every slice",
            "s_read": t_read, "s_file_md5": t_md5, "s_ifsc": t_ifsc, "s_encode": t_enc}
        print(json.dumps(res), flush=True)
    finally:
        shutil.rmtree(d, ignore_errors=True)


def batched_sets(seed, nsets=256):
    """The batched configuration's set list: file sizes log-uniform on
    [64 KiB, 256 MiB], slice size uniform over {4, 16, 64, 256, 1024} KiB
    (redrawn while the set would need more than 32768 input slices, the
    number of distinct PAR2 constants), redundancy uniform 1-20 %% with the
    creator's rule r = ceil(floor(k*S*pct/100) / S), even sets create and odd
    sets repair m ~ U{1..r} erased slices with the m lowest exponents."""
    rng = np.random.default_rng(seed)
    sets = []
    for j in range(nsets):
        size = int(np.exp(rng.uniform(np.log(64 << 10), np.log(256 << 20))))
        while True:
            S = int(rng.choice([4, 16, 64, 256, 1024])) << 10
            k = (size + S - 1) // S
            if k <= 32768:
                break
        pct = float(rng.uniform(1.0, 20.0))
        r = max(1, (int(k * S * pct / 100.0) + S - 1) // S)
        spec = {"k": k, "S": S, "r": r, "size": size, "create": j % 2 == 0}
        if not spec["create"]:
            m = int(rng.integers(1, r + 1))
            m = min(m, k)
            spec["m"] = m
            spec["missing"] = np.sort(rng.choice(k, m, replace=False))
        sets.append(spec)
    return sets


def run_batched(args):
    print(json.dumps(batched_leg()), flush=True)


def run_profile_batched(args):
    """An ncu-sized batch for the persistent kernel: the first 48 create sets
    of the batched distribution whose sources are at most 64 MiB, in one
    batch (one persistent launch), run `--warmup` + `--steps` times."""
    import torch

    import par2gpu

    dev = torch.device("cuda", 0)
    sets = [x for x in batched_sets(SEED + 7, 1024) if x["create"] and x["k"] * x["S"] <= 64 << 20][:48]
    g = torch.Generator(device=dev)
    g.manual_seed(SEED + 9)
    ctx = par2gpu.Context(0)
    jobs, keep = [], []
    for x in sets:
        src = torch.randint(0, 256, (x["k"], x["S"]), dtype=torch.uint8, device=dev, generator=g)
        out = torch.zeros((x["r"], x["S"]), dtype=torch.uint8, device=dev)
        keep += [src, out]
        jobs.append({"kind": par2gpu.JOB_CREATE, "k": x["k"], "slice_bytes": x["S"], "src": src,
                     "exps": np.arange(x["r"]), "out": out})
    ms = []
    for step in range(args.warmup + max(1, args.steps)):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        b = par2gpu.Batch(ctx, jobs)
        st = b.run()
        b.close()
        ms.append((time.perf_counter() - t0) * 1e3)
        assert all(v == 0 for v in st), st
    macs = sum(x["k"] * x["r"] * (x["S"] // 2) for x in sets)
    print(json.dumps({"workload": "profile_batched: 48 create sets of the batched distribution, "
                                  "sources at most 64 MiB each, one batch",
                      "sets": len(sets), "source_bytes": sum(x["k"] * x["S"] for x in sets),
                      "symbol_macs": macs, "ms_per_run": ms[args.warmup:]}), flush=True)
    ctx.close()


def batched_leg():
    """Many independent sets: per-set plain calls (p2g_encode / p2g_repair,
    one set after another) against the batch executor (one persistent kernel
    per phase over all sets' work items, longest first), and the batch's
    captured CUDA graph replayed.  Jobs/s and makespan; outputs compared.
    Returns the results."""
    import torch

    import par2gpu

    dev = torch.device("cuda", 0)
    sets = batched_sets(SEED + 7)
    ctx = par2gpu.Context(0)
    st = torch.cuda.current_stream(dev)
    ctx.set_stream(st.cuda_stream)
    ctx.set_timing(True)
    g = torch.Generator(device=dev)
    g.manual_seed(SEED + 8)
    total_src = sum(x["k"] * x["S"] for x in sets)
    # sources, recovery and two output copies per set
    for x in sets:
        x["src"] = torch.randint(0, 256, (x["k"], x["S"]), dtype=torch.uint8, device=dev,
                                 generator=g)
        if x["create"]:
            x["out_plain"] = torch.zeros((x["r"], x["S"]), dtype=torch.uint8, device=dev)
            x["out_batch"] = torch.zeros_like(x["out_plain"])
        else:
            m = x["m"]
            x["rec"] = torch.zeros((m, x["S"]), dtype=torch.uint8, device=dev)
            ctx.encode([x["src"][i] for i in range(x["k"])], x["S"], np.arange(m),
                       [x["rec"][q] for q in range(m)], device=True)
            # exponent 0 is the XOR of all slices: a cheap check of the setup
            par = x["src"]
            while par.shape[0] > 1:
                h = par.shape[0] // 2
                nxt = par[:h] ^ par[h:2 * h]
                if par.shape[0] % 2:
                    nxt[0] ^= par[-1]
                par = nxt
            x["rec0_ok"] = bool(torch.equal(par[0], x["rec"][0]))
            x["pristine"] = x["src"][torch.from_numpy(x["missing"]).to(dev)].clone()
            x["src"][torch.from_numpy(x["missing"]).to(dev)] = 0   # erased
            x["out_plain"] = torch.zeros((m, x["S"]), dtype=torch.uint8, device=dev)
            x["out_batch"] = torch.zeros_like(x["out_plain"])

    # each set's slice tables (device addresses, uint64), built once as a
    # caller holds them: neither arm times Python list building
    def rows(t, keep=None):
        a = np.uint64(t.data_ptr()) + np.arange(t.shape[0], dtype=np.uint64) * \
            np.uint64(t.stride(0))
        return a if keep is None else a[keep]

    for x in sets:
        x["t_src"] = rows(x["src"])
        x["t_out_plain"] = rows(x["out_plain"])
        x["t_out_batch"] = rows(x["out_batch"])
        if not x["create"]:
            keep = np.ones(x["k"], bool)
            keep[x["missing"]] = False
            x["t_present"] = rows(x["src"], keep)
            x["t_rec"] = rows(x["rec"])

    def plain_all():
        for x in sets:
            k, S = x["k"], x["S"]
            if x["create"]:
                ctx.encode(x["t_src"], S, np.arange(x["r"]), x["t_out_plain"], device=True)
            else:
                ctx.repair(k, S, x["missing"], x["t_present"], np.arange(x["m"]), x["t_rec"],
                           x["t_out_plain"], device=True)

    def jobs_for(xs):
        jobs = []
        for x in xs:
            k, S = x["k"], x["S"]
            if x["create"]:
                jobs.append({"kind": par2gpu.JOB_CREATE, "k": k, "slice_bytes": S,
                             "src": x["t_src"], "exps": np.arange(x["r"]),
                             "out": x["t_out_batch"]})
            else:
                jobs.append({"kind": par2gpu.JOB_REPAIR, "k": k, "slice_bytes": S,
                             "src": x["t_present"], "missing": x["missing"],
                             "exps": np.arange(x["m"]), "recovery": x["t_rec"],
                             "out": x["t_out_batch"]})
        return jobs

    # groups whose scratch (bit planes + records) fits the budget
    budget = 48 << 30
    groups, cur, used = [], [], 0
    for x in sets:
        n = x["r"] if x["create"] else x["m"]
        need = x["k"] * x["S"] + x["k"] * n * 64
        if cur and used + need > budget:
            groups.append(cur)
            cur, used = [], 0
        cur.append(x)
        used += need
    groups.append(cur)

    def batched_all():
        for grp in groups:
            b = par2gpu.Batch(ctx, jobs_for(grp))
            stv = b.run()
            b.close()
            assert all(v == 0 for v in stv), stv

    # the batch kernel's tile form per problem class, tuned on this device
    # before anything is timed
    forms, form_ms = ctx.batch_autotune(reps=2)
    names = {par2gpu.FORM_WIDE: "wide", par2gpu.FORM_SMALL: "small",
             par2gpu.FORM_PAIRED: "paired"}
    out = {"workload": "batched: 256 sets, file sizes log-uniform 64 KiB-256 MiB, slices "
                       "{4,16,64,256,1024} KiB, redundancy 1-20%, half create / half repair",
           "sets": len(sets), "source_bytes": total_src, "batches": len(groups),
           "tuned_forms": {f"outputs {o}, slices {sz}": names[forms[2 * i + j]]
                           for i, o in enumerate(("1-24", "25-104", "105-208", ">208"))
                           for j, sz in enumerate(("<=16KiB", ">16KiB"))}}
    for name, fn in (("plain", plain_all), ("batched", batched_all)):
        fn()  # warm-up
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
        out[name] = {"makespan_ms": ms, "jobs_per_s": len(sets) / (ms * 1e-3),
                     "source_gbs": total_src / (ms * 1e-3) / 1e9}
    # graph replay of the prepared batches (decode matrices supplied)
    graphs = []
    for grp in groups:
        jobs = jobs_for(grp)
        for x, jb in zip(grp, jobs):
            if not x["create"]:
                jb["inverse"] = ctx.reconstruction_matrix(x["k"], x["missing"], np.arange(x["m"]))
        graphs.append(par2gpu.Batch(ctx, jobs, graph=True))
    for b in graphs:
        b.run()
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for b in graphs:
        b.run()
    e1.record(st)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    out["graph_replay"] = {"makespan_ms": ms, "jobs_per_s": len(sets) / (ms * 1e-3),
                           "note": "decode matrices precomputed; device work only"}
    # the multiply-accumulate work of all sets (create: k x r, repair: one
    # pass of k sources x m outputs) against the LOP3 roofline, per arm
    macs = sum(x["k"] * (x["r"] if x["create"] else x["m"]) * (x["S"] // 2) for x in sets)
    int_peak, _ = probe_int_peak(0)
    out["symbol_macs"] = macs
    for name in ("plain", "batched", "graph_replay"):
        if int_peak:
            out[name]["int_frac"] = 2.0 * macs / (out[name]["makespan_ms"] * 1e-3) / int_peak
    for b in graphs:
        b.close()
    same = all(torch.equal(x["out_plain"], x["out_batch"]) for x in sets)
    bad = [(x["k"], x["S"], x["m"]) for x in sets
           if not x["create"] and not torch.equal(x["out_batch"], x["pristine"])]
    out["setup_rec0_ok"] = all(x["rec0_ok"] for x in sets if not x["create"])
    out["batched_equals_plain"] = bool(same)
    out["repairs_bit_exact"] = not bad
    if bad:
        out["repair_mismatch_sets"] = bad[:20]
    ctx.close()
    del sets, graphs
    torch.cuda.empty_cache()
    return out


def serving_pool(dev, nsets, seed):
    """Device-resident job data for the serving loop: sets drawn from the
    batched distribution; each arrival becomes a create (40 %), verify (40 %)
    or repair (20 %) job over one of them."""
    import torch

    sets = batched_sets(seed, nsets)
    g = torch.Generator(device=dev)
    g.manual_seed(seed + 1)
    pool = []
    for x in sets:
        src = torch.randint(0, 256, (x["k"], x["S"]), dtype=torch.uint8, device=dev, generator=g)
        pool.append({"spec": x, "src": src})
    return pool


def repair_data(p, ctx):
    """The recovery slices and erasures of a pool set's repair jobs, made once
    (its own generator: every job list sees the same data)."""
    import torch

    if "rec" not in p:
        x = p["spec"]
        m = max(1, min(x["k"], x.get("m", 1)))
        prng = np.random.default_rng(x["k"] * 7919 + x["S"])
        miss = np.sort(prng.choice(x["k"], m, replace=False))
        rec = torch.zeros((m, x["S"]), dtype=torch.uint8, device=p["src"].device)
        ctx.encode([p["src"][i] for i in range(x["k"])], x["S"], np.arange(m),
                   [rec[q] for q in range(m)], device=True)
        p["rec"], p["miss"] = rec, miss
    return p["miss"], p["rec"]


def make_jobs(pool, nj, rng, ctx):
    from par2gpu.serve import ServedJob

    jobs = []
    for jid in range(nj):
        p = pool[int(rng.integers(len(pool)))]
        x = p["spec"]
        u = rng.uniform()
        if u < 0.4:
            jobs.append(ServedJob(jid, "create", p["src"], r=x["r"]))
        elif u < 0.8:
            jobs.append(ServedJob(jid, "verify", p["src"]))
        else:
            miss, rec = repair_data(p, ctx)
            jobs.append(ServedJob(jid, "repair", p["src"], missing=miss, rec=rec))
    return jobs


def run_serving(args):
    print(json.dumps(serving_leg((10, 100, 500, 1000, 2000))), flush=True)


def serving_leg(rates):
    """Poisson arrivals at the given rates (jobs/s); continuous batching
    versus one job at a time on the same GPU and the same arrival times;
    jobs/s and p50/p95/p99 latency; every job's outputs compared between the
    two.  Returns the results."""
    import torch

    import par2gpu
    from par2gpu.serve import latency_stats, serve_continuous, serve_one_at_a_time

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    ctxs = [par2gpu.Context(0), par2gpu.Context(0), par2gpu.Context(0)]
    pool = serving_pool(dev, 48, SEED + 21)
    torch.cuda.synchronize(dev)
    # untimed warm-up of both servers to their steady state: every set of the
    # pool as a create, a verify and a repair job, so that every scratch
    # buffer has reached its size (growing one frees it, and a free
    # synchronises the device)
    from par2gpu.serve import ServedJob

    warm = []
    for p in pool:
        miss, rec = repair_data(p, ctxs[0])
        warm.append(ServedJob(len(warm), "create", p["src"], r=p["spec"]["r"]))
        warm.append(ServedJob(len(warm), "verify", p["src"]))
        warm.append(ServedJob(len(warm), "repair", p["src"], missing=miss, rec=rec))
    for _ in range(2):
        for j in warm:
            j.out = j.md5 = j.crc = j.inverse = None
        serve_continuous(ctxs, warm, np.zeros(len(warm)))
        serve_one_at_a_time(ctxs[0], warm, np.zeros(len(warm)))
    del warm
    torch.cuda.synchronize(dev)
    results = []
    for lam in rates:
        rng = np.random.default_rng(SEED + lam)
        nj = int(min(600, max(120, lam * 2)))  # p99 of 120-600 jobs
        arrivals = np.cumsum(rng.exponential(1.0 / lam, nj))
        jobs_a = make_jobs(pool, nj, np.random.default_rng(SEED + 100 + lam), ctxs[0])
        jobs_b = make_jobs(pool, nj, np.random.default_rng(SEED + 100 + lam), ctxs[0])
        torch.cuda.synchronize(dev)
        lat_a, wall_a = serve_continuous(ctxs, jobs_a, arrivals)
        torch.cuda.synchronize(dev)
        lat_b, wall_b = serve_one_at_a_time(ctxs[0], jobs_b, arrivals)
        torch.cuda.synchronize(dev)
        same = True
        for ja, jb in zip(jobs_a, jobs_b):
            if ja.kind == "verify":
                same = same and np.array_equal(ja.md5, jb.md5) and np.array_equal(ja.crc, jb.crc)
            else:
                same = same and bool(torch.equal(ja.out, jb.out))
        results.append({"rate_jobs_per_s": lam, "continuous": latency_stats(lat_a, wall_a),
                        "one_at_a_time": latency_stats(lat_b, wall_b),
                        "outputs_identical": bool(same)})
        del jobs_a, jobs_b
    for c in ctxs:
        c.close()
    del pool
    torch.cuda.empty_cache()
    return {"workload": "serving: Poisson arrivals, 40% create / 40% verify / 20% repair, "
                        "sizes from the batched distribution (48 device-resident sets), "
                        "120 GB admission budget",
            "all_outputs_identical": all(x["outputs_identical"] for x in results),
            "sweep": results}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="large_encode",
                    choices=sorted(WORKLOADS) + sorted(HASH_WORKLOADS) +
                    ["verify_repair", "invert", "create_files", "batched",
                     "serving", "profile_batched"])
    ap.add_argument("--no-autotune", action="store_true",
                    help="use the heuristic tile shape instead of the autotuned one")
    ap.add_argument("--quick", action="store_true",
                    help="device-resident timing only (no e2e, roofline probe or CPU baseline)")
    ap.add_argument("--no-legs", action="store_true",
                    help="large_encode without the repair / batched / serving parts")
    args = ap.parse_args()
    if args.workload in HASH_WORKLOADS:
        run_hash(args)
        return
    if args.workload == "verify_repair":
        run_verify_repair(args)
        return
    if args.workload == "invert":
        run_invert(args)
        return
        return
    if args.workload == "create_files":
        run_create_files(args)
        return
    if args.workload == "batched":
        run_batched(args)
        return
    if args.workload == "profile_batched":
        run_profile_batched(args)
        return
    if args.workload == "serving":
        run_serving(args)
        return
    global K_SRC, SLICE, R_REC, WORKLOAD
    K_SRC, SLICE, R_REC, WORKLOAD = WORKLOADS[args.workload]
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    try:
        run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
