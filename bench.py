"""Benchmark: primes tested/s of the plain BSGS sieve on the 100-sequence job.

Workload (config 2): 100 sequences k*2^n+-1 (50 with +1, 50 with -1), k odd
in [3,2^32), n in [4e6,1e7) kept with probability 0.03 (seeded synthetic
bitmap, ~1.8e7 candidate terms), sieved over consecutive windows of the
p-range [2^50, 2^50+2^38).  One step = one rs_run_range call over a window of
width --width (default 2^29, ~1.5e7 primes): prime generation, per-prime
set-up and the BSGS search, with factors accumulating on the device.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--width BITS] [--impl ours|reference]

Multi-GPU (torchrun, one rank per GPU): each rank sieves its own disjoint
windows (weak scaling, no data-path collective); the timed region is bracketed
by barriers and the max over ranks is reported.  `value` counts inputs already
resident in HBM; `e2e` runs the same windows through the C ABI with the job's
host buffers (pinned) uploaded and the factors downloaded every step.
--impl reference times the CPU port of the reference algorithm (oracle/,
kind "port": the reference ships only OpenCL kernels, no CPU path) on a
bounded sample of the same workload with every host thread.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "primes tested/s at 100 seqs, batched vs plain on 1 B200; p50/p99 unit latency"
WORKLOAD = ("config2 plain form: 100 seqs k*2^n+-1 (50 +1, 50 -1), k odd U[3,2^32), n in [4e6,1e7) "
            "kept w.p. 0.03, p windows from 2^50")
P_START = 1 << 50
# DRAM bytes (read + write) per prime of the BSGS kernel, from one ncu capture
# of a 2^20-wide window at 2^50 at the tuned Q = 8192 (69.36 MB for 30 203
# primes, FP64 steps and start values): the 2272-byte prime record plus
# claims.  Traffic grows in proportion to primes, so the per-launch figure is
# this times the primes one launch processes.
BSGS_DRAM_BYTES_PER_PRIME = 2296.4


def reference_params(nmin, nmax):
    """The reference's BSGS parameters for an n-range (cl_sieve.cpp:893-938): Q
    doubles from 1024 while below both 4096 and ceil(sqrt(L)); M = ceil(L/Q) giant
    steps for full-range sequences, MM = ceil(L/2Q) for single-parity ones."""
    L = nmax - nmin + 1
    target = math.ceil(math.sqrt(L))
    q = 1024
    while q < 4096 and q < target:
        q <<= 1
    return {"Q": q, "M": -(-L // q), "MM": -(-L // (2 * q))}


def mulmod_rates(counters, seconds, peak_g):
    """Giant-step products (one modular product each) and baby steps per second
    over a whole run, and the giant rate as a fraction of the measured peak."""
    g = counters["giant"] / seconds
    return {"giant_products_per_s": g, "baby_steps_per_s": counters["baby"] / seconds,
            "giant_frac_of_mulmod_peak": g / (peak_g * 1e9)}


def job_of(name, seed, W):
    """(job, first p, workload label) of the timed steps' job."""
    if name == "config2":
        return W.config2(seed), P_START, WORKLOAD
    if name == "config1":
        j = W.config1(1)
        return j, j["prange"][0], "config1 job: 8 seqs k*2^n-1, k odd < 2^20, n in [1e5,3e5), p windows from 1e12"
    if name == "config4":
        j = W.config4()
        return j, j["prange"][0], ("config4 job: 20 seqs b=5, k even < 2^40, n in [1e6,3e6), p windows from "
                                   "2^64-2^36")
    if name.startswith("config3:"):
        i = int(name.split(":")[1])
        j = W.config3(3)[i]
        return j, j["prange"][0], "config3 job %d: %d seqs b=%d, n in [%d,%d], p windows from %d" % (
            i, len(j["k"]), j["base"], j["nmin"], j["nmax"], j["prange"][0])
    raise ValueError("unknown --job %s" % name)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--width", type=int, default=29, help="log2 of the p-window per step")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--baby-steps", type=int, default=0, help="fix Q baby steps per prime (0: the per-job tuner)")
    ap.add_argument("--no-forms", action="store_true",
                    help="skip the batched (configs 2, 3, 4) and served (config 5) forms")
    ap.add_argument("--serve-rates", default="", help="extra arrival rates (units/s, comma-separated) to serve")
    ap.add_argument("--form", default="",
                    help="run only this form (config1, batched, batched_config2, batched_config4, served, "
                         "served_stated, served_stated_low) and print its result, for profiling it on its own")
    ap.add_argument("--job", default="config2",
                    help="job of the timed steps: config2 (the benchmark), config1, config4 or config3:<index>; "
                         "the others are for profiling single kernels on those shapes")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU-baseline sample length")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, gpu):
        self.path = os.path.join("/tmp", "rs_clocks_%d_%d.csv" % (os.getpid(), gpu))
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(self.path, "w")
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.fh.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in open(self.path):
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(seed, target_s, job=None):
    """The oracle's CPU port of the reference BSGS algorithm on a bounded sample of the workload."""
    from oracle import pyoracle as O
    from rssieve_b200 import workloads as W
    job = job or W.config2(seed)
    oj = O.Job(job["base"], job["k"], job["c"], job["nmin"], job["nmax"], job["bitmap"])
    threads = os.cpu_count() or 1
    pl = O.prp2(P_START, P_START + 400_000)           # the reference's own prime set (2-PRPs)
    t = time.perf_counter()
    O.bsgs(oj, pl[: 64 * threads], nthreads=threads)
    pilot = 64 * threads / max(time.perf_counter() - t, 1e-6)
    want = int(min(max(pilot * target_s, 32 * threads), 2_000_000))
    width = int(want * 36.0) + 1000
    pl = O.prp2(P_START, P_START + width)[:want]
    t = time.perf_counter()
    f, st, _ = O.bsgs(oj, pl, nthreads=threads)
    dt = time.perf_counter() - t
    return {"value": len(pl) / dt, "unit": "primes/s", "cores": threads, "kind": "port",
            "sample": "%d 2-PRPs from 2^50 (config2 job), %d threads, %.1f s; %.3g Montgomery products/s" % (
                len(pl), threads, dt, st["mulmods"] / dt)}


def measure_batched(torch, rs, W, peak_g, seed=3, njobs=48, window_log2=24):
    """Config-3 sample: the same jobs and p-windows through the single-job path, job
    after job, and through one batch.  CUDA events on one side stream bracket the
    uploads (each job's bitmap and tables, from pageable host memory) and the
    sieving separately, so the ratio is reported with and without the uploads."""
    jobs = W.config3(seed, njobs=njobs)
    seqs = [W.seqs_of(j) for j in jobs]
    wins = [(j["prange"][0], j["prange"][0] + (1 << window_log2)) for j in jobs]
    st = torch.cuda.Stream()

    def ev():
        return torch.cuda.Event(enable_timing=True)
    sv = rs.Sieve(torch.cuda.current_device())
    sv.set_stream(st.cuda_stream)
    plain_terms, plain_primes, load_ms, run_ms = [], 0, 0.0, 0.0
    plain_ctr = {"giant": 0, "baby": 0}
    torch.cuda.synchronize()
    for sq, (p0, p1) in zip(seqs, wins):
        e = [ev() for _ in range(3)]
        e[0].record(st)
        sv.load(sq)
        e[1].record(st)
        c = sv.run(p0, p1)
        plain_primes += c["primes"]
        for k in plain_ctr:
            plain_ctr[k] += c[k]
        e[2].record(st)
        torch.cuda.synchronize()
        load_ms += e[0].elapsed_time(e[1])
        run_ms += e[1].elapsed_time(e[2])
        f = sv.factors()
        plain_terms.append(set(zip(f["seq"].tolist(), f["n"].tolist())))
    sv.close()
    b = rs.Batch(torch.cuda.current_device(), max_jobs=njobs, range_slots=njobs + 8)
    b.set_stream(st.cuda_stream)
    e = [ev() for _ in range(3)]
    torch.cuda.synchronize()
    e[0].record(st)
    ids = [b.add(sq, p0, p1) for sq, (p0, p1) in zip(seqs, wins)]
    e[1].record(st)
    b.run(0)
    e[2].record(st)
    torch.cuda.synchronize()
    b_load, b_run = e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])
    batch_primes = sum(b.job_info(j)[1] for j in ids)
    same = all(set(zip(f["seq"].tolist(), f["n"].tolist())) == t
               for f, t in zip((b.factors(j) for j in ids), plain_terms))
    qs = sorted(set(b.job_info(j)[0] for j in ids))
    batch_ctr = b.counters()
    b.close()
    return {"workload": "config3 sample: %d jobs (1-100 seqs, b in {2,3,5,6,10}, n from 1e6, p from 2^44..2^60), "
                        "2^%d-wide p-window each" % (njobs, window_log2),
            "primes": int(batch_primes),
            "plain_primes_per_s": plain_primes / (run_ms / 1e3),
            "batched_primes_per_s": batch_primes / (b_run / 1e3),
            "batched_over_plain": run_ms / b_run,
            "with_uploads": {"plain_primes_per_s": plain_primes / ((load_ms + run_ms) / 1e3),
                             "batched_primes_per_s": batch_primes / ((b_load + b_run) / 1e3),
                             "batched_over_plain": (load_ms + run_ms) / (b_load + b_run),
                             "upload_ms": {"plain": load_ms, "batched": b_load}},
            "mulmods": {"plain": mulmod_rates(plain_ctr, run_ms / 1e3, peak_g),
                        "batched": mulmod_rates(batch_ctr, b_run / 1e3, peak_g)},
            "identical_eliminated_terms": bool(same and plain_primes == batch_primes), "baby_steps_used": qs}


def measure_one_job_batched(torch, rs, W, peak_g, job, p0, width_log2, nsplit, label):
    """One job over one p-window through the single-job path and through the batch
    (a resident copy of the job cloned over nsplit range slots, at the Q the
    single-job tuner measured for the job's shape); CUDA events on one side stream
    bracket the sieving of each, with the job already resident on the device
    (the single-job load and the batch's upload and clone outside)."""
    import numpy as np
    seqs = W.seqs_of(job)
    p1 = p0 + (1 << width_log2)
    st = torch.cuda.Stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    sv = rs.Sieve(torch.cuda.current_device())
    sv.set_stream(st.cuda_stream)
    sv.load(seqs)
    sv.run(p0, p0 + (1 << 26))                 # warm: the tuner measures this job shape's Q
    sv.load(seqs)
    torch.cuda.synchronize()
    ev[0].record(st)
    plain_ctr = sv.run(p0, p1)
    plain_primes = plain_ctr["primes"]
    ev[1].record(st)
    torch.cuda.synchronize()
    f = sv.factors()
    plain_terms = set(zip(f["seq"].tolist(), f["n"].tolist()))
    plain_bm = sv.bitmap()
    sv.close()
    b = rs.Batch(torch.cuda.current_device(), max_jobs=2, range_slots=nsplit)
    b.set_stream(st.cuda_stream)
    t = b.add(seqs, p0, p0)
    j = b.add_clone(t, p0, p1, nsplit)
    torch.cuda.synchronize()
    ev[2].record(st)                           # the job resident on both sides: sieving only
    b.run(0)
    ev[3].record(st)
    torch.cuda.synchronize()
    f = b.factors(j)
    q, batch_primes, _ = b.job_info(j)
    same = (set(zip(f["seq"].tolist(), f["n"].tolist())) == plain_terms and batch_primes == plain_primes
            and np.array_equal(b.bitmap(j), plain_bm))
    batch_ctr = b.counters()
    b.close()
    pms, bms = ev[0].elapsed_time(ev[1]), ev[2].elapsed_time(ev[3])
    return {"workload": "%s: one 2^%d-wide p-window from %s, batch over %d range slots" % (
                label, width_log2, hex(p0), nsplit),
            "primes": int(batch_primes), "plain_primes_per_s": plain_primes / (pms / 1e3),
            "batched_primes_per_s": batch_primes / (bms / 1e3), "batched_over_plain": pms / bms,
            "mulmods": {"plain": mulmod_rates(plain_ctr, pms / 1e3, peak_g),
                        "batched": mulmod_rates(batch_ctr, bms / 1e3, peak_g)},
            "identical_eliminated_terms": bool(same), "baby_steps_used": q}


def measure_config1(torch, rs, W, peak_g):
    """Config 1 end to end (8 sequences k*2^n-1, k < 2^20, n in [1e5, 3e5), the
    whole p-range [1e12, 1e12+1e8)): the GPU through the C ABI (upload, every
    prime, factors back) beside the CPU port of the reference algorithm on every
    host thread over the same range; term sets compared between the two, and
    with the brute-force oracle on the first 2e6 of the range."""
    import numpy as np
    from oracle import pyoracle as O
    job = W.config1(1)
    seqs = W.seqs_of(job)
    p0, p1 = job["prange"]
    st = torch.cuda.Stream()
    sv = rs.Sieve(torch.cuda.current_device())
    sv.set_stream(st.cuda_stream)
    sv.load(seqs)
    sv.run(p0, p1)                             # the tuner settles this job shape's Q
    sv.factors()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    ev[0].record(st)
    sv.load(seqs)
    c = sv.run(p0, p1)
    f = sv.factors()
    ev[1].record(st)
    torch.cuda.synchronize()
    gms = ev[0].elapsed_time(ev[1])
    q, _ = sv.baby_steps()
    gpu_terms = O.term_set(f)
    sub = sv
    sub.load(seqs)
    sub.run(p0, p0 + 2_000_000)
    fsub = sub.factors()
    sv.close()
    oj = O.Job(job["base"], job["k"], job["c"], job["nmin"], job["nmax"], job["bitmap"])
    threads = os.cpu_count() or 1
    pl = O.prp2(p0, p1)
    t = time.perf_counter()
    pf, pst, _ = O.bsgs(oj, pl, nthreads=threads)
    cdt = time.perf_counter() - t
    bf, _, _ = O.brute(oj, O.primes(p0, p0 + 2_000_000))
    return {"workload": "config1: 8 seqs k*2^n-1, k odd < 2^20, n in [1e5,3e5) kept w.p. 0.06, "
                        "p in [1e12, 1e12+1e8), whole range",
            "primes": int(c["primes"]), "baby_steps_used": q,
            "gpu_e2e_primes_per_s": c["primes"] / (gms / 1e3), "gpu_e2e_s": gms / 1e3,
            "cpu_port_primes_per_s": len(pl) / cdt, "cpu_port_s": cdt, "cpu_port_cores": threads,
            "cpu_port_prime_set": "base-2 strong probable primes (the reference's)",
            "gpu_over_cpu_port": (c["primes"] / (gms / 1e3)) / (len(pl) / cdt),
            "factors": len(gpu_terms),
            "identical_eliminated_terms_gpu_vs_port": gpu_terms == O.term_set(pf),
            "identical_eliminated_terms_gpu_vs_brute_first_2e6": O.term_set(fsub) == O.term_set(bf),
            "mulmods": {"gpu": mulmod_rates(c, gms / 1e3, peak_g)}}


def measure_served(rs, W, serve, peak_g, seed=5, nunits=60, rate=8.0, width_log2=(22, 26), rho=None,
                   primes_per_s=None, label=None):
    """Config-5 shape: 16 config-2-style files, Poisson arrivals at `rate` units/s
    (or, with rho, at the rate that loads the GPU to rho given its measured
    primes_per_s), unit widths 2^width_log2 (the full workload's are 2^30..2^36);
    latency from arrival and from admission, and each unit's latency over its own
    run time alone on the same server."""
    import numpy as np
    files = [W.seqs_of(f) for f in W.config5_files(seed)]
    if rho is not None:
        # mean service time of a unit alone: its primes (width / ln p0) at the measured rate
        probe = W.config5_units(seed, nunits, 1.0, len(files), width_log2)
        mean_primes = sum((p1 - p0) / math.log(p0) for _, _, p0, p1 in probe) / len(probe)
        rate = rho / (mean_primes / primes_per_s)
    raw = W.config5_units(seed, nunits, rate, len(files), width_log2)
    units = [serve.Unit(k, fi, p0, p1, t) for k, (t, fi, p0, p1) in enumerate(raw)]
    srv = serve.Server(files, max_units=48, range_slots=64)
    try:
        busy0, c0 = srv.busy_s, srv.batch.counters()
        out = srv.run(units)
        c1 = srv.batch.counters()
        st = serve.latency_stats(out)
        st["gpu_busy"] = (srv.busy_s - busy0) / st["span_s"]
        st["mulmods_while_busy"] = mulmod_rates({k: c1[k] - c0[k] for k in ("giant", "baby")},
                                                srv.busy_s - busy0, peak_g)
        ratios = []
        for u in out:
            v = serve.Unit(u.uid, u.file, u.p0, u.p1, 0.0)
            srv.run([v])
            ratios.append((u.finished - u.arrival) / max(v.finished - v.admitted, 1e-6))
    finally:
        srv.close()
    st.update({"workload": label or ("config5 shape scaled down: %d units over 16 files, Poisson %.0f units/s, "
                                     "widths 2^%d..2^%d, starts 2^44..2^62" % (nunits, rate, width_log2[0],
                                                                               width_log2[1])),
               "arrival_rate_per_s": rate,
               "latency_over_isolated_p50": float(np.percentile(ratios, 50)),
               "latency_over_isolated_p99": float(np.percentile(ratios, 99)),
               "latency_over_isolated_max": float(max(ratios)),
               "policy": "%s, %.0f ms rounds" % (srv.policy, srv.round_s * 1e3)})
    return st


def forms_of(torch, rs, W, peak, value, job, names):
    """The batched and served forms (and config 1) named in names."""
    from rssieve_b200 import serve
    makers = {
        "config1": lambda: measure_config1(torch, rs, W, peak),
        "batched": lambda: measure_batched(torch, rs, W, peak),
        "batched_config2": lambda: measure_one_job_batched(torch, rs, W, peak, job, P_START + (1 << 37), 29, 32,
                                                           "config2 job"),
        "batched_config4": lambda: measure_one_job_batched(
            torch, rs, W, peak, W.config4(), (1 << 64) - (1 << 36), 30, 32,
            "config4 job (b=5, 20 seqs, k even < 2^40, p near 2^64)"),
        "served": lambda: measure_served(rs, W, serve, peak),
        "served_stated": lambda: measure_served(
            rs, W, serve, peak, seed=6, nunits=5, width_log2=(30, 31), rho=0.5, primes_per_s=value,
            label="config5 units at the lower end of their stated widths: 5 units of 2^U{30..31} over 16 files, "
                  "starts log-uniform in [2^44, 2^62], Poisson arrivals at the rate that loads the GPU to 0.5"),
        "served_stated_low": lambda: measure_served(
            rs, W, serve, peak, seed=6, nunits=5, width_log2=(30, 31), rho=0.3, primes_per_s=value,
            label="config5 units at the lower end of their stated widths: 5 units of 2^U{30..31} over 16 files, "
                  "starts log-uniform in [2^44, 2^62], Poisson arrivals at the rate that loads the GPU to 0.3"),
    }
    return {n: makers[n]() for n in names}


def run_form(args, torch):
    """One form on its own (no timed steps), for profiling."""
    import rssieve_b200 as rs
    from rssieve_b200 import workloads as W
    with rs.Sieve(torch.cuda.current_device()) as sv:
        peak = sv.mulmod_peak()
    out = forms_of(torch, rs, W, peak, 1.5e7, W.config2(args.seed), [args.form])
    print(json.dumps(out), flush=True)


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    res = []
    from rssieve_b200 import workloads as W
    job = W.config2(args.seed)
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(args.seed, max(2.0, args.cpu_seconds / 2), job)
        if i >= args.warmup:
            res.append(r)
    v = statistics.median(r["value"] for r in res)
    line = {"metric": METRIC, "value": v, "unit": "primes/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "p_window": "bounded CPU sample from 2^50"},
            "cpu_baseline": {"value": v, "unit": "primes/s", "cores": res[0]["cores"], "kind": "port",
                             "sample": res[-1]["sample"]},
            "e2e": {"value": v, "unit": "primes/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    rank, world, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    if args.form:
        return run_form(args, torch)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    import numpy as np
    import rssieve_b200 as rs
    from rssieve_b200 import workloads as W

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM)
        return float(t.item())

    job, p_start, workload = job_of(args.job, args.seed, W)
    seqs = W.seqs_of(job)
    stream = torch.cuda.current_stream()
    sv = rs.Sieve(local)
    sv.set_stream(stream.cuda_stream)
    peak = sv.mulmod_peak()
    wide = sv.widemul_peak()
    fpeak = sv.fpmul_peak()
    sms = torch.cuda.get_device_properties(local).multi_processor_count
    sv.set_baby_steps(args.baby_steps)
    sv.load(seqs)
    width = 1 << args.width
    # disjoint windows per rank: rank r takes windows r, r+world, ...
    nwin = args.warmup + args.steps
    windows = [(p_start + (i * world + rank) * width, p_start + (i * world + rank + 1) * width) for i in range(nwin)]
    l2_flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    for i in range(args.warmup):
        sv.run(*windows[i])
    sv.factors()
    baby_q, tuning = sv.baby_steps()                  # the per-job tuner settles during the warm-up
    torch.cuda.synchronize()
    barrier()

    clk = Clocks(local)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    tot = {}
    bsgs_ms, bsgs_launches, kernel_launches = 0.0, 0, 0
    barrier()
    torch.cuda.synchronize()
    t_wall = time.perf_counter()
    for i in range(args.steps):
        l2_flush.zero_()                               # flush L2 between steps (outside the step events)
        evs[i][0].record(stream)
        c = sv.run(*windows[args.warmup + i])
        evs[i][1].record(stream)
        tm = sv.last_timing()
        bsgs_ms += tm["bsgs_ms_avg"] * tm["bsgs_launches"]
        bsgs_launches += tm["bsgs_launches"]
        kernel_launches += tm["kernel_launches"]
        for k, v in c.items():
            tot[k] = tot.get(k, 0) + v
    torch.cuda.synchronize()
    barrier()
    wall = time.perf_counter() - t_wall
    clocks = clk.stop()
    dev_ms = sum(a.elapsed_time(b) for a, b in evs)
    dev_ms_max = max_over_ranks(dev_ms)
    primes_all = sum_over_ranks(tot["primes"])
    value = primes_all / (dev_ms_max / 1e3)
    giant_all = sum_over_ranks(tot["giant"])
    bsgs_ms_avg = bsgs_ms / max(bsgs_launches, 1)
    # roofline of the BSGS kernel: its executed steps per launch (baby steps and
    # giant steps, one modular product -- or doublings for b^e <= 4 -- and one
    # table insert or probe each) / average launch time
    achieved = ((tot["giant"] + tot["baby"]) / max(bsgs_launches, 1)) / (bsgs_ms_avg / 1e3) / 1e9
    peak_mult = wide / 11.0                       # products the 32x32->64 multiplier allows
    # below 2^51 the steps' products run on the FP64 pipe: the roofline is then
    # the FP64 product rate; above, the Montgomery-product rate
    fp_steps = p_start + nwin * world * width <= (1 << 51)
    rpeak = fpeak if fp_steps else peak
    fac = sv.factors()

    e2e = None
    if not args.no_e2e:
        # end to end through the C ABI: pinned host job -> device each step, factors -> host each step
        bm = seqs.bitmap
        cudart = torch.cuda.cudart()
        cudart.cudaHostRegister(bm.ctypes.data, bm.nbytes, 0)
        ewin = [(p_start + ((nwin + i) * world + rank) * width, p_start + ((nwin + i) * world + rank + 1) * width)
                for i in range(args.steps)]
        sv.load(seqs)
        sv.run(*ewin[0])                               # warm the load/run/fetch path once
        sv.factors()
        torch.cuda.synchronize()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eprimes, d2h = 0, 0
        for i in range(args.steps):
            sv.load(seqs)
            c = sv.run(*ewin[i])
            f = sv.factors()
            eprimes += c["primes"]
            d2h += len(f) * 16 + 13 * 8
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ems = max_over_ranks(e0.elapsed_time(e1))
        cudart.cudaHostUnregister(bm.ctypes.data)
        e2e = {"value": sum_over_ranks(eprimes) / (ems / 1e3), "unit": "primes/s",
               "h2d_bytes_per_step": int(bm.nbytes + 2400), "d2h_bytes_per_step": int(d2h / args.steps)}

    cpu = None
    if rank == 0 and world == 1:
        cpu = cpu_baseline(args.seed, args.cpu_seconds, job)

    forms = None
    if rank == 0 and world == 1 and not args.no_forms:
        forms = forms_of(torch, rs, W, peak, value, W.config2(args.seed),
                         ["config1", "batched", "batched_config2", "batched_config4", "served", "served_stated",
                          "served_stated_low"])
        rates = [float(x) for x in args.serve_rates.split(",") if x] if args.serve_rates else []
        if rates:
            from rssieve_b200 import serve
            forms["served_sweep"] = [measure_served(rs, W, serve, peak, rate=r) for r in rates]

    # work per prime against the reference's parameter rule on the same primes: its Q
    # baby steps per searched prime, and per surviving target its M giant steps when b
    # is a quadratic residue mod p and MM when not (the parity split; each for about
    # half the primes), with the targets that survive here (the reference's filters,
    # which the character test here contains, keep at least as many)
    rp = reference_params(job["nmin"], job["nmax"])
    searched = tot["full"] + tot["parity"]
    work_ours = tot["baby"] + tot["giant"]
    work_ref = rp["Q"] * searched + tot["targets"] * 0.5 * (rp["M"] + rp["MM"])
    rp["work_per_prime_est"] = work_ref / max(tot["primes"], 1)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "primes/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
            "config": {"workload": workload, "p_window_log2": args.width, "seed": args.seed,
                       "baby_steps": baby_q, "baby_steps_tuned": not tuning,
                       "l2": "flushed between steps (256 MiB write outside the step events)",
                       "parallelism": "p-range windows per rank" if world > 1 else "1 GPU"},
            "e2e": e2e,
            "gpu_launches": kernel_launches,
            "roofline": {"bound": ("fp64 pipe (FMA-based modular products, p < 2^51)" if fp_steps
                                   else "int32-imad (64-bit Montgomery products)"),
                         "achieved": achieved, "peak": rpeak, "unit": "Gmulmod/s", "frac": achieved / rpeak,
                         "traffic": BSGS_DRAM_BYTES_PER_PRIME * tot["primes"] / max(bsgs_launches, 1),
                         "traffic_unit": "bytes per BSGS launch (ncu per-prime DRAM bytes x primes per launch)",
                         "work_unit": "baby + giant steps of the BSGS kernel (each one modular product or "
                                      "doublings, plus one table insert or probe)",
                         "peak_source": ("measured live: rs_fpmul_peak, independent chains of the steps' FP64 product"
                                         if fp_steps else
                                         "measured live: rs_mulmod_peak, independent Montgomery-product chains"),
                         "peak_fp64_products": fpeak,
                         "peak_montgomery_products": peak,
                         "frac_of_montgomery_peak": achieved / peak,
                         "peak_multiplier": peak_mult,
                         "frac_of_multiplier_peak": achieved / peak_mult,
                         "peak_multiplier_source": "measured live: rs_widemul_peak (independent mad.wide.u32 "
                                                   "chains) / 11 wide products per Montgomery product",
                         "r_wide_per_sm_clock": (wide * 1e9 / (sms * clocks["sm_mhz"] * 1e6)) if clocks else None,
                         "giant_only_frac": (tot["giant"] / max(bsgs_launches, 1)) / (bsgs_ms_avg / 1e3) / 1e9 / rpeak},
            "cpu_baseline": cpu,
            "forms": forms,
            "clocks": clocks,
            "detail": {"primes": tot["primes"], "giant_steps": tot["giant"], "baby_steps": tot["baby"],
                       "targets_per_prime": tot["targets"] / max(tot["full"] + tot["parity"], 1),
                       "giant_per_prime": tot["giant"] / max(tot["primes"], 1),
                       "skipped": tot["skipped"], "factors": int(len(fac)), "dups": tot["dups"],
                       "candidates": tot["candidates"], "bsgs_ms_avg": bsgs_ms_avg,
                       "bsgs_share": bsgs_ms / max(dev_ms, 1e-9), "wall_s": wall,
                       "mont_products_per_s": giant_all / (dev_ms_max / 1e3),
                       "work_per_prime": work_ours / max(tot["primes"], 1), "reference_rule": rp,
                       "work_ref_over_ours": work_ref / max(work_ours, 1)},
        }
        print(json.dumps(line), flush=True)
    sv.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
