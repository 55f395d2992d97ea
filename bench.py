"""Benchmark of the batched Kadanoff-Baym time stepping (libcntr dyson_timestep hot path) on B200.

Default workload: config 4, the self-consistent 32 x 32 square lattice (size1 = 1, nt = 2000,
ntau = 800, 3 predictor-corrector iterations per step), the configuration the metric's
mixed-versus-FP64 target is stated on.  One bench step = the whole time-stepping phase n = k+1..nt
of every k-point (the metric counts k-point time steps; Matsubara and bootstrap are set-up,
outside the timed region).  After the warm-up, one eager propagation gives the per-kernel device
times (and the roofline of the dominant kernel); the propagation is then recorded as one CUDA
graph and every timed step replays it (--no-graph: eager launches).  Inputs are resident in HBM
for `value`; `e2e` repeats the step through the public API with host buffers (Sigma, H and
bootstrap uploaded, the result downloaded every step).  The FP64 line also carries `mixed`: the
mixed-precision path on the same inputs, its throughput, its ratio to FP64 and its max relative
error per component against the FP64 result (--no-mixed skips it).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload config4|config4-small|config4-ncu|config1|config1-small|config1-ncu|
                                config2|config3|config3-small]
                    [--precision fp64|mixed] [--mixed-error] [--no-cpu] [--no-e2e] [--no-graph]

Under torchrun each rank advances its own k-grid (shifted by rank/N of a grid spacing): the
k-points of the chain workloads are independent, so ranks share no data ("scaling": "weak").
The lattice workloads (config4*) form ONE lattice from all ranks' grids: after every k-average
the ranks sum the weighted G_loc time-step slice with an NCCL all-reduce (nessi_b200.lattice),
and those steps launch eagerly.  `--impl reference` times the CPU restatement of libcntr's
serial path (oracle/, OpenMP over k-points) on a bounded sample of the same workload.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "k-point timesteps/s (batched Dyson), mixed vs FP64 on B200 at <=1e-8 rel err"
UNIT = "k-point time steps/s"


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


def fp64_peak_tflops(n=8192, reps=8):
    """FP64 tensor-core throughput measured in this run: a cuBLAS DGEMM (torch.matmul on float64
    tensors) of n x n x n, timed with CUDA events after a warm-up.  Only the roofline denominator
    of the FP64 contractions; nothing on the product path uses cuBLAS."""
    import torch
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    c = a @ b
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        c = a @ b
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (ms / 1000.0) / 1e12


# ------------------------------------------------------------------------------------------
# clocks during the timed region
# ------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = os.path.join("/tmp", "nessi_clocks_%d_%d.csv" % (os.getpid(), device_index))

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        load = [x for x in sm if smax and x > 0.3 * smax] or sm
        med = float(np.median(load)) if load else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------------------
# CPU baseline: the oracle (CPU restatement of libcntr's serial dyson_timestep), OpenMP over k
# ------------------------------------------------------------------------------------------
def cpu_sample(W, target_s=15.0, max_threads=None):
    """Time windows of consecutive time steps at several n for P problems in parallel, fit
    t(n) = a + b N + c N^2 (N = n+1) per step and integrate over n = k+1..nt.
    Returns (kpt_steps_per_s, threads, description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    import psutil
    from nessi_b200 import herm_matrix
    d0 = W.descs[0]
    nt, ntau, s, k = d0["nt"], d0["ntau"], d0["size1"], W.k
    threads = max_threads or os.cpu_count() or 1
    gbytes = 16.0 * s * s * ((nt + 1) * (nt + 2) + (nt + 1) * (ntau + 1)) / 1e9
    avail = psutil.virtual_memory().available / 1e9
    P = int(max(1, min(threads, W.nprob, (0.25 * avail) // max(gbytes, 1e-9))))
    Gs = []
    for p in range(P):
        G = herm_matrix(nt, ntau, s, d0["sig"])
        B = W.boot[p]
        G.mat[...] = B.mat
        for t in range(k + 1):
            G.set_timestep_data(t, B.get_timestep(t))
        Gs.append(G)
    Hs = np.ascontiguousarray(W.H[:P])
    beta, h, mu = d0["beta"], d0["h"], d0["mu"]
    if W.lattice:
        # a lattice step needs all of its k-points together: the sample lattice is the first P
        # k-points (same cost per k-point step; G_loc is their average)
        Gloc = herm_matrix(nt, ntau, s, d0["sig"])
        Sig = herm_matrix(nt, ntau, s, d0["sig"])
        Um = np.zeros((nt + 2, s, s), np.complex128)
        for i in range(s):
            Um[:, i, i] = W.U[:, i]

        def steps(a, b_):
            for n in range(a, b_ + 1):
                O.lattice2b_timestep(n, Gs, Gloc, Sig, Um, mu, Hs, beta, h, k, ncorr=W.ncorr, nthreads=threads)
    else:
        def steps(a, b_):
            O.dyson_timestep_batch(a, b_, Gs, mu, Hs, W.sigma, beta, h, k, threads)
    # probe one step at the largest n to size the windows
    t0 = time.perf_counter()
    steps(nt, nt)
    t1 = time.perf_counter() - t0
    pts = sorted(set([max(k + 1, int(nt * f)) for f in (0.1, 0.3, 0.6, 1.0)]))
    win = int(max(1, min(40, target_s / (len(pts) * max(t1, 1e-6)))))
    ns, ts = [], []
    for n in pts:
        a = max(k + 1, n - win + 1)
        t0 = time.perf_counter()
        steps(a, n)
        dt = (time.perf_counter() - t0) / (n - a + 1)
        ns.append(0.5 * (a + n) + 1)
        ts.append(dt)
    N = np.array(ns)
    A = np.stack([np.ones_like(N), N, N * N], 1)
    coef, *_ = np.linalg.lstsq(A, np.array(ts), rcond=None)
    allN = np.arange(k + 2, nt + 2, dtype=float)
    total = float(np.sum(coef[0] + coef[1] * allN + coef[2] * allN * allN))
    value = P * (nt - k) / total
    resid = float(np.max(np.abs(A @ coef - np.array(ts)) / np.array(ts)))
    desc = ("%d problems in parallel on %d threads, windows of %d steps at n=%s, fit t(n)=a+bN+cN^2 "
            "integrated over n=%d..%d (max fit residual %.1f%%)" % (P, threads, win, pts, k + 1, nt, 100 * resid))
    if W.lattice:
        desc += "; lattice steps with %d correctors, G_loc over the %d sampled k-points" % (W.ncorr, P)
    return value, threads, desc


# ------------------------------------------------------------------------------------------
def step_bytes(W, mixed):
    """Algorithmic HBM bytes of one propagation (time steps k+1..nt of every problem), by the
    per-problem-step formula of the history convolutions: with N = n+1, M = ntau+1,
      b s^2 (N M) [G^tv history] + 16 s^2 (2N + M) [G slice] + 16 s^2 (N M + N(N+1) + M) [Sigma^tv
      history, Sigma^R / Sigma^< triangles, G^mat], the Sigma part once per group and step,
    b = 16 (FP64) or 8 (FP32 history); a lattice step repeats the Dyson step once per corrector."""
    ncorr = getattr(W, "ncorr", None) or 1
    groups = {}
    for d in W.descs:
        groups.setdefault(d.get("sigma_group", 0), []).append(d)
    total = 0.0
    for members in groups.values():
        s2 = members[0]["size1"] ** 2
        M = members[0]["ntau"] + 1
        nts = np.array(sorted(d["nt"] for d in members))
        n = np.arange(W.k + 1, int(nts.max()) + 1, dtype=np.float64)
        N = n + 1
        active = len(nts) - np.searchsorted(nts, n, side="left")  # members with nt >= n
        b = 8.0 if mixed else 16.0
        per_problem = b * s2 * N * M + 16.0 * s2 * (2 * N + M)
        shared = 16.0 * s2 * (N * M + N * (N + 1) + M)
        total += float(np.sum(active * per_problem + (active > 0) * shared))
    return ncorr * total


def build_workload(name, rank, world):
    from nessi_b200 import workloads
    shift = 0.0 if world == 1 else (2 * math.pi / 256) * rank / world
    if name == "config0":  # one impurity problem (the CPU-sized case)
        return workloads.config0()
    if name == "config1":
        return workloads.config1(kshift=shift)
    if name == "config1-small":
        return workloads.config1(nk=64, nt=200, ntau=100, kshift=shift)
    if name == "config1-ncu":  # config-1 chain at nt=ntau=300: 1.5 GB of G^tv history, > L2
        return workloads.config1(nk=256, nt=300, ntau=300, kshift=shift)
    if name == "config2":  # one 32-k-point chunk of the 512-k 4-band chain (chunks are independent)
        return workloads.config2(chunk=32, chunk_index=rank % 16)
    if name == "config3":  # 96 uneven problems; ranks draw their own problems (seed + rank)
        return workloads.config3(seed=20261203 + rank)
    if name == "config3-small":
        return workloads.uneven(nprob=24, nt_range=(100, 400), ntau=100, seed=20261203 + rank)
    if name == "config4":
        return workloads.config4(kshift=shift)
    if name == "config4-small":  # 16x16 lattice, nt=400, ntau=200: quick checks of the lattice path
        return workloads.config4(nkx=16, nky=16, nt=400, ntau=200, kshift=shift)
    if name == "config4-ncu":  # 32x32 lattice (the config-4 grid), nt=400, ntau=200: ~4 GB, for ncu
        return workloads.config4(nkx=32, nky=32, nt=400, ntau=200, kshift=shift)
    raise SystemExit("unknown workload %s" % name)


def _result_sample(b, W, nt):
    """What the comparison looks at: G_loc of a lattice, else every component of up to 8
    problems (all time steps)."""
    from nessi_b200 import herm_matrix
    out = []
    if W.lattice:
        d = W.descs[0]
        L = herm_matrix(d["nt"], d["ntau"], d["size1"], d["sig"])
        b.get_gloc(0, L)
        out.append(L)
    else:
        for p in range(min(8, len(W.descs))):
            d = W.descs[p]
            G = herm_matrix(d["nt"], d["ntau"], d["size1"], d["sig"])
            b.get_G(p, G)
            out.append(G)
    return out


def compare_with_fp64(b, W, run_step, nt, k):
    """Max relative error max|x - x64| / max|x64| per component of the mixed result against the
    FP64 GPU path (itself parity-tested against the oracle at 1e-10) on the same inputs."""
    from nessi_b200 import gpu, workloads
    run_step()
    b.synchronize()
    mixed = _result_sample(b, W, nt)
    b.close()
    b64 = gpu.Batch(W.descs, precision=gpu.PREC_FP64)
    workloads.upload(b64, W)
    if W.lattice:
        b64.lattice_2b_start(max_iter=30, tol=1e-12)
        for n in range(k + 1, nt + 1):
            b64.lattice_2b_timestep(n, W.ncorr)
    else:
        for n in range(k + 1, nt + 1):
            b64.dyson_timestep(n)
    b64.synchronize()
    ref = _result_sample(b64, W, nt)
    b64.close()
    err = _max_rel(mixed, ref)
    err["compared"] = "G_loc, all time steps" if W.lattice else "all components of %d problems" % len(ref)
    return err


def _max_rel(xs, ys):
    err = {}
    for comp in ("ret", "les", "tv"):
        num = max(float(np.max(np.abs(getattr(x, comp) - getattr(y, comp)))) for x, y in zip(xs, ys))
        den = max(float(np.max(np.abs(getattr(y, comp)))) for y in ys)
        err[comp] = num / den if den else 0.0
    return err


def mixed_companion(b, W, nt, k, fp64_value, args, world, stream):
    """The mixed-precision path on the same inputs, after the FP64 measurement: its throughput
    (same step definition and timing as the FP64 line: a CUDA graph of the propagation replayed
    `--steps` times after an eager warm-up propagation) and the max relative error of its result
    against the FP64 result per component (G_loc of a lattice, else every component of up to 8
    problems).  The FP64 batch is released first."""
    import torch
    from nessi_b200 import gpu, workloads
    ref = _result_sample(b, W, nt)
    b.close()
    bm = gpu.Batch(W.descs, precision=gpu.PREC_MIXED)
    try:
        workloads.upload(bm, W)
        bm.set_stream(stream.cuda_stream)
        if W.lattice:
            bm.lattice_2b_start(max_iter=30, tol=1e-12)

        def prop():
            for n in range(k + 1, nt + 1):
                if W.lattice:
                    bm.lattice_2b_timestep(n, W.ncorr)
                else:
                    bm.dyson_timestep(n)
        prop()  # eager: the Volterra autotuner decides here
        bm.synchronize()
        bm.set_profiling(True)
        prop()
        bm.synchronize()
        prof = bm.read_profile()
        bm.set_profiling(False)
        bm.graph_record(bm.GRAPH_LATTICE if W.lattice else bm.GRAPH_DYSON, k + 1, nt, W.ncorr or 3)
        bm.graph_launch()
        bm.synchronize()
        barrier(world)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            bm.graph_launch()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        ms = allmax(e0.elapsed_time(e1), world)
        value = world * W.kpt_steps() * args.steps / (ms / 1000.0)
        err = _max_rel(_result_sample(bm, W, nt), ref)
        groups = sorted(W.sigma.keys()) if isinstance(W.sigma, dict) else [0]
        volterra = {str(gid): bm.volterra_choice(gid) for gid in groups}
    finally:
        bm.close()
    compared = "G_loc, all time steps" if W.lattice else "all components of %d problems, all time steps" % len(ref)
    return {"value": value, "unit": UNIT, "ms_per_step": ms / args.steps, "ratio_to_fp64": value / fp64_value,
            "max_rel_error_vs_fp64": err, "error_compared": compared,
            "kernels": {kname: {"ms": v[0], "launches": v[1]} for kname, v in prof.items()},
            "volterra_kernels": {g: {"ret": v[0], "les": v[1]} for g, v in volterra.items()},
            "dtype": "complex64 G^tv history / complex128 sums, solves and contractions"}


# kernel classes of the profile whose algorithmic count is flops (nessi_gpu_read_profile)
FLOP_KERNELS = ("ret", "les", "gemm")


def kernel_roofline(prof, prof_steps, peak_hbm, hbm_kind, peak_fp64, traffic_ratio):
    """Breakdown per kernel class and the roofline of the dominant one (largest device time):
    HBM bytes against the measured copy peak for the streaming kernels, FP64 flops against the
    FP64 tensor-core peak measured in this run for the contractions (k_zgemm, the Volterra
    recursions)."""
    total = max(1e-9, sum(v[0] for v in prof.values()))
    breakdown = {}
    for name, (ms, launches, work) in prof.items():
        e = {"ms": ms / prof_steps, "launches": launches // prof_steps, "share": ms / total}
        if ms > 0 and work > 0:
            if name in FLOP_KERNELS:
                e["tflops"] = work / (ms / 1000.0) / 1e12
            else:
                e["gbs"] = work / (ms / 1000.0) / 1e9
        breakdown[name] = e
    dom = max(prof, key=lambda x: prof[x][0])
    ms, launches, work = prof[dom]
    avg = ms / launches if launches else None
    if dom in FLOP_KERNELS:
        achieved = (work / launches) / (avg / 1000.0) / 1e12 if launches else 0.0
        roof = {"kernel": dom, "bound": "tensor", "achieved": achieved, "peak": peak_fp64, "unit": "TFLOP/s",
                "frac": achieved / peak_fp64, "peak_source": "measured in-run (cuBLAS DGEMM 8192^3, FP64 tensor cores)",
                "traffic": None, "algorithmic_flops_per_launch": work / launches if launches else None,
                "avg_launch_ms": avg}
    else:
        achieved = (work / launches) / (avg / 1000.0) / 1e9 if launches else 0.0
        roof = {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak_hbm, "unit": "GB/s",
                "frac": achieved / peak_hbm, "peak_source": hbm_kind,
                "traffic": (traffic_ratio * work / launches) if (traffic_ratio and launches and dom == "tv") else None,
                "algorithmic_bytes_per_launch": work / launches if launches else None, "avg_launch_ms": avg}
        if roof["traffic"] is not None:
            roof["traffic_note"] = ("DRAM bytes per algorithmic byte from one ncu capture of k_tv, scaled to this "
                                    "launch's algorithmic bytes")
    return breakdown, roof


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allmax(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args, rank, world):
    """The reference arm: the oracle (CPU restatement of libcntr's serial dyson_timestep and of
    the lattice driver) with OpenMP over k-points on the host cores.  Each step is a bounded
    sample of the workload (windows of time steps at several n); `value` is the throughput of the
    whole propagation integrated from the sample's fit, `ms_per_step` the sample's wall time."""
    if rank != 0:
        return
    W = build_workload(args.workload, 0, 1)
    vals, walls = [], []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        v, thr, desc = cpu_sample(W, target_s=args.cpu_seconds)
        if i >= args.warmup:
            vals.append(v)
            walls.append(time.perf_counter() - t0)
    value = float(np.median(vals))
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * float(np.mean(walls)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "complex128", "data": "synthetic",
            "impl": "reference",
            "config": dict(workload=args.workload, **W.info),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": thr, "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "ms_per_step_note": "wall time of one bounded sample (a step); the whole propagation would take "
                                "%.0f s at the fitted rate" % (W.kpt_steps() / value),
            "note": "libcntr needs Eigen3, absent here: the timed CPU path is the oracle's C++ restatement "
                    "of libcntr's serial dyson_timestep (and lattice driver) with OpenMP over k-points"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="config4")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--mixed-error", action="store_true",
                    help="with --precision mixed: afterwards run the FP64 path on the same inputs and report the "
                         "max relative error of the mixed result per component")
    ap.add_argument("--no-mixed", action="store_true", help="do not add the mixed-precision companion "
                    "measurement to the FP64 line")
    ap.add_argument("--no-graph", action="store_true", help="launch every step eagerly instead of replaying "
                    "a CUDA graph of the propagation")
    args = ap.parse_args()
    rank, world, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    from nessi_b200 import gpu, workloads
    torch.cuda.set_device(local)
    gpu.init(local)
    W = build_workload(args.workload, rank, world)
    prec = gpu.PREC_MIXED if args.precision == "mixed" else gpu.PREC_FP64
    b = gpu.Batch(W.descs, precision=prec)
    workloads.upload(b, W)
    stream = torch.cuda.Stream()
    b.set_stream(stream.cuda_stream)
    k = W.k
    nt = max(d["nt"] for d in W.descs)

    sharded = None
    if W.lattice and world > 1:
        # one lattice over the k-points of all ranks (each rank's grid is shifted, so together they
        # form a finer one): after every k-average the ranks sum the weighted G_loc slice with one
        # NCCL all-reduce; the steps launch eagerly (no graph around the collectives)
        from nessi_b200.lattice import ShardedLattice
        sharded = ShardedLattice(b, stream=stream)

    def lattice_start():
        if sharded is not None:
            return sharded.start(max_iter=30, tol=1e-12)
        return b.lattice_2b_start(max_iter=30, tol=1e-12)

    if W.lattice:
        # set-up (untimed): self-consistent bootstrap of steps 0..k
        boot_iters, boot_err = lattice_start()

    def propagate():
        if W.lattice:
            for n in range(k + 1, nt + 1):
                if sharded is not None:
                    sharded.timestep(n, W.ncorr)
                else:
                    b.lattice_2b_timestep(n, W.ncorr)
        else:
            for n in range(k + 1, nt + 1):
                b.dyson_timestep(n)

    for _ in range(args.warmup):
        propagate()
    b.synchronize()
    use_graph = not args.no_graph and sharded is None
    if use_graph:
        # per-kernel device times from one eager propagation (untimed); then the propagation is
        # recorded once as a CUDA graph and every timed step replays it
        b.set_profiling(True)
        propagate()
        b.synchronize()
        prof = b.read_profile()
        b.set_profiling(False)
        b.graph_record(b.GRAPH_LATTICE if W.lattice else b.GRAPH_DYSON, k + 1, nt, W.ncorr or 3)
        run_step = b.graph_launch
        run_step()  # first replay outside the timed region
        b.synchronize()
    else:
        b.set_profiling(True)
        run_step = propagate
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        run_step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms = allmax(e0.elapsed_time(e1), world)
    if not use_graph:
        prof = b.read_profile()
        b.set_profiling(False)
    prof_steps = 1 if use_graph else args.steps
    units = world * W.kpt_steps() * args.steps
    value = units / (ms / 1000.0)

    # per-kernel device times and the roofline of the dominant kernel class
    peak, peak_kind = load_peaks()
    peak_fp64 = fp64_peak_tflops()
    traffic_ratio = None
    tpath = os.path.join(ROOT, "profiles", "k_tv_config1-ncu.md")
    if os.path.exists(tpath):
        for line in open(tpath):
            if line.startswith("traffic_ratio:"):
                traffic_ratio = float(line.split(":")[1])
    breakdown, roofline = kernel_roofline(prof, prof_steps, peak, peak_kind, peak_fp64, traffic_ratio)
    # the whole step against the HBM peak: all algorithmic bytes of the propagation over its
    # time; low where the sequential Volterra recursions set the pace
    try:
        sb = step_bytes(W, args.precision == "mixed")
        ach = sb * args.steps / (ms / 1000.0) / 1e9
        step_roofline = {"achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "peak_source": peak_kind,
                         "bytes_per_step": sb,
                         "definition": "sum over problem-steps of the history-convolution bytes (G^tv, Sigma^tv "
                                       "histories, Sigma triangles, G slices) / device time of the timed steps"}
    except Exception as exc:  # the line stands without it
        step_roofline = {"error": "%s: %s" % (type(exc).__name__, exc)}

    # end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        from nessi_b200 import herm_matrix
        # the uneven batch holds ~135 GB of G: its result is the last time step of every problem
        last_only = W.name == "uneven"
        host = []
        for d in (W.descs[:1] if (W.lattice or last_only) else W.descs):
            host.append(herm_matrix(d["nt"], d["ntau"], d["size1"], d["sig"]))
        try:
            import torch as _t
            pinned = True
            for G in host:
                for nm in ("ret", "les", "tv", "mat"):
                    a = getattr(G, nm)
                    t = _t.empty(a.size * 2, dtype=_t.float64, pin_memory=True)
                    setattr(G, nm, t.numpy().view(np.complex128).reshape(a.shape))
        except Exception:
            pinned = False
        sig_bytes = sum(getattr(W.sigma, x).nbytes for x in ("ret", "les", "tv", "mat"))
        h2d = sig_bytes + W.H.nbytes + sum(B.mat.nbytes + sum(B.get_timestep(t).nbytes for t in range(k + 1))
                                           for B in W.boot)
        if W.lattice:
            h2d += W.U.nbytes
            # result of a lattice run: G_loc (all components) and the last time step of every G_k
            d0 = W.descs[0]
            gloc_host = host[0]
            last = np.zeros((len(W.descs), 2 * (nt + 1) + d0["ntau"] + 1, d0["size1"], d0["size1"]), np.complex128)
            d2h = sum(getattr(gloc_host, x).nbytes for x in ("ret", "les", "tv", "mat")) + last.nbytes
        elif last_only:
            lasts = [np.zeros((2 * (d["nt"] + 1) + d["ntau"] + 1, d["size1"], d["size1"]), np.complex128)
                     for d in W.descs]
            d2h = sum(a.nbytes for a in lasts)
        else:
            d2h = sum(G.ret.nbytes + G.les.nbytes + G.tv.nbytes + G.mat.nbytes for G in host)
        barrier(world)
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2e_steps = min(args.steps, 3)
        f0.record(stream)
        for _ in range(e2e_steps):
            workloads.upload(b, W)
            if W.lattice:
                lattice_start()
            run_step()
            if W.lattice:
                b.get_gloc(0, gloc_host)
                for p in range(len(W.descs)):
                    b.get_timestep(p, nt, last[p])
            elif last_only:
                for p, d in enumerate(W.descs):
                    b.get_timestep(p, d["nt"], lasts[p])
            else:
                for p, G in enumerate(host):
                    b.get_G(p, G)
        f1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        ems = allmax(f0.elapsed_time(f1), world)
        e2e = {"value": world * W.kpt_steps() * e2e_steps / (ems / 1000.0), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "pinned_host": pinned,
               "ms_per_step": ems / e2e_steps, "steps": e2e_steps}
        if W.lattice:
            e2e["includes"] = "upload, self-consistent bootstrap, propagation, download of G_loc and G_k(nt)"
        elif last_only:
            e2e["includes"] = "upload of Sigma, H and bootstrap steps, propagation, download of each G_p(nt_p)"
        # sanity: the downloaded result is finite
        if not last_only and not all(np.isfinite(G.tv[nt]).all() for G in host[:4]):
            e2e["warning"] = "non-finite values in the result"

    cpu = None
    if isinstance(W.sigma, dict):
        cpu = {"value": None, "note": "not sampled for the multi-size batch; see the config-1 and config-4 lines"}
    elif rank == 0 and world == 1 and not args.no_cpu:
        v, thr, desc = cpu_sample(W, target_s=args.cpu_seconds)
        cpu = {"value": v, "unit": UNIT, "cores": thr, "kind": "port", "sample": desc}

    groups = sorted(W.sigma.keys()) if isinstance(W.sigma, dict) else [0]
    volterra = {str(gid): b.volterra_choice(gid) for gid in groups}
    # own kernels launched per timed step, from the launch structure of one Dyson step per group:
    # k_prep_problem, k_prep_group, k_mat_operator, k_zgemm (Matsubara part), ret, k_les_operands_t,
    # k_zgemm (les*adv), k_tv, k_les_operands_t, k_zgemm (tv*vt), les; ret / les are two kernels
    # (k_*_start + k_volterra_cl) on the cluster path and one otherwise.  A lattice step adds
    # k_extrapolate, per corrector k_gloc + k_gloc_final + k_sigma_2b, and the final k-average.
    per_group = [10 + (2 if v[0] == 100 else 1) + (2 if v[1] == 100 else 1) for v in volterra.values()]
    if W.lattice:
        gpu_launches = (nt - k) * (1 + W.ncorr * (3 + sum(per_group)) + 2) * args.steps
    else:
        nts = {}
        for d in W.descs:
            nts.setdefault(d.get("sigma_group", 0), []).append(d["nt"])
        gpu_launches = sum((max(nts[int(g)]) - k) * c for g, c in zip(volterra.keys(), per_group)) * args.steps
    mixed_err = None
    if args.mixed_error and args.precision == "mixed":
        mixed_err = compare_with_fp64(b, W, run_step, nt, k)
    # the metric compares mixed with FP64: the default (FP64) line of the chain workloads also
    # carries the mixed path measured on the same inputs
    mixed_line = None
    closed = False
    if args.precision == "fp64" and sharded is None and not args.no_mixed:
        try:
            mixed_line = mixed_companion(b, W, nt, k, value, args, world, stream)
        except Exception as exc:  # the FP64 line stands on its own
            mixed_line = {"error": "%s: %s" % (type(exc).__name__, exc)}
        closed = True

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "complex128" if args.precision == "fp64" else "complex64 history / complex128 solves",
                "data": "synthetic",
                "config": dict(workload=args.workload, precision=args.precision,
                               l2="inputs larger than L2 (G^tv history %.1f GB per GPU)" % (
                                   sum(16.0 * (d["nt"] + 1) * (d["ntau"] + 1) * d["size1"] ** 2 for d in W.descs) / 1e9),
                               bootstrap=("free propagator of H_k(-1) for mat, then %d self-consistent "
                                          "dyson_start iterations (set-up, untimed)" % boot_iters) if W.lattice else
                               "free propagator of H_k(-1) for mat and steps 0..k (set-up, untimed)",
                               **W.info),
                "roofline": roofline, "step_roofline": step_roofline, "kernels": breakdown,
                "fp64_peak_tflops_in_run": peak_fp64, "cpu_baseline": cpu,
                "e2e": e2e,
                "gpu_launches": gpu_launches, "clocks": clk,
                "launch": "CUDA graph of the whole propagation, replayed each step" if use_graph else "eager",
                "volterra_kernels": {g: {"ret": v[0], "les": v[1]} for g, v in volterra.items()}}
        if sharded is not None:
            line["lattice_exchange"] = {
                "collective": "NCCL all-reduce of the weighted G_loc time-step slice after every k-average",
                "k_points_total": sharded.nk_total[0], "k_points_this_rank": len(W.descs),
                "bytes_per_all_reduce_at_nt": sharded.exchange_bytes(nt),
                "all_reduces_per_time_step": W.ncorr + 1}
        if mixed_err is not None:
            line["mixed_error_vs_fp64_gpu"] = mixed_err
        if mixed_line is not None:
            line["mixed"] = mixed_line
        print(json.dumps(line), flush=True)
    if not closed and not (args.mixed_error and args.precision == "mixed"):
        b.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
