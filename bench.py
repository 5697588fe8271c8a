"""Benchmark: fused energy + pose-gradient pair-terms/s on the 65536 x 65536 workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload 2]

One step = one energy + pose-gradient evaluation of the REF model (compi.cu:753-772
restated) over all N x M source/target pairs at one pose: the per-pose prologue, the
fused adjoint kernel and the FP64 reduction.  A pair-term is one (i, j) pair at one
pose.  Inputs are seeded synthetic clouds of the named workload (no dataset).

value       whole-job pair-terms/s with the clouds resident on the device (CUDA events
            around each step on the launching stream; the L2 is flushed between steps
            by writing 256 MiB on that stream before each step's start event).
e2e         the same metric through the C ABI with host buffers: dugma_init (FP64 clouds
            and covariances copied in from pinned host memory), dugma_energy_grad (E and g
            copied out) and dugma_fr_m per step, wall clock (max over ranks); the host thread
            and the pinned inputs on the CPUs NVML reports local to the GPU.
roofline    the adjoint kernel's FP32-pipe instruction rate (algorithmic instructions per
            pair x pairs per launch / launch time from CUDA events inside the library)
            against the FP32 fused-multiply-add rate measured in this run.
plain_fd    the plain form: energy + central finite differences (13 energy evaluations, 7 in 2D).
cpu_baseline  the FP64 C/OpenMP oracle on a bounded sample of source rows, all host cores.
accuracy    this run's relative error against that FP64 oracle on the same sampled rows
            (energy and the pose gradient of source rows [0, rows) over all targets).
configs     (default run, one GPU) compact results of the other configured workloads, each
            with its own device timing, roofline fraction, error against the FP64 oracle and
            clock record: the 1K and 6K spheres, the batch of 256 problems x 32 rotations, the
            300K depth views with 64 poses and the k = 8 neighbour pass, the 2D curve, the CONV
            model, update_sig / compi through the plugin interface at 64K, and the end-to-end
            registration of the reference's 30 real Kinect scenes (both modes).

Workloads (--workload): 0 1K sphere, 1 6K sphere with outliers, 2 the 64K harmonic surface
(default), 3 256 problems x 32 poses in one persistent launch, 4 300K depth views, 5 the 2D
path on two 64K samples of a closed curve.

With --poses P a step evaluates P multistart poses of the problem back to back (one
launch sequence per pose); the depth-camera workload is quoted with P = 64.  The
nearest-distance pass that sets sigma (update_sig) is timed separately (details).

Multi-GPU: each rank evaluates its own multistart poses of the same problem (independent
units, no collective on the data path): weak scaling, value = sum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# algorithmic per-pair operation counts of the REF kernels, 3D (see the kernel sources)
# REF adjoint: d 6, u = kC'd 9, d.u 3, B exponent (z = U d 6, |z|^2 3) 9, energy 2, S1 += e1 u 3,
# w = e2 z 3, D2 += w 3, Q2 += w z^T 6
FP32_INSTR_ADJOINT = 44
# REF adjoint in 2D: d 4, u 4, d.u 2, B exponent (z = U d 3, |z|^2 2) 5, energy 2, S1 2, w 2, D2 2, Q2 3
FP32_INSTR_ADJOINT_2D = 26
# CONV adjoint: d 6, S = Sx + C'y 6, adjugate 12, det 3, singularity test 3, h = adj d 9, d.h 3,
# exponent and normalisation 5, energy 1, nr and nr2 2, U 3 + w 3, UU 6, A 6; SFU: rsqrt + ex2
FP32_INSTR_CONV_ADJOINT = 68
FP32_INSTR_ENERGY = 26      # d 6, two Horner quadratic forms 9 + 9, accumulation 2
# compi in one pass: d 6, two quadratic forms 9 + 9 (Cholesky form z = U d 6 and |z|^2 3 each, or
# Horner), p = e1 + e2 1, source-side H2 += p g 10,
# target-side T += fw p 10
FP32_INSTR_COMPI = 45
SFU_PER_PAIR = 2            # two ex2


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1, help="ranks (one per GPU; launched by torchrun for N > 1)")
    ap.add_argument("--steps", type=int, default=50, help="timed steps")
    ap.add_argument("--warmup", type=int, default=3, help="untimed warm-up steps (at least 3 are run)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-gpu"],
                    help="ours: this library; reference: the path's CPU implementation (FP64 oracle port); "
                         "reference-gpu: the reference's own CUDA plugins built from its sources")
    ap.add_argument("--workload", type=int, default=2,
                    help="0 1K sphere, 1 6K sphere, 2 64K harmonic surface, 3 batched problems, 4 300K depth "
                         "views, 5 2D 64K curve")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end (host buffers) measurement")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline and the accuracy check")
    ap.add_argument("--no-fd", action="store_true", help="skip the plain form (energy + finite differences)")
    ap.add_argument("--no-tune", action="store_true", help="keep the default kernel shape (profiling runs)")
    ap.add_argument("--n", type=int, default=0, help="override the cloud size (small profiling cases)")
    ap.add_argument("--shape", default="", help="pin the adjoint kernel shape ipt,nt,tj,pack (skips tuning)")
    ap.add_argument("--model", type=int, default=0, choices=[0, 1],
                    help="0: the reference's per-pair model (REF), 1: convolved GMM (CONV)")
    ap.add_argument("--poses", type=int, default=1,
                    help="multistart poses evaluated per step and GPU (the depth workload uses 64)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the compact results of the other configured workloads (the `configs` key)")
    ap.add_argument("--plugin", default="", choices=["", "compi", "update_sig", "compi_range", "nn", "knn_covariance"],
                    help="profiling runs: only this call, --warmup + --steps times at the workload's first "
                         "multistart pose (one JSON line with the wall time per call and the library's device "
                         "time of its pair kernels): compi, update_sig, compi_range (the source-side coefficient "
                         "pass alone, as row-range compi runs it), nn (--knn nearest neighbours), knn_covariance "
                         "(the --knn neighbour covariance estimator on the source cloud)")
    ap.add_argument("--knn", type=int, default=8, help="k for --plugin nn and knn_covariance")
    return ap.parse_args()


def dist_setup(n):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != n and world != 1:
        raise SystemExit(f"--gpus {n} but WORLD_SIZE={world}")
    return rank, world, local


def dist_init(world, local):
    """This rank's device (local rank, wrapped over the visible devices) and, for world > 1, the
    process group: NCCL, or the backend named by DUGMA_DIST_BACKEND (gloo runs several ranks'
    host-side plumbing on fewer GPUs; each rank's kernels are independent)."""
    import datetime
    import torch
    dev = local % max(1, torch.cuda.device_count())
    torch.cuda.set_device(dev)
    if world > 1:
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = os.environ.get("DUGMA_DIST_BACKEND", "nccl")
        kw = {"device_id": torch.device("cuda", dev)} if backend == "nccl" else {}
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120), **kw)
    return dev


def all_reduce(values, op):
    """All-reduce a few host floats over the ranks (op "sum" or "max"); identity when alone."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64)
    if dist.get_backend() == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.SUM if op == "sum" else dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def gpu_local_cpus(dev):
    """The host CPUs NVML reports as local to CUDA device `dev` (its NUMA node), within this
    process's allowed set; empty when NVML cannot tell (read-only queries, nothing is changed)."""
    try:
        import pynvml
        import torch
        pynvml.nvmlInit()
        try:
            h = pynvml.nvmlDeviceGetHandleByUUID("GPU-" + str(torch.cuda.get_device_properties(dev).uuid))
            n = os.cpu_count() or 64
            masks = pynvml.nvmlDeviceGetCpuAffinity(h, (n + 63) // 64)
        finally:
            pynvml.nvmlShutdown()
        cpus = {64 * w + b for w, m in enumerate(masks) for b in range(64) if (int(m) >> b) & 1}
        return cpus & os.sched_getaffinity(0)
    except Exception:
        return set()


def workload(wl, n=0):
    from dugma_b200 import synth
    return synth.WORKLOADS[wl](n=n) if n else synth.WORKLOADS[wl]()


def config_for(P, poses=1, model=0):
    """The workload description, shared by both arms."""
    per = "one multistart pose" if poses == 1 else f"{poses} multistart poses"
    name = "REF" if model == 0 else "CONV"
    return {"workload": f"{P.name}: N={P.N}, M={P.M}, {name} model energy + pose gradient, {per} per step and GPU",
            "l2": "flushed between steps (256 MiB write on the launching stream, before the start event)"}


def profiled_traffic(shape_key):
    """DRAM bytes per launch of the adjoint kernel from the committed ncu summary, when this run
    uses the profiled kernel shape (its "shape:" line) on the profiled workload; otherwise None."""
    path = os.path.join(ROOT, "profiles", "adjoint_packed_harmonic64k.txt")
    if not os.path.exists(path):
        return None
    shape, traffic = None, None
    for line in open(path):
        if line.strip().startswith("shape:"):
            shape = tuple(int(v) for v in line.split(":")[1].split(","))
        if "traffic_bytes_per_launch:" in line:
            traffic = float(line.split(":")[1])
    return traffic if shape == tuple(shape_key) else None


def hbm_view(bytes_per_launch, kernel_ms):
    """The same launch against the HBM roofline of MEASURED_PEAKS.json (the algorithmic bytes,
    every record read once): shows how far from memory-bound the kernel is."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        peak = float(json.load(open(path))["hbm_gbs"])
    except Exception:
        return None
    gbs = bytes_per_launch / (kernel_ms * 1e-3) / 1e9
    return {"achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak}


def eval_pose(P, unit):
    """Multistart pose number `unit`: ground truth perturbed by a seeded 10 deg, 2 cm offset."""
    from dugma_b200.pose import expmap, rot2d
    rng = np.random.default_rng(100 + unit)
    D = P.X.shape[1]
    ax = rng.standard_normal(D)
    ax /= np.linalg.norm(ax)
    if D == 2:
        return P.R_G @ rot2d(np.radians(10.0) * np.sign(ax[0])), P.t_G + 0.02 * ax
    R = P.R_G @ expmap(ax * np.radians(10.0))
    t = P.t_G + 0.02 * ax
    return R, t


class Clocks:
    """nvidia-smi samples during the timed region (one reading right after it when the region is
    shorter than the sampler's start-up, marked in the summary)."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, path, index):
        self.path, self.index = path, index
        self.p = None
        self.window = "timed region"

    def _cmd(self):
        return ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits"]

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(self._cmd() + ["-lms", "50"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()
            self.f.close()
            try:
                empty = not open(self.path).read().strip()
                if empty:
                    with open(self.path, "w") as f:
                        subprocess.run(self._cmd(), stdout=f, stderr=subprocess.DEVNULL, timeout=30)
                    self.window = "right after the timed region (shorter than the sampler's start-up)"
            except Exception:
                pass

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and "Active" in r[5 + k] and "Not" not in r[5 + k]:
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows), "window": self.window}


def cpu_rate(P, R, t, sig, model=0, budget_s=8.0):
    """Oracle (FP64, OpenMP, all host threads) pair-terms/s on a bounded sample of source rows
    [0, i0); also returns the oracle's energy and pose gradient summed over those rows."""
    from oracle import oracle as orc
    orc.use_all_cores()
    st = orc.State(P.X, P.X_C, P.Y, P.Y_C)
    fn = st.energy_conv if model == 1 else st.energy
    rows = 64
    done = 0
    E, g = 0.0, 0.0
    t0 = time.perf_counter()
    i0 = 0
    while time.perf_counter() - t0 < budget_s and i0 < st.N:
        i1 = min(st.N, i0 + rows)
        e, gg, _ = fn(R, t, sig, i0=i0, i1=i1)
        E, g = E + e, g + gg
        done += (i1 - i0) * st.M
        i0 = i1
        rows = min(rows * 2, 4096)
    el = time.perf_counter() - t0
    return done / el, done, el, orc.num_threads(), (i0, E, g)


def run_reference(args, rank, world):
    """Reference arm: the CPU implementation of the path (the FP64 oracle port; the reference has no
    CPU code of its own), all host threads, rank 0 only, a bounded sample of rows per step."""
    if rank != 0:
        return
    from oracle import oracle as orc
    orc.use_all_cores()
    P = workload(args.workload, args.n)
    R, t = eval_pose(P, 0)
    st = orc.State(P.X, P.X_C, P.Y, P.Y_C)
    _, d2 = st.nn(R, t, 1)
    sig = float(np.mean(d2) / 3.0)
    rows = min(2048, st.N)
    fn = st.energy_conv if args.model == 1 else st.energy
    for _ in range(args.warmup):
        fn(R, t, sig, i0=0, i1=rows)
    t0 = time.perf_counter()
    for k in range(args.steps):
        i0 = (k * rows) % (st.N - rows + 1)
        fn(R, t, sig, i0=i0, i1=i0 + rows)
    el = time.perf_counter() - t0
    val = args.steps * rows * st.M / el
    line = {"impl": "reference", "metric": "energy+grad pair-terms/s", "value": val, "unit": "pair-terms/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_for(P, args.poses, args.model),
            "cpu_baseline": {"value": val, "unit": "pair-terms/s", "cores": orc.num_threads(), "kind": "port",
                             "sample": f"{rows} source rows x {st.M} targets per step"},
            "e2e": {"value": val, "unit": "pair-terms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference_gpu(args, rank):
    """The reference's own CUDA plugins (init.cu / update_sig.cu / compi.cu compiled unmodified for
    sm_100a into oracle/_ref) timed on this GPU beside this library's equivalents, on the 1K-sphere
    generator at sizes that are multiples of 32 (the reference compi kernel needs them)."""
    if rank != 0:
        return
    import torch
    from oracle import ref_plugins
    from dugma_b200 import api, synth
    if not ref_plugins.available():
        print(json.dumps({"impl": "reference-gpu", "unavailable": "oracle/_ref was not built"}))
        return
    rows = []
    # compi at 65536 points would take the reference ~30 s a call; 16384 is its largest size here
    for n, names in ((1024, ("update_sig", "compi")), (4096, ("update_sig", "compi")), (16384, ("update_sig", "compi")),
                     (65536, ("update_sig",))):
        P = synth.workload0(n=n)
        R, t = P.R_G, P.t_G
        ptr = ref_plugins.init(P.X, P.X_C, P.Y, P.Y_C)
        _, h = api.init(P.X, P.X_C, P.Y, P.Y_C)
        res = {"N": n, "M": n}
        calls = {"update_sig": (lambda: ref_plugins.update_sig(ptr, R, t, n, n, 3), lambda: api.update_sig(h, R, t)),
                 "compi": (lambda: ref_plugins.compi(ptr, R, t, n, n, 3, 0.01), lambda: api.compi(h, R, t, sig=0.01))}
        for name in names:
            fn_ref, fn_ours = calls[name]
            for tag, fn in (("reference", fn_ref), ("ours", fn_ours)):
                fn()
                torch.cuda.synchronize()
                reps, el = 0, 0.0
                t0 = time.perf_counter()
                while reps < 3 or (time.perf_counter() - t0 < 2.0 and reps < 50):
                    fn()
                    reps += 1
                el = time.perf_counter() - t0
                res[f"{name}_{tag}_ms"] = 1e3 * el / reps
                res[f"{name}_{tag}_pair_terms_per_s"] = n * n * reps / el
            res[f"{name}_speedup"] = res[f"{name}_reference_ms"] / res[f"{name}_ours_ms"]
        rows.append(res)
        api.fr_m(h)
    print(json.dumps({"impl": "reference-gpu", "unit": "pair-terms/s (one pair at one pose per term)",
                      "note": "host-to-host calls of each plugin, wall clock", "results": rows}), flush=True)


def run_batch(args, rank, world):
    """Workload 3: 256 problems (N, M uniform in [500, 8000]) x 32 multistart rotations on a uniform
    SO(3) grid, one persistent launch per evaluation (graph replay after the first), tile shape
    autotuned on these poses; the problems are split across ranks.  value: device time of each
    evaluation (the library's CUDA events, max over ranks); e2e: the synchronous batch call with
    host poses in and E, g out; accuracy: 4 sampled problem-poses against the FP64 oracle (rank 0);
    cpu_baseline: the oracle on one whole problem-pose, all host cores."""
    import torch
    from dugma_b200 import api, synth
    probs = synth.workload3()
    mine = probs[rank::world]
    grid = synth.so3_grid(synth.rng_for(3, 1), 32)
    Q = len(grid)
    sig = np.zeros((len(mine), Q))
    for k, P in enumerate(mine):
        _, h = api.init(P.X, P.X_C, P.Y, P.Y_C)
        sig[k, :] = api.update_sig(h, np.eye(3), P.t_G)
        api.fr_m(h)
    R = np.array([[g @ P.R_G for g in grid] for P in mine])
    t = np.array([[P.t_G for _ in grid] for P in mine])
    b = api.Batch([(P.X, P.X_C, P.Y, P.Y_C) for P in mine])
    pairs = Q * sum(P.N * P.M for P in mine)
    tune = b.autotune(R, t, sig)
    for _ in range(max(3, args.warmup)):
        E, g = b.energy_grad(R, t, sig)
    torch.cuda.synchronize()
    steps = max(3, min(args.steps, 20))
    import tempfile
    b.timing(1)
    with Clocks(os.path.join(tempfile.gettempdir(), f"dugma_clocks_batch_rank{rank}.csv"),
                torch.cuda.current_device()) as clk:
        t0 = time.perf_counter()
        for _ in range(steps):
            E, g = b.energy_grad(R, t, sig)
        el = time.perf_counter() - t0
    dev_ms, n_ev = b.timing(2)
    b.timing(0)
    shape = list(b.get_shape())
    b.close()
    tot = all_reduce([pairs], "sum") + all_reduce([el, dev_ms], "max")
    if rank != 0:
        return
    from oracle import oracle as orc
    orc.use_all_cores()
    peak = ctypes_peak()
    value = float(tot[0]) * steps / (float(tot[2]) * 1e-3)
    e2e = float(tot[0]) * steps / float(tot[1])
    n_pose = len(mine) * Q
    rng = np.random.default_rng(7)
    errs = []
    for p, q in zip(rng.choice(len(mine), 4, replace=False), rng.integers(0, Q, 4)):
        P = mine[p]
        Eo, go, _ = orc.State(P.X, P.X_C, P.Y, P.Y_C).energy(R[p, q], t[p, q], sig[p, q])
        errs.append((abs(E[p, q] - Eo) / abs(Eo), float(np.linalg.norm(g[p, q] - go) / np.linalg.norm(go))))
    P0 = mine[0]
    st0 = orc.State(P0.X, P0.X_C, P0.Y, P0.Y_C)
    c0 = time.perf_counter()
    st0.energy(R[0, 0], t[0, 0], sig[0, 0])
    cpu_s = time.perf_counter() - c0
    ms = float(tot[2]) / steps
    line = {"metric": "energy+grad pair-terms/s", "value": value, "unit": "pair-terms/s", "n_gpus": world,
            "steps": steps, "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "batch256x32: 256 problems, N, M uniform in [500, 8000], 32 rotations of a "
                                   "uniform SO(3) grid each, one evaluation per step",
                       "pair_terms_per_step": int(tot[0]),
                       "timing": "CUDA events around each evaluation on the batch stream, max over ranks",
                       "l2": "the records of all problems (4.5 GB) exceed L2; no flush"},
            "roofline": {"bound": "fp32", "achieved": FP32_INSTR_ADJOINT * float(tot[0]) / (ms * 1e-3) / 1e12,
                         "peak": peak / 1e12, "unit": "Tinstr/s (FP32 pipe, lane ops)",
                         "frac": FP32_INSTR_ADJOINT * float(tot[0]) / (ms * 1e-3) / peak,
                         "traffic": None, "kernel_ms": ms, "instr_per_pair": FP32_INSTR_ADJOINT,
                         "note": "device time of the whole evaluation (records prologue, pair launch, reduction)"},
            "kernel_shape": shape, "autotune": tune,
            # the batch call takes host poses and returns host results: the steps are end to end
            "e2e": {"value": e2e, "unit": "pair-terms/s", "h2d_bytes_per_step": 8 * 13 * n_pose,
                    "d2h_bytes_per_step": 8 * (1 + g.shape[-1]) * n_pose},
            "accuracy": {"pairs_checked": len(errs), "E_rel_err": max(e[0] for e in errs),
                         "grad_rel_err": max(e[1] for e in errs), "tolerance": {"E": 1e-6, "grad": 1e-5},
                         "against": "FP64 oracle, 4 sampled (problem, pose) pairs, all rows"},
            "cpu_baseline": {"value": P0.N * P0.M / cpu_s, "unit": "pair-terms/s", "cores": orc.num_threads(),
                             "kind": "port", "sample": f"problem 0 at its first pose: {P0.N} x {P0.M} pairs "
                                                       f"({cpu_s:.2f} s, FP64 oracle, OpenMP)"},
            "gpu_launches": 3 * steps}
    clocks = clk.summary()
    if clocks:
        line["clocks"] = clocks
    print(json.dumps(line), flush=True)


def ctypes_peak():
    """The FP32 fused-multiply-add lane rate of this GPU, measured now (dugma_calibrate)."""
    import ctypes
    from dugma_b200 import _lib
    peak = ctypes.c_double(0)
    _lib.load().dugma_calibrate(0, ctypes.byref(peak), None)
    return peak.value


# ---------------------------------------------------------------------------
# The other configured workloads, each measured compactly in the default run (`configs`)
# ---------------------------------------------------------------------------
def _oracle_rows(P, budget_pairs=2.7e8):
    """Source rows the FP64 oracle checks: all of them when that is cheap, else a prefix of about
    budget_pairs pairs."""
    return int(min(P.N, max(256, budget_pairs // P.M)))


def _accuracy(h, st, R, t, sig, model, rows):
    from dugma_b200 import api
    Eo, go, _ = (st.energy_conv if model == 1 else st.energy)(R, t, sig, i0=0, i1=rows)
    Eg, gg = api.energy_grad_range(h, R, t, sig, 0, rows, model=model)
    return {"rows": int(rows), "E_rel_err": abs(Eg - Eo) / abs(Eo),
            "grad_rel_err": float(np.linalg.norm(gg - go) / np.linalg.norm(go)),
            "tolerance": {"E": 1e-6, "grad": 1e-5}, "against": "FP64 oracle, same rows"}


def _instr(D, model):
    if model == 1:
        return FP32_INSTR_CONV_ADJOINT
    return FP32_INSTR_ADJOINT if D == 3 else FP32_INSTR_ADJOINT_2D


def config_single(L, name, P, model, peak, steps=20, poses=1, nn_k=0, clock_dir="/tmp"):
    """One problem: pose gradient of `poses` multistart poses per step, device-timed (CUDA events on
    the launching stream, L2 flushed between steps), the adjoint kernel's share from the library's
    events, the error against the FP64 oracle on the oracle's rows, clocks during the timed region."""
    import ctypes
    import torch
    from dugma_b200 import api
    from oracle import oracle as orc
    D = P.X.shape[1]
    R, t = eval_pose(P, 0)
    _, h = api.init(P.X, P.X_C, P.Y, P.Y_C)
    try:
        ent = {"workload": f"{P.name}: N={P.N}, M={P.M}, {'CONV' if model == 1 else 'REF'} model, "
                           f"{poses} pose(s) per step"}
        torch.cuda.synchronize()
        a0 = time.perf_counter()
        sig = api.update_sig(h, R, t)
        ent["update_sig_ms"] = 1e3 * (time.perf_counter() - a0)
        if nn_k:
            # the brute-force k-nearest-neighbour pass on the clouds (device time of its kernels)
            api.nn(h, R, t, nn_k)
            L.dugma_timing(h.arr, 1, None, None)
            api.nn(h, R, t, nn_k)
            kms, kl = ctypes.c_double(0), ctypes.c_int(0)
            L.dugma_timing(h.arr, 2, ctypes.byref(kms), ctypes.byref(kl))
            L.dugma_timing(h.arr, 0, None, None)
            ent["nn"] = {"k": nn_k, "kernel_ms": kms.value, "pairs_per_s": P.N * P.M / (kms.value * 1e-3)}
        ent["autotune"] = api.autotune(h, 0 if model == 0 else 3)
        stream = torch.cuda.Stream()
        pose = torch.zeros(poses, 16, dtype=torch.float64, device="cuda")
        for k in range(poses):
            Rk, tk = eval_pose(P, k)
            pose[k, :D * D] = torch.tensor(np.asarray(Rk).T.reshape(-1))
            pose[k, 9:9 + D] = torch.tensor(tk)
            pose[k, 12] = sig
        out = torch.zeros(poses, 8, dtype=torch.float64, device="cuda")
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

        def step(npose=poses):
            for k in range(npose):
                rc = L.dugma_energy_grad_async(h.arr, pose[k].data_ptr(), model, out[k].data_ptr(), None,
                                               stream.cuda_stream)
                if rc != 0:
                    raise RuntimeError(L.dugma_last_error().decode())

        with torch.cuda.stream(stream):
            for _ in range(3):
                step(1)
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        L.dugma_timing(h.arr, 1, None, None)
        with Clocks(os.path.join(clock_dir, f"dugma_clocks_{name}.csv"), torch.cuda.current_device()) as clk:
            for k in range(steps):
                with torch.cuda.stream(stream):   # the flush ends before the step's start event
                    flush.fill_(float(k))
                ev[k][0].record(stream)
                step()
                ev[k][1].record(stream)
            torch.cuda.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in ev) / steps
        kms, kl = ctypes.c_double(0), ctypes.c_int(0)
        L.dugma_timing(h.arr, 2, ctypes.byref(kms), ctypes.byref(kl))
        L.dugma_timing(h.arr, 0, None, None)
        kernel_ms = kms.value / max(kl.value, 1)
        pairs = P.N * P.M
        instr = _instr(D, model)
        ent.update({"steps": steps, "warmup": 3, "ms_per_step": ms, "pair_terms_per_s": pairs * poses / (ms * 1e-3),
                    "evals_per_s": poses / (ms * 1e-3),
                    "roofline": {"bound": "fp32", "instr_per_pair": instr, "kernel_ms": kernel_ms,
                                 "achieved": instr * pairs / (kernel_ms * 1e-3) / 1e12, "unit": "Tinstr/s",
                                 "frac": instr * pairs / (kernel_ms * 1e-3) / peak},
                    "kernel_shape": list(api.get_shape(h, 0 if model == 0 else 3)),
                    "l2": "flushed between steps (256 MiB write on the launching stream, before the start event)"})
        st = orc.State(P.X, P.X_C, P.Y, P.Y_C)
        ent["accuracy"] = _accuracy(h, st, R, t, sig, model, _oracle_rows(P))
        c = clk.summary()
        if c:
            ent["clocks"] = c
        return ent
    finally:
        api.fr_m(h)


def config_batch(L, peak, steps=5, clock_dir="/tmp"):
    """The batched workload: 256 problems x 32 grid rotations in one persistent launch per
    evaluation, tile shape autotuned, device time of each evaluation from the library's events."""
    import torch
    from dugma_b200 import api, synth
    from oracle import oracle as orc
    probs = synth.workload3()
    grid = synth.so3_grid(synth.rng_for(3, 1), 32)
    Q = len(grid)
    sig = np.zeros((len(probs), Q))
    for k, P in enumerate(probs):
        _, h = api.init(P.X, P.X_C, P.Y, P.Y_C)
        sig[k, :] = api.update_sig(h, np.eye(3), P.t_G)
        api.fr_m(h)
    R = np.array([[g @ P.R_G for g in grid] for P in probs])
    t = np.array([[P.t_G for _ in grid] for P in probs])
    pairs = Q * sum(P.N * P.M for P in probs)
    b = api.Batch([(P.X, P.X_C, P.Y, P.Y_C) for P in probs])
    try:
        tune = b.autotune(R, t, sig)
        for _ in range(3):
            E, g = b.energy_grad(R, t, sig)
        torch.cuda.synchronize()
        b.timing(1)
        with Clocks(os.path.join(clock_dir, "dugma_clocks_batch.csv"), torch.cuda.current_device()) as clk:
            t0 = time.perf_counter()
            for _ in range(steps):
                E, g = b.energy_grad(R, t, sig)
            wall = time.perf_counter() - t0
        dev_ms, n = b.timing(2)
        b.timing(0)
        ms = dev_ms / max(n, 1)
        instr = FP32_INSTR_ADJOINT
        rng = np.random.default_rng(7)
        errs = []
        for p, q in zip(rng.choice(len(probs), 4, replace=False), rng.integers(0, Q, 4)):
            P = probs[p]
            Eo, go, _ = orc.State(P.X, P.X_C, P.Y, P.Y_C).energy(R[p, q], t[p, q], sig[p, q])
            errs.append((abs(E[p, q] - Eo) / abs(Eo), float(np.linalg.norm(g[p, q] - go) / np.linalg.norm(go))))
        ent = {"workload": "batch256x32: 256 problems, N, M uniform in [500, 8000], 32 rotations of a uniform "
                           "SO(3) grid each, one persistent launch per evaluation (graph replay)",
               "pair_terms_per_eval": int(pairs), "steps": steps, "warmup": 3, "ms_per_step": ms,
               "pair_terms_per_s": pairs / (ms * 1e-3), "e2e_pair_terms_per_s": pairs * steps / wall,
               "e2e_ms_per_step": 1e3 * wall / steps,
               "roofline": {"bound": "fp32", "instr_per_pair": instr, "kernel_ms": ms,
                            "achieved": instr * pairs / (ms * 1e-3) / 1e12, "unit": "Tinstr/s",
                            "frac": instr * pairs / (ms * 1e-3) / peak,
                            "note": "device time of the whole evaluation (records prologue, pair launch, reduction)"},
               "kernel_shape": list(b.get_shape()), "autotune": tune,
               "accuracy": {"pairs_checked": len(errs), "E_rel_err": max(e[0] for e in errs),
                            "grad_rel_err": max(e[1] for e in errs), "tolerance": {"E": 1e-6, "grad": 1e-5},
                            "against": "FP64 oracle, 4 sampled (problem, pose) pairs, all rows"},
               "l2": "the records of all problems (4.5 GB) exceed L2; no flush"}
        c = clk.summary()
        if c:
            ent["clocks"] = c
        return ent
    finally:
        b.close()


def config_plugins(L, P, peak, reps=5, clock_dir="/tmp"):
    """update_sig and compi through the plugin interface at the headline size (host R, t in, sigma /
    637 coefficients out, like the reference's MEX gateways): wall time per call and the device
    time of the pair kernels; compi's coefficients checked against the FP64 oracle on the 6K
    workload, update_sig's nearest squared distances bit for bit on 4096 rows."""
    import ctypes
    import torch
    from dugma_b200 import api, synth
    from oracle import oracle as orc
    R, t = eval_pose(P, 0)
    _, h = api.init(P.X, P.X_C, P.Y, P.Y_C)
    res = {}
    try:
        sig = api.update_sig(h, R, t)
        for name, fn, instr in (("update_sig", lambda: api.update_sig(h, R, t), None),
                                ("compi", lambda: api.compi(h, R, t, sig=sig), FP32_INSTR_COMPI)):
            fn()
            torch.cuda.synchronize()
            L.dugma_timing(h.arr, 1, None, None)
            with Clocks(os.path.join(clock_dir, f"dugma_clocks_{name}.csv"), torch.cuda.current_device()) as clk:
                walls = []
                for _ in range(reps):
                    a0 = time.perf_counter()
                    fn()
                    walls.append(time.perf_counter() - a0)
            kms, kl = ctypes.c_double(0), ctypes.c_int(0)
            L.dugma_timing(h.arr, 2, ctypes.byref(kms), ctypes.byref(kl))
            L.dugma_timing(h.arr, 0, None, None)
            ms = 1e3 * float(np.median(walls))
            ent = {"workload": f"{P.name}: N={P.N}, M={P.M}, host-to-host plugin call", "reps": reps, "warmup": 1,
                   "ms_per_call": ms, "pair_terms_per_s": P.N * P.M / (ms * 1e-3),
                   "pair_kernel_ms_per_call": kms.value / reps}
            if instr:
                ent["roofline"] = {"bound": "fp32", "instr_per_pair": instr,
                                   "frac": instr * P.N * P.M / (kms.value / reps * 1e-3) / peak,
                                   "note": "one pass over the pairs: d 6, two quadratic forms (Cholesky) 18, p 1, source-side "
                                           "sums 10, target-side sums 10 FP32 lane-ops per pair"}
            c = clk.summary()
            if c:
                ent["clocks"] = c
            res[name] = ent
        # nearest squared distances of 4096 sampled rows, bit for bit
        rows = 4096
        idx, d2 = api.nn(h, R, t, 1)
        st = orc.State(P.X[:rows], P.X_C[:rows], P.Y, P.Y_C)
        oi, od = st.nn(R, t, 1)
        res["update_sig"]["accuracy"] = {"rows": rows, "nn_idx_exact": bool(np.array_equal(idx[:rows], oi)),
                                         "nn_d2_bit_exact": bool(np.array_equal(d2[:rows], od)),
                                         "against": "FP64 oracle's FP32 distance sequence (update_sig.cu:238-259)"}
    finally:
        api.fr_m(h)
    P1 = synth.workload1()
    R1, t1 = eval_pose(P1, 0)
    _, h = api.init(P1.X, P1.X_C, P1.Y, P1.Y_C)
    try:
        s1 = api.update_sig(h, R1, t1)
        A = api.compi(h, R1, t1, sig=s1)
        Ao = orc.State(P1.X, P1.X_C, P1.Y, P1.Y_C).coef(R1, t1, s1)[:637]
        res["compi"]["accuracy"] = {"workload": "sphere6k", "max_abs_err_over_max_abs": float(
            np.abs(A - Ao).max() / np.abs(Ao).max()), "tolerance": 2e-6, "against": "FP64 oracle, all 637"}
    finally:
        api.fr_m(h)
    # registration size: the plugin calls and one EM iteration (update_sig then compi at its sigma,
    # one captured graph) at 4096 x 4096, median wall time of 200 host-to-host calls each
    P4 = synth.workload0(n=4096)
    R4, t4 = eval_pose(P4, 0)
    _, h = api.init(P4.X, P4.X_C, P4.Y, P4.Y_C)
    try:
        s4 = api.update_sig(h, R4, t4)
        g = api.EMGraph(h)
        try:
            def med(fn, n=200):
                fn()
                fn()
                w = []
                for _ in range(n):
                    a0 = time.perf_counter()
                    fn()
                    w.append(time.perf_counter() - a0)
                return 1e3 * float(np.median(w))
            with Clocks(os.path.join(clock_dir, "dugma_clocks_sphere4k.csv"), torch.cuda.current_device()) as clk:
                ent = {"workload": "sphere4k: N = M = 4096, host-to-host calls, median of 200",
                       "compi_ms_per_call": med(lambda: api.compi(h, R4, t4, sig=s4)),
                       "update_sig_ms_per_call": med(lambda: api.update_sig(h, R4, t4)),
                       "em_iteration_ms": med(lambda: g(R4, t4))}
            c = clk.summary()
            if c:
                ent["clocks"] = c
            res["sphere4k_calls"] = ent
        finally:
            g.close()
    finally:
        api.fr_m(h)
    return res


def config_kinect(modes=(0, 1), clock_dir="/tmp"):
    """The reference's 30 real Kinect scenes (tests/golden/kinect_scenes.npz) registered end to end
    from the identity pose with main_kinect_real_application.m's settings: per mode, the medians of
    the error measures against the ground truth, the distance to the authors' recorded poses, and
    the seconds per scene (host clouds in, pose out) against the authors' recorded seconds, with
    the SM clocks sampled over the mode's 30 registrations."""
    import torch
    from dugma_b200 import evaluate
    path = os.path.join(ROOT, "tests", "golden", "kinect_scenes.npz")
    out = {"workload": "kinect30: the reference's 30 two-Kinect scenes (N, M 463..5334), identity start, 300 "
                       "iterations, tolerances 1e-4 / 1e-8 / 1e-9"}
    scenes = list(evaluate.scenes_from_npz(path))
    for mode in modes:
        with Clocks(os.path.join(clock_dir, f"dugma_clocks_kinect{mode}.csv"), torch.cuda.current_device()) as clk:
            rows = [evaluate.register(P, mode, 300, rec) for P, rec in scenes]
        s = evaluate.summarise(rows, mode)
        out[f"mode{mode}"] = {k: s[k]["median"] for k in ("error_R", "error_t", "deg", "iterations", "seconds",
                                                          "vs_recorded_deg", "vs_recorded_t", "recorded_error_R",
                                                          "recorded_error_t", "recorded_seconds")}
        out[f"mode{mode}"]["max_vs_recorded_deg"] = s["vs_recorded_deg"]["max"]
        out[f"mode{mode}"]["statistic"] = "median over the 30 scenes (max where named)"
        c = clk.summary()
        if c:
            out[f"mode{mode}"]["clocks"] = c
    return out


def config_simulation(clock_dir="/tmp", trials=100):
    """The reference's simulation protocol (main_simulation.m:17-56: random rotation within 30 deg,
    translation, noise, outliers and occlusion drawn per problem) on its own models
    (tests/golden/sim_models.npz: 2D shape and fish contours, the 3D surface), registered with
    the reference's loop from the identity with main_simulation.m's settings; per model set the
    medians of the error measures, the share of problems within 2 deg of the ground truth and the
    seconds per registration."""
    import torch
    from dugma_b200 import evaluate
    path = os.path.join(ROOT, "tests", "golden", "sim_models.npz")
    out = {"workload": f"simulation: {trials} problems per model set (2D_SHAPE_MODEL 'S', 2D_Fish_MODEL/dataset2D_200 "
                       "'F', 3D_SHAPE 'T'), seeded, mode 0, 700 iterations, tolerances 1e-4 / 1e-8 / 1e-9"}
    for models in ("S", "F", "T"):
        with Clocks(os.path.join(clock_dir, f"dugma_clocks_sim{models}.csv"), torch.cuda.current_device()) as clk:
            rows = [evaluate.register(P, 0, 700) for P, _ in evaluate.scenes_simulation(path, models, trials)]
        deg = np.array([r["deg"] for r in rows])
        ent = {k: float(np.median([r[k] for r in rows])) for k in ("error_R", "error_t", "deg", "iterations", "seconds")}
        ent["within_2deg"] = float(np.mean(deg < 2.0))
        ent["statistic"] = "median over the problems"
        c = clk.summary()
        if c:
            ent["clocks"] = c
        out[models] = ent
    return out


def run_configs(L, peak, clock_dir):
    """Compact results of every configured workload besides the headline one."""
    from dugma_b200 import synth
    out = {}
    timings = {}

    def run(key, fn):
        a0 = time.perf_counter()
        try:
            out[key] = fn()
        except Exception as e:   # one failing entry must not hide the others
            out[key] = {"error": f"{type(e).__name__}: {e}"}
        timings[key] = round(time.perf_counter() - a0, 1)

    run("cfg0_sphere1k", lambda: config_single(L, "cfg0", synth.workload0(), 0, peak, clock_dir=clock_dir))
    run("cfg1_sphere6k", lambda: config_single(L, "cfg1", synth.workload1(), 0, peak, clock_dir=clock_dir))
    run("cfg3_batch256x32", lambda: config_batch(L, peak, clock_dir=clock_dir))
    run("cfg4_depth300k_64poses", lambda: config_single(L, "cfg4", synth.workload4(), 0, peak, steps=1, poses=64,
                                                         nn_k=8, clock_dir=clock_dir))
    run("curve2d_64k", lambda: config_single(L, "cfg5", synth.workload5(), 0, peak, clock_dir=clock_dir))
    run("conv_harmonic64k", lambda: config_single(L, "conv", synth.workload2(), 1, peak, clock_dir=clock_dir))
    run("plugins_harmonic64k", lambda: config_plugins(L, synth.workload2(), peak, clock_dir=clock_dir))
    run("kinect30_registration", lambda: config_kinect(clock_dir=clock_dir))
    run("simulation_registration", lambda: config_simulation(clock_dir=clock_dir))
    out["seconds"] = timings
    return out


def run_plugin(args):
    """--plugin: one call repeated on the workload, for profiling."""
    import ctypes
    import torch
    from dugma_b200 import _lib, api
    P = workload(args.workload, args.n)
    R, t = eval_pose(P, 0)
    _, h = api.init(P.X, P.X_C, P.Y, P.Y_C)
    sig = api.update_sig(h, R, t)
    calls = {"compi": lambda: api.compi(h, R, t, sig=sig),
             "update_sig": lambda: api.update_sig(h, R, t),
             "compi_range": lambda: api.compi_range(h, R, t, sig, 0, P.N, 0, 0),
             "nn": lambda: api.nn(h, R, t, args.knn),
             "knn_covariance": lambda: api.knn_covariance(P.X, k=args.knn)}
    fn = calls[args.plugin]
    for _ in range(max(1, args.warmup)):
        fn()
    torch.cuda.synchronize()
    L = _lib.load()
    L.dugma_timing(h.arr, 1, None, None)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        fn()
    el = time.perf_counter() - t0
    kms, kl = ctypes.c_double(0), ctypes.c_int(0)
    L.dugma_timing(h.arr, 2, ctypes.byref(kms), ctypes.byref(kl))
    L.dugma_timing(h.arr, 0, None, None)
    api.fr_m(h)
    line = {"plugin": args.plugin, "workload": P.name, "N": P.N, "M": P.M, "calls": args.steps,
            "ms_per_call": 1e3 * el / max(1, args.steps)}
    if kl.value:   # the context's pair kernels (knn_covariance runs on a context of its own)
        line["pair_kernel_ms_per_call"] = kms.value / max(1, args.steps)
        line["pair_kernel_pairs_per_s"] = P.N * P.M * args.steps / (kms.value * 1e-3)
    if args.plugin in ("nn", "knn_covariance"):
        line["k"] = args.knn
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local = dist_setup(args.gpus)
    if args.plugin:
        if rank == 0:
            import torch
            torch.cuda.set_device(local % max(1, torch.cuda.device_count()))
            run_plugin(args)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.impl == "reference-gpu":
        run_reference_gpu(args, rank)
        return
    if args.workload == 3:
        dist_init(world, local)
        run_batch(args, rank, world)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import torch
    import torch.distributed as dist
    dev = dist_init(world, local)
    from dugma_b200 import _lib, api
    L = _lib.load(build_if_missing=False)

    P = workload(args.workload, args.n)
    D = P.X.shape[1]
    ng = 6 if D == 3 else 3
    if D == 2 and args.model == 1:
        raise SystemExit("the CONV model is measured on the 3D workloads")
    R, t = eval_pose(P, rank * max(1, args.poses))
    _, h = api.init(P.X, P.X_C, P.Y, P.Y_C)
    sig = api.update_sig(h, R, t)
    if args.shape:
        shape_key = tuple(int(v) for v in args.shape.split(","))
        api.set_shape(h, 0 if args.model == 0 else 3, shape_key)
        tune = f"pinned {args.shape}"
    else:
        kind = 0 if args.model == 0 else 3     # REF or CONV adjoint shapes
        tune = "" if args.no_tune else api.autotune(h, kind)
        shape_key = api.get_shape(h, kind)
        if tune:
            import re
            best = min(re.findall(r"\(ipt=(\d+),nt=(\d+),tj=(\d+),pack=(\d+)\):([0-9.]+)ms", tune), key=lambda m: float(m[4]))
            shape_key = tuple(int(v) for v in best[:4])
    if not args.no_fd and not args.shape and not args.no_tune:
        # the plain form's energy kernel gets the same treatment
        tune_energy = api.autotune(h, 1 if args.model == 0 else 4)
    else:
        tune_energy = ""
    pairs = P.N * P.M

    # a dedicated stream: handle 0 (the legacy default stream) means 'the context stream' in the C ABI
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    npose = max(1, args.poses)
    pose = torch.zeros(npose, 16, dtype=torch.float64, device="cuda")
    for k in range(npose):
        Rk, tk = (R, t) if k == 0 else eval_pose(P, rank * npose + k)
        pose[k, :D * D] = torch.tensor(np.asarray(Rk).T.reshape(-1))
        pose[k, 9:9 + D] = torch.tensor(tk)
        pose[k, 12] = sig
    out = torch.zeros(npose, 8, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def step():
        for k in range(npose):
            rc = L.dugma_energy_grad_async(h.arr, pose[k].data_ptr(), args.model, out[k].data_ptr(), None,
                                           stream.cuda_stream)
            if rc != 0:
                raise RuntimeError(L.dugma_last_error().decode())

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    import ctypes
    L.dugma_timing(h.arr, 1, None, None)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    import tempfile
    with Clocks(os.path.join(tempfile.gettempdir(), f"dugma_clocks_rank{rank}.csv"), dev) as clk:
        for k in range(args.steps):
            with torch.cuda.stream(stream):   # the flush ends before the step's start event
                flush.fill_(float(k))
            ev[k][0].record(stream)
            step()
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = sum(a.elapsed_time(b) for a, b in ev)
    kms = ctypes.c_double(0)
    kl = ctypes.c_int(0)
    L.dugma_timing(h.arr, 2, ctypes.byref(kms), ctypes.byref(kl))
    L.dugma_timing(h.arr, 0, None, None)
    ms = all_reduce([ms], "max")[0]
    value = world * pairs * npose * args.steps / (ms * 1e-3)
    res = out[0].cpu().numpy()

    # the nearest-distance pass behind sigma (update_sig through the C ABI, host pose in, sigma out)
    api.update_sig(h, R, t)
    reps = 5
    a0 = time.perf_counter()
    for _ in range(reps):
        api.update_sig(h, R, t)
    upd_ms = 1e3 * (time.perf_counter() - a0) / reps

    # roofline of the adjoint kernel
    peak = ctypes.c_double(0)
    L.dugma_calibrate(0, ctypes.byref(peak), None)
    sfu = ctypes.c_double(0)
    L.dugma_calibrate(1, ctypes.byref(sfu), None)
    kernel_ms = kms.value / max(kl.value, 1)
    instr = (FP32_INSTR_ADJOINT if D == 3 else FP32_INSTR_ADJOINT_2D) if args.model == 0 else FP32_INSTR_CONV_ADJOINT
    achieved = instr * pairs / (kernel_ms * 1e-3)
    sfu_frac = SFU_PER_PAIR * pairs / (kernel_ms * 1e-3) / sfu.value if sfu.value else None

    extra = {}
    if not args.no_fd and rank == 0:
        # plain form: energy + central FD over the pose coordinates (13 energy evaluations in 3D, 7 in 2D)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        api.energy_fd_grad(h, R, t, sig, model=args.model)
        reps = max(2, args.steps // 4)
        t0.record()
        for _ in range(reps):
            api.energy_fd_grad(h, R, t, sig, model=args.model)
        t1.record()
        torch.cuda.synchronize()
        fd_ms = t0.elapsed_time(t1) / reps
        adj_ms = ms / (args.steps * npose)
        extra["plain_fd"] = {"ms_per_gradient": fd_ms, "evals_per_s": 1e3 / fd_ms,
                             "adjoint_evals_per_s": 1e3 / adj_ms, "adjoint_speedup": fd_ms / adj_ms,
                             "energy_evals_per_gradient": 1 + 2 * ng}
        if args.model == 0:
            # the same at the reference's per-pair precision (FP64 d, quadratic forms and exp)
            api.energy_fd_grad(h, R, t, sig, model=2)
            fd64 = []
            for _ in range(2):
                t0.record()
                api.energy_fd_grad(h, R, t, sig, model=2)
                t1.record()
                torch.cuda.synchronize()
                fd64.append(t0.elapsed_time(t1))
            fd64_ms = min(fd64)
            extra["plain_fd"].update({"fp64_ms_per_gradient": fd64_ms,
                                      "fp64_energy_pair_terms_per_s": (1 + 2 * ng) * pairs / (fd64_ms * 1e-3),
                                      "adjoint_speedup_vs_fp64": fd64_ms / adj_ms})

    e2e = None
    if not args.no_e2e:
        # the host threads and the pinned inputs on the GPU's own NUMA node (NVML's CPU affinity of
        # the device), as a host application placed for this GPU would have them; restored after
        cpus_all = os.sched_getaffinity(0)
        cpus_local = gpu_local_cpus(torch.cuda.current_device())
        if cpus_local:
            os.sched_setaffinity(0, cpus_local)
        try:
            # the step's inputs in pinned host memory, laid out as the C ABI takes them (the
            # covariance arrays are views whose transpose is the contiguous MATLAB block order)
            def pinned(a):
                return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()

            Xh, Yh = pinned(P.X), pinned(P.Y)
            X_C = pinned(np.transpose(P.X_C, (0, 2, 1))).transpose(0, 2, 1)
            Y_C = pinned(np.transpose(P.Y_C, (0, 2, 1))).transpose(0, 2, 1)
            # the clouds and covariances, plus the 16-double pose block dugma_energy_grad uploads
            h2d = 8 * (Xh.size + X_C.size + Yh.size + Y_C.size) + 8 * 16
            # warm-up of the end-to-end path
            _, h2 = api.init(Xh, X_C, Yh, Y_C)
            api.energy_grad(h2, R, t, sig, model=args.model)
            api.fr_m(h2)
            ksteps = max(3, min(args.steps, 10))
            ph = [0.0, 0.0, 0.0]
            t0 = time.perf_counter()
            for _ in range(ksteps):
                a = time.perf_counter()
                _, h2 = api.init(Xh, X_C, Yh, Y_C)
                b = time.perf_counter()
                api.energy_grad(h2, R, t, sig, model=args.model)
                c = time.perf_counter()
                api.fr_m(h2)
                d = time.perf_counter()
                ph[0] += b - a
                ph[1] += c - b
                ph[2] += d - c
            el = time.perf_counter() - t0
            el = all_reduce([el], "max")[0]
            e2e = {"value": world * pairs * ksteps / el, "unit": "pair-terms/s", "host_memory": "pinned",
                   "h2d_bytes_per_step": int(h2d),
                   "d2h_bytes_per_step": 8 * (1 + ng) + 4, "steps": ksteps,
                   "ms_per_step": {"init": 1e3 * ph[0] / ksteps, "energy_grad": 1e3 * ph[1] / ksteps,
                                   "fr_m": 1e3 * ph[2] / ksteps}}
        finally:
            if cpus_local:
                os.sched_setaffinity(0, cpus_all)
        e2e["host_cpus"] = (f"{len(cpus_local)} CPUs local to the GPU (NVML affinity)" if cpus_local
                            else "all allowed CPUs (NVML gave no affinity)")

    cpu = None
    if not args.no_cpu and world == 1:
        rate, done, el, cores, (nrow, Eo, go) = cpu_rate(P, R, t, sig, args.model)
        cpu = {"value": rate, "unit": "pair-terms/s", "cores": cores, "kind": "port",
               "sample": f"{done // P.M} source rows x {P.M} targets ({el:.1f} s, FP64 oracle, OpenMP)"}
        # this run's error against the FP64 oracle on the same rows: the fused adjoint over source
        # rows [0, nrow) through the C ABI against the oracle's sum over those rows
        Eg, gg = api.energy_grad_range(h, R, t, sig, 0, nrow, model=args.model)
        go = np.asarray(go, np.float64)
        accuracy = {"rows": int(nrow), "targets": int(P.M), "E_oracle": float(Eo), "E": float(Eg),
                    "E_rel_err": abs(Eg - Eo) / abs(Eo) if Eo else None,
                    "grad_rel_err": float(np.max(np.abs(gg - go)) / np.max(np.abs(go))) if np.any(go) else None,
                    "tolerance": {"E": 1e-6, "grad": 1e-5}}

    configs = None
    if not args.no_configs and world == 1 and args.workload == 2 and not args.n and args.model == 0:
        import tempfile
        configs = run_configs(L, peak.value, tempfile.gettempdir())

    if rank == 0:
        clocks = clk.summary()
        line = {
            "metric": "energy+grad pair-terms/s", "value": value, "unit": "pair-terms/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_for(P, npose, args.model),
            "details": {"sigma": sig, "kernel_shape": list(shape_key), "poses_per_step": npose,
                        "update_sig_ms": upd_ms,
                        "update_sig_pair_terms_per_s": pairs / (upd_ms * 1e-3)},
            "roofline": {"bound": "fp32", "achieved": achieved / 1e12, "peak": peak.value / 1e12,
                         "unit": "Tinstr/s (FP32 pipe, lane ops)", "frac": achieved / peak.value,
                         "traffic": profiled_traffic(shape_key) if (args.workload == 2 and not args.n and args.model == 0)
                         else None,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of this bench command, "
                                           "committed in profiles/adjoint_packed_harmonic64k.txt (shape 4,64,64,2); "
                                           "null when this run's shape or workload differs",
                         "algorithmic_bytes": 64 * (P.N + P.M),
                         "peak_source": "FP32 FMA-chain kernel measured in this run (MEASURED_PEAKS.json has "
                                        "no FP32-pipe figure)",
                         "sfu_frac": sfu_frac, "kernel_ms": kernel_ms,
                         "instr_per_pair": instr,
                         "hbm_view": hbm_view(64 * (P.N + P.M), kernel_ms)},
            "gpu_launches": 3 * args.steps * npose,
            "result": {"E": float(res[0]), "g": [float(v) for v in res[1:1 + ng]]},
            "autotune": tune,
            "autotune_energy": tune_energy,
        }
        if e2e:
            line["e2e"] = e2e
        if cpu:
            line["cpu_baseline"] = cpu
            line["accuracy"] = accuracy
        if clocks:
            line["clocks"] = clocks
        line.update(extra)
        if configs:
            line["configs"] = configs
        print(json.dumps(line), flush=True)
    api.fr_m(h)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
