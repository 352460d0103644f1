"""Benchmark: worst-case load solve on the 128x128x64 configuration on one B200.

A step is one worst-case solve of the hot path on the resident design:
Galerkin coarse-stencil assembly + coarsest factorisation, then the largest
eigenvalue of the load-space compliance operator P K^-1 P by Lanczos (k=16
Krylov vectors) whose inner MG-PCG solves run to relative residual 1e-6, then
the worst-case displacement solve to 1e-6.  ``value`` uses the mixed form (FP32
V-cycles inside FP64 CG; FP64 residuals, dots, orthogonalisation, Rayleigh
quotient and coarsest solve); the all-FP64 form is reported beside it.

Input: seeded synthetic density (smoothed Gaussian field, sigmoid map), z=0
clamped, loadable set = top face; no dataset is read.

``--impl reference`` times the CPU restatement of the reference algorithm
(oracle/, OpenMP, all host cores) on the same configuration — the reference
itself cannot be built in this image (its sources need Eigen, CGAL and OpenVDB).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(nx=128, ny=128, nz=64, seed=0, k=16, tol=1e-6)
# plain: the reference's V-cycle made symmetric (8-colour GS, forward pre / backward post), all FP64
# mixed: FP32 V-cycle with Chebyshev(2) smoothing (8 steps on the coarse levels), FP64 coarsest solve,
#        FP32 flexible-CG vectors restarted from FP64 residuals (iterative refinement), FP64 V-cycles
#        once the FP32 ones stall
FORMS = {"plain": dict(precision="FP64", smoother="SMOOTH_SGS", sweeps=1, coarse_sweeps=0, cycle_gamma=1,
                       coarse_bf16=0, krylov_fp32=0),
         "mixed": dict(precision="FP32", smoother="SMOOTH_CHEBY", sweeps=2, coarse_sweeps=8, cycle_gamma=1,
                       coarse_bf16=0, krylov_fp32=2)}
# the batched graph runs FP64-vector CG (the Krylov form is a single-solve path): the sequential
# solves it is compared with use the same form
FORMS_BATCH = dict(FORMS["mixed"], krylov_fp32=0)
# on the 511x256x256 arch the W-cycle (coarse corrections twice per visit below level 1) wins
FORMS_C5 = {"plain": FORMS["plain"],
            "mixed": dict(precision="FP32", smoother="SMOOTH_CHEBY", sweeps=2, coarse_sweeps=0, cycle_gamma=2,
                          coarse_bf16=0, krylov_fp32=0),
            "fp64_same_cycle": dict(precision="FP64", smoother="SMOOTH_CHEBY", sweeps=2, coarse_sweeps=0,
                                    cycle_gamma=2, coarse_bf16=0, krylov_fp32=0)}


def apply_form(rb, G, form):
    p = G.params
    p.precision = getattr(rb, form["precision"])
    p.smoother = getattr(rb, form["smoother"])
    p.pre_sweeps = p.post_sweeps = form["sweeps"]
    p.coarse_sweeps = form["coarse_sweeps"]
    p.cycle_gamma = form["cycle_gamma"]
    p.coarse_bf16 = form["coarse_bf16"]
    p.krylov_fp32 = form.get("krylov_fp32", 0)
    G.set_params(p)


def form_text(form):
    return (f"{form['precision']} V-cycle{' (W below level 1)' if form['cycle_gamma'] == 2 else ''}, "
            f"{form['smoother'][7:].lower()}({form['sweeps']}) smoothing"
            f"{', ' + str(form['coarse_sweeps']) + ' steps on coarse levels' if form['coarse_sweeps'] else ''}"
            f"{', BF16 coarse stencils' if form['coarse_bf16'] else ''}"
            f"{', FP32 Krylov vectors with FP64 refinement' if form.get('krylov_fp32') else ''}")
METRIC = "worst-case solve (Lanczos k=16, MG-PCG inner solves to rel. residual 1e-6) on 128x128x64"


def init_replicas(ws, lrank, backend="nccl"):
    """One process per GPU: the process group the replicas use for their barriers and the
    max-over-ranks timing (no data-path collective: every replica solves its own problem).
    Returns the torch.distributed module, or None for a single process."""
    if ws <= 1:
        return None
    import datetime

    import torch
    import torch.distributed as dist

    if backend == "nccl":
        torch.cuda.set_device(lrank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", lrank))
    else:
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return dist


def max_over_ranks(dist, values, device="cuda"):
    """Element-wise maximum of a list of timings over all ranks (the job's time is its slowest
    replica's); the values unchanged for a single process."""
    if dist is None:
        return list(values)
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    lrank = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, lrank


def gpu_id(cuda_index):
    """The id nvidia-smi should sample for CUDA device ``cuda_index``: its UUID.  nvidia-smi numbers
    GPUs by NVML order and ignores CUDA_VISIBLE_DEVICES, so a CUDA ordinal can name another GPU."""
    try:
        import torch

        return f"GPU-{torch.cuda.get_device_properties(cuda_index).uuid}"
    except Exception:
        return str(cuda_index)


class Clocks:
    """nvidia-smi sampling during the timed region (``gpu`` is an id from gpu_id)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

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
        for l in self.lines:
            p = [x.strip() for x in l.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "gpu": self.gpu}


def build_problem(rb, configs, ctx, precision, dims=None):
    nx, ny, nz = dims or (WORKLOAD["nx"], WORKLOAD["ny"], WORKLOAD["nz"])
    cfg = configs.worst_case_box(nx, ny, nz, seed=WORKLOAD["seed"])
    params = rb.default_params(mode=cfg["mode"], youngs_modulus=1e6, poisson_ratio=0.4, power_penalty=3.0,
                               min_rho=1e-3, precision=precision, smoother=rb.SMOOTH_SGS, pre_sweeps=1,
                               post_sweeps=1)
    G = rb.HierarchyGrid(ctx, params)
    G.genFromBox(cfg["eact"])
    G[0].setRho(cfg["rho"].ravel())
    G.set_support(cfg["vfix"])
    G.set_load_nodes(cfg["load_nodes"], cfg["normals"])
    return cfg, G


def step(rb, G, seed):
    G.update_stencil()
    lam, info = G.worst_case(rb.WORST_LANCZOS, WORKLOAD["k"], WORKLOAD["tol"], seed=seed)
    return lam, info


def time_steps(rb, ctx, G, steps, seed0=100):
    """K steps bracketed by synchronize + CUDA events on the library's stream."""
    import torch

    stream = torch.cuda.ExternalStream(ctx_stream_handle(ctx))
    ctx.sync()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    l0 = ctx.launches()
    ev0.record(stream)
    lams, infos = [], []
    for s in range(steps):
        lam, info = step(rb, G, seed0 + s)
        lams.append(lam)
        infos.append(info)
    ev1.record(stream)
    ev1.synchronize()
    ctx.sync()
    return ev0.elapsed_time(ev1), lams, infos, ctx.launches() - l0


_STREAMS = {}


def ctx_stream_handle(ctx):
    return _STREAMS[id(ctx)]


def make_ctx(rb, device):
    import torch

    torch.cuda.set_device(device)
    s = torch.cuda.Stream(device=device)
    ctx = rb.Context(device, C.c_void_p(s.cuda_stream))
    _STREAMS[id(ctx)] = s.cuda_stream
    ctx._torch_stream = s
    return ctx


# algorithmic bytes per launch of the kernels that can dominate (per node of the level,
# level-0 sizes): u/f/r are 3 components of s bytes, w is 4 B per element, flags 1 B
def algorithmic_bytes(name, nv, ne, s):
    if name.startswith("fine_residual") or name.startswith("fine_jacobi"):
        return nv * (3 * s * 3 + 1 + 1) + ne * 4   # read u, f; write r/unew; vact, vfix; w
    if name.startswith("fine_cheby"):
        return nv * (3 * s * 5 + 1 + 1) + ne * 4   # read u, f, d; write unew, d; vact, vfix; w
    if name.startswith("fine_applyK"):
        return nv * (3 * s * 2 + 1 + 1) + ne * 4
    if name.startswith("fine_gs"):
        # one colour: read u of all nodes + w, read f / write u of 1/8 of the nodes
        return nv * (3 * s + 1 + 1) + ne * 4 + nv // 8 * (3 * s * 2)
    return None


# DRAM bytes (read + write) per launch from one ncu capture of the kernel on this workload,
# per node (1,081,665 nodes): register-marching variant (rows 2, z-chunk 8) 71.0 MB read +
# 3.3 MB written; tile variant (rows 4, z-chunk 8) 45.33 MB read + 0.31 MB written;
# pipelined tile variant (rows 8, z-chunk 8) 45.33 MB read + 0.26 MB written.  The tile
# variants' 26 MB of writes are still in the 126 MB L2 when the launch ends.  None for
# variants without a capture.
NCU_TRAFFIC_PER_NODE = {("fine_cheby_f32", "register_march"): (71.0e6 + 3.3e6) / 1081665,
                        ("fine_cheby_f32", "smem_tile"): (45.326e6 + 0.306e6) / 1081665,
                        ("fine_cheby_f32", "smem_tile_pipelined"): (45.329e6 + 0.256e6) / 1081665}


# DRAM bytes (read + write) per node of the finest-level kernels on the arch workload, from one ncu
# capture of the same kernel variant and launch shape (8 rows, z-chunk 32) on the 255x256x128
# worst-case box, whose vectors exceed L2 (8,487,168 nodes: 359.7 MB read + 171.8 MB written);
# traffic grows with the nodes, so the per-node figure scales to the arch's node box
NCU_TRAFFIC_ARCH = {("fine_cheby_f32", "smem_tile_pipelined"): (359.672064e6 + 171.792896e6) / 8487168,
                    ("fine_cheby_f32", "smem_tile_pipelined_tma"): (358.008320e6 + 168.810240e6) / 8487168,
                    ("fine_cheby_f32", "smem_tile_pipelined_tma_x31"): (358.434304e6 + 167.496448e6) / 8487168}
# warp-instructions per node of the same captures (smsp__inst_executed.sum / nodes)
NCU_INST_ARCH = {("fine_cheby_f32", "smem_tile_pipelined", (8, 32)): 222157952 / 8487168,
                 ("fine_cheby_f32", "smem_tile_pipelined_tma", (4, 32)): 256982264 / 8487168,
                 ("fine_cheby_f32", "smem_tile_pipelined_tma_x31", (8, 32)): 232812378 / 8487168}


def roofline(ctx, stats, G, peaks, tuning=None, traffic_table=None):
    # dominant kernel by device time
    name, (n, ms) = max(stats.items(), key=lambda kv: kv[1][1])
    nv, ne = G[0].nv, G[0].ne
    s = 4 if name.endswith("f32") else 8
    b = algorithmic_bytes(name, nv, ne, s)
    avg_s = ms / max(n, 1) * 1e-3
    out = {"kernel": name, "launches": n, "avg_us": avg_s * 1e6, "share": ms / sum(v[1] for v in stats.values())}
    if b is None:
        out.update({"bound": "hbm", "achieved": None, "peak": peaks.get("hbm_gbs"), "unit": "GB/s", "frac": None,
                    "traffic": None})
        return out
    ach = b / avg_s / 1e9
    peak = peaks.get("hbm_gbs", 6650.0)
    variant, shape = None, None
    if tuning and name.startswith("fine_cheby"):
        t = tuning.get("chebyshev_" + name.rsplit("_", 1)[1], {})
        variant, shape = t.get("variant"), (t.get("rows"), t.get("zchunk"))
    per_node = (NCU_TRAFFIC_PER_NODE if traffic_table is None else traffic_table).get((name, variant))
    out.update({"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                "frac": round(ach / peak, 4), "traffic": int(per_node * nv) if per_node else None,
                "traffic_source": "ncu capture of the same kernel variant on this workload" if per_node else None,
                "variant": variant, "rows_zchunk": shape, "algorithmic_bytes": int(b),
                "peak_source": "measured" if "hbm_gbs" in peaks else "fallback"})
    return out


# warp-instructions per node of the finest-level FP32 Chebyshev step (smsp__inst_executed.sum of one
# ncu launch on 128x128x64 at the bench's launch shape, divided by its 1,081,665 nodes)
NCU_INST_PER_NODE = {("fine_cheby_f32", "smem_tile", (4, 8)): 41640038 / 1081665}


def simt_peaks(rb, ctx):
    """FP32 FFMA, packed FFMA2 and FP64 DFMA throughput of this device (project microbenchmark)."""
    out = {}
    for kind, key in ((0, "fp32_tflops"), (1, "fp32x2_tflops"), (2, "fp64_tflops")):
        t = C.c_double()
        rb._capi.check(rb.lib().rt_bench_simt_peak(ctx.handle, kind, 5, C.byref(t)), ctx.handle)
        out[key] = round(t.value, 2)
    return out


def issue_roofline(rb, ctx, G, roof, clk, inst_table=None):
    """The matrix-free finest-level kernel is bound by instruction issue, not HBM: next to the HBM
    fraction, report its warp-instruction rate against 4 per SM per cycle at the measured SM clock,
    and the measured SIMT peaks."""
    import torch

    roof["simt_peaks"] = simt_peaks(rb, ctx)
    shape = tuple(roof["rows_zchunk"]) if roof.get("rows_zchunk") else None
    ipn = (NCU_INST_PER_NODE if inst_table is None else inst_table).get((roof.get("kernel"), roof.get("variant"),
                                                                          shape))
    mhz = (clk or {}).get("sm_mhz")
    if ipn is None or not mhz or not roof.get("avg_us"):
        return
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    inst = ipn * G[0].nv
    ach = inst / (roof["avg_us"] * 1e-6) / 1e9
    peak = 4 * sms * mhz * 1e6 / 1e9
    roof["issue"] = {"warp_inst_per_launch": int(inst), "achieved_ginst_s": round(ach, 1),
                     "peak_ginst_s": round(peak, 1), "frac": round(ach / peak, 4),
                     "source": "ncu smsp__inst_executed.sum of the same variant and shape; peak = 4 warp-"
                               "instructions per SM per cycle at the median SM clock of the timed region"}


def e2e_steps(rb, ctx, G, cfg, steps, seed0=100):
    """Same steps (same Lanczos start vectors as the device-timed ones) through the public
    API with host buffers: H2D of the density each step, worst-case solve, D2H of the
    worst-case load field."""
    import torch

    rho = np.ascontiguousarray(cfg["rho"].ravel(), np.float32)
    fout = np.zeros(3 * G[0].nv)
    stream = torch.cuda.ExternalStream(ctx_stream_handle(ctx))
    ctx.sync()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for s in range(steps):
        G[0].setRho(rho)
        step(rb, G, seed0 + s)
        fout = G[0].getForce()
    ev1.record(stream)
    ev1.synchronize()
    return ev0.elapsed_time(ev1), rho.nbytes, fout.nbytes


def cpu_baseline(gpu_inner_iters, gpu_vcycles, threads):
    """Oracle (plain FP64, OpenMP) on a bounded sample of the same workload:
    stencil assembly once + a few PCG iterations, extrapolated to the number of
    inner PCG iterations one GPU step used."""
    import oracle as O
    from robtop_b200 import configs

    os.environ["OMP_NUM_THREADS"] = str(threads)
    cfg = configs.worst_case_box(WORKLOAD["nx"], WORKLOAD["ny"], WORKLOAD["nz"], seed=WORKLOAD["seed"])
    H = O.Hierarchy(cfg["eact"], cfg["rho"], cfg["vfix"], p=3, E=1e6, nu=0.4)
    t0 = time.perf_counter()
    H.update_stencil()
    t_st = time.perf_counter() - t0
    nv = H.arrs[0]["u"].size // 3
    b = np.zeros(3 * nv)
    b[2 * nv + cfg["load_nodes"]] = 1.0 / np.sqrt(cfg["load_nodes"].size)
    n_it = 3
    t0 = time.perf_counter()
    x, it, rr = H.pcg(b, tol=1e-30, maxit=n_it, smoother=O.SMOOTH_SGS)
    t_it = (time.perf_counter() - t0) / n_it
    total = t_st + t_it * gpu_inner_iters
    return {"value": 1.0 / total, "unit": "solves/s", "cores": threads, "kind": "port", "extrapolated": True,
            "sample": f"oracle FP64 stencil assembly ({t_st:.2f} s) + {n_it} MG-PCG iterations "
                      f"({t_it:.3f} s each), extrapolated to the plain method's {gpu_inner_iters} PCG iterations "
                      "of one step on the GPU",
            "sampled_wall_s": t_st + t_it * n_it, "scale_factor": total / (t_st + t_it * n_it),
            "seconds_per_step": total}


def run_reference(args):
    """The reference arm: the CPU restatement of the reference algorithm (oracle/, plain FP64 SGS
    V-cycle PCG, OpenMP on all host cores) on the same workload as the default arm.  The
    reference's solve path cannot be built here (Grid.cpp and optimization.cpp need Eigen, CGAL and
    OpenVDB; only its element template, four kernels, stop test and voxeliser compile, and those
    pin the oracle).  A full step
    on the 511x256x256 arch takes the oracle tens of minutes, so each step is a bounded sample: the
    oracle runs stencil assembly and one inner solve to 1e-6 on the 127x64x64 arch, and the step
    time is extrapolated to the full arch by node count and to the 17 inner solves of a step (k = 16
    Lanczos solves + the displacement solve) at the sample's iterations per solve.  The line
    carries the sampled wall seconds and the scale factor beside the extrapolated value."""
    ws, rank, lrank = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    if args.workload == "worstcase128":
        return run_reference_128(args, threads)
    dims = tuple(int(v) for v in args.size.split("x")) if args.size else ARCH["dims"]
    solves = ARCH["k"] + 1
    samples = []
    for s_ in range(args.warmup + args.steps):
        # iterations per solve from this sample (no GPU count on this arm)
        smp = arch_cpu_sample(threads, dims, 0, solves)
        its_full = solves * smp["sample_pcg_iterations"]
        smp["plain_inner_iterations_full"] = its_full
        smp["extrapolated_s_per_step"] = smp["node_scale_factor"] * (smp["sample_assembly_s"] +
                                                                      smp["sample_s_per_iteration"] * its_full)
        samples.append(smp)
    tt = samples[args.warmup:]
    sec = sum(t["extrapolated_s_per_step"] for t in tt) / len(tt)
    wall = sum(t["sampled_wall_s"] for t in tt) / len(tt)
    val = 1.0 / sec
    last = tt[-1]
    nx, ny, nz = dims
    line = {"impl": "reference", "metric": METRIC_ARCH.replace(", learned+mixed form", ", plain FP64 method"),
            "value": val, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"arch {nx}x{ny}x{nz}, worst-case solve (Lanczos k=16, inner PCG to 1e-6)",
                       "threads": threads},
            "extrapolated": True,
            "sampled_wall_s_per_step": wall, "scale_factor": sec / wall,
            "sample": {k: last[k] for k in ("sample_dims", "sample_nodes", "sample_assembly_s", "sample_pcg_iterations",
                                            "sample_s_per_iteration", "node_scale_factor")},
            "cpu_baseline": {"value": val, "unit": "solves/s", "cores": threads, "kind": "port", "extrapolated": True,
                             "sample": "CPU restatement of the reference algorithm (the reference's solve path needs "
                                       "Eigen/CGAL/OpenVDB and cannot be built here; the restatement is pinned to the "
                                       "parts that can): stencil assembly + one inner solve to 1e-6 "
                                       f"on the {'x'.join(map(str, last['sample_dims']))} arch per step "
                                       f"({wall:.1f} s of CPU wall time), extrapolated by node count "
                                       f"(x{last['node_scale_factor']:.1f}) and to {solves} inner solves "
                                       f"(scale factor {sec / wall:.0f} overall)"},
            "e2e": {"value": val, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_reference_128(args, threads):
    """Reference arm of the 128x128x64 worst-case box: per step, stencil assembly + 2 of the 16
    Lanczos inner solves by the oracle, the time scaled by 17/2."""
    import oracle as O
    from robtop_b200 import configs

    os.environ["OMP_NUM_THREADS"] = str(threads)
    cfg = configs.worst_case_box(WORKLOAD["nx"], WORKLOAD["ny"], WORKLOAD["nz"], seed=WORKLOAD["seed"])
    H = O.Hierarchy(cfg["eact"], cfg["rho"], cfg["vfix"], p=3, E=1e6, nu=0.4)
    nv = H.arrs[0]["u"].size // 3
    nl = cfg["load_nodes"].size
    times, walls = [], []
    ksample = 2
    scale_f = (WORKLOAD["k"] + 1) / ksample
    for s in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        H.update_stencil()
        work = np.zeros((ksample + 1) * 3 * nl + 10 * 3 * nv)
        lam = np.zeros(1)
        O.lib().or_lanczos(H.LA, H.nlev, O.ptr(H.KE), O.SMOOTH_SGS, 1, 1, 0.6, nl, O.ptr(cfg["load_nodes"]),
                           O.ptr(np.ascontiguousarray(cfg["normals"])), 0, 0, None, 100 + s, ksample, WORKLOAD["tol"],
                           500, O.ptr(lam), None, O.ptr(work))
        dt = time.perf_counter() - t0
        walls.append(dt)
        times.append(dt * scale_f)
    tt = times[args.warmup:]
    sec = sum(tt) / len(tt)
    wall = sum(walls[args.warmup:]) / len(tt)
    val = 1.0 / sec
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "worst-case 128x128x64 (z=0 clamped, top-face load set, wsff), Lanczos k=16",
                       "inner_tol": WORKLOAD["tol"], "threads": threads},
            "extrapolated": True, "sampled_wall_s_per_step": wall, "scale_factor": scale_f,
            "cpu_baseline": {"value": val, "unit": "solves/s", "cores": threads, "kind": "port", "extrapolated": True,
                             "sample": "CPU restatement of the reference algorithm: stencil assembly + 2 of the 16 "
                                       "Lanczos inner solves per step, time scaled by 17/2"},
            "e2e": {"value": val, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_conv(args):
    """One U-Net convolution (rt_unet_conv3) on random bf16 data: --conv CIN,COUT --size XxYxZ
    (voxels); prints its per-launch device time (library CUDA events) and TFLOP/s."""
    import torch

    import robtop_b200 as rb

    cin, cout = (int(v) for v in args.conv.split(","))
    X, Y, Z = (int(v) for v in (args.size or "257x257x129").split("x"))
    V = X * Y * Z
    ctx = rb.Context(0)
    g = torch.Generator(device="cuda").manual_seed(0)
    inp = (torch.randn(V, cin, device="cuda", generator=g) * 0.3).to(torch.bfloat16)
    w = (torch.randn(cout, 27, cin, device="cuda", generator=g) * 0.05).to(torch.bfloat16)
    out = torch.empty(V, cout, device="cuda", dtype=torch.bfloat16)
    argv = (ctx.handle, C.c_void_p(inp.data_ptr()), cin, cin, C.c_void_p(w.data_ptr()), None, cout,
            C.c_void_p(out.data_ptr()), cout, 0, 1, 0, X, Y, Z)
    for _ in range(args.warmup):
        rb._capi.check(rb.lib().rt_unet_conv3(*argv), ctx.handle)
    ctx.profile(True)
    ctx.profile_reset()
    for _ in range(args.steps):
        rb._capi.check(rb.lib().rt_unet_conv3(*argv), ctx.handle)
    st = ctx.profile_stats()
    ctx.profile(False)
    n, ms = [v for k, v in st.items() if k.startswith("unet_conv3") and v[0]][0]
    us = ms / n * 1e3
    print(json.dumps({"kernel": "conv3", "cin": cin, "cout": cout, "dims": [X, Y, Z], "us_per_call": us,
                      "tflops": 2 * 27 * cin * cout * V / (us * 1e-6) / 1e12}))
    ctx.close()
    return 0


def vcycle_bytes(G, s, smoother_sweeps, smoother_bytes_node):
    """Algorithmic bytes of one V-cycle from the level sizes: per level its smoothing sweeps,
    one residual, the restriction into and prolongation from the next level; s = bytes per
    value.  Finest level matrix-free (u, f, r / unew 3 values each per node, 2 flag bytes,
    4 B weight per element); stencil levels 243 values per node plus the vectors."""
    total = 0
    n = G.n_grid()
    for i in range(n):
        L = G[i]
        nv, ne = L.nv, L.ne
        if i == 0:
            sweep = nv * (smoother_bytes_node * s + 2) + 4 * ne
            resid = nv * (9 * s + 2) + 4 * ne
        elif i < n - 1:
            sweep = nv * (243 * s + smoother_bytes_node * s)
            resid = nv * (243 * s + 9 * s)
        else:  # the coarsest level: dense solve on the active nodes
            total += (3 * nv) ** 2 // 64 * 8
            continue
        total += smoother_sweeps * sweep + resid
        total += 2 * (3 * s * nv + 3 * s * G[i + 1].nv)  # restriction and prolongation
    return total


def run_c1(args):
    """The plain method on the small cantilever: 64x32x32 elements, uniform density 0.4,
    x = 0 clamped, total load 1 in -z spread over the bottom edge of the x = 64 face (wsff).
    FP64 V-cycle PCG with 2 + 2 damped block-Jacobi sweeps to relative residual 1e-6, then
    one OC step (sensitivity, filter radius 2, OC update to volume 0.4).  Every step starts
    from the uniform density and zero displacement, so the steps are the same work.

    The timed sweeps use omega 0.5.  With omega 0.6 the Jacobi step amplifies the top of
    the spectrum: lambda_max(D^-1 K) is about 3.7 on the finest level, above 2 / 0.6.  PCG
    then stalls near 6e-5; the oracle and the library agree on this, and the line records
    that run beside the timed one.  The oracle runs the timed solve on the host cores as the
    CPU baseline."""
    import torch

    import robtop_b200 as rb
    from robtop_b200 import configs

    ctx = make_ctx(rb, 0)
    stream = torch.cuda.ExternalStream(ctx_stream_handle(ctx))
    cfg = configs.cantilever(64, 32, 32)
    p = rb.default_params(mode=cfg["mode"], youngs_modulus=1e6, poisson_ratio=0.4, power_penalty=3.0, min_rho=1e-3,
                          precision=rb.FP64, smoother=rb.SMOOTH_JACOBI, pre_sweeps=2, post_sweeps=2,
                          jacobi_omega=0.5, volume_ratio=0.4, design_step=0.03, damp_ratio=0.5, filter_radius=2.0)
    G = rb.HierarchyGrid(ctx, p)
    G.genFromBox(cfg["eact"])
    G.set_support(cfg["vfix"])
    G.set_load_nodes(cfg["load_nodes"], cfg["normals"])
    rho0 = np.ascontiguousarray(cfg["rho"].ravel(), np.float32)
    f = np.ascontiguousarray(cfg["fload"].ravel(), np.float64)
    lam, trials = C.c_float(), C.c_int()
    infos = []

    def one_step(read_back=False):
        G[0].setRho(rho0)
        G.update_stencil()
        G[0].setForce(f)
        G[0].reset_displacement()
        info = G.pcg(1e-6, 500)
        rb._capi.check(rb.lib().rt_sensitivity(G.handle, 1), ctx.handle)
        G[0].filterSensitivity(2.0)
        rb._capi.check(rb.lib().rt_oc_update(G.handle, 0.4, C.byref(lam), C.byref(trials)), ctx.handle)
        infos.append(info)
        return G[0].getRho() if read_back else None

    for _ in range(max(args.warmup, 3)):
        one_step()
    ctx.sync()
    clocks = Clocks(gpu_id(0))
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = ctx.launches()
    e0.record(stream)
    for _ in range(args.steps):
        one_step()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    launches = ctx.launches() - l0
    # end to end with a device-to-host read of the updated density every step
    e0.record(stream)
    for _ in range(args.steps):
        rho_out = one_step(read_back=True)
    e1.record(stream)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    it = infos[-1].iterations
    G[0].setRho(rho0)
    G.update_stencil()
    lmax0 = G.smoother_lmax(0)
    # the same solve with omega 0.6, for the record
    q = G.params
    q.jacobi_omega = 0.6
    G.set_params(q)
    one_step()
    bad = infos[-1]
    q.jacobi_omega = 0.5
    G.set_params(q)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    # per PCG iteration: one V-cycle, one FP64 K p (matrix-free) and ~10 vector passes of 24 B per node
    nv0, ne0 = G[0].nv, G[0].ne
    per_it = vcycle_bytes(G, 8, 4, 9) + nv0 * (6 * 8 + 2) + 4 * ne0 + 10 * 24 * nv0
    solve_ms = ms / args.steps
    line = {"metric": "plain MG-PCG solve to 1e-6 + one OC step, cantilever 64x32x32 (damped Jacobi 2+2)",
            "value": args.steps / (ms * 1e-3), "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": solve_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "cantilever 64x32x32, rho 0.4, x=0 clamped, bottom-edge load, wsff, FP64 V-cycle "
                                   "PCG (Jacobi 2+2, omega 0.5) to 1e-6, OC step (R 2, move 0.03, eta 0.5, V 0.4)",
                       "levels": G.n_grid(), "pcg_iterations": it, "rel_residual": infos[-2].rel_residual,
                       "smoother_lmax_level0": lmax0,
                       "omega_0.6": {"pcg_iterations": bad.iterations, "rel_residual": bad.rel_residual,
                                     "converged": bad.status == 0},
                       "oc_multiplier": lam.value,
                       "volume_after": float(rho_out.mean()),
                       "algorithmic_bytes_per_pcg_iteration": int(per_it),
                       "achieved_gbs_per_solve": per_it * it / (solve_ms * 1e-3) / 1e9,
                       "hbm_peak_gbs": peaks.get("hbm_gbs")},
            "clocks": clk, "gpu_launches": launches // max(args.steps, 1) * args.steps,
            "e2e": {"value": args.steps / (e2e_ms * 1e-3), "unit": "solves/s",
                    "h2d_bytes_per_step": int(rho0.nbytes + f.nbytes), "d2h_bytes_per_step": int(rho0.nbytes)}}
    if not args.no_cpu_baseline:
        import oracle as O

        t0 = time.perf_counter()
        H = O.Hierarchy(cfg["eact"], cfg["rho"], cfg["vfix"], p=3, E=1e6, nu=0.4)
        H.update_stencil()
        x, ito, rr = H.pcg(f, tol=1e-6, maxit=500, smoother=O.SMOOTH_JACOBI, npre=2, npost=2, omega=0.5)
        t_cpu = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": 1.0 / t_cpu, "unit": "solves/s", "cores": os.cpu_count() or 1,
                                "kind": "port", "sample": f"the oracle (OpenMP) stencil assembly + the same PCG solve "
                                                          f"({ito} iterations), one run, without the OC step"}
    print(json.dumps(line))
    G.close()
    ctx.close()
    return 0


def run_voxelize(args):
    """Solid voxelisation (voxelize_mesh, voxelizer/voxelize_main.cpp:344-402) of a closed
    mesh: an icosphere refined 7 times (327,680 triangles) merged with a rotated 256x128
    torus (65,536 triangles), prefer_reso 511 -> a 512^3 bit grid.  value = cube cells per
    second of device time (event pass + row pass, mesh resident); e2e = the same through
    rt_voxelize_mesh with host arrays (mesh upload, bits download); the oracle's
    restatement of the reference's CPU voxeliser is the CPU baseline."""
    import robtop_b200 as rb
    from robtop_b200 import configs

    ctx = rb.Context(0)
    sv, sf = configs.icosphere(7, (0.0, 0.0, 0.0), 1.0)
    tv, tf = configs.torus(1.6, 0.3, 256, 128, (0.0, 0.0, 0.0))  # encircles the sphere, disjoint
    v, f = configs.merge_meshes((sv, sf), (configs.rigid_transform(tv, 21), tf))
    prefer = 511
    R = rb.lib().rt_voxel_resolution(prefer)
    vf = np.ascontiguousarray(v, np.float32).reshape(-1)
    ff = np.ascontiguousarray(f, np.int32).reshape(-1)
    us = C.c_double()
    rb._capi.check(rb.lib().rt_bench_voxelize(ctx.handle, vf.ctypes.data, len(v), ff.ctypes.data, len(f), prefer,
                                              max(args.warmup, 3), C.byref(us)), ctx.handle)
    # one voxelisation takes well under a millisecond: time enough of them (about half a second)
    # for the clock sampler to see the timed region
    reps = max(args.steps, 6000)
    clocks = Clocks(gpu_id(0))
    clocks.start()
    rb._capi.check(rb.lib().rt_bench_voxelize(ctx.handle, vf.ctypes.data, len(v), ff.ctypes.data, len(f), prefer,
                                              reps, C.byref(us)), ctx.handle)
    clk = clocks.stop()
    # per-kernel split from the library's per-launch profile
    ctx.profile(True)
    ctx.profile_reset()
    rb._capi.check(rb.lib().rt_bench_voxelize(ctx.handle, vf.ctypes.data, len(v), ff.ctypes.data, len(f), prefer,
                                              args.steps, C.byref(us)), ctx.handle)
    st = {k: v_ for k, v_ in ctx.profile_stats().items() if k.startswith("vox") and v_[0]}
    ctx.profile(False)
    # end to end with host arrays
    import time as _t
    t0 = _t.perf_counter()
    for _ in range(args.steps):
        bits, R2, box = rb.voxelize_mesh(ctx, v, f, prefer)
    e2e_s = (_t.perf_counter() - t0) / args.steps
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    rows_n, rows_ms = st.get("vox_rows", (1, 0.0))
    row_bytes = 2 * R ** 3 // 8  # each row pass reads and writes the R^3-bit grid once
    ach = row_bytes / (rows_ms / max(rows_n, 1) * 1e-3) / 1e9 if rows_ms else None
    hbm = peaks.get("hbm_gbs", 6650.0)
    ev_n, ev_ms = st.get("vox_events", (1, 0.0))
    line = {"metric": "solid mesh voxelisation, 393,216-triangle closed mesh into a 512^3 bit grid",
            "value": R ** 3 / (us.value * 1e-6), "unit": "cells/s", "n_gpus": 1, "steps": reps,
            "warmup": max(args.warmup, 3), "ms_per_step": us.value * 1e-3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+u32", "data": "synthetic",
            "config": {"workload": "icosphere(7) + rotated torus(256x128), prefer_reso 511, R 512",
                       "triangles": int(len(f)), "solid_cells": int(_popcount_bits(bits)),
                       "event_pass_ms": ev_ms / max(ev_n, 1), "row_pass_ms": rows_ms / max(rows_n, 1),
                       "triangles_per_s": len(f) / (us.value * 1e-6)},
            "roofline": {"kernel": "vox_rows", "bound": "hbm", "achieved": round(ach, 1) if ach else None,
                         "peak": hbm, "unit": "GB/s", "frac": round(ach / hbm, 4) if ach else None, "traffic": None,
                         "algorithmic_bytes": row_bytes},
            "clocks": clk, "gpu_launches": 2 * reps,
            "e2e": {"value": R ** 3 / e2e_s, "unit": "cells/s", "h2d_bytes_per_step": int(vf.nbytes + ff.nbytes),
                    "d2h_bytes_per_step": int(bits.nbytes)}}
    if not args.no_cpu_baseline:
        import oracle as O

        t0 = _t.perf_counter()
        Ro, bmin, bmax, unit = O.voxel_box(v, prefer)
        ob = O.voxelize_solid(v, f, Ro, bmin, unit)
        t_cpu = _t.perf_counter() - t0
        line["cpu_baseline"] = {"value": R ** 3 / t_cpu, "unit": "cells/s", "cores": 1, "kind": "port",
                                "sample": "the oracle's single-threaded restatement of the reference's CPU solid "
                                          "voxeliser on the same mesh and cube, one run"}
        line["config"]["bit_exact_vs_oracle"] = bool(np.array_equal(ob, bits))
    print(json.dumps(line))
    ctx.close()
    return 0


def _popcount_bits(bits):
    return int(np.unpackbits(np.ascontiguousarray(bits, np.uint32).view(np.uint8)).sum())


def run_kernel(args):
    """Repeat one hot operator of the path on the bench workload (short command for
    ncu captures): fine_residual = rt_update_residual(level 0), fine_jacobi =
    rt_smooth(level 0, Jacobi), st_residual = rt_update_residual(level 1)."""
    import robtop_b200 as rb
    from robtop_b200 import configs

    ctx = rb.Context(0)
    dims = tuple(int(v) for v in args.size.split("x")) if args.size else None
    cfg, G = build_problem(rb, configs, ctx, rb.FP64, dims)
    G.update_stencil()
    u = np.random.default_rng(0).standard_normal(3 * G[0].nv) * np.tile(G[0].getVact(), 3)
    G[0].setDisplacement(u)
    G[0].setForce(u[::-1].copy())
    if args.kernel in ("fine_cheby_f32", "fine_residual_f64", "fine_applyK_f64", "fine_residual_f32"):
        # one finest-level kernel at the autotuned (or a given) launch shape, timed by the library (CUDA events)
        prec = rb.FP32 if args.kernel.endswith("f32") else rb.FP64
        mode = {"fine_residual": 0, "fine_applyK": 1, "fine_cheby": 3}[args.kernel.rsplit("_", 1)[0]]
        if args.shape:
            variant, ty, zc = (int(v) for v in args.shape.split(","))
            rb._capi.check(rb.lib().rt_set_tuning(G.handle, prec, mode, variant, ty, zc), ctx.handle)
            names = ["residual", "applyK", "jacobi", "chebyshev"]
            shapes = {f"{names[mode]}_{'f32' if prec == rb.FP32 else 'f64'}":
                      {"variant": ["smem_tile", "register_march", "register_march_prefetch", "smem_tile_pipelined",
                                   "smem_tile_pairs_f32", "sum_factorised", "smem_tile_pipelined_tma",
                                   "smem_tile_pipelined_tma_x31"][variant],
                       "rows": ty,
                       "zchunk": zc}}
        else:
            shapes = G.autotune()
        us = C.c_double()
        rb._capi.check(rb.lib().rt_bench_fine_kernel(G.handle, prec, mode, args.warmup, C.byref(us)), ctx.handle)
        rb._capi.check(rb.lib().rt_bench_fine_kernel(G.handle, prec, mode, args.steps, C.byref(us)), ctx.handle)
        key = {0: "residual", 1: "applyK", 3: "chebyshev"}[mode] + ("_f32" if prec == rb.FP32 else "_f64")
        print(json.dumps({"kernel": args.kernel, "us_per_call": us.value, "nodes": G[0].nv, "shape": shapes[key]}))
        G.close()
        ctx.close()
        return 0
    if args.kernel.startswith("st_") and args.kernel != "st_residual":
        # one stencil-level kernel on level --level, timed by the library (CUDA events)
        base, form = args.kernel.rsplit("_", 1)
        prec = rb.FP64 if form == "f64" else rb.FP32
        mode = {"st_residual": 0, "st_jacobi": 2, "st_cheby": 3}[base]
        if form == "bf16":
            p = G.params
            p.coarse_bf16 = 1
            G.set_params(p)
            G.update_stencil()
        variant = None
        if args.shape and prec == rb.FP32:  # 0 lane-split, 1 bulk-copy
            variant = int(args.shape)
            rb._capi.check(rb.lib().rt_set_level_kernel(G.handle, 1 if form == "bf16" else 0, variant), ctx.handle)
        us = C.c_double()
        rb._capi.check(rb.lib().rt_bench_level_kernel(G.handle, args.level, prec, mode, args.warmup, C.byref(us)),
                       ctx.handle)
        rb._capi.check(rb.lib().rt_bench_level_kernel(G.handle, args.level, prec, mode, args.steps, C.byref(us)),
                       ctx.handle)
        print(json.dumps({"kernel": args.kernel, "level": args.level, "variant": variant, "us_per_call": us.value,
                          "nodes": G[args.level].nv, "stencil_bytes": G[args.level].nv * 243 * {"f64": 8, "f32": 4,
                                                                                               "bf16": 2}[form]}))
        G.close()
        ctx.close()
        return 0
    ops = {"fine_residual": lambda: G[0].update_residual(),
           "fine_jacobi": lambda: G[0].smooth(rb.SMOOTH_JACOBI, 1, 0.6),
           "st_residual": lambda: G[1].update_residual()}
    op = ops[args.kernel]
    for _ in range(args.warmup):
        op()
    ctx.sync()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        op()
    ctx.sync()
    dt = (time.perf_counter() - t0) / args.steps
    print(json.dumps({"kernel": args.kernel, "us_per_call": dt * 1e6, "nodes": G[0].nv}))
    G.close()
    ctx.close()
    return 0


def run_batched(args):
    """Batched solves: 12 cantilever instances with per-axis sizes drawn from {48..160} (seed 1),
    smoothed random densities (seeds 2+i), x=0 clamped with the bottom-edge tip load, plus 8
    right-hand sides (random top-face loads) on one 256x256x128 worst-case box, all 20 MG-PCG
    solves (the mixed form: FP32 Chebyshev V-cycles in FP64 CG, to 1e-6 from zero) in ONE graph launch
    (rt_pcg_batch), timed against the same 20 solves one after another (rt_pcg)."""
    import torch

    import robtop_b200 as rb
    from robtop_b200 import configs

    ws_, rank, lrank = dist_env()
    ctx = make_ctx(rb, lrank)
    stream = torch.cuda.ExternalStream(ctx_stream_handle(ctx))

    def params(mode):
        return rb.default_params(mode=mode, youngs_modulus=1e6, poisson_ratio=0.4, power_penalty=3.0, min_rho=1e-3,
                                 precision=rb.FP32, smoother=rb.SMOOTH_CHEBY, pre_sweeps=4, post_sweeps=4)

    grids, insts, rhs = [], [], []
    sizes = configs.batch_instances(12, 48, 160, seed=1)
    for i, (nx, ny, nz) in enumerate(sizes):
        cfg = configs.cantilever(nx, ny, nz)
        cfg["rho"] = configs.smoothed_density(cfg["eact"].shape, 2 + i)
        G = rb.HierarchyGrid(ctx, params(cfg["mode"]))
        G.genFromBox(cfg["eact"])
        apply_form(rb, G, FORMS_BATCH)
        G[0].setRho(cfg["rho"].ravel())
        G.set_support(cfg["vfix"])
        G.update_stencil()
        G.autotune(reps=2)
        grids.append(G)
        insts.append(G)
        rhs.append(cfg["fload"].ravel())
    big_cfg = configs.worst_case_box(256, 256, 128, seed=0)
    big = rb.HierarchyGrid(ctx, params(big_cfg["mode"]))
    big.genFromBox(big_cfg["eact"])
    apply_form(rb, big, FORMS_BATCH)
    big[0].setRho(big_cfg["rho"].ravel())
    big.set_support(big_cfg["vfix"])
    big.update_stencil()
    big.autotune(reps=2)
    grids.append(big)
    rng = np.random.default_rng(7)
    for k in range(8):
        w = big.workspace()
        f = np.zeros(3 * big[0].nv)
        for c in range(3):
            f[c * big[0].nv + big_cfg["load_nodes"]] = rng.standard_normal(big_cfg["load_nodes"].size)
        insts.append(w)
        rhs.append(f)
    for g, f in zip(insts, rhs):
        g[0].setForce(f)
    zeros = torch.zeros(3 * max(g[0].nv for g in insts), dtype=torch.float64, device="cuda")

    def reset():
        for g in insts:
            rb._capi.check(rb.lib().rt_put_dev(g.handle, rb._capi.FIELD_U, 0, C.c_void_p(zeros.data_ptr())),
                           ctx.handle)

    def timed(fn):
        ctx.sync()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    maxit = args.maxit
    ncant = len(sizes)

    def batch_step(sub=None):
        reset()
        return rb.pcg_batch(insts[:sub] if sub else insts, WORKLOAD["tol"], maxit)

    def seq_step(sub=None):
        reset()
        return [g.pcg(WORKLOAD["tol"], maxit) for g in (insts[:sub] if sub else insts)]

    # one warm-up pass of each (graph capture and instantiation happen in the first); a step of
    # the 256x256x128 block takes about two minutes, so the default three are not repeated here
    warm = 1
    for _ in range(warm):
        batch_step()
        seq_step()
        batch_step(ncant)
        seq_step(ncant)
    clocks = Clocks(gpu_id(lrank))
    clocks.start()
    l0 = ctx.launches()
    tb, infos_b = 0.0, None
    for _ in range(args.steps):
        ms, infos_b = timed(batch_step)
        tb += ms
    launches = ctx.launches() - l0
    clk = clocks.stop()
    ts, infos_s = 0.0, None
    for _ in range(args.steps):
        ms, infos_s = timed(seq_step)
        ts += ms
    # the 12 cantilevers alone (small instances, where concurrent branches can overlap)
    tcb = tcs = 0.0
    for _ in range(args.steps):
        tcb += timed(lambda: batch_step(ncant))[0]
        tcs += timed(lambda: seq_step(ncant))[0]
    n = len(insts)
    line = {"metric": "batched MG-PCG solves (12 cantilevers U{48..160}^3 + 8-RHS block on 256x256x128) to rel. "
                      "residual 1e-6 in one graph launch",
            "value": n * args.steps / (tb * 1e-3), "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
            "warmup": warm, "ms_per_step": tb / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
            "config": {"workload": "12 cantilevers (sizes " + ";".join("x".join(map(str, s)) for s in sizes) +
                                   ") + 8 top-face loads on the 256x256x128 worst-case box",
                       "form": form_text(FORMS_BATCH) + " in FP64 flexible CG, per-step reset of u on the device",
                       "sequential_ms_per_step": ts / args.steps, "batch_speedup": ts / tb,
                       "cantilevers_only": {"batch_ms": tcb / args.steps, "sequential_ms": tcs / args.steps,
                                            "batch_speedup": tcs / tcb},
                       "maxit": maxit, "precision_fallbacks": sum(rb.lib().rt_hier_precision_fallbacks(g.handle)
                                                                  for g in grids),
                       "iterations": [i.iterations for i in infos_b],
                       "iterations_sequential": [i.iterations for i in infos_s],
                       "max_rel_residual": max(i.rel_residual for i in infos_b),
                       "all_converged": all(i.status == 0 for i in infos_b)},
            "clocks": clk, "gpu_launches": launches}
    if rank == 0:
        print(json.dumps(line))
    for g in grids:
        g.close()
    ctx.close()
    return 0


def run_learned(args):
    """Learned preconditioner: (density, residual, MG-error) samples harvested from 128^3 worst-case
    boxes with random densities (k = 2, 6, 14 plain MG-PCG iterations each), the U-Net trained by
    the library's kernels on random 33^3 crops of them, then used inside flexible MG-PCG on the
    256x256x128 box (z = Vcycle(r) + N(rho, r), plain V-cycle as fallback) against the same PCG
    without it.  Step = one solve of a top-face load to 1e-6 from zero, timed per form."""
    import torch

    import robtop_b200 as rb
    from robtop_b200 import configs, learned

    ws_, rank, lrank = dist_env()
    ctx = make_ctx(rb, lrank)
    stream = torch.cuda.ExternalStream(ctx_stream_handle(ctx))

    def grid(cfg):
        p = rb.default_params(mode=cfg["mode"], youngs_modulus=1e6, poisson_ratio=0.4, power_penalty=3.0,
                              min_rho=1e-3, precision=rb.FP32, smoother=rb.SMOOTH_CHEBY, pre_sweeps=4, post_sweeps=4)
        G = rb.HierarchyGrid(ctx, p)
        G.genFromBox(cfg["eact"])
        G[0].setRho(cfg["rho"].ravel())
        G.set_support(cfg["vfix"])
        G.update_stencil()
        return G

    n_train, iters, crop, n_crops = 8, (2, 6, 14), (33, 33, 33), 24
    rng = np.random.default_rng(11)
    t0 = time.perf_counter()
    samples, hnet = [], None
    for i in range(n_train):
        G = grid(configs.worst_case_box(128, 128, 128, seed=100 + i))
        if hnet is None:
            hnet = learned.UNet.for_grid(G, seed=0)
        for k in iters:
            inp, tgt = learned.harvest(G, hnet, k, seed=1000 * i + k)
            samples += learned.crops(inp, tgt, hnet.dims, crop, n_crops, rng)
        G.close()
    t_harvest = time.perf_counter() - t0
    net = learned.UNet(ctx, *crop, seed=1)
    net.output_scale = hnet.output_scale
    hnet.close()
    t0 = time.perf_counter()
    losses = learned.train(net, samples, steps=1200, batch=8, lr=1e-3, seed=0)
    t_train = time.perf_counter() - t0
    del samples
    torch.cuda.empty_cache()
    cfg = configs.worst_case_box(256, 256, 128, seed=0)
    G = grid(cfg)
    G.autotune(reps=2)
    enet = learned.UNet.for_grid(G)
    learned.transfer(net, enet)
    f = np.zeros(3 * G[0].nv)
    for c in range(3):
        f[c * G[0].nv + cfg["load_nodes"]] = np.random.default_rng(5).standard_normal(cfg["load_nodes"].size)
    G[0].setForce(f)
    zeros = torch.zeros(3 * G[0].nv, dtype=torch.float64, device="cuda")

    def solve():
        rb._capi.check(rb.lib().rt_put_dev(G.handle, rb._capi.FIELD_U, 0, C.c_void_p(zeros.data_ptr())), ctx.handle)
        ctx.sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        info = G.pcg(WORKLOAD["tol"], 1000)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), info

    res = {}
    for name, net_ in (("plain", None), ("learned", enet)):
        learned.attach(G, net_, fallback_ratio=1.0)
        for _ in range(max(args.warmup, 1)):
            solve()
        ms = [solve() for _ in range(args.steps)]
        res[name] = (sum(m for m, _ in ms) / len(ms), ms[-1][1])
    learned.attach(G, None)
    pl_ms, pl = res["plain"]
    ln_ms, ln = res["learned"]
    line = {"metric": "learned+mixed vs mixed MG-PCG, time to rel. residual 1e-6 on 256x256x128",
            "value": 1e3 / ln_ms, "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
            "warmup": max(args.warmup, 1), "ms_per_step": ln_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f32+bf16", "data": "synthetic",
            "config": {"workload": "worst-case box 256x256x128 (seed 0), random top-face load; U-Net trained on "
                                   f"{n_train * len(iters) * n_crops} crops {crop} of {n_train * len(iters)} samples "
                                   "harvested from 128^3 boxes (seeds 100-107)",
                       "plain_ms_per_solve": pl_ms, "learned_over_plain_speed": pl_ms / ln_ms,
                       "plain_iterations": pl.iterations, "learned_iterations": ln.iterations,
                       "learned_rel_residual": ln.rel_residual, "loss_first": float(np.mean(losses[:10])),
                       "loss_last": float(np.mean(losses[-50:])), "harvest_s": t_harvest, "train_s": t_train}}
    if rank == 0:
        print(json.dumps(line))
    enet.close()
    net.close()
    G.close()
    ctx.close()
    return 0


def run_c5(args):
    """Worst-case optimisation on the 511x256x256 arch (solid box minus a radius-96 tunnel along x,
    four 16x16 support pads at the bottom corners, top face loadable with normal-constrained loads,
    wscf; rho = 0.4 to start, volume target 0.4, filter radius 2, move limit 0.06, damping 0.5,
    p = 3).  A step is one OC iteration (stencil update, worst-case Lanczos k = 16 with MG-PCG inner
    solves to 1e-6, sensitivity, filter, OC update) in the mixed form.  After the timed steps the
    worst-case solve of the current design is timed in the mixed and the plain FP64 form and their
    eigenvalues compared."""
    import torch

    import robtop_b200 as rb
    from robtop_b200 import configs

    ws_, rank, lrank = dist_env()
    ctx = make_ctx(rb, lrank)
    stream = torch.cuda.ExternalStream(ctx_stream_handle(ctx))
    t0 = time.perf_counter()
    cfg = configs.arch(511, 256, 256)
    p = rb.default_params(mode=cfg["mode"], youngs_modulus=1e6, poisson_ratio=0.4, power_penalty=3.0, min_rho=1e-3,
                          volume_ratio=0.4, design_step=0.06, damp_ratio=0.5, filter_radius=2.0,
                          precision=rb.FP32, smoother=rb.SMOOTH_CHEBY, pre_sweeps=4, post_sweeps=4)
    G = rb.HierarchyGrid(ctx, p)
    G.genFromBox(cfg["eact"])
    apply_form(rb, G, FORMS_C5["mixed"])
    G[0].setRho(cfg["rho"].ravel())
    G.set_support(cfg["vfix"])
    G.set_load_nodes(cfg["load_nodes"], cfg["normals"])
    G.update_stencil()
    G.autotune(reps=2)
    t_setup = time.perf_counter() - t0

    def oc_step(seed):
        lam = C.c_double()
        rb._capi.check(rb.lib().rt_oc_iteration(G.handle, rb.WORST_LANCZOS, WORKLOAD["k"], WORKLOAD["tol"], seed,
                                                0.4, C.byref(lam)), ctx.handle)
        return lam.value

    def timed(fn):
        ctx.sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    for w in range(args.warmup):
        oc_step(10 + w)
    clocks = Clocks(gpu_id(lrank))
    clocks.start()
    l0 = ctx.launches()
    ms_oc, lams = 0.0, []
    for s_ in range(args.steps):
        ms, lam = timed(lambda: oc_step(100 + s_))
        ms_oc += ms
        lams.append(lam)
    launches = ctx.launches() - l0
    clk = clocks.stop()
    fb0 = int(rb.lib().rt_hier_precision_fallbacks(G.handle))
    forms = {}
    for name in ("mixed", "plain", "fp64_same_cycle"):
        apply_form(rb, G, FORMS_C5[name])
        ms, (lam, info) = timed(lambda: step(rb, G, 7))
        forms[name] = (ms, lam, info.inner_iterations)
    m_ms, m_lam, m_it = forms["mixed"]
    p_ms, p_lam, p_it = forms["plain"]
    s_ms, s_lam, s_it = forms["fp64_same_cycle"]
    line = {"metric": "worst-case optimisation on the 511x256x256 arch: OC iterations (stencil update, Lanczos k=16 "
                      "worst-case solve to 1e-6, sensitivity, filter, OC update)",
            "value": args.steps / (ms_oc * 1e-3), "unit": "OC iterations/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_oc / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
            "config": {"workload": "arch 511x256x256 (tunnel radius 96, 16x16 pads), wscf, V 0.4, R 2, move 0.06, "
                                   "eta 0.5, p 3, rho0 0.4",
                       "worst_case_lambda_per_step": lams, "setup_s": t_setup,
                       "form_mixed": form_text(FORMS_C5["mixed"]),
                       "worst_case_solve_ms_mixed": m_ms, "worst_case_solve_ms_plain_fp64": p_ms,
                       "speedup_mixed_vs_plain": p_ms / m_ms,
                       "worst_case_solve_ms_fp64_same_cycle": s_ms, "speedup_mixed_vs_fp64_same_cycle": s_ms / m_ms,
                       "inner_iterations_fp64_same_cycle": s_it,
                       "lambda_rel_diff_fp64_same_cycle": abs(s_lam - p_lam) / abs(p_lam),
                       "lambda_mixed": m_lam, "lambda_plain": p_lam,
                       "lambda_rel_diff": abs(m_lam - p_lam) / abs(p_lam),
                       "inner_iterations_mixed": m_it, "inner_iterations_plain": p_it,
                       "precision_fallbacks": int(rb.lib().rt_hier_precision_fallbacks(G.handle)),
                       "precision_fallbacks_in_timed_steps": fb0},
            "clocks": clk, "gpu_launches": launches}
    if rank == 0:
        print(json.dumps(line))
    G.close()
    ctx.close()
    return 0


# the default workload: the worst-case solve on the 511x256x256 arch, in the learned+mixed form
ARCH = dict(dims=(511, 256, 256), k=16, tol=1e-6, design_iters=4, harvest_k=(1, 4, 12), crop=(33, 33, 33),
            n_crops=32, train_steps=200, train_batch=8, vgoal=0.4)
METRIC_ARCH = ("worst-case solve on the 511x256x256 arch (stencil assembly + Lanczos k=16 with MG-PCG inner solves "
               "to rel. residual 1e-6 + the worst-case displacement solve), learned+mixed form")


def arch_config(configs, dims):
    """The arch of the given size; the tunnel radius (96 of 256) and the support pads (16 of 256)
    scale with ny for the reduced sizes used by quick runs and the CPU baseline's sample."""
    nx, ny, nz = dims
    return configs.arch(nx, ny, nz, tunnel=int(round(96 * ny / 256)), pad=max(2, int(round(16 * ny / 256))))


def arch_cpu_sample(threads, dims_full, plain_inner_its, solves, sample_dims=(127, 64, 64)):
    """The oracle (plain FP64 SGS V-cycle PCG, OpenMP) on a reduced arch with the same shape: stencil
    assembly plus one inner solve to 1e-6 of a top-face load.  Extrapolated to the full arch by node
    count, to ``solves`` inner solves of ``plain_inner_its / solves`` iterations each (the plain
    method's own iteration count on the full arch, measured on the GPU) plus one assembly."""
    import oracle as O
    from robtop_b200 import configs

    os.environ["OMP_NUM_THREADS"] = str(threads)
    cfg = arch_config(configs, sample_dims)
    ws = cfg["vfix"] is not None
    t0 = time.perf_counter()
    H = O.Hierarchy(cfg["eact"], cfg["rho"], cfg["vfix"], p=3, E=1e6, nu=0.4)
    H.update_stencil()
    t_st = time.perf_counter() - t0
    nv = H.arrs[0]["u"].size // 3
    b = np.zeros(3 * nv)
    b[2 * nv + cfg["load_nodes"]] = 1.0 / np.sqrt(cfg["load_nodes"].size)
    t0 = time.perf_counter()
    x, it, rr = H.pcg(b, tol=1e-6, maxit=200, smoother=O.SMOOTH_SGS)
    t_pcg = time.perf_counter() - t0
    t_it = t_pcg / max(it, 1)
    nx, ny, nz = dims_full
    scale = (nx + 1) * (ny + 1) * (nz + 1) / nv
    total = scale * (t_st + t_it * plain_inner_its)
    return {"sampled_wall_s": t_st + t_pcg, "sample_dims": list(sample_dims), "sample_nodes": int(nv),
            "sample_assembly_s": t_st, "sample_pcg_iterations": int(it), "sample_s_per_iteration": t_it,
            "node_scale_factor": scale, "extrapolated_s_per_step": total, "solves": solves,
            "plain_inner_iterations_full": int(plain_inner_its), "ws": ws}


def arch_design_and_network(rb, learned, ctx, G, design_iters, seed0=10, first_iter=0, on_iter=None):
    """``design_iters`` OC iterations of the current form (worst-case Lanczos k = 16, sensitivity,
    filter, OC update); after each, (density, residual, MG-error) samples harvested from the solver
    are cropped; then the U-Net is trained on the crops by the library's kernels and its weights are
    moved to a network over the full node box.  on_iter(i, lam) is called after iteration i."""
    import torch

    hnet = learned.UNet.for_grid(G, seed=0)
    rng = np.random.default_rng(11)
    samples, t_harvest = [], 0.0
    lam_c = C.c_double()
    for it in range(design_iters):
        rb._capi.check(rb.lib().rt_oc_iteration(G.handle, rb.WORST_LANCZOS, ARCH["k"], ARCH["tol"], seed0 + it,
                                                ARCH["vgoal"], C.byref(lam_c)), ctx.handle)
        if on_iter:
            on_iter(first_iter + it, lam_c.value)
        G.update_stencil()
        t0 = time.perf_counter()
        for kk in ARCH["harvest_k"]:
            inp, tgt = learned.harvest(G, hnet, kk, seed=1000 * it + kk)
            samples += learned.crops(inp, tgt, hnet.dims, ARCH["crop"], ARCH["n_crops"] // len(ARCH["harvest_k"]), rng)
            del inp, tgt
        t_harvest += time.perf_counter() - t0
    torch.cuda.empty_cache()
    net = learned.UNet(ctx, *ARCH["crop"], seed=1)
    net.output_scale = hnet.output_scale
    t0 = time.perf_counter()
    losses = learned.train(net, samples, steps=ARCH["train_steps"], batch=ARCH["train_batch"], lr=1e-3, seed=0)
    t_train = time.perf_counter() - t0
    learned.transfer(net, hnet)
    net.close()
    n = len(samples)
    del samples
    torch.cuda.empty_cache()
    return hnet, {"losses": losses, "harvest_s": t_harvest, "train_s": t_train, "samples": n}


def arch_attach_network(learned, G, cfg, hnet):
    """Attach the network with the cost-aware fallback ratio: the plain V-cycle PCG's rate and
    iteration time on this design (a unit top-face load, the second of two solves) against the
    network's time."""
    nv = G[0].nv
    f = np.zeros(3 * nv)
    f[2 * nv + cfg["load_nodes"]] = 1.0 / np.sqrt(cfg["load_nodes"].size)
    learned.attach(G, None)
    G[0].setForce(f)
    for _ in range(2):
        G[0].reset_displacement()
        cal = G.pcg(ARCH["tol"], 500)
    t_net = learned.forward_seconds(hnet)
    ratio = learned.cost_aware_ratio(cal.iterations, cal.rel_residual, cal.seconds, t_net)
    learned.attach(G, hnet, fallback_ratio=ratio)
    return cal, t_net, ratio


def run_c5_oc40(args):
    """The 40-iteration worst-case optimisation of the 511x256x256 arch (volume 0.4, filter radius 2,
    move 0.06, damping 0.5, p = 3): iterations 1-4 in the mixed form while training samples are
    harvested, the U-Net trained, iterations 5-40 in the learned+mixed form.  Every 10 iterations
    the design's worst-case eigenvalue and the compliance of a fixed unit top-face load are
    recomputed with the plain FP64 method and compared with the learned+mixed values on the same
    design.  Prints one JSON line with the per-iteration eigenvalues and the checks."""
    import torch

    import robtop_b200 as rb
    from robtop_b200 import configs, learned

    ws_, rank, lrank = dist_env()
    dims = tuple(int(v) for v in args.size.split("x")) if args.size else ARCH["dims"]
    n_iter = args.oc_iters
    ctx = make_ctx(rb, lrank)
    stream = torch.cuda.ExternalStream(ctx_stream_handle(ctx))
    cfg = arch_config(configs, dims)
    p = rb.default_params(mode=cfg["mode"], youngs_modulus=1e6, poisson_ratio=0.4, power_penalty=3.0, min_rho=1e-3,
                          volume_ratio=ARCH["vgoal"], design_step=0.06, damp_ratio=0.5, filter_radius=2.0)
    G = rb.HierarchyGrid(ctx, p)
    G.genFromBox(cfg["eact"])
    apply_form(rb, G, FORMS_C5["mixed"])
    G[0].setRho(cfg["rho"].ravel())
    G.set_support(cfg["vfix"])
    G.set_load_nodes(cfg["load_nodes"], cfg["normals"])
    G.update_stencil()
    G.autotune(reps=2)
    nv = G[0].nv
    fload = np.zeros(3 * nv)
    fload[2 * nv + cfg["load_nodes"]] = 1.0 / np.sqrt(cfg["load_nodes"].size)
    lams, ms_iter, checks = [], [], []

    def timed(fn):
        ctx.sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    def compliance():
        G[0].setForce(fload)
        G[0].reset_displacement()
        info = G.pcg(ARCH["tol"], 2000)
        return float(fload @ G[0].getDisplacement()), info.iterations

    applied_before = [0]  # corrections counted before each re-attach (attach resets the count)

    def check(i):
        # the current design in both forms (the stencil of the design before this OC update)
        applied_before[0] += learned.stats(G)[0]
        G.update_stencil()
        lam_l, _ = G.worst_case(rb.WORST_LANCZOS, ARCH["k"], ARCH["tol"], seed=7)
        c_l, it_l = compliance()
        net_saved = G_net[0]
        learned.attach(G, None)
        apply_form(rb, G, FORMS_C5["plain"])
        G.update_stencil()
        ms_p, (lam_p, info_p) = timed(lambda: G.worst_case(rb.WORST_LANCZOS, ARCH["k"], ARCH["tol"], seed=7))
        c_p, it_p = compliance()
        apply_form(rb, G, FORMS_C5["mixed"])
        G.update_stencil()
        if net_saved is not None:
            learned.attach(G, net_saved, fallback_ratio=G_net[1])
        checks.append({"iteration": i, "lambda": lam_l, "lambda_plain_fp64": lam_p,
                       "lambda_rel_diff": abs(lam_l - lam_p) / abs(lam_p), "compliance": c_l,
                       "compliance_plain_fp64": c_p, "compliance_rel_diff": abs(c_l - c_p) / abs(c_p),
                       "pcg_iterations": it_l, "pcg_iterations_plain_fp64": it_p, "plain_worst_case_ms": ms_p})

    G_net = [None, 1.0]
    t0 = time.perf_counter()
    n_design = min(ARCH["design_iters"], n_iter)
    hnet, tr = arch_design_and_network(rb, learned, ctx, G, n_design, seed0=10,
                                       on_iter=lambda i, lam: lams.append(lam))
    cal, t_net, ratio = arch_attach_network(learned, G, cfg, hnet)
    G_net[0], G_net[1] = hnet, ratio
    lam_c = C.c_double()
    stopped_early = False
    for it in range(n_design, n_iter):
        if (it + 1) % 10 == 0 or it + 1 == n_iter:
            check(it + 1)
            c = checks[-1]
            print(f"check at iteration {it + 1}: lambda rel diff {c['lambda_rel_diff']:.2e}, compliance rel diff "
                  f"{c['compliance_rel_diff']:.2e}, {c['pcg_iterations']} / {c['pcg_iterations_plain_fp64']} PCG "
                  "iterations", file=sys.stderr, flush=True)
        ms, _ = timed(lambda: rb._capi.check(rb.lib().rt_oc_iteration(G.handle, rb.WORST_LANCZOS, ARCH["k"],
                                                                        ARCH["tol"], 10 + it, ARCH["vgoal"],
                                                                        C.byref(lam_c)), ctx.handle))
        ms_iter.append(ms)
        lams.append(lam_c.value)
        print(f"OC iteration {it + 1}: {ms:.0f} ms, lambda {lam_c.value:.6e}", file=sys.stderr, flush=True)
        # the design sharpens towards 0/1 densities (nine decades of stiffness): later iterations
        # need many more PCG iterations; a time budget ends the run with the iterations done
        if args.time_budget > 0 and time.perf_counter() - t0 > args.time_budget and it + 1 < n_iter:
            stopped_early = True
            if not checks or checks[-1]["iteration"] != it + 1:
                check(it + 1)
            break
    wall = time.perf_counter() - t0
    applied, off = learned.stats(G)
    applied += applied_before[0]
    rho = G[0].getRho()
    eact = cfg["eact"].ravel().astype(bool)
    line = {"metric": "40-iteration worst-case optimisation of the 511x256x256 arch, learned+mixed form, checked "
                      "against the plain FP64 method every 10 iterations",
            "value": len(ms_iter) / (sum(ms_iter) * 1e-3) if ms_iter else None, "unit": "OC iterations/s",
            "n_gpus": 1, "steps": len(ms_iter), "warmup": n_design, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+f32+bf16", "data": "synthetic",
            "config": {"workload": f"arch {'x'.join(map(str, dims))}, {n_iter} OC iterations (the first {n_design} "
                                   "without the network, harvesting its training samples)",
                       "lambda_per_iteration": lams, "ms_per_iteration": ms_iter, "checks": checks,
                       "max_lambda_rel_diff": max((c["lambda_rel_diff"] for c in checks), default=None),
                       "max_compliance_rel_diff": max((c["compliance_rel_diff"] for c in checks), default=None),
                       "volume_fraction": float(rho[eact].mean()), "learned_corrections": applied,
                       "learned_judged_off_at_end": off, "fallback_ratio": ratio, "network_ms": t_net * 1e3,
                       "wall_s": wall, "iterations_completed": n_design + len(ms_iter),
                       "stopped_by_time_budget": stopped_early}}
    if rank == 0:
        print(json.dumps(line))
    hnet.close()
    G.close()
    ctx.close()
    return 0


def run_arch(args):
    """Default workload.  A step is one worst-case solve of the current design of the 511x256x256
    arch (solid box minus a radius-96 tunnel along x, four 16x16 support pads at the bottom corners,
    top face loadable with normal-constrained loads, wscf, p = 3): Galerkin stencil assembly, the
    largest eigenvalue of the load-space compliance operator by Lanczos (k = 16) whose inner MG-PCG
    solves run to relative residual 1e-6, and the worst-case displacement solve.

    Set-up (untimed): ``design_iters`` OC iterations (volume 0.4, filter radius 2, move 0.06,
    damping 0.5) give the design; after each, (density, residual, MG-error) samples are harvested
    from the solver and cropped; the U-Net is trained on the crops by the library's forward and
    backward kernels and attached to the full-size hierarchy with the cost-aware fallback ratio.
    ``value`` is the learned+mixed form (FP32 V-cycles inside FP64 flexible CG plus the network's
    correction while it pays); the mixed form without the network and the plain FP64 method are
    timed on the same design after the timed steps, with their eigenvalues."""
    import torch

    ws, rank, lrank = dist_env()
    dist = init_replicas(ws, lrank)

    import robtop_b200 as rb
    from robtop_b200 import configs, learned

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    dims = tuple(int(v) for v in args.size.split("x")) if args.size else ARCH["dims"]
    ctx = make_ctx(rb, lrank)
    stream = torch.cuda.ExternalStream(ctx_stream_handle(ctx))
    t_setup0 = time.perf_counter()
    cfg = arch_config(configs, dims)
    p = rb.default_params(mode=cfg["mode"], youngs_modulus=1e6, poisson_ratio=0.4, power_penalty=3.0, min_rho=1e-3,
                          volume_ratio=ARCH["vgoal"], design_step=0.06, damp_ratio=0.5, filter_radius=2.0)
    G = rb.HierarchyGrid(ctx, p)
    G.genFromBox(cfg["eact"])
    apply_form(rb, G, FORMS_C5["mixed"])
    G[0].setRho(cfg["rho"].ravel())
    G.set_support(cfg["vfix"])
    G.set_load_nodes(cfg["load_nodes"], cfg["normals"])
    G.update_stencil()
    tuning = G.autotune(reps=2) if args.tiles == "autotune" else G.set_tiles(*map(int, args.tiles.split(",")))
    nv = G[0].nv

    # design iterations, harvesting training samples from the solver after each, then training
    hnet, tr = arch_design_and_network(rb, learned, ctx, G, ARCH["design_iters"], seed0=10)
    cal, t_net, ratio = arch_attach_network(learned, G, cfg, hnet)
    losses, t_harvest, t_train, n_samples = tr["losses"], tr["harvest_s"], tr["train_s"], tr["samples"]
    t_setup = time.perf_counter() - t_setup0
    rho_design = G[0].getRho()

    warm = max(args.warmup, 3)
    for w in range(warm):
        step(rb, G, 10 + w)
    if dist:
        dist.barrier()
    applied0, _ = learned.stats(G)
    clocks = Clocks(gpu_id(lrank))
    clocks.start()
    torch.cuda.nvtx.range_push("timed_steps")  # the range a launch-list capture selects (ncu --nvtx)
    ms, lams, infos, nlaunch = time_steps(rb, ctx, G, args.steps)
    torch.cuda.nvtx.range_pop()
    applied1, judged_off = learned.stats(G)
    # end to end through the public API with host buffers: H2D of the design density, the solve,
    # D2H of the worst-case load field, every step
    n_e2e = min(args.steps, 5)
    e2e_ms, h2d, d2h = e2e_steps(rb, ctx, G, {"rho": rho_design}, n_e2e)
    clk = clocks.stop()
    ms, e2e_ms = max_over_ranks(dist, [ms, e2e_ms])

    # the same design in the mixed form without the network and in the plain FP64 method
    def timed(fn):
        ctx.sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), out

    learned.attach(G, None)
    forms = {}
    for name in ("mixed", "plain"):
        apply_form(rb, G, FORMS_C5[name])
        ms_f, (lam_f, info_f) = timed(lambda: step(rb, G, 100))
        forms[name] = (ms_f, lam_f, info_f.inner_iterations)
    apply_form(rb, G, FORMS_C5["mixed"])
    learned.attach(G, hnet, fallback_ratio=ratio)

    # per-kernel device time over one step (CUDA events around every launch; graphs off)
    ctx.profile(True)
    ctx.profile_reset()
    time_steps(rb, ctx, G, 1)
    stats = {k: v for k, v in ctx.profile_stats().items() if v[0] > 0}
    ctx.profile(False)
    roof = roofline(ctx, stats, G, peaks, tuning, traffic_table=NCU_TRAFFIC_ARCH)
    if roof.get("traffic_source"):
        roof["traffic_source"] = ("ncu capture of the same kernel variant and launch shape on the 255x256x128 "
                                  "worst-case box (vectors > L2), per node, scaled to this node box")
    issue_roofline(rb, ctx, G, roof, clk, inst_table=NCU_INST_ARCH)
    top = sorted(stats.items(), key=lambda kv: -kv[1][1])[:10]

    ms_step = ms / args.steps
    lam = lams[0]
    m_ms, m_lam, m_it = forms["mixed"]
    p_ms, p_lam, p_it = forms["plain"]
    nx, ny, nz = dims
    line = {
        "metric": METRIC_ARCH, "value": ws * args.steps / (ms * 1e-3), "unit": "solves/s", "n_gpus": ws,
        "steps": args.steps, "warmup": warm, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64+f32+bf16", "data": "synthetic",
        "config": {"workload": f"arch {nx}x{ny}x{nz} (tunnel radius {int(round(96 * ny / 256))}, support pads, top "
                               f"face loadable, wscf), design after {ARCH['design_iters']} OC iterations (V 0.4, R 2, "
                               "move 0.06, eta 0.5, p 3); Lanczos k=16, inner MG-PCG to 1e-6, stencil assembly included",
                   "form": "learned+mixed: " + form_text(FORMS_C5["mixed"]) + ", FP64 coarsest solve, FP64 flexible "
                           "CG vectors and dots; U-Net correction z += N(rho, r, Vcycle(r)) under the cost-aware gate",
                   "speedup_vs_plain_fp64": p_ms / ms_step, "speedup_vs_mixed_without_network": m_ms / ms_step,
                   "plain_fp64_ms_per_step": p_ms, "mixed_ms_per_step": m_ms,
                   "speedup_mixed_vs_plain_fp64": p_ms / m_ms,
                   "lambda_learned_mixed": lam, "lambda_mixed": m_lam, "lambda_plain_fp64": p_lam,
                   "lambda_rel_diff": abs(lam - p_lam) / abs(p_lam),
                   "lambda_rel_diff_mixed": abs(m_lam - p_lam) / abs(p_lam),
                   "inner_pcg_iterations": infos[0].inner_iterations, "inner_pcg_iterations_mixed": m_it,
                   "inner_pcg_iterations_plain_fp64": p_it,
                   "learned": {"fallback_ratio": ratio, "plain_rate_per_iteration":
                               float(cal.rel_residual) ** (1.0 / max(cal.iterations, 1)),
                               "plain_iteration_ms": cal.seconds * 1e3 / max(cal.iterations, 1),
                               "network_ms": t_net * 1e3, "corrections_in_timed_steps": applied1 - applied0,
                               "judged_off_at_end": judged_off, "train_steps": ARCH["train_steps"],
                               "train_crops": n_samples,
                               "loss_first": float(np.mean(losses[:10])), "loss_last": float(np.mean(losses[-20:])),
                               "harvest_s": t_harvest, "train_s": t_train},
                   "setup_s": t_setup, "e2e_steps": n_e2e,
                   "l2": "working set several GB of vectors and stencils >> 126 MB L2 per step",
                   "parallelism": f"replicas x{ws}", "tile_shapes": tuning},
        "clocks": clk, "gpu_launches": nlaunch, "roofline": roof,
        "kernel_top": {k: {"launches": v[0], "ms": round(v[1], 3)} for k, v in top},
        "e2e": {"value": ws * n_e2e / (e2e_ms * 1e-3), "unit": "solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
    }
    if rank == 0 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        smp = arch_cpu_sample(threads, dims, p_it, ARCH["k"] + 1)
        line["cpu_baseline"] = {"value": 1.0 / smp["extrapolated_s_per_step"], "unit": "solves/s", "cores": threads,
                                "kind": "port", "extrapolated": True,
                                "sample": f"oracle plain FP64 SGS V-cycle PCG on the {'x'.join(map(str, smp['sample_dims']))}"
                                          f" arch: assembly + one solve to 1e-6 ({smp['sample_pcg_iterations']} iterations,"
                                          f" {smp['sampled_wall_s']:.1f} s), scaled by node count x{smp['node_scale_factor']:.1f}"
                                          f" and to the plain method's {p_it} inner iterations per step on the GPU",
                                **smp}
    if rank == 0:
        print(json.dumps(line))
    hnet.close()
    G.close()
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="arch",
                    choices=["arch", "worstcase128", "batched", "learned", "c5", "c5oc40", "voxelize", "c1"],
                    help="arch (default): the worst-case solve on the 511x256x256 arch, learned+mixed vs mixed vs plain "
                         "FP64; worstcase128: the 128x128x64 worst-case box; batched: the 12-instance + 8-RHS batched "
                         "solves; c5: timed OC iterations of the arch; c5oc40: the 40-iteration arch optimisation with "
                         "the plain FP64 check every 10")
    ap.add_argument("--forms", default="both", choices=["both", "mixed"],
                    help="mixed: time only the mixed form (short command for launch-list captures)")
    ap.add_argument("--conv", default="16,16", help="--kernel conv3: input and output channels")
    ap.add_argument("--kernel", default=None, choices=["conv3", "fine_residual", "fine_jacobi", "st_residual",
                                                       "st_residual_f32", "st_residual_f64", "st_cheby_f32",
                                                       "st_cheby_bf16", "st_cheby_f64", "st_jacobi_f32",
                                                       "fine_cheby_f32", "fine_residual_f64", "fine_applyK_f64",
                                                       "fine_residual_f32"])
    ap.add_argument("--size", default=None, help="kernel mode and arch workload: grid NXxNYxNZ (default: the bench "
                                                  "workload)")
    ap.add_argument("--level", type=int, default=1, help="kernel mode, st_* kernels: the stencil level")
    ap.add_argument("--tiles", default="autotune",
                    help="finest-level launch shape of the worst-case bench: autotune, or variant,rows,zchunk for "
                         "every finest-level kernel")
    ap.add_argument("--fused", default="auto", choices=["auto", "on", "off"],
                    help="FP32 Chebyshev sweeps of the stencil levels as one cooperative launch per smoothing: the "
                         "library's setting (auto: off unless enabled), or on / off for every level")
    ap.add_argument("--shape", default=None, help="kernel mode: launch shape variant,rows,zchunk (default: autotune)")
    ap.add_argument("--oc-iters", type=int, default=40, help="c5oc40 workload: OC iterations")
    ap.add_argument("--maxit", type=int, default=3000, help="batched workload: PCG iteration limit per solve")
    ap.add_argument("--time-budget", type=float, default=900.0,
                    help="c5oc40 workload: seconds after which the run stops at the end of an OC iteration (0: none)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.kernel == "conv3":
        return run_conv(args)
    if args.kernel:
        return run_kernel(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "learned":
        return run_learned(args)
    if args.workload == "voxelize":
        return run_voxelize(args)
    if args.workload == "c1":
        return run_c1(args)
    if args.workload == "c5":
        return run_c5(args)
    if args.workload == "c5oc40":
        return run_c5_oc40(args)
    if args.workload == "arch":
        return run_arch(args)
    return run_worstcase128(args)


def run_worstcase128(args):
    """The worst-case solve on the 128x128x64 box (smoothed random density, z = 0 clamped, top face
    loadable, wsff): mixed form timed, plain FP64 beside it."""

    import torch

    ws, rank, lrank = dist_env()
    dist = init_replicas(ws, lrank)

    import robtop_b200 as rb
    from robtop_b200 import configs

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass

    ctx = make_ctx(rb, lrank)
    cfg, G = build_problem(rb, configs, ctx, rb.FP32)
    # launch shapes of the finest-level kernels, chosen once by the library's autotuner (or fixed by
    # --tiles, e.g. for a profiler run, under which the autotuner's timings are distorted)
    G.update_stencil()
    tuning = G.autotune() if args.tiles == "autotune" else G.set_tiles(*map(int, args.tiles.split(",")))
    if args.fused != "auto":  # fused Chebyshev sweeps on every stencil level, or on none
        for lvl in range(1, G.n_grid() - 1):
            rb._capi.check(rb.lib().rt_set_level_fused(G.handle, lvl, 1 if args.fused == "on" else 0), ctx.handle)
        tuning = G.tuning()
    results = {}
    for prec in ((rb.FP64, rb.FP32) if args.forms == "both" else (rb.FP32,)):
        apply_form(rb, G, FORMS["plain" if prec == rb.FP64 else "mixed"])
        for w in range(max(args.warmup, 3)):
            step(rb, G, 10 + w)
        if dist:
            dist.barrier()
        clocks = Clocks(gpu_id(lrank)) if prec == rb.FP32 else None
        if clocks:
            clocks.start()
        ms, lams, infos, nlaunch = time_steps(rb, ctx, G, args.steps)
        if prec == rb.FP32:
            # end to end through the public API with host buffers, under the same clock sampler
            e2e_ms, h2d, d2h = e2e_steps(rb, ctx, G, cfg, args.steps)
        clk = clocks.stop() if clocks else None
        if prec == rb.FP32:
            ms, e2e_ms = max_over_ranks(dist, [ms, e2e_ms])
        else:
            ms = max_over_ranks(dist, [ms])[0]
        results[prec] = dict(ms=ms, lams=lams, infos=[i.as_dict() for i in infos], launches=nlaunch, clocks=clk)

    # per-kernel device time over the same K steps (CUDA events around every launch; separate pass)
    ctx.profile(True)
    ctx.profile_reset()
    time_steps(rb, ctx, G, args.steps)
    stats = ctx.profile_stats()
    ctx.profile(False)
    stats = {k: v for k, v in stats.items() if v[0] > 0}
    roof = roofline(ctx, stats, G, peaks, tuning)
    issue_roofline(rb, ctx, G, roof, results[rb.FP32]["clocks"])
    top = sorted(stats.items(), key=lambda kv: -kv[1][1])[:8]

    r32, r64 = results[rb.FP32], results.get(rb.FP64)
    ms_step = r32["ms"] / args.steps
    value = ws * args.steps / (r32["ms"] * 1e-3)
    lam32 = float(np.mean(r32["lams"]))
    lam64 = float(np.mean(r64["lams"])) if r64 else None
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": ws, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
        "config": {"workload": "worst-case 128x128x64 (smoothed random density, z=0 clamped, top-face load set, "
                               "wsff), Lanczos k=16, inner MG-PCG to 1e-6, stencil assembly included",
                   "form": "mixed: " + form_text(FORMS["mixed"]) + ", FP64 coarsest solve, FP64 residual "
                           "recomputed at each refinement restart, one CUDA graph per inner solve; plain "
                           "(fp64_ms_per_step): FP64 symmetric-GS V-cycle in FP64 flexible CG",
                   "fp64_ms_per_step": r64["ms"] / args.steps if r64 else None,
                   "speedup_vs_fp64": r64["ms"] / r32["ms"] if r64 else None,
                   "lambda_mixed": lam32, "lambda_fp64": lam64,
                   "lambda_rel_diff": abs(lam32 - lam64) / abs(lam64) if r64 else None,
                   "inner_pcg_iterations": r32["infos"][0]["inner_iterations"],
                   "inner_pcg_iterations_fp64": r64["infos"][0]["inner_iterations"] if r64 else None,
                   "l2": "working set ~0.4 GB of vectors and stencils > 126 MB L2 per step",
                   "parallelism": f"replicas x{ws}",
                   "tile_shapes": tuning},
        "clocks": r32["clocks"],
        "gpu_launches": r32["launches"],
        "roofline": roof,
        "kernel_top": {k: {"launches": v[0], "ms": round(v[1], 3)} for k, v in top},
        "e2e": {"value": ws * args.steps / (e2e_ms * 1e-3), "unit": "solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
    }
    if rank == 0 and not args.no_cpu_baseline:
        # the CPU runs the plain method: its time is extrapolated to the plain method's own inner
        # iteration count on the GPU (the mixed form's count when the plain form was not run)
        its_plain = r64["infos"][0]["inner_iterations"] if r64 else r32["infos"][0]["inner_iterations"]
        line["cpu_baseline"] = cpu_baseline(its_plain, r32["infos"][0]["vcycles"], os.cpu_count() or 1)
    if rank == 0:
        print(json.dumps(line))
    G.close()
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
