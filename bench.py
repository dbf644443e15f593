"""Benchmark: seconds per design iteration of the GPU-TO topology-optimisation
loop on the 256x128x128 cantilever (4.19M hex8 elements, 12.83M DOF), MGCG
tolerance 1e-6, 6 multigrid levels, on one B200.

A step is one design iteration of the top3D125 loop: density filter, SIMP,
MGCG solve (hierarchy setup + PCG to relres < 1e-6), compliance sensitivity,
filtered sensitivities and the OC update, every field resident in HBM.  Every
step starts from the same design, so every step does the same work.  The
design is a mid-optimisation one: the 64x32x32 cantilever design after 50 OC
iterations (tests/golden/design_c1.npz, produced with the reference's solver),
upsampled 4x to 256x128x128 -- synthetic, deterministic, with the void/solid
contrast of a real run.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl gputo|reference]

The headline ``value`` is the mixed-precision path (FP32 V-cycle, flexible
FP64 PCG); ``fp64`` carries the plain FP64 MGCG on the same design.  ``e2e`` is
the same design iteration through the host-buffer C ABI a MATLAB caller uses
(gputo_density_filter, mgcg1, gputo_compliance_sens, gputo_oc_update), with all
host<->device copies inside the timed region.  ``--impl reference`` times the
reference's own OpenMP MEX (Cantilever/omp/mgcg1.c, compiled into oracle/_ref)
on the host cores on the same design.

With N > 1 (torchrun) every rank runs an independent replica ("replicas
only": the path has no exchange step); value = max-over-ranks time / (N K).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpu-to_b200"))

NELX, NELY, NELZ, NL = 256, 128, 128, 6
TOL, MAXIT = 1e-6, 500
VOLFRAC, PENAL, RMIN, MOVE = 0.12, 3.0, 3 ** 0.5, 0.2
METRIC = "s/design-iter @12.7M DOF, tol 1e-6: mixed+learned vs FP64 MGCG, same B200"
# PCG iterations the FP64 MGCG needs on the bench design at tol 1e-6, as the
# FP64 arm of this benchmark measures them on a B200 (the reference's MGCG
# runs the same algorithm and takes the same count; the tests check that
# iteration for iteration on smaller grids).  The CPU arm extrapolates its
# bounded sample to this count.
FP64_NIT_ON_BENCH_DESIGN = 71
# dram__bytes_read.sum + dram__bytes_write.sum of one FP32 Jacobi sweep launch
# (hsweep2_kernel) at 256x128x128 (188.7 MB + 37.1 MB), from an ncu capture of
# bench.py --micro jacobi32.
HSWEEP32_DRAM_BYTES = 225.8e6


def bench_design(nelx=NELX, nely=NELY, nelz=NELZ):
    d = np.load(os.path.join(ROOT, "tests", "golden", "design_c1.npz"))
    x = d["x"].astype(np.float64).reshape(64, 32, 32)  # (x, z, y) element order
    fx, fz, fy = nelx // 64, nelz // 32, nely // 32
    if fx * 64 != nelx or fz * 32 != nelz or fy * 32 != nely:
        return np.full(nelx * nely * nelz, VOLFRAC)
    xb = np.repeat(np.repeat(np.repeat(x, fx, 0), fz, 1), fy, 2)
    return np.ascontiguousarray(xb.reshape(-1))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [t.strip() for t in ln.split(",")]
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
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_init(backend="nccl"):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def max_over_ranks(v, ws):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seconds(t_max, steps, ws):
    """Whole-job seconds per design iteration for ws independent replicas
    that each ran 'steps' design iterations in t_max seconds (the slowest
    rank): ws designs finish per step."""
    return t_max / (steps * ws)


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def time_design_loop(gputo, torch, precision, x0, F, fixed, Ke0, steps, warmup, ws, stream,
                     clocks=None, tune=False):
    """Time 'steps' design iterations.  tune: after the first warm-up step,
    gputo_autotune_dev times complete solves of this design over the tunable
    options (Jacobi sweeps per smoothing step on all levels and on the finest
    level, smoother back end, host check interval) and keeps the fastest;
    the timed steps use that choice."""
    opts = gputo.default_options(precision=precision)
    dl = gputo.DesignLoop(NELX, NELY, NELZ, NL, F, fixed, Ke0, volfrac=VOLFRAC, penal=PENAL,
                          rmin=RMIN, move=MOVE, tol=TOL, maxit=MAXIT, options=opts, x0=x0,
                          stream=stream)
    x0_dev = dl.x.clone()
    infos = []

    def one():
        dl.x.copy_(x0_dev)
        return dl.step()

    dl.tuned = None
    for w in range(warmup):
        one()
        if tune and w == 0:
            torch.cuda.synchronize()
            best, bms, _ = gputo.autotune(dl.solver, dl.F, torch.zeros_like(dl.U), TOL, MAXIT)
            dl.tuned = {"nswp": best.nswp, "nswp_fine": best.nswp_fine, "nswp_coarse": best.nswp_coarse, "coarse_from": best.coarse_from, "sweep_xchunk": best.sweep_xchunk,
                        "tc_parts": best.tc_parts,
                        "check_every": best.check_every, "solve_ms": round(bms, 2)}
    torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = gputo.launch_count()
    ctx = clocks if clocks is not None else _Null()
    with ctx:
        e0.record(stream)
        for _ in range(steps):
            infos.append(one())
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(ws)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = gputo.launch_count() - launches0
    return dl, ms / 1000.0, infos, launches


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def time_filter(gputo, torch, inputs, reps, stream):
    """Mean time of one density-filter launch (imfilter, normalised), CUDA
    events on the launching stream, launches back to back inside the library
    (gputo_time_filter_dev).  They cycle through four inputs and four outputs
    (268 MB, more than L2), so each one reads from HBM."""
    outs = [torch.empty_like(inputs[0]) for _ in inputs]
    return gputo.time_filter_dev(inputs, outs, NELX, NELY, NELZ, RMIN, reps, stream=stream)


def mixed_parity(gputo, torch, dl, fixed, Ke0, stream):
    """Accuracy of the timed mixed-precision solve (the last step's U, at the
    benchmark tolerance): against an FP64 MGCG solve of the same design to
    1e-10, with the true residual of the mixed U from an FP64 apply.  For
    context, the same figures for a plain FP64 solve at the benchmark
    tolerance.  Outside the timed region."""
    Um, CX, Fd = dl.U.clone(), dl.CX.clone(), dl.F
    s64 = gputo.Solver(NELX, NELY, NELZ, NL, gputo.default_options())
    s64.set_problem(Ke0, fixed)
    s64.setup(CX, stream=stream)
    Uref = torch.zeros_like(Fd)
    rr_ref, nit_ref = s64.solve(Fd, Uref, 1e-10, 2000, stream=stream)
    U6 = torch.zeros_like(Fd)
    rr6, nit6 = s64.solve(Fd, U6, TOL, MAXIT, stream=stream)
    KU = torch.zeros_like(Fd)
    torch.cuda.synchronize()

    def figures(U):
        s64.apply(U, KU, stream=stream)
        torch.cuda.synchronize()
        c_ref, c = float(Fd @ Uref), float(Fd @ U)
        return {"compliance_rel_err": abs(c - c_ref) / abs(c_ref),
                "u_l2_rel_err": float(torch.linalg.norm(U - Uref) / torch.linalg.norm(Uref)),
                "true_relres": float(torch.linalg.norm(Fd - KU) / torch.linalg.norm(Fd))}

    out = {"vs": f"FP64 MGCG of the same design to relres {rr_ref:.2e} ({nit_ref} iterations)",
           **figures(Um), "fp64_at_tol": {"nit": nit6, **figures(U6)}}
    del s64
    return out


def e2e_design_iteration(gputo, x, F, fixed, Ke0, opts, state):
    """One design iteration through the host-buffer C ABI, as a C caller
    would run it with these drop-ins (top3D125modCuda.m:105-152).  Like the
    driver, dV and the U array are made once before the loop and kept in
    'state', and so are the host output arrays each C-ABI call writes into
    (a fresh output page costs a first-touch fault per call otherwise).
    Returns (xnew, info, h2d, d2h)."""
    nel = x.size
    nd = F.size
    if "U" not in state:
        state["U"] = np.zeros(nd)
        state["dV"] = np.full(nel, 1.0 / nel / VOLFRAC)
        for k in ("xPhys", "CX", "dsK", "ce", "dc", "dcf", "dV0", "xnew"):
            state[k] = np.zeros(nel)
    U, dV = state["U"], state["dV"]
    xPhys = gputo.density_filter(x, NELX, NELY, NELZ, RMIN, out=state["xPhys"])
    CX, dsK = gputo.simp(xPhys, PENAL, 1.0, 1e-9, out=(state["CX"], state["dsK"]))
    rr, nit = gputo.mgcg1(Ke0, F, U, CX, fixed, fixed.size, NELX, NELY, NELZ, NL, TOL, MAXIT,
                          printLev=0, options=opts)
    ce, dc, c = gputo.compliance_sens(Ke0, U, CX, dsK, NELX, NELY, NELZ, out=(state["ce"], state["dc"]))
    dcf = gputo.density_filter(dc, NELX, NELY, NELZ, RMIN, out=state["dcf"])
    dV0 = gputo.density_filter(dV, NELX, NELY, NELZ, RMIN, out=state["dV0"])
    xnew, lmid = gputo.oc_update(x, dcf, dV0, VOLFRAC, MOVE, out=state["xnew"])
    # bytes crossing PCIe, counted from the arrays each call copies
    h2d = 8 * (nel                       # filter(x)
               + nel                     # simp: xPhys
               + nd + nel + fixed.size   # mgcg1: F, CX, fixed
               + nd + 2 * nel            # compliance_sens: U, CX, dsK
               + nel + nel               # the two sensitivity filters
               + 3 * nel)                # oc_update: x, dc, dV0
    d2h = 8 * (nel + 2 * nel + nd + 2 * nel + 2 * nel + nel)
    return xnew, {"c": c, "nit": nit, "relres": rr}, h2d, d2h


def run_ours(args):
    import torch

    import gputo
    ws, rank, local = dist_init()
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream()
    Ke0 = gputo.hex8_stiffness(0.3)
    F, fixed = gputo.cantilever(NELX, NELY, NELZ)
    x0 = bench_design()
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "of measured" if "hbm_gbs" in peaks else "of fallback"

    with torch.cuda.stream(stream):
        clocks = ClockSampler(local)
        dl_m, t_m, inf_m, launches = time_design_loop(gputo, torch, gputo.PREC_MIXED, x0, F, fixed,
                                                      Ke0, args.steps, args.warmup, ws, stream,
                                                      clocks, tune=True)
        tuned = dl_m.tuned
        # per-kernel timing on the mixed hierarchy, for the roofline
        ms_apply64 = dl_m.solver.time_kernel(0, 20, stream)
        ms_jac32 = dl_m.solver.time_kernel(1, 20, stream)
        ms_lvl1_32 = dl_m.solver.time_kernel(2, 20, stream)
        ms_energy = dl_m.solver.time_kernel(5, 20, stream)
        ms_filter = time_filter(gputo, torch, [dl_m.x, dl_m.CX, dl_m.dsK, dl_m.dV], 20, stream)
        parity = mixed_parity(gputo, torch, dl_m, fixed, Ke0, stream)
        del dl_m
        torch.cuda.empty_cache()
        dl_d, t_d, inf_d, _ = time_design_loop(gputo, torch, gputo.PREC_FP64, x0, F, fixed, Ke0,
                                               max(1, args.steps // 2), args.warmup, ws, stream)
        ms_lvl1_64 = dl_d.solver.time_kernel(3, 20, stream)
        del dl_d
        torch.cuda.empty_cache()
        # the mixed solver on the reference's smoothing schedule (nswp 3 on every level)
        dl_u, t_u, inf_u, _ = time_design_loop(gputo, torch, gputo.PREC_MIXED, x0, F, fixed, Ke0,
                                               max(1, args.steps // 2), args.warmup, ws, stream)
        del dl_u
        torch.cuda.empty_cache()

    t_m = max_over_ranks(t_m, ws)
    t_d = max_over_ranks(t_d, ws)
    t_u = max_over_ranks(t_u, ws)
    K = args.steps
    s_mixed = replica_seconds(t_m, K, ws)
    s_fp64 = replica_seconds(t_d, max(1, args.steps // 2), ws)
    s_mixed_ref = replica_seconds(t_u, max(1, args.steps // 2), ws)

    # e2e: host buffers through the drop-in C ABI, with the options the
    # autotuner chose for the device-resident measurement (passed in the
    # mgcg1 call's options, as a caller would)
    opts = gputo.default_options(precision=gputo.PREC_MIXED)
    if tuned:
        for k in ("nswp", "nswp_fine", "nswp_coarse", "coarse_from", "sweep_xchunk", "tc_parts", "check_every"):
            setattr(opts, k, tuned[k])
    xhost = x0.copy()
    e2e_state = {}
    for _ in range(1):
        e2e_design_iteration(gputo, xhost, F, fixed, Ke0, opts, e2e_state)  # warm caches
    barrier(ws)
    t0 = time.perf_counter()
    ke2e = max(1, min(args.steps, 3))
    for _ in range(ke2e):
        _, inf_e, h2d, d2h = e2e_design_iteration(gputo, xhost, F, fixed, Ke0, opts, e2e_state)
    t_e2e = replica_seconds(max_over_ranks(time.perf_counter() - t0, ws), ke2e, ws)

    ndof = 3 * (NELX + 1) * (NELY + 1) * (NELZ + 1)
    nel = NELX * NELY * NELZ
    nel1 = nel // 8
    ndof1 = 3 * (NELX // 2 + 1) * (NELY // 2 + 1) * (NELZ // 2 + 1)
    nnod = (NELX + 1) * (NELY + 1) * (NELZ + 1)
    nnod1 = ndof1 // 3
    # Fine sweeps (Ke in its Hadamard basis): u (or f), out, CX, the mask byte per
    # node, plus f and 1/diag for the Jacobi sweep; ~149 operations per element
    # (the dense 24x24 product would be 1152 FLOP).
    kernels = {
        "fine_apply_fp64": {"ms": ms_apply64, "bytes": 16 * ndof + 8 * nel + nnod, "ops": 149 * nel},
        "fine_jacobi_fp32": {"ms": ms_jac32, "bytes": 16 * ndof + 4 * nel + nnod, "ops": 149 * nel},
        # level 1, matrix-free from the fine CX: u, f, 1/diag and the output
        # (4 vectors of ndof1), the fine CX and the level-1 mask byte per node;
        # the element pass's per-element scratch is not algorithmic traffic
        "level1_jacobi_fp32": {"ms": ms_lvl1_32, "bytes": 16 * ndof1 + 4 * nel + nnod1},
        "level1_jacobi_fp64": {"ms": ms_lvl1_64, "bytes": 32 * ndof1 + 8 * nel + nnod1},
        # the FP64 apply of the solution with ce, dc and |F - K U|^2 in its epilogue:
        # U and F read, ce written, CX read, the mask byte per node
        "energy_fused_fp64": {"ms": ms_energy, "bytes": 16 * ndof + 16 * nel + nnod},
        # density filter (3^3 stencil): x read, xPhys written
        "filter_fp64": {"ms": ms_filter, "bytes": 16 * nel},
    }
    for k in kernels.values():
        k["gbs"] = k["bytes"] / (k["ms"] * 1e-3) / 1e9
    # The dominant kernel of a mixed design iteration is the FP32 Jacobi sweep
    # (the largest share of an ncu launch list of one step); its DRAM traffic per
    # launch is read + write from one ncu capture of this workload.
    dom = kernels["fine_jacobi_fp32"]
    roofline = {"bound": "hbm", "kernel": "hsweep2_kernel<MODE_JACOBI> (damped Jacobi sweep, FP32, element pairs)",
                "achieved": round(dom["gbs"], 1), "peak": hbm_peak, "unit": "GB/s",
                "frac": round(dom["gbs"] / hbm_peak, 4), "peak_source": peak_src,
                "traffic": HSWEEP32_DRAM_BYTES,
                "note": "issue-bound, not HBM-bound: 39.1M warp instructions per launch at 51% issue activity"}

    result = {
        "metric": METRIC, "value": round(s_mixed, 5), "unit": "s/design-iter",
        "n_gpus": ws, "steps": K, "warmup": args.warmup,
        "ms_per_step": round(1000 * t_m / K, 3), "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 outer PCG / f32 V-cycle",
        "data": "synthetic: 256x128x128 cantilever, mid-optimisation design (64x32x32 design "
                "after 50 OC iterations, upsampled 4x); working set > L2",
        "config": {"workload": "one top3D125 design iteration (filter, SIMP, MGCG solve to "
                               "1e-6, sensitivity, filters, OC) on the 256x128x128 cantilever",
                   "nelx": NELX, "nely": NELY, "nelz": NELZ, "ndof": ndof, "nl": NL,
                   "tol": TOL, "rmin": RMIN, "volfrac": VOLFRAC,
                   "l2": "inputs larger than L2 (12.8M-DOF FP64 vectors of 103 MB; ~4 GB per step)",
                   "parallelism": f"replicas x{ws}",
                   "learned": "off: the learned correction does not lower the iteration count on the designs "
                              "measured, so its auto mode keeps the plain mixed V-cycle"},
        "fp64": {"value": round(s_fp64, 5), "unit": "s/design-iter", "schedule": "the reference's (nswp 3, every level)",
                 "nit": [i["nit"] for i in inf_d], "speedup_mixed_vs_fp64": round(s_fp64 / s_mixed, 3)},
        "mixed_reference_schedule": {"value": round(s_mixed_ref, 5), "unit": "s/design-iter",
                                     "nit": [i["nit"] for i in inf_u],
                                     "speedup_vs_fp64": round(s_fp64 / s_mixed_ref, 3)},
        "tuned": tuned,
        "true_relres": [i.get("true_relres") for i in inf_m],
        "nit": [i["nit"] for i in inf_m],
        "relres": [i["relres"] for i in inf_m],
        "compliance": inf_m[-1]["c"] if inf_m else None,
        "parity": parity,
        "dof_iters_per_s": round(ndof * np.mean([i["nit"] for i in inf_m]) / s_mixed, 1),   # all replicas
        "e2e": {"value": round(t_e2e, 5), "unit": "s/design-iter", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "timing": "host wall clock around synchronous "
                                                          "host-buffer C-ABI calls",
                "options": "the autotuned solver options of value" if tuned else "defaults"},
        "gpu_launches": int(launches),
        "roofline": roofline,
        "kernels": {k: {kk: (round(vv, 4) if isinstance(vv, float) else vv) for kk, vv in v.items()}
                    for k, v in kernels.items()},
        "clocks": clocks.summary(),
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline_sample(x0, inf_d)
    if rank == 0:
        print(json.dumps(result))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# the reference's CPU implementation (oracle/_ref: Cantilever/omp/mgcg1.c)
# ---------------------------------------------------------------------------

def _ref_module():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.ref_available():
        return None, "compiled reference oracle/_ref/libmgcg1_omp_ref.so is absent"
    return O, None


def _ref_call(O, p, CX, maxit):
    t = time.perf_counter()
    U, rr, nit = O.ref_mgcg1(p, CX, NL, TOL, maxit)
    return time.perf_counter() - t, U


def _design_rest_cpu(O, p, xPhys, U):
    """The MATLAB-side steps (filter, sensitivity, OC) on the host, timed once."""
    t = time.perf_counter()
    nel = p.nel
    CX, dsK = O.simp(xPhys)
    Uc = U.copy()
    Uc[1::3] *= -1
    ce = O.element_energy(p, Uc)
    dcf, hs = O.filter3d(dsK * ce, NELX, NELY, NELZ, RMIN)
    dv0, _ = O.filter3d(np.full(nel, 1.0 / nel / VOLFRAC), NELX, NELY, NELZ, RMIN)
    O.oc_update(xPhys, dcf / hs, dv0 / hs, VOLFRAC, MOVE)
    return time.perf_counter() - t


def _cores():
    lim = os.environ.get("OMP_THREAD_LIMIT")
    n = os.cpu_count() or 1
    # mgcg1.c:120-121 hard-codes 16 OpenMP threads
    return min(16, n, int(lim) if lim else n)


def cpu_baseline_sample(x0, inf_d=None):
    """The reference's OpenMP MEX on a bounded sample of the bench workload
    (about 25 s of CPU work): a cgmax=1 call (hierarchy setup, first V-cycle,
    one PCG iteration) and a cgmax=11 call; the per-iteration cost is their
    difference over 10 iterations, and the value extrapolates to the FP64
    iteration count of this design.  ``--impl reference`` times a complete
    design iteration instead."""
    O, why = _ref_module()
    if O is None:
        return {"value": None, "unit": "s/design-iter", "cores": 0, "kind": "reference",
                "sample": why}
    os.environ.setdefault("OMP_THREAD_LIMIT", str(os.cpu_count()))
    p = O.cantilever(NELX, NELY, NELZ)
    xf, hs = O.filter3d(x0, NELX, NELY, NELZ, RMIN)
    xPhys = xf / hs
    CX, _ = O.simp(xPhys)
    t1, U = _ref_call(O, p, CX, 1)
    t11, _ = _ref_call(O, p, CX, 11)
    t_iter = max(t11 - t1, 0.0) / 10.0
    nit = FP64_NIT_ON_BENCH_DESIGN
    if inf_d:
        nit = int(np.median([i["nit"] for i in inf_d]))
    t_rest = _design_rest_cpu(O, p, xPhys, U)
    est = t1 + (nit - 1) * t_iter + t_rest
    return {"value": round(est, 2), "unit": "s/design-iter", "cores": _cores(), "kind": "reference",
            "sample": f"reference OpenMP MEX (Cantilever/omp/mgcg1.c) on the bench design: "
                      f"cgmax=1 call (setup + 1 PCG iteration) {t1:.1f}s, cgmax=11 call {t11:.1f}s, "
                      f"so {t_iter:.2f}s per PCG iteration (10-iteration difference); extrapolated to "
                      f"{nit} iterations (the FP64 count) plus {t_rest:.1f}s for filter/sensitivity/OC "
                      f"(oracle restatement); bench.py --impl reference times a whole design iteration"}


def run_reference(args):
    """The reference's own CPU implementation of the path, timed whole: each
    timed step is one complete design iteration on the bench design -- the
    reference's OpenMP MEX (Cantilever/omp/mgcg1.c, unmodified) solving to
    tol 1e-6 from its own zero start, plus the MATLAB-side steps (filter,
    sensitivity, OC) in the oracle's numpy restatement (MATLAB is absent).
    About 80-125 s per step on 16 host cores, so only GPUTO_REF_STEPS steps
    (default 1) are timed, after one short warm-up call; the line reports the
    number of steps actually timed."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    O, why = _ref_module()
    if O is None:
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return
    os.environ.setdefault("OMP_THREAD_LIMIT", str(os.cpu_count()))
    p = O.cantilever(NELX, NELY, NELZ)
    x0 = bench_design()
    steps = max(1, min(args.steps, int(os.environ.get("GPUTO_REF_STEPS", "1"))))
    xf, hs = O.filter3d(x0, NELX, NELY, NELZ, RMIN)
    _ref_call(O, p, O.simp(xf / hs)[0], 1)   # warm-up: page-in, OpenMP thread start
    timed, nits = [], []
    for _ in range(steps):
        t0 = time.perf_counter()
        xf, hs = O.filter3d(x0, NELX, NELY, NELZ, RMIN)
        xPhys = xf / hs
        CX, _ = O.simp(xPhys)
        U, rr, nit = O.ref_mgcg1(p, CX, NL, TOL, MAXIT)
        t_solve = time.perf_counter() - t0
        _design_rest_cpu(O, p, xPhys, U)
        timed.append(time.perf_counter() - t0)
        nits.append(int(nit))
    value = float(np.mean(timed))
    cores = _cores()
    sample = (f"{steps} complete design iteration(s) timed, unextrapolated: the reference OpenMP MEX "
              f"(Cantilever/omp/mgcg1.c, unmodified) solving the bench design to tol {TOL} "
              f"({nits[-1]} PCG iterations, {t_solve:.1f}s for the MEX call) plus filter/sensitivity/OC "
              f"in the oracle's numpy restatement of the MATLAB steps; one cgmax=1 warm-up call before")
    out = {"metric": METRIC, "value": round(value, 3), "unit": "s/design-iter", "n_gpus": ws,
           "steps": steps, "steps_requested": args.steps, "warmup": args.warmup,
           "ms_per_step": round(1000 * value, 1),
           "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
           "dtype": "f64", "data": "synthetic: same design as the gputo arm",
           "config": {"workload": "one top3D125 design iteration on the 256x128x128 cantilever",
                      "nelx": NELX, "nely": NELY, "nelz": NELZ, "nl": NL, "tol": TOL, "nit": nits},
           "impl": "reference",
           "cpu_baseline": {"value": round(value, 3), "unit": "s/design-iter", "cores": cores,
                            "kind": "reference", "sample": sample},
           "e2e": {"value": round(value, 3), "unit": "s/design-iter", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


KERNELS = {"apply64": 0, "jacobi32": 1, "level1_32": 2, "level1_64": 3, "jacobi_tc": 4, "energy_fused": 5, "level2_32": 6,
           "energy64": -1, "energy_tc": -2, "filter": -3}


def run_micro(args):
    """Profiling aid: build one solver on the bench design and launch a single
    kernel kind a few times (for ncu -k ... -c ...); prints mean times."""
    import torch

    import gputo
    nelx, nely, nelz = (int(v) for v in args.size.split("x"))
    nl = args.nl
    F, fixed = gputo.cantilever(nelx, nely, nelz)
    x0 = bench_design(nelx, nely, nelz)
    kinds = list(KERNELS) if args.micro == "all" else [args.micro]
    mixed = any(k in ("jacobi32", "level1_32", "jacobi_tc", "level2_32") for k in kinds)
    opts = gputo.default_options(precision=gputo.PREC_MIXED if mixed else gputo.PREC_FP64,
                                 tc_parts=2 if "jacobi_tc" in kinds else 0, sweep_pairs=args.sweep_pairs)
    s = gputo.Solver(nelx, nely, nelz, nl, opts)
    s.set_problem(gputo.hex8_stiffness(), fixed)
    xd = torch.as_tensor(x0, dtype=torch.float64, device="cuda")
    xp = torch.empty_like(xd)
    gputo.density_filter_dev(xd, xp, nelx, nely, nelz, RMIN)
    CX = torch.empty_like(xd)
    gputo.simp_dev(xp, CX)
    s.setup(CX)
    out = {"micro": args.micro, "size": args.size, "nl": nl, "device_bytes": s.device_bytes}
    for k in kinds:
        if KERNELS[k] >= 0:
            out[k + "_ms"] = s.time_kernel(KERNELS[k], args.reps)
            continue
        if k == "filter":   # launches back to back over four inputs (more than L2)
            ins = [xd] + [torch.rand_like(xd) for _ in range(3)]
            outs = [torch.empty_like(xd) for _ in ins]
            out[k + "_ms"] = gputo.time_filter_dev(ins, outs, nelx, nely, nelz, RMIN, args.reps)
            continue
        # compliance sensitivity of a random displacement field: FP64 kernel or tensor cores
        U = torch.randn(3 * (nelx + 1) * (nely + 1) * (nelz + 1), dtype=torch.float64, device="cuda")
        dsK = -3.0 * xp * xp
        ce, dc = torch.empty_like(xd), torch.empty_like(xd)
        fn = gputo.compliance_sens_dev if KERNELS[k] == -1 else gputo.compliance_sens_tc_dev
        Ke = gputo.hex8_stiffness()
        fn(Ke, U, CX, dsK, nelx, nely, nelz, ce, dc)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.reps):
            fn(Ke, U, CX, dsK, nelx, nely, nelz, ce, dc)
        e1.record()
        torch.cuda.synchronize()
        out[k + "_ms_per_call"] = e0.elapsed_time(e1) / args.reps
    print(json.dumps(out))


def run_one_step(args):
    """Profiling aid: exactly one design iteration of the bench workload after
    the solver is built (for an ncu launch list of one step)."""
    import torch

    import gputo
    prec = gputo.PREC_MIXED if args.one_step == "mixed" else gputo.PREC_FP64
    F, fixed = gputo.cantilever(NELX, NELY, NELZ)
    opts = gputo.default_options(precision=prec, nswp_fine=args.nswp_fine,
                                 check_every=8 if args.nswp_fine else 1, sweep_pairs=args.sweep_pairs)
    if args.nswp:
        opts.nswp = args.nswp
    opts.nswp_coarse = args.nswp_coarse
    opts.coarse_from = args.coarse_from
    dl = gputo.DesignLoop(NELX, NELY, NELZ, NL, F, fixed, gputo.hex8_stiffness(), volfrac=VOLFRAC,
                          penal=PENAL, rmin=RMIN, move=MOVE, tol=TOL, maxit=MAXIT,
                          options=opts, x0=bench_design())
    info = dl.step()
    torch.cuda.synchronize()
    print(json.dumps({"one_step": args.one_step, **info}))


BATCH_SIZES = [(96, 48, 48), (128, 64, 64), (160, 80, 80), (192, 96, 96)]


def batch_designs(n=8, seed=7):
    """The uneven multi-design batch: grid sizes drawn (seeded) from
    BATCH_SIZES, each a cantilever at a uniform density drawn from U(0.1, 0.3);
    nl per design keeps the coarsest grid under ~2k dofs."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        shape = BATCH_SIZES[int(rng.integers(len(BATCH_SIZES)))]
        nl = 4 if shape[0] == 96 else 5
        out.append((shape, nl, float(rng.uniform(0.1, 0.3))))
    return out


def run_batch(args):
    """Multi-design batch: one batched solve of all designs (one CUDA graph
    launch per CG step, options autotuned per grid shape) against the same
    solves one after another; mixed precision, tol 1e-6."""
    import torch

    import gputo
    torch.cuda.set_device(0)
    Ke0 = gputo.hex8_stiffness(0.3)
    members, tuned = [], {}
    for shape, nl, rho in batch_designs():
        F, fixed = gputo.cantilever(*shape)
        CX = torch.full((shape[0] * shape[1] * shape[2],), 1e-9 + rho ** 3 * (1 - 1e-9), dtype=torch.float64,
                        device="cuda")
        s = gputo.Solver(*shape, nl, gputo.default_options(precision=gputo.PREC_MIXED))
        s.set_problem(Ke0, fixed)
        s.setup(CX)
        Fd = torch.as_tensor(F, dtype=torch.float64, device="cuda")
        U = torch.zeros_like(Fd)
        if shape not in tuned:
            tuned[shape] = gputo.autotune(s, Fd, U, TOL, MAXIT)[0]
        else:
            s.set_options(tuned[shape])
        members.append((s, Fd, shape))
    b = gputo.Batch([m[0] for m in members])
    Us = [torch.zeros_like(m[1]) for m in members]

    def seq():
        out = []
        for (s, Fd, _), U in zip(members, Us):
            out.append(s.solve(Fd, U, TOL, MAXIT))
        return out

    def bat():
        return b.solve([m[1] for m in members], Us, TOL, MAXIT, check_every=8)

    res = {}
    for name, fn in (("sequential", seq), ("batched", bat)):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            out = fn()
        e1.record()
        torch.cuda.synchronize()
        res[name] = (e0.elapsed_time(e1) / args.steps / 1000.0, out)
    nits = res["batched"][1][1]
    dofs = sum(3 * (sh[0] + 1) * (sh[1] + 1) * (sh[2] + 1) for _, _, sh in members)
    line = {"metric": "s per batched solve of 8 uneven designs, tol 1e-6", "value": round(res["batched"][0], 5),
            "unit": "s", "higher_is_better": False, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "sequential_s": round(res["sequential"][0], 5),
            "batch_speedup": round(res["sequential"][0] / res["batched"][0], 3),
            "dtype": "f64 outer / f32 V-cycle", "data": "synthetic",
            "config": {"workload": "uneven multi-design batch", "designs": [list(m[2]) for m in members],
                       "total_dofs": dofs, "nit": nits,
                       "tuned": {"x".join(map(str, k)): {"nswp": v.nswp, "nswp_fine": v.nswp_fine, "nswp_coarse": v.nswp_coarse, "coarse_from": v.coarse_from, "sweep_xchunk": v.sweep_xchunk,
                                                         "tc_parts": v.tc_parts,
                                                         "tc_xchunk": v.tc_xchunk} for k, v in tuned.items()}}}
    print(json.dumps(line))


HOMOG = (128, 6)   # unit cell n^3, levels (coarsest grid 4^3)


def run_homog(args):
    """Batched periodic homogenization: a 128^3 unit cell whose density is a
    seeded Gaussian random field (correlation length 8 voxels) through a
    sigmoid to [1e-3, 1], SIMP moduli; the six unit-strain load cases solved
    as six right-hand sides to tol 1e-6 (FP32 V-cycle, flexible FP64 PCG, one
    graph launch per iteration of all six), then the 6x6 effective tensor.  A
    step is one whole homogenization (hierarchy setup, solve, C_eff)."""
    import torch

    import gputo
    torch.cuda.set_device(0)
    n, nl = HOMOG
    x = gputo.random_field_density(n, n, n, seed=2024, corr_len=8.0)
    CX = torch.as_tensor(1e-9 + x ** 3 * (1 - 1e-9), dtype=torch.float64, device="cuda")
    Ke = gputo.hex8_stiffness(0.3)
    h = gputo.Homog(n, n, n, nl)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            C, rr, nit = h.solve(Ke, CX, tol=TOL, maxit=MAXIT, stream=stream)
        torch.cuda.synchronize()
        clocks = ClockSampler(0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches0 = gputo.launch_count()
        with clocks:
            e0.record(stream)
            for _ in range(args.steps):
                C, rr, nit = h.solve(Ke, CX, tol=TOL, maxit=MAXIT, stream=stream)
            e1.record(stream)
            torch.cuda.synchronize()
    s = e0.elapsed_time(e1) / args.steps / 1000.0
    ndof = 3 * n ** 3
    line = {"metric": "s per homogenization (6 load cases, 128^3 cell, tol 1e-6)", "value": round(s, 5),
            "unit": "s", "higher_is_better": False, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "dtype": "f64 outer PCG / f32 V-cycle", "data": "synthetic: seeded Gaussian random field",
            "gpu_launches": int((gputo.launch_count() - launches0) / max(1, args.steps)),
            "dof_iters_per_s": round(6 * ndof * float(np.mean(nit)) / s, 1),
            "clocks": clocks.summary(),
            "config": {"workload": "periodic homogenization, 6 unit-strain load cases as 6 right-hand sides",
                       "cell": [n, n, n], "nl": nl, "ndof_per_case": ndof, "tol": TOL, "nit": nit.tolist(),
                       "relres": rr.tolist(), "Ceff": np.round(C, 8).tolist(),
                       "device_gb": round(h.device_bytes / 1e9, 2)}}
    print(json.dumps(line))


BRIDGE = (512, 256, 256, 7)   # nelx, nely, nelz, levels (coarsest grid 8x4x4)


def run_bridge(args):
    """The 512x256x256 bridge (101.6M dofs): supports on the two bottom corner
    strips, unit uniform top load, volume fraction 0.15 from a uniform start.
    Seconds per design iteration for the mixed and the FP64 solver; the
    reference cannot run this size (its int workspace counter overflows)."""
    import torch

    import gputo
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    nelx, nely, nelz, nl = BRIDGE
    F, fixed = gputo.bridge(nelx, nely, nelz)
    Ke0 = gputo.hex8_stiffness(0.3)
    out = {}
    with torch.cuda.stream(stream):
        clocks = ClockSampler(0)
        for name, prec, steps in (("mixed", gputo.PREC_MIXED, args.steps),
                                  ("fp64", gputo.PREC_FP64, max(1, args.steps // 2))):
            dl = gputo.DesignLoop(nelx, nely, nelz, nl, F, fixed, Ke0, volfrac=0.15, penal=PENAL, rmin=RMIN,
                                  move=MOVE, tol=TOL, maxit=MAXIT, options=gputo.default_options(precision=prec),
                                  stream=stream)
            x0 = dl.x.clone()
            infos = []

            def one():
                dl.x.copy_(x0)
                return dl.step()

            for _ in range(args.warmup):
                one()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ctx = clocks if name == "mixed" else _Null()
            with ctx:
                e0.record(stream)
                for _ in range(steps):
                    infos.append(one())
                e1.record(stream)
                torch.cuda.synchronize()
            out[name] = {"s": e0.elapsed_time(e1) / steps / 1000.0, "nit": infos[-1]["nit"],
                         "relres": infos[-1]["relres"], "c": infos[-1]["c"], "steps": steps,
                         "solver_bytes": dl.solver.device_bytes}
            del dl, x0
            torch.cuda.empty_cache()
    ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1)
    m = out["mixed"]
    line = {"metric": "s per design iteration, 512x256x256 bridge, tol 1e-6", "value": round(m["s"], 4),
            "unit": "s", "higher_is_better": False, "n_gpus": 1, "steps": m["steps"], "warmup": args.warmup,
            "fp64_s": round(out["fp64"]["s"], 4), "mixed_vs_fp64": round(out["fp64"]["s"] / m["s"], 3),
            "dtype": "f64 outer / f32 V-cycle", "data": "synthetic",
            "clocks": clocks.summary(),
            "config": {"workload": "bridge design iteration (filter, SIMP, MGCG solve to 1e-6, ce, OC)",
                       "nelx": nelx, "nely": nely, "nelz": nelz, "nl": nl, "ndof": ndof, "volfrac": 0.15,
                       "nit": {k: v["nit"] for k, v in out.items()},
                       "relres": {k: v["relres"] for k, v in out.items()},
                       "compliance": {k: v["c"] for k, v in out.items()},
                       "solver_gb": {k: round(v["solver_bytes"] / 1e9, 2) for k, v in out.items()},
                       "inputs_vs_l2": "inputs larger than L2"}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gputo", choices=["gputo", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--micro", choices=list(KERNELS) + ["all"], help="profiling aid: one kernel kind")
    ap.add_argument("--size", default=f"{NELX}x{NELY}x{NELZ}")
    ap.add_argument("--nl", type=int, default=NL)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--sweep-pairs", type=int, default=1, choices=[0, 1],
                    help="profiling aid: FP32 fine sweeps with two element columns per lane (1) or one (0)")
    ap.add_argument("--one-step", choices=["mixed", "fp64"], help="profiling aid: one design iteration")
    ap.add_argument("--nswp", type=int, default=0, help="profiling aid: V-cycle sweeps for --one-step (0: 3)")
    ap.add_argument("--nswp-coarse", type=int, default=0, help="with --one-step: sweeps from level --coarse-from on")
    ap.add_argument("--coarse-from", type=int, default=0, help="with --one-step: first level of --nswp-coarse (0: 2)")
    ap.add_argument("--nswp-fine", type=int, default=0,
                    help="with --one-step: Jacobi sweeps on the finest level (the autotuner's choice)")
    ap.add_argument("--workload", default="cantilever", choices=["cantilever", "batch", "bridge", "homog"],
                    help="batch: the uneven multi-design batch; bridge: the 512x256x256 bridge; homog: the "
                         "128^3 periodic homogenization (instead of the headline design loop)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "batch":
        run_batch(args)
    elif args.workload == "bridge":
        run_bridge(args)
    elif args.workload == "homog":
        run_homog(args)
    elif args.micro:
        run_micro(args)
    elif args.one_step:
        run_one_step(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
