"""Benchmark of the explicit unstructured FV step on one B200 (or N replicas).

Workload (default): Mach 3 forward-facing step, ~1.0M triangles from a seeded
Delaunay of a jittered lattice, second-order Green-Gauss + smooth-switch
limiter with Venkatakrishnan phi (K = 5), Roe flux, 5-stage RK, CFL 0.8,
global time step.  One bench step = one RK5 time step over the whole mesh.

Metric: cell-updates per second per RK stage = n_real * stages * steps / time.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun every rank runs an independent replica of the workload (the
single-GPU path has no data exchange); value = all ranks' cell updates /
max-over-ranks device time.  Prints one JSON line on rank 0.
"""
import argparse
import json
import os
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "finite-volume-2d-cpp_b200")
ORACLE = os.path.join(ROOT, "oracle")
for _p in (PKG, ORACLE):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

import meshgen  # noqa: E402
import physics as P  # noqa: E402

METRIC = "cell-updates/s per RK stage"
UNIT = "cell-updates/s"
# Algorithmic (unique compulsory) bytes per real cell and launch, V = 4,
# E/N = 1.5 edges per cell: the flux + update kernel reads the
# stage state, its (limited) gradients, centroid, area, edge data
# (2 indices + normal, length, face centre) and the FP64 base state, and
# writes the new state.  FP64_EXACT keeps the reference's separate limiter
# array (296 B); FP64 folds the limiter into the gradients; FP32
# stores stage states, gradients and geometry in FP32, the base in FP64, and
# writes the FP64 state on the last of the 5 stages only.
# The fused stage kernel (gradients, limiter, fluxes, update and ghost fill
# of a two-ring tile in one launch) reads the stage state, centroid and area,
# the edge data (2 indices + normal, length, face centre, Green-Gauss weight)
# and the FP64 base state, and writes the new state: FP64 32 + 24 + 1.5*56 +
# 32 + 32 = 204; FP32 16 + 12 + 1.5*32 + 32 + 16 + 32/5 = 130.4.  Its time
# step comes from the dt kernel, once per step (reads the state, area and
# edge indices + normal and length; writes dt).
ALGO_BYTES = {
    "fp64_exact": {"stage": 296.0, "grad_lim": 224.0, "stage_o1": 160.0, "dt": 96.0, "fused": 204.0},
    "fp64": {"stage": 256.0, "grad_lim": 192.0, "stage_o1": 160.0, "dt": 96.0, "fused": 204.0},
    "fp32": {"stage": 156.4, "grad_lim": 102.0, "stage_o1": 110.0, "dt": 58.0, "fused": 130.4},
}
# The diffusive kinds (same accounting, s = 8 or 4).
# Navier-Stokes (V = 4, MUSCL): the stage kernel reads q, the raw gradients
# and the limiter (kept apart in every mode), centroid, area, edges
# (2 indices + normal, length, face centre), q_base and the local dt, and
# writes q_new: FP64 32*4 + 16 + 8 + 1.5*44 + 32 + 8 + 32 = 290; FP32 16*4 +
# 8 + 4 + 1.5*24 + 32 + 8 + 16 + 32/5 = 174.4.  The gradient kernel reads q,
# centroid, area, edges (+ Green-Gauss weight) and writes gx, gy, lim:
# FP64 32 + 16 + 8 + 1.5*52 + 96 = 230; FP32 16 + 8 + 4 + 1.5*28 + 48 = 118.
# Diffusion (V = 1, no MUSCL): stage reads q, gx, gy (+ lim in FP64_EXACT),
# centroid, area, edges (2 indices + normal, length), q_base and writes
# q_new: FP64 8*3 + 16 + 8 + 1.5*28 + 8 + 8 = 106 (114 exact); FP32 4*3 + 8 +
# 4 + 1.5*16 + 8 + 4 + 8/5 = 61.6.  Its gradient kernel needs no face centres:
# FP64 8 + 16 + 8 + 1.5*36 + 24 = 110; FP32 4 + 8 + 4 + 1.5*20 + 12 = 58.
ALGO_BYTES_KIND = {
    "ns": {"fp64_exact": {"stage": 290.0, "grad_lim": 230.0}, "fp64": {"stage": 290.0, "grad_lim": 230.0},
           "fp32": {"stage": 174.4, "grad_lim": 118.0}},
    "diffusion": {"fp64_exact": {"stage": 114.0, "grad_lim": 110.0}, "fp64": {"stage": 106.0, "grad_lim": 110.0},
                  "fp32": {"stage": 61.6, "grad_lim": 58.0}},
}


def algo_bytes(ph, precision, kernel):
    kind = {"ns": "ns", "diffusion": "diffusion"}.get(ph.flux)
    if kind is not None:
        return ALGO_BYTES_KIND[kind][precision][kernel]
    if kernel == "stage" and not ph.order2:
        kernel = "stage_o1"
    return ALGO_BYTES[precision][kernel]


# DRAM bytes per real cell of one stage-kernel launch on the forward-step
# workload (dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture
# per precision mode), scaled by the cells of a launch; each entry names the
# capture it comes from.  Modes and workloads without a capture report null.
TRAFFIC_B_PER_CELL = {
    ("step", "fp32", "split"): (153.2, "ncu --set full -k regex:k_tile_stage -s 30 -c 2, "
                                       "bench.py --precision fp32 --steps 20 --warmup 3 --no-cpu-baseline"),
    ("step", "fp32", "fused"): (150.6, "ncu --set full -k regex:k_tile_fused -s 10 -c 2, bench.py --precision "
                                       "fp32 --steps 20 --warmup 3 --no-cpu-baseline --batch-steps 0"),
    ("step", "fp64", "fused"): (231.3, "ncu --set full -k regex:k_tile_fused -s 10 -c 2, bench.py --precision "
                                       "fp64 --steps 20 --warmup 3 --no-cpu-baseline --batch-steps 0"),
}


def build_workload(name):
    """(element mesh or list of case meshes, physics, RK stages, ic(mesh, geometry) -> q, description)"""
    if name == "step":
        em = meshgen.forward_step()
        ph = P.forward_step(order2=True, limiter="venkat", K=5.0, cfl=0.8)
        # the reference scheme goes non-finite at t ~ 0.005 on this mesh; the
        # positivity guard (MUSCL face states with rho <= 0 or p <= 0 fall
        # back to the cell value) keeps it physical to t ~ 0.025
        ph.positivity_guard = True
        return em, ph, P.RK5_ALPHA, lambda mesh, geo: P.ic_forward_step(mesh.n_total).ravel(), \
            "forward step Mach 3, 2nd-order GG + Venkatakrishnan K=5 + positivity guard, RK5, CFL 0.8"
    if name == "sod":
        em = meshgen.sod_strip(400, 40)
        return em, P.sod(cfl=0.5), P.RK1_ALPHA, lambda mesh, geo: P.ic_sod(geo["ccx"]).ravel(), \
            "Sod shock tube 400x40x2, 1st-order Roe, RK1, CFL 0.5"
    if name == "naca":
        em = meshgen.naca_ogrid()
        return em, P.naca(), P.RK5_ALPHA, lambda mesh, geo: P.ic_naca(mesh.n_total).ravel(), \
            "NACA 0012 O-grid 1024x512x2, M 0.8, Michalak, local dt, RK5"
    if name == "batch":
        nx, states = meshgen.riemann_strip_sizes()
        ems = [meshgen.riemann_strip(n) for n in nx]

        def ic(mesh, geo):
            ccx = mesh.split(geo["ccx"], 1)
            return mesh.join([P.ic_riemann(c, st[:3], st[3:]) for c, st in zip(ccx, states)], 4)

        return ems, P.riemann_strip(), P.RK5_ALPHA, ic, \
            (f"{len(ems)} independent Riemann strips (nx x 8 x 2 triangles, 2k-200k cells log-uniform, seed 4), "
             f"2nd-order GG + Venkatakrishnan K=5, RK5, CFL 0.8, per-case global dt, one batched solver")
    if name == "flatplate":
        # examples/flatPlate's domain and grading pattern at 1.0M quadrilaterals
        # CFL 1: at the example's CFL 2 the scheme goes non-finite on this mesh
        # (by step 60 in the reference's exact arithmetic)
        em = meshgen.flat_plate(nx0=100, nx1=900, ny=1000, r_up=1.02, r_plate=1.004, r_y=1.004)
        return em, P.flat_plate(cfl=1.0), P.RK5_ALPHA, \
            lambda mesh, geo: P.ic_forward_step(mesh.n_total, mach=0.2).ravel(), \
            ("flat plate M 0.2 (examples/flatPlate), 1000x1000 graded quads, Navier-Stokes, MUSCL + Michalak, "
             "local viscous dt, RK5, CFL 1")
    if name == "heat":
        em = meshgen.rect_tri(708, 708, 1.0, 1.0, side_names=("wall", "wall"))
        return em, P.heat(dt=2e-7), P.RK5_ALPHA, lambda mesh, geo: P.ic_heat(geo["ccx"], geo["ccy"]).ravel(), \
            "heat equation (examples/heatTransfer), 708x708x2 triangles, diffusion flux with face gradients, RK5"
    raise SystemExit(f"unknown workload {name}")


# reference build, boundary aliases and constants timed as the CPU baseline of a workload
REF_FOR = {"step": ("forwardStep_o2venk5", {"step": "wall"}, dict(cfl=0.8)),
           "flatplate": ("flatPlate", {}, {}),
           "heat": ("heatTransfer", {}, {})}


def make_mesh(em):
    import fvgpu
    if isinstance(em, list):
        return fvgpu.Mesh.batch([fvgpu.Mesh.from_elements(e) for e in em])
    return fvgpu.Mesh.from_elements(em)


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled through NVML every
    few milliseconds while the timed region runs."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, index, period_s=0.005):
        self.index = index
        self.period = period_s
        self.sm, self.reasons = [], set()
        self.max_sm = None
        self._stop = threading.Event()

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_sm = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.thread = threading.Thread(target=self._loop, daemon=True)
            self.thread.start()
        except Exception:
            self.nv = None
        return self

    def _sample(self):
        nv = self.nv
        self.sm.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
        try:
            r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        except AttributeError:
            r = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
        for name, bit in self.REASONS.items():
            if r & bit:
                self.reasons.add(name)

    def _loop(self):
        while not self._stop.is_set():
            try:
                self._sample()
            except Exception:
                return
            time.sleep(self.period)

    def __exit__(self, *a):
        self._stop.set()
        if self.nv is not None:
            self.thread.join(timeout=2)
            try:
                self._sample()  # at least one sample at the end of the region
            except Exception:
                pass

    def summary(self):
        if not self.sm:
            return {"sm_mhz": None, "sm_max_mhz": self.max_sm, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(self.sm)), "sm_max_mhz": self.max_sm,
                "reasons": sorted(self.reasons), "samples": len(self.sm)}


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# --------------------------------------------------------------- reference --
def _ref_worker(args):
    """One single-rank reference process (spawned): K RK1 steps on the mesh
    from the example's own initial state (generate_initial_solution)."""
    variant, base, consts, aliases, n_total, warmup, steps = args
    from oracle import RefLib
    ref = RefLib(variant)
    for name, src in aliases.items():
        ref.bc_set(name, ref.bc_get(src))
    ref.set_consts(**consts)
    if ref.lib.ref_read_mesh(base.encode()) != 0:
        raise RuntimeError("reference reader failed")
    s = np.zeros(5, np.int64)
    import ctypes
    ref.lib.ref_mesh_sizes(s.ctypes.data_as(ctypes.c_void_p))
    ref.n_nodes, ref.n_real, ref.n_total, ref.n_edges, ref.n_bound = (int(x) for x in s)
    ref.nq = ref.V * ref.n_total
    q0 = ref.initial_state()
    r = ref.run_loop(q0, P.RK1_ALPHA, max(warmup, 1))
    t0 = time.perf_counter()
    ref.run_loop(r["q"], P.RK1_ALPHA, steps)
    return time.perf_counter() - t0, ref.n_real


def reference_samples(em, procs, warmup, steps, workload="step"):
    """Times the reference library (oracle/_ref, built from the reference's
    own sources) on a workload's mesh in `procs` independent single-rank
    processes.  Returns (cell-updates/s aggregate, n_real) or None."""
    import multiprocessing as mp
    from oracle import ref_available
    variant, aliases, consts = REF_FOR[workload]
    if not ref_available(variant):
        return None
    tmp = tempfile.mkdtemp(prefix="fvbench_")
    base = os.path.join(tmp, "mesh")
    meshgen.write_msh41(base + ".msh", em)
    job = (variant, base, consts, aliases, 0, warmup, steps)
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_ref_worker, [job] * procs)
    t = max(r[0] for r in res)
    n = res[0][1]
    return procs * n * steps / t, n


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    em, ph, alpha, ic, desc = build_workload("step")
    procs = os.cpu_count() or 1
    r = reference_samples(em, procs, args.warmup, args.steps)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built (reference sources absent when building)"}))
        return
    value, n = r
    sample = (f"{procs} independent single-rank processes of the reference library (no MPI on the box), "
              f"each {args.steps} single-stage steps (calc_dt + complete_calc_qt + update_cells + update_bounds) "
              f"of the {n}-cell forward step after {args.warmup} warm-up steps")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "n_real_cells": n, "parallelism": f"{procs} host processes"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "same_config": False,
            "comparability": ("the same mesh, physics and metric as the GPU arm (cell-updates per RK stage), but "
                              "each timed step is one single-stage step of the reference's stage functions, so "
                              "calc_dt runs once per stage instead of once per 5-stage step (1-2 % of its time); "
                              "the reference scheme has no positivity guard; the processes are independent "
                              "replicas (an upper bound of MPI scaling on these cores)")}
    print(json.dumps(line))


# ---------------------------------------------------------------- our arm --
def measure_mode(args, em, mesh, geo, ph, alpha, ic, precision, local, dist, world):
    """Times args.steps time steps of one precision mode (device resident)."""
    import torch
    import fvgpu

    q0 = ic(mesh, geo)
    if args.tile_cells < 0:  # autotuned tile size
        s = fvgpu.Solver.create_tuned(mesh, ph, precision, q0, alpha=alpha, steps=3, device=local)
    else:
        s = fvgpu.Solver(mesh, ph, precision, device=local, tile_cells=args.tile_cells,
                         stage_kernels=args.stage_kernels, schedule=args.schedule)
        s.tile_cells = args.tile_cells or 128
    # hybrid: the split kernels for the first stage, the fused kernel for the
    # other four (the dominant kernel)
    fused = s.stage_kernels in ("fused", "hybrid")
    stream = torch.cuda.Stream(device=local)
    s.set_stream(stream.cuda_stream)
    s.set_state(q0)
    stages = len(alpha)
    N = mesh.n_real
    s.run(args.warmup, alpha=alpha)  # warm-up, also captures the step graphs

    def barrier():
        if dist is not None:
            dist.barrier()

    barrier(); torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True); ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        info = s.run(args.warmup + args.steps, alpha=alpha, restart=False)
        ev1.record(stream)
        ev1.synchronize()
    barrier(); torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    if info["step"] != args.warmup + args.steps:
        raise SystemExit(f"{precision}: run stopped at step {info['step']} (R = {info['R']}): "
                         f"state check {s.check_state()}")
    launches = s.last_run_stats()[1]  # kernels launched inside the timed region
    import replicas
    ms_max = replicas.max_over_ranks(ms, dist, device=f"cuda:{local}")
    out = dict(solver=s, stream=stream, value=world * N * stages * args.steps / (ms_max / 1e3),
               ms_per_step=ms_max / args.steps, launches=int(launches), clocks=clk.summary(),
               state_finite=s.check_state() == 0, q_final=s.get_state(), case_times=s.case_times())
    # per-kernel device timing (events around every kernel, same stream)
    prof_steps = max(2, min(args.steps, 10))
    ms_k = np.zeros(6); cnt_k = np.zeros(6, np.int64)
    a = np.ascontiguousarray(alpha, np.float64)
    import ctypes as C
    fvgpu._check(fvgpu.lib().fv_profile_kernels(s._h, a.ctypes.data_as(C.POINTER(C.c_double)), C.c_int32(a.size),
                                                C.c_int32(prof_steps), ms_k.ctypes.data_as(C.POINTER(C.c_double)),
                                                cnt_k.ctypes.data_as(C.POINTER(C.c_int64))))
    kinds = ["step_begin", "dt", "grad_lim", "stage", "step_end", "fused"]
    out["per_launch_ms"] = {kinds[k]: (ms_k[k] / cnt_k[k] if cnt_k[k] else 0.0) for k in range(6)}
    out["share"] = {kinds[k]: float(ms_k[k] / ms_k.sum()) for k in range(6)}
    peak, peak_kind = measured_peak_hbm()
    kb = (ALGO_BYTES[precision]["fused"] if fused else algo_bytes(ph, precision, "stage")) * N
    achieved = kb / (out["per_launch_ms"]["fused" if fused else "stage"] / 1e3) / 1e9
    out["stage_kernels"] = s.stage_kernels
    out["schedule"] = s.schedule
    kname = ("gradients + limiter + flux + RK update + ghost fill of a two-ring tile (k_tile_fused)" if fused
             else "flux + RK update + ghost fill (k_tile_stage)")
    out["roofline"] = {"bound": "hbm", "kernel": kname,
                       "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                       "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                       "traffic": None, "traffic_source": "no ncu capture of this mode and workload",
                       "algorithmic_bytes_per_launch": kb}
    cap = TRAFFIC_B_PER_CELL.get((args.workload, precision, "fused" if fused else "split"))
    if cap is not None:
        out["roofline"]["traffic"] = cap[0] * N
        out["roofline"]["traffic_source"] = ("dram__bytes_read.sum + dram__bytes_write.sum per launch of the "
                                             "stage kernel, from: " + cap[1])
    if (ph.order2 or ph.diffusive) and not fused:
        kg = algo_bytes(ph, precision, "grad_lim") * N
        out["roofline_grad_lim"] = {"achieved": kg / (out["per_launch_ms"]["grad_lim"] / 1e3) / 1e9,
                                    "frac": kg / (out["per_launch_ms"]["grad_lim"] / 1e3) / 1e9 / peak}
    if out["per_launch_ms"]["dt"] > 0 and ph.V == 4:
        kd = ALGO_BYTES[precision]["dt"] * N
        out["roofline_dt"] = {"achieved": kd / (out["per_launch_ms"]["dt"] / 1e3) / 1e9,
                              "frac": kd / (out["per_launch_ms"]["dt"] / 1e3) / 1e9 / peak}
    return out


def e2e_mode(args, mesh, ph, alpha, m, local, dist, world):
    """Same metric through the C ABI with pinned host buffers: every step
    uploads a state from pinned host memory, runs one time step on it and
    reads the result back to pinned host memory.

    Pipelined (the reported figure): the upload of step k+1 and the read-back
    of step k-1 run on their own copy streams while step k computes
    (fv_set_state_device / fv_run / fv_get_state_device on the solver's
    stream, double-buffered device inputs and outputs).  Serial (reported
    beside it): upload, step and read-back one after the other with the
    blocking host-pointer calls.  Both produce the same output, checked."""
    import torch

    s = m["solver"]
    stream = m["stream"]
    nq = mesh.n_total * ph.V
    state = s.get_state()
    e2e_steps = max(3, min(args.steps, 50))
    s.set_chunk(1)
    s.set_state(state)
    s.run(1, alpha=alpha)  # builds the one-step graph outside the timed region
    import replicas
    dev = f"cuda:{local}"

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- serial
    h_in = torch.from_numpy(state.copy()).pin_memory()
    h_out = torch.empty(nq, dtype=torch.float64).pin_memory()
    barrier()
    t0 = time.perf_counter()
    for k in range(e2e_steps):
        s.set_state_ptr(h_in.data_ptr(), device=False)
        s.run(k + 1, alpha=alpha, restart=(k == 0))
        s.get_state_ptr(h_out.data_ptr(), device=False)
    torch.cuda.synchronize()
    wall_serial = time.perf_counter() - t0
    serial_out = h_out.numpy().copy()
    # ---- pipelined
    hi = [torch.from_numpy(state.copy()).pin_memory() for _ in range(2)]
    ho = [torch.empty(nq, dtype=torch.float64).pin_memory() for _ in range(2)]
    di = [torch.empty(nq, dtype=torch.float64, device=dev) for _ in range(2)]
    do = [torch.empty(nq, dtype=torch.float64, device=dev) for _ in range(2)]
    up, down = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
    in_ready = [torch.cuda.Event() for _ in range(2)]
    in_free = [torch.cuda.Event() for _ in range(2)]
    out_ready = [torch.cuda.Event() for _ in range(2)]
    out_free = [torch.cuda.Event() for _ in range(2)]
    used_in = [False, False]
    used_out = [False, False]
    barrier()
    t0 = time.perf_counter()
    with torch.cuda.stream(up):
        di[0].copy_(hi[0], non_blocking=True)
        in_ready[0].record(up)
    for k in range(e2e_steps):
        j = k % 2
        if k + 1 < e2e_steps:
            with torch.cuda.stream(up):
                if used_in[1 - j]:
                    up.wait_event(in_free[1 - j])
                di[1 - j].copy_(hi[1 - j], non_blocking=True)
                in_ready[1 - j].record(up)
        stream.wait_event(in_ready[j])
        s.set_state_ptr(di[j].data_ptr(), device=True)
        in_free[j].record(stream)
        used_in[j] = True
        s.run(k + 1, alpha=alpha, restart=(k == 0))
        if used_out[j]:
            stream.wait_event(out_free[j])
        s.get_state_ptr(do[j].data_ptr(), device=True)
        out_ready[j].record(stream)
        with torch.cuda.stream(down):
            down.wait_event(out_ready[j])
            ho[j].copy_(do[j], non_blocking=True)
            out_free[j].record(down)
        used_out[j] = True
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    same = bool(np.array_equal(ho[(e2e_steps - 1) % 2].numpy(), serial_out, equal_nan=True))
    s.set_chunk(16)
    cells = mesh.n_real * len(alpha) * e2e_steps
    return {"value": replicas.job_throughput(cells, wall, dist, dev), "unit": UNIT,
            "h2d_bytes_per_step": nq * 8, "d2h_bytes_per_step": nq * 8, "steps": e2e_steps,
            "mode": "pipelined: upload of step k+1 and read-back of step k-1 overlap step k",
            "serial_value": replicas.job_throughput(cells, wall_serial, dist, dev),
            "pipelined_output_equals_serial": same}


def err_rho_p(q, q_ref, n_real, gamma=1.4):
    """Relative L1 and L2 errors of density and pressure over the real cells."""
    a = q.reshape(-1, 4)[:n_real]; b = q_ref.reshape(-1, 4)[:n_real]

    def rp(x):
        return x[:, 0], (gamma - 1) * (x[:, 3] - 0.5 * (x[:, 1] ** 2 + x[:, 2] ** 2) / x[:, 0])

    (ra, pa), (rb, pb) = rp(a), rp(b)
    l1 = lambda u, v: float(np.sum(np.abs(u - v)) / np.sum(np.abs(v)))
    l2 = lambda u, v: float(np.sqrt(np.sum((u - v) ** 2) / np.sum(v ** 2)))
    return {"density": {"l1": l1(ra, rb), "l2": l2(ra, rb)}, "pressure": {"l1": l1(pa, pb), "l2": l2(pa, pb)}}


def exact_run_state(mesh, geo, ph, alpha, ic, steps, local):
    """The FP64_EXACT path's state after `steps` time steps: the reference's
    FP64 arithmetic, bit for bit (the oracle restates the positivity guard,
    which the reference does not have, the same way)."""
    import fvgpu
    s = fvgpu.Solver(mesh, ph, "fp64_exact", device=local)
    s.set_state(ic(mesh, geo))
    info = s.run(steps, alpha=alpha, print_interval=10 ** 9)
    q = s.get_state()
    s.close()
    return q, info["step"]


def run_batch_modes(args, local, dist, world):
    """The batched Riemann-strip workload (256 strips of 2k-200k cells in one
    solver, autotuned tile size, 500 RK5 steps) in FP32-bulk and plain FP64:
    cell-updates/s per stage and the L2 error against the exact Riemann
    solution."""
    import copy
    ba = copy.copy(args)
    ba.workload, ba.steps, ba.warmup, ba.tile_cells = "batch", args.batch_steps, 3, -1
    em, ph, alpha, ic, desc = build_workload("batch")
    mesh = make_mesh(em)
    geo = mesh.geometry()
    res = {prec: measure_mode(ba, em, mesh, geo, ph, alpha, ic, prec, local, dist, world) for prec in ("fp64", "fp32")}
    _, states = meshgen.riemann_strip_sizes()
    out = {"workload": desc, "n_real_cells": mesh.n_real, "n_cases": mesh.n_cases, "steps": ba.steps}
    for prec, r in res.items():
        out[prec] = {"value": r["value"], "ms_per_step": r["ms_per_step"], "tile_cells": r["solver"].tile_cells,
                     "stage_kernels": r["stage_kernels"], "schedule": r["schedule"],
                     "stage_roofline_frac": r["roofline"]["frac"],
                     "l2_error_vs_exact_riemann": batch_error_vs_exact(mesh, geo, r["q_final"], r["case_times"], states),
                     "state_finite": bool(r["state_finite"]), "clocks": r["clocks"]}
        r["solver"].close()
    out["fp32_speedup_over_fp64"] = out["fp32"]["value"] / out["fp64"]["value"]
    out["fp32_minus_fp64_density_error"] = (out["fp32"]["l2_error_vs_exact_riemann"]["density"]
                                            - out["fp64"]["l2_error_vs_exact_riemann"]["density"])
    return out


def batch_error_vs_exact(mesh, geo, q, times, states, gamma=1.4):
    """L2 density / pressure error of a batch of Riemann strips against the
    exact Riemann solution at each case's own time, area-weighted over all
    real cells of the batch, and the worst case."""
    import riemann
    qs = mesh.split(q, 4)
    ccx = mesh.split(geo["ccx"], 1)
    area = mesh.split(geo["area"], 1)
    ro, _ = mesh.case_offsets()
    num_r = num_p = den = 0.0
    worst = 0.0
    for k in range(len(qs)):
        n = int(ro[k + 1] - ro[k])
        x, A = ccx[k][:n], area[k][:n]
        ra, _, pa = riemann.sample(x, times[k], states[k][:3], states[k][3:], gamma)
        qq = qs[k].reshape(-1, 4)[:n]
        r = qq[:, 0]
        p = (gamma - 1) * (qq[:, 3] - 0.5 * (qq[:, 1] ** 2 + qq[:, 2] ** 2) / r)
        er, ep = float(((r - ra) ** 2 * A).sum()), float(((p - pa) ** 2 * A).sum())
        num_r += er; num_p += ep; den += float(A.sum())
        worst = max(worst, np.sqrt(er / A.sum()))
    return {"density": float(np.sqrt(num_r / den)), "pressure": float(np.sqrt(num_p / den)),
            "density_worst_case": float(worst)}


def run_adjoint_workload(args):
    """Discrete adjoint of the forward step at 250k cells: 500 RK5 steps,
    loss = time integral of the pressure force on the step face, gradient
    with respect to the inflow Mach number and 64 inflow density bins
    (delta ~ N(0, 0.01), seed 5), checkpoints every 50 steps; checked
    against central finite differences (h = 1e-6) on a few components."""
    import fvgpu

    em = meshgen.forward_step(n=220)
    # CFL 0.5: at CFL 0.8 the reference scheme's cell pressure at the step
    # corner goes negative near t = 0.037 (step 400 of 500 at this size)
    ph = P.forward_step(order2=True, limiter="venkat", K=5.0, cfl=0.5)
    ph.positivity_guard = True
    mesh = fvgpu.Mesh.from_elements(em)
    nb = 64
    import torch
    torch.cuda.init()
    free0 = torch.cuda.mem_get_info(0)[0]
    adj = fvgpu.Adjoint(mesh, ph, n_steps=args.steps, checkpoint_every=50, n_bins=nb)
    # the adjoint allocates everything it uses at creation
    adj_bytes = free0 - torch.cuda.mem_get_info(0)[0]
    theta = np.concatenate([[3.0], np.random.default_rng(5).normal(0.0, 0.01, nb)])
    for _ in range(max(1, args.warmup - 2)):
        adj.loss(theta)
    t0 = time.perf_counter(); L = adj.loss(theta); t_fwd = time.perf_counter() - t0
    t0 = time.perf_counter(); L2, g = adj.gradient(theta); t_grad = time.perf_counter() - t0
    def fd(i, h):
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h; tm[i] -= h
        return (adj.loss(tp) - adj.loss(tm)) / (2 * h)

    # the loss is piecewise smooth (limiter min/max, dt arg-min, guard): the
    # adjoint is the derivative of the code path taken, central differences
    # converge to it as h shrinks past the nearest kink
    checks = {"mach": {f"h={h:g}": {"adjoint": float(g[0]), "fd": fd(0, h),
                                    "rel_error": abs(float(g[0]) - fd(0, h)) / abs(fd(0, h))}
                       for h in (1e-5, 1e-6, 1e-7, 1e-8)}}
    # kink scan: one-sided slopes of the loss over M in steps of 2e-7 around
    # theta; an interval whose slope departs from the adjoint holds a kink
    step, K = 2e-7, 8
    Ls = [adj.loss(np.concatenate([[theta[0] + k * step], theta[1:]])) for k in range(-K, K + 1)]
    slopes = np.diff(Ls) / step
    rel = np.abs(slopes - float(g[0])) / abs(float(g[0]))
    checks["mach_kink_scan"] = {
        "step": step, "intervals": [[(k - K) * step, (k - K + 1) * step] for k in range(2 * K)],
        "slope_rel_error_vs_adjoint": rel.tolist(),
        "kink_intervals": [[(k - K) * step, (k - K + 1) * step] for k in range(2 * K) if rel[k] > 1e-6],
        "intervals_adjacent_to_theta_match_1e-6": bool(min(rel[K - 1], rel[K]) <= 1e-6)}
    top = [1 + int(i) for i in np.argsort(-np.abs(g[1:]))[:3]]
    checks["density_bins"] = {str(i - 1): {"adjoint": float(g[i]), "fd_h=1e-6": fd(i, 1e-6)} for i in top}
    cell_stages = mesh.n_real * 5 * args.steps
    line = {"metric": "cell-updates/s per RK stage (adjoint: forward + reverse sweep)",
            "value": cell_stages / t_grad, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * t_grad / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "adjoint of the forward step, 2nd-order GG + Venkatakrishnan K=5 + positivity "
                                   "guard, RK5, CFL 0.5; loss = time-integrated pressure force on the step face; "
                                   "theta = inflow Mach + 64 inflow density bins; checkpoints every 50 steps",
                       "n_real_cells": mesh.n_real, "n_params": 1 + nb},
            "forward_seconds": t_fwd, "gradient_seconds": t_grad, "loss": L, "loss_repeat_equal": L == L2,
            "device_memory_bytes": int(adj_bytes),
            "gradient_norm": float(np.linalg.norm(g)), "max_abs_density_bin_gradient": float(np.abs(g[1:]).max()),
            "fd_check": checks}
    print(json.dumps(line))
    adj.close()


def measure_decomposed(args, mesh, geo, ph, alpha, ic, prec, parts_per_gpu, local, dist, world, rank, steps,
                       timeout_ms=0.0, compare_single=False):
    """Times `steps` time steps of the workload as a domain decomposition
    (fv_group_*): n_parts = processes x parts_per_gpu parts, each a contiguous
    Hilbert range with a two-ring halo, one halo exchange of the stage state
    per RK stage (NCCL between processes, device reads between the parts of
    one process), dt minimum and residual sums by all-gather.  Strong
    scaling: the whole job is one mesh.  compare_single (one process): the
    single solver on the same steps, its time and whether the states agree
    bit for bit."""
    import torch
    import fvgpu
    import replicas

    q0 = ic(mesh, geo)
    n_parts = world * parts_per_gpu
    nid = None
    if world > 1:
        box = [fvgpu.nccl_id() if rank == 0 else None]
        dist.broadcast_object_list(box, src=0)
        nid = box[0]
        dist.barrier()
    grp = fvgpu.Group(mesh, ph, prec, n_parts=n_parts, rank=rank, n_ranks=world, nccl_id_bytes=nid, device=local,
                      serial_exchange=args.serial_exchange, timeout_ms=timeout_ms, transport=args.transport)
    try:
        grp.set_state(q0)
        grp.run(args.warmup, alpha=alpha)
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            info = grp.run(args.warmup + steps, alpha=alpha, restart=False)
        ms, launches = grp.last_run_stats()
        if info["step"] != args.warmup + steps:
            raise RuntimeError(f"decomposed run stopped at step {info['step']}")
        ms_max = replicas.max_over_ranks(ms, dist, device=f"cuda:{local}")
        gi = grp.info()
        cell_bytes = 4 * (4 if prec == "fp32" else 8)
        out = {"value": mesh.n_real * len(alpha) * steps / (ms_max / 1e3), "unit": UNIT, "ms_per_step": ms_max / steps,
               "steps": steps, "n_parts": n_parts, "precision": prec, "gpu_launches": int(launches),
               "clocks": clk.summary(), "rank_parts": gi, "halo_bytes_per_stage": gi["halo_cells"] * cell_bytes,
               "exchange": ("inside each stage launch: band tiles wait for their senders, store into the "
                            "readers' buffers and release an epoch, beside the interior tiles"
                            if gi["transport"] == "p2p" and ph.order2 else
                            "after all tiles" if args.serial_exchange else
                            "band tiles + exchange on a second stream beside the interior tiles"),
               "transport": gi["transport"],
               "parallelism": (f"{n_parts} parts over {world} processes (NCCL)" if world > 1
                               else f"{n_parts} parts on one GPU (device reads)")}
        if compare_single:
            s = fvgpu.Solver(mesh, ph, prec, device=local)
            s.set_state(q0)
            s.run(args.warmup, alpha=alpha)
            torch.cuda.synchronize()
            s.run(args.warmup + steps, alpha=alpha, restart=False)
            ms1, _ = s.last_run_stats()
            q1 = s.get_state()
            s.close()
            q = grp.get_state()
            out["single_solver"] = {"value": mesh.n_real * len(alpha) * steps / (ms1 / 1e3),
                                    "ms_per_step": ms1 / steps, "stage_kernels": "hybrid",
                                    "decomposition_time_ratio": ms / ms1,
                                    "states_bit_identical": q.tobytes() == q1.tobytes()}
        return out
    finally:
        grp.close()


def run_decomposed_workload(args):
    """The forward-step workload as a domain decomposition; one JSON line."""
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    em, ph, alpha, ic, desc = build_workload("step")
    mesh = make_mesh(em)
    geo = mesh.geometry()
    prec = "fp32" if args.precision == "all" else args.precision
    d = measure_decomposed(args, mesh, geo, ph, alpha, ic, prec, args.parts_per_gpu, local, dist, world, rank,
                           args.steps, timeout_ms=120000.0, compare_single=(world == 1))
    if rank == 0:
        line = {"metric": METRIC, "value": d["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": d["ms_per_step"], "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f32+f64" if prec == "fp32" else "f64",
                "data": "synthetic",
                "config": {"workload": desc + ", domain decomposition", "n_real_cells": mesh.n_real,
                           "n_parts": d["n_parts"], "precision": prec, "exchange": d["exchange"],
                           "parallelism": d["parallelism"],
                           "l2": "inputs larger than L2 (working set > 126 MB), no flush"},
                "transport": d["transport"],
                "gpu_launches": d["gpu_launches"], "clocks": d["clocks"], "rank0_parts": d["rank_parts"],
                "halo_bytes_per_stage_rank0": d["halo_bytes_per_stage"]}
        if "single_solver" in d:
            line["single_solver"] = d["single_solver"]
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="step",
                    choices=["step", "sod", "naca", "batch", "adjoint", "flatplate", "heat", "decomposed"])
    ap.add_argument("--parts-per-gpu", type=int, default=None,
                    help="decomposed workload: parts per process (default 4 on one GPU, else 1)")
    ap.add_argument("--transport", default="copy", choices=["copy", "p2p"],
                    help="decomposed workload: halo states by NCCL between processes and device reads within "
                         "one (copy), or stored straight into the reading part's memory with epoch flags (p2p)")
    ap.add_argument("--serial-exchange", action="store_true",
                    help="decomposed workload: halo exchange after all tiles of a stage (default: beside "
                         "the interior tiles)")
    ap.add_argument("--precision", default="all", choices=["all", "fp64_exact", "fp64", "fp32"],
                    help="all: FP32-bulk (headline) and plain FP64 in one line")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--stage-kernels", default="auto", choices=["auto", "split", "fused", "hybrid"],
                    help="second-order Euler stage kernels: fused (one per stage) where the physics allow, "
                         "or split gradient and flux kernels")
    ap.add_argument("--schedule", default="tile", choices=["tile", "worklist", "tile2"],
                    help="fused stage kernel: one CTA per tile, resident CTAs taking tiles from a work list, "
                         "or one CTA of two threads per cell per tile")
    ap.add_argument("--batch-steps", type=int, default=500,
                    help="steps of the batched Riemann-strip workload reported beside the forward step "
                         "(0: not run)")
    ap.add_argument("--tile-cells", type=int, default=None,
                    help="cells per tile: 64/128/256, 0 = library default (128), -1 = autotuned "
                         "(default: autotuned for the batch workload, else 0)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.tile_cells is None:
        args.tile_cells = -1 if args.workload == "batch" else 0
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import fvgpu

    if args.workload == "adjoint":
        return run_adjoint_workload(args)
    if args.workload == "decomposed":
        if args.parts_per_gpu is None:
            args.parts_per_gpu = 4 if int(os.environ.get("WORLD_SIZE", "1")) == 1 else 1
        return run_decomposed_workload(args)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    em, ph, alpha, ic, desc = build_workload(args.workload)
    mesh = make_mesh(em)
    geo = mesh.geometry()
    modes = ["fp64", "fp32"] if args.precision == "all" else [args.precision]
    res = {}
    for prec in modes:
        res[prec] = measure_mode(args, em, mesh, geo, ph, alpha, ic, prec, local, dist, world)
    head = modes[-1]  # FP32-bulk when both run
    m = res[head]
    e2e = e2e_mode(args, mesh, ph, alpha, m, local, dist, world)
    # the plain FP64 mode end to end as well (the same host transfers)
    e2e_other = {p: e2e_mode(args, mesh, ph, alpha, r, local, dist, world) for p, r in res.items() if p != head}
    batch_line = None
    if args.workload == "step" and args.batch_steps > 0:
        # every rank takes the same steps (replicas under torchrun)
        batch_line = run_batch_modes(args, local, dist, world)
    decomposed = None
    if args.workload == "step" and world > 1:
        # the same mesh split over the ranks (strong scaling), beside the
        # replicas; a rank that fails ends the others' waits within the limit
        try:
            decomposed = measure_decomposed(args, mesh, geo, ph, alpha, ic, head, 1, local, dist, world, rank,
                                            min(args.steps, 200), timeout_ms=60000.0)
        except Exception as e:  # reported in the line, the replica figures stand
            decomposed = {"error": str(e)[:300]}
    if rank == 0:
        line = {"metric": METRIC, "value": m["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": m["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if head == "fp32" else "f64",
                "data": "synthetic",
                "config": {"workload": desc, "n_real_cells": mesh.n_real, "n_edges": mesh.n_edges,
                           "stages": len(alpha), "precision": head, "n_cases": mesh.n_cases,
                           "tile_cells": m["solver"].tile_cells,
                           "tile_choice": "autotuned" if args.tile_cells < 0 else "fixed",
                           "l2": "inputs larger than L2 (working set > 126 MB), no flush",
                           "parallelism": f"{world} independent replicas" if world > 1 else "single GPU"},
                "e2e": e2e, "gpu_launches": m["launches"], "roofline": m["roofline"],
                "kernel_ms_per_launch": m["per_launch_ms"], "kernel_time_share": m["share"],
                "clocks": m["clocks"], "state_finite": bool(m["state_finite"])}
        line["modes"] = {p: {"value": r["value"], "ms_per_step": r["ms_per_step"], "roofline_frac": r["roofline"]["frac"],
                             "e2e": e2e if p == head else e2e_other.get(p),
                             "stage_kernels": r["stage_kernels"], "schedule": r["schedule"], "schedule": r["schedule"],
                             "grad_lim_frac": r.get("roofline_grad_lim", {}).get("frac"),
                             "dt_frac": r.get("roofline_dt", {}).get("frac"),
                             "kernel_ms_per_launch": r["per_launch_ms"], "clocks": r["clocks"],
                             "state_finite": bool(r["state_finite"])} for p, r in res.items()}
        if "fp64" in res and "fp32" in res and ph.V == 4:
            line["fp32_vs_fp64"] = {"speedup": res["fp32"]["value"] / res["fp64"]["value"]}
            if args.workload in ("step", "naca", "sod"):
                # both modes against the FP64_EXACT run of the same steps
                q_ex, n_ex = exact_run_state(mesh, geo, ph, alpha, ic, args.warmup + args.steps, local)
                line["error_vs_fp64_exact"] = {
                    "reference": "FP64_EXACT path (the reference's FP64 arithmetic bit for bit), same mesh, "
                                 "same initial state, same steps",
                    "after_steps": n_ex,
                    "fp32": err_rho_p(res["fp32"]["q_final"], q_ex, mesh.n_real),
                    "fp64": err_rho_p(res["fp64"]["q_final"], q_ex, mesh.n_real)}
        if args.workload == "batch":
            _, states = meshgen.riemann_strip_sizes()
            errs = {p: batch_error_vs_exact(mesh, geo, r["q_final"], r["case_times"], states) for p, r in res.items()}
            line["l2_error_vs_exact_riemann"] = errs
            if "fp64" in errs and "fp32" in errs:
                line["l2_error_vs_exact_riemann"]["fp32_minus_fp64_density"] = \
                    errs["fp32"]["density"] - errs["fp64"]["density"]
        if args.workload == "step" and args.batch_steps > 0:
            line["modes"]["batch"] = batch_line
        if decomposed is not None:
            line["decomposed"] = decomposed
        if not args.no_cpu_baseline and world == 1 and args.workload in REF_FOR:
            r = reference_samples(em, 1, 1, 25, args.workload)
            if r is not None:
                line["cpu_baseline"] = {"value": r[0], "unit": UNIT, "cores": 1, "kind": "reference",
                                        "sample": f"reference library (built from its sources, "
                                                  f"{REF_FOR[args.workload][0]}), 1 process, "
                                                  f"25 single-stage steps of the {r[1]}-cell mesh"}
        print(json.dumps(line))
    for r in res.values():
        r["solver"].close()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
