"""Benchmark: s/timestep of the ElmGMR + memLS hot path on a 4M-tet cylinder.

Workload (one "step" = one time step, itrdrv_iter_step): a 4.0M-tet jittered
cylinder (R = 1 cm, L = 10 cm, 80x80 cross-section masked to the disc, 133
layers, 6 tets per hex), pulsatile parabolic inflow 10 + 5 sin(2 pi t / 0.8)
cm/s, one RCR outlet (Rp = 100, C = 1e-4, Rd = 1000), rho = 1.06, mu = 0.04,
dt = 1e-3 s, 3 nonlinear iterations (ElmGMR + memLS NS solve + correct) per
step.  Inputs are synthetic and seeded.

Both arithmetic modes run on the same workload from the same initial state:
plain FP64 (memLS's arithmetic, the ``fp64`` object) and the mixed-precision
NS solve (FP32 matrices in the inner Krylov matvecs, FP64 refinement), which
is the headline ``value``; ``mixed_rel_err_vs_fp64`` compares their velocity
and pressure fields after the same number of steps.

Multi-GPU: the path does not shard (one GPU, no domain decomposition), so
``--gpus N`` under torchrun runs N independent replicas; time is the max over
ranks and ``value`` counts every rank's time steps (weak scaling).

``--impl reference`` times the CPU oracle (the reference algorithm restated
in C++, all host threads) on the same workload: one complete time step
(predict, 3 x [ElmGMR + SolFlow pack + full memLS NS solve + correct], RCR
update), measured, is the value; each of the W + K timed steps is a bounded
sample (one full-size ElmGMR + pack) so the run stays within minutes.

In this arm (N = 1) the CPU oracle also runs one complete nonlinear
iteration of the first time step on the full-size mesh (ElmGMR + pack + the
full memLS solve): 3 x its time is ``cpu_baseline``, and the same system
solved on the GPU gives the full-size parity figures (``full_size_parity``:
ElmGMR res/lhsK/lhsP and the FP64 and mixed memLS solutions against the
oracle, with the iteration counts).
"""
from __future__ import annotations

import argparse
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

METRIC = "s/timestep @4M tets (mixed vs FP64 GPU, ≤1e-6 rel err); Melem/s assembly"
NCROSS, NAXIAL = 80, 133
NITR = 3
# memLS NSSOLVER relative tolerance (epstol(8)).  1e-6 is below what the
# reference's residual estimate sqrt(|R0|^2 - xB.B) decides reliably: on the
# 107,520-tet cylinder the CPU oracle's first solve stops after 8 outer
# iterations with 8 threads and runs to the 10-iteration limit with 1 thread
# (estimates 6.9e-7 and 1.4e-6 of the initial norm), and the first solve of
# this workload reaches the 10-iteration limit on CPU and GPU alike.
EPSTOL_NS = 1e-5
REFINE_TOL = 0.0      # mixed precision: FP64 defect target (0: the NSSOLVER tolerance)
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one persistent
# CG iteration divided by cg_iter_bytes, from ncu captures of one launch of 50
# iterations on a 2.07M-tet cylinder (5.3M blocks, matrices and vectors
# larger than L2); the traffic of a launch grows with blocks x iterations, so
# the ratio scales the full-size algorithmic bytes to full-size traffic.
TRAFFIC_PER_ALG_F32 = 0.765
TRAFFIC_PER_ALG_F64 = 0.850
TRAFFIC_SOURCE = "ncu --set full, k_cg_persistent, 2.07M-tet cylinder, 50 iterations/launch, scaled by blocks"
# The same ratio for the CG on the explicit FP32 Schur operator (k_cg_schur);
# 1.0 until an ncu capture of that kernel replaces it.
TRAFFIC_PER_ALG_S2 = 1.0
TRAFFIC_SOURCE_S2 = "not yet captured: algorithmic bytes"


def _inflow(t: float) -> float:
    return 10.0 + 5.0 * np.sin(2.0 * np.pi * t / 0.8)


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    return ws, rank


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int = 0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.samples.append([v.strip() for v in out.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 4 + i and "Active" in s[4 + i]
                          and "Not" not in s[4 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def make_problem(ncross: int, naxial: int, epstol_ns: float = None, workload: str = "cylinder",
                 ybif_h: float = 0.036):
    from crimsonflowsolver_b200 import FlowParams, RCR, mesh

    tol = EPSTOL_NS if epstol_ns is None else epstol_ns
    if workload == "ybif":
        m = mesh.bifurcation(h=ybif_h, seed=3)
        P = FlowParams(rcr=[RCR(**d) for d in mesh.bifurcation_rcr(seed=3)], nitr=NITR, epstol_ns=tol)
        return m, P
    m = mesh.cylinder(ncross=ncross, naxial=naxial, seed=1)
    P = FlowParams(rcr=[RCR(srfid=3, Rp=100.0, C=1e-4, Rd=1000.0)], nitr=NITR, epstol_ns=tol)
    return m, P


def workload_name(args, m) -> str:
    if args.workload == "ybif":
        return (f"{m.nelem / 1e6:.1f}M-tet Y-bifurcation ({m.nelem} tets, {m.nshg} nodes; parent R 1 cm, daughters "
                "R 0.7 cm at +-30 deg, 2 RCR outlets +-20% seeded), pulsatile inflow, dt=1e-3, 3 nonlinear "
                "iterations/step")
    size = f"{m.nelem / 1e6:.1f}M" if m.nelem >= 1e6 else f"{m.nelem / 1e3:.0f}k"
    return (f"{size}-tet cylinder ({m.nelem} tets, {m.nshg} nodes), pulsatile inflow, RCR outlet, dt=1e-3, "
            "3 nonlinear iterations/step")


def _oracle_first_iteration(m, P, nthreads: int):
    """The first nonlinear iteration of time step 1 on the CPU oracle, timed:
    predict, ElmGMR (residual + tangent), SolFlow pack, the full memLS NS
    solve.  Returns the timings, the oracle's system and solution."""
    from oracle import pyoracle as po

    F = po.OracleFlow(m, P, nthreads=nthreads, inflow=_inflow)
    m.set_inflow(_inflow(P.Delt))
    fct = (P.gami - 1.0) / P.gami
    F.y = F.yold.copy()
    F.ac = F.acold * fct
    F._itr_bc(F.y)
    c1, c2 = F.implicit_coeffs(0, True)
    yA = F.y.copy()
    acA = F.ac.copy()
    yA[:, 0:3] = F.yold[:, 0:3] + P.alfi * (F.y[:, 0:3] - F.yold[:, 0:3])
    acA[:, 0:3] = F.acold[:, 0:3] + P.almi * (F.ac[:, 0:3] - F.acold[:, 0:3])
    acA[:, 3] = 0.0
    t0 = time.perf_counter()
    out = F.elm(yA, acA, lhs=True, srflist=F.srflist, coef1=c1, coef2=c2)
    t_elm = time.perf_counter() - t0
    t0 = time.perf_counter()
    Res4, Val4 = po.solflow_pack(m.nshg, F.colm, F.rowp, out["res"], out["lhsK"], out["lhsP"])
    t_pack = time.perf_counter() - t0
    faceRes = np.concatenate([[0.0], np.asarray(c1) * P.alfi * P.gami * P.Delt])
    V = Val4.copy()
    t0 = time.perf_counter()
    sol, st = F.memls.solve(Res4, V, faceRes)
    t_solve = time.perf_counter() - t0
    return {"t_elm": t_elm, "t_pack": t_pack, "t_solve": t_solve, "stats": st, "F": F, "inputs": (yA, acA, c1, c2),
            "out": out, "Res4": Res4, "Val4": Val4, "faceRes": faceRes, "sol": sol}


def full_size_parity(m, P, nthreads: int):
    """CPU baseline and full-size parity in one pass (rank 0, N = 1).

    The oracle runs the first nonlinear iteration of time step 1 on the
    benchmark mesh; 3 x (ElmGMR + pack + solve) is the CPU s/timestep (a
    measured sample: every nonlinear iteration repeats this work, the first
    solve being the one from the predicted state).  The GPU then assembles the
    same ElmGMR inputs and solves the oracle's packed system in FP64 and in
    mixed precision through the host-pointer C ABI.
    """
    from crimsonflowsolver_b200 import FlowParams, solver

    o = _oracle_first_iteration(m, P, nthreads)
    st = o["stats"]
    t_iter = o["t_elm"] + o["t_pack"] + o["t_solve"]
    cpu = {"value": P.nitr * t_iter, "unit": "s/timestep", "cores": nthreads, "kind": "port",
           "sample": (f"one complete nonlinear iteration of step 1 at full size, measured: ElmGMR {o['t_elm']:.2f}s + "
                      f"pack {o['t_pack']:.2f}s + full memLS NS solve {o['t_solve']:.2f}s ({st.RI.itr} outer, "
                      f"{st.GM.itr} GMRES, {st.CG.itr} CG its); x {P.nitr} nonlinear iterations per step")}
    yA, acA, c1, c2 = o["inputs"]
    par = {}
    with solver.ElmGMR(m, P) as elm:
        colm, rowp = elm.genadj()
        par["pattern_bit_exact"] = bool(np.array_equal(colm, o["F"].colm) and np.array_equal(rowp, o["F"].rowp))
        g = elm(yA, acA, c1, c2)
        for k in ("res", "lhsK", "lhsP"):
            par[f"elmgmr_{k}_rel_err"] = _relerr(g[k], o["out"][k])
        del g
        for prec in ("fp64", "mixed"):
            Pp = FlowParams(**{**P.__dict__, "precision": prec, "max_refine": 8})
            ms = solver.MemLS(Pp, 1 + len(P.rcr), nshg=m.nshg, colm=colm, rowp=rowp)
            nodes, sv = solver.dirichlet_face(m)
            ms.bc_create(1, nodes, 3, 0, sv)
            for k, r in enumerate(P.rcr):
                nn, vv = solver.neumann_face(m, r.srfid)
                ms.bc_create(2 + k, nn, 3, 1, vv)
            gsol, gst = ms.solve(o["Res4"], o["Val4"].copy(), o["faceRes"])
            ms.close()
            ref = o["sol"]
            par[f"memls_{prec}"] = {
                "velocity_rel_err": _relerr(gsol[:, 0:3], ref[:, 0:3]), "pressure_rel_err": _relerr(gsol[:, 3], ref[:, 3]),
                "iters_gpu": [gst.RI.itr, gst.GM.itr, gst.CG.itr], "iters_oracle": [st.RI.itr, st.GM.itr, st.CG.itr]}
    par["system"] = (f"first nonlinear iteration of step 1 ({m.nelem} tets, {m.nshg} nodes); ElmGMR on the same "
                     "y_alpha/a_alpha/RCR coefficients; memLS on the oracle's packed Res4/Val4")
    return cpu, par


def run_reference(args):
    """The reference algorithm on the CPU (the oracle on all host threads).

    value: one complete time step of the workload, measured.  Each of the
    W + K steps is a bounded sample of the same workload (one full-size
    ElmGMR + SolFlow pack, timed), reported in ms_per_step.
    """
    from oracle import pyoracle as po

    ws, rank = _dist()
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    m, P = make_problem(args.ncross, args.naxial, args.epstol_ns, args.workload, args.ybif_h)
    F = po.OracleFlow(m, P, nthreads=nthreads, inflow=_inflow)
    t0 = time.perf_counter()
    F.step()
    t_full = time.perf_counter() - t0
    its = [list(s[:3]) for s in F.stats]
    y, ac = F.y.copy(), F.ac.copy()
    cc = F.implicit_coeffs(1, True)
    samples = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        out = F.elm(y, ac, lhs=True, srflist=F.srflist, coef1=cc[0], coef2=cc[1])
        po.solflow_pack(m.nshg, F.colm, F.rowp, out["res"], out["lhsK"], out["lhsP"])
        if i >= args.warmup:
            samples.append(time.perf_counter() - t0)
        del out
    sample_s = float(np.median(samples))
    sample = (f"value: one complete time step measured ({len(its)} nonlinear iterations; outer/GMRES/CG its per "
              f"solve {its}); each timed step: one full-size ElmGMR (residual + tangent) + SolFlow pack")
    line = {"metric": METRIC, "value": t_full, "unit": "s/timestep", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sample_s * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": workload_name(args, m) + ", FP64", "parallelism": "replicas",
                       "epstol_ns": P.epstol_ns, "epstol_gmres_cg": [P.epstol_mom, P.epstol_cont]},
            "full_step_measured_s": t_full, "full_step_iters_per_solve": its,
            "sample_step_s": sample_s,
            "cpu_baseline": {"value": t_full, "unit": "s/timestep", "cores": nthreads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": t_full, "unit": "s/timestep", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _timed_steps(F, args, stream, local, dist):
    """W untimed steps, then K steps timed with CUDA events on the library stream."""
    import torch

    from crimsonflowsolver_b200 import _native as N

    L = N.lib()
    iters = []
    for _ in range(args.warmup):
        F.step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = L.crimson_launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            st = F.step()
            iters.append([(st.ri_itr[i], st.gm_itr[i], st.cg_itr[i], st.refine_steps[i], st.refine_rel[i])
                          for i in range(st.nsolves)])
        e1.record(stream)
        torch.cuda.synchronize()
    launches = L.crimson_launch_count() - l0
    t_ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    it = np.array([s for step in iters for s in step], dtype=float)
    per_solve = {"ri": float(it[:, 0].mean()), "gm": float(it[:, 1].mean()), "cg": float(it[:, 2].mean())}
    if it[:, 3].max() > 0:
        per_solve["refine_sweeps"] = float(it[:, 3].mean())
        per_solve["max_final_defect"] = float(it[:, 4].max())
    per_solve["outlet_q"] = [float(st.q_out[k]) for k in range(len(F.P.rcr))]
    per_solve["outlet_p"] = [float(st.p_out[k]) for k in range(len(F.P.rcr))]
    return t_ms, per_solve, int(launches), clk.summary()


def max_over_ranks(t_ms: float, dist, device: str) -> float:
    """The slowest rank's time: replicas run independently, so the job's time
    is the maximum (every rank takes the same collective steps)."""
    if not dist:
        return t_ms
    import torch

    t = torch.tensor([t_ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.barrier()
    return float(t.item())


def replica_value(t_ms: float, steps: int, world_size: int) -> float:
    """s/timestep of the whole job: every replica's steps count (weak scaling)."""
    return t_ms / 1e3 / (steps * world_size)


def _relerr(a, b):
    den = float(np.abs(b).max())
    return float(np.abs(a - b).max() / (den if den > 0 else 1.0))


def cg_iter_bytes(nnz: int, n: int, mbytes: int, nface: int, resident: bool = False) -> int:
    """Algorithmic HBM bytes of one iteration of the persistent CGRAD kernel.

    Per block (nnz real blocks, no padding): G (3 values) + Gt (3) + L (1) of
    mbytes each, and, unless the kernel keeps the column indices resident in
    shared memory for the whole launch (read once per launch, not per
    iteration), the column index read by each of the two SpMV phases
    (2 x 4).  Per row, once: {R, P_prev} read (16), {GP, P} written and
    gathered (2 x 4 mbytes), P written and read twice (24), SP written and
    read (16), X read and written (16), {R, P} written (16), and 2 x 8 per
    coupled face (w_f, z_f).
    """
    return nnz * ((0 if resident else 8) + 7 * mbytes) + n * (16 + 8 * mbytes + 24 + 16 + 16 + 16 + 16 * nface)


def cg_schur_iter_bytes(nnz2: int, n: int, nface: int) -> int:
    """Algorithmic HBM bytes of one iteration of the CG on the explicit FP32
    Schur operator: per 2-ring entry the FP32 value and its int16 column
    offset (6); per row, once: {R, P_prev} FP64 read in both phases and
    written (3 x 16), its FP32 copy written and gathered (2 x 8), S P written
    and read (2 x 8), X read and written (16), and w_f, z_f (phase 1) and z_f
    (phase 2) per coupled face (3 x 8)."""
    return nnz2 * 6 + n * (48 + 16 + 16 + 16 + 24 * nface)


def run_ours(args):
    import ctypes

    import torch

    from crimsonflowsolver_b200 import FlowParams
    from crimsonflowsolver_b200 import _native as N
    from crimsonflowsolver_b200 import solver

    ws, rank = _dist()
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    L = N.lib()
    m, P = make_problem(args.ncross, args.naxial, args.epstol_ns, args.workload, args.ybif_h)
    n = m.nshg
    # ---- FP64 (memLS arithmetic) ----
    F64 = solver.FlowSolver(m, P, inflow=_inflow)
    s64 = torch.cuda.ExternalStream(F64.elm.stream_handle)
    t64_ms, it64, l64, clk64 = _timed_steps(F64, args, s64, local, dist)
    # ---- mixed: FP32 inner matvecs, FP64 refinement ----
    Pm = FlowParams(**{**P.__dict__, "precision": "mixed", "max_refine": 8, "refine_tol": args.refine_tol})
    FM = solver.FlowSolver(m, Pm, inflow=_inflow)
    sm = torch.cuda.ExternalStream(FM.elm.stream_handle)
    tm_ms, itm, lm, clkm = _timed_steps(FM, args, sm, local, dist)
    y64, _ = F64.state()
    ym, _ = FM.state()
    acc = {"velocity": _relerr(ym[:, 0:3], y64[:, 0:3]), "pressure": _relerr(ym[:, 3], y64[:, 3]),
           "outlet_flow": _relerr(np.array(itm["outlet_q"]), np.array(it64["outlet_q"])),
           "outlet_pressure": _relerr(np.array(itm["outlet_p"]), np.array(it64["outlet_p"])),
           "after_steps": args.warmup + args.steps}
    value = replica_value(tm_ms, args.steps, ws)
    v64 = replica_value(t64_ms, args.steps, ws)
    # ---- mixed with FP32 element quadrature of the tangent (the mixed mode's
    # second form), same steps from the same state ----
    Pt = FlowParams(**{**Pm.__dict__, "precision": "mixed_f32_tangent"})
    FT = solver.FlowSolver(m, Pt, inflow=_inflow)
    st_ = torch.cuda.ExternalStream(FT.elm.stream_handle)
    tt_ms, itt, _, _ = _timed_steps(FT, args, st_, local, dist)
    yt, _ = FT.state()
    FT.close()
    del FT
    vt = replica_value(tt_ms, args.steps, ws)
    f32_tangent = {"value": vt, "unit": "s/timestep", "speedup_vs_fp64": v64 / vt,
                   "rel_err_vs_fp64": {"velocity": _relerr(yt[:, 0:3], y64[:, 0:3]),
                                       "pressure": _relerr(yt[:, 3], y64[:, 3]),
                                       "outlet_pressure": _relerr(np.array(itt["outlet_p"]),
                                                                  np.array(it64["outlet_p"])),
                                       "after_steps": args.warmup + args.steps},
                   "solver_iters_per_solve": itt}
    # ---- end to end through the host-buffer API: state in from pinned host, step, state out ----
    def end_to_end(FS, stream):
        y_h = torch.empty((4, n), dtype=torch.float64).pin_memory()
        ac_h = torch.empty((4, n), dtype=torch.float64).pin_memory()
        y0, a0 = FS.state()
        y_h.copy_(torch.from_numpy(np.ascontiguousarray(y0.T)))
        ac_h.copy_(torch.from_numpy(np.ascontiguousarray(a0.T)))
        yp = ctypes.cast(y_h.data_ptr(), N.c_dbl_p)
        ap = ctypes.cast(ac_h.data_ptr(), N.c_dbl_p)
        e_steps = max(1, min(args.steps, 3))
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(e_steps):
            N.check(L.crimson_state_set(FS.elm.h, yp, ap), "crimson_state_set")
            FS.step()
            N.check(L.crimson_state_get(FS.elm.h, yp, ap), "crimson_state_get")
        f1.record(stream)
        torch.cuda.synchronize()
        return f0.elapsed_time(f1) / 1e3 / e_steps

    e2e = end_to_end(FM, sm)
    e2e64 = end_to_end(F64, s64)
    # ---- assembly throughput, timed live on the library stream ----
    dres = torch.zeros((n, 4), dtype=torch.float64, device="cuda")
    nnz = FM.elm._nnz()
    dK = torch.empty((nnz, 9), dtype=torch.float64, device="cuda")
    dP = torch.empty((nnz, 4), dtype=torch.float64, device="cuda")
    dy = torch.tensor(FM.state()[0], device="cuda")
    dac = torch.tensor(FM.state()[1], device="cuda")
    torch.cuda.synchronize()
    for _ in range(2):
        FM.elm.device(dy, dac, dres, dK, dP, [100.0], [0.0])
    a0e = torch.cuda.Event(enable_timing=True)
    a1e = torch.cuda.Event(enable_timing=True)
    a0e.record(sm)
    reps = 5
    for _ in range(reps):
        FM.elm.device(dy, dac, dres, dK, dP, [100.0], [0.0])
    a1e.record(sm)
    torch.cuda.synchronize()
    t_asm = a0e.elapsed_time(a1e) / reps / 1e3
    # ---- kernel times: the persistent CG (events around every launch of the timed run) and the SpMVs ----
    kt = {}
    for lhs, which, name in ((FM.memls.lhs, 4, "cg_iter_f32"), (F64.memls.lhs, 1, "cg_iter_f64"),
                             (FM.memls.lhs, 5, "spmv_K_f32"), (F64.memls.lhs, 0, "spmv_K_f64"),
                             (F64.memls.lhs, 6, "spmv_K_f64_csr"),
                             (F64.memls.lhs, 2, "spmv_G_f64"), (F64.memls.lhs, 3, "mgs_f64")):
        ms = ctypes.c_double()
        rc = L.crimson_memls_kernel_time(lhs, which, 20, ctypes.byref(ms))
        kt[name] = ms.value if rc == 0 else None
    peaks = _peaks()
    nface = len(P.rcr)
    res64, res32, rbytes = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
    N.check(L.crimson_memls_cg_layout(F64.memls.lhs, ctypes.byref(res64), None, None), "crimson_memls_cg_layout")
    if L.crimson_memls_cg_layout(FM.memls.lhs, None, ctypes.byref(res32), ctypes.byref(rbytes)) != 0:
        res32.value = 0   # the mixed solve ran only the explicit-Schur CG
    s2_state, s2_nnz, s2_npad, s2_form_ms = FM.memls.schur_info()
    if s2_state == 1:
        cg_bytes = cg_schur_iter_bytes(s2_nnz, n, nface)
        cg_kernel = ("k_cg_schur<1> (one CGRAD iteration on the explicit FP32 Schur operator: S P, "
                     "coupled-face term, updates)")
    else:
        cg_bytes = cg_iter_bytes(nnz, n, 4, nface, bool(res32.value))
        cg_kernel = "k_cg_persistent<float> (one CGRAD iteration: G P, L P - Gt G P, updates)"
    achieved = cg_bytes / (kt["cg_iter_f32"] / 1e3) / 1e9 if kt["cg_iter_f32"] else None
    cg_bytes64 = cg_iter_bytes(nnz, n, 8, nface, bool(res64.value))
    achieved64 = cg_bytes64 / (kt["cg_iter_f64"] / 1e3) / 1e9 if kt["cg_iter_f64"] else None
    line = {
        "metric": METRIC, "value": value, "unit": "s/timestep", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tm_ms / args.steps, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 matrices in inner Krylov matvecs, f64 vectors/reductions/refinement",
        "data": "synthetic",
        "config": {"workload": workload_name(args, m) + f", {nnz} blocks, mixed-precision NS solve",
                   "parallelism": "replicas" if ws > 1 else "single GPU",
                   "epstol_ns": P.epstol_ns, "epstol_gmres_cg": [P.epstol_mom, P.epstol_cont],
                   "mixed_refine_tol": Pm.refine_tol if Pm.refine_tol > 0 else P.epstol_ns,
                   "l2": "inputs larger than L2 (sliced FP32 matrices 0.66 GB, FP64 1.33 GB per solve)"},
        "fp64": {"value": v64, "unit": "s/timestep", "ms_per_step": t64_ms / args.steps,
                 "e2e": {"value": e2e64, "unit": "s/timestep", "h2d_bytes_per_step": 2 * 4 * n * 8,
                         "d2h_bytes_per_step": 2 * 4 * n * 8},
                 "solver_iters_per_solve": it64, "gpu_launches": l64, "clocks": clk64},
        "mixed_speedup_vs_fp64": v64 / value,
        "mixed_rel_err_vs_fp64": acc,
        "mixed_f32_tangent": f32_tangent,
        "solver_iters_per_solve": itm,
        "assembly_melem_s": m.nelem / t_asm / 1e6,
        "assembly_ms": t_asm * 1e3,
        "kernel_ms": kt,
        "roofline": {"kernel": cg_kernel,
                     "bound": "hbm", "achieved": achieved, "peak": peaks[0], "unit": "GB/s",
                     "frac": achieved / peaks[0] if achieved else None,
                     "traffic": (TRAFFIC_PER_ALG_S2 if s2_state == 1 else TRAFFIC_PER_ALG_F32) * cg_bytes,
                     "traffic_source": TRAFFIC_SOURCE_S2 if s2_state == 1 else TRAFFIC_SOURCE,
                     "algorithmic_bytes_per_iter": cg_bytes, "peak_source": peaks[1],
                     "schur_operator": {"state": s2_state, "nnz": s2_nnz, "sliced_positions": s2_npad,
                                        "formation_ms": s2_form_ms},
                     "columns": ("int16 offsets streamed with the FP32 values" if s2_state == 1 else
                                 ("block-resident in shared memory" if res32.value else "read per phase")),
                     "fp64_kernel": {"achieved": achieved64, "frac": achieved64 / peaks[0] if achieved64 else None,
                                     "algorithmic_bytes_per_iter": cg_bytes64,
                                     "traffic": TRAFFIC_PER_ALG_F64 * cg_bytes64 if TRAFFIC_PER_ALG_F64 else None}},
        "e2e": {"value": e2e, "unit": "s/timestep", "h2d_bytes_per_step": 2 * 4 * n * 8,
                "d2h_bytes_per_step": 2 * 4 * n * 8},
        "gpu_launches": lm,
        "clocks": clkm,
    }
    FM.close()
    F64.close()
    if rank == 0 and ws == 1 and not args.no_cpu:
        try:
            line["cpu_baseline"], line["full_size_parity"] = full_size_parity(m, P, os.cpu_count() or 1)
        except Exception as ex:  # the CPU baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": "s/timestep", "cores": os.cpu_count(), "kind": "port",
                                    "sample": f"failed: {ex}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s"


def run_cg_capture(args):
    """Small fixed-work case for profiler captures of the persistent CG kernel.

    One time step with one nonlinear iteration, two NSSOLVER outer iterations
    and CG maxiters = --cg-iters with an unreachable CG tolerance, so every CG
    launch runs exactly --cg-iters iterations.
    """
    from crimsonflowsolver_b200 import FlowParams, RCR, mesh, solver

    m = mesh.cylinder(ncross=args.ncross, naxial=args.naxial, seed=1)
    P = FlowParams(rcr=[RCR(srfid=3)], precision=args.precision, maxiters=args.cg_iters, epstol_cont=1e-14,
                   nprjs=2, nitr=1, max_refine=1)
    F = solver.FlowSolver(m, P, inflow=lambda t: 10.0)
    st = F.step()
    print(json.dumps({"tets": m.nelem, "nodes": m.nshg, "blocks": F.elm._nnz(),
                      "solves": [(st.ri_itr[i], st.gm_itr[i], st.cg_itr[i]) for i in range(st.nsolves)]}))
    F.close()


def run_adjoint(args):
    """Gradient of the outlet-pressure misfit on a multi-outlet cylinder.

    Workload: cylinder (R 1 cm, L 10 cm) whose distal cap is split into 3 RCR
    outlets (Rp 100 / 120 / 100, C 1e-4 / 1.2e-4 / 1e-4, Rd 1000 / 1000 /
    900), pulsatile inflow, --adj-steps steps of dt 1e-3 with 10 nonlinear
    iterations each (converged), checkpoint every 10 steps; objective
    sum_k (mean_n P_k(t_n) - T_k)^2 with T = (2, 3, 1.5) x 1e3.  Times the
    forward pass alone and the full gradient (forward + recomputation +
    adjoint), and checks --adj-fd components against central differences
    with relative step 1e-6.
    """
    import torch

    from crimsonflowsolver_b200 import FlowParams, RCR, mesh
    from crimsonflowsolver_b200.adjoint import AdjointProblem

    m = mesh.cylinder(ncross=args.ncross, naxial=args.naxial, seed=1, n_outlets=3)
    P = FlowParams(rcr=[RCR(srfid=3), RCR(srfid=4, Rp=120.0, C=1.2e-4), RCR(srfid=5, Rd=900.0)], nitr=10)
    prob = AdjointProblem(m, P, targets=[2.0e3, 3.0e3, 1.5e3], nsteps=args.adj_steps, inflow=_inflow,
                          checkpoint_every=10)
    th = prob.theta0()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    J0 = prob.objective(th)
    t_fwd = time.perf_counter() - t0
    t0 = time.perf_counter()
    J, g = prob.gradient(th)
    t_grad = time.perf_counter() - t0
    its = prob.last_stats["adjoint_iterations"]
    comps = [int(c) for c in args.adj_fd.split(",") if c != ""]
    fd = {}
    for i in comps:
        h = 1e-6 * abs(th[i])
        tp, tm = th.copy(), th.copy()
        tp[i] += h
        tm[i] -= h
        fd[i] = (prob.objective(tp) - prob.objective(tm)) / (2 * h)
    names = ["mu"] + [f"{p}_{k + 1}" for k in range(3) for p in ("Rp", "C", "Rd")]
    line = {"workload": f"adjoint: {m.nelem}-tet cylinder, 3 RCR outlets, {args.adj_steps} steps, checkpoint 10, "
                        "10 nonlinear iterations/step, FP64",
            "tets": m.nelem, "nodes": m.nshg, "J": J, "J_forward_only": J0,
            "forward_s": t_fwd, "gradient_s": t_grad, "gradient_over_forward": t_grad / t_fwd,
            "adjoint_krylov_iterations_per_step": float(np.mean(its)),
            "gradient": dict(zip(names, g.tolist())),
            "fd_check": {names[i]: {"adjoint": float(g[i]), "central_fd": float(fd[i]),
                                    "rel_err": float(abs(g[i] - fd[i]) / abs(fd[i]))} for i in comps}}
    print(json.dumps(line), flush=True)


def run_microbench(args):
    """Assembly / SpMV microbenchmark on a jittered lattice of linear tets.

    Workload: --lattice n gives 6 n^3 tets on an (n+1)^3-node jittered unit
    lattice (n = 139: 16.1M tets, 2.74M nodes), nodal y = (u, v, w, p) and ac
    ~ N(0, 1) (seeded).  Measures ElmGMR residual + tangent assembly (Melem/s)
    and the 4x4 block SpMV (SPARMULVV, dof 4) on the assembled pattern with
    N(0, 1) blocks, FP64 and FP32, each against the HBM roofline, with CUDA
    events on the library stream.  Also ElmGMRSclr (scalar residual +
    tangent, 768 algorithmic B/elem: gathers 352 + rows 32 + tangent 128 of
    the interior pass, 256 of the flux projection) on the same mesh.
    """
    import ctypes

    import torch

    from crimsonflowsolver_b200 import FlowParams
    from crimsonflowsolver_b200 import _native as N
    from crimsonflowsolver_b200 import mesh, solver

    L = N.lib()
    m = mesh.lattice(args.lattice, seed=5)
    P = FlowParams()
    elm = solver.ElmGMR(m, P)
    nnz = elm._nnz()
    n = m.nshg
    stream = torch.cuda.ExternalStream(elm.stream_handle)
    y, ac = mesh.random_state(n, seed=5)
    dev = "cuda"
    dy = torch.tensor(y, device=dev)
    dac = torch.tensor(ac, device=dev)
    res = torch.empty((n, 4), dtype=torch.float64, device=dev)
    K = torch.empty((nnz, 9), dtype=torch.float64, device=dev)
    Pm = torch.empty((nnz, 4), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    def timed(fn, reps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps / 1e3

    peak, peak_src = _peaks()
    t_asm = timed(lambda: elm.device(dy, dac, res, K, Pm, lhs=True), 5)
    t_res = timed(lambda: elm.device(dy, dac, res, None, None, lhs=False), 5)
    rec = torch.empty((nnz, 16), dtype=torch.float32, device=dev)
    t_asm32 = timed(lambda: N.check(L.crimson_elmgmr_device_f32(elm.h, ctypes.c_void_p(dy.data_ptr()),
                                                                ctypes.c_void_p(dac.data_ptr()), None, None,
                                                                ctypes.c_void_p(res.data_ptr()),
                                                                ctypes.c_void_p(rec.data_ptr())), "f32"), 5)
    del rec
    asm_bytes = (2416 + 560) * m.nelem
    asm32_bytes = (624 + 128 + 16 * 13 * 4 + 560) * m.nelem
    out = {"workload": f"lattice {args.lattice}^3 x 6: {m.nelem} tets, {n} nodes, {nnz} blocks; y, ac ~ N(0,1)",
           "peak_gbs": peak, "peak_source": peak_src,
           "assembly_fp64": {"ms": t_asm * 1e3, "melem_s": m.nelem / t_asm / 1e6,
                             "algorithmic_bytes_per_elem": 2976, "achieved_gbs": asm_bytes / t_asm / 1e9,
                             "frac": asm_bytes / t_asm / 1e9 / peak},
           "assembly_fp32_tangent": {"ms": t_asm32 * 1e3, "melem_s": m.nelem / t_asm32 / 1e6,
                                     "algorithmic_bytes_per_elem": 2144,
                                     "achieved_gbs": asm32_bytes / t_asm32 / 1e9,
                                     "frac": asm32_bytes / t_asm32 / 1e9 / peak},
           "residual_only_fp64": {"ms": t_res * 1e3, "melem_s": m.nelem / t_res / 1e6}}
    # ElmGMRSclr on the same mesh: scalar and rate ~ N(0, 1), diffusivity 0.1
    gs = torch.Generator(device=dev).manual_seed(6)
    ds = torch.randn(n, dtype=torch.float64, device=dev, generator=gs)
    dsd = torch.randn(n, dtype=torch.float64, device=dev, generator=gs)
    rs = torch.empty(n, dtype=torch.float64, device=dev)
    del K, Pm
    S = torch.empty(nnz, dtype=torch.float64, device=dev)
    t_s = timed(lambda: elm.sclr_device(dy, ds, dsd, rs, S, isclr=1, diffus=0.1), 5)
    t_sr = timed(lambda: elm.sclr_device(dy, ds, dsd, rs, None, isclr=1, diffus=0.1, lhs=False), 5)
    sclr_bytes = 768 * m.nelem
    out["assembly_sclr_fp64"] = {"ms": t_s * 1e3, "melem_s": m.nelem / t_s / 1e6,
                                 "algorithmic_bytes_per_elem": 768, "achieved_gbs": sclr_bytes / t_s / 1e9,
                                 "frac": sclr_bytes / t_s / 1e9 / peak,
                                 "residual_only_ms": t_sr * 1e3}
    # size-independent checks at full size: two more calls give the same
    # bits; the patch test (zero velocity, linear scalar) leaves only
    # rounding on the interior nodes (the lattice has no boundary faces)
    ref_r, ref_S = rs.clone(), S.clone()
    elm.sclr_device(dy, ds, dsd, rs, S, isclr=1, diffus=0.1)
    elm.sclr_device(dy, ds, dsd, rs, S, isclr=1, diffus=0.1)
    torch.cuda.synchronize()
    repeatable = bool(torch.equal(rs, ref_r) and torch.equal(S, ref_S))
    scale = float(ref_r.abs().max())
    nn1 = args.lattice + 1
    ijk = np.stack(np.unravel_index(np.arange(n), (nn1, nn1, nn1), order="F"), axis=1)
    interior = torch.tensor(np.all((ijk > 0) & (ijk < args.lattice), axis=1), device=dev)
    ds.copy_(torch.tensor(m.x @ np.array([0.3, -1.2, 0.7]) + 2.0, device=dev))
    dsd.zero_()
    y0 = torch.zeros_like(dy)
    elm.sclr_device(y0, ds, dsd, rs, S, isclr=1, diffus=0.1)
    torch.cuda.synchronize()
    patch = float(rs[interior].abs().max())
    out["assembly_sclr_fp64"]["full_size_checks"] = {
        "repeatable_bitwise": repeatable, "patch_max_interior_res": patch,
        "patch_rel_to_random_state_res": patch / scale}
    del ds, dsd, rs, S, y0, ref_r, ref_S
    if not args.no_cpu:
        # cpu_baseline of the scalar assembly: the oracle restatement, one
        # thread, on a 40^3-cell lattice (384,000 tets) with the same fields
        from oracle import pyoracle as po

        ms = mesh.lattice(40, seed=5)
        cs, rs_ = po.genadj(ms.ien, ms.nshg)
        oe = po.Elm(ms, P, cs, rs_)
        rng = np.random.default_rng(6)
        ys = rng.standard_normal((ms.nshg, 4))
        s0, s1 = rng.standard_normal(ms.nshg), rng.standard_normal(ms.nshg)
        po.elmgmr_sclr(oe, ys, s0, s1, isclr=1, diffus=0.1)
        t0 = time.perf_counter()
        po.elmgmr_sclr(oe, ys, s0, s1, isclr=1, diffus=0.1)
        tc = time.perf_counter() - t0
        out["assembly_sclr_fp64"]["cpu_baseline"] = {"value": ms.nelem / tc / 1e6, "unit": "Melem/s", "cores": 1,
                                                     "kind": "port",
                                                     "sample": f"lattice 40^3 x 6 = {ms.nelem} tets, one call"}
    g = torch.Generator(device=dev).manual_seed(5)
    val = torch.randn((nnz, 16), dtype=torch.float64, device=dev, generator=g)
    u = torch.randn((n, 4), dtype=torch.float64, device=dev, generator=g)
    for prec, dt, bb, br in ((0, torch.float64, 132, 72), (1, torch.float32, 68, 40)):
        v = val.to(dt).contiguous()
        uu = u.to(dt).contiguous()
        ku = torch.empty_like(uu)
        torch.cuda.synchronize()
        N.check(L.crimson_spmv4_prepare(elm.h, prec, ctypes.c_void_p(v.data_ptr())), "crimson_spmv4_prepare")
        t = timed(lambda: N.check(L.crimson_spmv4_apply(elm.h, ctypes.c_void_p(uu.data_ptr()),
                                                        ctypes.c_void_p(ku.data_ptr())), "crimson_spmv4_apply"), 20)
        byt = nnz * bb + n * br
        out["spmv4_" + ("fp64" if prec == 0 else "fp32")] = {
            "ms": t * 1e3, "algorithmic_bytes": byt, "achieved_gbs": byt / t / 1e9, "frac": byt / t / 1e9 / peak}
        del v, uu, ku
    elm.close()
    print(json.dumps(out), flush=True)


def run_scale(args):
    """Large-mesh run, one arm at a time (both at once would not fit beyond
    ~45M tets): mesh from --ncross / --naxial (170 x 290 gives 39.5M tets),
    one warm-up step and one timed step per arm, device memory of each arm,
    the CG iteration time against its algorithmic bytes (columns streamed
    when they do not fit in shared memory), mixed vs FP64."""
    import ctypes

    import torch

    from crimsonflowsolver_b200 import FlowParams
    from crimsonflowsolver_b200 import _native as N
    from crimsonflowsolver_b200 import solver

    L = N.lib()
    t0 = time.perf_counter()
    m, P = make_problem(args.ncross, args.naxial, args.epstol_ns)
    gen_s = time.perf_counter() - t0
    peaks = _peaks()
    free0, total = torch.cuda.mem_get_info()
    out = {"workload": workload_name(args, m), "tets": m.nelem, "nodes": m.nshg, "mesh_generation_s": gen_s,
           "device_memory_gb": total / 1e9}
    y64 = None
    for prec in ("fp64", "mixed"):
        Pp = FlowParams(**{**P.__dict__, "precision": prec, "max_refine": 8, "refine_tol": args.refine_tol})
        F = solver.FlowSolver(m, Pp, inflow=_inflow)
        F.step()
        s = torch.cuda.ExternalStream(F.elm.stream_handle)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(s)
        st = F.step()
        e1.record(s)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        ms = ctypes.c_double()
        N.check(L.crimson_memls_kernel_time(F.memls.lhs, 1 if prec == "fp64" else 4, 1, ctypes.byref(ms)), "kt")
        r64, r32, rb = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        N.check(L.crimson_memls_cg_layout(F.memls.lhs, ctypes.byref(r64), ctypes.byref(r32), ctypes.byref(rb)),
                "cg_layout")
        resident = bool(r64.value if prec == "fp64" else r32.value)
        nnz = F.elm._nnz()
        byt = cg_iter_bytes(nnz, m.nshg, 8 if prec == "fp64" else 4, len(P.rcr), resident)
        y, _ = F.state()
        if y64 is None:
            y64 = y
        out[prec] = {"step_s": e0.elapsed_time(e1) / 1e3, "device_memory_used_gb": (free0 - free1) / 1e9,
                     "cg_iter_ms": ms.value, "cg_columns_resident": resident,
                     "cg_algorithmic_bytes_per_iter": byt, "cg_achieved_gbs": byt / ms.value / 1e6,
                     "cg_frac": byt / ms.value / 1e6 / peaks[0],
                     "iters_per_solve": [(st.ri_itr[i], st.gm_itr[i], st.cg_itr[i]) for i in range(st.nsolves)],
                     "rel_err_vs_fp64": _relerr(y, y64)}
        F.close()
        del F
        torch.cuda.synchronize()
    out["mixed_speedup_vs_fp64"] = out["fp64"]["step_s"] / out["mixed"]["step_s"]
    out["peak_source"] = peaks[1]
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ncross", type=int, default=NCROSS)
    ap.add_argument("--naxial", type=int, default=NAXIAL)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--workload", default="cylinder", choices=["cylinder", "ybif"],
                    help="cylinder: 4.0M-tet tube, 1 RCR outlet (default); ybif: ~3.9M-tet Y-bifurcation, 2 RCR "
                         "outlets, mixed arm refined to 1e-8")
    ap.add_argument("--ybif-h", type=float, default=0.036, help="grid spacing of the Y-bifurcation (cm)")
    ap.add_argument("--epstol-ns", type=float, default=EPSTOL_NS, help="NSSOLVER relative tolerance, both arms")
    ap.add_argument("--refine-tol", type=float, default=None,
                    help="mixed precision FP64 defect target (0: the NSSOLVER tolerance; default 0 for the "
                         "cylinder, 1e-8 for the Y-bifurcation)")
    ap.add_argument("--cg-capture", action="store_true",
                    help="run the small fixed-iteration CG case for profiler captures instead of the benchmark")
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"], help="--cg-capture only")
    ap.add_argument("--cg-iters", type=int, default=50, help="--cg-capture only")
    ap.add_argument("--microbench", action="store_true",
                    help="run the lattice assembly / 4x4 SpMV microbenchmark instead of the benchmark")
    ap.add_argument("--lattice", type=int, default=139, help="--microbench only: lattice cells per side")
    ap.add_argument("--adjoint", action="store_true",
                    help="run the adjoint-gradient workload (multi-outlet cylinder) instead of the benchmark")
    ap.add_argument("--adj-steps", type=int, default=100, help="--adjoint only")
    ap.add_argument("--adj-fd", default="0,1", help="--adjoint only: theta components checked by central FD")
    ap.add_argument("--scale", action="store_true",
                    help="large-mesh run of the cylinder, one arm at a time (e.g. --ncross 170 --naxial 290)")
    args = ap.parse_args()
    if args.refine_tol is None:
        args.refine_tol = 1e-8 if args.workload == "ybif" else REFINE_TOL
    if args.cg_capture:
        run_cg_capture(args)
    elif args.adjoint:
        run_adjoint(args)
    elif args.microbench:
        run_microbench(args)
    elif args.scale:
        run_scale(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
