#!/usr/bin/env python
"""Throughput benchmark of the B200 sintering operator.

Workload (one GPU): the 3D operator bench -- Q1 hexes, 128^3 unit cells, 8
seeded spheres with radii U[12, 18] overlapping by 2 cells, greedy colouring
to 4 order parameters (6 components, 12.88 M DoFs), tanh profiles of width 2
plus U(-1e-3, 1e-3) noise, tensorial mobility.  A step is one FP64
Jacobian-vector product J(u) v over the whole mesh (inputs already resident
in HBM); the metric is DoFs processed per second (GDoF/s).  The FP32
Jacobian-vector product and the FP64 residual are timed the same way and
reported under "kernels".

`e2e` times the same step through the public C ABI with host buffers: the
direction v is copied from pinned host memory, J v is computed and copied
back, every step.

`--impl reference`: hpsint itself cannot be built here (deal.II, p4est and
Trilinos are absent), so the reference arm times the CPU restatement of its
operator (oracle/) on the host cores instead.

Multi-GPU (`--gpus N` under torchrun): the operator path is run as N
independent replicas, one per GPU (no collective on the data path); value is
the sum over ranks, timed as the maximum over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Jacobian-vec GDoF/s & s/step: FP32-inner+learned vs FP64 plain, Newton tol 1e-8"
UNIT = "GDoF/s"
WORKLOAD = "3d-operator-bench-128^3-8spheres-G4"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=128, help="cells per direction")
    ap.add_argument("--scalar", action="store_true", help="scalar instead of tensorial mobility")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="budget of the CPU baseline sample")
    ap.add_argument("--workload", choices=["operator", "operator2d", "solve2d", "solve3d", "learned2d", "learned3d",
                                           "nnconv", "nn3d",
                                           "cutoff", "tracker", "advection"],
                    default="operator",
                    help="operator: J v throughput (headline); solve2d: s/step of the 2D two-particle solve; "
                         "learned2d: train the learned guess on 2D many-grain packings and compare s/step")
    ap.add_argument("--n3", type=int, default=192, help="cells per direction of the 3D solve workload")
    ap.add_argument("--spheres", type=int, default=51, help="3D solve: number of spheres")
    ap.add_argument("--median", type=float, default=10.0, help="3D solve: median sphere radius")
    ap.add_argument("--sigma", type=float, default=0.2, help="3D solve: sigma of log radius")
    ap.add_argument("--max-grains", type=int, default=10, help="3D solve: order-parameter budget")
    ap.add_argument("--no-solve", action="store_true", help="skip the s/step comparison of the operator run")
    ap.add_argument("--solve-compare-steps", type=int, default=40)
    ap.add_argument("--solve3d-steps", type=int, default=4,
                    help="steps of the C5 s/step comparison in the default line (0: skip)")
    ap.add_argument("--train-seeds", type=int, default=10)
    ap.add_argument("--train-steps", type=int, default=200, help="FP64 steps per training trajectory")
    ap.add_argument("--train-iters", type=int, default=4000)
    ap.add_argument("--smooth", type=float, default=4.0, help="learned2d: weight of the Laplacian error term")
    ap.add_argument("--eval-seeds", type=int, default=2)
    ap.add_argument("--eval-steps", type=int, default=100)
    ap.add_argument("--cells", type=int, default=512)
    ap.add_argument("--circles", type=int, default=100)
    ap.add_argument("--save-net", default=None, help="write the trained predictor (.npz) here")
    ap.add_argument("--net-width", type=int, default=32, help="learned2d: channels of the hidden layers")
    ap.add_argument("--solve-steps", type=int, default=100)
    ap.add_argument("--arms", default=None,
                    help="solve3d: comma-separated subset of the arms to run (default: all)")
    ap.add_argument("--predictor", default="none",
                    help="solve3d: comma-separated initial guesses (none, linear, euler, learned) each arm but the "
                         "FP64 reference runs with (hpsint's predictors; learned: the 3D network of --net3d or the "
                         "one learned3d trains)")
    ap.add_argument("--net3d", default=None, help="solve3d: trained 3D predictor (.npz of learned_guess.save_predictor)")
    ap.add_argument("--train-n3", type=int, default=64, help="learned3d: cells per direction of the training packings")
    ap.add_argument("--preconditioners", action="store_true",
                    help="solve3d: also run right-preconditioned GMRES with block-Jacobi and with the Gauss-Seidel "
                         "Cahn-Hilliard block")
    ap.add_argument("--cut-off", type=float, default=0.0,
                    help="solve3d: also run both solves with this GrainCutOffTolerance and time the cut-off J v")
    return ap.parse_args()


def make_state(n):
    from hpsint_b200 import packings as P
    centers, radii, colours = P.operator_bench_packing(n=n)
    G = int(colours.max()) + 1
    u = P.initial_state(3, (n, n, n), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), centers, radii, colours, width=2.0,
                        noise=1e-3, seed=1)
    rng = np.random.default_rng(2)
    v = rng.uniform(-1.0, 1.0, u.shape)
    return u, v, G


def model_params(G, tensorial):
    # EnergyAbstractData / MobilityAbstractData defaults (sintering/parameters.h:113-134)
    return dict(n_grains=G, A=16.0, B=1.0, kappa_c=1.0, kappa_p=0.5, Mvol=1e-2, Mvap=1e-10, Msurf=4.0, Mgb=0.4,
                L=1.0, tensorial=tensorial)


DT = 1e-3  # BDF1, dt0 of the solver configurations


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.file.flush()
        rows = [r.split(",") for r in open(self.file.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [x.strip() for x in r]
            if len(r) < 9:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for name, val in zip(names, r[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def fma_peaks(stream_ptr):
    """Measured FMA throughput (TFLOP/s) of this GPU in FP64 and FP32, from the
    bench-only probe library (hpsint_b200/libfma_probe.so, built with the
    operator library): the denominator of the ALU roofline."""
    import ctypes
    probe = ctypes.CDLL(os.path.join(ROOT, "hpsint_b200", "libfma_probe.so"))
    probe.fma_probe_tflops.restype = ctypes.c_int
    probe.fma_probe_tflops.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]
    out = {}
    for prec in (64, 32):
        t = ctypes.c_double()
        rc = probe.fma_probe_tflops(prec, ctypes.byref(t), stream_ptr)
        if rc != 0:
            raise RuntimeError(f"fma_probe_tflops({prec}) failed with CUDA error {rc}")
        out[prec] = t.value
    return out


SLAB_LAYERS = 16  # z-layers of cells in the CPU baseline's sample


def cpu_baseline(u, v, G, tensorial, budget_s, n, gpu_product=None):
    """Time the CPU restatement of the operator (oracle) on a bounded sample of
    the same workload: a slab of z-layers, repeated until `budget_s` elapses.
    With `gpu_product` (the GPU's J v on the full mesh, C x N), the oracle's
    product on the slab checks it: rows of the slab's nodes below its top
    layer (whose cells all lie inside the slab) must agree to 1e-12."""
    from oracle import oracle as O
    threads = os.cpu_count() or 1
    nz = max(2, min(n, SLAB_LAYERS))
    N_slab = (n + 1) * (n + 1) * (nz + 1)
    us = np.ascontiguousarray(u[:, :N_slab])
    vs = np.ascontiguousarray(v[:, :N_slab])
    mesh = O.make_mesh(3, [n, n, nz])
    prm = O.make_params(**{k: val for k, val in model_params(G, tensorial).items()})
    T = O.make_time(1.0 / DT, 1.0, [-1.0 / DT])
    ref = O.jvp(mesh, prm, T, us, vs, threads)  # warm-up, and the parity reference
    parity = None
    if gpu_product is not None:
        inner = (n + 1) * (n + 1) * nz  # nodes with z < nz
        ours, want = gpu_product[:, :inner], ref[:, :inner]
        parity = max(float(np.linalg.norm(ours[b] - want[b]) / np.linalg.norm(want[b])) for b in range(want.shape[0]))
    reps, t0 = 0, time.perf_counter()
    while True:
        O.jvp(mesh, prm, T, us, vs, threads)
        reps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or reps >= 1000:
            break
    dofs = (G + 2) * N_slab * reps
    out = {"value": dofs / el / 1e9, "unit": UNIT, "cores": threads, "kind": "port",
           "sample": f"FP64 Jacobian-vector product, CPU restatement (OpenMP, {threads} threads), "
                     f"{n}x{n}x{nz}-cell z-slab of the same state, {reps} reps in {el:.1f} s"}
    if parity is not None:
        out["parity_rel_err"] = parity
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    u, v, G = make_state(args.n)
    from oracle import oracle as O
    O.build()
    tensorial = not args.scalar
    # each step is a bounded sample (a z-slab) of the workload on all host cores
    per_step = max(1.0, args.cpu_seconds / max(1, args.steps + args.warmup))
    for _ in range(args.warmup):
        cpu_baseline(u, v, G, tensorial, 0.0, args.n)
    vals = []
    for _ in range(args.steps):
        vals.append(cpu_baseline(u, v, G, tensorial, per_step, args.n))
    value = float(np.mean([x["value"] for x in vals]))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "mobility": "scalar" if args.scalar else "tensorial", "n_cells": args.n,
                   "note": "hpsint needs deal.II/p4est/Trilinos (absent): CPU restatement of its operator"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": vals[0]["cores"], "kind": "port",
                         "sample": vals[0]["sample"]},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def two_particle_solve(args):
    """2D two-particle sintering: 256 x 128 Q1 cells on [-40, 40] x [-20, 20],
    circles R = 10 at (+-10, 0), tanh width 2, G = 2, hpsint's default
    constants, BDF1 with dt0 = 1e-3 and hpsint's dt control, Newton relative
    tolerance 1e-8.  Runs the plain FP64 solve, then the FP32-inner solve from
    the same state on the FP64 run's time grid, and reports s/step, iteration
    counts, and the FP32-inner run's error against the FP64 run."""
    import torch

    import hpsint_b200 as hb
    from hpsint_b200 import packings as P
    from hpsint_b200.time_integration import TimeIntegrationData, TimeIntegrator

    nx, ny = 256, 128
    h = (80.0 / nx, 40.0 / ny)
    centers, radii, colours = P.two_particle_2d()
    u0 = P.initial_state(2, (nx, ny), h, (-40.0, -20.0), centers, radii, colours, width=2.0)
    wx = np.full(nx + 1, h[0]); wx[[0, -1]] *= 0.5
    wy = np.full(ny + 1, h[1]); wy[[0, -1]] *= 0.5
    mass = np.outer(wy, wx).ravel()  # lumped weights: int c_h = sum_n m_n c_n

    runs, schedule = {}, None
    for label, prec in (("fp64", 64), ("fp32_inner", 32)):
        op = hb.SinteringOperatorGeneric(hb.Mesh(2, (nx, ny, 1), (h[0], h[1], 1.0)), hb.Params(2))
        ti = TimeIntegrator(op, hb.NonLinearData(nl_rel_tol=1e-8, inner_precision=prec),
                            TimeIntegrationData(time_step_init=1e-3))
        ti.initialize(op.to_device(u0))
        ti.run(2, dt_schedule=[1e-3, 1e-3])  # warm-up (discarded)
        ti.initialize(op.to_device(u0))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ti.run(args.solve_steps, dt_schedule=schedule)  # the FP32-inner run replays the FP64 time grid
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        if schedule is None:
            schedule = [r.dt for r in ti.records]
        u = op.to_host(ti.history[0])
        runs[label] = dict(u=u, wall=wall, t=ti.t, rec=ti.records)
    ref, mp = runs["fp64"], runs["fp32_inner"]
    line = {"metric": METRIC, "workload": "2d-two-particle-256x128-G2", "steps": args.solve_steps,
            "unit": "s/step", "higher_is_better": False, "dtype": "f64 Newton", "data": "synthetic"}
    for label, r in runs.items():
        recs = r["rec"]
        line[label] = {"s_per_step": r["wall"] / len(recs), "sim_time": r["t"],
                       "s_per_accepted_attempt": sum(x.accepted_wall_s for x in recs) / len(recs),
                       "newton_iterations": sum(x.newton_iterations for x in recs),
                       "linear_iterations": sum(x.linear_iterations for x in recs),
                       "preconditioner_setups": sum(x.preconditioner_setups for x in recs),
                       "predict_s_per_step": sum(x.predict_s for x in recs) / len(recs),
                       "failed_tries": sum(x.failed_tries for x in recs), "final_dt": recs[-1].dt}
    same_t = abs(ref["t"] - mp["t"]) <= 1e-12 * max(1.0, ref["t"])
    line["fp32_inner_vs_fp64"] = {
        "same_time_grid": same_t,
        "max_abs_diff_c": float(np.abs(mp["u"][0] - ref["u"][0]).max()),
        "max_abs_diff_eta": float(np.abs(mp["u"][2:] - ref["u"][2:]).max()),
        "int_c_conservation_fp64": float(abs(mass @ ref["u"][0] - mass @ u0[0]) / abs(mass @ u0[0])),
        "int_c_conservation_fp32_inner": float(abs(mass @ mp["u"][0] - mass @ u0[0]) / abs(mass @ u0[0])),
        "speedup_s_per_step": (ref["wall"] / len(ref["rec"])) / (mp["wall"] / len(mp["rec"])),
        "speedup_accepted_attempts": sum(x.accepted_wall_s for x in ref["rec"]) /
                                     sum(x.accepted_wall_s for x in mp["rec"]),
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_solve_baseline(u0, h, schedule, args.cpu_seconds)
    print(json.dumps(line), flush=True)


def cpu_solve_baseline(u0, h, schedule, budget_s):
    """The same solve on the host cores: the CPU restatement of the damped
    Newton-GMRES step (oracle/newton_cpu.py: FP64 GMRES(30), block-Jacobi,
    the oracle's residual and J v with OpenMP) on the first steps of the
    FP64 run's time grid, as many as fit in about `budget_s` seconds; plus
    the CPU residual and J v of the initial state."""
    from oracle import newton_cpu as NC
    from oracle import oracle as O
    O.build()
    threads = os.cpu_count() or 1
    nx, ny = 256, 128
    mesh = O.make_mesh(2, [nx, ny, 0], (h[0], h[1], 1.0))
    prm = O.make_params(**model_params(2, True))
    solver = NC.NewtonCPU(mesh, prm, threads, nl_rel_tol=1e-8)
    u = u0.copy()
    recs, t0 = [], time.perf_counter()
    for dt in schedule:
        T = O.make_time(1.0 / dt, 1.0, [-1.0 / dt])
        old = u.copy()
        recs.append(solver.solve(T, u, [old]))
        if time.perf_counter() - t0 >= budget_s:
            break
    el = time.perf_counter() - t0
    T = O.make_time(1.0 / schedule[0], 1.0, [-1.0 / schedule[0]])
    reps = 5
    t1 = time.perf_counter()
    for _ in range(reps):
        O.residual(mesh, prm, T, u0, [u0], 2, threads)
    t_res = (time.perf_counter() - t1) / reps
    t1 = time.perf_counter()
    for _ in range(reps):
        O.jvp(mesh, prm, T, u0, u0, threads)
    t_jvp = (time.perf_counter() - t1) / reps
    dofs = u0.size
    return {"value": el / len(recs), "unit": "s/step", "cores": threads, "kind": "port",
            "sample": f"first {len(recs)} steps of the FP64 run's time grid, FP64 Newton-GMRES(30) with "
                      f"block-Jacobi on the CPU restatement (oracle/newton_cpu.py, OpenMP, {threads} threads)",
            "newton_iterations": sum(r["newton_iterations"] for r in recs),
            "linear_iterations": sum(r["linear_iterations"] for r in recs),
            "residual_gdofs": dofs / t_res / 1e9, "jvp_gdofs": dofs / t_jvp / 1e9}


def operator_2d(args):
    """The kernels of one FP32-inner Newton step on the 2D many-grain state
    (512^2 cells, 100 circles, seed 0, G = 8, scalar mobility, 2.63 M DoFs,
    BDF1 with dt = 1e-3): CUDA-event time per call of J v (FP64, FP32), the
    residual and the FP32 block-Jacobi apply."""
    import torch

    from hpsint_b200 import learned_guess as LG
    from hpsint_b200.operator import BlockPreconditioner2

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    case = LG.make_case(0)
    op = case.op
    op.set_time_weights(1.0 / DT, [-1.0 / DT], 1.0)
    op.fill_quadrature_point_values(case.u0)
    gen = torch.Generator("cuda").manual_seed(3)
    v = torch.rand(case.u0.shape, dtype=torch.float64, device="cuda", generator=gen) * 2 - 1
    v[:, op.N:] = 0
    d = op.initialize_dof_vector()
    v32, d32 = v.float(), d.float()
    pc = BlockPreconditioner2(op)
    pc.do_update()

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    dofs = op.C * op.N
    res = {"jvp_f64": timed(lambda: op.vmult(d, v)), "jvp_f32": timed(lambda: op.vmult(d32, v32)),
           "residual_f64_bdf1": timed(lambda: op.evaluate_nonlinear_residual(d, case.u0, 2, [case.u0])),
           "precond_apply_f32": timed(lambda: pc.vmult(d32, v32))}
    print(json.dumps({"workload": f"2d-512x512-100-circles-G{case.G}-operator", "dofs": dofs, "unit": "ms",
                      "ms": res, "gdofs": {k: dofs / (t * 1e-3) / 1e9 for k, t in res.items()}}), flush=True)


def nn_conv(args):
    """The learned guess's hidden-layer convolution at inference size: 8 grain
    streams of 513 x 513 nodes, 32 -> 32 channels, 3x3 (38.8 GFLOP): the
    tcgen05 TF32 kernel and the FP32 kernel, CUDA-event time per call."""
    import torch

    from hpsint_b200 import predictor as P

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    G, H, W, C = 8, 513, 513, 32
    gen = torch.Generator("cuda").manual_seed(0)
    x = torch.randn((G, C, H, W), device="cuda", generator=gen)
    w = torch.randn((C, C, 3, 3), device="cuda", generator=gen) * 0.1
    b = torch.randn(C, device="cuda", generator=gen)
    out = torch.empty_like(x)
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    flops = 2.0 * G * H * W * C * C * 9

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    ms_tc = timed(lambda: P.conv3x3_tc(x, w, b, out, status))
    assert int(status.item()) == 0
    ms_fp32 = timed(lambda: P.conv3x3(x, w, b, out))
    print(json.dumps({"workload": "nn-conv3x3-8x32x513x513-to-32", "unit": "ms", "gflop": flops / 1e9,
                      "tcgen05_tf32": {"ms": ms_tc, "tflops": flops / (ms_tc * 1e-3) / 1e12},
                      "fp32_simt": {"ms": ms_fp32, "tflops": flops / (ms_fp32 * 1e-3) / 1e12}}), flush=True)


def solve_comparison(n_steps):
    """s/step of the metric's solve arms on a held-out 2D many-grain packing
    (512^2 cells, 100 circles, seed 1000, scalar mobility, Newton 1e-8): the
    plain FP64 solve (hpsint's method) fixes the time grid, the FP32-inner
    arms replay it with the previous-solution guess, hpsint's Linear and
    Euler predictors, and the learned guess raw and safeguarded (the net
    trained by --workload learned2d on seeds 0..9,
    hpsint_b200/weights/learned_guess_c4.npz); the last two arms add the
    grain cut-off (GrainCutOffTolerance 1e-5)."""
    from hpsint_b200 import learned_guess as LG
    wpath = os.path.join(ROOT, "hpsint_b200", "weights", "learned_guess_c4.npz")
    net, norm = LG.load_predictor(wpath)
    case = LG.make_case(1000)
    arms = ["fp64_plain", "fp32_inner_plain", "fp32_inner_linear", "fp32_inner_euler", "fp32_inner_learned",
            "fp32_inner_learned_safeguarded", "fp32_inner_linear_cut_off", "fp32_inner_learned_safeguarded_cut_off"]
    res = LG.compare_arms(case, n_steps, net, norm, arms=arms)
    plain = res["fp64_plain"]["s_per_step"]
    pick = lambda key: {a: res[a].get(key) for a in arms if a in res}
    return {"workload": f"2d-512x512-100-circles-G{case.G}-seed1000", "dofs": case.op.C * case.op.N,
            "steps": n_steps, "unit": "s/step", "newton_tol": 1e-8,
            "s_per_step": pick("s_per_step"),
            "speedup_vs_fp64_plain": {a: plain / res[a]["s_per_step"] for a in arms if "s_per_step" in res.get(a, {})},
            "newton_iterations": pick("newton_iterations"), "linear_iterations": pick("linear_iterations"),
            "guess_residual_ratio_gmean": pick("guess_residual_ratio_gmean"),
            "max_abs_diff_vs_fp64_plain": {a: max(res[a]["max_abs_diff_c"], res[a]["max_abs_diff_eta"])
                                           for a in arms if "max_abs_diff_c" in res.get(a, {})},
            "int_c_rel_change": pick("int_c_rel_change"),
            "weights": "hpsint_b200/weights/learned_guess_c4.npz"}


def mixed_precision_solve_3d(args, learned=None, train_info=None):
    print(json.dumps(solve3d_line(args, learned, train_info)), flush=True)


def solve_comparison_3d(n_steps):
    """The metric's s/step on the 3D combined configuration, a few steps:
    256^3 cells, 200 lognormal spheres (median 8, sigma 0.25), G = 10
    (203.7 M DoFs), tensorial mobility, Newton 1e-8.  The plain FP64 solve
    (hpsint's method) fixes the time grid; FP32-inner with the grain cut-off
    1e-7 and the matrix-based CH preconditioner replays it without a guess
    and with the committed 3D learned guess
    (hpsint_b200/weights/learned_guess_c5_3d_w8.npz)."""
    a = argparse.Namespace(n3=256, spheres=200, median=8.0, sigma=0.25, max_grains=12, scalar=False,
                           cut_off=1e-7, preconditioners=True, solve_steps=n_steps, predictor="none,learned",
                           net3d=os.path.join(ROOT, "hpsint_b200", "weights", "learned_guess_c5_3d_w8.npz"),
                           arms="fp64_inner,fp32_inner_cut_off_ch_gs_right", operator_rates=False)
    full = solve3d_line(a)
    arms = {"fp64_plain": "fp64_inner", "fp32_inner_cut_off_ch_gs": "fp32_inner_cut_off_ch_gs_right",
            "fp32_inner_cut_off_ch_gs_learned": "fp32_inner_cut_off_ch_gs_right_learned"}
    out = {"workload": full["workload"], "dofs": full["dofs"], "steps": n_steps, "unit": "s/step",
           "newton_tol": 1e-8, "weights": "hpsint_b200/weights/learned_guess_c5_3d_w8.npz"}
    plain = full["fp64_inner"]["s_per_step"]
    for name, key in (("s_per_step", "s_per_step"), ("newton_iterations", "newton_iterations"),
                      ("linear_iterations", "linear_iterations"), ("int_c_rel_change", "int_c_rel_change")):
        out[name] = {k: full[v][key] for k, v in arms.items() if v in full}
    out["speedup_vs_fp64_plain"] = {k: plain / full[v]["s_per_step"] for k, v in arms.items() if v in full}
    out["max_abs_diff_vs_fp64_plain"] = {
        k: max(full[v]["max_abs_diff_c_vs_fp64_inner"], full[v]["max_abs_diff_eta_vs_fp64_inner"])
        for k, v in arms.items() if v in full and "max_abs_diff_c_vs_fp64_inner" in full[v]}
    return out


def solve3d_line(args, learned=None, train_info=None):
    """3D mixed-precision solve: 192^3 Q1 cells at unit spacing, 51 spheres
    with lognormal radii (median 10, sigma 0.2) in a random sequential packing
    with 2-cell overlaps, coloured to <= 10 order parameters, width-2 tanh
    profiles, tensorial mobility with hpsint's default constants, BDF1 with
    dt0 = 1e-4 and hpsint's dt control, Newton relative tolerance 1e-8.  The
    FP64-inner solve fixes the time grid; the FP32-inner solve (FP32 GMRES(30)
    vectors, Jacobian and block-Jacobi inside FP64 Newton) replays it.  Reports
    s/step of both and the FP32-inner run's errors against the FP64-inner run.
    With --cut-off TOL both solves run again on the same grid with the grain
    cut-off (GrainCutOffTolerance = TOL; block-Jacobi from the full operator),
    the FP32-inner one once more with the preconditioner cut as well (the
    reference's assembly), and the J v throughput at the initial state is
    timed with and without the cut-off."""
    import torch

    import hpsint_b200 as hb
    from hpsint_b200 import packings as P
    from hpsint_b200.time_integration import TimeIntegrationData, TimeIntegrator

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n = args.n3
    centers, radii, colours = P.lognormal_packing_3d(n=n, n_spheres=args.spheres, median=args.median,
                                                     sigma=args.sigma, max_grains=args.max_grains)
    G = int(colours.max()) + 1
    u0 = P.initial_state(3, (n, n, n), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), centers, radii, colours, width=2.0)
    w = np.ones(n + 1)
    w[[0, -1]] = 0.5
    op = hb.SinteringOperatorGeneric(hb.Mesh(3, (n, n, n)), hb.Params(**model_params(G, not args.scalar)))
    u0d = op.to_device(u0)
    c0 = float(np.einsum("k,j,i,kji->", w, w, w, u0[0].reshape(n + 1, n + 1, n + 1)))
    del u0
    operator_rates = (cut_off_operator_rates(op, u0d, args.cut_off)
                      if args.cut_off > 0 and getattr(args, "operator_rates", True) else None)
    # (label, Krylov precision, cut-off tolerance, preconditioner with the cut-off too,
    #  block-0 preconditioner, right-preconditioned GMRES)
    BJ, GS = "block_jacobi", "ch_gauss_seidel"
    arms = [("fp64_inner", 64, 0.0, False, BJ, False), ("fp32_inner", 32, 0.0, False, BJ, False)]
    if args.cut_off > 0:
        arms += [("fp64_inner_cut_off", 64, args.cut_off, False, BJ, False),
                 ("fp32_inner_cut_off", 32, args.cut_off, False, BJ, False),
                 ("fp32_inner_cut_off_cut_preconditioner", 32, args.cut_off, True, BJ, False)]
    if args.preconditioners:
        arms += [("fp32_inner_right", 32, 0.0, False, BJ, True), ("fp32_inner_ch_gs_right", 32, 0.0, False, GS, True),
                 ("fp64_inner_ch_gs_right", 64, 0.0, False, GS, True)]
        if args.cut_off > 0:
            arms += [("fp32_inner_cut_off_ch_gs_right", 32, args.cut_off, False, GS, True)]
    if args.arms:
        keep = args.arms.split(",")
        arms = [a for a in arms if a[0] in keep]
        if not arms:
            raise SystemExit(f"--arms {args.arms}: no such arm")
    runs, schedule = {}, None
    from hpsint_b200 import learned_guess as LG
    from hpsint_b200 import learned_guess3d as LG3
    kinds = [k.strip() for k in args.predictor.split(",") if k.strip()]
    if "learned" in kinds and learned is None:
        if not args.net3d:
            raise SystemExit("--predictor learned needs --net3d (or the learned3d workload)")
        learned = LG.load_predictor(args.net3d)
    factories = {"none": None, "linear": LG.LinearPredictor, "euler": LG.EulerPredictor,
                 "learned": (lambda o: LG3.LearnedPredictor3D(o, *learned)) if learned else None}
    for k in kinds:
        if k not in factories:
            raise SystemExit(f"--predictor {k}: not one of {sorted(factories)}")
    # the FP64-inner reference arm keeps hpsint's default (no predictor); every
    # other arm runs once per predictor kind
    expanded = []
    for a in arms:
        if a[0] == "fp64_inner":
            expanded.append((a, "none"))
        else:
            expanded += [(a, k) for k in kinds]
    for (label, prec, tol, cut_pc, block0, right), kind in expanded:
        label = label if kind == "none" else f"{label}_{kind}"
        op.set_component_mask(u0d, tol)  # 0 switches a previous arm's cut-off off
        op.set_preconditioner_cut_off(cut_pc)
        op.set_preconditioner_type(block0)
        # predicted arms stop at the same absolute tolerance (old-solution base)
        pred = factories[kind](op) if factories[kind] else None
        ti = TimeIntegrator(op, hb.NonLinearData(nl_rel_tol=1e-8, inner_precision=prec, right_preconditioning=right),
                            TimeIntegrationData(time_step_init=1e-4), grain_cut_off_tolerance=tol, predictor=pred,
                            tolerance_base="old_solution" if pred else "initial_guess")
        ti.initialize(u0d)
        ti.run(2, dt_schedule=[1e-4, 1e-4])  # warm-up: workspaces, first launches (discarded)
        ti.initialize(u0d)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ti.run(args.solve_steps, dt_schedule=schedule)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        if schedule is None:
            schedule = [r.dt for r in ti.records]
        u = op.to_host(ti.history[0])
        c_int = float(np.einsum("k,j,i,kji->", w, w, w, u[0].reshape(n + 1, n + 1, n + 1)))
        recs = ti.records
        runs[label] = dict(u=u, wall=wall, recs=recs, c_int=c_int, stats=list(ti.cut_off_statistics))
        del ti
    ref, mp = runs.get("fp64_inner"), runs.get("fp32_inner")
    line = {"metric": METRIC, "workload": f"3d-{n}^3-{len(radii)}-lognormal-spheres-median{args.median:g}-G{G}",
            "unit": "s/step", "higher_is_better": False, "dofs": op.C * op.N, "grains": G,
            "steps": args.solve_steps, "dtype": "f64 Newton", "data": "synthetic seeded packing",
            "mobility": "scalar" if args.scalar else "tensorial"}
    for label, r in runs.items():
        recs = r["recs"]
        line[label] = {"s_per_step": r["wall"] / len(recs), "sim_time": float(sum(x.dt for x in recs)),
                       "s_per_accepted_attempt": sum(x.accepted_wall_s for x in recs) / len(recs),
                       "newton_iterations": sum(x.newton_iterations for x in recs),
                       "linear_iterations": sum(x.linear_iterations for x in recs),
                       "preconditioner_setups": sum(x.preconditioner_setups for x in recs),
                       "predict_s_per_step": sum(x.predict_s for x in recs) / len(recs),
                       "failed_tries": sum(x.failed_tries for x in recs),
                       "max_final_residual": max(x.final_residual for x in recs),
                       "int_c_rel_change": abs(r["c_int"] - c0) / abs(c0)}
    if ref and mp:
        line["fp32_inner_vs_fp64_inner"] = {
            "max_abs_diff_c": float(np.abs(mp["u"][0] - ref["u"][0]).max()),
            "max_abs_diff_eta": float(np.abs(mp["u"][2:] - ref["u"][2:]).max()),
            "speedup_s_per_step": (ref["wall"] / len(ref["recs"])) / (mp["wall"] / len(mp["recs"])),
            # failed FP64 attempts (dt halvings) fix the grid the FP32 run replays; without their time:
            "speedup_accepted_attempts": sum(x.accepted_wall_s for x in ref["recs"]) /
                                         sum(x.accepted_wall_s for x in mp["recs"]),
        }
    if ref:
        for label in runs:
            if label in ("fp64_inner", "fp32_inner") or label in ("fp64_inner_cut_off", "fp32_inner_cut_off",
                                                                  "fp32_inner_cut_off_cut_preconditioner"):
                continue
            if label in runs:
                r = runs[label]
                line[label].update({
                    "max_abs_diff_c_vs_fp64_inner": float(np.abs(r["u"][0] - ref["u"][0]).max()),
                    "max_abs_diff_eta_vs_fp64_inner": float(np.abs(r["u"][2:] - ref["u"][2:]).max()),
                    "speedup_s_per_step_vs_fp64_inner": (ref["wall"] / len(ref["recs"])) / (r["wall"] / len(r["recs"])),
                    "linear_iterations_per_newton": sum(x.linear_iterations for x in r["recs"]) /
                                                    max(1, sum(x.newton_iterations for x in r["recs"]))})
    if args.cut_off > 0 and ref:
        line["cut_off"] = {"tolerance": args.cut_off, "operator_at_initial_state": operator_rates}
        for label in ("fp64_inner_cut_off", "fp32_inner_cut_off", "fp32_inner_cut_off_cut_preconditioner"):
            if label not in runs:
                continue
            r = runs[label]
            st = np.sum(r["stats"], axis=0)
            line["cut_off"][label] = {
                "mean_relevant_grains_per_cell": float((np.arange(len(st)) * st).sum() / st.sum()),
                "max_abs_diff_c_vs_fp64_inner": float(np.abs(r["u"][0] - ref["u"][0]).max()),
                "max_abs_diff_eta_vs_fp64_inner": float(np.abs(r["u"][2:] - ref["u"][2:]).max()),
                "speedup_s_per_step_vs_fp64_inner": (ref["wall"] / len(ref["recs"])) / (r["wall"] / len(r["recs"]))}
    if train_info is not None:
        line["learned_training"] = train_info
    return line


def nn_inference_3d(args):
    """One whole-mesh inference of the 3D learned guess at the 3D solve size
    (--n3 cells per direction, --max-grains order parameters, the committed
    C5 net or --net3d): the one-pass convolutions against the slice-shifted
    tensor-core path, on the same seeded states, wall time per call (best of
    --steps after --warmup calls) and the largest difference of the guesses."""
    import torch

    import hpsint_b200 as hb
    from hpsint_b200 import learned_guess as LG
    from hpsint_b200 import learned_guess3d as LG3

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n, G = args.n3, args.max_grains
    net, norm = LG.load_predictor(args.net3d or os.path.join(ROOT, "hpsint_b200", "weights",
                                                             "learned_guess_c5_3d_w8.npz"))
    op = hb.SinteringOperatorGeneric(hb.Mesh(3, (n, n, n)), hb.Params(**model_params(G, not args.scalar)))
    gen = torch.Generator(device="cuda").manual_seed(0)
    un, um = op.initialize_dof_vector(), op.initialize_dof_vector()
    un[:, :op.N] = torch.rand((op.C, op.N), device="cuda", dtype=torch.float64, generator=gen)
    um[:, :op.N] = un[:, :op.N] - 1e-3 * torch.rand((op.C, op.N), device="cuda", dtype=torch.float64, generator=gen)
    line = {"workload": f"nn3d-inference-{n}^3-G{G}-width{net.cfg.width}-layers{net.cfg.layers}", "unit": "ms"}
    guesses = {}
    for name, kw in (("fused_fp32", dict(fused=True)), ("sliced_tcgen05", dict(fused=False, tensor_cores=True))):
        p = LG3.LearnedPredictor3D(op, net, norm, **kw)
        for _ in range(max(1, args.warmup)):
            p([un, um], [1e-4], 1e-4)
        times = []
        for _ in range(max(1, args.steps)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            p([un, um], [1e-4], 1e-4)
            torch.cuda.synchronize()
            times.append(time.perf_counter() - t0)
        net.check_tensor_cores()
        guesses[name] = p.guess.clone()
        line[name] = {"ms": 1e3 * min(times)}
        del p
        torch.cuda.empty_cache()
    line["max_abs_diff"] = float((guesses["fused_fp32"] - guesses["sliced_tcgen05"]).abs().max())
    print(json.dumps(line), flush=True)


def learned_guess_3d(args):
    """Trains the 3D learned guess (FP64 trajectories of --train-seeds
    lognormal packings of --train-n3 cells, --train-steps steps each; 3x3x3
    equivariant net of --net-width channels; --train-iters Adam steps on
    24^3 windows), optionally saves it (--save-net), then runs the 3D solve
    workload with the --predictor kinds (learned among them)."""
    import torch

    from hpsint_b200 import learned_guess as LG
    from hpsint_b200 import learned_guess3d as LG3
    from hpsint_b200.predictor import NetConfig

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    net, norm, tr, info = LG3.train_learned_guess3d(
        list(range(100, 100 + args.train_seeds)), n=args.train_n3, n_spheres=max(4, args.train_n3 ** 3 // 20000),
        n_steps=args.train_steps, net_cfg=NetConfig(dim=3, width=args.net_width, layers=3),
        train_cfg=LG.TrainConfig(window=24, batch=2, iterations=args.train_iters, smooth=args.smooth),
        median=args.median, sigma=args.sigma, max_grains=args.max_grains)
    info = {k: v for k, v in info.items() if k != "loss_history"} | {
        "loss_first_last": [info["loss_history"][0], info["loss_history"][-1]] if info["loss_history"] else None}
    if args.save_net:
        LG.save_predictor(args.save_net, net, norm)
    if "learned" not in args.predictor:
        args.predictor = args.predictor + ",learned"
    mixed_precision_solve_3d(args, learned=(net, norm), train_info=info)


def cut_off_operator(args):
    """Operator throughput with and without the grain cut-off (tolerance
    --cut-off, 1e-5 if unset) at the initial state of the 3D solve workload
    (--n3, --spheres, --median, --sigma, --max-grains; C3 by default)."""
    import torch

    import hpsint_b200 as hb
    from hpsint_b200 import packings as P

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n, tol = args.n3, args.cut_off if args.cut_off > 0 else 1e-5
    centers, radii, colours = P.lognormal_packing_3d(n=n, n_spheres=args.spheres, median=args.median,
                                                     sigma=args.sigma, max_grains=args.max_grains)
    G = int(colours.max()) + 1
    u0 = P.initial_state(3, (n, n, n), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), centers, radii, colours, width=2.0)
    op = hb.SinteringOperatorGeneric(hb.Mesh(3, (n, n, n)), hb.Params(**model_params(G, not args.scalar)))
    u0d = op.to_device(u0)
    del u0
    rates = cut_off_operator_rates(op, u0d, tol, reps=args.steps, warmup=args.warmup)
    print(json.dumps({"metric": "Jacobian-vec GDoF/s with and without the grain cut-off", "unit": "GDoF/s",
                      "workload": f"3d-{n}^3-{len(radii)}-lognormal-spheres-median{args.median:g}-G{G}",
                      "dofs": op.C * op.N, "grains": G, "tolerance": tol, "steps": args.steps,
                      "warmup": args.warmup, "data": "synthetic seeded packing", **rates}), flush=True)


def grain_tracker_detection(args):
    """Grain-tracker particle detection (flood fill, measures, centers, radii,
    maxima; threshold_lower 0.01) of every order parameter of the 3D solve
    workload's initial state (--n3, --spheres, ...; C3 by default): device
    time per tracker call (all order parameters, CUDA events, after --warmup
    calls), against the oracle's flood fill and properties on one host core,
    whose particle ids and counts must agree."""
    import torch

    import hpsint_b200 as hb
    from hpsint_b200 import grain_tracker as GT
    from hpsint_b200 import packings as P
    from oracle import oracle as O

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n = args.n3
    centers, radii, colours = P.lognormal_packing_3d(n=n, n_spheres=args.spheres, median=args.median,
                                                     sigma=args.sigma, max_grains=args.max_grains)
    G = int(colours.max()) + 1
    u0 = P.initial_state(3, (n, n, n), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), centers, radii, colours, width=2.0)
    op = hb.SinteringOperatorGeneric(hb.Mesh(3, (n, n, n)), hb.Params(**model_params(G, not args.scalar)))
    ud = op.to_device(u0)
    thr = 0.01

    def call():
        return [GT.detect_particles(op, ud, b, thr) for b in range(G)]

    for _ in range(args.warmup):
        call()
    stream = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    torch.cuda.synchronize()
    ev[0].record(stream)
    for _ in range(args.steps):
        parts = call()
    ev[1].record(stream)
    torch.cuda.synchronize()
    gpu_ms = ev[0].elapsed_time(ev[1]) / args.steps
    om = O.make_mesh(3, [n, n, n], (1.0, 1.0, 1.0))
    t0 = time.perf_counter()
    ref = [O.grain_segments(om, u0[2 + b], thr) for b in range(G)]
    props = [O.segment_properties(om, u0[2 + b], ids, k) for b, (ids, k) in enumerate(ref)]
    cpu_ms = (time.perf_counter() - t0) * 1e3
    agree = all(p.n_particles == k and np.array_equal(p.ids.cpu().numpy(), ids) for p, (ids, k) in zip(parts, ref))
    max_rel = max([float(np.max(np.abs(p.radii - q[:, 4]) / q[:, 4])) for p, q in zip(parts, props) if len(q)],
                  default=0.0)
    print(json.dumps({"metric": "grain-tracker particle detection, ms per tracker call", "unit": "ms",
                      "higher_is_better": False,
                      "workload": f"3d-{n}^3-{len(radii)}-lognormal-spheres-G{G}", "cells": n ** 3,
                      "order_parameters": G, "threshold_lower": thr, "steps": args.steps, "warmup": args.warmup,
                      "gpu_ms_per_call": gpu_ms, "cpu_oracle_ms_per_call": cpu_ms, "cpu_cores": 1,
                      "particles": [p.n_particles for p in parts], "ids_equal_oracle": bool(agree),
                      "max_rel_radius_diff_vs_oracle": max_rel, "data": "synthetic seeded packing"}), flush=True)


def advection_operator(args):
    """The operator with the advection mechanism at the initial state of the
    3D solve workload (--n3, --spheres, ...; C3 by default): segments = the
    particles of every order parameter (device tracker), k = 2.5, cgb = 0,
    ceq = 0.9, mt = mr = 1.  Reports the set-up (tracker + segment sort), the
    force evaluation, and J v / residual throughput with and without
    advection, also under the grain cut-off (--cut-off, 1e-5 if unset)."""
    import torch

    import hpsint_b200 as hb
    from hpsint_b200 import grain_tracker as GT
    from hpsint_b200 import packings as P

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n, tol = args.n3, args.cut_off if args.cut_off > 0 else 1e-5
    centers, radii, colours = P.lognormal_packing_3d(n=n, n_spheres=args.spheres, median=args.median,
                                                     sigma=args.sigma, max_grains=args.max_grains)
    G = int(colours.max()) + 1
    u0 = P.initial_state(3, (n, n, n), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), centers, radii, colours, width=2.0)
    op = hb.SinteringOperatorGeneric(hb.Mesh(3, (n, n, n)), hb.Params(**model_params(G, not args.scalar)))
    u = op.to_device(u0)
    del u0
    stream = torch.cuda.current_stream()

    def timed(fn, reps, warmup):
        for _ in range(warmup):
            fn()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        for _ in range(reps):
            fn()
        ev[1].record(stream)
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]) / reps

    prm = dict(k=2.5, cgb=0.0, ceq=0.9, smoothening=0.0, mt=1.0, mr=1.0)

    def set_up():
        seg, cen, owners = GT.advection_segments(op, u, 0.01)
        op.set_advection_mechanism(seg, cen, **prm)
        return owners

    owners = set_up()
    t0 = time.perf_counter()
    for _ in range(3):
        set_up()
    torch.cuda.synchronize()
    setup_ms = (time.perf_counter() - t0) * 1e3 / 3
    forces_ms = timed(lambda: op.advection_forces(u), args.steps, args.warmup)
    out = {"setup_ms_wall": setup_ms, "forces_ms": forces_ms, "segments": len(owners)}
    op.set_time_weights(1e4, [-1e4], 1.0)
    op.fill_quadrature_point_values(u)
    gen = torch.Generator(device="cuda").manual_seed(0)
    dst64, dst32 = op.initialize_dof_vector(), op.initialize_dof_vector(torch.float32)
    src64 = torch.rand((op.C, op.ld), dtype=torch.float64, device="cuda", generator=gen) - 0.5
    src32 = src64.float()
    dofs = op.C * op.N
    for cut in (0.0, tol):
        op.set_component_mask(u, cut)
        for adv in (False, True):
            if adv:
                set_up()
            else:
                op.set_advection_mechanism(None, None, **prm)
            tag = ("_advection" if adv else "") + ("_cut_off" if cut > 0 else "")
            out["jvp_f64" + tag + "_gdofs"] = dofs / timed(lambda: op.vmult(dst64, src64), args.steps,
                                                           args.warmup) / 1e6
            out["jvp_f32" + tag + "_gdofs"] = dofs / timed(lambda: op.vmult(dst32, src32), args.steps,
                                                           args.warmup) / 1e6
            out["residual_f64" + tag + "_gdofs"] = dofs / timed(
                lambda: op.evaluate_nonlinear_residual(dst64, u, 2, [u]), args.steps, args.warmup) / 1e6
    op.set_component_mask(u, 0.0)
    print(json.dumps({"metric": "operator GDoF/s with the advection mechanism", "unit": "GDoF/s",
                      "workload": f"3d-{n}^3-{len(radii)}-lognormal-spheres-G{G}", "dofs": dofs, "grains": G,
                      "cut_off_tolerance": tol, "advection": prm, "steps": args.steps, "warmup": args.warmup,
                      "note": "residual with advection includes the force evaluation from its state",
                      "data": "synthetic seeded packing", **out}), flush=True)


def cut_off_operator_rates(op, u, tol, reps=20, warmup=3):
    """GDoF/s of the FP64/FP32 Jacobian-vector products and the residual at
    state u, without and with the grain cut-off at tolerance tol (CUDA events
    on the current stream after `warmup` calls)."""
    import torch

    op.set_time_weights(1e4, [-1e4], 1.0)
    op.fill_quadrature_point_values(u)
    gen = torch.Generator(device="cuda").manual_seed(0)
    out = {}
    stream = torch.cuda.current_stream()
    for t in (0.0, tol):
        op.set_component_mask(u, t)
        for name, dt in (("jvp_f64", torch.float64), ("jvp_f32", torch.float32), ("residual_f64", None)):
            if dt is None:
                dst = op.initialize_dof_vector()
                fn = lambda: op.evaluate_nonlinear_residual(dst, u, 2, [u])  # noqa: E731
            else:
                src = torch.rand((op.C, op.ld), dtype=dt, device="cuda", generator=gen) - 0.5
                dst = op.initialize_dof_vector(dt)
                fn = lambda: op.vmult(dst, src)  # noqa: E731
            for _ in range(warmup):
                fn()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
            ev[0].record(stream)
            for _ in range(reps):
                fn()
            ev[1].record(stream)
            torch.cuda.synchronize()
            ms = ev[0].elapsed_time(ev[1]) / reps
            out[f"{name}{'_cut_off' if t > 0 else ''}_gdofs"] = op.C * op.N / (ms * 1e-3) / 1e9
        if t > 0:
            st = op.component_mask_statistics()
            out["mean_relevant_grains_per_cell"] = float((np.arange(len(st)) * st).sum() / st.sum())
            out["cells_per_relevant_grain_count"] = st.tolist()
    op.set_component_mask(u, 0.0)
    return out


def learned_guess_solve(args):
    """2D many-grain packings (cells^2 Q1 cells, circles with radii U[6, 12],
    <= 8 order parameters, scalar mobility, BDF1, dt0 = 1e-3, Newton
    relative tolerance 1e-8): FP64 training trajectories on train seeds,
    Adam training of the equivariant net on the device, then on held-out
    seeds the plain FP64 solve (previous-solution guess, hpsint's dt control)
    against FP64 + linear guess, FP64 + learned guess, FP32-inner plain and
    FP32-inner + learned guess on the plain run's time grid.  Every arm stops
    at the same absolute Newton tolerance (1e-8 relative to the residual of the
    old solution), so the final fields must agree."""
    import torch

    from hpsint_b200 import learned_guess as LG
    from hpsint_b200.predictor import NetConfig

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    train = list(range(args.train_seeds))
    held = list(range(1000, 1000 + args.eval_seeds))
    net, norm, trainer, info = LG.train_learned_guess(
        train, n=args.cells, n_circles=args.circles, n_steps=args.train_steps, net_cfg=NetConfig(width=args.net_width),
        train_cfg=LG.TrainConfig(iterations=args.train_iters, smooth=args.smooth), verbose=False)
    if args.save_net:
        LG.save_predictor(args.save_net, net, norm)
    evals = []
    for seed in held:
        case = LG.make_case(seed, n=args.cells, n_circles=args.circles)
        res = LG.compare_arms(case, args.eval_steps, net, norm)
        evals.append({"seed": seed, "G": case.G, "dofs": case.op.C * case.op.N, "arms": res})
        del case
        torch.cuda.empty_cache()

    def total(arm, key):
        return sum(e["arms"][arm][key] for e in evals if arm in e["arms"] and key in e["arms"][arm])

    steps = args.eval_steps * len(evals)
    plain_s = total("fp64_plain", "wall_s") / steps
    best_s = total("fp32_inner_learned_safeguarded", "wall_s") / steps
    line = {"metric": METRIC, "workload": f"2d-{args.cells}x{args.cells}-{args.circles}-circles-learned-guess",
            "value": best_s, "unit": "s/step", "higher_is_better": False, "n_gpus": 1,
            "dtype": "f64 Newton, f32 GMRES + f32 net", "data": "synthetic seeded packings",
            "fp64_plain_s_per_step": plain_s, "speedup_vs_fp64_plain": plain_s / best_s if best_s > 0 else None,
            "arms_s_per_step": {a: total(a, "wall_s") / steps for a in LG.ARMS},
            "arms_newton_iterations": {a: total(a, "newton_iterations") for a in LG.ARMS},
            "arms_linear_iterations": {a: total(a, "linear_iterations") for a in LG.ARMS},
            "guess_residual_ratio_gmean": {a: [e["arms"][a].get("guess_residual_ratio_gmean") for e in evals
                                               if a in e["arms"]] for a in LG.ARMS},
            "max_abs_diff_vs_fp64_plain": {a: max((max(e["arms"][a]["max_abs_diff_c"], e["arms"][a]["max_abs_diff_eta"])
                                                   for e in evals if "max_abs_diff_c" in e["arms"].get(a, {})),
                                                  default=None) for a in LG.ARMS},
            "training": {k: v for k, v in info.items() if k != "loss_history"},
            # (iteration, training loss, loss of the zero correction = linear extrapolation) at start and end
            "loss_first_last": [info["loss_history"][0], info["loss_history"][-1]],
            "eval": evals}
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "solve2d":
        two_particle_solve(args)
        return
    if args.workload == "operator2d":
        operator_2d(args)
        return
    if args.workload == "nnconv":
        nn_conv(args)
        return
    if args.workload == "learned3d":
        learned_guess_3d(args)
        return
    if args.workload == "nn3d":
        nn_inference_3d(args)
        return
    if args.workload == "solve3d":
        mixed_precision_solve_3d(args)
        return
    if args.workload == "cutoff":
        cut_off_operator(args)
        return
    if args.workload == "advection":
        return advection_operator(args)
    if args.workload == "tracker":
        grain_tracker_detection(args)
        return
    if args.workload == "learned2d":
        learned_guess_solve(args)
        return
    import torch

    from hpsint_b200 import replicas

    w = replicas.from_env()
    world, rank, local_rank = w.size, w.rank, w.local_rank
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    import hpsint_b200 as hb
    from hpsint_b200 import _lib as L

    tensorial = not args.scalar
    u, v, G = make_state(args.n)
    n = args.n
    op = hb.SinteringOperatorGeneric(hb.Mesh(3, (n, n, n)), hb.Params(**model_params(G, tensorial)))
    op.set_time_weights(1.0 / DT, [-1.0 / DT], 1.0)
    ud, vd = op.to_device(u), op.to_device(v)
    op.fill_quadrature_point_values(ud)
    dst = op.initialize_dof_vector()
    dofs = op.C * op.N
    stream = torch.cuda.current_stream()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def time_loop(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        barrier()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(stream)
        for _ in range(steps):
            fn()
        ev[1].record(stream)
        torch.cuda.synchronize()
        # the job's step time is the slowest rank's (replicas: no data-path collective)
        ms = replicas.max_over_ranks(ev[0].elapsed_time(ev[1]), dist)
        return ms / steps

    # --- headline: FP64 Jacobian-vector product --------------------------------
    sampler = ClockSampler(local_rank)
    for _ in range(args.warmup):
        op.vmult(dst, vd)
    barrier()
    launches0 = hb.kernel_launch_count()
    sampler.start()
    time.sleep(0.3)
    ms_jvp64 = time_loop(lambda: op.vmult(dst, vd), args.steps, 0)
    clocks = sampler.stop()
    launches = hb.kernel_launch_count() - launches0
    # the headline product on the oracle slab's nodes, for the parity check
    slab_nodes = (n + 1) * (n + 1) * (min(n, SLAB_LAYERS) + 1)
    gpu_slab = dst[:, :slab_nodes].cpu().numpy()

    # --- the other kernels of the path ----------------------------------------
    v32, dst32 = vd.float(), op.initialize_dof_vector(torch.float32)
    ms_jvp32 = time_loop(lambda: op.vmult(dst32, v32), args.steps, args.warmup)
    hist = [ud.clone()]
    res = op.initialize_dof_vector()
    ms_res = time_loop(lambda: op.evaluate_nonlinear_residual(res, ud, 2, hist), args.steps, args.warmup)
    pc = hb.BlockPreconditioner2(op)
    ms_pcsetup = time_loop(pc.do_update, max(1, args.steps // 4), 1)
    z32 = op.initialize_dof_vector(torch.float32)
    ms_pc32 = time_loop(lambda: pc.vmult(z32, v32), args.steps, args.warmup)

    # --- end to end through the C ABI with host buffers ------------------------
    import ctypes
    h_src = torch.empty((op.C, op.ld), dtype=torch.float64, pin_memory=True)
    h_src.copy_(vd.cpu())
    h_dst = torch.empty((op.C, op.ld), dtype=torch.float64, pin_memory=True)
    d_src = op.initialize_dof_vector()
    lib = L.lib()
    sp = ctypes.c_void_p(stream.cuda_stream)
    nbytes = op.C * op.ld * 8

    def e2e_step():
        d_src.copy_(h_src, non_blocking=True)
        L.check(lib.sint_jvp_f64(op._h, ctypes.c_void_p(dst.data_ptr()), ctypes.c_void_p(d_src.data_ptr()), sp),
                "sint_jvp_f64")
        h_dst.copy_(dst, non_blocking=True)

    ms_e2e_serial = time_loop(e2e_step, args.steps, args.warmup)
    torch.cuda.synchronize()
    assert np.isfinite(h_dst[:, :op.N].numpy()).all()
    # the same calls pipelined (copy-in / product / copy-out of consecutive steps overlap)
    pipe = hb.HostJvpPipeline(op)
    h_dsts = [torch.empty((op.C, op.ld), dtype=torch.float64, pin_memory=True) for _ in range(2)]
    step_no = [0]

    def e2e_pipelined():
        pipe.submit(h_dsts[step_no[0] % 2], h_src)
        step_no[0] += 1

    for _ in range(args.warmup):
        e2e_pipelined()
    pipe.end(stream)
    barrier()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ev[0].record(stream)
    pipe.begin(stream)
    for _ in range(args.steps):
        e2e_pipelined()
    pipe.end(stream)
    ev[1].record(stream)
    torch.cuda.synchronize()
    ms_e2e = replicas.max_over_ranks(ev[0].elapsed_time(ev[1]), dist) / args.steps
    assert torch.equal(h_dsts[0], h_dst)  # same product, bitwise

    # --- measured FMA throughput: denominator of the ALU roofline ---------------
    fma = fma_peaks(sp)

    # --- roofline of the dominant kernel (algorithmic bytes) ------------------
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    alg_bytes = 24 * dofs  # src + dst + linearisation point, FP64
    achieved = alg_bytes / (ms_jvp64 * 1e-3) / 1e9

    if rank != 0:
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    gdofs = lambda ms: dofs / (ms * 1e-3) / 1e9
    # per-launch DRAM traffic and executed FP64 operations of the FP64 J v kernel
    # from one ncu capture of this workload (profiles/jvp_f64_counters.json)
    traffic, flops = None, None
    tf = os.path.join(ROOT, "profiles", "jvp_f64_counters.json")
    if os.path.exists(tf):
        try:
            t = json.load(open(tf))
            if t.get("workload") == WORKLOAD and t.get("mobility") == ("tensorial" if tensorial else "scalar"):
                traffic = t.get("dram_bytes_per_launch")
                flops = t.get("fp64_flops_per_launch")
        except Exception:
            traffic, flops = None, None
    line = {
        "metric": METRIC,
        "value": gdofs(ms_jvp64) * world,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_jvp64,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "n_cells": [n, n, n], "n_grains": G, "n_components": op.C,
                   "dofs": dofs, "mobility": "tensorial" if tensorial else "scalar", "step": "FP64 J(u) v",
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                   "l2": "inputs larger than L2 (lin + src + dst = %.0f MB)" % (3 * dofs * 8 / 1e6)},
        "kernels": {
            "jvp_f64": {"ms": ms_jvp64, "gdofs": gdofs(ms_jvp64)},
            "jvp_f32": {"ms": ms_jvp32, "gdofs": gdofs(ms_jvp32)},
            "residual_f64_bdf1": {"ms": ms_res, "gdofs": gdofs(ms_res)},
            "precond_setup_f64": {"ms": ms_pcsetup},
            "precond_apply_f32": {"ms": ms_pc32, "gbs": (4 * 2 * dofs + 4 * (G + 4) * op.N) / (ms_pc32 * 1e-3) / 1e9},
        },
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak, "traffic": traffic,
                     "note": f"FP64 J v: algorithmic bytes 24*C*N = {alg_bytes/1e6:.1f} MB per launch; "
                             f"peak {peak_src}; kernel is FP64-ALU bound (on-the-fly linearisation)"},
        "roofline_alu": {"bound": "fp64", "peak_fp64_tflops": fma[64], "peak_fp32_tflops": fma[32],
                         "peak_note": "measured FMA-chain throughput on this GPU (bench-only libfma_probe.so)",
                         "achieved_fp64_tflops": (flops / (ms_jvp64 * 1e-3) / 1e12) if flops else None,
                         "frac": (flops / (ms_jvp64 * 1e-3) / 1e12 / fma[64]) if flops else None,
                         "flops_source": "executed FP64 add/mul/fma (fma = 2) of one ncu capture" if flops else None},
        "e2e": {"value": gdofs(ms_e2e) * world, "unit": UNIT, "h2d_bytes_per_step": nbytes,
                "d2h_bytes_per_step": nbytes,
                "note": "sint_jvp_f64 on pinned host vectors, copy-in / product / copy-out of consecutive "
                        "steps overlapped on three streams (operator.HostJvpPipeline)",
                "serial_value": gdofs(ms_e2e_serial) * world},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    if world == 1 and not args.no_solve:
        del ud, vd, dst, v32, dst32, hist, res, z32, d_src, pc
        torch.cuda.empty_cache()
        line["solve"] = solve_comparison(args.solve_compare_steps)
        torch.cuda.empty_cache()
        if args.solve3d_steps > 0:
            line["solve3d"] = solve_comparison_3d(args.solve3d_steps)
    if world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(u, v, G, tensorial, args.cpu_seconds, n, gpu_product=gpu_slab)
        # per-block relative l2 error of the headline product against the oracle
        # on the slab's interior rows (16 z-layers of cells, 4.4 M DoFs)
        line["parity_rel_err"] = cb.pop("parity_rel_err", None)
        line["cpu_baseline"] = cb
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
