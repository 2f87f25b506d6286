#!/usr/bin/env python
"""Benchmark of the FV right-hand side (FiniteVolumeSolver::ComputeRHSFunction) on B200.

One "step" is one RHS evaluation of the whole synthetic workload with the state resident in HBM.
Default workload: the 128^3 periodic Navier-Stokes Taylor-Green case (AUSM+up, least squares +
minmod, constant viscosity), run at FP64 and on the mixed path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload tgv3d|sod2d|shear3d]

With --gpus N > 1 it runs under torch.distributed.run, one rank per GPU: the Taylor-Green box is
(128 N) x 128 x 128 cut into x-slabs, 128^3 owned cells per GPU (weak scaling), and every step is the
two-layer halo exchange (pack kernel, NCCL point-to-point, unpack kernel) followed by the local RHS.
Device times come from CUDA events around each step on the launching stream, L2 flushed between timed
steps, max over ranks.
``--impl reference`` times the CPU restatement of the reference algorithm (the oracle; the reference
itself needs PETSc/MPI/TChem, absent here) on all host cores, rank 0 only.
At N = 1 the default run also measures two species configurations under their own keys
(``species_case``: 256^3, five NASA-7 species; ``tets_case``: 2M tetrahedra, nine species): RHS, JVP,
VJP and the FP64 error against the oracle at full size. ``--no-species-case`` skips them.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "FV RHS Mcell-updates/s (FP64 vs mixed @1e-6 rel), HBM GB/s, VJP/RHS cost"
UNIT = "Mcell-updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="tgv3d", choices=["tgv3d", "sod2d", "channel_tets", "shear3d", "wall3d"])
    ap.add_argument("--n", type=int, default=0, help="mesh cells per direction (default: the configuration's size)")
    ap.add_argument("--precision", default="both", choices=["fp64", "mixed", "both"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-species-case", action="store_true",
                    help="skip the species cases (256^3 five species, 2M tetrahedra nine species) measured beside the Taylor-Green headline")
    return ap.parse_args()


def make_workload(name, n):
    from ablate_b200 import workloads

    if name == "tgv3d":
        return workloads.tgv3d(n or 128)
    if name == "sod2d":
        return workloads.sod2d(n or 256)
    if name == "channel_tets":
        return workloads.channel_tets(n or 2_000_000, 9)
    if name == "wall3d":
        return workloads.wall3d(n or 128)
    return workloads.shear3d(n or 256, 5)


def workload_for(args, world, rank):
    """(workload, local domain or None) of this rank. At N > 1 the Taylor-Green box is (128 N) x 128 x 128
    cut in x-slabs and every rank holds its slab with a two-layer halo. Building it maps no library."""
    if world > 1:
        if args.workload != "tgv3d":
            raise SystemExit("multi-GPU runs partition the tgv3d case")
        from ablate_b200.workloads import tgv3d_slab
        dom, w = tgv3d_slab(args.n or 128, world, rank)
        return w, dom
    return make_workload(args.workload, args.n), None


def workload_config(w, world):
    """The `config` object of the bench line, identical for both arms (built from the workload alone)."""
    n_cells = int(w.mesh.n_interior)
    return {"workload": w.name, "n_cells": world * n_cells, "cells_per_gpu": n_cells, "n_faces": int(w.mesh.n_faces),
            "description": w.description,
            "parallelism": (f"dp{world}: x-slab partition, 2-layer halo exchanged over NCCL point-to-point before every RHS"
                            if world > 1 else "single GPU"),
            "l2": "flushed (256 MiB write) between timed steps, outside the timed events"}


def block_errors(F, F_ref, owned, dim):
    """Norm-wise relative error ||F - F_ref||_2 / ||F_ref||_2 and the largest absolute difference, per
    field block (euler, densityYi) over the owned cells."""
    neul = 2 + dim
    a, b = F[owned], F_ref[owned]
    out = {}
    for name, sl in (("euler", slice(0, neul)), ("densityYi", slice(neul, None))):
        x, y = a[:, sl], b[:, sl]
        if x.shape[1] == 0:
            continue
        d = x - y
        out[name] = {"rel_l2": float(np.linalg.norm(d) / max(np.linalg.norm(y), 1e-300)), "max_abs": float(np.abs(d).max()),
                     "max_abs_ref": float(np.abs(y).max())}
    return out


def algorithmic_bytes(w):
    """Compulsory traffic of one RHS: read the FP64 state once, write the residual once, read 1/V per
    owned cell; per face with an owned side read two int32 cell indices and the FP64 area normal."""
    from ablate_b200 import _lib as L
    n_cells = int(w.mesh.n_interior)
    nc = w.U.shape[1]
    kind, fc = w.mesh.cell_kind, w.mesh.face_cells
    n_faces = int(((kind[fc[:, 0]] == L.CELL_OWNED) | (kind[fc[:, 1]] == L.CELL_OWNED)).sum())
    return n_cells * (2 * nc * 8 + 8) + n_faces * (2 * 4 + w.mesh.dim * 8)


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5], parts[6], parts[7], parts[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        reasons = set()
        for r in rows:
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), r[2:]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows), "reasons": sorted(reasons),
                "samples": len(rows)}


def read_traffic(workload: str, precision: str, kernel: str, n_cells: int):
    """DRAM bytes per launch of one kernel from the committed ncu summary (profiles/traffic_<workload>.txt,
    a line "cells: <n>" and lines "<precision> <kernel>: <bytes>"), if it has that kernel at this size."""
    p = ROOT / "profiles" / f"traffic_{workload}.txt"
    if not p.exists():
        return None
    lines = p.read_text().splitlines()
    if f"cells: {n_cells}" not in lines:
        return None
    for line in lines:
        if line.startswith(f"{precision} {kernel}:"):
            return float(line.split(":")[1])
    return None


def implicit_vs_explicit(solver, U0, owned, dt_e, horizon, stream, dev, ms_of):
    """BDF2 (Newton-GMRES(30) on the JVP, frozen-limiter tangent) at 1, 2, 4 and 8 times the CFL-0.5
    step against SSP-RK3 at that step, both measured against SSP-RK3 at 1/8 of it over `horizon` steps."""
    import torch
    from ablate_b200 import _lib as L
    from ablate_b200.implicit import BDFStepper

    st = stream.cuda_stream

    def ssprk3(dt, n):
        Ux = U0.clone()
        for _ in range(n):
            solver.StepDevice(L.STEP_SSPRK3, 0.0, dt, Ux.data_ptr(), L.PRECISION_FP64, st)
        return Ux

    U_ref, ref_ms = ms_of(lambda: ssprk3(dt_e / 8, horizon * 8))
    scale = float((U_ref[owned] - U0[owned]).norm())

    def err(X):
        return float((X[owned] - U_ref[owned]).norm()) / scale

    U_ex, ex_ms = ms_of(lambda: ssprk3(dt_e, horizon))
    rows = [{"method": "ssprk3", "dt_over_cfl05": 1, "steps": horizon, "ms": ex_ms, "rel_error": err(U_ex)}]
    for m in (1, 2, 4, 8):
        bdf = BDFStepper(solver, m * dt_e)

        def run():
            Ux = U0.clone()
            for _ in range(horizon // m):
                bdf.step(Ux)
            return Ux

        U_im, im_ms = ms_of(run)
        rows.append({"method": "bdf2", "dt_over_cfl05": m, "steps": horizon // m, "ms": im_ms, "rel_error": err(U_im),
                     "newton": bdf.stats["newton"], "gmres_iterations": bdf.stats["gmres"], "jvp": bdf.stats["jvp"], "rhs": bdf.stats["rhs"],
                     "gmres_unconverged": bdf.stats["ksp_unconverged"], "newton_unconverged": bdf.stats["snes_unconverged"],
                     "newton_residual_reduction": [float(r) for r in bdf.reductions]})
    if solver.Status() != L.OK:
        raise RuntimeError("device status after the implicit/explicit comparison")
    ex_err = rows[0]["rel_error"]
    matched = [r for r in rows[1:] if r["rel_error"] <= ex_err]
    verdict = (f"BDF2 at {matched[-1]['dt_over_cfl05']}x the explicit step matches its accuracy in {matched[-1]['ms']:.1f} ms vs {ex_ms:.1f} ms"
               if matched else
               f"no BDF2 step size reaches the explicit error {ex_err:.2e}; the smallest BDF2 error is "
               f"{min(r['rel_error'] for r in rows[1:]):.2e}")
    return {"reference": f"ssprk3 at dt/8 ({horizon * 8} steps, {ref_ms:.1f} ms)", "runs": rows, "equal_accuracy": verdict}


def wall_studies(w, solver, U, stream, dev, K=10, horizon=8):
    """The wall-bounded channel's two uses of the derivatives, on the device:
    (1) the gradient of the wall-patch pressure after K SSP-RK3 steps (fixed step, half the CFL-1 step)
        with respect to the initial state and the inlet speed: forward march with checkpoints, then
        the adjoint march (VJP per stage + transposed ghost fill);
    (2) BDF2 with Newton-GMRES(30) on the JVP against SSP-RK3 at CFL 0.5, with the configured minmod
        limiter and with unlimited gradients (a differentiable residual)."""
    import torch
    from ablate_b200 import _lib as L
    from ablate_b200 import fv
    from ablate_b200.adjoint import ExplicitMarch, functional_gradient, inlet_state

    st = stream.cuda_stream
    table, cell_bc = w.boundary
    solver.SetBoundary(table, cell_bc)
    solver.SetPressureFunctional(*w.functional)
    U0 = U.clone()
    solver.FillGhostsDevice(U0.data_ptr(), st)
    dt_e = solver.CflTimeStepDevice(U0.data_ptr(), 0.5, st)

    def ms_of(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        a.record(stream)
        out = fn()
        b.record(stream)
        torch.cuda.synchronize(dev)
        return out, a.elapsed_time(b)

    march = ExplicitMarch(solver, L.STEP_SSPRK3, dt_e, K)
    functional_gradient(solver, march, U0)  # warm-up
    UK, fwd_ms = ms_of(lambda: march.forward(U0, keep=True))
    lam = torch.zeros_like(UK)
    J = solver.PressureFunctionalDevice(UK.data_ptr(), lam.data_ptr(), st)
    (lam0, vbar), adj_ms = ms_of(lambda: march.adjoint(lam))
    if solver.Status() != L.OK:
        raise RuntimeError("device status after the functional gradient")
    rho0, p0 = 101325.0 / (287.0 * 300.0), 101325.0
    V = 0.3 * np.sqrt(1.4 * 287.0 * 300.0)
    _, dvalue = inlet_state(rho0, p0, V, (1.0, 0.0, 0.0))
    grad = {"steps": K, "scheme": "ssprk3", "dt": dt_e, "J": J, "dJ_dVin": float(np.dot(vbar[0, :5], dvalue)),
            "dJ_dU0_norm": float(lam0.norm()), "forward_ms": fwd_ms, "adjoint_ms": adj_ms, "adjoint_over_forward": adj_ms / fwd_ms,
            "note": "adjoint = stage recomputation (RHS) + one VJP and one transposed ghost fill per stage; gradients checked against "
                    "central differences in the tests"}

    owned = torch.from_numpy(w.mesh.cell_kind == L.CELL_OWNED).to(dev)
    comp = {"t_end": horizon * dt_e, "horizon_steps": horizon,
            "minmod": implicit_vs_explicit(solver, U0, owned, dt_e, horizon, stream, dev, ms_of)}
    unlimited = fv.FiniteVolumeSolver(w.mesh, w.eos, w.processes, w.petscfv_type, "none", device=solver.device)
    unlimited.SetBoundary(table, cell_bc)
    comp["unlimited"] = implicit_vs_explicit(unlimited, U0, owned, dt_e, horizon, stream, dev, ms_of)
    unlimited.close()
    comp["note"] = ("rel_error = |U - U_ref| / |U_ref - U_0| over the owned cells; device time with CUDA events around each march; "
                    "Newton: SNES defaults (rtol 1e-8, stol 1e-8) capped at 10 iterations with a backtracking line search, "
                    "GMRES(30) at rtol 1e-5 capped at 300 iterations, state scaled per component")
    return grad, comp


def species_workload_case(args, dev, stream, flush, name, n):
    """A species configuration measured beside the headline, with the headline's protocol (L2 flushed
    between steps, CUDA events): the FP64 RHS, the mixed request, the JVP and the VJP, and the FP64
    residual against the oracle's on the same state. `shear3d` at 256: 3D Euler + 5 NASA-7 species,
    256^3 shear layer, AusmpUp, least squares + minmod (the large single-GPU case). `channel_tets` at
    2,000,000: Navier-Stokes + 9 NASA-7 species with constant-Lewis transport on Delaunay tetrahedra
    in a 1 x 0.2 x 0.2 channel."""
    import torch
    from ablate_b200 import _lib as L
    from ablate_b200.workloads import initial_aux
    from oracle import oracle as orc

    t_setup = time.perf_counter()
    w = make_workload(name, n)
    solver = w.solver(device=dev.index)
    aux0 = initial_aux(w)
    solver.SetAux(aux0)
    U = torch.from_numpy(w.U).to(dev)
    setup_s = time.perf_counter() - t_setup
    steps, warm = max(3, min(args.steps, 5)), max(3, min(args.warmup, 3))

    def timed(fn):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize(dev)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for k in range(steps):
            flush.zero_()
            ev[k][0].record(stream)
            fn()
            ev[k][1].record(stream)
        torch.cuda.synchronize(dev)
        if solver.Status() != L.OK:
            raise RuntimeError("device status after a timed call of the species case")
        return sum(a.elapsed_time(b) for a, b in ev) / steps

    F = torch.zeros_like(U)
    out = {"workload": w.name, "description": w.description, "n_cells": int(w.mesh.n_interior), "steps": steps, "warmup": warm,
           "state_bytes": int(w.U.nbytes), "record_classes": dict(zip(("cone_weights", "face_geometry"), solver.RecordClasses()))}
    ms = {}
    for name, prec in (("fp64", L.PRECISION_FP64), ("mixed", L.PRECISION_MIXED)):
        ms[name] = timed(lambda: solver.ComputeRHSDevice(0.0, U.data_ptr(), F.data_ptr(), prec, stream.cuda_stream))
    dU = torch.randn_like(U) * U.abs().mean(0, keepdim=True) * 1e-2
    dF = torch.zeros_like(U)
    ms["jvp"] = timed(lambda: solver.ComputeJVPDevice(0.0, U.data_ptr(), dU.data_ptr(), dF.data_ptr(), 0, stream.cuda_stream))
    Fbar = torch.randn_like(U)
    Ubar = torch.zeros_like(U)
    ms["vjp"] = timed(lambda: solver.ComputeVJPDevice(0.0, U.data_ptr(), Fbar.data_ptr(), Ubar.data_ptr(), stream.cuda_stream))
    B = algorithmic_bytes(w)
    n = out["n_cells"]
    out["fp64"] = {"ms_per_step": ms["fp64"], "mcell_per_s": n / (ms["fp64"] * 1e-3) / 1e6, "hbm_gbs": B / (ms["fp64"] * 1e-3) / 1e9}
    out["mixed"] = {"ms_per_step": ms["mixed"], "mcell_per_s": n / (ms["mixed"] * 1e-3) / 1e6,
                    "note": "with species a mixed request runs the FP64 kernels unless ABL_FV_MIXED_SPECIES=1 is set at create (the FP32-gradient kernels measured 1.18e-6 against FP64 on the 2M tetrahedra and 1.02-1.06x faster)"}
    out["jvp"] = {"ms_per_step": ms["jvp"], "over_rhs_fp64": ms["jvp"] / ms["fp64"]}
    out["vjp"] = {"ms_per_step": ms["vjp"], "over_rhs_fp64": ms["vjp"] / ms["fp64"],
                  "note": "limiter and EOS recomputed inside the VJP (no intermediates kept from a forward pass)"}
    out["algorithmic_bytes_per_rhs"] = B
    # FP64 residual of the state against the oracle's (mixture temperatures reset to the same guess)
    solver.SetAux(aux0)
    Fx = torch.zeros_like(U)
    solver.ComputeRHSDevice(0.0, U.data_ptr(), Fx.data_ptr(), L.PRECISION_FP64, stream.cuda_stream)
    torch.cuda.synchronize(dev)
    if not args.no_cpu_baseline:
        phys, keep = w.physics()
        R = orc.OracleRHS(w.mesh, phys)
        F_cpu = np.zeros_like(w.U)
        t0 = time.perf_counter()
        R(w.U, aux0, F_cpu, os.cpu_count() or 1)
        t_cpu = time.perf_counter() - t0
        R.close()
        out["parity"] = {"fp64_vs_oracle": block_errors(Fx.cpu().numpy(), F_cpu, w.mesh.cell_kind == L.CELL_OWNED, w.mesh.dim)}
        out["cpu_oracle"] = {"value": n / t_cpu / 1e6, "unit": UNIT, "cores": os.cpu_count() or 1, "sample": "one full RHS evaluation"}
    out["setup_s"] = setup_s
    solver.close()
    return out


def cpu_baseline(w, phys, seconds):
    from oracle import oracle as orc
    from ablate_b200.workloads import initial_aux

    threads = os.cpu_count() or 1
    R = orc.OracleRHS(w.mesh, phys)
    aux = initial_aux(w)
    F = np.zeros_like(w.U)
    R(w.U, aux, F, threads)  # warm-up
    times = []
    t_end = time.perf_counter() + seconds
    while time.perf_counter() < t_end or len(times) < 2:
        F[:] = 0.0
        t0 = time.perf_counter()
        R(w.U, aux, F, threads)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    out = {"value": w.mesh.n_interior / t / 1e6, "unit": UNIT, "cores": threads, "kind": "port",
           "sample": f"full workload, {len(times)} RHS evaluations (median), oracle restatement with OpenMP over {threads} threads"}
    # one thread (about one rank of the reference's MPI runs): one evaluation, when it fits in ~30 s
    if t * threads <= 30.0:
        F1 = np.zeros_like(w.U)
        t0 = time.perf_counter()
        R(w.U, aux, F1, 1)
        t1 = time.perf_counter() - t0
        out["single_thread"] = {"value": w.mesh.n_interior / t1 / 1e6, "unit": UNIT, "cores": 1,
                                "sample": "one full RHS evaluation on one thread"}
    R.close()
    return out, F


def run_reference(args):
    """The reference arm: the CPU restatement of the reference's RHS algorithm (the reference itself needs
    PETSc, MPI, Kokkos and TChem) on all host cores, rank 0 only. It builds the same workload and config
    as the GPU arm without mapping the CUDA library (the package loads it on first use only)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    w, dom = workload_for(args, world, 0)
    phys, keep = w.physics()
    from oracle import oracle as orc
    from ablate_b200.workloads import initial_aux

    threads = os.cpu_count() or 1
    R = orc.OracleRHS(w.mesh, phys)
    aux = initial_aux(w)
    F = np.zeros_like(w.U)
    for _ in range(args.warmup):
        R(w.U, aux, F, threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        R(w.U, aux, F, threads)
    t = (time.perf_counter() - t0) / args.steps
    R.close()
    n_cells = int(w.mesh.n_interior)
    value = n_cells / t / 1e6
    sample = (f"one full RHS of the workload per step, {threads} OpenMP threads" if world == 1 else
              f"one RHS of rank 0's slab ({n_cells} owned cells, its 2-layer halo included) per step, {threads} OpenMP threads; "
              "the host's cores are shared by all ranks, so the rate of one slab is the host's rate")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": workload_config(w, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    from ablate_b200 import _lib as L
    from ablate_b200.workloads import initial_aux

    drhs = None
    w, dom = workload_for(args, world, rank)
    if dom is not None:
        from ablate_b200.distributed import DistributedRHS
        drhs = DistributedRHS(dom, w.eos, w.processes, w.petscfv_type, w.limiter, device=local)
        solver = drhs.solver
    else:
        solver = w.solver(device=local)
    solver.SetAux(initial_aux(w))
    U = torch.from_numpy(w.U).to(dev)
    F = torch.zeros_like(U)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # 256 MiB > 126 MB L2
    stream = torch.cuda.current_stream(dev)
    precisions = {"fp64": [L.PRECISION_FP64], "mixed": [L.PRECISION_MIXED], "both": [L.PRECISION_FP64, L.PRECISION_MIXED]}[args.precision]

    def barrier():
        if world > 1:
            dist.barrier()

    def rhs(prec):
        if drhs is not None:
            drhs.ComputeRHSDevice(0.0, U, F, prec)
        else:
            solver.ComputeRHSDevice(0.0, U.data_ptr(), F.data_ptr(), prec, stream.cuda_stream)

    results = {}
    kernels = {}
    clocks = None
    for prec in precisions:
        for _ in range(args.warmup):
            rhs(prec)
        torch.cuda.synchronize(dev)
        barrier()
        torch.cuda.synchronize(dev)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        with ClockSampler(local) as cs:
            for k in range(args.steps):
                flush.zero_()
                evs[k][0].record(stream)
                rhs(prec)
                evs[k][1].record(stream)
            torch.cuda.synchronize(dev)
        barrier()
        torch.cuda.synchronize(dev)
        if clocks is None:
            clocks = cs.summary()
        total_ms = sum(a.elapsed_time(b) for a, b in evs)
        if world > 1:
            t = torch.tensor([total_ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            total_ms = float(t.item())
        rc = solver.Status()
        if rc != L.OK:
            raise RuntimeError(f"device status {rc} after the timed RHS")
        results[prec] = total_ms / args.steps
        # per-kernel split from a separate profiled pass (events between the launches inside the library)
        solver.Profile(True)
        acc: dict = {}
        for k in range(args.steps):
            flush.zero_()
            rhs(prec)
            for name, ms in solver.ProfileRead().items():
                acc[name] = acc.get(name, 0.0) + ms
        solver.Profile(False)
        kernels[prec] = {name: ms / args.steps for name, ms in acc.items()}

    # forward tangent (JVP) and adjoint (VJP) costs relative to one FP64 RHS, same protocol
    def timed(fn, what):
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize(dev)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record(stream)
            fn()
            ev[k][1].record(stream)
        torch.cuda.synchronize(dev)
        if solver.Status() != L.OK:
            raise RuntimeError(f"device status after the timed {what}")
        ms = sum(a.elapsed_time(b) for a, b in ev) / args.steps
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        solver.Profile(True)
        split: dict = {}
        for k in range(args.steps):
            flush.zero_()
            fn()
            for name, kms in solver.ProfileRead().items():
                split[name] = split.get(name, 0.0) + kms / args.steps
        solver.Profile(False)
        return ms, split

    jvp_ms = vjp_ms = None
    if L.PRECISION_FP64 in results and world == 1:
        dU = torch.randn_like(U) * U.abs().mean(0, keepdim=True) * 1e-2
        dF = torch.zeros_like(U)
        jvp_ms, kernels["jvp"] = timed(lambda: solver.ComputeJVPDevice(0.0, U.data_ptr(), dU.data_ptr(), dF.data_ptr(), 0, stream.cuda_stream), "JVP")
        Fbar = torch.randn_like(U)
        Ubar = torch.zeros_like(U)
        vjp_ms, kernels["vjp"] = timed(lambda: solver.ComputeVJPDevice(0.0, U.data_ptr(), Fbar.data_ptr(), Ubar.data_ptr(), stream.cuda_stream),
                                       "VJP")

    # the 2D Euler configuration also marches: 100 SSP-RK3 steps at CFL 0.5 with the CFL step of each
    # state, ghosts filled before every stage (one RHS was timed above)
    march = None
    head_prec = L.PRECISION_FP64 if L.PRECISION_FP64 in results else precisions[0]
    if w.name == "sod2d" and world == 1:
        Um = U.clone()
        t_dev = torch.zeros(1, dtype=torch.float64, device=dev)
        for _ in range(2):
            solver.StepCflDevice(L.STEP_SSPRK3, 0.5, Um.data_ptr(), head_prec, t_dev.data_ptr(), stream.cuda_stream)
        Um.copy_(U)
        t_dev.zero_()
        torch.cuda.synchronize(dev)
        m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m0.record(stream)
        for _ in range(100):
            solver.StepCflDevice(L.STEP_SSPRK3, 0.5, Um.data_ptr(), head_prec, t_dev.data_ptr(), stream.cuda_stream)
        m1.record(stream)
        torch.cuda.synchronize(dev)
        if solver.Status() != L.OK:
            raise RuntimeError("device status after the march")
        ms = m0.elapsed_time(m1)
        march = {"steps": 100, "scheme": "ssprk3", "cfl": 0.5, "ms": ms, "ms_per_step": ms / 100,
                 "mcell_per_s": 300 * int(w.mesh.n_interior) / (ms * 1e-3) / 1e6, "t_end": float(t_dev.item()),
                 "note": "per step on the device, nothing read back: CFL step (device minimum), 3 stages of ghost fill + RHS + stage update"}

    # the wall-bounded channel: functional gradient through the adjoint march, implicit vs explicit
    wall = None
    if w.name == "wall3d" and world == 1:
        grad, comp = wall_studies(w, solver, U, stream, dev)
        wall = {"functional_gradient": grad, "implicit_vs_explicit": comp}

    # the residuals of this workload's state at each precision (for the accuracy figures below); the
    # mixture EOS's resident temperatures are reset to the oracle's starting guess first
    F_dev = {}
    for prec in (L.PRECISION_FP64, L.PRECISION_MIXED):
        if prec in results or (prec == L.PRECISION_FP64 and L.PRECISION_MIXED in results):
            solver.SetAux(initial_aux(w))
            Fx = torch.zeros_like(U)
            if drhs is not None:
                drhs.ComputeRHSDevice(0.0, U, Fx, prec)
            else:
                solver.ComputeRHSDevice(0.0, U.data_ptr(), Fx.data_ptr(), prec, stream.cuda_stream)
            torch.cuda.synchronize(dev)
            F_dev[prec] = Fx.cpu().numpy()
    owned_np = w.mesh.cell_kind == L.CELL_OWNED
    # accuracy of the mixed path against FP64 on this workload
    mixed_err = None
    if L.PRECISION_MIXED in F_dev:
        mixed_err = {k: v["rel_l2"] for k, v in block_errors(F_dev[L.PRECISION_MIXED], F_dev[L.PRECISION_FP64], owned_np, w.mesh.dim).items()}

    # end to end through the public host API: pinned host buffers, H2D of U and F, RHS, D2H of F
    head = L.PRECISION_FP64 if L.PRECISION_FP64 in results else precisions[0]
    Uh = torch.from_numpy(w.U).pin_memory()
    Fh = torch.zeros_like(Uh).pin_memory()
    Un, Fn = Uh.numpy(), Fh.numpy()

    def e2e_step():
        if drhs is not None:
            # the rank's host state in, halo exchange + RHS, the residual out
            U.copy_(Uh, non_blocking=True)
            F.zero_()
            drhs.ComputeRHSDevice(0.0, U, F, head)
            Fh.copy_(F, non_blocking=True)
            torch.cuda.current_stream(dev).synchronize()
        else:
            solver.ComputeRHSFunction(0.0, Un, Fn, head)

    for _ in range(2):
        e2e_step()
    torch.cuda.synchronize(dev)
    barrier()
    e2e_steps = max(3, min(args.steps, 10))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    torch.cuda.synchronize(dev)
    e2e_ms = (time.perf_counter() - t0) * 1e3 / e2e_steps
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    state_bytes = int(w.U.nbytes)

    n_cells = int(w.mesh.n_interior)
    B = algorithmic_bytes(w)
    peak, peak_kind = measured_peaks()
    head_ms = results[head]
    value = world * n_cells / (head_ms * 1e-3) / 1e6
    achieved = B / (head_ms * 1e-3) / 1e9
    launches = solver.LaunchCount(head) * args.steps
    kt = kernels.get(head, {})
    dom_name, dom_ms = max(kt.items(), key=lambda kv: kv[1]) if kt else ("rhs", head_ms)
    dom_achieved = B / (dom_ms * 1e-3) / 1e9

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": head_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if head == L.PRECISION_FP64 else "mixed f32/f64", "data": "synthetic",
        "config": workload_config(w, world),
        "layout": {"record_classes": dict(zip(("cone_weights", "face_geometry"), solver.RecordClasses())),
                   "halo_bytes_per_rank_per_step": drhs.halo.bytes_per_exchange if drhs is not None else 0},
        "roofline": {"bound": "hbm", "kernel": dom_name, "achieved": dom_achieved, "peak": peak, "unit": "GB/s", "frac": dom_achieved / peak,
                     "traffic": read_traffic(w.name, "fp64" if head == L.PRECISION_FP64 else "mixed", dom_name, n_cells) if world == 1 else None,
                     "algorithmic_bytes_per_launch": B, "kernel_ms": dom_ms,
                     "peak_source": f"{peak_kind} MEASURED_PEAKS.json hbm_gbs" if peak_kind == "measured" else "fallback 6.65 TB/s",
                     "whole_rhs": {"achieved": achieved, "frac": achieved / peak, "ms": head_ms},
                     "note": "the dominant kernel touches every algorithmic byte of the RHS (state, residual, 1/V, face cells, normals)"},
        "kernel_ms": {({L.PRECISION_FP64: "fp64", L.PRECISION_MIXED: "mixed"}.get(p, p)): v for p, v in kernels.items()},
        "precisions": {("fp64" if p == L.PRECISION_FP64 else "mixed"): {"ms_per_step": ms, "mcell_per_s": world * n_cells / (ms * 1e-3) / 1e6,
                                                                          "hbm_gbs": B / (ms * 1e-3) / 1e9}
                       for p, ms in results.items()},
        "mixed_rel_err_vs_fp64": mixed_err,
        "vjp_over_rhs": (vjp_ms / results[L.PRECISION_FP64]) if vjp_ms else None,
        "vjp": {"ms_per_step": vjp_ms, "over_rhs_fp64": (vjp_ms / results[L.PRECISION_FP64]) if vjp_ms else None},
        "jvp": {"ms_per_step": jvp_ms, "over_rhs_fp64": (jvp_ms / results[L.PRECISION_FP64]) if jvp_ms else None},
        "e2e": {"value": world * n_cells / (e2e_ms * 1e-3) / 1e6, "unit": UNIT,
                "h2d_bytes_per_step": (state_bytes if world > 1 else 2 * state_bytes), "d2h_bytes_per_step": state_bytes, "ms_per_step": e2e_ms,
                "path": ("per rank: pinned host U copied in, halo exchange + RHS, F copied out, every step" if world > 1 else
                         "abl_fv_rhs_host: pinned host U and F copied in, RHS, F copied out, every step")},
        "march": march,
        "wall": wall,
        "gpu_launches": launches,
        "clocks": clocks,
    }
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        phys, keep = w.physics()
        cb, F_cpu = cpu_baseline(w, phys, args.cpu_seconds)
        line["cpu_baseline"] = cb
        # every number above states its error against the oracle's FP64 residual of the same state
        parity = {"reference": "oracle: CPU restatement of the reference RHS, FP64, same seeded state"}
        if L.PRECISION_FP64 in F_dev:
            parity["fp64_vs_oracle"] = block_errors(F_dev[L.PRECISION_FP64], F_cpu, owned_np, w.mesh.dim)
        if L.PRECISION_MIXED in F_dev:
            parity["mixed_vs_oracle"] = block_errors(F_dev[L.PRECISION_MIXED], F_cpu, owned_np, w.mesh.dim)
        line["parity"] = parity
    solver.close()
    if world == 1 and w.name == "tgv3d" and not args.no_species_case:
        # the species configurations, each under its own line key (the headline above stays the 128^3 case)
        del U, F
        torch.cuda.empty_cache()
        for key, name, n in (("species_case", "shear3d", 256), ("tets_case", "channel_tets", 2_000_000)):
            try:
                line[key] = species_workload_case(args, dev, stream, flush, name, n)
            except Exception as e:  # reported, the headline line stands
                line[key] = {"error": f"{type(e).__name__}: {e}"}
            torch.cuda.empty_cache()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
