"""Matrix-free implicit time stepping with the device JVP as the Jacobian: BDF1/BDF2 with Newton-GMRES.

This is the caller-side use of abl_fv_jvp that PETSc's implicit TS makes through a MatShell whose
MatMult is the JVP (TSBDF order 2, SNES Newton line search "basic", KSPGMRES restart 30, no
preconditioner). The residual of one step of size dt from U^n (and U^{n-1}) is, on the owned rows,

    R(U) = U - a1 U^n - a2 U^{n-1} - beta dt F(fill(U))

with (a1, a2, beta) = (1, 0, 1) for BDF1 and (4/3, -1/3, 2/3) for BDF2 at a constant step, and its
Jacobian J v = v - beta dt dF/dU (fill'(v)), fill' the tangent of the ghost fill. Vectors are torch
tensors (n_cells, nc) on the solver's GPU; rows that are not owned are kept at zero in the Krylov
vectors. GMRES is Saad and Schultz's (1986) with classical Gram-Schmidt applied twice (as PETSc's
KSPGMRESClassicalGramSchmidtOrthogonalization with refinement) and Givens rotations; convergence is
PETSc's default test, ||r|| <= max(rtol ||b||, atol).
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib as L


def gmres(apply, b, x0=None, restart: int = 30, rtol: float = 1e-5, atol: float = 1e-50, max_it: int = 10000):
    """Solve apply(x) = b. Returns (x, iterations, final residual norm). Vectors are torch tensors."""
    import torch
    x = torch.zeros_like(b) if x0 is None else x0.clone()
    bnorm = float(torch.linalg.vector_norm(b))
    target = max(rtol * bnorm, atol)
    n_it = 0
    r = b - apply(x) if x0 is not None else b.clone()
    beta = float(torch.linalg.vector_norm(r))
    while beta > target and n_it < max_it:
        m = restart
        Vb = torch.empty((m + 1,) + tuple(b.shape), dtype=b.dtype, device=b.device)
        Vf = Vb.view(m + 1, -1)
        Vb[0] = r / beta
        H = np.zeros((m + 1, m))
        cs, sn = np.zeros(m), np.zeros(m)
        g = np.zeros(m + 1)
        g[0] = beta
        k = 0
        for j in range(m):
            w = apply(Vb[j]).reshape(-1)
            h = Vf[: j + 1] @ w
            w -= Vf[: j + 1].T @ h
            h2 = Vf[: j + 1] @ w
            w -= Vf[: j + 1].T @ h2
            hc = (h + h2).double().cpu().numpy()
            hn = float(torch.linalg.vector_norm(w))
            H[: j + 1, j] = hc
            H[j + 1, j] = hn
            for i in range(j):
                t = cs[i] * H[i, j] + sn[i] * H[i + 1, j]
                H[i + 1, j] = -sn[i] * H[i, j] + cs[i] * H[i + 1, j]
                H[i, j] = t
            den = math.hypot(H[j, j], H[j + 1, j])
            cs[j], sn[j] = (1.0, 0.0) if den == 0.0 else (H[j, j] / den, H[j + 1, j] / den)
            H[j, j] = cs[j] * H[j, j] + sn[j] * H[j + 1, j]
            H[j + 1, j] = 0.0
            g[j + 1] = -sn[j] * g[j]
            g[j] = cs[j] * g[j]
            n_it += 1
            k = j + 1
            if abs(g[j + 1]) <= target or hn == 0.0 or n_it >= max_it:
                break
            Vb[j + 1] = (w / hn).view_as(b)
        y = np.linalg.solve(np.triu(H[:k, :k]), g[:k])
        x += (torch.from_numpy(y).to(b.device, b.dtype) @ Vf[:k]).view_as(b)
        r = b - apply(x)
        beta = float(torch.linalg.vector_norm(r))
    return x, n_it, beta


class BDFStepper:
    """BDF1 then BDF2 steps of constant size dt with Newton-GMRES on the device JVP."""

    COEFFS = {1: (1.0, 0.0, 1.0), 2: (4.0 / 3.0, -1.0 / 3.0, 2.0 / 3.0)}

    def __init__(self, solver, dt: float, snes_rtol: float = 1e-8, snes_atol: float = 1e-50, ksp_rtol: float = 1e-5, restart: int = 30,
                 max_newton: int = 20, stream: int | None = None):
        import torch
        self.torch = torch
        self.s = solver
        self.dt = float(dt)
        self.snes_rtol, self.snes_atol, self.ksp_rtol, self.restart, self.max_newton = snes_rtol, snes_atol, ksp_rtol, restart, max_newton
        self.stream = stream
        kind = torch.from_numpy(np.asarray(solver.mesh.cell_kind)).to(torch.device("cuda", solver.device))
        self.owned = (kind == L.CELL_OWNED)[:, None].to(torch.float64)
        self.prev = None
        self.stats = {"steps": 0, "newton": 0, "gmres": 0, "rhs": 0, "jvp": 0}

    def _st(self):
        return self.stream if self.stream is not None else self.torch.cuda.current_stream().cuda_stream

    def _F(self, U):
        self.s.FillGhostsDevice(U.data_ptr(), self._st())
        F = self.torch.zeros_like(U)
        self.s.ComputeRHSDevice(0.0, U.data_ptr(), F.data_ptr(), L.PRECISION_FP64, self._st())
        self.stats["rhs"] += 1
        return F

    def step(self, U):
        """One step in place on U (ghosts filled on return); BDF1 on the first call, BDF2 after."""
        torch = self.torch
        order = 1 if self.prev is None else 2
        a1, a2, beta = self.COEFFS[order]
        Un = U.clone()
        base = a1 * Un + (a2 * self.prev if order == 2 else 0.0)
        bdt = beta * self.dt
        st = self._st()

        def residual(X):
            return self.owned * (X - base - bdt * self._F(X))

        R = residual(U)
        r0 = float(torch.linalg.vector_norm(R))
        for _ in range(self.max_newton):
            rn = float(torch.linalg.vector_norm(R))
            if rn <= max(self.snes_rtol * r0, self.snes_atol):
                break

            def apply(v):
                dV = v.clone()
                self.s.FillGhostsJVPDevice(dV.data_ptr(), st)
                dF = torch.zeros_like(v)
                self.s.ComputeJVPDevice(0.0, U.data_ptr(), dV.data_ptr(), dF.data_ptr(), 0, st)
                self.stats["jvp"] += 1
                return self.owned * (v - bdt * dF)

            delta, its, _ = gmres(apply, -R, restart=self.restart, rtol=self.ksp_rtol)
            self.stats["gmres"] += its
            self.stats["newton"] += 1
            U += self.owned * delta
            R = residual(U)
        self.s.FillGhostsDevice(U.data_ptr(), st)
        self.prev = Un
        self.stats["steps"] += 1
        return U
