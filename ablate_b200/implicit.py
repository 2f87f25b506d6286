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
    """BDF1 then BDF2 steps of constant size dt with Newton-GMRES on the device JVP.

    Newton stops at ||R|| <= max(snes_rtol ||R_0||, snes_atol) or when the update is below
    snes_stol ||U|| (PETSc's SNES defaults 1e-8, 1e-50, 1e-8), after at most max_newton iterations;
    each update is backtracked (halved up to 4 times) until ||R|| falls by the Armijo factor
    1 - 1e-4 lambda (PETSc's SNESNEWTONLS uses a backtracking line search by default). Each GMRES solve
    stops at ksp_rtol or after ksp_max_it iterations; with `scale` it runs on the state divided by each
    component's RMS over the owned cells (density, energy and momenta differ by five orders of
    magnitude). The tangent is the frozen-limiter one by default (L.JVP_FROZEN_LIMITER): the exact
    derivative of a limited scheme holds 1/(grad . dx) terms and jumps where the minimising face
    changes, and GMRES(30) stagnates on it. Every Newton iteration is logged in `log` (step, iteration,
    ||R||, GMRES iterations, GMRES residual / ||b||, line-search factor)."""

    COEFFS = {1: (1.0, 0.0, 1.0), 2: (4.0 / 3.0, -1.0 / 3.0, 2.0 / 3.0)}

    def __init__(self, solver, dt: float, snes_rtol: float = 1e-8, snes_atol: float = 1e-50, snes_stol: float = 1e-8, ksp_rtol: float = 1e-5,
                 restart: int = 30, max_newton: int = 10, ksp_max_it: int = 300, jvp_mode: int = L.JVP_FROZEN_LIMITER, scale: bool = True,
                 stream: int | None = None):
        import torch
        self.torch = torch
        self.s = solver
        self.dt = float(dt)
        self.snes_rtol, self.snes_atol, self.snes_stol = snes_rtol, snes_atol, snes_stol
        self.ksp_rtol, self.restart, self.max_newton, self.ksp_max_it = ksp_rtol, restart, max_newton, ksp_max_it
        self.stream = stream
        self.jvp_mode, self.scale = jvp_mode, scale
        self.owned = self._owned_mask()
        self.prev = None
        self.stats = {"steps": 0, "newton": 0, "gmres": 0, "rhs": 0, "jvp": 0, "ksp_unconverged": 0, "snes_unconverged": 0}
        self.log: list = []
        self.reductions: list = []  # per step, final ||R|| / initial ||R||

    # the device operations (a test substitutes its own)
    def _owned_mask(self):
        kind = self.torch.from_numpy(np.asarray(self.s.mesh.cell_kind)).to(self.torch.device("cuda", self.s.device))
        return (kind == L.CELL_OWNED)[:, None].to(self.torch.float64)

    def _st(self):
        return self.stream if self.stream is not None else self.torch.cuda.current_stream().cuda_stream

    def _fill(self, U):
        self.s.FillGhostsDevice(U.data_ptr(), self._st())

    def _rhs(self, U):
        F = self.torch.zeros_like(U)
        self.s.ComputeRHSDevice(0.0, U.data_ptr(), F.data_ptr(), L.PRECISION_FP64, self._st())
        return F

    def _fill_tangent(self, dU):
        self.s.FillGhostsJVPDevice(dU.data_ptr(), self._st())

    def _set_mode(self, mode):
        self.s.SetJVPMode(mode)

    def _jvp(self, U, dU):
        dF = self.torch.zeros_like(U)
        self.s.ComputeJVPDevice(0.0, U.data_ptr(), dU.data_ptr(), dF.data_ptr(), 0, self._st())
        return dF

    def step(self, U):
        """One step in place on U (ghosts filled on return); BDF1 on the first call, BDF2 after."""
        self._set_mode(self.jvp_mode)
        try:
            return self._step(U)
        finally:
            self._set_mode(L.JVP_EXACT)

    def _step(self, U):
        torch = self.torch
        order = 1 if self.prev is None else 2
        a1, a2, beta = self.COEFFS[order]
        Un = U.clone()
        base = a1 * Un + (a2 * self.prev if order == 2 else 0.0)
        bdt = beta * self.dt
        if self.scale:
            n_owned = float(self.owned.sum())
            rms = torch.sqrt((self.owned * U * U).sum(0, keepdim=True) / max(n_owned, 1.0))
            D = torch.clamp(rms, min=float(rms.max()) * 1e-12 + 1e-300).expand_as(U)
        else:
            D = None

        def residual(X):
            self._fill(X)
            self.stats["rhs"] += 1
            return self.owned * (X - base - bdt * self._rhs(X))

        def apply(v):
            dV = v.clone()
            self._fill_tangent(dV)
            self.stats["jvp"] += 1
            return self.owned * (v - bdt * self._jvp(U, dV))

        R = residual(U)
        r0 = float(torch.linalg.vector_norm(R))
        rn = r0
        converged = r0 <= self.snes_atol
        for it in range(self.max_newton):
            if converged:
                break
            b = -R
            if D is not None:
                y, its, res = gmres(lambda z: apply(z * D) / D, b / D, restart=self.restart, rtol=self.ksp_rtol, max_it=self.ksp_max_it)
                delta = y * D
                bn = float(torch.linalg.vector_norm(b / D))
            else:
                delta, its, res = gmres(apply, b, restart=self.restart, rtol=self.ksp_rtol, max_it=self.ksp_max_it)
                bn = float(torch.linalg.vector_norm(b))
            self.stats["gmres"] += its
            self.stats["newton"] += 1
            if res > self.ksp_rtol * bn:
                self.stats["ksp_unconverged"] += 1
            U0 = U.clone()
            lam = 1.0
            for _ in range(5):
                U.copy_(U0 + lam * self.owned * delta)
                R = residual(U)
                rl = float(torch.linalg.vector_norm(R))
                if rl <= (1.0 - 1e-4 * lam) * rn:
                    break
                lam *= 0.5
            rn = rl
            self.log.append((self.stats["steps"], it, rn, its, res / bn if bn > 0 else 0.0, lam))
            small_step = lam * float(torch.linalg.vector_norm(delta)) <= self.snes_stol * float(torch.linalg.vector_norm(U))
            converged = rn <= max(self.snes_rtol * r0, self.snes_atol) or small_step
        if not converged:
            self.stats["snes_unconverged"] += 1
        self.reductions.append(rn / r0 if r0 > 0 else 0.0)
        self._fill(U)
        self.prev = Un
        self.stats["steps"] += 1
        return U
