"""Tangent and adjoint of a march of explicit steps on the device, for gradients of a functional of the
marched state (the wall-pressure functional of abl_fv_pressure_functional) with respect to the initial
state and the boundary-condition values.

The march is the one abl_fv_step runs (src/solver/timeStepper.cpp drives the same steps through PETSc
TS): every stage fills the ghost rows, evaluates the RHS and combines the owned rows; the step ends with
a fill. Written here from its pieces (abl_fv_fill_ghosts, abl_fv_rhs, abl_fv_rk_stage) so that the
backward pass can recompute the stage states bit for bit. The step size is fixed: a CFL-chosen step is
a minimum over cells and has no useful derivative. Species normalisation is a clip; the march is
differentiated without species only (the stepper raises otherwise).

Reverse of one stage V -> U' = a V0 + b (V + dt F(V)) on the owned rows, then V' = fill(U'):
    lambda_U'  = fill^T(lambda_V')            (abl_fv_fill_ghosts_vjp; the value adjoints accumulate)
    lambda_V  += b lambda_U' + b dt J(V)^T lambda_U'   (abl_fv_vjp)
    lambda_V0 += a lambda_U'
The reference has no adjoint; its counterpart would be PETSc's TSAdjoint over a finite-difference
Jacobian of ComputeRHSFunction.
"""
from __future__ import annotations

import numpy as np

from . import _lib as L


def _torch():
    import torch
    return torch


class ExplicitMarch:
    """n_steps explicit steps of size dt (L.STEP_EULER or L.STEP_SSPRK3) of `solver` on torch tensors of
    shape (n_cells, nc) on the solver's GPU, FP64."""

    # Shu-Osher stages: (a, b) of U' = a V0 + b (V + dt F(V))
    STAGES = {L.STEP_EULER: [(0.0, 1.0)], L.STEP_SSPRK3: [(0.0, 1.0), (0.75, 0.25), (1.0 / 3.0, 2.0 / 3.0)]}

    def __init__(self, solver, scheme: int, dt: float, n_steps: int, stream: int | None = None):
        if scheme not in self.STAGES:
            raise ValueError("unknown scheme")
        if solver.nc - 2 - solver.mesh.dim != 0:
            raise ValueError("the march is differentiated without species (normalisation is a clip)")
        self.s = solver
        self.scheme = scheme
        self.dt = float(dt)
        self.n_steps = int(n_steps)
        self.torch = _torch()
        self.stream = stream
        self.checkpoints: list = []

    def _st(self):
        return self.stream if self.stream is not None else self.torch.cuda.current_stream().cuda_stream

    def _rhs(self, V):
        F = self.torch.zeros_like(V)
        self.s.ComputeRHSDevice(0.0, V.data_ptr(), F.data_ptr(), L.PRECISION_FP64, self._st())
        return F

    def _stages(self, U):
        """The stage inputs V_0 .. V_{s-1} of one step from U (ghosts filled) and the step's output."""
        st = self._st()
        V0 = U.clone()
        self.s.FillGhostsDevice(V0.data_ptr(), st)
        Vs = [V0]
        V = V0
        for a, b in self.STAGES[self.scheme]:
            F = self._rhs(V)
            Un = V.clone()
            self.s.RkStageDevice(a, V0.data_ptr() if a != 0.0 else 0, b, V.data_ptr(), self.dt, F.data_ptr(), Un.data_ptr(), st)
            self.s.FillGhostsDevice(Un.data_ptr(), st)
            Vs.append(Un)
            V = Un
        return Vs[:-1], Vs[-1]

    def forward(self, U0, keep: bool = True):
        """March from U0 (not modified); keeps every step's starting state for the backward pass."""
        self.checkpoints = []
        U = U0.clone()
        for _ in range(self.n_steps):
            if keep:
                self.checkpoints.append(U.clone())
            _, U = self._stages(U)
        return U

    def tangent(self, U0, dU0):
        """Forward-mode derivative of the march: returns (U_K, dU_K) for the initial perturbation dU0 (the
        condition values held fixed)."""
        st = self._st()
        U, dU = U0.clone(), dU0.clone()
        for _ in range(self.n_steps):
            V0, dV0 = U.clone(), dU.clone()
            self.s.FillGhostsDevice(V0.data_ptr(), st)
            self.s.FillGhostsJVPDevice(dV0.data_ptr(), st)
            V, dV = V0, dV0
            for a, b in self.STAGES[self.scheme]:
                F = self.torch.zeros_like(V)
                dF = self.torch.zeros_like(V)
                self.s.ComputeJVPDevice(0.0, V.data_ptr(), dV.data_ptr(), dF.data_ptr(), F.data_ptr(), st)
                Un, dUn = V.clone(), dV.clone()
                self.s.RkStageDevice(a, V0.data_ptr() if a != 0.0 else 0, b, V.data_ptr(), self.dt, F.data_ptr(), Un.data_ptr(), st)
                self.s.RkStageDevice(a, dV0.data_ptr() if a != 0.0 else 0, b, dV.data_ptr(), self.dt, dF.data_ptr(), dUn.data_ptr(), st)
                self.s.FillGhostsDevice(Un.data_ptr(), st)
                self.s.FillGhostsJVPDevice(dUn.data_ptr(), st)
                V, dV = Un, dUn
            U, dU = V, dV
        return U, dU

    def adjoint(self, lam_K):
        """Reverse pass from the adjoint of the final state (after forward()). Returns (lambda_0, vbar):
        lambda_0 the gradient with respect to the initial state (every row; ghost rows 0, since the first
        fill overwrites them) and vbar[n_bc][16] the gradient with respect to the condition values."""
        if len(self.checkpoints) != self.n_steps:
            raise RuntimeError("run forward(keep=True) first")
        st = self._st()
        vbar = np.zeros((self.s._n_bc, L.BC_MAX_COMPONENTS))
        lam = lam_K.clone()
        stages = self.STAGES[self.scheme]
        for k in range(self.n_steps - 1, -1, -1):
            Vs, _ = self._stages(self.checkpoints[k])
            lamV = [self.torch.zeros_like(lam) for _ in Vs]
            lamU = lam
            for i in range(len(stages) - 1, -1, -1):
                a, b = stages[i]
                vbar += self.s.FillGhostsVJPDevice(lamU.data_ptr(), st)
                # U' = a V0 + b (V_i + dt F(V_i)) on the owned rows; lamU's ghost rows are 0 here
                lamV[i] += b * lamU
                Fbar = (b * self.dt) * lamU
                self.s.ComputeVJPDevice(0.0, Vs[i].data_ptr(), Fbar.data_ptr(), lamV[i].data_ptr(), st)
                if a != 0.0:
                    lamV[0] += a * lamU
                if i > 0:
                    lamU = lamV[i]
            lam = lamV[0]
            vbar += self.s.FillGhostsVJPDevice(lam.data_ptr(), st)
        return lam, vbar


def functional_gradient(solver, march: ExplicitMarch, U0):
    """J(U_K) of the registered pressure functional after the march, and its gradients: returns
    (J, dJ/dU0 as a torch tensor, dJ/d(condition values) as an array (n_bc, 16))."""
    torch = _torch()
    UK = march.forward(U0, keep=True)
    lam = torch.zeros_like(UK)
    J = solver.PressureFunctionalDevice(UK.data_ptr(), lam.data_ptr(), march._st())
    lam0, vbar = march.adjoint(lam)
    return J, lam0, vbar


def inlet_state(rho: float, p: float, speed: float, direction, gamma: float = 1.4) -> tuple[np.ndarray, np.ndarray]:
    """Conserved Dirichlet inlet state [rho, rho E, rho u] of a perfect gas entering at `speed` along
    `direction`, and its derivative with respect to the speed."""
    d = np.asarray(direction, float)
    d = d / np.linalg.norm(d)
    value = np.concatenate([[rho, p / (gamma - 1.0) + 0.5 * rho * speed ** 2], rho * speed * d])
    dvalue = np.concatenate([[0.0, rho * speed], rho * d])
    return value, dvalue
