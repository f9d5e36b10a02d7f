"""Reverse-mode gradients through Leapfrog trajectories, with step checkpointing, on the device.

The forward map of one step is the reference's NVE step (Leapfrog, vcorr = 1):

    v_h = v_k + c F_k,  r_{k+1} = r_k + dt v_h,  F_{k+1} = F(r_{k+1}),  v_{k+1} = v_h + c F_{k+1}

with c = dt / (2 m). ``mdgpu_traj_forward`` runs it keeping every ``checkpoint_every``-th state as a
device snapshot; ``mdgpu_traj_backward`` recomputes each segment from its snapshot on the device
and walks it backwards with the force map's vector-Jacobian product (the adjoint kernel) and the
Leapfrog part in small device kernels. Only the cotangents go in and the gradients come out.
"""
from __future__ import annotations

import numpy as np

from . import mdgpu as M


class TrajectoryAdjoint:
    """Gradient of a loss on the final forces/energy of an n-step NVE trajectory with respect to the
    initial positions and velocities and the component-pair parameters eps_ab, sigma_ab."""

    def __init__(self, system, nsteps: int, checkpoint_every: int = 10, device: int = 0, precision: int = M.FP64):
        self.system = system
        self.nsteps = int(nsteps)
        self.every = int(checkpoint_every)
        self.lc = M.LinkedCells.from_system(system, precision, device)
        self.dt = float(system.dt)
        self.checkpoints = list(range(0, self.nsteps, min(self.every, self.nsteps)))
        self.recomputed_steps = 0

    def close(self) -> None:
        self.lc.close()

    def forward(self, r0: np.ndarray, v0: np.ndarray):
        """Runs the trajectory keeping device snapshots; returns the final (r, v, F, U)."""
        self.lc.setState(r=r0, v=v0)
        u = self.lc.trajForward(self.nsteps, self.every, self.dt)
        st = self.lc.getParticles()
        return st["r"], st["v"], st["F"], u

    def backward(self, gF_final: np.ndarray, gU_final: float):
        """Cotangents of the final forces and energy -> (dL/dr0, dL/dv0, dL/deps_ab, dL/dsigma_ab)."""
        gr, gv, ge, gs, rec = self.lc.trajBackward(gF_final, gU_final)
        self.recomputed_steps = rec
        return gr, gv, ge, gs
