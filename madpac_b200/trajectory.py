"""Reverse-mode gradients through Leapfrog trajectories, with step checkpointing.

The forward map of one step is the device integration of ``mdgpu_leapfrog_pre`` /
``mdgpu_update`` / ``mdgpu_traverse_pairs`` / ``mdgpu_leapfrog_post`` (NVE, vcorr = 1):

    v_h = v_k + c F_k,  r_{k+1} = r_k + dt v_h,  F_{k+1} = F(r_{k+1}),  v_{k+1} = v_h + c F_{k+1}

with c = dt / (2 m). Going backwards through it needs the vector-Jacobian product of the force
map, which ``mdgpu_adjoint`` computes (``LinkedCells.adjoint``). Only every ``checkpoint_every``-th
state is kept during the forward pass; each segment is recomputed from its checkpoint when the
backward pass reaches it, so memory holds one segment of states instead of the whole trajectory.
"""
from __future__ import annotations

from typing import Callable, Dict, List, Tuple

import numpy as np

from . import mdgpu as M


class TrajectoryAdjoint:
    """Gradient of a loss on the final forces/energy of an n-step NVE trajectory with respect to the
    initial positions and velocities and the component-pair parameters eps_ab, sigma_ab."""

    def __init__(self, system, nsteps: int, checkpoint_every: int = 10, device: int = 0):
        self.system = system
        self.nsteps = int(nsteps)
        self.every = int(checkpoint_every)
        self.lc = M.LinkedCells.from_system(system, M.FP64, device)
        self.dt = float(system.dt)
        self.c = (0.5 * self.dt) / system.mass()[system.cid]  # per molecule, (n,)
        self.checkpoints: Dict[int, Tuple[np.ndarray, np.ndarray]] = {}
        self.recomputed_steps = 0

    def close(self) -> None:
        self.lc.close()

    # -- forward ----------------------------------------------------------------------------------
    def _forces(self, r: np.ndarray) -> Tuple[np.ndarray, float]:
        self.lc.setState(r=r)
        self.lc.update()
        u, _, _ = self.lc.traversePairs()
        st = self.lc.getParticles()
        return st["F"], u, st["r"]

    def _step(self, r: np.ndarray, v: np.ndarray, F: np.ndarray):
        """One step on the device; returns (r', v', F', U')."""
        self.lc.setState(r=r, v=v)
        self.lc.update()
        self.lc.traversePairs()  # F at r (the stored force the pre-kick uses)
        self.lc.leapfrogPre(self.dt, 1.0)
        self.lc.update()
        u, _, _ = self.lc.traversePairs()
        self.lc.leapfrogPost(0.5 * self.dt)
        st = self.lc.getParticles()
        return st["r"], st["v"], st["F"], u

    def forward(self, r0: np.ndarray, v0: np.ndarray):
        """Runs the trajectory keeping checkpoints; returns the final (r, v, F, U)."""
        F, u, r = self._forces(r0)
        v = np.array(v0, dtype=np.float64)
        self.checkpoints = {0: (r.copy(), v.copy())}
        for k in range(1, self.nsteps + 1):
            r, v, F, u = self._step(r, v, F)
            if k % self.every == 0 and k < self.nsteps:
                self.checkpoints[k] = (r.copy(), v.copy())
        return r, v, F, u

    def _segment(self, k0: int, k1: int) -> List[Tuple[np.ndarray, np.ndarray, np.ndarray]]:
        """States (r_k, v_k, F_k) for k0..k1 recomputed from the checkpoint at k0."""
        r, v = self.checkpoints[k0]
        F, _, r = self._forces(r)
        out = [(r.copy(), v.copy(), F.copy())]
        for _ in range(k0, k1):
            r, v, F, _ = self._step(r, v, F)
            self.recomputed_steps += 1
            out.append((r.copy(), v.copy(), F.copy()))
        return out

    # -- backward ---------------------------------------------------------------------------------
    def _vjp(self, r: np.ndarray, gF: np.ndarray, gU: float):
        self.lc.setState(r=r)
        self.lc.update()
        self.lc.traversePairs()
        return self.lc.adjoint(gF, gU)

    def backward(self, gF_final: np.ndarray, gU_final: float):
        """Cotangents of the final forces and energy -> (dL/dr0, dL/dv0, dL/deps_ab, dL/dsigma_ab)."""
        n = self.system.n
        ns = len(self.system.components)
        c = self.c[:, None]
        rbar = np.zeros((n, 3))
        vbar = np.zeros((n, 3))
        Fbar = np.array(gF_final, dtype=np.float64)
        gU = float(gU_final)
        geps = np.zeros((ns, ns))
        gsig = np.zeros((ns, ns))
        starts = sorted(self.checkpoints)
        for si in range(len(starts) - 1, -1, -1):
            k0 = starts[si]
            k1 = starts[si + 1] if si + 1 < len(starts) else self.nsteps
            states = self._segment(k0, k1)
            for k in range(k1, k0, -1):
                r_k1 = states[k - k0][0]
                # post-kick v_{k+1} = v_h + c F_{k+1}: F_{k+1} also reaches L through v_{k+1}
                Fbar = Fbar + c * vbar
                # F_{k+1} = F(r_{k+1}): rbar_{k+1} += J^T Fbar_{k+1} (plus the energy cotangent at the end)
                gr, ge, gs = self._vjp(r_k1, Fbar, gU)
                rbar += gr
                geps += ge
                gsig += gs
                gU = 0.0
                # r_{k+1} = r_k + dt v_h and v_h = v_k + c F_k
                vh_bar = vbar + self.dt * rbar
                vbar = vh_bar
                Fbar = c * vh_bar
            # rbar, vbar now belong to state k0; Fbar to F_k0
        gr, ge, gs = self._vjp(self.checkpoints[0][0], Fbar, gU)
        rbar += gr
        geps += ge
        gsig += gs
        return rbar, vbar, geps, gsig
