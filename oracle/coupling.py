"""NumPy restatement of the molecule-side operations of MaDPaC's coupled MD step
(MarDynSimulation::simulateStep, mardyn/coupling/MarDynSimulation.cpp:61-160 of the reference
bundle): the reflecting boundary, the boundary force and the cell-wise thermostat.

TEST INFRASTRUCTURE ONLY: imported by tests/ (the checker of madpac_b200's coupling kernels).

* reflect: ReflectingBoundary::applyBoundary (mardyn/coupling/boundary/ReflectingBoundary.cpp:47-130)
  with its own arithmetic, pinned by fixtures the compiled reference writes
  (tests/golden/make_coupling_golden.py).
* calc_fm: ForceBoundary::calcFm (mardyn/coupling/boundary/ForceBoundary.h:56-82), the
  piecewise-polynomial wall force fit, pinned by samples of the compiled function.
* force_boundary: the force ForceBoundary::applyBoundary (ForceBoundary.cpp:52-226) computes for
  each molecule of a boundary region (FBoundary::getLower/getUpper regions, FBoundary.cpp:25-56;
  LinkedCells::getRegion's low <= r < high, LinkedCells.cpp:397-442). In the reference the regions
  are collected into a copy of the list (getLower/getUpper take it by value), so the force is never
  applied; the fixtures record that. This function is what the code computes per molecule.
* CellWiseThermostat: CellWiseThermostat::applyThermostat / saveV / updateLocalE /
  adjustTemperature (mardyn/coupling/thermostat/CellWiseThermostat.cpp:46-195) on a coupling-cell
  grid given as DataContainer gives it (calcIndexX, madpac/core/DataContainer.cpp:209-261). The
  reference class needs the Peano coupling service to be built, so this part is restated from the
  source without a compiled pin.
"""
from __future__ import annotations

import numpy as np


def reflect(r, v, length, dim, stream_out_dir, moving_wall=False, stream_out=False):
    """ReflectingBoundary::applyBoundary on every molecule outside the box (the halo molecules
    after LinkedCells::update): returns (r, v, number streamed out)."""
    r = np.array(r, dtype=np.float64, copy=True)
    v = np.array(v, dtype=np.float64, copy=True)
    so = (not moving_wall) or stream_out  # ReflectingBoundary.cpp:33
    nout = 0
    for m in range(r.shape[0]):
        for i in range(dim):
            if r[m, i] < 0.0:
                a = [0.0, 0.0, 0.0]
                a[i] = -2.0 * v[m, i]
                for d in range(3):
                    v[m, d] = v[m, d] + a[d]
                newpos = -r[m, i] - 2 * r[m, i]
                r[m, i] = r[m, i] + newpos
            elif r[m, i] > length[i]:
                if i != stream_out_dir or not so:
                    a = [0.0, 0.0, 0.0]
                    a[i] = -2.0 * v[m, i]
                    for d in range(3):
                        v[m, d] = v[m, d] + a[d]
                    newpos = -2 * (r[m, i] - length[i])
                    r[m, i] = r[m, i] + newpos
                else:
                    nout += 1
    return r, v, nout


def calc_fm(r):
    """ForceBoundary::calcFm: the wall force at distance r from the boundary (same operation order)."""
    r_w = r / 2.95
    if r_w < 0.2975:
        return 10.8007 + 0.860717 * r_w - 172.468 * r_w * r_w + 86.9134 * r_w * r_w * r_w - 140.214 * r_w * r_w * r_w * r_w
    if r_w < 0.3475:
        return (-3621.30 + 44657.4 * r_w - 204844.0 * r_w * r_w + 414123.0 * r_w * r_w * r_w
                - 311674.0 * r_w * r_w * r_w * r_w)
    if r_w < 0.3975:
        return (4331.63 - 45188.5 * r_w + 176236.0 * r_w * r_w - 305157.0 * r_w * r_w * r_w
                + 198111.0 * r_w * r_w * r_w * r_w)
    if r_w < 1.0:
        return (-94.4796 + 576.282 * r_w - 1436.11 * r_w * r_w + 1804.53 * r_w * r_w * r_w
                - 1133.47 * r_w * r_w * r_w * r_w + 283.244 * r_w * r_w * r_w * r_w * r_w)
    return 0.0


def force_boundary(r, F, length, dim, border, stream_out_dir, stream_damping):
    """The boundary force of each molecule in a boundary region (X, then Y, then Z when dim is 3;
    lower region [0, border), upper region [L - border, L) in that dimension, [0, L) in the others):
    F_d += calcFm(r_d) at the lower face, F_d -= calcFm(L_d - r_d) (times the stream damping in
    the stream-out dimension) at the upper face."""
    F = np.array(F, dtype=np.float64, copy=True)
    L = np.asarray(length, dtype=np.float64)
    inside = np.all((r >= 0.0) & (r < L), axis=1)
    dims = (0, 1, 2) if dim == 3 else (0, 1)
    for d in dims:
        for m in np.nonzero(inside & (r[:, d] < 0.0 + border))[0]:
            F[m, d] = F[m, d] + calc_fm(r[m, d] - 0.0) * 1.0
        for m in np.nonzero(inside & (r[:, d] >= L[d] - border))[0]:
            f = -calc_fm(L[d] - r[m, d]) * 1.0
            if stream_out_dir == d:
                f *= stream_damping
            F[m, d] = F[m, d] + f
    return F


class CellWiseThermostat:
    """CellWiseThermostat on a coupling-cell grid: lower/upper corners, cell size, cells per
    dimension, dim (2 or 3); the target temperature, gamma, interval and the directed flags of its
    configuration."""

    def __init__(self, lower, upper, cell_size, size, dim, target_temperature, gamma, interval, directed):
        self.lower = np.asarray(lower, dtype=np.float64)
        self.upper = np.asarray(upper, dtype=np.float64)
        self.cell_size = float(cell_size)
        self.size = [int(x) for x in size]
        self.dim = int(dim)
        self.T = float(target_temperature)
        self.gamma = float(gamma)
        self.interval = int(interval)
        self.directed = [int(x) for x in directed]
        nc = self.size[0] * self.size[1] * self.size[2]
        self.vsum = np.zeros((nc, 4))
        self.e = np.zeros(nc)

    def index(self, pos):
        """DataContainer::calcIndexX: the cell of a position, -1 outside the coupling box (also at its
        upper corner, whose cell index would lie past the grid)."""
        ip = [0, 0, 0]
        for i in range(self.dim):
            if not (self.lower[i] <= pos[i] <= self.upper[i]):
                return -1
            ip[i] = int((pos[i] - self.lower[i]) / self.cell_size)
            if ip[i] >= self.size[i]:
                return -1
        if self.dim == 2:
            ip[2] = 0
        return (ip[0] * self.size[1] + ip[1]) * self.size[2] + ip[2]

    def apply(self, r, v, mass, iteration):
        """applyThermostat(iteration) on the molecules (r, v, per-molecule mass); returns the new v."""
        v = np.array(v, dtype=np.float64, copy=True)
        idx = np.array([self.index(p) for p in r])
        # saveV
        for m in range(len(idx)):
            k = idx[m]
            if k > -1:
                for i in range(3):
                    self.vsum[k, i] += v[m, i]
                self.vsum[k, 3] = self.vsum[k, 3] + 1
        if self.interval != 0 and iteration % self.interval == 0:
            # updateLocalE
            vc = np.zeros((len(self.vsum), 3))
            for j in range(len(self.vsum)):
                for i in range(3):
                    vc[j, i] = self.vsum[j, i] / self.vsum[j, 3] if self.directed[i] != 0 else 0.0
            self.e[:] = 0.0
            for m in range(len(idx)):
                k = idx[m]
                if k > -1:
                    e = 0.0
                    for i in range(3):
                        t = v[m, i] - vc[k, i]
                        e += t * t
                    e *= 0.5 * mass[m]
                    self.e[k] += e
            # adjustTemperature
            for m in range(len(idx)):
                k = idx[m]
                if k > -1:
                    target = 1.5 * self.vsum[k, 3] / float(self.interval) * self.T
                    beta = np.sqrt(target / self.e[k])
                    for i in range(3):
                        v[m, i] = v[m, i] - vc[k, i]
                    s = 1.0 + self.gamma * (beta - 1.0)
                    for i in range(3):
                        v[m, i] *= s
                    for i in range(3):
                        v[m, i] = v[m, i] + vc[k, i]
            self.vsum[:] = 0.0
        return v
