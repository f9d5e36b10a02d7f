"""Numpy restatement of MarDyn's step for rigid multi-centre LJ molecules (the checker).

TEST INFRASTRUCTURE ONLY: imported by tests/ and by the CPU-baseline leg of ``bench.py``. The
package never imports it. Pinned against the reference itself (oracle/_ref/ref_driver, golden
fixtures in tests/golden/rigid_*.npz made by tests/golden/make_rigid_golden.py).

What it restates, in the reference's own operation order where rounding matters:

* the site-pair parameter streams of ``Comp2Param::initialize`` (mardyn/molecules/Comp2Param.cpp:
  28-115): same component: eps24 = 24 sqrt(eps_i eps_j), sig2 = ((sig_i + sig_j)/2)^2, shift6 of
  the row centre (Component::addLJcenter's 24 eps ((sig/rc)^6 - (sig/rc)^12) when truncated-shifted,
  Component.cpp:44-72); different components: eps24 = 24 xi sqrt(eps_i eps_j),
  sig2 = (eta (sig_i + sig_j)/2)^2, shift6 always from rcLJ;
* the LJ block of ``PotForce`` (mardyn/molecules/potforce.h:319-363) for every molecule pair whose
  centres are closer than rc (strict, BlockTraverse.cpp:155), all centre pairs evaluated when
  dd < rcLJ^2: drs = drm + d_i - d_j (SiteSiteDistance, potforce.h:26-31), ``PotForceLJ``
  (potforce.h:41-53), u += shift6, site forces +f on i and -f on j, Upot6LJ += u,
  Virial += drm . f;
* its charge-charge block (potforce.h:372-386) for every such pair: ``PotForce2Charge``
  (potforce.h:244-253: u = q_i q_j / r with 1/r = sqrt(1/r^2), f = u / r^2 drs; the product
  q_i q_j of Comp2Param.cpp:126-135), UpotXpoles += u, Virial += drm . f;
  Upot = Upot6LJ / 6 + UpotXpoles (ParticlePairs2PotForceAdapter::finish);
* ``Molecule::upd_cache`` (Molecule.cpp:161-190): site offsets d = q.rotateinv(site) of the LJ
  centres and the charges;
* ``Molecule::calcFM`` (Molecule.cpp:386-411): F = sum of site forces, M = sum d x F_site over all
  sites;
* ``Molecule::upd_preF`` / ``upd_postF`` (Molecule.cpp:128-159, 193-216) with the quaternion
  algebra of Quaternion.cpp (rotate, rotateinv, differentiate);
* the periodic wrap of DomainDecompDummy::exchangeMolecules (r + L below 0, r - L at or above L).

Pairs use the minimum image (the box must exceed twice the cutoff), which is the reference's
halo image of the partner for every pair within rc.
"""
from __future__ import annotations

import math
from typing import Dict, List

import numpy as np


# ----------------------------------------------------------------------------- quaternions

def rotate(q: np.ndarray, d: np.ndarray) -> np.ndarray:
    """Quaternion::rotate (space frame -> body frame) for arrays q (N, 4) and d (N, 3)."""
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    ww, xx, yy, zz = w * w, x * x, y * y, z * z
    xy, zw, xz, yw = x * y, z * w, x * z, y * w
    yz, xw = y * z, x * w
    out = np.empty_like(d)
    out[:, 0] = (ww + xx - yy - zz) * d[:, 0] + 2. * (xy + zw) * d[:, 1] + 2. * (xz - yw) * d[:, 2]
    out[:, 1] = 2. * (xy - zw) * d[:, 0] + (ww - xx + yy - zz) * d[:, 1] + 2. * (yz + xw) * d[:, 2]
    out[:, 2] = 2. * (xz + yw) * d[:, 0] + 2. * (yz - xw) * d[:, 1] + (ww - xx - yy + zz) * d[:, 2]
    return out


def rotate_inv(q: np.ndarray, d: np.ndarray) -> np.ndarray:
    """Quaternion::rotateinv (body frame -> space frame)."""
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    ww, xx, yy, zz = w * w, x * x, y * y, z * z
    xy, zw, xz, yw = x * y, z * w, x * z, y * w
    yz, xw = y * z, x * w
    out = np.empty_like(d)
    out[:, 0] = (ww + xx - yy - zz) * d[:, 0] + 2. * (xy - zw) * d[:, 1] + 2. * (xz + yw) * d[:, 2]
    out[:, 1] = 2. * (xy + zw) * d[:, 0] + (ww - xx + yy - zz) * d[:, 1] + 2. * (yz - xw) * d[:, 2]
    out[:, 2] = 2. * (xz - yw) * d[:, 0] + 2. * (yz + xw) * d[:, 1] + (ww - xx - yy + zz) * d[:, 2]
    return out


def differentiate(q: np.ndarray, w: np.ndarray) -> np.ndarray:
    """Quaternion::differentiate: dq/dt for body angular velocity w."""
    qw, qx, qy, qz = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    out = np.empty_like(q)
    out[:, 0] = .5 * (-qx * w[:, 0] - qy * w[:, 1] - qz * w[:, 2])
    out[:, 1] = .5 * (qw * w[:, 0] - qz * w[:, 1] + qy * w[:, 2])
    out[:, 2] = .5 * (qz * w[:, 0] + qw * w[:, 1] - qx * w[:, 2])
    out[:, 3] = .5 * (-qy * w[:, 0] + qx * w[:, 1] + qw * w[:, 2])
    return out


# ----------------------------------------------------------------------------- parameters

class Model:
    """Per-component LJ centres and the site-pair parameter streams of a system."""

    def __init__(self, system):
        comps = system.components
        self.nc = len(comps)
        self.centres = [c.lj_centres() for c in comps]
        self.charges = [c.point_charges() for c in comps]
        # site positions: the LJ centres, then the charges (the reference's site order)
        self.site_r = [np.array([[t.x, t.y, t.z] for t in cs + qs]).reshape(-1, 3)
                       for cs, qs in zip(self.centres, self.charges)]
        self.nlj = [len(cs) for cs in self.centres]
        self.mass = np.array([c.mass for c in comps])
        self.I = np.stack([c.moments() for c in comps])
        self.invI = np.where(self.I != 0.0, 1.0 / np.where(self.I != 0.0, self.I, 1.0), 0.0)
        self.rc, self.rclj = float(system.cutoff), float(system.lj_cutoff)
        self.L = np.asarray(system.length, dtype=np.float64)
        rclj = self.rclj
        tab: Dict = {}
        k = 0
        for ci in range(self.nc):
            for si, a in enumerate(self.centres[ci]):
                shift_a = 0.0
                if a.do_shift:
                    s2 = a.sigma * a.sigma / (rclj * rclj)
                    s6 = s2 * s2 * s2
                    shift_a = 24.0 * a.eps * (s6 - s6 * s6)
                for sj, b in enumerate(self.centres[ci]):
                    sig2 = .5 * (a.sigma + b.sigma)
                    tab[(ci, ci, si, sj)] = (24. * math.sqrt(a.eps * b.eps), sig2 * sig2, shift_a)
            for cj in range(ci + 1, self.nc):
                xi, eta = float(system.mix[k, 0]), float(system.mix[k, 1])
                k += 1
                for si, a in enumerate(self.centres[ci]):
                    for sj, b in enumerate(self.centres[cj]):
                        e24 = 24. * xi * math.sqrt(a.eps * b.eps)
                        sig2 = eta * .5 * (a.sigma + b.sigma)
                        sig2 *= sig2
                        p2 = sig2 / (rclj * rclj)
                        p6 = p2 * p2 * p2
                        sh = e24 * (p6 - p6 * p6)
                        tab[(ci, cj, si, sj)] = (e24, sig2, sh)
                        tab[(cj, ci, sj, si)] = (e24, sig2, sh)
        self.tab = tab


# ----------------------------------------------------------------------------- forces

def site_offsets(model: Model, cid: np.ndarray, q: np.ndarray) -> List[np.ndarray]:
    """upd_cache: per site index s, the (N, 3) space-frame offsets (zero where a molecule has fewer
    centres)."""
    ns = max(len(r) for r in model.site_r)
    out = [np.zeros((cid.shape[0], 3)) for _ in range(ns)]
    for c in range(model.nc):
        sel = cid == c
        for s in range(len(model.site_r[c])):
            out[s][sel] = rotate_inv(q[sel], np.repeat(model.site_r[c][s][None, :], int(sel.sum()), axis=0))
    return out


def forces(model: Model, r: np.ndarray, cid: np.ndarray, q: np.ndarray) -> Dict:
    """F, M per molecule, Upot (Upot6LJ/6 + UpotXpoles), virial and the number of molecule pairs
    within rc."""
    n = r.shape[0]
    L = model.L
    d = site_offsets(model, cid, q)
    F = np.zeros((n, 3))
    M = np.zeros((n, 3))
    U6 = 0.0
    UX = 0.0
    W = 0.0
    npairs = 0
    rc2, rclj2 = model.rc * model.rc, model.rclj * model.rclj
    for i in range(n - 1):
        j = np.arange(i + 1, n)
        drm = r[i][None, :] - r[j]
        drm -= L[None, :] * np.round(drm / L[None, :])
        dd = np.einsum("ij,ij->i", drm, drm)
        near = dd < rc2
        j, drm, dd = j[near], drm[near], dd[near]
        npairs += int(j.shape[0])
        ci = int(cid[i])
        # charge-charge: every pair within rc
        for cj in range(model.nc):
            sel = cid[j] == cj
            if not sel.any() or not model.charges[ci] or not model.charges[cj]:
                continue
            jj, dm = j[sel], drm[sel]
            for a, qa in enumerate(model.charges[ci]):
                di = d[model.nlj[ci] + a][i]
                for b, qb in enumerate(model.charges[cj]):
                    dj = d[model.nlj[cj] + b][jj]
                    drs = dm + di[None, :] - dj
                    dr2 = np.einsum("ij,ij->i", drs, drs)
                    invdr2 = 1.0 / dr2
                    invdr = np.sqrt(invdr2)
                    u = (qa.q * qb.q) * invdr
                    f = (u * invdr2)[:, None] * drs
                    F[i] += f.sum(axis=0)
                    np.subtract.at(F, jj, f)
                    M[i] += np.cross(di[None, :], f).sum(axis=0)
                    np.subtract.at(M, jj, np.cross(dj, f))
                    UX += float(u.sum())
                    W += float(np.einsum("ij,ij->", dm, f))
        lj = dd < rclj2
        j, drm = j[lj], drm[lj]
        for cj in range(model.nc):
            sel = cid[j] == cj
            if not sel.any():
                continue
            jj, dm = j[sel], drm[sel]
            for si in range(len(model.centres[ci])):
                di = d[si][i]
                for sj in range(len(model.centres[cj])):
                    dj = d[sj][jj]
                    e24, sig2, sh6 = model.tab[(ci, cj, si, sj)]
                    drs = dm + di[None, :] - dj
                    dr2 = np.einsum("ij,ij->i", drs, drs)
                    inv = 1. / dr2
                    lj6 = sig2 * inv
                    lj6 = lj6 * lj6 * lj6
                    lj12 = lj6 * lj6
                    lj12m6 = lj12 - lj6
                    u = e24 * lj12m6 + sh6
                    fac = e24 * (lj12 + lj12m6) * inv
                    f = fac[:, None] * drs
                    F[i] += f.sum(axis=0)
                    np.subtract.at(F, jj, f)
                    M[i] += np.cross(di[None, :], f).sum(axis=0)
                    np.subtract.at(M, jj, np.cross(dj, f))
                    U6 += float(u.sum())
                    W += float(np.einsum("ij,ij->", dm, f))
    return dict(F=F, M=M, upot=U6 / 6.0 + UX, virial=W, npairs=npairs)


# ----------------------------------------------------------------------------- integration

def leapfrog_pre(model: Model, st: Dict, dt: float, vcorr: float = 1.0, Dcorr: float = 1.0) -> None:
    """Molecule::upd_preF for every molecule (in place on st's r, v, q, D)."""
    cid = st["cid"]
    m = model.mass[cid][:, None]
    invI = model.invI[cid]
    dt_half = .5 * dt
    st["v"] = vcorr * st["v"] + (dt_half / m) * st["F"]
    st["r"] = st["r"] + dt * st["v"]
    q = st["q"]
    w = rotate(q, st["D"]) * invI
    qh = differentiate(q, w) * dt_half + q
    qh = qh * (1. / np.sqrt(np.sum(qh * qh, axis=1)))[:, None]
    st["D"] = Dcorr * st["D"] + dt_half * st["M"]
    w = rotate(qh, st["D"]) * invI
    q = q + differentiate(qh, w) * dt
    st["q"] = q * (1. / np.sqrt(np.sum(q * q, axis=1)))[:, None]


def leapfrog_post(model: Model, st: Dict, dt_half: float) -> Dict:
    """Molecule::upd_postF for every molecule: the closing kicks, sum m v^2 and sum I w^2."""
    cid = st["cid"]
    m = model.mass[cid][:, None]
    st["v"] = st["v"] + (dt_half / m) * st["F"]
    st["D"] = st["D"] + dt_half * st["M"]
    w = rotate(st["q"], st["D"]) * model.invI[cid]
    return dict(summv2=float(np.sum(m * st["v"] * st["v"])),
                sum_iw2=float(np.sum(model.I[cid] * w * w)))


def wrap(model: Model, r: np.ndarray) -> np.ndarray:
    L = model.L[None, :]
    return np.where(r < 0.0, r + L, np.where(r >= L, r - L, r))


def run(system, nsteps: int, dump_steps=()) -> Dict:
    """prepare_start (forces of the start), then nsteps reference steps: upd_preF, wrap, forces,
    upd_postF. Returns per-step scalars and the states of dump_steps (0 = after prepare_start)."""
    model = Model(system)
    st = dict(cid=system.cid.astype(np.int64), r=wrap(model, system.r.copy()), v=system.v.copy(),
              q=system.q.copy(), D=system.D.copy())
    f = forces(model, st["r"], st["cid"], st["q"])
    st["F"], st["M"] = f["F"], f["M"]
    scal = [dict(step=0, upot=f["upot"], virial=f["virial"], npairs=f["npairs"])]
    dumps = {}
    if 0 in dump_steps:
        dumps[0] = {k: np.array(v) for k, v in st.items()}
    for k in range(1, nsteps + 1):
        leapfrog_pre(model, st, system.dt)
        st["r"] = wrap(model, st["r"])
        f = forces(model, st["r"], st["cid"], st["q"])
        st["F"], st["M"] = f["F"], f["M"]
        kin = leapfrog_post(model, st, .5 * system.dt)
        scal.append(dict(step=k, upot=f["upot"], virial=f["virial"], npairs=f["npairs"], **kin))
        if k in dump_steps:
            dumps[k] = {kk: np.array(v) for kk, v in st.items()}
    return dict(scalars=scal, dumps=dumps)
