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
        self.dipoles = [c.point_dipoles() for c in comps]
        self.quads = [c.point_quadrupoles() for c in comps]
        # site positions: the LJ centres, the charges, the dipoles, the quadrupoles (the reference's
        # site order); orientations of the dipoles and quadrupoles
        self.site_r = [np.array([[t.x, t.y, t.z] for t in cs + qs + ds + qq]).reshape(-1, 3)
                       for cs, qs, ds, qq in zip(self.centres, self.charges, self.dipoles, self.quads)]
        self.site_e = [np.array([[0.0, 0.0, 0.0]] * (len(cs) + len(qs)) + [[t.ex, t.ey, t.ez] for t in ds + qq])
                       .reshape(-1, 3) for cs, qs, ds, qq in zip(self.centres, self.charges, self.dipoles, self.quads)]
        self.nlj = [len(cs) for cs in self.centres]
        self.first_dip = [len(cs) + len(qs) for cs, qs in zip(self.centres, self.charges)]
        self.first_quad = [len(cs) + len(qs) + len(ds) for cs, qs, ds in zip(self.centres, self.charges, self.dipoles)]
        eps_rf = float(getattr(system, "epsilon_rf", 1.0e10))
        rc = float(system.cutoff)
        self.eps_rf_inv_rc3 = 2. * (eps_rf - 1.) / ((rc * rc * rc) * (2. * eps_rf + 1.))
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

def site_offsets(model: Model, cid: np.ndarray, q: np.ndarray, orient: bool = False):
    """upd_cache: per site index s, the (N, 3) space-frame offsets (zero where a molecule has fewer
    sites); with orient also the rotated orientation vectors of the dipoles and quadrupoles."""
    ns = max(len(r) for r in model.site_r)
    out = [np.zeros((cid.shape[0], 3)) for _ in range(ns)]
    oe = [np.zeros((cid.shape[0], 3)) for _ in range(ns)]
    for c in range(model.nc):
        sel = cid == c
        k = int(sel.sum())
        for s in range(len(model.site_r[c])):
            out[s][sel] = rotate_inv(q[sel], np.repeat(model.site_r[c][s][None, :], k, axis=0))
            oe[s][sel] = rotate_inv(q[sel], np.repeat(model.site_e[c][s][None, :], k, axis=0))
    return (out, oe) if orient else out


# Point-polarity pair terms of potforce.h, vectorised over pairs (dr: (P, 3), dr2: (P,), e: (P, 3)).

def _dot(a, b):
    return a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1] + a[:, 2] * b[:, 2]


def _cross(a, b):
    return np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1], a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                     a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], axis=1)


def charge_quadrupole(dr, dr2, ejj, qQ025):
    """PotForceChargeQuadrupole (potforce.h:256-281): f, m2 (torque on the quadrupole), u."""
    invdr2 = 1.0 / dr2
    invdr = np.sqrt(invdr2)
    costj = ((ejj[:, 0] * dr[:, 0] + ejj[:, 1] * dr[:, 1]) + ejj[:, 2] * dr[:, 2]) * invdr
    qQinv4dr3 = qQ025 * invdr * invdr2
    u = qQinv4dr3 * (3.0 * costj * costj - 1)
    pR = -3.0 * u * invdr2
    pT = 6.0 * costj * qQinv4dr3 * invdr
    fac = costj * pT * invdr - pR
    f = fac[:, None] * dr - pT[:, None] * ejj
    mx = np.stack([ejj[:, 2] * dr[:, 1] - ejj[:, 1] * dr[:, 2], ejj[:, 0] * dr[:, 2] - ejj[:, 2] * dr[:, 0],
                   ejj[:, 1] * dr[:, 0] - ejj[:, 0] * dr[:, 1]], axis=1)
    return f, pT[:, None] * mx, u


def charge_dipole(dr, dr2, ejj, minusqmy):
    """PotForceChargeDipole (potforce.h:284-311): f, m2 (torque on the dipole), u."""
    invdr2 = 1.0 / dr2
    invdr = np.sqrt(invdr2)
    costj = ((ejj[:, 0] * dr[:, 0] + ejj[:, 1] * dr[:, 1]) + ejj[:, 2] * dr[:, 2]) * invdr
    uInvcostj = minusqmy * invdr2
    u = uInvcostj * costj
    pT = uInvcostj * invdr
    fac = 3.0 * u * invdr * invdr2
    f = fac[:, None] * dr - pT[:, None] * ejj
    mx = np.stack([ejj[:, 2] * dr[:, 1] - ejj[:, 1] * dr[:, 2], ejj[:, 0] * dr[:, 2] - ejj[:, 2] * dr[:, 0],
                   ejj[:, 1] * dr[:, 0] - ejj[:, 0] * dr[:, 1]], axis=1)
    return f, pT[:, None] * mx, u


def _angles(dr, eii, ejj, invdr1):
    costi = ((eii[:, 0] * dr[:, 0] + eii[:, 1] * dr[:, 1]) + eii[:, 2] * dr[:, 2]) * invdr1
    costj = ((ejj[:, 0] * dr[:, 0] + ejj[:, 1] * dr[:, 1]) + ejj[:, 2] * dr[:, 2]) * invdr1
    cosgij = (eii[:, 0] * ejj[:, 0] + eii[:, 1] * ejj[:, 1]) + eii[:, 2] * ejj[:, 2]
    return costi, costj, cosgij


def two_dipole(dr, dr2, eii, ejj, my2, rffac):
    """PotForce2Dipole (potforce.h:66-113): f, m1, m2, u and the MyRF increment."""
    invdr2 = 1. / dr2
    invdr1 = np.sqrt(invdr2)
    myfac = my2 * invdr2 * invdr1
    costi, costj, cosgij = _angles(dr, eii, ejj, invdr1)
    u = myfac * (cosgij - 3. * costi * costj)
    rf = -rffac * cosgij
    pR = -3. * u * invdr2
    pTi = -myfac * 3. * costj * invdr1
    pTj = -myfac * 3. * costi * invdr1
    pG = myfac
    fac = -pR + (costi * pTi + costj * pTj) * invdr1
    f = fac[:, None] * dr - pTi[:, None] * eii - pTj[:, None] * ejj
    eiXej = _cross(eii, ejj)
    m1 = -pTi[:, None] * _cross(eii, dr) + (-pG + rffac)[:, None] * eiXej
    m2 = -pTj[:, None] * _cross(ejj, dr) + (pG - rffac)[:, None] * eiXej
    return f, m1, m2, u, rf


def two_quadrupole(dr, dr2, eii, ejj, q2075):
    """PotForce2Quadrupole (potforce.h:127-172): f, m1, m2, u."""
    invdr2 = 1. / dr2
    invdr1 = np.sqrt(invdr2)
    qfac = q2075 * invdr2 * invdr2 * invdr1
    costi, costj, cosgij = _angles(dr, eii, ejj, invdr1)
    c2i, c2j = costi * costi, costj * costj
    term = cosgij - 5. * costi * costj
    u = qfac * (1. - 5. * (c2i + c2j) - 15. * c2i * c2j + 2. * term * term)
    pR = -5. * u * invdr2
    pTi = -qfac * 10. * (costi + 3. * costi * c2j + 2. * costj * term) * invdr1
    pTj = -qfac * 10. * (costj + 3. * c2i * costj + 2. * costi * term) * invdr1
    pG = qfac * 4. * term
    fac = -pR + (costi * pTi + costj * pTj) * invdr1
    f = fac[:, None] * dr - pTi[:, None] * eii - pTj[:, None] * ejj
    eiXej = _cross(eii, ejj)
    m1 = -pTi[:, None] * _cross(eii, dr) - pG[:, None] * eiXej
    m2 = -pTj[:, None] * _cross(ejj, dr) + pG[:, None] * eiXej
    return f, m1, m2, u


def di_quadrupole(dr, dr2, eii, ejj, myq15):
    """PotForceDiQuadrupole (potforce.h:186-229), dipole eii, quadrupole ejj: f, m1, m2, u."""
    invdr2 = 1. / dr2
    invdr1 = np.sqrt(invdr2)
    myqfac = myq15 * invdr2 * invdr2
    costi, costj, cosgij = _angles(dr, eii, ejj, invdr1)
    c2j = costj * costj
    u = myqfac * (-costi * (5. * c2j - 1.) + 2. * cosgij * costj)
    pR = -4. * u * invdr2
    pTi = myqfac * (-5. * c2j + 1.) * invdr1
    pTj = myqfac * 2. * (-5. * costi * costj + cosgij) * invdr1
    pG = myqfac * 2. * costj
    fac = -pR + (costi * pTi + costj * pTj) * invdr1
    f = fac[:, None] * dr - pTi[:, None] * eii - pTj[:, None] * ejj
    eiXej = _cross(eii, ejj)
    m1 = -pTi[:, None] * _cross(eii, dr) - pG[:, None] * eiXej
    m2 = -pTj[:, None] * _cross(ejj, dr) + pG[:, None] * eiXej
    return f, m1, m2, u


def forces(model: Model, r: np.ndarray, cid: np.ndarray, q: np.ndarray, both_sided: bool = False) -> Dict:
    """F, M per molecule, Upot (Upot6LJ/6 + UpotXpoles + MyRF), virial and the number of molecule
    pairs within rc. Each unordered pair once, as the reference; with both_sided every molecule i
    takes PotForce(mi = i, mj = j) with every other j and keeps only its own share (the device
    path's order of work), the scalars halved."""
    n = r.shape[0]
    L = model.L
    d, oe = site_offsets(model, cid, q, orient=True)
    F = np.zeros((n, 3))
    M = np.zeros((n, 3))
    U6 = 0.0
    UX = 0.0
    RF = 0.0
    W = 0.0
    npairs = 0
    rc2, rclj2 = model.rc * model.rc, model.rclj * model.rclj
    Fs, Ms = (np.zeros((n, 3)), np.zeros((n, 3))) if both_sided else (F, M)   # partners' shares
    for i in range(n if both_sided else n - 1):
        j = np.delete(np.arange(n), i) if both_sided else np.arange(i + 1, n)
        drm = r[i][None, :] - r[j]
        drm -= L[None, :] * np.round(drm / L[None, :])
        dd = np.einsum("ij,ij->i", drm, drm)
        near = dd < rc2
        j, drm, dd = j[near], drm[near], dd[near]
        npairs += int(j.shape[0])
        ci = int(cid[i])
        # the point-polarity blocks of PotForce (potforce.h:365-542), mi = i, mj = j, every pair within rc
        for cj in range(model.nc):
            sel = cid[j] == cj
            if not sel.any():
                continue
            jj, dm = j[sel], drm[sel]
            UX, W, RF = _polar_blocks(model, ci, cj, i, jj, dm, d, oe, F, M, UX, W, RF, Fs, Ms)
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
                    np.subtract.at(Fs, jj, f)
                    M[i] += np.cross(di[None, :], f).sum(axis=0)
                    np.subtract.at(Ms, jj, np.cross(dj, f))
                    U6 += float(u.sum())
                    W += float(np.einsum("ij,ij->", dm, f))
    h = 0.5 if both_sided else 1.0
    # ParticlePairs2PotForceAdapter::finish: Upot6LJ/6 + UpotXpoles + MyRF, Virial + 3 MyRF
    return dict(F=F, M=M, upot=h * (U6 / 6.0 + UX + RF), virial=h * (W + 3.0 * RF), npairs=int(h * npairs))


def _polar_blocks(model, ci, cj, i, jj, dm, d, oe, F, M, UX, W, RF, Fs=None, Ms=None):
    """Charge, dipole and quadrupole pairs of molecule i (mi) with the molecules jj (mj) of component
    cj, drm = dm (from j to i), in PotForce's order (potforce.h:372-542): site forces (+f on the
    SiteSiteDistance side), the direct torques (Madd), UpotXpoles, Virial and MyRF."""
    nq_i, nq_j = len(model.charges[ci]), len(model.charges[cj])
    nd_i, nd_j = len(model.dipoles[ci]), len(model.dipoles[cj])
    nQ_i, nQ_j = len(model.quads[ci]), len(model.quads[cj])
    ch_i = lambda a: model.nlj[ci] + a  # noqa: E731
    ch_j = lambda b: model.nlj[cj] + b  # noqa: E731
    dp_i = lambda a: model.first_dip[ci] + a  # noqa: E731
    dp_j = lambda b: model.first_dip[cj] + b  # noqa: E731
    qd_i = lambda a: model.first_quad[ci] + a  # noqa: E731
    qd_j = lambda b: model.first_quad[cj] + b  # noqa: E731
    Wacc = [W]
    Fs = F if Fs is None else Fs
    Ms = M if Ms is None else Ms

    def apply(si, sj, f, sign, m_i=None, m_j=None):
        # sign +1: mi gets +f, mj gets -f; sign -1 the other way round (minusSiteSiteDistance blocks)
        di, dj = d[si][i], d[sj][jj]
        fi = sign * f
        F[i] += fi.sum(axis=0)
        np.subtract.at(Fs, jj, fi)
        M[i] += np.cross(di[None, :], fi).sum(axis=0)
        np.subtract.at(Ms, jj, np.cross(dj, fi))
        if m_i is not None:
            M[i] += m_i.sum(axis=0)
        if m_j is not None:
            np.add.at(Ms, jj, m_j)
        Wacc[0] += sign * float(np.einsum("ij,ij->", dm, f))

    def plus(si, sj):
        drs = dm + d[si][i][None, :] - d[sj][jj]
        return drs, np.einsum("ij,ij->i", drs, drs)

    def minus(si, sj):
        drs = d[sj][jj] - dm - d[si][i][None, :]
        return drs, np.einsum("ij,ij->i", drs, drs)

    for a in range(nq_i):
        qa = model.charges[ci][a].q
        for b in range(nq_j):
            drs, dr2 = plus(ch_i(a), ch_j(b))
            invdr2 = 1.0 / dr2
            u = (qa * model.charges[cj][b].q) * np.sqrt(invdr2)
            apply(ch_i(a), ch_j(b), (u * invdr2)[:, None] * drs, 1.0)
            UX += float(u.sum())
        for b in range(nQ_j):
            drs, dr2 = plus(ch_i(a), qd_j(b))
            f, m2, u = charge_quadrupole(drs, dr2, oe[qd_j(b)][jj], 0.25 * qa * model.quads[cj][b].abs_q)
            apply(ch_i(a), qd_j(b), f, 1.0, m_j=m2)
            UX += float(u.sum())
        for b in range(nd_j):
            drs, dr2 = plus(ch_i(a), dp_j(b))
            f, m2, u = charge_dipole(drs, dr2, oe[dp_j(b)][jj], -qa * model.dipoles[cj][b].abs_my)
            apply(ch_i(a), dp_j(b), f, 1.0, m_j=m2)
            UX += float(u.sum())
    for a in range(nQ_i):
        Qa = model.quads[ci][a].abs_q
        ei = np.repeat(oe[qd_i(a)][i][None, :], jj.shape[0], axis=0)
        for b in range(nq_j):
            drs, dr2 = minus(qd_i(a), ch_j(b))
            f, m1, u = charge_quadrupole(drs, dr2, ei, 0.25 * model.charges[cj][b].q * Qa)
            apply(qd_i(a), ch_j(b), f, -1.0, m_i=m1)
            UX += float(u.sum())
        for b in range(nQ_j):
            drs, dr2 = plus(qd_i(a), qd_j(b))
            f, m1, m2, u = two_quadrupole(drs, dr2, ei, oe[qd_j(b)][jj], .75 * Qa * model.quads[cj][b].abs_q)
            apply(qd_i(a), qd_j(b), f, 1.0, m_i=m1, m_j=m2)
            UX += float(u.sum())
        for b in range(nd_j):
            drs, dr2 = minus(qd_i(a), dp_j(b))
            f, m_dip, m_quad, u = di_quadrupole(drs, dr2, oe[dp_j(b)][jj], ei, 1.5 * Qa * model.dipoles[cj][b].abs_my)
            apply(qd_i(a), dp_j(b), f, -1.0, m_i=m_quad, m_j=m_dip)
            UX += float(u.sum())
    for a in range(nd_i):
        mya = model.dipoles[ci][a].abs_my
        ei = np.repeat(oe[dp_i(a)][i][None, :], jj.shape[0], axis=0)
        for b in range(nq_j):
            drs, dr2 = minus(dp_i(a), ch_j(b))
            f, m1, u = charge_dipole(drs, dr2, ei, -model.charges[cj][b].q * mya)
            apply(dp_i(a), ch_j(b), f, -1.0, m_i=m1)
            UX += float(u.sum())
        for b in range(nQ_j):
            drs, dr2 = plus(dp_i(a), qd_j(b))
            f, m1, m2, u = di_quadrupole(drs, dr2, ei, oe[qd_j(b)][jj], 1.5 * mya * model.quads[cj][b].abs_q)
            apply(dp_i(a), qd_j(b), f, 1.0, m_i=m1, m_j=m2)
            UX += float(u.sum())
        for b in range(nd_j):
            drs, dr2 = plus(dp_i(a), dp_j(b))
            my2 = mya * model.dipoles[cj][b].abs_my
            f, m1, m2, u, rf = two_dipole(drs, dr2, ei, oe[dp_j(b)][jj], my2, my2 * model.eps_rf_inv_rc3)
            apply(dp_i(a), dp_j(b), f, 1.0, m_i=m1, m_j=m2)
            UX += float(u.sum())
            RF += float(rf.sum())
    return UX, Wacc[0], RF


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
