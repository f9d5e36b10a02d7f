"""Seeded synthetic LJ systems and MarDyn's old-style phase-space format.

The workloads are the single-site Lennard-Jones systems the benchmark and the parity tests run
(FCC lattices with Maxwell-Boltzmann velocities drawn from ``numpy.random.default_rng(seed)``, zero
net momentum, rescaled to the exact target temperature), and fluids of rigid multi-centre LJ
molecules (the same lattices with seeded random orientations and angular momenta). No public
dataset is involved.

``write_inp``/``read_inp`` implement the subset of MarDyn's old-style phase-space format used by
LJ components: the header of ``InputOldstyle::readPhaseSpaceHeader``
(mardyn/io/InputOldstyle.cpp:35-261: ``Length``, ``Temperature``, ``NumberOfComponents`` with the LJ
centre lines ``x y z m eps sigma tcutoff do_shift`` of each component (:162-166), the inertia line
(:188-195), the mixing coefficients ``xi eta`` for i<j (:206-215) and epsilon_RF) and the molecule
section of ``InputOldstyle::readPhaseSpace`` (:263-392) in the ``ICRV`` or ``ICRVQD`` layouts.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Optional, Sequence

import numpy as np


@dataclasses.dataclass
class Site:
    """One LJ centre of a rigid molecule at (x, y, z) in the molecule's principal-axes frame (the
    origin is the centre of mass, Component::addLJcenter, mardyn/molecules/Component.cpp:44-72)."""

    x: float
    y: float
    z: float
    mass: float
    eps: float
    sigma: float
    do_shift: bool = False


@dataclasses.dataclass
class Charge:
    """A point charge of a rigid molecule at (x, y, z) in the principal-axes frame, with its mass
    (Component::addCharge, mardyn/molecules/Component.cpp:115-133)."""

    x: float
    y: float
    z: float
    mass: float
    q: float


@dataclasses.dataclass
class Dipole:
    """A massless point dipole at (x, y, z) with orientation e (body frame) and strength abs_my
    (Component::addDipole, mardyn/molecules/Component.cpp:135-139; e is used as given)."""

    x: float
    y: float
    z: float
    ex: float
    ey: float
    ez: float
    abs_my: float


@dataclasses.dataclass
class Quadrupole:
    """A massless linear point quadrupole at (x, y, z) with axis e and strength abs_q
    (Component::addQuadrupole, Component.cpp:141-145)."""

    x: float
    y: float
    z: float
    ex: float
    ey: float
    ez: float
    abs_q: float


@dataclasses.dataclass
class Component:
    """One LJ component: a single LJ centre at the molecule origin (eps, sigma, mass, do_shift) or,
    with ``sites`` (and ``charges``, ``dipoles``, ``quadrupoles``), a rigid molecule of several LJ
    centres and point polarities (``rigid_component``)."""

    eps: float = 1.0
    sigma: float = 1.0
    mass: float = 1.0
    do_shift: bool = False
    sites: Optional[List[Site]] = None
    inertia: Optional[Sequence[float]] = None   # the header's inertia line; values > 0 replace the moments
    charges: Optional[List[Charge]] = None
    dipoles: Optional[List[Dipole]] = None
    quadrupoles: Optional[List[Quadrupole]] = None

    def lj_centres(self) -> List[Site]:
        if self.sites is not None:
            return list(self.sites)
        return [Site(0.0, 0.0, 0.0, self.mass, self.eps, self.sigma, self.do_shift)]

    def point_charges(self) -> List[Charge]:
        return list(self.charges) if self.charges else []

    def point_dipoles(self) -> List[Dipole]:
        return list(self.dipoles) if self.dipoles else []

    def point_quadrupoles(self) -> List[Quadrupole]:
        return list(self.quadrupoles) if self.quadrupoles else []

    def moments(self) -> np.ndarray:
        """Principal moments I11, I22, I33: sum m (y^2+z^2), sum m (x^2+z^2), sum m (x^2+y^2) over the
        centres and charges, each replaced by the header's value where that is > 0
        (InputOldstyle.cpp:188-195)."""
        I = np.zeros(3)
        for c in list(self.lj_centres()) + self.point_charges():
            I[0] += c.mass * (c.y * c.y + c.z * c.z)
            I[1] += c.mass * (c.x * c.x + c.z * c.z)
            I[2] += c.mass * (c.x * c.x + c.y * c.y)
        if self.inertia is not None:
            for d in range(3):
                if self.inertia[d] > 0.0:
                    I[d] = float(self.inertia[d])
        return I

    @property
    def is_rigid(self) -> bool:
        return self.sites is not None


def rigid_component(sites: Sequence[Site], inertia: Optional[Sequence[float]] = None,
                    charges: Optional[Sequence[Charge]] = None, dipoles: Optional[Sequence[Dipole]] = None,
                    quadrupoles: Optional[Sequence[Quadrupole]] = None) -> Component:
    """A rigid multi-centre component; its mass is the sum of the centres' and charges' masses
    (dipoles and quadrupoles are massless)."""
    sites = list(sites)
    charges = list(charges) if charges else None
    mass = float(sum(c.mass for c in sites) + sum(c.mass for c in (charges or [])))
    return Component(sites[0].eps, sites[0].sigma, mass, sites[0].do_shift,
                     sites=sites, inertia=None if inertia is None else list(inertia), charges=charges,
                     dipoles=list(dipoles) if dipoles else None, quadrupoles=list(quadrupoles) if quadrupoles else None)


def dipolar_two_centre(my: float = 1.0, elongation: float = 0.5) -> Component:
    """A two-centre LJ molecule with a point dipole of strength my at the centre of mass along the
    molecule axis (2CLJD)."""
    base = two_centre(elongation)
    return rigid_component(base.sites, dipoles=[Dipole(0.0, 0.0, 0.0, 0.0, 0.0, 1.0, my)])


def quadrupolar_two_centre(Q: float = 1.0, elongation: float = 0.5) -> Component:
    """A two-centre LJ molecule with a linear point quadrupole of strength Q at the centre of mass
    along the molecule axis (2CLJQ)."""
    base = two_centre(elongation)
    return rigid_component(base.sites, quadrupoles=[Quadrupole(0.0, 0.0, 0.0, 0.0, 0.0, 1.0, Q)])


def charged_two_centre(q: float = 0.5, elongation: float = 0.5, charge_offset: float = 0.35) -> Component:
    """A two-centre LJ molecule (as ``two_centre``) with two massless point charges +q and -q at
    z = +-charge_offset: a neutral molecule with a dipole of 2 q charge_offset."""
    base = two_centre(elongation)
    return rigid_component(base.sites, charges=[Charge(0.0, 0.0, charge_offset, 0.0, q),
                                                Charge(0.0, 0.0, -charge_offset, 0.0, -q)])


def two_centre(elongation: float = 0.5, eps: float = 1.0, sigma: float = 1.0, mass: float = 1.0,
               do_shift: bool = True) -> Component:
    """A two-centre LJ molecule (2CLJ): equal centres at z = +-elongation/2, half the mass each."""
    h = 0.5 * elongation
    return rigid_component([Site(0.0, 0.0, -h, 0.5 * mass, eps, sigma, do_shift),
                            Site(0.0, 0.0, h, 0.5 * mass, eps, sigma, do_shift)])


def three_centre_linear() -> Component:
    """A linear three-centre molecule with a different middle centre (CO2-like proportions in LJ
    units): middle (eps 0.6, sigma 0.9, m 0.4) at the origin, ends (eps 1.0, sigma 1.05, m 0.3) at
    z = +-0.6; truncated-shifted."""
    return rigid_component([Site(0.0, 0.0, 0.0, 0.4, 0.6, 0.9, True),
                            Site(0.0, 0.0, -0.6, 0.3, 1.0, 1.05, True),
                            Site(0.0, 0.0, 0.6, 0.3, 1.0, 1.05, True)])


def bent_three_centre() -> Component:
    """A bent three-centre molecule with three non-zero principal moments (centre of mass at the
    origin, principal axes along x, y, z), plain truncated LJ."""
    return rigid_component([Site(0.0, 0.0, 0.3, 0.5, 0.9, 1.0, False),
                            Site(0.45, 0.0, -0.3, 0.25, 1.1, 0.95, False),
                            Site(-0.45, 0.0, -0.3, 0.25, 1.1, 0.95, False)])


@dataclasses.dataclass
class System:
    """A periodic box of single-site LJ molecules (all arrays in molecule order)."""

    length: np.ndarray                 # (3,) box edge lengths; the box is [0, L)
    components: List[Component]
    mix: np.ndarray                    # (ncomp*(ncomp-1)/2, 2) xi, eta for i<j
    ids: np.ndarray                    # (N,) uint64 molecule ids
    cid: np.ndarray                    # (N,) int32 0-based component ids
    r: np.ndarray                      # (N, 3) float64 positions
    v: np.ndarray                      # (N, 3) float64 velocities
    temperature: float = 1.0           # target temperature written to the header
    cutoff: float = 2.5                # cutoffRadius (cells and pair search)
    lj_cutoff: float = 2.5             # LJCutoffRadius
    dt: float = 0.002                  # timestepLength
    nve: bool = True
    name: str = "system"
    q: Optional[np.ndarray] = None     # (N, 4) orientation quaternions (w, x, y, z) of rigid molecules
    D: Optional[np.ndarray] = None     # (N, 3) angular momenta (space frame) of rigid molecules
    epsilon_rf: float = 1.0e10         # reaction-field permittivity (the header's epsilon_RF)

    @property
    def n(self) -> int:
        return int(self.ids.shape[0])

    @property
    def is_rigid(self) -> bool:
        return any(c.is_rigid for c in self.components)

    def eps(self) -> np.ndarray:
        return np.array([c.eps for c in self.components], dtype=np.float64)

    def sigma(self) -> np.ndarray:
        return np.array([c.sigma for c in self.components], dtype=np.float64)

    def mass(self) -> np.ndarray:
        return np.array([c.mass for c in self.components], dtype=np.float64)

    def do_shift(self) -> np.ndarray:
        return np.array([1 if c.do_shift else 0 for c in self.components], dtype=np.int32)


# ----------------------------------------------------------------------------- generators

def fcc_sites(ncell: Sequence[int], a: Sequence[float], offset: Sequence[float]) -> np.ndarray:
    """FCC lattice sites of ncell[0] x ncell[1] x ncell[2] cubic unit cells of edge a."""
    basis = np.array([[0.0, 0.0, 0.0], [0.5, 0.5, 0.0], [0.5, 0.0, 0.5], [0.0, 0.5, 0.5]])
    ix, iy, iz = np.meshgrid(np.arange(ncell[0]), np.arange(ncell[1]), np.arange(ncell[2]),
                             indexing="ij")
    cells = np.stack([ix.ravel(), iy.ravel(), iz.ravel()], axis=1).astype(np.float64)
    pts = (cells[:, None, :] + basis[None, :, :]).reshape(-1, 3)
    return pts * np.asarray(a, dtype=np.float64) + np.asarray(offset, dtype=np.float64)


def maxwell_boltzmann(rng: np.random.Generator, mass: np.ndarray, temperature: float) -> np.ndarray:
    """Velocities with zero net momentum, scaled so that sum m v^2 / (3N) equals temperature
    (the reference's temperature with no rotational degrees of freedom, Domain.cpp:244-246)."""
    n = mass.shape[0]
    v = rng.standard_normal((n, 3)) * np.sqrt(temperature / mass)[:, None]
    p = (mass[:, None] * v).sum(axis=0) / mass.sum()
    v -= p[None, :]
    summv2 = float((mass[:, None] * v * v).sum())
    v *= math.sqrt(3.0 * n * temperature / summv2)
    return v


def _wrap(r: np.ndarray, length: np.ndarray) -> np.ndarray:
    r = np.mod(r, length[None, :])
    r[r >= length[None, :]] = 0.0
    return r


def lj_fcc_box(n_cells: int, density: float, temperature: float, seed: int, cutoff: float,
               components: Optional[List[Component]] = None, fractions: Optional[Sequence[float]] = None,
               mix: Optional[np.ndarray] = None, dt: float = 0.002, nve: bool = True,
               n_atoms: Optional[int] = None, name: str = "fcc") -> System:
    """A cubic periodic FCC box of 4*n_cells^3 sites at the given number density.

    If n_atoms is given (fewer than the sites), a seeded random subset of the sites is kept and
    the box edge follows from n_atoms/density. The lattice is offset by a/4 so that no molecule
    sits on a cell face.
    """
    rng = np.random.default_rng(seed)
    nsites = 4 * n_cells ** 3
    n = nsites if n_atoms is None else int(n_atoms)
    if n > nsites:
        raise ValueError("n_atoms exceeds the lattice sites")
    L = (n / density) ** (1.0 / 3.0)
    a = L / n_cells
    r = fcc_sites([n_cells] * 3, [a] * 3, [a / 4.0] * 3)
    if n < nsites:
        keep = np.sort(rng.choice(nsites, size=n, replace=False))
        r = r[keep]
    components = components or [Component(1.0, 1.0, 1.0, False)]
    nc = len(components)
    if nc == 1:
        cid = np.zeros(n, dtype=np.int32)
    else:
        fr = np.asarray(fractions if fractions is not None else [1.0 / nc] * nc, dtype=np.float64)
        counts = np.floor(fr / fr.sum() * n).astype(np.int64)
        counts[0] += n - counts.sum()
        cid = np.repeat(np.arange(nc, dtype=np.int32), counts)
        cid = cid[rng.permutation(n)]
    if mix is None:
        mix = np.ones((nc * (nc - 1) // 2, 2), dtype=np.float64)
    length = np.array([L, L, L], dtype=np.float64)
    mass = np.array([components[c].mass for c in range(nc)])[cid]
    v = maxwell_boltzmann(rng, mass, temperature)
    return System(length=length, components=components, mix=np.asarray(mix, dtype=np.float64),
                  ids=np.arange(1, n + 1, dtype=np.uint64), cid=cid, r=_wrap(r, length), v=v,
                  temperature=temperature, cutoff=cutoff, lj_cutoff=cutoff, dt=dt, nve=nve, name=name)


def two_species() -> List[Component]:
    """Species A/B: sigma_A=1.0, sigma_B=0.9, eps_A=1.0, eps_B=0.8, m=1, truncated-shifted."""
    return [Component(1.0, 1.0, 1.0, True), Component(0.8, 0.9, 1.0, True)]


def config_c1(seed: int = 1) -> System:
    """32,000-atom single-species FCC box, rho=0.8, T=1.0, rc=2.5, dt=0.002, plain truncated LJ."""
    return lj_fcc_box(20, 0.8, 1.0, seed, 2.5, [Component(1.0, 1.0, 1.0, False)], name="c1_32k")


def config_c2(seed: int = 2) -> System:
    """1,048,576-atom single-species FCC box, rho=0.75, T=0.9, rc=3.0, truncated-shifted LJ."""
    return lj_fcc_box(64, 0.75, 0.9, seed, 3.0, [Component(1.0, 1.0, 1.0, True)], name="c2_1m")


def config_c3(seed: int = 3, n_total: int = 4194304) -> System:
    """Two-species slab: Lx=Ly, Lz=3Lx; FCC liquid (rho~0.70) in the middle third and a sparse
    vapour (rho~0.02) elsewhere; A/B 50/50 with Lorentz-Berthelot mixing (xi=eta=1); T=0.85;
    rc=2.5 (sigma_A units)."""
    rng = np.random.default_rng(seed)
    Lx = (n_total / (0.70 + 0.02 * 2.0)) ** (1.0 / 3.0)
    n_cells = int(round((0.70 * Lx ** 3 / 4.0) ** (1.0 / 3.0)))
    a = Lx / n_cells
    liquid = fcc_sites([n_cells] * 3, [a] * 3, [a / 4.0, a / 4.0, Lx + a / 4.0])
    n_vap = n_total - liquid.shape[0]
    # vapour on a simple-cubic grid filling z in [0, Lx) and [2Lx, 3Lx); a seeded subset is kept
    m = int(math.ceil((n_vap / 2.0) ** (1.0 / 3.0))) + 1
    av = Lx / m
    g = (np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1)
         .reshape(-1, 3).astype(np.float64) + 0.5) * av
    sites = np.concatenate([g, g + np.array([0.0, 0.0, 2.0 * Lx])])
    keep = np.sort(rng.choice(sites.shape[0], size=n_vap, replace=False))
    r = np.concatenate([liquid, sites[keep]])
    n = r.shape[0]
    comps = two_species()
    cid = np.repeat(np.arange(2, dtype=np.int32), [n - n // 2, n // 2])[rng.permutation(n)]
    length = np.array([Lx, Lx, 3.0 * Lx])
    mass = np.ones(n)
    v = maxwell_boltzmann(rng, mass, 0.85)
    return System(length=length, components=comps, mix=np.ones((1, 2)), ids=np.arange(1, n + 1, dtype=np.uint64),
                  cid=cid, r=_wrap(r, length), v=v, temperature=0.85, cutoff=2.5, lj_cutoff=2.5,
                  dt=0.002, nve=True, name="c3_slab_4m")


def config_c4(seed: int = 4, n_boxes: int = 512) -> List[System]:
    """Independent cubic boxes: N log-uniform in [256, 8192], rho U[0.6, 0.9], T U[0.7, 1.5],
    rc=2.5, truncated-shifted single-species LJ."""
    rng = np.random.default_rng(seed)
    out = []
    for b in range(n_boxes):
        n = int(round(math.exp(rng.uniform(math.log(256), math.log(8192)))))
        rho = float(rng.uniform(0.6, 0.9))
        T = float(rng.uniform(0.7, 1.5))
        ncell = int(math.ceil((n / 4.0) ** (1.0 / 3.0)))
        out.append(lj_fcc_box(ncell, rho, T, int(rng.integers(1 << 31)), 2.5,
                              [Component(1.0, 1.0, 1.0, True)], n_atoms=n, name=f"c4_box{b}"))
    return out


def rotate_inv(q: np.ndarray, d: np.ndarray) -> np.ndarray:
    """Body frame -> space frame for unit quaternions q (N, 4) = (w, x, y, z) and vectors d (N, 3):
    the matrix of Quaternion::rotateinv (mardyn/molecules/Quaternion.cpp:50-66), used here only to
    draw space-frame angular momenta."""
    w, x, y, z = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    ww, xx, yy, zz = w * w, x * x, y * y, z * z
    xy, zw, xz, yw, yz, xw = x * y, z * w, x * z, y * w, y * z, x * w
    out = np.empty_like(d)
    out[:, 0] = (ww + xx - yy - zz) * d[:, 0] + 2.0 * (xy - zw) * d[:, 1] + 2.0 * (xz + yw) * d[:, 2]
    out[:, 1] = 2.0 * (xy + zw) * d[:, 0] + (ww - xx + yy - zz) * d[:, 1] + 2.0 * (yz - xw) * d[:, 2]
    out[:, 2] = 2.0 * (xz - yw) * d[:, 0] + 2.0 * (yz + xw) * d[:, 1] + (ww - xx - yy + zz) * d[:, 2]
    return out


def rigid_fcc_box(n_cells: int, density: float, temperature: float, seed: int, cutoff: float,
                  components: List[Component], fractions: Optional[Sequence[float]] = None,
                  mix: Optional[np.ndarray] = None, dt: float = 0.002, nve: bool = True,
                  n_atoms: Optional[int] = None, name: str = "rigid") -> System:
    """A fluid start of rigid multi-centre molecules: the molecule centres on the FCC lattice of
    ``lj_fcc_box`` (density counts molecules), seeded uniformly random orientations, and angular
    momenta whose body-frame angular velocities are Maxwell-Boltzmann about every axis with a
    non-zero moment, scaled so that sum I w^2 equals rotDOF * T (the rotational part of the
    reference's temperature, Domain.cpp:244-246)."""
    s = lj_fcc_box(n_cells, density, temperature, seed, cutoff, components, fractions, mix, dt, nve, n_atoms, name)
    rng = np.random.default_rng(seed + 7919)
    n = s.n
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1)[:, None]
    I = np.stack([c.moments() for c in components])[s.cid]
    has = I > 0.0
    w = np.where(has, rng.standard_normal((n, 3)) * np.sqrt(temperature / np.where(has, I, 1.0)), 0.0)
    sum_iw2 = float((I * w * w).sum())
    rot_dof = int(has.sum())
    if sum_iw2 > 0.0:
        w *= math.sqrt(rot_dof * temperature / sum_iw2)
    s.q = q
    s.D = rotate_inv(q, I * w)
    return s


def config_2clj(seed: int = 6, n_cells: int = 40, density: float = 0.3, temperature: float = 2.0,
                cutoff: float = 3.0, charged: bool = False) -> System:
    """A two-centre LJ fluid (elongation 0.5, truncated-shifted, cutoff 3.0 on the molecule centres):
    4 n_cells^3 molecules (256,000 at the default) at molecular density 0.3 and T = 2.0; with
    ``charged`` the molecules carry the point charges +-0.5 of ``charged_two_centre``."""
    comp = charged_two_centre() if charged else two_centre()
    tag = "2cljq" if charged else "2clj"
    return rigid_fcc_box(n_cells, density, temperature, seed, cutoff, [comp], name=f"{tag}_{4 * n_cells ** 3}")


def config_c5(seed: int = 5) -> System:
    """16,384-atom two-species FCC box (A/B 50/50 of the slab species), rho=0.8, T=1.0, rc=2.5."""
    return lj_fcc_box(16, 0.8, 1.0, seed, 2.5, two_species(), [0.5, 0.5], np.ones((1, 2)), name="c5_16k")


# ----------------------------------------------------------------------------- file format

def write_inp(sys_: System, path: str, fmt: Optional[str] = None) -> None:
    """Write the old-style phase-space file (header + molecules, component ids 1-based). The molecule
    layout defaults to ICRVQD for rigid molecules (orientations and angular momenta) and ICRV
    otherwise."""
    if fmt is None:
        fmt = "ICRVQD" if sys_.is_rigid else "ICRV"
    nc = len(sys_.components)
    lines = ["mardyn trunk 20090721", "currentTime 0.0",
             f"Temperature {float(sys_.temperature)!r}",
             "Length {!r} {!r} {!r}".format(*[float(x) for x in sys_.length]),
             f"NumberOfComponents {nc}"]
    for c in sys_.components:
        centres = c.lj_centres()
        charges = c.point_charges()
        dips, quads = c.point_dipoles(), c.point_quadrupoles()
        lines.append(f"{len(centres)} {len(charges)} {len(dips)} {len(quads)} 0")
        for t in centres:
            lines.append(f"{float(t.x)!r} {float(t.y)!r} {float(t.z)!r} {float(t.mass)!r} {float(t.eps)!r} "
                         f"{float(t.sigma)!r} {float(sys_.lj_cutoff)!r} {1 if t.do_shift else 0}")
        for t in charges:
            lines.append(f"{float(t.x)!r} {float(t.y)!r} {float(t.z)!r} {float(t.mass)!r} {float(t.q)!r}")
        for t in dips:
            lines.append(f"{float(t.x)!r} {float(t.y)!r} {float(t.z)!r} {float(t.ex)!r} {float(t.ey)!r} "
                         f"{float(t.ez)!r} {float(t.abs_my)!r}")
        for t in quads:
            lines.append(f"{float(t.x)!r} {float(t.y)!r} {float(t.z)!r} {float(t.ex)!r} {float(t.ey)!r} "
                         f"{float(t.ez)!r} {float(t.abs_q)!r}")
        inertia = [0.0, 0.0, 0.0] if c.inertia is None else [float(x) for x in c.inertia]
        lines.append("{!r} {!r} {!r}".format(*inertia))
    k = 0
    for i in range(nc):
        for j in range(i + 1, nc):
            lines.append(f"{float(sys_.mix[k, 0])!r} {float(sys_.mix[k, 1])!r}")
            k += 1
    lines.append(repr(float(sys_.epsilon_rf)))
    lines.append(f"NumberOfMolecules {sys_.n}")
    lines.append(f"MoleculeFormat {fmt}")
    head = "\n".join(lines) + "\n"
    cols = [sys_.ids.astype(np.float64), (sys_.cid + 1).astype(np.float64), sys_.r[:, 0], sys_.r[:, 1],
            sys_.r[:, 2], sys_.v[:, 0], sys_.v[:, 1], sys_.v[:, 2]]
    with open(path, "w") as f:
        f.write(head)
        if fmt == "ICRV":
            body = np.column_stack(cols)
            np.savetxt(f, body, fmt=["%d", "%d"] + ["%.17g"] * 6)
        elif fmt == "ICRVQD":
            n = sys_.n
            q = sys_.q if sys_.q is not None else np.tile([1.0, 0.0, 0.0, 0.0], (n, 1))
            D = sys_.D if sys_.D is not None else np.zeros((n, 3))
            body = np.column_stack(cols + [q, D])
            np.savetxt(f, body, fmt=["%d", "%d"] + ["%.17g"] * 13)
        else:
            raise ValueError(f"unsupported molecule format {fmt}")


def read_inp(path: str) -> System:
    """Read an old-style phase-space file with single-site LJ components (ICRV/ICRVQD/IRV)."""
    with open(path) as f:
        text = "\n".join(ln for ln in f.read().splitlines() if not ln.lstrip().startswith("#"))
    toks = text.split()
    pos = 0

    def nxt() -> str:
        nonlocal pos
        t = toks[pos]
        pos += 1
        return t

    magic = nxt()
    if magic not in ("mardyn", "MOLDY", "ls1r1", "mrdyn", "MDProject", "Mardyn", "MARDYN"):
        raise ValueError(f"{path}: not a valid OldStyle input file")
    if nxt() != "trunk":
        raise ValueError(f"{path}: wrong input file specifier")
    nxt()
    temperature, length, comps, mix, epsilon_rf = 1.0, None, [], [], 1.0e10
    while True:
        t = nxt()
        if t in ("currentTime", "t"):
            nxt()
        elif t in ("Temperature", "T"):
            temperature = float(nxt())
        elif t in ("Length", "L"):
            length = np.array([float(nxt()), float(nxt()), float(nxt())])
        elif t in ("NumberOfComponents", "C"):
            nc = int(nxt())
            for _ in range(nc):
                nlj, nq, nd, nqq, nt = (int(nxt()) for _ in range(5))
                if nlj < 1 or nt:
                    raise ValueError("only LJ centres and point polarities are supported")
                centres = []
                for _ in range(nlj):
                    x, y, z, m, eps, sig, tcut, shift = (float(nxt()) for _ in range(8))
                    centres.append(Site(x, y, z, m, eps, sig, shift != 0))
                charges = []
                for _ in range(nq):
                    x, y, z, m, q = (float(nxt()) for _ in range(5))
                    charges.append(Charge(x, y, z, m, q))
                dips = [Dipole(*(float(nxt()) for _ in range(7))) for _ in range(nd)]
                quads = [Quadrupole(*(float(nxt()) for _ in range(7))) for _ in range(nqq)]
                inertia = [float(nxt()) for _ in range(3)]
                if (nlj == 1 and not (nq or nd or nqq) and not (centres[0].x or centres[0].y or centres[0].z)
                        and not any(inertia)):
                    t = centres[0]
                    comps.append(Component(t.eps, t.sigma, t.mass, t.do_shift))
                else:
                    comps.append(rigid_component(centres, inertia if any(inertia) else None, charges or None,
                                                 dips or None, quads or None))
            for i in range(nc):
                for j in range(i + 1, nc):
                    mix.append((float(nxt()), float(nxt())))
            epsilon_rf = float(nxt())
            break
        else:
            raise ValueError(f"unsupported header token {t}")
    t = nxt()
    if t not in ("NumberOfMolecules", "N"):
        raise ValueError("expected NumberOfMolecules")
    n = int(nxt())
    fmt = "ICRVQD"
    if toks[pos] in ("MoleculeFormat", "M"):
        pos += 1
        fmt = nxt()
    ncol = {"ICRVQD": 15, "ICRV": 8, "IRV": 7, "ICRVFQDM": 21}[fmt]
    body = np.array(toks[pos:pos + n * ncol], dtype=np.float64).reshape(n, ncol)
    if fmt == "IRV":
        ids, cid, r, v = body[:, 0], np.ones(n), body[:, 1:4], body[:, 4:7]
    else:
        ids, cid, r, v = body[:, 0], body[:, 1], body[:, 2:5], body[:, 5:8]
    q = D = None
    if fmt == "ICRVQD":
        q, D = body[:, 8:12].copy(), body[:, 12:15].copy()
    elif fmt == "ICRVFQDM":
        q, D = body[:, 11:15].copy(), body[:, 15:18].copy()
    nc = len(comps)
    rigid = any(c.is_rigid for c in comps)
    return System(length=length, components=comps,
                  mix=np.array(mix, dtype=np.float64).reshape(nc * (nc - 1) // 2, 2),
                  ids=ids.astype(np.uint64), cid=(cid.astype(np.int32) - 1), r=r.copy(), v=v.copy(),
                  temperature=temperature, name=path, q=q if rigid else None, D=D if rigid else None,
                  epsilon_rf=epsilon_rf)


def write_cfg(sys_: System, cfg_path: str, inp_name: str) -> None:
    """Old-style MarDyn config for the system (tokens of Simulation::initConfigOldstyle)."""
    lines = ["mardynconfig", f"timestepLength {float(sys_.dt)!r}", f"cutoffRadius {float(sys_.cutoff)!r}",
             f"LJCutoffRadius {float(sys_.lj_cutoff)!r}", f"phaseSpaceFile OldStyle {inp_name}",
             "datastructure LinkedCells 1"]
    if sys_.nve:
        lines.append("NVE")
    with open(cfg_path, "w") as f:
        f.write("\n".join(lines) + "\n")
