"""Python host side of the B200 LJ hot path, over the C ABI of libmdgpu.so (include/mdgpu.h).

The classes mirror the reference's interfaces for this path so that code written against MarDyn's
sequential LJ loop reads the same (paths relative to madpac/mardyn/):

* ``LinkedCells``  -- ParticleContainer/LinkedCells (particleContainer/LinkedCells.h:60-312): ``update``,
  ``traversePairs`` (with the ParticlePairs2PotForceAdapter folded in), ``deleteOuterParticles``,
  ``getNumberOfParticles``, ``getCellIndexOfMolecule``.
* ``Leapfrog``     -- the three-state integrator (integrators/Leapfrog.cpp:14-108):
  ``eventNewTimestep`` / ``eventForcesCalculated``.
* ``Domain``       -- the Upot/virial/temperature/thermostat part of Domain (Domain.cpp:102-376).
* ``Simulation``   -- ``prepare_start`` and ``simulateStep`` in the order of Simulation.cpp:907-1229.

Errors raise ``MdgpuError`` carrying the status code (the reference calls ``exit(code)``).
The compute path is the CUDA library only: if libmdgpu.so cannot be loaded, every constructor
raises; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import math
import os
from typing import Dict, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmdgpu.so")

FP64 = 0
MIXED = 1

STATUS_NAMES = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_STATE", 5: "ERR_BOX_TOO_SMALL",
                6: "ERR_OUTSIDE_HALO", 7: "ERR_SAME_POSITION", 8: "ERR_NONFINITE", 9: "ERR_TIMEOUT",
                10: "ERR_CAPACITY"}

# Every entry point of include/mdgpu.h: name -> (restype, argtypes)
_VP = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
SIGNATURES = {
    "mdgpu_create": (_I, [ctypes.POINTER(_VP), _VP, _D, _D, _D, _I, _VP, _VP, _I, _I]),
    "mdgpu_destroy": (_I, [_VP]),
    "mdgpu_last_error": (ctypes.c_char_p, [_VP]),
    "mdgpu_set_precision": (_I, [_VP, _I]),
    "mdgpu_set_pair_kernel": (_I, [_VP, _I]),
    "mdgpu_set_particles": (_I, [_VP, _I64, _VP, _VP, _VP, _VP, _VP]),
    "mdgpu_set_state": (_I, [_VP, _I64, _VP, _VP]),
    "mdgpu_get_particles": (_I, [_VP, _I64, _VP, _VP, _VP, _VP, _VP]),
    "mdgpu_num_particles": (_I, [_VP, _VP]),
    "mdgpu_get_geometry": (_I, [_VP, _VP, _VP, _VP]),
    "mdgpu_update": (_I, [_VP]),
    "mdgpu_get_cell_index": (_I, [_VP, _I64, _VP]),
    "mdgpu_traverse_pairs": (_I, [_VP, _VP, _VP, _VP]),
    "mdgpu_leapfrog_pre": (_I, [_VP, _D, _D]),
    "mdgpu_leapfrog_post": (_I, [_VP, _D, _VP]),
    "mdgpu_scale_velocities": (_I, [_VP, _D]),
    "mdgpu_far_field_correction": (_I, [_VP, _VP, _VP]),
    "mdgpu_step": (_I, [_VP, _D, _D, _VP]),
    "mdgpu_run": (_I, [_VP, _I32, _D, _VP]),
    "mdgpu_run_async": (_I, [_VP, _I32, _D]),
    "mdgpu_read_steps": (_I, [_VP, _I32, _VP]),
    "mdgpu_device_peaks": (_I, [_I, _VP, _VP]),
    "mdgpu_adjoint": (_I, [_VP, _VP, _D, _VP, _VP, _VP]),
    "mdgpu_traj_forward": (_I, [_VP, _I32, _I32, _D, _VP]),
    "mdgpu_traj_backward": (_I, [_VP, _VP, _D, _VP, _VP, _VP, _VP, _VP]),
    "mdgpu_traj_adjoint_time": (_I, [_VP, _VP, _VP]),
    "mdgpu_reflect_boundary": (_I, [_VP, _I32, _I32, _I32, _I32, _VP]),
    "mdgpu_force_boundary": (_I, [_VP, _I32, _D, _I32, _D]),
    "mdgpu_thermostat_create": (_I, [ctypes.POINTER(_VP), _VP, _VP, _D, _D, _I32, _VP]),
    "mdgpu_thermostat_apply": (_I, [_VP, _I64]),
    "mdgpu_thermostat_destroy": (_I, [_VP]),
    "mdgpu_profile_enable": (_I, [_VP, _I]),
    "mdgpu_profile_read": (_I, [_VP, _VP, _VP, _I]),
    "mdgpu_get_stream": (_I, [_VP, _VP]),
    "mdgpu_synchronize": (_I, [_VP]),
    "mdgpu_forces_noalloc": (_I, [_I, _VP, _I64, _VP, _VP, _VP, _D, _D, _I, _VP, _VP, _I, _VP, _VP, _VP,
                                  ctypes.c_char_p, _I]),
    "mdgpu_set_skin": (_I, [_VP, _D]),
    "mdgpu_write_checkpoint": (_I, [_VP, ctypes.c_char_p, _D, _D, _D, _I]),
    "mdgpu_read_phase_space": (_I, [_VP, ctypes.c_char_p, _VP, _VP]),
    "mdgpu_skin_builds": (_I, [_VP, _VP]),
    "mdgpu_set_list_prune": (_I, [_VP, _D]),
    "mdgpu_list_prunes": (_I, [_VP, _VP]),
    "mdgpu_batch_create": (_I, [ctypes.POINTER(_VP), _I32, _VP, _VP, _D, _D, _D, _I, _VP, _VP, _I, _I]),
    "mdgpu_batch_destroy": (_I, [_VP]),
    "mdgpu_batch_last_error": (ctypes.c_char_p, [_VP]),
    "mdgpu_batch_set_particles": (_I, [_VP, _I64, _VP, _VP, _VP, _VP]),
    "mdgpu_batch_get_particles": (_I, [_VP, _I64, _VP, _VP, _VP, _VP, _VP]),
    "mdgpu_batch_prepare": (_I, [_VP, _VP]),
    "mdgpu_batch_run": (_I, [_VP, _I32, _D, _VP]),
    "mdgpu_batch_set_tiles": (_I, [_VP, _I32, _I32, _I32]),
    "mdgpu_batch_get_tiles": (_I, [_VP, _VP]),
    "mdgpu_batch_autotune": (_I, [_VP, _D, _I32, _VP, _VP]),
    "mdgpu_batch_last_run_ms": (_I, [_VP, _VP]),
    "mdgpu_batch_set_barrier_timeout": (_I, [_VP, _I64]),
    "mdgpu_batch_set_skin": (_I, [_VP, _D]),
    "mdgpu_batch_skin_builds": (_I, [_VP, _VP]),
    "mdgpu_rigid_create": (_I, [ctypes.POINTER(_VP), _VP, _D, _D, _D, _I, _VP, _VP, _VP, _VP, _VP, _VP, _I, _I]),
    "mdgpu_rigid_destroy": (_I, [_VP]),
    "mdgpu_rigid_set_polarities": (_I, [_VP, _VP, _VP, _VP, _VP, _D]),
    "mdgpu_rigid_far_field_correction": (_I, [_I, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _D, _D, _D, _VP, _VP,
                                              ctypes.c_char_p, _I]),
    "mdgpu_rigid_last_error": (ctypes.c_char_p, [_VP]),
    "mdgpu_rigid_set_precision": (_I, [_VP, _I]),
    "mdgpu_rigid_get_inertia": (_I, [_VP, _I32, _VP, _VP]),
    "mdgpu_rigid_set_particles": (_I, [_VP, _I64, _VP, _VP, _VP, _VP, _VP, _VP]),
    "mdgpu_rigid_get_particles": (_I, [_VP, _I64, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _VP]),
    "mdgpu_rigid_update": (_I, [_VP]),
    "mdgpu_rigid_traverse_pairs": (_I, [_VP, _VP, _VP, _VP]),
    "mdgpu_rigid_leapfrog_pre": (_I, [_VP, _D, _D, _D]),
    "mdgpu_rigid_leapfrog_post": (_I, [_VP, _D, _VP, _VP]),
    "mdgpu_rigid_run": (_I, [_VP, _I32, _D, _VP]),
    "mdgpu_rigid_set_skin": (_I, [_VP, _D, _I32]),
    "mdgpu_rigid_skin_builds": (_I, [_VP, _VP]),
    "mdgpu_rigid_get_stream": (_I, [_VP, _VP]),
    "mdgpu_rigid_profile_enable": (_I, [_VP, _I]),
    "mdgpu_rigid_profile_read": (_I, [_VP, _VP, _VP, _I]),
}

_lib = None


class MdgpuError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"mdgpu status {code} ({STATUS_NAMES.get(code, '?')}): {message}")
        self.code = code


class _MdComponent(ctypes.Structure):
    _fields_ = [("eps", ctypes.c_double), ("sigma", ctypes.c_double), ("mass", ctypes.c_double),
                ("do_shift", ctypes.c_int)]


class _MdSite(ctypes.Structure):
    _fields_ = [("r", ctypes.c_double * 3), ("mass", ctypes.c_double), ("eps", ctypes.c_double),
                ("sigma", ctypes.c_double), ("do_shift", ctypes.c_int)]


class _MdCharge(ctypes.Structure):
    _fields_ = [("r", ctypes.c_double * 3), ("mass", ctypes.c_double), ("q", ctypes.c_double)]


class _MdOriented(ctypes.Structure):
    _fields_ = [("r", ctypes.c_double * 3), ("e", ctypes.c_double * 3), ("strength", ctypes.c_double)]


def _site_tables(components):
    """ctypes arrays of the components' LJ centres and charges: (nsites, sites, ncharges, charges)."""
    centres = [c.lj_centres() for c in components]
    nsites = np.array([len(cs) for cs in centres], dtype=np.int32)
    sites = (_MdSite * int(nsites.sum()))()
    k = 0
    for cs in centres:
        for t in cs:
            sites[k].r[0], sites[k].r[1], sites[k].r[2] = float(t.x), float(t.y), float(t.z)
            sites[k].mass, sites[k].eps, sites[k].sigma = float(t.mass), float(t.eps), float(t.sigma)
            sites[k].do_shift = 1 if t.do_shift else 0
            k += 1
    qs = [c.point_charges() if hasattr(c, "point_charges") else [] for c in components]
    ncharges = np.array([len(x) for x in qs], dtype=np.int32)
    charges = (_MdCharge * max(1, int(ncharges.sum())))()
    k = 0
    for x in qs:
        for t in x:
            charges[k].r[0], charges[k].r[1], charges[k].r[2] = float(t.x), float(t.y), float(t.z)
            charges[k].mass, charges[k].q = float(t.mass), float(t.q)
            k += 1
    return nsites, sites, ncharges, charges


def rigid_far_field_correction(system):
    """Domain::initFarFieldCorr (Domain.cpp:574-677) for the system's rigid components and molecule
    counts: (UpotCorr, VirialCorr). Host arithmetic in libmdgpu.so; no device needed."""
    lib = load_library()
    comps = system.components
    nsites, sites, ncharges, charges = _site_tables(comps)
    nd, da = _oriented([c.point_dipoles() if hasattr(c, "point_dipoles") else [] for c in comps], "abs_my")
    counts = np.bincount(np.asarray(system.cid, dtype=np.int64), minlength=len(comps)).astype(np.int64)
    length = _c64(system.length)
    mix = _c64(system.mix).reshape(-1)
    u, w = ctypes.c_double(), ctypes.c_double()
    err = ctypes.create_string_buffer(256)
    st = lib.mdgpu_rigid_far_field_correction(len(comps), _ptr(nsites), ctypes.cast(sites, ctypes.c_void_p),
                                              _ptr(ncharges), ctypes.cast(charges, ctypes.c_void_p), _ptr(nd),
                                              ctypes.cast(da, ctypes.c_void_p), _ptr(mix) if mix.size else None,
                                              _ptr(counts), _ptr(length), float(system.cutoff),
                                              float(system.lj_cutoff), float(getattr(system, "epsilon_rf", 1.0e10)),
                                              ctypes.byref(u), ctypes.byref(w), err, 256)
    if st != 0:
        raise MdgpuError(st, "far-field correction: " + err.value.decode())
    return u.value, w.value


def _oriented(lists, strength_attr):
    counts = np.array([len(x) for x in lists], dtype=np.int32)
    arr = (_MdOriented * max(1, int(counts.sum())))()
    k = 0
    for x in lists:
        for t in x:
            arr[k].r[0], arr[k].r[1], arr[k].r[2] = float(t.x), float(t.y), float(t.z)
            arr[k].e[0], arr[k].e[1], arr[k].e[2] = float(t.ex), float(t.ey), float(t.ez)
            arr[k].strength = float(getattr(t, strength_attr))
            k += 1
    return counts, arr


def load_library(path: str = LIB_PATH):
    """Load libmdgpu.so (built by madpac_b200.build) and declare every entry point."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise OSError(f"{path} is missing: build it with `python -m madpac_b200.build`")
        lib = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c64(a, dtype=np.float64, shape=None) -> np.ndarray:
    out = np.ascontiguousarray(a, dtype=dtype)
    if shape is not None:
        out = out.reshape(shape)
    return out


def device_peaks(device: int = 0):
    """(FP32, FP64) peak FMA throughput of the device in TFLOP/s, measured by a short kernel."""
    lib = load_library()
    a, b = ctypes.c_double(), ctypes.c_double()
    st = lib.mdgpu_device_peaks(int(device), ctypes.byref(a), ctypes.byref(b))
    if st != 0:
        raise MdgpuError(st, "device peak measurement failed")
    return a.value, b.value


def forces_noalloc(d_r: int, d_cid: int, d_F: int, n: int, length, cutoff: float, components, mixcoeff=None,
                   LJCutoffRadius: float = 0.0, precision: int = FP64, device: int = 0, stream: int = 0):
    """Forces, local Upot and virial of one box with no device allocation inside the call.

    For callers that cannot allocate device memory while they run (a host owning all memory
    through its own pool, a latency-bound loop): d_r, d_cid and d_F are device addresses of
    buffers the caller owns ((n, 3) float64, (n,) int32, (n, 3) float64). At most 32768 molecules
    and 32768 cells (the size of the library's static scratch array). The call is synchronous (it
    waits for `stream`) and leaves the current device as it found it. Returns (upot, virial).
    """
    lib = load_library()
    comps = (_MdComponent * len(components))()
    for k, c in enumerate(components):
        comps[k].eps, comps[k].sigma, comps[k].mass = float(c.eps), float(c.sigma), float(c.mass)
        comps[k].do_shift = 1 if c.do_shift else 0
    length = _c64(length)
    mix = None if mixcoeff is None else _c64(mixcoeff).reshape(-1)
    if mix is not None and mix.size == 0:
        mix = None
    u, w = ctypes.c_double(), ctypes.c_double()
    err = ctypes.create_string_buffer(256)
    st = lib.mdgpu_forces_noalloc(int(device), stream or None, int(n), d_r, d_cid, _ptr(length), float(cutoff),
                                  float(LJCutoffRadius), len(components), ctypes.cast(comps, ctypes.c_void_p),
                                  _ptr(mix), int(precision), d_F, ctypes.byref(u), ctypes.byref(w), err, 256)
    if st != 0:
        raise MdgpuError(st, err.value.decode())
    return u.value, w.value


def _components(components):
    comps = (_MdComponent * len(components))()
    for k, c in enumerate(components):
        comps[k].eps, comps[k].sigma, comps[k].mass = float(c.eps), float(c.sigma), float(c.mass)
        comps[k].do_shift = 1 if c.do_shift else 0
    return comps


class Batch:
    """An ensemble of independent periodic boxes (no reference counterpart: the reference runs one
    Simulation per box). All boxes share cutoffs, components and precision; every step of every box
    is one persistent kernel launch, replayed from a captured CUDA graph. Molecule arrays are
    box-major (box 0's molecules, then box 1's, ...)."""

    TILE_CANDIDATES = [(cap, ctas, dyn) for cap in (32, 64) for ctas in (1, 2) for dyn in (0, 1)]

    def __init__(self, lengths, counts, cutoffRadius: float, components, mixcoeff=None,
                 LJCutoffRadius: float = 0.0, precision: int = FP64, device: int = 0):
        self.lib = load_library()
        self._lengths = _c64(lengths).reshape(-1, 3)
        self.counts = _c64(counts, np.int64).reshape(-1)
        if self._lengths.shape[0] != self.counts.shape[0]:
            raise ValueError("one length triple per box")
        self.nboxes = int(self.counts.shape[0])
        self.ntotal = int(self.counts.sum())
        self.offsets = np.concatenate([[0], np.cumsum(self.counts)]).astype(np.int64)
        comps = _components(components)
        mix = None if mixcoeff is None else _c64(mixcoeff).reshape(-1)
        if mix is not None and mix.size == 0:
            mix = None
        h = ctypes.c_void_p()
        st = self.lib.mdgpu_batch_create(ctypes.byref(h), self.nboxes, _ptr(self._lengths), _ptr(self.counts),
                                         float(cutoffRadius), float(LJCutoffRadius), 1.0, len(components),
                                         ctypes.cast(comps, ctypes.c_void_p), _ptr(mix), int(precision), int(device))
        self.h = h.value
        if st != 0:
            msg = self.lib.mdgpu_batch_last_error(self.h).decode() if self.h else ""
            if self.h:
                self.lib.mdgpu_batch_destroy(self.h)
            self.h = None
            raise MdgpuError(st, msg)

    @classmethod
    def from_systems(cls, systems, precision: int = FP64, device: int = 0) -> "Batch":
        s0 = systems[0]
        b = cls([s.length for s in systems], [s.n for s in systems], s0.cutoff, s0.components, s0.mix, s0.lj_cutoff,
                precision, device)
        b.setParticles(np.concatenate([s.ids for s in systems]), np.concatenate([s.cid for s in systems]),
                       np.concatenate([s.r for s in systems]), np.concatenate([s.v for s in systems]))
        return b

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.mdgpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        if st != 0:
            raise MdgpuError(st, self.lib.mdgpu_batch_last_error(self.h).decode())

    def setParticles(self, ids, cid, r, v) -> None:
        n = self.ntotal
        self._check(self.lib.mdgpu_batch_set_particles(self.h, n, _ptr(_c64(ids, np.uint64)), _ptr(_c64(cid, np.int32)),
                                                       _ptr(_c64(r, shape=(n, 3))), _ptr(_c64(v, shape=(n, 3)))))

    def getParticles(self) -> Dict[str, np.ndarray]:
        n = self.ntotal
        ids = np.zeros(n, dtype=np.uint64)
        cid = np.zeros(n, dtype=np.int32)
        r, v, F = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3))
        self._check(self.lib.mdgpu_batch_get_particles(self.h, n, _ptr(ids), _ptr(cid), _ptr(r), _ptr(v), _ptr(F)))
        return dict(id=ids, cid=cid, r=r, v=v, F=F)

    def box(self, state: Dict[str, np.ndarray], k: int) -> Dict[str, np.ndarray]:
        """The slice of a getParticles() result that belongs to box k."""
        a, b = self.offsets[k], self.offsets[k + 1]
        return {key: val[a:b] for key, val in state.items()}

    def prepare(self) -> np.ndarray:
        """Initial binning and forces of every box; returns (nboxes, 4) {Upot, virial, sum m v^2, pairs}."""
        out = np.zeros((self.nboxes, 4))
        self._check(self.lib.mdgpu_batch_prepare(self.h, _ptr(out)))
        return out

    def run(self, nsteps: int, dt: float, record: bool = True) -> Optional[np.ndarray]:
        """nsteps NVE steps of every box; returns (nsteps, nboxes, 4) step records."""
        out = np.zeros((nsteps, self.nboxes, 4)) if record else None
        self._check(self.lib.mdgpu_batch_run(self.h, int(nsteps), float(dt), _ptr(out)))
        return out

    def setTiles(self, list_cap: int, ctas_per_sm: int, dynamic: int) -> None:
        self._check(self.lib.mdgpu_batch_set_tiles(self.h, int(list_cap), int(ctas_per_sm), int(dynamic)))

    def tiles(self):
        t = np.zeros(3, dtype=np.int32)
        self._check(self.lib.mdgpu_batch_get_tiles(self.h, _ptr(t)))
        return tuple(int(x) for x in t)

    def autotune(self, dt: float, trial_steps: int = 5):
        """Times every tile shape from the current state (restored afterwards) and keeps the fastest.
        Returns (best (list_cap, ctas_per_sm, dynamic), {candidate: ms per step}); a candidate not
        timed reads -1 (staging that does not fit; in the Verlet-skin mode every list depth other
        than the current one, since the depth does not act on skin-mode lists)."""
        best = np.zeros(3, dtype=np.int32)
        ms = np.zeros(len(self.TILE_CANDIDATES))
        self._check(self.lib.mdgpu_batch_autotune(self.h, float(dt), int(trial_steps), _ptr(best), _ptr(ms)))
        return tuple(int(x) for x in best), dict(zip(self.TILE_CANDIDATES, ms.tolist()))

    def lastRunMs(self) -> float:
        ms = ctypes.c_double()
        self._check(self.lib.mdgpu_batch_last_run_ms(self.h, ctypes.byref(ms)))
        return ms.value

    def setBarrierTimeout(self, ns: int) -> None:
        self._check(self.lib.mdgpu_batch_set_barrier_timeout(self.h, int(ns)))

    def setSkin(self, skin: float) -> None:
        """Verlet-skin mode per box (0 = off); takes effect at the next prepare()."""
        self._check(self.lib.mdgpu_batch_set_skin(self.h, float(skin)))

    def skinBuilds(self) -> int:
        b = ctypes.c_int64()
        self._check(self.lib.mdgpu_batch_skin_builds(self.h, ctypes.byref(b)))
        return b.value


class RigidLinkedCells:
    """The GPU container for rigid multi-centre LJ molecules with point charges (include/mdgpu.h, mdgpu_rigid_*): the
    molecule centres binned into cells of edge >= rc as in ``LinkedCells``, every molecule with an
    orientation q, angular momentum D and torque M. Mirrors the same reference sequence:
    ``update`` (LinkedCells::update), ``traversePairs`` (Molecule::upd_cache, traversePairs with
    PotForce's loop over LJ centre pairs, Molecule::calcFM), ``eventNewTimestep`` /
    ``eventForcesCalculated`` (Molecule::upd_preF / upd_postF) and ``run`` (Simulation::simulateStep,
    NVE). ``components`` are ``workloads.Component`` objects (single-centre ones count as one
    centre at the origin)."""

    def __init__(self, length: Sequence[float], cutoffRadius: float, components, mixcoeff=None,
                 LJCutoffRadius: float = 0.0, cellsInCutoffRadius: float = 1.0, precision: int = FP64,
                 device: int = 0, epsilonRF: float = 1.0e10):
        self.lib = load_library()
        centres = [c.lj_centres() for c in components]
        nsites = np.array([len(cs) for cs in centres], dtype=np.int32)
        sites = (_MdSite * int(nsites.sum()))()
        k = 0
        for cs in centres:
            for t in cs:
                sites[k].r[0], sites[k].r[1], sites[k].r[2] = float(t.x), float(t.y), float(t.z)
                sites[k].mass, sites[k].eps, sites[k].sigma = float(t.mass), float(t.eps), float(t.sigma)
                sites[k].do_shift = 1 if t.do_shift else 0
                k += 1
        qs = [c.point_charges() if hasattr(c, "point_charges") else [] for c in components]
        ncharges = np.array([len(x) for x in qs], dtype=np.int32)
        charges = (_MdCharge * max(1, int(ncharges.sum())))()
        k = 0
        for x in qs:
            for t in x:
                charges[k].r[0], charges[k].r[1], charges[k].r[2] = float(t.x), float(t.y), float(t.z)
                charges[k].mass, charges[k].q = float(t.mass), float(t.q)
                k += 1
        inertia = np.zeros((len(components), 3))
        for i, c in enumerate(components):
            if getattr(c, "inertia", None) is not None:
                inertia[i] = c.inertia
        self._length = _c64(length)
        mix = None if mixcoeff is None else _c64(mixcoeff).reshape(-1)
        if mix is not None and mix.size == 0:
            mix = None
        h = ctypes.c_void_p()
        st = self.lib.mdgpu_rigid_create(ctypes.byref(h), _ptr(self._length), float(cutoffRadius),
                                         float(LJCutoffRadius), float(cellsInCutoffRadius), len(components),
                                         _ptr(nsites), ctypes.cast(sites, ctypes.c_void_p), _ptr(ncharges),
                                         ctypes.cast(charges, ctypes.c_void_p), _ptr(inertia), _ptr(mix),
                                         int(precision), int(device))
        self.h = h.value
        if st != 0:
            msg = self.lib.mdgpu_rigid_last_error(self.h).decode() if self.h else ""
            if self.h:
                self.lib.mdgpu_rigid_destroy(self.h)
            self.h = None
            raise MdgpuError(st, msg)
        self.n = 0
        self.components = components
        dips = [c.point_dipoles() if hasattr(c, "point_dipoles") else [] for c in components]
        quads = [c.point_quadrupoles() if hasattr(c, "point_quadrupoles") else [] for c in components]
        if any(dips) or any(quads) or epsilonRF != 1.0e10:
            nd, da = _oriented(dips, "abs_my")
            nqq, qa = _oriented(quads, "abs_q")
            self._check(self.lib.mdgpu_rigid_set_polarities(self.h, _ptr(nd), ctypes.cast(da, ctypes.c_void_p),
                                                            _ptr(nqq), ctypes.cast(qa, ctypes.c_void_p),
                                                            float(epsilonRF)))

    @classmethod
    def from_system(cls, system, precision: int = FP64, device: int = 0) -> "RigidLinkedCells":
        lc = cls(system.length, system.cutoff, system.components, system.mix, system.lj_cutoff, 1.0, precision, device,
                 getattr(system, "epsilon_rf", 1.0e10))
        n = system.n
        q = system.q if system.q is not None else np.tile([1.0, 0.0, 0.0, 0.0], (n, 1))
        D = system.D if system.D is not None else np.zeros((n, 3))
        lc.addParticles(system.ids, system.cid, system.r, system.v, q, D)
        return lc

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.mdgpu_rigid_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        if st != 0:
            raise MdgpuError(st, self.lib.mdgpu_rigid_last_error(self.h).decode())

    def setPrecision(self, precision: int) -> None:
        self._check(self.lib.mdgpu_rigid_set_precision(self.h, int(precision)))

    def inertia(self, comp: int):
        """(mass, (I11, I22, I33)) of component comp."""
        m = ctypes.c_double()
        I = np.zeros(3)
        self._check(self.lib.mdgpu_rigid_get_inertia(self.h, int(comp), ctypes.byref(m), _ptr(I)))
        return m.value, I

    def addParticles(self, ids, cid, r, v, q, D) -> None:
        n = int(np.asarray(ids).shape[0])
        self._check(self.lib.mdgpu_rigid_set_particles(
            self.h, n, _ptr(_c64(ids, np.uint64)), _ptr(_c64(cid, np.int32)), _ptr(_c64(r, shape=(n, 3))),
            _ptr(_c64(v, shape=(n, 3))), _ptr(_c64(q, shape=(n, 4))), _ptr(_c64(D, shape=(n, 3)))))
        self.n = n

    def getParticles(self) -> Dict[str, np.ndarray]:
        n = self.n
        ids = np.zeros(n, dtype=np.uint64)
        cid = np.zeros(n, dtype=np.int32)
        r, v, F, D, M = (np.zeros((n, 3)) for _ in range(5))
        q = np.zeros((n, 4))
        self._check(self.lib.mdgpu_rigid_get_particles(self.h, n, _ptr(ids), _ptr(cid), _ptr(r), _ptr(v), _ptr(F),
                                                       _ptr(q), _ptr(D), _ptr(M)))
        return dict(id=ids, cid=cid, r=r, v=v, F=F, q=q, D=D, M=M)

    def update(self) -> None:
        self._check(self.lib.mdgpu_rigid_update(self.h))

    def traversePairs(self):
        """(Upot, virial, molecule pairs within the cutoff); F and M of every molecule on the device."""
        u, w, p = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.mdgpu_rigid_traverse_pairs(self.h, ctypes.byref(u), ctypes.byref(w), ctypes.byref(p)))
        return u.value, w.value, p.value

    def eventNewTimestep(self, dt: float, vcorr: float = 1.0, Dcorr: float = 1.0) -> None:
        self._check(self.lib.mdgpu_rigid_leapfrog_pre(self.h, float(dt), float(vcorr), float(Dcorr)))

    def eventForcesCalculated(self, dt: float):
        """The closing half-kicks; returns (sum m v^2, sum I w^2)."""
        a, b = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.mdgpu_rigid_leapfrog_post(self.h, 0.5 * float(dt), ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def run(self, nsteps: int, dt: float, record: bool = True) -> Optional[np.ndarray]:
        """nsteps NVE steps; returns (nsteps, 5) {Upot, virial, sum m v^2, sum I w^2, pairs}."""
        out = np.zeros((nsteps, 5)) if record else None
        self._check(self.lib.mdgpu_rigid_run(self.h, int(nsteps), float(dt), _ptr(out)))
        return out

    def setSkin(self, skin: float, listCap: int = 0) -> None:
        """Verlet-skin mode of ``run`` (0 turns it off): candidate lists of radius rc + skin, rebuilt
        when a molecule moved more than skin/2; listCap entries per molecule (0: automatic)."""
        self._check(self.lib.mdgpu_rigid_set_skin(self.h, float(skin), int(listCap)))

    def skinBuilds(self) -> int:
        b = ctypes.c_int64()
        self._check(self.lib.mdgpu_rigid_skin_builds(self.h, ctypes.byref(b)))
        return b.value

    def launches(self) -> int:
        return int(self.profileRead()[1][3])

    def profileEnable(self, enable: bool = True) -> None:
        self._check(self.lib.mdgpu_rigid_profile_enable(self.h, 1 if enable else 0))

    def profileRead(self, reset: bool = False):
        """(ms per group [binning, site rotation + pairs, integration], launch counts [3 groups, all])."""
        t = np.zeros(3)
        cnt = np.zeros(4, dtype=np.int64)
        self._check(self.lib.mdgpu_rigid_profile_read(self.h, _ptr(t), _ptr(cnt), 1 if reset else 0))
        return t, cnt

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.lib.mdgpu_rigid_get_stream(self.h, ctypes.byref(s)))
        return s.value or 0


class LinkedCells:
    """The GPU container: the molecules of one periodic box [0, L) binned into cells of edge >= rc."""

    def __init__(self, length: Sequence[float], cutoffRadius: float, components, mixcoeff=None,
                 LJCutoffRadius: float = 0.0, cellsInCutoffRadius: float = 1.0, precision: int = FP64,
                 device: int = 0):
        self.lib = load_library()
        comps = (_MdComponent * len(components))()
        for k, c in enumerate(components):
            comps[k].eps, comps[k].sigma, comps[k].mass = float(c.eps), float(c.sigma), float(c.mass)
            comps[k].do_shift = 1 if c.do_shift else 0
        self._length = _c64(length)
        mix = None if mixcoeff is None else _c64(mixcoeff).reshape(-1)
        if mix is not None and mix.size == 0:
            mix = None
        self._mix = mix
        h = ctypes.c_void_p()
        st = self.lib.mdgpu_create(ctypes.byref(h), _ptr(self._length), float(cutoffRadius), float(LJCutoffRadius),
                                   float(cellsInCutoffRadius), len(components), ctypes.cast(comps, ctypes.c_void_p),
                                   _ptr(mix), int(precision), int(device))
        self.h = h.value
        if st != 0:
            msg = self.lib.mdgpu_last_error(self.h).decode() if self.h else ""
            if self.h:
                self.lib.mdgpu_destroy(self.h)
            self.h = None
            raise MdgpuError(st, msg)
        self.n = 0
        self.components = components

    @classmethod
    def from_system(cls, system, precision: int = FP64, device: int = 0) -> "LinkedCells":
        lc = cls(system.length, system.cutoff, system.components, system.mix, system.lj_cutoff, 1.0, precision,
                 device)
        lc.addParticles(system.ids, system.cid, system.r, system.v)
        return lc

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.mdgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int) -> None:
        if st != 0:
            raise MdgpuError(st, self.lib.mdgpu_last_error(self.h).decode())

    # -- ParticleContainer-like surface ---------------------------------------------------------
    def addParticles(self, ids, cid, r, v, F=None) -> None:
        ids = _c64(ids, np.uint64)
        n = ids.shape[0]
        self._check(self.lib.mdgpu_set_particles(self.h, n, _ptr(ids), _ptr(_c64(cid, np.int32)),
                                                 _ptr(_c64(r, shape=(n, 3))), _ptr(_c64(v, shape=(n, 3))),
                                                 _ptr(None if F is None else _c64(F, shape=(n, 3)))))
        self.n = n

    def setState(self, r=None, v=None) -> None:
        self._check(self.lib.mdgpu_set_state(self.h, self.n, _ptr(None if r is None else _c64(r, shape=(self.n, 3))),
                                             _ptr(None if v is None else _c64(v, shape=(self.n, 3)))))

    def getNumberOfParticles(self) -> int:
        n = ctypes.c_int64()
        self._check(self.lib.mdgpu_num_particles(self.h, ctypes.byref(n)))
        return n.value

    def update(self) -> None:
        self._check(self.lib.mdgpu_update(self.h))

    def deleteOuterParticles(self) -> None:
        """No-op: the periodic wrap happens inside update()."""

    def traversePairs(self):
        """Forces on all molecules; returns (local Upot, local virial, unordered pairs within rc)."""
        u, w, p = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.mdgpu_traverse_pairs(self.h, ctypes.byref(u), ctypes.byref(w), ctypes.byref(p)))
        return u.value, w.value, p.value

    def getCellIndexOfMolecule(self) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.int64)
        self._check(self.lib.mdgpu_get_cell_index(self.h, self.n, _ptr(out)))
        return out

    def getParticles(self) -> Dict[str, np.ndarray]:
        n = self.n
        ids = np.zeros(n, dtype=np.uint64)
        cid = np.zeros(n, dtype=np.int32)
        r, v, F = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3))
        self._check(self.lib.mdgpu_get_particles(self.h, n, _ptr(ids), _ptr(cid), _ptr(r), _ptr(v), _ptr(F)))
        return dict(id=ids, cid=cid, r=r, v=v, F=F)

    def geometry(self) -> Dict[str, np.ndarray]:
        nc = np.zeros(3, dtype=np.int32)
        cl, hm = np.zeros(3), np.zeros(3)
        self._check(self.lib.mdgpu_get_geometry(self.h, _ptr(nc), _ptr(cl), _ptr(hm)))
        return dict(box_cells=nc, cell_length=cl, halo_min=hm)

    def setPairKernel(self, kind: int) -> None:
        """0 = shared-memory brick kernel (default), 1 = simple gather kernel."""
        self._check(self.lib.mdgpu_set_pair_kernel(self.h, int(kind)))

    def setPrecision(self, precision: int) -> None:
        self._check(self.lib.mdgpu_set_precision(self.h, int(precision)))

    def setSkin(self, skin: float) -> None:
        """Verlet-skin mode of step/run (0 = off): candidate lists of radius rc + skin rebuilt on the
        device when a molecule moved more than skin/2; exact cutoff test on every pair."""
        self._check(self.lib.mdgpu_set_skin(self.h, float(skin)))

    def skinBuilds(self) -> int:
        """List builds of the Verlet-skin mode so far."""
        b = ctypes.c_int64()
        self._check(self.lib.mdgpu_skin_builds(self.h, ctypes.byref(b)))
        return b.value

    def setListPrune(self, prune: float) -> None:
        """Pruned lists of the Verlet-skin mode (0 = off; in effect while 0 < prune < skin): the steps
        evaluate the entries within rc + prune at the last prune, re-pruned on the device after each
        build and when the summed largest drifts since the last prune reach prune/2."""
        self._check(self.lib.mdgpu_set_list_prune(self.h, float(prune)))

    def listPrunes(self) -> int:
        """Prunes of the pruned lists so far."""
        b = ctypes.c_int64()
        self._check(self.lib.mdgpu_list_prunes(self.h, ctypes.byref(b)))
        return b.value

    # -- phase-space files ---------------------------------------------------------------------------
    def writeCheckpoint(self, path: str, current_time: float = 0.0, temperature: float = 1.0,
                        epsilon_rf: float = 1.0e10, digits: int = 0) -> None:
        """The loaded molecules as an old-style phase-space file in the reference's checkpoint layout
        (Domain::writeCheckpoint); digits 0 = the reference's 6 significant digits."""
        self._check(self.lib.mdgpu_write_checkpoint(self.h, os.fsencode(path), float(current_time),
                                                    float(temperature), float(epsilon_rf), int(digits)))

    def readPhaseSpace(self, path: str):
        """Load the molecules of an old-style phase-space file (InputOldstyle); returns the header's
        (currentTime, Temperature)."""
        t, T = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.mdgpu_read_phase_space(self.h, os.fsencode(path), ctypes.byref(t), ctypes.byref(T)))
        self.n = self.getNumberOfParticles()
        return t.value, T.value

    # -- integrator primitives -------------------------------------------------------------------
    def leapfrogPre(self, dt: float, vcorr: float) -> None:
        self._check(self.lib.mdgpu_leapfrog_pre(self.h, float(dt), float(vcorr)))

    def leapfrogPost(self, dt_half: float) -> float:
        s = ctypes.c_double()
        self._check(self.lib.mdgpu_leapfrog_post(self.h, float(dt_half), ctypes.byref(s)))
        return s.value

    def scaleVelocities(self, beta: float) -> None:
        self._check(self.lib.mdgpu_scale_velocities(self.h, float(beta)))

    def farFieldCorrection(self):
        u, w = ctypes.c_double(), ctypes.c_double()
        self._check(self.lib.mdgpu_far_field_correction(self.h, ctypes.byref(u), ctypes.byref(w)))
        return u.value, w.value

    def adjoint(self, gF, gU: float):
        """(dL/dr (n, 3), dL/d eps_ab, dL/d sigma_ab) for cotangents gF = dL/dF, gU = dL/dUpot at the
        current positions (after update)."""
        ns = len(self.components)
        gr = np.zeros((self.n, 3))
        ge = np.zeros((ns, ns))
        gs = np.zeros((ns, ns))
        self._check(self.lib.mdgpu_adjoint(self.h, _ptr(_c64(gF, shape=(self.n, 3))), float(gU), _ptr(gr), _ptr(ge),
                                           _ptr(gs)))
        return gr, ge, gs

    def trajForward(self, nsteps: int, checkpoint_every: int, dt: float) -> float:
        """nsteps NVE steps on the device from the loaded state, snapshots every checkpoint_every
        steps kept on the device; returns the final local Upot (the final state is in the context)."""
        u = ctypes.c_double()
        self._check(self.lib.mdgpu_traj_forward(self.h, int(nsteps), int(checkpoint_every), float(dt), ctypes.byref(u)))
        return u.value

    def trajBackward(self, gF, gU: float):
        """Gradients of a loss with cotangents gF = dL/dF_final, gU = dL/dUpot_final through the
        trajectory of the last trajForward: (dL/dr0, dL/dv0, dL/d eps_ab, dL/d sigma_ab, recomputed
        steps). The context holds the start state afterwards."""
        ns = len(self.components)
        gr, gv = np.zeros((self.n, 3)), np.zeros((self.n, 3))
        ge, gs = np.zeros((ns, ns)), np.zeros((ns, ns))
        rec = ctypes.c_int64()
        self._check(self.lib.mdgpu_traj_backward(self.h, _ptr(_c64(gF, shape=(self.n, 3))), float(gU), _ptr(gr),
                                                 _ptr(gv), _ptr(ge), _ptr(gs), ctypes.byref(rec)))
        return gr, gv, ge, gs, rec.value

    # -- molecule-side operations of MaDPaC's coupled step ---------------------------------------
    def reflectBoundary(self, dim: int, streamOutDir: int, movingWall: bool = False, streamOut: bool = False) -> int:
        """ReflectingBoundary::applyBoundary on the device (after leapfrogPre, before update);
        returns the molecules left beyond the stream-out face."""
        out = ctypes.c_int64()
        self._check(self.lib.mdgpu_reflect_boundary(self.h, int(dim), int(streamOutDir), 1 if movingWall else 0,
                                                    1 if streamOut else 0, ctypes.byref(out)))
        return out.value

    def forceBoundary(self, dim: int, border: float, streamOutDir: int, streamDamping: float = 1.0) -> None:
        """The wall force ForceBoundary computes for the boundary regions (after traversePairs)."""
        self._check(self.lib.mdgpu_force_boundary(self.h, int(dim), float(border), int(streamOutDir),
                                                  float(streamDamping)))

    def trajAdjointTime(self):
        """(ms, launches) of the adjoint kernel in the last trajBackward run with profiling on."""
        ms, k = ctypes.c_double(), ctypes.c_int64()
        self._check(self.lib.mdgpu_traj_adjoint_time(self.h, ctypes.byref(ms), ctypes.byref(k)))
        return ms.value, k.value

    def step(self, dt: float, vcorr: float = 1.0) -> np.ndarray:
        out = np.zeros(4)
        self._check(self.lib.mdgpu_step(self.h, float(dt), float(vcorr), _ptr(out)))
        return out

    def run(self, nsteps: int, dt: float, record: bool = True) -> Optional[np.ndarray]:
        out = np.zeros((nsteps, 4)) if record else None
        self._check(self.lib.mdgpu_run(self.h, int(nsteps), float(dt), _ptr(out)))
        return out

    def runAsync(self, nsteps: int, dt: float) -> None:
        self._check(self.lib.mdgpu_run_async(self.h, int(nsteps), float(dt)))

    def readSteps(self, nsteps: int) -> np.ndarray:
        out = np.zeros((nsteps, 4))
        self._check(self.lib.mdgpu_read_steps(self.h, int(nsteps), _ptr(out)))
        return out

    def profileEnable(self, on: bool = True) -> None:
        self._check(self.lib.mdgpu_profile_enable(self.h, 1 if on else 0))

    def profileRead(self, reset: bool = False):
        t = np.zeros(3)
        cnt = np.zeros(4, dtype=np.int64)
        self._check(self.lib.mdgpu_profile_read(self.h, _ptr(t), _ptr(cnt), 1 if reset else 0))
        return t, cnt

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.lib.mdgpu_get_stream(self.h, ctypes.byref(s)))
        return s.value or 0

    def synchronize(self) -> None:
        self._check(self.lib.mdgpu_synchronize(self.h))


class _MdCouplingCells(ctypes.Structure):
    _fields_ = [("lower", ctypes.c_double * 3), ("upper", ctypes.c_double * 3), ("cell_size", ctypes.c_double),
                ("size", ctypes.c_int32 * 3), ("dim", ctypes.c_int32)]


class CellWiseThermostat:
    """CellWiseThermostat (coupling/thermostat/CellWiseThermostat.cpp:46-156) on the molecules of a
    LinkedCells, over the coupling-cell grid lower..upper of cells of edge cellSize (size cells per
    dimension; size[2] = 1 when dim is 2). applyThermostat(iteration) samples the velocities every
    call and rescales them towards targetTemperature every `interval` iterations. Destroy it (close)
    before its container."""

    def __init__(self, container: LinkedCells, lower, upper, cellSize: float, size, dim: int,
                 targetTemperature: float, gamma: float, interval: int, directed=(0, 0, 0)):
        self.lib = container.lib
        self.container = container
        g = _MdCouplingCells()
        for d in range(3):
            g.lower[d], g.upper[d], g.size[d] = float(lower[d]), float(upper[d]), int(size[d])
        g.cell_size, g.dim = float(cellSize), int(dim)
        dirs = (ctypes.c_int32 * 3)(*[int(x) for x in directed])
        h = ctypes.c_void_p()
        container._check(self.lib.mdgpu_thermostat_create(ctypes.byref(h), container.h, ctypes.byref(g),
                                                          float(targetTemperature), float(gamma), int(interval),
                                                          ctypes.cast(dirs, ctypes.c_void_p)))
        self.h = h.value

    def applyThermostat(self, iteration: int) -> None:
        self.container._check(self.lib.mdgpu_thermostat_apply(self.h, int(iteration)))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.mdgpu_thermostat_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


MIN_BETA = 0.9  # Domain.h:33


class Domain:
    """Upot, virial, temperature and the thermostat factors (Domain.cpp:102-263, one thermostat),
    with the rotational degrees of freedom of rigid molecules (sum I w^2, rotDOF, beta_rot)."""

    def __init__(self, target_temperature: float = 1.0, nve: bool = True):
        self.target_temperature = float(target_temperature)
        self.nve = nve
        self.local_upot = 0.0
        self.local_virial = 0.0
        self.summv2 = 0.0
        self.upot_corr = 0.0
        self.virial_corr = 0.0
        self.global_upot = 0.0
        self.global_virial = 0.0
        self.temperature = target_temperature
        self.beta_trans = 1.0
        self.beta_rot = 1.0
        self.sum_iw2 = 0.0
        self.rot_dof = 0
        self.n = 0

    def setLocalUpot(self, u: float) -> None:
        self.local_upot = u

    def setLocalVirial(self, w: float) -> None:
        self.local_virial = w

    def getGlobalBetaTrans(self) -> float:
        return self.beta_trans

    def getGlobalBetaRot(self) -> float:
        return self.beta_rot

    def calculateGlobalValues(self, tfactor: float = 1.0) -> None:
        """Domain::calculateGlobalValues (Domain.cpp:158-263) for one process and one thermostat."""
        self.global_upot = self.local_upot + self.upot_corr
        self.global_virial = self.local_virial + self.virial_corr
        n = self.n
        rot_dof = self.rot_dof
        sum_iw2 = self.sum_iw2 if rot_dof > 0 else 0.0
        self.temperature = ((self.summv2 + sum_iw2) / float(3 * n + rot_dof) if n > 0
                            else self.target_temperature)
        ti = tfactor * self.target_temperature
        if ti > 0.0 and not self.nve:
            self.beta_trans = math.pow(3.0 * n * ti / self.summv2, 0.4)
            self.beta_rot = 1.0 if sum_iw2 == 0.0 else math.pow(rot_dof * ti / sum_iw2, 0.4)
        else:
            self.beta_trans = 1.0
            self.beta_rot = 1.0
        if self.beta_trans < MIN_BETA or self.beta_rot < MIN_BETA:
            raise MdgpuError(8, "explosion: beta below MIN_BETA (the selective thermostat is not provided)")


class Leapfrog:
    """MarDyn's three-state Leapfrog (integrators/Leapfrog.cpp:14-108) driving the GPU kernels."""

    def __init__(self, timestepLength: float):
        self._state = 3
        self._dt = float(timestepLength)

    def getTimestepLength(self) -> float:
        return self._dt

    def eventNewTimestep(self, cont: LinkedCells, domain: Domain) -> None:
        if self._state == 3:
            self._state = 1
            vcorr = 2. - 1. / domain.getGlobalBetaTrans()
            cont.leapfrogPre(self._dt, vcorr)
            self._state = 2

    def eventForcesCalculated(self, cont: LinkedCells, domain: Domain) -> None:
        if self._state == 2:
            domain.summv2 = cont.leapfrogPost(0.5 * self._dt)
            domain.n = cont.getNumberOfParticles()
            self._state = 3


class Simulation:
    """The reference's step sequence (Simulation.cpp:907-1229) on the GPU container."""

    def __init__(self, system, precision: int = FP64, device: int = 0):
        self.system = system
        self.container = LinkedCells.from_system(system, precision, device)
        self.domain = Domain(system.temperature, system.nve)
        self.domain.n = system.n
        self.domain.upot_corr, self.domain.virial_corr = self.container.farFieldCorrection()
        self.integrator = Leapfrog(system.dt)
        self.npairs = 0.0
        self.simstep = 0

    def _forces(self) -> None:
        u, w, p = self.container.traversePairs()
        self.domain.setLocalUpot(u)
        self.domain.setLocalVirial(w)
        self.npairs = p

    def prepare_start(self) -> None:
        self.container.update()
        self._forces()
        self.domain.summv2 = self._summv2()
        self.domain.calculateGlobalValues(1.0)

    def _summv2(self) -> float:
        st = self.container.getParticles()
        m = self.system.mass()[st["cid"]]
        return float(np.sum(m * np.sum(st["v"] * st["v"], axis=1)))

    def simulateStep(self, tfactor: float = 1.0) -> None:
        self.integrator.eventNewTimestep(self.container, self.domain)
        self.container.update()
        self._forces()
        self.container.deleteOuterParticles()
        self.integrator.eventForcesCalculated(self.container, self.domain)
        self.domain.calculateGlobalValues(tfactor)
        if not self.domain.nve:
            self.container.scaleVelocities(self.domain.getGlobalBetaTrans())
        self.simstep += 1

    def scalars(self) -> Dict[str, float]:
        d = self.domain
        return dict(upot=d.local_upot, virial=d.local_virial, summv2=d.summv2, global_upot=d.global_upot,
                    global_virial=d.global_virial, T=d.temperature, beta_trans=d.beta_trans, npairs=self.npairs)

    def state(self) -> Dict[str, np.ndarray]:
        st = self.container.getParticles()
        o = np.argsort(st["id"], kind="stable")
        st = {k: a[o] for k, a in st.items()}
        st["cell"] = self.container.getCellIndexOfMolecule()[o]
        return st
