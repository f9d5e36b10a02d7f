"""ctypes wrapper around the plain-C oracle (oracle/ljmd_oracle.c) and the reference harness.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` and by the
CPU-baseline leg of ``bench.py``. The package never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# Where the reference's MarDyn sources lie (the one place this location is set; the environment
# variable MADPAC_REFERENCE_MARDYN overrides it). Only the recipe that compiles the reference into
# oracle/_ref reads it; without the sources, the prebuilt oracle/_ref is used as it is.
REFERENCE_MARDYN = os.environ.get("MADPAC_REFERENCE_MARDYN", "/root/reference/madpac/mardyn")
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DRIVER = os.path.join(HERE, "_ref", "ref_driver")

_lib = None


def build() -> None:
    """Compile liboracle.so (and, when the reference tree is present, the reference harness)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def build_reference(ref_dir: str = REFERENCE_MARDYN) -> bool:
    """Compile the reference sources into oracle/_ref when the reference tree is present."""
    if not os.path.isdir(ref_dir):
        return False
    subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref", f"REF={ref_dir}"], check=True)
    return True


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [dp, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                 dp, dp, dp, ip, dp]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        for name in ("orc_status", "orc_update", "orc_exchange", "orc_traverse", "orc_delete_outer",
                     "orc_prepare_start"):
            getattr(L, name).argtypes = [ctypes.c_void_p]
            getattr(L, name).restype = ctypes.c_int
        L.orc_add_particles.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p]
        L.orc_add_particles.restype = ctypes.c_int
        L.orc_init.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.orc_init.restype = ctypes.c_int
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        L.orc_step.restype = ctypes.c_int
        L.orc_count.argtypes = [ctypes.c_void_p]
        L.orc_count.restype = ctypes.c_long
        L.orc_get.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 6
        L.orc_scalars.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_geometry.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_cell_index.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.orc_cell_index.restype = ctypes.c_long
        L.orc_params.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        L.orc_rdf_enable.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.orc_rdf_counts.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class OracleError(RuntimeError):
    pass


class Oracle:
    """One MarDyn-equivalent sequential LJ simulation held by the C oracle."""

    def __init__(self, system, add_particles: bool = True):
        L = lib()
        self.system = system
        nc = len(system.components)
        length = np.ascontiguousarray(system.length, dtype=np.float64)
        eps = np.ascontiguousarray(system.eps())
        sig = np.ascontiguousarray(system.sigma())
        mass = np.ascontiguousarray(system.mass())
        shift = np.ascontiguousarray(system.do_shift(), dtype=np.int32)
        mix = np.ascontiguousarray(np.asarray(system.mix, dtype=np.float64).reshape(-1))
        if mix.size == 0:
            mix = np.zeros(2)
        dp = ctypes.POINTER(ctypes.c_double)
        self._keep = (length, eps, sig, mass, shift, mix)
        self.h = L.orc_create(length.ctypes.data_as(dp), system.cutoff, system.lj_cutoff, 1.0, nc,
                              eps.ctypes.data_as(dp), sig.ctypes.data_as(dp), mass.ctypes.data_as(dp),
                              shift.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), mix.ctypes.data_as(dp))
        self._check(L.orc_status(self.h))
        if add_particles:
            self.add_particles(system)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def _check(self, st: int) -> None:
        if st != 0:
            raise OracleError(f"oracle status {st}")

    def add_particles(self, system) -> None:
        ids = np.ascontiguousarray(system.ids, dtype=np.uint64)
        cid = np.ascontiguousarray(system.cid, dtype=np.int32)
        r = np.ascontiguousarray(system.r, dtype=np.float64)
        v = np.ascontiguousarray(system.v, dtype=np.float64)
        self._check(lib().orc_add_particles(self.h, system.n, _p(ids), _p(cid), _p(r), _p(v)))

    def init(self) -> None:
        self._check(lib().orc_init(self.h, float(self.system.temperature), 1 if self.system.nve else 0))

    def prepare_start(self) -> None:
        self._check(lib().orc_prepare_start(self.h))

    def step(self, dt: Optional[float] = None, tfactor: float = 1.0) -> None:
        self._check(lib().orc_step(self.h, float(self.system.dt if dt is None else dt), tfactor))

    def update(self) -> None:
        self._check(lib().orc_update(self.h))

    def exchange(self) -> None:
        self._check(lib().orc_exchange(self.h))

    def traverse(self) -> None:
        self._check(lib().orc_traverse(self.h))

    def delete_outer(self) -> None:
        self._check(lib().orc_delete_outer(self.h))

    def rdf_enable(self, interval: float, bins: int) -> None:
        lib().orc_rdf_enable(self.h, interval, bins)
        self._bins = bins

    def rdf_counts(self) -> np.ndarray:
        out = np.zeros(self._bins, dtype=np.uint64)
        lib().orc_rdf_counts(self.h, _p(out))
        return out

    def state(self, sort: bool = True) -> Dict[str, np.ndarray]:
        n = lib().orc_count(self.h)
        ids = np.zeros(n, dtype=np.uint64)
        cid = np.zeros(n, dtype=np.int32)
        r = np.zeros((n, 3))
        v = np.zeros((n, 3))
        F = np.zeros((n, 3))
        cell = np.zeros(n, dtype=np.int64)
        lib().orc_get(self.h, _p(ids), _p(cid), _p(r), _p(v), _p(F), _p(cell))
        out = dict(id=ids, cid=cid, r=r, v=v, F=F, cell=cell)
        if sort:
            o = np.argsort(ids, kind="stable")
            out = {k: a[o] for k, a in out.items()}
        return out

    def scalars(self) -> Dict[str, float]:
        out = np.zeros(13)
        lib().orc_scalars(self.h, _p(out))
        keys = ["upot", "virial", "summv2", "global_upot", "global_virial", "T", "beta_trans",
                "upot_corr", "virial_corr", "npairs", "summv2_end", "upot_exact", "virial_exact"]
        return dict(zip(keys, out.tolist()))

    def geometry(self):
        oi = np.zeros(9, dtype=np.int32)
        od = np.zeros(9)
        lib().orc_geometry(self.h, _p(oi), _p(od))
        return dict(box_cells=oi[0:3], halo_cells=oi[3:6], cells_per_dim=oi[6:9], cell_length=od[0:3],
                    halo_min=od[3:6], halo_max=od[6:9])

    def cell_index(self, r) -> int:
        a = np.ascontiguousarray(r, dtype=np.float64)
        return int(lib().orc_cell_index(self.h, _p(a)))

    def params(self, ci: int, cj: int) -> np.ndarray:
        out = np.zeros(3)
        lib().orc_params(self.h, ci, cj, _p(out))
        return out


def run_oracle(system, nsteps: int, dump_steps=()) -> Dict:
    """Reference step sequence on the oracle: init, prepare_start, then nsteps simulateStep."""
    o = Oracle(system)
    o.init()
    o.prepare_start()
    scal = [o.scalars()]
    dumps = {}
    if 0 in dump_steps:
        dumps[0] = o.state()
    for k in range(1, nsteps + 1):
        o.step()
        scal.append(o.scalars())
        if k in dump_steps:
            dumps[k] = o.state()
    return dict(scalars=scal, dumps=dumps)


def read_ref_dump(path: str) -> Dict[str, np.ndarray]:
    """Read one step dump written by oracle/_ref/ref_driver."""
    with open(path, "rb") as f:
        n = int(np.frombuffer(f.read(8), dtype=np.int64)[0])
        ids = np.frombuffer(f.read(8 * n), dtype=np.uint64)
        cid = np.frombuffer(f.read(8 * n), dtype=np.int64)
        r = np.frombuffer(f.read(24 * n), dtype=np.float64).reshape(n, 3)
        v = np.frombuffer(f.read(24 * n), dtype=np.float64).reshape(n, 3)
        F = np.frombuffer(f.read(24 * n), dtype=np.float64).reshape(n, 3)
        cell = np.frombuffer(f.read(8 * n), dtype=np.int64)
    out = dict(id=ids, cid=cid.astype(np.int32), r=r, v=v, F=F, cell=cell)
    rot = path[:-4] + ".rot.bin"
    if os.path.exists(rot):
        with open(rot, "rb") as f:
            m = int(np.frombuffer(f.read(8), dtype=np.int64)[0])
            out["q"] = np.frombuffer(f.read(32 * m), dtype=np.float64).reshape(m, 4)
            out["D"] = np.frombuffer(f.read(24 * m), dtype=np.float64).reshape(m, 3)
            out["M"] = np.frombuffer(f.read(24 * m), dtype=np.float64).reshape(m, 3)
    return out


def run_reference(system, nsteps: int, dump_steps=(), workdir: Optional[str] = None) -> Dict:
    """Run the compiled reference harness (oracle/_ref/ref_driver) on the system."""
    from madpac_b200.workloads import write_cfg, write_inp

    if not os.path.exists(REF_DRIVER):
        raise FileNotFoundError("oracle/_ref/ref_driver is not built")
    tmp = workdir or tempfile.mkdtemp(prefix="mdref_")
    write_inp(system, os.path.join(tmp, "sys.inp"))
    write_cfg(system, os.path.join(tmp, "sys.cfg"), "sys.inp")
    dl = ",".join(str(s) for s in dump_steps) or "-1"
    subprocess.run([REF_DRIVER, "sys.cfg", str(nsteps), ".", dl], cwd=tmp, check=True,
                   stdout=subprocess.DEVNULL)
    scal = []
    with open(os.path.join(tmp, "scalars.txt")) as f:
        for line in f:
            p = line.split()
            scal.append(dict(step=int(p[0]), upot=float(p[1]), virial=float(p[2]), summv2=float(p[3]),
                             n=int(p[4])))
    with open(os.path.join(tmp, "rot.txt")) as f:
        for rec, line in zip(scal, f):
            rec["sum_iw2"] = float(line.split()[1])
    dumps = {s: read_ref_dump(os.path.join(tmp, f"step{s:06d}.bin")) for s in dump_steps}
    return dict(scalars=scal, dumps=dumps, workdir=tmp)


def _run_oracle_job(args):
    system, nsteps, dump_steps = args
    return run_oracle(system, nsteps, dump_steps)


def run_oracle_many(systems, nsteps: int, dump_steps=(), processes: Optional[int] = None):
    """run_oracle on many independent boxes, spread over the host cores by a pool of freshly
    spawned processes (spawn, not fork: the caller may hold a CUDA context). Results in the order
    of `systems`."""
    import multiprocessing as mp

    if processes is None:
        processes = max(1, min(len(systems), os.cpu_count() or 1, 32))
    jobs = [(s, nsteps, tuple(dump_steps)) for s in systems]
    if processes == 1:
        return [_run_oracle_job(j) for j in jobs]
    ctx = mp.get_context("spawn")
    with ctx.Pool(processes) as pool:
        # largest boxes first, so that the pool ends together
        order = sorted(range(len(jobs)), key=lambda k: -systems[k].n)
        out = pool.map(_run_oracle_job, [jobs[k] for k in order], chunksize=1)
    res = [None] * len(jobs)
    for k, r in zip(order, out):
        res[k] = r
    return res
