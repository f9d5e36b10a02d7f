"""MarDyn's own simulation loop on the device container: the reference's Simulation (configuration
reader, prepare_start, simulateStart / simulateStep / simulateFinish, Domain, thermostat, checkpoint
writer) compiled from its sources and linked with the shim (madpac_b200/mardyn_shim: GpuLinkedCells,
GpuLeapfrog, GpuSimulation) and libmdgpu.so, run on the five golden systems and compared with the
reference's own runs (the golden fixtures, made by the unmodified reference with the same harness
loop):

  * step 0 forces within 1e-12 of the reference's (max |dF| / max(rms F, 1)), Upot and virial
    within 1e-10;
  * every step's Upot, virial and sum m v^2 within 1e-9; at the dumped steps r within 1e-9, v within
    1e-8 and F within 1e-8 (the device sums in another order and MD amplifies the last bits);
  * the thermostatted system goes through the host mirror (the Domain's velocity scaling acts on
    host molecules and is uploaded before the next device step);
  * the mixed form through the same loop within 1e-5 (rms force) of the reference.

The shim harness is built by madpac_b200/mardyn_shim/Makefile against the reference's headers
and objects; where it was not built (no reference sources on the machine that built the tree)
the tests are skipped.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN_NAMES, ROOT, system_from_golden
from madpac_b200 import workloads as W

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(ROOT, "madpac_b200", "mardyn_shim", "_build", "shim_driver")


def force_err_max(F, Fref):
    rms = max(np.sqrt(np.mean(np.sum(Fref * Fref, axis=1))), 1.0)
    return float(np.max(np.linalg.norm(F - Fref, axis=1)) / rms)


def force_err_rms(F, Fref):
    rms = np.sqrt(np.mean(np.sum(Fref * Fref, axis=1)))
    return float(np.sqrt(np.mean(np.sum((F - Fref) ** 2, axis=1))) / rms)


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def run_shim(system, nsteps, dumps, precision="fp64"):
    if not os.path.exists(DRIVER):
        pytest.skip("the MarDyn shim harness was not built (needs the reference sources)")
    tmp = tempfile.mkdtemp(prefix="mdshim_")
    W.write_inp(system, os.path.join(tmp, "sys.inp"))
    W.write_cfg(system, os.path.join(tmp, "sys.cfg"), "sys.inp")
    dl = ",".join(str(s) for s in sorted(dumps)) or "-1"
    r = subprocess.run([DRIVER, "sys.cfg", str(nsteps), ".", dl, precision], cwd=tmp, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    scal = np.loadtxt(os.path.join(tmp, "scalars.txt"), ndmin=2)
    out = {k: O.read_ref_dump(os.path.join(tmp, f"step{k:06d}.bin")) for k in dumps}
    return scal, out


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_mardyn_loop_on_the_device_matches_reference(name):
    system, g, meta = system_from_golden(name)
    nsteps = meta["nsteps"]
    dumps = set(meta["dumps"]) | {0}
    scal, out = run_shim(system, nsteps, dumps)
    assert scal.shape[0] == nsteps + 1
    np.testing.assert_array_equal(scal[:, 4], [system.n] * (nsteps + 1))
    d0 = out[0]
    np.testing.assert_array_equal(d0["id"], g["s0_id"])
    assert force_err_max(d0["F"], g["s0_F"]) <= 1e-12
    assert rel(scal[0, 1], g["upot"][0]) <= 1e-10
    assert rel(scal[0, 2], g["virial"][0]) <= 1e-10
    for k in range(1, nsteps + 1):
        assert rel(scal[k, 1], g["upot"][k]) <= 1e-9, (k, scal[k], g["upot"][k])
        assert rel(scal[k, 2], g["virial"][k]) <= 1e-9, k
        assert rel(scal[k, 3], g["summv2"][k]) <= 1e-9, k
    for k in meta["dumps"]:
        if k == 0:
            continue
        d = out[k]
        np.testing.assert_array_equal(d["id"], g[f"s{k}_id"])
        np.testing.assert_allclose(d["r"], g[f"s{k}_r"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(d["v"], g[f"s{k}_v"], rtol=0, atol=1e-8)
        assert force_err_max(d["F"], g[f"s{k}_F"]) <= 1e-8


def test_mardyn_loop_mixed_form():
    system, g, meta = system_from_golden("two_species_2048")
    k = max(meta["dumps"])
    scal, out = run_shim(system, k, {k}, precision="mixed")
    assert force_err_rms(out[k]["F"], g[f"s{k}_F"]) <= 1e-5
    for j in range(1, k + 1):
        assert rel(scal[j, 1], g["upot"][j]) <= 1e-6
        assert rel(scal[j, 3], g["summv2"][j]) <= 1e-6
