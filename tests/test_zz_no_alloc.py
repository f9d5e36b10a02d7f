"""mdgpu_forces_noalloc, the entry point for callers that cannot allocate device memory while they
run (hosts owning all device memory through their own pool, latency-bound loops). It must give the forces, Upot and virial of the regular context path
(mdgpu_create / mdgpu_update / mdgpu_traverse_pairs) on two calls in a row -- the second call
reuses the static scratch array the first one left behind -- within the tolerances of the other
GPU tests. This file is collected last so that a run stopping at the first failure has already
run every other test."""
import numpy as np
import pytest

from madpac_b200 import mdgpu as M
from madpac_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _thermalised(system, steps=40):
    lc = M.LinkedCells.from_system(system, M.FP64)
    lc.update()
    lc.traversePairs()
    lc.run(steps, system.dt)
    r = lc.getParticles()["r"]
    lc.close()
    return r


def _context_forces(system, r, precision):
    lc = M.LinkedCells.from_system(system, precision)
    lc.setState(r=r)
    lc.update()
    u, w, _ = lc.traversePairs()
    F = lc.getParticles()["F"]
    lc.close()
    return F, u, w


@pytest.mark.parametrize("precision,tol", [(M.FP64, 1e-12), (M.MIXED, 1e-5)])
def test_noalloc_matches_context_path_on_two_calls(precision, tol):
    torch = pytest.importorskip("torch")
    system = W.config_c5()  # 16,384 molecules, two species, 1,000 cells
    r = _thermalised(system)
    F_ref, u_ref, w_ref = _context_forces(system, r, precision)
    F_fp64, _, _ = _context_forces(system, r, M.FP64)
    scale = max(float(np.sqrt(np.mean(np.sum(F_fp64 ** 2, axis=1)))), 1.0)
    d_r = torch.tensor(r, dtype=torch.float64, device="cuda").contiguous()
    d_cid = torch.tensor(system.cid, dtype=torch.int32, device="cuda").contiguous()
    outs = []
    for _ in range(2):
        d_F = torch.full((system.n, 3), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        u, w = M.forces_noalloc(d_r.data_ptr(), d_cid.data_ptr(), d_F.data_ptr(), system.n, system.length,
                                system.cutoff, system.components, system.mix, system.lj_cutoff, precision)
        F = d_F.cpu().numpy()
        outs.append((F, u, w))
        assert np.all(np.isfinite(F))
        assert np.max(np.abs(F - F_ref)) / scale <= tol
        assert abs(u - u_ref) <= tol * abs(u_ref)
        assert abs(w - w_ref) <= tol * abs(w_ref)
    # the second call, on the scratch the first one left, gives the same answer
    np.testing.assert_array_equal(outs[0][0], outs[1][0])
    assert outs[0][1:] == outs[1][1:]


def test_noalloc_rejects_more_molecules_than_its_scratch_holds():
    with pytest.raises(M.MdgpuError) as e:
        M.forces_noalloc(1, 1, 1, 32769, [60.0, 60.0, 60.0], 2.5, [W.Component()])
    assert e.value.code == 10
    assert "32768" in str(e.value)


def test_noalloc_rejects_a_negative_lj_cutoff():
    with pytest.raises(M.MdgpuError) as e:
        M.forces_noalloc(1, 1, 1, 100, [60.0, 60.0, 60.0], 2.5, [W.Component()], None, -1.0)
    assert e.value.code == 1
    assert "lj_cutoff" in str(e.value)


def test_noalloc_leaves_the_current_device_as_it_found_it():
    torch = pytest.importorskip("torch")
    system = W.lj_fcc_box(6, 0.8, 1.0, 3, 2.5)
    dev = torch.cuda.device_count() - 1
    torch.cuda.set_device(dev)
    d_r = torch.tensor(system.r, dtype=torch.float64, device=f"cuda:{dev}")
    d_cid = torch.tensor(system.cid, dtype=torch.int32, device=f"cuda:{dev}")
    d_F = torch.zeros((system.n, 3), dtype=torch.float64, device=f"cuda:{dev}")
    torch.cuda.synchronize()
    M.forces_noalloc(d_r.data_ptr(), d_cid.data_ptr(), d_F.data_ptr(), system.n, system.length, system.cutoff,
                     system.components, system.mix, system.lj_cutoff, M.FP64, device=dev)
    assert torch.cuda.current_device() == dev
    torch.cuda.set_device(0)
