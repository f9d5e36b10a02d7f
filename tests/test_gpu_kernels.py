"""The shared-memory brick pair kernel against the simple gather kernel (two independent CUDA
implementations of the same per-pair arithmetic) on boxes of every shape the brick kernel treats
specially: 2 or 3 cells per dimension (periodic images staged twice), non-cubic boxes, two
species, and a dense system whose staged region exceeds shared memory (gather fallback)."""
import numpy as np
import pytest

from madpac_b200 import mdgpu as M
from madpac_b200 import workloads as W

pytestmark = pytest.mark.gpu


def systems():
    out = [W.config_c5(), W.lj_fcc_box(3, 0.8, 1.0, 41, 2.5, [W.Component(1, 1, 1, True)], name="nc2"),
           W.lj_fcc_box(4, 0.7, 1.0, 42, 2.5, [W.Component(1, 1, 1, False)], name="nc3"),
           W.config_c3(seed=43, n_total=20000),
           W.lj_fcc_box(10, 0.9, 1.0, 44, 4.5, [W.Component(1, 1, 1, True)], name="dense_rc4.5")]
    return out


def thermalise(s, steps=30):
    lc = M.LinkedCells.from_system(s, M.FP64)
    lc.update()
    lc.traversePairs()
    lc.run(steps, s.dt)
    st = lc.getParticles()
    lc.close()
    return st["r"]


def forces(s, r, precision, kernel):
    lc = M.LinkedCells.from_system(s, precision)
    lc.setPairKernel(kernel)
    lc.setState(r=r)
    lc.update()
    u, w, npairs = lc.traversePairs()
    F = lc.getParticles()["F"]
    lc.close()
    return F, u, w, npairs


@pytest.mark.parametrize("idx", range(5))
def test_brick_matches_gather_fp64(idx):
    s = systems()[idx]
    r = thermalise(s)
    Fa, ua, wa, na = forces(s, r, M.FP64, 0)
    Fb, ub, wb, nb = forces(s, r, M.FP64, 1)
    assert na == nb
    scale = max(np.sqrt(np.mean(np.sum(Fb ** 2, axis=1))), 1.0)
    assert np.max(np.abs(Fa - Fb)) / scale <= 1e-12
    assert abs(ua - ub) <= 1e-12 * abs(ub)
    assert abs(wa - wb) <= 1e-12 * abs(wb)


@pytest.mark.parametrize("idx", range(5))
def test_brick_mixed_matches_fp64(idx):
    s = systems()[idx]
    r = thermalise(s)
    Fa, ua, wa, na = forces(s, r, M.MIXED, 0)
    Fb, ub, wb, nb = forces(s, r, M.FP64, 1)
    assert na == nb
    rms = np.sqrt(np.mean(np.sum(Fb ** 2, axis=1)))
    assert np.sqrt(np.mean(np.sum((Fa - Fb) ** 2, axis=1))) / rms <= 1e-5
    assert abs(ua - ub) <= 1e-5 * abs(ub)


def test_brick_is_deterministic():
    s = W.config_c5()
    r = thermalise(s, 5)
    a = forces(s, r, M.MIXED, 0)
    b = forces(s, r, M.MIXED, 0)
    np.testing.assert_array_equal(a[0], b[0])
    assert a[1:] == b[1:]
