"""The adjoint of forces and energy (mdgpu_adjoint) and gradients through Leapfrog trajectories.

Loss L = sum_i |F_i - F_i^t|^2 + 0.1 (U - U^t)^2 with targets made by the method itself at
eps_AB x 1.1 and sigma_AB x 0.95 (two species, 50/50, sigma_A 1, sigma_B 0.9, eps_A 1, eps_B 0.8,
Lorentz-Berthelot mixing, truncated-shifted). Checks:
  * against an independent O(N^2) NumPy FP64 gradient on a 2,048-molecule box (relative 1e-10);
  * against FP64 central finite differences of positions and of eps_ab / sigma_ab (relative 1e-6);
  * through a torch.autograd.Function wrapper (torch.autograd.gradcheck on a 108-molecule box);
  * through 50 Leapfrog steps with checkpoints every 10 steps, against finite differences.
"""
import numpy as np
import pytest

from madpac_b200 import mdgpu as M
from madpac_b200 import workloads as W
from madpac_b200.trajectory import TrajectoryAdjoint

pytestmark = pytest.mark.gpu


# ------------------------------------------------------------------------ helpers

def thermalised_two_species(n_cells, seed, steps=100):
    s = W.lj_fcc_box(n_cells, 0.8, 1.0, seed, 2.5, W.two_species(), [0.5, 0.5], np.ones((1, 2)))
    lc = M.LinkedCells.from_system(s)
    lc.update()
    lc.traversePairs()
    lc.run(steps, s.dt)
    st = lc.getParticles()
    lc.close()
    s.r, s.v = st["r"], st["v"]
    return s


def with_pair_params(system, eps_ab, sig_ab):
    """The same molecules with component-pair parameters eps_ab, sigma_ab (symmetric ns x ns):
    components carry the diagonal, the mixing coefficients xi, eta the off-diagonal entries."""
    ns = len(system.components)
    comps = [W.Component(float(eps_ab[a][a]), float(sig_ab[a][a]), c.mass, c.do_shift)
             for a, c in enumerate(system.components)]
    mix = []
    for a in range(ns):
        for b in range(a + 1, ns):
            mix.append((eps_ab[a][b] / np.sqrt(eps_ab[a][a] * eps_ab[b][b]),
                        2.0 * sig_ab[a][b] / (sig_ab[a][a] + sig_ab[b][b])))
    out = W.System(**{**system.__dict__})
    out.components = comps
    out.mix = np.array(mix, dtype=np.float64).reshape(-1, 2)
    return out


def pair_params(system):
    ns = len(system.components)
    eps = np.zeros((ns, ns))
    sig = np.zeros((ns, ns))
    k = 0
    for a in range(ns):
        eps[a, a] = system.components[a].eps
        sig[a, a] = system.components[a].sigma
    for a in range(ns):
        for b in range(a + 1, ns):
            xi, eta = system.mix[k]
            k += 1
            eps[a, b] = eps[b, a] = xi * np.sqrt(eps[a, a] * eps[b, b])
            sig[a, b] = sig[b, a] = eta * 0.5 * (sig[a, a] + sig[b, b])
    return eps, sig


class Evaluator:
    """FP64 forces and energy of a fixed set of molecules at any positions."""

    def __init__(self, system):
        self.lc = M.LinkedCells.from_system(system, M.FP64)

    def __call__(self, r):
        self.lc.setState(r=r)
        self.lc.update()
        u, _, _ = self.lc.traversePairs()
        return self.lc.getParticles()["F"], u

    def close(self):
        self.lc.close()


def targets(system):
    eps, sig = pair_params(system)
    eps_t, sig_t = eps.copy(), sig.copy()
    eps_t[0, 1] = eps_t[1, 0] = eps[0, 1] * 1.1
    sig_t[0, 1] = sig_t[1, 0] = sig[0, 1] * 0.95
    ev = Evaluator(with_pair_params(system, eps_t, sig_t))
    Ft, Ut = ev(system.r)
    ev.close()
    return Ft, Ut


def loss(F, U, Ft, Ut):
    return float(np.sum((F - Ft) ** 2) + 0.1 * (U - Ut) ** 2)


def numpy_gradient(system, r, gF, gU):
    """Independent O(N^2) FP64 adjoint with the minimum-image convention."""
    eps, sig = pair_params(system)
    ns = len(system.components)
    rc = system.cutoff
    L = system.length
    n = r.shape[0]
    iu, ju = np.triu_indices(n, 1)
    d = r[iu] - r[ju]
    d -= L * np.round(d / L)
    q = np.sum(d * d, axis=1)
    m = q < rc * rc
    iu, ju, d, q = iu[m], ju[m], d[m], q[m]
    ti, tj = system.cid[iu], system.cid[ju]
    e24 = 24.0 * eps[ti, tj]
    sg2 = sig[ti, tj] ** 2
    shifted = np.array([[c.do_shift for c in system.components]] * ns)
    shifted = shifted | ~np.eye(ns, dtype=bool)  # cross pairs are always shifted
    shf = shifted[ti, tj]
    s6 = (sg2 / q) ** 3
    s12 = s6 * s6
    fac = e24 * (2 * s12 - s6) / q
    dfac = e24 * (4 * s6 - 14 * s12) / q ** 2
    w = gF[iu] - gF[ju]
    dw = np.sum(d * w, axis=1)
    gi = fac[:, None] * w + (2 * dfac * dw)[:, None] * d - gU * fac[:, None] * d
    gr = np.zeros((n, 3))
    np.add.at(gr, iu, gi)
    np.add.at(gr, ju, -gi)
    sr6 = (sg2 / rc ** 2) ** 3
    c6 = np.where(shf, sr6 - sr6 ** 2, 0.0)
    c6s = np.where(shf, 3 * sr6 - 6 * sr6 ** 2, 0.0)
    de24 = fac * dw / e24 + gU * (s12 - s6 + c6) / 6
    dsg2 = e24 * (12 * s12 - 3 * s6) / (q * sg2) * dw + gU * e24 * (6 * s12 - 3 * s6 + c6s) / (6 * sg2)
    ge = np.zeros((ns, ns))
    gs = np.zeros((ns, ns))
    lo, hi = np.minimum(ti, tj), np.maximum(ti, tj)
    np.add.at(ge, (lo, hi), de24 * 24.0)
    np.add.at(gs, (lo, hi), dsg2 * 2.0 * np.sqrt(sg2))
    ge = ge + np.triu(ge, 1).T
    gs = gs + np.triu(gs, 1).T
    return gr, ge, gs


# ------------------------------------------------------------------------ tests

@pytest.fixture(scope="module")
def box2048():
    s = thermalised_two_species(8, 61)
    Ft, Ut = targets(s)
    return s, Ft, Ut


def test_adjoint_matches_numpy_o_n2_gradient(box2048):
    s, Ft, Ut = box2048
    ev = Evaluator(s)
    F, U = ev(s.r)
    gF, gU = 2 * (F - Ft), 0.2 * (U - Ut)
    gr, ge, gs = ev.lc.adjoint(gF, gU)
    ev.close()
    nr, ne, nsg = numpy_gradient(s, s.r, gF, gU)
    scale = np.max(np.abs(nr))
    assert np.max(np.abs(gr - nr)) <= 1e-10 * scale
    np.testing.assert_allclose(ge, ne, rtol=1e-10, atol=1e-10 * np.max(np.abs(ne)))
    np.testing.assert_allclose(gs, nsg, rtol=1e-10, atol=1e-10 * np.max(np.abs(nsg)))


def test_adjoint_matches_central_differences_in_positions(box2048):
    s, Ft, Ut = box2048
    ev = Evaluator(s)
    F, U = ev(s.r)
    gr, _, _ = ev.lc.adjoint(2 * (F - Ft), 0.2 * (U - Ut))
    rng = np.random.default_rng(7)
    h = 1e-6
    scale = np.sqrt(np.mean(gr ** 2))
    for k, d in zip(rng.integers(0, s.n, 12), rng.integers(0, 3, 12)):
        rp, rm = s.r.copy(), s.r.copy()
        rp[k, d] += h
        rm[k, d] -= h
        fd = (loss(*ev(rp), Ft, Ut) - loss(*ev(rm), Ft, Ut)) / (2 * h)
        assert abs(fd - gr[k, d]) <= 1e-6 * max(abs(gr[k, d]), scale), (k, d, fd, gr[k, d])
    ev.close()


def test_adjoint_matches_central_differences_in_pair_parameters(box2048):
    s, Ft, Ut = box2048
    ev = Evaluator(s)
    F, U = ev(s.r)
    _, ge, gs = ev.lc.adjoint(2 * (F - Ft), 0.2 * (U - Ut))
    ev.close()
    eps, sig = pair_params(s)

    def L_at(e, g):
        e2 = Evaluator(with_pair_params(s, e, g))
        val = loss(*e2(s.r), Ft, Ut)
        e2.close()
        return val

    for (a, b) in [(0, 0), (0, 1), (1, 1)]:
        for which in ("eps", "sig"):
            h = 1e-7
            p_plus, p_minus = (eps.copy(), sig.copy()), (eps.copy(), sig.copy())
            idx = 0 if which == "eps" else 1
            p_plus[idx][a, b] += h
            p_plus[idx][b, a] = p_plus[idx][a, b]
            p_minus[idx][a, b] -= h
            p_minus[idx][b, a] = p_minus[idx][a, b]
            fd = (L_at(*p_plus) - L_at(*p_minus)) / (2 * h)
            ad = (ge if which == "eps" else gs)[a, b]
            assert abs(fd - ad) <= 1e-6 * abs(ad), (which, a, b, fd, ad)


def test_torch_autograd_function_gradcheck():
    torch = pytest.importorskip("torch")
    s = thermalised_two_species(3, 62, steps=50)  # 108 molecules, 2 cells per dimension

    class LJ(torch.autograd.Function):
        """(positions, [eps_AA, eps_AB, eps_BB], [sigma_AA, sigma_AB, sigma_BB]) -> (F, Upot) on the
        GPU; the backward pass is mdgpu_adjoint."""

        @staticmethod
        def forward(ctx, r, ep, sp):
            e = np.array([[ep[0].item(), ep[1].item()], [ep[1].item(), ep[2].item()]])
            g = np.array([[sp[0].item(), sp[1].item()], [sp[1].item(), sp[2].item()]])
            ev = Evaluator(with_pair_params(s, e, g))
            F, U = ev(r.detach().numpy())
            ev.close()
            ctx.saved = (r.detach().numpy().copy(), e, g)
            return torch.from_numpy(F.copy()), torch.tensor(U, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gF, gU):
            r_, e, g = ctx.saved
            ev = Evaluator(with_pair_params(s, e, g))
            ev(r_)
            gr, ge, gs = ev.lc.adjoint(gF.detach().numpy(), float(gU))
            ev.close()
            pe = torch.tensor([ge[0, 0], ge[0, 1], ge[1, 1]], dtype=torch.float64)
            ps = torch.tensor([gs[0, 0], gs[0, 1], gs[1, 1]], dtype=torch.float64)
            return torch.from_numpy(gr), pe, ps

    eps, sig = pair_params(s)
    r = torch.tensor(s.r, dtype=torch.float64, requires_grad=True)
    ep = torch.tensor([eps[0, 0], eps[0, 1], eps[1, 1]], dtype=torch.float64, requires_grad=True)
    sp = torch.tensor([sig[0, 0], sig[0, 1], sig[1, 1]], dtype=torch.float64, requires_grad=True)

    def scalar(r_, ep_, sp_):
        F, U = LJ.apply(r_, ep_, sp_)
        return (F ** 2).sum() * 1e-4 + 0.1 * U

    assert torch.autograd.gradcheck(scalar, (r, ep, sp), eps=1e-6, atol=1e-6, rtol=1e-5)


def test_gradient_through_50_leapfrog_steps_with_checkpoints(box2048):
    s, Ft, Ut = box2048
    steps, every = 50, 10
    tr = TrajectoryAdjoint(s, steps, every)
    r, v, F, U = tr.forward(s.r, s.v)
    gr0, gv0, ge, gs = tr.backward(2 * (F - Ft), 0.2 * (U - Ut))
    # each segment is recomputed once from its checkpoint
    assert tr.recomputed_steps == steps
    assert sorted(tr.checkpoints) == [0, 10, 20, 30, 40]
    tr.close()

    def L_final(r0, v0, system=s):
        t = TrajectoryAdjoint(system, steps, every)
        _, _, Fe, Ue = t.forward(r0, v0)
        t.close()
        return loss(Fe, Ue, Ft, Ut)

    rng = np.random.default_rng(11)
    h = 1e-6
    scale = np.sqrt(np.mean(gr0 ** 2))
    for k, d in zip(rng.integers(0, s.n, 4), rng.integers(0, 3, 4)):
        rp, rm = s.r.copy(), s.r.copy()
        rp[k, d] += h
        rm[k, d] -= h
        fd = (L_final(rp, s.v) - L_final(rm, s.v)) / (2 * h)
        assert abs(fd - gr0[k, d]) <= 1e-6 * max(abs(gr0[k, d]), scale), (k, d, fd, gr0[k, d])
    # one velocity component and the cross-species epsilon
    vp, vm = s.v.copy(), s.v.copy()
    vp[5, 1] += h
    vm[5, 1] -= h
    fd = (L_final(s.r, vp) - L_final(s.r, vm)) / (2 * h)
    assert abs(fd - gv0[5, 1]) <= 1e-6 * max(abs(gv0[5, 1]), np.sqrt(np.mean(gv0 ** 2)))
    eps, sig = pair_params(s)
    hp = 1e-7
    e_p, e_m = eps.copy(), eps.copy()
    e_p[0, 1] = e_p[1, 0] = eps[0, 1] + hp
    e_m[0, 1] = e_m[1, 0] = eps[0, 1] - hp
    fd = (L_final(s.r, s.v, with_pair_params(s, e_p, sig)) - L_final(s.r, s.v, with_pair_params(s, e_m, sig))) / (2 * hp)
    assert abs(fd - ge[0, 1]) <= 1e-6 * abs(ge[0, 1]), (fd, ge[0, 1])


def test_adjoint_on_the_16k_two_species_box():
    """The differentiation configuration: 16,384 molecules, rho 0.8, T 1.0, 50/50 A/B."""
    s = W.config_c5()
    lc = M.LinkedCells.from_system(s)
    lc.update()
    lc.traversePairs()
    lc.run(100, s.dt)
    s.r = lc.getParticles()["r"]
    lc.close()
    Ft, Ut = targets(s)
    ev = Evaluator(s)
    F, U = ev(s.r)
    gr, ge, gs = ev.lc.adjoint(2 * (F - Ft), 0.2 * (U - Ut))
    rng = np.random.default_rng(3)
    h = 1e-6
    scale = np.sqrt(np.mean(gr ** 2))
    for k, d in zip(rng.integers(0, s.n, 6), rng.integers(0, 3, 6)):
        rp, rm = s.r.copy(), s.r.copy()
        rp[k, d] += h
        rm[k, d] -= h
        fd = (loss(*ev(rp), Ft, Ut) - loss(*ev(rm), Ft, Ut)) / (2 * h)
        assert abs(fd - gr[k, d]) <= 1e-6 * max(abs(gr[k, d]), scale)
    ev.close()


class HostLoopTrajectoryAdjoint:
    """The same backward pass driven from the host one C-ABI call at a time (checkpoints as host
    arrays, the Leapfrog algebra in NumPy, mdgpu_adjoint per step): an independent second
    implementation of what mdgpu_traj_forward / mdgpu_traj_backward do on the device."""

    def __init__(self, system, nsteps, every):
        self.system, self.nsteps, self.every = system, nsteps, every
        self.lc = M.LinkedCells.from_system(system, M.FP64)
        self.dt = float(system.dt)
        self.c = ((0.5 * self.dt) / system.mass()[system.cid])[:, None]

    def close(self):
        self.lc.close()

    def _forces_at(self, r):
        self.lc.setState(r=r)
        self.lc.update()
        self.lc.traversePairs()
        return self.lc.getParticles()["F"]

    def _step(self, r, v):
        self.lc.setState(r=r, v=v)
        self.lc.update()
        self.lc.traversePairs()
        self.lc.leapfrogPre(self.dt, 1.0)
        self.lc.update()
        self.lc.traversePairs()
        self.lc.leapfrogPost(0.5 * self.dt)
        st = self.lc.getParticles()
        return st["r"], st["v"]

    def run(self, r0, v0, gF, gU):
        r, v = np.array(r0), np.array(v0)
        snaps = {0: (r.copy(), v.copy())}
        for k in range(1, self.nsteps + 1):
            r, v = self._step(r, v)
            if k % self.every == 0 and k < self.nsteps:
                snaps[k] = (r.copy(), v.copy())
        ns = len(self.system.components)
        rbar, vbar, Fbar = np.zeros_like(r), np.zeros_like(r), np.array(gF, dtype=np.float64)
        ge, gs = np.zeros((ns, ns)), np.zeros((ns, ns))
        starts = sorted(snaps)
        for si in range(len(starts) - 1, -1, -1):
            k0 = starts[si]
            k1 = starts[si + 1] if si + 1 < len(starts) else self.nsteps
            pos = {k0: snaps[k0][0]}
            rr, vv = snaps[k0]
            for k in range(k0 + 1, k1 + 1):
                rr, vv = self._step(rr, vv)
                pos[k] = rr
            for k in range(k1, k0, -1):
                Fbar = Fbar + self.c * vbar
                self._forces_at(pos[k])
                a, b, d = self.lc.adjoint(Fbar, gU)
                rbar, ge, gs = rbar + a, ge + b, gs + d
                gU = 0.0
                vbar = vbar + self.dt * rbar
                Fbar = self.c * vbar
        self._forces_at(snaps[0][0])
        a, b, d = self.lc.adjoint(Fbar, gU)
        return rbar + a, vbar, ge + b, gs + d


def test_device_trajectory_adjoint_equals_the_host_driven_loop(box2048):
    s, Ft, Ut = box2048
    steps, every = 20, 6
    dev = TrajectoryAdjoint(s, steps, every)
    r, v, F, U = dev.forward(s.r, s.v)
    gF, gU = 2 * (F - Ft), 0.2 * (U - Ut)
    gr, gv, ge, gs = dev.backward(gF, gU)
    assert dev.recomputed_steps == steps
    dev.close()
    host = HostLoopTrajectoryAdjoint(s, steps, every)
    hr, hv, he, hs = host.run(s.r, s.v, gF, gU)
    host.close()
    for a, b in ((gr, hr), (gv, hv)):
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))
    np.testing.assert_allclose(ge, he, rtol=1e-12, atol=0)
    np.testing.assert_allclose(gs, hs, rtol=1e-12, atol=0)


def test_mixed_adjoint_against_fp64_and_central_differences(box2048):
    """The mixed form of the adjoint (FP32 pair derivative terms from the FP64 difference vector,
    FP64 sums) against the FP64 adjoint (rms relative 1e-5, as the mixed forces) and against FP64
    central differences of the loss in positions (1e-5 of the gradient's scale)."""
    s, Ft, Ut = box2048
    ev = Evaluator(s)
    F, U = ev(s.r)
    gF, gU = 2 * (F - Ft), 0.2 * (U - Ut)
    g64, e64, s64 = ev.lc.adjoint(gF, gU)
    m = M.LinkedCells.from_system(s, M.MIXED)
    m.update()
    m.traversePairs()
    g32, e32, s32 = m.adjoint(gF, gU)
    m.close()
    scale = np.sqrt(np.mean(g64 ** 2))
    assert np.sqrt(np.mean((g32 - g64) ** 2)) / scale <= 1e-5
    np.testing.assert_allclose(e32, e64, rtol=1e-5)
    np.testing.assert_allclose(s32, s64, rtol=1e-5)
    rng = np.random.default_rng(17)
    h = 1e-6
    for k, d in zip(rng.integers(0, s.n, 4), rng.integers(0, 3, 4)):
        rp, rm = s.r.copy(), s.r.copy()
        rp[k, d] += h
        rm[k, d] -= h
        fd = (loss(*ev(rp), Ft, Ut) - loss(*ev(rm), Ft, Ut)) / (2 * h)
        assert abs(fd - g32[k, d]) <= 1e-5 * max(abs(g64[k, d]), scale), (k, d, fd, g32[k, d])
    ev.close()


def test_adjoint_is_deterministic(box2048):
    s, Ft, Ut = box2048
    outs = []
    for _ in range(2):
        ev = Evaluator(s)
        F, U = ev(s.r)
        outs.append(ev.lc.adjoint(2 * (F - Ft), 0.2 * (U - Ut)))
        ev.close()
    for a, b in zip(outs[0], outs[1]):
        np.testing.assert_array_equal(a, b)
