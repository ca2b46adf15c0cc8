"""Adjoint of mean drag: gradient w.r.t. a per-node body force and the inlet profile, checked
against central finite differences of the FP64 forward run, plus the body-force forward term
and the torch.autograd bridge."""
import numpy as np
import pytest

from cases import CASES
from mrlbm_2d_b200.config import WALL_REFERENCE, cylinder_case

pytestmark = pytest.mark.gpu


def _case():
    # 96 x 32 channel, D = 8 at (24, 16.5): curved wall with label-15 poles, free-slip walls
    return cylinder_case(96, 32, 8, 24.0, 16.5, 100.0, 0.05, seed=11, noise=1e-2)


def _params(sim, seed):
    rng = np.random.default_rng(seed)
    body = 1e-5 * rng.standard_normal((2, sim.nx, sim.ny))
    uin = 0.05 + 1e-3 * rng.standard_normal(sim.ny)
    return body, uin


def test_body_force_adds_its_momentum(mrlbm):
    """A uniform body force g adds g per node and step to the momentum (the run without the
    force is subtracted; the reference's periodic corner wraps duplicate a few populations, so
    the balance holds to 1e-3) and leaves the mass unchanged."""
    cfg = CASES["periodic_channel_no_cylinder"]()
    ex = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1])
    ey = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1])
    out = []
    for force in (False, True):
        s = mrlbm.Simulation(cfg)
        if force:
            g = np.zeros((2, s.nx, s.ny))
            g[0] = 2e-6
            g[1] = -1e-6
            s.set_body_force(g)
        s.step(10)
        f = s.get_state()
        out.append(((f * ex).sum(), (f * ey).sum(), f.sum()))
        nodes = s.nx * s.ny
        s.close()
    for c, gc in ((0, 2e-6), (1, -1e-6)):
        dm = out[1][c] - out[0][c]
        assert abs(dm - 10 * gc * nodes) < 1e-3 * abs(10 * gc * nodes)
    assert abs(out[1][2] - out[0][2]) < 1e-10 * out[0][2]


def test_adjoint_objective_is_the_forward_mean_drag(mrlbm):
    s = mrlbm.Simulation(_case())
    body, uin = _params(s, 1)
    s.set_body_force(body)
    s.set_inlet_profile(uin)
    J = s.adjoint_drag(120, 50, 40, grads=False)
    assert s.iter == 1                               # the handle is not advanced
    s.step(120)
    it, fd, fl, _ = s.forces()
    acc = 0.0
    for v in fd[-50:]:
        acc = acc + v
    assert J == acc / 50
    s.close()


@pytest.mark.parametrize("K", [37, 1000])
def test_adjoint_matches_central_differences(mrlbm, K):
    s = mrlbm.Simulation(_case())
    body, uin = _params(s, 2)
    s.set_body_force(body)
    s.set_inlet_profile(uin)
    N, T = 200, 80
    J, gb, gu = s.adjoint_drag(N, T, K)
    assert np.all(np.isfinite(gb)) and np.all(np.isfinite(gu))
    rng = np.random.default_rng(5)
    for _ in range(4):
        db = 1e-5 * rng.standard_normal(body.shape)
        du = 1e-3 * rng.standard_normal(uin.shape)
        eps = 1e-4
        vals = []
        for sgn in (1.0, -1.0):
            s.set_body_force(body + sgn * eps * db)
            s.set_inlet_profile(uin + sgn * eps * du)
            vals.append(s.adjoint_drag(N, T, K, grads=False))
        fd = (vals[0] - vals[1]) / (2 * eps)
        ad = float((gb * db).sum() + (gu * du).sum())
        assert abs(ad - fd) <= 1e-3 * abs(fd) + 1e-15, (ad, fd)
        # each block separately too
        for part in ("body", "inlet"):
            vals = []
            for sgn in (1.0, -1.0):
                s.set_body_force(body + (sgn * eps * db if part == "body" else 0.0))
                s.set_inlet_profile(uin + (sgn * eps * du if part == "inlet" else 0.0))
                vals.append(s.adjoint_drag(N, T, K, grads=False))
            fdp = (vals[0] - vals[1]) / (2 * eps)
            adp = float((gb * db).sum()) if part == "body" else float((gu * du).sum())
            assert abs(adp - fdp) <= 1e-3 * abs(fdp) + 1e-15, (part, adp, fdp)
    s.set_body_force(body)
    s.set_inlet_profile(uin)
    s.close()


def test_checkpoint_interval_does_not_change_the_gradient(mrlbm):
    s = mrlbm.Simulation(_case())
    body, uin = _params(s, 3)
    s.set_body_force(body)
    s.set_inlet_profile(uin)
    J1, gb1, gu1 = s.adjoint_drag(150, 60, 7)
    J2, gb2, gu2 = s.adjoint_drag(150, 60, 150)
    assert J1 == J2
    assert np.abs(gb1 - gb2).max() <= 1e-10 * np.abs(gb1).max()
    assert np.abs(gu1 - gu2).max() <= 1e-10 * np.abs(gu1).max()
    s.close()


def test_torch_autograd_bridge(mrlbm):
    torch = pytest.importorskip("torch")
    from mrlbm_2d_b200.autograd import mean_drag
    s = mrlbm.Simulation(_case())
    body, uin = _params(s, 4)
    b = torch.tensor(body, requires_grad=True)
    u = torch.tensor(uin, requires_grad=True)
    J = mean_drag(s, b, u, 100, 40, 25)
    (2.0 * J).backward()
    J0, gb, gu = s.adjoint_drag(100, 40, 25)
    assert float(J.detach()) == J0
    assert np.allclose(b.grad.numpy(), 2.0 * gb, rtol=1e-10, atol=1e-14 * np.abs(gb).max())
    assert np.allclose(u.grad.numpy(), 2.0 * gu, rtol=1e-10, atol=1e-14 * np.abs(gu).max())
    s.close()


@pytest.mark.parametrize("kw", [dict(), dict(strong_mass_bc=0, weak_mass_bc=1), dict(rotated_coordinate=0)])
def test_fp32_adjoint_tracks_fp64_adjoint(mrlbm, kw):
    """FP32 trajectory with FP64 adjoint arithmetic against the FP64 adjoint: the directional
    derivatives agree to 1e-3 relative (default, weak and unrotated curved-wall closures)."""
    out = {}
    for prec in (64, 32):
        s = mrlbm.Simulation(_case().replace(**kw), precision=prec)
        body, uin = _params(s, 6)
        s.set_body_force(body)
        s.set_inlet_profile(uin)
        out[prec] = s.adjoint_drag(200, 80, 37)
        s.close()
    rng = np.random.default_rng(9)
    assert abs(out[32][0] - out[64][0]) <= 1e-4 * abs(out[64][0])
    for _ in range(4):
        db = rng.standard_normal(out[64][1].shape)
        du = rng.standard_normal(out[64][2].shape)
        d64 = float((out[64][1] * db).sum() + (out[64][2] * du).sum())
        d32 = float((out[32][1] * db).sum() + (out[32][2] * du).sum())
        assert abs(d32 - d64) <= 1e-3 * abs(d64), (d32, d64)


def test_adjoint_rejects_unsupported_cases(mrlbm):
    """x-periodic lattices have no inlet or outlet to differentiate through."""
    s = mrlbm.Simulation(CASES["freeslip_xperiodic"]())
    with pytest.raises(mrlbm.MrlbmError):
        s.adjoint_drag(10, 5, 5)
    s.close()


def test_adjoint_y_periodic_case_matches_central_differences(mrlbm):
    """Top and bottom y-periodic instead of free-slip (another streaming map for the edge
    rows), inlet-profile direction only."""
    cfg = cylinder_case(96, 40, 8, 24.0, 20.5, 100.0, 0.05, seed=13, noise=1e-2).replace(y_periodic=1)
    s = mrlbm.Simulation(cfg)
    _, uin = _params(s, 8)
    s.set_inlet_profile(uin)
    N, T, K = 150, 60, 50
    J, gb, gu = s.adjoint_drag(N, T, K)
    du = 1e-3 * np.random.default_rng(3).standard_normal(uin.shape)
    eps = 1e-4
    vals = []
    for sgn in (1.0, -1.0):
        s.set_inlet_profile(uin + sgn * eps * du)
        vals.append(s.adjoint_drag(N, T, K, grads=False))
    fd = (vals[0] - vals[1]) / (2 * eps)
    ad = float((gu * du).sum())
    assert abs(ad - fd) <= 1e-3 * abs(fd), (ad, fd)
    s.close()


@pytest.mark.parametrize("kw", [dict(wall_mode=WALL_REFERENCE), dict(incomp_bc=1, incomp_bulk=1),
                                dict(wall_mode=WALL_REFERENCE, incomp_bc=1, incomp_bulk=1),
                                dict(strong_mass_bc=0, weak_mass_bc=1), dict(strong_mass_bc=0, eq_mass_bc=1),
                                dict(rotated_coordinate=0), dict(vel_interp=0), dict(strong_mass_bc=0)])
def test_adjoint_wall_and_closure_variants_match_central_differences(mrlbm, kw):
    """No-slip reference walls (apply_bc wall rows, 2d_mrlbm.f90:1327-1359, their closure
    winning at the corners), the incompressible edge closures and bulk collision
    (apply_bc_incomp, 2d_mrlbm.f90:1368-1494; 419-428), and the curved-wall closure variants
    (weak 1767-1871, rho_eq 1873-1972, unrotated with Cramer's rule 1496-1633 and 1974-2003, no
    velocity extrapolation, no mass closure): both parameter blocks against central
    differences."""
    s = mrlbm.Simulation(_case().replace(**kw))
    body, uin = _params(s, 12)
    s.set_body_force(body)
    s.set_inlet_profile(uin)
    N, T, K = 150, 60, 50
    J, gb, gu = s.adjoint_drag(N, T, K)
    assert np.all(np.isfinite(gb)) and np.all(np.isfinite(gu))
    rng = np.random.default_rng(21)
    eps = 1e-4
    for _ in range(2):
        db = 1e-5 * rng.standard_normal(body.shape)
        du = 1e-3 * rng.standard_normal(uin.shape)
        vals = []
        for sgn in (1.0, -1.0):
            s.set_body_force(body + sgn * eps * db)
            s.set_inlet_profile(uin + sgn * eps * du)
            vals.append(s.adjoint_drag(N, T, K, grads=False))
        fd = (vals[0] - vals[1]) / (2 * eps)
        ad = float((gb * db).sum() + (gu * du).sum())
        assert abs(ad - fd) <= 1e-3 * abs(fd) + 1e-15, (ad, fd)
    s.close()
