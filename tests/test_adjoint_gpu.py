"""The adjoint march against central finite differences of the forward (the run has no reference counterpart:
the reference has no adjoint). The forward is the FP64 form with exact fields (the real fields kept in FP64 and
gathered by the push), so that J = mean p_z of the live beam after K s-steps is a smooth function of the laser
mode coefficients and of the beam momenta at s = 0 (start field held fixed). Central differences with a step
eps; directional derivatives along seeded random directions, and single components.

Bound: relative difference <= 1e-6 between the adjoint's directional derivative and the central difference.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = 1e-6
TOL = 1e-6


def objective(p):
    a = p["alive"] == 1
    return float(np.sum(p["w"][a] * p["pz"][a]) / np.sum(p["w"][a]))


def central(pp, pm, eps):
    """(J(+) - J(-)) / (2 eps) from the two final beams: the weighted sum of the per-particle differences, so that
    the rounding of the sum of p_z ~ gamma does not enter the difference."""
    assert np.array_equal(pp["alive"], pm["alive"])
    a = pp["alive"] == 1
    return float(np.sum(pp["w"][a] * (pp["pz"][a] - pm["pz"][a])) / np.sum(pp["w"][a]) / (2 * eps))


def forward(cfg, coef=None, dp=None, exact=True, precision="fp64"):
    from g3d import Simulation
    s = Simulation(cfg, precision=precision)
    s.load_bunch()
    s.set_laser_modes(coef)
    if exact:
        s.set_exact_fields(True)
    s.init_fields()
    if dp is not None:
        p = s.host_particles()
        p["px"] += dp[:, 0]; p["py"] += dp[:, 1]; p["pz"] += dp[:, 2]
        s.set_particles(p)
    for _ in range(cfg.steps):
        s.step()
    p = s.host_particles()
    s.close()
    return p


def adjoint(cfg, exact=True, precision="fp64"):
    from g3d import Simulation
    s = Simulation(cfg, precision=precision)
    s.load_bunch()
    s.set_laser_modes(None)
    if exact:
        s.set_exact_fields(True)
    s.init_fields()
    J, gm, gp = s.adjoint(cfg.steps)
    Jh = objective(s.host_particles())
    s.close()
    return J, gm, gp, Jh


def case():
    from g3d import configs
    return configs.adjoint_small()


def test_adjoint_objective_is_the_forward_objective():
    cfg = case()
    J, gm, gp, Jh = adjoint(cfg)
    assert abs(J - Jh) <= 1e-13 * abs(J)
    assert abs(J - objective(forward(cfg))) <= 1e-13 * abs(J)
    assert np.all(np.isfinite(gm)) and np.all(np.isfinite(gp))


def test_laser_mode_gradient_against_central_differences():
    cfg = case()
    J, gm, gp, _ = adjoint(cfg)
    rng = np.random.default_rng(11)
    H = cfg.nx // 2 + 1
    d = rng.standard_normal((cfg.ny, H)) + 1j * rng.standard_normal((cfg.ny, H))
    ad = float(np.real(np.sum(np.conj(gm) * d)))
    fd = central(forward(cfg, coef=1 + EPS * d), forward(cfg, coef=1 - EPS * d), EPS)
    print(f"J = {J:.12e}, laser modes: adjoint {ad:.12e}, central difference {fd:.12e}")
    assert abs(ad - fd) <= TOL * abs(fd), (ad, fd)
    # the largest single component, real and imaginary parts
    j, k = np.unravel_index(np.argmax(np.abs(gm)), gm.shape)
    for unit in (1.0, 1j):
        e = np.zeros((cfg.ny, H), dtype=complex)
        e[j, k] = unit
        fd1 = central(forward(cfg, coef=1 + EPS * e), forward(cfg, coef=1 - EPS * e), EPS)
        ad1 = float(np.real(np.conj(gm[j, k]) * unit))
        assert abs(ad1 - fd1) <= TOL * max(abs(fd1), 1e-3 * np.max(np.abs(gm))), (unit, ad1, fd1)


def test_momentum_gradient_against_central_differences():
    cfg = case()
    J, gm, gp, _ = adjoint(cfg)
    rng = np.random.default_rng(12)
    D = rng.standard_normal(gp.shape)
    ad = float(np.sum(gp * D))
    fd = central(forward(cfg, dp=EPS * D), forward(cfg, dp=-EPS * D), EPS)
    print(f"momenta: adjoint {ad:.12e}, central difference {fd:.12e}")
    assert abs(ad - fd) <= TOL * abs(fd), (ad, fd)


def test_workload4_gradients_against_central_differences():
    """At the size of workload 4 without its plasma (64 x 64 modes x 512 slices, 65,536 electrons, gamma 100,
    40 s-steps): the FP64 adjoint (exact fields) and the mixed adjoint (the mixed forward with the float F, the
    reverse sweep in FP64) against central differences of the FP64 forward."""
    from g3d import configs
    cfg = configs.config4()
    H = cfg.nx // 2 + 1
    d = np.random.default_rng(11).standard_normal((cfg.ny, H)) + 1j * np.random.default_rng(13).standard_normal((cfg.ny, H))
    fl = central(forward(cfg, coef=1 + EPS * d), forward(cfg, coef=1 - EPS * d), EPS)
    res = {}
    for form, kw in [("fp64", dict(exact=True)), ("mixed", dict(exact=False, precision="mixed"))]:
        J, gm, gp, _ = adjoint(cfg, **kw)
        if form == "fp64":
            D = np.random.default_rng(12).standard_normal(gp.shape)
            fm = central(forward(cfg, dp=EPS * D), forward(cfg, dp=-EPS * D), EPS)
        al, am = float(np.real(np.sum(np.conj(gm) * d))), float(np.sum(gp * D))
        res[form] = (abs(al - fl) / abs(fl), abs(am - fm) / abs(fm))
    print("workload 4 without plasma, relative differences (laser modes, momenta):", res)
    for form, (el, em) in res.items():
        assert el <= TOL and em <= TOL, (form, el, em)
