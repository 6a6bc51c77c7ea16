"""The adjoint march against central finite differences of the forward (the run has no reference counterpart:
the reference has no adjoint). The forward is the FP64 form with exact fields (the real fields kept in FP64 and
gathered by the push), so that J = mean p_z of the live beam after K s-steps is a smooth function of the laser
mode coefficients and of the beam momenta at s = 0: as loaded, before the start field which the bunch's currents
and beta make (G3D_ADJ_THROUGH_START), or right after init with that start field held (G3D_ADJ_AFTER_START).
Central differences with a step eps; directional derivatives along seeded random directions, and single
components.

Bound: relative difference <= 1e-6 between the adjoint's directional derivative and the central difference.

The step is eps = 1e-6, except for the momenta before the start field at the size of workload 4. There the
bunch's beta (gamma 100) is, bit for bit as in the reference, the sequential sum of w p_z / gamma over 65,536
particles divided by the sum of w: terms near 1 whose sum carries a rounding error of ~1e-14 that changes
erratically with the momenta, while a step of 1e-6 along a random direction moves beta by ~1e-14 too, and J
depends on beta through gamma^-2 = 1 - beta^2 of the co-moving field. The difference quotient then carries noise
~ dJ/dbeta x 1e-14 / 2e-6, about 1e-5 of the derivative, which falls as 1/eps (measured on 20 s-steps:
1.5e-7, 1.2e-8, 2e-9 and 3e-11 absolute at eps = 1e-7, 1e-6, 1e-5 and 1e-4, the derivative being 1.6e-3).
eps = 1e-4 takes it below 1e-7 relative; the step's own truncation error (eps^2 times the third derivative) stays
below that.
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


def forward(cfg, coef=None, dp=None, exact=True, precision="fp64", through_start=True):
    """The final beam; dp added to the momenta as loaded (through_start) or right after init."""
    from g3d import Simulation
    s = Simulation(cfg, precision=precision)
    s.load_bunch()

    def perturb():
        p = s.host_particles()
        p["px"] += dp[:, 0]; p["py"] += dp[:, 1]; p["pz"] += dp[:, 2]
        s.set_particles(p)
    if dp is not None and through_start:
        perturb()
    s.set_laser_modes(coef)
    if exact:
        s.set_exact_fields(True)
    s.init_fields()
    if dp is not None and not through_start:
        perturb()
    for _ in range(cfg.steps):
        s.step()
    p = s.host_particles()
    s.close()
    return p


def adjoint(cfg, exact=True, precision="fp64", through_start=True):
    from g3d import Simulation
    s = Simulation(cfg, precision=precision)
    s.load_bunch()
    s.set_laser_modes(None)
    if exact:
        s.set_exact_fields(True)
    s.init_fields()
    J, gm, gp = s.adjoint(cfg.steps, through_start=through_start)
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


@pytest.mark.parametrize("through_start", [True, False])
def test_momentum_gradient_against_central_differences(through_start):
    cfg = case()
    J, gm, gp, _ = adjoint(cfg, through_start=through_start)
    rng = np.random.default_rng(12)
    D = rng.standard_normal(gp.shape)
    ad = float(np.sum(gp * D))
    fd = central(forward(cfg, dp=EPS * D, through_start=through_start),
                 forward(cfg, dp=-EPS * D, through_start=through_start), EPS)
    print(f"momenta (through the start field: {through_start}): adjoint {ad:.12e}, central difference {fd:.12e}")
    assert abs(ad - fd) <= TOL * abs(fd), (ad, fd)


def test_start_field_part_of_the_momentum_gradient():
    """The difference of the two momentum gradients is the start field's part (its currents, its beta, the
    relaxation marches, init's march(0)): against the difference of the two central differences, per momentum
    component, with a self field 100 times the test case's (1 pC)."""
    from g3d import configs
    cfg = configs.adjoint_small(charge_pC=1.0)
    _, _, g1, _ = adjoint(cfg, through_start=True)
    _, _, g0, _ = adjoint(cfg, through_start=False)
    R = np.random.default_rng(12).standard_normal(g1.shape)
    for k in range(3):
        D = np.zeros_like(R)
        D[:, k] = R[:, k]
        f1 = central(forward(cfg, dp=EPS * D), forward(cfg, dp=-EPS * D), EPS)
        f0 = central(forward(cfg, dp=EPS * D, through_start=False), forward(cfg, dp=-EPS * D, through_start=False), EPS)
        part_ad, part_fd = float(np.sum((g1 - g0) * D)), f1 - f0
        print(f"component {k}: start field part, adjoint {part_ad:.9e}, central differences {part_fd:.9e}")
        assert abs(part_ad - part_fd) <= 1e-4 * abs(part_fd) + TOL * abs(f1), (k, part_ad, part_fd)


def reference_final(cfg, dp):
    """The final beam of the reference CPU code (oracle/_ref) with dp added to the momenta as loaded."""
    ref = pytest.importorskip("ref")
    if not ref.available():
        pytest.skip("reference build oracle/_ref not present")
    r = ref.RefSimulation(cfg, threads=8)
    try:
        r.load_bunch()
        p = r.host_particles()
        p["px"] += dp[:, 0]; p["py"] += dp[:, 1]; p["pz"] += dp[:, 2]
        r.set_particles(p)
        r.init_fields()
        for _ in range(cfg.steps):
            r.step()
        return r.host_particles()
    finally:
        r.close()


@pytest.mark.parametrize("charge_pC", [0.01, 1.0])
def test_momentum_gradient_against_central_differences_of_the_reference(charge_pC):
    """Central differences of the reference's own CPU code (its FP64 arithmetic, its real fields rounded to float as
    it stores them) against the adjoint of the same forward (float F, the rounding linearised as the identity).
    The float F puts a rounding floor into the reference's difference quotient (~1e-4 at eps = 1e-6, falling with
    eps), so eps = 3e-3, where the floor is below 1e-5 and the truncation error too. The forward here takes the same
    difference to 1e-9: it is the reference's arithmetic."""
    from g3d import configs
    cfg = configs.adjoint_small(charge_pC=charge_pC)
    _, _, gf, _ = adjoint(cfg, exact=False)
    D = np.random.default_rng(12).standard_normal(gf.shape)
    e = 3e-3
    fr = central(reference_final(cfg, e * D), reference_final(cfg, -e * D), e)
    fo = central(forward(cfg, dp=e * D, exact=False), forward(cfg, dp=-e * D, exact=False), e)
    ad = float(np.sum(gf * D))
    print(f"momenta, {charge_pC} pC: reference central difference {fr:.12e}, this forward's {fo:.12e}, adjoint {ad:.12e}")
    assert abs(fo - fr) <= 1e-9 * abs(fr), (fo, fr)
    assert abs(ad - fr) <= 1e-5 * abs(fr), (ad, fr)


def hermitian_direction(rng, ny, nx):
    """A random direction over the stored modes [j][k_x], k_x = 0 .. nx/2, that keeps a real field real: on the
    columns k_x = 0 and k_x = nx/2, whose modes j and -j are both stored, d(-j) = conj d(j) (real at j = 0, ny/2)."""
    H = nx // 2 + 1
    d = rng.standard_normal((ny, H)) + 1j * rng.standard_normal((ny, H))
    for c in (0, H - 1):
        for j in range(ny // 2 + 1):
            m = (-j) % ny
            if m == j:
                d[j, c] = d[j, c].real
            else:
                d[m, c] = np.conj(d[j, c])
    return d


def full_coefficients(a_half, nx):
    """The stored half [j][k_x <= nx/2] of the mode coefficients as a full [j][ix] array: conj a(-j, nx - ix) on the
    other half, as the library's Hermitian storage implies."""
    ny, H = a_half.shape
    full = np.empty((ny, nx), dtype=np.complex128)
    full[:, :H] = a_half
    for ix in range(H, nx):
        full[:, ix] = np.conj(a_half[(-np.arange(ny)) % ny, nx - ix])
    return full


def reference_final_modes(cfg, a_half):
    """The final beam of the reference CPU code with every grid laser's spectrum multiplied by the coefficients a:
    the reference's init, then its last stages after the lasers are added replayed from R + (a - 1) s, s the laser
    spectrum added at init (R of an init with the lasers minus R of one without them). Those stages, march(0) and
    sponge_and_real_fields without a sponge, take R as it is, and j0 = jk then, so the replay is the reference's
    init with a (a patch of the reference's add_grid_lasers would give the same)."""
    import copy
    ref = pytest.importorskip("ref")
    if not ref.available():
        pytest.skip("reference build oracle/_ref not present")
    assert cfg.params.get("sponge", 0) == 0
    bare = copy.deepcopy(cfg)
    bare.glasers = []
    r0 = ref.RefSimulation(bare, threads=8)
    r0.init()
    R0 = {k: r0.array(k) for k in ("Rx", "Ry")}
    r0.close()
    r = ref.RefSimulation(cfg, threads=8)
    try:
        r.init()
        A = np.tile(full_coefficients(a_half, cfg.nx).ravel(), cfg.nzeta)
        for k in ("Rx", "Ry"):
            R = r.array(k)
            r.set_array(k, R + (A - 1) * (R - R0[k]))
        r.march(0.0)
        r.sponge_and_real_fields()
        for _ in range(cfg.steps):
            r.step()
        return r.host_particles()
    finally:
        r.close()


def test_laser_mode_gradient_against_central_differences_of_the_reference():
    """dJ/da along a random direction against central differences of the reference's own CPU code, and this
    library's forward taking the same differences to 1e-9 (measured 1e-12: they are the reference's arithmetic).
    The reference keeps the real fields in float, and their rounding reaches J: its difference quotients for the laser
    modes scatter by ~1e-4 relative at steps of 1e-3 (measured: 1.00907e-3 and 1.00916e-3 at eps = 4e-3 and 2e-3),
    more than their truncation error, so the adjoint is held to 5e-4 of their Richardson extrapolation
    (4 D(eps/2) - D(eps)) / 3 here; the same adjoint matches the central differences of the forward with FP64 real
    fields to 1e-6 (test_laser_mode_gradient_against_central_differences)."""
    from g3d import configs
    cfg = configs.adjoint_small(charge_pC=1.0)
    _, gm, _, _ = adjoint(cfg, exact=False)
    d = hermitian_direction(np.random.default_rng(21), cfg.ny, cfg.nx)
    quot = {}
    for e in (4e-3, 2e-3):
        fr = central(reference_final_modes(cfg, 1 + e * d), reference_final_modes(cfg, 1 - e * d), e)
        fo = central(forward(cfg, coef=1 + e * d, exact=False), forward(cfg, coef=1 - e * d, exact=False), e)
        assert abs(fo - fr) <= 1e-9 * abs(fr), (e, fo, fr)
        quot[e] = fr
    rich = (4 * quot[2e-3] - quot[4e-3]) / 3
    ad = float(np.real(np.sum(np.conj(gm) * d)))
    print(f"laser modes: reference central differences {quot}, extrapolated {rich:.12e}, adjoint {ad:.12e}")
    assert abs(ad - rich) <= 5e-4 * abs(rich), (ad, rich)


def autograd_inputs(cfg):
    import torch
    from g3d.sim import sample_bunches
    n = len(sample_bunches(cfg)[0])
    coef = torch.zeros(cfg.ny, cfg.nx // 2 + 1, 2, dtype=torch.float64)
    coef[..., 0] = 1
    return coef.requires_grad_(), torch.zeros(n, 3, dtype=torch.float64, requires_grad=True)


def test_autograd_function_backward_is_the_adjoint():
    from g3d.autograd import MarchObjective
    cfg = case()
    coef, dp = autograd_inputs(cfg)
    J, gm, gp, _ = adjoint(cfg)
    out = MarchObjective.apply(coef, dp, cfg)
    assert abs(out.item() - J) <= 1e-13 * abs(J)
    (2.0 * out).backward()
    # two runs: the gradients differ in the order of their atomic adds only
    scale_m, scale_p = np.max(np.abs(gm)), np.max(np.abs(gp))
    assert np.allclose(coef.grad[..., 0].numpy(), 2 * gm.real, rtol=1e-9, atol=1e-12 * scale_m)
    assert np.allclose(coef.grad[..., 1].numpy(), 2 * gm.imag, rtol=1e-9, atol=1e-12 * scale_m)
    assert np.allclose(dp.grad.numpy(), 2 * gp, rtol=1e-9, atol=1e-12 * scale_p)


@pytest.mark.parametrize("through_start", [True, False])
def test_autograd_function_passes_gradcheck(through_start):
    """torch.autograd.gradcheck through g3d.autograd.MarchObjective, fast mode (per input one random unit
    direction u: the central difference of the forward with step eps along u against the adjoint's
    vector-Jacobian product along u), eps = 1e-6, relative tolerance 1e-6, no absolute tolerance."""
    import torch
    from g3d.autograd import MarchObjective
    cfg = case()
    coef, dp = autograd_inputs(cfg)
    j0 = MarchObjective.apply(coef, dp, cfg, "fp64", True, through_start).item()

    def fn(c, d):
        return MarchObjective.apply(c, d, cfg, "fp64", True, through_start, j0)
    assert torch.autograd.gradcheck(fn, (coef, dp), eps=EPS, atol=0.0, rtol=TOL, fast_mode=True)


def test_adjoint_momentum_mode_is_checked():
    from g3d import Simulation
    from g3d.sim import G3DError
    s = Simulation(case())
    try:
        with pytest.raises(G3DError):
            s._c(s.lib.g3d_set_adjoint_momenta(s.ctx, 2))
    finally:
        s.close()


def test_workload4_gradients_against_central_differences():
    """At the size of workload 4 without its plasma (64 x 64 modes x 512 slices, 65,536 electrons, gamma 100,
    40 s-steps): the FP64 adjoint (exact fields) and the mixed adjoint (the mixed forward with the float F, the
    reverse sweep in FP64) against central differences of the FP64 forward: the laser modes and the momenta
    after the start field with eps = 1e-6, the momenta before it with eps = 1e-4 (the module's note)."""
    from g3d import configs
    cfg = configs.config4()
    H = cfg.nx // 2 + 1
    d = np.random.default_rng(11).standard_normal((cfg.ny, H)) + 1j * np.random.default_rng(13).standard_normal((cfg.ny, H))
    fl = central(forward(cfg, coef=1 + EPS * d), forward(cfg, coef=1 - EPS * d), EPS)
    D = np.random.default_rng(12).standard_normal((cfg.bunches[0]["nmacro"], 3))
    fa = central(forward(cfg, dp=EPS * D, through_start=False), forward(cfg, dp=-EPS * D, through_start=False), EPS)
    E4 = 1e-4
    fb = central(forward(cfg, dp=E4 * D), forward(cfg, dp=-E4 * D), E4)
    res = {}
    for form, kw in [("fp64", dict(exact=True)), ("mixed", dict(exact=False, precision="mixed"))]:
        _, gm, gb, _ = adjoint(cfg, **kw)
        _, _, ga, _ = adjoint(cfg, through_start=False, **kw)
        assert gb.shape == D.shape
        al, ab, aa = float(np.real(np.sum(np.conj(gm) * d))), float(np.sum(gb * D)), float(np.sum(ga * D))
        res[form] = (abs(al - fl) / abs(fl), abs(aa - fa) / abs(fa), abs(ab - fb) / abs(fb))
    print("workload 4 without plasma, relative differences (laser modes, momenta after / before the start field):", res)
    for form, errs in res.items():
        assert max(errs) <= TOL, (form, errs)
