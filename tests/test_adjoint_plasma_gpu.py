"""The adjoint march with a streaming plasma (the structure of workload 4: a witness bunch inside a Gaussian grid
laser in a plasma with mobile H+ ions) against central finite differences of the forward. The reference has no
adjoint. The forward is the FP64 form with exact fields: the real fields kept in FP64 and gathered by the beam push
and, through the midpoint fields, by the streaming push, so that J = mean p_z of the live beam after K s-steps is a
smooth function of the laser mode coefficients and of the beam momenta. The plasma couples both ways: the beam's
current and the laser drive the plasma, whose current enters the fields the beam feels. The adjoint runs each
s-step again from its level checkpoint with the march recorded and transposes the march half-cell by half-cell
(passes, prediction, correction, the Boris pushes and deposits of every streaming particle).

Bound: relative difference <= 1e-6 between the adjoint's directional derivative and the central difference
(eps = 1e-6), as for the adjoint without plasma.
"""
import numpy as np
import pytest

from test_adjoint_gpu import (EPS, TOL, adjoint, autograd_inputs, central, forward, hermitian_direction, objective,
                              reference_final, reference_final_modes)

pytestmark = pytest.mark.gpu


def case(**kw):
    from g3d import configs
    return configs.adjoint_plasma_small(**kw)


def test_plasma_adjoint_objective_and_the_run_it_leaves():
    """J is the forward's J, and the run is left at s = K dz as K steps leave it (the adjoint runs the steps again
    from their levels)."""
    from g3d import Simulation
    cfg = case()
    s = Simulation(cfg)
    s.load_bunch()
    s.set_laser_modes(None)
    s.set_exact_fields(True)
    s.init_fields()
    J, gm, gp = s.adjoint(cfg.steps)
    assert s.streaming_count() > 0
    p = s.host_particles()
    F = s.array("F")
    rx = s.array("Rx")
    s.close()
    assert np.all(np.isfinite(gm)) and np.all(np.isfinite(gp))
    assert abs(J - objective(p)) <= 1e-13 * abs(J)
    # the same run without the adjoint
    s = Simulation(cfg)
    s.load_bunch()
    s.set_laser_modes(None)
    s.set_exact_fields(True)
    s.init_fields()
    for _ in range(cfg.steps):
        s.step()
    p2, F2, rx2 = s.host_particles(), s.array("F"), s.array("Rx")
    s.close()
    assert abs(J - objective(p2)) <= 1e-12 * abs(J)
    assert np.linalg.norm(F - F2) <= 1e-6 * np.linalg.norm(F2)
    assert np.linalg.norm(rx - rx2) <= 1e-10 * np.linalg.norm(rx2)


@pytest.mark.parametrize("kw", [dict(), dict(passes=1), dict(extrapolate=0, smooth=0.5), dict(ions=False, passes=3)],
                         ids=["two-passes", "one-pass", "previous-smoothed", "electrons-three-passes"])
def test_plasma_laser_mode_gradient_against_central_differences(kw):
    cfg = case(**kw)
    J, gm, gp, _ = adjoint(cfg)
    d = hermitian_direction(np.random.default_rng(31), cfg.ny, cfg.nx)
    ad = float(np.real(np.sum(np.conj(gm) * d)))
    fd = central(forward(cfg, coef=1 + EPS * d), forward(cfg, coef=1 - EPS * d), EPS)
    print(f"{kw}: J = {J:.12e}, laser modes: adjoint {ad:.12e}, central difference {fd:.12e}")
    assert abs(ad - fd) <= TOL * abs(fd), (ad, fd)


@pytest.mark.parametrize("through_start", [True, False])
def test_plasma_momentum_gradient_against_central_differences(through_start):
    cfg = case(charge_pC=1.0)
    J, gm, gp, _ = adjoint(cfg, through_start=through_start)
    D = np.random.default_rng(32).standard_normal(gp.shape)
    ad = float(np.sum(gp * D))
    fd = central(forward(cfg, dp=EPS * D, through_start=through_start),
                 forward(cfg, dp=-EPS * D, through_start=through_start), EPS)
    print(f"momenta (through the start field: {through_start}): adjoint {ad:.12e}, central difference {fd:.12e}")
    assert abs(ad - fd) <= TOL * abs(fd), (ad, fd)


@pytest.mark.parametrize("what", ["momenta", "laser modes"])
def test_plasma_gradients_against_central_differences_of_the_reference(what):
    """The plasma adjoint (FP64, exact fields) against central differences of the reference's own CPU code with its
    streaming plasma, whose real fields are rounded to float as it stores them: the float rounding puts a floor into
    its difference quotients, so the steps are those of the adjoint without plasma (3e-3 for the momenta; for the
    laser modes the Richardson extrapolation of 4e-3 and 2e-3), and this library's forward with float fields takes
    the same differences to 1e-7 (its arithmetic is the reference's; its atomic adds run in another order)."""
    cfg = case(charge_pC=1.0)
    J, gm, gp, _ = adjoint(cfg)
    if what == "momenta":
        D = np.random.default_rng(41).standard_normal(gp.shape)
        e = 3e-3
        fr = central(reference_final(cfg, e * D), reference_final(cfg, -e * D), e)
        fo = central(forward(cfg, dp=e * D, exact=False), forward(cfg, dp=-e * D, exact=False), e)
        ad = float(np.sum(gp * D))
        print(f"plasma, momenta: reference central difference {fr:.12e}, this forward's {fo:.12e}, adjoint {ad:.12e}")
        assert abs(fo - fr) <= 1e-7 * abs(fr), (fo, fr)
        assert abs(ad - fr) <= 1e-4 * abs(fr), (ad, fr)
        return
    d = hermitian_direction(np.random.default_rng(42), cfg.ny, cfg.nx)
    quot = {}
    for e in (4e-3, 2e-3):
        fr = central(reference_final_modes(cfg, 1 + e * d), reference_final_modes(cfg, 1 - e * d), e)
        fo = central(forward(cfg, coef=1 + e * d, exact=False), forward(cfg, coef=1 - e * d, exact=False), e)
        assert abs(fo - fr) <= 1e-7 * abs(fr), (e, fo, fr)
        quot[e] = fr
    rich = (4 * quot[2e-3] - quot[4e-3]) / 3
    ad = float(np.real(np.sum(np.conj(gm) * d)))
    print(f"plasma, laser modes: reference central differences {quot}, extrapolated {rich:.12e}, adjoint {ad:.12e}")
    assert abs(ad - rich) <= 5e-4 * abs(rich), (ad, rich)


@pytest.mark.parametrize("what", ["laser modes", "momenta"])
def test_plasma_gradients_with_trapped_electrons(what):
    """At a0 = 1 about 130 plasma electrons a step advance a whole step in z inside the window: the forward traps them
    (they stop inside their half-cell) and they join the next step's march at their zeta, in its partial half-cell.
    The adjoint keeps these events as the forward took them and differentiates the trapped pushes (the third Boris
    push over dtp = (s1 - z) / v_z, the stop in zeta) and the joining paths across the steps."""
    from g3d import Simulation
    cfg = case(a0=1.0, charge_pC=1.0)
    s = Simulation(cfg)
    s.load_bunch()
    s.set_exact_fields(True)
    s.init_fields()
    s.step()
    trapped = int(np.sum(s.streaming_particles()["alive"] == 5))
    s.close()
    assert trapped > 0
    J, gm, gp, _ = adjoint(cfg)
    rng = np.random.default_rng(33)
    if what == "laser modes":
        d = hermitian_direction(rng, cfg.ny, cfg.nx)
        ad = float(np.real(np.sum(np.conj(gm) * d)))
        fd = central(forward(cfg, coef=1 + EPS * d), forward(cfg, coef=1 - EPS * d), EPS)
    else:
        D = rng.standard_normal(gp.shape)
        ad = float(np.sum(gp * D))
        fd = central(forward(cfg, dp=EPS * D), forward(cfg, dp=-EPS * D), EPS)
    print(f"trapping, {what}: J = {J:.12e}, adjoint {ad:.12e}, central difference {fd:.12e}")
    assert abs(ad - fd) <= TOL * abs(fd), (ad, fd)


def test_plasma_adjoint_stored_and_recomputed_records_agree(monkeypatch):
    """The march records kept from the forward (the default when they fit) and those made by running every step again
    from its level checkpoint (G3D_ADJ_RECOMPUTE) give the same gradients, with trapped electrons joining later steps."""
    cfg = case(a0=1.0, charge_pC=1.0)
    J1, gm1, gp1, _ = adjoint(cfg)
    monkeypatch.setenv("G3D_ADJ_RECOMPUTE", "1")
    J2, gm2, gp2, _ = adjoint(cfg)
    assert J1 == J2
    assert np.linalg.norm(gm1 - gm2) <= 1e-10 * np.linalg.norm(gm1)
    assert np.linalg.norm(gp1 - gp2) <= 1e-10 * np.linalg.norm(gp1)


def test_plasma_second_evaluation_on_the_same_context():
    """g3d_set_particles + g3d_init start the next evaluation on the same context: the plasma starts afresh (no
    streaming current of a level before, no trapped electron waiting from the last run), so the second evaluation
    after a run that trapped electrons is the first one again."""
    from g3d import Simulation
    cfg = case(a0=1.0, charge_pC=1.0, steps=1)
    s = Simulation(cfg)
    s.load_bunch()
    p0 = s.host_particles()
    s.set_laser_modes(None)
    s.set_exact_fields(True)
    out = []
    for _ in range(2):
        s.set_particles(p0)
        s.init_fields()
        out.append(s.adjoint(cfg.steps))
    s.close()
    assert out[0][0] == out[1][0]
    for k in (1, 2):
        assert np.linalg.norm(out[0][k] - out[1][k]) <= 1e-12 * np.linalg.norm(out[0][k])


@pytest.mark.parametrize("a0", [0.5, 1.0], ids=["streaming", "trapping"])
def test_mixed_plasma_adjoint_against_central_differences_of_the_fp64_forward(a0):
    """The mixed form (FP32 streaming gathers and deposit, complex64 storage of E_z, B_z, L and the currents) with its
    march records widened and the reverse sweep in FP64: it linearises the mixed forward, whose fields differ from the
    FP64 form's by the FP32 rounding; against the FP64 forward's central differences it is held to the 1e-6 of the FP64
    adjoint (measured 2e-9 ... 6e-9)."""
    cfg = case(a0=a0, charge_pC=1.0)
    J, gm, gp, _ = adjoint(cfg, exact=False, precision="mixed")
    rng = np.random.default_rng(34)
    d = hermitian_direction(rng, cfg.ny, cfg.nx)
    D = rng.standard_normal(gp.shape)
    fl = central(forward(cfg, coef=1 + EPS * d), forward(cfg, coef=1 - EPS * d), EPS)
    fm = central(forward(cfg, dp=EPS * D), forward(cfg, dp=-EPS * D), EPS)
    al, am = float(np.real(np.sum(np.conj(gm) * d))), float(np.sum(gp * D))
    print(f"mixed, a0 {a0}: laser modes {abs(al - fl) / abs(fl):.3e}, momenta {abs(am - fm) / abs(fm):.3e}")
    assert abs(al - fl) <= TOL * abs(fl), (al, fl)
    assert abs(am - fm) <= TOL * abs(fm), (am, fm)


def test_autograd_gradcheck_with_trapped_electrons():
    """torch.autograd.gradcheck through g3d.autograd.MarchObjective on the plasma case with trapping (fast mode: per
    input one random direction, central difference at eps = 1e-6 against the adjoint's vector-Jacobian product,
    relative tolerance 1e-6, no absolute tolerance)."""
    import torch
    from g3d.autograd import MarchObjective
    cfg = case(a0=1.0, charge_pC=1.0)
    coef, dp = autograd_inputs(cfg)
    j0 = MarchObjective.apply(coef, dp, cfg, "fp64", True, True).item()

    def fn(c, d):
        return MarchObjective.apply(c, d, cfg, "fp64", True, True, j0)
    assert torch.autograd.gradcheck(fn, (coef, dp), eps=EPS, atol=0.0, rtol=TOL, fast_mode=True)


def test_plasma_adjoint_refuses_what_it_does_not_differentiate():
    """Ionization and the FP64 form without exact fields are refused with G3D_ERR_ARG before anything runs."""
    from g3d import G3DError, Simulation, configs
    cfg = case()
    s = Simulation(cfg)
    s.load_bunch()
    s.set_laser_modes(None)
    s.init_fields()
    with pytest.raises(G3DError):
        s.adjoint(cfg.steps)
    s.close()
    ion = configs.ionization_small()
    ion.params.update(sponge=0.0, sponge_y=0.0)
    s = Simulation(ion)
    s.set_laser_modes(None)
    s.set_exact_fields(True)
    s.init_fields()
    with pytest.raises(G3DError):
        s.adjoint(1, momenta=False)
    s.close()
