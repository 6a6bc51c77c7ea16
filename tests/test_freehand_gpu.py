"""Parity of the march on the free-hand y grid (a graded table of nodes between conducting walls) with the reference
GEM-PIC-3D FP64 CPU path: stage by stage (currents with the filters along y, the march with the tridiagonal solves
along y, the sponge with the bound field from the LU factors, the real fields, the co-moving start field from the
eigenvectors of the y Laplacian, the push with the half-node gather and the walls) and a run of init + 2 s-steps.

Tolerances as in test_parity_gpu.py: spectra <= 1e-10 relative L2 against the field state norm (stages: 1e-12),
particles <= 1e-10, float F <= 1e-6.
"""
import numpy as np
import pytest

from conftest import CURRENTS, FIELDS, assert_state, rel_l2

pytestmark = pytest.mark.gpu
ref = pytest.importorskip("ref")
needs_ref = pytest.mark.skipif(not ref.available(), reason="reference build oracle/_ref not present")


def pair(cfg):
    from g3d import Simulation
    r = ref.RefSimulation(cfg, threads=1)
    r.load_bunch()
    s = Simulation(cfg)
    s.load_bunch()
    return s, r


def case(**kw):
    from g3d import configs
    return configs.freehand_small(**kw)


@needs_ref
def test_bunch_on_the_free_hand_grid_is_the_reference_bunch():
    s, r = pair(case())
    p, q = s.host_particles(), r.host_particles()
    assert len(p) == len(q)
    for f in p.dtype.names:
        assert np.array_equal(p[f], q[f]), f
    assert s.status().Y0 == r.status().Y0 == 0.0


@needs_ref
@pytest.mark.parametrize("kf", [1, 0])
def test_currents_stage(kf):
    s, r = pair(case(k_filter=kf))
    s.currents(); r.currents()
    assert rel_l2(s.array("jw"), r.array("jw")) <= 1e-13
    for a in CURRENTS:
        assert rel_l2(s.array(a), r.array(a)) <= 1e-12, a


@needs_ref
def test_comoving_and_relax_stage():
    s, r = pair(case())
    s.currents(); r.currents()
    s.comoving_field(); r.comoving_field()
    assert s.status().beta_b == r.status().beta_b
    for a in ["Rx", "Ry"]:
        assert rel_l2(s.array(a), r.array(a)) <= 1e-12, a
    s.relax_start_field(); r.relax_start_field()
    assert_state({a: s.array(a) for a in FIELDS}, {a: r.array(a) for a in FIELDS}, FIELDS, 1e-11)


@needs_ref
@pytest.mark.parametrize("D", [0.0, 1.5, 300.0])
def test_march_stage(D):
    s, r = pair(case())
    r.init_fields(); r.currents()
    for a in FIELDS + ["j0x", "j0y"] + CURRENTS:
        s.set_array(a, r.array(a))
    s.march(D); r.march(D)
    assert_state({a: s.array(a) for a in FIELDS}, {a: r.array(a) for a in FIELDS}, FIELDS, 1e-12)


@needs_ref
def test_sponge_and_real_fields_stage():
    s, r = pair(case())
    r.init_fields(); r.currents(); r.march(1.5)
    s.currents(); s.comoving_field()             # beta of the bunch, as the reference took it in init
    for a in FIELDS + ["jkz"]:
        s.set_array(a, r.array(a))
    s.sponge_and_real_fields(); r.sponge_and_real_fields()
    for a in ["Rx", "Ry"]:
        assert rel_l2(s.array(a), r.array(a)) <= 1e-12, a
    assert rel_l2(s.array("F"), r.array("F")) <= 1e-6


@needs_ref
def test_push_stage():
    cfg = case()
    s, r = pair(cfg)
    r.init_fields()
    s.set_array("F", r.array("F"))
    dz = cfg.params["dz"]
    s.push(0.0, dz); r.push(0.0, dz)
    p, q = s.host_particles(), r.host_particles()
    assert np.array_equal(p["alive"], q["alive"])
    for f in ["x", "y", "zeta", "px", "py", "pz", "z"]:
        assert rel_l2(p[f], q[f]) <= 1e-12, f


@needs_ref
@pytest.mark.parametrize("sponge", [1.5, 0.0])
def test_run_matches_reference(sponge):
    from g3d import Simulation
    cfg = case(sponge=sponge)
    r = ref.RefSimulation(cfg, threads=1)
    r.init()
    s = Simulation(cfg)
    s.init()
    for tag in ["init", "step1", "step2"]:
        if tag != "init":
            s.step(); r.step()
        assert_state({a: s.array(a) for a in FIELDS}, {a: r.array(a) for a in FIELDS}, FIELDS, 1e-10, tag=tag)
        assert_state({a: s.array(a) for a in CURRENTS}, {a: r.array(a) for a in CURRENTS}, CURRENTS, 1e-10, tag=tag)
        assert rel_l2(s.array("F"), r.array("F")) <= 1e-6, tag
        p, q = s.host_particles(), r.host_particles()
        assert np.array_equal(p["alive"], q["alive"]), tag
        for f in ["x", "y", "zeta", "px", "py", "pz"]:
            assert rel_l2(p[f], q[f]) <= 1e-10, (tag, f)
    d, dr = s.diagnostics_sums(), r.diagnostics_sums()
    assert np.allclose(d, dr, rtol=1e-9, atol=1e-300)


def compare_plasma_state(s, r, tol, tag):
    assert_state({a: s.array(a) for a in FIELDS}, {a: r.array(a) for a in FIELDS}, FIELDS, tol, comp_tol=1e-5, tag=tag)
    assert_state({a: s.array(a) for a in CURRENTS}, {a: r.array(a) for a in CURRENTS}, CURRENTS, tol, comp_tol=1e-5, tag=tag)
    assert rel_l2(s.array("F"), r.array("F")) <= 1e-6, tag


@needs_ref
@pytest.mark.parametrize("ions,extrap,passes,smooth", [(True, 1, 2, 0.0), (False, 0, 1, 0.0), (True, 1, 2, 0.4)])
def test_plasma_run_matches_reference(ions, extrap, passes, smooth):
    """The streaming-plasma march on the free-hand y grid: a grid laser on the nodes and half-nodes, the plasma
    lattice between the wall cells, the half-node deposit and gather of the streaming particles, the filters and
    the smoothing along y, the march of one slice by the solves along y, and the walls."""
    from g3d import Simulation, configs
    cfg = configs.on_freehand_y(configs.lwfa_small(ions=ions, extrapolate=extrap, passes=passes, smooth=smooth))
    r = ref.RefSimulation(cfg, threads=1)
    r.init()
    s = Simulation(cfg)
    s.init()
    compare_plasma_state(s, r, 1e-10, "init")
    for k in range(2):
        s.step(); r.step()
        compare_plasma_state(s, r, 1e-10, f"step{k + 1}")
        ps, pr = s.streaming_particles(), r.streaming_particles()
        assert len(ps) == len(pr)
        assert np.array_equal(ps["alive"], pr["alive"])
        for f in ["x", "y", "zeta", "px", "py", "pz", "z"]:
            assert rel_l2(ps[f], pr[f]) <= 1e-9, (k, f, rel_l2(ps[f], pr[f]))
        bs, br = s.host_particles(), r.host_particles()
        assert np.array_equal(bs["alive"], br["alive"])
        for f in ["x", "y", "zeta", "px", "py", "pz"]:
            assert rel_l2(bs[f], br[f]) <= 1e-10, (k, f)
    assert s.status().np == r.status().np


@needs_ref
def test_plasma_walls_take_the_particles_that_reach_them():
    """A narrow free-hand grid (walls at about +-4.6) with a strong driver: streaming electrons reach the wall
    cells and leave the march, as in the reference."""
    from g3d import Simulation, configs
    cfg = configs.on_freehand_y(configs.lwfa_small(a0=3.0, n0=0.02, ions=False, passes=1, extrapolate=0),
                                half=8, dy0=0.5, grow=1.1, core=2.0)
    r = ref.RefSimulation(cfg, threads=1)
    r.init()
    s = Simulation(cfg)
    s.init()
    for k in range(2):
        s.step(); r.step()
        compare_plasma_state(s, r, 1e-9, f"step{k + 1}")
    assert s.status().np == r.status().np
    assert s.status().lost == r.status().lost


@needs_ref
def test_ionization_on_the_free_hand_grid():
    from g3d import configs
    cfg = configs.on_freehand_y(configs.ionization_small())
    r = ref.RefSimulation(cfg, threads=1)
    r.init()
    from g3d import Simulation
    s = Simulation(cfg)
    s.init()
    for k in range(2):
        s.step(); r.step()
        ps, pr = sort_by_id(s.streaming_particles()), sort_by_id(r.streaming_particles())
        assert len(ps) == len(pr), (len(ps), len(pr))
        assert np.array_equal(ps["id"], pr["id"]) and np.array_equal(ps["sp"], pr["sp"])
        assert np.array_equal(ps["q"], pr["q"])
        assert np.array_equal(ps["alive"], pr["alive"])
        for f in ["x", "y", "zeta", "px", "py", "pz"]:
            assert rel_l2(ps[f], pr[f]) <= 1e-9, (k, f)
    assert len(ps[(ps["sp"] >= 50) & (ps["sp"] < 100)]) > 0, "the case must ionize"


def sort_by_id(p):
    return p[np.lexsort((np.round(p["x"], 6), np.round(p["zeta"], 6), p["sp"], p["id"]))]


@needs_ref
@pytest.mark.parametrize("ygrid", ["fourier", "freehand"])
def test_graded_zeta_frozen_bunch(ygrid):
    """A free-hand zeta grid (steps h/2 at the bunch growing by 15 % per slice to 2h): the graded zeta filter, the
    slice weights w_lo, w_hi of the march, the half-cell locate of the deposit and gather, the zeta terms of the
    sponge and of the co-moving field."""
    from g3d import Simulation, configs
    base = configs.config1(nx=16, ny=16, nzeta=48, nmacro=3000, steps=2) if ygrid == "fourier" else case()
    cfg = configs.on_graded_zeta(base)
    r = ref.RefSimulation(cfg, threads=1)
    r.init()
    s = Simulation(cfg)
    s.init()
    for tag in ["init", "step1", "step2"]:
        if tag != "init":
            s.step(); r.step()
        assert_state({a: s.array(a) for a in FIELDS}, {a: r.array(a) for a in FIELDS}, FIELDS, 1e-10, tag=tag)
        assert rel_l2(s.array("F"), r.array("F")) <= 1e-6, tag
        p, q = s.host_particles(), r.host_particles()
        assert np.array_equal(p["alive"], q["alive"]), tag
        for f in ["x", "y", "zeta", "px", "py", "pz"]:
            assert rel_l2(p[f], q[f]) <= 1e-10, (tag, f)


@needs_ref
def test_graded_zeta_plasma_on_the_free_hand_grid():
    """The structure of the ionization-injection workload at test size: free-hand y and zeta, streaming plasma
    with ions and a grid laser."""
    from g3d import Simulation, configs
    cfg = configs.on_graded_zeta(configs.on_freehand_y(configs.lwfa_small()))
    r = ref.RefSimulation(cfg, threads=1)
    r.init()
    s = Simulation(cfg)
    s.init()
    compare_plasma_state(s, r, 1e-10, "init")
    for k in range(2):
        s.step(); r.step()
        compare_plasma_state(s, r, 1e-10, f"step{k + 1}")
        ps, pr = s.streaming_particles(), r.streaming_particles()
        assert len(ps) == len(pr) and np.array_equal(ps["alive"], pr["alive"])
        for f in ["x", "y", "zeta", "px", "py", "pz", "z"]:
            assert rel_l2(ps[f], pr[f]) <= 1e-9, (k, f)
