"""Parity of the streaming-plasma march (libg3d.so) with the reference FP64 CPU path, small cases against the live
reference build: init with a grid laser, then s-steps with streaming plasma (mobile ions, passes, the extrapolating
predictor and the correction, trapping), and ADK ionization of a neutral gas.

Tolerances as in test_parity_gpu.py: fields <= 1e-10 relative L2 against the field state norm (a laser-driven
plasma is chaotic only over many steps; two steps stay at rounding level), streaming particles <= 1e-9 relative L2.
The ionization event set must be identical: the same ions reach the same charge states, and the freed electrons
are the same (matched by id; the order in which the GPU appends them differs).
"""
import numpy as np
import pytest

from conftest import CURRENTS, FIELDS, assert_state, rel_l2

pytestmark = pytest.mark.gpu
ref = pytest.importorskip("ref")
needs_ref = pytest.mark.skipif(not ref.available(), reason="reference build oracle/_ref not present")


def run_pair(cfg, steps):
    from g3d import Simulation
    r = ref.RefSimulation(cfg, threads=1)
    r.init()
    s = Simulation(cfg)
    s.init()
    return s, r


def compare_fields(s, r, tol=1e-10, tag=""):
    assert_state({a: s.array(a) for a in FIELDS}, {a: r.array(a) for a in FIELDS}, FIELDS, tol, comp_tol=1e-5, tag=tag)
    assert_state({a: s.array(a) for a in CURRENTS}, {a: r.array(a) for a in CURRENTS}, CURRENTS, tol, comp_tol=1e-5, tag=tag)
    assert rel_l2(s.array("F"), r.array("F")) <= 1e-6, tag


def sort_by_id(p):
    # electrons freed from one ion share its id: order them by where they are
    return p[np.lexsort((np.round(p["x"], 6), np.round(p["zeta"], 6), p["sp"], p["id"]))]


@needs_ref
@pytest.mark.parametrize("ions,extrap,passes", [(True, 1, 2), (False, 0, 1), (True, 1, 3)])
def test_lwfa_small_matches_reference(ions, extrap, passes):
    from g3d import configs
    cfg = configs.lwfa_small(ions=ions, extrapolate=extrap, passes=passes)
    s, r = run_pair(cfg, 2)
    compare_fields(s, r, tag="init")
    for k in range(2):
        s.step(); r.step()
        compare_fields(s, r, tag=f"step{k + 1}")
        ps, pr = s.streaming_particles(), r.streaming_particles()
        assert len(ps) == len(pr)
        assert np.array_equal(ps["alive"], pr["alive"])
        for f in ["x", "y", "zeta", "px", "py", "pz", "z"]:
            assert rel_l2(ps[f], pr[f]) <= 1e-9, (k, f, rel_l2(ps[f], pr[f]))
        bs, br = s.host_particles(), r.host_particles()
        assert len(bs) == len(br)
        for f in ["x", "y", "zeta", "px", "py", "pz"]:
            assert rel_l2(bs[f], br[f]) <= 1e-10, (k, f)


@needs_ref
@pytest.mark.parametrize("ygrid", ["fourier", "freehand"])
def test_plasma_channel_cutoff_and_profile_match_reference(ygrid):
    """Lattice points of zero density (beyond r_max), a parabolic channel and a longitudinal density profile. The
    fresh plasma of every step is built on the device with the points of zero density left out (a running
    count); its particles must be the reference loader's: the same count, order, ids and, bit for bit, weights."""
    from g3d import configs
    cfg = configs.lwfa_small()
    cfg.plasma.update(r_max=7.0, parabolic=1, channel_depth=0.6, r_channel=5.0,
                      z_points=[0.0, 2.0, 4.0], z_values=[0.4, 1.0, 0.7])
    if ygrid == "freehand":
        cfg = configs.on_freehand_y(cfg)
    s, r = run_pair(cfg, 2)
    compare_fields(s, r, tag="init")
    full = cfg.nx * cfg.ny * cfg.plasma["ppc_x"] * cfg.plasma["ppc_y"] * 2       # electrons and H+ at every point
    for k in range(2):
        s.step(); r.step()
        compare_fields(s, r, tag=f"step{k + 1}")
        ps, pr = s.streaming_particles(), r.streaming_particles()
        assert 0 < len(ps) == len(pr) < full, (len(ps), len(pr), full)
        assert np.array_equal(ps["id"], pr["id"]) and np.array_equal(ps["sp"], pr["sp"])
        assert np.array_equal(ps["w"], pr["w"]) and np.array_equal(ps["alive"], pr["alive"])
        for f in ["x", "y", "zeta", "px", "py", "pz", "z"]:
            assert rel_l2(ps[f], pr[f]) <= 1e-9, (k, f, rel_l2(ps[f], pr[f]))


@needs_ref
def test_window_shift_moves_the_joining_particles():
    """A driver strong enough to trap electrons too slow to join the beam: they wait, on the device, to stream
    again in the next march. A window shift between two steps must move them with everything else, as the
    reference moves its joining list."""
    from g3d import configs
    cfg = configs.lwfa_small(a0=3.0, n0=0.02)
    s, r = run_pair(cfg, 2)
    s.step(); r.step()
    s.shift_window(3, -2); r.shift_window(3, -2)
    s.step(); r.step()
    compare_fields(s, r, tol=1e-9, tag="after the shift")
    ps, pr = s.streaming_particles(), r.streaming_particles()
    fresh = cfg.nx * cfg.ny * cfg.plasma["ppc_x"] * cfg.plasma["ppc_y"] * 2
    assert len(ps) == len(pr) > fresh, (len(ps), len(pr), fresh)        # the lattice and joining particles
    assert np.array_equal(ps["id"], pr["id"]) and np.array_equal(ps["alive"], pr["alive"])
    for f in ["x", "y", "zeta", "px", "py", "pz", "z"]:
        assert rel_l2(ps[f], pr[f]) <= 1e-9, (f, rel_l2(ps[f], pr[f]))
    # the density lines through the axis follow the shifted window origin
    for a in ["rho_lines", "rho_lines_i"]:
        x, y = s.array(a), r.array(a)
        assert x.size == y.size > 0 and np.abs(y).max() > 0, a
        assert rel_l2(x, y) <= 1e-9, (a, rel_l2(x, y))


@needs_ref
def test_smoothing_and_trapping_small():
    """The smoothing 1/(1 + a^2 k^2) of the streaming current, and a driver strong enough to trap electrons."""
    from g3d import configs
    cfg = configs.lwfa_small(a0=3.0, n0=0.02, smooth=0.4)
    s, r = run_pair(cfg, 2)
    for k in range(2):
        s.step(); r.step()
        compare_fields(s, r, tol=1e-9, tag=f"step{k + 1}")
    assert s.status().np == r.status().np


@needs_ref
def test_ionization_event_set_is_identical():
    from g3d import configs
    cfg = configs.ionization_small()
    s, r = run_pair(cfg, 2)
    for k in range(2):
        s.step(); r.step()
        ps, pr = sort_by_id(s.streaming_particles()), sort_by_id(r.streaming_particles())
        assert len(ps) == len(pr), (len(ps), len(pr))
        # the same particles (ions and the electrons they freed), the same charge states
        assert np.array_equal(ps["id"], pr["id"]) and np.array_equal(ps["sp"], pr["sp"])
        assert np.array_equal(ps["q"], pr["q"])
        assert np.array_equal(ps["alive"], pr["alive"])
        for f in ["x", "y", "zeta", "px", "py", "pz"]:
            assert rel_l2(ps[f], pr[f]) <= 1e-9, (k, f)
    freed = ps[(ps["sp"] >= 50) & (ps["sp"] < 100)]
    assert len(freed) > 0, "the case must ionize"


@needs_ref
def test_plasma_checkpoint_restarts_the_reference_and_back(tmp_path):
    """With a plasma a checkpoint also holds the streaming current of level s0 and the particles that join the next
    march (reference src/sim_checkpoint.cpp:39-58). A driver strong enough to trap: libg3d's checkpoint after step 1
    restarts the reference, the reference's after step 2 restarts libg3d, and each continues as the other."""
    from g3d import Simulation, configs
    cfg = configs.lwfa_small(a0=3.0, n0=0.02)
    s, r = run_pair(cfg, 2)
    s.step(); r.step()
    s.write_checkpoint(tmp_path / "checkpoint_000001_r0000.bin")
    r2 = ref.RefSimulation(cfg, threads=1)
    r2.read_checkpoint(tmp_path, 1)
    for a in ["Rx", "Ry", "Ez", "Bz", "Lx", "Ly", "j0x", "j0y"]:
        assert np.array_equal(s.array(a), r2.array(a)), a
    s.step(); r2.step()
    compare_fields(s, r2, tol=1e-9, tag="reference from libg3d's checkpoint")
    ps, pr = s.streaming_particles(), r2.streaming_particles()
    fresh = cfg.nx * cfg.ny * cfg.plasma["ppc_x"] * cfg.plasma["ppc_y"] * 2
    assert len(ps) == len(pr) > fresh and np.array_equal(ps["id"], pr["id"])      # the joining particles came along
    for f in ["x", "y", "zeta", "px", "py", "pz", "z"]:
        assert rel_l2(ps[f], pr[f]) <= 1e-9, f
    r2.write_checkpoint(tmp_path)
    s2 = Simulation(cfg)
    s2.read_checkpoint(tmp_path / "checkpoint_000002_r0000.bin")
    s2.step(); r2.step()
    compare_fields(s2, r2, tol=1e-9, tag="libg3d from the reference's checkpoint")
    assert s2.status().istep == r2.status().istep == 3
    for sim in (s, s2, r, r2):
        sim.close()
