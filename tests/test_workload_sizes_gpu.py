"""Parity with the reference FP64 CPU path at the workloads' own sizes (the other parity tests shrink the grids):

  1  the frozen-bunch wake in full: 64 x 64 modes x 256 slices, 262,144 macro-electrons, all 10 s-steps
  2  the oblique plane wave on its full 128 x 128 x 1024 grid with 1,048,576 macro-electrons (the Gaussian envelope,
     which the reference has), 3 s-steps
  3  the laser wakefield with plasma in FP64 on its full 256 x 256 transverse grid at its own h = 0.2, on a window
     shortened to 256 slices (mobile H+ ions, grid laser, 4,194,304-electron witness), 2 s-steps
  5  ionization injection on its free-hand grids (256 Fourier modes in x, 193 graded y nodes between walls, graded
     zeta) on a window of 256 slices, H and N neutral gas with ADK over every level, 2 s-steps: the ionization event
     set identical

The reference runs on every host core (its OpenMP reductions then add in another order: 1 vs 8 threads agree to
~1e-14 here, well inside the bounds). Bounds as in test_parity_gpu.py: the field state <= 1e-10 relative L2 against
its norm, beam coordinates <= 1e-10, streaming particles <= 1e-9, F (float in both codes) <= 1e-6, <p_z> <= 1e-10.
"""
import os

import numpy as np
import pytest

from conftest import CURRENTS, FIELDS, assert_state, rel_l2

pytestmark = pytest.mark.gpu
ref = pytest.importorskip("ref")
needs_ref = pytest.mark.skipif(not ref.available(), reason="reference build oracle/_ref not present")
THREADS = os.cpu_count() or 1


def both(cfg):
    from g3d import Simulation
    r = ref.RefSimulation(cfg, threads=THREADS)
    r.init()
    s = Simulation(cfg)
    s.init()
    return s, r


def fields_match(s, r, tag, tol=1e-10, comp_tol=1e-6, currents=True):
    assert_state({a: s.array(a) for a in FIELDS}, {a: r.array(a) for a in FIELDS}, FIELDS, tol, comp_tol, tag=tag)
    if currents:
        assert_state({a: s.array(a) for a in CURRENTS}, {a: r.array(a) for a in CURRENTS}, CURRENTS, tol, comp_tol,
                     tag=tag)
    e = rel_l2(s.array("F"), r.array("F"))
    assert e <= 1e-6, (tag, "F", e)


def beam_match(s, r, tag, tol=1e-10):
    p, q = s.host_particles(), r.host_particles()
    assert len(p) == len(q), (tag, len(p), len(q))
    assert np.array_equal(p["alive"], q["alive"]), tag
    for f in ["x", "y", "zeta", "px", "py", "pz", "z"]:
        e = rel_l2(p[f], q[f])
        assert e <= tol, (tag, f, e)
    d, dr = s.diagnostics_sums(), r.diagnostics_sums()
    assert abs(d[9] / d[0] - dr[9] / dr[0]) <= 1e-10 * abs(dr[9] / dr[0]), (tag, "<p_z>")


def sort_streaming(p):
    return p[np.lexsort((np.round(p["x"], 6), np.round(p["zeta"], 6), p["sp"], p["id"]))]


@needs_ref
def test_workload1_in_full_matches_the_reference():
    from g3d import configs
    cfg = configs.config1()
    assert (cfg.nx, cfg.ny, cfg.nzeta, cfg.particles, cfg.steps) == (64, 64, 256, 262144, 10)
    s, r = both(cfg)
    fields_match(s, r, "init")
    beam_match(s, r, "init")
    for k in range(cfg.steps):
        s.step(); r.step()
    fields_match(s, r, "step 10")
    beam_match(s, r, "step 10")
    assert s.status().istep == r.status().istep == 10
    s.close(); r.close()


@needs_ref
def test_workload2_full_grid_matches_the_reference():
    from g3d import configs
    cfg = configs.config2(envelope=0)
    assert (cfg.nx, cfg.ny, cfg.nzeta, cfg.particles) == (128, 128, 1024, 1048576)
    s, r = both(cfg)
    fields_match(s, r, "init")
    for k in range(3):
        s.step(); r.step()
    fields_match(s, r, "step 3")
    beam_match(s, r, "step 3")
    assert abs(s.field_energy() - r.field_energy()) <= 1e-9 * abs(r.field_energy())
    s.close(); r.close()


@needs_ref
def test_workload3_fp64_full_transverse_grid_on_a_short_window():
    from g3d import configs
    cfg = configs.config3(nzeta=256, h=0.2)
    assert (cfg.nx, cfg.ny, cfg.particles) == (256, 256, 4194304) and abs(cfg.h - 0.2) < 1e-15
    s, r = both(cfg)
    fields_match(s, r, "init")
    for k in range(2):
        s.step(); r.step()
        fields_match(s, r, f"step {k + 1}", comp_tol=1e-5)
        ps, pr = s.streaming_particles(), r.streaming_particles()
        assert len(ps) == len(pr) > 500000, (len(ps), len(pr))
        assert np.array_equal(ps["id"], pr["id"]) and np.array_equal(ps["alive"], pr["alive"])
        for f in ["x", "y", "zeta", "px", "py", "pz", "z"]:
            e = rel_l2(ps[f], pr[f])
            assert e <= 1e-9, (k, f, e)
    beam_match(s, r, "step 2")
    s.close(); r.close()


@needs_ref
def test_workload5_structure_on_a_short_window():
    from g3d import configs
    cfg = configs.config5(nzeta=256, ppc=1)
    assert cfg.nx == 256 and len(cfg.ynode) == 193 and cfg.ynode is not None and cfg.zeta_table is not None
    s, r = both(cfg)
    fields_match(s, r, "init")
    for k in range(2):
        s.step(); r.step()
        fields_match(s, r, f"step {k + 1}", comp_tol=1e-5)
        ps, pr = sort_streaming(s.streaming_particles()), sort_streaming(r.streaming_particles())
        assert len(ps) == len(pr), (len(ps), len(pr))
        assert np.array_equal(ps["id"], pr["id"]) and np.array_equal(ps["sp"], pr["sp"])
        assert np.array_equal(ps["q"], pr["q"]) and np.array_equal(ps["alive"], pr["alive"])
        for f in ["x", "y", "zeta", "px", "py", "pz"]:
            e = rel_l2(ps[f], pr[f])
            assert e <= 1e-9, (k, f, e)
    freed = ps[(ps["sp"] >= 50) & (ps["sp"] < 100)]
    assert len(freed) > 0, "the laser must ionize"
    n_states = {int(q) for q in ps["q"][ps["sp"] == 4]}  # nitrogen (the second ion species: sp = 3 + 1)
    assert max(n_states) >= 2, n_states                    # beyond its first level
    s.close(); r.close()
