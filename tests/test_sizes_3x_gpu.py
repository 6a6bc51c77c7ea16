"""Transverse sizes three times a power of two (24..384): the transforms take a radix-3 pass (k_fft.cuh), as the
reference's mixed-radix FFT takes such lengths (src/fft.hpp). Against the reference's CPU build on the same config and
seed: a vacuum wake on a 48 x 24 grid and a laser wakefield with plasma and ions on 24 x 48 (FP64, the parity bounds of
the other tests), and the mixed form on 96 x 96 against the FP64 form (its stated bound)."""
import numpy as np
import pytest

from conftest import CURRENTS, FIELDS, assert_state, rel_l2

pytestmark = pytest.mark.gpu
ref = pytest.importorskip("ref")
needs_ref = pytest.mark.skipif(not ref.available(), reason="reference build oracle/_ref not present")


def pair(cfg):
    from g3d import Simulation
    r = ref.RefSimulation(cfg, threads=8)
    r.init()
    s = Simulation(cfg)
    s.init()
    return s, r


def compare(s, r, tag):
    assert_state({a: s.array(a) for a in FIELDS}, {a: r.array(a) for a in FIELDS}, FIELDS, 1e-10, comp_tol=1e-5, tag=tag)
    assert_state({a: s.array(a) for a in CURRENTS}, {a: r.array(a) for a in CURRENTS}, CURRENTS, 1e-10, comp_tol=1e-5, tag=tag)
    assert rel_l2(s.array("F"), r.array("F")) <= 1e-6, tag


@needs_ref
def test_vacuum_wake_on_a_48_by_24_grid_matches_the_reference():
    from g3d import configs
    cfg = configs.config1(nx=48, ny=24, nzeta=64, nmacro=20000, steps=2)
    s, r = pair(cfg)
    try:
        compare(s, r, "init")
        for k in range(2):
            s.step(); r.step()
            compare(s, r, f"step{k + 1}")
        ps, pr = s.host_particles(), r.host_particles()
        for f in ["x", "y", "zeta", "px", "py", "pz"]:
            assert rel_l2(ps[f], pr[f]) <= 1e-10, f
    finally:
        s.close(); r.close()


@needs_ref
def test_laser_wakefield_on_a_24_by_48_grid_matches_the_reference():
    from g3d import configs
    cfg = configs.lwfa_small(nx=24, ny=48, steps=2)
    s, r = pair(cfg)
    try:
        compare(s, r, "init")
        for k in range(2):
            s.step(); r.step()
            compare(s, r, f"step{k + 1}")
            ps, pr = s.streaming_particles(), r.streaming_particles()
            assert len(ps) == len(pr)
            for f in ["x", "y", "zeta", "px", "py", "pz", "z"]:
                assert rel_l2(ps[f], pr[f]) <= 1e-9, (k, f)
    finally:
        s.close(); r.close()


def test_mixed_form_on_a_96_by_96_grid():
    from g3d import Simulation, configs
    cfg = configs.config1(nx=96, ny=96, nzeta=64, nmacro=20000, steps=3)
    out = {}
    for form in ("fp64", "mixed"):
        s = Simulation(cfg, precision=form)
        s.load_bunch(); s.init()
        for _ in range(cfg.steps):
            s.step()
        out[form] = (np.concatenate([s.array(a).ravel() for a in FIELDS]), s.array("F"), s.host_particles()["pz"])
        s.close()
    (a, fa, pa), (b, fb, pb) = out["fp64"], out["mixed"]
    assert rel_l2(b, a) <= 1e-5 and rel_l2(fb, fa) <= 1e-5 and rel_l2(pb, pa) <= 1e-6
