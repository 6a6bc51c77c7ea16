"""The oracle, pinned before it is trusted (CPU only).

1. The reference build (oracle/_ref) reproduces the committed golden fixtures bit for bit (single thread).
2. The numpy restatement (oracle/g3d_oracle.py) matches the golden fixtures within the parity tolerances,
   stage by stage against the live reference, and on the flat-top envelope (which only it restates)
   against an independent finite difference of the vector potential.
"""
import math

import numpy as np
import pytest

from conftest import CURRENTS, FIELDS, assert_state, rel_l2

import ref
import g3d_oracle
from g3d import configs

needs_ref = pytest.mark.skipif(not ref.available(), reason="reference build oracle/_ref not present")


def golden_cfg(name):
    if name == "wake16":
        return configs.config1(nx=16, ny=16, nzeta=32, nmacro=3000, steps=2)
    return configs.config2(nx=16, ny=16, nzeta=48, nmacro=4000, steps=2, envelope=0)


@needs_ref
@pytest.mark.parametrize("name", ["wake16", "oblique16"])
def test_reference_build_reproduces_golden(name, golden):
    g = golden(name)
    r = ref.RefSimulation(golden_cfg(name), threads=1)
    r.load_bunch()
    p = r.host_particles()
    for f in p.dtype.names:
        assert np.array_equal(p[f], g["loaded_particles"][f])
    r.init_fields()
    for a in FIELDS + CURRENTS + ["F"]:
        assert np.array_equal(r.array(a), g[f"init_{a}"]), a
    r.step(); r.step()
    for a in FIELDS + CURRENTS + ["F"]:
        assert np.array_equal(r.array(a), g[f"step2_{a}"]), a
    assert np.array_equal(r.diagnostics_sums(), g["step2_diag"])


@pytest.mark.parametrize("name", ["wake16", "oblique16"])
def test_restatement_matches_golden(name, golden):
    g = golden(name)
    cfg = golden_cfg(name)
    o = g3d_oracle.Oracle(cfg)
    o.set_particles(g["loaded_particles"])
    o.set_origin(-0.5 * cfg.Lx, -0.5 * cfg.Ly)
    o.init_fields()
    for tag in ["init", "step2"]:
        if tag == "step2":
            o.step(); o.step()
        got = {a: o.array(a) for a in FIELDS + CURRENTS}
        ref_ = {a: g[f"{tag}_{a}"] for a in FIELDS + CURRENTS}
        assert_state(got, ref_, FIELDS, 1e-10, tag=tag)
        assert_state(got, ref_, CURRENTS, 1e-10, tag=tag)
        assert rel_l2(o.array("F"), g[f"{tag}_F"]) <= 1e-6
        p, q = o.host_particles(), g[f"{tag}_particles"]
        assert np.array_equal(p["alive"], q["alive"])
        for f in ["x", "y", "zeta", "px", "py", "pz"]:
            assert rel_l2(p[f], q[f]) <= 1e-10, (tag, f)
    d, dr = o.diagnostics_sums(), g["step2_diag"]
    assert np.allclose(d, dr, rtol=1e-10, atol=0)


@needs_ref
def test_restatement_stages_against_reference():
    cfg = configs.config2(nx=16, ny=8, nzeta=40, nmacro=3000, steps=1, envelope=0)
    r = ref.RefSimulation(cfg, threads=1)
    r.load_bunch()
    o = g3d_oracle.Oracle(cfg)
    o.set_particles(r.host_particles())
    o.set_origin(-0.5 * cfg.Lx, -0.5 * cfg.Ly)
    r.currents(); o.currents()
    assert rel_l2(o.array("jw"), r.array("jw")) <= 1e-14
    for a in CURRENTS:
        assert rel_l2(o.array(a), r.array(a)) <= 1e-13
    r.comoving_field(); o.comoving_field()
    assert o.beta_b == r.status().beta_b or abs(o.beta_b - r.status().beta_b) < 1e-12
    for a in ["Rx", "Ry"]:
        assert rel_l2(o.array(a), r.array(a)) <= 1e-11
    for D in (0.0, 1.0):
        for a in FIELDS + ["j0x", "j0y"] + CURRENTS:
            o.set_array(a, r.array(a))
        r.march(D); o.march(D)
        assert_state({a: o.array(a) for a in FIELDS}, {a: r.array(a) for a in FIELDS}, FIELDS, 1e-12)
    r.sponge_and_real_fields(); o.sponge_and_real_fields()
    assert rel_l2(o.array("Rx"), r.array("Rx")) <= 1e-12
    assert rel_l2(o.array("F"), r.array("F")) <= 1e-6


def test_flattop_envelope_is_the_derivative_of_the_potential():
    """E = -dA/deta for the flat-top + sin^2 envelope (the restated field against a central difference of
    A = a0 g(eta) cos(kL (eta - eta_c) + cep)), at points on the plateau, on both ramps and outside."""
    cfg = configs.config2(nx=16, ny=16, nzeta=48, nmacro=10, steps=1)
    o = g3d_oracle.Oracle(cfg)
    L = o.laser
    L.update(pol=0)                    # E along y: E_y = -dA/deta

    def A(eta):
        xi = eta - L["eta_c"]
        ax, hf, rp = abs(xi), 0.5 * L["flat"], L["ramp"]
        g = 1.0 if ax <= hf else (math.sin(0.5 * math.pi * (hf + rp - ax) / rp) ** 2 if ax < hf + rp else 0.0)
        return L["a0"] * g * math.cos(L["kL"] * xi + L["cep"])

    for eta in [0.3, 29.0, 31.7, 35.0, 39.5, -33.3, -38.0, 45.0]:
        E, _ = o.laser_field(np.array([0.0]), np.array([0.0]), np.array([eta]))
        h = 1e-5
        fd = -(A(eta + h) - A(eta - h)) / (2 * h)
        assert abs(E[1][0] - fd) <= 1e-8 * max(1.0, abs(fd)), eta


@needs_ref
def test_element_table_matches_the_reference():
    """The elements the workloads use carry the reference table's mass and ionization energies."""
    for sym, (mass_u, ip) in configs.ELEMENTS.items():
        rm, rip = ref.element(sym)
        assert mass_u == rm, sym
        assert ip == rip, sym
