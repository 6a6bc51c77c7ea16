"""The density lines of the streaming plasma (rho_lines, rho_lines_i: the charge of the negative and the positive
streaming particles of every half-cell on the row and the column through the axis, src/sim_plasma.cpp:363-374)
against the reference's CPU build on the same config and seed: Fourier y with mobile ions, the free-hand y grid,
field ionization (freed electrons), and the mixed form against the FP64 form."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu
ref = pytest.importorskip("ref")
needs_ref = pytest.mark.skipif(not ref.available(), reason="reference build oracle/_ref not present")

LINES = ["rho_lines", "rho_lines_i"]


def run_pair(cfg, steps=2):
    from g3d import Simulation
    r = ref.RefSimulation(cfg, threads=8)
    s = Simulation(cfg)
    try:
        r.init(); s.init()
        out = []
        for k in range(steps):
            s.step(); r.step()
            out.append(({a: s.array(a) for a in LINES}, {a: r.array(a) for a in LINES}))
        return out
    finally:
        s.close(); r.close()


def check(out, ions, tol=1e-9):
    for k, (a, b) in enumerate(out):
        for name in LINES:
            if name == "rho_lines_i" and not ions:
                assert a[name].size == 0 and b[name].size == 0, (k, name)
                continue
            assert a[name].shape == b[name].shape and a[name].size > 0, (k, name, a[name].shape, b[name].shape)
            assert np.abs(b[name]).max() > 0, (k, name)
            e = rel_l2(a[name], b[name])
            assert e <= tol, (k, name, e)


@needs_ref
@pytest.mark.parametrize("ions", [True, False])
def test_density_lines_on_the_fourier_grid(ions):
    from g3d import configs
    check(run_pair(configs.lwfa_small(ions=ions, a0=2.0, n0=0.02)), ions)


@needs_ref
def test_density_lines_on_the_free_hand_grid():
    from g3d import configs
    check(run_pair(configs.on_freehand_y(configs.lwfa_small(ions=True))), True)


@needs_ref
def test_density_lines_with_field_ionization():
    from g3d import configs
    check(run_pair(configs.ionization_small()), True)


def test_density_lines_of_the_mixed_form():
    from g3d import Simulation, configs
    cfg = configs.lwfa_small(ions=True, a0=2.0, n0=0.02)
    out = {}
    for form in ("fp64", "mixed"):
        s = Simulation(cfg, precision=form)
        s.init()
        s.step()
        out[form] = {a: s.array(a) for a in LINES}
        s.close()
    for a in LINES:
        assert out["fp64"][a].size > 0
        assert rel_l2(out["mixed"][a], out["fp64"][a]) <= 1e-5, a


def test_no_density_lines_without_a_plasma():
    from g3d import Simulation, configs
    s = Simulation(configs.config1(nx=16, ny=16, nzeta=32, nmacro=2000, steps=1))
    try:
        s.init()
        for a in LINES:
            assert s.array(a).size == 0
    finally:
        s.close()
