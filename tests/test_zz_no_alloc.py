"""g3d_beam_beta_sums_static: the bunch's beta sums taken with the library's static device scratch instead of a
per-call allocation. Checked against the beta g3d_comoving_field takes from the same sums (the status' beta_b
after init), on two calls in a row, and for its capacity check above G3D_BETA_STATIC_MAX. Collected last so that
it also runs after every other GPU test in one process (the scratch is shared by the contexts of a device)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

BETA_STATIC_MAX = 1048576      # G3D_BETA_STATIC_MAX of include/g3d.h
G3D_ERR_CAPACITY = 3


def beta_sums_static(sim):
    out = (C.c_double * 2)()
    rc = sim.lib.g3d_beam_beta_sums_static(sim.ctx, out)
    return rc, out[0], out[1]


def small_case():
    from g3d import configs
    return configs.config2(nx=16, ny=16, nzeta=48, nmacro=4000, steps=2, envelope=0)


def test_static_beta_sums_match_the_comoving_beta():
    from g3d import Simulation
    sim = Simulation(small_case())
    sim.load_bunch()
    sim.init_fields()
    beta = sim.status().beta_b
    first, second = beta_sums_static(sim), beta_sums_static(sim)
    assert first[0] == 0 and second[0] == 0, sim.lib.g3d_last_error(sim.ctx)
    assert first[1:] == second[1:]                      # the same bits on the second call
    assert abs(first[1] / first[2] - beta) <= 1e-15 * abs(beta)
    p = sim.host_particles()
    a = p["alive"] == 1
    g = np.sqrt(1 + p["px"][a] ** 2 + p["py"][a] ** 2 + p["pz"][a] ** 2)
    s0, s1 = np.sum(p["w"][a] * p["pz"][a] / g), np.sum(p["w"][a])
    assert abs(first[1] - s0) <= 1e-12 * abs(s0) and abs(first[2] - s1) <= 1e-12 * abs(s1)
    sim.step()
    third = beta_sums_static(sim)                       # after a step: still the sums of the live bunch
    assert third[0] == 0 and third[2] > 0
    sim.close()


def test_static_beta_sums_reject_more_particles_than_the_scratch_holds():
    from g3d import Simulation
    sim = Simulation(small_case())
    sim.load_bunch()
    p = sim.host_particles()
    big = np.resize(p, BETA_STATIC_MAX + 1)
    sim.set_particles(big)
    rc, _, _ = beta_sums_static(sim)
    assert rc == G3D_ERR_CAPACITY
    assert b"G3D_BETA_STATIC_MAX" in sim.lib.g3d_last_error(sim.ctx)
    sim.set_particles(p)
    rc, s0, s1 = beta_sums_static(sim)
    assert rc == 0 and s1 > 0
    sim.close()
