"""The mixed FP32/FP64 form (G3D_PREC_MIXED) against the FP64 form.

Bounds, stated per quantity (relative L2 unless noted):
  * field state R, E_z, B_z, L stacked: <= 1e-5 against the FP64 golden state of the reference;
  * float F (the six real field components): <= 1e-5;
  * <p_z> of the bunch: <= 1e-6 relative; particle coordinates: <= 1e-6;
on the reference's golden cases, and the same bounds between the two forms on the GPU for the 64 x 64 x 256
frozen-bunch wake (262,144 particles, 10 s-steps). The FP64 form is pinned to the reference elsewhere
(test_parity_gpu.py); this file states the distance of the mixed form from it.
"""
import numpy as np
import pytest

from conftest import CURRENTS, FIELDS, rel_l2, state_errors

pytestmark = pytest.mark.gpu

TOL_FIELD = 1e-5
TOL_PZ = 1e-6
TOL_PART = 1e-6


def stacked_error(got, ref, names):
    d = np.sqrt(sum(np.linalg.norm(np.asarray(got[n]) - np.asarray(ref[n])) ** 2 for n in names))
    r = np.sqrt(sum(np.linalg.norm(np.asarray(ref[n])) ** 2 for n in names))
    return d / r


def mean_pz(diag):
    return diag[9] / diag[0]


def golden_cases():
    from g3d import configs
    return {
        "wake16": configs.config1(nx=16, ny=16, nzeta=32, nmacro=3000, steps=2),
        "oblique16": configs.config2(nx=16, ny=16, nzeta=48, nmacro=4000, steps=2, envelope=0),
    }


@pytest.mark.parametrize("name", ["wake16", "oblique16"])
def test_mixed_form_against_the_reference_golden(name, golden):
    from g3d import Simulation
    cfg = golden_cases()[name]
    g = golden(name)
    sim = Simulation(cfg, precision="mixed")
    sim.load_bunch()
    sim.init_fields()
    for tag in ["init", "step2"]:
        if tag == "step2":
            sim.step(); sim.step()
        got = {a: sim.array(a) for a in FIELDS + CURRENTS}
        ref_ = {a: g[f"{tag}_{a}"] for a in FIELDS + CURRENTS}
        e = stacked_error(got, ref_, FIELDS)
        assert e <= TOL_FIELD, (tag, "fields", e, state_errors(got, ref_, FIELDS))
        e = stacked_error(got, ref_, CURRENTS)
        assert e <= TOL_FIELD, (tag, "currents", e)
        e = rel_l2(sim.array("F"), g[f"{tag}_F"])
        assert e <= TOL_FIELD, (tag, "F", e)
        p, q = sim.host_particles(), g[f"{tag}_particles"]
        assert np.array_equal(p["alive"], q["alive"])
        for f in ["x", "y", "zeta", "px", "py", "pz"]:
            assert rel_l2(p[f], q[f]) <= TOL_PART, (tag, f, rel_l2(p[f], q[f]))
    d, dr = sim.diagnostics_sums(), g["step2_diag"]
    assert abs(mean_pz(d) - mean_pz(dr)) <= TOL_PZ * abs(mean_pz(dr))
    sim.close()


def run(cfg, precision, steps):
    from g3d import Simulation
    sim = Simulation(cfg, precision=precision)
    sim.load_bunch()
    sim.init_fields()
    for _ in range(steps):
        sim.step()
    out = {a: sim.array(a) for a in FIELDS + ["F"]}
    out["diag"] = sim.diagnostics_sums()
    out["parts"] = sim.host_particles()
    sim.close()
    return out


def test_mixed_form_error_table_frozen_bunch_wake():
    """The error table of the mixed form on the 64 x 64 x 256 frozen-bunch wake after 10 s-steps."""
    from g3d import configs
    cfg = configs.config1()
    a = run(cfg, "fp64", 10)
    b = run(cfg, "mixed", 10)
    table = {n: rel_l2(b[n], a[n]) for n in FIELDS + ["F"]}
    table["state"] = stacked_error(b, a, FIELDS)
    table["<p_z>"] = abs(mean_pz(b["diag"]) - mean_pz(a["diag"])) / abs(mean_pz(a["diag"]))
    for f in ["x", "y", "zeta", "px", "py", "pz"]:
        table[f] = rel_l2(b["parts"][f], a["parts"][f])
    print("mixed vs FP64 (64x64x256, 262144 particles, 10 steps):", {k: f"{v:.2e}" for k, v in table.items()})
    assert table["state"] <= TOL_FIELD
    assert table["F"] <= TOL_FIELD
    assert table["<p_z>"] <= TOL_PZ
    for f in ["x", "y", "zeta", "px", "py", "pz"]:
        assert table[f] <= TOL_PART, (f, table[f])


def test_precision_is_fixed_after_init():
    from g3d import Simulation, G3DError, configs, abi
    sim = Simulation(configs.config1(nx=16, ny=16, nzeta=32, nmacro=3000, steps=2), precision="mixed")
    sim.load_bunch()
    sim.init_fields()
    with pytest.raises(G3DError):
        sim._c(sim.lib.g3d_set_precision(sim.ctx, abi.G3D_PREC_FP64))
    sim.close()


def run_plasma(cfg, precision, steps):
    from g3d import Simulation
    sim = Simulation(cfg, precision=precision)
    sim.init()
    for _ in range(steps):
        sim.step()
    out = {a: sim.array(a) for a in FIELDS + ["F"]}
    out["diag"] = sim.diagnostics_sums()
    out["strm"] = sim.streaming_particles()
    out["np"] = sim.status().np
    sim.close()
    return out


@pytest.mark.parametrize("ions,passes", [(True, 2), (False, 1)])
def test_mixed_form_plasma_error_table(ions, passes):
    """The streaming-plasma march in the mixed form (FP32 gathers and streaming deposit, complex64 spectra, FP64
    R and particles) against the FP64 form on the small laser-wakefield case, 3 s-steps."""
    from g3d import configs
    cfg = configs.lwfa_small(ions=ions, extrapolate=1, passes=passes)
    a = run_plasma(cfg, "fp64", 3)
    b = run_plasma(cfg, "mixed", 3)
    table = {n: rel_l2(b[n], a[n]) for n in FIELDS + ["F"]}
    table["state"] = stacked_error(b, a, FIELDS)
    assert len(b["strm"]) == len(a["strm"]) and b["np"] == a["np"]
    for f in ["x", "y", "px", "py", "pz"]:
        table["plasma " + f] = rel_l2(b["strm"][f], a["strm"][f])
    print(f"mixed vs FP64, plasma (ions={ions}, passes={passes}, 3 steps):", {k: f"{v:.2e}" for k, v in table.items()})
    assert table["state"] <= TOL_FIELD
    assert table["F"] <= TOL_FIELD
    for f in ["x", "y", "px", "py", "pz"]:
        assert table["plasma " + f] <= 1e-5, (f, table["plasma " + f])


def test_mixed_form_free_hand_plasma_error_table():
    """On the free-hand y grid the mixed form is the FP32 streaming plasma (gathers and deposit) over FP64 spectra
    (the march there is the serial solves along y per k_x line, latency-bound, not bandwidth-bound): its
    distance from the FP64 form on the small laser wakefield on a free-hand y and zeta grid, 3 s-steps."""
    from g3d import configs
    cfg = configs.on_graded_zeta(configs.on_freehand_y(configs.lwfa_small(extrapolate=1, passes=2)))
    a = run_plasma(cfg, "fp64", 3)
    b = run_plasma(cfg, "mixed", 3)
    table = {n: rel_l2(b[n], a[n]) for n in FIELDS + ["F"]}
    table["state"] = stacked_error(b, a, FIELDS)
    assert len(b["strm"]) == len(a["strm"]) and b["np"] == a["np"]
    for f in ["x", "y", "px", "py", "pz"]:
        table["plasma " + f] = rel_l2(b["strm"][f], a["strm"][f])
    print("mixed vs FP64, plasma on the free-hand y and zeta grid (3 steps):", {k: f"{v:.2e}" for k, v in table.items()})
    assert table["state"] <= TOL_FIELD
    assert table["F"] <= TOL_FIELD
    for f in ["x", "y", "px", "py", "pz"]:
        assert table["plasma " + f] <= 1e-5, (f, table["plasma " + f])
