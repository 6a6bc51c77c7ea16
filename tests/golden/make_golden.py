"""Generates the golden fixtures of tests/golden/ from the reference GEM-PIC-3D CPU build
(oracle/_ref/libg3dref.so, built by `make -C oracle`), single-threaded for reproducibility.

Each fixture is one small run of a benchmark workload: the particles after the bunch load, the state after
init (Simulation::init) and after `steps` s-steps (Simulation::step): the FP64 spectra Rx, Ry, Ez, Bz, Lx, Ly,
the filtered currents jkx, jky, jkz, the float fields F, the particles and the 19 diagnostics sums.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
sys.path.insert(0, os.path.join(REPO, "gem-pic-3d_b200"))

import ref  # noqa: E402
from g3d import configs  # noqa: E402

SPECTRA = ["Rx", "Ry", "Ez", "Bz", "Lx", "Ly", "jkx", "jky", "jkz"]


def cases():
    """Name -> (config, steps). Small sizes of workloads 1 and 2 (workload 2 with the reference's
    Gaussian envelope, which the reference can run)."""
    return {
        "wake16": (configs.config1(nx=16, ny=16, nzeta=32, nmacro=3000, steps=2), 2),
        "oblique16": (configs.config2(nx=16, ny=16, nzeta=48, nmacro=4000, steps=2, envelope=0), 2),
    }


def snapshot(sim, tag):
    out = {}
    for a in SPECTRA:
        out[f"{tag}_{a}"] = sim.array(a)
    out[f"{tag}_F"] = sim.array("F")
    out[f"{tag}_particles"] = sim.host_particles()
    out[f"{tag}_diag"] = sim.diagnostics_sums()
    st = sim.status()
    out[f"{tag}_status"] = np.array([st.s, st.X0, st.Y0, st.beta_b, st.gm2_b, st.istep, st.np, st.lost], dtype=np.float64)
    return out


def make(name, cfg, steps):
    sim = ref.RefSimulation(cfg, threads=1)
    sim.load_bunch()
    data = {"loaded_particles": sim.host_particles()}
    sim.init_fields()
    data.update(snapshot(sim, "init"))
    for _ in range(steps):
        sim.step()
    data.update(snapshot(sim, f"step{steps}"))
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **data)
    return path


if __name__ == "__main__":
    for name, (cfg, steps) in cases().items():
        print(make(name, cfg, steps), os.path.getsize(os.path.join(HERE, f"{name}.npz")))
