"""The drop-in boundary from the reference's side: g3d_run (gem-pic-3d_b200/shim) reads a GEM-PIC-3D deck with the
reference's own deck and Config layers, maps every key onto the C-ABI (g3dshim::setup_from) and runs the march in
libg3d; the reference's own command line (oracle/_ref/gempic3d) runs the same deck on the host. The decks are written
here. Compared: the checkpoint both write after the same step (the reference's binary layout: every array at the
parity bounds of test_parity_gpu.py) and diag.txt (every column to its printed digits), for a vacuum wake and for a
laser wakefield with streaming plasma and ions. tests/test_shim.py covers the deck mapping without a device."""
import math
import os
import subprocess

import numpy as np
import pytest

from conftest import FIELDS, REPO, assert_state, rel_l2

pytestmark = pytest.mark.gpu
SHIM = os.path.join(REPO, "gem-pic-3d_b200", "shim", "_build", "g3d_run")
REF_CLI = os.path.join(REPO, "oracle", "_ref", "gempic3d")
needs_both = pytest.mark.skipif(not (os.path.exists(SHIM) and os.path.exists(REF_CLI)),
                                reason="g3d_run or the reference CLI not built (they need the reference's sources)")
UM = 0.8 / (2 * math.pi)          # um per code length 1/k0 at lambda0 = 0.8 um


def L(x):
    return f"{x * UM:.10g} um"


def wake_deck(out):
    return f"""grid {{
  lambda0 = 0.8 um
  nx = 32
  ny = 32
  Lx = {L(40)}
  nzeta = 64
  window_length = {L(63)}
  dz = {L(5)}
  z_end = {L(15)}
  sponge = {L(4)}
  move_x = false
  move_y = false
}}
bunch {{
  charge = 0.5 pC
  gamma = 1000
  sigma_x = {L(2)}
  sigma_z = {L(4)}
  emittance_x = {L(0.2)}
  zeta_center = {L(40)}
  macroparticles = 20000
  seed = 3
}}
bunch2 {{
  charge = 0.2 pC
  gamma = 60
  sigma_x = {L(1)}
  sigma_z = {L(1.5)}
  zeta_center = {L(20)}
  macroparticles = 6000
  seed = 9
}}
output {{
  dir = {out}
  every = 1
  checkpoint_every = 3
  fields = none
  particles = false
}}
"""


def lwfa_deck(out):
    return f"""grid {{
  lambda0 = 0.8 um
  nx = 16
  ny = 16
  Lx = {L(24)}
  nzeta = 64
  window_length = {L(25.2)}
  dz = {L(2)}
  z_end = {L(4)}
  sponge = {L(2.4)}
  move_x = false
  move_y = false
}}
laser {{
  type = gaussian
  a0 = 1
  waist = {L(6)}
  tau_fwhm = {6 * UM / 0.299792458:.10g} fs
  zeta_center = {L(17.6)}
  z_focus = {L(2)}
}}
plasma {{
  density = 0.01 n_c
  ppc_x = 2
  ppc_y = 2
}}
ion {{
  element = H
}}
bunch {{
  charge = 0.05 pC
  gamma = 50
  sigma_x = {L(1)}
  sigma_z = {L(1.5)}
  emittance_x = {L(0.05)}
  zeta_center = {L(7.6)}
  macroparticles = 600
  seed = 3
}}
output {{
  dir = {out}
  every = 1
  checkpoint_every = 2
  fields = none
  particles = false
}}
"""


def external_deck(out):
    """The vacuum wake with a lower-gamma bunch through an undulator, a quadrupole, a plasma lens and a solenoid
    (reference src/external.hpp) along the run's 2 um of z."""
    text = wake_deck(out).replace("  gamma = 1000\n", "  gamma = 50\n", 1)
    return text + """undulator {
  period = 1.5 um
  K = 0.3
  z_start = 0.05 um
  periods = 1
  ramp_periods = 0
}
quadrupole {
  z_start = 0.3 um
  length = 0.5 um
  gradient = 2e5 T/m
}
plasma_lens {
  z_start = 0.85 um
  length = 0.4 um
  gradient = 3e5 T/m
  radius = 0.1 um
}
solenoid {
  z_start = 1.3 um
  length = 0.5 um
  field = 3e3 T
  ramp = 0.1 um
}
"""


def chicane_deck(out):
    """The two-bunch wake with an energy spread through a thin chicane inside the second step."""
    text = wake_deck(out).replace("  gamma = 1000\n", "  gamma = 1000\n  energy_spread = 0.01\n", 1)
    return text + f"""chicane {{
  z = {L(7)}
  r56 = {L(200)}
  delay = {L(2)}
  gamma = 990
}}
"""


def run(cmd, cwd):
    return subprocess.run(cmd, cwd=cwd, capture_output=True, text=True, timeout=600)


def read_checkpoint(path):
    """The arrays of a checkpoint file in the reference's layout (src/sim_checkpoint.cpp:9-58)."""
    from g3d import abi
    raw = open(path, "rb").read()
    pos = 128
    out = {}

    def take(dtype):
        nonlocal pos
        n = int(np.frombuffer(raw, "<u8", 1, pos)[0])
        pos += 8
        a = np.frombuffer(raw, dtype, n, pos)
        pos += n * np.dtype(dtype).itemsize
        return a
    for name in FIELDS + ["j0x", "j0y", "js0x", "js0y", "js0z"]:
        out[name] = take("<c16")
    out["F"] = take("<f4")
    out["particles"] = take(abi.PARTICLE_DTYPE)
    return out


def diag_rows(path):
    return np.array([[float(v) for v in line.split()] for line in open(path) if line.strip() and line[0] != "#"])


def bunches_rows(path):
    """bunches.txt as {species: rows of numbers (step, z, N, Q, ...)}"""
    out = {}
    for line in open(path):
        if not line.strip() or line[0] == "#":
            continue
        f = line.split()
        out.setdefault(f[2], []).append([float(v) for v in f[:2] + f[3:]])
    return {k: np.array(v) for k, v in out.items()}


def bunches_close(a, b, tag):
    assert sorted(a) == sorted(b), (tag, sorted(a), sorted(b))
    for k in a:
        x, y = a[k], b[k]
        assert x.shape == y.shape, (tag, k, x.shape, y.shape)
        tol = 3e-4 * np.maximum(np.abs(x), np.abs(y)) + 2e-5
        bad = np.argwhere(np.abs(x - y) > tol)
        assert len(bad) == 0, (tag, k, [(int(i), int(j), x[i, j], y[i, j]) for i, j in bad[:5]])


def diag_close(a, b, tag):
    """Every column to its printed digits: within a few units of the last digit of either side. With mobile ions both
    tables have a 22nd column, the largest ion density on the axis (the density lines of the plasma march)."""
    assert a.shape == b.shape and a.shape[1] in (21, 22), (tag, a.shape, b.shape)
    for i in range(a.shape[0]):
        for j in range(a.shape[1]):
            x, y = a[i, j], b[i, j]
            tol = 3e-4 * max(abs(x), abs(y)) + 2e-4       # the %10.4f columns and the %11.4e ones
            assert abs(x - y) <= tol, (tag, "row", i, "column", j, x, y)


@needs_both
def test_vacuum_wake_deck_matches_the_reference_cli(tmp_path):
    ref_dir, our_dir = tmp_path / "ref", tmp_path / "g3d"
    for d, exe in ((ref_dir, REF_CLI), (our_dir, SHIM)):
        d.mkdir()
        deck = d / "wake.deck"
        deck.write_text(wake_deck(d / "out"))
        env_cmd = [exe, str(deck)]
        r = run(env_cmd, d)
        assert r.returncode == 0, (exe, r.stdout[-2000:], r.stderr[-2000:])
        assert "done: 4 steps" in r.stdout or "done: 3 steps" in r.stdout, r.stdout[-500:]
    a = read_checkpoint(our_dir / "out" / "checkpoint_000003_r0000.bin")
    b = read_checkpoint(ref_dir / "out" / "checkpoint_000003_r0000.bin")
    assert_state({k: a[k] for k in FIELDS}, {k: b[k] for k in FIELDS}, FIELDS, 1e-10, tag="checkpoint")
    assert rel_l2(a["F"], b["F"]) <= 1e-6
    p, q = a["particles"], b["particles"]
    assert len(p) == len(q) == 26000 and set(np.unique(p["sp"])) == {0, -1}
    for f in ["x", "y", "zeta", "px", "py", "pz", "z"]:
        assert rel_l2(p[f], q[f]) <= 1e-10, f
    diag_close(diag_rows(our_dir / "out" / "diag.txt"), diag_rows(ref_dir / "out" / "diag.txt"), "wake")
    bunches_close(bunches_rows(our_dir / "out" / "bunches.txt"), bunches_rows(ref_dir / "out" / "bunches.txt"), "wake")


@needs_both
def test_laser_wakefield_deck_matches_the_reference_cli(tmp_path):
    ref_dir, our_dir = tmp_path / "ref", tmp_path / "g3d"
    for d, exe in ((ref_dir, REF_CLI), (our_dir, SHIM)):
        d.mkdir()
        deck = d / "lwfa.deck"
        deck.write_text(lwfa_deck(d / "out"))
        r = run([exe, str(deck)], d)
        assert r.returncode == 0, (exe, r.stdout[-2000:], r.stderr[-2000:])
    a, b = diag_rows(our_dir / "out" / "diag.txt"), diag_rows(ref_dir / "out" / "diag.txt")
    assert a.shape[0] >= 3 and a.shape[1] == 22 and np.all(a[1:, 21] > 0)      # no march before the first step
    diag_close(a, b, "lwfa")
    # the checkpoint after step 2, with the streaming plasma's state (written here while the run went on)
    ca = read_checkpoint(our_dir / "out" / "checkpoint_000002_r0000.bin")
    cb = read_checkpoint(ref_dir / "out" / "checkpoint_000002_r0000.bin")
    assert_state({k: ca[k] for k in FIELDS}, {k: cb[k] for k in FIELDS}, FIELDS, 1e-10, tag="checkpoint")
    for k in ("js0x", "js0y", "js0z"):
        assert rel_l2(ca[k], cb[k]) <= 1e-9, k
    assert rel_l2(ca["F"], cb["F"]) <= 1e-6
    assert len(ca["particles"]) == len(cb["particles"])
    bunches_close(bunches_rows(our_dir / "out" / "bunches.txt"), bunches_rows(ref_dir / "out" / "bunches.txt"), "lwfa")


@needs_both
def test_external_elements_deck_matches_the_reference_cli(tmp_path):
    """Undulator, quadrupole, plasma lens and solenoid fields in the push and its sub-steps ending on their
    breakpoints: the checkpoint after step 3 and diag.txt as for the plain wake."""
    ref_dir, our_dir = tmp_path / "ref", tmp_path / "g3d"
    for d, exe in ((ref_dir, REF_CLI), (our_dir, SHIM)):
        d.mkdir()
        deck = d / "ext.deck"
        deck.write_text(external_deck(d / "out"))
        r = run([exe, str(deck)], d)
        assert r.returncode == 0, (exe, r.stdout[-2000:], r.stderr[-2000:])
    a = read_checkpoint(our_dir / "out" / "checkpoint_000003_r0000.bin")
    b = read_checkpoint(ref_dir / "out" / "checkpoint_000003_r0000.bin")
    assert_state({k: a[k] for k in FIELDS}, {k: b[k] for k in FIELDS}, FIELDS, 1e-10, tag="checkpoint")
    p, q = a["particles"], b["particles"]
    assert len(p) == len(q)
    for f in ["x", "y", "zeta", "px", "py", "pz", "z"]:
        assert rel_l2(p[f], q[f]) <= 1e-10, f
    diag_close(diag_rows(our_dir / "out" / "diag.txt"), diag_rows(ref_dir / "out" / "diag.txt"), "external")


@needs_both
def test_chicane_deck_matches_the_reference_cli(tmp_path):
    """A thin chicane passed in step 2: the beam moved in zeta by its energy, its co-moving field traded, E_z, B_z, L
    and the real fields rebuilt; the checkpoint after step 3 and diag.txt as for the plain wake."""
    ref_dir, our_dir = tmp_path / "ref", tmp_path / "g3d"
    for d, exe in ((ref_dir, REF_CLI), (our_dir, SHIM)):
        d.mkdir()
        deck = d / "chicane.deck"
        deck.write_text(chicane_deck(d / "out"))
        r = run([exe, str(deck)], d)
        assert r.returncode == 0, (exe, r.stdout[-2000:], r.stderr[-2000:])
    a = read_checkpoint(our_dir / "out" / "checkpoint_000003_r0000.bin")
    b = read_checkpoint(ref_dir / "out" / "checkpoint_000003_r0000.bin")
    assert_state({k: a[k] for k in FIELDS}, {k: b[k] for k in FIELDS}, FIELDS, 1e-10, tag="checkpoint")
    p, q = a["particles"], b["particles"]
    assert len(p) == len(q)
    for f in ["x", "y", "zeta", "px", "py", "pz", "z"]:
        assert rel_l2(p[f], q[f]) <= 1e-10, f
    diag_close(diag_rows(our_dir / "out" / "diag.txt"), diag_rows(ref_dir / "out" / "diag.txt"), "chicane")
