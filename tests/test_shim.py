"""g3d_run without a device: --check reads a deck through the reference's deck and Config layers and maps it onto the
C-ABI structs (g3dshim::setup_from) without creating a context, and a deck asking for what libg3d does not run is
refused there, with the key, before any device work (exit code 2, as the reference's command line exits on an
error)."""
import os
import subprocess

import pytest

from test_shim_gpu import L, SHIM, chicane_deck, external_deck, lwfa_deck, wake_deck

needs_shim = pytest.mark.skipif(not os.path.exists(SHIM), reason="g3d_run not built (it needs the reference's sources)")


def check(text, tmp_path):
    deck = tmp_path / "t.deck"
    deck.write_text(text)
    return subprocess.run([SHIM, str(deck), "--check"], capture_output=True, text=True, timeout=120)


@needs_shim
@pytest.mark.parametrize("which", ["wake", "lwfa"])
def test_supported_decks_map(which, tmp_path):
    r = check((wake_deck if which == "wake" else lwfa_deck)(tmp_path / "out"), tmp_path)
    assert r.returncode == 0, r.stderr
    assert "march: libg3d" in r.stdout and "FP64 form" in r.stdout
    assert not (tmp_path / "out").exists()             # --check runs nothing


@needs_shim
@pytest.mark.parametrize("extra,key", [
    ("  ux_function = 0.001\n", "profile functions"),
])
def test_what_the_library_does_not_run_is_refused(extra, key, tmp_path):
    text = wake_deck(tmp_path / "out").replace("  seed = 3\n", "  seed = 3\n" + extra, 1)
    r = check(text, tmp_path)
    assert r.returncode == 2 and "libg3d does not run" in r.stderr and key in r.stderr, (r.stdout[-500:], r.stderr)


@needs_shim
def test_a_plasma_density_function_is_refused(tmp_path):
    text = lwfa_deck(tmp_path / "out").replace("  ppc_y = 2\n", "  ppc_y = 2\n  density_function = 1 + 0.1 * r\n", 1)
    r = check(text, tmp_path)
    assert r.returncode == 2 and "libg3d does not run" in r.stderr and "density_function" in r.stderr, r.stderr


@needs_shim
def test_fawley_shot_noise_maps(tmp_path):
    text = wake_deck(tmp_path / "out").replace("  seed = 3\n", f"  seed = 3\n  shot_noise = fawley\n  noise_wavelength = {L(1)}\n", 1)
    r = check(text, tmp_path)
    assert r.returncode == 0 and "fawley" in r.stdout, r.stderr


@needs_shim
def test_external_elements_map(tmp_path):
    r = check(external_deck(tmp_path / "out"), tmp_path)
    assert r.returncode == 0, r.stderr
    for name in ("undulator", "quadrupole", "plasma lens", "solenoid"):
        assert name in r.stdout, name


@needs_shim
def test_chicanes_map(tmp_path):
    r = check(chicane_deck(tmp_path / "out"), tmp_path)
    assert r.returncode == 0 and "chicane at z" in r.stdout, r.stderr
