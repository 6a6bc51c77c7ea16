"""The drop-in boundary: libg3d.so loads without a GPU, exports every entry point include/g3d.h declares,
and its records have the C layout (checked against gcc's offsetof). No compute call needs a device here."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import REPO

HEADER = os.path.join(REPO, "include", "g3d.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^[A-Za-z_][\w\s\*]*?\b(g3d_\w+)\(", text, flags=re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ["g3d_create", "g3d_destroy", "g3d_step", "g3d_init", "g3d_solve_fields", "g3d_march", "g3d_currents",
                 "g3d_push", "g3d_diagnostics", "g3d_write_checkpoint", "g3d_read_checkpoint", "g3d_last_error"]:
        assert must in names


def test_library_exports_every_declared_symbol():
    from g3d import abi
    lib = abi.load_library()
    names = declared_functions()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    bound = {n for n, _, _ in abi.SIGNATURES}
    assert set(names) == bound, set(names) ^ bound
    out = subprocess.run(["nm", "-D", "--defined-only", abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (g3d_\w+)", out))
    assert set(names) <= exported


def test_array_ids_match_the_header():
    """The Python mirror's array names map to the ids include/g3d.h defines, and cover all of them."""
    from g3d import abi
    text = open(HEADER).read()
    ids = {m.group(1): int(m.group(2)) for m in re.finditer(r"^#define G3D_A_(\w+)\s+(\d+)", text, flags=re.M)}
    count = ids.pop("COUNT")
    assert sorted(abi.ARRAYS.values()) == sorted(ids.values()) == list(range(count))
    names = {"RX": "Rx", "RY": "Ry", "EZ": "Ez", "BZ": "Bz", "LX": "Lx", "LY": "Ly", "J0X": "j0x", "J0Y": "j0y",
             "JKX": "jkx", "JKY": "jky", "JKZ": "jkz", "JW": "jw", "F": "F", "RHO_E": "rho_lines", "RHO_I": "rho_lines_i"}
    assert {names[k]: v for k, v in ids.items()} == abi.ARRAYS


def test_version_string():
    from g3d import abi
    assert b"sm_100a" in abi.load_library().g3d_version()


def test_records_match_the_c_layout(tmp_path):
    """Offsets of every field of the ctypes mirrors against the C compiler's."""
    from g3d import abi
    structs = {"g3d_grid": abi.Grid, "g3d_params": abi.Params, "g3d_bunch": abi.Bunch, "g3d_status": abi.Status}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "g3d.h"', "int main(void){"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    for f in abi.PARTICLE_DTYPE.names:
        lines.append(f'printf("g3d_particle.{f} %zu\\n", offsetof(g3d_particle, {f}));')
    lines.append('printf("g3d_particle %zu\\n", sizeof(g3d_particle)); return 0;}')
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(py, f).offset, (cname, f)
    for f in abi.PARTICLE_DTYPE.names:
        assert int(got[f"g3d_particle.{f}"]) == abi.PARTICLE_DTYPE.fields[f][1], f
    assert int(got["g3d_particle"]) == 104


def test_create_reports_missing_device_or_bad_grid():
    """Without a device g3d_create returns G3D_ERR_NODEV with a message; with one, a bad grid is G3D_ERR_ARG."""
    from g3d import abi, configs
    lib = abi.load_library()
    cfg = configs.config1(nx=16, ny=16, nzeta=8, nmacro=10)
    cfg.nx = 12                                 # neither a power of two in 8..512 nor three times one in 24..384
    g, z = cfg.grid_struct()
    p = cfg.params_struct()
    h = C.c_void_p()
    rc = lib.g3d_create(C.byref(g), C.byref(p), C.byref(h))
    assert rc in (abi.G3D_ERR_NODEV, abi.G3D_ERR_ARG)
    assert lib.g3d_last_error(None)
    assert not h.value


def test_sample_bunches_matches_the_reference_loader(golden):
    """The host bunch sampler reproduces the reference's particles bit for bit (same libstdc++ generators)."""
    from g3d import configs, sample_bunches
    for name, cfg in [("wake16", configs.config1(nx=16, ny=16, nzeta=32, nmacro=3000, steps=2)),
                      ("oblique16", configs.config2(nx=16, ny=16, nzeta=48, nmacro=4000, steps=2, envelope=0))]:
        ref = golden(name)["loaded_particles"]
        got, lost, x0, y0 = sample_bunches(cfg)
        assert len(got) == len(ref)
        for f in ref.dtype.names:
            assert np.array_equal(got[f], ref[f]), (name, f)
        assert x0 == -0.5 * cfg.Lx and y0 == -0.5 * cfg.Ly


def test_sample_bunches_rejects_bad_input():
    from g3d import G3DError, configs, sample_bunches
    cfg = configs.config1(nx=16, ny=16, nzeta=32, nmacro=10)
    cfg.bunches[0]["gamma"] = 0.5
    with pytest.raises(G3DError):
        sample_bunches(cfg)


def test_march_objective_checks_its_tensors_before_any_device_work():
    """The autograd wrapper of the adjoint march rejects mis-shaped inputs on the host, before a context is made."""
    import torch
    from g3d import configs
    from g3d.autograd import MarchObjective
    cfg = configs.config1(nx=16, ny=16, nzeta=32, nmacro=10, steps=1)
    dp = torch.zeros(10, 3, dtype=torch.float64)
    with pytest.raises(ValueError, match=r"coef must be \[16, 9, 2\]"):
        MarchObjective.apply(torch.zeros(16, 16, 2, dtype=torch.float64), dp, cfg)
    with pytest.raises(ValueError, match=r"coef must be"):
        MarchObjective.apply(torch.zeros(16, 9, dtype=torch.float64), dp, cfg)


@pytest.mark.parametrize("beamlet", [4, 7])
def test_fawley_beamlets_match_the_reference_loader(beamlet):
    """Shot noise by Fawley's beamlets (Phys. Rev. ST Accel. Beams 5, 070701 (2002); the deck's shot_noise = fawley):
    the host sampler, without a device, against the reference build's loader, bit for bit."""
    ref = pytest.importorskip("ref")
    if not ref.available():
        pytest.skip("reference build oracle/_ref not present")
    from g3d import configs, sample_bunches
    cfg = configs.config2(nx=16, ny=16, nzeta=48, nmacro=4200, steps=2, envelope=0)
    cfg.bunches[0].update(beamlet=beamlet, noise_lambda=0.35)
    got, lost, _, _ = sample_bunches(cfg)
    r = ref.RefSimulation(cfg, threads=1)
    r.load_bunch()
    want = r.host_particles()
    r.close()
    assert len(got) == len(want) > 4000 - 200
    for f in want.dtype.names:
        assert np.array_equal(got[f], want[f]), f
    # the groups: each draws one position and momentum, M phases spread over the wavelength
    z = got["zeta"][:beamlet]
    assert np.all(got["px"][:beamlet] == got["px"][0]) and np.ptp(z) > 0


def test_fawley_beamlets_need_a_divisible_count():
    from g3d import G3DError, configs, sample_bunches
    cfg = configs.config1(nx=16, ny=16, nzeta=32, nmacro=1001)
    cfg.bunches[0].update(beamlet=4, noise_lambda=0.5)
    with pytest.raises(G3DError):
        sample_bunches(cfg)
