"""Failure paths of the C-ABI, made on the host: a missing, truncated or foreign checkpoint file gives G3D_ERR_IO and
leaves the context usable; a list of freed electrons capped below what the ionization frees gives G3D_ERR_CAPACITY
(the device's bounds check raises a flag that the host turns into the status); bad arguments give G3D_ERR_ARG.
No test faults, traps or hangs the GPU: every failing write is skipped by a bounds check."""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import REPO, rel_l2

pytestmark = pytest.mark.gpu

G3D_ERR_TIMEOUT, G3D_ERR_CAPACITY, G3D_ERR_ARG, G3D_ERR_IO = 2, 3, 4, 6


def small():
    from g3d import configs
    return configs.config1(nx=16, ny=16, nzeta=32, nmacro=3000, steps=2)


def test_checkpoint_failures_give_io_errors(tmp_path):
    from g3d import G3DError, Simulation
    sim = Simulation(small())
    sim.init()
    sim.step()
    good = tmp_path / "ckpt.bin"
    sim.write_checkpoint(good)
    data = good.read_bytes()
    cases = {
        "missing": None,
        "truncated header": data[:64],
        "truncated arrays": data[: len(data) // 2],
        "foreign magic": b"NOTACKPT" + data[8:],
    }
    for name, blob in cases.items():
        path = tmp_path / f"{name.replace(' ', '_')}.bin"
        if blob is not None:
            path.write_bytes(blob)
        with pytest.raises(G3DError) as e:
            sim.read_checkpoint(path)
        assert e.value.code == G3D_ERR_IO, (name, e.value)
    # the context still works after the failed reads: the good file restores the state, the next step matches
    other = Simulation(small())
    other.read_checkpoint(good)
    before = sim.array("Rx")
    sim.read_checkpoint(good)
    assert np.array_equal(sim.array("Rx"), before)
    sim.step(); other.step()
    assert rel_l2(sim.array("Rx"), other.array("Rx")) == 0.0
    sim.close(); other.close()


def test_checkpoint_of_another_grid_is_refused(tmp_path):
    from g3d import G3DError, Simulation, configs
    a = Simulation(small())
    a.init()
    path = tmp_path / "a.bin"
    a.write_checkpoint(path)
    b = Simulation(configs.config1(nx=16, ny=16, nzeta=48, nmacro=3000, steps=2))
    with pytest.raises(G3DError) as e:
        b.read_checkpoint(path)
    assert e.value.code == G3D_ERR_IO and "differ" in str(e.value)
    a.close(); b.close()


def test_bad_arguments_give_arg_errors():
    import ctypes as C
    from g3d import G3DError, Simulation
    sim = Simulation(small())
    with pytest.raises(G3DError) as e:
        sim._c(sim.lib.g3d_get_array(sim.ctx, 99, None, 0))        # no array 99
    assert e.value.code == G3D_ERR_ARG
    n = C.c_int64()
    sim.load_bunch()
    rc = sim.lib.g3d_get_particles(sim.ctx, None, 0, C.byref(n))
    assert rc == G3D_ERR_CAPACITY and n.value == 3000
    sim.close()


CAPACITY_SCRIPT = r"""
import sys
sys.path.insert(0, sys.argv[1])
from g3d import G3DError, Simulation, configs
cfg = configs.ionization_small()
sim = Simulation(cfg)
sim.init()
try:
    sim.step()
except G3DError as e:
    print("code", e.code, str(e))
    sys.exit(0)
print("no error")
"""


def test_freed_electron_overflow_gives_capacity_error():
    """With the list of freed electrons capped at one slot the first ionizing step overflows it: the march skips
    the writes past the end, raises the device flag, and the step returns G3D_ERR_CAPACITY. Run in a child process,
    since the cap is read from its environment."""
    env = dict(os.environ, G3D_BORN_CAPACITY_LIMIT="1")
    out = subprocess.run([sys.executable, "-c", CAPACITY_SCRIPT, os.path.join(REPO, "gem-pic-3d_b200")], env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    assert f"code {G3D_ERR_CAPACITY}" in out.stdout and "overflowed" in out.stdout, out.stdout


TIMEOUT_SCRIPT = r"""
import sys
sys.path.insert(0, sys.argv[1])
from g3d import G3DError, Simulation, configs
cfg = configs.config2(nx=16, ny=16, nzeta=32, nmacro=2000, steps=1, envelope=0)
sim = Simulation(cfg)
try:
    sim.init()
    print("no error")
except G3DError as e:
    print("code", e.code, str(e))
sim.close()
"""


def test_tma_tile_wait_that_runs_out_gives_timeout():
    """The TMA column kernels wait for their tiles on an mbarrier with a bounded number of polls. With the barrier
    told to expect 16 bytes more than the tiles bring (G3D_TMA_EXTRA_BYTES, read at creation) its phase never
    completes: every wait gives up after G3D_TMA_POLLS polls, sets the error word and returns, and the call reports
    G3D_ERR_TIMEOUT. The tiles themselves land (no copy is left in flight) and the GPU stays usable: a context made
    afterwards in this process, without the settings, runs the same start field and step."""
    env = dict(os.environ, G3D_TMA_EXTRA_BYTES="16", G3D_TMA_POLLS="2000")
    out = subprocess.run([sys.executable, "-c", TIMEOUT_SCRIPT, os.path.join(REPO, "gem-pic-3d_b200")], env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    assert f"code {G3D_ERR_TIMEOUT}" in out.stdout and "bounded wait" in out.stdout, out.stdout
    from g3d import Simulation, configs
    sim = Simulation(configs.config2(nx=16, ny=16, nzeta=32, nmacro=2000, steps=1, envelope=0))
    sim.init()
    sim.step()
    sim.close()
