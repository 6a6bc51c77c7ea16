"""Asynchronous checkpoints (g3d_write_checkpoint_async, no counterpart in the reference): the file a host thread of
the library writes while the run goes on is, byte for byte, the synchronous checkpoint of the same state (the
reference's format), for a run with a streaming plasma and particles waiting to join it (FP64) and for the mixed
form's narrow storage; a write that fails reports G3D_ERR_IO at the wait and leaves the context usable."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run_and_compare(cfg, tmp_path, precision="fp64", before=2, after=2):
    from g3d import Simulation
    s = Simulation(cfg, precision=precision)
    s.load_bunch()
    s.init()
    for _ in range(before):
        s.step()
    a, b = tmp_path / "sync.ckpt", tmp_path / "async.ckpt"
    s.write_checkpoint(a)
    s.write_checkpoint_async(b)
    for _ in range(after):            # the state changes while the file is written
        s.step_async()
    s.checkpoint_wait()
    s.close()
    da, db = a.read_bytes(), b.read_bytes()
    assert len(da) == len(db) and da == db


def test_async_checkpoint_with_plasma_and_joining_particles(tmp_path):
    from g3d import configs
    cfg = configs.adjoint_plasma_small(a0=1.0, steps=4)        # electrons trapped each step wait for the next march
    run_and_compare(cfg, tmp_path)


def test_async_checkpoint_of_the_mixed_form(tmp_path):
    from g3d import configs
    cfg = configs.config1(nx=32, ny=32, nzeta=64, nmacro=20000, steps=4)
    run_and_compare(cfg, tmp_path, precision="mixed")


def test_async_checkpoint_write_error_is_reported_at_the_wait(tmp_path):
    from g3d import G3DError, Simulation, configs, abi
    cfg = configs.config1(nx=16, ny=16, nzeta=32, nmacro=3000, steps=2)
    s = Simulation(cfg)
    s.load_bunch()
    s.init()
    s.write_checkpoint_async(tmp_path / "no_such_dir" / "x.ckpt")
    s.step()
    with pytest.raises(G3DError) as e:
        s.checkpoint_wait()
    assert e.value.code == abi.G3D_ERR_IO
    s.write_checkpoint(tmp_path / "ok.ckpt")                  # the context goes on
    s.step()
    s.close()
    assert (tmp_path / "ok.ckpt").stat().st_size > 0
