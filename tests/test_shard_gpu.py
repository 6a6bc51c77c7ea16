"""A sharded run against the whole window on one device: two and three ranks (processes on one GPU, gloo, so the
collectives are host copies and no kernel waits on another rank), each holding a zeta slab, against a one-rank run of
the same particles in every rank's own context.

Expected: the real fields of every slab (its ns slices and the two ghost slices b, b + 1) and the spectra of every slab
equal the one-rank run's planes a .. b-1 to 1e-12 of the field state (the deposit is exact integer arithmetic with a
global scale, the march of a mode is the same arithmetic on the pencil; only the beta sums of the start field and the
diagnostics add per-rank partial sums, a rounding apart from the one-rank sums), every particle (matched by id) to
1e-12, the union of the ranks' particles the one-rank list, and the diagnostics to 1e-12. The window is cut inside
the bunch, and a bunch of gamma 10 drifts back across the cut, so particles are handed to the rank below and finish
their push there."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

SPECTRA = ["Rx", "Ry", "Ez", "Bz", "Lx", "Ly"]
HALF = ["jkx", "jky", "jkz"]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _cases():
    from g3d import configs
    return {
        # a witness bunch of gamma 10 across the cut, in a grid laser (no sponge, fixed window)
        "laser_bunch": configs.adjoint_small(nx=16, ny=16, nzeta=64, nmacro=4000, steps=4, gamma=10.0),
        # the oblique plane wave on a bunch of workload 2 at test size (sponge, window following the bunch)
        "oblique16": configs.config2(nx=16, ny=16, nzeta=48, nmacro=4000, steps=3, envelope=0),
    }


def _rank(rank, world, port, name, mode, out):
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(repo, "gem-pic-3d_b200"))
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    if mode == "transpose":
        os.environ["G3D_SHARD_TRANSPOSE"] = "1"
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        from g3d import Simulation, shard
        from g3d.sim import sample_bunches
        cfg = _cases()[name]
        parts, _, _, _ = sample_bunches(cfg)
        parts["id"] = np.arange(1, len(parts) + 1)
        N, nk = cfg.nzeta, cfg.nx * cfg.ny
        a, b, _, _ = shard.layout(N, cfg.ny * (cfg.nx // 2 + 1), rank, world)
        ns = b - a
        z = cfg.zeta
        nxt = shard.layout(N, cfg.ny * (cfg.nx // 2 + 1), rank + 1, world)[0] if rank < world - 1 else None
        lo = z[a + 1] if rank > 0 else -np.inf
        hi = z[nxt + 1] if nxt is not None else np.inf
        full = Simulation(cfg)
        full.set_particles(parts)
        comm = shard.RankComm(device="cuda:0")
        sh = Simulation(cfg, comm=comm)
        sh.set_particles(parts[(parts["zeta"] >= lo) & (parts["zeta"] < hi)])
        np0 = sh.status().np
        full.init_fields()
        sh.init_fields()
        sh.profile(True)
        res = []
        for step in range(cfg.steps + 1):
            if step:
                full.step()
                sh.step()
            err = {}
            fs = {n: full.array(n).reshape(N, nk) for n in SPECTRA}
            ss = {n: sh.array(n).reshape(ns, nk) for n in SPECTRA}
            norm = np.sqrt(sum(np.linalg.norm(fs[n]) ** 2 for n in SPECTRA))
            err["spectra"] = max(np.linalg.norm(ss[n] - fs[n][a:b]) for n in SPECTRA) / norm
            fj = {n: full.array(n).reshape(N + 1, nk) for n in HALF}
            sj = {n: sh.array(n).reshape(ns + 1, nk) for n in HALF}
            jn = np.sqrt(sum(np.linalg.norm(fj[n]) ** 2 for n in HALF))
            err["currents"] = max(np.linalg.norm(sj[n] - fj[n][a:b + 1]) for n in HALF) / max(jn, 1e-300)
            F = full.array("F").reshape(6, N + 2, nk)
            Fs = sh.array("F").reshape(6, ns + 2, nk)
            err["F"] = float(np.abs(Fs - F[:, a:b + 2]).max() / max(np.abs(F).max(), 1e-300))
            p_full = full.host_particles()
            p_full = p_full[p_full["alive"] == 1]
            p_sh = sh.host_particles()
            p_sh = p_sh[p_sh["alive"] == 1]
            ids = dist_all_ids(dist, p_sh["id"])
            err["ids_match"] = bool(np.array_equal(np.sort(ids), np.sort(p_full["id"])))
            ref = {int(i): k for k, i in enumerate(p_full["id"])}
            idx = np.array([ref[int(i)] for i in p_sh["id"]], dtype=np.int64)
            e = 0.0
            for f in ("x", "y", "zeta", "px", "py", "pz"):
                e = max(e, float(np.abs(p_sh[f] - p_full[f][idx]).max(initial=0.0) /
                                 max(np.abs(p_full[f]).max(initial=0.0), 1e-300)))
            err["particles"] = e
            own = (p_sh["zeta"] >= lo) & (p_sh["zeta"] < hi)
            err["owned"] = bool(own.all())
            d_full, d_sh = full.diagnostics_sums(), sh.diagnostics_sums()
            err["diag"] = max(abs(d_sh[k] - d_full[k]) / max(abs(d_full[k]), 1e-300) for k in range(16))
            res.append(err)
        out[rank] = (res, np0, sh.status().np, comm.calls, sorted(sh.profile_results()))
        full.close()
        sh.close()
    finally:
        dist.destroy_process_group()


def dist_all_ids(dist, ids):
    got = [None] * dist.get_world_size()
    dist.all_gather_object(got, np.asarray(ids).tolist())
    return np.concatenate([np.asarray(g, dtype=np.int64) for g in got])


@pytest.mark.parametrize("name,world,mode", [("laser_bunch", 2, "peer"), ("laser_bunch", 3, "peer"), ("oblique16", 2, "peer"),
                                             ("laser_bunch", 2, "transpose"), ("laser_bunch", 3, "transpose")])
def test_sharded_run_matches_the_whole_window(name, world, mode):
    """mode peer: the march reads and writes the other ranks' slabs through CUDA IPC mappings (one fused kernel);
    transpose (G3D_SHARD_TRANSPOSE): the all-to-all transposes around the pencil march."""
    port = _free_port()
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_rank, args=(world, port, name, mode, out), nprocs=world, start_method="spawn", join=True)
    handed = 0
    for r in range(world):
        res, np0, np_end, calls, kernels = out[r]
        if mode == "peer":
            assert "march_peer" in kernels and "shard_transpose" not in kernels, kernels
        else:
            assert "shard_transpose" in kernels and "march_peer" not in kernels, kernels
        handed += max(0, np0 - np_end) if r > 0 else 0
        assert calls > 0
        for s, e in enumerate(res):
            assert e["ids_match"] and e["owned"], (r, s, e)
            assert e["spectra"] <= 1e-12 and e["currents"] <= 1e-12, (r, s, e)
            assert e["F"] <= 1e-6, (r, s, e)
            assert e["particles"] <= 1e-12 and e["diag"] <= 1e-12, (r, s, e)
        print(name, world, r, res[-1], np0, np_end)
    if name == "laser_bunch":
        assert handed > 0, "no particle crossed a cut: the handover is untested"
