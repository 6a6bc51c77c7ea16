"""The zeta-slab / mode-pencil partition of a sharded run on CPU: the layout against the reference's split of the
slices (src/sim_setup.cpp:9-15), and the library's own transpose plans (g3d_shard_transpose_plan) driven over gloo
ranks by the same RankComm the GPU path uses, on the field planes of a reference run (the oblique16 golden state),
which every rank must get back exactly: the pencils are the whole window's modes of the rank, the slabs after the
return trip the whole window's slices. No GPU: the plan's copies run in numpy on host buffers."""
import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import GOLDEN


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_layout_is_the_reference_split():
    from g3d import shard
    for N, P in ((48, 2), (49, 3), (1024, 8), (2048, 7), (13, 3)):
        a = 0
        for r in range(P):
            ns = N // P + (1 if r < N % P else 0)          # rank P-1 at the front of the window
            got = shard.layout(N, 144, r, P)
            assert got[:2] == (a, a + ns)
            a += ns
        m = 0
        for q in range(P):
            mq = 144 // P + (1 if q < 144 % P else 0)
            assert shard.layout(N, 144, q, P)[2:] == (m, m + mq)
            m += mq
    from g3d.sim import G3DError
    with pytest.raises(G3DError, match="at least 4 slices"):
        shard.layout(15, 144, 0, 4)
    assert shard.layout(7, 144, 0, 1) == (0, 7, 0, 144)


def _half(full, planes, nx, ny):
    """The stored half spectrum [plane][j][k_x <= nx/2] of the reference's full spectra [plane][j][i]."""
    return np.ascontiguousarray(full.reshape(planes, ny, nx)[:, :, : nx // 2 + 1].reshape(planes, -1))


class _HostComm:
    """RankComm on host buffers: the plan's pointers are numpy arrays here, not device memory."""

    @staticmethod
    def make(group=None):
        from g3d import shard
        import torch

        class HostComm(shard.RankComm):
            def __init__(self):
                super().__init__(group, device="cpu")

            def _view(self, ptr, nbytes):
                if nbytes == 0:
                    return torch.empty(0, dtype=torch.uint8)
                return torch.frombuffer((C.c_uint8 * nbytes).from_address(ptr), dtype=torch.uint8)

            def _sync(self):
                pass
        return HostComm()


def _run_plan(plan, arrays, buf, to_buf):
    """The copies of a plan: arrays[k] and buf are flat complex128 numpy arrays (element offsets)."""
    for b in plan:
        src = buf if b["src_array"] < 0 else arrays[b["src_array"]]
        dst = buf if b["dst_array"] < 0 else arrays[b["dst_array"]]
        for r in range(b["rows"]):
            s0, d0 = b["src"] + r * b["src_stride"], b["dst"] + r * b["dst_stride"]
            dst[d0:d0 + b["cols"]] = src[s0:s0 + b["cols"]]


def _rank(rank, world, port, out):
    import datetime
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(repo, "gem-pic-3d_b200"))
    import torch.distributed as dist
    from g3d import abi, shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        g = np.load(os.path.join(GOLDEN, "oblique16.npz"))
        nx = ny = 16
        N = 48
        nkh = ny * (nx // 2 + 1)
        node = {n: _half(g[f"step2_{n}"], N, nx, ny) for n in ("Rx", "Ry", "Ez", "Bz")}
        half = {n: _half(g[f"step2_{n}"], N + 1, nx, ny) for n in ("jkx", "jky", "jkz")}
        a, b, m0, m1 = shard.layout(N, nkh, rank, world)
        ns, mq = b - a, m1 - m0
        names = ["Rx", "Ry", "Ez", "Bz", "jkx", "jky", "jkz"]
        kinds = [abi.G3D_SLAB_NODES] * 4 + [abi.G3D_SLAB_HALF] * 3
        # this rank's slab arrays: ns node planes, ns + 1 half-cell planes (a - 1/2 .. b - 1/2)
        slab = [np.ascontiguousarray(node[n][a:b]).ravel() for n in names[:4]]
        slab += [np.ascontiguousarray(half[n][a:b + 1]).ravel() for n in names[4:]]
        comm = _HostComm.make()
        plan = shard.transpose_plan(N, nkh, rank, world, kinds, True, 16)
        send = np.zeros(max(1, sum(plan["send_bytes"]) // 16), dtype=np.complex128)
        recv = np.zeros(max(1, sum(plan["recv_bytes"]) // 16), dtype=np.complex128)
        _run_plan(plan["pack"], slab, send, True)
        assert comm._call(None, C.pointer(abi.CommOp(op=abi.G3D_COMM_ALLTOALL, send=send.ctypes.data,
                                                     send_bytes=(C.c_int64 * world)(*plan["send_bytes"]),
                                                     recv=recv.ctypes.data,
                                                     recv_bytes=(C.c_int64 * world)(*plan["recv_bytes"])))) == 0, comm.error
        pen = [np.full(N * mq, np.nan + 0j) for _ in range(4)] + [np.full((N + 1) * mq, np.nan + 0j) for _ in range(3)]
        _run_plan(plan["unpack"], pen, recv, False)
        ok_in = all(np.array_equal(pen[k].reshape(-1, mq), (node[n] if k < 4 else half[n])[:, m0:m1])
                    for k, n in enumerate(names))
        # back: the node arrays of the pencil to the slabs
        back = shard.transpose_plan(N, nkh, rank, world, kinds[:4], False, 16)
        send = np.zeros(max(1, sum(back["send_bytes"]) // 16), dtype=np.complex128)
        recv = np.zeros(max(1, sum(back["recv_bytes"]) // 16), dtype=np.complex128)
        _run_plan(back["pack"], pen[:4], send, True)
        comm.all_to_all(send.ctypes.data, back["send_bytes"], recv.ctypes.data, back["recv_bytes"])
        slab2 = [np.full(ns * nkh, np.nan + 0j) for _ in range(4)]
        _run_plan(back["unpack"], slab2, recv, False)
        ok_back = all(np.array_equal(slab2[k].reshape(ns, nkh), node[n][a:b]) for k, n in enumerate(names[:4]))
        # sums in place: doubles and 64-bit integers
        v = np.array([rank + 0.5, 2.0 ** -40 * rank], dtype=np.float64)
        comm.sum(v.ctypes.data, 2, abi.G3D_SUM_F64)
        iv = np.array([rank + 1, (1 << 50) * rank], dtype=np.int64)
        comm.sum(iv.ctypes.data, 2, abi.G3D_SUM_I64)
        out[rank] = (ok_in, ok_back, v.tolist(), iv.tolist(), (a, b, m0, m1))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_transposes_move_the_reference_planes_exactly(world):
    port = _free_port()
    out = mp.get_context("spawn").Manager().dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, start_method="spawn", join=True)
    W = range(world)
    for r in W:
        ok_in, ok_back, v, iv, lay = out[r]
        assert ok_in, f"rank {r}: the pencil differs from the window's modes {lay[2]}..{lay[3]}"
        assert ok_back, f"rank {r}: the slab after the return trip differs from the window's slices {lay[0]}..{lay[1]}"
        assert v == [sum(q + 0.5 for q in W), sum(2.0 ** -40 * q for q in W)]
        assert iv == [sum(q + 1 for q in W), sum((1 << 50) * q for q in W)]
    assert out[0][4][0] == 0 and out[world - 1][4][1] == 48
    assert all(out[r][4][1] == out[r + 1][4][0] for r in range(world - 1))


def test_plan_blocks_cover_every_plane_once():
    """Every (plane, mode) of the window is written exactly once on some pencil, for uneven splits too."""
    from g3d import abi, shard
    N, nkh = 49, 144
    for P in (2, 3, 5):
        cover = np.zeros((N + 1, nkh), dtype=int)
        for q in range(P):
            _, _, m0, m1 = shard.layout(N, nkh, q, P)
            plan = shard.transpose_plan(N, nkh, q, P, [abi.G3D_SLAB_HALF], True, 16)
            mq = m1 - m0
            for b in plan["unpack"]:
                assert b["dst_stride"] == mq and b["cols"] == mq
                p0 = b["dst"] // mq
                cover[p0:p0 + b["rows"], m0:m1] += 1
        assert (cover == 1).all(), P
    from g3d.sim import G3DError
    with pytest.raises(G3DError, match="unknown array kind"):
        shard.transpose_plan(N, nkh, 0, 2, [7], True, 16)
