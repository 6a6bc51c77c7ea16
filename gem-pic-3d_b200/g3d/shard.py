"""Sharded runs: the zeta slabs and mode pencils of libg3d (g3d_set_ranks) over torch.distributed.

The library does no communication of its own. It asks its caller for two collectives over device buffers
(struct g3d_comm_op): a sum in place (doubles or 64-bit integers) and an all-to-all with byte counts per rank.
RankComm answers them on a torch.distributed process group: with NCCL directly on tensors that alias the
library's device buffers, with other backends (gloo) through host copies. One process per GPU, every rank
driving its own Simulation with the same calls in the same order (the reference runs one MPI rank per GPU,
src/comm.hpp:11-46).
"""
import ctypes as C

import torch
import torch.distributed as dist

from . import abi


def layout(nzeta, nkh, rank, world, lib=None):
    """(a, b, m0, m1): the slab [a, b) of the slices and the pencil [m0, m1) of the stored modes of `rank`."""
    lib = lib or abi.load_library()
    out = (C.c_int64 * 4)()
    rc = lib.g3d_shard_layout(nzeta, nkh, rank, world, out)
    if rc != abi.G3D_OK:
        from .sim import G3DError
        raise G3DError(rc, lib.g3d_last_error(None).decode(errors="replace"))
    return tuple(int(v) for v in out)


def transpose_plan(nzeta, nkh, rank, world, kinds, to_pencil, elem_bytes, lib=None):
    """The copies and byte counts of one slab <-> pencil transpose on `rank` (g3d_shard_transpose_plan): a dict of
    `pack` and `unpack` (lists of dicts of the g3d_block fields), `send_bytes` and `recv_bytes` (lists per rank)."""
    lib = lib or abi.load_library()
    K = len(kinds)
    kv = (C.c_int32 * K)(*kinds)
    cap = 4 * K * world + 4
    pack, unpack = (abi.Block * cap)(), (abi.Block * cap)()
    npk, nun = C.c_int32(), C.c_int32()
    sb, rb = (C.c_int64 * world)(), (C.c_int64 * world)()
    rc = lib.g3d_shard_transpose_plan(nzeta, nkh, rank, world, kv, K, 1 if to_pencil else 0, elem_bytes, pack, cap,
                                      C.byref(npk), unpack, cap, C.byref(nun), sb, rb)
    if rc != abi.G3D_OK:
        from .sim import G3DError
        raise G3DError(rc, lib.g3d_last_error(None).decode(errors="replace"))
    blk = lambda b: {f: getattr(b, f) for f, _ in abi.Block._fields_}
    return {"pack": [blk(pack[i]) for i in range(npk.value)], "unpack": [blk(unpack[i]) for i in range(nun.value)],
            "send_bytes": list(sb), "recv_bytes": list(rb)}


class _DeviceBytes:
    """A device buffer of the library as a CUDA array interface (bytes), for torch.as_tensor."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False), "strides": None,
                                         "version": 2}


class RankComm:
    """The g3d_comm_fn of one rank on a torch.distributed group (the default group if None). `device`: the CUDA
    device of this rank's context. Pass it to Simulation(cfg, comm=...)."""

    def __init__(self, group=None, device=None):
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.nccl = dist.get_backend(group) == "nccl"
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.error = None
        self.calls = 0
        self.fn = abi.COMM_FN(self._call)          # kept alive as long as this object

    # memory of the library: device bytes (overridden by tests that drive a plan with host buffers)
    def _view(self, ptr, nbytes):
        if nbytes == 0:
            return torch.empty(0, dtype=torch.uint8, device=self.device)
        return torch.as_tensor(_DeviceBytes(ptr, nbytes), device=self.device)

    def _sync(self):
        torch.cuda.current_stream(self.device).synchronize()

    def _call(self, user, op_p):
        try:
            op = op_p.contents
            self.calls += 1
            if op.op == abi.G3D_COMM_SUM:
                self.sum(op.data, op.count, op.kind)
            elif op.op == abi.G3D_COMM_ALLTOALL:
                sb = [int(op.send_bytes[i]) for i in range(self.world)]
                rb = [int(op.recv_bytes[i]) for i in range(self.world)]
                self.all_to_all(op.send, sb, op.recv, rb)
            else:
                raise ValueError(f"unknown collective {op.op}")
            return 0
        except BaseException as e:                 # nothing may unwind through the C library
            self.error = e
            return 1

    def sum(self, ptr, count, kind):
        dtype = {abi.G3D_SUM_F64: torch.float64, abi.G3D_SUM_I64: torch.int64}[kind]
        t = self._view(ptr, 8 * count).view(dtype)
        if self.nccl:
            dist.all_reduce(t, group=self.group)
        else:
            h = t.cpu()
            dist.all_reduce(h, group=self.group)
            t.copy_(h)
        self._sync()

    def all_to_all(self, send, send_bytes, recv, recv_bytes):
        s = self._view(send, sum(send_bytes))
        r = self._view(recv, sum(recv_bytes))
        if self.nccl:
            dist.all_to_all_single(r, s, output_split_sizes=recv_bytes, input_split_sizes=send_bytes, group=self.group)
        else:
            hr = torch.empty(sum(recv_bytes), dtype=torch.uint8)
            dist.all_to_all_single(hr, s.cpu(), output_split_sizes=recv_bytes, input_split_sizes=send_bytes,
                                   group=self.group)
            r.copy_(hr)
        self._sync()
