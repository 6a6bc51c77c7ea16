// A run of the beam sharded over ranks by zeta slabs, with the march and the co-moving solve on mode pencils
// (g3d_shard.cu; the ABI is g3d_set_ranks and the g3d_shard_* functions of include/g3d.h).
#pragma once
#include <vector>
#include "g3d_ctx.hpp"

namespace g3d {

// The partition of N slices and nkh modes over P ranks: the slab [a[r], a[r] + ns[r]) of the reference's split
// (src/sim_setup.cpp:9-15) and the pencil [m0[q], m0[q] + mq[q]) of the modes, split the same way.
struct ShardLayout {
    int P = 1, N = 0;
    long nkh = 0;
    std::vector<int> a, ns;
    std::vector<long> m0, mq;
    ShardLayout(int N, long nkh, int P);
};

// The copies and byte counts of one transpose of a list of arrays on one rank (g3d_shard_transpose_plan).
struct ShardPlan {
    std::vector<g3d_block> pack, unpack;
    std::vector<int64_t> send_bytes, recv_bytes;
    long pack_max = 0, unpack_max = 0;          // the largest block, elements
    DevBuf<g3d_block> dpack, dunpack;           // the blocks on the device, uploaded once
};
void shard_plan(const ShardLayout& L, int rank, const int* kinds, int narrays, bool to_pencil, long elem_bytes, ShardPlan& out);

// State of a sharded run kept by the context.
struct Shard {
    ShardLayout L;
    Geo pencil{};                               // the geometry of this rank's pencil (all slices, its modes)
    // pencil arrays: R_x, R_y, E_z, B_z, L_x, L_y (N planes), j0x, j0y, jkx, jky, jkz (N + 1 half-cell planes)
    DevBuf<cpx> pen[11];
    DevBuf<double> cpb;                         // the co-moving Thomas coefficients of the pencil
    DevBuf<cpx> dpb;
    DevBuf<unsigned char> sendb, recvb;         // all-to-all buffers
    ShardPlan march_in, march_out, como_in, como_out;
    // the particle exchange
    DevBuf<unsigned char> keep, hand;           // flags per particle
    DevBuf<unsigned long long> cnt;             // handed, dropped
    DevBuf<int64_t> hv;                         // the handed counts of the ranks
    DevBuf<int> nsel;
    DevBuf<unsigned char> cubtmp;
    DevBuf<g3d_particle> stage2, handrec;
    // the fused march over peer memory: every rank's slab arrays mapped here (CUDA IPC), as set up (j0 and jk in
    // their first roles); off when a rank cannot map them, above SHARD_PEER_MAX ranks or with G3D_SHARD_TRANSPOSE
    bool peer = false;
    SlabPeers peers;
    const void* orig_j0x = nullptr;
    std::vector<void*> opened;                  // the peers' mappings, closed with the shard
    DevBuf<int64_t> one;                        // the barrier's value
    explicit Shard(const ShardLayout& l) : L(l) {}
    ~Shard();
};

void set_ranks(Ctx& c, int rank, int world, g3d_comm_fn comm, void* user);

}  // namespace g3d
