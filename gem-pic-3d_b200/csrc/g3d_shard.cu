// A run of the beam sharded over ranks by zeta slabs: the reference's MPI decomposition (src/sim_setup.cpp:9-15,
// Comm src/comm.hpp:11-46) with the march over the ranks replaced by a transpose.
//
// Rank r holds the slices [a, b) of the window and the beam particles above zeta[a + 1] (and below the next rank's
// bound), and runs on them what is local in zeta: the push, the deposit, the transverse transforms, the sponge and
// the real fields. The march and the co-moving solve are serial in zeta but independent per mode, so they run on
// mode pencils: an all-to-all gives rank q all N slices of the modes [m0_q, m0_q + mq_q) (every rank sends its slab's
// rows of those modes), the per-mode kernels run there unchanged (a Geo with a = 0, b = ns = N and the mode offset
// m0), and a second all-to-all returns the results to the slabs. Each rank's work is 1/P of the whole; what crosses
// the links per s-step is 15 complex planes of the window (9 in, 6 out), (P - 1)/P of it off the rank.
//
// Between neighbours the exchanges are the reference's: the three top raw current half-cells of a slab are the
// bottom ghosts of the slab above (sim_particles.cpp:108-119), the filtered j_z half-cells a - 2 and b come from the
// neighbours for the sponge's bound field (:210-226), the two lowest real-field slices of a slab are the ghosts b,
// b + 1 of the slab below (sim_fields.cpp:295-306), and particles that cross below zeta[a + 1] in the push are
// handed to the rank below, which finishes their push (sim_particles.cpp:28-48). The library communicates only
// through the caller's function (g3d_set_ranks): sums and all-to-alls of device buffers, every rank calling the same
// collectives in the same order. Neighbour exchanges are all-to-alls with zero bytes for the other ranks.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <cub/device/device_select.cuh>
#include "g3d_shard.hpp"

namespace g3d {

// ---------------------------------------------------------------- collectives through the caller
void Ctx::all_sum(void* data, long count, int kind) {
    if (!sharded() || count <= 0) return;
    G3D_CUDA(cudaStreamSynchronize(stream));
    g3d_comm_op op{};
    op.op = G3D_COMM_SUM; op.kind = kind; op.count = count; op.data = data;
    if (comm_fn(comm_user, &op) != 0) throw Error(G3D_ERR_CUDA, "the sum over the ranks failed (the g3d_set_ranks function)");
}
void Ctx::all_to_all(const void* send, const int64_t* send_bytes, void* recv, const int64_t* recv_bytes) {
    if (!sharded()) return;
    G3D_CUDA(cudaStreamSynchronize(stream));
    g3d_comm_op op{};
    op.op = G3D_COMM_ALLTOALL; op.send = send; op.send_bytes = send_bytes; op.recv = recv; op.recv_bytes = recv_bytes;
    if (comm_fn(comm_user, &op) != 0) throw Error(G3D_ERR_CUDA, "the all-to-all over the ranks failed (the g3d_set_ranks function)");
}

// ---------------------------------------------------------------- partition and transpose plans
ShardLayout::ShardLayout(int N_, long nkh_, int P_) : P(P_), N(N_), nkh(nkh_) {
    if (P < 1 || N < 1 || nkh < 1) throw Error(G3D_ERR_ARG, "shard layout: world, slices and modes must be positive");
    const int base = N / P, rem = N % P;
    if (P > 1 && base < 4)
        throw Error(G3D_ERR_ARG, "a sharded run needs at least 4 slices a rank (" + std::to_string(N) + " slices, " +
                                     std::to_string(P) + " ranks)");
    a.resize(size_t(P)); ns.resize(size_t(P)); m0.resize(size_t(P)); mq.resize(size_t(P));
    const long mb = nkh / P, mr = nkh % P;
    int s = 0;
    long m = 0;
    for (int r = 0; r < P; ++r) {
        a[size_t(r)] = s; ns[size_t(r)] = base + (r < rem ? 1 : 0); s += ns[size_t(r)];
        m0[size_t(r)] = m; mq[size_t(r)] = mb + (r < mr ? 1 : 0); m += mq[size_t(r)];
    }
}

// A slab array of kind G3D_SLAB_NODES has ns planes (slices a .. b-1); G3D_SLAB_HALF ns + 1 (half cells a - 1/2 ..
// b - 1/2), of which the last is the next slab's first: the top rank alone sends it. On the pencil both start at
// plane a: slice n is plane n, half cell n - 1/2 plane n (N + 1 planes).
void shard_plan(const ShardLayout& L, int rank, const int* kinds, int K, bool to_pencil, long eb, ShardPlan& o) {
    const int P = L.P;
    if (rank < 0 || rank >= P || K < 1 || !kinds || eb < 1) throw Error(G3D_ERR_ARG, "shard plan: bad arguments");
    for (int k = 0; k < K; ++k)
        if (kinds[k] != G3D_SLAB_NODES && kinds[k] != G3D_SLAB_HALF) throw Error(G3D_ERR_ARG, "shard plan: unknown array kind");
    auto rows = [&](int k, int r) -> long { return L.ns[size_t(r)] + (kinds[k] == G3D_SLAB_HALF && r == P - 1 ? 1 : 0); };
    o.pack.clear(); o.unpack.clear();
    o.send_bytes.assign(size_t(P), 0); o.recv_bytes.assign(size_t(P), 0);
    o.pack_max = o.unpack_max = 0;
    auto add = [](std::vector<g3d_block>& v, long& mx, const g3d_block& b) {
        if (b.rows * b.cols == 0) return;
        v.push_back(b);
        mx = std::max<long>(mx, long(b.rows * b.cols));
    };
    long off = 0;
    if (to_pencil) {
        for (int q = 0; q < P; ++q) {            // this rank's slab rows of the modes of q, array after array
            const long o0 = off, mq = L.mq[size_t(q)];
            for (int k = 0; k < K; ++k) {
                add(o.pack, o.pack_max, g3d_block{L.m0[size_t(q)], off, rows(k, rank), mq, L.nkh, mq, k, -1});
                off += rows(k, rank) * mq;
            }
            o.send_bytes[size_t(q)] = (off - o0) * eb;
        }
        off = 0;
        const long mq = L.mq[size_t(rank)];
        for (int r = 0; r < P; ++r) {            // the rows of slab r into planes a_r ... of this rank's pencil
            const long o0 = off;
            for (int k = 0; k < K; ++k) {
                add(o.unpack, o.unpack_max, g3d_block{off, long(L.a[size_t(r)]) * mq, rows(k, r), mq, mq, mq, -1, k});
                off += rows(k, r) * mq;
            }
            o.recv_bytes[size_t(r)] = (off - o0) * eb;
        }
    } else {
        const long mq = L.mq[size_t(rank)];
        for (int r = 0; r < P; ++r) {            // this rank's pencil rows of slab r
            const long o0 = off;
            for (int k = 0; k < K; ++k) {
                add(o.pack, o.pack_max, g3d_block{long(L.a[size_t(r)]) * mq, off, rows(k, r), mq, mq, mq, k, -1});
                off += rows(k, r) * mq;
            }
            o.send_bytes[size_t(r)] = (off - o0) * eb;
        }
        off = 0;
        for (int q = 0; q < P; ++q) {            // the modes of q into this rank's slab
            const long o0 = off, mqq = L.mq[size_t(q)];
            for (int k = 0; k < K; ++k) {
                add(o.unpack, o.unpack_max, g3d_block{off, L.m0[size_t(q)], rows(k, rank), mqq, mqq, L.nkh, -1, k});
                off += rows(k, rank) * mqq;
            }
            o.recv_bytes[size_t(q)] = (off - o0) * eb;
        }
    }
}

namespace {
constexpr int MAXA = 12;
struct BlockArrays { cpx* p[MAXA]; };

// One CTA row per block of the plan (blockIdx.y), the CTAs of a row striding over its elements: consecutive
// threads copy consecutive modes of a plane, 16-byte elements, coalesced on both sides.
__global__ void __launch_bounds__(256) k_blocks(const g3d_block* __restrict__ B, BlockArrays A, cpx* buf) {
    const g3d_block b = B[blockIdx.y];
    const cpx* src = (b.src_array < 0 ? buf : A.p[b.src_array]) + b.src;
    cpx* dst = (b.dst_array < 0 ? buf : A.p[b.dst_array]) + b.dst;
    const long n = long(b.rows) * long(b.cols);
    for (long e = long(blockIdx.x) * blockDim.x + threadIdx.x; e < n; e += long(gridDim.x) * blockDim.x) {
        const long r = e / b.cols, k = e - r * b.cols;
        dst[r * b.dst_stride + k] = src[r * b.src_stride + k];
    }
}

void run_blocks(Ctx& c, const DevBuf<g3d_block>& B, size_t nb, long mx, cpx* const* arrays, int K, void* buf) {
    if (nb == 0) return;
    BlockArrays A{};
    for (int k = 0; k < K && k < MAXA; ++k) A.p[k] = arrays[k];
    const long gx = std::min<long>(std::max<long>((mx + 255) / 256, 1), 1024);
    k_blocks<<<dim3(unsigned(gx), unsigned(nb)), 256, 0, c.stream>>>(B.p, A, static_cast<cpx*>(buf));
    c.check_launch("k_blocks");
}

template <class T>
void ensure(DevBuf<T>& b, size_t n, cudaStream_t s) {
    if (b.n < n) b.alloc(n + n / 8, s);
}
long total(const std::vector<int64_t>& v) {
    long t = 0;
    for (int64_t x : v) t += long(x);
    return t;
}

// slab -> pencil or back: pack into the send buffer, the all-to-all, unpack from the receive buffer
void transpose(Ctx& c, ShardPlan& pl, cpx* const* src, int ks, cpx* const* dst, int kd) {
    Shard& S = *c.sh;
    const int tok = c.prof_begin("shard_transpose");
    ensure(S.sendb, size_t(std::max<long>(total(pl.send_bytes), 16)), c.stream);
    ensure(S.recvb, size_t(std::max<long>(total(pl.recv_bytes), 16)), c.stream);
    if (pl.dpack.n != pl.pack.size() && !pl.pack.empty()) pl.dpack.upload(pl.pack, c.stream);
    if (pl.dunpack.n != pl.unpack.size() && !pl.unpack.empty()) pl.dunpack.upload(pl.unpack, c.stream);
    run_blocks(c, pl.dpack, pl.pack.size(), pl.pack_max, src, ks, S.sendb.p);
    c.prof_end(tok);
    c.all_to_all(S.sendb.p, pl.send_bytes.data(), S.recvb.p, pl.recv_bytes.data());
    const int tok2 = c.prof_begin("shard_transpose");
    run_blocks(c, pl.dunpack, pl.unpack.size(), pl.unpack_max, dst, kd, S.recvb.p);
    c.prof_end(tok2);
}

// ---------------------------------------------------------------- particle exchange kernels
// keep: alive 1 (beam) or 4 (slow, streaming); hand: alive 2 (below zeta[a + 1]); the rest is lost. Counts by
// warp sums and integer atomics.
__global__ void k_exchange_flags(const int32_t* __restrict__ alive, long n, unsigned char* __restrict__ keep,
                                 unsigned char* __restrict__ hand, unsigned long long* __restrict__ cnt) {
    unsigned long long nh = 0, nd = 0;
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const int al = alive[i];
        const bool k = al == 1 || al == 4, h = al == 2;
        if (keep) keep[i] = k ? 1 : 0;
        if (hand) hand[i] = h ? 1 : 0;
        nh += h ? 1 : 0;
        nd += (!k && !h) ? 1 : 0;
    }
    for (int o = 16; o > 0; o >>= 1) {
        nh += __shfl_down_sync(0xffffffffu, nh, o);
        nd += __shfl_down_sync(0xffffffffu, nd, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (nh) atomicAdd(cnt, nh);
        if (nd) atomicAdd(cnt + 1, nd);
    }
}
// records -> the columns [i0, i0 + n); alive >= 0 replaces the records' state
__global__ void k_unpack_at(const g3d_particle* __restrict__ in, PartsDev P, long i0, long n, int alive) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const g3d_particle p = in[i];
        const long j = i0 + i;
        P.x[j] = p.x; P.y[j] = p.y; P.zeta[j] = p.zeta; P.px[j] = p.px; P.py[j] = p.py; P.pz[j] = p.pz;
        P.w[j] = p.w; P.rem[j] = p.rem; P.z[j] = p.z; P.q[j] = p.q; P.qm[j] = p.qm;
        P.alive[j] = alive >= 0 ? alive : p.alive; P.sp[j] = p.sp; P.id[j] = p.id;
    }
}
unsigned grid_for(long n) { return unsigned(std::min<long>(std::max<long>((n + 255) / 256, 1), 148 * 8)); }

void counts(Ctx& c, const int32_t* alive, long n, unsigned char* keep, unsigned char* hand, unsigned long long out[2]) {
    Shard& S = *c.sh;
    G3D_CUDA(cudaMemsetAsync(S.cnt.p, 0, 2 * sizeof(unsigned long long), c.stream));
    if (n > 0) {
        k_exchange_flags<<<grid_for(n), 256, 0, c.stream>>>(alive, n, keep, hand, S.cnt.p);
        c.check_launch("k_exchange_flags");
    }
    G3D_CUDA(cudaMemcpyAsync(out, S.cnt.p, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
}
long select_flagged(Ctx& c, const g3d_particle* in, const unsigned char* flags, g3d_particle* out, long n) {
    Shard& S = *c.sh;
    size_t tb = 0;
    G3D_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, in, flags, out, S.nsel.p, int(n), c.stream));
    ensure(S.cubtmp, tb, c.stream);
    tb = S.cubtmp.n;
    G3D_CUDA(cub::DeviceSelect::Flagged(S.cubtmp.p, tb, in, flags, out, S.nsel.p, int(n), c.stream));
    int k = 0;
    G3D_CUDA(cudaMemcpyAsync(&k, S.nsel.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
    return k;
}
}  // namespace

// ---------------------------------------------------------------- set-up
static void setup_peers(Ctx& c, Shard& S);
void set_ranks(Ctx& c, int rank, int world, g3d_comm_fn comm, void* user) {
    if (world < 1 || rank < 0 || rank >= world) throw Error(G3D_ERR_ARG, "g3d_set_ranks: rank must be in [0, world)");
    if (world > 1 && !comm) throw Error(G3D_ERR_ARG, "g3d_set_ranks: several ranks need a communication function");
    if (c.np > 0 || c.fields_ready) throw Error(G3D_ERR_STATE, "g3d_set_ranks: before particles are loaded and before g3d_init");
    if (world > 1) {
        if (!c.yf) throw Error(G3D_ERR_STATE, "g3d_set_ranks: a run on a free-hand y grid is not sharded");
        if (c.mixed || c.f32s) throw Error(G3D_ERR_STATE, "g3d_set_ranks: a sharded run is FP64");
        if (c.pl) throw Error(G3D_ERR_STATE, "g3d_set_ranks: a run with plasma is not sharded");
        if (!c.chicanes.empty()) throw Error(G3D_ERR_STATE, "g3d_set_ranks: a run with chicanes is not sharded");
        if (c.Fd.p) throw Error(G3D_ERR_STATE, "g3d_set_ranks: exact fields are not sharded");
    }
    const ShardLayout L(c.N, c.nkh, world);
    c.rank = rank; c.world = world;
    c.comm_fn = world > 1 ? comm : nullptr; c.comm_user = world > 1 ? user : nullptr;
    c.a = L.a[size_t(rank)]; c.ns = L.ns[size_t(rank)]; c.b = c.a + c.ns;
    c.sh.reset();
    realloc_slab(c);
    if (world == 1) return;
    auto S = std::make_unique<Shard>(L);
    Geo& g = S->pencil;
    g = c.geo();
    g.a = 0; g.b = c.N; g.ns = c.N; g.nh = c.N + 3;
    g.nkh = L.mq[size_t(rank)]; g.m0 = L.m0[size_t(rank)];
    const size_t mq = size_t(L.mq[size_t(rank)]), N = size_t(c.N);
    for (int k = 0; k < 11; ++k) S->pen[k].alloc((k < 6 ? N : N + 1) * std::max<size_t>(mq, 1), c.stream);
    S->cpb.alloc(N * std::max<size_t>(mq, 1), c.stream);
    S->dpb.alloc(N * std::max<size_t>(mq, 1), c.stream);
    const int NODE = G3D_SLAB_NODES, HALF = G3D_SLAB_HALF;
    const int k_march_in[9] = {NODE, NODE, NODE, NODE, HALF, HALF, HALF, HALF, HALF};
    const int k_nodes[6] = {NODE, NODE, NODE, NODE, NODE, NODE};
    const int k_half[1] = {HALF};
    shard_plan(L, rank, k_march_in, 9, true, sizeof(cpx), S->march_in);
    shard_plan(L, rank, k_nodes, 6, false, sizeof(cpx), S->march_out);
    shard_plan(L, rank, k_half, 1, true, sizeof(cpx), S->como_in);
    shard_plan(L, rank, k_nodes, 4, false, sizeof(cpx), S->como_out);
    S->cnt.alloc(2, c.stream);
    S->hv.alloc(size_t(world), c.stream);
    S->nsel.alloc(1, c.stream);
    S->one.alloc(1, c.stream);
    c.sh = std::move(S);
    setup_peers(c, *c.sh);
    G3D_CUDA(cudaStreamSynchronize(c.stream));
}

Shard::~Shard() {
    for (void* p : opened) cudaIpcCloseMemHandle(p);          // nothing to report from a destructor
}

// every rank has reached this point with its stream drained (a sum of nothing over the ranks)
static void shard_barrier(Ctx& c) {
    Shard& S = *c.sh;
    c.all_sum(S.one.p, 1, G3D_SUM_I64);
}
// Map every rank's slab arrays into this GPU's address space (CUDA IPC handles exchanged by the all-to-all): the
// fused march then reads and writes them directly. All ranks agree on the outcome (a failure anywhere is summed),
// so either every rank marches over peer memory or every rank uses the transposes.
static void setup_peers(Ctx& c, Shard& S) {
    const int P = c.world, r = c.rank;
    const bool want = P <= SHARD_PEER_MAX && std::getenv("G3D_SHARD_TRANSPOSE") == nullptr;
    cpx* mine[11] = {c.Rx.p, c.Ry.p, c.Ez.p, c.Bz.p, c.Lx.p, c.Ly.p, c.j0x.p, c.j0y.p, c.jkx.p, c.jky.p, c.jkz.p};
    std::vector<cudaIpcMemHandle_t> h(11);
    int64_t fail = want ? 0 : 1;
    for (int k = 0; k < 11 && !fail; ++k)
        if (cudaIpcGetMemHandle(&h[size_t(k)], mine[k]) != cudaSuccess) { fail = 1; cudaGetLastError(); }
    auto agree = [&](int64_t f) {                // the sum of the ranks' failure flags
        G3D_CUDA(cudaMemcpyAsync(S.one.p, &f, sizeof(f), cudaMemcpyHostToDevice, c.stream));
        c.all_sum(S.one.p, 1, G3D_SUM_I64);
        int64_t t = 0;
        G3D_CUDA(cudaMemcpyAsync(&t, S.one.p, sizeof(t), cudaMemcpyDeviceToHost, c.stream));
        G3D_CUDA(cudaMemsetAsync(S.one.p, 0, sizeof(int64_t), c.stream));
        G3D_CUDA(cudaStreamSynchronize(c.stream));
        return t;
    };
    if (agree(fail) != 0) return;
    const size_t hb = 11 * sizeof(cudaIpcMemHandle_t);
    std::vector<unsigned char> send(size_t(P) * hb), recv(size_t(P) * hb);
    for (int q = 0; q < P; ++q) std::memcpy(send.data() + size_t(q) * hb, h.data(), hb);
    DevBuf<unsigned char> ds, dr;
    ds.upload(send, c.stream);
    dr.alloc(size_t(P) * hb, c.stream);
    const std::vector<int64_t> bytes(static_cast<size_t>(P), static_cast<int64_t>(hb));
    c.all_to_all(ds.p, bytes.data(), dr.p, bytes.data());
    G3D_CUDA(cudaMemcpyAsync(recv.data(), dr.p, recv.size(), cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
    SlabPeers sp;
    sp.P = P;
    sp.nkh = c.nkh;
    for (int q = 0; q < P; ++q) {
        sp.a[q] = S.L.a[size_t(q)];
        sp.ns[q] = S.L.ns[size_t(q)];
        for (int k = 0; k < 11; ++k) {
            if (q == r) { sp.arr[q][k] = mine[k]; continue; }
            cudaIpcMemHandle_t hq;
            std::memcpy(&hq, recv.data() + size_t(q) * hb + size_t(k) * sizeof(cudaIpcMemHandle_t), sizeof(hq));
            void* p = nullptr;
            if (fail == 0 && cudaIpcOpenMemHandle(&p, hq, cudaIpcMemLazyEnablePeerAccess) == cudaSuccess) {
                S.opened.push_back(p);
                sp.arr[q][k] = p;
            } else {
                fail = 1;
                cudaGetLastError();
            }
        }
    }
    if (agree(fail) != 0) {
        for (void* p : S.opened) cudaIpcCloseMemHandle(p);
        S.opened.clear();
        return;
    }
    S.peers = sp;
    S.orig_j0x = c.j0x.p;
    S.peer = true;
}

bool shard_owns(const Ctx& c, double zeta) {
    if (!c.sharded()) return true;
    const ShardLayout& L = c.sh->L;
    const int r = c.rank;
    const double lo = r > 0 ? c.zeta[size_t(c.a) + 1] : -1e300;
    const double hi = r < L.P - 1 ? c.zeta[size_t(L.a[size_t(r) + 1]) + 1] : 1e300;
    return zeta >= lo && zeta < hi;
}

// ---------------------------------------------------------------- the march and the co-moving solve on pencils
void shard_march(Ctx& c, double D) {
    Shard& S = *c.sh;
    if (S.peer) {
        // j0 and jk trade buffers after every field solve, on every rank alike: the peers' current roles follow ours
        SlabPeers sp = S.peers;
        if (c.j0x.p != S.orig_j0x)
            for (int q = 0; q < sp.P; ++q) { std::swap(sp.arr[q][6], sp.arr[q][8]); std::swap(sp.arr[q][7], sp.arr[q][9]); }
        shard_barrier(c);                        // every slab's inputs are complete
        launch_march_peer(c, S.pencil, sp, D);
        shard_barrier(c);                        // every rank's march has written its modes into every slab
        return;
    }
    cpx* slab_in[9] = {c.Rx.p, c.Ry.p, c.Ez.p, c.Bz.p, c.j0x.p, c.j0y.p, c.jkx.p, c.jky.p, c.jkz.p};
    cpx* pen_in[9] = {S.pen[0].p, S.pen[1].p, S.pen[2].p, S.pen[3].p, S.pen[6].p, S.pen[7].p, S.pen[8].p, S.pen[9].p, S.pen[10].p};
    transpose(c, S.march_in, slab_in, 9, pen_in, 9);
    cpx* all[11];
    for (int k = 0; k < 11; ++k) all[k] = S.pen[k].p;
    launch_march_pencil(c, S.pencil, all, D);
    cpx* slab_out[6] = {c.Rx.p, c.Ry.p, c.Ez.p, c.Bz.p, c.Lx.p, c.Ly.p};
    transpose(c, S.march_out, all, 6, slab_out, 6);
}

void shard_comoving(Ctx& c, double beta, double gm2) {
    Shard& S = *c.sh;
    cpx* slab_in[1] = {c.jkz.p};
    cpx* pen_in[1] = {S.pen[10].p};
    transpose(c, S.como_in, slab_in, 1, pen_in, 1);
    cpx* pen_out[4] = {S.pen[0].p, S.pen[1].p, S.pen[2].p, S.pen[3].p};
    launch_comoving_pencil(c, S.pencil, S.pen[10].p, S.cpb.p, S.dpb.p, pen_out, beta, gm2);
    cpx* slab_out[4] = {c.Rx.p, c.Ry.p, c.Ez.p, c.Bz.p};
    transpose(c, S.como_out, pen_out, 4, slab_out, 4);
}

// ---------------------------------------------------------------- neighbour exchanges
// raw current planes [3][ns + 3][nk]: planes ns .. ns + 2 (cells b - 2 .. b) go up as planes 0 .. 2 of the slab above
void shard_raw_halo(Ctx& c) {
    Shard& S = *c.sh;
    const int P = c.world, r = c.rank;
    const size_t pl = size_t(c.nk), nh = size_t(c.ns) + 3, chunk = 3 * pl * sizeof(double);
    std::vector<int64_t> sb(size_t(P), 0), rb(size_t(P), 0);
    ensure(S.sendb, 3 * chunk, c.stream);
    ensure(S.recvb, 3 * chunk, c.stream);
    if (r < P - 1) {
        for (size_t comp = 0; comp < 3; ++comp)
            G3D_CUDA(cudaMemcpyAsync(S.sendb.p + comp * chunk, c.jw.p + (comp * nh + size_t(c.ns)) * pl, chunk,
                                     cudaMemcpyDeviceToDevice, c.stream));
        sb[size_t(r) + 1] = int64_t(3 * chunk);
    }
    if (r > 0) rb[size_t(r) - 1] = int64_t(3 * chunk);
    c.all_to_all(S.sendb.p, sb.data(), S.recvb.p, rb.data());
    if (r > 0)
        for (size_t comp = 0; comp < 3; ++comp)
            G3D_CUDA(cudaMemcpyAsync(c.jw.p + comp * nh * pl, S.recvb.p + comp * chunk, chunk, cudaMemcpyDeviceToDevice, c.stream));
}

// filtered j_z [ns + 1][nkh]: plane ns - 1 (half cell b - 3/2) is the low ghost of the slab above, plane 1 (a + 1/2)
// the high ghost of the slab below; a slab without a neighbour keeps a zero ghost
void shard_jz_ghosts(Ctx& c) {
    Shard& S = *c.sh;
    const int P = c.world, r = c.rank;
    const size_t ph = size_t(c.nkh), plane = ph * sizeof(cpx);
    std::vector<int64_t> sb(size_t(P), 0), rb(size_t(P), 0);
    ensure(S.sendb, 2 * plane, c.stream);
    ensure(S.recvb, 2 * plane, c.stream);
    size_t so = 0;
    if (r > 0) {                               // to the rank below first (rank order of the send buffer)
        G3D_CUDA(cudaMemcpyAsync(S.sendb.p + so, c.jkz.p + ph, plane, cudaMemcpyDeviceToDevice, c.stream));
        sb[size_t(r) - 1] = int64_t(plane); so += plane;
        rb[size_t(r) - 1] = int64_t(plane);
    }
    if (r < P - 1) {
        G3D_CUDA(cudaMemcpyAsync(S.sendb.p + so, c.jkz.p + size_t(c.ns - 1) * ph, plane, cudaMemcpyDeviceToDevice, c.stream));
        sb[size_t(r) + 1] = int64_t(plane);
        rb[size_t(r) + 1] = int64_t(plane);
    }
    c.all_to_all(S.sendb.p, sb.data(), S.recvb.p, rb.data());
    size_t ro = 0;
    if (r > 0) {
        G3D_CUDA(cudaMemcpyAsync(c.jzg.p, S.recvb.p, plane, cudaMemcpyDeviceToDevice, c.stream));
        ro += plane;
    }
    if (r < P - 1) G3D_CUDA(cudaMemcpyAsync(c.jzg.p + ph, S.recvb.p + ro, plane, cudaMemcpyDeviceToDevice, c.stream));
}

// real fields [6][ns + 2][nk]: planes 0, 1 (slices a, a + 1) go down as the ghost planes ns, ns + 1 of the slab below
void shard_field_ghosts(Ctx& c) {
    Shard& S = *c.sh;
    const int P = c.world, r = c.rank;
    const size_t pl = size_t(c.nk), fpl = (size_t(c.ns) + 2) * pl, chunk = 2 * pl * sizeof(float);
    std::vector<int64_t> sb(size_t(P), 0), rb(size_t(P), 0);
    ensure(S.sendb, 6 * chunk, c.stream);
    ensure(S.recvb, 6 * chunk, c.stream);
    if (r > 0) {
        for (size_t comp = 0; comp < 6; ++comp)
            G3D_CUDA(cudaMemcpyAsync(S.sendb.p + comp * chunk, c.F.p + comp * fpl, chunk, cudaMemcpyDeviceToDevice, c.stream));
        sb[size_t(r) - 1] = int64_t(6 * chunk);
    }
    if (r < P - 1) rb[size_t(r) + 1] = int64_t(6 * chunk);
    c.all_to_all(S.sendb.p, sb.data(), S.recvb.p, rb.data());
    if (r < P - 1)
        for (size_t comp = 0; comp < 6; ++comp)
            G3D_CUDA(cudaMemcpyAsync(c.F.p + comp * fpl + size_t(c.ns) * pl, S.recvb.p + comp * chunk, chunk,
                                     cudaMemcpyDeviceToDevice, c.stream));
}

// ---------------------------------------------------------------- particle handover (sim_particles.cpp:28-48)
// After the push: the particles marked 2 (below zeta[a + 1] with the rest of their step in rem) go to the rank below,
// the lost ones (0) are dropped and counted, and the particles from the rank above are appended marked 3 and pushed
// for their rest with this slab's fields. The list is rebuilt in storage order (kept ones, then adopted ones) only
// when something left or arrived; every rank learns every rank's handed count by a sum, so that all take part in
// the all-to-all of the records exactly when one hands any.
void shard_exchange_particles(Ctx& c, double s1) {
    Shard& S = *c.sh;
    const int P = c.world, r = c.rank;
    const long n = c.np;
    if (n > 0) { ensure(S.keep, size_t(n), c.stream); ensure(S.hand, size_t(n), c.stream); }
    unsigned long long hc[2] = {0, 0};
    counts(c, c.parts.alive, n, S.keep.p, S.hand.p, hc);
    const long hand = long(hc[0]), drop = long(hc[1]);
    if (r == 0 && hand > 0) throw Error(G3D_ERR_STATE, "particle handover below rank 0");
    std::vector<int64_t> v(size_t(P), 0);
    v[size_t(r)] = hand;
    G3D_CUDA(cudaMemcpyAsync(S.hv.p, v.data(), size_t(P) * sizeof(int64_t), cudaMemcpyHostToDevice, c.stream));
    c.all_sum(S.hv.p, P, G3D_SUM_I64);
    G3D_CUDA(cudaMemcpyAsync(v.data(), S.hv.p, size_t(P) * sizeof(int64_t), cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
    long any = 0;
    for (int64_t x : v) any += long(x);
    const long nin = r < P - 1 ? long(v[size_t(r) + 1]) : 0;
    if (any == 0 && drop == 0) return;
    const int tok = c.prof_begin("shard_exchange");
    // the own list as records
    if (c.pstage.n < size_t(std::max<long>(n, 1))) c.pstage.alloc(size_t(n) + size_t(n) / 4 + 64, c.stream);
    if (n > 0) launch_parts_pack(c, n);
    if (hand > 0) {
        ensure(S.handrec, size_t(hand), c.stream);
        if (select_flagged(c, c.pstage.p, S.hand.p, S.handrec.p, n) != hand)
            throw Error(G3D_ERR_STATE, "particle handover: selection count mismatch");
    }
    long nkeep = n;
    const g3d_particle* kept = c.pstage.p;
    if (hand + drop > 0) {
        ensure(S.stage2, size_t(std::max<long>(n, 1)), c.stream);
        nkeep = select_flagged(c, c.pstage.p, S.keep.p, S.stage2.p, n);
        if (nkeep != n - hand - drop) throw Error(G3D_ERR_STATE, "particle handover: selection count mismatch");
        kept = S.stage2.p;
    }
    // the records to the rank below, from the rank above
    if (any > 0) {
        std::vector<int64_t> sb(size_t(P), 0), rb(size_t(P), 0);
        if (r > 0) sb[size_t(r) - 1] = int64_t(hand) * int64_t(sizeof(g3d_particle));
        if (r < P - 1) rb[size_t(r) + 1] = int64_t(nin) * int64_t(sizeof(g3d_particle));
        ensure(S.recvb, size_t(std::max<long>(nin, 1)) * sizeof(g3d_particle), c.stream);
        if (!S.handrec.p) ensure(S.handrec, 1, c.stream);
        c.all_to_all(S.handrec.p, sb.data(), S.recvb.p, rb.data());
    }
    // the new list: kept ones, then the adopted ones
    const long nnew = nkeep + nin;
    if (nnew > 0x7fffffffL) throw Error(G3D_ERR_CAPACITY, "more than 2^31 particles");
    reserve_particles(c, nnew);
    if (nkeep > 0) {
        k_unpack_at<<<grid_for(nkeep), 256, 0, c.stream>>>(kept, c.parts, 0, nkeep, -1);
        c.check_launch("k_unpack_at");
    }
    if (nin > 0) {
        k_unpack_at<<<grid_for(nin), 256, 0, c.stream>>>(reinterpret_cast<const g3d_particle*>(S.recvb.p), c.parts, nkeep, nin, 3);
        c.check_launch("k_unpack_at");
    }
    c.np = nnew;
    c.lost_total += drop;
    c.prof_end(tok);
    if (nin > 0) {
        launch_push_range(c, s1, s1, nkeep, nin);
        unsigned long long again[2] = {0, 0};
        counts(c, c.parts.alive + nkeep, nin, nullptr, nullptr, again);
        if (again[0] > 0) throw Error(G3D_ERR_STATE, "an adopted particle crossed a whole slab in one step (slabs too thin)");
    }
    sort_particles(c);
}

}  // namespace g3d
