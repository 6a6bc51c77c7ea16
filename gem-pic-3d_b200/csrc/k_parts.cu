// Transposition between the reference's 104-byte particle records (struct Particle, src/sim.hpp:217) and the
// structure-of-arrays columns the kernels read. One thread per particle; each record is moved as thirteen
// 8-byte words (104 = 13 x 8), the columns are written and read coalesced.
#include <cub/device/device_scan.cuh>
#include "g3d_ctx.hpp"

namespace g3d {

static_assert(sizeof(g3d_particle) == 104, "particle record");

__global__ void k_parts_unpack(const g3d_particle* __restrict__ in, PartsDev P, long n) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const g3d_particle p = in[i];
        P.x[i] = p.x; P.y[i] = p.y; P.zeta[i] = p.zeta; P.px[i] = p.px; P.py[i] = p.py; P.pz[i] = p.pz;
        P.w[i] = p.w; P.rem[i] = p.rem; P.z[i] = p.z; P.q[i] = p.q; P.qm[i] = p.qm;
        P.alive[i] = p.alive; P.sp[i] = p.sp; P.id[i] = p.id;
    }
}

__global__ void k_parts_pack(PartsDev P, g3d_particle* __restrict__ out, long n) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        g3d_particle p;
        p.x = P.x[i]; p.y = P.y[i]; p.zeta = P.zeta[i]; p.px = P.px[i]; p.py = P.py[i]; p.pz = P.pz[i];
        p.w = P.w[i]; p.rem = P.rem[i]; p.z = P.z[i]; p.q = P.q[i]; p.qm = P.qm[i];
        p.alive = P.alive[i]; p.sp = P.sp[i]; p.id = P.id[i];
        out[i] = p;
    }
}

static unsigned blocks_for(long n) {
    const long b = (n + 255) / 256;
    return unsigned(b < 148 * 8 ? (b < 1 ? 1 : b) : 148 * 8);
}

void launch_parts_unpack(Ctx& c, long n) {
    const int tok = c.prof_begin("parts_unpack");
    k_parts_unpack<<<blocks_for(n), 256, 0, c.stream>>>(c.pstage.p, c.parts, n);
    c.check_launch("k_parts_unpack");
    c.prof_end(tok);
}

void launch_parts_pack(Ctx& c, long n) {
    const int tok = c.prof_begin("parts_pack");
    k_parts_pack<<<blocks_for(n), 256, 0, c.stream>>>(c.parts, c.pstage.p, n);
    c.check_launch("k_parts_pack");
    c.prof_end(tok);
}

// flag[i] = particle i is alive (1), flag[n] = 0 (its exclusive sum is the count of live particles)
__global__ void k_live_flags(const int32_t* __restrict__ alive, long n, int32_t* __restrict__ flag) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i <= n; i += long(gridDim.x) * blockDim.x)
        flag[i] = i < n && alive[i] == 1 ? 1 : 0;
}
// the record of every live particle to its place off[i] among the live ones (the list's order kept)
__global__ void k_pack_live(PartsDev P, const int32_t* __restrict__ flag, const int32_t* __restrict__ off,
                            g3d_particle* __restrict__ out, long n) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        if (!flag[i]) continue;
        g3d_particle p;
        p.x = P.x[i]; p.y = P.y[i]; p.zeta = P.zeta[i]; p.px = P.px[i]; p.py = P.py[i]; p.pz = P.pz[i];
        p.w = P.w[i]; p.rem = P.rem[i]; p.z = P.z[i]; p.q = P.q[i]; p.qm = P.qm[i];
        p.alive = P.alive[i]; p.sp = P.sp[i]; p.id = P.id[i];
        out[off[i]] = p;
    }
}

// The beam list after a plasma march (src/sim_plasma.cpp:459-466, the trapped electrons that join the beam): its live
// particles in their order, then the joining ones, as the host's filter and set_particles make it, on the device: the
// live records are packed at their exclusive sums into the staging buffer, the joining records are copied behind
// them, and the columns are rebuilt from it. The list does not cross PCIe.
bool beam_keep_live_and_append(Ctx& c, const g3d_particle* add, long na) {
    const long n = c.np;
    if (n + na > c.pcap || n + 1 > 0x7fffffffL) return false;
    if (c.jflag.n < size_t(c.pcap + 1)) {
        c.jflag.alloc(size_t(c.pcap + 1), c.stream);
        c.joff.alloc(size_t(c.pcap + 1), c.stream);
        size_t tb = 0;
        G3D_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, c.jflag.p, c.joff.p, int(c.pcap + 1), c.stream));
        c.jtmp.alloc(tb, c.stream);
    }
    if (c.pstage.n < size_t(n + na)) c.pstage.alloc(size_t(n + na) + size_t(n + na) / 4 + 64, c.stream);
    const int tok = c.prof_begin("beam_join");
    k_live_flags<<<blocks_for(n + 1), 256, 0, c.stream>>>(c.parts.alive, n, c.jflag.p);
    c.check_launch("k_live_flags");
    size_t tb = c.jtmp.n;
    G3D_CUDA(cub::DeviceScan::ExclusiveSum(c.jtmp.p, tb, c.jflag.p, c.joff.p, int(n + 1), c.stream));
    int32_t live = 0;
    G3D_CUDA(cudaMemcpyAsync(&live, c.joff.p + n, sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
    if (n) k_pack_live<<<blocks_for(n), 256, 0, c.stream>>>(c.parts, c.jflag.p, c.joff.p, c.pstage.p, n);
    c.check_launch("k_pack_live");
    G3D_CUDA(cudaStreamSynchronize(c.stream));
    if (na) G3D_CUDA(cudaMemcpyAsync(c.pstage.p + live, add, size_t(na) * sizeof(g3d_particle), cudaMemcpyHostToDevice, c.stream));
    c.np = long(live) + na;
    if (c.np) launch_parts_unpack(c, c.np);
    c.prof_end(tok);
    sort_particles(c);
    G3D_CUDA(cudaStreamSynchronize(c.stream));       // the caller's records may go on return
    return true;
}

}  // namespace g3d
