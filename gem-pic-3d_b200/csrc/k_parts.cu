// Transposition between the reference's 104-byte particle records (struct Particle, src/sim.hpp:217) and the
// structure-of-arrays columns the kernels read. One thread per particle; each record is moved as thirteen
// 8-byte words (104 = 13 x 8), the columns are written and read coalesced.
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

}  // namespace g3d
