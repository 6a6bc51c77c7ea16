// Locality order of the particles for the push and the deposit.
//
// The particles stay stored in the order they were given (the reference's order: the ABI, checkpoints and
// the sums that follow array order see it unchanged); `perm` lists them by cell instead: zeta slice first,
// then 8 x 8 tiles of transverse cells, so the 32 particles of a warp gather the same few planes of F and
// deposit into the same lines of jw. The order is a stable radix sort of the cell keys (CUB's
// DeviceRadixSort: a utility sort at upload time and every few steps, not a per-step kernel). Particles move
// far less than a cell per step in zeta, so the order stays good between re-sorts; it only affects speed.
#include <cub/device/device_radix_sort.cuh>
#include "g3d_ctx.hpp"

namespace g3d {

__global__ void k_cell_keys(PartsDev P, long np, Geo g, uint32_t* __restrict__ key, int32_t* __restrict__ idx) {
    const int tx = (g.nx + 7) / 8, ty = (g.ny + 7) / 8;
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < np; i += long(gridDim.x) * blockDim.x) {
        int m; double f;
        g.zax.locate(P.zeta[i], m, f);
        m = m < 0 ? 0 : (m > g.N - 1 ? g.N - 1 : m);
        const double xs = P.x[i] / g.dx, ys = P.y[i] / g.dy;
        int ix = int(floor(xs)) % g.nx, jy = int(floor(ys)) % g.ny;
        ix += ix < 0 ? g.nx : 0; jy += jy < 0 ? g.ny : 0;
        uint32_t k = (uint32_t(m) * uint32_t(ty) + uint32_t(jy / 8)) * uint32_t(tx) + uint32_t(ix / 8);
        if (P.alive[i] != 1) k = 0xffffffffu;                     // dead particles last
        key[i] = k;
        idx[i] = int32_t(i);
    }
}

void sort_particles(Ctx& c) {
    const long n = c.np;
    if (n == 0) return;
    if (n > 0x7fffffffL) throw Error(G3D_ERR_CAPACITY, "more than 2^31 particles");
    // buffers sized for the particle capacity and kept: no allocation (and no implicit synchronisation of
    // cudaFree) inside a step
    if (c.perm.n < size_t(c.pcap)) {
        c.perm.alloc(size_t(c.pcap), c.stream);
        c.sort_keys.alloc(size_t(2 * c.pcap), c.stream);
        c.sort_idx.alloc(size_t(c.pcap), c.stream);
        size_t tb = 0;
        G3D_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, c.sort_keys.p, c.sort_keys.p + c.pcap, c.sort_idx.p, c.perm.p,
                                                 int(c.pcap), 0, 32, c.stream));
        c.sort_tmp.alloc(tb, c.stream);
    }
    const long blocks = std::min<long>((n + 255) / 256, 148 * 8);
    k_cell_keys<<<unsigned(blocks), 256, 0, c.stream>>>(c.parts, n, c.geo(), c.sort_keys.p, c.sort_idx.p);
    c.check_launch("k_cell_keys");
    size_t tmp_bytes = c.sort_tmp.n;
    G3D_CUDA(cub::DeviceRadixSort::SortPairs(c.sort_tmp.p, tmp_bytes, c.sort_keys.p, c.sort_keys.p + n, c.sort_idx.p, c.perm.p,
                                             int(n), 0, 32, c.stream));
    c.steps_since_sort = 0;
}

}  // namespace g3d
