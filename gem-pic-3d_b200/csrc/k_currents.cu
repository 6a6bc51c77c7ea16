// Current deposition of the beam list, the (1,2,1)/4 zeta filter, the forward transverse FFT pair and
// the transverse filters: Simulation::currents of the reference (src/sim_particles.cpp:56-207), Fourier y.
//
// Kernels (per call):
//   k_deposit      one thread per particle: NGP over the zeta half-cell, TSC in x and y, FP64 atomics
//                  into the raw current planes jw [3][ns+3][ny][nx] (sim_particles.cpp:66-106)
//   k_cur_cols     per (half-cell plane, tile of 8 columns): zeta filter of the raw planes (:120-138),
//                  packing jx + i jy and jz, FFT along y of both -> S1, jkz
//   k_cur_rows     per (half-cell plane, pairs of rows j and ny-j): FFT along x of both fields, then the
//                  Hermitian split of jx + i jy and the cos^2 k-filters (:146-156) -> jkx, jky, jkz
#include "g3d_ctx.hpp"
#include "k_fft.cuh"
#include "k_dispatch.cuh"

namespace g3d {

// ---------------------------------------------------------------- deposit
__global__ void __launch_bounds__(256) k_deposit(PartsDev P, long np, Geo g, double* __restrict__ J) {
    const long ip = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (ip >= np || P.alive[ip] != 1) return;
    int m; double fz;
    g.zax.locate(P.zeta[ip], m, fz);
    const int hw = m - (g.a - 2);
    if (hw < 0 || hw >= g.nh || m < 0 || m > g.N - 2) return;
    const double px = P.px[ip], py = P.py[ip], pz = P.pz[ip];
    const double gm = sqrt(1 + px * px + py * py + pz * pz);
    const double vx = px / gm, vy = py / gm, vz = pz / gm;
    const double f = P.q[ip] * P.w[ip] / (g.hcg[m + 2] * g.dx);
    int ix[3], jn[3]; double wx[3], wn[3];
    tsc_periodic(P.x[ip], g.dx, g.nx, ix, wx);
    tsc_periodic(P.y[ip], g.dy, g.ny, jn, wn);
    const double ia0 = g.iA[0];
    const long nk = g.nk, pl = long(g.nh) * nk;
    double* J0 = J + long(hw) * nk;
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int u = 0; u < 3; ++u) {
            const long k = long(jn[v]) * g.nx + ix[u];
            const double w = f * wx[u] * wn[v] * ia0;
            atomicAdd(J0 + k, w * vx / vz);
            atomicAdd(J0 + pl + k, w * vy / vz);
            atomicAdd(J0 + 2 * pl + k, w);
        }
}

// ---------------------------------------------------------------- zeta filter + FFT along y
// Tile of CW columns x NY rows of one half-cell plane; NY/E threads per column.
template <int NY, int CW>
__global__ void __launch_bounds__(CW * FftShape<NY>::T) k_cur_cols(Geo g, const double* __restrict__ J, cpx* __restrict__ S1,
                                                                   cpx* __restrict__ JZ, int zf) {
    using S = FftShape<NY>;
    extern __shared__ cpx sm[];
    cpx* s0 = sm;                    // jx + i jy
    cpx* s1 = sm + NY * CW;          // jz
    const int hk = blockIdx.y, c0 = blockIdx.x * CW, tid = threadIdx.x, nthr = CW * S::T;
    const int nx = g.nx;
    const long nk = g.nk;
    const int hc_ = g.a - 1 + hk, hw = hk + 1;
    const bool live = hc_ >= 0 && hc_ <= g.N - 2;
    const double* Jp[3] = {J, J + long(g.nh) * nk, J + 2L * g.nh * nk};
    double hm = 0, h0 = 1, hp = 0;
    if (live && zf && !g.zeta_uniform) { hm = g.hcg[hc_ + 1]; h0 = g.hcg[hc_ + 2]; hp = g.hcg[hc_ + 3]; }
    for (int e = tid; e < NY * CW; e += nthr) {
        const int p = e / CW, c = e - p * CW;
        const long i = long(p) * nx + c0 + c;
        double v[3] = {0, 0, 0};
        if (live) {
#pragma unroll
            for (int comp = 0; comp < 3; ++comp) {
                const double* Jc = Jp[comp];
                if (zf && g.zeta_uniform)
                    v[comp] = 0.25 * Jc[(hw - 1) * nk + i] + 0.5 * Jc[hw * nk + i] + 0.25 * Jc[(hw + 1) * nk + i];
                else if (zf)
                    v[comp] = (0.25 * hm * Jc[(hw - 1) * nk + i] + 0.5 * h0 * Jc[hw * nk + i] + 0.25 * hp * Jc[(hw + 1) * nk + i]) / h0;
                else
                    v[comp] = Jc[hw * nk + i];
            }
        }
        s0[e] = C(v[0], v[1]);
        s1[e] = C(v[2], 0.0);
    }
    __syncthreads();
    const int c = tid % CW, t = tid / CW;
    fft_line<NY>(s0, ColAddr<CW>{c}, t, g.twy);
    fft_line<NY>(s1, ColAddr<CW>{c}, t, g.twy);
    cpx* o0 = S1 + long(hk) * nk;
    cpx* o1 = JZ + long(hk) * nk;
    for (int e = tid; e < NY * CW; e += nthr) {
        const int p = e / CW, cc = e - p * CW;
        const long i = long(p) * nx + c0 + cc;
        o0[i] = s0[e];
        o1[i] = s1[e];
    }
}

// ---------------------------------------------------------------- FFT along x of row pairs + unpack
// Slots 2u and 2u+1 of the CTA hold the rows j and (ny - j) % ny of one half-cell plane.
template <int NX>
__global__ void __launch_bounds__(128) k_cur_rows(Geo g, cpx* __restrict__ S1, cpx* __restrict__ JX, cpx* __restrict__ JY,
                                                 cpx* __restrict__ JZ, int keep0) {
    using S = FftShape<NX>;
    constexpr int LPC = 128 / S::T, PPC = LPC / 2, RS = row_stride<NX>();
    extern __shared__ cpx sm[];
    cpx* a0 = sm;                   // jx + i jy rows
    cpx* a1 = sm + LPC * RS;        // jz rows
    const int hk = blockIdx.y, tid = threadIdx.x;
    const int ny = g.ny;
    const long nk = g.nk;
    const long base = long(hk) * nk;
    auto row_of = [&](int slot, bool& valid) {
        const int jp = blockIdx.x * PPC + (slot >> 1);
        valid = jp <= ny / 2;
        return (slot & 1) ? (ny - jp) % ny : jp;
    };
    for (int e = tid; e < LPC * NX; e += 128) {
        const int r = e / NX, p = e - r * NX;
        bool valid;
        const int row = row_of(r, valid);
        cpx u0 = C(0), u1 = C(0);
        if (valid) { const long i = base + long(row) * NX + p; u0 = S1[i]; u1 = JZ[i]; }
        a0[r * RS + p + (p >> 3)] = u0;
        a1[r * RS + p + (p >> 3)] = u1;
    }
    __syncthreads();
    const int r = tid / S::T, t = tid - r * S::T;
    fft_line<NX>(a0, RowAddr{r * RS}, t, g.twx);
    fft_line<NX>(a1, RowAddr{r * RS}, t, g.twx);
    for (int e = tid; e < LPC * NX; e += 128) {
        const int rr = e / NX, p = e - rr * NX;
        bool valid;
        const int row = row_of(rr, valid);
        if (!valid) continue;
        if ((rr & 1) && row == row_of(rr ^ 1, valid)) continue;    // a self-paired row is written once
        const int pm = (NX - p) % NX;
        const cpx z = a0[rr * RS + p + (p >> 3)], zm = conj(a0[(rr ^ 1) * RS + pm + (pm >> 3)]);
        const double f = (p == 0 && row == 0 && !keep0) ? 0.0 : g.filt[p] * g.filty[row];
        const cpx d = z - zm;
        const long i = base + long(row) * NX + p;
        JX[i] = f * (0.5 * (z + zm));
        JY[i] = f * (0.5 * C(d.y, -d.x));
        JZ[i] = f * a1[rr * RS + p + (p >> 3)];
    }
}

// ---------------------------------------------------------------- launchers
void launch_deposit(Ctx& c) {
    c.jw.zero(c.stream);
    if (c.np == 0) return;
    const int tok = c.prof_begin("deposit");
    const unsigned blocks = unsigned((c.np + 255) / 256);
    k_deposit<<<blocks, 256, 0, c.stream>>>(c.parts, c.np, c.geo(), c.jw.p);
    c.check_launch("k_deposit");
    c.prof_end(tok);
}

template <int NY>
static void cur_cols(Ctx& c) {
    constexpr int CW = 8;
    const Geo g = c.geo();
    const int cw = c.nx < CW ? c.nx : CW;
    if (cw != CW) throw Error(G3D_ERR_ARG, "nx must be >= 8");
    const size_t smem = size_t(2) * NY * CW * sizeof(cpx);
    auto kern = k_cur_cols<NY, CW>;
    G3D_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    const dim3 grid(unsigned(c.nx / CW), unsigned(c.ns + 1));
    const int tok = c.prof_begin("cur_cols");
    kern<<<grid, CW * FftShape<NY>::T, smem, c.stream>>>(g, c.jw.p, c.S1.p, c.jkz.p, c.P.zeta_filter ? 1 : 0);
    c.check_launch("k_cur_cols");
    c.prof_end(tok);
}
template <int NX>
static void cur_rows(Ctx& c, bool keep0) {
    using S = FftShape<NX>;
    constexpr int LPC = 128 / S::T, PPC = LPC / 2;
    const size_t smem = size_t(2) * LPC * row_stride<NX>() * sizeof(cpx);
    auto kern = k_cur_rows<NX>;
    G3D_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    const dim3 grid(unsigned((c.ny / 2 + 1 + PPC - 1) / PPC), unsigned(c.ns + 1));
    const int tok = c.prof_begin("cur_rows");
    kern<<<grid, 128, smem, c.stream>>>(c.geo(), c.S1.p, c.jkx.p, c.jky.p, c.jkz.p, keep0 ? 1 : 0);
    c.check_launch("k_cur_rows");
    c.prof_end(tok);
}

void launch_cur_fft(Ctx& c, bool keep0) {
    G3D_DISPATCH_N(c.ny, NY, cur_cols<NY>(c));
    G3D_DISPATCH_N(c.nx, NX, cur_rows<NX>(c, keep0));
}

}  // namespace g3d
