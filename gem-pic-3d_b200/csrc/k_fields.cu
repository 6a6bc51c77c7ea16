// Sponge and real-space fields (Simulation::sponge_and_real_fields, src/sim_fields.cpp:156-307, Fourier y),
// the window shift (src/sim_setup.cpp:249-281), the half <-> full spectrum layouts and small elementwise kernels.
//
// The spectra are kept for k_x = 0 .. nx/2 (H columns): every field is real, so X(-k) = conj X(k).
// A transverse 2-D transform is a pass along y over the H columns (k_*_cols) and a pass along x over the
// rows (k_*_rows), where a row's other half follows from X(nx - k_x) = conj X(k_x) of the y-transformed data.
//
// Sponge: the radiation part R - R_b of the forward field (R_b = (1 + beta) E_perp of the slice charge,
// psi = (rho + gamma^-2 d_zeta^2 rho / k^2) / k^2) is multiplied in real space by maskx(x) masky(y):
//   k_sp_cols_inv  bound field psi -> W3, U = R_x - R_bx and V = R_y - R_by, inverse FFT along y
//   k_sp_rows      per row: u + i v by one inverse FFT along x, 1/(nx ny), the mask, one forward FFT along x,
//                  split back into the half spectra of u and v
//   k_sp_cols_fwd  forward FFT along y, + R_b
// Real fields: k_rf_cols transforms R_x, R_y, L_x, L_y, E_z, B_z along y (a pair per CTA); k_rf_rows rebuilds R_x + i R_y,
// L_x + i L_y, E_z + i B_z per row, transforms along x and writes the six float components of F with the
// reference's combinations (E_x = (r1 + l1)/2, ...).
#include "g3d_ctx.hpp"
#include "k_fft.cuh"
#include "k_dispatch.cuh"
#include "k_tma.cuh"

namespace g3d {

namespace {
constexpr int NT = 128;    // threads of the row kernels
constexpr int CW = 8;      // columns per tile of the column kernels

// psi of the slice charge of slice n = a + l at the half-spectrum mode i (reference: the Fourier-y lambda
// of sim_fields.cpp:176-201)
__device__ __forceinline__ cpx bound_psi(const Geo& g, const cpx* __restrict__ jz, const cpx* __restrict__ jg, int l, long i,
                                         double kx, double ky, double g2) {
    const long nk = g.nkh;
    const int n = g.a + l;
    auto half = [&](int hk) -> cpx {
        if (hk < 0) return jg[i];
        if (hk > g.ns) return jg[nk + i];
        return jz[long(hk) * nk + i];
    };
    auto rho_at = [&](int dl) -> cpx {
        const int nn = n + dl;
        if (nn < 0 || nn > g.N - 1) return C(0);
        return g.wlo[nn] * half(l + dl) + g.whi[nn] * half(l + dl + 1);
    };
    const double hm = g.hcg[n + 1], hp = g.hcg[n + 2];
    const double cm = 2 / ((hm + hp) * hm), cp_ = 2 / ((hm + hp) * hp);
    const double k2 = kx * kx + ky * ky;
    cpx psi = C(0);
    if (k2 > 0) {
        const cpx d2 = g2 * (cp_ * rho_at(1) - (cm + cp_) * rho_at(0) + cm * rho_at(-1));
        psi = (rho_at(0) + d2 / k2) / k2;
    }
    return psi;
}

// Full row z[0..NX) from the half rows A, B (k_x = 0..NX/2) of two real fields: z = A + i B with
// A(NX - k) = conj A(k), B(NX - k) = conj B(k); stored conjugated for an inverse transform.
template <int NX>
__device__ __forceinline__ void full_row_conj(cpx* line, int p, cpx a, cpx b, bool mirror) {
    // p in 0..NX/2: position p gets a + i b; its mirror NX - p gets conj(a) + i conj(b)
    const cpx z = C(a.x - b.y, a.y + b.x);
    line[p + (p >> 3)] = conj(z);
    if (mirror) {
        const int q = NX - p;
        const cpx zm = C(a.x + b.y, -a.y + b.x);                     // conj(a) + i conj(b)
        line[q + (q >> 3)] = conj(zm);
    }
}
}  // namespace

// ---------------------------------------------------------------- sponge, pass 1: columns (psi, pack, inverse y)
template <int NY>
__global__ void __launch_bounds__(CW * FftShape<NY>::T) k_sp_cols_inv(Geo g, const cpx* __restrict__ Rx, const cpx* __restrict__ Ry,
                                                                      const cpx* __restrict__ jz, const cpx* __restrict__ jg,
                                                                      cpx* __restrict__ U, cpx* __restrict__ V,
                                                                      cpx* __restrict__ PSI, double g2, double opb) {
    using S = FftShape<NY>;
    extern __shared__ cpx sm[];
    cpx* s0 = sm;
    cpx* s1 = sm + ColTile<NY, CW>::size;
    const int l = blockIdx.y, c0 = blockIdx.x * CW, tid = threadIdx.x, nthr = CW * S::T;
    const int H = g.H;
    const long base = long(l) * g.nkh;
    #pragma unroll
    for (int u_ = 0; u_ < (NY * CW + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * CW) break;
        const int p = e / CW, c = e - p * CW, kxi = c0 + c;
        cpx u = C(0), v = C(0);
        if (kxi < H) {
            const long i = long(p) * H + kxi, o = base + i;
            const double kx = g.kxd[kxi], ky = g.kyd[p];
            const cpx psi = bound_psi(g, jz, jg, l, i, kx, ky, g2);
            PSI[o] = psi;
            u = Rx[o] - (-opb * ik(kx, psi));
            v = Ry[o] - (-opb * ik(ky, psi));
        }
        s0[ColTile<NY, CW>::at(p, c)] = conj(u);
        s1[ColTile<NY, CW>::at(p, c)] = conj(v);
    }
    __syncthreads();
    const int c = tid % CW, t = tid / CW;
    {
        decltype(s0) const ls_[2] = {s0, s1};
        fft_lines<NY, 2>(ls_, RowAddr{c * ColTile<NY, CW>::RS}, t, g.twy);
    }
    #pragma unroll
    for (int u_ = 0; u_ < (NY * CW + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * CW) break;
        const int p = e / CW, cc = e - p * CW, kxi = c0 + cc;
        if (kxi >= H) continue;
        const long o = base + long(p) * H + kxi;
        U[o] = conj(s0[ColTile<NY, CW>::at(p, cc)]);
        V[o] = conj(s1[ColTile<NY, CW>::at(p, cc)]);
    }
}

// The same with the tiles of R_x, R_y (maps 0, 1) loaded by the TMA (k_tma.cuh); psi per element as above.
template <int NY>
__global__ void __launch_bounds__(8 * FftShape<NY>::T) k_sp_cols_inv_tma(Geo g, const __grid_constant__ TileMaps maps,
                                                                        const cpx* __restrict__ jz, const cpx* __restrict__ jg,
                                                                        cpx* __restrict__ U, cpx* __restrict__ V,
                                                                        cpx* __restrict__ PSI, double g2, double opb,
                                                                        TmaWait wt) {
    using S = FftShape<NY>;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int ok;
    const int l = blockIdx.y, c0 = blockIdx.x * 8, tid = threadIdx.x, nthr = 8 * S::T;
    const int H = g.H;
    const long base = long(l) * g.nkh;
    cpx* s0 = reinterpret_cast<cpx*>(smraw + ((128 - (smem_addr(smraw) & 127)) & 127));
    cpx* s1 = s0 + NY * 8;
    const int idx[2] = {0, 1};
    cpx* const dst[2] = {s0, s1};
    if (!tma_tiles<NY>(maps, idx, 2, dst, c0, l * g.ny, &bar, &ok, wt)) return;
    #pragma unroll
    for (int u_ = 0; u_ < (NY * 8 + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * 8) break;
        const int p = e / 8, c = e - p * 8, kxi = c0 + c;
        cpx u = C(0), v = C(0);
        if (kxi < H) {
            const long i = long(p) * H + kxi, o = base + i;
            const double kx = g.kxd[kxi], ky = g.kyd[p];
            const cpx psi = bound_psi(g, jz, jg, l, i, kx, ky, g2);
            PSI[o] = psi;
            u = s0[e] - (-opb * ik(kx, psi));
            v = s1[e] - (-opb * ik(ky, psi));
        }
        s0[e] = conj(u);
        s1[e] = conj(v);
    }
    __syncthreads();
    const int c = tid % 8, t = tid / 8;
    {
        decltype(s0) const ls_[2] = {s0, s1};
        fft_lines<NY, 2>(ls_, TileCol{c}, t, g.twy);
    }
    #pragma unroll
    for (int u_ = 0; u_ < (NY * 8 + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * 8) break;
        const int p = e / 8, cc = e - p * 8, kxi = c0 + cc;
        if (kxi >= H) continue;
        const long o = base + long(p) * H + kxi;
        U[o] = conj(s0[e]);
        V[o] = conj(s1[e]);
    }
}

// ---------------------------------------------------------------- sponge, pass 2: rows (inverse x, mask, forward x)
template <int NX>
__global__ void __launch_bounds__(NT) k_sp_rows(Geo g, cpx* __restrict__ U, cpx* __restrict__ V) {
    using S = FftShape<NX>;
    constexpr int LPC = NT / S::T, RS = row_stride<NX>(), H = NX / 2 + 1;
    extern __shared__ cpx sm[];
    const int l = blockIdx.y, r0 = blockIdx.x * LPC, tid = threadIdx.x;
    const long base = long(l) * g.nkh;
    #pragma unroll
    for (int u_ = 0; u_ < (LPC * H + NT - 1) / NT; ++u_) {
        const int e = tid + u_ * NT;
        if (e >= LPC * H) break;
        const int r = e / H, p = e - r * H, row = r0 + r;
        cpx a = C(0), b = C(0);
        if (row < g.ny) { const long o = base + long(row) * H + p; a = U[o]; b = V[o]; }
        full_row_conj<NX>(sm + r * RS, p, a, b, p > 0 && p < NX / 2);
    }
    __syncthreads();
    const int r = tid / S::T, t = tid - r * S::T;
    fft_line<NX>(sm, RowAddr{r * RS}, t, g.twx);
    const double s = g.yf ? 1.0 / double(g.nk) : 1.0 / double(g.nx);   // free-hand y: rows only, 1/nx
    #pragma unroll
    for (int u_ = 0; u_ < (LPC * NX + NT - 1) / NT; ++u_) {
        const int e = tid + u_ * NT;
        if (e >= LPC * NX) break;
        const int rr = e / NX, p = e - rr * NX, row = r0 + rr;
        const int q = rr * RS + p + (p >> 3);
        const cpx z = s * conj(sm[q]);                                  // u + i v in real space
        const double mx = g.maskx[p];
        const double mn = row < g.ny ? g.masky_n[row] : 0.0, mh = row < g.ny ? g.masky_h[row] : 0.0;
        sm[q] = C(mx * mn * z.x, mx * mh * z.y);
    }
    __syncthreads();
    fft_line<NX>(sm, RowAddr{r * RS}, t, g.twx);
    #pragma unroll
    for (int u_ = 0; u_ < (LPC * H + NT - 1) / NT; ++u_) {
        const int e = tid + u_ * NT;
        if (e >= LPC * H) break;
        const int rr = e / H, p = e - rr * H, row = r0 + rr;
        if (row >= g.ny) continue;
        const int pm = (NX - p) % NX;
        const cpx z = sm[rr * RS + p + (p >> 3)], zm = conj(sm[rr * RS + pm + (pm >> 3)]);
        const cpx d = z - zm;
        const long o = base + long(row) * H + p;
        U[o] = 0.5 * (z + zm);
        V[o] = 0.5 * C(d.y, -d.x);
    }
}

// ---------------------------------------------------------------- sponge, pass 3: columns (forward y, + R_b)
template <int NY>
__global__ void __launch_bounds__(CW * FftShape<NY>::T) k_sp_cols_fwd(Geo g, const cpx* __restrict__ U, const cpx* __restrict__ V,
                                                                      const cpx* __restrict__ PSI, cpx* __restrict__ Rx,
                                                                      cpx* __restrict__ Ry, double opb) {
    using S = FftShape<NY>;
    extern __shared__ cpx sm[];
    cpx* s0 = sm;
    cpx* s1 = sm + ColTile<NY, CW>::size;
    const int l = blockIdx.y, c0 = blockIdx.x * CW, tid = threadIdx.x, nthr = CW * S::T;
    const int H = g.H;
    const long base = long(l) * g.nkh;
    #pragma unroll
    for (int u_ = 0; u_ < (NY * CW + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * CW) break;
        const int p = e / CW, c = e - p * CW, kxi = c0 + c;
        cpx u = C(0), v = C(0);
        if (kxi < H) { const long o = base + long(p) * H + kxi; u = U[o]; v = V[o]; }
        s0[ColTile<NY, CW>::at(p, c)] = u; s1[ColTile<NY, CW>::at(p, c)] = v;
    }
    __syncthreads();
    const int c = tid % CW, t = tid / CW;
    {
        decltype(s0) const ls_[2] = {s0, s1};
        fft_lines<NY, 2>(ls_, RowAddr{c * ColTile<NY, CW>::RS}, t, g.twy);
    }
    #pragma unroll
    for (int u_ = 0; u_ < (NY * CW + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * CW) break;
        const int p = e / CW, cc = e - p * CW, kxi = c0 + cc;
        if (kxi >= H) continue;
        const long o = base + long(p) * H + kxi;
        const cpx psi = PSI[o];
        Rx[o] = s0[ColTile<NY, CW>::at(p, cc)] - opb * ik(g.kxd[kxi], psi);
        Ry[o] = s1[ColTile<NY, CW>::at(p, cc)] - opb * ik(g.kyd[p], psi);
    }
}

// The same with the tiles of U, V, PSI (maps 0, 1, 2) loaded by the TMA (k_tma.cuh).
template <int NY>
__global__ void __launch_bounds__(8 * FftShape<NY>::T) k_sp_cols_fwd_tma(Geo g, const __grid_constant__ TileMaps maps,
                                                                        cpx* __restrict__ Rx, cpx* __restrict__ Ry, double opb,
                                                                        TmaWait wt) {
    using S = FftShape<NY>;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int ok;
    const int l = blockIdx.y, c0 = blockIdx.x * 8, tid = threadIdx.x, nthr = 8 * S::T;
    const int H = g.H;
    const long base = long(l) * g.nkh;
    cpx* s0 = reinterpret_cast<cpx*>(smraw + ((128 - (smem_addr(smraw) & 127)) & 127));
    cpx* s1 = s0 + NY * 8;
    cpx* s2 = s1 + NY * 8;
    const int idx[3] = {0, 1, 2};
    cpx* const dst[3] = {s0, s1, s2};
    if (!tma_tiles<NY>(maps, idx, 3, dst, c0, l * g.ny, &bar, &ok, wt)) return;
    const int c = tid % 8, t = tid / 8;
    {
        decltype(s0) const ls_[2] = {s0, s1};
        fft_lines<NY, 2>(ls_, TileCol{c}, t, g.twy);
    }
    #pragma unroll
    for (int u_ = 0; u_ < (NY * 8 + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * 8) break;
        const int p = e / 8, cc = e - p * 8, kxi = c0 + cc;
        if (kxi >= H) continue;
        const long o = base + long(p) * H + kxi;
        const cpx psi = s2[e];
        Rx[o] = s0[e] - opb * ik(g.kxd[kxi], psi);
        Ry[o] = s1[e] - opb * ik(g.kyd[p], psi);
    }
}

// ---------------------------------------------------------------- real fields: columns (inverse y of the six spectra)
// blockIdx.z picks the pair (R_x, R_y), (L_x, L_y) or (E_z, B_z): two fields per CTA keep the shared memory small
// enough for several CTAs per SM, so loads of one CTA overlap the transforms of another.
template <int NY, int CWT>
__global__ void __launch_bounds__(CWT * FftShape<NY>::T) k_rf_cols(Geo g, const cpx* __restrict__ Rx, const cpx* __restrict__ Ry,
                                                                  const cpx* __restrict__ Lx, const cpx* __restrict__ Ly,
                                                                  const cpx* __restrict__ Ez, const cpx* __restrict__ Bz,
                                                                  cpx* __restrict__ W0, cpx* __restrict__ W1, cpx* __restrict__ W2,
                                                                  cpx* __restrict__ W3, cpx* __restrict__ W4, cpx* __restrict__ W5,
                                                                  int l0) {
    using S = FftShape<NY>;
    extern __shared__ cpx sm[];
    const int l = l0 + blockIdx.y, c0 = blockIdx.x * CWT, tid = threadIdx.x, nthr = CWT * S::T, pr = blockIdx.z;
    const int H = g.H;
    const long base = long(l) * g.nkh;
    const cpx* in0 = pr == 0 ? Rx : pr == 1 ? Lx : Ez;
    const cpx* in1 = pr == 0 ? Ry : pr == 1 ? Ly : Bz;
    cpx* out0 = pr == 0 ? W0 : pr == 1 ? W2 : W4;
    cpx* out1 = pr == 0 ? W1 : pr == 1 ? W3 : W5;
    cpx* s0 = sm;
    cpx* s1 = sm + ColTile<NY, CWT>::size;
    #pragma unroll
    for (int u_ = 0; u_ < (NY * CWT + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * CWT) break;
        const int p = e / CWT, c = e - p * CWT, kxi = c0 + c;
        const long o = base + long(p) * H + kxi;
        s0[ColTile<NY, CWT>::at(p, c)] = kxi < H ? conj(in0[o]) : C(0);
        s1[ColTile<NY, CWT>::at(p, c)] = kxi < H ? conj(in1[o]) : C(0);
    }
    __syncthreads();
    const int c = tid % CWT, t = tid / CWT;
    {
        decltype(s0) const ls_[2] = {s0, s1};
        fft_lines<NY, 2>(ls_, RowAddr{c * ColTile<NY, CWT>::RS}, t, g.twy);
    }
    #pragma unroll
    for (int u_ = 0; u_ < (NY * CWT + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * CWT) break;
        const int p = e / CWT, cc = e - p * CWT, kxi = c0 + cc;
        if (kxi >= H) continue;
        const long o = base + long(p) * H + kxi;
        out0[o] = conj(s0[ColTile<NY, CWT>::at(p, cc)]);
        out1[o] = conj(s1[ColTile<NY, CWT>::at(p, cc)]);
    }
}

// The same transforms of the whole window with the tiles loaded by the TMA (k_tma.cuh): the 8-column tiles of the
// pair land row-major in shared memory, are conjugated in place, transformed along their columns (stride 8) and
// written back conjugated; maps 0..5 are R_x, R_y, L_x, L_y, E_z, B_z.
template <int NY>
__global__ void __launch_bounds__(8 * FftShape<NY>::T) k_rf_cols_tma(Geo g, const __grid_constant__ TileMaps maps,
                                                                    cpx* __restrict__ W0, cpx* __restrict__ W1,
                                                                    cpx* __restrict__ W2, cpx* __restrict__ W3,
                                                                    cpx* __restrict__ W4, cpx* __restrict__ W5, int l0,
                                                                    TmaWait wt) {
    using S = FftShape<NY>;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int ok;
    const int l = l0 + blockIdx.y, c0 = blockIdx.x * 8, tid = threadIdx.x, nthr = 8 * S::T, pr = blockIdx.z;
    const int H = g.H;
    const long base = long(l) * g.nkh;
    cpx* s0 = reinterpret_cast<cpx*>(smraw + ((128 - (smem_addr(smraw) & 127)) & 127));
    cpx* s1 = s0 + NY * 8;
    cpx* out0 = pr == 0 ? W0 : pr == 1 ? W2 : W4;
    cpx* out1 = pr == 0 ? W1 : pr == 1 ? W3 : W5;
    const int idx[2] = {2 * pr, 2 * pr + 1};
    cpx* const dst[2] = {s0, s1};
    if (!tma_tiles<NY>(maps, idx, 2, dst, c0, l * g.ny, &bar, &ok, wt)) return;
    for (int e = tid; e < NY * 8; e += nthr) { s0[e] = conj(s0[e]); s1[e] = conj(s1[e]); }
    __syncthreads();
    const int c = tid % 8, t = tid / 8;
    {
        decltype(s0) const ls_[2] = {s0, s1};
        fft_lines<NY, 2>(ls_, TileCol{c}, t, g.twy);
    }
    #pragma unroll
    for (int u_ = 0; u_ < (NY * 8 + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * 8) break;
        const int p = e / 8, cc = e - p * 8, kxi = c0 + cc;
        if (kxi >= H) continue;
        const long o = base + long(p) * H + kxi;
        out0[o] = conj(s0[e]);
        out1[o] = conj(s1[e]);
    }
}

// ---------------------------------------------------------------- real fields: rows (inverse x, F)
// XM (exact fields with midpoint fields, FP64 Fourier y): the midpoint fields from the FP64 values of both slices
// (Fd), so that the streaming push of the exact forward gathers unrounded fields like the beam push does
template <int NX, bool XM = false>
__global__ void __launch_bounds__(NT) k_rf_rows(Geo g, const cpx* __restrict__ W0, const cpx* __restrict__ W1,
                                               const cpx* __restrict__ W2, const cpx* __restrict__ W3,
                                               const cpx* __restrict__ W4, const cpx* __restrict__ W5, float* __restrict__ F, int l0,
                                               double* __restrict__ Fd, FmidOut fm) {
    using S = FftShape<NX>;
    constexpr int LPC = NT / S::T, RS = row_stride<NX>(), H = NX / 2 + 1;
    extern __shared__ cpx sm[];
    cpx* a0 = sm;
    cpx* a1 = sm + LPC * RS;
    cpx* a2 = sm + 2 * LPC * RS;
    const int l = l0 + blockIdx.y, r0 = blockIdx.x * LPC, tid = threadIdx.x;
    const long base = long(l) * g.nkh;
    const long fpl = long(g.ns + 2) * g.nk, fbase = long(l) * g.nk;
    constexpr int EO = (LPC * NX + NT - 1) / NT;                    // output elements of a thread
    float oth[XM ? 1 : EO][6];                                      // the midpoint fields' other slice
    double othd[XM ? EO : 1][6];
    if (fm.out) {
    #pragma unroll
        for (int u_ = 0; u_ < EO; ++u_) {
            const int e = tid + u_ * NT, rr = e / NX, p = e - rr * NX, row = r0 + rr;
            if (e >= LPC * NX || row >= g.ny) continue;
            if constexpr (XM) {
#pragma unroll
                for (int comp = 0; comp < 6; ++comp) othd[u_][comp] = Fd[comp * fpl + long(fm.other) * g.nk + long(row) * NX + p];
            } else {
                fmid_load(fm, F, fpl, g.nk, long(row) * NX + p, oth[u_]);
            }
        }
    }
    #pragma unroll
    for (int u_ = 0; u_ < (LPC * H + NT - 1) / NT; ++u_) {      // unrolled: the loads of all elements in flight
        const int e = tid + u_ * NT;
        if (e >= LPC * H) continue;
        const int r = e / H, p = e - r * H, row = r0 + r;
        cpx v[6] = {C(0), C(0), C(0), C(0), C(0), C(0)};
        if (row < g.ny) {
            const long o = base + long(row) * H + p;
            v[0] = W0[o]; v[1] = W1[o]; v[2] = W2[o]; v[3] = W3[o]; v[4] = W4[o]; v[5] = W5[o];
        }
        const bool mirror = p > 0 && p < NX / 2;
        full_row_conj<NX>(a0 + r * RS, p, v[0], v[1], mirror);
        full_row_conj<NX>(a1 + r * RS, p, v[2], v[3], mirror);
        full_row_conj<NX>(a2 + r * RS, p, v[4], v[5], mirror);
    }
    __syncthreads();
    const int r = tid / S::T, t = tid - r * S::T;
    {
        decltype(a0) const ls_[3] = {a0, a1, a2};
        fft_lines<NX, 3>(ls_, RowAddr{r * RS}, t, g.twx);
    }
    const double s = g.yf ? 1.0 / double(g.nk) : 1.0 / double(g.nx);   // free-hand y: rows only, 1/nx
    #pragma unroll
    for (int u_ = 0; u_ < EO; ++u_) {
        const int e = tid + u_ * NT;
        if (e >= LPC * NX) continue;
        const int rr = e / NX, p = e - rr * NX, row = r0 + rr;
        if (row >= g.ny) continue;
        const int q = rr * RS + p + (p >> 3);
        const cpx z1 = s * conj(a0[q]), z2 = s * conj(a1[q]), z3 = s * conj(a2[q]);
        const long idx = fbase + long(row) * NX + p;
        const double r1 = z1.x, r2 = z1.y, l1 = z2.x, l2 = z2.y;
        const float fv[6] = {float(0.5 * (r1 + l1)), float(0.5 * (r2 + l2)), float(z3.x),    // E_x, E_y, E_z
                             float(0.5 * (l2 - r2)), float(0.5 * (r1 - l1)), float(z3.y)};  // B_x, B_y, B_z
#pragma unroll
        for (int comp = 0; comp < 6; ++comp) F[comp * fpl + idx] = fv[comp];
        if constexpr (XM) {
            const double dv[6] = {0.5 * (r1 + l1), 0.5 * (r2 + l2), z3.x, 0.5 * (l2 - r2), 0.5 * (r1 - l1), z3.y};
            if (fm.rec_f) {                            // the adjoint's record of the slice
                double* R = *fm.rec_f + fm.rec_off + long(row) * NX + p;
#pragma unroll
                for (int comp = 0; comp < 6; ++comp) R[comp * g.nk] = dv[comp];
            }
            double2* o = reinterpret_cast<double2*>(fm.out) + 3 * (long(row) * NX + p);
            o[0] = make_double2(0.5 * (dv[0] + othd[u_][0]), 0.5 * (dv[1] + othd[u_][1]));
            o[1] = make_double2(0.5 * (dv[2] + othd[u_][2]), 0.5 * (dv[3] + othd[u_][3]));
            o[2] = make_double2(0.5 * (dv[4] + othd[u_][4]), 0.5 * (dv[5] + othd[u_][5]));
        } else if (fm.out) {
            fmid_store(fm, long(row) * NX + p, fv, oth[u_]);
        }
        if (Fd) {                                      // exact fields: the same values before the rounding
            Fd[0 * fpl + idx] = 0.5 * (r1 + l1); Fd[1 * fpl + idx] = 0.5 * (r2 + l2);
            Fd[3 * fpl + idx] = 0.5 * (l2 - r2); Fd[4 * fpl + idx] = 0.5 * (r1 - l1);
            Fd[2 * fpl + idx] = z3.x; Fd[5 * fpl + idx] = z3.y;
        }
    }
}

// ---------------------------------------------------------------- launchers
template <class K>
static void allow_smem(K kern, size_t smem) {
    smem_attr(reinterpret_cast<const void*>(kern), smem);
}
static unsigned col_tiles(const Ctx& c) { return unsigned((c.H + CW - 1) / CW); }

template <int NY>
static void sp_cols_inv(Ctx& c) {
    if constexpr (NY <= 256 && (NY & (NY - 1)) == 0) {
        const cpx* p[2] = {c.Rx.p, c.Ry.p};
        if (c.use_tma && c.tma_spi.get(p, 2, c.H, long(c.ns) * c.ny, c.ny)) {
            const size_t smem = size_t(2) * NY * 8 * sizeof(cpx) + 128;
            allow_smem(k_sp_cols_inv_tma<NY>, smem);
            const int tok = c.prof_begin("sponge_cols_inv");
            k_sp_cols_inv_tma<NY><<<dim3(col_tiles(c), unsigned(c.ns)), 8 * FftShape<NY>::T, smem, c.stream>>>(
                c.geo(), c.tma_spi.maps, c.jkz.p, c.jzg.p, c.W[0].p, c.W[1].p, c.W[3].p, c.gm2_b, 1 + c.beta_b, c.tma_wait());
            c.check_launch("k_sp_cols_inv_tma");
            c.prof_end(tok);
            return;
        }
    }
    const size_t smem = size_t(2) * ColTile<NY, CW>::size * sizeof(cpx);
    allow_smem(k_sp_cols_inv<NY>, smem);
    const int tok = c.prof_begin("sponge_cols_inv");
    k_sp_cols_inv<NY><<<dim3(col_tiles(c), unsigned(c.ns)), CW * FftShape<NY>::T, smem, c.stream>>>(
        c.geo(), c.Rx.p, c.Ry.p, c.jkz.p, c.jzg.p, c.W[0].p, c.W[1].p, c.W[3].p, c.gm2_b, 1 + c.beta_b);
    c.check_launch("k_sp_cols_inv");
    c.prof_end(tok);
}
template <int NX>
static void sp_rows(Ctx& c) {
    constexpr int LPC = NT / FftShape<NX>::T;
    const size_t smem = size_t(LPC) * row_stride<NX>() * sizeof(cpx);
    allow_smem(k_sp_rows<NX>, smem);
    const int tok = c.prof_begin("sponge_rows");
    k_sp_rows<NX><<<dim3(unsigned((c.ny + LPC - 1) / LPC), unsigned(c.ns)), NT, smem, c.stream>>>(c.geo(), c.W[0].p, c.W[1].p);
    c.check_launch("k_sp_rows");
    c.prof_end(tok);
}
template <int NY>
static void sp_cols_fwd(Ctx& c) {
    if constexpr (NY <= 256 && (NY & (NY - 1)) == 0) {
        const cpx* p[3] = {c.W[0].p, c.W[1].p, c.W[3].p};
        if (c.use_tma && c.tma_spf.get(p, 3, c.H, long(c.ns) * c.ny, c.ny)) {
            const size_t smem = size_t(3) * NY * 8 * sizeof(cpx) + 128;
            allow_smem(k_sp_cols_fwd_tma<NY>, smem);
            const int tok = c.prof_begin("sponge_cols_fwd");
            k_sp_cols_fwd_tma<NY><<<dim3(col_tiles(c), unsigned(c.ns)), 8 * FftShape<NY>::T, smem, c.stream>>>(
                c.geo(), c.tma_spf.maps, c.Rx.p, c.Ry.p, 1 + c.beta_b, c.tma_wait());
            c.check_launch("k_sp_cols_fwd_tma");
            c.prof_end(tok);
            return;
        }
    }
    const size_t smem = size_t(2) * ColTile<NY, CW>::size * sizeof(cpx);
    allow_smem(k_sp_cols_fwd<NY>, smem);
    const int tok = c.prof_begin("sponge_cols_fwd");
    k_sp_cols_fwd<NY><<<dim3(col_tiles(c), unsigned(c.ns)), CW * FftShape<NY>::T, smem, c.stream>>>(
        c.geo(), c.W[0].p, c.W[1].p, c.W[3].p, c.Rx.p, c.Ry.p, 1 + c.beta_b);
    c.check_launch("k_sp_cols_fwd");
    c.prof_end(tok);
}
void launch_sponge(Ctx& c) {
    G3D_DISPATCH_N(c.ny, NY, sp_cols_inv<NY>(c));
    G3D_DISPATCH_N(c.nx, NX, sp_rows<NX>(c));
    G3D_DISPATCH_N(c.ny, NY, sp_cols_fwd<NY>(c));
}

// one slice (the plasma march): tiles of 2 columns, so that 3 x 65 CTAs spread the slice's latency over the SMs
template <int NY, int CWT>
static void rf_cols_w(Ctx& c, int l0, int nl) {
    const size_t smem = size_t(2) * ColTile<NY, CWT>::size * sizeof(cpx);
    allow_smem(k_rf_cols<NY, CWT>, smem);
    const int tok = c.prof_begin(nl == 1 ? "real_cols_slice" : "real_cols");
    k_rf_cols<NY, CWT><<<dim3(unsigned((c.H + CWT - 1) / CWT), unsigned(nl), 3), CWT * FftShape<NY>::T, smem, c.stream>>>(
        c.geo(), c.Rx.p, c.Ry.p, c.Lx.p, c.Ly.p, c.Ez.p, c.Bz.p, c.W[0].p, c.W[1].p, c.W[2].p, c.W[3].p, c.W[4].p, c.W[5].p, l0);
    c.check_launch("k_rf_cols");
    c.prof_end(tok);
}
// the tensor maps of R_x, R_y, L_x, L_y, E_z, B_z for tiles of 8 columns x ny rows, made once per set of buffers;
// false where the TMA path does not apply (ny > 256, or the encoder is unavailable)
static bool rf_maps(Ctx& c) {
    const cpx* p[6] = {c.Rx.p, c.Ry.p, c.Lx.p, c.Ly.p, c.Ez.p, c.Bz.p};
    return c.tma_rf.get(p, 6, c.H, long(c.ns) * c.ny, c.ny);
}
template <int NY>
static void rf_cols_tma(Ctx& c, int l0, int nl) {
    const size_t smem = size_t(2) * NY * 8 * sizeof(cpx) + 128;
    allow_smem(k_rf_cols_tma<NY>, smem);
    const int tok = c.prof_begin("real_cols");
    k_rf_cols_tma<NY><<<dim3(unsigned((c.H + 7) / 8), unsigned(nl), 3), 8 * FftShape<NY>::T, smem, c.stream>>>(
        c.geo(), c.tma_rf.maps, c.W[0].p, c.W[1].p, c.W[2].p, c.W[3].p, c.W[4].p, c.W[5].p, l0, c.tma_wait());
    c.check_launch("k_rf_cols_tma");
    c.prof_end(tok);
}
template <int NY>
static void rf_cols(Ctx& c, int l0, int nl) {
    if (nl == 1) { rf_cols_w<NY, 2>(c, l0, nl); return; }
    if constexpr (NY <= 256 && (NY & (NY - 1)) == 0) {
        if (c.use_tma && rf_maps(c)) { rf_cols_tma<NY>(c, l0, nl); return; }
    }
    rf_cols_w<NY, CW>(c, l0, nl);
}
template <int NX>
static void rf_rows(Ctx& c, int l0, int nl, FmidOut fm = FmidOut()) {
    constexpr int LPC = NT / FftShape<NX>::T;
    const size_t smem = size_t(3) * LPC * row_stride<NX>() * sizeof(cpx);
    const int tok = c.prof_begin(nl == 1 ? "real_rows_slice" : "real_rows");
    const dim3 grid(unsigned((c.ny + LPC - 1) / LPC), unsigned(nl));
    if (c.Fd.p && fm.out && !fm.f32 && !fm.fh) {       // exact fields: unrounded midpoint fields
        allow_smem(k_rf_rows<NX, true>, smem);
        k_rf_rows<NX, true><<<grid, NT, smem, c.stream>>>(c.geo(), c.W[0].p, c.W[1].p, c.W[2].p, c.W[3].p, c.W[4].p, c.W[5].p, c.F.p,
                                                          l0, c.Fd.p, fm);
    } else {
        allow_smem(k_rf_rows<NX>, smem);
        k_rf_rows<NX><<<grid, NT, smem, c.stream>>>(c.geo(), c.W[0].p, c.W[1].p, c.W[2].p, c.W[3].p, c.W[4].p, c.W[5].p, c.F.p, l0,
                                                    c.Fd.p, fm);
    }
    c.check_launch("k_rf_rows");
    c.prof_end(tok);
}
void launch_real_fields(Ctx& c) {
    G3D_DISPATCH_N(c.ny, NY, rf_cols<NY>(c, 0, c.ns));
    G3D_DISPATCH_N(c.nx, NX, rf_rows<NX>(c, 0, c.ns));
}
// free-hand y: the spectra are already real in y; one inverse transform along x per row of R, L and E_z + i B_z
template <int NX>
static void rf_rows_direct(Ctx& c, int l0, int nl, FmidOut fm = FmidOut()) {
    constexpr int LPC = NT / FftShape<NX>::T;
    const size_t smem = size_t(3) * LPC * row_stride<NX>() * sizeof(cpx);
    allow_smem(k_rf_rows<NX>, smem);
    const int tok = c.prof_begin(nl == 1 ? "real_rows_slice" : "real_rows");
    k_rf_rows<NX><<<dim3(unsigned((c.ny + LPC - 1) / LPC), unsigned(nl)), NT, smem, c.stream>>>(
        c.geo(), c.Rx.p, c.Ry.p, c.Lx.p, c.Ly.p, c.Ez.p, c.Bz.p, c.F.p, l0, c.Fd.p, fm);
    c.check_launch("k_rf_rows");
    c.prof_end(tok);
}
void launch_real_fields_fh(Ctx& c) { G3D_DISPATCH_N(c.nx, NX, rf_rows_direct<NX>(c, 0, c.ns)); }
void launch_real_fields_slice_fh(Ctx& c, int l, FmidOut fm) { G3D_DISPATCH_N(c.nx, NX, rf_rows_direct<NX>(c, l, 1, fm)); }
// the sponge's row pass alone (inverse x, mask, forward x) on W0, W1: the free-hand y sponge
void launch_sp_rows(Ctx& c) { G3D_DISPATCH_N(c.nx, NX, sp_rows<NX>(c)); }
// E and B of one slice (plane l) in real space (Simulation::real_fields_slice, src/sim_plasma.cpp:200-220)
void launch_real_fields_slice(Ctx& c, int l, FmidOut fm, bool cols) {
    if (cols) G3D_DISPATCH_N(c.ny, NY, rf_cols<NY>(c, l, 1));
    G3D_DISPATCH_N(c.nx, NX, rf_rows<NX>(c, l, 1, fm));
}

// ---------------------------------------------------------------- half <-> full spectrum layouts
// full[p][j][ix] = half[p][j][ix] (ix <= nx/2), conj(half[p][(ny - j) % ny][nx - ix]) (ix > nx/2; free-hand y:
// conj(half[p][j][nx - ix]))
__global__ void k_half_to_full(Geo g, const cpx* __restrict__ half, cpx* __restrict__ full, long planes) {
    const long n = planes * g.nk;
    for (long idx = long(blockIdx.x) * blockDim.x + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
        const long pl = idx / g.nk, i = idx - pl * g.nk;
        const int ixx = int(i % g.nx), j = int(i / g.nx);
        const long hb = pl * g.nkh;
        const int jm = g.yf ? (g.ny - j) % g.ny : j;      // free-hand y: y is real space, only k_x mirrors
        full[idx] = ixx <= g.nx / 2 ? half[hb + long(j) * g.H + ixx]
                                    : conj(half[hb + long(jm) * g.H + (g.nx - ixx)]);
    }
}
__global__ void k_full_to_half(Geo g, const cpx* __restrict__ full, cpx* __restrict__ half, long planes) {
    const long n = planes * g.nkh;
    for (long idx = long(blockIdx.x) * blockDim.x + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
        const long pl = idx / g.nkh, i = idx - pl * g.nkh;
        const int kx = int(i % g.H), j = int(i / g.H);
        half[idx] = full[pl * g.nk + long(j) * g.nx + kx];
    }
}

// ---------------------------------------------------------------- elementwise
__global__ void k_axpy_c(cpx* __restrict__ y, const cpx* __restrict__ x, double a, long n) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) y[i] = y[i] + a * x[i];
}
__global__ void k_copy_c(cpx* __restrict__ y, const cpx* __restrict__ x, long n) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) y[i] = x[i];
}
static unsigned ew_blocks(long n) {
    long b = (n + 255) / 256;
    return unsigned(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}
void launch_half_to_full(Ctx& c, const cpx* half, cpx* full, long planes) {
    k_half_to_full<<<ew_blocks(planes * c.nk), 256, 0, c.stream>>>(c.geo(), half, full, planes);
    c.check_launch("k_half_to_full");
}
void launch_full_to_half(Ctx& c, const cpx* full, cpx* half, long planes) {
    k_full_to_half<<<ew_blocks(planes * c.nkh), 256, 0, c.stream>>>(c.geo(), full, half, planes);
    c.check_launch("k_full_to_half");
}
void launch_zero_c(Ctx& c, cpx* p, size_t n) { if (n) G3D_CUDA(cudaMemsetAsync(p, 0, n * sizeof(cpx), c.stream)); }
void launch_axpy_c(Ctx& c, cpx* y, const cpx* x, double a, size_t n) {
    if (!n) return;
    const int tok = c.prof_begin("axpy");
    k_axpy_c<<<ew_blocks(long(n)), 256, 0, c.stream>>>(y, x, a, long(n));
    c.check_launch("k_axpy_c");
    c.prof_end(tok);
}
void launch_copy_c(Ctx& c, cpx* y, const cpx* x, size_t n) {
    if (!n) return;
    const int tok = c.prof_begin("copy");
    k_copy_c<<<ew_blocks(long(n)), 256, 0, c.stream>>>(y, x, long(n));
    c.check_launch("k_copy_c");
    c.prof_end(tok);
}

// ---------------------------------------------------------------- window shift
// Spectra: exact phase factor exp(i (k_x s_x + k_y s_y)) with the shift tables kxs, kys (Nyquist kept).
__global__ void k_rotate(Geo g, cpx* __restrict__ p, long n, double sx, double sy, int nys) {
    const long nk = g.nkh;
    for (long idx = long(blockIdx.x) * blockDim.x + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
        const long i = idx % nk;
        const double ph = g.kxs[i % g.H] * sx + (nys ? g.kys[i / g.H] * sy : 0.0);
        p[idx] = p[idx] * C(cos(ph), sin(ph));
    }
}
// Real fields: index roll of every plane.
__global__ void k_roll(Geo g, const float* __restrict__ f, float* __restrict__ t, long n, int nxs, int nys) {
    const long nk = g.nk;
    for (long idx = long(blockIdx.x) * blockDim.x + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
        const long i = idx % nk, base = idx - i;
        const int ixx = int(i % g.nx), j = int(i / g.nx);
        const int sxx = ((ixx + nxs) % g.nx + g.nx) % g.nx, syy = ((j + nys) % g.ny + g.ny) % g.ny;
        t[idx] = f[base + long(syy) * g.nx + sxx];
    }
}
__global__ void k_shift_parts(PartsDev P, long np, double sx, double sy) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < np; i += long(gridDim.x) * blockDim.x) {
        P.x[i] -= sx; P.y[i] -= sy;
    }
}
void launch_rotate(Ctx& c, cpx* p, size_t n, double sx, double sy, int nys) {
    if (!n) return;
    k_rotate<<<ew_blocks(long(n)), 256, 0, c.stream>>>(c.geo(), p, long(n), sx, sy, nys);
    c.check_launch("k_rotate");
}
void launch_shift(Ctx& c, int nxs, int nys, double sx, double sy) {
    const Geo g = c.geo();
    if (c.np) {
        k_shift_parts<<<ew_blocks(c.np), 256, 0, c.stream>>>(c.parts, c.np, sx, sy);
        c.check_launch("k_shift_parts");
    }
    if (!c.P.self_fields) return;
    for (DevBuf<cpx>* a : {&c.Rx, &c.Ry, &c.Ez, &c.Bz, &c.j0x, &c.j0y}) {
        if (!a->n) continue;                     // the mixed form keeps E_z, B_z, j0 in complex64 (k_mixed.cu)
        k_rotate<<<ew_blocks(long(a->n)), 256, 0, c.stream>>>(g, a->p, long(a->n), sx, sy, nys);
        c.check_launch("k_rotate");
    }
    DevBuf<float> tmp;
    tmp.alloc(c.F.n, c.stream);
    k_roll<<<ew_blocks(long(c.F.n)), 256, 0, c.stream>>>(g, c.F.p, tmp.p, long(c.F.n), nxs, nys);
    c.check_launch("k_roll");
    std::swap(c.F.p, tmp.p);
    G3D_CUDA(cudaStreamSynchronize(c.stream));
}

}  // namespace g3d
