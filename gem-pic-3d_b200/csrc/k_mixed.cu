// The mixed FP32/FP64 form of the vacuum march (G3D_PREC_MIXED): the deposit, the zeta filter, the transverse
// FFTs, the sponge and the real fields in FP32 (complex64 half spectra, FP32 atomics), with E_z, B_z, L and the
// current spectra stored in complex64 and R_x, R_y in complex128. Each kernel restates the FP64 kernel of the
// same name (k_currents.cu, k_fields.cu, k_march.cu) with another element type; the march itself is the FP64
// kernel instantiated on complex64 storage (k_march.cu). Precision is kept where it decides the result:
//   * R_x, R_y stay complex128 across s-steps; the sponge is applied as an FP32 correction
//     dR = FFT((mask - 1) IFFT(R - R_b)) added to R in FP64 (R_b + FFT(mask IFFT(R - R_b)) = R + dR, and mask - 1
//     vanishes inside the box, so the FP32 error of dR is relative to the absorbed part, not to R); R - R_b is
//     formed in FP64 before it is rounded;
//   * the (1,2,1)/4 zeta filter sums with error-free transformations (two-sum), i.e. compensated FP32;
//   * the march recurrence and the bound field psi run in FP64 on widened inputs;
//   * the particles and their push are FP64 (the push reads the float F of both forms).
#include "g3d_ctx.hpp"
#include "k_fft.cuh"
#include "k_dispatch.cuh"

namespace g3d {

namespace {
constexpr int NT = 128;
constexpr int CW = 8;

// error-free sum of two floats (Knuth's two-sum); the _rn intrinsics are never fused into an FMA with the
// products that feed them, which would break the exactness of the error term
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = __fadd_rn(a, b);
    const float bb = __fsub_rn(s, a);
    e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
}
// a + b + c with the rounding errors of both additions added back
__device__ __forceinline__ float sum3c(float a, float b, float c) {
    float s1, e1, s2, e2;
    two_sum(a, b, s1, e1);
    two_sum(s1, c, s2, e2);
    return s2 + (e1 + e2);
}
}  // namespace

// ---------------------------------------------------------------- deposit (FP32 atomics)
// k_deposit (k_currents.cu) with FP32 values and FP32 atomics into FP32 raw planes: the cell location and the
// TSC fractions stay FP64 (zeta needs every digit; x / dx and y / dy near 128 would keep only 5 of them in FP32),
// the weights and the velocity ratios are rounded once.
__global__ void __launch_bounds__(256) k_deposit_f(PartsDev P, const int32_t* __restrict__ perm, long np, Geo g,
                                                  float* __restrict__ J) {
    const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const long ip = perm[t];
    if (P.alive[ip] != 1) return;
    int m; double fz;
    g.zax.locate(P.zeta[ip], m, fz);
    const int hw = m - (g.a - 2);
    if (hw < 0 || hw >= g.nh || m < 0 || m > g.N - 2) return;
    const double pz = P.pz[ip];
    const float vxz = float(P.px[ip] / pz), vyz = float(P.py[ip] / pz);      // v_x / v_z, v_y / v_z
    const float f = float(P.q[ip] * P.w[ip] / (g.hcg[m + 2] * g.dx) * g.iA[0]);
    int ix[3], jn[3]; double wx[3], wn[3];
    tsc_periodic(P.x[ip], g.dx, g.nx, ix, wx);
    tsc_periodic(P.y[ip], g.dy, g.ny, jn, wn);
    const long nk = g.nk, pl = long(g.nh) * nk;
    float* J0 = J + long(hw) * nk;
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int u = 0; u < 3; ++u) {
            const long k = long(jn[v]) * g.nx + ix[u];
            const float w = f * float(wx[u] * wn[v]);
            atomicAdd(J0 + k, w * vxz);
            atomicAdd(J0 + pl + k, w * vyz);
            atomicAdd(J0 + 2 * pl + k, w);
        }
}

// ---------------------------------------------------------------- zeta filter + FFT along x (FP32)
template <int NX>
__global__ void __launch_bounds__(NT) k_cur_rows_f(Geo g, const float* __restrict__ J, const cpxf* __restrict__ tw,
                                                  cpxf* __restrict__ TX, cpxf* __restrict__ TY, cpxf* __restrict__ TZ, int zf) {
    using S = FftShape<NX>;
    constexpr int LPC = NT / S::T, RS = row_stride<NX>(), H = NX / 2 + 1;
    extern __shared__ cpxf smf[];
    cpxf* a0 = smf;
    cpxf* a1 = smf + LPC * RS;
    const int tid = threadIdx.x, r0 = blockIdx.x * LPC, hk = blockIdx.y;
    const long nk = g.nk, cpl = long(g.nh) * nk, nkh = long(g.ny) * H;
    const int hw = hk + 1, hc = g.a - 1 + hk;
    const bool live = hc >= 0 && hc <= g.N - 2;
    float wm = 0.25f, w0 = 0.5f, wp = 0.25f, inv = 1.0f;
    if (zf && !g.zeta_uniform && live) {
        wm = float(0.25 * g.hcg[hc + 1]); w0 = float(0.5 * g.hcg[hc + 2]); wp = float(0.25 * g.hcg[hc + 3]); inv = float(g.hcg[hc + 2]);
    }
    #pragma unroll
    for (int u_ = 0; u_ < (LPC * NX + NT - 1) / NT; ++u_) {
        const int e = tid + u_ * NT;
        if (e >= LPC * NX) break;
        const int rr = e / NX, p = e - rr * NX, row = r0 + rr;
        float v[3] = {0, 0, 0};
        if (live && row < g.ny) {
            const long i = long(row) * NX + p;
#pragma unroll
            for (int comp = 0; comp < 3; ++comp) {
                const float* Jc = J + comp * cpl + i;
                const float jm = __ldg(Jc + (hw - 1) * nk), j0 = __ldg(Jc + hw * nk), jp = __ldg(Jc + (hw + 1) * nk);
                if (zf) v[comp] = sum3c(__fmul_rn(wm, jm), __fmul_rn(w0, j0), __fmul_rn(wp, jp)) / inv;
                else v[comp] = j0;
            }
        }
        a0[rr * RS + p + (p >> 3)] = Cf(v[0], v[1]);
        a1[rr * RS + p + (p >> 3)] = Cf(v[2], 0.0f);
    }
    __syncthreads();
    const int r = tid / S::T, t = tid - r * S::T;
    {
        decltype(a0) const ls_[2] = {a0, a1};
        fft_lines<NX, 2>(ls_, RowAddr{r * RS}, t, tw);
    }
    const long base = long(hk) * nkh;
    #pragma unroll
    for (int u_ = 0; u_ < (LPC * H + NT - 1) / NT; ++u_) {
        const int e = tid + u_ * NT;
        if (e >= LPC * H) break;
        const int rr = e / H, kx = e - rr * H, row = r0 + rr;
        if (row >= g.ny) continue;
        const int km = (NX - kx) % NX;
        const cpxf z = a0[rr * RS + kx + (kx >> 3)], zm = conj(a0[rr * RS + km + (km >> 3)]);
        const cpxf d = z - zm;
        const long o = base + long(row) * H + kx;
        TX[o] = 0.5f * (z + zm);
        TY[o] = 0.5f * Cf(d.y, -d.x);
        TZ[o] = a1[rr * RS + kx + (kx >> 3)];
    }
}

template <int NY>
__global__ void __launch_bounds__(CW * FftShape<NY>::T) k_cur_cols_f(Geo g, const cpxf* __restrict__ tw, const cpxf* __restrict__ TX,
                                                                     const cpxf* __restrict__ TY, const cpxf* __restrict__ TZ,
                                                                     cpxf* __restrict__ JX, cpxf* __restrict__ JY, cpxf* __restrict__ JZ,
                                                                     int keep0) {
    using S = FftShape<NY>;
    extern __shared__ cpxf smf[];
    cpxf* s0 = smf;
    cpxf* s1 = smf + ColTile<NY, CW>::size;
    cpxf* s2 = smf + 2 * ColTile<NY, CW>::size;
    const int hk = blockIdx.y, c0 = blockIdx.x * CW, tid = threadIdx.x, nthr = CW * S::T, H = g.H;
    const long base = long(hk) * g.nkh;
    #pragma unroll
    for (int u_ = 0; u_ < (NY * CW + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * CW) break;
        const int p = e / CW, c = e - p * CW, kx = c0 + c;
        cpxf u0 = Cf(0), u1 = Cf(0), u2 = Cf(0);
        if (kx < H) { const long o = base + long(p) * H + kx; u0 = TX[o]; u1 = TY[o]; u2 = TZ[o]; }
        s0[ColTile<NY, CW>::at(p, c)] = u0; s1[ColTile<NY, CW>::at(p, c)] = u1; s2[ColTile<NY, CW>::at(p, c)] = u2;
    }
    __syncthreads();
    const int c = tid % CW, t = tid / CW;
    {
        decltype(s0) const ls_[3] = {s0, s1, s2};
        fft_lines<NY, 3>(ls_, RowAddr{c * ColTile<NY, CW>::RS}, t, tw);
    }
    #pragma unroll
    for (int u_ = 0; u_ < (NY * CW + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * CW) break;
        const int p = e / CW, cc = e - p * CW, kx = c0 + cc;
        if (kx >= H) continue;
        const float f = (kx == 0 && p == 0 && !keep0) ? 0.0f : float(g.filt[kx] * g.filty[p]);
        const long o = base + long(p) * H + kx;
        JX[o] = f * s0[ColTile<NY, CW>::at(p, cc)]; JY[o] = f * s1[ColTile<NY, CW>::at(p, cc)]; JZ[o] = f * s2[ColTile<NY, CW>::at(p, cc)];
    }
}

// ---------------------------------------------------------------- co-moving start field (FP64 solve, mixed storage)
__global__ void __launch_bounds__(128) k_comoving_mixed(Geo g, const cpxf* __restrict__ jz, double* __restrict__ cpb,
                                                       cpx* __restrict__ dpb, cpx* __restrict__ Rx, cpx* __restrict__ Ry,
                                                       cpxf* __restrict__ Ez, cpxf* __restrict__ Bz, double beta, double gm2) {
    const long nk = g.nkh;
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nk) return;
    const int kxi = int(i % g.H), j = int(i / g.H);
    const double kx = g.kxd[kxi], ky = g.kyd[j], ev = ky * ky;
    double cprev = 0;
    cpx dprev = C(0);
    for (int l = 0; l < g.ns; ++l) {
        const long o = long(l) * nk + i;
        const int n = g.a + l;
        const double hm = g.hcg[n + 1], hp = g.hcg[n + 2];
        const double lo = -gm2 * 2 / ((hm + hp) * hm), up = -gm2 * 2 / ((hm + hp) * hp);
        const double dg = kx * kx + ev + gm2 * 2 / (hm * hp);
        if (dg == 0) { cpb[o] = 0; dpb[o] = C(0); continue; }
        const cpx rhs = (1 / beta) * (g.wlo[n] * to_d(jz[o]) + g.whi[n] * to_d(jz[o + nk]));
        if (n == 0) { cprev = 0; dprev = C(0); }
        const double den = dg - lo * cprev;
        const double cpv = up / den;
        const cpx dpv = (rhs - lo * dprev) / den;
        cpb[o] = cpv; dpb[o] = dpv;
        cprev = cpv; dprev = dpv;
    }
    cpx next = C(0);
    const double opb = 1 + beta;
    for (int l = g.ns - 1; l >= 0; --l) {
        const long o = long(l) * nk + i;
        next = dpb[o] - cpb[o] * next;
        Rx[o] = -opb * ik(kx, next);
        Ry[o] = -opb * ik(ky, next);
        Ez[o] = Cf(0); Bz[o] = Cf(0);
    }
}

// ---------------------------------------------------------------- sponge: the FP32 correction dR, added to R in FP64
template <int NY>
__global__ void __launch_bounds__(CW * FftShape<NY>::T) k_sp_cols_inv_f(Geo g, const cpxf* __restrict__ tw, const cpx* __restrict__ Rx,
                                                                        const cpx* __restrict__ Ry, const cpxf* __restrict__ jz,
                                                                        cpxf* __restrict__ U, cpxf* __restrict__ V, double g2, double opb) {
    using S = FftShape<NY>;
    extern __shared__ cpxf smf[];
    cpxf* s0 = smf;
    cpxf* s1 = smf + ColTile<NY, CW>::size;
    const int l = blockIdx.y, c0 = blockIdx.x * CW, tid = threadIdx.x, nthr = CW * S::T, H = g.H;
    const long nk = g.nkh, base = long(l) * nk;
    const int n = g.a + l;
    #pragma unroll
    for (int u_ = 0; u_ < (NY * CW + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * CW) break;
        const int p = e / CW, c = e - p * CW, kxi = c0 + c;
        cpxf u = Cf(0), v = Cf(0);
        if (kxi < H) {
            const long i = long(p) * H + kxi, o = base + i;
            const double kx = g.kxd[kxi], ky = g.kyd[p], k2 = kx * kx + ky * ky;
            // bound field psi of the slice charge (one rank: no ghost half-cells)
            auto half = [&](int hk) -> cpx { return (hk < 0 || hk > g.ns) ? C(0) : to_d(jz[long(hk) * nk + i]); };
            auto rho_at = [&](int dl) -> cpx {
                const int nn = n + dl;
                if (nn < 0 || nn > g.N - 1) return C(0);
                return g.wlo[nn] * half(l + dl) + g.whi[nn] * half(l + dl + 1);
            };
            const double hm = g.hcg[n + 1], hp = g.hcg[n + 2];
            const double cm = 2 / ((hm + hp) * hm), cp_ = 2 / ((hm + hp) * hp);
            cpx psi = C(0);
            if (k2 > 0) {
                const cpx d2 = g2 * (cp_ * rho_at(1) - (cm + cp_) * rho_at(0) + cm * rho_at(-1));
                psi = (rho_at(0) + d2 / k2) / k2;
            }
            u = to_f(Rx[o] + opb * ik(kx, psi));              // R - R_b, R_b = -(1 + beta) i k psi
            v = to_f(Ry[o] + opb * ik(ky, psi));
        }
        s0[ColTile<NY, CW>::at(p, c)] = conj(u); s1[ColTile<NY, CW>::at(p, c)] = conj(v);
    }
    __syncthreads();
    const int c = tid % CW, t = tid / CW;
    {
        decltype(s0) const ls_[2] = {s0, s1};
        fft_lines<NY, 2>(ls_, RowAddr{c * ColTile<NY, CW>::RS}, t, tw);
    }
    #pragma unroll
    for (int u_ = 0; u_ < (NY * CW + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * CW) break;
        const int p = e / CW, cc = e - p * CW, kxi = c0 + cc;
        if (kxi >= H) continue;
        const long o = base + long(p) * H + kxi;
        U[o] = conj(s0[ColTile<NY, CW>::at(p, cc)]); V[o] = conj(s1[ColTile<NY, CW>::at(p, cc)]);
    }
}
template <int NX>
__global__ void __launch_bounds__(NT) k_sp_rows_f(Geo g, const cpxf* __restrict__ tw, cpxf* __restrict__ U, cpxf* __restrict__ V) {
    using S = FftShape<NX>;
    constexpr int LPC = NT / S::T, RS = row_stride<NX>(), H = NX / 2 + 1;
    extern __shared__ cpxf smf[];
    const int l = blockIdx.y, r0 = blockIdx.x * LPC, tid = threadIdx.x;
    const long base = long(l) * g.nkh;
    #pragma unroll
    for (int u_ = 0; u_ < (LPC * H + NT - 1) / NT; ++u_) {
        const int e = tid + u_ * NT;
        if (e >= LPC * H) break;
        const int r = e / H, p = e - r * H, row = r0 + r;
        cpxf a = Cf(0), b = Cf(0);
        if (row < g.ny) { const long o = base + long(row) * H + p; a = U[o]; b = V[o]; }
        const cpxf z = Cf(a.x - b.y, a.y + b.x);
        smf[r * RS + p + (p >> 3)] = conj(z);
        if (p > 0 && p < NX / 2) {
            const int q = NX - p;
            smf[r * RS + q + (q >> 3)] = conj(Cf(a.x + b.y, -a.y + b.x));
        }
    }
    __syncthreads();
    const int r = tid / S::T, t = tid - r * S::T;
    fft_line<NX>(smf, RowAddr{r * RS}, t, tw);
    const float s = 1.0f / float(g.nk);
    #pragma unroll
    for (int u_ = 0; u_ < (LPC * NX + NT - 1) / NT; ++u_) {
        const int e = tid + u_ * NT;
        if (e >= LPC * NX) break;
        const int rr = e / NX, p = e - rr * NX, row = r0 + rr;
        const int q = rr * RS + p + (p >> 3);
        const cpxf z = s * conj(smf[q]);
        const float mx = float(g.maskx[p]);
        const float mn = row < g.ny ? float(g.masky_n[row]) : 1.0f, mh = row < g.ny ? float(g.masky_h[row]) : 1.0f;
        smf[q] = Cf((mx * mn - 1.0f) * z.x, (mx * mh - 1.0f) * z.y);      // (mask - 1): the correction only
    }
    __syncthreads();
    fft_line<NX>(smf, RowAddr{r * RS}, t, tw);
    #pragma unroll
    for (int u_ = 0; u_ < (LPC * H + NT - 1) / NT; ++u_) {
        const int e = tid + u_ * NT;
        if (e >= LPC * H) break;
        const int rr = e / H, p = e - rr * H, row = r0 + rr;
        if (row >= g.ny) continue;
        const int pm = (NX - p) % NX;
        const cpxf z = smf[rr * RS + p + (p >> 3)], zm = conj(smf[rr * RS + pm + (pm >> 3)]);
        const cpxf d = z - zm;
        const long o = base + long(row) * H + p;
        U[o] = 0.5f * (z + zm);
        V[o] = 0.5f * Cf(d.y, -d.x);
    }
}
template <int NY>
__global__ void __launch_bounds__(CW * FftShape<NY>::T) k_sp_cols_fwd_f(Geo g, const cpxf* __restrict__ tw, const cpxf* __restrict__ U,
                                                                        const cpxf* __restrict__ V, cpx* __restrict__ Rx,
                                                                        cpx* __restrict__ Ry) {
    using S = FftShape<NY>;
    extern __shared__ cpxf smf[];
    cpxf* s0 = smf;
    cpxf* s1 = smf + ColTile<NY, CW>::size;
    const int l = blockIdx.y, c0 = blockIdx.x * CW, tid = threadIdx.x, nthr = CW * S::T, H = g.H;
    const long base = long(l) * g.nkh;
    #pragma unroll
    for (int u_ = 0; u_ < (NY * CW + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * CW) break;
        const int p = e / CW, c = e - p * CW, kxi = c0 + c;
        cpxf u = Cf(0), v = Cf(0);
        if (kxi < H) { const long o = base + long(p) * H + kxi; u = U[o]; v = V[o]; }
        s0[ColTile<NY, CW>::at(p, c)] = u; s1[ColTile<NY, CW>::at(p, c)] = v;
    }
    __syncthreads();
    const int c = tid % CW, t = tid / CW;
    {
        decltype(s0) const ls_[2] = {s0, s1};
        fft_lines<NY, 2>(ls_, RowAddr{c * ColTile<NY, CW>::RS}, t, tw);
    }
    #pragma unroll
    for (int u_ = 0; u_ < (NY * CW + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * CW) break;
        const int p = e / CW, cc = e - p * CW, kxi = c0 + cc;
        if (kxi >= H) continue;
        const long o = base + long(p) * H + kxi;
        Rx[o] = Rx[o] + to_d(s0[ColTile<NY, CW>::at(p, cc)]);                   // R + dR in FP64
        Ry[o] = Ry[o] + to_d(s1[ColTile<NY, CW>::at(p, cc)]);
    }
}

// ---------------------------------------------------------------- real fields (FP32 transforms of the FP64 R)
template <int NY, int CWT>
__global__ void __launch_bounds__(CWT * FftShape<NY>::T) k_rf_cols_f(Geo g, const cpxf* __restrict__ tw, const cpx* __restrict__ Rx,
                                                                    const cpx* __restrict__ Ry, const cpxf* __restrict__ Lx,
                                                                    const cpxf* __restrict__ Ly, const cpxf* __restrict__ Ez,
                                                                    const cpxf* __restrict__ Bz, cpxf* __restrict__ W0,
                                                                    cpxf* __restrict__ W1, cpxf* __restrict__ W2,
                                                                    cpxf* __restrict__ W3, cpxf* __restrict__ W4, cpxf* __restrict__ W5,
                                                                    int l0) {
    using S = FftShape<NY>;
    extern __shared__ cpxf smf[];
    const int l = l0 + blockIdx.y, c0 = blockIdx.x * CWT, tid = threadIdx.x, nthr = CWT * S::T, pr = blockIdx.z, H = g.H;
    const long base = long(l) * g.nkh;
    cpxf* out0 = pr == 0 ? W0 : pr == 1 ? W2 : W4;
    cpxf* out1 = pr == 0 ? W1 : pr == 1 ? W3 : W5;
    cpxf* s0 = smf;
    cpxf* s1 = smf + ColTile<NY, CWT>::size;
    #pragma unroll
    for (int u_ = 0; u_ < (NY * CWT + nthr - 1) / nthr; ++u_) {      // unrolled: the loads of all elements in flight
        const int e = tid + u_ * nthr;
        if (e >= NY * CWT) continue;
        const int p = e / CWT, c = e - p * CWT, kxi = c0 + c;
        const long o = base + long(p) * H + kxi;
        cpxf a = Cf(0), b = Cf(0);
        if (kxi < H) {
            if (pr == 0) { a = to_f(Rx[o]); b = to_f(Ry[o]); }
            else if (pr == 1) { a = Lx[o]; b = Ly[o]; }
            else { a = Ez[o]; b = Bz[o]; }
        }
        s0[ColTile<NY, CWT>::at(p, c)] = conj(a); s1[ColTile<NY, CWT>::at(p, c)] = conj(b);
    }
    __syncthreads();
    const int c = tid % CWT, t = tid / CWT;
    {
        decltype(s0) const ls_[2] = {s0, s1};
        fft_lines<NY, 2>(ls_, RowAddr{c * ColTile<NY, CWT>::RS}, t, tw);
    }
    #pragma unroll 1
    for (int u_ = 0; u_ < (NY * CWT + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * CWT) break;
        const int p = e / CWT, cc = e - p * CWT, kxi = c0 + cc;
        if (kxi >= H) continue;
        const long o = base + long(p) * H + kxi;
        out0[o] = conj(s0[ColTile<NY, CWT>::at(p, cc)]); out1[o] = conj(s1[ColTile<NY, CWT>::at(p, cc)]);
    }
}
template <int NX>
__global__ void __launch_bounds__(NT) k_rf_rows_f(Geo g, const cpxf* __restrict__ tw, const cpxf* __restrict__ W0,
                                                 const cpxf* __restrict__ W1, const cpxf* __restrict__ W2,
                                                 const cpxf* __restrict__ W3, const cpxf* __restrict__ W4,
                                                 const cpxf* __restrict__ W5, float* __restrict__ F, int l0, FmidOut fm) {
    using S = FftShape<NX>;
    constexpr int LPC = NT / S::T, RS = row_stride<NX>(), H = NX / 2 + 1;
    extern __shared__ cpxf smf[];
    cpxf* a[3] = {smf, smf + LPC * RS, smf + 2 * LPC * RS};
    const int l = l0 + blockIdx.y, r0 = blockIdx.x * LPC, tid = threadIdx.x;
    const long base = long(l) * g.nkh;
    const cpxf* in[6] = {W0, W1, W2, W3, W4, W5};
    const long fpl = long(g.ns + 2) * g.nk, fbase = long(l) * g.nk;
    constexpr int EO = (LPC * NX + NT - 1) / NT;                    // output elements of a thread
    float oth[EO][6];                                               // the midpoint fields' other slice
    if (fm.out) {
    #pragma unroll
        for (int u_ = 0; u_ < EO; ++u_) {
            const int e = tid + u_ * NT, rr = e / NX, p = e - rr * NX, row = r0 + rr;
            if (e < LPC * NX && row < g.ny) fmid_load(fm, F, fpl, g.nk, long(row) * NX + p, oth[u_]);
        }
    }
    #pragma unroll
    for (int u_ = 0; u_ < (LPC * H + NT - 1) / NT; ++u_) {
        const int e = tid + u_ * NT;
        if (e >= LPC * H) break;
        const int r = e / H, p = e - r * H, row = r0 + r;
        for (int f = 0; f < 3; ++f) {
            cpxf x = Cf(0), y = Cf(0);
            if (row < g.ny) { const long o = base + long(row) * H + p; x = in[2 * f][o]; y = in[2 * f + 1][o]; }
            a[f][r * RS + p + (p >> 3)] = conj(Cf(x.x - y.y, x.y + y.x));
            if (p > 0 && p < NX / 2) { const int q = NX - p; a[f][r * RS + q + (q >> 3)] = conj(Cf(x.x + y.y, -x.y + y.x)); }
        }
    }
    __syncthreads();
    const int r = tid / S::T, t = tid - r * S::T;
    fft_lines<NX, 3>(a, RowAddr{r * RS}, t, tw);
    const float s = 1.0f / float(g.nk);
    #pragma unroll
    for (int u_ = 0; u_ < EO; ++u_) {
        const int e = tid + u_ * NT;
        if (e >= LPC * NX) continue;
        const int rr = e / NX, p = e - rr * NX, row = r0 + rr;
        if (row >= g.ny) continue;
        const int q = rr * RS + p + (p >> 3);
        const cpxf z1 = s * conj(a[0][q]), z2 = s * conj(a[1][q]), z3 = s * conj(a[2][q]);
        const long idx = fbase + long(row) * NX + p;
        const float fv[6] = {0.5f * (z1.x + z2.x), 0.5f * (z1.y + z2.y), z3.x,      // E_x, E_y, E_z
                             0.5f * (z2.y - z1.y), 0.5f * (z1.x - z2.x), z3.y};     // B_x, B_y, B_z
#pragma unroll
        for (int comp = 0; comp < 6; ++comp) F[comp * fpl + idx] = fv[comp];
        if (fm.out) fmid_store(fm, long(row) * NX + p, fv, oth[u_]);
        if (fm.rec_f) {                                // the adjoint's record of the slice (widened)
            double* R = *fm.rec_f + fm.rec_off + long(row) * NX + p;
#pragma unroll
            for (int comp = 0; comp < 6; ++comp) R[comp * g.nk] = double(fv[comp]);
        }
    }
}

// ---------------------------------------------------------------- elementwise on complex64 arrays
__global__ void k_half_to_full_f(Geo g, const cpxf* __restrict__ half, cpx* __restrict__ full, long planes) {
    const long n = planes * g.nk;
    for (long idx = long(blockIdx.x) * blockDim.x + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
        const long pl = idx / g.nk, i = idx - pl * g.nk;
        const int ixx = int(i % g.nx), j = int(i / g.nx);
        const long hb = pl * g.nkh;
        full[idx] = ixx <= g.nx / 2 ? to_d(half[hb + long(j) * g.H + ixx])
                                    : conj(to_d(half[hb + long((g.ny - j) % g.ny) * g.H + (g.nx - ixx)]));
    }
}
__global__ void k_full_to_half_f(Geo g, const cpx* __restrict__ full, cpxf* __restrict__ half, long planes) {
    const long n = planes * g.nkh;
    for (long idx = long(blockIdx.x) * blockDim.x + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
        const long pl = idx / g.nkh, i = idx - pl * g.nkh;
        const int kx = int(i % g.H), j = int(i / g.H);
        half[idx] = to_f(full[pl * g.nk + long(j) * g.nx + kx]);
    }
}
__global__ void k_rotate_f(Geo g, cpxf* __restrict__ p, long n, double sx, double sy, int nys) {
    const long nk = g.nkh;
    for (long idx = long(blockIdx.x) * blockDim.x + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
        const long i = idx % nk;
        const double ph = g.kxs[i % g.H] * sx + (nys ? g.kys[i / g.H] * sy : 0.0);
        p[idx] = to_f(to_d(p[idx]) * C(cos(ph), sin(ph)));
    }
}
__global__ void k_axpy_fc(cpxf* __restrict__ y, const cpx* __restrict__ x, double a, long n) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x)
        y[i] = to_f(to_d(y[i]) + a * x[i]);
}
__global__ void k_copy_f(cpxf* __restrict__ y, const cpxf* __restrict__ x, long n) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) y[i] = x[i];
}

// ---------------------------------------------------------------- launchers
static unsigned ew_blocks(long n) {
    long b = (n + 255) / 256;
    return unsigned(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}
template <class K>
static void allow_smem(K kern, size_t smem) {
    smem_attr(reinterpret_cast<const void*>(kern), smem);
}

void launch_deposit_f(Ctx& c) {
    c.mx.jw.zero(c.stream);
    if (c.np == 0) return;
    const int tok = c.prof_begin("deposit");
    k_deposit_f<<<unsigned((c.np + 255) / 256), 256, 0, c.stream>>>(c.parts, c.perm.p, c.np, c.geo(), c.mx.jw.p);
    c.check_launch("k_deposit_f");
    c.prof_end(tok);
}
template <int NX>
static void cur_rows_f(Ctx& c) {
    constexpr int LPC = NT / FftShape<NX>::T;
    const size_t smem = size_t(2) * LPC * row_stride<NX>() * sizeof(cpxf);
    allow_smem(k_cur_rows_f<NX>, smem);
    const int tok = c.prof_begin("cur_rows");
    k_cur_rows_f<NX><<<dim3(unsigned((c.ny + LPC - 1) / LPC), unsigned(c.ns + 1)), NT, smem, c.stream>>>(
        c.geo(), c.mx.jw.p, c.mx.twx.p, c.mx.W[0].p, c.mx.W[1].p, c.mx.W[2].p, c.P.zeta_filter ? 1 : 0);
    c.check_launch("k_cur_rows_f");
    c.prof_end(tok);
}
template <int NY>
static void cur_cols_f(Ctx& c, bool keep0) {
    const size_t smem = size_t(3) * ColTile<NY, CW>::size * sizeof(cpxf);
    allow_smem(k_cur_cols_f<NY>, smem);
    const int tok = c.prof_begin("cur_cols");
    k_cur_cols_f<NY><<<dim3(unsigned((c.H + CW - 1) / CW), unsigned(c.ns + 1)), CW * FftShape<NY>::T, smem, c.stream>>>(
        c.geo(), c.mx.twy.p, c.mx.W[0].p, c.mx.W[1].p, c.mx.W[2].p, c.mx.jkx.p, c.mx.jky.p, c.mx.jkz.p, keep0 ? 1 : 0);
    c.check_launch("k_cur_cols_f");
    c.prof_end(tok);
}
void launch_cur_fft_f(Ctx& c, bool keep0) {
    G3D_DISPATCH_N(c.nx, NX, cur_rows_f<NX>(c));
    G3D_DISPATCH_N(c.ny, NY, cur_cols_f<NY>(c, keep0));
}
void launch_comoving_f(Ctx& c, double beta, double gm2) {
    DevBuf<cpx> dp;
    dp.alloc(size_t(c.ns) * c.nkh, c.stream);
    k_comoving_mixed<<<unsigned((c.nkh + 127) / 128), 128, 0, c.stream>>>(c.geo(), c.mx.jkz.p, c.rscratch.p, dp.p, c.Rx.p, c.Ry.p,
                                                                          c.mx.Ez.p, c.mx.Bz.p, beta, gm2);
    c.check_launch("k_comoving_mixed");
    G3D_CUDA(cudaStreamSynchronize(c.stream));
}
template <int NY>
static void sp_cols_inv_f(Ctx& c) {
    const size_t smem = size_t(2) * ColTile<NY, CW>::size * sizeof(cpxf);
    allow_smem(k_sp_cols_inv_f<NY>, smem);
    const int tok = c.prof_begin("sponge_cols_inv");
    k_sp_cols_inv_f<NY><<<dim3(unsigned((c.H + CW - 1) / CW), unsigned(c.ns)), CW * FftShape<NY>::T, smem, c.stream>>>(
        c.geo(), c.mx.twy.p, c.Rx.p, c.Ry.p, c.mx.jkz.p, c.mx.W[0].p, c.mx.W[1].p, c.gm2_b, 1 + c.beta_b);
    c.check_launch("k_sp_cols_inv_f");
    c.prof_end(tok);
}
template <int NX>
static void sp_rows_f(Ctx& c) {
    constexpr int LPC = NT / FftShape<NX>::T;
    const size_t smem = size_t(LPC) * row_stride<NX>() * sizeof(cpxf);
    allow_smem(k_sp_rows_f<NX>, smem);
    const int tok = c.prof_begin("sponge_rows");
    k_sp_rows_f<NX><<<dim3(unsigned((c.ny + LPC - 1) / LPC), unsigned(c.ns)), NT, smem, c.stream>>>(c.geo(), c.mx.twx.p,
                                                                                                      c.mx.W[0].p, c.mx.W[1].p);
    c.check_launch("k_sp_rows_f");
    c.prof_end(tok);
}
template <int NY>
static void sp_cols_fwd_f(Ctx& c) {
    const size_t smem = size_t(2) * ColTile<NY, CW>::size * sizeof(cpxf);
    allow_smem(k_sp_cols_fwd_f<NY>, smem);
    const int tok = c.prof_begin("sponge_cols_fwd");
    k_sp_cols_fwd_f<NY><<<dim3(unsigned((c.H + CW - 1) / CW), unsigned(c.ns)), CW * FftShape<NY>::T, smem, c.stream>>>(
        c.geo(), c.mx.twy.p, c.mx.W[0].p, c.mx.W[1].p, c.Rx.p, c.Ry.p);
    c.check_launch("k_sp_cols_fwd_f");
    c.prof_end(tok);
}
void launch_sponge_f(Ctx& c) {
    G3D_DISPATCH_N(c.ny, NY, sp_cols_inv_f<NY>(c));
    G3D_DISPATCH_N(c.nx, NX, sp_rows_f<NX>(c));
    G3D_DISPATCH_N(c.ny, NY, sp_cols_fwd_f<NY>(c));
}
template <int NY, int CWT>
static void rf_cols_fw(Ctx& c, int l0, int nl) {
    const size_t smem = size_t(2) * ColTile<NY, CWT>::size * sizeof(cpxf);
    allow_smem(k_rf_cols_f<NY, CWT>, smem);
    const int tok = c.prof_begin(nl == 1 ? "real_cols_slice" : "real_cols");
    auto& m = c.mx;
    k_rf_cols_f<NY, CWT><<<dim3(unsigned((c.H + CWT - 1) / CWT), unsigned(nl), 3), CWT * FftShape<NY>::T, smem, c.stream>>>(
        c.geo(), m.twy.p, c.Rx.p, c.Ry.p, m.Lx.p, m.Ly.p, m.Ez.p, m.Bz.p, m.W[0].p, m.W[1].p, m.W[2].p, m.W[3].p, m.W[4].p, m.W[5].p,
        l0);
    c.check_launch("k_rf_cols_f");
    c.prof_end(tok);
}
// one slice (the plasma march): tiles of 2 columns, so that 3 x 65 CTAs spread the slice's latency over the SMs
template <int NY>
static void rf_cols_f(Ctx& c, int l0, int nl) {
    if (nl == 1) rf_cols_fw<NY, 2>(c, l0, nl);
    else rf_cols_fw<NY, CW>(c, l0, nl);
}
template <int NX>
static void rf_rows_f(Ctx& c, int l0, int nl, FmidOut fm = FmidOut()) {
    constexpr int LPC = NT / FftShape<NX>::T;
    const size_t smem = size_t(3) * LPC * row_stride<NX>() * sizeof(cpxf);
    allow_smem(k_rf_rows_f<NX>, smem);
    const int tok = c.prof_begin(nl == 1 ? "real_rows_slice" : "real_rows");
    auto& m = c.mx;
    k_rf_rows_f<NX><<<dim3(unsigned((c.ny + LPC - 1) / LPC), unsigned(nl)), NT, smem, c.stream>>>(
        c.geo(), m.twx.p, m.W[0].p, m.W[1].p, m.W[2].p, m.W[3].p, m.W[4].p, m.W[5].p, c.F.p, l0, fm);
    c.check_launch("k_rf_rows_f");
    c.prof_end(tok);
}
void launch_real_fields_f(Ctx& c) {
    G3D_DISPATCH_N(c.ny, NY, rf_cols_f<NY>(c, 0, c.ns));
    G3D_DISPATCH_N(c.nx, NX, rf_rows_f<NX>(c, 0, c.ns));
}
// E and B of one slice (plane l) of the mixed form (the real fields of one slice of the plasma march)
void launch_real_fields_slice_f(Ctx& c, int l, FmidOut fm, bool cols) {
    if (cols) G3D_DISPATCH_N(c.ny, NY, rf_cols_f<NY>(c, l, 1));
    G3D_DISPATCH_N(c.nx, NX, rf_rows_f<NX>(c, l, 1, fm));
}
void launch_half_to_full_f(Ctx& c, const cpxf* half, cpx* full, long planes) {
    k_half_to_full_f<<<ew_blocks(planes * c.nk), 256, 0, c.stream>>>(c.geo(), half, full, planes);
    c.check_launch("k_half_to_full_f");
}
void launch_full_to_half_f(Ctx& c, const cpx* full, cpxf* half, long planes) {
    k_full_to_half_f<<<ew_blocks(planes * c.nkh), 256, 0, c.stream>>>(c.geo(), full, half, planes);
    c.check_launch("k_full_to_half_f");
}
void launch_rotate_f(Ctx& c, cpxf* p, size_t n, double sx, double sy, int nys) {
    if (!n) return;
    k_rotate_f<<<ew_blocks(long(n)), 256, 0, c.stream>>>(c.geo(), p, long(n), sx, sy, nys);
    c.check_launch("k_rotate_f");
}
void launch_axpy_fc(Ctx& c, cpxf* y, const cpx* x, double a, size_t n) {
    if (!n) return;
    k_axpy_fc<<<ew_blocks(long(n)), 256, 0, c.stream>>>(y, x, a, long(n));
    c.check_launch("k_axpy_fc");
}
void launch_copy_f(Ctx& c, cpxf* y, const cpxf* x, size_t n) {
    if (!n) return;
    k_copy_f<<<ew_blocks(long(n)), 256, 0, c.stream>>>(y, x, long(n));
    c.check_launch("k_copy_f");
}

}  // namespace g3d
