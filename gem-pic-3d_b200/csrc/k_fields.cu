// Sponge and real-space fields (Simulation::sponge_and_real_fields, src/sim_fields.cpp:156-307, Fourier y),
// the window shift (src/sim_setup.cpp:249-281) and small elementwise kernels.
//
// Sponge: the radiation part R - R_b of the forward field (R_b = (1 + beta) E_perp of the slice charge,
// psi = (rho + gamma^-2 d_zeta^2 rho / k^2) / k^2) is multiplied in real space by the separable mask
// maskx(x) masky(y). Three kernels: k_sp_rows (bound field psi -> S2, pack R - R_b, inverse FFT along x),
// k_sp_cols (inverse FFT along y, 1/(nx ny), mask, forward FFT along y), k_sp_rowpairs (forward FFT along
// x, Hermitian split, + R_b).
// Real fields: k_rf_cols packs R_x + i R_y, L_x + i L_y, E_z + i B_z and transforms them along y; k_rf_rows
// transforms along x, normalises and writes the six float components of F.
#include "g3d_ctx.hpp"
#include "k_fft.cuh"
#include "k_dispatch.cuh"

namespace g3d {

namespace {
constexpr int NT = 128;    // threads of the row kernels
constexpr int CW = 8;      // columns per tile of the column kernels

// psi of the slice charge of slice n = a + l at the mode i (reference: the Fourier-y lambda of
// sim_fields.cpp:176-201)
__device__ __forceinline__ cpx bound_psi(const Geo& g, const cpx* __restrict__ jz, const cpx* __restrict__ jg, int l, long i,
                                         double kx, double ky, double g2) {
    const long nk = g.nk;
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
}  // namespace

// ---------------------------------------------------------------- sponge, pass 1: rows (inverse x)
template <int NX>
__global__ void __launch_bounds__(NT) k_sp_rows(Geo g, const cpx* __restrict__ Rx, const cpx* __restrict__ Ry,
                                               const cpx* __restrict__ jz, const cpx* __restrict__ jg, cpx* __restrict__ S1,
                                               cpx* __restrict__ S2, double g2, double opb) {
    using S = FftShape<NX>;
    constexpr int LPC = NT / S::T, RS = row_stride<NX>();
    extern __shared__ cpx sm[];
    const int l = blockIdx.y, r0 = blockIdx.x * LPC, tid = threadIdx.x;
    const long nk = g.nk, base = long(l) * nk;
    for (int e = tid; e < LPC * NX; e += NT) {
        const int r = e / NX, p = e - r * NX, row = r0 + r;
        cpx v = C(0);
        if (row < g.ny) {
            const long i = long(row) * NX + p, idx = base + i;
            const double kx = g.kxd[p], ky = g.kyd[row];
            const cpx psi = bound_psi(g, jz, jg, l, i, kx, ky, g2);
            S2[idx] = psi;
            const cpx bx = -opb * ik(kx, psi), by = -opb * ik(ky, psi);
            const cpx u = Rx[idx] - bx, w = Ry[idx] - by;
            v = conj(C(u.x - w.y, u.y + w.x));                       // u + i w, conjugated: inverse transform
        }
        sm[r * RS + p + (p >> 3)] = v;
    }
    __syncthreads();
    const int r = tid / S::T, t = tid - r * S::T;
    fft_line<NX>(sm, RowAddr{r * RS}, t, g.twx);
    for (int e = tid; e < LPC * NX; e += NT) {
        const int rr = e / NX, p = e - rr * NX, row = r0 + rr;
        if (row < g.ny) S1[base + long(row) * NX + p] = conj(sm[rr * RS + p + (p >> 3)]);
    }
}

// ---------------------------------------------------------------- sponge, pass 2: columns (inverse y, mask, forward y)
template <int NY>
__global__ void __launch_bounds__(CW * FftShape<NY>::T) k_sp_cols(Geo g, cpx* __restrict__ S1) {
    using S = FftShape<NY>;
    extern __shared__ cpx sm[];
    const int l = blockIdx.y, c0 = blockIdx.x * CW, tid = threadIdx.x, nthr = CW * S::T;
    const long nk = g.nk, base = long(l) * nk;
    const int nx = g.nx;
    for (int e = tid; e < NY * CW; e += nthr) {
        const int p = e / CW, c = e - p * CW;
        sm[e] = conj(S1[base + long(p) * nx + c0 + c]);
    }
    __syncthreads();
    const int c = tid % CW, t = tid / CW;
    fft_line<NY>(sm, ColAddr<CW>{c}, t, g.twy);
    const double s = 1.0 / double(g.nk);
    for (int e = tid; e < NY * CW; e += nthr) {
        const int p = e / CW, cc = e - p * CW, ixx = c0 + cc;
        const cpx z = s * conj(sm[e]);                                 // real-space value (x and y inverse done)
        const double mx = g.maskx[ixx];
        sm[e] = C(mx * g.masky_n[p] * z.x, mx * g.masky_h[p] * z.y);
    }
    __syncthreads();
    fft_line<NY>(sm, ColAddr<CW>{c}, t, g.twy);
    for (int e = tid; e < NY * CW; e += nthr) {
        const int p = e / CW, cc = e - p * CW;
        S1[base + long(p) * nx + c0 + cc] = sm[e];
    }
}

// ---------------------------------------------------------------- sponge, pass 3: row pairs (forward x, split, + R_b)
template <int NX>
__global__ void __launch_bounds__(NT) k_sp_rowpairs(Geo g, const cpx* __restrict__ S1, const cpx* __restrict__ S2,
                                                   cpx* __restrict__ Rx, cpx* __restrict__ Ry, double opb) {
    using S = FftShape<NX>;
    constexpr int LPC = NT / S::T, PPC = LPC / 2, RS = row_stride<NX>();
    extern __shared__ cpx sm[];
    const int l = blockIdx.y, tid = threadIdx.x, ny = g.ny;
    const long nk = g.nk, base = long(l) * nk;
    auto row_of = [&](int slot, bool& valid) {
        const int jp = blockIdx.x * PPC + (slot >> 1);
        valid = jp <= ny / 2;
        return (slot & 1) ? (ny - jp) % ny : jp;
    };
    for (int e = tid; e < LPC * NX; e += NT) {
        const int r = e / NX, p = e - r * NX;
        bool valid;
        const int row = row_of(r, valid);
        sm[r * RS + p + (p >> 3)] = valid ? S1[base + long(row) * NX + p] : C(0);
    }
    __syncthreads();
    const int r = tid / S::T, t = tid - r * S::T;
    fft_line<NX>(sm, RowAddr{r * RS}, t, g.twx);
    for (int e = tid; e < LPC * NX; e += NT) {
        const int rr = e / NX, p = e - rr * NX;
        bool valid, v2;
        const int row = row_of(rr, valid);
        if (!valid) continue;
        if ((rr & 1) && row == row_of(rr ^ 1, v2)) continue;
        const int pm = (NX - p) % NX;
        const cpx z = sm[rr * RS + p + (p >> 3)], zm = conj(sm[(rr ^ 1) * RS + pm + (pm >> 3)]);
        const cpx d = z - zm;
        const long idx = base + long(row) * NX + p;
        const cpx psi = S2[idx];
        Rx[idx] = 0.5 * (z + zm) - opb * ik(g.kxd[p], psi);
        Ry[idx] = 0.5 * C(d.y, -d.x) - opb * ik(g.kyd[row], psi);
    }
}

// ---------------------------------------------------------------- real fields: columns (pack, inverse y)
template <int NY>
__global__ void __launch_bounds__(CW * FftShape<NY>::T) k_rf_cols(Geo g, const cpx* __restrict__ Rx, const cpx* __restrict__ Ry,
                                                                  const cpx* __restrict__ Lx, const cpx* __restrict__ Ly,
                                                                  const cpx* __restrict__ Ez, const cpx* __restrict__ Bz,
                                                                  cpx* __restrict__ S1, cpx* __restrict__ S2, cpx* __restrict__ S3) {
    using S = FftShape<NY>;
    extern __shared__ cpx sm[];
    cpx* a0 = sm;
    cpx* a1 = sm + NY * CW;
    cpx* a2 = sm + 2 * NY * CW;
    const int l = blockIdx.y, c0 = blockIdx.x * CW, tid = threadIdx.x, nthr = CW * S::T;
    const long nk = g.nk, base = long(l) * nk;
    const int nx = g.nx;
    for (int e = tid; e < NY * CW; e += nthr) {
        const int p = e / CW, c = e - p * CW;
        const long idx = base + long(p) * nx + c0 + c;
        const cpx rx = Rx[idx], ry = Ry[idx], lx = Lx[idx], ly = Ly[idx], ez = Ez[idx], bz = Bz[idx];
        a0[e] = conj(C(rx.x - ry.y, rx.y + ry.x));
        a1[e] = conj(C(lx.x - ly.y, lx.y + ly.x));
        a2[e] = conj(C(ez.x - bz.y, ez.y + bz.x));
    }
    __syncthreads();
    const int c = tid % CW, t = tid / CW;
    fft_line<NY>(a0, ColAddr<CW>{c}, t, g.twy);
    fft_line<NY>(a1, ColAddr<CW>{c}, t, g.twy);
    fft_line<NY>(a2, ColAddr<CW>{c}, t, g.twy);
    for (int e = tid; e < NY * CW; e += nthr) {
        const int p = e / CW, cc = e - p * CW;
        const long idx = base + long(p) * nx + c0 + cc;
        S1[idx] = a0[e]; S2[idx] = a1[e]; S3[idx] = a2[e];          // still conjugated
    }
}

// ---------------------------------------------------------------- real fields: rows (inverse x, F)
template <int NX>
__global__ void __launch_bounds__(NT) k_rf_rows(Geo g, const cpx* __restrict__ S1, const cpx* __restrict__ S2,
                                               const cpx* __restrict__ S3, float* __restrict__ F) {
    using S = FftShape<NX>;
    constexpr int LPC = NT / S::T, RS = row_stride<NX>();
    extern __shared__ cpx sm[];
    cpx* a0 = sm;
    cpx* a1 = sm + LPC * RS;
    cpx* a2 = sm + 2 * LPC * RS;
    const int l = blockIdx.y, r0 = blockIdx.x * LPC, tid = threadIdx.x;
    const long nk = g.nk, base = long(l) * nk;
    for (int e = tid; e < LPC * NX; e += NT) {
        const int r = e / NX, p = e - r * NX, row = r0 + r;
        cpx u0 = C(0), u1 = C(0), u2 = C(0);
        if (row < g.ny) { const long idx = base + long(row) * NX + p; u0 = S1[idx]; u1 = S2[idx]; u2 = S3[idx]; }
        const int q = r * RS + p + (p >> 3);
        a0[q] = u0; a1[q] = u1; a2[q] = u2;
    }
    __syncthreads();
    const int r = tid / S::T, t = tid - r * S::T;
    fft_line<NX>(a0, RowAddr{r * RS}, t, g.twx);
    fft_line<NX>(a1, RowAddr{r * RS}, t, g.twx);
    fft_line<NX>(a2, RowAddr{r * RS}, t, g.twx);
    const double s = 1.0 / double(nk);
    const long fpl = long(g.ns + 2) * nk;
    for (int e = tid; e < LPC * NX; e += NT) {
        const int rr = e / NX, p = e - rr * NX, row = r0 + rr;
        if (row >= g.ny) continue;
        const int q = rr * RS + p + (p >> 3);
        const cpx z1 = s * conj(a0[q]), z2 = s * conj(a1[q]), z3 = s * conj(a2[q]);
        const long idx = base + long(row) * NX + p;
        const double r1 = z1.x, r2 = z1.y, l1 = z2.x, l2 = z2.y;
        F[0 * fpl + idx] = float(0.5 * (r1 + l1));     // E_x
        F[1 * fpl + idx] = float(0.5 * (r2 + l2));     // E_y
        F[3 * fpl + idx] = float(0.5 * (l2 - r2));     // B_x
        F[4 * fpl + idx] = float(0.5 * (r1 - l1));     // B_y
        F[2 * fpl + idx] = float(z3.x);                // E_z
        F[5 * fpl + idx] = float(z3.y);                // B_z
    }
}

// ---------------------------------------------------------------- launchers
template <int NX>
static void sp_rows(Ctx& c) {
    using S = FftShape<NX>;
    constexpr int LPC = NT / S::T;
    const size_t smem = size_t(LPC) * row_stride<NX>() * sizeof(cpx);
    auto kern = k_sp_rows<NX>;
    G3D_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    const int tok = c.prof_begin("sponge_rows");
    kern<<<dim3(unsigned((c.ny + LPC - 1) / LPC), unsigned(c.ns)), NT, smem, c.stream>>>(
        c.geo(), c.Rx.p, c.Ry.p, c.jkz.p, c.jzg.p, c.S1.p, c.S2.p, c.gm2_b, 1 + c.beta_b);
    c.check_launch("k_sp_rows");
    c.prof_end(tok);
}
template <int NY>
static void sp_cols(Ctx& c) {
    const size_t smem = size_t(NY) * CW * sizeof(cpx);
    auto kern = k_sp_cols<NY>;
    G3D_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    const int tok = c.prof_begin("sponge_cols");
    kern<<<dim3(unsigned(c.nx / CW), unsigned(c.ns)), CW * FftShape<NY>::T, smem, c.stream>>>(c.geo(), c.S1.p);
    c.check_launch("k_sp_cols");
    c.prof_end(tok);
}
template <int NX>
static void sp_rowpairs(Ctx& c) {
    using S = FftShape<NX>;
    constexpr int LPC = NT / S::T, PPC = LPC / 2;
    const size_t smem = size_t(LPC) * row_stride<NX>() * sizeof(cpx);
    auto kern = k_sp_rowpairs<NX>;
    G3D_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    const int tok = c.prof_begin("sponge_rowpairs");
    kern<<<dim3(unsigned((c.ny / 2 + 1 + PPC - 1) / PPC), unsigned(c.ns)), NT, smem, c.stream>>>(
        c.geo(), c.S1.p, c.S2.p, c.Rx.p, c.Ry.p, 1 + c.beta_b);
    c.check_launch("k_sp_rowpairs");
    c.prof_end(tok);
}
void launch_sponge(Ctx& c) {
    if (c.nx < CW) throw Error(G3D_ERR_ARG, "nx must be >= 8");
    G3D_DISPATCH_N(c.nx, NX, sp_rows<NX>(c));
    G3D_DISPATCH_N(c.ny, NY, sp_cols<NY>(c));
    G3D_DISPATCH_N(c.nx, NX, sp_rowpairs<NX>(c));
}

template <int NY>
static void rf_cols(Ctx& c) {
    const size_t smem = size_t(3) * NY * CW * sizeof(cpx);
    auto kern = k_rf_cols<NY>;
    G3D_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    const int tok = c.prof_begin("real_cols");
    kern<<<dim3(unsigned(c.nx / CW), unsigned(c.ns)), CW * FftShape<NY>::T, smem, c.stream>>>(
        c.geo(), c.Rx.p, c.Ry.p, c.Lx.p, c.Ly.p, c.Ez.p, c.Bz.p, c.S1.p, c.S2.p, c.S3.p);
    c.check_launch("k_rf_cols");
    c.prof_end(tok);
}
template <int NX>
static void rf_rows(Ctx& c) {
    using S = FftShape<NX>;
    constexpr int LPC = NT / S::T;
    const size_t smem = size_t(3) * LPC * row_stride<NX>() * sizeof(cpx);
    auto kern = k_rf_rows<NX>;
    G3D_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    const int tok = c.prof_begin("real_rows");
    kern<<<dim3(unsigned((c.ny + LPC - 1) / LPC), unsigned(c.ns)), NT, smem, c.stream>>>(c.geo(), c.S1.p, c.S2.p, c.S3.p, c.F.p);
    c.check_launch("k_rf_rows");
    c.prof_end(tok);
}
void launch_real_fields(Ctx& c) {
    if (c.nx < CW) throw Error(G3D_ERR_ARG, "nx must be >= 8");
    G3D_DISPATCH_N(c.ny, NY, rf_cols<NY>(c));
    G3D_DISPATCH_N(c.nx, NX, rf_rows<NX>(c));
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
    const long nk = g.nk;
    for (long idx = long(blockIdx.x) * blockDim.x + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
        const long i = idx % nk;
        const double ph = g.kxs[i % g.nx] * sx + (nys ? g.kys[i / g.nx] * sy : 0.0);
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
void launch_shift(Ctx& c, int nxs, int nys, double sx, double sy) {
    const Geo g = c.geo();
    if (c.np) {
        k_shift_parts<<<ew_blocks(c.np), 256, 0, c.stream>>>(c.parts, c.np, sx, sy);
        c.check_launch("k_shift_parts");
    }
    if (!c.P.self_fields) return;
    for (DevBuf<cpx>* a : {&c.Rx, &c.Ry, &c.Ez, &c.Bz, &c.j0x, &c.j0y}) {
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
