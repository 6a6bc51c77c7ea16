// The adjoint march: the reverse sweep of the s-steps of the beam and its fields (Fourier y), which the reference
// does not have. It differentiates J = mean p_z of the live beam after K s-steps with respect to the laser
// mode coefficients of the start field and the beam momenta at s = 0 (through the start field, or after it). Each kernel is the transposed program of
// one forward kernel, in reverse order; every transform, filter and march coefficient is real or a multiple of
// i k, so the transposes are the conjugated coefficients and the inverse transforms (no normalisation).
//   k_adj_objective  J = sum w p_z / sum w over the live particles (one CTA, fixed order)
//   k_adj_rf_rows/cols  transposed real fields (F <- IFFT of R, L, E_z + i B_z; sim_fields.cpp:282-292): forward
//                    transforms of the field adjoints, the half-row fold of the Hermitian rows
//   k_adj_march      transposed per-mode march (march_point, sim_kernels.hpp:173-210), slices rear to front
//   k_adj_cur_cols/rows, k_adj_zfilter  transposed currents (filters, transforms, the zeta filter;
//                    sim_particles.cpp:120-156)
//   k_adj_deposit    transposed deposit (sim_particles.cpp:88-106): a gather of the current adjoints with the
//                    TSC weights and their derivatives
//   k_adj_push       transposed RK4 push (push_one, sim_kernels.hpp:98-149): the sub-steps recomputed from the
//                    level's checkpoint with the same sub-step rule (frozen schedule), then reversed stage by
//                    stage; the gather adjoint is a deposit of the field adjoints into dJ/dF
//   k_adj_lmodes     dJ/d(laser mode coefficient) = sum over slices of conj(laser spectrum) dJ/dR
//   k_adj_comoving   transposed co-moving field of the start (sim_fields.cpp:44-151): the tridiagonal solves
//                    along zeta by parallel cyclic reduction, one CTA per mode; dJ/dj_z of the start currents
//                    and dJ/dbeta per mode
//   k_adj_wsum, k_adj_beta  beta = sum w p_z / gamma / sum w (sim_fields.cpp:45-51): dJ/dbeta to every particle
#include "k_push.cuh"
#include "k_fft.cuh"
#include "k_dispatch.cuh"

namespace g3d {

namespace {
constexpr int ANT = 128;          // threads of the row kernels
constexpr int ACW = 8;            // columns per tile of the column kernels

// derivative of the TSC weights with respect to the index coordinate (tsc_weights of g3d_common.cuh)
__device__ __forceinline__ void tsc_dweights(double xi, double d[3]) {
    const double f = xi - floor(xi + 0.5);
    d[0] = -(0.5 - f); d[1] = -2 * f; d[2] = 0.5 + f;
}
// d(fz)/d(zeta) of AxisDev::locate at the cell i it returned
__device__ __forceinline__ double locate_slope(const AxisDev& ax, int i) {
    if (ax.uniform) return ax.ih;
    if (i < 0) return 1 / (ax.X[1] - ax.X[0]);
    if (i >= ax.n - 1) return 1 / (ax.X[ax.n - 1] - ax.X[ax.n - 2]);
    return 1 / (ax.X[i + 1] - ax.X[i]);
}
}  // namespace

// ---------------------------------------------------------------- objective
__global__ void __launch_bounds__(1024) k_adj_objective(PartsDev P, long np, double* __restrict__ out) {
    __shared__ double s0[1024], s1[1024];
    double a = 0, b = 0;
    for (long i = threadIdx.x; i < np; i += 1024)
        if (P.alive[i] == 1) { a += P.w[i] * P.pz[i]; b += P.w[i]; }
    s0[threadIdx.x] = a; s1[threadIdx.x] = b;
    __syncthreads();
    for (int s = 512; s > 0; s >>= 1) {
        if (int(threadIdx.x) < s) { s0[threadIdx.x] += s0[threadIdx.x + s]; s1[threadIdx.x] += s1[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { out[0] = s0[0]; out[1] = s1[0]; }
}
// dJ/d(final state): w / W on p_z of the live particles
__global__ void k_adj_seed(PartsDev P, long np, double W, double* __restrict__ lam) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= np) return;
    for (int k = 0; k < 5; ++k) lam[k * np + i] = 0;
    lam[5 * np + i] = P.alive[i] == 1 ? P.w[i] / W : 0.0;
}

// ---------------------------------------------------------------- transposed real fields
// rows: per row of slice l, Lambda_R = (lEx + lBy)/2 + i (lEy - lBx)/2, Lambda_L = (lEx - lBy)/2 + i (lEy + lBx)/2,
// Lambda_E = lEz + i lBz; their forward transforms times 1/nk, folded onto the half rows of the two fields of
// each pair: lA(k) = z(k) + conj z(nx-k), lB(k) = -i z(k) + i conj z(nx-k) (mirror terms for 0 < k < nx/2)
template <int NX>
__global__ void __launch_bounds__(ANT) k_adj_rf_rows(Geo g, const double* __restrict__ lF, cpx* __restrict__ W0, cpx* __restrict__ W1,
                                                    cpx* __restrict__ W2, cpx* __restrict__ W3, cpx* __restrict__ W4,
                                                    cpx* __restrict__ W5, long fpl) {
    using S = FftShape<NX>;
    constexpr int LPC = ANT / S::T, RS = row_stride<NX>(), H = NX / 2 + 1;
    extern __shared__ cpx sm[];
    cpx* a0 = sm;
    cpx* a1 = sm + LPC * RS;
    cpx* a2 = sm + 2 * LPC * RS;
    const int l = blockIdx.y, r0 = blockIdx.x * LPC, tid = threadIdx.x;
    const long fbase = long(l) * g.nk;
    for (int e = tid; e < LPC * NX; e += ANT) {
        const int rr = e / NX, p = e - rr * NX, row = r0 + rr;
        double f[6] = {0, 0, 0, 0, 0, 0};
        if (row < g.ny) {
            const long idx = fbase + long(row) * NX + p;
            for (int k = 0; k < 6; ++k) f[k] = lF[k * fpl + idx];
        }
        const int q = rr * RS + p + (p >> 3);
        a0[q] = C(0.5 * (f[0] + f[4]), 0.5 * (f[1] - f[3]));
        a1[q] = C(0.5 * (f[0] - f[4]), 0.5 * (f[1] + f[3]));
        a2[q] = C(f[2], f[5]);
    }
    __syncthreads();
    const int r = tid / S::T, t = tid - r * S::T;
    {
        decltype(a0) const ls_[3] = {a0, a1, a2};
        fft_lines<NX, 3>(ls_, RowAddr{r * RS}, t, g.twx);
    }
    const double s = 1.0 / double(g.nk);
    const long base = long(l) * g.nkh;
    for (int e = tid; e < LPC * H; e += ANT) {
        const int rr = e / H, kx = e - rr * H, row = r0 + rr;
        if (row >= g.ny) continue;
        const bool mirror = kx > 0 && kx < NX / 2;
        const int km = NX - kx;
        const long o = base + long(row) * H + kx;
        cpx* outA[3] = {W0, W2, W4};
        cpx* outB[3] = {W1, W3, W5};
        const cpx* a[3] = {a0, a1, a2};
        for (int pr = 0; pr < 3; ++pr) {
            const cpx z = s * a[pr][rr * RS + kx + (kx >> 3)];
            cpx lA = z, lB = mul_mi(z);
            if (mirror) {
                const cpx zm = conj(s * a[pr][rr * RS + km + (km >> 3)]);
                lA = lA + zm; lB = lB + mul_i(zm);
            }
            outA[pr][o] = lA; outB[pr][o] = lB;
        }
    }
}
// columns: forward transforms along y of the six half-row adjoints, added to the spectrum adjoints of slice l
// (R, E_z, B_z; assigned for L, whose adjoint the transposed march leaves stale), or all six assigned (`assign`: one
// slice of the streaming-plasma march, whose slice fields are read by nothing but its own real fields)
template <int NY>
__global__ void __launch_bounds__(ACW * FftShape<NY>::T) k_adj_rf_cols(Geo g, const cpx* __restrict__ W0, const cpx* __restrict__ W1,
                                                                      const cpx* __restrict__ W2, const cpx* __restrict__ W3,
                                                                      const cpx* __restrict__ W4, const cpx* __restrict__ W5,
                                                                      cpx* __restrict__ lRx, cpx* __restrict__ lRy, cpx* __restrict__ lLx,
                                                                      cpx* __restrict__ lLy, cpx* __restrict__ lEz, cpx* __restrict__ lBz,
                                                                      int assign) {
    using S = FftShape<NY>;
    extern __shared__ cpx sm[];
    const int l = blockIdx.y, c0 = blockIdx.x * ACW, tid = threadIdx.x, nthr = ACW * S::T, pr = blockIdx.z;
    const int H = g.H;
    const long base = long(l) * g.nkh;
    const cpx* in0 = pr == 0 ? W0 : pr == 1 ? W2 : W4;
    const cpx* in1 = pr == 0 ? W1 : pr == 1 ? W3 : W5;
    cpx* out0 = pr == 0 ? lRx : pr == 1 ? lLx : lEz;
    cpx* out1 = pr == 0 ? lRy : pr == 1 ? lLy : lBz;
    cpx* s0 = sm;
    cpx* s1 = sm + ColTile<NY, ACW>::size;
    for (int e = tid; e < NY * ACW; e += nthr) {
        const int p = e / ACW, c = e - p * ACW, kxi = c0 + c;
        const long o = base + long(p) * H + kxi;
        s0[ColTile<NY, ACW>::at(p, c)] = kxi < H ? in0[o] : C(0);
        s1[ColTile<NY, ACW>::at(p, c)] = kxi < H ? in1[o] : C(0);
    }
    __syncthreads();
    const int c = tid % ACW, t = tid / ACW;
    {
        decltype(s0) const ls_[2] = {s0, s1};
        fft_lines<NY, 2>(ls_, RowAddr{c * ColTile<NY, ACW>::RS}, t, g.twy);
    }
    for (int e = tid; e < NY * ACW; e += nthr) {
        const int p = e / ACW, cc = e - p * ACW, kxi = c0 + cc;
        if (kxi >= H) continue;
        const long o = base + long(p) * H + kxi;
        if (pr == 1 || assign) { out0[o] = s0[ColTile<NY, ACW>::at(p, cc)]; out1[o] = s1[ColTile<NY, ACW>::at(p, cc)]; }   // L: not an input of the forward march
        else { out0[o] = out0[o] + s0[ColTile<NY, ACW>::at(p, cc)]; out1[o] = out1[o] + s1[ColTile<NY, ACW>::at(p, cc)]; }
    }
}

// ---------------------------------------------------------------- transposed march
// The transposed per-mode march in the two-lane form of the forward (k_march.cu): with E~ = i E_z, B~ = i B_z
// every coefficient is real, so lane c = 0 carries the adjoints of (Re R, Re L, -Im E_z, -Im B_z) and lane c = 1
// those of (Im R, Im L, Re E_z, Re B_z); each lane is the transpose of the forward lane's real recurrence. Slices
// n = a .. N-1 (the reverse of the forward's N-1 .. a): the adjoints of the new level at slice n (given, plus what
// slice n-1 passed up through the values of slice n+1 it read) become those of the old level (R, E_z, B_z; the
// old L is not read by the forward, so lLx, lLy are left to the next transposed real fields, which assign
// them) and of the currents. The two half-cells of a slice are written once each: the upper one's terms ride
// in registers to the next slice, where it is the lower one. lj0 is written; ljk_x, ljk_y hold on entry the
// adjoint of jk as the j0 of the next step and are overwritten with the total; ljk_z is written, or added to
// (accz: the marches of the start field's relaxation, whose j_z adjoint adds to that of init's march(0)). Per
// slice each lane streams its 8 values (the 6 adjoints of the new level, the 2 pending ones; with accz a third,
// j_z, so that no plain load waits inside the chain) and the slice's coefficients DEPTH slices ahead into a
// shared-memory ring with cp.async, as the forward does.
namespace {
constexpr int AMA = 9, AMC = 3;
constexpr int aslot(int bt) { return (AMA + AMC) * bt; }
__device__ __forceinline__ void acp8(void* smem, const void* gmem) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void acommit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void await_() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
}  // namespace

template <int BT, int DEPTH>
__global__ void __launch_bounds__(BT) k_adj_march(Geo g, cpx* __restrict__ lRx, cpx* __restrict__ lRy, cpx* __restrict__ lEz,
                                                 cpx* __restrict__ lBz, cpx* __restrict__ lLx, cpx* __restrict__ lLy,
                                                 cpx* __restrict__ lj0x, cpx* __restrict__ lj0y, cpx* __restrict__ ljkx,
                                                 cpx* __restrict__ ljky, cpx* __restrict__ ljkz, double D, int accz) {
    extern __shared__ double ringa[];
    const long nk = g.nkh;
    const int tid = threadIdx.x;
    const long gt = long(blockIdx.x) * BT + tid;
    const int c = int(gt & 1);
    const long i = gt >> 1;
    const bool live = i < nk;
    const long ii = live ? i : 0;
    const int kxi = int(ii % g.H), j = int(ii / g.H);
    const double kx = g.kxd[kxi], ky = g.kyd[j], k2 = kx * kx + ky * ky;
    const double sgn = c ? 1.0 : -1.0;
    auto own = [&](long o) { return 2 * o + c; };
    auto oth = [&](long o) { return 2 * o + 1 - c; };
    double* Rx = reinterpret_cast<double*>(lRx);
    double* Ry = reinterpret_cast<double*>(lRy);
    double* Ez = reinterpret_cast<double*>(lEz);
    double* Bz = reinterpret_cast<double*>(lBz);
    double* Lx = reinterpret_cast<double*>(lLx);
    double* Ly = reinterpret_cast<double*>(lLy);
    double* j0x = reinterpret_cast<double*>(lj0x);
    double* j0y = reinterpret_cast<double*>(lj0y);
    double* jkx = reinterpret_cast<double*>(ljkx);
    double* jky = reinterpret_cast<double*>(ljky);
    double* jkz = reinterpret_cast<double*>(ljkz);
    auto cell = [&](int sl, int k) { return ringa + size_t(sl) * aslot(BT) + k * BT + tid; };
    // ring cells: 0 R_x, 1 R_y, 2 L_x, 3 L_y (own), 4 E_z, 5 B_z (other), 6 jk_x, 7 jk_y pending (own); w_lo, w_hi,
    // h; 11 jk_z pending (other; accz only)
    auto fetch = [&](int n) {
        const int sl = (n - g.a) % DEPTH;
        const long o = long(n - g.a) * nk + ii;
        acp8(cell(sl, 0), Rx + own(o)); acp8(cell(sl, 1), Ry + own(o));
        acp8(cell(sl, 2), Lx + own(o)); acp8(cell(sl, 3), Ly + own(o));
        acp8(cell(sl, 4), Ez + oth(o)); acp8(cell(sl, 5), Bz + oth(o));
        acp8(cell(sl, 6), jkx + own(o)); acp8(cell(sl, 7), jky + own(o));
        acp8(cell(sl, 8), g.wlo + n); acp8(cell(sl, 9), g.whi + n); acp8(cell(sl, 10), g.hcg + n + 2);
        if (accz) acp8(cell(sl, 11), jkz + oth(o));
    };
#pragma unroll
    for (int q = 0; q < DEPTH; ++q) {
        const int n = g.a + q;
        if (n <= g.b - 1) fetch(n);
        acommit();
    }
    double qRx = 0, qRy = 0, qLx = 0, qLy = 0, qE = 0, qB = 0;          // adjoints of the p-values of slice n
    double c0x = 0, c0y = 0, ckx = 0, cky = 0, ckz = 0;                 // lower half-cell terms from slice n-1
    double rden = 0;
    bool have_rden = false;
    for (int n = g.a; n <= g.b - 1; ++n) {
        await_<DEPTH - 1>();
        const int sl = (n - g.a) % DEPTH;
        const long o = long(n - g.a) * nk + ii;
        const double ARx = *cell(sl, 0) + qRx, ARy = *cell(sl, 1) + qRy;
        const double ALx = *cell(sl, 2) + qLx, ALy = *cell(sl, 3) + qLy;
        double AE = sgn * *cell(sl, 4) + qE, AB = sgn * *cell(sl, 5) + qB;
        const double pkx = *cell(sl, 6), pky = *cell(sl, 7);
        const double wl = *cell(sl, 8), wu = *cell(sl, 9), h = *cell(sl, 10);
        const double pkz = accz ? *cell(sl, 11) : 0.0;
        if (!have_rden) rden = 1 / (1 + 0.25 * h * (D + 0.25 * h) * k2);
        double rden_next = 0;                 // the next slice's inverse denominator, off the chain
        if (n < g.b - 1) {
            await_<DEPTH - 2>();
            const double hn = *cell((sl + 1) % DEPTH, 10);
            rden_next = 1 / (1 + 0.25 * hn * (D + 0.25 * hn) * k2);
        }
        double lRsx = ARx, lRsy = ARy;
        double ux = 0, uy = 0, uz = 0;                                   // adjoints of jk of the upper half-cell
        if (n == g.N - 1) {
            qRx = qRy = qLx = qLy = qE = qB = 0;
        } else {
            double lLsx = ALx, lLsy = ALy;
            AB += -0.25 * h * kx * ALy + 0.25 * h * ky * ALx - D * kx * ARy + D * ky * ARx;
            AE += -0.25 * h * ky * ALy - 0.25 * h * kx * ALx + D * ky * ARy + D * kx * ARx;
            const double tE = AE * rden, tB = AB * rden;
            const double liQp = -0.5 * h * tE, liSE = -0.25 * h * tE, lupz = -h * tE;
            const double liCp = -0.5 * h * tB, liSB = -0.25 * h * tB;
            // iSE = kx Rsx - kx Lsx - ky Lsy + ky Rsy; iSB = -kx Rsy - kx Lsy + ky Rsx + ky Lsx
            lRsx += kx * liSE + ky * liSB;
            lLsx += -kx * liSE + ky * liSB;
            lLsy += -ky * liSE - kx * liSB;
            lRsy += ky * liSE - kx * liSB;
            // iQp = kx (pRx - pLx)/2 - ky (pLy - pRy)/2; iCp = (-kx (pRy + pLy) + ky (pRx + pLx))/2
            double lpRx = 0.5 * kx * liQp + 0.5 * ky * liCp;
            double lpLx = -0.5 * kx * liQp + 0.5 * ky * liCp;
            double lpLy = -0.5 * ky * liQp - 0.5 * kx * liCp;
            double lpRy = 0.5 * ky * liQp - 0.5 * kx * liCp;
            double lpE = tE, lpB = tB;
            // Lsy = pLy - (h/4)(kx pB + ky pE) - (h/2) upy; Lsx = pLx - (h/4)(kx pE - ky pB) - (h/2) upx
            lpLy += lLsy; lpB += -0.25 * h * kx * lLsy; lpE += -0.25 * h * ky * lLsy;
            lpLx += lLsx; lpE += -0.25 * h * kx * lLsx; lpB += 0.25 * h * ky * lLsx;
            ux = -0.5 * h * lLsx; uy = -0.5 * h * lLsy; uz = lupz;
            qRx = lpRx; qRy = lpRy; qLx = lpLx; qLy = lpLy; qE = lpE; qB = lpB;
        }
        // Rsx = rx + D (kx e + ky b) - D Jx; Rsy = ry + D (ky e - kx b) - D Jy
        const double le = D * kx * lRsx + D * ky * lRsy, lb = D * ky * lRsx - D * kx * lRsy;
        const double lJx = -D * lRsx, lJy = -D * lRsy;
        if (live) {                           // (the adjoints of the old L stay: the old L is not read)
            Rx[own(o)] = lRsx; Ry[own(o)] = lRsy; Ez[oth(o)] = sgn * le; Bz[oth(o)] = sgn * lb;
            // the lower half-cell (plane n - a): this slice's w_lo terms and the previous slice's upper terms
            j0x[own(o)] = c0x + wl * lJx; j0y[own(o)] = c0y + wl * lJy;
            jkx[own(o)] = pkx + ckx + wl * lJx; jky[own(o)] = pky + cky + wl * lJy;
            jkz[oth(o)] = pkz + sgn * ckz;
        }
        rden = rden_next;
        have_rden = n < g.b - 1;
        c0x = wu * lJx; c0y = wu * lJy; ckx = wu * lJx + ux; cky = wu * lJy + uy; ckz = uz;
        const int nn = n + DEPTH;
        if (nn <= g.b - 1) fetch(nn);
        acommit();
    }
    await_<0>();
    if (live) {                                                          // the upper half-cell of the front slice
        const long ou = long(g.ns) * nk + ii;
        j0x[own(ou)] = c0x; j0y[own(ou)] = c0y;
        jkx[own(ou)] = jkx[own(ou)] + ckx; jky[own(ou)] = jky[own(ou)] + cky;
        jkz[oth(ou)] = accz ? jkz[oth(ou)] + sgn * ckz : sgn * ckz;
    }
}

// ---------------------------------------------------------------- transposed currents
// columns: per half-cell plane, the filters f(k) (zero at k = 0 unless keep0: the box mean of a run with plasma) with
// the smoothing 1 / (1 + a2 k_perp^2) (a2 > 0: the streaming current's spectra, k_ss_cols) and the unnormalised
// inverse transform along y
template <int NY>
__global__ void __launch_bounds__(ACW * FftShape<NY>::T) k_adj_cur_cols(Geo g, const cpx* __restrict__ JX, const cpx* __restrict__ JY,
                                                                       const cpx* __restrict__ JZ, cpx* __restrict__ TX,
                                                                       cpx* __restrict__ TY, cpx* __restrict__ TZ, int keep0,
                                                                       double a2) {
    using S = FftShape<NY>;
    extern __shared__ cpx sm[];
    cpx* s0 = sm;
    cpx* s1 = sm + ColTile<NY, ACW>::size;
    cpx* s2 = sm + 2 * ColTile<NY, ACW>::size;
    const int hk = blockIdx.y, c0 = blockIdx.x * ACW, tid = threadIdx.x, nthr = ACW * S::T;
    const int H = g.H;
    const long base = long(hk) * g.nkh;
    for (int e = tid; e < NY * ACW; e += nthr) {
        const int p = e / ACW, c = e - p * ACW, kx = c0 + c;
        cpx u0 = C(0), u1 = C(0), u2 = C(0);
        if (kx < H) {
            const double k2 = g.kxs[kx] * g.kxs[kx] + g.kys[p] * g.kys[p];
            const double f = (kx == 0 && p == 0 && !keep0) ? 0.0 : g.filt[kx] * g.filty[p] / (1 + a2 * k2);
            const long o = base + long(p) * H + kx;
            u0 = conj(f * JX[o]); u1 = conj(f * JY[o]); u2 = conj(f * JZ[o]);
        }
        s0[ColTile<NY, ACW>::at(p, c)] = u0; s1[ColTile<NY, ACW>::at(p, c)] = u1; s2[ColTile<NY, ACW>::at(p, c)] = u2;
    }
    __syncthreads();
    const int c = tid % ACW, t = tid / ACW;
    {
        decltype(s0) const ls_[3] = {s0, s1, s2};
        fft_lines<NY, 3>(ls_, RowAddr{c * ColTile<NY, ACW>::RS}, t, g.twy);
    }
    for (int e = tid; e < NY * ACW; e += nthr) {
        const int p = e / ACW, cc = e - p * ACW, kx = c0 + cc;
        if (kx >= H) continue;
        const long o = base + long(p) * H + kx;
        TX[o] = conj(s0[ColTile<NY, ACW>::at(p, cc)]); TY[o] = conj(s1[ColTile<NY, ACW>::at(p, cc)]); TZ[o] = conj(s2[ColTile<NY, ACW>::at(p, cc)]);
    }
}
// rows: the transposed Hermitian split (lz(k) = (lTX + i lTY)/2, lz(nx-k) = (conj lTX + i conj lTY)/2; at
// k = 0, nx/2: Re lTX + i Re lTY) and the unnormalised inverse transform along x: Re -> lv_x, Im -> lv_y; j_z
// from lTZ (zero above nx/2), real part -> lv_z. Out: V [3][ns+1][ny][nx].
template <int NX>
__global__ void __launch_bounds__(ANT) k_adj_cur_rows(Geo g, const cpx* __restrict__ TX, const cpx* __restrict__ TY,
                                                     const cpx* __restrict__ TZ, double* __restrict__ V, long vpl) {
    using S = FftShape<NX>;
    constexpr int LPC = ANT / S::T, RS = row_stride<NX>(), H = NX / 2 + 1;
    extern __shared__ cpx sm[];
    cpx* a0 = sm;
    cpx* a1 = sm + LPC * RS;
    const int tid = threadIdx.x, r0 = blockIdx.x * LPC, hk = blockIdx.y;
    const long base = long(hk) * g.nkh;
    for (int e = tid; e < LPC * NX; e += ANT) {                 // zero the rows (the mirror halves are added)
        const int rr = e / NX, p = e - rr * NX;
        a0[rr * RS + p + (p >> 3)] = C(0); a1[rr * RS + p + (p >> 3)] = C(0);
    }
    __syncthreads();
    for (int e = tid; e < LPC * H; e += ANT) {
        const int rr = e / H, kx = e - rr * H, row = r0 + rr;
        if (row >= g.ny) continue;
        const long o = base + long(row) * H + kx;
        const cpx lx = TX[o], ly = TY[o];
        cpx zk;
        if (kx == 0 || kx == NX / 2) zk = C(lx.x, ly.x);
        else {
            zk = 0.5 * (lx + mul_i(ly));
            const int km = NX - kx;
            a0[rr * RS + km + (km >> 3)] = conj(0.5 * (conj(lx) + mul_i(conj(ly))));
        }
        a0[rr * RS + kx + (kx >> 3)] = conj(zk);
        a1[rr * RS + kx + (kx >> 3)] = conj(TZ[o]);
    }
    __syncthreads();
    const int r = tid / S::T, t = tid - r * S::T;
    {
        decltype(a0) const ls_[2] = {a0, a1};
        fft_lines<NX, 2>(ls_, RowAddr{r * RS}, t, g.twx);
    }
    const long nk = g.nk;
    for (int e = tid; e < LPC * NX; e += ANT) {
        const int rr = e / NX, p = e - rr * NX, row = r0 + rr;
        if (row >= g.ny) continue;
        const cpx u = conj(a0[rr * RS + p + (p >> 3)]), w = conj(a1[rr * RS + p + (p >> 3)]);
        const long idx = long(hk) * nk + long(row) * NX + p;
        V[idx] = u.x; V[vpl + idx] = u.y; V[2 * vpl + idx] = w.x;
    }
}
// the transposed zeta filter: plane hk read the raw planes hk, hk+1, hk+2 with weights (cm, c0, cp)(hk)
__device__ __forceinline__ void zf_weights(const Geo& g, int hk, int zf, double w[3]) {
    const int hc = g.a - 1 + hk;
    if (hk < 0 || hk > g.ns || hc < 0 || hc > g.N - 2) { w[0] = w[1] = w[2] = 0; return; }
    if (!zf) { w[0] = 0; w[1] = 1; w[2] = 0; return; }
    if (g.zeta_uniform) { w[0] = 0.25; w[1] = 0.5; w[2] = 0.25; return; }
    const double inv = g.hcg[hc + 2];
    w[0] = 0.25 * g.hcg[hc + 1] / inv; w[1] = 0.5 * g.hcg[hc + 2] / inv; w[2] = 0.25 * g.hcg[hc + 3] / inv;
}
__global__ void k_adj_zfilter(Geo g, const double* __restrict__ V, double* __restrict__ lJ, int zf) {
    const long nk = g.nk, vpl = long(g.ns + 1) * nk, jpl = long(g.nh) * nk, n = 3 * jpl;
    for (long idx = long(blockIdx.x) * blockDim.x + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
        const int comp = int(idx / jpl);
        const long r = idx - comp * jpl;
        const int h = int(r / nk);
        const long k = r - long(h) * nk;
        double s = 0;
        for (int d = 0; d < 3; ++d) {
            const int hk = h - d;
            if (hk < 0 || hk > g.ns) continue;
            double w[3];
            zf_weights(g, hk, zf, w);
            if (w[d] != 0) s += w[d] * V[comp * vpl + long(hk) * nk + k];
        }
        lJ[idx] = s;
    }
}

// ---------------------------------------------------------------- transposed deposit
// j = f W(x, y) (p_x/p_z, p_y/p_z, 1), f = q w / (h_m dx dy), NGP in zeta (no zeta derivative)
__global__ void __launch_bounds__(256) k_adj_deposit(PartsDev P, const double* __restrict__ X, const int32_t* __restrict__ alive,
                                                    long np, Geo g, const double* __restrict__ lJ, double* __restrict__ lam) {
    const long ip = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (ip >= np || alive[ip] != 1) return;
    const double x = X[ip], y = X[np + ip], zeta = X[2 * np + ip], px = X[3 * np + ip], py = X[4 * np + ip], pz = X[5 * np + ip];
    int m; double fz;
    g.zax.locate(zeta, m, fz);
    const int hw = m - (g.a - 2);
    if (hw < 0 || hw >= g.nh || m < 0 || m > g.N - 2) return;
    const double f = P.q[ip] * P.w[ip] / (g.hcg[m + 2] * g.dx) * g.iA[0];
    int ix[3], jn[3]; double wx[3], wn[3], dwx[3], dwn[3];
    tsc_periodic(x, g.dx, g.nx, ix, wx);
    tsc_periodic(y, g.dy, g.ny, jn, wn);
    tsc_dweights(x / g.dx, dwx);
    tsc_dweights(y / g.dy, dwn);
    const long nk = g.nk, pl = long(g.nh) * nk;
    const double* J0 = lJ + long(hw) * nk;
    const double ux = px / pz, uy = py / pz;
    double Gx = 0, Gy = 0, Dx = 0, Dy = 0;
    for (int v = 0; v < 3; ++v)
        for (int u = 0; u < 3; ++u) {
            const long k = long(jn[v]) * g.nx + ix[u];
            const double ax = J0[k], ay = J0[pl + k], az = J0[2 * pl + k];
            const double W = wx[u] * wn[v];
            Gx += W * ax; Gy += W * ay;
            const double s = ax * ux + ay * uy + az;
            Dx += dwx[u] * wn[v] * s; Dy += wx[u] * dwn[v] * s;
        }
    lam[ip] += f * Dx / g.dx;
    lam[np + ip] += f * Dy / g.dy;
    lam[3 * np + ip] += f * Gx / pz;
    lam[4 * np + ip] += f * Gy / pz;
    lam[5 * np + ip] += -f * (Gx * ux + Gy * uy) / pz;
}

// ---------------------------------------------------------------- transposed push
// The stencil of one gather: the field adjoints A[6] and where they go in dJ/dF (the TSC points, the two slice
// planes and their weights). The four stages of an RK4 sub-step usually share the stencil (a sub-step moves a
// particle by far less than a cell), so their deposits are summed per point before the atomics.
struct Sten {
    double A[6], wx[3], wn[3], fz;
    int ix[3], jn[3], fl;                     // fl < 0: nothing to deposit
};
// The fields at one stage point with their gradients (per component: value, d/dx, d/dy, d/dzeta), gathered as
// the forward gathers them, and the stencil the field adjoints of that point go to (A is filled by the reverse
// chain). The forward recompute of a sub-step gathers each of its four stage points once; the reverse chain then
// reads no memory.
struct Gat { double F[6], dx[6], dy[6], dz[6]; };
template <class FT>
__device__ __forceinline__ void gather_grad(const PushArgs& c, const FT* __restrict__ Fp, double x, double y, double zeta, Gat& G,
                                            Sten& st) {
#pragma unroll
    for (int comp = 0; comp < 6; ++comp) G.F[comp] = G.dx[comp] = G.dy[comp] = G.dz[comp] = 0;
    st.fl = -1;
    if (!c.self) return;
    const Geo& g = c.g;
    int n; double fz;
    g.zax.locate(zeta, n, fz);
    if (n == g.a - 1 && fz > 1 - 1e-9) { n = g.a; fz = 0; }
    const int fl = n - g.a;
    if (fl < 0 || fl > g.ns) return;
    const double dfz = locate_slope(g.zax, n);
    double dwx[3], dwn[3];
    tsc_periodic(x, g.dx, g.nx, st.ix, st.wx);
    tsc_periodic(y, g.dy, g.ny, st.jn, st.wn);
    tsc_dweights(x / g.dx, dwx);
    tsc_dweights(y / g.dy, dwn);
    const double idx_ = 1 / g.dx, idy = 1 / g.dy;
    const long nk = g.nk;
#pragma unroll
    for (int comp = 0; comp < 6; ++comp) {
        const FT* p0 = Fp + (long(comp) * (g.ns + 2) + fl) * nk;
        const FT* p1 = p0 + nk;
        double v = 0, sx = 0, sy = 0, sz = 0;
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const long k = long(st.jn[j]) * g.nx + st.ix[i];
                const double f0 = double(__ldg(p0 + k)), f1 = double(__ldg(p1 + k));
                const double val = (1 - fz) * f0 + fz * f1;
                v += st.wx[i] * st.wn[j] * val;
                sx += dwx[i] * st.wn[j] * val; sy += st.wx[i] * dwn[j] * val; sz += st.wx[i] * st.wn[j] * (f1 - f0);
            }
        G.F[comp] = v; G.dx[comp] = sx * idx_; G.dy[comp] = sy * idy; G.dz[comp] = sz * dfz;
    }
    st.fz = fz; st.fl = fl;
}
// the right-hand side of the characteristics at Y with the gathered fields (rhs of k_push.cuh, no analytic laser:
// the adjoint march rejects it)
__device__ __forceinline__ St rhs_g(const St& Y, double qm, const Gat& G) {
    const double g = sqrt(1 + Y.px * Y.px + Y.py * Y.py + Y.pz * Y.pz);
    const double gm = (1 + Y.px * Y.px + Y.py * Y.py) / (g + Y.pz);
    const double* E = G.F;
    const double* B = G.F + 3;
    const double ip = 1 / Y.pz;
    return St{Y.px * ip, Y.py * ip, -gm * ip, qm * (g * E[0] + Y.py * B[2] - Y.pz * B[1]) * ip,
              qm * (g * E[1] + Y.pz * B[0] - Y.px * B[2]) * ip, qm * (g * E[2] + Y.px * B[1] - Y.py * B[0]) * ip};
}
// the field adjoints of the stencils st[0..ns) into dJ/dF: summed per point when every stencil has the same
// points and planes, else one by one
__device__ __forceinline__ void flush_stencils(const Geo& g, const Sten* st, int ns, double* __restrict__ lF) {
    const long nk = g.nk;
    bool same = true;
    int first = -1;
    for (int s = 0; s < ns; ++s) {
        if (st[s].fl < 0) continue;
        if (first < 0) { first = s; continue; }
        same = same && st[s].fl == st[first].fl && st[s].ix[0] == st[first].ix[0] && st[s].jn[0] == st[first].jn[0];
    }
    if (first < 0) return;
    for (int s = (same ? first : 0); s < (same ? first + 1 : ns); ++s) {
        const Sten& b = st[s];
        if (b.fl < 0) continue;
        for (int comp = 0; comp < 6; ++comp) {
            const long off = (long(comp) * (g.ns + 2) + b.fl) * nk;
            for (int j = 0; j < 3; ++j)
                for (int i = 0; i < 3; ++i) {
                    double c0 = 0, c1 = 0;
                    if (same) {
                        for (int u = 0; u < ns; ++u) {
                            if (st[u].fl < 0) continue;
                            const double w = st[u].A[comp] * st[u].wx[i] * st[u].wn[j];
                            c0 += w * (1 - st[u].fz); c1 += w * st[u].fz;
                        }
                    } else {
                        const double w = b.A[comp] * b.wx[i] * b.wn[j];
                        c0 = w * (1 - b.fz); c1 = w * b.fz;
                    }
                    const long k = long(b.jn[j]) * g.nx + b.ix[i];
                    if (c0 != 0) atomicAdd(lF + off + k, c0);
                    if (c1 != 0) atomicAdd(lF + off + nk + k, c1);
                }
        }
    }
}
// lY += d(mu . rhs)/dY at Y from the gathered fields and gradients; the field adjoints A into the stencil st
__device__ __forceinline__ void rhs_adj(const St& Y, double qm, const St& mu, const Gat& G, St& lY, Sten& st) {
    const double px = Y.px, py = Y.py, pz = Y.pz;
    const double g = sqrt(1 + px * px + py * py + pz * pz);
    const double gpz = g + pz, gm = (1 + px * px + py * py) / gpz, ip = 1 / pz;
    double A[6];
    A[0] = mu.px * qm * g * ip; A[1] = mu.py * qm * g * ip; A[2] = mu.pz * qm * g * ip;
    A[3] = qm * ip * (mu.py * pz - mu.pz * py);
    A[4] = qm * ip * (mu.pz * px - mu.px * pz);
    A[5] = qm * ip * (mu.px * py - mu.py * px);
    double gx = 0, gy = 0, gz = 0;
#pragma unroll
    for (int comp = 0; comp < 6; ++comp) {
        gx += A[comp] * G.dx[comp]; gy += A[comp] * G.dy[comp]; gz += A[comp] * G.dz[comp];
        st.A[comp] = A[comp];
    }
    const double* E = G.F;
    const double* B = G.F + 3;
    const double Fx = qm * (g * E[0] + py * B[2] - pz * B[1]);
    const double Fy = qm * (g * E[1] + pz * B[0] - px * B[2]);
    const double Fz = qm * (g * E[2] + px * B[1] - py * B[0]);
    const double Gm = mu.px * E[0] + mu.py * E[1] + mu.pz * E[2];
    const double dgx = (2 * px - gm * px / g) / gpz, dgy = (2 * py - gm * py / g) / gpz, dgz = -gm * (pz / g + 1) / gpz;
    lY.x += gx; lY.y += gy; lY.zeta += gz;
    lY.px += mu.x * ip - mu.zeta * ip * dgx + qm * ip * (Gm * px / g - mu.py * B[2] + mu.pz * B[1]);
    lY.py += mu.y * ip - mu.zeta * ip * dgy + qm * ip * (Gm * py / g + mu.px * B[2] - mu.pz * B[0]);
    lY.pz += -(mu.x * px + mu.y * py) * ip * ip - mu.zeta * ip * dgz + mu.zeta * gm * ip * ip +
             qm * ip * (Gm * pz / g - mu.px * B[1] + mu.py * B[0]) - ip * ip * (mu.px * Fx + mu.py * Fy + mu.pz * Fz);
}
__device__ __forceinline__ St scale(const St& a, double h) { return St{h * a.x, h * a.y, h * a.zeta, h * a.px, h * a.py, h * a.pz}; }
__device__ __forceinline__ St add(const St& a, const St& b) {
    return St{a.x + b.x, a.y + b.y, a.zeta + b.zeta, a.px + b.px, a.py + b.py, a.pz + b.pz};
}
// the adjoint of one RK4 sub-step at its start state Y: lam (of the end state) -> lam (of Y). The forward stages
// are recomputed with each stage point gathered once (values and gradients); the reverse chain uses those.
template <class FT>
__device__ __forceinline__ St rk4_adj(const PushArgs& c, const FT* __restrict__ Fp, const St& Y, double ds, double qm, const St& lam,
                                      double* __restrict__ lF) {
    const Geo& g = c.g;
    Gat G1, G2, G3, G4;
    Sten st[4];
    gather_grad(c, Fp, wrap_periodic(Y.x, g.Lx), wrap_periodic(Y.y, g.Ly), Y.zeta, G1, st[0]);
    const St Y2 = axpy(Y, 0.5 * ds, rhs_g(Y, qm, G1));
    gather_grad(c, Fp, wrap_periodic(Y2.x, g.Lx), wrap_periodic(Y2.y, g.Ly), Y2.zeta, G2, st[1]);
    const St Y3 = axpy(Y, 0.5 * ds, rhs_g(Y2, qm, G2));
    gather_grad(c, Fp, wrap_periodic(Y3.x, g.Lx), wrap_periodic(Y3.y, g.Ly), Y3.zeta, G3, st[2]);
    const St Y4 = axpy(Y, ds, rhs_g(Y3, qm, G3));
    gather_grad(c, Fp, wrap_periodic(Y4.x, g.Lx), wrap_periodic(Y4.y, g.Ly), Y4.zeta, G4, st[3]);
    St lY = lam;
    St m1 = scale(lam, ds / 6), m2 = scale(lam, ds / 3), m3 = scale(lam, ds / 3);
    const St m4 = scale(lam, ds / 6);
    St a{0, 0, 0, 0, 0, 0};
    rhs_adj(Y4, qm, m4, G4, a, st[3]);                // k4 = f(Y + ds k3)
    lY = add(lY, a); m3 = add(m3, scale(a, ds));
    a = St{0, 0, 0, 0, 0, 0};
    rhs_adj(Y3, qm, m3, G3, a, st[2]);                // k3 = f(Y + ds/2 k2)
    lY = add(lY, a); m2 = add(m2, scale(a, 0.5 * ds));
    a = St{0, 0, 0, 0, 0, 0};
    rhs_adj(Y2, qm, m2, G2, a, st[1]);                // k2 = f(Y + ds/2 k1)
    lY = add(lY, a); m1 = add(m1, scale(a, 0.5 * ds));
    a = St{0, 0, 0, 0, 0, 0};
    rhs_adj(Y, qm, m1, G1, a, st[0]);                 // k1 = f(Y)
    flush_stencils(c.g, st, 4, lF);
    return add(lY, a);
}
constexpr int ADJ_MAXSUB = 64;
// per particle: the level's checkpoint X (x, y, zeta, px, py, pz) and alive flags; lam in/out [6][np]
template <class FT>
__global__ void __launch_bounds__(128) k_adj_push(PushArgs c, const FT* __restrict__ Fp, PartsDev P, const int32_t* __restrict__ perm,
                                                 const double* __restrict__ X, const int32_t* __restrict__ alive, long np, double s0,
                                                 double* __restrict__ lam, double* __restrict__ lF, int* __restrict__ err) {
    const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const long ip = perm[t];                 // cell order: the warp's deposits into dJ/dF meet in the same lines
    const int al = alive[ip];
    if (al != 1) {                           // not pushed: the state passes unchanged
        if (al == 3) atomicOr(err, 1);
        return;
    }
    if (c.freeze && P.sp[ip] <= 0) return;
    St lm{lam[ip], lam[np + ip], lam[2 * np + ip], lam[3 * np + ip], lam[4 * np + ip], lam[5 * np + ip]};
    if (lm.x == 0 && lm.y == 0 && lm.zeta == 0 && lm.px == 0 && lm.py == 0 && lm.pz == 0) return;
    const St Y0{X[ip], X[np + ip], X[2 * np + ip], X[3 * np + ip], X[4 * np + ip], X[5 * np + ip]};
    const double qm = P.qm[ip], s1 = c.s1;
    const double zend = s1 - 1e-12 * fabs(s1);
    int nsub = 0;
    {                                         // the sub-step count of the forward (the last one is not taken)
        St Y = Y0;
        double z = s0;
        while (z < zend) {
            const double ds = substep(c, Y, z, s1);
            if (nsub == ADJ_MAXSUB) { atomicOr(err, 2); return; }
            ++nsub;
            if (!(z + ds < zend)) break;
            if (!rk4_step(c, Fp, Y, z, ds, qm)) return;      // lost in the forward: no adjoint
            z += ds;
        }
    }
    for (int t = nsub - 1; t >= 0; --t) {     // sub-step t from its start state, the schedule recomputed as taken
        St Y = Y0;
        double z = s0;
        for (int u = 0; u < t; ++u) {
            const double ds = substep(c, Y, z, s1);
            rk4_step(c, Fp, Y, z, ds, qm);
            z += ds;
        }
        lm = rk4_adj(c, Fp, Y, substep(c, Y, z, s1), qm, lm, lF);
    }
    lam[ip] = lm.x; lam[np + ip] = lm.y; lam[2 * np + ip] = lm.zeta;
    lam[3 * np + ip] = lm.px; lam[4 * np + ip] = lm.py; lam[5 * np + ip] = lm.pz;
}

// ---------------------------------------------------------------- laser mode coefficients
// R += a(k) s(k, l) at init: dJ/da(k) = sum_l conj(s_x) dJ/dR_x + conj(s_y) dJ/dR_y. A CTA takes 32 modes
// (coalesced along k_x) x LMS slice lanes, each lane summing every LMS-th slice; the lanes are added in a fixed order.
namespace { constexpr int LMS = 8; }
__global__ void __launch_bounds__(32 * LMS) k_adj_lmodes(Geo g, const cpx* __restrict__ lRx, const cpx* __restrict__ lRy,
                                                         const cpx* __restrict__ sx, const cpx* __restrict__ sy,
                                                         cpx* __restrict__ out) {
    __shared__ cpx part[LMS][32];
    const long nk = g.nkh;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const long i = long(blockIdx.x) * 32 + tx;
    cpx s = C(0);
    if (i < nk)
        for (int l = ty; l < g.ns; l += LMS) {
            const long o = long(l) * nk + i;
            s = s + conj(sx[o]) * lRx[o] + conj(sy[o]) * lRy[o];
        }
    part[ty][tx] = s;
    __syncthreads();
    if (ty == 0 && i < nk) {
        for (int q = 1; q < LMS; ++q) s = s + part[q][tx];
        out[i] = s;
    }
}

// ---------------------------------------------------------------- the start field's dependence on the bunch
// transposed co-moving field (Fourier y; k_comoving of k_march.cu, Simulation::comoving_field,
// src/sim_fields.cpp:44-151): per mode, R = -(1 + beta) i k psi with A(gm2) psi = rhs along zeta,
// rhs(l) = (w_lo j_z(l) + w_hi j_z(l+1)) / beta. In: dJ/dR; out: dJ/dj_z added to ljz and, when dbeta is given,
// dJ/dbeta of the mode (through 1 + beta, 1/beta and gm2 = 1 - beta^2):
//   dJ/dpsi = conj(-(1 + beta) i k) dJ/dR = (1 + beta) i k dJ/dR;  A^T dJ/drhs = dJ/dpsi;
//   dJ/dbeta = -Re<dJ/dR, i k psi> - Re<dJ/drhs, rhs> / beta - 2 beta Re<dJ/drhs, (dA/dgm2) psi>.
// One CTA per mode: the tridiagonal systems along zeta (A for psi, needed only for dbeta, and A^T) are solved
// by parallel cyclic reduction in shared memory, ceil(log2 ns) halvings of the coupling distance, so a mode
// costs a few microseconds instead of a 4 x ns-long dependent chain. The k = 0 mode is skipped: R(k = 0) =
// -(1 + beta) i 0 psi = 0 whatever psi is, so it has no adjoint.
namespace {
constexpr int CMT = 256;                            // threads per mode
// a_i x_{i-1} + b_i x_i + c_i x_{i+1} = d_i, i < n (a_0 = c_{n-1} = 0); on return d_i = x_i. Rows tid + r CMT.
template <int RPT>
__device__ void pcr_solve(double* a, double* b, double* c, cpx* d, int n) {
    const int tid = threadIdx.x;
    for (int s = 1; s < n; s <<= 1) {
        double na[RPT], nb[RPT], nc[RPT];
        cpx nd[RPT];
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = tid + r * CMT;
            if (i >= n) continue;
            double A2 = 0, B2 = b[i], C2 = 0;
            cpx D2 = d[i];
            if (i - s >= 0) {
                const double al = -a[i] / b[i - s];
                A2 = al * a[i - s]; B2 += al * c[i - s]; D2 = D2 + al * d[i - s];
            }
            if (i + s < n) {
                const double ga = -c[i] / b[i + s];
                C2 = ga * c[i + s]; B2 += ga * a[i + s]; D2 = D2 + ga * d[i + s];
            }
            na[r] = A2; nb[r] = B2; nc[r] = C2; nd[r] = D2;
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int i = tid + r * CMT;
            if (i < n) { a[i] = na[r]; b[i] = nb[r]; c[i] = nc[r]; d[i] = nd[r]; }
        }
        __syncthreads();
    }
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int i = tid + r * CMT;
        if (i < n) d[i] = (1 / b[i]) * d[i];
    }
    __syncthreads();
}
__device__ __forceinline__ double cdot(cpx u, cpx v) { return u.x * v.x + u.y * v.y; }
}  // namespace

template <int RPT>
__global__ void __launch_bounds__(CMT) k_adj_comoving(Geo g, const cpx* __restrict__ lRx, const cpx* __restrict__ lRy,
                                                     const cpx* __restrict__ jz, double beta, double gm2, cpx* __restrict__ ljz,
                                                     double* __restrict__ dbeta) {
    extern __shared__ double smc[];
    const int ns = g.ns, tid = threadIdx.x;
    cpx* d = reinterpret_cast<cpx*>(smc);
    double* a = smc + 2 * ns;
    double* b = a + ns;
    double* c = b + ns;
    const long nk = g.nkh, i = blockIdx.x;
    const int kxi = int(i % g.H), j = int(i / g.H);
    const double kx = g.kxd[kxi], ky = g.kyd[j], k2 = kx * kx + ky * ky;
    if (k2 == 0) {
        if (dbeta && tid == 0) dbeta[i] = 0;
        return;
    }
    // row l: lo(l) = gm2 lo1(l), up(l) = gm2 up1(l), dg(l) = k^2 + gm2 dg1(l) (k_comoving's coefficients)
    auto d1 = [&](int l, double& lo1, double& up1, double& dg1) {
        const int n = g.a + l;
        const double hm = g.hcg[n + 1], hp = g.hcg[n + 2];
        lo1 = -2 / ((hm + hp) * hm); up1 = -2 / ((hm + hp) * hp); dg1 = 2 / (hm * hp);
    };
    auto rhs_at = [&](int l) {
        const int n = g.a + l;
        const long o = long(l) * nk + i;
        return (1 / beta) * (g.wlo[n] * jz[o] + g.whi[n] * jz[o + nk]);
    };
    const bool tri = gm2 != 0;                       // gm2 = 0: A is the diagonal k^2
    cpx ps[RPT];
    if (dbeta) {                                     // psi = A^-1 rhs, kept per row in registers
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int l = tid + r * CMT;
            if (l >= ns) continue;
            double lo1, up1, dg1;
            d1(l, lo1, up1, dg1);
            a[l] = l > 0 ? gm2 * lo1 : 0; b[l] = k2 + gm2 * dg1; c[l] = l + 1 < ns ? gm2 * up1 : 0;
            d[l] = rhs_at(l);
        }
        __syncthreads();
        if (tri) pcr_solve<RPT>(a, b, c, d, ns);
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int l = tid + r * CMT;
            ps[r] = l < ns ? (tri ? d[l] : (1 / b[l]) * d[l]) : C(0);
        }
        __syncthreads();
    }
    // A^T lrhs = lpsi: row l of A^T is (up(l-1), dg(l), lo(l+1))
    const double opb = 1 + beta;
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int l = tid + r * CMT;
        if (l >= ns) continue;
        double lo1, up1, dg1, lo1n = 0, up1p = 0, t0, t1;
        d1(l, lo1, up1, dg1);
        if (l > 0) d1(l - 1, t0, up1p, t1);
        if (l + 1 < ns) d1(l + 1, lo1n, t0, t1);
        a[l] = l > 0 ? gm2 * up1p : 0; b[l] = k2 + gm2 * dg1; c[l] = l + 1 < ns ? gm2 * lo1n : 0;
        const long o = long(l) * nk + i;
        d[l] = opb * (ik(kx, lRx[o]) + ik(ky, lRy[o]));
    }
    __syncthreads();
    if (tri) pcr_solve<RPT>(a, b, c, d, ns);
    else {
#pragma unroll
        for (int r = 0; r < RPT; ++r) {
            const int l = tid + r * CMT;
            if (l < ns) d[l] = (1 / b[l]) * d[l];
        }
        __syncthreads();
    }
    // dJ/dj_z of plane p (0 .. ns): rhs(p) reads it with w_lo(p), rhs(p - 1) with w_hi(p - 1)
    for (int p = tid; p <= ns; p += CMT) {
        cpx v = C(0);
        if (p < ns) v = v + g.wlo[g.a + p] * d[p];
        if (p > 0) v = v + g.whi[g.a + p - 1] * d[p - 1];
        const long o = long(p) * nk + i;
        ljz[o] = ljz[o] + (1 / beta) * v;
    }
    if (!dbeta) return;
    double t1 = 0, t2 = 0, t3 = 0;
#pragma unroll
    for (int r = 0; r < RPT; ++r) {
        const int l = tid + r * CMT;
        if (l >= ns) continue;
        const long o = long(l) * nk + i;
        t1 -= cdot(lRx[o], ik(kx, ps[r])) + cdot(lRy[o], ik(ky, ps[r]));
        t2 -= cdot(d[l], rhs_at(l)) / beta;
        // Re<lrhs, (dA/dgm2) psi> = sum_m Re<psi_m, up1(m-1) lrhs(m-1) + dg1(m) lrhs(m) + lo1(m+1) lrhs(m+1)>
        double lo1, up1, dg1, lo1n = 0, up1p = 0, t0, tt;
        d1(l, lo1, up1, dg1);
        cpx v = dg1 * d[l];
        if (l > 0) { d1(l - 1, t0, up1p, tt); v = v + up1p * d[l - 1]; }
        if (l + 1 < ns) { d1(l + 1, lo1n, t0, tt); v = v + lo1n * d[l + 1]; }
        t3 -= cdot(ps[r], v);
    }
    // block sums in a fixed order
    __shared__ double red[3][CMT / 32];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        t1 += __shfl_down_sync(0xffffffffu, t1, off);
        t2 += __shfl_down_sync(0xffffffffu, t2, off);
        t3 += __shfl_down_sync(0xffffffffu, t3, off);
    }
    if ((tid & 31) == 0) { red[0][tid >> 5] = t1; red[1][tid >> 5] = t2; red[2][tid >> 5] = t3; }
    __syncthreads();
    if (tid == 0) {
        double s1 = 0, s2 = 0, s3 = 0;
        for (int w = 0; w < CMT / 32; ++w) { s1 += red[0][w]; s2 += red[1][w]; s3 += red[2][w]; }
        dbeta[i] = s1 + s2 + (-2 * beta) * s3;
    }
}
// sum of w over the particles alive at a level (one CTA, fixed order)
__global__ void __launch_bounds__(1024) k_adj_wsum(PartsDev P, const int32_t* __restrict__ alive, long np, double* __restrict__ out) {
    __shared__ double s0[1024];
    double a = 0;
    for (long i = threadIdx.x; i < np; i += 1024)
        if (alive[i] == 1) a += P.w[i];
    s0[threadIdx.x] = a;
    __syncthreads();
    for (int s = 512; s > 0; s >>= 1) {
        if (int(threadIdx.x) < s) s0[threadIdx.x] += s0[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = s0[0];
}
// beta = sum w p_z / gamma / sum w over the live bunch: dJ/dp += dJ/dbeta (w / W) d(p_z / gamma)/dp
__global__ void k_adj_beta(PartsDev P, const double* __restrict__ X, const int32_t* __restrict__ alive, long np, double c,
                           double* __restrict__ lam) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= np || alive[i] != 1) return;
    const double px = X[3 * np + i], py = X[4 * np + i], pz = X[5 * np + i];
    const double g = sqrt(1 + px * px + py * py + pz * pz), ig3 = 1 / (g * g * g), f = c * P.w[i];
    lam[3 * np + i] += f * (-pz * px * ig3);
    lam[4 * np + i] += f * (-pz * py * ig3);
    lam[5 * np + i] += f * ((1 + px * px + py * py) * ig3);
}
// complex64 -> complex128 (the start currents of the mixed form for the transposed co-moving field)
__global__ void k_adj_widen(const cpxf* __restrict__ a, cpx* __restrict__ b, long n) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) b[i] = to_d(a[i]);
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

void launch_adj_objective(Ctx& c, double* dev_out2) {
    k_adj_objective<<<1, 1024, 0, c.stream>>>(c.parts, c.np, dev_out2);
    c.check_launch("k_adj_objective");
}
void launch_adj_seed(Ctx& c, double W, double* lam) {
    k_adj_seed<<<unsigned((c.np + 255) / 256), 256, 0, c.stream>>>(c.parts, c.np, W, lam);
    c.check_launch("k_adj_seed");
}
template <int NX>
static void adj_rf_rows(Ctx& c, const double* lF, cpx* const* W) {
    constexpr int LPC = ANT / FftShape<NX>::T;
    const size_t smem = size_t(3) * LPC * row_stride<NX>() * sizeof(cpx);
    allow_smem(k_adj_rf_rows<NX>, smem);
    k_adj_rf_rows<NX><<<dim3(unsigned((c.ny + LPC - 1) / LPC), unsigned(c.ns)), ANT, smem, c.stream>>>(c.geo(), lF, W[0], W[1], W[2],
                                                                                                         W[3], W[4], W[5],
                                                                                                         long(c.ns + 2) * c.nk);
    c.check_launch("k_adj_rf_rows");
}
template <int NY>
static void adj_rf_cols(Ctx& c, cpx* const* W, cpx* const* lS) {
    const size_t smem = size_t(2) * ColTile<NY, ACW>::size * sizeof(cpx);
    allow_smem(k_adj_rf_cols<NY>, smem);
    k_adj_rf_cols<NY><<<dim3(unsigned((c.H + ACW - 1) / ACW), unsigned(c.ns), 3), ACW * FftShape<NY>::T, smem, c.stream>>>(
        c.geo(), W[0], W[1], W[2], W[3], W[4], W[5], lS[0], lS[1], lS[4], lS[5], lS[2], lS[3], 0);
    c.check_launch("k_adj_rf_cols");
}
// lS = {Rx, Ry, Ez, Bz, Lx, Ly}; W: 6 half-spectrum scratch arrays of ns planes
void launch_adj_real_fields(Ctx& c, const double* lF, cpx* const* W, cpx* const* lS) {
    const int tok = c.prof_begin("adj_real_fields");
    G3D_DISPATCH_N(c.nx, NX, adj_rf_rows<NX>(c, lF, W));
    G3D_DISPATCH_N(c.ny, NY, adj_rf_cols<NY>(c, W, lS));
    c.prof_end(tok);
}
// One slice of the streaming-plasma march: the transposed real fields of lF (6 planes of one slice, component stride
// fpl) assigned to the slice's spectrum adjoints lsl = {Rx, Ry, Ez, Bz, Lx, Ly} (one plane each); W: 6 planes of scratch
template <int NX>
static void adj_rf_rows_slice(Ctx& c, const double* lF, long fpl, cpx* const* W) {
    constexpr int LPC = ANT / FftShape<NX>::T;
    const size_t smem = size_t(3) * LPC * row_stride<NX>() * sizeof(cpx);
    allow_smem(k_adj_rf_rows<NX>, smem);
    k_adj_rf_rows<NX><<<dim3(unsigned((c.ny + LPC - 1) / LPC), 1u), ANT, smem, c.stream>>>(c.geo(), lF, W[0], W[1], W[2], W[3],
                                                                                          W[4], W[5], fpl);
    c.check_launch("k_adj_rf_rows");
}
template <int NY>
static void adj_rf_cols_slice(Ctx& c, cpx* const* W, cpx* const* lsl) {
    const size_t smem = size_t(2) * ColTile<NY, ACW>::size * sizeof(cpx);
    allow_smem(k_adj_rf_cols<NY>, smem);
    k_adj_rf_cols<NY><<<dim3(unsigned((c.H + ACW - 1) / ACW), 1u, 3u), ACW * FftShape<NY>::T, smem, c.stream>>>(
        c.geo(), W[0], W[1], W[2], W[3], W[4], W[5], lsl[0], lsl[1], lsl[4], lsl[5], lsl[2], lsl[3], 1);
    c.check_launch("k_adj_rf_cols");
}
void launch_adj_real_fields_slice(Ctx& c, const double* lF, long fpl, cpx* const* W, cpx* const* lsl) {
    const int tok = c.prof_begin("adj_real_fields_slice");
    G3D_DISPATCH_N(c.nx, NX, adj_rf_rows_slice<NX>(c, lF, fpl, W));
    G3D_DISPATCH_N(c.ny, NY, adj_rf_cols_slice<NY>(c, W, lsl));
    c.prof_end(tok);
}
// The transposed spectra of one half-cell's streaming current (k_ss_rows + the column part of k_pass_cols): ljsn (3 half
// planes) -> lJ (3 real planes, component stride nk); T: 3 planes of scratch
template <int NY>
static void adj_ss_cols(Ctx& c, cpx* const* ljsn, cpx* const* T, bool keep0, double a2) {
    const size_t smem = size_t(3) * ColTile<NY, ACW>::size * sizeof(cpx);
    allow_smem(k_adj_cur_cols<NY>, smem);
    k_adj_cur_cols<NY><<<dim3(unsigned((c.H + ACW - 1) / ACW), 1u), ACW * FftShape<NY>::T, smem, c.stream>>>(
        c.geo(), ljsn[0], ljsn[1], ljsn[2], T[0], T[1], T[2], keep0 ? 1 : 0, a2);
    c.check_launch("k_adj_cur_cols");
}
template <int NX>
static void adj_ss_rows(Ctx& c, cpx* const* T, double* lJ) {
    constexpr int LPC = ANT / FftShape<NX>::T;
    const size_t smem = size_t(2) * LPC * row_stride<NX>() * sizeof(cpx);
    allow_smem(k_adj_cur_rows<NX>, smem);
    k_adj_cur_rows<NX><<<dim3(unsigned((c.ny + LPC - 1) / LPC), 1u), ANT, smem, c.stream>>>(c.geo(), T[0], T[1], T[2], lJ, long(c.nk));
    c.check_launch("k_adj_cur_rows");
}
void launch_adj_rf_rows_slice(Ctx& c, const double* lF, long fpl, cpx* const* W) {
    const int tok = c.prof_begin("adj_rf_rows_slice");
    G3D_DISPATCH_N(c.nx, NX, adj_rf_rows_slice<NX>(c, lF, fpl, W));
    c.prof_end(tok);
}
void launch_adj_ss_rows(Ctx& c, cpx* const* T, double* lJ) {
    const int tok = c.prof_begin("adj_ss_rows");
    G3D_DISPATCH_N(c.nx, NX, adj_ss_rows<NX>(c, T, lJ));
    c.prof_end(tok);
}
void launch_adj_stream_spectra(Ctx& c, cpx* const* ljsn, cpx* const* T, double* lJ, bool keep0, double a2) {
    const int tok = c.prof_begin("adj_stream_spectra");
    G3D_DISPATCH_N(c.ny, NY, adj_ss_cols<NY>(c, ljsn, T, keep0, a2));
    G3D_DISPATCH_N(c.nx, NX, adj_ss_rows<NX>(c, T, lJ));
    c.prof_end(tok);
}
template <int BT, int DEPTH>
static void adj_march_launch(Ctx& c, cpx* const* lS, cpx* const* lj0, cpx* const* ljk, double D, int accz) {
    const unsigned blocks = unsigned((2 * c.nkh + BT - 1) / BT);
    const size_t smem = size_t(DEPTH) * aslot(BT) * sizeof(double);
    allow_smem(k_adj_march<BT, DEPTH>, smem);
    k_adj_march<BT, DEPTH><<<blocks, BT, smem, c.stream>>>(c.geo(), lS[0], lS[1], lS[2], lS[3], lS[4], lS[5], lj0[0], lj0[1], ljk[0],
                                                           ljk[1], ljk[2], D, accz);
}
// lS = {Rx, Ry, Ez, Bz, Lx, Ly}; ljk holds the pending adjoints of jk (x, y; z is added to)
void launch_adj_march(Ctx& c, cpx* const* lS, cpx* const* lj0, cpx* const* ljk, double D, int accz) {
    const int tok = c.prof_begin("adj_march");
    if (2 * c.nkh < 2L * 148 * 64) adj_march_launch<32, 6>(c, lS, lj0, ljk, D, accz);
    else adj_march_launch<64, 6>(c, lS, lj0, ljk, D, accz);
    c.check_launch("k_adj_march");
    c.prof_end(tok);
}
template <int NY>
static void adj_cur_cols(Ctx& c, cpx* const* ljk, cpx* const* T, bool keep0) {
    const size_t smem = size_t(3) * ColTile<NY, ACW>::size * sizeof(cpx);
    allow_smem(k_adj_cur_cols<NY>, smem);
    k_adj_cur_cols<NY><<<dim3(unsigned((c.H + ACW - 1) / ACW), unsigned(c.ns + 1)), ACW * FftShape<NY>::T, smem, c.stream>>>(
        c.geo(), ljk[0], ljk[1], ljk[2], T[0], T[1], T[2], keep0 ? 1 : 0, 0.0);
    c.check_launch("k_adj_cur_cols");
}
template <int NX>
static void adj_cur_rows(Ctx& c, cpx* const* T, double* V) {
    constexpr int LPC = ANT / FftShape<NX>::T;
    const size_t smem = size_t(2) * LPC * row_stride<NX>() * sizeof(cpx);
    allow_smem(k_adj_cur_rows<NX>, smem);
    k_adj_cur_rows<NX><<<dim3(unsigned((c.ny + LPC - 1) / LPC), unsigned(c.ns + 1)), ANT, smem, c.stream>>>(c.geo(), T[0], T[1], T[2], V,
                                                                                                          long(c.ns + 1) * c.nk);
    c.check_launch("k_adj_cur_rows");
}
// ljk (3 half-cell spectra) -> lJ (3 x (ns+3) raw planes); T: 3 scratch arrays of ns+1 planes, V: 3 (ns+1) real planes;
// keep0: the k_perp = 0 current kept (the steps of a run with plasma and box_mean, currents() of g3d_host.cu)
void launch_adj_currents(Ctx& c, cpx* const* ljk, cpx* const* T, double* V, double* lJ, bool keep0) {
    const int tok = c.prof_begin("adj_currents");
    G3D_DISPATCH_N(c.ny, NY, adj_cur_cols<NY>(c, ljk, T, keep0));
    G3D_DISPATCH_N(c.nx, NX, adj_cur_rows<NX>(c, T, V));
    k_adj_zfilter<<<ew_blocks(3L * (c.ns + 3) * c.nk), 256, 0, c.stream>>>(c.geo(), V, lJ, c.P.zeta_filter ? 1 : 0);
    c.check_launch("k_adj_zfilter");
    c.prof_end(tok);
}
void launch_adj_deposit(Ctx& c, const double* X, const int32_t* alive, const double* lJ, double* lam) {
    if (c.np == 0) return;
    const int tok = c.prof_begin("adj_deposit");
    k_adj_deposit<<<unsigned((c.np + 255) / 256), 256, 0, c.stream>>>(c.parts, X, alive, c.np, c.geo(), lJ, lam);
    c.check_launch("k_adj_deposit");
    c.prof_end(tok);
}
// the push from s0 to s1 of the level checkpointed in (X, alive) with the level's fields Ff (float) or Fd
void launch_adj_push(Ctx& c, const float* Ff, const double* Fd, const double* X, const int32_t* alive, double s0, double s1,
                     double* lam, double* lF, int* err) {
    if (c.np == 0) return;
    const PushArgs a = push_args(c, s1);
    const int tok = c.prof_begin("adj_push");
    const unsigned blocks = unsigned((c.np + 127) / 128);
    if (Fd) k_adj_push<double><<<blocks, 128, 0, c.stream>>>(a, Fd, c.parts, c.perm.p, X, alive, c.np, s0, lam, lF, err);
    else k_adj_push<float><<<blocks, 128, 0, c.stream>>>(a, Ff, c.parts, c.perm.p, X, alive, c.np, s0, lam, lF, err);
    c.check_launch("k_adj_push");
    c.prof_end(tok);
}
template <int RPT>
static void adj_comoving_launch(Ctx& c, const cpx* lRx, const cpx* lRy, const cpx* jz, double beta, double gm2, cpx* ljz,
                                double* dbeta) {
    const size_t smem = size_t(c.ns) * (sizeof(cpx) + 3 * sizeof(double));
    smem_attr(reinterpret_cast<const void*>(k_adj_comoving<RPT>), smem);
    k_adj_comoving<RPT><<<unsigned(c.nkh), CMT, smem, c.stream>>>(c.geo(), lRx, lRy, jz, beta, gm2, ljz, dbeta);
}
void launch_adj_comoving(Ctx& c, const cpx* lRx, const cpx* lRy, const cpx* jz, double beta, double gm2, cpx* ljz, double* dbeta) {
    const int ns = c.ns;
    if (ns <= 2 * CMT) adj_comoving_launch<2>(c, lRx, lRy, jz, beta, gm2, ljz, dbeta);
    else if (ns <= 4 * CMT) adj_comoving_launch<4>(c, lRx, lRy, jz, beta, gm2, ljz, dbeta);
    else if (ns <= 8 * CMT) adj_comoving_launch<8>(c, lRx, lRy, jz, beta, gm2, ljz, dbeta);
    else if (ns <= 16 * CMT) adj_comoving_launch<16>(c, lRx, lRy, jz, beta, gm2, ljz, dbeta);
    else throw Error(G3D_ERR_CAPACITY, "the adjoint's co-moving field takes at most 4096 slices");
    c.check_launch("k_adj_comoving");
}
void launch_adj_wsum(Ctx& c, const int32_t* alive, double* out) {
    k_adj_wsum<<<1, 1024, 0, c.stream>>>(c.parts, alive, c.np, out);
    c.check_launch("k_adj_wsum");
}
void launch_adj_beta(Ctx& c, const double* X, const int32_t* alive, double coef, double* lam) {
    if (c.np == 0) return;
    k_adj_beta<<<unsigned((c.np + 255) / 256), 256, 0, c.stream>>>(c.parts, X, alive, c.np, coef, lam);
    c.check_launch("k_adj_beta");
}
void launch_adj_widen(Ctx& c, const cpxf* a, cpx* b, long n) {
    k_adj_widen<<<ew_blocks(n), 256, 0, c.stream>>>(a, b, n);
    c.check_launch("k_adj_widen");
}
void launch_adj_lmodes(Ctx& c, const cpx* lRx, const cpx* lRy, cpx* out) {
    k_adj_lmodes<<<unsigned((c.nkh + 31) / 32), 32 * LMS, 0, c.stream>>>(c.geo(), lRx, lRy, c.lspx.p, c.lspy.p, out);
    c.check_launch("k_adj_lmodes");
}

}  // namespace g3d
