// The per-mode march over the slices (Fourier y) and the co-moving start field, on the half spectrum
// k_x = 0 .. nx/2 (every field is real, so its spectrum is Hermitian and the other half is implied).
//
// k_march: Simulation::march / march_point of the reference (src/sim_fields.cpp:7-39,
// src/sim_kernels.hpp:169-210). Every mode (k_x, k_y) is an independent recurrence from the front slice
// b-1 down to a: R by the trapezoidal rule in s, L, E_z, B_z by the trapezoidal rule over the half-cell
// of length h_n, B_z and E_z in closed form with the denominator 1 + (h/4)(D + h/4) k_perp^2, the current
// of slice n interpolated as w_lo (j0 + jk)_{n-1/2} + w_hi (j0 + jk)_{n+1/2}. One thread per mode keeps
// the values of slice n+1 (level s1) and of the upper half-cell in registers; each slice costs 9 loads
// (R_x, R_y, E_z, B_z of level s0 and the five current spectra of the lower half-cell) and 6 stores.
// The loads do not depend on the recurrence, so every thread streams them MS slices ahead into its own
// ring of shared memory with cp.async (16-byte copies, one commit group per slice): several hundred
// bytes per thread in flight keep HBM busy although one thread owns a whole chain of slices.
//
// k_comoving: Simulation::comoving_field for Fourier y (src/sim_fields.cpp:44-151): per mode the
// tridiagonal system of -(k_perp^2 + gamma^-2 d_zeta^2) psi = rho along zeta (Thomas), then
// R = -(1 + beta) i k psi, E_z = B_z = 0.
#include "g3d_ctx.hpp"

namespace g3d {

namespace {
constexpr int MT = 64;      // threads (modes) per block
constexpr int MS = 6;       // prefetch depth in slices
constexpr int MA = 9;       // complex arrays streamed per slice
constexpr int MC = 3;       // per-slice coefficients streamed with them: w_lo, w_hi, h
constexpr int SLOT = MA * MT * 2 + MC * MT;   // doubles per ring slot

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
}  // namespace

__device__ __forceinline__ cpx widen(cpx a) { return a; }
__device__ __forceinline__ cpx widen(cpxf a) { return to_d(a); }
template <class T> __device__ __forceinline__ T narrow(cpx a);
template <> __device__ __forceinline__ cpx narrow<cpx>(cpx a) { return a; }
template <> __device__ __forceinline__ cpxf narrow<cpxf>(cpx a) { return to_f(a); }

// One thread per mode. Per slice the thread's own loads (9 arrays) and its copies of the slice's coefficients
// land in its column of a ring of MS slots; the recurrence itself touches only registers and that ring. The
// denominator 1 + (h/4)(D + h/4) k_perp^2 is inverted one slice ahead, off the chain.
// T is the storage of E_z, B_z, L and the currents: complex128 (the FP64 form) or complex64 (the mixed form,
// 8-byte copies into the 16-byte ring cells). R stays complex128, and the recurrence runs in FP64 in both
// forms: its carried values (level s1 of R, L, E_z, B_z) never leave the registers, so the mixed form only
// rounds what it stores, and the cancellations in curl R and div R that make E_z, B_z gamma^-2 small are
// taken in FP64.
template <class T>
__global__ void __launch_bounds__(MT) k_march(Geo g, cpx* __restrict__ Rx, cpx* __restrict__ Ry, T* __restrict__ Ez,
                                             T* __restrict__ Bz, T* __restrict__ Lx, T* __restrict__ Ly,
                                             const T* __restrict__ j0x, const T* __restrict__ j0y,
                                             const T* __restrict__ jkx, const T* __restrict__ jky,
                                             const T* __restrict__ jkz, double D) {
    extern __shared__ double ringd[];        // MS slots of [MA arrays][MT] complex, then [MC][MT] double
    const long nk = g.nkh;
    const int tid = threadIdx.x;
    const long i = long(blockIdx.x) * MT + tid;
    const bool live = i < nk;
    const long ii = live ? i : 0;             // idle threads stream mode 0 and store nothing
    const int kxi = int(ii % g.H), j = int(ii / g.H);
    const double kx = g.kxd[kxi], ky = g.kyd[j], k2 = kx * kx + ky * ky;
    const T* srct[7] = {j0x, jkx, j0y, jky, jkz, Ez, Bz};
    auto arr = [&](int sl, int k) { return reinterpret_cast<cpx*>(ringd + size_t(sl) * SLOT) + k * MT + tid; };
    auto coef = [&](int sl, int k) { return ringd + size_t(sl) * SLOT + 2 * MA * MT + k * MT + tid; };
    // ring cell k: j0x, jkx, j0y, jky, jkz, R_x, R_y, E_z, B_z
    auto cell = [&](int sl, int k) -> cpx {
        if (k == 5 || k == 6) return *arr(sl, k);
        return widen(*reinterpret_cast<const T*>(arr(sl, k)));
    };
    auto fetch = [&](int n) {                  // slice n (plane n - a) into its ring slot
        const int sl = (g.b - 1 - n) % MS;
        const long o = long(n - g.a) * nk + ii;
#pragma unroll
        for (int k = 0; k < MA; ++k) {
            if (k == 5) cp_async16(arr(sl, k), Rx + o);
            else if (k == 6) cp_async16(arr(sl, k), Ry + o);
            else {
                const T* sp = srct[k < 5 ? k : k - 2] + o;
                if (sizeof(T) == 16) cp_async16(arr(sl, k), sp);
                else cp_async8(arr(sl, k), sp);
            }
        }
        cp_async8(coef(sl, 0), g.wlo + n);
        cp_async8(coef(sl, 1), g.whi + n);
        cp_async8(coef(sl, 2), g.hcg + n + 2);
    };
    // upper half-cell of the front slice: plane ns
    const long ou = long(g.ns) * nk + ii;
    cpx jxu = widen(j0x[ou]) + widen(jkx[ou]), jyu = widen(j0y[ou]) + widen(jky[ou]);
    cpx upx = widen(jkx[ou]), upy = widen(jky[ou]), upz = widen(jkz[ou]);
    cpx pRx = C(0), pRy = C(0), pEz = C(0), pBz = C(0), pLx = C(0), pLy = C(0);
#pragma unroll
    for (int q = 0; q < MS; ++q) {
        const int n = g.b - 1 - q;
        if (n >= g.a) fetch(n);
        cp_commit();                          // empty groups keep the count of groups per slice uniform
    }
    double rden = 0;                          // 1 / denominator of the slice being solved
    bool have_rden = false;
    for (int n = g.b - 1; n >= g.a; --n) {
        cp_wait<MS - 1>();                    // the group of slice n has landed (this thread's own copies)
        const int sl = (g.b - 1 - n) % MS;
        const cpx dx0 = cell(sl, 0), dxk = cell(sl, 1), dy0 = cell(sl, 2), dyk = cell(sl, 3);
        const cpx dzk = cell(sl, 4), rx = cell(sl, 5), ry = cell(sl, 6), ez = cell(sl, 7), bz = cell(sl, 8);
        const double wl = *coef(sl, 0), wu = *coef(sl, 1), h = *coef(sl, 2);
        if (!have_rden) rden = 1 / (1 + 0.25 * h * (D + 0.25 * h) * k2);
        // the next slice's inverse denominator, while this slice's chain runs
        double rden_next = 0;
        if (n > g.a) {
            cp_wait<MS - 2>();
            const double hn = *coef((sl + 1) % MS, 2);
            rden_next = 1 / (1 + 0.25 * hn * (D + 0.25 * hn) * k2);
        }
        const long o = long(n - g.a) * nk + ii;
        const cpx jxd = dx0 + dxk, jyd = dy0 + dyk;
        const cpx Jx = wl * jxd + wu * jxu;
        const cpx Jy = wl * jyd + wu * jyu;
        const cpx Rsx = rx + D * (ik(kx, ez) + ik(ky, bz)) - D * Jx;
        const cpx Rsy = ry + D * (ik(ky, ez) - ik(kx, bz)) - D * Jy;
        if (n == g.N - 1) {          // front of the window: L = E_z = B_z = 0
            if (live) {
                Rx[o] = Rsx; Ry[o] = Rsy;
                Ez[o] = narrow<T>(C(0)); Bz[o] = narrow<T>(C(0)); Lx[o] = narrow<T>(C(0)); Ly[o] = narrow<T>(C(0));
            }
            pRx = Rsx; pRy = Rsy; pEz = C(0); pBz = C(0); pLx = C(0); pLy = C(0);
        } else {
            const cpx Lsx = pLx - 0.25 * h * (ik(kx, pEz) - ik(ky, pBz)) - 0.5 * h * upx;
            const cpx Lsy = pLy - 0.25 * h * (ik(kx, pBz) + ik(ky, pEz)) - 0.5 * h * upy;
            const cpx Cp = 0.5 * (ik(kx, pRy + pLy) - ik(ky, pRx + pLx));
            const cpx Qp = -0.5 * ik(kx, pRx - pLx) + 0.5 * ik(ky, pLy - pRy);
            const cpx SB = ik(kx, Rsy) + ik(kx, Lsy) - ik(ky, Rsx) - ik(ky, Lsx);
            const cpx SE = -ik(kx, Rsx) + ik(kx, Lsx) + ik(ky, Lsy) - ik(ky, Rsy);
            const cpx Bzn = (pBz - 0.5 * h * Cp - 0.25 * h * SB) * rden;
            const cpx Ezn = (pEz - 0.5 * h * Qp - 0.25 * h * SE - h * upz) * rden;
            const cpx nRx = Rsx + D * (ik(kx, Ezn) + ik(ky, Bzn));
            const cpx nRy = Rsy + D * (ik(ky, Ezn) - ik(kx, Bzn));
            const cpx nLx = Lsx - 0.25 * h * (ik(kx, Ezn) - ik(ky, Bzn));
            const cpx nLy = Lsy - 0.25 * h * (ik(kx, Bzn) + ik(ky, Ezn));
            if (live) {
                Ez[o] = narrow<T>(Ezn); Bz[o] = narrow<T>(Bzn); Rx[o] = nRx; Ry[o] = nRy;
                Lx[o] = narrow<T>(nLx); Ly[o] = narrow<T>(nLy);
            }
            pRx = nRx; pRy = nRy; pEz = Ezn; pBz = Bzn; pLx = nLx; pLy = nLy;
        }
        rden = rden_next;
        have_rden = n > g.a;
        // the lower half-cell of this slice is the upper one of the next
        jxu = jxd; jyu = jyd; upx = dxk; upy = dyk; upz = dzk;
        // refill this slot (its values are consumed above) with the slice MS below
        const int nn = n - MS;
        if (nn >= g.a) fetch(nn);
        cp_commit();
    }
    cp_wait<0>();
}

__global__ void __launch_bounds__(128) k_comoving(Geo g, const cpx* __restrict__ jz, double* __restrict__ cpb,
                                                 cpx* __restrict__ dpb, cpx* __restrict__ Rx, cpx* __restrict__ Ry,
                                                 cpx* __restrict__ Ez, cpx* __restrict__ Bz, double beta, double gm2) {
    const long nk = g.nkh;
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nk) return;
    const int kxi = int(i % g.H), j = int(i / g.H);
    const double kx = g.kxd[kxi], ky = g.kyd[j];
    const double ev = ky * ky;                      // Fourier y: the eigenvalue of -Lap_y is k_y^2
    double cprev = 0;
    cpx dprev = C(0);
    for (int l = 0; l < g.ns; ++l) {
        const long o = long(l) * nk + i;
        const int n = g.a + l;
        const double hm = g.hcg[n + 1], hp = g.hcg[n + 2];
        const double lo = -gm2 * 2 / ((hm + hp) * hm), up = -gm2 * 2 / ((hm + hp) * hp);
        const double dg = kx * kx + ev + gm2 * 2 / (hm * hp);
        if (dg == 0) { cpb[o] = 0; dpb[o] = C(0); continue; }
        const cpx rhs = (1 / beta) * (g.wlo[n] * jz[o] + g.whi[n] * jz[o + nk]);
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
        Ez[o] = C(0); Bz[o] = C(0);
    }
}

void launch_march(Ctx& c, double D) {
    const int tok = c.prof_begin("march");
    const unsigned blocks = unsigned((c.nkh + MT - 1) / MT);
    const size_t smem = size_t(MS) * SLOT * sizeof(double);
    G3D_CUDA(cudaFuncSetAttribute(k_march<cpx>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    k_march<cpx><<<blocks, MT, smem, c.stream>>>(c.geo(), c.Rx.p, c.Ry.p, c.Ez.p, c.Bz.p, c.Lx.p, c.Ly.p, c.j0x.p, c.j0y.p,
                                              c.jkx.p, c.jky.p, c.jkz.p, D);
    c.check_launch("k_march");
    c.prof_end(tok);
}

void launch_march_f(Ctx& c, double D) {
    const int tok = c.prof_begin("march");
    const unsigned blocks = unsigned((c.nkh + MT - 1) / MT);
    const size_t smem = size_t(MS) * SLOT * sizeof(double);
    MixedBufs& m = c.mx;
    G3D_CUDA(cudaFuncSetAttribute(k_march<cpxf>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    k_march<cpxf><<<blocks, MT, smem, c.stream>>>(c.geo(), c.Rx.p, c.Ry.p, m.Ez.p, m.Bz.p, m.Lx.p, m.Ly.p, m.j0x.p, m.j0y.p,
                                               m.jkx.p, m.jky.p, m.jkz.p, D);
    c.check_launch("k_march_f");
    c.prof_end(tok);
}

void launch_comoving(Ctx& c, double beta, double gm2) {
    const int tok = c.prof_begin("comoving");
    const unsigned blocks = unsigned((c.nkh + 127) / 128);
    k_comoving<<<blocks, 128, 0, c.stream>>>(c.geo(), c.jkz.p, c.rscratch.p, c.W[3].p, c.Rx.p, c.Ry.p, c.Ez.p, c.Bz.p, beta, gm2);
    c.check_launch("k_comoving");
    c.prof_end(tok);
}

}  // namespace g3d
