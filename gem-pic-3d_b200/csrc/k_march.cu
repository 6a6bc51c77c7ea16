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
constexpr int MA = 9;       // complex arrays streamed per slice
constexpr int MC = 3;       // per-slice coefficients streamed with them: w_lo, w_hi, h
constexpr int slot_doubles(int bt) { return MA * bt + MC * bt; }   // doubles per ring slot (one value per lane)

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
}  // namespace

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
template <class Re>
__device__ __forceinline__ void cp_async_re(double* cell, const Re* src) {
    if constexpr (sizeof(Re) == 8) cp_async8(cell, src);
    else cp_async4(cell, src);
}
template <class Re>
__device__ __forceinline__ double ring_re(const double* cell) {
    if constexpr (sizeof(Re) == 8) return *cell;
    else return double(*reinterpret_cast<const float*>(cell));
}

// Two lanes per mode. With E~ = i E_z and B~ = i B_z every coefficient of the march is real (i k_x, i k_y only
// ever multiply E_z, B_z or come in pairs), so the real parts of (R, L, E~, B~) and their imaginary parts are two
// independent real recurrences: lane c = 0 carries (Re R, Re L, -Im E_z, -Im B_z), lane c = 1 carries
// (Im R, Im L, Re E_z, Re B_z); each lane makes the same products and sums as the component c of the complex
// formulas (i k z contributes +-k times the other component, an exact sign change), so nothing is rounded
// differently. The pair of a mode sits in adjacent lanes, so a warp's 8-byte loads cover 16 modes contiguously.
// Per slice each lane streams its 9 values (R_x, R_y, E_z, B_z, j0x, j0y, jkx, jky, jkz) and the slice's
// coefficients DEPTH slices ahead with per-thread cp.async into its own column of a shared-memory ring; the
// recurrence touches only registers and that ring. The denominator 1 + (h/4)(D + h/4) k_perp^2 is inverted one
// slice ahead, off the chain.
// T is the storage of E_z, B_z, L and the currents: complex128 (the FP64 form) or complex64 (the mixed form).
// R stays complex128 and the recurrence runs in FP64 in both forms: its carried values never leave the
// registers, so the mixed form only rounds what it stores, and the cancellations in curl R and div R that make
// E_z, B_z gamma^-2 small are taken in FP64.
//
// PEER (a sharded run with the ranks' slab buffers mapped into this GPU's address space, g3d_shard.cu): the lanes of
// the modes [g.m0, g.m0 + g.nkh) fetch slice n straight from the slab of the rank that holds it and store its results
// there, so the transposes before and after the march are this kernel's own loads and stores over NVLink (peer
// loads through the cp.async ring, plain peer stores) instead of an all-to-all and two copies; the pointer arguments
// are unused then.
template <class T, int BT, int DEPTH, bool PEER = false>
__global__ void __launch_bounds__(BT) k_march(Geo g, cpx* __restrict__ Rx, cpx* __restrict__ Ry, T* __restrict__ Ez,
                                             T* __restrict__ Bz, T* __restrict__ Lx, T* __restrict__ Ly,
                                             const T* __restrict__ j0x, const T* __restrict__ j0y,
                                             const T* __restrict__ jkx, const T* __restrict__ jky,
                                             const T* __restrict__ jkz, double D, SlabPeers sp = SlabPeers()) {
    typedef typename RealOf<T>::type Re;
    static_assert(!PEER || sizeof(Re) == 8, "the peer march is the FP64 form's");
    extern __shared__ double ringd[];        // DEPTH slots of [MA arrays][BT] values, then [MC][BT] coefficients
    const long nk = g.nkh;
    const int tid = threadIdx.x;
    const long gt = long(blockIdx.x) * BT + tid;
    const int c = int(gt & 1);                // component of this lane
    const long i = gt >> 1;                   // mode
    const bool live = i < nk;
    const long ii = live ? i : 0;             // idle lanes stream mode 0 and store nothing
    const int kxi = int((g.m0 + ii) % g.H), j = int((g.m0 + ii) / g.H);
    const double kx = g.kxd[kxi], ky = g.kyd[j], k2 = kx * kx + ky * ky;
    const double sgn = c ? 1.0 : -1.0;        // (i z)_c = sgn z_(1-c)
    // element offsets of the own component (R, L, j_perp) and of the other one (E_z, B_z, j_z)
    auto own = [&](long o) { return 2 * o + c; };
    auto oth = [&](long o) { return 2 * o + 1 - c; };
    const Re* j0xr = reinterpret_cast<const Re*>(j0x);
    const Re* jkxr = reinterpret_cast<const Re*>(jkx);
    const Re* j0yr = reinterpret_cast<const Re*>(j0y);
    const Re* jkyr = reinterpret_cast<const Re*>(jky);
    const Re* jkzr = reinterpret_cast<const Re*>(jkz);
    Re* Ezr = reinterpret_cast<Re*>(Ez);
    Re* Bzr = reinterpret_cast<Re*>(Bz);
    Re* Lxr = reinterpret_cast<Re*>(Lx);
    Re* Lyr = reinterpret_cast<Re*>(Ly);
    double* Rxr = reinterpret_cast<double*>(Rx);
    double* Ryr = reinterpret_cast<double*>(Ry);
    auto cell = [&](int sl, int k) { return ringd + size_t(sl) * slot_doubles(BT) + k * BT + tid; };
    auto coef = [&](int sl, int k) { return ringd + size_t(sl) * slot_doubles(BT) + MA * BT + k * BT + tid; };
    // ring cells: 0 j0x, 1 jkx, 2 j0y, 3 jky (own), 4 jkz (other), 5 R_x, 6 R_y (own), 7 E_z, 8 B_z (other)
    // PEER: the slab arrays of the rank holding slice n (R_x, R_y, E_z, B_z, L_x, L_y, j0x, j0y, jkx, jky, jkz) and the
    // element offset of this lane's mode in its plane
    auto peer = [&](int n, long& o) -> double* const* {
        int r = 0;
        while (r + 1 < sp.P && n >= sp.a[r + 1]) ++r;
        o = long(n - sp.a[r]) * sp.nkh + g.m0 + ii;
        return reinterpret_cast<double* const*>(sp.arr[r]);
    };
    auto fetch = [&](int n) {                  // slice n (plane n - a) into its ring slot
        const int sl = (g.b - 1 - n) % DEPTH;
        if constexpr (PEER) {
            long o;
            double* const* q = peer(n, o);
            cp_async8(cell(sl, 0), q[6] + own(o));
            cp_async8(cell(sl, 1), q[8] + own(o));
            cp_async8(cell(sl, 2), q[7] + own(o));
            cp_async8(cell(sl, 3), q[9] + own(o));
            cp_async8(cell(sl, 4), q[10] + oth(o));
            cp_async8(cell(sl, 5), q[0] + own(o));
            cp_async8(cell(sl, 6), q[1] + own(o));
            cp_async8(cell(sl, 7), q[2] + oth(o));
            cp_async8(cell(sl, 8), q[3] + oth(o));
        } else {
            const long o = long(n - g.a) * nk + ii;
            cp_async_re(cell(sl, 0), j0xr + own(o));
            cp_async_re(cell(sl, 1), jkxr + own(o));
            cp_async_re(cell(sl, 2), j0yr + own(o));
            cp_async_re(cell(sl, 3), jkyr + own(o));
            cp_async_re(cell(sl, 4), jkzr + oth(o));
            cp_async8(cell(sl, 5), Rxr + own(o));
            cp_async8(cell(sl, 6), Ryr + own(o));
            cp_async_re(cell(sl, 7), Ezr + oth(o));
            cp_async_re(cell(sl, 8), Bzr + oth(o));
        }
        cp_async8(coef(sl, 0), g.wlo + n);
        cp_async8(coef(sl, 1), g.whi + n);
        cp_async8(coef(sl, 2), g.hcg + n + 2);
    };
    // upper half-cell of the front slice: plane ns (PEER: the top rank's last half-cell plane)
    const Re* uj0x = j0xr; const Re* ujkx = jkxr; const Re* uj0y = j0yr; const Re* ujky = jkyr; const Re* ujkz = jkzr;
    long ou = long(g.ns) * nk + ii;
    if constexpr (PEER) {
        const int r = sp.P - 1;
        ou = long(sp.ns[r]) * sp.nkh + g.m0 + ii;
        uj0x = static_cast<const Re*>(sp.arr[r][6]); uj0y = static_cast<const Re*>(sp.arr[r][7]);
        ujkx = static_cast<const Re*>(sp.arr[r][8]); ujky = static_cast<const Re*>(sp.arr[r][9]);
        ujkz = static_cast<const Re*>(sp.arr[r][10]);
    }
    double jxu = double(uj0x[own(ou)]) + double(ujkx[own(ou)]), jyu = double(uj0y[own(ou)]) + double(ujky[own(ou)]);
    double upx = ujkx[own(ou)], upy = ujky[own(ou)], upz = sgn * double(ujkz[oth(ou)]);
    double pRx = 0, pRy = 0, pE = 0, pB = 0, pLx = 0, pLy = 0;    // level s1 of the slice above: R, E~, B~, L
#pragma unroll
    for (int q = 0; q < DEPTH; ++q) {
        const int n = g.b - 1 - q;
        if (n >= g.a) fetch(n);
        cp_commit();                          // empty groups keep the count of groups per slice uniform
    }
    double rden = 0;                          // 1 / denominator of the slice being solved
    bool have_rden = false;
    for (int n = g.b - 1; n >= g.a; --n) {
        cp_wait<DEPTH - 1>();                 // the group of slice n has landed (this lane's own copies)
        const int sl = (g.b - 1 - n) % DEPTH;
        const double dx0 = ring_re<Re>(cell(sl, 0)), dxk = ring_re<Re>(cell(sl, 1));
        const double dy0 = ring_re<Re>(cell(sl, 2)), dyk = ring_re<Re>(cell(sl, 3));
        const double dzk = sgn * ring_re<Re>(cell(sl, 4));
        const double rx = *cell(sl, 5), ry = *cell(sl, 6);
        const double e = sgn * ring_re<Re>(cell(sl, 7)), b = sgn * ring_re<Re>(cell(sl, 8));
        const double wl = *coef(sl, 0), wu = *coef(sl, 1), h = *coef(sl, 2);
        if (!have_rden) rden = 1 / (1 + 0.25 * h * (D + 0.25 * h) * k2);
        // the next slice's inverse denominator, while this slice's chain runs
        double rden_next = 0;
        if (n > g.a) {
            cp_wait<DEPTH - 2>();
            const double hn = *coef((sl + 1) % DEPTH, 2);
            rden_next = 1 / (1 + 0.25 * hn * (D + 0.25 * hn) * k2);
        }
        long o = long(n - g.a) * nk + ii;
        Re* sEz = Ezr; Re* sBz = Bzr; Re* sLx = Lxr; Re* sLy = Lyr;
        double* sRx = Rxr; double* sRy = Ryr;
        if constexpr (PEER) {                  // the results go to the slab of the rank holding slice n
            double* const* q = peer(n, o);
            sRx = q[0]; sRy = q[1]; sEz = q[2]; sBz = q[3]; sLx = q[4]; sLy = q[5];
        }
        const double jxd = dx0 + dxk, jyd = dy0 + dyk;
        const double Jx = wl * jxd + wu * jxu;
        const double Jy = wl * jyd + wu * jyu;
        const double Rsx = rx + D * (kx * e + ky * b) - D * Jx;
        const double Rsy = ry + D * (ky * e - kx * b) - D * Jy;
        if (n == g.N - 1) {          // front of the window: L = E_z = B_z = 0
            if (live) {
                sRx[own(o)] = Rsx; sRy[own(o)] = Rsy;
                sEz[oth(o)] = Re(0); sBz[oth(o)] = Re(0); sLx[own(o)] = Re(0); sLy[own(o)] = Re(0);
            }
            pRx = Rsx; pRy = Rsy; pE = 0; pB = 0; pLx = 0; pLy = 0;
        } else {
            const double Lsx = pLx - 0.25 * h * (kx * pE - ky * pB) - 0.5 * h * upx;
            const double Lsy = pLy - 0.25 * h * (kx * pB + ky * pE) - 0.5 * h * upy;
            const double iCp = 0.5 * ((-kx * (pRy + pLy)) - (-ky * (pRx + pLx)));        // (i C_p)_c
            const double iQp = -0.5 * (-kx * (pRx - pLx)) + 0.5 * (-ky * (pLy - pRy));    // (i Q_p)_c
            const double iSB = (-kx * Rsy) + (-kx * Lsy) - (-ky * Rsx) - (-ky * Lsx);     // (i S_B)_c
            const double iSE = (kx * Rsx) + (-kx * Lsx) + (-ky * Lsy) - (-ky * Rsy);      // (i S_E)_c
            const double Bn = (pB - 0.5 * h * iCp - 0.25 * h * iSB) * rden;                // (i B_z)_c
            const double En = (pE - 0.5 * h * iQp - 0.25 * h * iSE - h * upz) * rden;      // (i E_z)_c
            const double nRx = Rsx + D * (kx * En + ky * Bn);
            const double nRy = Rsy + D * (ky * En - kx * Bn);
            const double nLx = Lsx - 0.25 * h * (kx * En - ky * Bn);
            const double nLy = Lsy - 0.25 * h * (kx * Bn + ky * En);
            if (live) {
                sEz[oth(o)] = Re(sgn * En); sBz[oth(o)] = Re(sgn * Bn); sRx[own(o)] = nRx; sRy[own(o)] = nRy;
                sLx[own(o)] = Re(nLx); sLy[own(o)] = Re(nLy);
            }
            pRx = nRx; pRy = nRy; pE = En; pB = Bn; pLx = nLx; pLy = nLy;
        }
        rden = rden_next;
        have_rden = n > g.a;
        // the lower half-cell of this slice is the upper one of the next
        jxu = jxd; jyu = jyd; upx = dxk; upy = dyk; upz = dzk;
        // refill this slot (its values are consumed above) with the slice DEPTH below
        const int nn = n - DEPTH;
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
    const int kxi = int((g.m0 + i) % g.H), j = int((g.m0 + i) / g.H);
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

// Block size and ring depth: 32 lanes per block when blocks of 64 would give fewer than two per SM (the
// 128 x 128 grid has 8,320 half-spectrum modes, 16,640 lanes), else 64. The mixed form streams 44 bytes per lane
// and slice instead of 72, so it keeps more slices in flight for the same bytes.
template <class T, int BT, int DEPTH>
static void march_launch(Ctx& c, const Geo& g, cpx* Rx, cpx* Ry, T* Ez, T* Bz, T* Lx, T* Ly, const T* j0x, const T* j0y,
                         const T* jkx, const T* jky, const T* jkz, double D) {
    const unsigned blocks = unsigned((2 * g.nkh + BT - 1) / BT);
    if (blocks == 0) return;
    const size_t smem = size_t(DEPTH) * slot_doubles(BT) * sizeof(double);
    smem_attr(reinterpret_cast<const void*>(k_march<T, BT, DEPTH>), smem);
    k_march<T, BT, DEPTH><<<blocks, BT, smem, c.stream>>>(g, Rx, Ry, Ez, Bz, Lx, Ly, j0x, j0y, jkx, jky, jkz, D);
}
template <class T, int DEPTH>
static void march_any(Ctx& c, const Geo& g, cpx* Rx, cpx* Ry, T* Ez, T* Bz, T* Lx, T* Ly, const T* j0x, const T* j0y,
                      const T* jkx, const T* jky, const T* jkz, double D) {
    if (2 * g.nkh < 2L * 148 * 64) march_launch<T, 32, DEPTH>(c, g, Rx, Ry, Ez, Bz, Lx, Ly, j0x, j0y, jkx, jky, jkz, D);
    else march_launch<T, 64, DEPTH>(c, g, Rx, Ry, Ez, Bz, Lx, Ly, j0x, j0y, jkx, jky, jkz, D);
}

void launch_march(Ctx& c, double D) {
    const int tok = c.prof_begin("march");
    march_any<cpx, 6>(c, c.geo(), c.Rx.p, c.Ry.p, c.Ez.p, c.Bz.p, c.Lx.p, c.Ly.p, c.j0x.p, c.j0y.p, c.jkx.p, c.jky.p, c.jkz.p, D);
    c.check_launch("k_march");
    c.prof_end(tok);
}
// the march of a mode pencil (a sharded run): all N slices of the modes [g.m0, g.m0 + g.nkh), arrays in the order
// R_x, R_y, E_z, B_z, L_x, L_y, j0x, j0y, jkx, jky, jkz
void launch_march_pencil(Ctx& c, const Geo& g, cpx* const* p, double D) {
    const int tok = c.prof_begin("march");
    march_any<cpx, 6>(c, g, p[0], p[1], p[2], p[3], p[4], p[5], p[6], p[7], p[8], p[9], p[10], D);
    c.check_launch("k_march");
    c.prof_end(tok);
}

// the fused transpose and march of a sharded run: the modes of this rank's pencil, every slice read from and written to
// the slab of the rank that holds it (sp: the slabs' mapped buffers)
void launch_march_peer(Ctx& c, const Geo& g, const SlabPeers& sp, double D) {
    const int tok = c.prof_begin("march_peer");
    if (2 * g.nkh < 2L * 148 * 64) {
        const unsigned blocks = unsigned((2 * g.nkh + 31) / 32);
        const size_t smem = size_t(6) * slot_doubles(32) * sizeof(double);
        smem_attr(reinterpret_cast<const void*>(k_march<cpx, 32, 6, true>), smem);
        if (blocks) k_march<cpx, 32, 6, true><<<blocks, 32, smem, c.stream>>>(g, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, D, sp);
    } else {
        const unsigned blocks = unsigned((2 * g.nkh + 63) / 64);
        const size_t smem = size_t(6) * slot_doubles(64) * sizeof(double);
        smem_attr(reinterpret_cast<const void*>(k_march<cpx, 64, 6, true>), smem);
        k_march<cpx, 64, 6, true><<<blocks, 64, smem, c.stream>>>(g, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, D, sp);
    }
    c.check_launch("k_march_peer");
    c.prof_end(tok);
}

void launch_march_f(Ctx& c, double D) {
    const int tok = c.prof_begin("march");
    MixedBufs& m = c.mx;
    march_any<cpxf, 10>(c, c.geo(), c.Rx.p, c.Ry.p, m.Ez.p, m.Bz.p, m.Lx.p, m.Ly.p, m.j0x.p, m.j0y.p, m.jkx.p, m.jky.p, m.jkz.p, D);
    c.check_launch("k_march_f");
    c.prof_end(tok);
}

static void comoving_launch(Ctx& c, const Geo& g, const cpx* jz, double* cpb, cpx* dpb, cpx* Rx, cpx* Ry, cpx* Ez, cpx* Bz,
                            double beta, double gm2) {
    const int tok = c.prof_begin("comoving");
    const unsigned blocks = unsigned((g.nkh + 127) / 128);
    if (blocks) k_comoving<<<blocks, 128, 0, c.stream>>>(g, jz, cpb, dpb, Rx, Ry, Ez, Bz, beta, gm2);
    c.check_launch("k_comoving");
    c.prof_end(tok);
}
void launch_comoving(Ctx& c, double beta, double gm2) {
    comoving_launch(c, c.geo(), c.jkz.p, c.rscratch.p, c.W[3].p, c.Rx.p, c.Ry.p, c.Ez.p, c.Bz.p, beta, gm2);
}
// the co-moving solve of a mode pencil: j_z (N + 1 half cells) in, R_x, R_y, E_z, B_z (N slices) out
void launch_comoving_pencil(Ctx& c, const Geo& g, const cpx* jz, double* cpb, cpx* dpb, cpx* const* out, double beta,
                            double gm2) {
    comoving_launch(c, g, jz, cpb, dpb, out[0], out[1], out[2], out[3], beta, gm2);
}

}  // namespace g3d
