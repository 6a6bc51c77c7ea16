// The per-mode march over the slices (Fourier y) and the co-moving start field.
//
// k_march: Simulation::march / march_point of the reference (src/sim_fields.cpp:7-39,
// src/sim_kernels.hpp:169-210). Every mode (k_x, k_y) is an independent recurrence from the front slice
// b-1 down to a: R by the trapezoidal rule in s, L, E_z, B_z by the trapezoidal rule over the half-cell
// of length h_n, B_z and E_z in closed form with the denominator 1 + (h/4)(D + h/4) k_perp^2, the current
// of slice n interpolated as w_lo (j0 + jk)_{n-1/2} + w_hi (j0 + jk)_{n+1/2}. One thread per mode keeps
// the values of slice n+1 (level s1) and of the upper half-cell in registers, so each slice costs 9 loads
// (R_x, R_y, E_z, B_z of level s0 and the five current spectra of the lower half-cell) and 6 stores.
//
// k_comoving: Simulation::comoving_field for Fourier y (src/sim_fields.cpp:44-151): per mode the
// tridiagonal system of -(k_perp^2 + gamma^-2 d_zeta^2) psi = rho along zeta (Thomas), then
// R = -(1 + beta) i k psi, E_z = B_z = 0.
#include "g3d_ctx.hpp"

namespace g3d {

__global__ void __launch_bounds__(128) k_march(Geo g, cpx* __restrict__ Rx, cpx* __restrict__ Ry, cpx* __restrict__ Ez,
                                              cpx* __restrict__ Bz, cpx* __restrict__ Lx, cpx* __restrict__ Ly,
                                              const cpx* __restrict__ j0x, const cpx* __restrict__ j0y,
                                              const cpx* __restrict__ jkx, const cpx* __restrict__ jky,
                                              const cpx* __restrict__ jkz, double D) {
    const long nk = g.nk;
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nk) return;
    const int ixx = int(i % g.nx), j = int(i / g.nx);
    const double kx = g.kxd[ixx], ky = g.kyd[j], k2 = kx * kx + ky * ky;
    // upper half-cell of the front slice: plane ns
    long ou = long(g.ns) * nk + i;
    cpx jxu = j0x[ou] + jkx[ou], jyu = j0y[ou] + jky[ou];
    cpx upx = jkx[ou], upy = jky[ou], upz = jkz[ou];
    cpx pRx = C(0), pRy = C(0), pEz = C(0), pBz = C(0), pLx = C(0), pLy = C(0);
    // prefetched inputs of the slice being solved
    int n = g.b - 1;
    long o = long(n - g.a) * nk + i;
    cpx dx0 = j0x[o], dxk = jkx[o], dy0 = j0y[o], dyk = jky[o], dzk = jkz[o];
    cpx rx = Rx[o], ry = Ry[o], ez = Ez[o], bz = Bz[o];
    for (; n >= g.a; --n) {
        // next slice's inputs first (independent of this slice's result)
        const long on = o - nk;
        cpx ndx0, ndxk, ndy0, ndyk, ndzk, nrx, nry, nez, nbz;
        if (n > g.a) {
            ndx0 = j0x[on]; ndxk = jkx[on]; ndy0 = j0y[on]; ndyk = jky[on]; ndzk = jkz[on];
            nrx = Rx[on]; nry = Ry[on]; nez = Ez[on]; nbz = Bz[on];
        }
        const double wl = g.wlo[n], wu = g.whi[n];
        const cpx jxd = dx0 + dxk, jyd = dy0 + dyk;
        const cpx Jx = wl * jxd + wu * jxu;
        const cpx Jy = wl * jyd + wu * jyu;
        const cpx Rsx = rx + D * (ik(kx, ez) + ik(ky, bz)) - D * Jx;
        const cpx Rsy = ry + D * (ik(ky, ez) - ik(kx, bz)) - D * Jy;
        if (n == g.N - 1) {          // front of the window: L = E_z = B_z = 0
            Rx[o] = Rsx; Ry[o] = Rsy;
            Ez[o] = C(0); Bz[o] = C(0); Lx[o] = C(0); Ly[o] = C(0);
            pRx = Rsx; pRy = Rsy; pEz = C(0); pBz = C(0); pLx = C(0); pLy = C(0);
        } else {
            const double h = g.hcg[n + 2];
            const cpx Lsx = pLx - 0.25 * h * (ik(kx, pEz) - ik(ky, pBz)) - 0.5 * h * upx;
            const cpx Lsy = pLy - 0.25 * h * (ik(kx, pBz) + ik(ky, pEz)) - 0.5 * h * upy;
            const cpx Cp = 0.5 * (ik(kx, pRy + pLy) - ik(ky, pRx + pLx));
            const cpx Qp = -0.5 * ik(kx, pRx - pLx) + 0.5 * ik(ky, pLy - pRy);
            const cpx SB = ik(kx, Rsy) + ik(kx, Lsy) - ik(ky, Rsx) - ik(ky, Lsx);
            const cpx SE = -ik(kx, Rsx) + ik(kx, Lsx) + ik(ky, Lsy) - ik(ky, Rsy);
            const double den = 1 + 0.25 * h * (D + 0.25 * h) * k2;
            const cpx Bzn = (pBz - 0.5 * h * Cp - 0.25 * h * SB) / den;
            const cpx Ezn = (pEz - 0.5 * h * Qp - 0.25 * h * SE - h * upz) / den;
            const cpx nRx = Rsx + D * (ik(kx, Ezn) + ik(ky, Bzn));
            const cpx nRy = Rsy + D * (ik(ky, Ezn) - ik(kx, Bzn));
            const cpx nLx = Lsx - 0.25 * h * (ik(kx, Ezn) - ik(ky, Bzn));
            const cpx nLy = Lsy - 0.25 * h * (ik(kx, Bzn) + ik(ky, Ezn));
            Ez[o] = Ezn; Bz[o] = Bzn; Rx[o] = nRx; Ry[o] = nRy; Lx[o] = nLx; Ly[o] = nLy;
            pRx = nRx; pRy = nRy; pEz = Ezn; pBz = Bzn; pLx = nLx; pLy = nLy;
        }
        // the lower half-cell of this slice is the upper one of the next
        jxu = jxd; jyu = jyd; upx = dxk; upy = dyk; upz = dzk;
        dx0 = ndx0; dxk = ndxk; dy0 = ndy0; dyk = ndyk; dzk = ndzk;
        rx = nrx; ry = nry; ez = nez; bz = nbz;
        o = on;
    }
}

__global__ void __launch_bounds__(128) k_comoving(Geo g, const cpx* __restrict__ jz, double* __restrict__ cpb,
                                                 cpx* __restrict__ dpb, cpx* __restrict__ Rx, cpx* __restrict__ Ry,
                                                 cpx* __restrict__ Ez, cpx* __restrict__ Bz, double beta, double gm2) {
    const long nk = g.nk;
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nk) return;
    const int ixx = int(i % g.nx), j = int(i / g.nx);
    const double kx = g.kxd[ixx], ky = g.kyd[j];
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
    const unsigned blocks = unsigned((c.nk + 127) / 128);
    k_march<<<blocks, 128, 0, c.stream>>>(c.geo(), c.Rx.p, c.Ry.p, c.Ez.p, c.Bz.p, c.Lx.p, c.Ly.p, c.j0x.p, c.j0y.p, c.jkx.p,
                                          c.jky.p, c.jkz.p, D);
    c.check_launch("k_march");
    c.prof_end(tok);
}

void launch_comoving(Ctx& c, double beta, double gm2) {
    const int tok = c.prof_begin("comoving");
    const unsigned blocks = unsigned((c.nk + 127) / 128);
    k_comoving<<<blocks, 128, 0, c.stream>>>(c.geo(), c.jkz.p, c.rscratch.p, c.S2.p, c.Rx.p, c.Ry.p, c.Ez.p, c.Bz.p, beta, gm2);
    c.check_launch("k_comoving");
    c.prof_end(tok);
}

}  // namespace g3d
