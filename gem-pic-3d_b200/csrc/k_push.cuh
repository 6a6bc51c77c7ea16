// Device functions of the beam push shared by the push (k_push.cu) and its adjoint (k_adjoint.cu), so that the
// adjoint recomputes the forward trajectory with the same arithmetic: the gather of the grid fields (TSC in x
// and y, linear in zeta; reference gather, src/sim_kernels.hpp:44-72) and the right-hand side of the
// characteristics (rhs, sim_kernels.hpp:75-92). FT is the element type of the real-space fields: float (the
// reference's F) or double (the exact fields of the gradient check).
#pragma once
#include "g3d_plasma.hpp"
#include "k_external.cuh"

namespace g3d {

struct PushArgs {
    const float* __restrict__ F;
    const double* __restrict__ Fd;        // exact fields (FP64 copy of F) or null
    Geo g;
    LaserDev laser;
    double X0, Y0, zc, dz_push, push_phase, zhand, zmax, ylo, yhi, s1, vz_min, hmin;
    int freeze, self;
    ExtDev ext;                           // external magnetic elements (none: nu = nm = 0)
};

struct St { double x, y, zeta, px, py, pz; };

PushArgs push_args(Ctx& c, double s1);          // the arguments of the push to the plane s1 (k_push.cu)

template <class FT>
__device__ __forceinline__ void gather(const PushArgs& c, const FT* __restrict__ Fp, double x, double y, double zeta, double E[3],
                                       double B[3]) {
    E[0] = E[1] = E[2] = B[0] = B[1] = B[2] = 0;
    if (!c.self) return;
    const Geo& g = c.g;
    int n; double fz;
    g.zax.locate(zeta, n, fz);
    if (n == g.a - 1 && fz > 1 - 1e-9) { n = g.a; fz = 0; }    // on the lowest slice (rounding of locate)
    const int fl = n - g.a;
    if (fl < 0 || fl > g.ns) return;
    int ix[3], jn[3]; double wx[3], wn[3];
    tsc_periodic(x, g.dx, g.nx, ix, wx);
    const long nk = g.nk;
    if (!g.yf) {                       // free-hand y: E_y, B_x, B_z on the half-nodes, nothing beyond the walls
        int jh[3]; double wh[3];
        tsc_y(g.yax, y, jn, wn, jh, wh);
        for (int comp = 0; comp < 6; ++comp) {
            const FT* p0 = Fp + (long(comp) * (g.ns + 2) + fl) * nk;
            const FT* p1 = p0 + nk;
            const bool hf = is_half(comp);
            const int* jj = hf ? jh : jn;
            const double* wy = hf ? wh : wn;
            double v = 0;
            for (int j = 0; j < 3; ++j) {
                if (jj[j] < 0 || jj[j] >= g.ny) continue;
                for (int i = 0; i < 3; ++i) {
                    const long k = long(jj[j]) * g.nx + ix[i];
                    v += wx[i] * wy[j] * ((1 - fz) * double(__ldg(p0 + k)) + fz * double(__ldg(p1 + k)));
                }
            }
            if (comp < 3) E[comp] = v; else B[comp - 3] = v;
        }
        return;
    }
    tsc_periodic(y, g.dy, g.ny, jn, wn);
#pragma unroll
    for (int comp = 0; comp < 6; ++comp) {
        const FT* p0 = Fp + (long(comp) * (g.ns + 2) + fl) * nk;
        const FT* p1 = p0 + nk;
        double v = 0;
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                const long k = long(jn[j]) * g.nx + ix[i];
                v += wx[i] * wn[j] * ((1 - fz) * double(__ldg(p0 + k)) + fz * double(__ldg(p1 + k)));
            }
        if (comp < 3) E[comp] = v; else B[comp - 3] = v;
    }
}

template <class FT>
__device__ __forceinline__ bool rhs(const PushArgs& c, const FT* __restrict__ Fp, const St& Y, double z, double qm, St& d) {
    const double g = sqrt(1 + Y.px * Y.px + Y.py * Y.py + Y.pz * Y.pz);
    if (Y.pz < 0.3 * g) return false;
    const double gm = (1 + Y.px * Y.px + Y.py * Y.py) / (g + Y.pz);
    double E[3], B[3], Ee[3], Be[3];
    gather(c, Fp, wrap_periodic(Y.x, c.g.Lx), c.g.yf ? wrap_periodic(Y.y, c.g.Ly) : Y.y, Y.zeta, E, B);
    c.laser.field(Y.x + c.X0, z, z - (Y.zeta - c.zc), Ee, Be);
#pragma unroll
    for (int k = 0; k < 3; ++k) { E[k] += Ee[k]; B[k] += Be[k]; }
    if (c.ext.any()) add_external(c.ext, Y.x + c.X0, Y.y + c.Y0, z, B);
    const double ip = 1 / Y.pz;
    d.x = Y.px * ip; d.y = Y.py * ip; d.zeta = -gm * ip;
    d.px = qm * (g * E[0] + Y.py * B[2] - Y.pz * B[1]) * ip;
    d.py = qm * (g * E[1] + Y.pz * B[0] - Y.px * B[2]) * ip;
    d.pz = qm * (g * E[2] + Y.px * B[1] - Y.py * B[0]) * ip;
    return true;
}
// The next sub-step from z towards s1: at most dz_push, at most push_phase of the laser phase, and a zeta
// advance of at most hmin/2 (reference push_one, src/sim_kernels.hpp:110-125)
__device__ __forceinline__ double substep(const PushArgs& c, const St& Y, double z, double s1) {
    double ds = c.dz_push < s1 - z ? c.dz_push : s1 - z;
    {
        const double g = sqrt(1 + Y.px * Y.px + Y.py * Y.py + Y.pz * Y.pz);
        const double lz = 0.5 * c.hmin * Y.pz * (g + Y.pz) / (1 + Y.px * Y.px + Y.py * Y.py);
        if (lz < ds) ds = (s1 - z) / ceil((s1 - z) / lz);
    }
    if (c.laser.on) {
        const double g = sqrt(1 + Y.px * Y.px + Y.py * Y.py + Y.pz * Y.pz);
        const double hl = g - Y.px * c.laser.kx - Y.pz * c.laser.kz;
        const double lim = c.push_phase * Y.pz / (c.laser.kL * (hl > 1e-12 ? hl : 1e-12));
        if (lim < ds) ds = (s1 - z) / ceil((s1 - z) / lim);
    }
    if (c.ext.any()) ds = external_step(c.ext, z, ds);       // the external elements resolved
    return ds;
}
__device__ __forceinline__ St axpy(const St& a, double h, const St& b) {
    return St{a.x + h * b.x, a.y + h * b.y, a.zeta + h * b.zeta, a.px + h * b.px, a.py + h * b.py, a.pz + h * b.pz};
}

// One RK4 sub-step of length ds from z (reference push_one, src/sim_kernels.hpp:126-143); k1 + 2 k2 + 2 k3 + k4
// summed left to right as each stage completes (fewer live registers). False: the particle is too slow
// (rhs), and Y is left unchanged.
template <class FT>
__device__ __forceinline__ bool rk4_step(const PushArgs& c, const FT* __restrict__ Fp, St& Y, double z, double ds, double qm) {
    St k, acc;
    // with external elements the first and last stages take the field just inside the sub-step, which ends on the
    // elements' breakpoints, where the field or its derivative jumps
    const double e = c.ext.any() ? 1e-9 * ds : 0.0;
    bool ok = rhs(c, Fp, Y, z + e, qm, k);
    acc = k;
    ok = ok && rhs(c, Fp, axpy(Y, 0.5 * ds, k), z + 0.5 * ds, qm, k);
    acc = axpy(acc, 2.0, k);
    ok = ok && rhs(c, Fp, axpy(Y, 0.5 * ds, k), z + 0.5 * ds, qm, k);
    acc = axpy(acc, 2.0, k);
    ok = ok && rhs(c, Fp, axpy(Y, ds, k), z + ds - e, qm, k);
    if (!ok) return false;
    acc = axpy(acc, 1.0, k);
    const double w = ds / 6;
    Y.x += w * acc.x; Y.y += w * acc.y; Y.zeta += w * acc.zeta;
    Y.px += w * acc.px; Y.py += w * acc.py; Y.pz += w * acc.pz;
    return true;
}

}  // namespace g3d
