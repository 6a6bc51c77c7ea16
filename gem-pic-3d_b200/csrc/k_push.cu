// Push of the beam list to the next plane s1 (Simulation::push, src/sim_particles.cpp:6-24): characteristics
// with z as the independent variable, dr/dz = p/p_z, dzeta/dz = -(gamma - p_z)/p_z, dp/dz = q (gamma E + p x B)/p_z,
// integrated by RK4 (src/sim_kernels.hpp:73-149). The fields are the grid fields of level s0 (float F, TSC in x
// and y, linear in zeta between the slices; gather, sim_kernels.hpp:44-72) plus the analytic plane wave.
// A sub-step is at most dz_push, at most push_phase of the laser phase and moves the particle by at most
// hmin/2 in zeta. One thread per particle, FP64 arithmetic on the float field data.
#include "g3d_plasma.hpp"

namespace g3d {

struct PushArgs {
    const float* __restrict__ F;
    Geo g;
    LaserDev laser;
    double X0, Y0, zc, dz_push, push_phase, zhand, zmax, ylo, yhi, s1, vz_min, hmin;
    int freeze, self;
};

struct St { double x, y, zeta, px, py, pz; };

__device__ __forceinline__ void gather(const PushArgs& c, double x, double y, double zeta, double E[3], double B[3]) {
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
            const float* p0 = c.F + (long(comp) * (g.ns + 2) + fl) * nk;
            const float* p1 = p0 + nk;
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
        const float* p0 = c.F + (long(comp) * (g.ns + 2) + fl) * nk;
        const float* p1 = p0 + nk;
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

__device__ __forceinline__ bool rhs(const PushArgs& c, const St& Y, double z, double qm, St& d) {
    const double g = sqrt(1 + Y.px * Y.px + Y.py * Y.py + Y.pz * Y.pz);
    if (Y.pz < 0.3 * g) return false;
    const double gm = (1 + Y.px * Y.px + Y.py * Y.py) / (g + Y.pz);
    double E[3], B[3], Ee[3], Be[3];
    gather(c, wrap_periodic(Y.x, c.g.Lx), c.g.yf ? wrap_periodic(Y.y, c.g.Ly) : Y.y, Y.zeta, E, B);
    c.laser.field(Y.x + c.X0, z, z - (Y.zeta - c.zc), Ee, Be);
#pragma unroll
    for (int k = 0; k < 3; ++k) { E[k] += Ee[k]; B[k] += Be[k]; }
    const double ip = 1 / Y.pz;
    d.x = Y.px * ip; d.y = Y.py * ip; d.zeta = -gm * ip;
    d.px = qm * (g * E[0] + Y.py * B[2] - Y.pz * B[1]) * ip;
    d.py = qm * (g * E[1] + Y.pz * B[0] - Y.px * B[2]) * ip;
    d.pz = qm * (g * E[2] + Y.px * B[1] - Y.py * B[0]) * ip;
    return true;
}
__device__ __forceinline__ St axpy(const St& a, double h, const St& b) {
    return St{a.x + h * b.x, a.y + h * b.y, a.zeta + h * b.zeta, a.px + h * b.px, a.py + h * b.py, a.pz + h * b.pz};
}

// RK4 from z0 to the plane s1 (reference push_one, src/sim_kernels.hpp:98-149).
__global__ void __launch_bounds__(128, 4) k_push(PushArgs c, PartsDev P, const int32_t* __restrict__ perm, long np, double s0) {
    const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const long ip = perm[t];                 // cell order: the warp's particles gather the same planes of F
    const int alive = P.alive[ip];
    if (alive != 1 && alive != 3) return;
    const double s1 = c.s1;
    if (c.freeze && P.sp[ip] <= 0) { P.z[ip] = s1; return; }       // numerics.freeze_bunch: rigid bunch
    St Y{P.x[ip], P.y[ip], P.zeta[ip], P.px[ip], P.py[ip], P.pz[ip]};
    const double qm = P.qm[ip];
    double z = alive == 1 ? s0 : s1 - P.rem[ip];
    while (z < s1 - 1e-12 * fabs(s1)) {
        if (Y.zeta < c.zhand) {          // handed to the rank below with the rest of the step
            P.x[ip] = Y.x; P.y[ip] = Y.y; P.zeta[ip] = Y.zeta; P.px[ip] = Y.px; P.py[ip] = Y.py; P.pz[ip] = Y.pz;
            P.alive[ip] = 2; P.rem[ip] = s1 - z;
            return;
        }
        if (c.vz_min > 0 && Y.pz < c.vz_min * sqrt(1 + Y.px * Y.px + Y.py * Y.py + Y.pz * Y.pz)) {
            // too slow for the beam list: streams in the current march from (z, zeta)
            P.x[ip] = Y.x; P.y[ip] = Y.y; P.zeta[ip] = Y.zeta; P.px[ip] = Y.px; P.py[ip] = Y.py; P.pz[ip] = Y.pz;
            P.z[ip] = z; P.alive[ip] = 4;
            return;
        }
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
        // k1 + 2 k2 + 2 k3 + k4 summed left to right as each stage completes (fewer live registers)
        St k, acc;
        bool ok = rhs(c, Y, z, qm, k);
        acc = k;
        ok = ok && rhs(c, axpy(Y, 0.5 * ds, k), z + 0.5 * ds, qm, k);
        acc = axpy(acc, 2.0, k);
        ok = ok && rhs(c, axpy(Y, 0.5 * ds, k), z + 0.5 * ds, qm, k);
        acc = axpy(acc, 2.0, k);
        ok = ok && rhs(c, axpy(Y, ds, k), z + ds, qm, k);
        if (!ok) {
            P.alive[ip] = 0;
            return;
        }
        acc = axpy(acc, 1.0, k);
        const double w = ds / 6;
        Y.x += w * acc.x; Y.y += w * acc.y; Y.zeta += w * acc.zeta;
        Y.px += w * acc.px; Y.py += w * acc.py; Y.pz += w * acc.pz;
        z += ds;
    }
    P.x[ip] = Y.x; P.y[ip] = Y.y; P.zeta[ip] = Y.zeta; P.px[ip] = Y.px; P.py[ip] = Y.py; P.pz[ip] = Y.pz; P.z[ip] = s1;
    // lost: out of the window in zeta, or within one cell of a wall in y
    int al = (Y.zeta < 0 || Y.zeta >= c.zmax || Y.y < c.ylo || Y.y > c.yhi) ? 0 : 1;
    if (al == 1 && Y.zeta < c.zhand) { al = 2; P.rem[ip] = 0; }
    P.alive[ip] = al;
}

void launch_push(Ctx& c, double s0, double s1) {
    if (c.np == 0) return;
    PushArgs a;
    a.F = c.F.p; a.g = c.geo(); a.laser = c.laser;
    a.X0 = c.X0; a.Y0 = c.Y0; a.zc = c.P.zeta_center; a.dz_push = c.P.dz_push; a.push_phase = c.P.push_phase;
    a.zhand = -1e300;                                   // one rank: nothing is handed over
    a.zmax = c.zeta[c.N - 1]; a.s1 = s1; a.hmin = c.hmin;
    a.ylo = c.yf ? -1e300 : c.ynode_h[1];              // free-hand y: lost within one cell of a wall
    a.yhi = c.yf ? 1e300 : c.ynode_h[size_t(c.ny) - 1];
    a.vz_min = c.pl ? c.pl->cfg.vz_min : 0;            // slower beam particles stream in the plasma march
    a.freeze = c.P.freeze_bunch; a.self = c.P.self_fields;
    const int tok = c.prof_begin("push");
    k_push<<<unsigned((c.np + 127) / 128), 128, 0, c.stream>>>(a, c.parts, c.perm.p, c.np, s0);
    c.check_launch("k_push");
    c.prof_end(tok);
}

}  // namespace g3d
