// Push of the beam list to the next plane s1 (Simulation::push, src/sim_particles.cpp:6-24): characteristics
// with z as the independent variable, dr/dz = p/p_z, dzeta/dz = -(gamma - p_z)/p_z, dp/dz = q (gamma E + p x B)/p_z,
// integrated by RK4 (src/sim_kernels.hpp:73-149). The fields are the grid fields of level s0 (float F, TSC in x
// and y, linear in zeta between the slices; gather, sim_kernels.hpp:44-72) plus the analytic plane wave.
// A sub-step is at most dz_push, at most push_phase of the laser phase and moves the particle by at most
// hmin/2 in zeta. One thread per particle, FP64 arithmetic on the float field data.
#include "k_push.cuh"

namespace g3d {

// RK4 from z0 to the plane s1 (reference push_one, src/sim_kernels.hpp:98-149).
// perm: the particles in cell order, or null for the particles [i0, i0 + np) in storage order
template <class FT>
__global__ void __launch_bounds__(128, 4) k_push(PushArgs c, const FT* __restrict__ Fp, PartsDev P, const int32_t* __restrict__ perm,
                                                long i0, long np, double s0) {
    const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const long ip = perm ? perm[t] : i0 + t;     // cell order: the warp's particles gather the same planes of F
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
        const double ds = substep(c, Y, z, s1);
        if (!rk4_step(c, Fp, Y, z, ds, qm)) {
            P.alive[ip] = 0;
            return;
        }
        z += ds;
    }
    P.x[ip] = Y.x; P.y[ip] = Y.y; P.zeta[ip] = Y.zeta; P.px[ip] = Y.px; P.py[ip] = Y.py; P.pz[ip] = Y.pz; P.z[ip] = s1;
    // lost: out of the window in zeta, or within one cell of a wall in y
    int al = (Y.zeta < 0 || Y.zeta >= c.zmax || Y.y < c.ylo || Y.y > c.yhi) ? 0 : 1;
    if (al == 1 && Y.zeta < c.zhand) { al = 2; P.rem[ip] = 0; }
    P.alive[ip] = al;
}

PushArgs push_args(Ctx& c, double s1) {
    PushArgs a;
    a.F = c.F.p; a.Fd = c.Fd.p; a.g = c.geo(); a.laser = c.laser;
    a.X0 = c.X0; a.Y0 = c.Y0; a.zc = c.P.zeta_center; a.dz_push = c.P.dz_push; a.push_phase = c.P.push_phase;
    // a sharded run: particles below zeta[a + 1] go to the rank below (sim_particles.cpp:10); rank 0 keeps all
    a.zhand = c.sharded() && c.rank > 0 ? c.zeta[size_t(c.a) + 1] : -1e300;
    a.zmax = c.zeta[c.N - 1]; a.s1 = s1; a.hmin = c.hmin;
    a.ylo = c.yf ? -1e300 : c.ynode_h[1];              // free-hand y: lost within one cell of a wall
    a.yhi = c.yf ? 1e300 : c.ynode_h[size_t(c.ny) - 1];
    a.vz_min = c.pl ? c.pl->cfg.vz_min : 0;            // slower beam particles stream in the plasma march
    a.freeze = c.P.freeze_bunch; a.self = c.P.self_fields;
    a.ext = c.ext;
    return a;
}
static void push_launch(Ctx& c, double s0, double s1, const int32_t* perm, long i0, long n) {
    if (n <= 0) return;
    const PushArgs a = push_args(c, s1);
    const int tok = c.prof_begin("push");
    if (c.Fd.p) k_push<double><<<unsigned((n + 127) / 128), 128, 0, c.stream>>>(a, c.Fd.p, c.parts, perm, i0, n, s0);
    else k_push<float><<<unsigned((n + 127) / 128), 128, 0, c.stream>>>(a, c.F.p, c.parts, perm, i0, n, s0);
    c.check_launch("k_push");
    c.prof_end(tok);
}
void launch_push(Ctx& c, double s0, double s1) { push_launch(c, s0, s1, c.perm.p, 0, c.np); }
// the particles [i0, i0 + n) in storage order (those adopted from the rank above finish their push)
void launch_push_range(Ctx& c, double s0, double s1, long i0, long n) { push_launch(c, s0, s1, nullptr, i0, n); }

}  // namespace g3d
