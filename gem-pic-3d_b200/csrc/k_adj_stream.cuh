// The reverse of one streaming particle's push through a whole half-cell (FP64), for the adjoint of the
// streaming-plasma march. The forward is stream_one of k_plasma.cu (src/sim_stream.hpp:104-171) for a particle
// that crosses the whole half-cell (the only case the adjoint admits: no trapping, no analytic wave, no external
// elements): the midpoint gather, the relativistic Boris push over dt0 = h / (1 - v_z0), the time dt of the
// half-cell from the mean of 1 - v_z before and after, the second Boris push over dt, and the TSC deposit of
// f (v_x, v_y, v_z) at the midpoint of the move, f = q w dt / (Delta h dx).
//
// Everything here is __host__ __device__ and reads memory only through two functors, so the same code runs in
// the kernels of the adjoint (the fields and the current adjoints on the device) and in a host harness that
// checks it against central differences with analytic fields:
//   Gat: gather(xm, ym, E, B)                 the fields at the midpoint of the push
//        adjoint(xm, ym, lE, lB, lxm, lym)    dJ/dE, dJ/dB into dJ/dF; dJ/dxm, dJ/dym out
//   Dep: gather(xd, yd, G, Dx, Dy)            G_c = sum_k W_k(xd, yd) lJ_c[k] of the current adjoints lJ (times
//                                             the deposit's 1/A), Dx_c, Dy_c their derivatives in xd, yd
#pragma once
#include "g3d_common.cuh"

namespace g3d {

// the relativistic Boris push (boris of k_plasma.cu, src/sim_stream.hpp:8-18) with the intermediates its
// reverse reads
struct BorisTape {
    double qh, um[3], gm, qg, t[3], up[3], sf;
};
G3D_HD void boris_taped(const double u[3], const double E[3], const double B[3], double qm, double dt, double out[3], BorisTape& T) {
    T.qh = 0.5 * qm * dt;
    for (int k = 0; k < 3; ++k) T.um[k] = u[k] + T.qh * E[k];
    T.gm = sqrt(1.0 + T.um[0] * T.um[0] + T.um[1] * T.um[1] + T.um[2] * T.um[2]);
    T.qg = T.qh / T.gm;
    for (int k = 0; k < 3; ++k) T.t[k] = T.qg * B[k];
    const double t2 = T.t[0] * T.t[0] + T.t[1] * T.t[1] + T.t[2] * T.t[2];
    T.up[0] = T.um[0] + (T.um[1] * T.t[2] - T.um[2] * T.t[1]);
    T.up[1] = T.um[1] + (T.um[2] * T.t[0] - T.um[0] * T.t[2]);
    T.up[2] = T.um[2] + (T.um[0] * T.t[1] - T.um[1] * T.t[0]);
    T.sf = 2.0 / (1.0 + t2);
    const double v[3] = {T.um[0] + T.sf * (T.up[1] * T.t[2] - T.up[2] * T.t[1]),
                         T.um[1] + T.sf * (T.up[2] * T.t[0] - T.up[0] * T.t[2]),
                         T.um[2] + T.sf * (T.up[0] * T.t[1] - T.up[1] * T.t[0])};
    for (int k = 0; k < 3; ++k) out[k] = v[k] + T.qh * E[k];
}
G3D_HD void cross3(const double a[3], const double b[3], double c[3]) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}
G3D_HD double dot3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// The transposed Boris push: lo = dJ/d(out) -> lu = dJ/du (assigned), dJ/dE, dJ/dB, dJ/ddt (added). Reverse of
// out = v + qh E, v = um + sf (up x t), sf = 2 / (1 + t.t), up = um + um x t, t = qg B, qg = qh / gm,
// gm = |(1, um)|, um = u + qh E, qh = qm dt / 2; for c = a x b the adjoints are la += b x lc, lb += lc x a.
G3D_HD void boris_reverse(const double E[3], const double B[3], double qm, const BorisTape& T, const double lo[3], double lu[3],
                          double lE[3], double lB[3], double& ldt) {
    double lqh = dot3(lo, E), lum[3], lt[3], lup[3], sv[3], tmp[3];
    for (int k = 0; k < 3; ++k) { lE[k] += T.qh * lo[k]; lum[k] = lo[k]; sv[k] = T.sf * lo[k]; }
    double ut[3];
    cross3(T.up, T.t, ut);
    const double lsf = dot3(lo, ut);
    cross3(T.t, sv, lup);                       // up: b x lc with a = up, b = t
    cross3(sv, T.up, lt);                       // t: lc x a
    const double lt2 = -0.5 * lsf * T.sf * T.sf;
    cross3(T.t, lup, tmp);                      // up = um + um x t
    for (int k = 0; k < 3; ++k) lum[k] += lup[k] + tmp[k];
    cross3(lup, T.um, tmp);
    for (int k = 0; k < 3; ++k) lt[k] += tmp[k] + 2.0 * T.t[k] * lt2;
    const double lqg = dot3(lt, B);
    for (int k = 0; k < 3; ++k) lB[k] += T.qg * lt[k];
    lqh += lqg / T.gm;
    const double lgm = -lqg * T.qh / (T.gm * T.gm);
    for (int k = 0; k < 3; ++k) lum[k] += lgm * T.um[k] / T.gm;
    lqh += dot3(lum, E);
    for (int k = 0; k < 3; ++k) { lu[k] = lum[k]; lE[k] += T.qh * lum[k]; }
    ldt += 0.5 * qm * lqh;
}

// One particle through a whole half-cell of height h: state (x, y, p) in, (xn, yn, u) out, the deposit f v at
// (xd, yd). fscale = 1 / (Delta h dx).
struct StreamTape {
    double g0, ig0, omv0, dt0, hd, xm, ym, E[3], B[3];
    BorisTape b1, b2;
    double u1[3], g1a, Q, dt, u[3], ig1, v[3], xn, yn, f;
};
template <class Gat>
G3D_HD void stream_push_taped(double x, double y, const double p[3], double qm, double qw, double h, double fscale, Gat& gat,
                              StreamTape& T) {
    T.g0 = sqrt(1.0 + p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    T.ig0 = 1.0 / T.g0;
    T.omv0 = (1.0 + p[0] * p[0] + p[1] * p[1]) / (T.g0 * (T.g0 + p[2]));      // 1 - v_z, no cancellation
    T.dt0 = h / T.omv0;
    T.hd = 0.5 * T.dt0 * T.ig0;
    T.xm = x + T.hd * p[0];
    T.ym = y + T.hd * p[1];
    gat.gather(T.xm, T.ym, T.E, T.B);
    boris_taped(p, T.E, T.B, qm, T.dt0, T.u1, T.b1);
    T.g1a = sqrt(1.0 + T.u1[0] * T.u1[0] + T.u1[1] * T.u1[1] + T.u1[2] * T.u1[2]);
    T.Q = T.omv0 + (1.0 + T.u1[0] * T.u1[0] + T.u1[1] * T.u1[1]) / (T.g1a * (T.g1a + T.u1[2]));
    T.dt = 2.0 * h / T.Q;
    boris_taped(p, T.E, T.B, qm, T.dt, T.u, T.b2);
    T.ig1 = 1.0 / sqrt(1.0 + T.u[0] * T.u[0] + T.u[1] * T.u[1] + T.u[2] * T.u[2]);
    for (int k = 0; k < 3; ++k) T.v[k] = 0.5 * (p[k] * T.ig0 + T.u[k] * T.ig1);
    T.xn = x + T.v[0] * T.dt;
    T.yn = y + T.v[1] * T.dt;
    T.f = qw * T.dt * fscale;
}

// The reverse: lout = dJ/d(xn, yn, u_x, u_y, u_z) and the current adjoints (through dep) -> lin = dJ/d(x, y, p_x,
// p_y, p_z) (assigned) and the field adjoints (through gat.adjoint). Each line below is the transpose of one line
// of stream_push_taped, taken in the reverse order.
template <class Gat, class Dep>
G3D_HD void stream_push_reverse(double x, double y, const double p[3], double qm, double qw, double h, double fscale, Gat& gat,
                                Dep& dep, const double lout[5], double lin[5]) {
    StreamTape T;
    stream_push_taped(x, y, p, qm, qw, h, fscale, gat, T);
    // the deposit f v at (xd, yd) = ((x + xn) / 2, (y + yn) / 2)
    double G[3], Dx[3], Dy[3];
    dep.gather(0.5 * (x + T.xn), 0.5 * (y + T.yn), G, Dx, Dy);
    double lv[3];
    for (int k = 0; k < 3; ++k) lv[k] = T.f * G[k];
    const double lf = dot3(T.v, G);
    const double lxd = T.f * dot3(T.v, Dx), lyd = T.f * dot3(T.v, Dy);
    double ldt = lf * qw * fscale;
    double lx = 0.5 * lxd, ly = 0.5 * lyd;
    const double lxn = 0.5 * lxd + lout[0], lyn = 0.5 * lyd + lout[1];
    // xn = x + v_x dt, yn = y + v_y dt
    lx += lxn; ly += lyn;
    lv[0] += lxn * T.dt; lv[1] += lyn * T.dt;
    ldt += lxn * T.v[0] + lyn * T.v[1];
    // v = (p / g0 + u / g1) / 2
    double lp[3], lu[3];
    double lig0 = 0, lig1 = 0;
    for (int k = 0; k < 3; ++k) {
        lp[k] = 0.5 * T.ig0 * lv[k];
        lig0 += 0.5 * p[k] * lv[k];
        lu[k] = 0.5 * T.ig1 * lv[k] + lout[2 + k];
        lig1 += 0.5 * T.u[k] * lv[k];
    }
    const double ig13 = T.ig1 * T.ig1 * T.ig1;
    for (int k = 0; k < 3; ++k) lu[k] -= lig1 * T.u[k] * ig13;
    // u = boris(p, E, B, dt)
    double lE[3] = {0, 0, 0}, lB[3] = {0, 0, 0}, lpb[3];
    boris_reverse(T.E, T.B, qm, T.b2, lu, lpb, lE, lB, ldt);
    for (int k = 0; k < 3; ++k) lp[k] += lpb[k];
    // dt = 2 h / Q, Q = omv0 + (1 - u1_z / g1a)
    const double lQ = -ldt * T.dt / T.Q;
    double lomv0 = lQ;
    const double g3 = 1.0 / (T.g1a * T.g1a * T.g1a);
    const double lu1[3] = {lQ * T.u1[2] * T.u1[0] * g3, lQ * T.u1[2] * T.u1[1] * g3,
                           -lQ * (1.0 + T.u1[0] * T.u1[0] + T.u1[1] * T.u1[1]) * g3};
    // u1 = boris(p, E, B, dt0)
    double ldt0 = 0;
    boris_reverse(T.E, T.B, qm, T.b1, lu1, lpb, lE, lB, ldt0);
    for (int k = 0; k < 3; ++k) lp[k] += lpb[k];
    // the gather at (xm, ym)
    double lxm = 0, lym = 0;
    gat.adjoint(T.xm, T.ym, lE, lB, lxm, lym);
    // xm = x + hd p_x, ym = y + hd p_y, hd = dt0 / (2 g0)
    lx += lxm; ly += lym;
    const double lhd = lxm * p[0] + lym * p[1];
    lp[0] += lxm * T.hd; lp[1] += lym * T.hd;
    ldt0 += 0.5 * T.ig0 * lhd;
    lig0 += 0.5 * T.dt0 * lhd;
    // dt0 = h / omv0, omv0 = 1 - p_z / g0
    lomv0 -= ldt0 * T.dt0 / T.omv0;
    const double ig03 = T.ig0 * T.ig0 * T.ig0;
    lp[0] += lomv0 * p[2] * p[0] * ig03;
    lp[1] += lomv0 * p[2] * p[1] * ig03;
    lp[2] -= lomv0 * (1.0 + p[0] * p[0] + p[1] * p[1]) * ig03;
    // ig0 = 1 / g0
    for (int k = 0; k < 3; ++k) lp[k] -= lig0 * p[k] * ig03;
    lin[0] = lx; lin[1] = ly; lin[2] = lp[0]; lin[3] = lp[1]; lin[4] = lp[2];
}

}  // namespace g3d
