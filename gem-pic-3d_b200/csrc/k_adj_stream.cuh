// The reverse of one streaming particle's push through a half-cell (FP64), for the adjoint of the streaming-plasma
// march. The forward is stream_one of k_plasma.cu (src/sim_stream.hpp:104-171) without an analytic wave or external
// elements: the gather half-way along the path, the relativistic Boris push over dt0 = hl / (1 - v_z0), the time dt
// of the path from the mean of 1 - v_z before and after, the second Boris push over dt (a third over the shorter dtp
// when the particle is trapped inside the half-cell), and the TSC deposit of f (v_x, v_y, v_z) at the midpoint of
// the move, f = q w dt / (Delta h dx). Whether a particle is trapped is an event of the forward that the reverse
// keeps as it was.
//
// Everything here is __host__ __device__ and reads memory only through two functors, so the same code runs in
// the kernels of the adjoint (the fields and the current adjoints on the device) and in a host harness that
// checks it against central differences with analytic fields:
//   Gat: gather(xm, ym, zetam, E, B)                  the fields at the midpoint of the push
//        adjoint(xm, ym, zetam, lE, lB, lxm, lym, lzm) dJ/dE, dJ/dB into dJ/dF; dJ/dxm, dJ/dym, dJ/dzetam added
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

// One particle through half-cell n (slices zn < zn1, h = zn1 - zn) from its state (x, y, zeta, z, p): the whole
// half-cell (hl = h), or from zeta down (hl = zeta - zn, a particle joining the march inside the half-cell); the
// fields at the midpoint of its path (xm, ym, zetam = zeta - hl / 2); out (xn, yn, zeta_out, z_out, u). A trapped
// particle (its lab position advanced to sTrap inside the half-cell) is pushed over dtp = (sTrap - z) / max(v_z, 1e-3)
// instead of dt, stops at zeta - (1 - v_z) dtp and takes z = s1. fscale = 1 / (Delta h dx).
struct StreamCase {
    double zn, h, fscale, sTrap;
    bool partial;              // hl = zeta - zn (the forward: zeta below zn1 - 1e-9 h)
    int trap;                  // 0: not trapped, 1: trapped (a recorded event), 2: as the forward decides
};
struct StreamTape {
    double hl, g0, ig0, omv0, dt0, hd, xm, ym, zetam, E[3], B[3];
    BorisTape b1, b2, b3;
    double u1[3], g1a, Q, dt, u2[3], ig2, v2[3], vv, dtp, u[3], ig1, v[3], dte, xn, yn, zeta_out, z_out, f;
    bool trapped;
};
template <class Gat>
G3D_HD void stream_push_taped(double x, double y, double zeta, double z, const double p[3], double qm, double qw, const StreamCase& K,
                              Gat& gat, StreamTape& T) {
    T.hl = K.partial ? (zeta - K.zn > 0 ? zeta - K.zn : 0.0) : K.h;
    T.g0 = sqrt(1.0 + p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    T.ig0 = 1.0 / T.g0;
    T.omv0 = (1.0 + p[0] * p[0] + p[1] * p[1]) / (T.g0 * (T.g0 + p[2]));      // 1 - v_z, no cancellation
    T.dt0 = T.hl / T.omv0;
    T.hd = 0.5 * T.dt0 * T.ig0;
    T.xm = x + T.hd * p[0];
    T.ym = y + T.hd * p[1];
    T.zetam = zeta - 0.5 * T.hl;
    gat.gather(T.xm, T.ym, T.zetam, T.E, T.B);
    boris_taped(p, T.E, T.B, qm, T.dt0, T.u1, T.b1);
    T.g1a = sqrt(1.0 + T.u1[0] * T.u1[0] + T.u1[1] * T.u1[1] + T.u1[2] * T.u1[2]);
    T.Q = T.omv0 + (1.0 + T.u1[0] * T.u1[0] + T.u1[1] * T.u1[1]) / (T.g1a * (T.g1a + T.u1[2]));
    T.dt = 2.0 * T.hl / T.Q;
    boris_taped(p, T.E, T.B, qm, T.dt, T.u2, T.b2);
    T.ig2 = 1.0 / sqrt(1.0 + T.u2[0] * T.u2[0] + T.u2[1] * T.u2[1] + T.u2[2] * T.u2[2]);
    for (int k = 0; k < 3; ++k) T.v2[k] = 0.5 * (p[k] * T.ig0 + T.u2[k] * T.ig2);
    T.trapped = K.trap == 1 || (K.trap == 2 && z + T.v2[2] * T.dt >= K.sTrap);
    if (T.trapped) {
        T.vv = T.v2[2] > 1e-3 ? T.v2[2] : 1e-3;
        T.dtp = (K.sTrap - z) / T.vv > 0 ? (K.sTrap - z) / T.vv : 0.0;
        boris_taped(p, T.E, T.B, qm, T.dtp, T.u, T.b3);
        T.ig1 = 1.0 / sqrt(1.0 + T.u[0] * T.u[0] + T.u[1] * T.u[1] + T.u[2] * T.u[2]);
        for (int k = 0; k < 3; ++k) T.v[k] = 0.5 * (p[k] * T.ig0 + T.u[k] * T.ig1);
        T.dte = T.dtp;
        T.zeta_out = zeta - (1.0 - T.v[2]) * T.dtp;
        T.z_out = 0;                                   // s1: a constant
    } else {
        for (int k = 0; k < 3; ++k) { T.u[k] = T.u2[k]; T.v[k] = T.v2[k]; }
        T.ig1 = T.ig2;
        T.dte = T.dt;
        T.zeta_out = K.zn;
        T.z_out = z + T.v2[2] * T.dt;
    }
    T.xn = x + T.v[0] * T.dte;
    T.yn = y + T.v[1] * T.dte;
    T.f = qw * T.dte * K.fscale;
}

// The reverse: lout = dJ/d(xn, yn, zeta_out, z_out, u_x, u_y, u_z) and the current adjoints (through dep) ->
// lin = dJ/d(x, y, zeta, z, p_x, p_y, p_z) (assigned) and the field adjoints (through gat.adjoint). Each line below is
// the transpose of one line of stream_push_taped, in the reverse order.
template <class Gat, class Dep>
G3D_HD void stream_push_reverse(double x, double y, double zeta, double z, const double p[3], double qm, double qw, const StreamCase& K,
                                Gat& gat, Dep& dep, const double lout[7], double lin[7]) {
    StreamTape T;
    stream_push_taped(x, y, zeta, z, p, qm, qw, K, gat, T);
    // the deposit f v at (xd, yd) = ((x + xn) / 2, (y + yn) / 2), f = q w dte fscale
    double G[3], Dx[3], Dy[3];
    dep.gather(0.5 * (x + T.xn), 0.5 * (y + T.yn), G, Dx, Dy);
    double lv[3];
    for (int k = 0; k < 3; ++k) lv[k] = T.f * G[k];
    const double lf = dot3(T.v, G);
    const double lxd = T.f * dot3(T.v, Dx), lyd = T.f * dot3(T.v, Dy);
    double ldte = lf * qw * K.fscale;
    double lx = 0.5 * lxd, ly = 0.5 * lyd, lzeta = 0, lz = 0, ldt = 0;
    const double lxn = 0.5 * lxd + lout[0], lyn = 0.5 * lyd + lout[1];
    // xn = x + v_x dte, yn = y + v_y dte
    lx += lxn; ly += lyn;
    lv[0] += lxn * T.dte; lv[1] += lyn * T.dte;
    ldte += lxn * T.v[0] + lyn * T.v[1];
    double lp[3], lu[3], lig0 = 0, lig1 = 0, lE[3] = {0, 0, 0}, lB[3] = {0, 0, 0}, lpb[3];
    if (T.trapped) {
        // zeta_out = zeta - (1 - v_z) dtp (z_out = s1 holds no dependence)
        lzeta += lout[2];
        lv[2] += lout[2] * T.dtp;
        ldte -= (1.0 - T.v[2]) * lout[2];
    } else {
        // z_out = z + v_z dt (zeta_out = zn holds none)
        lz += lout[3];
        lv[2] += lout[3] * T.dt;
        ldte += lout[3] * T.v[2];
    }
    // v = (p / g0 + u / g1) / 2
    for (int k = 0; k < 3; ++k) {
        lp[k] = 0.5 * T.ig0 * lv[k];
        lig0 += 0.5 * p[k] * lv[k];
        lu[k] = 0.5 * T.ig1 * lv[k] + lout[4 + k];
        lig1 += 0.5 * T.u[k] * lv[k];
    }
    const double ig13 = T.ig1 * T.ig1 * T.ig1;
    for (int k = 0; k < 3; ++k) lu[k] -= lig1 * T.u[k] * ig13;
    double lu2[3] = {0, 0, 0};
    if (T.trapped) {
        // u = boris(p, dtp), dtp = (sTrap - z) / vv, vv = max(v2_z, 1e-3), v2 = (p / g0 + u2 / g2) / 2
        double ldtp = ldte;
        boris_reverse(T.E, T.B, qm, T.b3, lu, lpb, lE, lB, ldtp);
        for (int k = 0; k < 3; ++k) lp[k] += lpb[k];
        if (T.dtp > 0) {
            lz -= ldtp / T.vv;
            if (T.v2[2] > 1e-3) {
                const double lv2z = -ldtp * T.dtp / T.vv;
                lp[2] += 0.5 * T.ig0 * lv2z;
                lig0 += 0.5 * p[2] * lv2z;
                lu2[2] += 0.5 * T.ig2 * lv2z;
                const double lig2 = 0.5 * T.u2[2] * lv2z, ig23 = T.ig2 * T.ig2 * T.ig2;
                for (int k = 0; k < 3; ++k) lu2[k] -= lig2 * T.u2[k] * ig23;
            }
        }
    } else {
        for (int k = 0; k < 3; ++k) lu2[k] = lu[k];
        ldt = ldte;
    }
    // u2 = boris(p, dt)
    boris_reverse(T.E, T.B, qm, T.b2, lu2, lpb, lE, lB, ldt);
    for (int k = 0; k < 3; ++k) lp[k] += lpb[k];
    // dt = 2 hl / Q, Q = omv0 + (1 - u1_z / g1a)
    double lhl = 2.0 * ldt / T.Q;
    const double lQ = -ldt * T.dt / T.Q;
    double lomv0 = lQ;
    const double g3 = 1.0 / (T.g1a * T.g1a * T.g1a);
    const double lu1[3] = {lQ * T.u1[2] * T.u1[0] * g3, lQ * T.u1[2] * T.u1[1] * g3,
                           -lQ * (1.0 + T.u1[0] * T.u1[0] + T.u1[1] * T.u1[1]) * g3};
    // u1 = boris(p, dt0)
    double ldt0 = 0;
    boris_reverse(T.E, T.B, qm, T.b1, lu1, lpb, lE, lB, ldt0);
    for (int k = 0; k < 3; ++k) lp[k] += lpb[k];
    // the gather at (xm, ym, zetam), zetam = zeta - hl / 2
    double lxm = 0, lym = 0, lzm = 0;
    gat.adjoint(T.xm, T.ym, T.zetam, lE, lB, lxm, lym, lzm);
    lzeta += lzm;
    lhl -= 0.5 * lzm;
    // xm = x + hd p_x, ym = y + hd p_y, hd = dt0 / (2 g0)
    lx += lxm; ly += lym;
    const double lhd = lxm * p[0] + lym * p[1];
    lp[0] += lxm * T.hd; lp[1] += lym * T.hd;
    ldt0 += 0.5 * T.ig0 * lhd;
    lig0 += 0.5 * T.dt0 * lhd;
    // dt0 = hl / omv0, omv0 = 1 - p_z / g0
    lhl += ldt0 / T.omv0;
    lomv0 -= ldt0 * T.dt0 / T.omv0;
    const double ig03 = T.ig0 * T.ig0 * T.ig0;
    lp[0] += lomv0 * p[2] * p[0] * ig03;
    lp[1] += lomv0 * p[2] * p[1] * ig03;
    lp[2] -= lomv0 * (1.0 + p[0] * p[0] + p[1] * p[1]) * ig03;
    // ig0 = 1 / g0
    for (int k = 0; k < 3; ++k) lp[k] -= lig0 * p[k] * ig03;
    // hl = zeta - zn (partial)
    if (K.partial && zeta - K.zn > 0) lzeta += lhl;
    lin[0] = lx; lin[1] = ly; lin[2] = lzeta; lin[3] = lz; lin[4] = lp[0]; lin[5] = lp[1]; lin[6] = lp[2];
}

}  // namespace g3d
