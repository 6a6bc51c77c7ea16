// Host check of the transposed streaming push (gem-pic-3d_b200/csrc/k_adj_stream.cuh) against central differences
// of its forward, with analytic fields and an analytic current adjoint, for the whole half-cell, a particle joining
// inside it, a trapped one and one joining and trapped again; compiled by tests/test_stream_reverse.py with nvcc and
// run on the CPU (no GPU). Prints one line per case: the largest relative difference.
#include <cstdio>
#include <cmath>
#include "k_adj_stream.cuh"

using namespace g3d;

// fields M_c(x, y, zeta) = a_c sin(kx x + ph_c) cos(ky y + ps_c) (1 + bz_c zeta) + m_c, plus offsets dE, dB the check
// differentiates
struct AnaGat {
    double a[6], ph[6], ps[6], m[6], bz[6], kx, ky, dE[3], dB[3];
    double lE[3], lB[3];
    __host__ __device__ double t(int c, double x, double y) const { return a[c] * sin(kx * x + ph[c]) * cos(ky * y + ps[c]); }
    __host__ __device__ double val(int c, double x, double y, double z) const { return t(c, x, y) * (1 + bz[c] * z) + m[c]; }
    __host__ __device__ double dx(int c, double x, double y, double z) const {
        return a[c] * kx * cos(kx * x + ph[c]) * cos(ky * y + ps[c]) * (1 + bz[c] * z);
    }
    __host__ __device__ double dy(int c, double x, double y, double z) const {
        return -a[c] * ky * sin(kx * x + ph[c]) * sin(ky * y + ps[c]) * (1 + bz[c] * z);
    }
    __host__ __device__ void gather(double x, double y, double z, double E[3], double B[3]) const {
        for (int k = 0; k < 3; ++k) { E[k] = val(k, x, y, z) + dE[k]; B[k] = val(3 + k, x, y, z) + dB[k]; }
    }
    __host__ __device__ void adjoint(double x, double y, double z, const double le[3], const double lb[3], double& lx, double& ly,
                                     double& lz) {
        for (int k = 0; k < 3; ++k) {
            lE[k] = le[k]; lB[k] = lb[k];
            lx += le[k] * dx(k, x, y, z) + lb[k] * dx(3 + k, x, y, z);
            ly += le[k] * dy(k, x, y, z) + lb[k] * dy(3 + k, x, y, z);
            lz += le[k] * t(k, x, y) * bz[k] + lb[k] * t(3 + k, x, y) * bz[3 + k];
        }
    }
};
// current adjoints lJ_c(x, y) = b_c cos(qx x + r_c) sin(qy y + t_c) + n_c
struct AnaDep {
    double b[3], r[3], t[3], n[3], qx, qy;
    __host__ __device__ double val(int c, double x, double y) const { return b[c] * cos(qx * x + r[c]) * sin(qy * y + t[c]) + n[c]; }
    __host__ __device__ void gather(double x, double y, double G[3], double Dx[3], double Dy[3]) const {
        for (int c = 0; c < 3; ++c) {
            G[c] = val(c, x, y);
            Dx[c] = -b[c] * qx * sin(qx * x + r[c]) * sin(qy * y + t[c]);
            Dy[c] = b[c] * qy * cos(qx * x + r[c]) * cos(qy * y + t[c]);
        }
    }
};

struct Case { double x, y, zeta, z, p[3], qm, qw; StreamCase K; const char* what; };

// the scalar the reverse differentiates: lout . (xn, yn, zeta_out, z_out, u) + f v . lJ(xd, yd)
static double scalar(const Case& s, AnaGat& g, const AnaDep& d, const double lout[7]) {
    StreamTape T;
    stream_push_taped(s.x, s.y, s.zeta, s.z, s.p, s.qm, s.qw, s.K, g, T);
    const double xd = 0.5 * (s.x + T.xn), yd = 0.5 * (s.y + T.yn);
    double J = lout[0] * T.xn + lout[1] * T.yn + lout[2] * T.zeta_out + lout[3] * T.z_out + lout[4] * T.u[0] + lout[5] * T.u[1] +
               lout[6] * T.u[2];
    for (int c = 0; c < 3; ++c) J += T.f * T.v[c] * d.val(c, xd, yd);
    return J;
}

int main() {
    AnaGat g{};
    const double amp[6] = {0.3, -0.2, 0.05, 0.1, 0.25, -0.04};
    for (int c = 0; c < 6; ++c) {
        g.a[c] = amp[c]; g.ph[c] = 0.3 * c + 0.1; g.ps[c] = 0.7 - 0.2 * c; g.m[c] = 0.02 * (c - 2); g.bz[c] = 0.05 * (c + 1);
    }
    g.kx = 0.31; g.ky = 0.23;
    AnaDep d{};
    for (int c = 0; c < 3; ++c) { d.b[c] = 1.0 + 0.5 * c; d.r[c] = 0.4 * c; d.t[c] = 0.2 + 0.3 * c; d.n[c] = 0.1 * c; }
    d.qx = 0.17; d.qy = 0.29;
    const double lout[7] = {0.7, -0.4, 0.35, 0.6, 0.9, -0.3, 0.5};
    // half-cell [zn, zn + h]; the whole one starts at zn + h, a joining particle inside it; a trapped particle is
    // pushed over dtp to sTrap (its case holds the recorded event)
    const StreamCase whole{3.0, 0.2, 1.7, 1e9, false, 0}, whole2{3.0, 0.25, 0.9, 1e9, false, 0};
    const StreamCase part{3.0, 0.2, 1.7, 1e9, true, 0}, trapc{3.0, 0.2, 1.7, 10.3, false, 1}, trapj{3.0, 0.2, 1.7, 10.25, true, 1};
    const Case cases[6] = {
        {1.3, -0.8, 3.2, 10.0, {0.2, -0.1, 0.05}, -1.0, -0.8, whole, "a plasma electron through the whole half-cell"},
        {-2.1, 0.6, 3.25, 10.0, {1.5, 0.7, 3.0}, -1.0, -0.5, whole2, "a fast one"},
        {0.4, 2.2, 3.2, 10.0, {0.01, 0.02, -0.005}, 1.0 / 1836.0, 0.8, whole, "a mobile ion"},
        {1.1, 0.3, 3.13, 10.0, {0.3, 0.2, 0.4}, -1.0, -0.7, part, "joining inside the half-cell"},
        {0.9, -1.4, 3.2, 10.0, {0.6, -0.3, 1.2}, -1.0, -0.6, trapc, "trapped inside the half-cell"},
        {-0.5, 0.8, 3.12, 10.0, {0.5, 0.4, 1.5}, -1.0, -0.9, trapj, "joining and trapped again"},
    };
    double worst = 0;
    for (int ci = 0; ci < 6; ++ci) {
        const Case s0 = cases[ci];
        double lin[7];
        stream_push_reverse(s0.x, s0.y, s0.zeta, s0.z, s0.p, s0.qm, s0.qw, s0.K, g, d, lout, lin);
        double lE[3], lB[3];
        for (int k = 0; k < 3; ++k) { lE[k] = g.lE[k]; lB[k] = g.lB[k]; }
        StreamTape T;
        stream_push_taped(s0.x, s0.y, s0.zeta, s0.z, s0.p, s0.qm, s0.qw, s0.K, g, T);
        double err = 0;
        // the seven state components
        for (int k = 0; k < 7; ++k) {
            const double eps = 1e-6 * (k < 4 ? 1.0 : fmax(1.0, fabs(s0.p[k - 4])));
            Case a = s0, b = s0;
            double* pa[7] = {&a.x, &a.y, &a.zeta, &a.z, &a.p[0], &a.p[1], &a.p[2]};
            double* pb[7] = {&b.x, &b.y, &b.zeta, &b.z, &b.p[0], &b.p[1], &b.p[2]};
            *pa[k] += eps; *pb[k] -= eps;
            const double fd = (scalar(a, g, d, lout) - scalar(b, g, d, lout)) / (2 * eps);
            const double e = fabs(fd - lin[k]) / fmax(1e-3, fabs(fd));
            if (e > err) err = e;
        }
        // the six field offsets
        for (int k = 0; k < 6; ++k) {
            const double eps = 1e-6;
            double* o = k < 3 ? &g.dE[k] : &g.dB[k - 3];
            *o = eps;
            const double jp = scalar(s0, g, d, lout);
            *o = -eps;
            const double jm = scalar(s0, g, d, lout);
            *o = 0;
            const double fd = (jp - jm) / (2 * eps);
            const double an = k < 3 ? lE[k] : lB[k - 3];
            const double e = fabs(fd - an) / fmax(1e-3, fabs(fd));
            if (e > err) err = e;
        }
        std::printf("case %d (%s%s): largest relative difference %.3e\n", ci, s0.what, T.trapped ? ", dtp > 0" : "", err);
        if ((s0.K.trap == 1) != T.trapped || (T.trapped && !(T.dtp > 0))) { std::printf("case %d: not the intended branch\n", ci); return 2; }
        if (err > worst) worst = err;
    }
    std::printf("worst %.3e\n", worst);
    return worst < 1e-6 ? 0 : 1;
}
