// Streaming plasma: the march of a step with plasma, half-cell by half-cell (Simulation::march_plasma,
// src/sim_plasma.cpp:228-470, one rank, Fourier y).
//
// Per half-cell n (front to rear) and pass:
//   k_stream       one thread per streaming particle: the push through the half-cell (stream_one,
//                  src/sim_stream.hpp:104-171): mid-point gather of the grid fields + analytic wave, two relativistic
//                  Boris pushes (a third when the particle is trapped inside the half-cell), TSC deposit of its
//                  current and charge into the real planes jsr (stream_deposit, :33-64), ADK ionization of the ions
//                  with the counter-based random numbers (ionize, :80-101; ionization.hpp:25-46)
//   k_ss_rows/cols the spectra of jsr: FFT of jx + i jy and jz of one plane, the k-filters, the smoothing
//                  1 / (1 + a^2 k_perp^2) (stream_spectra, src/sim_plasma.cpp:94-157) -> jsn (half spectrum)
//   k_replace_pred replace the streaming part of jk(n) by jsn and, with the extrapolating predictor, of jk(n-1) by
//                  js0(n-1) + d + w (d - dl), d = jsn - js0(n) (sim_plasma.cpp:339-351)
//   k_march_slice  the march of the modes of slice n (march_point, src/sim_kernels.hpp:173-210)
//   real fields of slice n: the column and row kernels of k_fields.cu on one plane
// On the Fourier y grid the column transform of the spectra, the replace and prediction, the slice march and the
// column transforms of the real fields are one kernel per k_x column (k_pass_cols), between k_ss_rows and the
// rows kernel of the real fields.
// A pass before the last (the predictor) deposits, transforms and marches like the last one but leaves the
// particles unchanged (StreamArgs::dry), so every pass starts from the same particle state without a copy.
// After the passes: k_correct (R of slice n+1 corrected for the prediction it used; dl, js0 updated,
// sim_plasma.cpp:381-403) and k_born_append (the freed electrons join the march).
#include <type_traits>
#include <cub/device/device_scan.cuh>
#include "g3d_plasma.hpp"
#include "k_external.cuh"
#include "k_fft.cuh"
#include "k_dispatch.cuh"

namespace g3d {

// ---------------------------------------------------------------- relativistic Boris (sim_stream.hpp:8-18)
// A: the arithmetic type of the push (double in both forms)
template <class A>
__device__ __forceinline__ void boris(A& ux, A& uy, A& uz, const A E[3], const A B[3], A qm, A dt) {
    const A qh = A(0.5) * qm * dt;
    const A umx = ux + qh * E[0], umy = uy + qh * E[1], umz = uz + qh * E[2];
    const A qg = qh / sqrt(A(1) + umx * umx + umy * umy + umz * umz);     // q dt / (2 m gamma-)
    const A tx = qg * B[0], ty = qg * B[1], tz = qg * B[2];
    const A t2 = tx * tx + ty * ty + tz * tz;
    const A upx = umx + (umy * tz - umz * ty), upy = umy + (umz * tx - umx * tz), upz = umz + (umx * ty - umy * tx);
    const A sf = A(2) / (A(1) + t2);
    const A vx = umx + sf * (upy * tz - upz * ty), vy = umy + sf * (upz * tx - upx * tz), vz = umz + sf * (upx * ty - upy * tx);
    ux = vx + qh * E[0]; uy = vy + qh * E[1]; uz = vz + qh * E[2];
}

// grid fields of the F planes (TSC in x, y, linear in zeta) as in the beam push. F32 (the mixed form): the
// weights and the sums in FP32; else FP64 arithmetic on the float data.
template <bool F32, bool YF, int NC = 6>
__device__ __forceinline__ void sgather(const StreamArgs& c, double x, double y, double zeta, double E[3], double B[3]) {
    E[0] = E[1] = E[2] = B[0] = B[1] = B[2] = 0;
    const Geo& g = c.g;
    int n; double fz;
    g.zax.locate(zeta, n, fz);
    if (n == g.a - 1 && fz > 1 - 1e-9) { n = g.a; fz = 0; }
    const int fl = n - g.a;
    if (fl < 0 || fl > g.ns) return;
    int ix[3], jn[3]; double wx[3], wn[3];
    tsc_periodic(x, g.dx, g.nx, ix, wx);
    const long nk = g.nk;
    typedef typename std::conditional<F32, float, double>::type R;
    if constexpr (!YF) {               // free-hand y: E_y, B_x, B_z on the half-nodes, nothing beyond the walls
        int jh[3]; double wh[3];
        tsc_y(g.yax, y, jn, wn, jh, wh);
        const R f1 = R(fz), f0 = R(1 - fz);
#pragma unroll
        for (int comp = 0; comp < NC; ++comp) {
            const float* p0 = c.F + (long(comp) * (g.ns + 2) + fl) * nk;
            const float* p1 = p0 + nk;
            const bool hf = is_half(comp);
            R v0 = 0, v1 = 0;
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                const int jy = hf ? jh[j] : jn[j];
                const double wy = hf ? wh[j] : wn[j];
                if (jy < 0 || jy >= g.ny) continue;
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    const long k = long(jy) * g.nx + ix[i];
                    const R w = R(wx[i] * wy);
                    v0 += w * R(p0[k]); v1 += w * R(p1[k]);
                }
            }
            const double v = double(f0 * v0 + f1 * v1);
            if (comp < 3) E[comp] = v; else B[comp - 3] = v;
        }
        return;
    }
    tsc_periodic(y, g.dy, g.ny, jn, wn);
    R w9[9];
    int k9[9];
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int i = 0; i < 3; ++i) { w9[3 * j + i] = R(wx[i] * wn[j]); k9[3 * j + i] = jn[j] * g.nx + ix[i]; }
    // both slices summed with the TSC weights, then interpolated in zeta
    const R f1 = R(fz), f0 = R(1 - fz);
#pragma unroll
    for (int comp = 0; comp < NC; ++comp) {
        const float* p0 = c.F + (long(comp) * (g.ns + 2) + fl) * nk;
        const float* p1 = p0 + nk;
        R v0 = 0, v1 = 0;
#pragma unroll
        for (int q = 0; q < 9; ++q) { v0 += w9[q] * R(p0[k9[q]]); v1 += w9[q] * R(p1[k9[q]]); }
        const double v = double(f0 * v0 + f1 * v1);
        if (comp < 3) E[comp] = v; else B[comp - 3] = v;
    }
}
// The exact fields (the FP64 planes Fd of the FP64 form) at (x, y, zeta), TSC in x and y, linear in zeta: the gather of
// a particle that starts inside the half-cell when the fields are kept exact (a variant of its own, k_stream's EX)
__device__ __forceinline__ void sgather_exact(const StreamArgs& c, double x, double y, double zeta, double E[3], double B[3]) {
    E[0] = E[1] = E[2] = B[0] = B[1] = B[2] = 0;
    const Geo& g = c.g;
    int n; double fz;
    g.zax.locate(zeta, n, fz);
    if (n == g.a - 1 && fz > 1 - 1e-9) { n = g.a; fz = 0; }
    const int fl = n - g.a;
    if (fl < 0 || fl > g.ns) return;
    int ix[3], jn[3]; double wx[3], wn[3];
    tsc_periodic(x, g.dx, g.nx, ix, wx);
    tsc_periodic(y, g.dy, g.ny, jn, wn);
    const long nk = g.nk;
    for (int comp = 0; comp < 6; ++comp) {
        const double* p0 = c.Fd + (long(comp) * (g.ns + 2) + fl) * nk;
        const double* p1 = p0 + nk;
        double v0 = 0, v1 = 0;
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                const long k = long(jn[j]) * g.nx + ix[i];
                v0 += wx[i] * wn[j] * p0[k]; v1 += wx[i] * wn[j] * p1[k];
            }
        const double v = (1 - fz) * v0 + fz * v1;
        if (comp < 3) E[comp] = v; else B[comp - 3] = v;
    }
}
// The gather half-way through the half-cell (zeta = the slice midpoint, a particle crossing the whole half-cell):
// TSC in x and y of the interleaved midpoint fields, one vector load per point (Fourier y).
template <bool F32>
__device__ __forceinline__ void sgather_mid(const StreamArgs& c, double x, double y, double E[3], double B[3]) {
    const Geo& g = c.g;
    int ix[3], jn[3]; double wx[3], wn[3];
    tsc_periodic(x, g.dx, g.nx, ix, wx);
    tsc_periodic(y, g.dy, g.ny, jn, wn);
    typedef typename std::conditional<F32, float, double>::type R;
    R a[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const long k = long(jn[j]) * g.nx + ix[i];
            const R w = R(wx[i] * wn[j]);
            if constexpr (F32) {
                const float4* p = reinterpret_cast<const float4*>(c.Fmid) + 2 * k;
                const float4 u = __ldg(p), v = __ldg(p + 1);
                a[0] += w * u.x; a[1] += w * u.y; a[2] += w * u.z; a[3] += w * u.w; a[4] += w * v.x; a[5] += w * v.y;
            } else {
                const double2* p = reinterpret_cast<const double2*>(c.Fmid) + 3 * k;
                const double2 u = __ldg(p), v = __ldg(p + 1), q = __ldg(p + 2);
                a[0] += w * u.x; a[1] += w * u.y; a[2] += w * v.x; a[3] += w * v.y; a[4] += w * q.x; a[5] += w * q.y;
            }
        }
    E[0] = double(a[0]); E[1] = double(a[1]); E[2] = double(a[2]);
    B[0] = double(a[3]); B[1] = double(a[4]); B[2] = double(a[5]);
}
// The mixed form's TSC on a periodic grid: the cell coordinate t = x / d and the nearest node in FP64 (x spans the
// box, so the index needs the double), the offset from that node in FP32, the three weights in FP32.
__device__ __forceinline__ void tsc_f32(double x, double inv_d, int n, int idx[3], float w[3]) {
    const double t = x * inv_d;
    const double c = floor(t + 0.5);
    const float f = float(t - c);
    w[0] = 0.5f * (0.5f - f) * (0.5f - f);
    w[1] = 0.75f - f * f;
    w[2] = 0.5f * (0.5f + f) * (0.5f + f);
    int b = (int(c) - 1) % n;
    if (b < 0) b += n;
    const int b1 = b + 1 == n ? 0 : b + 1;
    idx[0] = b; idx[1] = b1; idx[2] = b1 + 1 == n ? 0 : b1 + 1;
}
// The mixed form's midpoint gather (Fourier y): the interleaved midpoint fields with FP32 weights, straight into
// the FP32 fields of the Boris push.
__device__ __forceinline__ void sgather_mid_f32(const StreamArgs& c, double x, double y, float E[3], float B[3]) {
    int ix[3], jn[3]; float wx[3], wn[3];
    tsc_f32(x, c.inv_dx, c.g.nx, ix, wx);
    tsc_f32(y, c.inv_dy, c.g.ny, jn, wn);
    float a[6] = {0, 0, 0, 0, 0, 0};
    const float4* F4 = reinterpret_cast<const float4*>(c.Fmid);
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            const long k = long(jn[j]) * c.g.nx + ix[i];
            const float w = wx[i] * wn[j];
            const float4 u = __ldg(F4 + 2 * k), v = __ldg(F4 + 2 * k + 1);
            a[0] += w * u.x; a[1] += w * u.y; a[2] += w * u.z; a[3] += w * u.w; a[4] += w * v.x; a[5] += w * v.y;
        }
    E[0] = a[0]; E[1] = a[1]; E[2] = a[2]; B[0] = a[3]; B[1] = a[4]; B[2] = a[5];
}
// The mixed form's midpoint gather on the free-hand y grid: per TSC point one float4 of the node row (E_x, E_z, B_y)
// and one of the half-node row (E_y, B_x, B_z) of the interleaved midpoint fields, rows beyond the walls left out
// (as sgather does); the weights as in sgather's FP32 form (FP64 TSC weights, their products rounded to FP32).
__device__ __forceinline__ void sgather_mid_fh_f32(const StreamArgs& c, double x, double y, float E[3], float B[3]) {
    const Geo& g = c.g;
    int ix[3], jn[3], jh[3]; double wx[3], wn[3], wh[3];
    tsc_periodic(x, g.dx, g.nx, ix, wx);
    tsc_y(g.yax, y, jn, wn, jh, wh);
    float a[6] = {0, 0, 0, 0, 0, 0};
    const float4* F4 = reinterpret_cast<const float4*>(c.Fmid);
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const bool nod = jn[j] >= 0 && jn[j] < g.ny, hal = jh[j] >= 0 && jh[j] < g.ny;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            if (nod) {
                const float w = float(wx[i] * wn[j]);
                const float4 u = __ldg(F4 + 2 * (long(jn[j]) * g.nx + ix[i]));
                a[0] += w * u.x; a[2] += w * u.y; a[4] += w * u.z;
            }
            if (hal) {
                const float w = float(wx[i] * wh[j]);
                const float4 v = __ldg(F4 + 2 * (long(jh[j]) * g.nx + ix[i]) + 1);
                a[1] += w * v.x; a[3] += w * v.y; a[5] += w * v.z;
            }
        }
    }
    E[0] = a[0]; E[1] = a[1]; E[2] = a[2]; B[0] = a[3]; B[1] = a[4]; B[2] = a[5];
}
// The charge of a particle's TSC points on the lines through the axis of half-cell n (the density lines,
// src/sim_plasma.cpp:363-374, of the charge planes that stream_deposit fills, src/sim_stream.hpp:33-64): the points of
// row j0 at their column, those of column i0 at nx + their row. W(u, v) is the charge of point (ix[u], jn[v]); a point
// with jn[v] < 0 has none. Negative particles go to rl[0], positive ones to rl[1] (null: not recorded).
template <typename T, typename Wf>
__device__ __forceinline__ void sdeposit_lines(const StreamArgs& c, T f, const int ix[3], const int jn[3], Wf W) {
    double* rl = c.rl[f < T(0) ? 0 : 1];
    if (!rl) return;
    const int i0 = c.sv->i0, j0 = c.sv->j0;
#pragma unroll
    for (int v = 0; v < 3; ++v)
        if (jn[v] == j0)
#pragma unroll
            for (int u = 0; u < 3; ++u) atomicAdd(rl + ix[u], double(W(u, v)));
#pragma unroll
    for (int u = 0; u < 3; ++u)
        if (ix[u] == i0)
#pragma unroll
            for (int v = 0; v < 3; ++v)
                if (jn[v] >= 0) atomicAdd(rl + c.g.nx + jn[v], double(W(u, v)));
}
__device__ __forceinline__ double wrapx(const Geo& g, double x) { return wrap_periodic(x, g.Lx); }
template <bool YF>
__device__ __forceinline__ double wrapy(const Geo& g, double y) { return YF ? wrap_periodic(y, g.Ly) : y; }   // free-hand: walls

// TSC deposit of f v at (x, y) into jsr: jx, jy, jz (stream_deposit, sim_stream.hpp:33-64). The reference also
// deposits the charge of negative and positive particles into whole planes 3 and 4, of which it keeps only the lines
// through the axis (rho_lines; openPMD n_e / n_i, not written here, take the planes): the last pass adds the charge of
// the points on those lines alone (sdeposit_lines). F32: into the FP32 planes; on the Fourier y grid interleaved per
// point as (jx, jy, jz, 0), one vector atomic add per TSC point instead of three (the adds into L2 bound the
// streaming push).
template <bool F32, bool YF>
__device__ __forceinline__ void sdeposit(const StreamArgs& c, double x, double y, double f, double vx, double vy, double vz) {
    const Geo& g = c.g;
    int ix_[3], jn[3]; double wx[3], wn[3];
    tsc_periodic(x, g.dx, g.nx, ix_, wx);
    const long nk = g.nk;
    if constexpr (!YF) {               // free-hand y: j_x, j_z on the nodes, j_y on the half-nodes
        int jh[3]; double wh[3];
        tsc_y(g.yax, y, jn, wn, jh, wh);
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const bool nod = jn[v] >= 1 && jn[v] <= g.ny - 1, hal = jh[v] >= 0 && jh[v] <= g.ny - 1;
#pragma unroll
            for (int u = 0; u < 3; ++u) {
                if (nod) {
                    const long k = long(jn[v]) * g.nx + ix_[u];
                    const double w = f * wx[u] * wn[v] * g.iA[jn[v]];
                    if constexpr (F32) {
                        atomicAdd(&c.Jf[k], float(w * vx)); atomicAdd(&c.Jf[2 * nk + k], float(w * vz));
                    } else {
                        atomicAdd(&c.J[k], w * vx); atomicAdd(&c.J[2 * nk + k], w * vz);
                    }
                }
                if (hal) {
                    const long k = long(jh[v]) * g.nx + ix_[u];
                    const double w = f * wx[u] * wh[v] * g.iD[jh[v]] * vy;
                    if constexpr (F32) atomicAdd(&c.Jf[nk + k], float(w));
                    else atomicAdd(&c.J[nk + k], w);
                }
            }
        }
        int jl[3];                     // the charge lives on the inner nodes 1 .. ny - 1
#pragma unroll
        for (int v = 0; v < 3; ++v) jl[v] = jn[v] >= 1 && jn[v] <= g.ny - 1 ? jn[v] : -1;
        sdeposit_lines(c, f, ix_, jl, [&](int u, int v) { return f * wx[u] * wn[v] * g.iA[jl[v]]; });
        return;
    }
    tsc_periodic(y, g.dy, g.ny, jn, wn);
    const double ia0 = g.iA[0];
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int u = 0; u < 3; ++u) {
            const long k = long(jn[v]) * g.nx + ix_[u];
            const double w = f * wx[u] * wn[v] * ia0;
            if constexpr (F32) {
                atomicAdd(reinterpret_cast<float4*>(c.Jf) + k, make_float4(float(w * vx), float(w * vy), float(w * vz), 0.f));
            } else {
                atomicAdd(&c.J[k], w * vx); atomicAdd(&c.J[nk + k], w * vy); atomicAdd(&c.J[2 * nk + k], w * vz);
            }
        }
    sdeposit_lines(c, f, ix_, jn, [&](int u, int v) { return f * wx[u] * wn[v] * ia0; });
}

// |E| of the grid and the wave at (x, y), lab z, slice position zeta (field_abs, sim_stream.hpp:67-74)
template <bool F32, bool YF>
__device__ __forceinline__ double field_abs(const StreamArgs& c, double x, double y, double z, double zeta) {
    double E[3], B[3], Ee[3], Be[3];
    sgather<F32, YF, 3>(c, wrapx(c.g, x), wrapy<YF>(c.g, y), zeta, E, B);      // |E| needs the electric field only
    c.laser.field(x + c.sv->X0, z, z - (zeta - c.zc), Ee, Be);
    for (int k = 0; k < 3; ++k) E[k] += Ee[k];
    return sqrt(E[0] * E[0] + E[1] * E[1] + E[2] * E[2]);
}

// ADK rate of a level (ionization.hpp:198-202) and the counter-based random numbers (ionization.hpp:209-218)
__device__ __forceinline__ double adk_rate(const AdkDev& L, double E) {
    if (!(E >= L.Emin) || !(E > 0)) return 0.0;
    E = E < L.Epeak ? E : L.Epeak;
    return exp(L.logpre - L.power * log(E) + L.expo / E);
}
G3D_HD uint64_t mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double uniform01(uint64_t key) { return double(mix64(key) >> 11) * (1.0 / 9007199254740992.0); }

// Monte Carlo field ionization during dt (ionize, sim_stream.hpp:80-101): sequential levels with exponential
// waiting times; each event frees an electron at the ion (a copy with q = -1 into the born list).
__device__ void ionize(const StreamArgs& c, const StrmDev& S, long i, double E1, double E0, double dt) {
    const int sp = S.sp[i];
    const IonDevC& I = c.ions[sp - SP_ION];
    if (!I.ionizing || (E1 < I.Emin && E0 < I.Emin)) return;
    const uint64_t key = mix64(c.sv->key_step ^ ((uint64_t(c.n) << 8) | uint64_t(c.pass)));   // ion_key_slice
    const uint64_t base = mix64(key ^ mix64(S.id[i]));            // ion_key_particle(key_slice, id)
    int Z = int(floor(S.q[i] + 0.5));
    const int Z0 = Z;
    unsigned draw = 0;
    double tleft = dt;
    while (Z < I.Zmax) {
        const AdkDev& L = c.adk[I.off + Z];
        const double w = 0.5 * (adk_rate(L, E1) + adk_rate(L, E0));
        if (!(w > 0)) break;
        const double tw = -log(1.0 - uniform01(base + draw++)) / w;
        if (tw > tleft) break;
        tleft -= tw; ++Z;
        const int j = atomicAdd(c.bcnt, 1);
        if (j < c.bcap) {
            const StrmDev Bn = c.sd[1];
            Bn.x[j] = S.x[i]; Bn.y[j] = S.y[i]; Bn.zeta[j] = S.zeta[i]; Bn.px[j] = S.px[i]; Bn.py[j] = S.py[i];
            Bn.pz[j] = S.pz[i]; Bn.w[j] = S.w[i]; Bn.z[j] = S.z[i]; Bn.q[j] = -1; Bn.qm[j] = -1;
            Bn.alive[j] = 1; Bn.sp[j] = SP_FREED + (sp - SP_ION); Bn.id[j] = S.id[i];
        }
    }
    if (Z != Z0 && !c.dry) { S.q[i] = Z; S.qm[i] = Z / I.mass; }
}

// The deposit of one particle in one half-cell: f (v_x, v_y, v_z, 1) at (x, y) (stream_deposit)
struct DepReq {
    double x, y, f, vx, vy, vz;
    bool on;
    bool f32;                  // the mixed form on the Fourier y grid: FP32 deposit weights from ff, fv (sdeposit_warp)
    float ff, fv[3];
};

// one streaming particle through half-cell n (stream_one, sim_stream.hpp:104-171); its deposit is returned to
// the caller, the rare second deposit of a trapped particle that joins the beam list is made here. A predictor
// pass (c.dry) computes and deposits the same but leaves the particle as it was, so every pass of a half-cell
// starts from the same state without a copy of the particles.
// ION: some species ionizes (else the field magnitudes and the ADK sampling are left out); LASER: the analytic
// plane wave is on. Both are fixed for a run; the variants without them hold fewer registers.
// EX: exact fields (FP64 form, Fourier y, neither ionization nor the analytic wave): the gathers from the FP64 planes.
// REC: the variant that writes the adjoint's record (c.recd, first pass), launched only when recording.
template <bool F32, bool ION, bool LASER, bool YF, bool EX = false, bool REC = false>
__device__ __forceinline__ DepReq stream_one(const StreamArgs& c, const StrmDev& S, long i) {
    DepReq d{0, 0, 0, 0, 0, 0, false, false, 0.f, {0.f, 0.f, 0.f}};
    const Geo& g = c.g;
    const int n = c.n;
    const double zn = g.zs[n], zn1 = g.zs[n + 1], h = zn1 - zn;
    // The whole state is loaded at once, before any branch or store: a load behind a branch waits for the
    // branch's own load, and a load behind a store to another array of the state (which the compiler must
    // assume may alias it) waits for that store. Every index below the count is a valid slot of every array.
    typedef double A;     // the push arithmetic: FP64 in both forms (the mixed form's FP32 push gave 3-4x its F error)
    int alive = S.alive[i];
    const int sp = S.sp[i];
    const double zeta = S.zeta[i], x = S.x[i], y = S.y[i], z = S.z[i];
    const double px_ = S.px[i], py_ = S.py[i], pz_ = S.pz[i], qm_ = S.qm[i];
    const double qw = S.q[i] * S.w[i];
    const double sTrap = c.sv->sTrap, s1 = c.sv->s1;
    if constexpr (REC) {
        if (c.recd && c.pass == 0) {                 // the adjoint's record: the state entering half-cell n
            const RecDev R = *c.recd;
            double* xr = R.x + 7 * R.rs * long(n + 1) + i;
            xr[0] = x; xr[R.rs] = y; xr[2 * R.rs] = zeta; xr[3 * R.rs] = z;
            xr[4 * R.rs] = px_; xr[5 * R.rs] = py_; xr[6 * R.rs] = pz_;
            R.a[R.rs * long(n + 1) + i] = alive;
        }
    }
    if (alive == 6) {                 // waiting: joins the march inside the half-cell that holds its zeta
        if (zeta > zn) { alive = 1; if (!c.dry) S.alive[i] = 1; }
        else return d;
    }
    if (alive != 1) return d;
    const double hl = zeta >= zn1 - 1e-9 * h ? h : (zeta - zn > 0 ? zeta - zn : 0.0);
    const bool ion = sp >= SP_ION && sp < SP_FREED;
    if (ion && !c.ions[sp - SP_ION].mobile) {        // fixed ion: its charge, then the ionization
        const double f = qw * hl / (c.Delta * h * g.dx);
        if (f != 0) d = DepReq{x, y, f, 0, 0, 0, true, false, 0.f, {0.f, 0.f, 0.f}};
        if (!c.dry) S.zeta[i] = zn;
        if constexpr (ION) {
            const double E1 = field_abs<F32, YF>(c, x, y, z, zeta), E0 = field_abs<F32, YF>(c, x, y, z, zn);
            ionize(c, S, i, E1, E0, hl);
        }
        return d;
    }
    // the push in FP64 in both forms: the mixed form gathers FP32 fields and deposits into FP32 planes, but its Boris
    // steps, gamma, 1 - v_z and velocities are FP64 (measured on the laser-plasma workload: FP32 arithmetic here put
    // 3-4x more error into F over 1-5 s-steps, for 2.6 % less time in this kernel)
    const A px = A(px_), py = A(py_), pz = A(pz_), qm = A(qm_);
    const A g0 = sqrt(A(1) + px * px + py * py + pz * pz), ig0 = A(1) / g0;
    const A omv0 = (A(1) + px * px + py * py) / (g0 * (g0 + pz));     // 1 - v_z, no cancellation
    const A dt0 = A(hl) / omv0;
    const A hd = A(0.5) * dt0 * ig0;
    const double xm = x + double(hd * px), ym = y + double(hd * py);
    const double zm = z + double(hd * pz), zetam = zeta - 0.5 * hl;
    A E[3], B[3];
    const bool mid = c.Fmid && zeta == zn1;                       // the whole half-cell: the midpoint fields
    if (qm_ == 0) {
        // a neutral atom: the Boris pushes below leave u exactly as it is whatever the (finite) fields, so they
        // are not gathered (the gas of an ionization-injection run is mostly neutral until the laser arrives)
        for (int k = 0; k < 3; ++k) { E[k] = A(0); B[k] = A(0); }
    } else if (F32 && mid && !LASER && !c.ext.any()) {
        if constexpr (F32) {
            float Ef[3], Bf[3];
            if constexpr (YF) sgather_mid_f32(c, wrapx(g, xm), wrapy<YF>(g, ym), Ef, Bf);
            else sgather_mid_fh_f32(c, wrapx(g, xm), ym, Ef, Bf);
            for (int k = 0; k < 3; ++k) { E[k] = A(Ef[k]); B[k] = A(Bf[k]); }
        }
    } else {
        double Ed[3], Bd[3], Ee[3], Be[3];
        if (YF && mid) sgather_mid<F32>(c, wrapx(g, xm), wrapy<YF>(g, ym), Ed, Bd);   // free-hand: Fmid is FP32-only
        else if (EX) sgather_exact(c, wrapx(g, xm), wrapy<YF>(g, ym), zetam, Ed, Bd);
        else sgather<F32, YF>(c, wrapx(g, xm), wrapy<YF>(g, ym), zetam, Ed, Bd);
        if constexpr (LASER) {
            c.laser.field(xm + c.sv->X0, zm, zm - (zetam - c.zc), Ee, Be);
            for (int k = 0; k < 3; ++k) { Ed[k] += Ee[k]; Bd[k] += Be[k]; }
        }
        if (c.ext.any()) add_external(c.ext, xm + c.sv->X0, ym + c.sv->Y0, zm, Bd);   // sim_stream.hpp:133
        for (int k = 0; k < 3; ++k) { E[k] = A(Ed[k]); B[k] = A(Bd[k]); }
    }
    A ux = px, uy = py, uz = pz;
    boris<A>(ux, uy, uz, E, B, qm, dt0);
    A g1 = sqrt(A(1) + ux * ux + uy * uy + uz * uz);
    A dt = A(2) * A(hl) / (omv0 + (A(1) + ux * ux + uy * uy) / (g1 * (g1 + uz)));
    ux = px; uy = py; uz = pz;
    boris<A>(ux, uy, uz, E, B, qm, dt);
    g1 = sqrt(A(1) + ux * ux + uy * uy + uz * uz);
    A ig1 = A(1) / g1;
    A vx = A(0.5) * (px * ig0 + ux * ig1), vy = A(0.5) * (py * ig0 + uy * ig1), vz = A(0.5) * (pz * ig0 + uz * ig1);
    double zeta_end = zn;
    bool trapped = false;
    if (z + double(vz * dt) >= sTrap) {       // advanced trap_advance steps inside this half-cell: trapped
        const double vv = double(vz) > 1e-3 ? double(vz) : 1e-3;
        const double dtp = (sTrap - z) / vv > 0 ? (sTrap - z) / vv : 0.0;
        ux = px; uy = py; uz = pz;
        boris<A>(ux, uy, uz, E, B, qm, A(dtp));
        g1 = sqrt(A(1) + ux * ux + uy * uy + uz * uz);
        ig1 = A(1) / g1;
        vx = A(0.5) * (px * ig0 + ux * ig1); vy = A(0.5) * (py * ig0 + uy * ig1); vz = A(0.5) * (pz * ig0 + uz * ig1);
        dt = A(dtp);
        zeta_end = zeta - (1 - double(vz)) * dtp;
        trapped = true;
    }
    const double xn = x + double(vx * dt), yn = y + double(vy * dt);
    if (!c.dry) {
        S.x[i] = xn; S.y[i] = yn;
        S.z[i] = trapped ? s1 : z + double(vz * dt);
        S.px[i] = ux; S.py[i] = uy; S.pz[i] = uz;
        S.zeta[i] = zeta_end;
    }
    if constexpr (F32) {
        if constexpr (YF) {           // FP32 deposit: the factor 1 / (Delta h dx) taken once per half-cell
            const float ff = float(qw * c.dep_norm) * float(dt);
            if (ff != 0.f) d = DepReq{0.5 * (x + xn), 0.5 * (y + yn), 0, 0, 0, 0, true, true, ff, {float(vx), float(vy), float(vz)}};
        } else {
            const double f = qw * double(dt) / (c.Delta * h * g.dx);
            if (f != 0) d = DepReq{0.5 * (x + xn), 0.5 * (y + yn), f, double(vx), double(vy), double(vz), true, false, 0.f, {0.f, 0.f, 0.f}};
        }
    } else {
        const double f = qw * double(dt) / (c.Delta * h * g.dx);
        if (f != 0) d = DepReq{0.5 * (x + xn), 0.5 * (y + yn), f, double(vx), double(vy), double(vz), true, false, 0.f, {0.f, 0.f, 0.f}};
    }
    if (!YF && (yn < c.ylo || yn > c.yhi)) {        // free-hand y: reached the cell at a wall
        if (!c.dry) S.alive[i] = 0;
        return d;
    }
    if constexpr (ION)
        if (ion && !trapped && c.ions[sp - SP_ION].ionizing)
            ionize(c, S, i, field_abs<F32, YF>(c, xm, ym, zm, zeta), field_abs<F32, YF>(c, xm, ym, zm, zn), double(dt));
    if (trapped) {
        if (!c.dry) S.alive[i] = 5;
        const double vze = double(uz * ig1);
        if (vze >= c.vz_beam)         // joins the beam list: its beam current of level s1 from now on
            sdeposit<F32, YF>(c, xn, yn, qw / (h * g.dx * vze), double(ux * ig1), double(uy * ig1), vze);
    }
    return d;
}

// The deposit of a warp's particles on the Fourier y grid, the adds of particles that share a TSC stencil summed in
// registers first. Lanes whose stencils start at the same grid point form a group (a match on the stencil's first
// point): on the plasma lattice the electron and the ion of a lattice point and the neighbouring points that round to
// the same node, about three lanes. A tree inside each group (every round, each lane of even rank in the group adds
// the value of the next remaining member above it, and the odd ranks leave) leaves the group's sum with its lowest
// lane, which alone issues the adds: a third of the reductions into L2, which bound the streaming push (measured:
// without its deposit adds the FP64 push takes 36 % less time, the mixed one 21 %). Row by row (three points of
// three components), so that few values are live. Every lane of the warp calls it; `on` false: nothing to deposit.
template <bool F32>
__device__ __forceinline__ void sdeposit_warp(const StreamArgs& c, const DepReq& d, bool on, int lane) {
    typedef typename std::conditional<F32, float, double>::type T;
    const Geo& g = c.g;
    int ix[3], jn[3];
    T wx[3], wn[3], fa, v3[3];
    if constexpr (F32) {
        tsc_f32(d.x, c.inv_dx, g.nx, ix, wx);
        tsc_f32(d.y, c.inv_dy, g.ny, jn, wn);
        fa = d.ff * float(g.iA[0]);
        v3[0] = d.fv[0]; v3[1] = d.fv[1]; v3[2] = d.fv[2];
    } else {
        tsc_periodic(d.x, g.dx, g.nx, ix, wx);
        tsc_periodic(d.y, g.dy, g.ny, jn, wn);
        fa = d.f;
        v3[0] = d.vx; v3[1] = d.vy; v3[2] = d.vz;
    }
    const double ia0 = g.iA[0];
    const unsigned all = 0xffffffffu;
    const int key = on ? jn[0] * g.nx + ix[0] : -1 - lane;
    const unsigned peers = __match_any_sync(all, key);
    const unsigned rank0 = unsigned(__popc(peers & ((1u << lane) - 1u)));
    const unsigned above0 = peers & ~((2u << lane) - 1u);
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        T a[3][3];
#pragma unroll
        for (int u = 0; u < 3; ++u) {
            T w;
            if constexpr (F32) w = fa * wx[u] * wn[v];
            else w = fa * wx[u] * wn[v] * ia0;
#pragma unroll
            for (int k = 0; k < 3; ++k) a[u][k] = on ? w * v3[k] : T(0);
        }
        unsigned above = above0, rank = rank0;
        while (__any_sync(all, above != 0u)) {
            const int nxt = above ? __ffs(int(above)) - 1 : lane;
            const bool take = above != 0u && !(rank & 1u);
#pragma unroll
            for (int u = 0; u < 3; ++u)
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const T t = __shfl_sync(all, a[u][k], nxt);
                    if (take) a[u][k] += t;
                }
            const unsigned gone = __ballot_sync(all, (rank & 1u) != 0u);
            if (rank & 1u) above = 0u;
            above &= ~gone;
            rank >>= 1;
        }
        if (on && rank0 == 0u) {
#pragma unroll
            for (int u = 0; u < 3; ++u) {
                const long k = long(jn[v]) * g.nx + ix[u];
                if constexpr (F32) {
                    atomicAdd(reinterpret_cast<float4*>(c.Jf) + k, make_float4(a[u][0], a[u][1], a[u][2], 0.f));
                } else {
                    atomicAdd(&c.J[k], a[u][0]); atomicAdd(&c.J[g.nk + k], a[u][1]); atomicAdd(&c.J[2 * g.nk + k], a[u][2]);
                }
            }
        }
    }
    if (on) {
        if constexpr (F32) sdeposit_lines(c, d.ff, ix, jn, [&](int u, int v) { return fa * wx[u] * wn[v]; });
        else sdeposit_lines(c, d.f, ix, jn, [&](int u, int v) { return d.f * wx[u] * wn[v] * ia0; });
    }
}

// One thread per streaming particle, a fixed grid striding over their count (which freed electrons raise; it is
// read on the device). The deposit adds go straight to global memory: without a use of the old value they are
// fire-and-forget reductions in L2, cheaper for the SM than accumulating in shared memory the many adds that
// neighbouring lattice particles make to the same points. F32 (the mixed form): the gathers in FP32 from FP32 field
// planes, the deposit into FP32 planes; the push arithmetic and the particle state stay FP64.
constexpr int ST_NT = 128;
// Resident CTAs per SM the register budget of the plain variant is sized for, by form. With the per-thread deposit,
// 5 (96 registers) against 6 (80) gave 55.8 against 57.8 us per launch in the mixed form and 89.7 against 91.8 us in
// the FP64 form (laser-plasma workload, one box); 4, 7 and 8 were slower. With the warp-summed deposit the mixed form
// prefers 6 (47.1 and 46.6 against 47.7 and 48.9 us, 4: 52.6) and the FP64 form keeps 5 (66.5 against 66.8 at 6, 71.4
// at 4; 256 x 256 x 128 case, all builds alternated in one call).
#ifndef G3D_STREAM_MINB
#define G3D_STREAM_MINB 5
#endif
#ifndef G3D_STREAM_MINB_F32
#define G3D_STREAM_MINB_F32 6
#endif
// YF: the Fourier y grid (true) or the free-hand one, fixed for a run, so that each variant holds only its own grid's
// gathers and deposits (fewer registers and no local arrays).
template <bool F32, bool ION, bool LASER, bool YF, bool EX = false, bool REC = false>
__global__ void __launch_bounds__(ST_NT, (ION || LASER) ? 4 : F32 ? G3D_STREAM_MINB_F32 : G3D_STREAM_MINB) k_stream(StreamArgs c,
                                                                                       const long* __restrict__ nstrm) {
    const StrmDev S = c.sd[0];
    const long n = *nstrm;
    const int lane = int(threadIdx.x & 31u);
    // the warp strides as a whole (its lanes meet in the warp's deposit): b is the warp's first particle
    for (long b = long(blockIdx.x) * ST_NT + long(threadIdx.x & ~31u); b < n; b += long(gridDim.x) * ST_NT) {
        const long i = b + lane;
        DepReq d{0, 0, 0, 0, 0, 0, false, false, 0.f, {0.f, 0.f, 0.f}};
        if (i < n) d = stream_one<F32, ION, LASER, YF, EX, REC>(c, S, i);
        if constexpr (YF) {
            const bool warp = d.on && (!F32 || d.f32);   // F32: a fixed ion's charge alone takes the plain deposit
            sdeposit_warp<F32>(c, d, warp, lane);
            if (d.on && !warp) sdeposit<F32, YF>(c, d.x, d.y, d.f, d.vx, d.vy, d.vz);
        } else if (d.on) {
            sdeposit<F32, YF>(c, d.x, d.y, d.f, d.vx, d.vy, d.vz);
        }
    }
}
template <bool F32, bool YF>
static void stream_launch_y(Ctx& c, const StreamArgs& a, unsigned blocks) {
    PlasmaState& P = *c.pl;
    const bool ion = P.any_ionizing, las = c.laser.on != 0;
    if constexpr (!F32 && YF) {
        if (a.Fd && !ion && !las) {                  // exact fields (the adjoint's forward, writing its record when asked)
            k_stream<false, false, false, true, true, true><<<blocks, ST_NT, 0, c.stream>>>(a, P.nstrm_dev.p);
            return;
        }
    }
    if constexpr (F32 && YF) {
        if (a.recd && !ion && !las) {                // the mixed form's forward of the adjoint, writing its record
            k_stream<true, false, false, true, false, true><<<blocks, ST_NT, 0, c.stream>>>(a, P.nstrm_dev.p);
            return;
        }
    }
    if (ion && las) k_stream<F32, true, true, YF><<<blocks, ST_NT, 0, c.stream>>>(a, P.nstrm_dev.p);
    else if (ion) k_stream<F32, true, false, YF><<<blocks, ST_NT, 0, c.stream>>>(a, P.nstrm_dev.p);
    else if (las) k_stream<F32, false, true, YF><<<blocks, ST_NT, 0, c.stream>>>(a, P.nstrm_dev.p);
    else k_stream<F32, false, false, YF><<<blocks, ST_NT, 0, c.stream>>>(a, P.nstrm_dev.p);
}
template <bool F32>
static void stream_launch(Ctx& c, const StreamArgs& a, unsigned blocks) {
    if (c.yf) stream_launch_y<F32, true>(c, a, blocks);
    else stream_launch_y<F32, false>(c, a, blocks);
}

// ---------------------------------------------------------------- spectra of the streaming current
// rows: per row, FFT along x of jx + i jy (split) and of jz -> three half rows in T0..T2
template <int NX, class JT>
__global__ void __launch_bounds__(128) k_ss_rows(Geo g, JT* __restrict__ J, cpx* __restrict__ T0, cpx* __restrict__ T1,
                                                cpx* __restrict__ T2, int clear, int* __restrict__ bcnt) {
    using S = FftShape<NX>;
    constexpr int LPC = 128 / S::T, RS = row_stride<NX>(), H = NX / 2 + 1;
    extern __shared__ cpx sm[];
    cpx* a0 = sm;
    cpx* a1 = sm + LPC * RS;
    const int tid = threadIdx.x, r0 = blockIdx.x * LPC;
    const long nk = g.nk;
    // every load first, then the clears for the next pass's deposit, then shared memory: a clear between two loads
    // would keep the second waiting for the first (the compiler cannot move a load above a store it may alias)
    constexpr int EPT = LPC * NX / 128;
    double jx[EPT], jy[EPT], jz[EPT];
#pragma unroll
    for (int u = 0; u < EPT; ++u) {
        const int e = tid + u * 128, rr = e / NX, p = e - rr * NX, row = r0 + rr;
        jx[u] = jy[u] = jz[u] = 0;
        if (row < g.ny) {
            const long i = long(row) * NX + p;
            if constexpr (std::is_same<JT, float4>::value) {            // interleaved per point (FP32, Fourier y)
                const float4 v = J[i];
                jx[u] = v.x; jy[u] = v.y; jz[u] = v.z;
            } else {
                jx[u] = J[i]; jy[u] = J[nk + i]; jz[u] = J[2 * nk + i];
            }
        }
    }
    if (clear) {
#pragma unroll
        for (int u = 0; u < EPT; ++u) {
            const int e = tid + u * 128, rr = e / NX, p = e - rr * NX, row = r0 + rr;
            if (row >= g.ny) continue;
            const long i = long(row) * NX + p;
            if constexpr (std::is_same<JT, float4>::value) J[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            else { J[i] = JT(0); J[nk + i] = JT(0); J[2 * nk + i] = JT(0); }
        }
    }
#pragma unroll
    for (int u = 0; u < EPT; ++u) {
        const int e = tid + u * 128, rr = e / NX, p = e - rr * NX;
        a0[rr * RS + p + (p >> 3)] = C(jx[u], jy[u]);
        a1[rr * RS + p + (p >> 3)] = C(jz[u], 0.0);
    }
    if (bcnt && blockIdx.x == 0 && tid == 0) *bcnt = 0;          // the freed electrons of the next pass
    __syncthreads();
    const int r = tid / S::T, t = tid - r * S::T;
    {
        decltype(a0) const ls_[2] = {a0, a1};
        fft_lines<NX, 2>(ls_, RowAddr{r * RS}, t, g.twx);
    }
    for (int e = tid; e < LPC * H; e += 128) {
        const int rr = e / H, kx = e - rr * H, row = r0 + rr;
        if (row >= g.ny) continue;
        const int km = (NX - kx) % NX;
        const cpx z = a0[rr * RS + kx + (kx >> 3)], zm = conj(a0[rr * RS + km + (km >> 3)]);
        const cpx d = z - zm;
        const long o = long(row) * H + kx;
        T0[o] = 0.5 * (z + zm);
        T1[o] = 0.5 * C(d.y, -d.x);
        T2[o] = a1[rr * RS + kx + (kx >> 3)];
    }
}
// columns: FFT along y, filters and smoothing -> jsn (3 half planes)
template <int NY, int CW>
__global__ void __launch_bounds__(CW * FftShape<NY>::T) k_ss_cols(Geo g, const cpx* __restrict__ T0, const cpx* __restrict__ T1,
                                                                  const cpx* __restrict__ T2, cpx* __restrict__ out, double a2, int keep0,
                                                                  int filter) {
    using S = FftShape<NY>;
    extern __shared__ cpx sm[];
    cpx* s0 = sm;
    cpx* s1 = sm + ColTile<NY, CW>::size;
    cpx* s2 = sm + 2 * ColTile<NY, CW>::size;
    const int c0 = blockIdx.x * CW, tid = threadIdx.x, nthr = CW * S::T, H = g.H;
#pragma unroll
    for (int u = 0; u < NY / S::T; ++u) {      // unrolled: the loads of all elements in flight together
        const int e = tid + u * nthr, p = e / CW, c = e - p * CW, kx = c0 + c;
        cpx u0 = C(0), u1 = C(0), u2 = C(0);
        if (kx < H) { const long o = long(p) * H + kx; u0 = T0[o]; u1 = T1[o]; u2 = T2[o]; }
        s0[ColTile<NY, CW>::at(p, c)] = u0; s1[ColTile<NY, CW>::at(p, c)] = u1; s2[ColTile<NY, CW>::at(p, c)] = u2;
    }
    __syncthreads();
    const int c = tid % CW, t = tid / CW;
    {
        decltype(s0) const ls_[3] = {s0, s1, s2};
        fft_lines<NY, 3>(ls_, RowAddr{c * ColTile<NY, CW>::RS}, t, g.twy);
    }
    const long nkh = g.nkh;
    constexpr int EPT = NY / S::T;            // elements of a thread (e = tid + u nthr)
    double f[EPT];
#pragma unroll
    for (int u = 0; u < EPT; ++u) {            // the filter factors first: their loads wait for no store
        const int e = tid + u * nthr, p = e / CW, kx = c0 + (e - p * CW);
        f[u] = 0;
        if (kx < H) {
            const double k2 = g.kxs[kx] * g.kxs[kx] + g.kys[p] * g.kys[p];
            f[u] = !filter ? 1.0 : (kx == 0 && p == 0 && !keep0) ? 0.0 : g.filt[kx] * g.filty[p] / (1 + a2 * k2);
        }
    }
#pragma unroll
    for (int u = 0; u < EPT; ++u) {
        const int e = tid + u * nthr, p = e / CW, cc = e - p * CW, kx = c0 + cc;
        if (kx >= H) continue;
        const long o = long(p) * H + kx;
        out[o] = f[u] * s0[ColTile<NY, CW>::at(p, cc)];
        out[nkh + o] = f[u] * s1[ColTile<NY, CW>::at(p, cc)];
        out[2 * nkh + o] = f[u] * s2[ColTile<NY, CW>::at(p, cc)];
    }
}

// ---------------------------------------------------------------- elementwise steps of the half-cell
// jk(m) += nw - old; old <- nw (the `replace` of sim_plasma.cpp:257-264), three half planes
template <class T>
__global__ void k_replace(T* __restrict__ jx, T* __restrict__ jy, T* __restrict__ jz, cpx* __restrict__ old,
                          const cpx* __restrict__ nw, long nkh) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < nkh; i += long(gridDim.x) * blockDim.x) {
        jx[i] = narrow<T>(widen(jx[i]) + nw[i] - old[i]);
        jy[i] = narrow<T>(widen(jy[i]) + nw[nkh + i] - old[nkh + i]);
        jz[i] = narrow<T>(widen(jz[i]) + nw[2 * nkh + i] - old[2 * nkh + i]);
        old[i] = nw[i]; old[nkh + i] = nw[nkh + i]; old[2 * nkh + i] = nw[2 * nkh + i];
    }
}
// after a pass: replace the streaming part of jk(n) by jsn (old = sin); with the extrapolating predictor and
// n >= 1 the prediction of half-cell n-1: tmp = js0(n-1) + d + w (d - dl), d = jsn - js0(n); replace(n-1, pin, tmp)
template <class T>
__device__ __forceinline__ void replace_pred_mode(const PlasmaPtrs& p, int n, int extrap, double w, long i) {
    const long nkh = p.nkh;
    const long hp = long(n + 1) * nkh, hq = long(n) * nkh;        // planes of half-cells n and n-1 (a = 0)
    cpx u[3];
    for (int k = 0; k < 3; ++k) u[k] = p.jsn[k * nkh + i];
    T* jk[3] = {static_cast<T*>(p.jkx), static_cast<T*>(p.jky), static_cast<T*>(p.jkz)};
    for (int k = 0; k < 3; ++k) {
        jk[k][hp + i] = narrow<T>(widen(jk[k][hp + i]) + u[k] - p.sin_[k * nkh + i]);
        p.sin_[k * nkh + i] = u[k];
    }
    if (extrap && n >= 1) {
        const cpx* s0[3] = {p.js0x, p.js0y, p.js0z};
        for (int k = 0; k < 3; ++k) {
            const cpx d = u[k] - s0[k][hp + i];
            const cpx t = s0[k][hq + i] + d + w * (d - p.dl[k * nkh + i]);
            jk[k][hq + i] = narrow<T>(widen(jk[k][hq + i]) + t - p.pin[k * nkh + i]);
            p.pin[k * nkh + i] = t;
        }
    }
}
template <class T>
__global__ void k_replace_pred(PlasmaPtrs p, int n, int extrap, double w) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < p.nkh; i += long(gridDim.x) * blockDim.x)
        replace_pred_mode<T>(p, n, extrap, w, i);
}
// half-cell n is final (sim_plasma.cpp:381-403): R at slice n+1 corrected for the prediction it used; the
// change s0 -> s1 kept for the extrapolation; the current kept as the prediction of the next step
__device__ __forceinline__ void correct_mode(const PlasmaPtrs& p, cpx* Rx, cpx* Ry, int n, double q, int own, long i) {
    const long nkh = p.nkh;
    const long hp = long(n + 1) * nkh, sp1 = long(n + 1) * nkh;
    cpx* s0[3] = {p.js0x, p.js0y, p.js0z};
    const cpx u0 = p.jsn[i], u1 = p.jsn[nkh + i], u2 = p.jsn[2 * nkh + i];
    if (own) {
        Rx[sp1 + i] = Rx[sp1 + i] - q * (u0 - p.si0[i]);
        Ry[sp1 + i] = Ry[sp1 + i] - q * (u1 - p.si0[nkh + i]);
    }
    p.dl[i] = u0 - s0[0][hp + i]; p.dl[nkh + i] = u1 - s0[1][hp + i]; p.dl[2 * nkh + i] = u2 - s0[2][hp + i];
    s0[0][hp + i] = u0; s0[1][hp + i] = u1; s0[2][hp + i] = u2;
}
__global__ void k_correct(PlasmaPtrs p, cpx* __restrict__ Rx, cpx* __restrict__ Ry, int n, double q, int own) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < p.nkh; i += long(gridDim.x) * blockDim.x)
        correct_mode(p, Rx, Ry, n, q, own, i);
}
// the march of slice n, one mode (march_point, sim_kernels.hpp:173-210, one rank: b = N, no boundary slice). The
// current pointers carry no __restrict__: the fused kernel below writes jk just before.
template <class T>
__device__ __forceinline__ void march_slice_mode(const Geo& g, cpx* Rx, cpx* Ry, T* Ez, T* Bz, T* Lx, T* Ly, const T* j0x,
                                                 const T* j0y, const T* jkx, const T* jky, const T* jkz, double D, int n, long i) {
    const long nk = g.nkh;
    const int kxi = int(i % g.H), j = int(i / g.H);
    const double kx = g.kxd[kxi], ky = g.kyd[j], k2 = kx * kx + ky * ky, wl = g.wlo[n], wu = g.whi[n];
    const long o = long(n - g.a) * nk + i, od = o, ou = o + nk;
    const cpx Jx = wl * (widen(j0x[od]) + widen(jkx[od])) + wu * (widen(j0x[ou]) + widen(jkx[ou]));
    const cpx Jy = wl * (widen(j0y[od]) + widen(jky[od])) + wu * (widen(j0y[ou]) + widen(jky[ou]));
    const cpx ez = widen(Ez[o]), bz = widen(Bz[o]);
    const cpx Rsx = Rx[o] + D * (ik(kx, ez) + ik(ky, bz)) - D * Jx;
    const cpx Rsy = Ry[o] + D * (ik(ky, ez) - ik(kx, bz)) - D * Jy;
    if (n == g.N - 1) {
        Rx[o] = Rsx; Ry[o] = Rsy;
        Ez[o] = narrow<T>(C(0)); Bz[o] = narrow<T>(C(0)); Lx[o] = narrow<T>(C(0)); Ly[o] = narrow<T>(C(0));
        return;
    }
    const long pp = o + nk;
    const cpx pRx = Rx[pp], pRy = Ry[pp], pEz = widen(Ez[pp]), pBz = widen(Bz[pp]), pLx = widen(Lx[pp]), pLy = widen(Ly[pp]);
    const double h = g.hcg[n + 2];
    const cpx upx = widen(jkx[ou]), upy = widen(jky[ou]), upz = widen(jkz[ou]);
    const cpx Lsx = pLx - 0.25 * h * (ik(kx, pEz) - ik(ky, pBz)) - 0.5 * h * upx;
    const cpx Lsy = pLy - 0.25 * h * (ik(kx, pBz) + ik(ky, pEz)) - 0.5 * h * upy;
    const cpx Cp = 0.5 * (ik(kx, pRy + pLy) - ik(ky, pRx + pLx));
    const cpx Qp = -0.5 * ik(kx, pRx - pLx) + 0.5 * ik(ky, pLy - pRy);
    const cpx SB = ik(kx, Rsy) + ik(kx, Lsy) - ik(ky, Rsx) - ik(ky, Lsx);
    const cpx SE = -ik(kx, Rsx) + ik(kx, Lsx) + ik(ky, Lsy) - ik(ky, Rsy);
    const double den = 1 + 0.25 * h * (D + 0.25 * h) * k2;
    const cpx Bzn = (pBz - 0.5 * h * Cp - 0.25 * h * SB) / den;
    const cpx Ezn = (pEz - 0.5 * h * Qp - 0.25 * h * SE - h * upz) / den;
    Ez[o] = narrow<T>(Ezn); Bz[o] = narrow<T>(Bzn);
    Rx[o] = Rsx + D * (ik(kx, Ezn) + ik(ky, Bzn)); Ry[o] = Rsy + D * (ik(ky, Ezn) - ik(kx, Bzn));
    Lx[o] = narrow<T>(Lsx - 0.25 * h * (ik(kx, Ezn) - ik(ky, Bzn)));
    Ly[o] = narrow<T>(Lsy - 0.25 * h * (ik(kx, Bzn) + ik(ky, Ezn)));
}
template <class T>
__global__ void __launch_bounds__(128) k_march_slice(Geo g, cpx* Rx, cpx* Ry, T* Ez, T* Bz, T* Lx, T* Ly, const T* j0x, const T* j0y,
                                                    const T* jkx, const T* jky, const T* jkz, double D, int n) {
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < g.nkh) march_slice_mode<T>(g, Rx, Ry, Ez, Bz, Lx, Ly, j0x, j0y, jkx, jky, jkz, D, n, i);
}
// ---------------------------------------------------------------- one pass's column work, fused (Fourier y)
// k_pass_cols: one CTA per k_x column, one thread per k_y (per mode). (1) Each thread loads what the march of its
// mode reads (the loads of the replace and march below; they are in flight during the transform). (2) The y
// transforms of the streaming current's three row spectra, the filters and the smoothing (k_ss_cols) -> jsn. (3)
// Per mode the replace and the march of slice n (replace_pred_mode + march_slice_mode in one). (4) The inverse y transforms of slice n's new
// R, L, E_z, B_z from shared memory (k_rf_cols, or k_rf_cols_f in FP32 for the mixed form) -> W, which the rows
// kernel of the real fields takes. One launch and one pass over the spectra instead of three. The transforms
// run on three groups of FftShape<NY>::T threads (a line or a line pair each); all threads take the barriers.
template <int NY, class T, class WT>
__global__ void __launch_bounds__(NY) k_pass_cols(PlasmaPtrs p, Geo g, const cpx* __restrict__ T0, const cpx* __restrict__ T1,
                                                  const cpx* __restrict__ T2, double a2, int keep0, cpx* __restrict__ Rx,
                                                  cpx* __restrict__ Ry, T* __restrict__ Ez, T* __restrict__ Bz, T* __restrict__ Lx,
                                                  T* __restrict__ Ly, const T* __restrict__ j0x, const T* __restrict__ j0y,
                                                  double D, int n, int extrap, double w, const cpx* __restrict__ bk,
                                                  const WT* __restrict__ twi, WT* __restrict__ W0, WT* __restrict__ W1,
                                                  WT* __restrict__ W2, WT* __restrict__ W3, WT* __restrict__ W4, WT* __restrict__ W5) {
    using S = FftShape<NY>;
    using Tile = ColTile<NY, 1>;
    extern __shared__ double smp[];
    cpx* fl[3] = {reinterpret_cast<cpx*>(smp), reinterpret_cast<cpx*>(smp) + Tile::size, reinterpret_cast<cpx*>(smp) + 2 * Tile::size};
    WT* ib = reinterpret_cast<WT*>(reinterpret_cast<cpx*>(smp) + 3 * Tile::size);
    const int kxi = blockIdx.x, j = threadIdx.x;
    const long nk = g.nkh, i = long(j) * g.H + kxi;
    // the transforms: three groups of S::T threads, one line (forward) or one line pair (inverse) each
    const int grp = j / S::T < 2 ? j / S::T : 2, tl = j - (j / S::T) * S::T;
    const bool act = j < 3 * S::T;
    // (1) the march's loads
    const long hp = long(n + 1) * nk + i, hq = long(n) * nk + i;      // half-cells n and n-1
    T* jk[3] = {static_cast<T*>(p.jkx), static_cast<T*>(p.jky), static_cast<T*>(p.jkz)};
    const bool pred = extrap && n >= 1;
    cpx sn[3], kp[3], kq[3], s0p[3], s0q[3], dl[3], pn[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        sn[k] = p.sin_[k * nk + i];
        kp[k] = widen(jk[k][hp]); kq[k] = widen(jk[k][hq]);
        if (pred) {
            const cpx* s0[3] = {p.js0x, p.js0y, p.js0z};
            s0p[k] = s0[k][hp]; s0q[k] = s0[k][hq]; dl[k] = p.dl[k * nk + i]; pn[k] = p.pin[k * nk + i];
        }
    }
    const double kx = g.kxd[kxi], ky = g.kyd[j], k2 = kx * kx + ky * ky, wl = g.wlo[n], wu = g.whi[n];
    const long o = long(n - g.a) * nk + i, ou = o + nk;
    const cpx j0xd = widen(j0x[o]), j0xu = widen(j0x[ou]), j0yd = widen(j0y[o]), j0yu = widen(j0y[ou]);
    const cpx rx = bk ? bk[i] : Rx[o], ry = bk ? bk[nk + i] : Ry[o];
    const cpx ez = bk ? widen(narrow<T>(bk[2 * nk + i])) : widen(Ez[o]), bz = bk ? widen(narrow<T>(bk[3 * nk + i])) : widen(Bz[o]);
    const bool front = n == g.N - 1;
    cpx pRx = C(0), pRy = C(0), pEz = C(0), pBz = C(0), pLx = C(0), pLy = C(0);
    if (!front) {
        const long pp = o + nk;
        pRx = Rx[pp]; pRy = Ry[pp]; pEz = widen(Ez[pp]); pBz = widen(Bz[pp]); pLx = widen(Lx[pp]); pLy = widen(Ly[pp]);
    }
    const double h = front ? 0.0 : g.hcg[n + 2];
    // (2) the current's column, transformed and filtered
    const long ot = long(j) * g.H + kxi;
    fl[0][Tile::at(j, 0)] = T0[ot]; fl[1][Tile::at(j, 0)] = T1[ot]; fl[2][Tile::at(j, 0)] = T2[ot];
    __syncthreads();
    {
        cpx* const ls_[1] = {fl[grp]};
        fft_lines_some<NY, 1>(ls_, RowAddr{0}, tl, g.twy, act);
    }
    const double k2f = g.kxs[kxi] * g.kxs[kxi] + g.kys[j] * g.kys[j];
    const double f = (kxi == 0 && j == 0 && !keep0) ? 0.0 : g.filt[kxi] * g.filty[j] / (1 + a2 * k2f);
    cpx u[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) { u[k] = f * fl[k][Tile::at(j, 0)]; p.jsn[k * nk + i] = u[k]; }
    // (3) replace(n, sin, jsn), the prediction of n-1, the march of slice n
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const T np_ = narrow<T>(kp[k] + u[k] - sn[k]);
        jk[k][hp] = np_; kp[k] = widen(np_);
        p.sin_[k * nk + i] = u[k];
        if (pred) {
            const cpx d = u[k] - s0p[k];
            const cpx t = s0q[k] + d + w * (d - dl[k]);
            const T nq_ = narrow<T>(kq[k] + t - pn[k]);
            jk[k][hq] = nq_; kq[k] = widen(nq_);
            p.pin[k * nk + i] = t;
        }
    }
    const cpx Jx = wl * (j0xd + kq[0]) + wu * (j0xu + kp[0]);
    const cpx Jy = wl * (j0yd + kq[1]) + wu * (j0yu + kp[1]);
    const cpx Rsx = rx + D * (ik(kx, ez) + ik(ky, bz)) - D * Jx;
    const cpx Rsy = ry + D * (ik(ky, ez) - ik(kx, bz)) - D * Jy;
    cpx nv[6];                                        // slice n as stored: R_x, R_y, L_x, L_y, E_z, B_z
    if (front) {
        Rx[o] = Rsx; Ry[o] = Rsy;
        Ez[o] = narrow<T>(C(0)); Bz[o] = narrow<T>(C(0)); Lx[o] = narrow<T>(C(0)); Ly[o] = narrow<T>(C(0));
        nv[0] = Rsx; nv[1] = Rsy;
        nv[2] = nv[3] = nv[4] = nv[5] = widen(narrow<T>(C(0)));
    } else {
        const cpx upx = kp[0], upy = kp[1], upz = kp[2];
        const cpx Lsx = pLx - 0.25 * h * (ik(kx, pEz) - ik(ky, pBz)) - 0.5 * h * upx;
        const cpx Lsy = pLy - 0.25 * h * (ik(kx, pBz) + ik(ky, pEz)) - 0.5 * h * upy;
        const cpx Cp = 0.5 * (ik(kx, pRy + pLy) - ik(ky, pRx + pLx));
        const cpx Qp = -0.5 * ik(kx, pRx - pLx) + 0.5 * ik(ky, pLy - pRy);
        const cpx SB = ik(kx, Rsy) + ik(kx, Lsy) - ik(ky, Rsx) - ik(ky, Lsx);
        const cpx SE = -ik(kx, Rsx) + ik(kx, Lsx) + ik(ky, Lsy) - ik(ky, Rsy);
        const double den = 1 + 0.25 * h * (D + 0.25 * h) * k2;
        const cpx Bzn = (pBz - 0.5 * h * Cp - 0.25 * h * SB) / den;
        const cpx Ezn = (pEz - 0.5 * h * Qp - 0.25 * h * SE - h * upz) / den;
        const T ezs = narrow<T>(Ezn), bzs = narrow<T>(Bzn);
        const cpx nRx = Rsx + D * (ik(kx, Ezn) + ik(ky, Bzn)), nRy = Rsy + D * (ik(ky, Ezn) - ik(kx, Bzn));
        const T lxs = narrow<T>(Lsx - 0.25 * h * (ik(kx, Ezn) - ik(ky, Bzn)));
        const T lys = narrow<T>(Lsy - 0.25 * h * (ik(kx, Bzn) + ik(ky, Ezn)));
        Ez[o] = ezs; Bz[o] = bzs; Rx[o] = nRx; Ry[o] = nRy; Lx[o] = lxs; Ly[o] = lys;
        nv[0] = nRx; nv[1] = nRy; nv[2] = widen(lxs); nv[3] = widen(lys); nv[4] = widen(ezs); nv[5] = widen(bzs);
    }
    // (4) the real fields' y transforms of slice n (pairs as k_rf_cols: R -> W0, W1; L -> W2, W3; E_z, B_z -> W4, W5)
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        if constexpr (std::is_same<WT, cpx>::value) ib[k * Tile::size + Tile::at(j, 0)] = conj(nv[k]);
        else ib[k * Tile::size + Tile::at(j, 0)] = conj(to_f(nv[k]));
    }
    __syncthreads();
    {
        WT* const ls_[2] = {ib + (2 * grp) * Tile::size, ib + (2 * grp + 1) * Tile::size};
        fft_lines_some<NY, 2>(ls_, RowAddr{0}, tl, twi, act);
    }
    WT* out[6] = {W0, W1, W2, W3, W4, W5};
    const long ow = long(n) * nk + long(j) * g.H + kxi;
#pragma unroll
    for (int k = 0; k < 6; ++k) out[k][ow] = conj(ib[k * Tile::size + Tile::at(j, 0)]);
}
// freed electrons join the march (appended after the streaming particles; the count stays on the device)
__global__ void k_born_append(const StrmDev* __restrict__ sd, const int* __restrict__ bcnt, int bcap, long* __restrict__ nstrm_dev,
                              int* __restrict__ overflow) {
    const StrmDev S = sd[0], Bn = sd[1];
    const int cnt = *bcnt;
    const long base = *nstrm_dev;
    if (cnt > bcap) { if (blockIdx.x == 0 && threadIdx.x == 0) *overflow = 1; return; }
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < cnt; k += gridDim.x * blockDim.x) {
        const long d = base + k;
        S.x[d] = Bn.x[k]; S.y[d] = Bn.y[k]; S.zeta[d] = Bn.zeta[k]; S.px[d] = Bn.px[k]; S.py[d] = Bn.py[k];
        S.pz[d] = Bn.pz[k]; S.w[d] = Bn.w[k]; S.z[d] = Bn.z[k]; S.q[d] = Bn.q[k]; S.qm[d] = Bn.qm[k];
        S.alive[d] = Bn.alive[k]; S.sp[d] = Bn.sp[k]; S.id[d] = Bn.id[k];
    }
}
__global__ void k_count_add(long* __restrict__ nstrm_dev, const int* __restrict__ bcnt, int bcap) {
    const int cnt = *bcnt;
    if (cnt <= bcap) *nstrm_dev += cnt;
}

// ---------------------------------------------------------------- per half-cell set-up, fused
// Start of half-cell n (sim_plasma.cpp:236-262): sin <- pin and si0 <- pin (copy_in); the prediction of half-cell
// pred_m starts from its level s0 with the prediction buffer cleared: jk(pred_m) += js0(pred_m), pin <- js0(pred_m)
// (pred_m < 0: none); the slice's R_x, R_y, E_z, B_z saved for the passes (backup).
template <class T>
__device__ __forceinline__ void slice_prologue_mode(const PlasmaPtrs& p, cpx* sin_, cpx* si0, cpx* bk, const cpx* Rx, const cpx* Ry,
                                                    const T* Ez, const T* Bz, long o, int pred_m, int copy_in, int backup, long i) {
    const long nkh = p.nkh;
    const long hm = long(pred_m + 1) * nkh;
    T* jk[3] = {static_cast<T*>(p.jkx), static_cast<T*>(p.jky), static_cast<T*>(p.jkz)};
    const cpx* s0[3] = {p.js0x, p.js0y, p.js0z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const long q = k * nkh + i;
        if (copy_in) { const cpx v = p.pin[q]; sin_[q] = v; si0[q] = v; }
        if (pred_m >= 0) {
            const cpx t = s0[k][hm + i];
            jk[k][hm + i] = narrow<T>(widen(jk[k][hm + i]) + t);
            p.pin[q] = t;
        }
    }
    if (backup) {
        bk[i] = Rx[o + i]; bk[nkh + i] = Ry[o + i];
        bk[2 * nkh + i] = widen(Ez[o + i]); bk[3 * nkh + i] = widen(Bz[o + i]);
    }
}
template <class T>
__global__ void k_slice_prologue(PlasmaPtrs p, cpx* __restrict__ sin_, cpx* __restrict__ si0, cpx* __restrict__ bk,
                                 const cpx* __restrict__ Rx, const cpx* __restrict__ Ry, const T* __restrict__ Ez,
                                 const T* __restrict__ Bz, long o, int pred_m, int copy_in, int backup) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < p.nkh; i += long(gridDim.x) * blockDim.x)
        slice_prologue_mode<T>(p, sin_, si0, bk, Rx, Ry, Ez, Bz, o, pred_m, copy_in, backup, i);
}
// half-cell n final (correct_mode) and the prologue of half-cell n-1 (slice_prologue_mode, copy_in), per mode in
// one thread. Every value is loaded before anything is stored: the correction reads si0 before the prologue
// refills it, the prologue's slice n-1 and half-cell n-1 are not touched by the correction (slice n+1, half-cell
// n), and pin and jk are each read before they are written; so the stores see the values of the sequential
// code, and the ~26 loads of a mode wait together instead of behind stores they might alias.
template <class T>
__global__ void k_correct_prologue(PlasmaPtrs p, cpx* __restrict__ Rx, cpx* __restrict__ Ry, int n, double q, int own,
                                   cpx* __restrict__ sin_, cpx* __restrict__ si0, cpx* __restrict__ bk, const T* __restrict__ Ez,
                                   const T* __restrict__ Bz, long o_next, int pred_m, int backup) {
    const long nkh = p.nkh, hp = long(n + 1) * nkh, hm = long(pred_m + 1) * nkh;
    cpx* s0[3] = {p.js0x, p.js0y, p.js0z};
    T* jk[3] = {static_cast<T*>(p.jkx), static_cast<T*>(p.jky), static_cast<T*>(p.jkz)};
    const bool pred = pred_m >= 0;
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < nkh; i += long(gridDim.x) * blockDim.x) {
        cpx u[3], sh[3], pn[3], t[3], jm[3], sx = C(0), sy = C(0), rx = C(0), ry = C(0);
        cpx b0 = C(0), b1 = C(0), b2 = C(0), b3 = C(0);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            u[k] = p.jsn[k * nkh + i]; sh[k] = s0[k][hp + i]; pn[k] = p.pin[k * nkh + i];
            t[k] = pred ? s0[k][hm + i] : C(0);
            jm[k] = pred ? widen(jk[k][hm + i]) : C(0);
        }
        if (own) { sx = p.si0[i]; sy = p.si0[nkh + i]; rx = Rx[hp + i]; ry = Ry[hp + i]; }
        if (backup) { b0 = Rx[o_next + i]; b1 = Ry[o_next + i]; b2 = widen(Ez[o_next + i]); b3 = widen(Bz[o_next + i]); }
        if (own) { Rx[hp + i] = rx - q * (u[0] - sx); Ry[hp + i] = ry - q * (u[1] - sy); }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            p.dl[k * nkh + i] = u[k] - sh[k];
            s0[k][hp + i] = u[k];
            sin_[k * nkh + i] = pn[k]; si0[k * nkh + i] = pn[k];
            if (pred) { jk[k][hm + i] = narrow<T>(jm[k] + t[k]); p.pin[k * nkh + i] = t[k]; }
        }
        if (backup) { bk[i] = b0; bk[nkh + i] = b1; bk[2 * nkh + i] = b2; bk[3 * nkh + i] = b3; }
    }
}
// Start of a pass on the free-hand y grid: the slice restored from the backup (restore), the streaming-current
// planes and the count of freed electrons cleared. (Fourier y: the fused march reads the backup, the rows kernel
// of the spectra clears the planes and the count.)
template <class T, class JT>
__global__ void k_pass_prologue(const cpx* __restrict__ bk, cpx* __restrict__ Rx, cpx* __restrict__ Ry, T* __restrict__ Ez,
                                T* __restrict__ Bz, long o, long nkh, JT* __restrict__ J, long nj, int* __restrict__ bcnt,
                                int restore) {
    const long t0 = long(blockIdx.x) * blockDim.x + threadIdx.x, st = long(gridDim.x) * blockDim.x;
    if (restore)
        for (long i = t0; i < nkh; i += st) {
            Rx[o + i] = bk[i]; Ry[o + i] = bk[nkh + i];
            Ez[o + i] = narrow<T>(bk[2 * nkh + i]); Bz[o + i] = narrow<T>(bk[3 * nkh + i]);
        }
    for (long i = t0; i < nj; i += st) J[i] = JT(0);
    if (t0 == 0) *bcnt = 0;
}

// ---------------------------------------------------------------- count of particles in one state
__global__ void k_count_state(const int32_t* __restrict__ alive, long n, const long* __restrict__ n_dev, int state,
                              int* __restrict__ out) {
    const long m = n_dev ? *n_dev : n;
    int k = 0;
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += long(gridDim.x) * blockDim.x) k += alive[i] == state;
    for (int o = 16; o > 0; o >>= 1) k += __shfl_down_sync(0xffffffffu, k, o);
    if ((threadIdx.x & 31) == 0 && k) atomicAdd(out, k);
}

// ---------------------------------------------------------------- the fresh plasma lattice
// Lattice point L: its position (x, y), row height hy and density n with the host loader's operations, no
// contraction into FMAs (the host code has none), so the same points get particles and the same values.
__device__ __forceinline__ void lattice_point(const LatticeArgs& a, long L, double& x, double& y, double& hy, double& n) {
    const int a2 = int(L % a.px);
    long r = L / a.px;
    const int b2 = int(r % a.py);
    r /= a.py;
    const int i = int(r % a.nx), j = a.j0 + int(r / a.nx);
    double y0 = __dmul_rn(double(j), a.dy);
    hy = a.dy;
    if (a.yn) { y0 = a.yn[j]; hy = __dsub_rn(a.yn[j + 1], a.yn[j]); }
    x = __dmul_rn(__dadd_rn(double(i), __ddiv_rn(__dadd_rn(double(a2), 0.5), double(a.px))), a.dx);
    y = __dadd_rn(y0, __dmul_rn(__ddiv_rn(__dadd_rn(double(b2), 0.5), double(a.py)), hy));
    const double xx = __dadd_rn(x, a.X0), yy = __dadd_rn(y, a.Y0);
    const double r2 = __dadd_rn(__dmul_rn(xx, xx), __dmul_rn(yy, yy));
    n = 0;
    if (r2 >= a.rmax2) return;
    const double g = a.parabolic ? __dadd_rn(1.0, __ddiv_rn(__dmul_rn(a.depth, r2), a.rc2)) : 1.0;
    if (__dmul_rn(a.f, g) > 0) n = __dmul_rn(__dmul_rn(a.n0, a.f), g);
}
__global__ void k_lattice_flags(LatticeArgs a, long npts, int* __restrict__ flag) {
    for (long L = long(blockIdx.x) * blockDim.x + threadIdx.x; L <= npts; L += long(gridDim.x) * blockDim.x) {
        if (L == npts) { flag[L] = 0; continue; }
        double x, y, hy, n;
        lattice_point(a, L, x, y, hy, n);
        flag[L] = n > 0;
    }
}
__global__ void k_lattice_fill(LatticeArgs a, long npts, const int* __restrict__ off, StrmDev S) {
    for (long L = long(blockIdx.x) * blockDim.x + threadIdx.x; L < npts; L += long(gridDim.x) * blockDim.x) {
        double x, y, hy, n;
        lattice_point(a, L, x, y, hy, n);
        if (!(n > 0)) continue;
        const double w = __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(n, a.dx), hy), a.Delta), double(a.px * a.py));
        long k = long(off[L]) * a.m;
        auto put = [&](double ww, double q, double qm, int sp) {
            S.x[k] = x; S.y[k] = y; S.zeta[k] = a.zf; S.px[k] = 0; S.py[k] = 0; S.pz[k] = 0;
            S.w[k] = ww; S.z[k] = a.s0; S.q[k] = q; S.qm[k] = qm; S.alive[k] = 1; S.sp[k] = sp;
            S.id[k] = a.id0 + uint64_t(k);
            ++k;
        };
        if (a.electrons) put(w, -1, -1, SP_PLASMA);
        for (int t = 0; t < a.nion; ++t) put(__dmul_rn(a.ion_atoms[t], w), a.ion_q[t], a.ion_qm[t], a.ion_sp[t]);
    }
}
// ---------------------------------------------------------------- trapped particles, split on the device
// A trapped streaming particle (alive 5) joins the beam when v_z = p_z / gamma >= vz_beam, else it streams again in
// the next march (Simulation::march_plasma's trapping, src/sim_plasma.cpp:404-433). v_z with the host's
// operations, so the split is the host's.
__device__ __forceinline__ bool trapped_fast(const StrmDev& S, long i, double vzb) {
    const double px = S.px[i], py = S.py[i], pz = S.pz[i];
    const double g = __dsqrt_rn(__dadd_rn(__dadd_rn(__dadd_rn(1.0, __dmul_rn(px, px)), __dmul_rn(py, py)), __dmul_rn(pz, pz)));
    return __ddiv_rn(pz, g) >= vzb;
}
__global__ void k_trap_flags(StrmDev S, const long* __restrict__ n_dev, long cap, double vzb, int fast, int* __restrict__ flag) {
    const long n = *n_dev < cap ? *n_dev : cap;
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i <= cap; i += long(gridDim.x) * blockDim.x)
        flag[i] = i < n && S.alive[i] == 5 && trapped_fast(S, i, vzb) == (fast != 0);
}
// the flagged particles in list order into T from T[base]: z = s1, and (slow) alive 6, waiting for their zeta
__global__ void k_trap_gather(StrmDev S, const int* __restrict__ flag, const int* __restrict__ off, long cap, StrmDev T, long base,
                              int slow, double s1) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < cap; i += long(gridDim.x) * blockDim.x) {
        if (!flag[i]) continue;
        const long k = base + off[i];
        T.x[k] = S.x[i]; T.y[k] = S.y[i]; T.zeta[k] = S.zeta[i]; T.px[k] = S.px[i]; T.py[k] = S.py[i]; T.pz[k] = S.pz[i];
        T.w[k] = S.w[i]; T.z[k] = s1; T.q[k] = S.q[i]; T.qm[k] = S.qm[i]; T.alive[k] = slow ? 6 : S.alive[i]; T.sp[k] = S.sp[i];
        T.id[k] = S.id[i];
    }
}
// the freed-electron capacity the joining ions need: sum of Zmax - round(q) over the ions of ionizing species
__global__ void k_join_cap(StrmDev J, long n, const IonDevC* __restrict__ ions, int nion, unsigned long long* __restrict__ out) {
    unsigned long long a = 0;
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const int sp = J.sp[i];
        if (sp >= SP_ION && sp < SP_FREED && sp - SP_ION < nion && ions[sp - SP_ION].ionizing)
            a += (unsigned long long)(ions[sp - SP_ION].Zmax - llround(J.q[i]));
    }
    for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
    if ((threadIdx.x & 31) == 0 && a) atomicAdd(out, a);
}
// x, y of the joining particles on the device moved with the window
__global__ void k_join_shift(StrmDev J, long n, double sx, double sy) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) { J.x[i] -= sx; J.y[i] -= sy; }
}

// ---------------------------------------------------------------- launchers
static unsigned ew_blocks(long n) {
    long b = (n + 255) / 256;
    return unsigned(b < 148 * 8 ? (b < 1 ? 1 : b) : 148 * 8);
}
void launch_stream(Ctx& c, const StreamArgs& a) {
    PlasmaState& P = *c.pl;
    if (P.s.cap <= 0) return;
    const int tok = c.prof_begin("stream");
    const unsigned blocks = 148 * 16;             // fixed (the kernel strides over the count on the device), so
                                                  // that the graph of the slice loop does not depend on the list
    if (c.f32s) stream_launch<true>(c, a, blocks);
    else stream_launch<false>(c, a, blocks);
    c.check_launch("k_stream");
    c.prof_end(tok);
}
// Half spectra of three real planes J[0..2] (jx, jy, jz layout) into out[0..2]; T is scratch (3 half planes).
template <int NX, class JT>
static void ss_rows(Ctx& c, JT* J, cpx* T, int clear = 0, int* bcnt = nullptr) {
    using S = FftShape<NX>;
    constexpr int LPC = 128 / S::T;
    const size_t smem = size_t(2) * LPC * row_stride<NX>() * sizeof(cpx);
    smem_attr(reinterpret_cast<const void*>(k_ss_rows<NX, JT>), smem);
    k_ss_rows<NX, JT><<<unsigned((c.ny + LPC - 1) / LPC), 128, smem, c.stream>>>(c.geo(), J, T, T + c.nkh, T + 2 * c.nkh, clear, bcnt);
    c.check_launch("k_ss_rows");
}
template <int NY>
static void ss_cols(Ctx& c, const cpx* T, cpx* out, double a2, int keep0, int filter) {
    constexpr int CW = 2;              // one slice: 2-column tiles spread its latency over 65 SMs (measured: 8 used 17)
    const size_t smem = size_t(3) * ColTile<NY, CW>::size * sizeof(cpx);
    smem_attr(reinterpret_cast<const void*>(k_ss_cols<NY, CW>), smem);
    k_ss_cols<NY, CW><<<unsigned((c.H + CW - 1) / CW), CW * FftShape<NY>::T, smem, c.stream>>>(
        c.geo(), T, T + c.nkh, T + 2 * c.nkh, out, a2, keep0, filter);
    c.check_launch("k_ss_cols");
}
void launch_stream_spectra(Ctx& c) {
    const int tok = c.prof_begin("stream_spectra");
    PlasmaState& P = *c.pl;
    const double a2 = P.cfg.smooth_length * P.cfg.smooth_length;
    if (c.f32s && c.yf) {
        float4* J4 = reinterpret_cast<float4*>(P.jsrf.p);
        G3D_DISPATCH_N(c.nx, NX, (ss_rows<NX, float4>(c, J4, P.tsp.p, 1, P.bcnt.p)));
    } else if (c.f32s) {
        G3D_DISPATCH_N(c.nx, NX, (ss_rows<NX, float>(c, P.jsrf.p, P.tsp.p, 1, P.bcnt.p)));
    } else {
        G3D_DISPATCH_N(c.nx, NX, (ss_rows<NX, double>(c, P.jsr.p, P.tsp.p, 1, P.bcnt.p)));
    }
    if (!c.yf) launch_ss_lines_fh(c, P.tsp.p, P.jsn.p, a2);           // free-hand y: filters along the y lines
    else G3D_DISPATCH_N(c.ny, NY, ss_cols<NY>(c, P.tsp.p, P.jsn.p, a2, P.box_mean ? 1 : 0, 1));
    c.prof_end(tok);
}
// plain transverse spectra (no filters) of three real planes: the grid-laser profile (free-hand y: the x spectra
// of the rows alone)
void launch_real_to_half3(Ctx& c, const double* J3, cpx* T3, cpx* out3) {
    double* J = const_cast<double*>(J3);      // read only: the rows kernel clears nothing here
    if (!c.yf) { G3D_DISPATCH_N(c.nx, NX, (ss_rows<NX, double>(c, J, out3))); return; }
    G3D_DISPATCH_N(c.nx, NX, (ss_rows<NX, double>(c, J, T3)));
    G3D_DISPATCH_N(c.ny, NY, ss_cols<NY>(c, T3, out3, 0.0, 1, 0));
}

// exclusive running sum of P.cflag[0 .. n] into P.coff (n + 1 entries); returns the total (a synchronisation)
static long scan_flags(Ctx& c, long n) {
    PlasmaState& P = *c.pl;
    if (n + 1 > 0x7fffffffL) throw Error(G3D_ERR_CAPACITY, "more than 2^31 items in one compaction");
    size_t tb = 0;
    G3D_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, P.cflag.p, P.coff.p, int(n + 1), c.stream));
    if (P.ctmp.n < tb) P.ctmp.alloc(tb, c.stream);
    G3D_CUDA(cub::DeviceScan::ExclusiveSum(P.ctmp.p, tb, P.cflag.p, P.coff.p, int(n + 1), c.stream));
    int h = 0;
    G3D_CUDA(cudaMemcpyAsync(&h, P.coff.p + n, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
    return h;
}
static void reserve_flags(Ctx& c, long n) {
    PlasmaState& P = *c.pl;
    if (long(P.cflag.n) < n + 1) {
        P.cflag.alloc(size_t(n + 1) + size_t(n + 1) / 8, c.stream);
        P.coff.alloc(P.cflag.n, c.stream);
    }
}
long launch_lattice_count(Ctx& c, const LatticeArgs& a, long npts) {
    reserve_flags(c, npts);
    k_lattice_flags<<<ew_blocks(npts + 1), 256, 0, c.stream>>>(a, npts, c.pl->cflag.p);
    c.check_launch("k_lattice_flags");
    return scan_flags(c, npts);
}
void launch_lattice_fill(Ctx& c, const LatticeArgs& a, long npts, StrmDev S) {
    k_lattice_fill<<<ew_blocks(npts), 256, 0, c.stream>>>(a, npts, c.pl->coff.p, S);
    c.check_launch("k_lattice_fill");
}
// The trapped streaming particles after a march: the slow ones appended on the device to the joining list (P.jb,
// P.njb), the fast ones into P.tr; returns how many fast ones.
long launch_trapped_split(Ctx& c, double s1) {
    PlasmaState& P = *c.pl;
    const long cap = P.s.cap;
    if (cap <= 0) return 0;
    reserve_flags(c, cap);
    const double vzb = P.cfg.vz_beam;
    k_trap_flags<<<ew_blocks(cap + 1), 256, 0, c.stream>>>(P.strm, P.nstrm_dev.p, cap, vzb, 0, P.cflag.p);
    c.check_launch("k_trap_flags");
    const long ns = scan_flags(c, cap);
    if (ns > 0) {
        if (P.jb.cap < P.njb + ns) {                     // grow, keeping the particles already there
            StrmBuf nb;
            nb.alloc(2 * (P.njb + ns) + 64, c.stream);
            if (P.njb > 0) {
                for (int m = 0; m < 10; ++m)
                    G3D_CUDA(cudaMemcpyAsync(nb.d.p + size_t(m) * nb.cap, P.jb.d.p + size_t(m) * P.jb.cap, size_t(P.njb) * 8,
                                             cudaMemcpyDeviceToDevice, c.stream));
                for (int m = 0; m < 2; ++m)
                    G3D_CUDA(cudaMemcpyAsync(nb.i.p + size_t(m) * nb.cap, P.jb.i.p + size_t(m) * P.jb.cap, size_t(P.njb) * 4,
                                             cudaMemcpyDeviceToDevice, c.stream));
                G3D_CUDA(cudaMemcpyAsync(nb.u.p, P.jb.u.p, size_t(P.njb) * 8, cudaMemcpyDeviceToDevice, c.stream));
            }
            G3D_CUDA(cudaStreamSynchronize(c.stream));
            std::swap(P.jb.d.p, nb.d.p); std::swap(P.jb.d.n, nb.d.n);
            std::swap(P.jb.i.p, nb.i.p); std::swap(P.jb.i.n, nb.i.n);
            std::swap(P.jb.u.p, nb.u.p); std::swap(P.jb.u.n, nb.u.n);
            std::swap(P.jb.v, nb.v); std::swap(P.jb.cap, nb.cap);             // nb frees the old buffers
        }
        k_trap_gather<<<ew_blocks(cap), 256, 0, c.stream>>>(P.strm, P.cflag.p, P.coff.p, cap, P.jb.v, P.njb, 1, s1);
        c.check_launch("k_trap_gather");
        P.njb += ns;
    }
    k_trap_flags<<<ew_blocks(cap + 1), 256, 0, c.stream>>>(P.strm, P.nstrm_dev.p, cap, vzb, 1, P.cflag.p);
    c.check_launch("k_trap_flags");
    const long nf = scan_flags(c, cap);
    if (nf > 0) {
        if (P.tr.cap < nf) P.tr.alloc(nf + nf / 4 + 64, c.stream);
        k_trap_gather<<<ew_blocks(cap), 256, 0, c.stream>>>(P.strm, P.cflag.p, P.coff.p, cap, P.tr.v, 0, 0, s1);
        c.check_launch("k_trap_gather");
    }
    return nf;
}
// The adjoint march across steps: the slow trapped particles of a march (in list order, as launch_trapped_split takes
// them) are the next march's joining particles (its list from index fresh). Their state adjoints (7 components of
// stride rs: x, y, zeta, z, p_x, p_y, p_z) go from the next march's list to this one's.
__global__ void k_join_adj_out(const double* __restrict__ lam, long rs, long fresh, long n, double* __restrict__ jl) {
    for (long j = long(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += long(gridDim.x) * blockDim.x)
        for (int q = 0; q < 7; ++q) jl[q * n + j] = lam[q * rs + fresh + j];
}
// the slow trapped particles of a recorded march: alive 5 after it and v_z of their final momenta below vzb (the
// operations of trapped_fast)
__global__ void k_join_flags(RecDev R, long np, double vzb, int* __restrict__ flag) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i <= np; i += long(gridDim.x) * blockDim.x) {
        bool f = false;
        if (i < np && R.a[i] == 5) {
            const double px = R.x[4 * R.rs + i], py = R.x[5 * R.rs + i], pz = R.x[6 * R.rs + i];
            const double g = __dsqrt_rn(__dadd_rn(__dadd_rn(__dadd_rn(1.0, __dmul_rn(px, px)), __dmul_rn(py, py)), __dmul_rn(pz, pz)));
            f = !(__ddiv_rn(pz, g) >= vzb);
        }
        flag[i] = f ? 1 : 0;
    }
}
__global__ void k_join_adj_in(const int* __restrict__ flag, const int* __restrict__ off, long cap, const double* __restrict__ jl,
                              long njl, double* __restrict__ lam, long rs) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < cap; i += long(gridDim.x) * blockDim.x) {
        if (!flag[i]) continue;
        const long j = off[i];
        if (j >= njl) continue;
        for (int q = 0; q < 7; ++q) lam[q * rs + i] = jl[q * njl + j];
    }
}
long launch_join_adjoint_out(Ctx& c, const double* lam, long rs, long fresh, long n, double* jl) {
    if (n <= 0) return 0;
    k_join_adj_out<<<ew_blocks(n), 256, 0, c.stream>>>(lam, rs, fresh, n, jl);
    c.check_launch("k_join_adj_out");
    return n;
}
long launch_join_adjoint_in(Ctx& c, const RecDev& rec, long np, const double* jl, long njl, double* lam) {
    PlasmaState& P = *c.pl;
    if (np <= 0) return 0;
    reserve_flags(c, np);
    k_join_flags<<<ew_blocks(np + 1), 256, 0, c.stream>>>(rec, np, P.cfg.vz_beam, P.cflag.p);
    c.check_launch("k_join_flags");
    const long ns = scan_flags(c, np);
    if (ns > 0 && njl > 0) {
        k_join_adj_in<<<ew_blocks(np), 256, 0, c.stream>>>(P.cflag.p, P.coff.p, np, jl, njl, lam, rec.rs);
        c.check_launch("k_join_adj_in");
    }
    return ns;
}
// The adjoint's record of the particles entering half-cell n (n < 0: after the last one, with their charges): the
// seven state columns and alive of every streaming particle at slot n + 1 of the record that rd points at; the count
// read on the device, so that the recording slice loop can run as a graph
__global__ void k_rec_particles(const StrmDev* __restrict__ sd, const long* __restrict__ n_dev, const RecDev* __restrict__ rd, int n,
                                const IonDevC* __restrict__ ions) {
    const StrmDev S = sd[0];
    const RecDev R = *rd;
    const long rs = R.rs, m = *n_dev < rs ? *n_dev : rs;
    double* x = R.x + 7 * rs * long(n + 1);
    int32_t* a = R.a + rs * long(n + 1);
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += long(gridDim.x) * blockDim.x) {
        x[i] = S.x[i]; x[rs + i] = S.y[i]; x[2 * rs + i] = S.zeta[i]; x[3 * rs + i] = S.z[i];
        x[4 * rs + i] = S.px[i]; x[5 * rs + i] = S.py[i]; x[6 * rs + i] = S.pz[i];
        a[i] = S.alive[i];
        if (n < 0) {
            const int sp = S.sp[i];
            const bool fixed = sp >= SP_ION && sp < SP_FREED && !ions[sp - SP_ION].mobile;
            R.q[i] = fixed ? 0.0 : S.q[i] * S.w[i];
            R.q[rs + i] = S.qm[i];
        }
    }
}
void launch_record_particles(Ctx& c, int n) {
    PlasmaState& P = *c.pl;
    k_rec_particles<<<ew_blocks(P.s.cap), 256, 0, c.stream>>>(P.sdev.p, P.nstrm_dev.p, P.recd.p, n, P.ion_dev.p);
    c.check_launch("k_rec_particles");
}
// ... and of the real fields of slice l after pass p (the exact FP64 planes, or the float F of the mixed form widened)
template <class FT>
__global__ void k_rec_fields(const RecDev* __restrict__ rd, const FT* __restrict__ Fd, long fpl, long nk, long l, int passes, int p) {
    double* f = rd->f + 6 * nk * (long(passes) * l + p);
    for (long e = long(blockIdx.x) * blockDim.x + threadIdx.x; e < 6 * nk; e += long(gridDim.x) * blockDim.x) {
        const long comp = e / nk, k = e - comp * nk;
        f[e] = double(Fd[comp * fpl + l * nk + k]);
    }
}
void launch_record_fields(Ctx& c, int l, int p) {
    PlasmaState& P = *c.pl;
    if (c.Fd.p)
        k_rec_fields<double><<<ew_blocks(6L * c.nk), 256, 0, c.stream>>>(P.recd.p, c.Fd.p, long(c.ns + 2) * c.nk, long(c.nk),
                                                                        long(l - c.a), P.cfg.iterations, p);
    else
        k_rec_fields<float><<<ew_blocks(6L * c.nk), 256, 0, c.stream>>>(P.recd.p, c.F.p, long(c.ns + 2) * c.nk, long(c.nk),
                                                                       long(l - c.a), P.cfg.iterations, p);
    c.check_launch("k_rec_fields");
}

long launch_join_cap(Ctx& c) {
    PlasmaState& P = *c.pl;
    if (P.njb == 0 || !P.any_ionizing) return 0;
    G3D_CUDA(cudaMemsetAsync(P.ucount.p, 0, sizeof(unsigned long long), c.stream));
    k_join_cap<<<ew_blocks(P.njb), 256, 0, c.stream>>>(P.jb.v, P.njb, P.ion_dev.p, int(P.ion_dev.n), P.ucount.p);
    c.check_launch("k_join_cap");
    unsigned long long h = 0;
    G3D_CUDA(cudaMemcpyAsync(&h, P.ucount.p, sizeof h, cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
    return long(h);
}
void launch_join_shift(Ctx& c, double sx, double sy) {
    PlasmaState& P = *c.pl;
    if (P.njb == 0) return;
    k_join_shift<<<ew_blocks(P.njb), 256, 0, c.stream>>>(P.jb.v, P.njb, sx, sy);
    c.check_launch("k_join_shift");
}

long count_state(Ctx& c, const int32_t* alive, long n, const long* n_dev, int state) {
    PlasmaState& P = *c.pl;
    G3D_CUDA(cudaMemsetAsync(P.tally.p, 0, sizeof(int), c.stream));
    k_count_state<<<148 * 4, 256, 0, c.stream>>>(alive, n, n_dev, state, P.tally.p);
    c.check_launch("k_count_state");
    int h = 0;
    G3D_CUDA(cudaMemcpyAsync(&h, P.tally.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
    return h;
}
void launch_slice_prologue(Ctx& c, int n, int pred_m, int copy_in, int backup) {
    PlasmaState& P = *c.pl;
    const long o = long(n - c.a) * c.nkh;
    const int tok = c.prof_begin("slice_prologue");
    if (c.mixed)
        k_slice_prologue<cpxf><<<ew_blocks(c.nkh), 256, 0, c.stream>>>(P.ptrs(c), P.jsin.p, P.jsi0.p, P.bk.p, c.Rx.p, c.Ry.p,
                                                                       c.mx.Ez.p, c.mx.Bz.p, o, pred_m, copy_in, backup);
    else
        k_slice_prologue<cpx><<<ew_blocks(c.nkh), 256, 0, c.stream>>>(P.ptrs(c), P.jsin.p, P.jsi0.p, P.bk.p, c.Rx.p, c.Ry.p,
                                                                      c.Ez.p, c.Bz.p, o, pred_m, copy_in, backup);
    c.check_launch("k_slice_prologue");
    c.prof_end(tok);
}
void launch_pass_prologue(Ctx& c, int n, int restore) {
    PlasmaState& P = *c.pl;
    const long o = long(n - c.a) * c.nkh, nj = 3 * long(c.nk);
    const int tok = c.prof_begin("pass_prologue");
    if (c.mixed)
        k_pass_prologue<cpxf, float><<<ew_blocks(nj), 256, 0, c.stream>>>(P.bk.p, c.Rx.p, c.Ry.p, c.mx.Ez.p, c.mx.Bz.p, o, c.nkh,
                                                                          P.jsrf.p, nj, P.bcnt.p, restore);
    else if (c.f32s)                  // free-hand y, mixed: FP64 spectra, FP32 streaming planes
        k_pass_prologue<cpx, float><<<ew_blocks(nj), 256, 0, c.stream>>>(P.bk.p, c.Rx.p, c.Ry.p, c.Ez.p, c.Bz.p, o, c.nkh,
                                                                         P.jsrf.p, nj, P.bcnt.p, restore);
    else
        k_pass_prologue<cpx, double><<<ew_blocks(nj), 256, 0, c.stream>>>(P.bk.p, c.Rx.p, c.Ry.p, c.Ez.p, c.Bz.p, o, c.nkh,
                                                                          P.jsr.p, nj, P.bcnt.p, restore);
    c.check_launch("k_pass_prologue");
    c.prof_end(tok);
}
void launch_replace(Ctx& c, int m, cpx* old, const cpx* nw) {
    const long h = long(m + 1) * c.nkh;
    if (c.mixed)
        k_replace<cpxf><<<ew_blocks(c.nkh), 256, 0, c.stream>>>(c.mx.jkx.p + h, c.mx.jky.p + h, c.mx.jkz.p + h, old, nw, c.nkh);
    else
        k_replace<cpx><<<ew_blocks(c.nkh), 256, 0, c.stream>>>(c.jkx.p + h, c.jky.p + h, c.jkz.p + h, old, nw, c.nkh);
    c.check_launch("k_replace");
}
void launch_replace_pred(Ctx& c, int n, int extrap, double w) {
    const int tok = c.prof_begin("replace_pred");
    if (c.mixed) k_replace_pred<cpxf><<<ew_blocks(c.nkh), 256, 0, c.stream>>>(c.pl->ptrs(c), n, extrap, w);
    else k_replace_pred<cpx><<<ew_blocks(c.nkh), 256, 0, c.stream>>>(c.pl->ptrs(c), n, extrap, w);
    c.check_launch("k_replace_pred");
    c.prof_end(tok);
}
void launch_correct(Ctx& c, int n, double q, int own) {
    k_correct<<<ew_blocks(c.nkh), 256, 0, c.stream>>>(c.pl->ptrs(c), c.Rx.p, c.Ry.p, n, q, own);
    c.check_launch("k_correct");
}
// correct(n) and slice_prologue(n - 1, pred_m, copy_in = 1, backup) in one launch
void launch_correct_prologue(Ctx& c, int n, double q, int own, int pred_m, int backup) {
    PlasmaState& P = *c.pl;
    const long o = long(n - 1 - c.a) * c.nkh;
    const int tok = c.prof_begin("correct_prologue");
    if (c.mixed)
        k_correct_prologue<cpxf><<<ew_blocks(c.nkh), 256, 0, c.stream>>>(P.ptrs(c), c.Rx.p, c.Ry.p, n, q, own, P.jsin.p, P.jsi0.p, P.bk.p,
                                                                         c.mx.Ez.p, c.mx.Bz.p, o, pred_m, backup);
    else
        k_correct_prologue<cpx><<<ew_blocks(c.nkh), 256, 0, c.stream>>>(P.ptrs(c), c.Rx.p, c.Ry.p, n, q, own, P.jsin.p, P.jsi0.p, P.bk.p,
                                                                        c.Ez.p, c.Bz.p, o, pred_m, backup);
    c.check_launch("k_correct_prologue");
    c.prof_end(tok);
}
void launch_march_slice(Ctx& c, double D, int n) {
    if (!c.yf) { launch_march_slice_fh(c, D, n); return; }
    const int tok = c.prof_begin("march_slice");
    const unsigned blocks = unsigned((c.nkh + 127) / 128);
    if (c.mixed) {
        MixedBufs& m = c.mx;
        k_march_slice<cpxf><<<blocks, 128, 0, c.stream>>>(c.geo(), c.Rx.p, c.Ry.p, m.Ez.p, m.Bz.p, m.Lx.p, m.Ly.p, m.j0x.p, m.j0y.p,
                                                          m.jkx.p, m.jky.p, m.jkz.p, D, n);
    } else {
        k_march_slice<cpx><<<blocks, 128, 0, c.stream>>>(c.geo(), c.Rx.p, c.Ry.p, c.Ez.p, c.Bz.p, c.Lx.p, c.Ly.p, c.j0x.p, c.j0y.p,
                                                         c.jkx.p, c.jky.p, c.jkz.p, D, n);
    }
    c.check_launch("k_march_slice");
    c.prof_end(tok);
}
template <int NY>
static void pass_cols(Ctx& c, double D, int n, int extrap, double w, int restore) {
    PlasmaState& P = *c.pl;
    const PlasmaPtrs pp = P.ptrs(c);
    const cpx* bk = restore ? P.bk.p : nullptr;
    const double a2 = P.cfg.smooth_length * P.cfg.smooth_length;
    const int keep0 = P.box_mean ? 1 : 0;
    const cpx* T = P.tsp.p;
    using Tile = ColTile<NY, 1>;
    if (c.mixed) {
        MixedBufs& m = c.mx;
        const size_t smem = 3 * Tile::size * sizeof(cpx) + 6 * Tile::size * sizeof(cpxf);
        smem_attr(reinterpret_cast<const void*>(k_pass_cols<NY, cpxf, cpxf>), smem);
        k_pass_cols<NY, cpxf, cpxf><<<unsigned(c.H), NY, smem, c.stream>>>(
            pp, c.geo(), T, T + c.nkh, T + 2 * c.nkh, a2, keep0, c.Rx.p, c.Ry.p, m.Ez.p, m.Bz.p, m.Lx.p, m.Ly.p, m.j0x.p, m.j0y.p,
            D, n, extrap, w, bk, m.twy.p, m.W[0].p, m.W[1].p, m.W[2].p, m.W[3].p, m.W[4].p, m.W[5].p);
    } else {
        const size_t smem = 9 * Tile::size * sizeof(cpx);
        smem_attr(reinterpret_cast<const void*>(k_pass_cols<NY, cpx, cpx>), smem);
        k_pass_cols<NY, cpx, cpx><<<unsigned(c.H), NY, smem, c.stream>>>(
            pp, c.geo(), T, T + c.nkh, T + 2 * c.nkh, a2, keep0, c.Rx.p, c.Ry.p, c.Ez.p, c.Bz.p, c.Lx.p, c.Ly.p, c.j0x.p, c.j0y.p,
            D, n, extrap, w, bk, c.twy.p, c.W[0].p, c.W[1].p, c.W[2].p, c.W[3].p, c.W[4].p, c.W[5].p);
    }
}
void launch_pass_cols(Ctx& c, double D, int n, int extrap, double w, int restore) {
    const int tok = c.prof_begin("pass_cols");
    G3D_DISPATCH_N(c.ny, NY, pass_cols<NY>(c, D, n, extrap, w, restore));
    c.check_launch("k_pass_cols");
    c.prof_end(tok);
}
void launch_stream_spectra_rows(Ctx& c) {
    const int tok = c.prof_begin("stream_spectra");
    PlasmaState& P = *c.pl;
    if (c.f32s) {
        float4* J4 = reinterpret_cast<float4*>(P.jsrf.p);
        G3D_DISPATCH_N(c.nx, NX, (ss_rows<NX, float4>(c, J4, P.tsp.p, 1, P.bcnt.p)));
    } else {
        G3D_DISPATCH_N(c.nx, NX, (ss_rows<NX, double>(c, P.jsr.p, P.tsp.p, 1, P.bcnt.p)));
    }
    c.prof_end(tok);
}
void launch_born_append(Ctx& c) {
    PlasmaState& P = *c.pl;
    k_born_append<<<ew_blocks(P.born_cap), 256, 0, c.stream>>>(P.sdev.p, P.bcnt.p, int(P.born_cap), P.nstrm_dev.p,
                                                               P.flags.p);
    c.check_launch("k_born_append");
    k_count_add<<<1, 1, 0, c.stream>>>(P.nstrm_dev.p, P.bcnt.p, int(P.born_cap));
    c.check_launch("k_count_add");
}

}  // namespace g3d
