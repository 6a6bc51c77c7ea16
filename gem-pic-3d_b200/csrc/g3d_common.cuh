// Common device/host definitions of libg3d: complex arithmetic on double2/float2, the zeta and
// y axis lookup, TSC weights, and the error plumbing of the C-ABI.
#pragma once
#include <cuda_runtime.h>
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#define G3D_HD __host__ __device__ __forceinline__

// ---------------------------------------------------------------- errors
// Host-side failures travel as g3d::Error (with the status code of include/g3d.h) up to the
// extern "C" layer, which turns them into a status and a message.
namespace g3d {
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
}  // namespace g3d

#define G3D_CUDA(call)                                                                                   \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess)                                                                           \
            throw g3d::Error(1, std::string(#call) + ": " + cudaGetErrorString(e_) + " (" + __FILE__ + \
                                    ":" + std::to_string(__LINE__) + ")");                             \
    } while (0)

// ---------------------------------------------------------------- complex numbers
// cpx is a double2 = {re, im}, the layout of the reference's `struct cpx` (src/portable.hpp:25).
typedef double2 cpx;
G3D_HD cpx C(double r, double i = 0.0) { return make_double2(r, i); }
G3D_HD cpx operator+(cpx a, cpx b) { return make_double2(a.x + b.x, a.y + b.y); }
G3D_HD cpx operator-(cpx a, cpx b) { return make_double2(a.x - b.x, a.y - b.y); }
G3D_HD cpx operator-(cpx a) { return make_double2(-a.x, -a.y); }
G3D_HD cpx operator*(cpx a, cpx b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
G3D_HD cpx operator*(double s, cpx a) { return make_double2(s * a.x, s * a.y); }
G3D_HD cpx operator*(cpx a, double s) { return make_double2(s * a.x, s * a.y); }
G3D_HD cpx operator/(cpx a, double s) { return make_double2(a.x / s, a.y / s); }
G3D_HD cpx cdiv(cpx a, cpx b) {
    const double d = b.x * b.x + b.y * b.y;
    return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
G3D_HD cpx conj(cpx a) { return make_double2(a.x, -a.y); }
// i k * z for a real k (the derivative factor of a spectral mode)
G3D_HD cpx ik(double k, cpx z) { return make_double2(-k * z.y, k * z.x); }
G3D_HD cpx mul_i(cpx z) { return make_double2(-z.y, z.x); }          // i z
G3D_HD cpx mul_mi(cpx z) { return make_double2(z.y, -z.x); }         // -i z

// cpxf is the FP32 complex of the mixed form (float2), with the same operators.
typedef float2 cpxf;
G3D_HD cpxf Cf(float r, float i = 0.0f) { return make_float2(r, i); }
G3D_HD cpxf operator+(cpxf a, cpxf b) { return make_float2(a.x + b.x, a.y + b.y); }
G3D_HD cpxf operator-(cpxf a, cpxf b) { return make_float2(a.x - b.x, a.y - b.y); }
G3D_HD cpxf operator-(cpxf a) { return make_float2(-a.x, -a.y); }
G3D_HD cpxf operator*(cpxf a, cpxf b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
G3D_HD cpxf operator*(float s, cpxf a) { return make_float2(s * a.x, s * a.y); }
G3D_HD cpxf operator*(cpxf a, float s) { return make_float2(s * a.x, s * a.y); }
G3D_HD cpxf operator/(cpxf a, float s) { return make_float2(a.x / s, a.y / s); }
G3D_HD cpxf conj(cpxf a) { return make_float2(a.x, -a.y); }
G3D_HD cpxf ik(float k, cpxf z) { return make_float2(-k * z.y, k * z.x); }
G3D_HD cpxf mul_i(cpxf z) { return make_float2(-z.y, z.x); }
G3D_HD cpxf mul_mi(cpxf z) { return make_float2(z.y, -z.x); }
G3D_HD cpx to_d(cpxf a) { return make_double2(a.x, a.y); }
G3D_HD cpxf to_f(cpx a) { return make_float2(float(a.x), float(a.y)); }

// Storage <-> arithmetic of the two forms: complex128 or complex64 storage, FP64 arithmetic.
G3D_HD cpx widen(cpx a) { return a; }
G3D_HD cpx widen(cpxf a) { return to_d(a); }
template <class T> G3D_HD T narrow(cpx a);
template <> G3D_HD cpx narrow<cpx>(cpx a) { return a; }
template <> G3D_HD cpxf narrow<cpxf>(cpx a) { return to_f(a); }

// Real type of a complex type.
template <class T> struct RealOf;
template <> struct RealOf<double2> { typedef double type; };
template <> struct RealOf<float2> { typedef float type; };
template <class T> G3D_HD T mk(typename RealOf<T>::type r, typename RealOf<T>::type i);
template <> G3D_HD double2 mk<double2>(double r, double i) { return make_double2(r, i); }
template <> G3D_HD float2 mk<float2>(float r, float i) { return make_float2(r, i); }

// ---------------------------------------------------------------- axes
// Location of a coordinate on a grid of nodes (uniform: direct; else binary search), with the end
// cells continued beyond the ends. Same contract as the reference's Axis::locate (src/grid.hpp:325-341).
struct AxisDev {
    const double* X;            // nodes (device), n of them
    int n, uniform;
    double x0, ih;
    // a non-uniform axis on the device: bins of width <= its smallest cell from X[0], bins[b] the last node at or
    // below the bin's start, so a point's cell is one table load and a step or two away (null: a binary search)
    const int* bins = nullptr;
    int nb = 0;
    double bih = 0;
    G3D_HD void locate(double x, int& i, double& f) const {
        if (uniform) { const double t = (x - x0) * ih; i = int(floor(t)); f = t - i; return; }
        if (x < X[0]) { const double t = (x - X[0]) / (X[1] - X[0]); i = int(floor(t)); f = t - i; return; }
        if (x >= X[n - 1]) {
            const double t = (x - X[n - 1]) / (X[n - 1] - X[n - 2]);
            const int k = int(floor(t));
            i = n - 1 + k; f = t - k; return;
        }
        int lo;
        if (bins) {            // the same cell as the search below: the one lo with X[lo] <= x < X[lo + 1]
            int b = int((x - X[0]) * bih);
            b = b < 0 ? 0 : (b >= nb ? nb - 1 : b);
            lo = bins[b];
            while (lo > 0 && X[lo] > x) --lo;
            while (lo < n - 2 && X[lo + 1] <= x) ++lo;
        } else {
            lo = 0;
            int hi = n - 1;
            while (hi - lo > 1) { const int m = (lo + hi) >> 1; if (X[m] <= x) lo = m; else hi = m; }
        }
        i = lo; f = (x - X[lo]) / (X[lo + 1] - X[lo]);
    }
};
// the bin table of a non-uniform axis (host): nb bins of width <= its smallest cell
inline std::vector<int> axis_bins(const std::vector<double>& X, double& bih) {
    const size_t n = X.size();
    double hmin = 1e300;
    for (size_t k = 0; k + 1 < n; ++k) hmin = std::min(hmin, X[k + 1] - X[k]);
    const double span = X[n - 1] - X[0];
    const long nb = std::max<long>(1, std::min<long>(long(std::ceil(span / hmin)) + 1, 1L << 22));
    bih = double(nb) / span;
    std::vector<int> bins(size_t(nb), 0);
    int lo = 0;
    for (long b = 0; b < nb; ++b) {
        const double start = X[0] + double(b) / bih;
        while (lo + 2 < int(n) && X[size_t(lo) + 1] <= start) ++lo;
        bins[size_t(b)] = lo;
    }
    return bins;
}

// Quadratic (TSC) weights of the three points around the nearest integer of the index coordinate
// (reference tsc_index, src/sim_kernels.hpp:21-26).
G3D_HD void tsc_weights(double xi, int idx[3], double w[3]) {
    const int i0 = int(floor(xi + 0.5));
    const double f = xi - i0;
    w[0] = 0.5 * (0.5 - f) * (0.5 - f);
    w[1] = 0.75 - f * f;
    w[2] = 0.5 * (0.5 + f) * (0.5 + f);
    idx[0] = i0 - 1; idx[1] = i0; idx[2] = i0 + 1;
}
// TSC on a periodic uniform grid with nodes at i*d (reference tsc, src/sim_kernels.hpp:28-31). The three
// indices are consecutive, so one modulo wraps the first and the other two follow by a compare (the same
// indices as wrapping each one).
G3D_HD void tsc_periodic(double x, double d, int n, int idx[3], double w[3]) {
    tsc_weights(x / d, idx, w);
    int b = idx[0] % n;
    if (b < 0) b += n;
    const int b1 = b + 1 == n ? 0 : b + 1;
    idx[0] = b; idx[1] = b1; idx[2] = b1 + 1 == n ? 0 : b1 + 1;
}

// TSC on the free-hand y grid in the index coordinate xi(y) (linear within a cell): nodes at the integers,
// half-nodes at the half-integers (stored at index j for j + 1/2); points outside 0..ny-1 are walls or beyond
// (reference tsc_y, src/sim_kernels.hpp:34-40).
G3D_HD void tsc_y(const AxisDev& ax, double y, int jn[3], double wn[3], int jh[3], double wh[3]) {
    int i; double f;
    ax.locate(y, i, f);
    const double xi = i + f;
    tsc_weights(xi, jn, wn);
    tsc_weights(xi - 0.5, jh, wh);
}
// the components of F that live on the half-nodes of the free-hand y grid: E_y, B_x, B_z
G3D_HD bool is_half(int comp) { return comp == 1 || comp == 3 || comp == 5; }

// fmod(x, L) for L > 0, bit for bit (fmod is exact): |x| < L is x itself, L <= |x| < 2L is x -+ L (exact by
// Sterbenz's lemma); larger |x| falls back to fmod. The periodic wrap of the reference's gather call,
// fmod(fmod(x, L) + L, L) (src/sim_kernels.hpp), meets only the first two cases in practice.
G3D_HD double fmod_pos(double x, double L) {
    const double a = fabs(x);
    if (a < L) return x;
    if (a < 2 * L) return x > 0 ? x - L : x + L;
    return fmod(x, L);
}
G3D_HD double wrap_periodic(double x, double L) { return fmod_pos(fmod_pos(x, L) + L, L); }
