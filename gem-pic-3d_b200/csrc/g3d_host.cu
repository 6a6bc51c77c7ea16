// Host side of libg3d: the context (grids, tables, buffers), the orchestration of a step, the bunch
// loader, checkpoints and the extern "C" entry points of include/g3d.h.
#include <limits>
#include <algorithm>
#include <mutex>
#include <map>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <random>
#include <thread>
#include "g3d_plasma.hpp"
#include "g3d_shard.hpp"

namespace g3d {

namespace {
constexpr double c_SI = 299792458.0, e_SI = 1.602176634e-19, me_SI = 9.1093837015e-31, eps0 = 8.8541878128e-12;
thread_local std::string g_create_err;

bool pow2_ok(int n) { return n >= 4 && n <= 512 && (n & (n - 1)) == 0; }
// the transverse sizes the transforms take: a power of two in 4..512, or three times one in 24..384 (k_fft.cuh)
bool fft_size_ok(int n) { return pow2_ok(n) || (n % 3 == 0 && n >= 24 && n <= 384 && ((n / 3) & (n / 3 - 1)) == 0); }
}  // namespace

// ---------------------------------------------------------------- context plumbing
Ctx::Ctx() = default;
Ctx::~Ctx() = default;

// The spectra other than R of one form: complex128 (FP64) or complex64 (mixed), with the raw current planes
// and the transform scratch; the other form's buffers are released.
static void alloc_spectra(Ctx& c, bool mixed) {
    const cudaStream_t s = c.stream;
    const size_t pl = size_t(c.nk), ph = size_t(c.nkh), ns = size_t(c.ns);
    if (mixed) {
        for (DevBuf<cpx>* p : {&c.Ez, &c.Bz, &c.Lx, &c.Ly, &c.j0x, &c.j0y, &c.jkx, &c.jky, &c.jkz, &c.jzg}) p->release();
        for (DevBuf<cpx>& w : c.W) w.release();
        c.jw.release();
        MixedBufs& m = c.mx;
        for (DevBuf<cpxf>* p : {&m.Ez, &m.Bz, &m.Lx, &m.Ly}) p->alloc(ns * ph, s);
        for (DevBuf<cpxf>* p : {&m.j0x, &m.j0y, &m.jkx, &m.jky, &m.jkz}) p->alloc((ns + 1) * ph, s);
        for (DevBuf<cpxf>& w : m.W) w.alloc((ns + 1) * ph, s);
        m.jw.alloc(3 * (ns + 3) * pl, s);
        auto tw = [&](int n) {
            std::vector<cpxf> t(static_cast<size_t>(n));
            for (int k = 0; k < n; ++k) {
                const std::complex<double> w = std::polar(1.0, -2.0 * M_PI * k / n);
                t[size_t(k)] = Cf(float(w.real()), float(w.imag()));
            }
            return t;
        };
        m.twx.upload(tw(c.nx), s); m.twy.upload(tw(c.ny), s);
    } else {
        MixedBufs& m = c.mx;
        for (DevBuf<cpxf>* p : {&m.Ez, &m.Bz, &m.Lx, &m.Ly, &m.j0x, &m.j0y, &m.jkx, &m.jky, &m.jkz, &m.twx, &m.twy}) p->release();
        for (DevBuf<cpxf>& w : m.W) w.release();
        m.jw.release();
        for (DevBuf<cpx>* p : {&c.Ez, &c.Bz, &c.Lx, &c.Ly}) p->alloc(ns * ph, s);
        for (DevBuf<cpx>* p : {&c.j0x, &c.j0y, &c.jkx, &c.jky, &c.jkz}) p->alloc((ns + 1) * ph, s);
        for (DevBuf<cpx>& w : c.W) w.alloc((ns + 1) * ph, s);
        c.jzg.alloc(2 * ph, s);
        c.jw.alloc(3 * (ns + 3) * pl, s);
    }
    c.mixed = mixed;
    c.f32s = mixed;
    c.jk_is_j0 = false;
    G3D_CUDA(cudaStreamSynchronize(s));
}

static void set_precision(Ctx& c, int mode) {
    if (mode != G3D_PREC_FP64 && mode != G3D_PREC_MIXED) throw Error(G3D_ERR_ARG, "unknown precision " + std::to_string(mode));
    const bool mixed = mode == G3D_PREC_MIXED;
    if (mixed == c.f32s) return;
    if (c.fields_ready) throw Error(G3D_ERR_STATE, "the precision is set before g3d_init");
    if (!c.yf) { c.f32s = mixed; return; }       // free-hand y: FP32 streaming plasma, FP64 spectra
    alloc_spectra(c, mixed);
}

void smem_attr(const void* kern, size_t smem) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> have;
    int dev = 0;
    G3D_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    size_t& v = have[{kern, dev}];
    if (v >= smem) return;
    G3D_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    v = smem;
}

Geo Ctx::geo() const {
    Geo g;
    g.nx = nx; g.ny = ny; g.nk = nk; g.N = N; g.a = a; g.b = b; g.ns = ns; g.nh = ns + 3;
    g.H = H; g.nkh = nkh; g.m0 = 0;
    g.yf = yf ? 1 : 0; g.zeta_uniform = zax.uniform;
    g.dx = dx; g.dy = dy; g.Lx = nx * dx; g.Ly = ny * dy;
    g.kxd = kxd.p; g.kxs = kxs.p; g.filt = filt.p; g.maskx = maskx.p;
    g.kyd = kyd.p; g.kys = kys.p; g.filty = filty.p; g.masky_n = masky_n.p; g.masky_h = masky_h.p; g.iD = iD.p; g.iA = iA.p;
    g.zs = zs.p; g.hcg = hcg.p; g.wlo = wlo.p; g.whi = whi.p; g.wsl = wsl.p;
    g.yn = yn.p; g.pcp = pcp.p; g.pid = pid.p; g.evf = evf.p; g.evb = evb.p; g.evl = evl.p;
    g.zax = zax; g.yax = yax;
    g.twx = twx.p; g.twy = twy.p;
    return g;
}

int Ctx::prof_begin(const char* name) {
    if (!profiling) return -1;
    int e = -1;
    for (size_t k = 0; k < prof.size(); ++k) if (prof[k].name == name) { e = int(k); break; }
    if (e < 0) { prof.push_back(ProfEntry{name, 0, 0}); e = int(prof.size()) - 1; }
    PendingEvent pe{e, nullptr, nullptr};
    for (cudaEvent_t* ev : {&pe.e0, &pe.e1}) {
        if (!event_pool.empty()) { *ev = event_pool.back(); event_pool.pop_back(); }
        else G3D_CUDA(cudaEventCreate(ev));
    }
    G3D_CUDA(cudaEventRecord(pe.e0, stream));
    pending.push_back(pe);
    return int(pending.size()) - 1;
}
void Ctx::prof_end(int tok) {
    if (tok < 0) return;
    G3D_CUDA(cudaEventRecord(pending[size_t(tok)].e1, stream));
}
void Ctx::prof_collect() {
    if (pending.empty()) return;
    G3D_CUDA(cudaStreamSynchronize(stream));
    for (auto& pe : pending) {
        float ms = 0;
        G3D_CUDA(cudaEventElapsedTime(&ms, pe.e0, pe.e1));
        prof[size_t(pe.entry)].ms += ms;
        prof[size_t(pe.entry)].launches += 1;
        event_pool.push_back(pe.e0); event_pool.push_back(pe.e1);
    }
    pending.clear();
}
void Ctx::check_launch(const char* what) {
    ++launches;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw Error(G3D_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------- set-up (reference sim_setup.cpp:5-164)
// Eigenpairs of a symmetric tridiagonal matrix T with diagonal t[0..n) and nonzero couplings u[i] between rows i and
// i + 1 (an irreducible T: its eigenvalues are simple).
//  * Eigenvalues by bisection on Sturm counts (Givens 1954; Barth, Martin & Wilkinson 1967): the number of negative
//    pivots of the LDL^T factorisation of T - x I is the number of eigenvalues below x, so the k-th eigenvalue is
//    bracketed inside the Gershgorin interval and halved down to the spacing of doubles.
//  * Eigenvectors by inverse iteration (Wilkinson 1965; Peters & Wilkinson 1971): a few solves of (T - lambda I) v = b
//    with an LU factorisation with row interchanges, the start vector fixed, each iterate orthogonalised (modified
//    Gram-Schmidt) against the vectors already found for eigenvalues within 1e-3 ||T|| of it, so that the vectors
//    of close eigenvalues stay orthogonal.
// Returns the eigenvalues ascending and the unit eigenvectors, vector m in vec[m * n .. m * n + n).
struct TridiagEigen {
    std::vector<double> val, vec;
};
static int sturm_below(const std::vector<double>& t, const std::vector<double>& u2, double x, double tiny) {
    int neg = 0;
    double q = t[0] - x;
    for (size_t i = 0;; ++i) {
        if (q == 0) q = -tiny;                   // a zero pivot counts as a tiny negative one
        neg += q < 0;
        if (i + 1 == t.size()) break;
        q = (t[i + 1] - x) - u2[i] / q;
    }
    return neg;
}
static TridiagEigen tridiag_eigen(const std::vector<double>& t, const std::vector<double>& u) {
    const int n = int(t.size());
    TridiagEigen out;
    out.val.assign(size_t(n), 0.0);
    out.vec.assign(size_t(n) * n, 0.0);
    if (n == 0) return out;
    std::vector<double> u2(size_t(std::max(n - 1, 0)));
    double lo = 1e300, hi = -1e300, norm = 0;
    for (int i = 0; i < n; ++i) {
        const double r = (i > 0 ? std::fabs(u[size_t(i) - 1]) : 0.0) + (i + 1 < n ? std::fabs(u[size_t(i)]) : 0.0);
        lo = std::min(lo, t[size_t(i)] - r); hi = std::max(hi, t[size_t(i)] + r);
        norm = std::max(norm, std::fabs(t[size_t(i)]) + r);
        if (i + 1 < n) u2[size_t(i)] = u[size_t(i)] * u[size_t(i)];
    }
    const double eps = std::numeric_limits<double>::epsilon();
    const double tiny = eps * eps * std::max(norm, 1e-300);
    for (int k = 0; k < n; ++k) {               // the k-th smallest: count(x) <= k below a, > k below b
        double a = lo - eps * norm, b = hi + eps * norm;
        for (int it = 0; it < 200 && b - a > 2 * eps * std::max(std::fabs(a), std::fabs(b)) + tiny; ++it) {
            const double m = 0.5 * (a + b);
            if (m <= a || m >= b) break;
            if (sturm_below(t, u2, m, tiny) > k) b = m; else a = m;
        }
        out.val[size_t(k)] = 0.5 * (a + b);
    }
    // inverse iteration
    std::vector<double> dd(static_cast<size_t>(n)), du(static_cast<size_t>(n)), du2(static_cast<size_t>(n)),
        dl(static_cast<size_t>(n)), x(static_cast<size_t>(n));
    std::vector<int> swp(static_cast<size_t>(n));
    const double pivot_floor = eps * std::max(norm, 1e-300);
    int cluster_start = 0;
    for (int k = 0; k < n; ++k) {
        const double lam = out.val[size_t(k)];
        if (k > 0 && lam - out.val[size_t(k) - 1] > 1e-3 * norm) cluster_start = k;
        // LU of T - lam I with partial pivoting: row i of U holds dd[i], du[i], du2[i] (two superdiagonals)
        double diag = t[0] - lam, sup = n > 1 ? u[0] : 0.0, sup2 = 0;
        for (int i = 0; i + 1 < n; ++i) {
            const double sub = u[size_t(i)], nd = t[size_t(i) + 1] - lam, nsup = i + 2 < n ? u[size_t(i) + 1] : 0.0;
            if (std::fabs(diag) >= std::fabs(sub)) {       // no interchange
                const double l = sub / (diag != 0 ? diag : pivot_floor);
                dd[size_t(i)] = diag; du[size_t(i)] = sup; du2[size_t(i)] = sup2; dl[size_t(i)] = l; swp[size_t(i)] = 0;
                diag = nd - l * sup; sup = nsup; sup2 = 0;
            } else {                                       // rows i and i + 1 interchanged
                const double l = diag / sub;
                dd[size_t(i)] = sub; du[size_t(i)] = nd; du2[size_t(i)] = nsup; dl[size_t(i)] = l; swp[size_t(i)] = 1;
                diag = sup - l * nd; sup = -l * nsup; sup2 = 0;
            }
        }
        dd[size_t(n) - 1] = diag; du[size_t(n) - 1] = 0; du2[size_t(n) - 1] = 0;
        for (int i = 0; i < n; ++i)
            if (std::fabs(dd[size_t(i)]) < pivot_floor) dd[size_t(i)] = dd[size_t(i)] < 0 ? -pivot_floor : pivot_floor;
        for (int i = 0; i < n; ++i) x[size_t(i)] = 1.0 + 0.1 * std::sin(1.0 + 3.0 * i);   // fixed, not special
        for (int sweep = 0; sweep < 3; ++sweep) {
            for (int i = 0; i + 1 < n; ++i) {              // forward: apply the interchanges and L
                if (swp[size_t(i)]) std::swap(x[size_t(i)], x[size_t(i) + 1]);
                x[size_t(i) + 1] -= dl[size_t(i)] * x[size_t(i)];
            }
            for (int i = n - 1; i >= 0; --i) {             // back substitution with U
                double v = x[size_t(i)];
                if (i + 1 < n) v -= du[size_t(i)] * x[size_t(i) + 1];
                if (i + 2 < n) v -= du2[size_t(i)] * x[size_t(i) + 2];
                x[size_t(i)] = v / dd[size_t(i)];
            }
            for (int m = cluster_start; m < k; ++m) {      // orthogonal to the cluster's earlier vectors
                const double* w = &out.vec[size_t(m) * n];
                double dot = 0;
                for (int i = 0; i < n; ++i) dot += w[i] * x[size_t(i)];
                for (int i = 0; i < n; ++i) x[size_t(i)] -= dot * w[i];
            }
            double nr = 0;
            for (int i = 0; i < n; ++i) nr += x[size_t(i)] * x[size_t(i)];
            nr = std::sqrt(nr);
            for (int i = 0; i < n; ++i) x[size_t(i)] /= nr;
        }
        std::copy(x.begin(), x.end(), out.vec.begin() + size_t(k) * n);
    }
    return out;
}

// Free-hand y (the grid of the reference's setup_y, src/sim_setup.cpp:84-143): ny cells between the conducting walls
// at the nodes 0 and ny. Cell j runs from node j to node j + 1 (size Delta_j, its centre the half-node j); the dual
// cell of node j has size A_j = (Delta_{j-1} + Delta_j) / 2, A_0 = Delta_0 / 2. E_x, B_y, E_z, j_x, j_z live on the
// nodes; E_y, B_x, B_z, j_y on the half-nodes. The tables built here:
//   * 1/Delta_j, 1/A_j and the sponge profile at the nodes and half-nodes;
//   * the elimination of k_x^2 - Lap_y on the interior nodes 1..ny-1 (Lap_y = the three-point operator
//     A_j^-1 [(f_{j+1} - f_j)/Delta_j - (f_j - f_{j-1})/Delta_{j-1}], zero at the walls), per k_x: the reciprocal
//     pivots and the multipliers of the forward sweep, for the sponge's bound field;
//   * the eigenvectors of -Lap_y for the co-moving start field. -Lap_y = A^-1 K with K symmetric, so it is
//     similar to the symmetric tridiagonal A^-1/2 K A^-1/2; its orthonormal eigenvectors u_m give the modes
//     v_m = A^-1/2 u_m, orthonormal in the A-weighted product. A profile f on the nodes then has the coefficients
//     c_m = sum_j v_m(j) A_j f_j = sum_j u_m(j) sqrt(A_j) f_j, and f_j = sum_m v_m(j) c_m = sum_m u_m(j) c_m / sqrt(A_j).
//     Tables: forward [slot][j] = u_m(j) sqrt(A_j), back [j][slot] = u_m(j) / sqrt(A_j), eigenvalue [slot], with
//     slot = m + 1 (slot 0 left at zero: the wall node has no mode).
static double sponge_factor(double dist_from_edge, double width, double rate) {
    if (width <= 0 || dist_from_edge >= width) return 1.0;
    const double r = 1 - dist_from_edge / width;
    return 1 - rate * r * r;
}
static void setup_y_free(Ctx& c, const g3d_grid& G, const g3d_params& P, cudaStream_t s) {
    const int ny = c.ny, H = c.H;
    const std::vector<double> node(G.ynode, G.ynode + ny + 1);
    for (int j = 0; j < ny; ++j)
        if (!(node[size_t(j) + 1] > node[size_t(j)])) throw Error(G3D_ERR_ARG, "ynode must increase");
    const double Ly = node[size_t(ny)] - node[0];
    c.dy = Ly / ny;
    std::vector<double> cell(static_cast<size_t>(ny)), dual(static_cast<size_t>(ny));
    std::vector<double> inv_cell(static_cast<size_t>(ny)), inv_dual(static_cast<size_t>(ny));
    std::vector<double> mask_node(static_cast<size_t>(ny)), mask_half(static_cast<size_t>(ny));
    for (int j = 0; j < ny; ++j) cell[size_t(j)] = node[size_t(j) + 1] - node[size_t(j)];
    for (int j = 0; j < ny; ++j) dual[size_t(j)] = j == 0 ? 0.5 * cell[0] : 0.5 * (cell[size_t(j) - 1] + cell[size_t(j)]);
    for (int j = 0; j < ny; ++j) {
        inv_cell[size_t(j)] = 1 / cell[size_t(j)];
        inv_dual[size_t(j)] = 1 / dual[size_t(j)];
        const double y_half = 0.5 * (node[size_t(j)] + node[size_t(j) + 1]);
        mask_node[size_t(j)] = sponge_factor(0.5 * Ly - std::fabs(node[size_t(j)]), P.sponge_y, P.sponge_rate);
        mask_half[size_t(j)] = sponge_factor(0.5 * Ly - std::fabs(y_half), P.sponge_y, P.sponge_rate);
    }
    c.ynode_h = node;
    c.ia_max = 0;
    for (int j = 0; j < ny; ++j) c.ia_max = std::max(c.ia_max, std::max(inv_cell[size_t(j)], inv_dual[size_t(j)]));
    c.yn.upload(node, s); c.iD.upload(inv_cell, s); c.iA.upload(inv_dual, s);
    c.masky_n.upload(mask_node, s); c.masky_h.upload(mask_half, s);
    const bool equal_cells = std::all_of(cell.begin(), cell.end(), [&](double d) { return d == cell[0]; });
    c.yax = AxisDev{c.yn.p, ny + 1, equal_cells ? 1 : 0, node[0], 1 / cell[0]};
    if (!equal_cells) {
        c.ybins.upload(axis_bins(node, c.yax.bih), s);
        c.yax.bins = c.ybins.p; c.yax.nb = int(c.ybins.n);
    }
    // the y tables of the Fourier form are not used; zeros keep the device pointers valid
    const std::vector<double> zero(static_cast<size_t>(ny), 0.0);
    c.kyd.upload(zero, s); c.kys.upload(zero, s); c.filty.upload(zero, s);
    c.kyd_h = zero;
    // -Lap_y on the interior nodes: row j couples j - 1 (below), j, j + 1 (above)
    auto below = [&](int j) { return j > 1 ? -inv_dual[size_t(j)] * inv_cell[size_t(j) - 1] : 0.0; };
    auto above = [&](int j) { return j < ny - 1 ? -inv_dual[size_t(j)] * inv_cell[size_t(j)] : 0.0; };
    auto centre = [&](int j) { return inv_dual[size_t(j)] * (inv_cell[size_t(j) - 1] + inv_cell[size_t(j)]); };
    // forward elimination of k_x^2 - Lap_y per k_x <= nx/2: pivot_j = k_x^2 + centre_j - below_j m_{j-1},
    // m_j = above_j / pivot_j; stored 1/pivot_j and m_j at [j][k_x]
    std::vector<double> mult(size_t(ny) * H, 0.0), inv_piv(size_t(ny) * H, 0.0);
    for (int i = 0; i < H; ++i) {
        const double k2 = c.kxd_h[size_t(i)] * c.kxd_h[size_t(i)];
        double m_prev = 0;
        for (int j = 1; j < ny; ++j) {
            const double piv = k2 + centre(j) - below(j) * m_prev;
            inv_piv[size_t(j) * H + i] = 1 / piv;
            m_prev = above(j) / piv;
            mult[size_t(j) * H + i] = m_prev;
        }
    }
    c.pcp.upload(mult, s); c.pid.upload(inv_piv, s);
    // modes of -Lap_y: the symmetric form A^-1/2 K A^-1/2 (diagonal centre_j, couplings -1/(Delta_j sqrt(A_j A_{j+1})))
    const int M = ny - 1;
    std::vector<double> t(static_cast<size_t>(M)), u(static_cast<size_t>(std::max(M - 1, 0)));
    for (int j = 1; j < ny; ++j) t[size_t(j) - 1] = centre(j);
    for (int j = 1; j + 1 < ny; ++j) u[size_t(j) - 1] = -inv_cell[size_t(j)] / std::sqrt(dual[size_t(j)] * dual[size_t(j) + 1]);
    const TridiagEigen ev = tridiag_eigen(t, u);
    // check: largest |S v - mu v| and |v_m . v_k - delta_mk| against the spectrum's size
    double big = 0, resid = 0, orth = 0;
    for (int m = 0; m < M; ++m) big = std::max(big, std::fabs(ev.val[size_t(m)]));
    for (int m = 0; m < M; ++m) {
        const double* v = &ev.vec[size_t(m) * M];
        for (int k = 0; k < M; ++k) {
            double r = (t[size_t(k)] - ev.val[size_t(m)]) * v[k];
            if (k > 0) r += u[size_t(k) - 1] * v[k - 1];
            if (k + 1 < M) r += u[size_t(k)] * v[k + 1];
            resid = std::max(resid, std::fabs(r));
        }
        for (int q = m; q < std::min(M, m + 8); ++q) {     // neighbours in the spectrum are the ones at risk
            const double* w = &ev.vec[size_t(q) * M];
            double dot = 0;
            for (int k = 0; k < M; ++k) dot += v[k] * w[k];
            orth = std::max(orth, std::fabs(dot - (q == m ? 1.0 : 0.0)));
        }
    }
    if (!(resid <= 1e-10 * big) || !(orth <= 1e-10))
        throw Error(G3D_ERR_ARG, "modes of the y Laplacian: residual " + std::to_string(resid / big) + ", orthogonality " +
                                     std::to_string(orth));
    std::vector<double> fwd(size_t(ny) * ny, 0.0), back(size_t(ny) * ny, 0.0), eig(static_cast<size_t>(ny), 0.0);
    for (int m = 0; m < M; ++m) {
        const int slot = m + 1;
        eig[size_t(slot)] = ev.val[size_t(m)];
        for (int j = 1; j < ny; ++j) {
            const double um = ev.vec[size_t(m) * M + size_t(j) - 1], root = std::sqrt(dual[size_t(j)]);
            fwd[size_t(slot) * ny + j] = um * root;
            back[size_t(j) * ny + slot] = um / root;
        }
    }
    c.evf.upload(fwd, s); c.evb.upload(back, s); c.evl.upload(eig, s);
}

// field buffers of the slab [a, b): real planes of the reference layouts, spectra as half spectra (FP64 form)
void realloc_slab(Ctx& c) {
    const cudaStream_t s = c.stream;
    const size_t pl = size_t(c.nk), ph = size_t(c.nkh), ns = size_t(c.ns);
    for (DevBuf<cpx>* p : {&c.Rx, &c.Ry}) p->alloc(ns * ph, s);
    alloc_spectra(c, false);
    c.F.alloc(6 * (ns + 2) * pl, s);
    c.rscratch.alloc(ns * ph, s);
}

static void setup(Ctx& c, const g3d_grid& G, const g3d_params& P) {
    if (!G.y_fourier && !G.ynode) throw Error(G3D_ERR_ARG, "free-hand y needs the ny + 1 nodes (ynode)");
    if (!fft_size_ok(G.nx) || G.nx < 8 || (G.y_fourier && !fft_size_ok(G.ny)) || (!G.y_fourier && (G.ny < 3 || G.ny > 512)))
        throw Error(G3D_ERR_ARG, "nx must be a power of two in 8..512 or three times one in 24..384; ny likewise (4..512, Fourier y) "
                                 "or 3..512 (free-hand)");
    if (G.nzeta < 4 || !G.zeta) throw Error(G3D_ERR_ARG, "nzeta must be >= 4 with a zeta table");
    if (!(G.Lx > 0) || !(G.Ly > 0)) throw Error(G3D_ERR_ARG, "Lx, Ly must be positive");
    if (P.precision != G3D_FP64 && P.precision != G3D_MIXED) throw Error(G3D_ERR_ARG, "precision must be G3D_FP64 or G3D_MIXED");
    if (!(P.dz > 0) || !(P.dz_push > 0) || !(P.lambda0 > 0)) throw Error(G3D_ERR_ARG, "dz, dz_push, lambda0 must be positive");
    for (int m = 0; m + 1 < G.nzeta; ++m)
        if (!(G.zeta[m + 1] > G.zeta[m])) throw Error(G3D_ERR_ARG, "zeta slices must increase");
    c.P = P;
    c.N = G.nzeta; c.nx = G.nx; c.ny = G.ny; c.nk = c.nx * c.ny;
    c.H = c.nx / 2 + 1; c.nkh = long(c.ny) * c.H;
    c.a = 0; c.ns = c.N; c.b = c.N;
    c.dx = G.Lx / c.nx;
    c.yf = true;
    c.zeta.assign(G.zeta, G.zeta + G.nzeta);
    cudaStream_t s = c.stream;

    // x: Fourier modes; Nyquist zeroed for derivatives, kept for the shift; cos^2 current filter; sponge
    const int nx = c.nx, ny = c.ny;
    std::vector<double> hkx(nx), hsx(nx), hf(nx), hm(nx);
    auto prof = [&](double dd, double w) {
        if (w <= 0 || dd >= w) return 1.0;
        const double r = 1 - dd / w;
        return 1 - P.sponge_rate * r * r;
    };
    for (int ixx = 0; ixx < nx; ++ixx) {
        const int mx = ixx <= nx / 2 ? ixx : ixx - nx;
        hsx[ixx] = 2 * M_PI * mx / G.Lx;
        hkx[ixx] = (2 * ixx == nx) ? 0 : hsx[ixx];
        hf[ixx] = P.k_filter ? std::pow(std::cos(0.5 * hsx[ixx] * c.dx), 2) : 1.0;
        if (2 * ixx == nx) hf[ixx] = 0;
        hm[ixx] = prof(std::min(ixx * c.dx, G.Lx - ixx * c.dx), P.sponge);
    }
    c.kxd.upload(hkx, s); c.kxs.upload(hsx, s); c.filt.upload(hf, s); c.maskx.upload(hm, s);
    c.kxd_h = hkx;
    c.yf = G.y_fourier != 0;
    if (!c.yf) setup_y_free(c, G, P, s);
    // y: Fourier modes (reference setup_y_fourier, sim_setup.cpp:63-82)
    if (c.yf) {
    c.dy = G.Ly / ny;
    std::vector<double> hky(ny), hsy(ny), hfy(ny), hmy(ny), hi(ny, 1 / c.dy);
    for (int j = 0; j < ny; ++j) {
        const int my = j <= ny / 2 ? j : j - ny;
        hsy[j] = 2 * M_PI * my / G.Ly;
        hky[j] = (2 * j == ny) ? 0 : hsy[j];
        hfy[j] = P.k_filter ? std::pow(std::cos(0.5 * hsy[j] * c.dy), 2) : 1.0;
        if (2 * j == ny) hfy[j] = 0;
        const double dd = std::min(j * c.dy, G.Ly - j * c.dy), w = P.sponge_y;
        double m = 1;
        if (w > 0 && dd < w) { const double r = 1 - dd / w; m = 1 - P.sponge_rate * r * r; }
        hmy[j] = m;
    }
    c.kyd.upload(hky, s); c.kys.upload(hsy, s); c.filty.upload(hfy, s); c.masky_n.upload(hmy, s); c.masky_h.upload(hmy, s);
    c.iD.upload(hi, s); c.iA.upload(hi, s);
    c.kyd_h = hky;
    c.yax = AxisDev{nullptr, ny + 1, 1, 0.0, 1 / c.dy};
    }
    // zeta (reference setup_zeta, sim_setup.cpp:148-164)
    const int N = c.N;
    const std::vector<double>& Z = c.zeta;
    std::vector<double> hh(N - 1);
    for (int m = 0; m < N - 1; ++m) hh[m] = Z[m + 1] - Z[m];
    bool uni = true;
    for (int m = 0; m < N - 1; ++m) uni = uni && hh[m] == hh[0];
    if (uni) for (double& v : hh) v = Z.back() / (N - 1);
    std::vector<double> g(N + 3), lo(N), hi2(N), ws(N);
    for (int m = -2; m <= N; ++m) g[m + 2] = hh[std::min(std::max(m, 0), N - 2)];
    for (int n = 0; n < N; ++n) {
        const double hmn = g[n - 1 + 2], hpn = g[n + 2];
        lo[n] = hpn / (hmn + hpn); hi2[n] = hmn / (hmn + hpn);
        ws[n] = 0.5 * ((n > 0 ? hh[n - 1] : 0) + (n < N - 1 ? hh[n] : 0));
    }
    c.zs.upload(Z, s); c.hcg.upload(g, s); c.wlo.upload(lo, s); c.whi.upload(hi2, s); c.wsl.upload(ws, s);
    c.hcg_h = g; c.wlo_h = lo; c.whi_h = hi2; c.wsl_h = ws;
    c.zax = AxisDev{c.zs.p, N, uni ? 1 : 0, 0.0, 1 / hh[0]};
    if (!uni) {
        c.zbins.upload(axis_bins(Z, c.zax.bih), s);
        c.zax.bins = c.zbins.p; c.zax.nb = int(c.zbins.n);
    }
    c.hmin = 1e300;
    for (int m = 0; m + 1 < N; ++m) c.hmin = std::min(c.hmin, Z[m + 1] - Z[m]);
    // twiddles exp(-2 pi i s / n)
    auto tw = [&](int n) {
        std::vector<cpx> t(n);
        for (int k = 0; k < n; ++k) { const std::complex<double> w = std::polar(1.0, -2.0 * M_PI * k / n); t[k] = C(w.real(), w.imag()); }
        return t;
    };
    c.twx.upload(tw(nx), s); c.twy.upload(tw(ny), s);
    realloc_slab(c);
    c.red.alloc(size_t(297) * 17, s);
    c.kerr.alloc(1, s);
    c.use_tma = std::getenv("G3D_NO_TMA") == nullptr;
    if (const char* v = std::getenv("G3D_TMA_POLLS")) c.tma_polls = std::max(1L, std::atol(v));
    if (const char* v = std::getenv("G3D_TMA_EXTRA_BYTES")) c.tma_extra = unsigned(std::min(4096L, std::max(0L, std::atol(v))));
    // the plane wave (reference sim_setup.cpp:51-54; eta_c given directly)
    c.laser.on = P.laser_on; c.laser.pol = P.laser_pol; c.laser.env = P.laser_envelope;
    c.laser.a0 = P.a0; c.laser.kL = P.kL; c.laser.tau = P.tau; c.laser.cep = P.cep; c.laser.eta_c = P.eta_c;
    c.laser.kx = std::sin(P.theta); c.laser.kz = std::cos(P.theta);
    c.laser.flat = P.flat_length; c.laser.ramp = P.ramp_length;
    // box origin as Simulation::init sets it (load_bunch, src/sim_bunches.cpp:216, also without bunches)
    c.X0 = -0.5 * G.Lx; c.Y0 = c.yf ? -0.5 * G.Ly : 0.0;    // free-hand y: y is the physical coordinate
    if (P.laser_on && P.laser_envelope == G3D_ENV_FLATTOP && !(P.ramp_length > 0))
        throw Error(G3D_ERR_ARG, "flat-top envelope needs ramp_length > 0");
    if (!c.yf) {
        c.fhs.alloc(5 * size_t(ny) * c.H, s);
        c.fhcp.alloc(size_t(ny) * c.H, s);
    }
    if (P.precision == G3D_MIXED) {
        if (c.yf) alloc_spectra(c, true);
        else c.f32s = true;                      // free-hand y: FP32 streaming plasma, FP64 spectra
    }
    G3D_CUDA(cudaStreamSynchronize(s));
}

// ---------------------------------------------------------------- particles
void reserve_particles(Ctx& c, long n) {
    if (n <= c.pcap && c.pcap <= 2 * n + 1024) return;
    const long cap = n + n / 4 + 64;
    c.pbuf_d.alloc(size_t(cap) * 11, c.stream);
    c.pbuf_i.alloc(size_t(cap) * 2, c.stream);
    c.pbuf_u.alloc(size_t(cap), c.stream);
    double* d = c.pbuf_d.p;
    PartsDev& P = c.parts;
    double** cols[11] = {&P.x, &P.y, &P.zeta, &P.px, &P.py, &P.pz, &P.w, &P.rem, &P.z, &P.q, &P.qm};
    for (int k = 0; k < 11; ++k) *cols[k] = d + size_t(k) * cap;
    P.alive = c.pbuf_i.p; P.sp = c.pbuf_i.p + cap;
    P.id = c.pbuf_u.p;
    c.pcap = cap;
}

// Host records (104-byte AoS) <-> device columns: one DMA of the records into a device staging buffer
// and a transposition kernel (k_parts_unpack / k_parts_pack, k_parts.cu).
void set_particles(Ctx& c, const g3d_particle* v, long n) {
    reserve_particles(c, n);
    c.np = n;
    if (!n) return;
    if (c.pstage.n < size_t(n)) c.pstage.alloc(size_t(n) + size_t(n) / 4 + 64, c.stream);
    G3D_CUDA(cudaMemcpyAsync(c.pstage.p, v, size_t(n) * sizeof(g3d_particle), cudaMemcpyHostToDevice, c.stream));
    launch_parts_unpack(c, n);
    sort_particles(c);
    G3D_CUDA(cudaStreamSynchronize(c.stream));     // the caller may reuse its buffer on return
}

static void get_particles_into(Ctx& c, g3d_particle* out) {
    const long n = c.np;
    if (!n) return;
    if (c.pstage.n < size_t(n)) c.pstage.alloc(size_t(n) + size_t(n) / 4 + 64, c.stream);
    launch_parts_pack(c, n);
    G3D_CUDA(cudaMemcpyAsync(out, c.pstage.p, size_t(n) * sizeof(g3d_particle), cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
}

std::vector<g3d_particle> get_particles(Ctx& c) {
    std::vector<g3d_particle> out(static_cast<size_t>(c.np));
    get_particles_into(c, out.data());
    return out;
}

// Bunch sampling with the reference's random sequence for the built-in profiles (sim_bunches.cpp:92-217,
// shot_noise = random): per particle G for x, y, (U or G) for z, G for px and py when sigma > 0, G for pz.
// Host code only: it needs the grid, not a device.
static void sample_bunches(const g3d_grid& G, const g3d_params& P, const g3d_bunch* list, int count,
                           std::vector<g3d_particle>& mine, long& lost, double& X0, double& Y0) {
    const double Lu = P.lambda0 / (2 * M_PI), w0 = c_SI / Lu;
    const double nc = eps0 * me_SI * w0 * w0 / (e_SI * e_SI);
    const bool yf = G.y_fourier != 0;
    const double yoff = yf ? 0.5 * G.Ly : 0.0;        // Fourier y: box coordinate, physical y = p.y + Y0
    const double ylo = yf ? -1e300 : G.ynode[1], yhi = yf ? 1e300 : G.ynode[G.ny - 1];   // free-hand: inside the walls
    const int N = G.nzeta;
    // the zeta axis as the set-up builds it (uniform: direct location with 1 / h)
    bool uni = true;
    const double h0 = G.zeta[1] - G.zeta[0];
    for (int m = 0; m + 1 < N; ++m) uni = uni && (G.zeta[m + 1] - G.zeta[m]) == h0;
    const AxisDev zax{G.zeta, N, uni ? 1 : 0, 0.0, 1 / (uni ? G.zeta[N - 1] / (N - 1) : h0)};
    lost = 0;
    for (int kb = 0; kb < count; ++kb) {
        const g3d_bunch& B = list[kb];
        if (!(B.gamma > 1)) throw Error(G3D_ERR_ARG, "bunch gamma must be > 1");
        std::mt19937_64 rng(B.seed);
        std::normal_distribution<double> Gs(0, 1);
        std::uniform_real_distribution<double> U(-0.5, 0.5);
        const double Ne = B.charge_C / e_SI;
        const double W = (B.nmacro > 0 ? Ne / double(B.nmacro) : 0) / (nc * std::pow(Lu, 3));
        const double p0 = std::sqrt(B.gamma * B.gamma - 1);
        // Fawley's beamlets (shot_noise = fawley): groups of M particles sharing a draw
        const int M = B.beamlet > 1 ? B.beamlet : 1;
        if (M > 1 && (M < 3 || B.nmacro % M || !(B.noise_lambda > 0)))
            throw Error(G3D_ERR_ARG, "Fawley shot noise needs beamlet >= 3 dividing the macroparticles and noise_lambda > 0");
        const long groups = B.nmacro / M;
        const double Ne_group = groups > 0 ? Ne / double(groups) : 0;
        std::vector<double> dz(static_cast<size_t>(M), 0.0), dth(static_cast<size_t>(M));
        mine.reserve(mine.size() + size_t(B.nmacro));
        for (long ib = 0; ib < groups; ++ib) {
            const double x = B.x0 + B.sigx * Gs(rng);
            const double y = B.y0 + B.sigy * Gs(rng);
            const double z = B.length > 0 ? B.length * U(rng) : B.sigz * Gs(rng);
            const double px = B.sigx > 0 ? B.emitx / B.sigx * Gs(rng) : 0;
            const double py = B.sigy > 0 ? B.emity / B.sigy * Gs(rng) : 0;
            const double pz = p0 * (1 + B.espread * Gs(rng));
            if (M > 1) {
                // M particles evenly spaced in the phase theta = 2 pi z / noise_lambda from a random theta0, each
                // displaced by sum_h Re(c_h e^{-i h theta_j}), c_h = -2 i b_h / h with b_h the bunching factor of
                // Ne_group random electrons at harmonic h (complex Gaussian of variance 1 / Ne_group), h < M / 2
                using cplx = std::complex<double>;
                const cplx I(0, 1);
                const double th0 = 2 * M_PI * std::uniform_real_distribution<double>(0, 1)(rng);
                std::fill(dth.begin(), dth.end(), 0.0);
                for (int hh = 1; 2 * hh < M; ++hh) {
                    const double gi = Gs(rng);               // the imaginary part is drawn first (the reference's order)
                    const double gr = Gs(rng);
                    const cplx bh = std::sqrt(0.5 / Ne_group) * cplx(gr, gi);
                    const cplx ch = -2.0 * I * bh / double(hh);
                    for (int j = 0; j < M; ++j) dth[size_t(j)] += std::real(ch * std::exp(-I * double(hh) * (th0 + 2 * M_PI * j / M)));
                }
                for (int j = 0; j < M; ++j) dz[size_t(j)] = B.noise_lambda * ((th0 + 2 * M_PI * j / M + dth[size_t(j)]) / (2 * M_PI) - 0.5);
            }
            for (int j = 0; j < M; ++j) {
                const double g = std::sqrt(1 + px * px + py * py + pz * pz);
                const double vx = px / g, vy = py / g, vz = pz / g;
                const double zz = z + dz[size_t(j)];
                g3d_particle p{};
                p.x = x - vx * zz / vz + 0.5 * G.Lx; p.y = y - vy * zz / vz + yoff;
                p.zeta = B.zeta_center + zz / vz;
                p.px = px; p.py = py; p.pz = pz; p.w = W; p.alive = 1;
                p.q = B.q; p.qm = B.q; p.sp = -kb; p.z = 0;
                int hc; double f;
                zax.locate(p.zeta, hc, f);
                if (p.zeta < 0 || hc > N - 2 || p.y < ylo || p.y > yhi) { ++lost; continue; }
                mine.push_back(p);
            }
        }
    }
    X0 = -0.5 * G.Lx; Y0 = -yoff;
}

static void load_bunches(Ctx& c, const g3d_grid& G, const g3d_bunch* list, int count) {
    std::vector<g3d_particle> mine;
    long lost = 0;
    sample_bunches(G, c.P, list, count, mine, lost, c.X0, c.Y0);
    if (c.sharded()) {                               // every rank samples the beam and keeps the particles of its slab
        std::vector<g3d_particle> own;
        for (const g3d_particle& p : mine)
            if (shard_owns(c, p.zeta)) own.push_back(p);
        mine.swap(own);
    }
    set_particles(c, mine.data(), long(mine.size()));
    c.lost_total += c.rank == 0 ? lost : 0;          // every rank samples the same beam: its losses count once
    c.nbunch = count > 1 ? count : 1;
}

// ---------------------------------------------------------------- the march path
static void currents(Ctx& c) {
    c.jk_is_j0 = false;
    if (!c.mixed && c.yf) launch_deposit(c);
    // with plasma the k = 0 current is kept (a 1D plasma wave, the return current), but not in the start field
    // (sim_particles.cpp:143-145)
    const bool keep0 = c.pl && c.pl->box_mean && !c.starting_;
    if (!c.yf) { launch_deposit_fh(c); launch_cur_fft_fh(c, keep0); return; }
    if (c.mixed) { launch_deposit_f(c); launch_cur_fft_f(c, keep0); return; }
    launch_cur_fft(c, keep0);
    if (c.sharded()) shard_jz_ghosts(c);
    // one rank: the filtered j_z ghosts of the neighbours are zero (exchange_jz_ghosts, sim_particles.cpp:210-226)
}
static void march(Ctx& c, double D) {
    if (c.jk_is_j0) throw Error(G3D_ERR_STATE, "march needs the currents of level s1 (call currents first)");
    if (!c.yf) launch_march_fh(c, D);
    else if (c.mixed) launch_march_f(c, D);
    else if (c.sharded()) shard_march(c, D);
    else launch_march(c, D);
}
static void sponge_and_real_fields(Ctx& c) {
    if (c.fd_next) { c.Fd.p = c.fd_next; c.fd_next = nullptr; }
    if (c.f_next) { c.F.p = c.f_next; c.f_next = nullptr; }
    if (!c.yf) {
        if (c.P.sponge > 0 || c.P.sponge_y > 0) launch_sponge_fh(c);
        launch_real_fields_fh(c);
        return;
    }
    if (c.mixed) {
        if (c.P.sponge > 0 || c.P.sponge_y > 0) launch_sponge_f(c);
        launch_real_fields_f(c);
        return;
    }
    if (c.P.sponge > 0 || c.P.sponge_y > 0) launch_sponge(c);
    launch_real_fields(c);
    if (c.sharded()) shard_field_ghosts(c);
}
// j0 <- jk (sim_fields.cpp:313-315): the buffers are swapped; until the next deposit jk reads as j0.
static void j0_from_jk(Ctx& c) {
    if (c.mixed) {
        std::swap(c.mx.j0x.p, c.mx.jkx.p);
        std::swap(c.mx.j0y.p, c.mx.jky.p);
    } else {
        std::swap(c.j0x.p, c.jkx.p);
        std::swap(c.j0y.p, c.jky.p);
    }
    c.jk_is_j0 = true;
}
static void materialize_jk(Ctx& c) {
    if (!c.jk_is_j0) return;
    if (c.mixed) {
        launch_copy_f(c, c.mx.jkx.p, c.mx.j0x.p, c.mx.jkx.n);
        launch_copy_f(c, c.mx.jky.p, c.mx.j0y.p, c.mx.jky.n);
        c.jk_is_j0 = false;
        return;
    }
    launch_copy_c(c, c.jkx.p, c.j0x.p, c.jkx.n);
    launch_copy_c(c, c.jky.p, c.j0y.p, c.jky.n);
    c.jk_is_j0 = false;
}
static void solve_fields(Ctx& c, double D) {
    currents(c);
    march(c, D);
    sponge_and_real_fields(c);
    j0_from_jk(c);
}
static void comoving_field(Ctx& c) {
    double sums[2];
    launch_beta_sums(c, sums);
    const double beta = c.comoving_c_ ? 1 : sums[1] > 0 ? sums[0] / sums[1] : 1;
    const double gm2 = 1 - beta * beta;
    if (!c.comoving_c_) { c.beta_b = beta; c.gm2_b = gm2; }
    if (!c.yf) launch_comoving_fh(c, beta, gm2);
    else if (c.mixed) launch_comoving_f(c, beta, gm2);
    else if (c.sharded()) shard_comoving(c, beta, gm2);
    else launch_comoving(c, beta, gm2);
}
// Several bunch blocks (reference Simulation::comoving_fields_per_bunch, src/sim_bunches.cpp:223-248): the co-moving
// equation -(Lap_perp + gamma^-2 d_zeta^2) psi = rho is linear but its gamma is the bunch's, so each block k (the
// particles with sp == -k, in storage order) gets its own currents and co-moving R with its own beta, and the R of
// the blocks are summed in block order into zeroed accumulators. The currents are then those of all particles, and
// the beta kept for the sponge's bound field is the mean over all of them. Init only: the blocks go through host
// records.
static void comoving_fields_per_bunch(Ctx& c) {
    const std::vector<g3d_particle> all = get_particles(c);
    const size_t n = size_t(c.ns) * c.nkh;
    DevBuf<cpx> sx, sy;                          // alloc zeroes them
    sx.alloc(n, c.stream); sy.alloc(n, c.stream);
    std::vector<g3d_particle> one;
    for (int k = 0; k < c.nbunch; ++k) {
        one.clear();
        for (const g3d_particle& p : all)
            if (p.sp == -k) one.push_back(p);
        set_particles(c, one.data(), long(one.size()));
        currents(c);
        comoving_field(c);
        launch_axpy_c(c, sx.p, c.Rx.p, 1.0, n);
        launch_axpy_c(c, sy.p, c.Ry.p, 1.0, n);
    }
    set_particles(c, all.data(), long(all.size()));
    currents(c);
    launch_copy_c(c, c.Rx.p, sx.p, n);
    launch_copy_c(c, c.Ry.p, sy.p, n);
    double sums[2];
    launch_beta_sums(c, sums);
    c.beta_b = sums[1] > 0 ? sums[0] / sums[1] : 1;
    c.gm2_b = 1 - c.beta_b * c.beta_b;
    G3D_CUDA(cudaStreamSynchronize(c.stream));
}
static void relax_start_field(Ctx& c) {
    const size_t n = size_t(c.ns) * c.nkh, nj = size_t(c.ns + 1) * c.nkh;
    if (c.mixed) {
        // the same three backward-Euler marches; R stays complex128, so its two copies are too
        DevBuf<cpx> rx, ry;
        rx.alloc(n, c.stream); ry.alloc(n, c.stream);
        launch_copy_c(c, rx.p, c.Rx.p, n);
        launch_copy_c(c, ry.p, c.Ry.p, n);
        c.comoving_c_ = true; comoving_field(c); c.comoving_c_ = false;
        launch_axpy_c(c, rx.p, c.Rx.p, -1.0, n);
        launch_axpy_c(c, ry.p, c.Ry.p, -1.0, n);
        const double D = 100 * c.P.dz;
        for (int it = 0; it < 3; ++it) {
            c.mx.Ez.zero(c.stream); c.mx.Bz.zero(c.stream); c.mx.j0x.zero(c.stream); c.mx.j0y.zero(c.stream);
            march(c, D);
        }
        launch_axpy_c(c, c.Rx.p, rx.p, 1.0, n);
        launch_axpy_c(c, c.Ry.p, ry.p, 1.0, n);
        G3D_CUDA(cudaStreamSynchronize(c.stream));
        return;
    }
    cpx* dxr = c.W[4].p; cpx* dyr = c.W[5].p;      // R of the bunch's beta (the co-moving solve uses W3)
    launch_copy_c(c, dxr, c.Rx.p, n);
    launch_copy_c(c, dyr, c.Ry.p, n);
    c.comoving_c_ = true; comoving_field(c); c.comoving_c_ = false;
    launch_axpy_c(c, dxr, c.Rx.p, -1.0, n);
    launch_axpy_c(c, dyr, c.Ry.p, -1.0, n);
    const double D = 100 * c.P.dz;
    for (int it = 0; it < 3; ++it) {
        launch_zero_c(c, c.Ez.p, n); launch_zero_c(c, c.Bz.p, n);
        launch_zero_c(c, c.j0x.p, nj); launch_zero_c(c, c.j0y.p, nj);
        march(c, D);
    }
    launch_axpy_c(c, c.Rx.p, dxr, 1.0, n);
    launch_axpy_c(c, c.Ry.p, dyr, 1.0, n);
}
// The thin chicanes passed in the step s0 -> s1 (reference Simulation::apply_chicanes, src/sim_external.cpp:108-151):
// every live beam particle moves in zeta by r56 (gamma / gamma_ref - 1) - delay, those leaving the window are lost;
// R keeps its radiation and trades the beam's co-moving field of the old positions for that of the new ones (each
// made as at the start: per bunch block, relaxed, vacuum); E_z, B_z, L, the real fields and j0 follow as at the start.
static void apply_chicanes(Ctx& c, double s0, double s1) {
    for (const g3d_chicane& ch : c.chicanes) {
        if (!(ch.z > s0 && ch.z <= s1)) continue;
        const size_t n = size_t(c.ns) * c.nkh;
        DevBuf<cpx> keep_x, keep_y, old_x, old_y;
        auto comoving_into = [&](DevBuf<cpx>& rx, DevBuf<cpx>& ry) {
            c.starting_ = true;                          // vacuum at the chicane: no k_perp = 0 current
            if (c.nbunch > 1) comoving_fields_per_bunch(c);
            else { currents(c); comoving_field(c); }
            if (c.P.start_relax) relax_start_field(c);
            c.starting_ = false;
            rx.alloc(n, c.stream); ry.alloc(n, c.stream);
            launch_copy_c(c, rx.p, c.Rx.p, n);
            launch_copy_c(c, ry.p, c.Ry.p, n);
        };
        if (c.P.self_fields) {
            keep_x.alloc(n, c.stream); keep_y.alloc(n, c.stream);
            launch_copy_c(c, keep_x.p, c.Rx.p, n);
            launch_copy_c(c, keep_y.p, c.Ry.p, n);
            comoving_into(old_x, old_y);
        }
        const std::vector<g3d_particle> all = get_particles(c);
        std::vector<g3d_particle> kept;
        kept.reserve(all.size());
        const double zmax = c.zeta[size_t(c.N) - 1];
        for (g3d_particle p : all) {
            if (p.alive != 1) continue;
            const double g = std::sqrt(1 + p.px * p.px + p.py * p.py + p.pz * p.pz);
            p.zeta += ch.r56 * (g / ch.gamma_ref - 1) - ch.delay;
            if (p.zeta < 0 || p.zeta >= zmax) { ++c.lost_total; continue; }
            kept.push_back(p);
        }
        set_particles(c, kept.data(), long(kept.size()));
        if (!c.P.self_fields) continue;
        DevBuf<cpx> new_x, new_y;
        comoving_into(new_x, new_y);
        // R = (R before + new) - old, in that order
        launch_axpy_c(c, keep_x.p, new_x.p, 1.0, n);
        launch_axpy_c(c, keep_x.p, old_x.p, -1.0, n);
        launch_axpy_c(c, keep_y.p, new_y.p, 1.0, n);
        launch_axpy_c(c, keep_y.p, old_y.p, -1.0, n);
        launch_copy_c(c, c.Rx.p, keep_x.p, n);
        launch_copy_c(c, c.Ry.p, keep_y.p, n);
        march(c, 0.0);                                   // E_z, B_z, L of R, as at the start
        sponge_and_real_fields(c);
        j0_from_jk(c);
        G3D_CUDA(cudaStreamSynchronize(c.stream));
    }
}
static void shift_window(Ctx& c, int nxs, int nys) {
    if (c.Fd.p) throw Error(G3D_ERR_STATE, "exact fields need a fixed window");
    materialize_jk(c);
    c.X0 += nxs * c.dx; c.Y0 += nys * c.dy;
    launch_shift(c, nxs, nys, nxs * c.dx, nys * c.dy);
    if (c.mixed && c.P.self_fields)
        for (DevBuf<cpxf>* a : {&c.mx.Ez, &c.mx.Bz, &c.mx.j0x, &c.mx.j0y}) launch_rotate_f(c, a->p, a->n, nxs * c.dx, nys * c.dy, nys);
    if (c.pl) {
        for (auto& p : c.pl->joining) { p.x -= nxs * c.dx; p.y -= nys * c.dy; }
        launch_join_shift(c, nxs * c.dx, nys * c.dy);
        launch_rotate(c, c.pl->js0x.p, c.pl->js0x.n, nxs * c.dx, nys * c.dy, nys);
        launch_rotate(c, c.pl->js0y.p, c.pl->js0y.n, nxs * c.dx, nys * c.dy, nys);
        launch_rotate(c, c.pl->js0z.p, c.pl->js0z.n, nxs * c.dx, nys * c.dy, nys);
    }
}
static void window_shift_post(Ctx& c) {
    if (!c.P.move_x && !(c.yf && c.P.move_y)) return;
    double a[3];
    launch_centroid(c, a);
    c.cent_.push_back({a[0], a[1], a[2]});
}
static void window_shift_start(Ctx& c) {
    if (!c.P.move_x && !(c.yf && c.P.move_y)) return;
    if (long(c.cent_.size()) < c.P.window_lag) return;
    const std::array<double, 3> v = c.cent_.front();
    c.cent_.pop_front();
    if (v[2] <= 0) return;
    const double Lx = c.nx * c.dx, Ly = c.ny * c.dy;
    const int nxs = c.P.move_x ? int(std::lround((v[0] / v[2] - (c.X0 + 0.5 * Lx)) / c.dx)) : 0;
    const int nys = c.yf && c.P.move_y ? int(std::lround((v[1] / v[2] - (c.Y0 + 0.5 * Ly)) / c.dy)) : 0;
    if (std::abs(nxs) >= 2 || std::abs(nys) >= 2) shift_window(c, nxs, nys);
}
static void check_kernel_errors(Ctx& c);
static void init_fields(Ctx& c) {
    c.s = 0; c.istep = 0;
    c.fields_ready = true;
    if (c.pl) reset_plasma_march(c);                 // a run starts with no streaming current and no waiting particle
    if (c.P.self_fields) {
        c.starting_ = true;
        if (c.nbunch > 1) comoving_fields_per_bunch(c);
        else { currents(c); comoving_field(c); }
        if (c.P.start_relax) relax_start_field(c);
        add_grid_lasers(c);
        march(c, 0.0);
        c.starting_ = false;
        sponge_and_real_fields(c);
        j0_from_jk(c);
    }
    window_shift_post(c);
}
static void step(Ctx& c, bool sync) {
    if (++c.steps_since_sort >= 16) sort_particles(c);
    window_shift_start(c);
    launch_push(c, c.s, c.s + c.P.dz);
    if (c.sharded()) shard_exchange_particles(c, c.s + c.P.dz);
    if (c.pl) collect_restreaming(c);
    c.s += c.P.dz; ++c.istep;
    if (c.P.self_fields && c.pl) {
        currents(c);
        march_plasma(c, c.s - c.P.dz, c.s);
        sponge_and_real_fields(c);
        j0_from_jk(c);
    } else if (c.P.self_fields) solve_fields(c, 0.5 * c.P.dz);
    if (!c.chicanes.empty()) apply_chicanes(c, c.s - c.P.dz, c.s);
    window_shift_post(c);
    if (sync) check_kernel_errors(c);
}
static bool finished(const Ctx& c) { return c.s >= c.P.z_end - 1e-9 || c.stop_; }
// the error word of the kernels' bounded waits (after the stream is synchronized): G3D_ERR_TIMEOUT, reset
static void check_kernel_errors(Ctx& c) {
    int e = 0;
    G3D_CUDA(cudaMemcpyAsync(&e, c.kerr.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
    if (e == 0) return;
    G3D_CUDA(cudaMemsetAsync(c.kerr.p, 0, sizeof(int), c.stream));
    throw Error(G3D_ERR_TIMEOUT, "a tile load of the TMA column transforms did not land within its bounded wait");
}

// ---------------------------------------------------------------- arrays
// Storage of an array id: device pointer, element count and size of the storage, the planes of a spectrum
// (0 for the real arrays jw and F, which are stored in the reference layout), and whether the storage is the
// mixed form's (complex64 spectra, float jw) while the boundary keeps the reference's complex128 / double.
struct ArrayRef { void* p; size_t count, eb; long planes; bool narrow; };
static ArrayRef array_ref(Ctx& c, int which) {
    if (which == G3D_A_RHO_E || which == G3D_A_RHO_I) {            // the density lines of the plasma march
        const size_t nl = size_t(c.N) * size_t(c.nx + c.ny);
        if (!c.pl || (which == G3D_A_RHO_I && !c.pl->ion_lines)) return ArrayRef{nullptr, 0, sizeof(double), 0, false};
        return ArrayRef{c.pl->rhol.p + (which == G3D_A_RHO_I ? nl : 0), nl, sizeof(double), 0, false};
    }
    if (c.mixed && which != G3D_A_RX && which != G3D_A_RY && which != G3D_A_F) {
        DevBuf<cpxf>* cb = nullptr;
        long planes = c.ns;
        MixedBufs& m = c.mx;
        switch (which) {
            case G3D_A_EZ: cb = &m.Ez; break; case G3D_A_BZ: cb = &m.Bz; break;
            case G3D_A_LX: cb = &m.Lx; break; case G3D_A_LY: cb = &m.Ly; break;
            case G3D_A_J0X: cb = &m.j0x; planes = c.ns + 1; break;
            case G3D_A_J0Y: cb = &m.j0y; planes = c.ns + 1; break;
            case G3D_A_JKX: cb = c.jk_is_j0 ? &m.j0x : &m.jkx; planes = c.ns + 1; break;
            case G3D_A_JKY: cb = c.jk_is_j0 ? &m.j0y : &m.jky; planes = c.ns + 1; break;
            case G3D_A_JKZ: cb = &m.jkz; planes = c.ns + 1; break;
            case G3D_A_JW: return ArrayRef{m.jw.p, m.jw.n, sizeof(double), 0, true};
            default: throw Error(G3D_ERR_ARG, "unknown array id " + std::to_string(which));
        }
        return ArrayRef{cb->p, cb->n, sizeof(cpx), planes, true};
    }
    DevBuf<cpx>* cb = nullptr;
    long planes = c.ns;
    switch (which) {
        case G3D_A_RX: cb = &c.Rx; break; case G3D_A_RY: cb = &c.Ry; break;
        case G3D_A_EZ: cb = &c.Ez; break; case G3D_A_BZ: cb = &c.Bz; break;
        case G3D_A_LX: cb = &c.Lx; break; case G3D_A_LY: cb = &c.Ly; break;
        case G3D_A_J0X: cb = &c.j0x; planes = c.ns + 1; break;
        case G3D_A_J0Y: cb = &c.j0y; planes = c.ns + 1; break;
        case G3D_A_JKX: cb = c.jk_is_j0 ? &c.j0x : &c.jkx; planes = c.ns + 1; break;
        case G3D_A_JKY: cb = c.jk_is_j0 ? &c.j0y : &c.jky; planes = c.ns + 1; break;
        case G3D_A_JKZ: cb = &c.jkz; planes = c.ns + 1; break;
        case G3D_A_JW:
            if (c.jw_fixed) launch_deposit_finish(c);   // the reference's doubles at the boundary
            return ArrayRef{c.jw.p, c.jw.n, sizeof(double), 0, false};
        case G3D_A_F: return ArrayRef{c.F.p, c.F.n, sizeof(float), 0, false};
        default: throw Error(G3D_ERR_ARG, "unknown array id " + std::to_string(which));
    }
    return ArrayRef{cb->p, cb->n, sizeof(cpx), planes, false};
}
// Element count of an array in the reference layout (spectra in full: planes x ny x nx).
static size_t ref_count(Ctx& c, const ArrayRef& a) { return a.planes ? size_t(a.planes) * c.nk : a.count; }

// Copy out in the reference layout (spectra expanded from the half spectrum by X(-k) = conj X(k); the mixed
// form's complex64 and float values widened to complex128 and double).
static void get_array(Ctx& c, int which, void* host) {
    const ArrayRef a = array_ref(c, which);
    if (!a.planes && a.narrow) {
        std::vector<float> v(a.count);
        if (a.count) G3D_CUDA(cudaMemcpyAsync(v.data(), a.p, a.count * sizeof(float), cudaMemcpyDeviceToHost, c.stream));
        G3D_CUDA(cudaStreamSynchronize(c.stream));
        double* out = static_cast<double*>(host);
        for (size_t i = 0; i < a.count; ++i) out[i] = v[i];
    } else if (!a.planes) {
        if (a.count) G3D_CUDA(cudaMemcpyAsync(host, a.p, a.count * a.eb, cudaMemcpyDeviceToHost, c.stream));
    } else {
        DevBuf<cpx> full;
        full.alloc(ref_count(c, a), c.stream);
        if (a.narrow) launch_half_to_full_f(c, static_cast<const cpxf*>(a.p), full.p, a.planes);
        else launch_half_to_full(c, static_cast<const cpx*>(a.p), full.p, a.planes);
        G3D_CUDA(cudaMemcpyAsync(host, full.p, full.bytes(), cudaMemcpyDeviceToHost, c.stream));
        G3D_CUDA(cudaStreamSynchronize(c.stream));
    }
    G3D_CUDA(cudaStreamSynchronize(c.stream));
}
// Copy in from the reference layout (spectra keep k_x = 0 .. nx/2: the data are the spectra of real fields;
// the mixed form rounds to complex64 and float).
static void set_array(Ctx& c, int which, const void* host) {
    const ArrayRef a = array_ref(c, which);
    if (!a.planes && a.narrow) {
        const double* in = static_cast<const double*>(host);
        std::vector<float> v(a.count);
        for (size_t i = 0; i < a.count; ++i) v[i] = float(in[i]);
        if (a.count) G3D_CUDA(cudaMemcpyAsync(a.p, v.data(), a.count * sizeof(float), cudaMemcpyHostToDevice, c.stream));
        G3D_CUDA(cudaStreamSynchronize(c.stream));
    } else if (!a.planes) {
        if (a.count) G3D_CUDA(cudaMemcpyAsync(a.p, host, a.count * a.eb, cudaMemcpyHostToDevice, c.stream));
    } else {
        DevBuf<cpx> full;
        full.alloc(ref_count(c, a), c.stream);
        G3D_CUDA(cudaMemcpyAsync(full.p, host, full.bytes(), cudaMemcpyHostToDevice, c.stream));
        if (a.narrow) launch_full_to_half_f(c, full.p, static_cast<cpxf*>(a.p), a.planes);
        else launch_full_to_half(c, full.p, static_cast<cpx*>(a.p), a.planes);
        G3D_CUDA(cudaStreamSynchronize(c.stream));
    }
    G3D_CUDA(cudaStreamSynchronize(c.stream));
}

// ---------------------------------------------------------------- checkpoints (sim_checkpoint.cpp:9-58)
namespace {
const char MAGIC[8] = {'G', '3', 'D', 'C', 'K', 'P', 'T', '1'};
struct CkptHeader {                  // the reference's native struct layout (128 bytes on x86-64)
    char magic[8];
    int32_t ranks, rank, N, a, b, ns, nk, nx, ny, plasma;
    int64_t istep, lost, trapped, restreamed;
    double s, X0, Y0, beta_b, gm2_b;
    int32_t stop, ncent;
};
static_assert(sizeof(CkptHeader) == 128, "checkpoint header layout");
template <class T>
void put(FILE* f, const T* p, uint64_t n) {
    if (std::fwrite(&n, sizeof n, 1, f) != 1 || (n && std::fwrite(p, sizeof(T), n, f) != n)) throw Error(G3D_ERR_IO, "checkpoint: write error");
}
template <class T>
std::vector<T> get(FILE* f) {
    uint64_t n = 0;
    if (std::fread(&n, sizeof n, 1, f) != 1) throw Error(G3D_ERR_IO, "checkpoint: file too short");
    if (n > (uint64_t(1) << 40)) throw Error(G3D_ERR_IO, "checkpoint: corrupt array length");
    std::vector<T> v(n);
    if (n && std::fread(v.data(), sizeof(T), n, f) != n) throw Error(G3D_ERR_IO, "checkpoint: file too short");
    return v;
}
template <class T>
[[maybe_unused]] std::vector<T> d2h(Ctx& c, const T* p, size_t n) {
    std::vector<T> v(n);
    if (n) G3D_CUDA(cudaMemcpyAsync(v.data(), p, n * sizeof(T), cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
    return v;
}
}  // namespace

static void checkpoint_wait(Ctx& c);
static void write_checkpoint(Ctx& c, const char* path) {
    checkpoint_wait(c);
    CkptHeader h{};
    std::memcpy(h.magic, MAGIC, 8);
    h.ranks = 1; h.rank = 0; h.N = c.N; h.a = c.a; h.b = c.b; h.ns = c.ns; h.nk = c.nk; h.nx = c.nx; h.ny = c.ny;
    h.plasma = c.pl ? 1 : 0;
    h.istep = c.istep; h.lost = c.lost_total;
    long trapped = 0, restreamed = 0;
    get_plasma_counters(c, trapped, restreamed);
    h.trapped = trapped; h.restreamed = restreamed;
    h.s = c.s; h.X0 = c.X0; h.Y0 = c.Y0; h.beta_b = c.beta_b; h.gm2_b = c.gm2_b; h.stop = c.stop_; h.ncent = int(c.cent_.size());
    const std::string tmp = std::string(path) + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) throw Error(G3D_ERR_IO, "cannot write " + tmp);
    try {
        if (std::fwrite(&h, sizeof h, 1, f) != 1) throw Error(G3D_ERR_IO, "checkpoint: write error");
        for (int w : {G3D_A_RX, G3D_A_RY, G3D_A_EZ, G3D_A_BZ, G3D_A_LX, G3D_A_LY, G3D_A_J0X, G3D_A_J0Y}) {
            std::vector<cpx> v(ref_count(c, array_ref(c, w)));
            get_array(c, w, v.data());
            put(f, v.data(), v.size());
        }
        for (int k = 0; k < 3; ++k) {                              // js0x, js0y, js0z: the streaming current of s0
            if (c.pl) { const std::vector<cpx> v = get_js0(c, k); put(f, v.data(), v.size()); }
            else put<cpx>(f, nullptr, 0);
        }
        const std::vector<float> fv = d2h(c, c.F.p, c.F.n);
        put(f, fv.data(), fv.size());
        const std::vector<g3d_particle> pv = get_particles(c);
        put(f, pv.data(), pv.size());
        if (c.pl) { const std::vector<g3d_particle> jv = get_joining(c); put(f, jv.data(), jv.size()); }
        else put<g3d_particle>(f, nullptr, 0);                     // joining: no plasma
        for (const auto& v : c.cent_) put(f, v.data(), 3);
    } catch (...) { std::fclose(f); throw; }
    std::fclose(f);
    if (std::rename(tmp.c_str(), path) != 0) throw Error(G3D_ERR_IO, std::string("cannot rename to ") + path);
}

// ---------------------------------------------------------------- asynchronous checkpoints
// The checkpoint above stops the caller until the file is written: the arrays go to the host one by one with the
// stream drained. The asynchronous one copies the state on the device, on the context's stream (so the next calls
// may change the state at once), and a host thread of the library waits for that copy, brings it to the host plane by
// plane, expands the half spectra to the reference's full layout on the host (as k_half_to_full does) and writes the
// same file while the march goes on. One job per context; a new one, the synchronous checkpoints, g3d_checkpoint_wait
// and g3d_destroy wait for the one in flight.
struct CkptJob {
    std::thread th;
    int code = G3D_OK;
    std::string msg;
    cudaStream_t s2 = nullptr;
    cudaEvent_t ready = nullptr;
    ~CkptJob() {
        if (th.joinable()) th.join();
        if (ready) cudaEventDestroy(ready);
        if (s2) cudaStreamDestroy(s2);
    }
};
// the job in flight ends; its outcome (the error of a failed write is thrown here, once)
static void checkpoint_wait(Ctx& c) {
    if (!c.ckjob) return;
    CkptJob& j = *static_cast<CkptJob*>(c.ckjob.get());
    if (j.th.joinable()) j.th.join();
    const int code = j.code;
    const std::string msg = j.msg;
    c.ckjob.reset();
    if (code != G3D_OK) throw Error(code, msg);
}

static void write_checkpoint_async(Ctx& c, const char* path) {
    checkpoint_wait(c);
    auto job = std::make_shared<CkptJob>();
    CkptJob& J = *job;
    cudaStream_t st = c.stream;
    // what the file holds, in its order: the spectra, js0, F, the particles, the joining list, the centroid history
    struct Seg { size_t off, bytes; long planes; bool narrow; };
    std::vector<Seg> spec;
    size_t tot = 0;
    auto add = [&](size_t bytes) { const size_t o = tot; tot += (bytes + 255) / 256 * 256; return o; };
    const int ws[8] = {G3D_A_RX, G3D_A_RY, G3D_A_EZ, G3D_A_BZ, G3D_A_LX, G3D_A_LY, G3D_A_J0X, G3D_A_J0Y};
    std::vector<ArrayRef> refs;
    for (int w : ws) {
        const ArrayRef a = array_ref(c, w);
        const size_t b = a.count * (a.narrow ? sizeof(cpxf) : sizeof(cpx));
        spec.push_back(Seg{add(b), b, a.planes, a.narrow});
        refs.push_back(a);
    }
    const bool pl = c.pl != nullptr;
    const size_t hb = size_t(c.ns + 1) * c.nkh * sizeof(cpx);
    size_t ojs[3] = {0, 0, 0};
    if (pl) for (int k = 0; k < 3; ++k) ojs[k] = add(hb);
    const size_t oF = add(c.F.n * sizeof(float));
    const long np = c.np;
    const size_t oP = add(size_t(np) * sizeof(g3d_particle));
    const long njb = pl ? c.pl->njb : 0;
    const size_t oJ = add(size_t(njb) * (10 * 8 + 2 * 4 + 8));
    if (c.ckpt_snap.n < tot) c.ckpt_snap.alloc(tot, st);
    unsigned char* S = c.ckpt_snap.p;
    for (size_t q = 0; q < spec.size(); ++q)
        if (spec[q].bytes) G3D_CUDA(cudaMemcpyAsync(S + spec[q].off, refs[q].p, spec[q].bytes, cudaMemcpyDeviceToDevice, st));
    if (pl) {
        const cpx* js[3] = {c.pl->js0x.p, c.pl->js0y.p, c.pl->js0z.p};
        for (int k = 0; k < 3; ++k) G3D_CUDA(cudaMemcpyAsync(S + ojs[k], js[k], hb, cudaMemcpyDeviceToDevice, st));
    }
    if (c.F.n) G3D_CUDA(cudaMemcpyAsync(S + oF, c.F.p, c.F.n * sizeof(float), cudaMemcpyDeviceToDevice, st));
    if (np) {
        if (c.pstage.n < size_t(np)) c.pstage.alloc(size_t(np) + size_t(np) / 4 + 64, st);
        launch_parts_pack(c, np);
        G3D_CUDA(cudaMemcpyAsync(S + oP, c.pstage.p, size_t(np) * sizeof(g3d_particle), cudaMemcpyDeviceToDevice, st));
    }
    if (njb) {                                        // the device joining list as columns: 10 doubles, alive, sp, id
        const StrmDev& V = c.pl->jb.v;
        const double* dc[10] = {V.x, V.y, V.zeta, V.px, V.py, V.pz, V.w, V.z, V.q, V.qm};
        unsigned char* o = S + oJ;
        for (int m = 0; m < 10; ++m, o += size_t(njb) * 8) G3D_CUDA(cudaMemcpyAsync(o, dc[m], size_t(njb) * 8, cudaMemcpyDeviceToDevice, st));
        G3D_CUDA(cudaMemcpyAsync(o, V.alive, size_t(njb) * 4, cudaMemcpyDeviceToDevice, st)); o += size_t(njb) * 4;
        G3D_CUDA(cudaMemcpyAsync(o, V.sp, size_t(njb) * 4, cudaMemcpyDeviceToDevice, st)); o += size_t(njb) * 4;
        G3D_CUDA(cudaMemcpyAsync(o, V.id, size_t(njb) * 8, cudaMemcpyDeviceToDevice, st));
    }
    G3D_CUDA(cudaEventCreateWithFlags(&J.ready, cudaEventDisableTiming));
    G3D_CUDA(cudaEventRecord(J.ready, st));
    G3D_CUDA(cudaStreamCreateWithFlags(&J.s2, cudaStreamNonBlocking));
    // the host values of the header and the rest, as they are now
    CkptHeader h{};
    std::memcpy(h.magic, MAGIC, 8);
    h.ranks = 1; h.rank = 0; h.N = c.N; h.a = c.a; h.b = c.b; h.ns = c.ns; h.nk = c.nk; h.nx = c.nx; h.ny = c.ny;
    h.plasma = pl ? 1 : 0;
    h.istep = c.istep; h.lost = c.lost_total;
    long trapped = 0, restreamed = 0;
    get_plasma_counters(c, trapped, restreamed);
    h.trapped = trapped; h.restreamed = restreamed;
    h.s = c.s; h.X0 = c.X0; h.Y0 = c.Y0; h.beta_b = c.beta_b; h.gm2_b = c.gm2_b; h.stop = c.stop_; h.ncent = int(c.cent_.size());
    std::vector<std::array<double, 3>> cent(c.cent_.begin(), c.cent_.end());
    std::vector<g3d_particle> joining_host = pl ? c.pl->joining : std::vector<g3d_particle>();
    const int dev = c.device, nx = c.nx, ny = c.ny, H = c.H, yf = c.yf ? 1 : 0;
    const long nkh = c.nkh, nk = c.nk, fn = long(c.F.n);
    const std::string out = path;
    J.th = std::thread([&J, S, spec, ojs, oF, oP, oJ, np, njb, pl, h, cent, joining_host, dev, nx, ny, H, yf, nkh, nk, fn, hb, out]() {
        FILE* f = nullptr;
        const std::string tmp = out + ".tmp";
        try {
            G3D_CUDA(cudaSetDevice(dev));
            G3D_CUDA(cudaEventSynchronize(J.ready));
            f = std::fopen(tmp.c_str(), "wb");
            if (!f) throw Error(G3D_ERR_IO, "cannot write " + tmp);
            auto wr = [&](const void* p, size_t b) {
                if (b && std::fwrite(p, 1, b, f) != b) throw Error(G3D_ERR_IO, "checkpoint: write error");
            };
            auto d2h = [&](void* dst, const unsigned char* src, size_t b) {
                if (!b) return;
                G3D_CUDA(cudaMemcpyAsync(dst, src, b, cudaMemcpyDeviceToHost, J.s2));
                G3D_CUDA(cudaStreamSynchronize(J.s2));
            };
            wr(&h, sizeof h);
            // the spectra: per plane the half spectrum widened and expanded to the full layout (k_half_to_full)
            std::vector<cpx> half(static_cast<size_t>(nkh)), full(static_cast<size_t>(nk));
            std::vector<cpxf> halff(static_cast<size_t>(nkh));
            auto expand = [&](const std::vector<cpx>& hv) {
                for (int j = 0; j < ny; ++j) {
                    const int jm = yf ? (ny - j) % ny : j;
                    for (int ix = 0; ix < nx; ++ix) {
                        const cpx v = ix <= nx / 2 ? hv[size_t(j) * H + ix] : conj(hv[size_t(jm) * H + (nx - ix)]);
                        full[size_t(j) * nx + ix] = v;
                    }
                }
            };
            for (const Seg& g : spec) {
                const uint64_t cnt = uint64_t(g.planes) * uint64_t(nk);
                wr(&cnt, sizeof cnt);
                for (long q = 0; q < g.planes; ++q) {
                    if (g.narrow) {
                        d2h(halff.data(), S + g.off + size_t(q) * nkh * sizeof(cpxf), size_t(nkh) * sizeof(cpxf));
                        for (long i = 0; i < nkh; ++i) half[size_t(i)] = to_d(halff[size_t(i)]);
                    } else {
                        d2h(half.data(), S + g.off + size_t(q) * nkh * sizeof(cpx), size_t(nkh) * sizeof(cpx));
                    }
                    expand(half);
                    wr(full.data(), size_t(nk) * sizeof(cpx));
                }
            }
            for (int k = 0; k < 3; ++k) {                 // js0: the streaming current of s0, full layout
                const uint64_t cnt = pl ? uint64_t(hb / sizeof(cpx) / nkh) * uint64_t(nk) : 0;
                wr(&cnt, sizeof cnt);
                for (uint64_t q = 0; pl && q < uint64_t(hb / sizeof(cpx) / nkh); ++q) {
                    d2h(half.data(), S + ojs[k] + size_t(q) * nkh * sizeof(cpx), size_t(nkh) * sizeof(cpx));
                    expand(half);
                    wr(full.data(), size_t(nk) * sizeof(cpx));
                }
            }
            {                                             // F, in chunks
                const uint64_t cnt = uint64_t(fn);
                wr(&cnt, sizeof cnt);
                std::vector<float> buf(size_t(1) << 22);
                for (long o = 0; o < fn; o += long(buf.size())) {
                    const size_t m = size_t(std::min<long>(long(buf.size()), fn - o));
                    d2h(buf.data(), S + oF + size_t(o) * sizeof(float), m * sizeof(float));
                    wr(buf.data(), m * sizeof(float));
                }
            }
            {                                             // the particles
                const uint64_t cnt = uint64_t(np);
                wr(&cnt, sizeof cnt);
                std::vector<g3d_particle> buf(size_t(1) << 16);
                for (long o = 0; o < np; o += long(buf.size())) {
                    const size_t m = size_t(std::min<long>(long(buf.size()), np - o));
                    d2h(buf.data(), S + oP + size_t(o) * sizeof(g3d_particle), m * sizeof(g3d_particle));
                    wr(buf.data(), m * sizeof(g3d_particle));
                }
            }
            if (pl) {                                     // the joining list: the device's, then the host's
                std::vector<unsigned char> raw(size_t(njb) * (10 * 8 + 2 * 4 + 8));
                d2h(raw.data(), S + oJ, raw.size());
                std::vector<g3d_particle> jv(static_cast<size_t>(njb));
                const double* dc = reinterpret_cast<const double*>(raw.data());
                const int32_t* ic = reinterpret_cast<const int32_t*>(raw.data() + size_t(njb) * 80);
                const uint64_t* uc = reinterpret_cast<const uint64_t*>(raw.data() + size_t(njb) * 88);
                for (long k = 0; k < njb; ++k) {
                    g3d_particle& p = jv[size_t(k)];
                    double* dst[10] = {&p.x, &p.y, &p.zeta, &p.px, &p.py, &p.pz, &p.w, &p.z, &p.q, &p.qm};
                    for (int m = 0; m < 10; ++m) *dst[m] = dc[size_t(m) * njb + k];
                    p.alive = ic[k]; p.sp = ic[njb + k]; p.id = uc[k];
                }
                jv.insert(jv.end(), joining_host.begin(), joining_host.end());
                const uint64_t cnt = jv.size();
                wr(&cnt, sizeof cnt);
                wr(jv.data(), jv.size() * sizeof(g3d_particle));
            } else {
                const uint64_t cnt = 0;
                wr(&cnt, sizeof cnt);
            }
            for (const auto& v : cent) { const uint64_t cnt = 3; wr(&cnt, sizeof cnt); wr(v.data(), 3 * sizeof(double)); }
            if (std::fclose(f) != 0) { f = nullptr; throw Error(G3D_ERR_IO, "checkpoint: write error"); }
            f = nullptr;
            if (std::rename(tmp.c_str(), out.c_str()) != 0) throw Error(G3D_ERR_IO, "cannot rename to " + out);
        } catch (const Error& e) {
            if (f) std::fclose(f);
            J.code = e.code; J.msg = e.what();
        } catch (const std::exception& e) {
            if (f) std::fclose(f);
            J.code = G3D_ERR_IO; J.msg = e.what();
        }
    });
    c.ckjob = job;
}

static void read_checkpoint(Ctx& c, const char* path) {
    checkpoint_wait(c);
    FILE* f = std::fopen(path, "rb");
    if (!f) throw Error(G3D_ERR_IO, std::string("cannot read ") + path);
    try {
        CkptHeader h{};
        if (std::fread(&h, sizeof h, 1, f) != 1 || std::memcmp(h.magic, MAGIC, 8))
            throw Error(G3D_ERR_IO, std::string(path) + ": not a GEM-PIC-3D checkpoint");
        if (h.ranks != 1) throw Error(G3D_ERR_IO, std::string(path) + ": written by " + std::to_string(h.ranks) + " ranks; restart with as many");
        if (h.N != c.N || h.a != c.a || h.b != c.b || h.nx != c.nx || h.ny != c.ny || h.plasma != (c.pl ? 1 : 0))
            throw Error(G3D_ERR_IO, std::string(path) + ": the grid (nx, ny, zeta slices) or the plasma differ");
        std::vector<std::vector<cpx>> arrays;
        for (int k = 0; k < 11; ++k) arrays.push_back(get<cpx>(f));
        const std::vector<float> fv = get<float>(f);
        const std::vector<g3d_particle> pv = get<g3d_particle>(f);
        const std::vector<g3d_particle> jv = get<g3d_particle>(f);
        std::deque<std::array<double, 3>> cent;
        for (int k = 0; k < h.ncent; ++k) {
            const std::vector<double> v = get<double>(f);
            if (v.size() != 3) throw Error(G3D_ERR_IO, std::string(path) + ": bad centroid record");
            cent.push_back({v[0], v[1], v[2]});
        }
        std::fclose(f);
        f = nullptr;
        if (fv.size() != c.F.n) throw Error(G3D_ERR_IO, std::string(path) + ": array sizes differ from the grid");
        c.jk_is_j0 = false;
        const int ids[8] = {G3D_A_RX, G3D_A_RY, G3D_A_EZ, G3D_A_BZ, G3D_A_LX, G3D_A_LY, G3D_A_J0X, G3D_A_J0Y};
        for (int k = 0; k < 8; ++k)
            if (arrays[size_t(k)].size() != ref_count(c, array_ref(c, ids[k])))
                throw Error(G3D_ERR_IO, std::string(path) + ": array sizes differ from the grid");
        for (int k = 0; k < 8; ++k) set_array(c, ids[k], arrays[size_t(k)].data());
        if (!c.pl) {
            for (int k = 8; k < 11; ++k)
                if (!arrays[size_t(k)].empty()) throw Error(G3D_ERR_IO, std::string(path) + ": streaming currents present but no plasma");
            if (!jv.empty()) throw Error(G3D_ERR_IO, std::string(path) + ": joining particles present but no plasma");
        } else {
            for (int k = 8; k < 11; ++k) set_js0(c, k - 8, arrays[size_t(k)]);
            set_joining(c, jv);
            set_plasma_counters(c, h.trapped, h.restreamed);
        }
        G3D_CUDA(cudaMemcpyAsync(c.F.p, fv.data(), c.F.bytes(), cudaMemcpyHostToDevice, c.stream));
        set_particles(c, pv.data(), long(pv.size()));
        c.istep = h.istep; c.lost_total = h.lost; c.s = h.s; c.X0 = h.X0; c.Y0 = h.Y0;
        c.beta_b = h.beta_b; c.gm2_b = h.gm2_b; c.stop_ = h.stop != 0;
        c.cent_ = cent;
        c.fields_ready = true;
        G3D_CUDA(cudaStreamSynchronize(c.stream));
    } catch (...) {
        if (f) std::fclose(f);
        throw;
    }
}


// ---------------------------------------------------------------- adjoint march
// Laser mode coefficients a(k) (per stored mode [j][k_x]) multiply every grid laser's spectrum added at init;
// the unmultiplied spectra are kept for the gradient. They take effect at the next g3d_init.
static void set_laser_modes(Ctx& c, const double* coef) {
    std::vector<cpx> a(size_t(c.nkh), C(1.0));
    if (coef)
        for (size_t i = 0; i < a.size(); ++i) a[i] = C(coef[2 * i], coef[2 * i + 1]);
    c.lmode.upload(a, c.stream);
    c.lspx.alloc(size_t(c.ns) * c.nkh, c.stream);
    c.lspy.alloc(size_t(c.ns) * c.nkh, c.stream);
    G3D_CUDA(cudaStreamSynchronize(c.stream));
}
// Exact fields: the real fields are also kept in FP64 and the beam push gathers from them (the differentiable
// forward that central differences are taken of). FP64 form; they take effect at the next g3d_init.
static void set_exact_fields(Ctx& c, bool on) {
    if (on && c.mixed) throw Error(G3D_ERR_ARG, "exact fields are an option of the FP64 form");
    if (on) c.Fd.alloc(c.F.n, c.stream);
    else c.Fd.release();
    G3D_CUDA(cudaStreamSynchronize(c.stream));
}
// What dJ/dp of the adjoint holds: through the start field (false) or with the start field held (true).
static void set_adjoint_momenta(Ctx& c, int mode) {
    if (mode != G3D_ADJ_THROUGH_START && mode != G3D_ADJ_AFTER_START) throw Error(G3D_ERR_ARG, "unknown adjoint momentum mode");
    c.adj_after_start = mode == G3D_ADJ_AFTER_START;
}
// From the start field (right after g3d_init): K s-steps forward with a checkpoint of the beam (x, y, zeta,
// p, alive) and of the real fields at every level (with a streaming plasma also the spectra R, E_z, B_z, j0 and the
// streaming current js0: each step is run again from its level in the reverse sweep, with the march recorded, and
// its march transposed, k_adj_plasma.cu), J = mean p_z of the live beam, then the reverse sweep
// (k_adjoint.cu): per step the transposed real fields, march, currents, deposit and push; then init's march(0),
// relaxation marches and co-moving fields back to the start currents and beta. Out: J, dJ/da per stored laser
// mode [j][k_x] (complex, interleaved) and dJ/dp of every particle at s = 0 [np][3] through both the s-steps and
// the start field the bunch made (its currents, its beta), or (G3D_ADJ_AFTER_START) through the s-steps alone, the
// momenta then being those the start field was made with held apart from it. The forward leaves the run at
// s = K dz, as K calls of g3d_step; g3d_set_particles + g3d_init start the next evaluation on the same context,
// which reuses the workspace.
static void adjoint(Ctx& c, int K, double* J, double* grad_modes, double* grad_p) {
    if (K < 1) throw Error(G3D_ERR_ARG, "the adjoint march needs at least one s-step");
    if (!c.yf) throw Error(G3D_ERR_ARG, "the adjoint march needs the Fourier y grid");
    const bool plasma = c.pl != nullptr;
    if (plasma) {
        if (!c.mixed && !c.Fd.p)
            throw Error(G3D_ERR_ARG, "the FP64 form's adjoint of the streaming plasma differentiates the forward with exact fields "
                                     "(g3d_set_exact_fields)");
        if (c.pl->any_ionizing) throw Error(G3D_ERR_ARG, "the adjoint march does not differentiate ionization");
        if (c.pl->njb || !c.pl->joining.empty())
            throw Error(G3D_ERR_STATE, "the adjoint march starts with no particle waiting to join the streaming plasma");
    }
    if (c.P.sponge > 0 || c.P.sponge_y > 0) throw Error(G3D_ERR_ARG, "the adjoint march needs sponge = 0");
    if (c.P.move_x || c.P.move_y) throw Error(G3D_ERR_ARG, "the adjoint march needs a fixed window (move_x = move_y = 0)");
    if (c.laser.on) throw Error(G3D_ERR_ARG, "the adjoint march differentiates grid lasers, not the analytic laser");
    if (!c.P.self_fields || c.P.freeze_bunch) throw Error(G3D_ERR_ARG, "the adjoint march needs self fields and a free bunch");
    if (!c.fields_ready || c.istep != 0) throw Error(G3D_ERR_STATE, "the adjoint march starts right after g3d_init");
    if (c.world > 1) throw Error(G3D_ERR_STATE, "the adjoint march of a sharded run is not built");
    if (c.ext.any() || !c.chicanes.empty())
        throw Error(G3D_ERR_STATE, "the adjoint march does not differentiate external elements or chicanes");
    if (grad_modes && !c.lmode.p) throw Error(G3D_ERR_STATE, "set the laser mode coefficients (g3d_set_laser_modes) before g3d_init");
    const long np = c.np;
    const size_t Fn = c.F.n, ns = size_t(c.ns), nkh = size_t(c.nkh), nk = size_t(c.nk);
    const bool ex = c.Fd.p != nullptr;
    const bool fdl = ex || plasma;                   // the levels' real fields in FP64 (the mixed form's float F widened)
    cudaStream_t st = c.stream;
    // one workspace, kept between calls: the checkpoints of the K + 1 levels (beam x, y, zeta, p; alive; the real
    // fields), the adjoints of the spectra, currents, real fields and beam, and transform scratch
    size_t need = 0;
    auto carve = [&](size_t bytes) { const size_t o = need; need += (bytes + 255) / 256 * 256; return o; };
    const size_t oX = carve(size_t(K + 1) * 6 * size_t(np) * 8), oAL = carve(size_t(K + 1) * size_t(np) * 4);
    const size_t oF = carve(size_t(K + 1) * Fn * (fdl ? 8 : 4));
    size_t oS[6], oj0[2], ojk[3], oW[6];
    for (auto& o : oS) o = carve(ns * nkh * sizeof(cpx));
    for (auto& o : oj0) o = carve((ns + 1) * nkh * sizeof(cpx));
    for (auto& o : ojk) o = carve((ns + 1) * nkh * sizeof(cpx));
    for (auto& o : oW) o = carve((ns + 1) * nkh * sizeof(cpx));
    const size_t olF = carve(Fn * 8), oV = carve(3 * (ns + 1) * nk * 8), olJ = carve(3 * (ns + 3) * nk * 8);
    const size_t olam = carve(6 * size_t(np) * 8), oerr = carve(sizeof(int)), ojo = carve(2 * 8), ogm = carve(nkh * sizeof(cpx));
    // the start field's dependence on the bunch: j_z of the start currents, dJ/dR of the relaxation's beta part,
    // dJ/dbeta per mode
    const size_t ojz = carve((ns + 1) * nkh * sizeof(cpx)), odx = carve(2 * ns * nkh * sizeof(cpx)), odb = carve(nkh * 8);
    // with a streaming plasma: per level the spectra R_x, R_y, E_z, B_z, j0 (x, y) and js0 (x, y, z); the adjoints of
    // js0 and of one slice's values, the adjoint's carried planes and one plane each of transform scratch
    const size_t lv = plasma ? size_t(K + 1) : 0, hp = (ns + 1) * nkh;
    const size_t oSP = carve(lv * 4 * ns * nkh * sizeof(cpx)), oJ0 = carve(lv * 2 * hp * sizeof(cpx)), oJS = carve(lv * 3 * hp * sizeof(cpx));
    const size_t ojs0 = carve(plasma ? 3 * hp * sizeof(cpx) : 0), osl = carve(plasma ? 31 * nkh * sizeof(cpx) : 0);
    const size_t oFa = carve(plasma ? 21 * nk * 8 : 0);
    if (c.adjws.n < need) c.adjws.alloc(need, st);
    unsigned char* ws = c.adjws.p;
    double* X = reinterpret_cast<double*>(ws + oX);
    int32_t* AL = reinterpret_cast<int32_t*>(ws + oAL);
    float* FF = fdl ? nullptr : reinterpret_cast<float*>(ws + oF);
    double* FD = fdl ? reinterpret_cast<double*>(ws + oF) : nullptr;
    cpx* lS[6]; cpx* lj0[2]; cpx* ljk[3]; cpx* W[6];
    for (int q = 0; q < 6; ++q) { lS[q] = reinterpret_cast<cpx*>(ws + oS[q]); W[q] = reinterpret_cast<cpx*>(ws + oW[q]); }
    for (int q = 0; q < 2; ++q) lj0[q] = reinterpret_cast<cpx*>(ws + oj0[q]);
    for (int q = 0; q < 3; ++q) ljk[q] = reinterpret_cast<cpx*>(ws + ojk[q]);
    double* lF = reinterpret_cast<double*>(ws + olF);
    double* V = reinterpret_cast<double*>(ws + oV);
    double* lJ = reinterpret_cast<double*>(ws + olJ);
    double* lam = reinterpret_cast<double*>(ws + olam);
    int* err = reinterpret_cast<int*>(ws + oerr);
    double* jo = reinterpret_cast<double*>(ws + ojo);
    cpx* gmd = reinterpret_cast<cpx*>(ws + ogm);
    cpx* jz0 = reinterpret_cast<cpx*>(ws + ojz);
    cpx* ldx = reinterpret_cast<cpx*>(ws + odx);
    double* dbm = reinterpret_cast<double*>(ws + odb);
    cpx* SP = reinterpret_cast<cpx*>(ws + oSP);
    cpx* J0 = reinterpret_cast<cpx*>(ws + oJ0);
    cpx* JS = reinterpret_cast<cpx*>(ws + oJS);
    AdjPlasmaPtrs ap{};
    AdjPlasmaWs aw{};
    if (plasma) {
        ap.nkh = long(nkh);
        for (int q = 0; q < 6; ++q) ap.lS[q] = lS[q];
        cpx* js = reinterpret_cast<cpx*>(ws + ojs0);
        for (int q = 0; q < 3; ++q) ap.ljs0[q] = js + q * hp;
        cpx* sl0 = reinterpret_cast<cpx*>(ws + osl);           // 31 planes: lsl 6, lold 4, ljsnA 3, ljsn 3, ldl 3, lsi0 6, W 6
        for (int q = 0; q < 6; ++q) ap.lsl[q] = sl0 + q * nkh;
        ap.lold = sl0 + 6 * nkh; ap.ljsnA = sl0 + 10 * nkh; ap.ljsn = sl0 + 13 * nkh; ap.ldl = sl0 + 16 * nkh;
        ap.lsi0[0] = sl0 + 19 * nkh; ap.lsi0[1] = sl0 + 22 * nkh;
        for (int q = 0; q < 6; ++q) aw.Wsc[q] = sl0 + (25 + q) * nkh;
        for (int q = 0; q < 3; ++q) aw.Tsc[q] = W[q] ;                // the currents' scratch is free during the march
        double* fa = reinterpret_cast<double*>(ws + oFa);      // 21 real planes: lFup 2 x 6, lFcur 6, ljsr 3
        aw.lFup[0] = fa; aw.lFup[1] = fa + 6 * nk; aw.lFcur = fa + 12 * nk; aw.ljsr = fa + 18 * nk;
    }
    // the start currents' j_z (init deposited them; jkz is not swapped into j0)
    if (c.mixed) launch_adj_widen(c, c.mx.jkz.p, jz0, long((ns + 1) * nkh));
    else G3D_CUDA(cudaMemcpyAsync(jz0, c.jkz.p, (ns + 1) * nkh * sizeof(cpx), cudaMemcpyDeviceToDevice, st));
    const double beta0 = c.beta_b, gm20 = c.gm2_b;
    std::vector<double> sl(size_t(K + 1));
    // the plasma state of a level: the spectra R_x, R_y, E_z, B_z (the march reads their old values), j0 x, y, js0
    auto plasma_state = [&](int k, bool out) {
        cpx* sp_[4] = {c.Rx.p, c.Ry.p, c.Ez.p, c.Bz.p};
        cpx* j0_[2] = {c.j0x.p, c.j0y.p};
        cpx* js_[3] = {c.pl->js0x.p, c.pl->js0y.p, c.pl->js0z.p};
        const cudaMemcpyKind d2d = cudaMemcpyDeviceToDevice;
        for (int q = 0; q < 4; ++q) {
            cpx* ck = SP + (size_t(k) * 4 + q) * ns * nkh;
            G3D_CUDA(cudaMemcpyAsync(out ? ck : sp_[q], out ? sp_[q] : ck, ns * nkh * sizeof(cpx), d2d, st));
        }
        for (int q = 0; q < 2; ++q) {
            cpx* ck = J0 + (size_t(k) * 2 + q) * hp;
            G3D_CUDA(cudaMemcpyAsync(out ? ck : j0_[q], out ? j0_[q] : ck, hp * sizeof(cpx), d2d, st));
        }
        for (int q = 0; q < 3; ++q) {
            cpx* ck = JS + (size_t(k) * 3 + q) * hp;
            G3D_CUDA(cudaMemcpyAsync(out ? ck : js_[q], out ? js_[q] : ck, hp * sizeof(cpx), d2d, st));
        }
    };
    // the particles waiting to join the streaming plasma at each level (slow trapped ones of the step before; few)
    std::vector<std::vector<g3d_particle>> joins(plasma ? size_t(K + 1) : 0);
    auto save = [&](int k) {
        if (plasma) joins[size_t(k)] = get_joining(c);
        double* x = X + size_t(k) * 6 * size_t(np);
        double* src[6] = {c.parts.x, c.parts.y, c.parts.zeta, c.parts.px, c.parts.py, c.parts.pz};
        if (np > 0) {
            for (int q = 0; q < 6; ++q)
                G3D_CUDA(cudaMemcpyAsync(x + size_t(q) * np, src[q], size_t(np) * 8, cudaMemcpyDeviceToDevice, st));
            G3D_CUDA(cudaMemcpyAsync(AL + size_t(k) * np, c.parts.alive, size_t(np) * 4, cudaMemcpyDeviceToDevice, st));
        }
        if (plasma && !c.mixed) plasma_state(k, true);   // the mixed form keeps the records: no step is run again
        sl[size_t(k)] = c.s;
    };
    // back to level k (the beam, the exact real fields, the plasma state, s), to run step k + 1 again
    auto restore = [&](int k) {
        const double* x = X + size_t(k) * 6 * size_t(np);
        double* dst[6] = {c.parts.x, c.parts.y, c.parts.zeta, c.parts.px, c.parts.py, c.parts.pz};
        if (np > 0) {
            for (int q = 0; q < 6; ++q)
                G3D_CUDA(cudaMemcpyAsync(dst[q], x + size_t(q) * np, size_t(np) * 8, cudaMemcpyDeviceToDevice, st));
            G3D_CUDA(cudaMemcpyAsync(c.parts.alive, AL + size_t(k) * np, size_t(np) * 4, cudaMemcpyDeviceToDevice, st));
        }
        G3D_CUDA(cudaMemcpyAsync(c.Fd.p, FD + size_t(k) * Fn, Fn * 8, cudaMemcpyDeviceToDevice, st));
        plasma_state(k, false);
        set_joining(c, joins[size_t(k)]);
        c.jk_is_j0 = true;
        c.s = sl[size_t(k)];
        c.istep = k;
    };
    long tr0 = 0, rs0 = 0, npl_max = 0;
    if (plasma) get_plasma_counters(c, tr0, rs0);
    // The record of the marches (k_adj_plasma.cu): kept from the forward for every step when it fits in half of the free
    // device memory (stride rs: twice the fresh plasma's most particles, room for the joining ones), else, or when a
    // march outgrows rs, or with G3D_ADJ_RECOMPUTE set, each step is run again from its level in the reverse sweep with
    // one march's record (the checkpoints of the levels are the only memory that grows with K).
    struct RecInfo { RecDev rec; long np, fresh; };
    std::vector<RecInfo> recinfo(plasma ? size_t(K + 1) : 0);
    bool stored = false, overflow = false;
    size_t step_bytes = 0, common = 0;
    long rs_rec = 0;
    int k_cur = 0;
    auto rup = [](size_t b) { return (b + 255) / 256 * 256; };
    auto rec_bytes = [&](long rs) {
        const size_t passes = size_t(c.pl->cfg.iterations);
        return rup((ns + 1) * 7 * size_t(rs) * 8) + rup(ns * passes * 6 * nk * 8) + rup((ns + 1) * size_t(rs) * 4) + rup(2 * size_t(rs) * 8);
    };
    auto carve_rec = [&](unsigned char* base, long rs) {
        const size_t passes = size_t(c.pl->cfg.iterations);
        RecDev r{};
        size_t o = 0;
        r.x = reinterpret_cast<double*>(base + o); o += rup((ns + 1) * 7 * size_t(rs) * 8);
        r.f = reinterpret_cast<double*>(base + o); o += rup(ns * passes * 6 * nk * 8);
        r.a = reinterpret_cast<int32_t*>(base + o); o += rup((ns + 1) * size_t(rs) * 4);
        r.q = reinterpret_cast<double*>(base + o);
        r.rs = rs;
        return r;
    };
    // lam, jl (7 rs each) and the step's values after the records
    auto carve_common = [&](unsigned char* base, long rs) {
        aw.lam = reinterpret_cast<double*>(base);
        aw.jl = reinterpret_cast<double*>(base + rup(7 * size_t(rs) * 8));
        aw.stepd = reinterpret_cast<AdjStepDev*>(base + 2 * rup(7 * size_t(rs) * 8));
    };
    struct RecOff {
        PlasmaState* P;
        ~RecOff() { if (P) { P->rec_on = false; P->rec_step = nullptr; } }
    } rec_off{plasma ? c.pl.get() : nullptr};
    if (plasma) {
        PlasmaState& Pl = *c.pl;
        if (!Pl.recd.p) Pl.recd.alloc(1, st);
        long m = Pl.cfg.free_electrons ? 1 : 0;
        for (const auto& is : Pl.ions) m += is.loaded() ? 1 : 0;
        const long fresh_bound = long(c.yf ? c.ny : c.ny - 2) * c.nx * Pl.cfg.ppc_x * Pl.cfg.ppc_y * m;
        rs_rec = 2 * fresh_bound + 1024;
        step_bytes = rec_bytes(rs_rec);
        common = 2 * rup(7 * size_t(rs_rec) * 8) + rup(sizeof(AdjStepDev));
        size_t fr = 0, tot = 0;
        G3D_CUDA(cudaMemGetInfo(&fr, &tot));
        const size_t have = c.adjrec.n >= size_t(K) * step_bytes + common ? c.adjrec.n : 0;
        stored = !std::getenv("G3D_ADJ_RECOMPUTE") && (have || size_t(K) * step_bytes + common <= fr / 2);
        if (stored) {
            if (c.adjrec.n < size_t(K) * step_bytes + common) c.adjrec.alloc(size_t(K) * step_bytes + common, st);
            carve_common(c.adjrec.p + size_t(K) * step_bytes, rs_rec);
            Pl.rec_on = true;
            Pl.rec_step = [&](long nstrm, long fresh) {
                if (nstrm > rs_rec || k_cur < 1 || k_cur > K) { overflow = true; return false; }
                RecInfo& ri = recinfo[size_t(k_cur)];
                ri.rec = carve_rec(c.adjrec.p + size_t(k_cur - 1) * step_bytes, rs_rec);
                ri.np = nstrm; ri.fresh = fresh;
                G3D_CUDA(cudaMemcpyAsync(c.pl->recd.p, &ri.rec, sizeof(RecDev), cudaMemcpyHostToDevice, c.stream));
                return true;
            };
        }
    }
    // the real fields of level k are written by step k straight into checkpoint k (the push of step k + 1 reads
    // them there; with a plasma they are copied there after the step); the context's own F / Fd come back, with the
    // last level's fields, when the forward is done
    struct Own {
        Ctx& c; double* fd; float* f;
        ~Own() { c.Fd.p = fd; c.F.p = f; c.fd_next = nullptr; c.f_next = nullptr; }
    } own{c, c.Fd.p, c.F.p};
    if (ex) G3D_CUDA(cudaMemcpyAsync(FD, c.Fd.p, Fn * 8, cudaMemcpyDeviceToDevice, st));
    else if (fdl) launch_f2d(c, c.F.p, FD, long(Fn));
    else G3D_CUDA(cudaMemcpyAsync(FF, c.F.p, Fn * 4, cudaMemcpyDeviceToDevice, st));
    save(0);
    for (int k = 1; k <= K; ++k) {
        // with a plasma the march writes the real fields slice by slice into the context's F during the step, so
        // the step keeps its own F and the level is copied after it (the level before must stay as it was)
        if (plasma) {
            k_cur = k;
            step(c, false);
            if (ex) G3D_CUDA(cudaMemcpyAsync(FD + size_t(k) * Fn, c.Fd.p, Fn * 8, cudaMemcpyDeviceToDevice, st));
            else launch_f2d(c, c.F.p, FD + size_t(k) * Fn, long(Fn));
            npl_max = std::max(npl_max, c.pl->nstrm);
        } else {
            if (ex) c.fd_next = FD + size_t(k) * Fn;
            else c.f_next = FF + size_t(k) * Fn;
            step(c, false);
        }
        save(k);
    }
    if (plasma) {
        long tr = 0, rs = 0;
        get_plasma_counters(c, tr, rs);
        if (tr != tr0 || rs != rs0)
            throw Error(G3D_ERR_STATE, "the adjoint march does not differentiate particles that join the beam (fast trapped or "
                                       "restreamed ones), and the forward had some");
        c.pl->rec_on = false;
        if (c.mixed && (!stored || overflow))
            throw Error(G3D_ERR_CAPACITY, "the mixed form's adjoint of the streaming plasma keeps the records of every step, and "
                                          "they do not fit in half the free device memory (or G3D_ADJ_RECOMPUTE is set)");
        if (!stored || overflow) {                    // one march's record, filled by running each step again
            stored = false;
            const long rs = npl_max;
            const size_t need = rec_bytes(rs) + 2 * rup(7 * size_t(rs) * 8) + rup(sizeof(AdjStepDev));
            if (c.adjrec.n < need) c.adjrec.alloc(need, st);
            const RecDev one = carve_rec(c.adjrec.p, rs);
            carve_common(c.adjrec.p + rec_bytes(rs), rs);
            c.pl->rec_step = [&, one](long nstrm, long fresh) {
                if (nstrm > one.rs) return false;
                RecInfo& ri = recinfo[size_t(k_cur)];
                ri.rec = one; ri.np = nstrm; ri.fresh = fresh;
                G3D_CUDA(cudaMemcpyAsync(c.pl->recd.p, &ri.rec, sizeof(RecDev), cudaMemcpyHostToDevice, c.stream));
                return true;
            };
        }
    }
    if (ex) G3D_CUDA(cudaMemcpyAsync(own.fd, FD + size_t(K) * Fn, Fn * 8, cudaMemcpyDeviceToDevice, st));
    else if (!fdl) G3D_CUDA(cudaMemcpyAsync(own.f, FF + size_t(K) * Fn, Fn * 4, cudaMemcpyDeviceToDevice, st));
    c.Fd.p = own.fd; c.F.p = own.f;
    launch_adj_objective(c, jo);
    double jh[2];
    G3D_CUDA(cudaMemcpyAsync(jh, jo, 16, cudaMemcpyDeviceToHost, st));
    G3D_CUDA(cudaStreamSynchronize(st));
    if (!(jh[1] > 0)) throw Error(G3D_ERR_STATE, "the adjoint march: no live particle at the end");
    *J = jh[0] / jh[1];
    // the reverse sweep
    for (int q = 0; q < 6; ++q) G3D_CUDA(cudaMemsetAsync(lS[q], 0, ns * nkh * sizeof(cpx), st));
    for (int q = 0; q < 3; ++q) G3D_CUDA(cudaMemsetAsync(ljk[q], 0, (ns + 1) * nkh * sizeof(cpx), st));
    G3D_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st));
    if (np > 0) launch_adj_seed(c, jh[1], lam);
    if (plasma) G3D_CUDA(cudaMemsetAsync(ap.ljs0[0], 0, 3 * hp * sizeof(cpx), st));
    for (int k = K; k >= 1; --k) {
        if (k < K) launch_adj_real_fields(c, lF, W, lS);
        for (int q = 0; q < 2; ++q) G3D_CUDA(cudaMemsetAsync(lj0[q], 0, (ns + 1) * nkh * sizeof(cpx), st));
        if (plasma) {
            PlasmaState& Pl = *c.pl;
            if (!stored) {
                // step k again from level k-1 with its march recorded
                restore(k - 1);
                k_cur = k;
                const long tr1 = Pl.trapped_total;
                Pl.rec_on = true;
                step(c, false);
                Pl.rec_on = false;
                if (Pl.nstrm > npl_max || Pl.trapped_total != tr1)
                    throw Error(G3D_ERR_STATE, "the adjoint march: a step run again from its level did not repeat its plasma");
            }
            const RecInfo& ri = recinfo[size_t(k)];
            // the streaming particles' adjoints after the march: the slow trapped ones are the next march's joining ones
            G3D_CUDA(cudaMemsetAsync(aw.lam, 0, 7 * size_t(ri.rec.rs) * 8, st));
            const long njl = k < K ? long(joins[size_t(k)].size()) : 0;
            const long nslow = launch_join_adjoint_in(c, ri.rec, ri.np, aw.jl, njl, aw.lam);
            if (k < K && nslow != njl)
                throw Error(G3D_ERR_STATE, "the adjoint march: the trapped particles of a step differ from those joining the next");
            // the march transposed; the level k-1 fields' adjoint takes the reads of the streaming pushes, then those of
            // the beam push
            G3D_CUDA(cudaMemsetAsync(lF, 0, Fn * 8, st));
            G3D_CUDA(cudaMemsetAsync(ljk[2], 0, (ns + 1) * nkh * sizeof(cpx), st));
            for (int q = 0; q < 2; ++q) ap.lj0[q] = lj0[q];
            for (int q = 0; q < 3; ++q) ap.ljk[q] = ljk[q];
            AdjPlasmaWs awk = aw;
            awk.np = ri.np; awk.fresh = ri.fresh; awk.rec = ri.rec;
            adjoint_march_plasma(c, awk, ap, FD + size_t(k - 1) * Fn, lF, sl[size_t(k - 1)], sl[size_t(k)]);
            // the joining particles of this march (after its fresh plasma) pass their adjoints to the march before
            launch_join_adjoint_out(c, aw.lam, ri.rec.rs, ri.fresh, long(joins[size_t(k - 1)].size()), aw.jl);
            launch_adj_currents(c, ljk, W, V, lJ, Pl.box_mean);
        } else {
            launch_adj_march(c, lS, lj0, ljk, 0.5 * c.P.dz);
            launch_adj_currents(c, ljk, W, V, lJ);
        }
        launch_adj_deposit(c, X + size_t(k) * 6 * np, AL + size_t(k) * np, lJ, lam);
        for (int q = 0; q < 2; ++q) std::swap(ljk[q], lj0[q]);           // jk of level k-1 as the j0 of step k
        if (!plasma) G3D_CUDA(cudaMemsetAsync(lF, 0, Fn * 8, st));
        launch_adj_push(c, fdl ? nullptr : FF + size_t(k - 1) * Fn, fdl ? FD + size_t(k - 1) * Fn : nullptr, X + size_t(k - 1) * 6 * np,
                        AL + size_t(k - 1) * np, sl[size_t(k - 1)], sl[size_t(k)], lam, lF, err);
    }
    // level 0: the real fields of the start field, then init's march(0) back to R with the lasers added
    launch_adj_real_fields(c, lF, W, lS);
    for (int q = 0; q < 2; ++q) G3D_CUDA(cudaMemsetAsync(lj0[q], 0, (ns + 1) * nkh * sizeof(cpx), st));
    launch_adj_march(c, lS, lj0, ljk, 0.0);
    int eh = 0;
    G3D_CUDA(cudaMemcpyAsync(&eh, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (grad_modes) {
        launch_adj_lmodes(c, lS[0], lS[1], gmd);
        G3D_CUDA(cudaMemcpyAsync(grad_modes, gmd, nkh * sizeof(cpx), cudaMemcpyDeviceToHost, st));
        G3D_CUDA(cudaStreamSynchronize(st));
    }
    if (grad_p && np > 0 && !c.adj_after_start) {
        // dJ/dR before the lasers is dJ/dR of the start field R_co(beta) + (relaxed R_co(1) - R_co(1)): through the
        // three relaxation marches (D = 100 dz; their E_z, B_z, j0 are zeroed and their E_z, B_z, L outputs unread)
        // and the two co-moving fields, to the start currents' j_z and to beta
        const size_t pn = ns * nkh;
        if (c.P.start_relax) {
            for (int q = 0; q < 2; ++q) G3D_CUDA(cudaMemcpyAsync(ldx + q * pn, lS[q], pn * sizeof(cpx), cudaMemcpyDeviceToDevice, st));
            for (int it = 0; it < 3; ++it) {
                for (int q = 2; q < 6; ++q) G3D_CUDA(cudaMemsetAsync(lS[q], 0, pn * sizeof(cpx), st));
                for (int q = 0; q < 2; ++q) G3D_CUDA(cudaMemsetAsync(lj0[q], 0, (ns + 1) * nkh * sizeof(cpx), st));
                launch_adj_march(c, lS, lj0, ljk, 100 * c.P.dz, 1);
            }
            // dJ/dR_co(1) = (through the marches) - dJ/dR_co(beta)
            for (int q = 0; q < 2; ++q) launch_axpy_c(c, lS[q], ldx + q * pn, -1.0, pn);
            launch_adj_comoving(c, lS[0], lS[1], jz0, 1.0, 0.0, ljk[2], nullptr);
            launch_adj_comoving(c, ldx, ldx + pn, jz0, beta0, gm20, ljk[2], dbm);
        } else {
            launch_adj_comoving(c, lS[0], lS[1], jz0, beta0, gm20, ljk[2], dbm);
        }
        // the start currents (deposit of the bunch at s = 0) and beta = sum w p_z / gamma / sum w
        launch_adj_currents(c, ljk, W, V, lJ);
        launch_adj_deposit(c, X, AL, lJ, lam);
        std::vector<double> db(nkh);
        G3D_CUDA(cudaMemcpyAsync(db.data(), dbm, nkh * 8, cudaMemcpyDeviceToHost, st));
        launch_adj_wsum(c, AL, jo);
        double W0 = 0;
        G3D_CUDA(cudaMemcpyAsync(&W0, jo, 8, cudaMemcpyDeviceToHost, st));
        G3D_CUDA(cudaStreamSynchronize(st));
        double dbeta = 0;
        for (double v : db) dbeta += v;
        if (W0 > 0) launch_adj_beta(c, X, AL, dbeta / W0, lam);
    }
    if (grad_p && np > 0) {
        std::vector<double> h(3 * size_t(np));
        G3D_CUDA(cudaMemcpyAsync(h.data(), lam + 3 * size_t(np), 3 * size_t(np) * 8, cudaMemcpyDeviceToHost, st));
        G3D_CUDA(cudaStreamSynchronize(st));
        for (long i = 0; i < np; ++i)
            for (int q = 0; q < 3; ++q) grad_p[3 * i + q] = h[size_t(q) * np + i];
    }
    if (plasma && !stored) {                          // the run as the forward left it, at level K
        restore(K);
        launch_d2f(c, c.Fd.p, c.F.p, long(Fn));
    }
    G3D_CUDA(cudaStreamSynchronize(st));
    if (eh & 1) throw Error(G3D_ERR_STATE, "the adjoint march: a particle in the handed-over state");
    if (eh & 2) throw Error(G3D_ERR_CAPACITY, "the adjoint march: more than 64 push sub-steps in one s-step");
}

}  // namespace g3d

// ================================================================ extern "C"
using g3d::Ctx;
using g3d::Error;

namespace {
template <class Fn>
int guarded(g3d_ctx* ctx, Fn&& fn) {
    try {
        // every call works on the device the context was created on, whatever device the calling thread has current
        if (ctx) G3D_CUDA(cudaSetDevice(ctx->c.device));
        fn();
        if (ctx) ctx->c.err.clear();
        return G3D_OK;
    } catch (const Error& e) {
        (ctx ? ctx->c.err : g3d::g_create_err) = e.what();
        return e.code;
    } catch (const std::exception& e) {
        (ctx ? ctx->c.err : g3d::g_create_err) = e.what();
        return G3D_ERR_ARG;
    }
}
}  // namespace

extern "C" {

const char* g3d_version(void) { return "libg3d 0.2 (sm_100a; FP64 and mixed forms; Fourier and free-hand y; adjoint)"; }

int g3d_create(const g3d_grid* grid, const g3d_params* params, g3d_ctx** out) {
    if (!grid || !params || !out) { g3d::g_create_err = "null argument"; return G3D_ERR_ARG; }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        g3d::g_create_err = "no CUDA device visible";
        return G3D_ERR_NODEV;
    }
    g3d_ctx* ctx = new g3d_ctx();
    try {
        G3D_CUDA(cudaGetDevice(&ctx->c.device));
        G3D_CUDA(cudaStreamCreateWithFlags(&ctx->c.stream, cudaStreamNonBlocking));
        g3d::setup(ctx->c, *grid, *params);
    } catch (const Error& e) {
        g3d::g_create_err = e.what();
        g3d_destroy(ctx);
        return e.code;
    } catch (const std::exception& e) {
        g3d::g_create_err = e.what();
        g3d_destroy(ctx);
        return G3D_ERR_ARG;
    }
    *out = ctx;
    return G3D_OK;
}

void g3d_destroy(g3d_ctx* ctx) {
    if (!ctx) return;
    Ctx& c = ctx->c;
    cudaSetDevice(c.device);
    c.ckjob.reset();                 // an asynchronous checkpoint in flight ends first (its error is dropped)
    if (c.stream) cudaStreamSynchronize(c.stream);
    for (auto& pe : c.pending) { cudaEventDestroy(pe.e0); cudaEventDestroy(pe.e1); }
    for (auto e : c.event_pool) cudaEventDestroy(e);
    cudaStream_t s = c.stream;
    delete ctx;                      // DevBuf destructors free the device memory
    if (s) cudaStreamDestroy(s);
}

const char* g3d_last_error(const g3d_ctx* ctx) { return ctx ? ctx->c.err.c_str() : g3d::g_create_err.c_str(); }

int g3d_set_particles(g3d_ctx* ctx, const g3d_particle* parts, int64_t n) {
    return guarded(ctx, [&] {
        if (n < 0 || (n > 0 && !parts)) throw Error(G3D_ERR_ARG, "bad particle array");
        g3d::set_particles(ctx->c, parts, long(n));
    });
}
int g3d_get_particles(g3d_ctx* ctx, g3d_particle* out, int64_t capacity, int64_t* n) {
    return guarded(ctx, [&] {
        if (n) *n = ctx->c.np;
        if (capacity < ctx->c.np) throw Error(G3D_ERR_CAPACITY, "output capacity below the particle count");
        g3d::get_particles_into(ctx->c, out);
    });
}
int g3d_load_bunches(g3d_ctx* ctx, const g3d_bunch* b, int32_t count) {
    return guarded(ctx, [&] {
        if (count < 0 || (count > 0 && !b)) throw Error(G3D_ERR_ARG, "bad bunch list");
        Ctx& c = ctx->c;
        const g3d_grid G{c.nx, c.ny, c.N, c.yf ? 1 : 0, c.nx * c.dx, c.ny * c.dy, c.zeta.data(),
                         c.yf ? nullptr : c.ynode_h.data()};
        g3d::load_bunches(c, G, b, count);
    });
}
int g3d_sample_bunches(const g3d_grid* grid, const g3d_params* params, const g3d_bunch* b, int32_t count,
                       g3d_particle* out, int64_t capacity, int64_t* n, int64_t* lost, double* X0, double* Y0) {
    try {
        if (!grid || !params || !n || count < 0 || (count > 0 && !b) || grid->nzeta < 4 || !grid->zeta)
            throw Error(G3D_ERR_ARG, "bad arguments");
        std::vector<g3d_particle> v;
        long ls = 0;
        double x0 = 0, y0 = 0;
        g3d::sample_bunches(*grid, *params, b, count, v, ls, x0, y0);
        *n = int64_t(v.size());
        if (lost) *lost = ls;
        if (X0) *X0 = x0;
        if (Y0) *Y0 = y0;
        if (int64_t(v.size()) > capacity) throw Error(G3D_ERR_CAPACITY, "output capacity below the particle count");
        if (!v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(g3d_particle));
        return G3D_OK;
    } catch (const Error& e) {
        g3d::g_create_err = e.what();
        return e.code;
    }
}
int g3d_init(g3d_ctx* ctx) { return guarded(ctx, [&] { g3d::init_fields(ctx->c); g3d::check_kernel_errors(ctx->c); }); }
int g3d_step(g3d_ctx* ctx) { return guarded(ctx, [&] { g3d::step(ctx->c, true); ctx->c.prof_collect(); }); }
int g3d_step_async(g3d_ctx* ctx) { return guarded(ctx, [&] { g3d::step(ctx->c, false); }); }
int g3d_solve_fields(g3d_ctx* ctx, double D) {
    return guarded(ctx, [&] { g3d::solve_fields(ctx->c, D); g3d::check_kernel_errors(ctx->c); });
}
int g3d_currents(g3d_ctx* ctx) { return guarded(ctx, [&] { g3d::currents(ctx->c); G3D_CUDA(cudaStreamSynchronize(ctx->c.stream)); }); }
int g3d_march(g3d_ctx* ctx, double D) {
    return guarded(ctx, [&] { g3d::materialize_jk(ctx->c); g3d::march(ctx->c, D); G3D_CUDA(cudaStreamSynchronize(ctx->c.stream)); });
}
int g3d_sponge_and_real_fields(g3d_ctx* ctx) {
    return guarded(ctx, [&] { g3d::sponge_and_real_fields(ctx->c); g3d::check_kernel_errors(ctx->c); });
}
int g3d_push(g3d_ctx* ctx, double s0, double s1) {
    return guarded(ctx, [&] { g3d::launch_push(ctx->c, s0, s1); G3D_CUDA(cudaStreamSynchronize(ctx->c.stream)); });
}
int g3d_comoving_field(g3d_ctx* ctx) {
    return guarded(ctx, [&] { g3d::comoving_field(ctx->c); G3D_CUDA(cudaStreamSynchronize(ctx->c.stream)); });
}
int g3d_set_precision(g3d_ctx* ctx, int32_t mode) {
    return guarded(ctx, [&] {
        if (ctx->c.sharded() && mode != G3D_PREC_FP64) throw Error(G3D_ERR_STATE, "a sharded run is FP64");
        g3d::set_precision(ctx->c, mode);
    });
}
int g3d_beam_beta_sums_static(g3d_ctx* ctx, double out[2]) {
    return guarded(ctx, [&] {
        if (!out) throw Error(G3D_ERR_ARG, "null output");
        g3d::launch_beta_sums_static(ctx->c, out);
    });
}
int g3d_relax_start_field(g3d_ctx* ctx) {
    return guarded(ctx, [&] {
        g3d::materialize_jk(ctx->c);
        g3d::relax_start_field(ctx->c);
        G3D_CUDA(cudaStreamSynchronize(ctx->c.stream));
    });
}
int g3d_shift_window(g3d_ctx* ctx, int32_t nxs, int32_t nys) { return guarded(ctx, [&] { g3d::shift_window(ctx->c, nxs, nys); }); }
int g3d_set_plasma(g3d_ctx* ctx, const g3d_plasma* plasma, const g3d_ion* ions, int32_t nions) {
    return guarded(ctx, [&] {
        if (!plasma || nions < 0 || (nions > 0 && !ions)) throw Error(G3D_ERR_ARG, "bad plasma arguments");
        if (ctx->c.world > 1) throw Error(G3D_ERR_STATE, "a sharded run has no plasma");
        g3d::set_plasma(ctx->c, *plasma, ions, nions);
    });
}
int g3d_add_grid_laser(g3d_ctx* ctx, const g3d_grid_laser* laser) {
    return guarded(ctx, [&] {
        if (!laser || !(laser->waist > 0) || !(laser->tau > 0)) throw Error(G3D_ERR_ARG, "grid laser: waist and tau must be positive");
        ctx->c.glasers.push_back(*laser);
    });
}
int g3d_set_external(g3d_ctx* ctx, const g3d_undulator* u, int32_t nu, const g3d_magnet* m, int32_t nm, const double* kt,
                     int32_t nkt) {
    return guarded(ctx, [&] {
        if (nu < 0 || nm < 0 || nkt < 0 || (nu && !u) || (nm && !m) || (nkt && !kt))
            throw Error(G3D_ERR_ARG, "g3d_set_external: bad element arrays");
        for (int k = 0; k < nu; ++k) {
            const g3d_undulator& U = u[k];
            if (!(U.ku > 0) || !(U.z1 > U.z0) || U.ramp < 0 || (U.nk > 0 && (U.nk < 2 || U.koff < 0 || U.koff + U.nk > nkt || !(U.dzk > 0))))
                throw Error(G3D_ERR_ARG, "g3d_set_external: undulator " + std::to_string(k) + " (period, extent, ramp or taper table)");
        }
        for (int k = 0; k < nm; ++k)
            if (m[k].kind < 0 || m[k].kind > 2 || !(m[k].z1 > m[k].z0) || m[k].ramp < 0 || !(m[k].dsmax > 0))
                throw Error(G3D_ERR_ARG, "g3d_set_external: magnet " + std::to_string(k) + " (kind, extent, ramp or dsmax)");
        Ctx& c = ctx->c;
        c.und.upload(std::vector<g3d_undulator>(u, u + nu), c.stream);
        c.mag.upload(std::vector<g3d_magnet>(m, m + nm), c.stream);
        c.ktab.upload(std::vector<double>(kt, kt + nkt), c.stream);
        G3D_CUDA(cudaStreamSynchronize(c.stream));
        c.ext = g3d::ExtDev{nu, nm, c.und.p, c.mag.p, c.ktab.p};
    });
}
int g3d_set_ranks(g3d_ctx* ctx, int32_t rank, int32_t world, g3d_comm_fn comm, void* user) {
    return guarded(ctx, [&] { g3d::set_ranks(ctx->c, rank, world, comm, user); });
}
int g3d_shard_layout(int32_t nzeta, int64_t nkh, int32_t rank, int32_t world, int64_t out[4]) {
    return guarded(nullptr, [&] {
        if (!out || rank < 0 || rank >= world) throw Error(G3D_ERR_ARG, "g3d_shard_layout: bad arguments");
        const g3d::ShardLayout L(nzeta, long(nkh), world);
        out[0] = L.a[size_t(rank)]; out[1] = L.a[size_t(rank)] + L.ns[size_t(rank)];
        out[2] = L.m0[size_t(rank)]; out[3] = L.m0[size_t(rank)] + L.mq[size_t(rank)];
    });
}
int g3d_shard_transpose_plan(int32_t nzeta, int64_t nkh, int32_t rank, int32_t world, const int32_t* kinds, int32_t narrays,
                             int32_t to_pencil, int64_t elem_bytes, g3d_block* pack, int32_t pack_cap, int32_t* npack,
                             g3d_block* unpack, int32_t unpack_cap, int32_t* nunpack, int64_t* send_bytes,
                             int64_t* recv_bytes) {
    return guarded(nullptr, [&] {
        if (!npack || !nunpack || !send_bytes || !recv_bytes || rank < 0 || rank >= world)
            throw Error(G3D_ERR_ARG, "g3d_shard_transpose_plan: bad arguments");
        const g3d::ShardLayout L(nzeta, long(nkh), world);
        g3d::ShardPlan pl;
        g3d::shard_plan(L, rank, kinds, narrays, to_pencil != 0, long(elem_bytes), pl);
        *npack = int32_t(pl.pack.size()); *nunpack = int32_t(pl.unpack.size());
        std::copy(pl.send_bytes.begin(), pl.send_bytes.end(), send_bytes);
        std::copy(pl.recv_bytes.begin(), pl.recv_bytes.end(), recv_bytes);
        if (int64_t(pl.pack.size()) > pack_cap || int64_t(pl.unpack.size()) > unpack_cap || (!pack && !pl.pack.empty()) ||
            (!unpack && !pl.unpack.empty()))
            throw Error(G3D_ERR_CAPACITY, "g3d_shard_transpose_plan: more blocks than the capacity");
        std::copy(pl.pack.begin(), pl.pack.end(), pack);
        std::copy(pl.unpack.begin(), pl.unpack.end(), unpack);
    });
}
int g3d_set_chicanes(g3d_ctx* ctx, const g3d_chicane* ch, int32_t n) {
    return guarded(ctx, [&] {
        if (n < 0 || (n && !ch)) throw Error(G3D_ERR_ARG, "g3d_set_chicanes: bad chicane array");
        if (n && ctx->c.sharded()) throw Error(G3D_ERR_STATE, "g3d_set_chicanes: a sharded run has no chicanes");
        for (int k = 0; k < n; ++k)
            if (!(ch[k].gamma_ref > 1)) throw Error(G3D_ERR_ARG, "g3d_set_chicanes: the reference gamma must be > 1");
        ctx->c.chicanes.assign(ch, ch + n);
    });
}
int g3d_march_plasma(g3d_ctx* ctx, double s0, double s1) {
    return guarded(ctx, [&] {
        if (!ctx->c.pl) throw Error(G3D_ERR_STATE, "no plasma set (g3d_set_plasma)");
        g3d::materialize_jk(ctx->c);
        g3d::march_plasma(ctx->c, s0, s1);
        G3D_CUDA(cudaStreamSynchronize(ctx->c.stream));
    });
}
int g3d_get_streaming(g3d_ctx* ctx, g3d_particle* out, int64_t capacity, int64_t* n) {
    return guarded(ctx, [&] {
        if (!ctx->c.pl) { if (n) *n = 0; return; }
        const std::vector<g3d_particle> v = g3d::get_streaming(ctx->c);
        if (n) *n = int64_t(v.size());
        if (int64_t(v.size()) > capacity) throw Error(G3D_ERR_CAPACITY, "output capacity below the streaming particle count");
        if (!v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(g3d_particle));
    });
}

int g3d_diagnostics(g3d_ctx* ctx, double out[19]) {
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        double S[19] = {0};
        g3d::launch_diag(c, S);
        S[15] = c.P.self_fields ? g3d::launch_field_energy(c) : 0;
        S[16] = double(c.lost_total);
        if (c.sharded()) {                               // the particles lost on every rank
            g3d::DevBuf<double> lost;
            lost.alloc(1, c.stream);
            G3D_CUDA(cudaMemcpyAsync(lost.p, &S[16], sizeof(double), cudaMemcpyHostToDevice, c.stream));
            c.all_sum(lost.p, 1, G3D_SUM_F64);
            G3D_CUDA(cudaMemcpyAsync(&S[16], lost.p, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
            G3D_CUDA(cudaStreamSynchronize(c.stream));
        }
        c.field_energy = S[15];
        // stop condition of the analytic laser (sim_output.cpp:30-31)
        const double w = S[0] > 0 ? S[0] : 1;
        if (c.laser.on && c.P.stop_fwhm > 0 && c.laser.tau > 0 && (S[13] / w - c.laser.eta_c) / c.laser.tau > c.P.stop_fwhm)
            c.stop_ = true;
        std::memcpy(out, S, sizeof S);
    });
}
int g3d_beam_moments(g3d_ctx* ctx, int32_t capacity, double* s1, double* s2, int32_t* ngroups) {
    return guarded(ctx, [&] {
        const int G = g3d::beam_groups(ctx->c);
        if (ngroups) *ngroups = G;
        if (!s1 || !s2) throw Error(G3D_ERR_ARG, "g3d_beam_moments: null output");
        if (capacity < G) throw Error(G3D_ERR_CAPACITY, "g3d_beam_moments: capacity below the " + std::to_string(G) + " beam species");
        g3d::launch_beam_moments(ctx->c, s1, s2);
    });
}
int g3d_field_energy(g3d_ctx* ctx, double* out) {
    return guarded(ctx, [&] { *out = ctx->c.P.self_fields ? g3d::launch_field_energy(ctx->c) : 0; });
}
int g3d_get_status(const g3d_ctx* ctx, g3d_status* o) {
    if (!ctx || !o) return G3D_ERR_ARG;
    const Ctx& c = ctx->c;
    o->s = c.s; o->X0 = c.X0; o->Y0 = c.Y0; o->beta_b = c.beta_b; o->gm2_b = c.gm2_b; o->field_energy = c.field_energy;
    o->istep = c.istep; o->np = c.np; o->lost = c.lost_total; o->stop = g3d::finished(c) ? 1 : 0;
    return G3D_OK;
}

int g3d_array_info(const g3d_ctx* ctx, int32_t which, size_t* count, size_t* eb) {
    return guarded(const_cast<g3d_ctx*>(ctx), [&] {
        Ctx& c = const_cast<g3d_ctx*>(ctx)->c;
        const g3d::ArrayRef a = g3d::array_ref(c, which);
        *count = g3d::ref_count(c, a); *eb = a.eb;
    });
}
int g3d_get_array(g3d_ctx* ctx, int32_t which, void* host, size_t count) {
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        const size_t n = g3d::ref_count(c, g3d::array_ref(c, which));
        if (count != n) throw Error(G3D_ERR_ARG, "count differs from the array size " + std::to_string(n));
        g3d::get_array(c, which, host);
    });
}
int g3d_set_array(g3d_ctx* ctx, int32_t which, const void* host, size_t count) {
    return guarded(ctx, [&] {
        Ctx& c = ctx->c;
        if (which == G3D_A_JKX || which == G3D_A_JKY || which == G3D_A_J0X || which == G3D_A_J0Y) g3d::materialize_jk(c);
        const size_t n = g3d::ref_count(c, g3d::array_ref(c, which));
        if (count != n) throw Error(G3D_ERR_ARG, "count differs from the array size " + std::to_string(n));
        g3d::set_array(c, which, host);
    });
}
void* g3d_device_ptr(g3d_ctx* ctx, int32_t which) {
    void* p = nullptr;
    guarded(ctx, [&] { p = g3d::array_ref(ctx->c, which).p; });
    return p;
}

int g3d_write_checkpoint_async(g3d_ctx* ctx, const char* path) {
    return guarded(ctx, [&] {
        if (!path) throw Error(G3D_ERR_ARG, "g3d_write_checkpoint_async: no path");
        if (ctx->c.world > 1) throw Error(G3D_ERR_STATE, "checkpoints of a sharded run are not built");
        g3d::write_checkpoint_async(ctx->c, path);
    });
}
int g3d_checkpoint_wait(g3d_ctx* ctx) { return guarded(ctx, [&] { g3d::checkpoint_wait(ctx->c); }); }
int g3d_write_checkpoint(g3d_ctx* ctx, const char* path) {
    return guarded(ctx, [&] {
        if (ctx->c.world > 1) throw Error(G3D_ERR_STATE, "checkpoints of a sharded run are not written");
        g3d::write_checkpoint(ctx->c, path);
    });
}
int g3d_read_checkpoint(g3d_ctx* ctx, const char* path) {
    return guarded(ctx, [&] {
        if (ctx->c.world > 1) throw Error(G3D_ERR_STATE, "checkpoints of a sharded run are not read");
        g3d::read_checkpoint(ctx->c, path);
    });
}

void* g3d_stream(g3d_ctx* ctx) { return ctx ? static_cast<void*>(ctx->c.stream) : nullptr; }
int g3d_synchronize(g3d_ctx* ctx) {
    return guarded(ctx, [&] { g3d::check_kernel_errors(ctx->c); ctx->c.prof_collect(); });
}
int g3d_profile_enable(g3d_ctx* ctx, int32_t on) {
    return guarded(ctx, [&] {
        ctx->c.prof_collect();
        ctx->c.profiling = on != 0;
        ctx->c.prof.clear();
    });
}
int32_t g3d_profile_count(const g3d_ctx* ctx) { return ctx ? int32_t(ctx->c.prof.size()) : 0; }
int g3d_profile_get(g3d_ctx* ctx, int32_t k, const char** name, int64_t* launches, double* total_ms) {
    return guarded(ctx, [&] {
        ctx->c.prof_collect();
        if (k < 0 || size_t(k) >= ctx->c.prof.size()) throw Error(G3D_ERR_ARG, "profile index out of range");
        const g3d::ProfEntry& e = ctx->c.prof[size_t(k)];
        *name = e.name.c_str(); *launches = e.launches; *total_ms = e.ms;
    });
}
int64_t g3d_launch_count(const g3d_ctx* ctx) { return ctx ? ctx->c.launches : 0; }

int g3d_set_laser_modes(g3d_ctx* ctx, const double* coef) { return guarded(ctx, [&] { g3d::set_laser_modes(ctx->c, coef); }); }
int g3d_set_exact_fields(g3d_ctx* ctx, int32_t on) {
    return guarded(ctx, [&] {
        if (on && ctx->c.sharded()) throw Error(G3D_ERR_STATE, "g3d_set_exact_fields: not in a sharded run");
        g3d::set_exact_fields(ctx->c, on != 0);
    });
}
int g3d_set_adjoint_momenta(g3d_ctx* ctx, int32_t mode) { return guarded(ctx, [&] { g3d::set_adjoint_momenta(ctx->c, mode); }); }
int g3d_adjoint(g3d_ctx* ctx, int32_t nsteps, double* objective, double* grad_modes, double* grad_p) {
    return guarded(ctx, [&] {
        if (!objective) throw Error(G3D_ERR_ARG, "g3d_adjoint: objective is required");
        g3d::adjoint(ctx->c, nsteps, objective, grad_modes, grad_p);
        ctx->c.prof_collect();
    });
}

}  // extern "C"
