// Host context of libg3d and the plain structs its kernels take by value.
#pragma once
#include <array>
#include <deque>
#include <memory>
#include <string>
#include <vector>
#include "g3d.h"
#include "g3d_common.cuh"
#include "k_tma.cuh"

namespace g3d {

// ---------------------------------------------------------------- device structs (kernel arguments)
// Grid, k-tables, zeta weights and FFT twiddles. Tables follow the reference's set-up
// (Simulation::Simulation, setup_y_fourier, setup_zeta: src/sim_setup.cpp:17-35, 63-82, 148-164).
struct Geo {
    int nx, ny, nk, N, a, b, ns, nh;     // nh = ns + 3 planes of the raw deposit
    int H;                               // nx/2 + 1 columns of a half spectrum (k_x = 0 .. nx/2)
    long nkh;                            // ny * H modes of a half-spectrum plane
    long m0;                             // the first mode of the planes (a mode pencil of a sharded run; else 0)
    int yf, zeta_uniform;
    double dx, dy, Lx, Ly;
    const double *kxd, *kxs, *filt, *maskx;
    const double *kyd, *kys, *filty, *masky_n, *masky_h, *iD, *iA;
    const double *zs, *hcg, *wlo, *whi, *wsl;
    // free-hand y (yf == 0): node positions (ny + 1), LU factors of k_x^2 - Lap_y on the nodes per (j, k_x)
    // ([j][k_x], k_x <= nx/2), eigenvectors of -Lap_y (forward [s][j], back [j][s]) and eigenvalues [s]
    const double *yn, *pcp, *pid, *evf, *evb, *evl;
    AxisDev zax, yax;
    const cpx *twx, *twy;               // exp(-2 pi i s / nx), exp(-2 pi i s / ny)
};

// Particles as structure of arrays (the reference keeps an array of 104-byte records).
struct PartsDev {
    double *x, *y, *zeta, *px, *py, *pz, *w, *rem, *z, *q, *qm;
    int32_t *alive, *sp;
    uint64_t* id;
};

// Analytic plane wave A = a0 g(eta) cos(kL (eta - eta_c) + cep) (reference struct Laser,
// src/sim.hpp:191-210), with the Gaussian envelope of the reference and a flat-top envelope with
// sin^2 ramps added here.
struct LaserDev {
    int on, pol, env;
    double a0, kL, tau, cep, eta_c, kx, kz, flat, ramp;
    G3D_HD double eta(double x, double z, double t) const { return t - kx * x - kz * z; }
    // envelope g and dg/dxi at xi = eta - eta_c; false outside the pulse
    G3D_HD bool envelope(double xi, double& g, double& gp) const {
        if (env == G3D_ENV_GAUSSIAN) {
            if (fabs(xi) > 5 * tau) return false;
            g = exp(-1.3862943611198906 * xi * xi / (tau * tau));       // 2 ln 2
            gp = -2.7725887222397811 * xi / (tau * tau) * g;             // 4 ln 2
            return true;
        }
        const double ax = fabs(xi), hf = 0.5 * flat;
        if (ax <= hf) { g = 1; gp = 0; return true; }
        if (ax >= hf + ramp) return false;
        const double u = (hf + ramp - ax) / ramp;                       // 1 at the plateau edge, 0 outside
        const double sn = sin(1.5707963267948966 * u), cs = cos(1.5707963267948966 * u);
        g = sn * sn;
        gp = (xi > 0 ? -1.0 : 1.0) * (3.1415926535897932 / ramp) * sn * cs;
        return true;
    }
    G3D_HD void field(double x, double z, double t, double E[3], double B[3]) const {
        E[0] = E[1] = E[2] = B[0] = B[1] = B[2] = 0;
        if (!on) return;
        const double xi = eta(x, z, t) - eta_c;
        double g, gp;
        if (!envelope(xi, g, gp)) return;
        const double ph = kL * xi + cep, c = cos(ph), s = sin(ph);
        const double d1 = a0 * (gp * c - kL * g * s), d2 = a0 * (gp * s + kL * g * c);
        if (pol == 0) { E[1] = -d1; }
        else if (pol == 1) { E[0] = -d1 * kz; E[2] = d1 * kx; }
        else { E[0] = -d1 * kz; E[2] = d1 * kx; E[1] = -d2; }
        B[0] = -kz * E[1]; B[1] = kz * E[0] - kx * E[2]; B[2] = kx * E[1];
    }
};

// External magnetic elements on the device (k_external.cuh): the undulators and magnets of g3d_set_external and
// the taper table of the undulators.
struct ExtDev {
    int nu, nm;
    const g3d_undulator* u;
    const g3d_magnet* m;
    const double* kt;
    G3D_HD bool any() const { return nu > 0 || nm > 0; }
};

// ---------------------------------------------------------------- device buffers
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void alloc(size_t count, cudaStream_t s) {
        release();
        n = count;
        if (n) {
            G3D_CUDA(cudaMalloc(&p, n * sizeof(T)));
            G3D_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
        }
    }
    void release() { if (p) cudaFree(p); p = nullptr; n = 0; }
    void zero(cudaStream_t s) { if (n) G3D_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s)); }
    void upload(const std::vector<T>& v, cudaStream_t s) {
        if (v.size() != n) alloc(v.size(), s);
        if (n) G3D_CUDA(cudaMemcpyAsync(p, v.data(), n * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    size_t bytes() const { return n * sizeof(T); }
};

// ---------------------------------------------------------------- profiling
struct ProfEntry { std::string name; long launches = 0; double ms = 0; };
struct PendingEvent { int entry; cudaEvent_t e0, e1; };

struct PlasmaState;               // g3d_plasma.hpp
// The slabs of a sharded run's ranks as one GPU sees them (g3d_shard.cu, the peer march of k_march.cu): each rank's
// first slice, slice count and its 11 slab arrays (R_x, R_y, E_z, B_z, L_x, L_y, j0x, j0y, jkx, jky, jkz) mapped here
constexpr int SHARD_PEER_MAX = 8;
struct SlabPeers {
    int P = 0;
    int a[SHARD_PEER_MAX] = {}, ns[SHARD_PEER_MAX] = {};
    long nkh = 0;
    void* arr[SHARD_PEER_MAX][11] = {};
};
// Tensor maps of a TMA column kernel over a set of buffers (k_tma.cuh), rebuilt when the buffers move
struct TmaCache {
    bool valid = false;
    const void* base[6] = {};
    long rows = 0;
    TileMaps maps{};
    // the maps of n arrays [rows][H] for 8-column tiles of ny rows; false where the TMA path does not apply
    bool get(const cpx* const* p, int n, long H, long rows_, int ny) {
        bool same = valid && rows == rows_;
        for (int k = 0; k < n && same; ++k) same = base[k] == p[k];
        if (same) return true;
        valid = false;
        if (ny > 256 || n > 6) return false;
        for (int k = 0; k < n; ++k) {
            if (!tma_map_columns(&maps.m[k], p[k], H, rows_, ny)) return false;
            base[k] = p[k];
        }
        rows = rows_;
        valid = true;
        return true;
    }
};
struct Shard;                     // g3d_shard.cu

// Buffers of the mixed FP32/FP64 form (k_mixed.cu): complex64 half spectra of E_z, B_z, L and the currents, FP32
// raw currents; R_x, R_y stay in Ctx::Rx, Ry (complex128), F is float in both forms.
struct MixedBufs {
    DevBuf<cpxf> Ez, Bz, Lx, Ly;                 // ns planes
    DevBuf<cpxf> j0x, j0y, jkx, jky, jkz;        // ns+1 half-cell planes
    DevBuf<cpxf> W[6];                           // transform scratch, ns+1 planes each
    DevBuf<float> jw;                            // 3 x (ns+3) real planes
    DevBuf<cpxf> twx, twy;                       // FP32 twiddles
};

// ---------------------------------------------------------------- the context
struct Ctx {
    // grid (single rank: a = 0, b = ns = N)
    int nx = 0, ny = 0, N = 0, a = 0, b = 0, ns = 0, nk = 0;
    int H = 0;                                   // nx/2 + 1: spectra are kept for k_x = 0 .. nx/2
    long nkh = 0;                                // ny * H
    double dx = 0, dy = 0;
    bool yf = true;
    g3d_params P{};
    std::vector<double> zeta;
    std::vector<double> hcg_h, wlo_h, whi_h, wsl_h, kxd_h, kyd_h;
    // tables
    DevBuf<double> kxd, kxs, filt, maskx, kyd, kys, filty, masky_n, masky_h, iD, iA;
    DevBuf<double> zs, hcg, wlo, whi, wsl;
    DevBuf<int> zbins, ybins;                    // bin tables of the graded zeta axis and the free-hand y axis
    DevBuf<cpx> twx, twy;
    DevBuf<double> yn, pcp, pid, evf, evb, evl;  // free-hand y tables (empty for Fourier y)
    std::vector<double> ynode_h;
    DevBuf<cpx> fhs;                             // free-hand march scratch: 5 lines of ny x H complex
    DevBuf<double> fhcp;                         // and the Thomas coefficients, ny x H
    // field state: the reference's arrays (src/sim.hpp:265-276); spectra as half spectra [plane][j][k_x <= nx/2]
    DevBuf<cpx> Rx, Ry, Ez, Bz, Lx, Ly;          // ns planes
    DevBuf<cpx> j0x, j0y, jkx, jky, jkz;         // ns+1 half-cell planes
    DevBuf<cpx> jzg;                             // 2 ghost planes of filtered j_z (zero on one rank)
    DevBuf<double> jw;                           // 3 x (ns+3) real planes
    bool jw_fixed = false;                       // jw holds the fixed-point deposit's integers (Fourier y, FP64)
    DevBuf<double> depfix;                       // the fixed-point deposit's bound partials and scale (k_currents.cu)
    double ia_max = 0;                           // the largest dual-cell factor 1/A_j, 1/Delta_j of the y grid
    DevBuf<float> F;                             // 6 x (ns+2) real planes
    DevBuf<double> Fd;                           // exact fields: F kept in FP64 too, gathered by the beam push
                                                 // (the differentiable forward of the gradient check), or empty
    DevBuf<cpx> lmode;                           // laser mode coefficients per stored mode (ny x H), or empty
    DevBuf<cpx> lspx, lspy;                      // the grid-laser spectra added at init before the coefficients
    DevBuf<unsigned char> adjws;                 // workspace of the adjoint march, kept between calls
    DevBuf<unsigned char> adjrec;                // the adjoint's record of one plasma march, kept between calls
    bool adj_after_start = false;                // dJ/dp with the start field held (G3D_ADJ_AFTER_START)
    // where the next real fields go instead of F / Fd (taken once by sponge_and_real_fields): the adjoint's forward
    // writes each level's fields straight into its checkpoint
    double* fd_next = nullptr;
    float* f_next = nullptr;
    DevBuf<cpx> W[6];                            // half-spectrum scratch, ns+1 planes each
    DevBuf<double> rscratch;                     // real scratch (Thomas coefficients), ns half planes
    // TMA tile loads of the whole-window column transforms (k_tma.cuh): on unless G3D_NO_TMA is set; the error word
    // of their bounded waits (bit 1: a tile never landed)
    bool use_tma = true;
    TmaCache tma_rf, tma_cur, tma_spi, tma_spf;
    DevBuf<int> kerr;
    long tma_polls = 1L << 24;
    unsigned tma_extra = 0;
    TmaWait tma_wait() { return TmaWait{kerr.p, tma_polls, tma_extra}; }
    bool jk_is_j0 = false;                       // after solve_fields jk == j0: the j0/jk buffers were swapped
    bool mixed = false;                          // G3D_PREC_MIXED: the spectra above except Rx, Ry are not allocated
    bool f32s = false;                           // G3D_PREC_MIXED: FP32 gathers and deposit of the streaming plasma
                                                 // (free-hand y: the mixed form is this alone, the spectra stay FP64)
    MixedBufs mx;
    bool fields_ready = false;                   // init has run (the precision is fixed from then on)
    // particles
    DevBuf<double> pbuf_d;                       // 11 double columns
    DevBuf<int32_t> pbuf_i;                      // 2 int columns
    DevBuf<uint64_t> pbuf_u;                     // ids
    DevBuf<g3d_particle> pstage;                 // device staging of the 104-byte records
    PartsDev parts{};
    long np = 0, pcap = 0;
    int nbunch = 1;                              // bunch blocks of the last g3d_load_bunches (sp = 0, -1, ...)
    DevBuf<int32_t> perm;                        // particles in cell order (k_sort.cu); storage order unchanged
    DevBuf<uint32_t> sort_keys;                  // sort buffers, sized for the particle capacity
    DevBuf<int32_t> sort_idx;
    DevBuf<unsigned char> sort_tmp;
    int steps_since_sort = 0;
    DevBuf<int32_t> jflag, joff;                 // the join of trapped particles: live flags of the list, their sums
    DevBuf<unsigned char> jtmp;
    // reductions
    DevBuf<double> red;                          // per-block partial sums
    DevBuf<double> momw;                         // the beam moments' partial sums, totals and means
    std::vector<double> red_h;
    // scalars (reference members)
    double s = 0, X0 = 0, Y0 = 0, beta_b = 1, gm2_b = 0, field_energy = 0, hmin = 1e300;
    long istep = 0, lost_total = 0;
    bool stop_ = false, starting_ = false, comoving_c_ = false;
    LaserDev laser{};
    AxisDev zax{}, yax{};
    std::deque<std::array<double, 3>> cent_;     // centroid sums awaiting their step (window lag)
    // device, stream, launches, profiling
    int device = 0;                              // the CUDA device current at g3d_create; every call runs on it
    std::shared_ptr<void> ckjob;                 // the asynchronous checkpoint in flight (g3d_host.cu), or none
    DevBuf<unsigned char> ckpt_snap;             // its device copy of the state, kept for the next one
    cudaStream_t stream = nullptr;
    long launches = 0;
    bool profiling = false;
    std::vector<ProfEntry> prof;
    std::vector<PendingEvent> pending;
    std::vector<cudaEvent_t> event_pool;
    std::string err;
    // streaming plasma (null without plasma) and the grid lasers of the start field
    std::unique_ptr<PlasmaState> pl;
    std::vector<g3d_grid_laser> glasers;
    // external magnetic elements (g3d_set_external)
    DevBuf<g3d_undulator> und;
    DevBuf<g3d_magnet> mag;
    DevBuf<double> ktab;
    ExtDev ext{0, 0, nullptr, nullptr, nullptr};
    std::vector<g3d_chicane> chicanes;           // thin chicanes (g3d_set_chicanes)
    // a sharded run (g3d_set_ranks, g3d_shard.cu): this rank's slab and mode pencil, the caller's collectives
    int rank = 0, world = 1;
    g3d_comm_fn comm_fn = nullptr;
    void* comm_user = nullptr;
    std::unique_ptr<Shard> sh;
    bool sharded() const { return world > 1; }
    // sums `count` values at the device pointer `data` across the ranks (nothing on one rank)
    void all_sum(void* data, long count, int kind);
    // the all-to-all of device buffers with host byte counts per rank
    void all_to_all(const void* send, const int64_t* send_bytes, void* recv, const int64_t* recv_bytes);

    Ctx();
    ~Ctx();
    Geo geo() const;
    // kernel launch bookkeeping: call before/after each launch
    int prof_begin(const char* name);
    void prof_end(int token);
    void prof_collect();
    void check_launch(const char* what);
};

// ---------------------------------------------------------------- launchers (k_*.cu)
void launch_deposit(Ctx& c);
const double* launch_deposit_scale(Ctx& c, double ia_max);   // fixed-point deposit: its scale, then the planes to doubles
void launch_deposit_finish(Ctx& c);
void launch_cur_fft(Ctx& c, bool keep0);
void launch_march(Ctx& c, double D);
// free-hand y (k_freehand.cu)
void launch_deposit_fh(Ctx& c);
void launch_cur_fft_fh(Ctx& c, bool keep0);
void launch_march_fh(Ctx& c, double D);
void launch_sponge_fh(Ctx& c);
void launch_real_fields_fh(Ctx& c);
void launch_comoving_fh(Ctx& c, double beta, double gm2);
void launch_march_slice_fh(Ctx& c, double D, int n);
// The midpoint fields that the rows kernel of one slice also writes, for the streaming gather of the next pass:
// 0.5 (F(l) + F(other)) per point, interleaved (FP32: 8 floats, FP64: 6 doubles); out null: none
struct FmidOut {
    void* out = nullptr;
    int other = 0, f32 = 0;
    int fh = 0;               // free-hand y (FP32): per point (E_x, E_z, B_y, 0) of the node row, (E_y, B_x, B_z, 0) of the half-node row
    // the adjoint's record of the slice's exact fields (the exact midpoint variant only): the device address of the
    // record's field array and the offset of this slice and pass in it (6 planes of nk)
    double* const* rec_f = nullptr;
    long rec_off = 0;
};
// the other slice's six values at point k (loaded by the rows kernel before it stores its own slice: the other
// slice is never this one, so the loads need not wait behind those stores)
__device__ __forceinline__ void fmid_load(const FmidOut& fm, const float* F, long fpl, long nk, long k, float o[6]) {
#pragma unroll
    for (int comp = 0; comp < 6; ++comp) o[comp] = F[comp * fpl + long(fm.other) * nk + k];
}
__device__ __forceinline__ void fmid_store(const FmidOut& fm, long k, const float v[6], const float oth[6]) {
    double m[6];
#pragma unroll
    for (int comp = 0; comp < 6; ++comp) m[comp] = 0.5 * (double(v[comp]) + double(oth[comp]));
    if (fm.fh) {
        float4* o = reinterpret_cast<float4*>(fm.out) + 2 * k;
        o[0] = make_float4(float(m[0]), float(m[2]), float(m[4]), 0.f);
        o[1] = make_float4(float(m[1]), float(m[3]), float(m[5]), 0.f);
    } else if (fm.f32) {
        float4* o = reinterpret_cast<float4*>(fm.out) + 2 * k;
        o[0] = make_float4(float(m[0]), float(m[1]), float(m[2]), float(m[3]));
        o[1] = make_float4(float(m[4]), float(m[5]), 0.f, 0.f);
    } else {
        double2* o = reinterpret_cast<double2*>(fm.out) + 3 * k;
        o[0] = make_double2(m[0], m[1]); o[1] = make_double2(m[2], m[3]); o[2] = make_double2(m[4], m[5]);
    }
}
void launch_real_fields_slice_fh(Ctx& c, int l, FmidOut fm = FmidOut());
void launch_ss_lines_fh(Ctx& c, const cpx* T3, cpx* out3, double a2);
void launch_sp_rows(Ctx& c);                // k_fields.cu
void launch_cur_rows_to_jk(Ctx& c);         // k_currents.cu
void launch_sponge(Ctx& c);
void launch_real_fields(Ctx& c);
void launch_comoving(Ctx& c, double beta, double gm2);
void launch_push(Ctx& c, double s0, double s1);
void launch_push_range(Ctx& c, double s0, double s1, long i0, long n);
void launch_march_pencil(Ctx& c, const Geo& g, cpx* const* p, double D);
void launch_march_peer(Ctx& c, const Geo& g, const SlabPeers& sp, double D);
void launch_comoving_pencil(Ctx& c, const Geo& g, const cpx* jz, double* cpb, cpx* dpb, cpx* const* out, double beta, double gm2);
void realloc_slab(Ctx& c);                        // the field buffers of the slab [a, b) (g3d_host.cu)
void reserve_particles(Ctx& c, long n);           // particle columns for n (contents not kept when they move)
// a sharded run (g3d_shard.cu)
void shard_raw_halo(Ctx& c);
void shard_jz_ghosts(Ctx& c);
void shard_field_ghosts(Ctx& c);
void shard_march(Ctx& c, double D);
void shard_comoving(Ctx& c, double beta, double gm2);
void shard_exchange_particles(Ctx& c, double s1);
bool shard_owns(const Ctx& c, double zeta);
void launch_zero_c(Ctx& c, cpx* p, size_t n);
void launch_axpy_c(Ctx& c, cpx* y, const cpx* x, double a, size_t n);   // y = y + a x
void launch_copy_c(Ctx& c, cpx* y, const cpx* x, size_t n);
void launch_beta_sums(Ctx& c, double out[2]);
void launch_beta_sums_static(Ctx& c, double out[2]);
void launch_centroid(Ctx& c, double out[3]);
int beam_groups(const Ctx& c);              // beam species: bunch blocks, trapped, injected per ion species
void launch_beam_moments(Ctx& c, double* s1, double* s2);
void launch_diag(Ctx& c, double S[19]);
double launch_field_energy(Ctx& c);
void launch_shift(Ctx& c, int nxs, int nys, double sx, double sy);
void launch_rotate(Ctx& c, cpx* p, size_t n, double sx, double sy, int nys);
void launch_half_to_full(Ctx& c, const cpx* half, cpx* full, long planes);
void launch_full_to_half(Ctx& c, const cpx* full, cpx* half, long planes);
void sort_particles(Ctx& c);                // refresh perm
// the mixed form (k_mixed.cu)
void launch_deposit_f(Ctx& c);
void launch_cur_fft_f(Ctx& c, bool keep0);
void launch_march_f(Ctx& c, double D);
void launch_comoving_f(Ctx& c, double beta, double gm2);
void launch_sponge_f(Ctx& c);
void launch_real_fields_f(Ctx& c);
void launch_half_to_full_f(Ctx& c, const cpxf* half, cpx* full, long planes);
void launch_full_to_half_f(Ctx& c, const cpx* full, cpxf* half, long planes);
void launch_rotate_f(Ctx& c, cpxf* p, size_t n, double sx, double sy, int nys);
void launch_copy_f(Ctx& c, cpxf* y, const cpxf* x, size_t n);
void launch_axpy_fc(Ctx& c, cpxf* y, const cpx* x, double a, size_t n);   // y = y + a x
void launch_real_fields_slice_f(Ctx& c, int l, FmidOut fm = FmidOut(), bool cols = true);   // cols false: rows only (W given)
// particles and plasma (g3d_host.cu, g3d_plasma.cu)
void set_particles(Ctx& c, const g3d_particle* v, long n);
std::vector<g3d_particle> get_particles(Ctx& c);
void set_plasma(Ctx& c, const g3d_plasma& P, const g3d_ion* ions, int nions);
void march_plasma(Ctx& c, double s0, double s1);
void reset_plasma_march(Ctx& c);   // g3d_init: no streaming current of level s0, no particle waiting to join
void collect_restreaming(Ctx& c);
void add_grid_lasers(Ctx& c);
// The dynamic shared memory a kernel may use, raised to smem once per kernel and device (a host call per
// launch would leave the GPU waiting on the host between the small per-slice kernels)
void smem_attr(const void* kern, size_t smem);
// the adjoint march (k_adjoint.cu)
void launch_adj_objective(Ctx& c, double* dev_out2);
void launch_adj_seed(Ctx& c, double W, double* lam);
void launch_adj_real_fields(Ctx& c, const double* lF, cpx* const* W, cpx* const* lS);
void launch_adj_march(Ctx& c, cpx* const* lS, cpx* const* lj0, cpx* const* ljk, double D, int accz = 0);
void launch_adj_currents(Ctx& c, cpx* const* ljk, cpx* const* T, double* V, double* lJ, bool keep0 = false);
void launch_adj_deposit(Ctx& c, const double* X, const int32_t* alive, const double* lJ, double* lam);
// one slice of the streaming-plasma march (k_adjoint.cu): the transposed real fields and current spectra
void launch_adj_real_fields_slice(Ctx& c, const double* lF, long fpl, cpx* const* W, cpx* const* lsl);
void launch_adj_stream_spectra(Ctx& c, cpx* const* ljsn, cpx* const* T, double* lJ, bool keep0, double a2);
void launch_adj_rf_rows_slice(Ctx& c, const double* lF, long fpl, cpx* const* W);   // the rows half of each
void launch_adj_ss_rows(Ctx& c, cpx* const* T, double* lJ);
void launch_adj_push(Ctx& c, const float* Ff, const double* Fd, const double* X, const int32_t* alive, double s0, double s1,
                     double* lam, double* lF, int* err);
void launch_adj_lmodes(Ctx& c, const cpx* lRx, const cpx* lRy, cpx* out);
void launch_adj_comoving(Ctx& c, const cpx* lRx, const cpx* lRy, const cpx* jz, double beta, double gm2, cpx* ljz, double* dbeta);
void launch_adj_wsum(Ctx& c, const int32_t* alive, double* out);
void launch_adj_beta(Ctx& c, const double* X, const int32_t* alive, double coef, double* lam);
void launch_adj_widen(Ctx& c, const cpxf* a, cpx* b, long n);
std::vector<g3d_particle> get_streaming(Ctx& c);
// the plasma state of a checkpoint (g3d_plasma.cu): the joining list, the trapping counters, the streaming current
// of level s0 in the reference's full layout
std::vector<g3d_particle> get_joining(Ctx& c);
void set_joining(Ctx& c, const std::vector<g3d_particle>& v);
void get_plasma_counters(const Ctx& c, long& trapped, long& restreamed);
void set_plasma_counters(Ctx& c, long trapped, long restreamed);
std::vector<cpx> get_js0(Ctx& c, int comp);
void set_js0(Ctx& c, int comp, const std::vector<cpx>& v);
void launch_parts_unpack(Ctx& c, long n);   // pstage (records) -> parts (columns)
void launch_parts_pack(Ctx& c, long n);     // parts (columns) -> pstage (records)
// the live particles (alive 1) of the list in order, then the na records `add` (host): false when the capacity is short
bool beam_keep_live_and_append(Ctx& c, const g3d_particle* add, long na);

}  // namespace g3d

struct g3d_ctx {
    g3d::Ctx c;
};
