// Device reductions of the diagnostics (src/sim_output.cpp:5-77), of the window centroid
// (src/sim_setup.cpp:222-235) and of the mean beta of the bunch (src/sim_fields.cpp:45-51).
//
// The reference copies every particle to the host (or sums with atomics); here each reduction is a
// fixed-order two-level tree: a persistent grid of RB blocks accumulates grid-stride partial sums,
// each block reduces them in shared memory, and one block sums the block results in index order. The
// result depends only on the input, never on the thread schedule, so reruns are bit-identical.
#include "g3d_plasma.hpp"

namespace g3d {

namespace {
constexpr int RB = 296;     // blocks of the first level (2 per SM)
constexpr int RT = 256;     // threads per block

template <int NV>
__device__ void block_store(double (&acc)[NV], double* __restrict__ out) {
    __shared__ double sh[RT];
    for (int v = 0; v < NV; ++v) {
        sh[threadIdx.x] = acc[v];
        __syncthreads();
        for (int s = RT / 2; s > 0; s >>= 1) {
            if (int(threadIdx.x) < s) sh[threadIdx.x] += sh[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[long(blockIdx.x) * NV + v] = sh[0];
        __syncthreads();
    }
}

template <int NV>
__global__ void __launch_bounds__(RT) k_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
    double acc[NV];
    for (int v = 0; v < NV; ++v) acc[v] = 0;
    for (int b = threadIdx.x; b < nb; b += RT)
        for (int v = 0; v < NV; ++v) acc[v] += part[long(b) * NV + v];
    block_store<NV>(acc, out);
}

// ------------------------------------------------ particle sums of diag.txt
struct DiagArgs { LaserDev laser; double X0, Y0, s, zc; };
constexpr int NDIAG = 17;    // S[0..14], trapped count, trapped charge
__global__ void __launch_bounds__(RT) k_diag(PartsDev P, long np, DiagArgs d, double* __restrict__ part) {
    double acc[NDIAG];
    for (int v = 0; v < NDIAG; ++v) acc[v] = 0;
    for (long i = long(blockIdx.x) * RT + threadIdx.x; i < np; i += long(gridDim.x) * RT) {
        if (P.alive[i] != 1) continue;
        const double w = P.w[i];
        if (P.sp[i] > 0) { acc[15] += 1; acc[16] += P.q[i] * w; continue; }     // trapped plasma electrons
        const double px = P.px[i], py = P.py[i], pz = P.pz[i], zeta = P.zeta[i];
        const double g = sqrt(1 + px * px + py * py + pz * pz);
        const double X = P.x[i] + d.X0, Y = P.y[i] + d.Y0;
        const double et = d.laser.eta(X, d.s, d.s - (zeta - d.zc));
        const double v[14] = {1, X, Y, zeta, X * X, Y * Y, zeta * zeta, px, py, pz, g, px * d.laser.kx + pz * d.laser.kz, pz * pz, et};
        for (int k = 0; k < 14; ++k) acc[k] += w * v[k];
        acc[14] += 1;
    }
    block_store<NDIAG>(acc, part);
}

// ------------------------------------------------ field energy: sum over slices of 1/2 w E^2 (dual cells)
__global__ void __launch_bounds__(RT) k_energy(Geo g, const float* __restrict__ F, double* __restrict__ part) {
    double acc[1] = {0};
    const long nk = g.nk, fpl = long(g.ns + 2) * nk;
    for (long i = long(blockIdx.x) * RT + threadIdx.x; i < nk; i += long(gridDim.x) * RT) {
        const int j = int(i / g.nx);
        const double wn = 1 / g.iA[j], wh = 1 / g.iD[j];
        double e = 0;
        for (int l = 0; l < g.ns; ++l) {
            const double w = g.wsl[g.a + l];
            for (int comp = 0; comp < 6; ++comp) {
                const double v = F[comp * fpl + l * nk + i];
                const bool half = comp == 1 || comp == 3 || comp == 5;
                e += 0.5 * w * (half ? wh : wn) * v * v;
            }
        }
        acc[0] += e;
    }
    block_store<1>(acc, part);
}

// ------------------------------------------------ centroid of the bunch (window shift)
__global__ void __launch_bounds__(RT) k_centroid(PartsDev P, long np, double X0, double Y0, double* __restrict__ part) {
    double acc[3] = {0, 0, 0};
    for (long i = long(blockIdx.x) * RT + threadIdx.x; i < np; i += long(gridDim.x) * RT) {
        if (P.alive[i] != 1 || P.sp[i] > 0) continue;
        const double w = P.w[i];
        acc[0] += w * (P.x[i] + X0); acc[1] += w * (P.y[i] + Y0); acc[2] += w;
    }
    block_store<3>(acc, part);
}

// ------------------------------------------------ mean beta of the alive particles (co-moving field)
// The reference sums w v_z and w over the particles in array order on the host (sim_fields.cpp:45-47). The
// mean beta enters 1 - beta^2 = gamma^-2 with a cancellation of 1 - 1/gamma^2, so the sum is taken in the
// same order with the same IEEE operations (no FMA contraction): every term in parallel, then one warp adds
// them in index order, 32 terms per coalesced load. Bit for bit the reference's value; used once per start.
__global__ void k_beta_terms(PartsDev P, long np, double* __restrict__ t, double* __restrict__ w) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < np; i += long(gridDim.x) * blockDim.x) {
        const bool al = P.alive[i] == 1;
        const double px = P.px[i], py = P.py[i], pz = P.pz[i], wi = P.w[i];
        const double g2 = __dadd_rn(__dadd_rn(__dadd_rn(1.0, __dmul_rn(px, px)), __dmul_rn(py, py)), __dmul_rn(pz, pz));
        t[i] = al ? __ddiv_rn(__dmul_rn(wi, pz), __dsqrt_rn(g2)) : 0.0;
        w[i] = al ? wi : 0.0;
    }
}
__global__ void k_seq_sum2(const double* __restrict__ t, const double* __restrict__ w, long n, const int32_t* __restrict__ alive,
                           double* __restrict__ out) {
    const int lane = threadIdx.x;
    double s0 = 0, s1 = 0;
    for (long b = 0; b < n; b += 32) {
        const long i = b + lane;
        const double ti = i < n ? t[i] : 0.0, wi = i < n ? w[i] : 0.0;
        const int al = i < n ? alive[i] : 0;
        const unsigned live = __ballot_sync(0xffffffffu, al == 1);
        for (int k = 0; k < 32; ++k) {
            const double a = __shfl_sync(0xffffffffu, ti, k), c = __shfl_sync(0xffffffffu, wi, k);
            if (live >> k & 1u) { s0 = __dadd_rn(s0, a); s1 = __dadd_rn(s1, c); }
        }
    }
    if (lane == 0) { out[0] = s0; out[1] = s1; }
}

// ------------------------------------------------ moments of the beam species (bunches.txt)
// group of a beam particle: bunch block k (sp = -k) -> k, trapped plasma electrons -> nbunch, electrons injected
// from ion species m (sp = 100 + m) -> nbunch + 1 + m (the reference's Config::beam_index); -1: none
constexpr int MOM_G = 16, MOM_NV = 8 * MOM_G;
__device__ __forceinline__ int beam_group(int sp, int nbunch, int ngroups) {
    const int g = sp <= 0 ? -sp : (sp >= 100 ? nbunch + 1 + (sp - 100) : nbunch);
    return g < ngroups ? g : -1;
}
__device__ __forceinline__ void beam_values(const PartsDev& P, long i, double X0, double Y0, double v[6]) {
    const double px = P.px[i], py = P.py[i], pz = P.pz[i];
    v[0] = P.x[i] + X0; v[1] = P.y[i] + Y0; v[2] = P.zeta[i]; v[3] = px; v[4] = py;
    v[5] = sqrt(1 + px * px + py * py + pz * pz);
}
// first pass: w, count and w v per group; second pass (mean given): the centred second moments
template <int PASS>
__global__ void __launch_bounds__(RT) k_moments(PartsDev P, long np, double X0, double Y0, int nbunch, int ngroups,
                                               const double* __restrict__ mean, double* __restrict__ part) {
    double acc[MOM_NV];
    for (int v = 0; v < MOM_NV; ++v) acc[v] = 0;
    for (long i = long(blockIdx.x) * RT + threadIdx.x; i < np; i += long(gridDim.x) * RT) {
        if (P.alive[i] != 1) continue;
        const int g = beam_group(P.sp[i], nbunch, ngroups);
        if (g < 0) continue;
        double v[6];
        beam_values(P, i, X0, Y0, v);
        const double w = P.w[i];
        double* a = acc + 8 * g;
        if (PASS == 1) {
            a[0] += w; a[1] += 1;
            for (int k = 0; k < 6; ++k) a[2 + k] += w * v[k];
        } else {
            double d[6];
            for (int k = 0; k < 6; ++k) d[k] = v[k] - mean[6 * g + k];
            a[0] += w * d[0] * d[0]; a[1] += w * d[1] * d[1]; a[2] += w * d[2] * d[2]; a[3] += w * d[3] * d[3];
            a[4] += w * d[4] * d[4]; a[5] += w * d[0] * d[3]; a[6] += w * d[1] * d[4]; a[7] += w * d[5] * d[5];
        }
    }
    block_store<MOM_NV>(acc, part);
}

// `sum`: a sum over the particles, which a sharded run adds across the ranks
template <int NV>
void finish(Ctx& c, double* out, bool sum) {
    k_final<NV><<<1, RT, 0, c.stream>>>(c.red.p, RB, c.red.p + RB * NV);
    c.check_launch("k_final");
    if (sum) c.all_sum(c.red.p + RB * NV, NV, G3D_SUM_F64);
    G3D_CUDA(cudaMemcpyAsync(out, c.red.p + RB * NV, NV * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
}
}  // namespace

void launch_diag(Ctx& c, double S[19]) {
    double r[NDIAG];
    DiagArgs d{c.laser, c.X0, c.Y0, c.s, c.P.zeta_center};
    const int tok = c.prof_begin("diag");
    k_diag<<<RB, RT, 0, c.stream>>>(c.parts, c.np, d, c.red.p);
    c.check_launch("k_diag");
    c.prof_end(tok);
    finish<NDIAG>(c, r, true);
    for (int k = 0; k < 15; ++k) S[k] = r[k];
    S[17] = r[15]; S[18] = r[16];
}

double launch_field_energy(Ctx& c) {
    double r[1];
    const int tok = c.prof_begin("field_energy");
    k_energy<<<RB, RT, 0, c.stream>>>(c.geo(), c.F.p, c.red.p);
    c.check_launch("k_energy");
    c.prof_end(tok);
    finish<1>(c, r, true);                    // a sharded run: the energies of the slabs
    return r[0] * c.dx;
}

int beam_groups(const Ctx& c) { return c.nbunch + 1 + (c.pl ? int(c.pl->ions.size()) : 0); }
void launch_beam_moments(Ctx& c, double* s1, double* s2) {
    const int G = beam_groups(c);
    if (G > MOM_G) throw Error(G3D_ERR_CAPACITY, "beam moments: more than " + std::to_string(MOM_G) + " beam species");
    if (c.momw.n < size_t(RB + 2) * MOM_NV) c.momw.alloc(size_t(RB + 2) * MOM_NV, c.stream);
    double* part = c.momw.p;
    double* tot = part + size_t(RB) * MOM_NV;
    double* mean = tot + MOM_NV;
    std::vector<double> r(MOM_NV), mh(MOM_NV, 0.0);
    k_moments<1><<<RB, RT, 0, c.stream>>>(c.parts, c.np, c.X0, c.Y0, c.nbunch, G, mean, part);
    c.check_launch("k_moments");
    k_final<MOM_NV><<<1, RT, 0, c.stream>>>(part, RB, tot);
    c.check_launch("k_final");
    c.all_sum(tot, MOM_NV, G3D_SUM_F64);
    G3D_CUDA(cudaMemcpyAsync(r.data(), tot, MOM_NV * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
    for (int g = 0; g < G; ++g) {
        for (int k = 0; k < 8; ++k) s1[8 * g + k] = r[size_t(8 * g + k)];
        for (int k = 0; k < 6; ++k) mh[size_t(6 * g + k)] = r[size_t(8 * g)] > 0 ? r[size_t(8 * g + 2 + k)] / r[size_t(8 * g)] : 0;
    }
    G3D_CUDA(cudaMemcpyAsync(mean, mh.data(), MOM_NV * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    k_moments<2><<<RB, RT, 0, c.stream>>>(c.parts, c.np, c.X0, c.Y0, c.nbunch, G, mean, part);
    c.check_launch("k_moments");
    k_final<MOM_NV><<<1, RT, 0, c.stream>>>(part, RB, tot);
    c.check_launch("k_final");
    c.all_sum(tot, MOM_NV, G3D_SUM_F64);
    G3D_CUDA(cudaMemcpyAsync(r.data(), tot, MOM_NV * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
    for (int g = 0; g < G; ++g)
        for (int k = 0; k < 8; ++k) s2[8 * g + k] = r[size_t(8 * g + k)];
}

void launch_centroid(Ctx& c, double out[3]) {
    k_centroid<<<RB, RT, 0, c.stream>>>(c.parts, c.np, c.X0, c.Y0, c.red.p);
    c.check_launch("k_centroid");
    finish<3>(c, out, true);
}

void launch_beta_sums(Ctx& c, double out[2]) {
    out[0] = out[1] = 0;
    if (c.np == 0 && !c.sharded()) return;
    DevBuf<double> tw;
    tw.alloc(size_t(2 * c.np + 2), c.stream);                       // zeroed: a rank without particles adds 0
    if (c.np > 0) {
        k_beta_terms<<<RB, RT, 0, c.stream>>>(c.parts, c.np, tw.p, tw.p + c.np);
        c.check_launch("k_beta_terms");
        k_seq_sum2<<<1, 32, 0, c.stream>>>(tw.p, tw.p + c.np, c.np, c.parts.alive, tw.p + 2 * c.np);
        c.check_launch("k_seq_sum2");
    }
    c.all_sum(tw.p + 2 * c.np, 2, G3D_SUM_F64);   // a sharded run: the ranks' sums in rank order of the reducer
    G3D_CUDA(cudaMemcpyAsync(out, tw.p + 2 * c.np, 2 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
}

// ------------------------------------------------ the same beta sums with file-scope scratch (no allocation)
// Scratch of g3d_beam_beta_sums_static: the per-particle terms t[0..np), w[0..np) and the two sums at [2 np],
// [2 np + 1], for at most G3D_BETA_STATIC_MAX particles (16 MiB + 16 B). It is a static device symbol of this
// library: one copy per device, shared by every context on that device, so two calls in flight at once on one
// device (two streams, threads or contexts) race on it. Nothing in it has to start at zero: every term below np
// is written before the sequential sum reads it, and the two sums are stored, not accumulated.
static __device__ __align__(256) double g_beta_scratch[2 * G3D_BETA_STATIC_MAX + 2];

void launch_beta_sums_static(Ctx& c, double out[2]) {
    if (c.np > G3D_BETA_STATIC_MAX)
        throw Error(G3D_ERR_CAPACITY, "g3d_beam_beta_sums_static: " + std::to_string(c.np) +
                                          " particles exceed the static scratch of G3D_BETA_STATIC_MAX = " +
                                          std::to_string(G3D_BETA_STATIC_MAX) + "; use g3d_comoving_field");
    out[0] = out[1] = 0;
    if (c.np == 0) return;
    void* sym = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress(&sym, g_beta_scratch);      // per device: the current one
    if (rc != cudaSuccess)
        throw Error(G3D_ERR_CUDA, std::string("cudaGetSymbolAddress(g_beta_scratch): ") + cudaGetErrorString(rc));
    double* tw = static_cast<double*>(sym);
    k_beta_terms<<<RB, RT, 0, c.stream>>>(c.parts, c.np, tw, tw + c.np);
    c.check_launch("k_beta_terms");
    k_seq_sum2<<<1, 32, 0, c.stream>>>(tw, tw + c.np, c.np, c.parts.alive, tw + 2 * c.np);
    c.check_launch("k_seq_sum2");
    G3D_CUDA(cudaMemcpyAsync(out, tw + 2 * c.np, 2 * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
}

}  // namespace g3d
