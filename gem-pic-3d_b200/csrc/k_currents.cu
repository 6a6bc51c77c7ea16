// Current deposition of the beam list, the (1,2,1)/4 zeta filter, the forward transverse FFTs and the
// transverse filters: Simulation::currents of the reference (src/sim_particles.cpp:56-207), Fourier y.
//
// The currents are real fields, so their spectra are Hermitian; only k_x = 0 .. nx/2 is kept (H = nx/2 + 1
// columns, [plane][j][k_x]).
//   k_deposit   one thread per particle: NGP over the zeta half-cell, TSC in x and y, into the raw current planes
//               jw [3][ns+3][ny][nx] (sim_particles.cpp:66-106) as fixed-point integer adds (see below), so that
//               the sums, and the whole run, do not depend on the order of the adds
//   k_cur_rows  per (block of rows, half-cell plane): zeta filter (sim_particles.cpp:120-138) of the three raw
//               planes (read as the deposit's integers and scaled to doubles on the way in), then per row one
//               complex FFT along x of jx + i jy, split by Hermitian symmetry into the half spectra of jx and jy,
//               and one of jz -> three half-spectrum planes (scratch W0, W1, W2)
//   k_cur_cols  per (half-cell plane, tile of 8 k_x columns): FFT along y, the cos^2 filters and the k_perp = 0
//               removal (sim_particles.cpp:146-156) -> jkx, jky, jkz
#include <algorithm>
#include "g3d_ctx.hpp"
#include "k_fft.cuh"
#include "k_dispatch.cuh"
#include "k_tma.cuh"

namespace g3d {

// ---------------------------------------------------------------- deposit
// Fixed-point deposit. Floating-point atomic adds make each sum depend on the order the adds arrive in, so two runs
// of the same input differ at the last bits and drift apart. Here every deposit value v of component c goes in as
// the integer round(v 2^e_c) with a 64-bit integer atomic add, which is associative: the sums, and all that follows
// them, are the same bits on every run. 2^e_c is the largest power of two with B_c 2^e_c < 2^62, B_c a bound on the
// sum of |v| over all particles and points of the component (per particle |f| x the largest dual-cell factor x
// |v_x/v_z|, |v_y/v_z| or 1, the TSC weights of a particle summing to 1), taken by a fixed-order two-level tree on
// the device, so no sum can overflow; each add is rounded to 2^-e_c < 2^-61 B_c, a scale of its own for each
// component because j_x and j_y of a relativistic bunch are far below j_z. A last pass turns the planes back into
// doubles (times 2^-e_c, exact for a power of two): the raw planes of the reference's layout that the filter reads.
constexpr int DB = 296, DT = 256;     // blocks and threads of the bound's first level

__device__ __forceinline__ void dep_bound_one(const PartsDev& P, long ip, const Geo& g, double ia_max, double b[3]) {
    if (P.alive[ip] != 1) return;
    int m; double fz;
    g.zax.locate(P.zeta[ip], m, fz);
    const int hw = m - (g.a - 2);
    if (hw < 0 || hw >= g.nh || m < 0 || m > g.N - 2) return;
    const double pz = P.pz[ip];               // the ratios v/v_z are p/p_z
    const double f = fabs(P.q[ip] * P.w[ip] / (g.hcg[m + 2] * g.dx)) * ia_max;
    b[0] += f * fabs(P.px[ip] / pz); b[1] += f * fabs(P.py[ip] / pz); b[2] += f;
}
__device__ __forceinline__ void block_sum3(double v[3], double* __restrict__ out) {
    __shared__ double sh[3][DT];
    for (int k = 0; k < 3; ++k) sh[k][threadIdx.x] = v[k];
    __syncthreads();
    for (int st = DT / 2; st > 0; st >>= 1) {
        if (int(threadIdx.x) < st)
            for (int k = 0; k < 3; ++k) sh[k][threadIdx.x] += sh[k][threadIdx.x + st];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 3; ++k) out[k] = sh[k][0];
}
__global__ void __launch_bounds__(DT) k_dep_bound(PartsDev P, long np, Geo g, double ia_max, double* __restrict__ part) {
    double acc[3] = {0, 0, 0};
    for (long i = long(blockIdx.x) * DT + threadIdx.x; i < np; i += long(gridDim.x) * DT) dep_bound_one(P, i, g, ia_max, acc);
    block_sum3(acc, part + 3 * blockIdx.x);
}
// the bound's three totals into tot[0..2]
__global__ void __launch_bounds__(DT) k_dep_total(const double* __restrict__ part, double* __restrict__ tot) {
    double acc[3] = {0, 0, 0};
    for (int b = threadIdx.x; b < DB; b += DT)
        for (int k = 0; k < 3; ++k) acc[k] += part[3 * b + k];
    block_sum3(acc, tot);
}
// scale[c] = 2^e_c, scale[3 + c] = 2^-e_c from the totals
__global__ void k_dep_scale(const double* __restrict__ tot, double* __restrict__ scale) {
    if (threadIdx.x < 3) {
        const double B = tot[threadIdx.x] * (1 + 1e-12) + 1e-300;   // the rounding of the bound's own sum; never 0
        int x;
        frexp(B, &x);                                               // B < 2^x
        const int e = min(62 - x, 1000);
        scale[threadIdx.x] = ldexp(1.0, e); scale[3 + threadIdx.x] = ldexp(1.0, -e);
    }
}
// pl: the values of one component (its planes)
__global__ void k_fix_to_double(double* __restrict__ J, long n, long pl, const double* __restrict__ scale) {
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += long(gridDim.x) * blockDim.x) {
        const long long q = reinterpret_cast<const long long*>(J)[i];
        J[i] = double(q) * scale[3 + int(i / pl)];
    }
}

__device__ __forceinline__ void fix_add(double* p, double v, double sc) {
    atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(__double2ll_rn(v * sc)));
}

// One thread per particle in cell order, 27 integer atomics each. (Summing the lanes of a warp that hit the same point
// first, with match-any and the warp's integer reductions, made this kernel 4x slower on the dense bunch of the
// oblique-wave workload: the integer adds in L2 are not what bounds it.)
__global__ void __launch_bounds__(256) k_deposit(PartsDev P, const int32_t* __restrict__ perm, long np, Geo g,
                                                double* __restrict__ J, const double* __restrict__ scale) {
    const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const long ip = perm[t];                 // cell order: neighbouring threads add into the same lines
    if (P.alive[ip] != 1) return;
    int m; double fz;
    g.zax.locate(P.zeta[ip], m, fz);
    const int hw = m - (g.a - 2);
    if (hw < 0 || hw >= g.nh || m < 0 || m > g.N - 2) return;
    const double px = P.px[ip], py = P.py[ip], pz = P.pz[ip];
    const double gm = sqrt(1 + px * px + py * py + pz * pz);
    const double vx = px / gm, vy = py / gm, vz = pz / gm;
    const double f = P.q[ip] * P.w[ip] / (g.hcg[m + 2] * g.dx);
    int ix[3], jn[3]; double wx[3], wn[3];
    tsc_periodic(P.x[ip], g.dx, g.nx, ix, wx);
    tsc_periodic(P.y[ip], g.dy, g.ny, jn, wn);
    const double ia0 = g.iA[0];
    const long nk = g.nk, pl = long(g.nh) * nk;
    double* J0 = J + long(hw) * nk;
#pragma unroll
    for (int v = 0; v < 3; ++v)
#pragma unroll
        for (int u = 0; u < 3; ++u) {
            const long k = long(jn[v]) * g.nx + ix[u];
            const double w = f * wx[u] * wn[v] * ia0;
            fix_add(J0 + k, w * vx / vz, scale[0]);
            fix_add(J0 + pl + k, w * vy / vz, scale[1]);
            fix_add(J0 + 2 * pl + k, w, scale[2]);
        }
}

// ---------------------------------------------------------------- zeta filter + FFT along x (rows)
constexpr int CUR_NT = 128;     // threads of the row kernel

// One CTA = LPC rows of one half-cell plane. The filter reads the three raw planes hk, hk+1, hk+2; the CTAs
// of neighbouring planes run together (blockIdx.x = rows is the fast index), so each raw plane comes from
// DRAM once and from L2 for its two neighbours.
// iscale (the fixed-point deposit's 2^-e_c per component, or null): the raw planes still hold the deposit's 64-bit
// integers, turned into doubles here as they are read (the same product as k_fix_to_double, without its pass over
// the planes)
template <int NX>
__global__ void __launch_bounds__(CUR_NT) k_cur_rows(Geo g, const double* __restrict__ J, cpx* __restrict__ TX,
                                                    cpx* __restrict__ TY, cpx* __restrict__ TZ, int zf,
                                                    const double* __restrict__ iscale) {
    using S = FftShape<NX>;
    constexpr int LPC = CUR_NT / S::T, RS = row_stride<NX>(), H = NX / 2 + 1;
    extern __shared__ cpx sm[];
    cpx* a0 = sm;                    // jx + i jy lines
    cpx* a1 = sm + LPC * RS;         // jz lines
    const int tid = threadIdx.x, r0 = blockIdx.x * LPC, hk = blockIdx.y;
    const long nk = g.nk, cpl = long(g.nh) * nk, nkh = long(g.ny) * H;
    const int hw = hk + 1, hc = g.a - 1 + hk;
    const bool live = hc >= 0 && hc <= g.N - 2;
    double wm = 0.25, w0 = 0.5, wp = 0.25, inv = 1.0;
    if (zf && !g.zeta_uniform && live) { wm = 0.25 * g.hcg[hc + 1]; w0 = 0.5 * g.hcg[hc + 2]; wp = 0.25 * g.hcg[hc + 3]; inv = g.hcg[hc + 2]; }
    #pragma unroll 1
    for (int u_ = 0; u_ < (LPC * NX + CUR_NT - 1) / CUR_NT; ++u_) {
        const int e = tid + u_ * CUR_NT;
        if (e >= LPC * NX) break;
        const int rr = e / NX, p = e - rr * NX, row = r0 + rr;
        double v[3] = {0, 0, 0};
        if (live && row < g.ny) {
            const long i = long(row) * NX + p;
#pragma unroll
            for (int comp = 0; comp < 3; ++comp) {
                const double* Jc = J + comp * cpl + i;
                double jm, j0, jp;
                if (iscale) {
                    const long long* Qc = reinterpret_cast<const long long*>(Jc);
                    const double sc = iscale[comp];
                    jm = double(__ldg(Qc + (hw - 1) * nk)) * sc; j0 = double(__ldg(Qc + hw * nk)) * sc;
                    jp = double(__ldg(Qc + (hw + 1) * nk)) * sc;
                } else {
                    jm = __ldg(Jc + (hw - 1) * nk); j0 = __ldg(Jc + hw * nk); jp = __ldg(Jc + (hw + 1) * nk);
                }
                if (zf && g.zeta_uniform) v[comp] = 0.25 * jm + 0.5 * j0 + 0.25 * jp;
                else if (zf) v[comp] = (wm * jm + w0 * j0 + wp * jp) / inv;
                else v[comp] = j0;
            }
        }
        a0[rr * RS + p + (p >> 3)] = C(v[0], v[1]);
        a1[rr * RS + p + (p >> 3)] = C(v[2], 0.0);
    }
    __syncthreads();
    const int r = tid / S::T, t = tid - r * S::T;
    {
        decltype(a0) const ls_[2] = {a0, a1};
        fft_lines<NX, 2>(ls_, RowAddr{r * RS}, t, g.twx);
    }
    const long base = long(hk) * nkh;
    #pragma unroll 1
    for (int u_ = 0; u_ < (LPC * H + CUR_NT - 1) / CUR_NT; ++u_) {
        const int e = tid + u_ * CUR_NT;
        if (e >= LPC * H) break;
        const int rr = e / H, kx = e - rr * H, row = r0 + rr;
        if (row >= g.ny) continue;
        const int km = (NX - kx) % NX;
        const cpx z = a0[rr * RS + kx + (kx >> 3)], zm = conj(a0[rr * RS + km + (km >> 3)]);
        const cpx d = z - zm;
        const long o = base + long(row) * H + kx;
        TX[o] = 0.5 * (z + zm);
        TY[o] = 0.5 * C(d.y, -d.x);
        TZ[o] = a1[rr * RS + kx + (kx >> 3)];
    }
}

// ---------------------------------------------------------------- FFT along y (columns) + k-filters
template <int NY, int CW>
__global__ void __launch_bounds__(CW * FftShape<NY>::T) k_cur_cols(Geo g, const cpx* __restrict__ TX, const cpx* __restrict__ TY,
                                                                   const cpx* __restrict__ TZ, cpx* __restrict__ JX,
                                                                   cpx* __restrict__ JY, cpx* __restrict__ JZ, int keep0) {
    using S = FftShape<NY>;
    extern __shared__ cpx sm[];
    cpx* s0 = sm;
    cpx* s1 = sm + ColTile<NY, CW>::size;
    cpx* s2 = sm + 2 * ColTile<NY, CW>::size;
    const int hk = blockIdx.y, c0 = blockIdx.x * CW, tid = threadIdx.x, nthr = CW * S::T;
    const int H = g.H;
    const long base = long(hk) * g.nkh;
    #pragma unroll
    for (int u_ = 0; u_ < (NY * CW + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * CW) break;
        const int p = e / CW, c = e - p * CW, kx = c0 + c;
        cpx u0 = C(0), u1 = C(0), u2 = C(0);
        if (kx < H) { const long o = base + long(p) * H + kx; u0 = TX[o]; u1 = TY[o]; u2 = TZ[o]; }
        s0[ColTile<NY, CW>::at(p, c)] = u0; s1[ColTile<NY, CW>::at(p, c)] = u1; s2[ColTile<NY, CW>::at(p, c)] = u2;
    }
    __syncthreads();
    const int c = tid % CW, t = tid / CW;
    {
        decltype(s0) const ls_[3] = {s0, s1, s2};
        fft_lines<NY, 3>(ls_, RowAddr{c * ColTile<NY, CW>::RS}, t, g.twy);
    }
    #pragma unroll
    for (int u_ = 0; u_ < (NY * CW + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * CW) break;
        const int p = e / CW, cc = e - p * CW, kx = c0 + cc;
        if (kx >= H) continue;
        const double f = (kx == 0 && p == 0 && !keep0) ? 0.0 : g.filt[kx] * g.filty[p];
        const long o = base + long(p) * H + kx;
        JX[o] = f * s0[ColTile<NY, CW>::at(p, cc)];
        JY[o] = f * s1[ColTile<NY, CW>::at(p, cc)];
        JZ[o] = f * s2[ColTile<NY, CW>::at(p, cc)];
    }
}

// The same with the tiles of TX, TY, TZ (maps 0, 1, 2) loaded by the TMA (k_tma.cuh): row-major 8-column tiles,
// transformed along their columns (stride 8).
template <int NY>
__global__ void __launch_bounds__(8 * FftShape<NY>::T) k_cur_cols_tma(Geo g, const __grid_constant__ TileMaps maps,
                                                                     cpx* __restrict__ JX, cpx* __restrict__ JY,
                                                                     cpx* __restrict__ JZ, int keep0, TmaWait wt) {
    using S = FftShape<NY>;
    extern __shared__ __align__(128) unsigned char smraw[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ int ok;
    const int hk = blockIdx.y, c0 = blockIdx.x * 8, tid = threadIdx.x, nthr = 8 * S::T;
    const int H = g.H;
    const long base = long(hk) * g.nkh;
    cpx* s0 = reinterpret_cast<cpx*>(smraw + ((128 - (smem_addr(smraw) & 127)) & 127));
    cpx* s1 = s0 + NY * 8;
    cpx* s2 = s1 + NY * 8;
    const int idx[3] = {0, 1, 2};
    cpx* const dst[3] = {s0, s1, s2};
    if (!tma_tiles<NY>(maps, idx, 3, dst, c0, hk * g.ny, &bar, &ok, wt)) return;
    const int c = tid % 8, t = tid / 8;
    {
        decltype(s0) const ls_[3] = {s0, s1, s2};
        fft_lines<NY, 3>(ls_, TileCol{c}, t, g.twy);
    }
    #pragma unroll
    for (int u_ = 0; u_ < (NY * 8 + nthr - 1) / nthr; ++u_) {
        const int e = tid + u_ * nthr;
        if (e >= NY * 8) break;
        const int p = e / 8, cc = e - p * 8, kx = c0 + cc;
        if (kx >= H) continue;
        const double f = (kx == 0 && p == 0 && !keep0) ? 0.0 : g.filt[kx] * g.filty[p];
        const long o = base + long(p) * H + kx;
        JX[o] = f * s0[e];
        JY[o] = f * s1[e];
        JZ[o] = f * s2[e];
    }
}

// ---------------------------------------------------------------- launchers
// the scales 2^e_c, 2^-e_c of the fixed-point deposit (six values; ia_max: the largest dual-cell factor); returns
// where they are
const double* launch_deposit_scale(Ctx& c, double ia_max) {
    if (c.depfix.n < size_t(3 * DB + 9)) c.depfix.alloc(size_t(3 * DB + 9), c.stream);
    double* tot = c.depfix.p + 3 * DB + 6;
    k_dep_bound<<<DB, DT, 0, c.stream>>>(c.parts, c.np, c.geo(), ia_max, c.depfix.p);
    c.check_launch("k_dep_bound");
    k_dep_total<<<1, DT, 0, c.stream>>>(c.depfix.p, tot);
    c.check_launch("k_dep_total");
    c.all_sum(tot, 3, G3D_SUM_F64);                      // a sharded run: the bound of every rank's particles
    k_dep_scale<<<1, 32, 0, c.stream>>>(tot, c.depfix.p + 3 * DB);
    c.check_launch("k_dep_scale");
    return c.depfix.p + 3 * DB;
}
// the fixed-point planes back to doubles (the free-hand deposit, and the raw planes read through the ABI)
void launch_deposit_finish(Ctx& c) {
    c.jw_fixed = false;
    const long n = long(c.jw.n);
    const long b = std::min<long>((n + 255) / 256, 148 * 16);
    k_fix_to_double<<<unsigned(b), 256, 0, c.stream>>>(c.jw.p, n, n / 3, c.depfix.p + 3 * DB);
    c.check_launch("k_fix_to_double");
}
void launch_deposit(Ctx& c) {
    c.jw.zero(c.stream);
    c.jw_fixed = false;                              // zero planes read the same either way
    if (c.np == 0 && !c.sharded()) return;           // a sharded rank without particles still takes part in the sums
    const int tok = c.prof_begin("deposit");
    const double* scale = launch_deposit_scale(c, 1 / c.dy);
    if (c.np > 0) {
        const unsigned blocks = unsigned((c.np + 255) / 256);
        k_deposit<<<blocks, 256, 0, c.stream>>>(c.parts, c.perm.p, c.np, c.geo(), c.jw.p, scale);
        c.check_launch("k_deposit");
    }
    c.jw_fixed = true;                               // k_cur_rows turns the integers into doubles as it reads them
    if (c.sharded()) shard_raw_halo(c);              // integer planes of one global scale: copied as they are
    c.prof_end(tok);
}

template <int NX>
static void cur_rows(Ctx& c, cpx* TX, cpx* TY, cpx* TZ) {
    using S = FftShape<NX>;
    constexpr int LPC = CUR_NT / S::T;
    const size_t smem = size_t(2) * LPC * row_stride<NX>() * sizeof(cpx);
    auto kern = k_cur_rows<NX>;
    smem_attr(reinterpret_cast<const void*>(kern), smem);
    const dim3 grid(unsigned((c.ny + LPC - 1) / LPC), unsigned(c.ns + 1));
    const int tok = c.prof_begin("cur_rows");
    kern<<<grid, CUR_NT, smem, c.stream>>>(c.geo(), c.jw.p, TX, TY, TZ, c.P.zeta_filter ? 1 : 0,
                                           c.jw_fixed ? c.depfix.p + 3 * DB + 3 : nullptr);
    c.check_launch("k_cur_rows");
    c.prof_end(tok);
}
// the tensor maps of TX, TY, TZ (the transform scratch W0..W2, ns + 1 planes), made once per set of buffers
static bool cur_maps(Ctx& c) {
    const cpx* p[3] = {c.W[0].p, c.W[1].p, c.W[2].p};
    return c.tma_cur.get(p, 3, c.H, long(c.ns + 1) * c.ny, c.ny);
}
template <int NY>
static void cur_cols(Ctx& c, bool keep0) {
    constexpr int CW = 8;
    if constexpr (NY <= 256 && (NY & (NY - 1)) == 0) {
        if (c.use_tma && cur_maps(c)) {
            const size_t smem = size_t(3) * NY * 8 * sizeof(cpx) + 128;
            smem_attr(reinterpret_cast<const void*>(k_cur_cols_tma<NY>), smem);
            const int tok = c.prof_begin("cur_cols");
            k_cur_cols_tma<NY><<<dim3(unsigned((c.H + 7) / 8), unsigned(c.ns + 1)), 8 * FftShape<NY>::T, smem, c.stream>>>(
                c.geo(), c.tma_cur.maps, c.jkx.p, c.jky.p, c.jkz.p, keep0 ? 1 : 0, c.tma_wait());
            c.check_launch("k_cur_cols_tma");
            c.prof_end(tok);
            return;
        }
    }
    const size_t smem = size_t(3) * ColTile<NY, CW>::size * sizeof(cpx);
    auto kern = k_cur_cols<NY, CW>;
    smem_attr(reinterpret_cast<const void*>(kern), smem);
    const dim3 grid(unsigned((c.H + CW - 1) / CW), unsigned(c.ns + 1));
    const int tok = c.prof_begin("cur_cols");
    kern<<<grid, CW * FftShape<NY>::T, smem, c.stream>>>(c.geo(), c.W[0].p, c.W[1].p, c.W[2].p, c.jkx.p, c.jky.p, c.jkz.p, keep0 ? 1 : 0);
    c.check_launch("k_cur_cols");
    c.prof_end(tok);
}

void launch_cur_fft(Ctx& c, bool keep0) {
    G3D_DISPATCH_N(c.nx, NX, cur_rows<NX>(c, c.W[0].p, c.W[1].p, c.W[2].p));
    G3D_DISPATCH_N(c.ny, NY, cur_cols<NY>(c, keep0));
}

// the zeta filter and the transform along x straight into jkx, jky, jkz (free-hand y: no transform along y)
void launch_cur_rows_to_jk(Ctx& c) { G3D_DISPATCH_N(c.nx, NX, cur_rows<NX>(c, c.jkx.p, c.jky.p, c.jkz.p)); }

}  // namespace g3d
