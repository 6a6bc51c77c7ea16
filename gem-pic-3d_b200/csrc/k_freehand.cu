// The march on the free-hand y grid (y_fourier = 0): x stays Fourier (half spectra k_x = 0 .. nx/2), y is a
// table of ny + 1 nodes between conducting walls, with E_x, B_y, E_z, j_x, j_z on the nodes and E_y, B_x, B_z, j_y
// on the half-nodes. The arrays keep the layout [plane][j][k_x] of the Fourier form, with j a point of y.
//   k_deposit_fh    TSC in x and along the y table (nodes and half-nodes), FP64 atomics
//                   (Simulation::currents, src/sim_particles.cpp:88-106)
//   k_cur_lines_fh  per (half-cell, k_x) line: (1,2,1)/4 on the cell charges along y (nodes: zero at the walls;
//                   half-nodes: mirrored), the y-mean of j_y removed at k_x = 0 (TEM), the x filter
//                   (sim_particles.cpp:165-205); the zeta filter and the x transform are the rows kernel of
//                   k_currents.cu
//   k_march_lines   one CTA per k_x line, a thread per y row, slices front to rear: the known parts of R and L,
//                   E_z on the nodes and B_z on the half-nodes from two tridiagonal systems along y solved together
//                   by parallel cyclic reduction in shared memory, then R and L (the scheme of march_line,
//                   src/sim_kernels.hpp:213-313)
//   k_sp_psi_fh     sponge: the bound field psi = T^-1 (rho + gamma^-2 T^-1 d_zeta^2 rho), T = k_x^2 - Lap_y with
//                   the precomputed LU factors, and R - R_b (sim_fields.cpp:199-232); then the rows kernel of
//                   k_fields.cu (inverse x, mask, forward x) and k_sp_add_fh (+ R_b, R_x = 0 at the wall node)
//   k_comoving_fh_* the co-moving start field in the eigenvectors of -Lap_y: projection of the charge, Thomas in
//                   zeta per (eigenvalue, k_x), back to the nodes, R (sim_fields.cpp:44-151)
// The other kernels take one thread per line (the lines of a window are many); the filters and solves along y in
// them are serial in the reference's order.
#include "g3d_ctx.hpp"

namespace g3d {

namespace {
__device__ __forceinline__ cpx ikx(double k, cpx z) { return ik(k, z); }     // i k_x z
}  // namespace

// ---------------------------------------------------------------- deposit
__device__ __forceinline__ void fix_add_fh(double* p, double v, double sc) {   // fixed-point add (k_currents.cu)
    atomicAdd(reinterpret_cast<unsigned long long*>(p), static_cast<unsigned long long>(__double2ll_rn(v * sc)));
}
__global__ void __launch_bounds__(256) k_deposit_fh(PartsDev P, const int32_t* __restrict__ perm, long np, Geo g,
                                                   double* __restrict__ J, const double* __restrict__ scale) {
    const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= np) return;
    const long ip = perm[t];
    if (P.alive[ip] != 1) return;
    int m; double fz;
    g.zax.locate(P.zeta[ip], m, fz);
    const int hw = m - (g.a - 2);
    if (hw < 0 || hw >= g.nh || m < 0 || m > g.N - 2) return;
    const double px = P.px[ip], py = P.py[ip], pz = P.pz[ip];
    const double gm = sqrt(1 + px * px + py * py + pz * pz);
    const double vx = px / gm, vy = py / gm, vz = pz / gm;
    const double f = P.q[ip] * P.w[ip] / (g.hcg[m + 2] * g.dx);
    int ix[3], jn[3], jh[3]; double wx[3], wn[3], wh[3];
    tsc_periodic(P.x[ip], g.dx, g.nx, ix, wx);
    tsc_y(g.yax, P.y[ip], jn, wn, jh, wh);
    const long nk = g.nk, pl = long(g.nh) * nk;
    double* J0 = J + long(hw) * nk;
    for (int v = 0; v < 3; ++v) {
        const bool nod = jn[v] >= 1 && jn[v] <= g.ny - 1, hal = jh[v] >= 0 && jh[v] <= g.ny - 1;
        for (int u = 0; u < 3; ++u) {
            if (nod) {
                const long k = long(jn[v]) * g.nx + ix[u];
                const double w = f * wx[u] * wn[v] * g.iA[jn[v]];
                fix_add_fh(J0 + k, w * vx / vz, scale[0]);
                fix_add_fh(J0 + 2 * pl + k, w, scale[2]);
            }
            if (hal) {
                const long k = long(jh[v]) * g.nx + ix[u];
                fix_add_fh(J0 + pl + k, f * wx[u] * wh[v] * g.iD[jh[v]] * vy / vz, scale[1]);
            }
        }
    }
}

// ---------------------------------------------------------------- filters along the y lines of the currents
__global__ void k_cur_lines_fh(Geo g, cpx* __restrict__ jx, cpx* __restrict__ jy, cpx* __restrict__ jz, int kf, int keep0) {
    const long nl = long(g.ns + 1) * g.H;
    const long line = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (line >= nl) return;
    const int H = g.H, ny = g.ny, kxi = int(line % H);
    const long o = (line / H) * g.nkh + kxi;         // element j at o + j H
    const double* ia = g.iA; const double* id = g.iD;
    const double fx = g.filt[kxi];
    if (kf) {
        cpx* nodal[2] = {jx, jz};
        for (int t = 0; t < 2; ++t) {                // nodes: charges Q_j = A_j J_j, Q = 0 at the walls
            cpx* A = nodal[t];
            cpx qm = C(0), q0 = A[o + H] / ia[1];
            for (int j = 1; j < ny; ++j) {
                const cpx qp = j + 1 < ny ? A[o + long(j + 1) * H] / ia[j + 1] : C(0);
                A[o + long(j) * H] = (0.25 * qm + 0.5 * q0 + 0.25 * qp) * ia[j];
                qm = q0; q0 = qp;
            }
        }
        cpx qm = jy[o] / id[0], q0 = qm;             // half-nodes: Q_j = Delta_j J_j, mirrored at the walls
        for (int j = 0; j < ny; ++j) {
            const cpx qp = j + 1 < ny ? jy[o + long(j + 1) * H] / id[j + 1] : q0;
            jy[o + long(j) * H] = (0.25 * qm + 0.5 * q0 + 0.25 * qp) * id[j];
            qm = q0; q0 = qp;
        }
    }
    cpx mean = C(0);
    if (kxi == 0 && !keep0) {
        for (int j = 0; j < ny; ++j) mean = mean + jy[o + long(j) * H] / id[j];
        mean = mean / (g.yn[ny] - g.yn[0]);
    }
    jx[o] = C(0); jz[o] = C(0);
    for (int j = 0; j < ny; ++j) {
        const long k = o + long(j) * H;
        jx[k] = fx * jx[k]; jz[k] = fx * jz[k]; jy[k] = fx * (jy[k] - mean);
    }
}

// ---------------------------------------------------------------- filters of the streaming current along y
// per k_x line of one half-cell (Simulation::stream_spectra, src/sim_plasma.cpp:146-180): the (1,2,1)/4 filters of
// the cell charges as for the beam (no TEM mean removed), j_x = j_z = 0 at the wall node, the x filter, then the
// smoothing (1 - a^2 Lap_perp)^-1: (1 + a^2 (k_x^2 - b- b+)) f = g on the nodes (f = 0 at the walls, as E_z in the
// march) and (1 + a^2 (k_x^2 - b+ b-)) f = g on the half-nodes (as B_z). One CTA per k_x line, a thread per y row:
// the charges Q_j of a row and its neighbours from shared memory (the same products and sums as a sweep along the
// line), the smoothing systems (one matrix for j_x and j_z on the nodes, one for j_y on the half-nodes, strictly
// diagonally dominant) by parallel cyclic reduction as in the march of the lines.
template <int MAXT>
__global__ void __launch_bounds__(MAXT) k_ss_lines_fh(Geo g, const cpx* __restrict__ T, cpx* __restrict__ out, int kf, double a2) {
    extern __shared__ double2 sm[];
    const int ny = g.ny, H = g.H, kxi = blockIdx.x, j = threadIdx.x;
    const bool row = j < ny;
    const long nkh = g.nkh, k = long(row ? j : 0) * H + kxi;
    cpx* qx = sm; cpx* qy = sm + ny; cpx* qz = sm + 2 * ny;        // charges of the rows
    cpx* rx = sm + 3 * ny; cpx* ry = sm + 4 * ny; cpx* rz = sm + 5 * ny;
    double* lo_n = reinterpret_cast<double*>(sm + 6 * ny);
    double* dg_n = lo_n + ny; double* up_n = dg_n + ny; double* lo_h = up_n + ny; double* dg_h = lo_h + ny; double* up_h = dg_h + ny;
    const double* ia = g.iA; const double* id = g.iD;
    cpx vx = C(0), vy = C(0), vz = C(0);
    if (row) { vx = T[k]; vy = T[nkh + k]; vz = T[2 * nkh + k]; }
    if (kf) {
        // nodes (j_x, j_z): Q_j = J_j / (1/A_j), zero on the wall node 0 and beyond the last node; half-nodes (j_y):
        // Q_j = J_j / (1/Delta_j), mirrored at both walls
        if (row) {
            qx[j] = j == 0 ? C(0) : vx / ia[j]; qz[j] = j == 0 ? C(0) : vz / ia[j];
            qy[j] = vy / id[j];
        }
        __syncthreads();
        if (row) {
            if (j > 0) {
                const cpx xm = j > 1 ? qx[j - 1] : C(0), zm = j > 1 ? qz[j - 1] : C(0);
                const cpx xp = j + 1 < ny ? qx[j + 1] : C(0), zp = j + 1 < ny ? qz[j + 1] : C(0);
                vx = (0.25 * xm + 0.5 * qx[j] + 0.25 * xp) * ia[j];
                vz = (0.25 * zm + 0.5 * qz[j] + 0.25 * zp) * ia[j];
            }
            const cpx ym = j > 0 ? qy[j - 1] : qy[0], yp = j + 1 < ny ? qy[j + 1] : qy[ny - 1];
            vy = (0.25 * ym + 0.5 * qy[j] + 0.25 * yp) * id[j];
        }
    }
    const double fx = g.filt[kxi];
    if (j == 0) { vx = C(0); vz = C(0); }
    vx = fx * vx; vy = fx * vy; vz = fx * vz;
    if (a2 > 0) {
        const double kx2 = g.kxs[kxi] * g.kxs[kxi];
        // nodes 1..ny-1 (row 0, the wall, stays 0) and half-nodes 0..ny-1
        double an = 0, bn = 1, cn = 0, ah = 0, bh = 1, ch = 0;
        if (row) {
            if (j > 0) {
                an = j > 1 ? -a2 * ia[j] * id[j - 1] : 0;
                cn = j < ny - 1 ? -a2 * ia[j] * id[j] : 0;
                bn = 1 + a2 * kx2 + a2 * ia[j] * (id[j - 1] + id[j]);
            }
            const double al = j > 0 ? ia[j] : 0, au = j < ny - 1 ? ia[j + 1] : 0;
            ah = -a2 * id[j] * al; ch = -a2 * id[j] * au;
            bh = 1 + a2 * kx2 + a2 * id[j] * (al + au);
        }
        for (int st = 1; st < ny; st <<= 1) {
            __syncthreads();                                        // the previous step's reads are done
            if (row) {
                lo_n[j] = an; dg_n[j] = bn; up_n[j] = cn; rx[j] = vx; rz[j] = vz;
                lo_h[j] = ah; dg_h[j] = bh; up_h[j] = ch; ry[j] = vy;
            }
            __syncthreads();
            if (row) {
                const int m = j - st, q = j + st;
                double nan_ = 0, ncn = 0, nah = 0, nch = 0, nbn = bn, nbh = bh;
                cpx dx = vx, dz = vz, dy = vy;
                if (m >= 0) {
                    const double fn = an / dg_n[m], fh = ah / dg_h[m];
                    nan_ = -lo_n[m] * fn; nah = -lo_h[m] * fh;
                    nbn -= up_n[m] * fn; nbh -= up_h[m] * fh;
                    dx = dx - fn * rx[m]; dz = dz - fn * rz[m]; dy = dy - fh * ry[m];
                }
                if (q < ny) {
                    const double gn = cn / dg_n[q], gh = ch / dg_h[q];
                    ncn = -up_n[q] * gn; nch = -up_h[q] * gh;
                    nbn -= lo_n[q] * gn; nbh -= lo_h[q] * gh;
                    dx = dx - gn * rx[q]; dz = dz - gn * rz[q]; dy = dy - gh * ry[q];
                }
                an = nan_; cn = ncn; bn = nbn; ah = nah; ch = nch; bh = nbh;
                vx = dx; vz = dz; vy = dy;
            }
        }
        if (row) {
            vx = j == 0 ? C(0) : vx / bn; vz = j == 0 ? C(0) : vz / bn;
            vy = vy / bh;
        }
    }
    if (row) { out[k] = vx; out[nkh + k] = vy; out[2 * nkh + k] = vz; }
}

// ---------------------------------------------------------------- the march of the k_x lines
// One CTA per k_x line, one thread per y row j (nodes for E_z, R_x, L_x; half-nodes for B_z, R_y, L_y), slices
// from the top of the range down. Per slice (the scheme of the reference's march_line, src/sim_kernels.hpp:213-313):
//   1. the parts of R known at level s0 (R + D (curl terms of E_z, B_z) - D J, J the slice current interpolated
//      between its two half-cells with w_lo, w_hi);
//   2. the parts of L known from the slice above (level s1);
//   3. E_z on the nodes (Dirichlet at both walls) and B_z on the half-nodes (Neumann) from two tridiagonal systems
//      along y, both solved together by parallel cyclic reduction: ceil(log2 ny) halving steps in shared memory, each
//      row eliminating its neighbours at distance s = 1, 2, 4, ... (the systems are strictly diagonally dominant,
//      diagonal 1 + cc (k_x^2 + ...) against off-diagonals summing to cc (...), so the reduction is stable);
//   4. R and L from the new E_z, B_z.
// The slice above stays in shared memory from one slice to the next, so a slice reads only its own level-s0 fields
// and one current plane (the other current plane is the one the slice above read), and the loads of the next slice
// are issued before this slice's work. Rows beyond ny (the padding of the CTA) take part in the barriers only.
struct LineArrays {
    cpx *Rx, *Ry, *Ez, *Bz, *Lx, *Ly;
    const cpx *j0x, *j0y, *jkx, *jky, *jkz;
};
constexpr int LINE_MAX_NY = 512;
// shared memory of one line: the slice above (6 planes), this slice's level-s0 E_z and B_z, the known parts (4),
// the new E_z and B_z, and the two reduction systems (3 real coefficients and a complex right side per row each)
static size_t line_smem(int ny) { return size_t(ny) * (14 * sizeof(cpx) + 2 * (3 * sizeof(double) + sizeof(cpx))); }

struct SliceIn {           // what a row reads of one slice: level-s0 fields and the slice's lower current plane
    cpx rx, ry, ez, bz, jx, jy, kx_, ky_, kz_;
};
__device__ __forceinline__ SliceIn load_slice(const LineArrays& A, long o) {
    SliceIn v;
    v.rx = A.Rx[o]; v.ry = A.Ry[o]; v.ez = A.Ez[o]; v.bz = A.Bz[o];
    v.kx_ = A.jkx[o]; v.ky_ = A.jky[o]; v.kz_ = A.jkz[o];
    v.jx = A.j0x[o] + v.kx_; v.jy = A.j0y[o] + v.ky_;
    return v;
}

template <int MAXT>
__global__ void __launch_bounds__(MAXT) k_march_lines(Geo g, LineArrays A, double D, int n_top, int n_bot) {
    extern __shared__ double2 sm[];
    const int ny = g.ny, H = g.H, line = blockIdx.x, j = threadIdx.x;
    const bool row = j < ny;
    const long nk = g.nkh, col = long(row ? j : 0) * H + line;
    cpx* up6 = sm;                       // the slice above: R_x, R_y, E_z, B_z, L_x, L_y (ny each)
    cpx* lvE = sm + 6 * ny;              // this slice, level s0: E_z, B_z
    cpx* lvB = lvE + ny;
    cpx* kn = lvB + ny;                  // known parts: R_x, R_y, L_x, L_y
    cpx* nwE = kn + 4 * ny;              // the new E_z, B_z
    cpx* nwB = nwE + ny;
    cpx* rhsE = nwB + ny;                // reduction systems: right sides, then lower, diagonal, upper
    cpx* rhsB = rhsE + ny;
    double* lo_E = reinterpret_cast<double*>(rhsB + ny);
    double* dg_E = lo_E + ny; double* up_E = dg_E + ny;
    double* lo_B = up_E + ny; double* dg_B = lo_B + ny; double* up_B = dg_B + ny;
    cpx* uRx = up6; cpx* uRy = up6 + ny; cpx* uEz = up6 + 2 * ny; cpx* uBz = up6 + 3 * ny; cpx* uLx = up6 + 4 * ny;
    cpx* uLy = up6 + 5 * ny;
    cpx* kRx = kn; cpx* kRy = kn + ny; cpx* kLx = kn + 2 * ny; cpx* kLy = kn + 3 * ny;

    const double kx = g.kxd[line], kx2 = kx * kx;
    const double iAj = row ? g.iA[j] : 0, iDj = row ? g.iD[j] : 0;
    const double iDm = (row && j > 0) ? g.iD[j - 1] : 0, iAp = (row && j + 1 < ny) ? g.iA[j + 1] : 0;
    const cpx Z = C(0);
    // the slice above the range (unless the range starts at the window front) and the upper current plane of
    // the first slice
    SliceIn up{};
    if (row) {
        const long o = long(n_top + 1 - g.a) * nk + col;
        if (n_top < g.N - 1) {
            uRx[j] = A.Rx[o]; uRy[j] = A.Ry[o]; uEz[j] = A.Ez[o]; uBz[j] = A.Bz[o]; uLx[j] = A.Lx[o]; uLy[j] = A.Ly[o];
        }
        up.kx_ = A.jkx[o]; up.ky_ = A.jky[o]; up.kz_ = A.jkz[o];
        up.jx = A.j0x[o] + up.kx_; up.jy = A.j0y[o] + up.ky_;
    }
    SliceIn cur{};
    if (row) cur = load_slice(A, long(n_top - g.a) * nk + col);
    for (int n = n_top; n >= n_bot; --n) {
        const long o = long(n - g.a) * nk + col;
        SliceIn nxt{};
        if (row && n > n_bot) nxt = load_slice(A, o - nk);        // the next slice's inputs, in flight meanwhile
        if (row) { lvE[j] = cur.ez; lvB[j] = cur.bz; }
        __syncthreads();
        // 1. known part of R
        const double wl = g.wlo[n], wu = g.whi[n];
        cpx sRx = Z, sRy = Z;
        if (row) {
            const cpx Jx = wl * cur.jx + wu * up.jx, Jy = wl * cur.jy + wu * up.jy;
            if (j > 0) sRx = cur.rx + D * (ik(kx, cur.ez) + (cur.bz - lvB[j - 1]) * iAj) - D * Jx;
            const cpx ez_up = j + 1 < ny ? lvE[j + 1] : Z;
            sRy = cur.ry + D * ((ez_up - cur.ez) * iDj - ik(kx, cur.bz)) - D * Jy;
        }
        cpx oRx, oRy, oEz = Z, oBz = Z, oLx = Z, oLy = Z;
        if (n == g.N - 1) {                                      // window front: L = E_z = B_z = 0
            oRx = sRx; oRy = sRy;
            __syncthreads();                                     // the neighbours' reads of lvE, lvB are done
        } else {
            // 2. known part of L from the slice above
            const double h = g.hcg[n + 2], cc = 0.25 * h * (D + 0.25 * h);
            cpx sLx = Z, sLy = Z, pe = Z;
            if (row) {
                pe = j == 0 ? Z : uEz[j];                         // E_z vanishes on the wall node
                const cpx pe_up = j + 1 < ny ? uEz[j + 1] : Z;
                if (j > 0) sLx = uLx[j] - 0.25 * h * (ik(kx, pe) - (uBz[j] - uBz[j - 1]) * iAj) - 0.5 * h * up.kx_;
                sLy = uLy[j] - 0.25 * h * (ik(kx, uBz[j]) + (pe_up - pe) * iDj) - 0.5 * h * up.ky_;
                kRx[j] = sRx; kRy[j] = sRy; kLx[j] = sLx; kLy[j] = sLy;
            }
            __syncthreads();
            // 3. the rows of the two systems: E_z on the nodes 1..ny-1 (row 0 is the wall: E_z = 0), B_z on the
            // half-nodes 0..ny-1
            double aE = 0, bE = 1, cE = 0, aB = 0, bB = 1, cB = 0;
            cpx rE = Z, rB = Z;
            if (row) {
                if (j > 0) {
                    const cpx Qp = 0.5 * (-ik(kx, uRx[j] - uLx[j]) + ((uLy[j] - uRy[j]) - (uLy[j - 1] - uRy[j - 1])) * iAj);
                    const cpx SE = -ik(kx, sRx - sLx) + ((sLy - sRy) - (kLy[j - 1] - kRy[j - 1])) * iAj;
                    rE = pe - 0.5 * h * Qp - 0.25 * h * SE - h * up.kz_;
                    aE = j > 1 ? -cc * iAj * iDm : 0;
                    cE = j < ny - 1 ? -cc * iAj * iDj : 0;
                    bE = 1 + cc * kx2 + cc * iAj * (iDm + iDj);
                }
                const cpx fu = j + 1 < ny ? uRx[j + 1] + uLx[j + 1] : Z, f0 = uRx[j] + uLx[j];
                const cpx Cp = 0.5 * (ik(kx, uRy[j] + uLy[j]) - (fu - f0) * iDj);
                const cpx su = j + 1 < ny ? kRx[j + 1] + kLx[j + 1] : Z, s0 = sRx + sLx;
                const cpx SB = ik(kx, sRy + sLy) - (su - s0) * iDj;
                rB = uBz[j] - 0.5 * h * Cp - 0.25 * h * SB;
                const double al = j > 0 ? iAj : 0, au = j < ny - 1 ? iAp : 0;
                aB = -cc * iDj * al; cB = -cc * iDj * au;
                bB = 1 + cc * kx2 + cc * iDj * (al + au);
            }
            // parallel cyclic reduction of both systems
            for (int st = 1; st < ny; st <<= 1) {
                if (row) {
                    lo_E[j] = aE; dg_E[j] = bE; up_E[j] = cE; rhsE[j] = rE;
                    lo_B[j] = aB; dg_B[j] = bB; up_B[j] = cB; rhsB[j] = rB;
                }
                __syncthreads();
                if (row) {
                    const int m = j - st, p = j + st;
                    double fE = 0, gE = 0, fB = 0, gB = 0;
                    double naE = 0, ncE = 0, naB = 0, ncB = 0;
                    cpx dE = rE, dB = rB;
                    double nbE = bE, nbB = bB;
                    if (m >= 0) {
                        fE = aE / dg_E[m]; fB = aB / dg_B[m];
                        naE = -lo_E[m] * fE; naB = -lo_B[m] * fB;
                        nbE -= up_E[m] * fE; nbB -= up_B[m] * fB;
                        dE = dE - fE * rhsE[m]; dB = dB - fB * rhsB[m];
                    }
                    if (p < ny) {
                        gE = cE / dg_E[p]; gB = cB / dg_B[p];
                        ncE = -up_E[p] * gE; ncB = -up_B[p] * gB;
                        nbE -= lo_E[p] * gE; nbB -= lo_B[p] * gB;
                        dE = dE - gE * rhsE[p]; dB = dB - gB * rhsB[p];
                    }
                    aE = naE; cE = ncE; bE = nbE; rE = dE;
                    aB = naB; cB = ncB; bB = nbB; rB = dB;
                }
                __syncthreads();
            }
            if (row) {
                oEz = j == 0 ? Z : rE / bE;
                oBz = rB / bB;
                nwE[j] = oEz; nwB[j] = oBz;
            }
            __syncthreads();
            // 4. R and L
            if (row) {
                if (j > 0) {
                    const cpx bm = (oBz - nwB[j - 1]) * iAj;
                    oRx = sRx + D * (ik(kx, oEz) + bm);
                    oLx = sLx - 0.25 * h * (ik(kx, oEz) - bm);
                } else {
                    oRx = Z; oLx = Z;
                }
                const cpx ez_up = j + 1 < ny ? nwE[j + 1] : Z;
                const cpx bp = (ez_up - oEz) * iDj;
                oRy = sRy + D * (bp - ik(kx, oBz));
                oLy = sLy - 0.25 * h * (ik(kx, oBz) + bp);
            }
        }
        if (row) {
            A.Rx[o] = oRx; A.Ry[o] = oRy; A.Ez[o] = oEz; A.Bz[o] = oBz; A.Lx[o] = oLx; A.Ly[o] = oLy;
            uRx[j] = oRx; uRy[j] = oRy; uEz[j] = oEz; uBz[j] = oBz; uLx[j] = oLx; uLy[j] = oLy;
        }
        up = cur;                                                // this slice's lower plane is the next one's upper
        cur = nxt;
    }
}

// ---------------------------------------------------------------- sponge
// psi of the slice charge per (slice, k_x) line into PSI; U = R_x - R_bx, V = R_y - R_by
__global__ void k_sp_psi_fh(Geo g, const cpx* __restrict__ Rx, const cpx* __restrict__ Ry, const cpx* __restrict__ jz,
                            cpx* __restrict__ U, cpx* __restrict__ V, cpx* __restrict__ PSI, double g2, double opb) {
    const long nl = long(g.ns) * g.H;
    const long line = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (line >= nl) return;
    const int H = g.H, ny = g.ny, kxi = int(line % H), l = int(line / H), n = g.a + l;
    const long nk = g.nkh, o = long(l) * nk + kxi;
    const double* ia = g.iA; const double* id = g.iD;
    auto half = [&](int hk, long jo) -> cpx {           // half-cell plane hk = -1 .. ns+1 (no ghosts on one rank)
        if (hk < 0 || hk > g.ns) return C(0);
        return jz[long(hk) * nk + kxi + jo];
    };
    auto rho_at = [&](int dl, long jo) -> cpx {          // charge of slice n + dl at the y offset jo
        const int nn = n + dl;
        if (nn < 0 || nn > g.N - 1) return C(0);
        return g.wlo[nn] * half(l + dl, jo) + g.whi[nn] * half(l + dl + 1, jo);
    };
    const double hm = g.hcg[n + 1], hp = g.hcg[n + 2];
    const double cm = 2 / ((hm + hp) * hm), cp_ = 2 / ((hm + hp) * hp);
    for (int second = 0; second < 2; ++second) {         // T^-1 of the d_zeta^2 term, then of rho + that
        cpx dpv = C(0);
        for (int j = 1; j < ny; ++j) {
            const long jo = long(j) * H, k = o + jo;
            cpx r;
            if (!second) r = g2 * (cp_ * rho_at(1, jo) - (cm + cp_) * rho_at(0, jo) + cm * rho_at(-1, jo));
            else r = rho_at(0, jo) + PSI[k];
            const double lo = j > 1 ? -ia[j] * id[j - 1] : 0;
            dpv = (r - lo * dpv) * g.pid[long(j) * H + kxi];
            PSI[k] = dpv;
        }
        cpx next = C(0);
        for (int j = ny - 1; j >= 1; --j) {
            next = PSI[o + long(j) * H] - g.pcp[long(j) * H + kxi] * next;
            PSI[o + long(j) * H] = next;
        }
    }
    PSI[o] = C(0);
    const double kx = g.kxd[kxi];
    for (int j = 0; j < ny; ++j) {
        const long k = o + long(j) * H;
        const cpx pu = j + 1 < ny ? PSI[k + H] : C(0);
        const cpx bx = -opb * ikx(kx, PSI[k]), by = -opb * ((pu - PSI[k]) * id[j]);
        U[k] = Rx[k] - bx; V[k] = Ry[k] - by;
    }
}
// after the mask: R = (masked R - R_b) + R_b, R_x = 0 at the wall node
__global__ void k_sp_add_fh(Geo g, const cpx* __restrict__ U, const cpx* __restrict__ V, const cpx* __restrict__ PSI,
                            cpx* __restrict__ Rx, cpx* __restrict__ Ry, double opb) {
    const long n = long(g.ns) * g.nkh;
    for (long idx = long(blockIdx.x) * blockDim.x + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
        const long i = idx % g.nkh;
        const int j = int(i / g.H), kxi = int(i % g.H);
        const cpx pu = j + 1 < g.ny ? PSI[idx + g.H] : C(0);
        const cpx bx = -opb * ikx(g.kxd[kxi], PSI[idx]), by = -opb * ((pu - PSI[idx]) * g.iD[j]);
        Rx[idx] = j == 0 ? C(0) : U[idx] + bx;
        Ry[idx] = V[idx] + by;
    }
}

// ---------------------------------------------------------------- co-moving start field
// half-cell charges to the eigen-coefficients: E1[l][s][k_x] = sum_j evf[s][j] jz[l][j][k_x] (slot 0 stays 0)
__global__ void k_comoving_fh_proj(Geo g, const cpx* __restrict__ jz, cpx* __restrict__ E1) {
    const long n = long(g.ns + 1) * g.nkh;
    for (long idx = long(blockIdx.x) * blockDim.x + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
        const long i = idx % g.nkh, base = idx - i;
        const int s = int(i / g.H), kxi = int(i % g.H);
        cpx v = C(0);
        if (s > 0)
            for (int j = 1; j < g.ny; ++j) v = v + g.evf[long(s) * g.ny + j] * jz[base + long(j) * g.H + kxi];
        E1[idx] = v;
    }
}
// per (eigenvalue slot, k_x): the tridiagonal system of -(k_x^2 + mu_s + gamma^-2 d_zeta^2) psi = rho along zeta
__global__ void k_comoving_fh_thomas(Geo g, const cpx* __restrict__ E1, double* __restrict__ cpb, cpx* __restrict__ dpb,
                                     double beta, double gm2) {
    const long nk = g.nkh;
    const long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= nk) return;
    const int s = int(i / g.H), kxi = int(i % g.H);
    const double kx = g.kxd[kxi], ev = g.evl[s];
    double cprev = 0;
    cpx dprev = C(0);
    for (int l = 0; l < g.ns; ++l) {
        const long o = long(l) * nk + i;
        const int n = g.a + l;
        const double hm = g.hcg[n + 1], hp = g.hcg[n + 2];
        const double lo = -gm2 * 2 / ((hm + hp) * hm), up = -gm2 * 2 / ((hm + hp) * hp);
        const double dg = kx * kx + ev + gm2 * 2 / (hm * hp);
        if (s == 0 || dg == 0) { cpb[o] = 0; dpb[o] = C(0); continue; }
        const cpx rhs = (1 / beta) * (g.wlo[n] * E1[o] + g.whi[n] * E1[o + nk]);
        if (n == 0) { cprev = 0; dprev = C(0); }
        const double den = dg - lo * cprev;
        const double cpv = up / den;
        const cpx dpv = (rhs - lo * dprev) / den;
        cpb[o] = cpv; dpb[o] = dpv;
        cprev = cpv; dprev = dpv;
    }
    cpx next = C(0);
    for (int l = g.ns - 1; l >= 0; --l) {
        const long o = long(l) * nk + i;
        next = dpb[o] - cpb[o] * next;
        dpb[o] = next;
    }
}
// back to the nodes: psi[l][j][k_x] = sum_s evb[j][s] psi_s (psi = 0 at the wall node)
__global__ void k_comoving_fh_back(Geo g, const cpx* __restrict__ psis, cpx* __restrict__ psi) {
    const long n = long(g.ns) * g.nkh;
    for (long idx = long(blockIdx.x) * blockDim.x + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
        const long i = idx % g.nkh, base = idx - i;
        const int j = int(i / g.H), kxi = int(i % g.H);
        cpx v = C(0);
        if (j > 0)
            for (int s = 1; s < g.ny; ++s) v = v + g.evb[long(j) * g.ny + s] * psis[base + long(s) * g.H + kxi];
        psi[idx] = v;
    }
}
// R = -(1 + beta) E_perp of psi, E_z = B_z = 0
__global__ void k_comoving_fh_field(Geo g, const cpx* __restrict__ psi, cpx* __restrict__ Rx, cpx* __restrict__ Ry,
                                    cpx* __restrict__ Ez, cpx* __restrict__ Bz, double beta) {
    const long n = long(g.ns) * g.nkh;
    for (long idx = long(blockIdx.x) * blockDim.x + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
        const long i = idx % g.nkh;
        const int j = int(i / g.H), kxi = int(i % g.H);
        Rx[idx] = -(1 + beta) * ikx(g.kxd[kxi], psi[idx]);
        const cpx up = j + 1 < g.ny ? psi[idx + g.H] : C(0);
        Ry[idx] = -(1 + beta) * ((up - psi[idx]) * g.iD[j]);
        Ez[idx] = C(0); Bz[idx] = C(0);
    }
}

// ---------------------------------------------------------------- launchers
static unsigned ew_blocks(long n) {
    long b = (n + 255) / 256;
    return unsigned(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}

void launch_deposit_fh(Ctx& c) {
    c.jw.zero(c.stream);
    if (c.np == 0 && !c.sharded()) return;
    const int tok = c.prof_begin("deposit");
    const double* scale = launch_deposit_scale(c, c.ia_max);
    if (c.np > 0) {
        k_deposit_fh<<<unsigned((c.np + 255) / 256), 256, 0, c.stream>>>(c.parts, c.perm.p, c.np, c.geo(), c.jw.p, scale);
        c.check_launch("k_deposit_fh");
    }
    launch_deposit_finish(c);
    c.prof_end(tok);
}
void launch_cur_fft_fh(Ctx& c, bool keep0) {
    launch_cur_rows_to_jk(c);
    const long nl = long(c.ns + 1) * c.H;
    const int tok = c.prof_begin("cur_lines");
    k_cur_lines_fh<<<unsigned((nl + 127) / 128), 128, 0, c.stream>>>(c.geo(), c.jkx.p, c.jky.p, c.jkz.p, c.P.k_filter ? 1 : 0,
                                                                      keep0 ? 1 : 0);
    c.check_launch("k_cur_lines_fh");
    c.prof_end(tok);
}
static void march_lines(Ctx& c, double D, int n_top, int n_bot, const char* name) {
    if (c.ny > LINE_MAX_NY) throw Error(G3D_ERR_ARG, "free-hand march: ny above " + std::to_string(LINE_MAX_NY));
    const size_t smem = line_smem(c.ny);
    const LineArrays A{c.Rx.p, c.Ry.p, c.Ez.p, c.Bz.p, c.Lx.p, c.Ly.p, c.j0x.p, c.j0y.p, c.jkx.p, c.jky.p, c.jkz.p};
    const int threads = (c.ny + 31) / 32 * 32;
    const int tok = c.prof_begin(name);
    if (threads <= 256) {         // up to 255 registers a thread
        smem_attr(reinterpret_cast<const void*>(k_march_lines<256>), line_smem(256));
        k_march_lines<256><<<unsigned(c.H), unsigned(threads), smem, c.stream>>>(c.geo(), A, D, n_top, n_bot);
    } else {
        smem_attr(reinterpret_cast<const void*>(k_march_lines<LINE_MAX_NY>), line_smem(LINE_MAX_NY));
        k_march_lines<LINE_MAX_NY><<<unsigned(c.H), unsigned(threads), smem, c.stream>>>(c.geo(), A, D, n_top, n_bot);
    }
    c.check_launch("k_march_lines");
    c.prof_end(tok);
}
void launch_march_fh(Ctx& c, double D) { march_lines(c, D, c.b - 1, c.a, "march"); }
// the march of the one slice n (the streaming-plasma march, Simulation::march_slice, src/sim_plasma.cpp:186-196)
void launch_march_slice_fh(Ctx& c, double D, int n) { march_lines(c, D, n, n, "march_slice"); }
// the lines of the streaming spectra: T0..T2 (the x spectra of the rows of j_x, j_y, j_z) -> out (3 half planes)
void launch_ss_lines_fh(Ctx& c, const cpx* T3, cpx* out3, double a2) {
    if (c.ny > LINE_MAX_NY) throw Error(G3D_ERR_ARG, "free-hand streaming spectra: ny above " + std::to_string(LINE_MAX_NY));
    const size_t smem = size_t(c.ny) * (6 * sizeof(cpx) + 6 * sizeof(double));
    const int threads = (c.ny + 31) / 32 * 32;
    if (threads <= 256) {
        smem_attr(reinterpret_cast<const void*>(k_ss_lines_fh<256>), size_t(256) * (6 * sizeof(cpx) + 6 * sizeof(double)));
        k_ss_lines_fh<256><<<unsigned(c.H), unsigned(threads), smem, c.stream>>>(c.geo(), T3, out3, c.P.k_filter ? 1 : 0, a2);
    } else {
        smem_attr(reinterpret_cast<const void*>(k_ss_lines_fh<LINE_MAX_NY>),
                  size_t(LINE_MAX_NY) * (6 * sizeof(cpx) + 6 * sizeof(double)));
        k_ss_lines_fh<LINE_MAX_NY><<<unsigned(c.H), unsigned(threads), smem, c.stream>>>(c.geo(), T3, out3, c.P.k_filter ? 1 : 0, a2);
    }
    c.check_launch("k_ss_lines_fh");
}
void launch_sponge_fh(Ctx& c) {
    const long nl = long(c.ns) * c.H;
    const double opb = 1 + c.beta_b;
    int tok = c.prof_begin("sponge_psi");
    k_sp_psi_fh<<<unsigned((nl + 127) / 128), 128, 0, c.stream>>>(c.geo(), c.Rx.p, c.Ry.p, c.jkz.p, c.W[0].p, c.W[1].p,
                                                                   c.W[3].p, c.gm2_b, opb);
    c.check_launch("k_sp_psi_fh");
    c.prof_end(tok);
    launch_sp_rows(c);
    tok = c.prof_begin("sponge_add");
    k_sp_add_fh<<<ew_blocks(long(c.ns) * c.nkh), 256, 0, c.stream>>>(c.geo(), c.W[0].p, c.W[1].p, c.W[3].p, c.Rx.p, c.Ry.p, opb);
    c.check_launch("k_sp_add_fh");
    c.prof_end(tok);
}
// scratch: W0 the eigen-coefficients of the charge, W3 psi_s, W2 psi on the nodes (W4, W5 hold the copies of R
// that relax_start_field makes around this call)
void launch_comoving_fh(Ctx& c, double beta, double gm2) {
    const int tok = c.prof_begin("comoving");
    const Geo g = c.geo();
    k_comoving_fh_proj<<<ew_blocks(long(c.ns + 1) * c.nkh), 256, 0, c.stream>>>(g, c.jkz.p, c.W[0].p);
    c.check_launch("k_comoving_fh_proj");
    k_comoving_fh_thomas<<<unsigned((c.nkh + 127) / 128), 128, 0, c.stream>>>(g, c.W[0].p, c.rscratch.p, c.W[3].p, beta, gm2);
    c.check_launch("k_comoving_fh_thomas");
    k_comoving_fh_back<<<ew_blocks(long(c.ns) * c.nkh), 256, 0, c.stream>>>(g, c.W[3].p, c.W[2].p);
    c.check_launch("k_comoving_fh_back");
    k_comoving_fh_field<<<ew_blocks(long(c.ns) * c.nkh), 256, 0, c.stream>>>(g, c.W[2].p, c.Rx.p, c.Ry.p, c.Ez.p, c.Bz.p, beta);
    c.check_launch("k_comoving_fh_field");
    c.prof_end(tok);
}

}  // namespace g3d
