// Host orchestration of the streaming plasma (one rank, Fourier y): set-up, the fresh plasma of a step, the
// march half-cell by half-cell with its passes, prediction and correction, the freed electrons, trapping and
// restreaming (src/sim_plasma.cpp:21-491, src/sim_ions.cpp:68-87, src/ionization.cpp:28-53), and the grid
// lasers of the start field (src/sim_fields.cpp:321-374).
#include <cstdlib>
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include "g3d_plasma.hpp"

namespace g3d {

namespace {
constexpr double c_SI = 299792458.0, e_SI = 1.602176634e-19, me_SI = 9.1093837015e-31;
constexpr double U_H_EV = 13.605693122994, E_ATOMIC_VM = 5.14220674763e11, OMEGA_ATOMIC = 4.1341373335e16;
}  // namespace

void StrmBuf::alloc(long n, cudaStream_t s) {
    cap = n;
    d.alloc(size_t(n) * 10, s);
    i.alloc(size_t(n) * 2, s);
    u.alloc(size_t(n), s);
    double** cols[10] = {&v.x, &v.y, &v.zeta, &v.px, &v.py, &v.pz, &v.w, &v.z, &v.q, &v.qm};
    for (int k = 0; k < 10; ++k) *cols[k] = d.p + size_t(k) * n;
    v.alive = i.p; v.sp = i.p + n;
    v.id = u.p;
}

PlasmaPtrs PlasmaState::ptrs(const Ctx& c) const {
    PlasmaPtrs p;
    p.nkh = c.nkh;
    if (c.mixed) { p.jkx = c.mx.jkx.p; p.jky = c.mx.jky.p; p.jkz = c.mx.jkz.p; }
    else { p.jkx = c.jkx.p; p.jky = c.jky.p; p.jkz = c.jkz.p; }
    p.js0x = js0x.p; p.js0y = js0y.p; p.js0z = js0z.p;
    p.jsn = jsn.p; p.sin_ = jsin.p; p.si0 = jsi0.p; p.pin = jpred.p; p.tmp = jtmp.p; p.dl = dlt.p;
    return p;
}

// ---------------------------------------------------------------- ADK tables (src/ionization.cpp:28-53)
// ln of omega_a C^2 (U/2U_H) (2 (U/U_H)^{3/2} E_a)^{2n*-1}, the power 2n*-1 and the exponent factor
// -(2/3)(U/U_H)^{3/2} E_a of the ADK rate (s-states, l* = n* - 1, m = 0) in SI units
static void adk_coefficients(double U_eV, int Zafter, double& logpre, double& power, double& expo) {
    const double x = U_eV / U_H_EV;
    const double nstar = Zafter / std::sqrt(x);
    const double logC2 = 2.0 * nstar * std::log(2.0) - std::log(nstar) - std::lgamma(nstar + 1.0) - std::lgamma(nstar);
    power = 2.0 * nstar - 1.0;
    logpre = std::log(OMEGA_ATOMIC) + logC2 + std::log(0.5 * x) + power * std::log(2.0 * std::pow(x, 1.5) * E_ATOMIC_VM);
    expo = -(2.0 / 3.0) * std::pow(x, 1.5) * E_ATOMIC_VM;
}
static double adk_raw(const AdkDev& L, double E) {
    E = std::min(E, L.Epeak);
    return E > 0 ? std::exp(L.logpre - L.power * std::log(E) + L.expo / E) : 0.0;
}
// levels Z0 .. Zmax-1 in code units; Emin: below it a level is not ionized within T with probability > 1e-10
static std::vector<AdkDev> adk_levels(const std::vector<double>& ip_eV, int Z0, int Zmax, double E0_SI, double omega0, double T) {
    std::vector<AdkDev> lev(size_t(std::max(Zmax, 0)), AdkDev{0, 0, 0, 1e300, 1e300});
    for (int k = Z0; k < Zmax; ++k) {
        AdkDev& L = lev[size_t(k)];
        double logpre, power, expo;
        adk_coefficients(ip_eV[size_t(k)], k + 1, logpre, power, expo);
        L.power = power;
        L.logpre = logpre - std::log(omega0) - power * std::log(E0_SI);
        L.expo = expo / E0_SI;
        L.Epeak = power > 0 ? -L.expo / power : 1e300;
        double lo = 1e-12, hi = std::min(L.Epeak, 1e6);
        if (adk_raw(L, hi) * T < 1e-10) L.Emin = hi;
        else {
            for (int it = 0; it < 200; ++it) {
                const double mid = std::sqrt(lo * hi);
                (adk_raw(L, mid) * T < 1e-10 ? lo : hi) = mid;
            }
            L.Emin = lo;
        }
    }
    return lev;
}

// ---------------------------------------------------------------- set-up (setup_plasma, setup_ions)
void set_plasma(Ctx& c, const g3d_plasma& P, const g3d_ion* ions, int nions) {
    if (P.ppc_x < 1 || P.ppc_y < 1) throw Error(G3D_ERR_ARG, "plasma: ppc_x, ppc_y must be >= 1");
    if (P.iterations < 1) throw Error(G3D_ERR_ARG, "plasma: iterations must be >= 1");
    if (!(P.vz_min > 0 && P.vz_min < P.vz_beam && P.vz_beam < 1)) throw Error(G3D_ERR_ARG, "plasma: need 0 < vz_min < vz_beam < 1");
    if (!(P.trap_advance >= 1)) throw Error(G3D_ERR_ARG, "plasma: trap_advance must be >= 1");
    if (!(P.n0 > 0)) throw Error(G3D_ERR_ARG, "plasma: n0 must be positive");
    auto pl = std::make_unique<PlasmaState>();
    pl->cfg = P;
    if (P.n_z > 0) {
        pl->zpts.assign(P.z_points, P.z_points + P.n_z);
        pl->zvals.assign(P.z_values, P.z_values + P.n_z);
    }
    pl->cfg.z_points = nullptr; pl->cfg.z_values = nullptr;
    pl->box_mean = P.box_mean != 0;
    for (int k = 0; k < nions; ++k) {
        const g3d_ion& I = ions[k];
        IonSpec s;
        s.mass = I.mass; s.atoms = I.atoms; s.Z0 = I.Z0; s.Zmax = I.Zmax; s.mobile = I.mobile; s.ionization = I.ionization;
        if (I.n_ip > 0) s.ip_eV.assign(I.ip_eV, I.ip_eV + I.n_ip);
        if (s.ionization && (int(s.ip_eV.size()) < s.Zmax || s.Zmax <= s.Z0))
            throw Error(G3D_ERR_ARG, "ion: ionization needs Zmax > Z0 and Zmax ionization energies");
        pl->ions.push_back(s);
        if (s.loaded()) pl->ion_lines = true;
    }
    cudaStream_t s = c.stream;
    const size_t ph = size_t(c.nkh);
    for (DevBuf<cpx>* b : {&pl->js0x, &pl->js0y, &pl->js0z}) b->alloc(size_t(c.ns + 1) * ph, s);
    pl->jsr.alloc(size_t(5) * c.nk, s);
    pl->jsrf.alloc(size_t(5) * c.nk, s);               // FP32: three planes, or on the Fourier y grid (jx, jy, jz, 0) per point
    if (c.yf || c.f32s) pl->fmid.alloc(size_t(6) * c.nk, s);      // 6 doubles or 8 floats per point
    pl->rhol.alloc(size_t(pl->ion_lines ? 2 : 1) * size_t(c.N) * size_t(c.nx + c.ny), s);
    pl->stepv.alloc(1, s);
    for (DevBuf<cpx>* b : {&pl->jsn, &pl->jsin, &pl->jpred, &pl->jtmp, &pl->jsi0, &pl->dlt, &pl->tsp}) b->alloc(3 * ph, s);
    pl->bk.alloc(4 * ph, s);
    pl->nstrm_dev.alloc(1, s);
    pl->sdev.alloc(2, s);
    pl->bcnt.alloc(1, s);
    pl->tally.alloc(1, s);
    pl->ucount.alloc(1, s);
    pl->flags.alloc(1, s);
    // ion tables on the device (setup_ions, src/sim_ions.cpp:68-87)
    const double Lu = c.P.lambda0 / (2 * M_PI), omega0 = c_SI / Lu, E0 = me_SI * c_SI * omega0 / e_SI;
    const double Lwin = c.zeta.back() - c.zeta.front();
    std::vector<IonDevC> iv;
    std::vector<AdkDev> lev;
    for (const auto& sp : pl->ions) {
        IonDevC d{};
        d.mass = sp.mass; d.mobile = sp.mobile; d.ionizing = sp.ionization; d.Zmax = sp.Zmax; d.off = int(lev.size()); d.Emin = 1e300;
        if (sp.ionization) pl->any_ionizing = true;
        if (sp.ionization) {
            const std::vector<AdkDev> L = adk_levels(sp.ip_eV, sp.Z0, sp.Zmax, E0, omega0, 2 * Lwin);
            for (int k = sp.Z0; k < sp.Zmax; ++k) d.Emin = std::min(d.Emin, L[size_t(k)].Emin);
            lev.insert(lev.end(), L.begin(), L.end());
        }
        iv.push_back(d);
    }
    if (!iv.empty()) pl->ion_dev.upload(iv, s);
    if (!lev.empty()) pl->adk_dev.upload(lev, s);
    G3D_CUDA(cudaStreamSynchronize(s));
    c.pl = std::move(pl);
}

// n = n0 f(z) g(r) for r < r_max (Config::plasma_density, src/sim_config.cpp:49-66; no density function): f(z),
// the longitudinal profile, here; g(r) and the cut at r_max per lattice point on the device (lattice_point).
static double density_zfactor(const PlasmaState& P, double z) {
    double f = 1;
    if (!P.zpts.empty()) {
        if (z <= P.zpts.front()) f = P.zvals.front();
        else if (z >= P.zpts.back()) f = P.zvals.back();
        else {
            size_t k = 1;
            while (P.zpts[k] < z) ++k;
            const double t = (z - P.zpts[k - 1]) / (P.zpts[k] - P.zpts[k - 1]);
            f = (1 - t) * P.zvals[k - 1] + t * P.zvals[k];
        }
    }
    return f;
}

// Fresh plasma at the front of the window in the reference's order (load_plasma, src/sim_plasma.cpp:43-90):
// rows j, cells i, sub-cells b2, a2; the electron, then the loaded ions of every species; then the particles
// that join the march at their zeta. The lattice is built on the device (k_lattice_flags / k_lattice_fill: the
// points of positive density counted, their particles written at the running count, ids in list order); the
// joining particles are the last march's slow trapped ones, kept on the device, then the beam particles that
// slowed down, from the host (the order of the reference's list).
static void load_plasma(Ctx& c, double s0, double s1) {
    PlasmaState& P = *c.pl;
    const double zmid = 0.5 * (s0 + s1), Delta = s1 - s0;
    LatticeArgs a{};
    a.nx = c.nx; a.px = P.cfg.ppc_x; a.py = P.cfg.ppc_y;
    a.j0 = c.yf ? 0 : 1;                                 // free-hand y: no plasma in the cells at the walls
    const long nrows = c.yf ? c.ny : c.ny - 2;
    a.electrons = P.cfg.free_electrons ? 1 : 0;
    a.dx = c.dx; a.dy = c.dy; a.X0 = c.X0; a.Y0 = c.Y0; a.Delta = Delta;
    a.zf = c.zeta[size_t(c.N - 1)]; a.s0 = s0;
    a.yn = c.yf ? nullptr : c.yn.p;
    a.f = density_zfactor(P, zmid); a.n0 = P.cfg.n0;
    a.rmax2 = P.cfg.r_max * P.cfg.r_max;
    a.parabolic = P.cfg.parabolic ? 1 : 0;
    a.depth = P.cfg.channel_depth; a.rc2 = P.cfg.r_channel * P.cfg.r_channel;
    a.id0 = uint64_t(c.istep + 1) << 32;
    long ion_cap = 0;                                    // freed-electron capacity per point (ionizing ions)
    for (size_t k = 0; k < P.ions.size(); ++k) {
        const IonSpec& is = P.ions[k];
        if (!is.loaded()) continue;
        if (a.nion == LAT_MAXION) throw Error(G3D_ERR_ARG, "more than 8 loaded ion species");
        a.ion_atoms[a.nion] = is.atoms; a.ion_q[a.nion] = is.Z0; a.ion_qm[a.nion] = is.Z0 / is.mass;
        a.ion_sp[a.nion] = SP_ION + int(k);
        ++a.nion;
        if (is.ionization) ion_cap += is.Zmax - is.Z0;
    }
    a.m = a.electrons + a.nion;
    const long npts = nrows > 0 ? nrows * c.nx * a.px * a.py : 0;
    const long pts = (npts > 0 && a.m > 0) ? launch_lattice_count(c, a, npts) : 0;
    const long fresh = pts * a.m;
    long cap = pts * ion_cap + launch_join_cap(c);
    for (const auto& p : P.joining)
        if (p.sp >= SP_ION && p.sp < SP_FREED && P.ions[size_t(p.sp - SP_ION)].ionization)
            cap += P.ions[size_t(p.sp - SP_ION)].Zmax - std::lround(p.q);
    // G3D_BORN_CAPACITY_LIMIT (environment, > 0): a smaller list of freed electrons than the ionization can fill, so
    // that the overflow check (device flag -> G3D_ERR_CAPACITY) can be exercised; every write stays inside the list
    if (const char* lim = std::getenv("G3D_BORN_CAPACITY_LIMIT")) {
        const long l = std::atol(lim);
        if (l > 0 && l < cap) cap = l;
    }
    const long jd = P.njb;                               // joining on the device (the last march's slow trapped)
    const long n = fresh + jd + long(P.joining.size());
    P.fresh_last = fresh;
    P.nstrm = n;
    P.born_cap = cap;
    const long need = n + cap;
    if (P.s.cap < need) {             // doubled: the list grows by the joining particles step after step
        const long nn = 2 * need + 64;
        P.s.alloc(nn, c.stream);
    }
    if (cap > 0 && P.bn.cap < cap) P.bn.alloc(cap, c.stream);
    P.strm = P.s.v;
    P.born = P.bn.v;
    P.sdh[0] = P.strm; P.sdh[1] = P.born;
    G3D_CUDA(cudaMemcpyAsync(P.sdev.p, P.sdh, sizeof(P.sdh), cudaMemcpyHostToDevice, c.stream));
    if (fresh) launch_lattice_fill(c, a, npts, P.strm);
    if (jd) {                                            // the device's joining particles after the lattice
        const StrmDev& J = P.jb.v;
        const double* src[10] = {J.x, J.y, J.zeta, J.px, J.py, J.pz, J.w, J.z, J.q, J.qm};
        double* dst[10] = {P.strm.x, P.strm.y, P.strm.zeta, P.strm.px, P.strm.py, P.strm.pz, P.strm.w, P.strm.z, P.strm.q, P.strm.qm};
        for (int m = 0; m < 10; ++m)
            G3D_CUDA(cudaMemcpyAsync(dst[m] + fresh, src[m], size_t(jd) * 8, cudaMemcpyDeviceToDevice, c.stream));
        G3D_CUDA(cudaMemcpyAsync(P.strm.alive + fresh, J.alive, size_t(jd) * 4, cudaMemcpyDeviceToDevice, c.stream));
        G3D_CUDA(cudaMemcpyAsync(P.strm.sp + fresh, J.sp, size_t(jd) * 4, cudaMemcpyDeviceToDevice, c.stream));
        G3D_CUDA(cudaMemcpyAsync(P.strm.id + fresh, J.id, size_t(jd) * 8, cudaMemcpyDeviceToDevice, c.stream));
        P.njb = 0;
    }
    const long nj = long(P.joining.size()), jo = fresh + jd;
    if (nj) {                                            // then the host's (restreamed beam particles), as columns
        std::vector<double> hd(size_t(nj) * 10);
        std::vector<int32_t> hi(size_t(nj) * 2);
        std::vector<uint64_t> hu(static_cast<size_t>(nj));
        for (long k = 0; k < nj; ++k) {
            const g3d_particle& p = P.joining[size_t(k)];
            const double vals[10] = {p.x, p.y, p.zeta, p.px, p.py, p.pz, p.w, p.z, p.q, p.qm};
            for (int m = 0; m < 10; ++m) hd[size_t(m) * nj + k] = vals[m];
            hi[size_t(k)] = 6; hi[size_t(nj) + k] = p.sp; hu[size_t(k)] = p.id;
        }
        double* cols[10] = {P.strm.x, P.strm.y, P.strm.zeta, P.strm.px, P.strm.py, P.strm.pz, P.strm.w, P.strm.z, P.strm.q, P.strm.qm};
        for (int m = 0; m < 10; ++m)
            G3D_CUDA(cudaMemcpyAsync(cols[m] + jo, hd.data() + size_t(m) * nj, size_t(nj) * 8, cudaMemcpyHostToDevice, c.stream));
        G3D_CUDA(cudaMemcpyAsync(P.strm.alive + jo, hi.data(), size_t(nj) * 4, cudaMemcpyHostToDevice, c.stream));
        G3D_CUDA(cudaMemcpyAsync(P.strm.sp + jo, hi.data() + nj, size_t(nj) * 4, cudaMemcpyHostToDevice, c.stream));
        G3D_CUDA(cudaMemcpyAsync(P.strm.id + jo, hu.data(), size_t(nj) * 8, cudaMemcpyHostToDevice, c.stream));
    }
    P.joining.clear();
    G3D_CUDA(cudaMemcpyAsync(P.nstrm_dev.p, &P.nstrm, sizeof(long), cudaMemcpyHostToDevice, c.stream));
    G3D_CUDA(cudaMemsetAsync(P.flags.p, 0, sizeof(int), c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
}

// The streaming particles back on the host (the reference's `strm` after a march).
// n streaming particles of a device list as host records
static std::vector<g3d_particle> records_of(Ctx& c, const StrmDev& S, long n) {
    std::vector<g3d_particle> out(static_cast<size_t>(n));
    if (!n) return out;
    std::vector<double> hd(size_t(n) * 10);
    std::vector<int32_t> hi(size_t(n) * 2);
    std::vector<uint64_t> hu(static_cast<size_t>(n));
    const double* cols[10] = {S.x, S.y, S.zeta, S.px, S.py, S.pz, S.w, S.z, S.q, S.qm};
    for (int m = 0; m < 10; ++m)
        G3D_CUDA(cudaMemcpyAsync(hd.data() + size_t(m) * n, cols[m], size_t(n) * 8, cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaMemcpyAsync(hi.data(), S.alive, size_t(n) * 4, cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaMemcpyAsync(hi.data() + n, S.sp, size_t(n) * 4, cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaMemcpyAsync(hu.data(), S.id, size_t(n) * 8, cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
    for (long k = 0; k < n; ++k) {
        g3d_particle& p = out[size_t(k)];
        double* dst[10] = {&p.x, &p.y, &p.zeta, &p.px, &p.py, &p.pz, &p.w, &p.z, &p.q, &p.qm};
        for (int m = 0; m < 10; ++m) *dst[m] = hd[size_t(m) * n + k];
        p.alive = hi[size_t(k)]; p.sp = hi[size_t(n) + k]; p.id = hu[size_t(k)];
    }
    return out;
}

// The start of a run (g3d_init): the streaming current of level s0 is zero and no particle waits to join the march, as
// in a new Simulation (src/sim_setup.cpp), also when the context ran before.
void reset_plasma_march(Ctx& c) {
    PlasmaState& P = *c.pl;
    for (DevBuf<cpx>* b : {&P.js0x, &P.js0y, &P.js0z}) G3D_CUDA(cudaMemsetAsync(b->p, 0, b->bytes(), c.stream));
    P.njb = 0;
    P.joining.clear();
}

std::vector<g3d_particle> get_streaming(Ctx& c) {
    PlasmaState& P = *c.pl;
    long n = 0;
    G3D_CUDA(cudaMemcpyAsync(&n, P.nstrm_dev.p, sizeof(long), cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
    return records_of(c, P.strm, n);
}

// The particles that join the next march, in the order the next march appends them (the last march's slow trapped
// ones kept on the device, then those from the host): the reference's joining list of a checkpoint.
std::vector<g3d_particle> get_joining(Ctx& c) {
    PlasmaState& P = *c.pl;
    std::vector<g3d_particle> out = records_of(c, P.jb.v, P.njb);
    out.insert(out.end(), P.joining.begin(), P.joining.end());
    return out;
}
// A checkpoint's joining list: all of it joins from the host
void set_joining(Ctx& c, const std::vector<g3d_particle>& v) {
    PlasmaState& P = *c.pl;
    P.njb = 0;
    P.joining = v;
}
void get_plasma_counters(const Ctx& c, long& trapped, long& restreamed) {
    trapped = c.pl ? c.pl->trapped_total : 0;
    restreamed = c.pl ? c.pl->restreamed_total : 0;
}
void set_plasma_counters(Ctx& c, long trapped, long restreamed) {
    if (!c.pl) return;
    c.pl->trapped_total = trapped;
    c.pl->restreamed_total = restreamed;
}
// the streaming current of level s0 (ns + 1 half-cell planes) in the reference's full layout, and back
std::vector<cpx> get_js0(Ctx& c, int comp) {
    PlasmaState& P = *c.pl;
    const DevBuf<cpx>& b = comp == 0 ? P.js0x : comp == 1 ? P.js0y : P.js0z;
    const long planes = long(c.ns + 1);
    DevBuf<cpx> full;
    full.alloc(size_t(planes) * c.nk, c.stream);
    launch_half_to_full(c, b.p, full.p, planes);
    std::vector<cpx> v(size_t(planes) * c.nk);
    G3D_CUDA(cudaMemcpyAsync(v.data(), full.p, v.size() * sizeof(cpx), cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
    return v;
}
void set_js0(Ctx& c, int comp, const std::vector<cpx>& v) {
    PlasmaState& P = *c.pl;
    DevBuf<cpx>& b = comp == 0 ? P.js0x : comp == 1 ? P.js0y : P.js0z;
    const long planes = long(c.ns + 1);
    if (v.size() != size_t(planes) * c.nk) throw Error(G3D_ERR_IO, "checkpoint: streaming current of another grid");
    DevBuf<cpx> full;
    full.alloc(v.size(), c.stream);
    G3D_CUDA(cudaMemcpyAsync(full.p, v.data(), v.size() * sizeof(cpx), cudaMemcpyHostToDevice, c.stream));
    launch_full_to_half(c, full.p, b.p, planes);
    G3D_CUDA(cudaStreamSynchronize(c.stream));
}

// The trapped streaming particles that join the beam (P.tr after launch_trapped_split, n of them) on the host.
static std::vector<g3d_particle> fast_trapped(Ctx& c, long n) {
    PlasmaState& P = *c.pl;
    std::vector<g3d_particle> out(static_cast<size_t>(n));
    if (!n) return out;
    const StrmDev& T = P.tr.v;
    std::vector<double> hd(size_t(n) * 10);
    std::vector<int32_t> hi(size_t(n) * 2);
    std::vector<uint64_t> hu(static_cast<size_t>(n));
    const double* cols[10] = {T.x, T.y, T.zeta, T.px, T.py, T.pz, T.w, T.z, T.q, T.qm};
    for (int m = 0; m < 10; ++m)
        G3D_CUDA(cudaMemcpyAsync(hd.data() + size_t(m) * n, cols[m], size_t(n) * 8, cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaMemcpyAsync(hi.data(), T.alive, size_t(n) * 4, cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaMemcpyAsync(hi.data() + n, T.sp, size_t(n) * 4, cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaMemcpyAsync(hu.data(), T.id, size_t(n) * 8, cudaMemcpyDeviceToHost, c.stream));
    G3D_CUDA(cudaStreamSynchronize(c.stream));
    for (long k = 0; k < n; ++k) {
        g3d_particle& p = out[size_t(k)];
        double* dst[10] = {&p.x, &p.y, &p.zeta, &p.px, &p.py, &p.pz, &p.w, &p.z, &p.q, &p.qm};
        for (int m = 0; m < 10; ++m) *dst[m] = hd[size_t(m) * n + k];
        p.alive = hi[size_t(k)]; p.sp = hi[size_t(n) + k]; p.id = hu[size_t(k)];
    }
    return out;
}

// ---------------------------------------------------------------- the march of a step with plasma
static uint64_t mix64h(uint64_t z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// E and B of slice l; Fourier y: with the midpoint fields of slice `target` (l for the next pass of half-cell l,
// l - 1 for the first pass of half-cell l - 1, -1: none) for the streaming gather
static void real_fields_slice(Ctx& c, int l, int target = -1, bool cols = true, long rec_slot = -1) {
    FmidOut fm;
    if (rec_slot >= 0) {                              // the adjoint's record of the slice (exact fields)
        fm.rec_f = &c.pl->recd.p->f;
        fm.rec_off = 6 * long(c.nk) * rec_slot;
    }
    if (target >= c.a && (c.yf || c.f32s) && c.pl->fmid.p) {   // free-hand y: the mixed form's FP32 gather only
        fm.out = c.pl->fmid.p;
        fm.other = (target == l ? l + 1 : l - 1) - c.a;
        fm.f32 = c.f32s ? 1 : 0;
        fm.fh = c.yf ? 0 : 1;
    }
    if (!c.yf) { launch_real_fields_slice_fh(c, l, fm); return; }
    if (c.mixed) launch_real_fields_slice_f(c, l, fm, cols);
    else launch_real_fields_slice(c, l, fm, cols);
}

void march_plasma(Ctx& c, double s0, double s1) {
    PlasmaState& P = *c.pl;
    const double Delta = s1 - s0, D = 0.5 * Delta;
    const int N = c.N;
    const int nhi = N - 2;
    load_plasma(c, s0, s1);
    const bool extrap = P.cfg.predictor_extrapolate != 0;
    std::vector<double> cen(size_t(N - 1));
    for (int m = 0; m < N - 1; ++m) cen[size_t(m)] = 0.5 * (c.zeta[size_t(m)] + c.zeta[size_t(m + 1)]);
    // the values that change from step to step go to the device; the captured loop reads them there
    // the box column and row through the axis (src/sim_plasma.cpp:364-366)
    const int i0 = ((int(std::lround(-c.X0 / c.dx)) % c.nx) + c.nx) % c.nx;
    const int j0 = c.yf ? ((int(std::lround(-c.Y0 / c.dy)) % c.ny) + c.ny) % c.ny : c.ny / 2;
    const StepVals stv{s1, s1 + (P.cfg.trap_advance - 1) * Delta, c.X0, c.Y0,
                       mix64h(P.cfg.seed * 0x9E3779B97F4A7C15ULL + uint64_t(c.istep)), i0, j0};   // ion_key_step
    G3D_CUDA(cudaMemcpyAsync(P.stepv.p, &stv, sizeof(StepVals), cudaMemcpyHostToDevice, c.stream));
    const bool ionz = P.born_cap > 0;
    const int passes = P.cfg.iterations;
    // The slice loop is some 20 launches per half-cell (about 41,000 for 2,048 slices and two passes). Launched
    // one by one, the host's launch rate would bound the march; as one CUDA graph they run back to back. The
    // graph is captured once and launched every step; it is captured again only when something it holds by value
    // changes (a buffer of the window moved, the capacity of the freed-electron list, the step length). The
    // streaming and freed-electron lists are reached through a descriptor on the device, so they may move. While per-kernel events
    // are recorded the loop is launched directly.
    uint64_t key = 1469598103934665603ULL;
    auto mixk = [&](uint64_t v) { key = (key ^ v) * 1099511628211ULL; };
    auto ptr = [](const void* q) { return uint64_t(reinterpret_cast<uintptr_t>(q)); };
    const PlasmaPtrs pp = P.ptrs(c);
    const bool rec = P.rec_on && P.rec_step && P.rec_step(P.nstrm, P.fresh_last);   // the adjoint's record of this march
    // the record written by the kernels that hold the values (the exact streaming variant and the exact midpoint rows),
    // else by copy kernels of its own
    const bool rec_fourier = c.yf && (c.mixed || c.Fd.p);        // the exact FP64 forward or the mixed one
    const bool rec_x = rec && rec_fourier && !P.any_ionizing && !c.laser.on, rec_fld = rec && rec_fourier;
    mixk(ptr(c.F.p)); mixk(ptr(c.Fd.p)); mixk(uint64_t(rec)); mixk(ptr(P.recd.p)); mixk(uint64_t(P.s.cap > 0)); mixk(uint64_t(P.born_cap));
    mixk(ptr(c.ext.u)); mixk(ptr(c.ext.m)); mixk(ptr(c.ext.kt)); mixk(uint64_t(c.ext.nu) << 32 | uint64_t(c.ext.nm));
    mixk(uint64_t(passes)); mixk(uint64_t(c.mixed) | uint64_t(c.f32s) << 1); mixk(ptr(c.Rx.p));
    mixk(ptr(pp.jkx)); mixk(ptr(pp.jky)); mixk(ptr(c.mixed ? static_cast<const void*>(c.mx.j0x.p) : c.j0x.p));
    uint64_t dbits;
    std::memcpy(&dbits, &Delta, sizeof dbits);
    mixk(dbits);
    auto issue = [&]() {
        bool have_dl = false;
        const bool fh = !c.yf;
        // the deposit planes and the count of freed electrons start cleared (the rows kernel of every pass clears
        // them again for the next one)
        if (c.f32s) G3D_CUDA(cudaMemsetAsync(P.jsrf.p, 0, size_t(c.yf ? 4 : 3) * c.nk * sizeof(float), c.stream));
        else G3D_CUDA(cudaMemsetAsync(P.jsr.p, 0, size_t(3) * c.nk * sizeof(double), c.stream));
        G3D_CUDA(cudaMemsetAsync(P.bcnt.p, 0, sizeof(int), c.stream));
        G3D_CUDA(cudaMemsetAsync(P.rhol.p, 0, P.rhol.n * sizeof(double), c.stream));
        // front: half-cell N-2 predicted with its value of level s0; the front slice solved with it
        launch_slice_prologue(c, N - 1, N - 2, 0, 0);
        launch_march_slice(c, D, N - 1);
        real_fields_slice(c, N - 1, N - 2, true, rec_fld ? long(passes) * (N - 1) + passes - 1 : -1);
        if (rec && !rec_fld) launch_record_fields(c, N - 1, passes - 1);

        StreamArgs sa;
        sa.F = c.F.p; sa.g = c.geo(); sa.laser = c.laser; sa.sv = P.stepv.p; sa.zc = c.P.zeta_center;
        sa.Delta = Delta; sa.vz_beam = P.cfg.vz_beam;
        sa.J = P.jsr.p; sa.Jf = P.jsrf.p; sa.ions = P.ion_dev.p; sa.adk = P.adk_dev.p; sa.sd = P.sdev.p; sa.bcnt = P.bcnt.p;
        sa.bcap = ionz ? int(P.born_cap) : 0; sa.dry = 0; sa.n = 0; sa.pass = 0;
        sa.ylo = c.yf ? -1e300 : c.ynode_h[1]; sa.yhi = c.yf ? 1e300 : c.ynode_h[size_t(c.ny) - 1];
        sa.Fmid = c.yf || c.f32s ? static_cast<const void*>(P.fmid.p) : nullptr;   // null if never allocated
        sa.inv_dx = 1 / c.dx; sa.inv_dy = 1 / c.dy; sa.dep_norm = 0;
        sa.Fd = c.mixed ? nullptr : c.Fd.p;
        sa.recd = rec_x ? P.recd.p : nullptr;
        sa.ext = c.ext;
        const long nl = long(c.nx) + c.ny;
        for (int n = nhi; n >= c.a; --n) {
            // sin, si0 <- pin; the prediction of half-cell n-1 from its level s0; the slice saved for the passes
            // (for the half-cells below the first, fused into the correction of the half-cell above)
            if (n == nhi) launch_slice_prologue(c, n, n >= 1 ? n - 1 : -1, 1, passes > 1 ? 1 : 0);
            const double wex = (n >= 1 && n + 1 <= N - 2 && have_dl)
                                   ? (cen[size_t(n)] - cen[size_t(n - 1)]) / (cen[size_t(n + 1)] - cen[size_t(n)]) : 0.0;
            if (rec && !rec_x) launch_record_particles(c, n);
            for (int pass = 0; pass < passes; ++pass) {
                if (fh) launch_pass_prologue(c, n, pass > 0 ? 1 : 0);
                sa.n = n;
                sa.dep_norm = 1 / (Delta * (c.zeta[size_t(n) + 1] - c.zeta[size_t(n)]) * c.dx);
                sa.pass = pass;
                sa.dry = pass + 1 < passes ? 1 : 0;
                sa.rl[0] = sa.dry ? nullptr : P.rhol.p + long(n) * nl;
                sa.rl[1] = sa.dry || !P.ion_lines ? nullptr : P.rhol.p + (long(N) + n) * nl;
                launch_stream(c, sa);
                // freed electrons join the march (after the last pass's stream, before its rows kernel clears the count)
                if (ionz && pass + 1 == passes) launch_born_append(c);
                if (!fh) {                     // rows of the current's spectra; columns, march and field columns fused
                    launch_stream_spectra_rows(c);
                    launch_pass_cols(c, D, n, extrap ? 1 : 0, wex, pass > 0 ? 1 : 0);
                    real_fields_slice(c, n, pass + 1 < passes ? n : n - 1, false, rec_fld ? long(passes) * n + pass : -1);
                    if (rec && !rec_fld) launch_record_fields(c, n, pass);
                } else {
                    launch_stream_spectra(c);
                    launch_replace_pred(c, n, extrap ? 1 : 0, wex);
                    launch_march_slice(c, D, n);
                    real_fields_slice(c, n, pass + 1 < passes ? n : n - 1);
                }
            }
            // half-cell n is final: correct R at slice n+1, keep the change and the current
            const double q = D * c.wlo_h[size_t(n + 1)];
            if (n - 1 >= c.a) launch_correct_prologue(c, n, q, n + 1 < c.b ? 1 : 0, n - 1 >= 1 ? n - 2 : -1, passes > 1 ? 1 : 0);
            else launch_correct(c, n, q, n + 1 < c.b ? 1 : 0);
            have_dl = true;
        }
        if (rec) launch_record_particles(c, -1);         // the states after the last half-cell
    };
    PlasmaState::LoopGraph* hit = nullptr;
    for (auto& l : P.loops) if (l.key == key) hit = &l;
    if (c.profiling) {
        issue();
    } else if (hit) {
        c.launches += hit->launches;
        G3D_CUDA(cudaGraphLaunch(hit->exec, c.stream));
    } else {
        if (P.loops.size() >= 4) { cudaGraphExecDestroy(P.loops.front().exec); P.loops.erase(P.loops.begin()); }
        const long l0 = c.launches;
        G3D_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeRelaxed));
        try {
            issue();
        } catch (...) {
            cudaGraph_t gr = nullptr;
            cudaStreamEndCapture(c.stream, &gr);
            if (gr) cudaGraphDestroy(gr);
            cudaGetLastError();
            throw;
        }
        cudaGraph_t gr = nullptr;
        G3D_CUDA(cudaStreamEndCapture(c.stream, &gr));
        cudaGraphExec_t ex = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&ex, gr, 0);
        cudaGraphDestroy(gr);
        G3D_CUDA(e);
        P.loops.push_back(PlasmaState::LoopGraph{key, ex, c.launches - l0});
        G3D_CUDA(cudaGraphLaunch(ex, c.stream));
    }
    G3D_CUDA(cudaStreamSynchronize(c.stream));
    int flag = 0;
    G3D_CUDA(cudaMemcpy(&flag, P.flags.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) throw Error(G3D_ERR_CAPACITY, "ionization: list of freed electrons overflowed");
    // trapped particles: fast ones join the beam list, slow ones stream again in the next step (split on the device
    // in list order, z = s1: the slow ones stay there as the next march's joining particles, alive 6; only the ones
    // joining the beam come to the host)
    std::vector<g3d_particle> add = fast_trapped(c, launch_trapped_split(c, s1));
    for (auto& p : add) {
        p.alive = 1;
        p.sp = (p.sp >= SP_FREED && p.sp < SP_INJECTED) ? p.sp - SP_FREED + SP_INJECTED : p.sp >= SP_INJECTED ? p.sp : SP_TRAPPED;
        ++P.trapped_total;
    }
    if (!add.empty() && !beam_keep_live_and_append(c, add.data(), long(add.size()))) {   // short of capacity: on the host
        std::vector<g3d_particle> all = get_particles(c), keep;
        keep.reserve(all.size() + add.size());
        for (auto& p : all) if (p.alive == 1) keep.push_back(p);
        keep.insert(keep.end(), add.begin(), add.end());
        set_particles(c, keep.data(), long(keep.size()));
    }
    // the sponge damps R - R_b with the bound field of the beam list only: jkz -= js0z
    if (c.mixed) launch_axpy_fc(c, c.mx.jkz.p, P.js0z.p, -1.0, size_t(c.ns + 1) * c.nkh);
    else launch_axpy_c(c, c.jkz.p, P.js0z.p, -1.0, size_t(c.ns + 1) * c.nkh);
}

// The beam particles that became slower than vz_min stream in the current march (collect_restreaming,
// src/sim_plasma.cpp:474-491, one rank).
void collect_restreaming(Ctx& c) {
    PlasmaState& P = *c.pl;
    // counted on the device first: the whole beam list comes to the host only when a particle left it
    if (c.np == 0 || count_state(c, c.parts.alive, c.np, nullptr, 4) == 0) return;
    std::vector<g3d_particle> all = get_particles(c), keep;
    bool any = false;
    for (auto& p : all) if (p.alive == 4) { any = true; break; }
    if (!any) return;
    for (auto& p : all) {
        if (p.alive == 4) {
            g3d_particle q = p; q.alive = 6; ++P.restreamed_total;
            P.joining.push_back(q);
        } else if (p.alive == 1) keep.push_back(p);
    }
    set_particles(c, keep.data(), long(keep.size()));
}

// ---------------------------------------------------------------- grid lasers (add_grid_lasers)
// The transverse profile exp(-(x^2 + y^2) / (w^2 qb)) / qb of a paraxial beam is separable; its two real parts
// are transformed once, and every slice adds 2 Re(c_n P) (c_n = amp env_n carrier_n) times the polarisation.
// Free-hand y: R_x on the nodes (zero at the wall node j = 0) and R_y on the half-nodes, so the profile is taken at
// both (planes 0, 1 and 3, 4; planes 2 and 5 stay zero) and transformed along x only.
__device__ __forceinline__ void glaser_point(double xp, double yp, double w2, double qr, double qi, double& re, double& im) {
    // exp(-(r^2/w^2) / qb) / qb, qb = qr + i qi
    const double r2 = (xp * xp + yp * yp) / w2;
    const double d = qr * qr + qi * qi;
    const double ir = qr / d, ii = -qi / d;                   // 1 / qb
    const double er = -r2 * ir, ei = -r2 * ii;
    const double m = exp(er);
    const double pr = m * cos(ei), pi = m * sin(ei);          // exp(-r^2/(w^2 qb))
    re = pr * ir - pi * ii;                                   // real part of the product with 1/qb
    im = pr * ii + pi * ir;                                   // imaginary part
}
__global__ void k_glaser_profile(Geo g, double X0, double Y0, double w2, double qr, double qi, double* __restrict__ out) {
    const long nk = g.nk;
    for (long i = long(blockIdx.x) * blockDim.x + threadIdx.x; i < nk; i += long(gridDim.x) * blockDim.x) {
        const int ix = int(i % g.nx), j = int(i / g.nx);
        const double xp = ix * g.dx + X0;
        if (g.yf) { glaser_point(xp, j * g.dy + Y0, w2, qr, qi, out[i], out[nk + i]); continue; }
        if (j == 0) { out[i] = 0; out[nk + i] = 0; }
        else glaser_point(xp, g.yn[j], w2, qr, qi, out[i], out[nk + i]);
        glaser_point(xp, 0.5 * (g.yn[j] + g.yn[j + 1]), w2, qr, qi, out[3 * nk + i], out[4 * nk + i]);
    }
}
__global__ void k_glaser_add(Geo g, const cpx* __restrict__ PR, const cpx* __restrict__ PI, const cpx* __restrict__ QR,
                             const cpx* __restrict__ QI, const double* __restrict__ cre, const double* __restrict__ cim,
                             cpx* __restrict__ Rx, cpx* __restrict__ Ry, double ax, double ay, double bx, double by,
                             const cpx* __restrict__ lm, cpx* __restrict__ sx, cpx* __restrict__ sy) {
    // R_x += 2 (ax (cre PR - cim PI) + bx (cim PR + cre PI)), R_y likewise with ay, by and the profile Q of the
    // R_y points (real-valued field factors)
    const long nk = g.nkh, n = long(g.ns) * nk;
    for (long idx = long(blockIdx.x) * blockDim.x + threadIdx.x; idx < n; idx += long(gridDim.x) * blockDim.x) {
        const long l = idx / nk, i = idx - l * nk;
        const double cr = cre[l], ci = cim[l];
        if (cr == 0 && ci == 0) continue;
        const cpx re = cr * PR[i] - ci * PI[i];          // spectrum of Re(c P)
        const cpx im = ci * PR[i] + cr * PI[i];          // spectrum of Im(c P)
        const cpx rq = cr * QR[i] - ci * QI[i], iq = ci * QR[i] + cr * QI[i];
        cpx ux = 2.0 * (ax * re + bx * im), uy = 2.0 * (ay * rq + by * iq);
        if (sx) { sx[idx] = sx[idx] + ux; sy[idx] = sy[idx] + uy; }      // kept for the laser-mode gradient
        if (lm) { ux = lm[i] * ux; uy = lm[i] * uy; }                     // the mode coefficients
        Rx[idx] = Rx[idx] + ux;
        Ry[idx] = Ry[idx] + uy;
    }
}

void launch_real_to_half3(Ctx& c, const double* J3, cpx* T3, cpx* out3);   // k_plasma.cu

void add_grid_lasers(Ctx& c) {
    if (c.lspx.p) { c.lspx.zero(c.stream); c.lspy.zero(c.stream); }
    if (c.glasers.empty()) return;
    DevBuf<double> prof;
    prof.alloc(size_t(6) * c.nk, c.stream);          // Re P, Im P, a zero plane (free-hand y: twice)
    G3D_CUDA(cudaMemsetAsync(prof.p, 0, size_t(6) * c.nk * sizeof(double), c.stream));
    DevBuf<cpx> spec, tsc;
    spec.alloc(size_t(6) * c.nkh, c.stream);
    tsc.alloc(size_t(3) * c.nkh, c.stream);
    DevBuf<double> coef;
    coef.alloc(size_t(2) * c.ns, c.stream);
    for (const auto& Lz : c.glasers) {
        const double amp = Lz.a0 * Lz.kL;
        const double zR = 0.5 * Lz.kL * Lz.waist * Lz.waist;
        const std::complex<double> qb(1.0, (0.0 - Lz.z_focus) / zR);
        const std::complex<double> rot(std::cos(Lz.pol_angle), std::sin(Lz.pol_angle));
        std::vector<double> cre(size_t(c.ns), 0.0), cim(size_t(c.ns), 0.0);
        for (int n = 0; n < c.ns; ++n) {
            const double d = c.zeta[size_t(c.a + n)] - Lz.zeta_c;
            const double env = std::exp(-2 * std::log(2.0) * d * d / (Lz.tau * Lz.tau));
            if (std::fabs(env) < 1e-12) continue;
            const std::complex<double> car = std::exp(std::complex<double>(0, Lz.kL * d + Lz.cep));
            const std::complex<double> cn = amp * env * car;
            cre[size_t(n)] = cn.real(); cim[size_t(n)] = cn.imag();
        }
        k_glaser_profile<<<148 * 4, 256, 0, c.stream>>>(c.geo(), c.X0, c.Y0, Lz.waist * Lz.waist, qb.real(), qb.imag(), prof.p);
        c.check_launch("k_glaser_profile");
        launch_real_to_half3(c, prof.p, tsc.p, spec.p);
        if (!c.yf) launch_real_to_half3(c, prof.p + 3 * c.nk, tsc.p, spec.p + 3 * c.nkh);
        const cpx* q = c.yf ? spec.p : spec.p + 3 * c.nkh;      // the profile at the points of R_y
        G3D_CUDA(cudaMemcpyAsync(coef.p, cre.data(), size_t(c.ns) * 8, cudaMemcpyHostToDevice, c.stream));
        G3D_CUDA(cudaMemcpyAsync(coef.p + c.ns, cim.data(), size_t(c.ns) * 8, cudaMemcpyHostToDevice, c.stream));
        // linear: ex = Re(E) cos(pol), ey = Re(E) sin(pol); circular: ex = Re E, ey = helicity Im E
        double ax, ay, bx, by;
        if (Lz.circular) { ax = 1; bx = 0; ay = 0; by = Lz.helicity; }
        else { ax = rot.real(); bx = 0; ay = rot.imag(); by = 0; }
        k_glaser_add<<<148 * 8, 256, 0, c.stream>>>(c.geo(), spec.p, spec.p + c.nkh, q, q + c.nkh, coef.p, coef.p + c.ns,
                                                     c.Rx.p, c.Ry.p, ax, ay, bx, by, c.lmode.p, c.lspx.p, c.lspy.p);
        c.check_launch("k_glaser_add");
        G3D_CUDA(cudaStreamSynchronize(c.stream));
    }
}

}  // namespace g3d
