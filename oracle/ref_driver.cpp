// Test infrastructure only: a C driver around the reference GEM-PIC-3D CPU build, used as the
// parity oracle and as the timed CPU baseline. It is compiled together with the reference's own
// sources where they lie (oracle/Makefile) into oracle/_ref/libg3dref.so; nothing of the
// product links it. Its entry points mirror include/g3d.h with the prefix ref_ so the tests can
// run both sides with one parameter set.
//
// What it calls in the reference: Config::base_units / zeta_uniform / y_uniform (sim_config.cpp:5-39),
// Simulation::Simulation, init, step, solve_fields, currents, march, sponge_and_real_fields,
// push, comoving_field, relax_start_field, shift_window, local_field_energy, set_particles,
// host_particles (sim.hpp:222-351). The diagnostics sums restate sim_output.cpp:10-26.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "sim.hpp"
#include "atomic_data.hpp"
#include "g3d.h"

static_assert(sizeof(Particle) == sizeof(g3d_particle), "particle record must be the reference's 104 bytes");

namespace {
std::string g_err;
Comm g_comm;

struct RefCtx {
    Config cfg;
    std::unique_ptr<Simulation> sim;
};

int fail(const std::exception& e) { g_err = e.what(); return G3D_ERR_ARG; }

Config make_config(const g3d_grid* g, const g3d_params* p) {
    Config c = Config::base_units(p->lambda0);
    c.nx = g->nx; c.Lx = g->Lx;
    if (g->y_fourier) {
        c.y_uniform(g->ny, g->Ly);
    } else {                        // free-hand y: the node table as Config::y_table leaves it (walls at 0 and ny)
        if (!g->ynode) throw std::runtime_error("oracle driver: free-hand y needs ynode");
        c.ny = g->ny;
        c.ynode.assign(g->ynode, g->ynode + g->ny + 1);
        c.y_fourier = false; c.move_y = false;
        c.Ly = c.ynode.back() - c.ynode.front();
        c.y_change = 0;
    }
    // zeta: copy the slice table; zeta_uniform when it is uniform (sim_config.cpp:14-20)
    c.nzeta = g->nzeta;
    c.zeta.assign(g->zeta, g->zeta + g->nzeta);
    c.Lwin = c.zeta.back();
    c.zeta_change = 0;
    c.dz = p->dz; c.z_end = p->z_end; c.dz_push = p->dz_push;
    c.sponge = p->sponge; c.sponge_y = p->sponge_y; c.sponge_rate = p->sponge_rate;
    c.move_x = p->move_x != 0; c.move_y = p->move_y != 0; c.window_lag = p->window_lag;
    c.self_fields = p->self_fields != 0; c.zeta_filter = p->zeta_filter != 0; c.k_filter = p->k_filter != 0;
    c.push_phase = p->push_phase;
    c.laser_on = p->laser_on != 0;
    if (p->laser_on && p->laser_envelope != G3D_ENV_GAUSSIAN)
        throw std::runtime_error("oracle driver: the reference has only the Gaussian envelope");
    c.a0 = p->a0; c.kL = p->kL; c.theta = p->theta; c.tau = p->tau; c.cep = p->cep;
    c.pol = p->laser_pol == G3D_POL_S ? "s" : p->laser_pol == G3D_POL_P ? "p" : "circular";
    c.start_fwhm = p->tau > 0 ? p->eta_c / p->tau : 0;
    c.stop_fwhm = p->stop_fwhm;
    c.zeta_center = p->zeta_center;
    c.freeze_bunch = p->freeze_bunch != 0; c.start_relax = p->start_relax != 0; c.box_mean = p->box_mean != 0;
    c.every = 0; c.dump_particles = false;
    return c;
}
}  // namespace

extern "C" {

const char* ref_last_error() { return g_err.c_str(); }

int ref_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n; return 1;
#endif
}

int ref_create(const g3d_grid* g, const g3d_params* p, const g3d_bunch* bunches, int nb, void** out) {
    try {
        auto* r = new RefCtx();
        r->cfg = make_config(g, p);
        r->cfg.bunches.clear();
        for (int k = 0; k < nb; ++k) {
            const g3d_bunch& b = bunches[k];
            Config::Bunch u;
            u.name = k == 0 ? "bunch" : "bunch" + std::to_string(k + 1);
            u.q = b.q; u.charge = b.charge_C; u.gamma = b.gamma; u.sigx = b.sigx; u.sigy = b.sigy; u.sigz = b.sigz;
            u.length = b.length; u.emitx = b.emitx; u.emity = b.emity; u.espread = b.espread;
            u.zeta_center = b.zeta_center; u.x0 = b.x0; u.y0 = b.y0; u.nmacro = long(b.nmacro); u.seed = (unsigned long)b.seed;
            if (b.beamlet > 1) { u.noise = "fawley"; u.beamlet = b.beamlet; u.noise_lambda = b.noise_lambda; }
            r->cfg.bunches.push_back(u);
        }
        if (nb > 0) {
            const Config::Bunch& f = r->cfg.bunches[0];
            r->cfg.charge = f.charge; r->cfg.gamma = f.gamma; r->cfg.sigx = f.sigx; r->cfg.sigy = f.sigy;
            r->cfg.sigz = f.sigz; r->cfg.nmacro = f.nmacro; r->cfg.seed = f.seed;
        }
        r->sim.reset(new Simulation(r->cfg, g_comm));
        *out = r;
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

void ref_destroy(void* h) { delete static_cast<RefCtx*>(h); }

// The same with a plasma, ion species and grid lasers (Config fields of src/sim.hpp:95-131).
int ref_create2(const g3d_grid* g, const g3d_params* p, const g3d_bunch* bunches, int nb, const g3d_plasma* pl,
                const g3d_ion* ions, int nions, const g3d_grid_laser* gl, int ngl, void** out) {
    try {
        void* h = nullptr;
        // build the config as ref_create does, then add the plasma before constructing the Simulation
        Config c = make_config(g, p);
        c.bunches.clear();
        for (int k = 0; k < nb; ++k) {
            const g3d_bunch& b = bunches[k];
            Config::Bunch u;
            u.name = k == 0 ? "bunch" : "bunch" + std::to_string(k + 1);
            u.q = b.q; u.charge = b.charge_C; u.gamma = b.gamma; u.sigx = b.sigx; u.sigy = b.sigy; u.sigz = b.sigz;
            u.length = b.length; u.emitx = b.emitx; u.emity = b.emity; u.espread = b.espread;
            u.zeta_center = b.zeta_center; u.x0 = b.x0; u.y0 = b.y0; u.nmacro = long(b.nmacro); u.seed = (unsigned long)b.seed;
            if (b.beamlet > 1) { u.noise = "fawley"; u.beamlet = b.beamlet; u.noise_lambda = b.noise_lambda; }
            c.bunches.push_back(u);
        }
        if (nb > 0) {
            const Config::Bunch& f = c.bunches[0];
            c.charge = f.charge; c.gamma = f.gamma; c.sigx = f.sigx; c.sigy = f.sigy; c.sigz = f.sigz; c.nmacro = f.nmacro;
        }
        if (pl) {
            c.plasma_on = true;
            c.n0 = pl->n0; c.r_max = pl->r_max; c.channel_depth = pl->channel_depth; c.r_channel = pl->r_channel;
            c.parabolic = pl->parabolic != 0; c.smooth_length = pl->smooth_length;
            c.pz_points.assign(pl->z_points, pl->z_points + pl->n_z);
            c.pz_values.assign(pl->z_values, pl->z_values + pl->n_z);
            c.ppc_x = pl->ppc_x; c.ppc_y = pl->ppc_y; c.iterations = pl->iterations;
            c.vz_min = pl->vz_min; c.vz_beam = pl->vz_beam; c.trap_advance = pl->trap_advance;
            c.predictor_extrapolate = pl->predictor_extrapolate != 0; c.free_electrons = pl->free_electrons != 0;
            c.box_mean = pl->box_mean != 0;
            c.seed = (unsigned long)pl->seed;
        }
        for (int k = 0; k < nions; ++k) {
            const g3d_ion& I = ions[k];
            Config::IonSpecies s;
            s.name = "ion" + std::to_string(k + 1);
            s.mass = I.mass; s.atoms = I.atoms; s.Z0 = I.Z0; s.Zmax = I.Zmax; s.mobile = I.mobile != 0;
            s.ionization = I.ionization != 0;
            s.ip_eV.assign(I.ip_eV, I.ip_eV + I.n_ip);
            c.ions.push_back(s);
        }
        for (int k = 0; k < ngl; ++k) {
            Config::GridLaser L;
            L.a0 = gl[k].a0; L.kL = gl[k].kL; L.waist = gl[k].waist; L.tau = gl[k].tau; L.zeta_c = gl[k].zeta_c;
            L.z_focus = gl[k].z_focus; L.cep = gl[k].cep; L.pol_angle = gl[k].pol_angle;
            L.circular = gl[k].circular != 0; L.helicity = gl[k].helicity;
            c.glasers.push_back(L);
        }
        auto* r = new RefCtx();
        r->cfg = c;
        r->sim.reset(new Simulation(r->cfg, g_comm));
        h = r;
        *out = h;
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

// Streaming particles of the last plasma march (the reference's `strm`, nstrm records).
int ref_get_streaming(void* h, g3d_particle* out, long cap, long* n) {
    try {
        Simulation& s = *static_cast<RefCtx*>(h)->sim;
        *n = s.nstrm;
        if (s.nstrm > cap) throw std::runtime_error("capacity");
        if (s.nstrm) s.strm.to_host(reinterpret_cast<Particle*>(out), 0, size_t(s.nstrm));
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}
int ref_march_plasma(void* h, double s0, double s1) {
    try { static_cast<RefCtx*>(h)->sim->march_plasma(s0, s1); return 0; } catch (const std::exception& e) { return fail(e); }
}
// Element data of the reference's table (mass [u], ionization energies [eV]); returns Znuc or -1.
int ref_element(const char* sym, double* mass_u, double* ip, int cap) {
    const gem::Element* e = gem::findElement(sym);
    if (!e) return -1;
    *mass_u = e->mass_u;
    for (int k = 0; k < e->Znuc && k < cap; ++k) ip[k] = e->ip_eV[size_t(k)];
    return e->Znuc;
}

#define SIM (static_cast<RefCtx*>(h)->sim)
#define TRY(body) try { body; return 0; } catch (const std::exception& e) { return fail(e); }

int ref_load_bunches(void* h) { TRY(SIM->load_bunch()) }
int ref_init(void* h) {
    // Simulation::init without the bunch load when particles were set by hand
    TRY(SIM->init())
}
int ref_init_fields(void* h) {
    // init() after load_bunch: the field part (sim_setup.cpp:180-196) for externally set particles
    try {
        Simulation& s = *SIM;
        s.s = 0; s.istep = 0;
        if (s.cfg.self_fields) {
            s.starting_ = true;
            if (s.cfg.nbunch() > 1) s.comoving_fields_per_bunch();
            else { s.currents(); s.comoving_field(); }
            if (s.cfg.start_relax) s.relax_start_field();
            s.add_grid_lasers();
            s.march(0.0);
            s.starting_ = false;
            s.sponge_and_real_fields();
            const size_t n = size_t(s.ns + 1) * s.nk;
            std::memcpy(s.j0x.data(), s.jkx.data(), n * sizeof(cpx));
            std::memcpy(s.j0y.data(), s.jky.data(), n * sizeof(cpx));
        }
        s.window_shift_post();
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}
int ref_step(void* h) { TRY(SIM->step()) }
int ref_solve_fields(void* h, double D) { TRY(SIM->solve_fields(D)) }
int ref_currents(void* h) { TRY(SIM->currents()) }
int ref_march(void* h, double D) { TRY(SIM->march(D)) }
int ref_sponge_and_real_fields(void* h) { TRY(SIM->sponge_and_real_fields()) }
int ref_push(void* h, double s0, double s1) { TRY(SIM->push(s0, s1, 0, SIM->np)) }
int ref_comoving_field(void* h) { TRY(SIM->comoving_field()) }
int ref_relax_start_field(void* h) { TRY(SIM->relax_start_field()) }
int ref_shift_window(void* h, int nxs, int nys) { TRY(SIM->shift_window(nxs, nys)) }
int ref_set_starting(void* h, int v) { TRY(SIM->starting_ = v != 0) }
int ref_set_origin(void* h, double X0, double Y0) { TRY(SIM->X0 = X0; SIM->Y0 = Y0) }

int ref_set_particles(void* h, const g3d_particle* p, long n) {
    try {
        std::vector<Particle> v(static_cast<size_t>(n));
        if (n) std::memcpy(static_cast<void*>(v.data()), p, static_cast<size_t>(n) * sizeof(Particle));
        SIM->set_particles(v);
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}
long ref_num_particles(void* h) { return SIM->np; }
int ref_get_particles(void* h, g3d_particle* out, long cap) {
    try {
        const std::vector<Particle> v = SIM->host_particles();
        if (long(v.size()) > cap) throw std::runtime_error("capacity");
        if (!v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(Particle));
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

int ref_get_status(void* h, g3d_status* o) {
    Simulation& s = *SIM;
    o->s = s.s; o->X0 = s.X0; o->Y0 = s.Y0; o->beta_b = s.beta_b; o->gm2_b = s.gm2_b; o->field_energy = s.field_energy;
    o->istep = s.istep; o->np = s.np; o->lost = s.lost_total; o->stop = s.finished() ? 1 : 0;
    return 0;
}

// Array access by the ids of include/g3d.h.
static int array_of(Simulation& s, int which, Buf<cpx>** c, Buf<double>** d, Buf<float>** f) {
    *c = nullptr; *d = nullptr; *f = nullptr;
    switch (which) {
        case G3D_A_RX: *c = &s.Rx; break; case G3D_A_RY: *c = &s.Ry; break;
        case G3D_A_EZ: *c = &s.Ez; break; case G3D_A_BZ: *c = &s.Bz; break;
        case G3D_A_LX: *c = &s.Lx; break; case G3D_A_LY: *c = &s.Ly; break;
        case G3D_A_J0X: *c = &s.j0x; break; case G3D_A_J0Y: *c = &s.j0y; break;
        case G3D_A_JKX: *c = &s.jkx; break; case G3D_A_JKY: *c = &s.jky; break;
        case G3D_A_JKZ: *c = &s.jkz; break;
        case G3D_A_JW: *d = &s.jw; break;
        case G3D_A_F: *f = &s.F; break;
        case G3D_A_RHO_E: *d = &s.rho_lines; break;
        case G3D_A_RHO_I: *d = &s.rho_lines_i; break;
        default: return -1;
    }
    return 0;
}
int ref_array_info(void* h, int which, size_t* count, size_t* eb) {
    Buf<cpx>* c; Buf<double>* d; Buf<float>* f;
    if (array_of(*SIM, which, &c, &d, &f)) { g_err = "unknown array"; return G3D_ERR_ARG; }
    if (c) { *count = c->size(); *eb = sizeof(cpx); }
    if (d) { *count = d->size(); *eb = sizeof(double); }
    if (f) { *count = f->size(); *eb = sizeof(float); }
    return 0;
}
int ref_get_array(void* h, int which, void* out, size_t count) {
    Buf<cpx>* c; Buf<double>* d; Buf<float>* f;
    if (array_of(*SIM, which, &c, &d, &f)) { g_err = "unknown array"; return G3D_ERR_ARG; }
    const size_t n = c ? c->size() : d ? d->size() : f->size();
    if (count != n) { g_err = "count mismatch"; return G3D_ERR_ARG; }
    if (c) c->to_host(static_cast<cpx*>(out), 0, n);
    if (d) d->to_host(static_cast<double*>(out), 0, n);
    if (f) f->to_host(static_cast<float*>(out), 0, n);
    return 0;
}
int ref_set_array(void* h, int which, const void* in, size_t count) {
    Buf<cpx>* c; Buf<double>* d; Buf<float>* f;
    if (array_of(*SIM, which, &c, &d, &f)) { g_err = "unknown array"; return G3D_ERR_ARG; }
    const size_t n = c ? c->size() : d ? d->size() : f->size();
    if (count != n) { g_err = "count mismatch"; return G3D_ERR_ARG; }
    if (c) c->from_host(static_cast<const cpx*>(in), 0, n);
    if (d) d->from_host(static_cast<const double*>(in), 0, n);
    if (f) f->from_host(static_cast<const float*>(in), 0, n);
    return 0;
}

double ref_field_energy(void* h) { return SIM->local_field_energy(); }

// The 19 sums of Simulation::diagnostics (sim_output.cpp:10-26), without printing.
int ref_diagnostics(void* h, double* S) {
    try {
        Simulation& s = *SIM;
        for (int k = 0; k < 19; ++k) S[k] = 0;
        for (const auto& p : s.host_particles()) {
            if (p.alive != 1) continue;
            if (!is_bunch(p.sp)) { S[17] += 1; S[18] += p.q * p.w; continue; }
            const double g = std::sqrt(1 + p.px * p.px + p.py * p.py + p.pz * p.pz);
            const double X = p.x + s.X0, Y = p.y + s.Y0;
            const double et = s.laser.eta(X, s.s, s.s - (p.zeta - s.cfg.zeta_center));
            const double v[] = {1, X, Y, p.zeta, X * X, Y * Y, p.zeta * p.zeta, p.px, p.py, p.pz, g,
                                p.px * s.laser.kx + p.pz * s.laser.kz, p.pz * p.pz, et};
            for (int k = 0; k < 14; ++k) S[k] += p.w * v[k];
            S[14] += 1;
        }
        S[15] = s.cfg.self_fields ? s.local_field_energy() : 0;
        S[16] = double(s.lost_total);
        s.field_energy = S[15];
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}

int ref_write_checkpoint(void* h, const char* dir) {
    try {
        Simulation& s = *SIM;
        s.cfg.dir = dir;
        s.write_checkpoint();
        return 0;
    } catch (const std::exception& e) { return fail(e); }
}
int ref_read_checkpoint(void* h, const char* dir, long step) {
    try {
        Simulation& s = *SIM;
        s.cfg.dir = dir;
        s.read_checkpoint(step);
        return 0;
    } catch (const std::exception& e) { g_err = e.what(); return G3D_ERR_IO; }
}

}  // extern "C"
