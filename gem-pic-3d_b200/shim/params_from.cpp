// setup_from: every Config field the march reads, mapped onto g3d_grid, g3d_params, g3d_bunch, g3d_plasma, g3d_ion and
// g3d_grid_laser (include/g3d.h). The Config comes from the reference's own deck reader (Config::from_deck,
// src/sim_config.cpp:69-343), so a deck keeps its keys, units and defaults. What the library does not run is refused
// here, before any device work, with the key that asks for it.
#include "params_from.hpp"

#include <string>
#include "sim.hpp"

namespace g3dshim {

namespace {
[[noreturn]] void refuse(const std::string& what) {
    throw std::runtime_error("libg3d does not run " + what + " (the reference's CPU/GPU build does)");
}
}  // namespace

Setup setup_from(const Config& c) {
    Setup s;
    // grid: Fourier x; Fourier y, or the free-hand y table between walls; the zeta slice table
    s.grid.nx = c.nx; s.grid.ny = c.ny; s.grid.nzeta = c.nzeta;
    s.grid.y_fourier = c.y_fourier ? 1 : 0;
    s.grid.Lx = c.Lx; s.grid.Ly = c.Ly;
    s.zeta = c.zeta;
    if (int(s.zeta.size()) != c.nzeta) refuse("a zeta table whose length differs from grid.nzeta");
    if (!c.y_fourier) s.ynode = c.ynode;
    // run and numerics keys
    g3d_params& p = s.params;
    p.lambda0 = c.lambda0;
    p.dz = c.dz; p.dz_push = c.dz_push; p.z_end = c.z_end;
    p.sponge = c.sponge; p.sponge_y = c.sponge_y; p.sponge_rate = c.sponge_rate;
    p.move_x = c.move_x; p.move_y = c.move_y; p.window_lag = c.window_lag;
    p.self_fields = c.self_fields; p.zeta_filter = c.zeta_filter; p.k_filter = c.k_filter;
    p.push_phase = c.push_phase;
    // the analytic plane wave (laser block without a type; src/sim.hpp:191-210, its centre at start_fwhm tau)
    p.laser_on = c.laser_on;
    if (c.pol == "s") p.laser_pol = G3D_POL_S;
    else if (c.pol == "p") p.laser_pol = G3D_POL_P;
    else if (c.pol == "circular") p.laser_pol = G3D_POL_CIRCULAR;
    else refuse("laser.polarization = " + c.pol);
    p.laser_envelope = G3D_ENV_GAUSSIAN;
    p.a0 = c.a0; p.kL = c.kL; p.theta = c.theta; p.tau = c.tau; p.cep = c.cep;
    p.eta_c = c.start_fwhm * c.tau;
    p.stop_fwhm = c.stop_fwhm;
    p.zeta_center = c.zeta_center;
    p.freeze_bunch = c.freeze_bunch; p.start_relax = c.start_relax; p.box_mean = c.box_mean;
    p.precision = G3D_FP64;
    // external elements (src/external.hpp: the same fields, code units) and their taper table
    for (const Undulator& U : c.undulators)
        s.undulators.push_back(g3d_undulator{U.helical, U.focusing, U.ku, U.B0, U.z0, U.z1, U.ramp, U.nk, U.koff, U.dzk});
    for (const Magnet& M : c.magnets) s.magnets.push_back(g3d_magnet{M.kind, 0, M.z0, M.z1, M.g, M.R, M.ramp, M.dsmax});
    s.ktab = c.ktab;
    for (const Config::Chicane& ch : c.chicanes) s.chicanes.push_back(g3d_chicane{ch.z, ch.r56, ch.delay, ch.gamma_ref});
    // bunch blocks: the built-in Gaussian / flat-top profiles with random shot noise
    for (const Config::Bunch& B : c.bunch_list()) {
        if (B.from_file) refuse("bunch.file (" + B.name + ")");
        if (!B.profile_z.empty() || !B.gamma_fn.empty() || !B.profile_r.empty() || !B.ux_fn.empty() || !B.uy_fn.empty())
            refuse("bunch profile functions (" + B.name + ")");
        if (B.noise != "random" && B.noise != "fawley") refuse("bunch.shot_noise = " + B.noise + " (" + B.name + ")");
        g3d_bunch b{};
        b.charge_C = B.charge; b.gamma = B.gamma; b.sigx = B.sigx; b.sigy = B.sigy; b.sigz = B.sigz; b.length = B.length;
        b.emitx = B.emitx; b.emity = B.emity; b.espread = B.espread; b.zeta_center = B.zeta_center;
        b.x0 = B.x0; b.y0 = B.y0; b.q = B.q; b.nmacro = B.nmacro; b.seed = B.seed;
        if (B.noise == "fawley") { b.beamlet = B.beamlet; b.noise_lambda = B.noise_lambda; }
        if (c.bunches.empty() && b.nmacro == 0) continue;      // no bunch block in the deck: no bunch
        s.bunches.push_back(b);
    }
    // plasma and ion blocks
    if (c.plasma_on) {
        if (!c.density_fn.empty()) refuse("plasma.density_function");
        s.plasma_on = true;
        g3d_plasma& q = s.plasma;
        q.n0 = c.n0; q.r_max = c.r_max; q.channel_depth = c.channel_depth; q.r_channel = c.r_channel;
        q.smooth_length = c.smooth_length;
        q.vz_min = c.vz_min; q.vz_beam = c.vz_beam; q.trap_advance = c.trap_advance;
        s.z_points = c.pz_points; s.z_values = c.pz_values;
        q.ppc_x = c.ppc_x; q.ppc_y = c.ppc_y; q.iterations = c.iterations;
        q.predictor_extrapolate = c.predictor_extrapolate; q.free_electrons = c.free_electrons;
        q.parabolic = c.parabolic; q.box_mean = c.box_mean;
        q.seed = c.seed;                 // the ionization's random numbers: the first bunch block's seed
        for (const Config::IonSpecies& I : c.ions) {
            g3d_ion ion{};
            ion.mass = I.mass; ion.atoms = I.atoms; ion.Z0 = I.Z0; ion.Zmax = I.Zmax;
            ion.mobile = I.mobile; ion.ionization = I.ionization;
            s.ions.push_back(ion);
            s.ion_ip.push_back(I.ip_eV);
        }
    }
    // grid lasers (laser blocks of type gaussian)
    for (const Config::GridLaser& L : c.glasers) {
        if (L.file) refuse("laser.type = file (" + L.file_path + ")");
        if (!L.profile.empty() || !L.envelope.empty()) refuse("laser profile or envelope functions");
        g3d_grid_laser g{};
        g.a0 = L.a0; g.kL = L.kL; g.waist = L.waist; g.tau = L.tau; g.zeta_c = L.zeta_c; g.z_focus = L.z_focus;
        g.cep = L.cep; g.pol_angle = L.pol_angle; g.circular = L.circular; g.helicity = L.helicity;
        s.lasers.push_back(g);
    }
    return s;
}

}  // namespace g3dshim
