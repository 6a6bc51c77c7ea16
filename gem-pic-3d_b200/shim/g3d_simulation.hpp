// The drop-in on the reference's side of the boundary: a C++17 host-side mirror of the reference's `class
// Simulation` (src/sim.hpp:222-360) over the C-ABI of libg3d (include/g3d.h), for a caller that keeps the
// reference's deck, expression and Config layers and hands the march to the B200.
//
//   g3dshim::Setup      the g3d structs of a run, built from a reference Config by setup_from (params_from.cpp),
//                       which maps every deck key the march uses and rejects, with std::runtime_error, the ones
//                       the library does not run (bunch files and profile functions, laser files, density functions,
//                       beamlet noise)
//   g3dshim::Simulation the reference's method names (init, step, finished, solve_fields, currents, march, push,
//                       shift_window, host_particles, set_particles, write/read_checkpoint, diagnostics sums), each
//                       a call of the C-ABI whose non-zero status becomes a std::runtime_error with the library's
//                       message, as the reference's gpu_check throws (src/portable.hpp:43-49)
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>
#include "g3d.h"

namespace g3dshim {

// A run's parameters as the C-ABI takes them. The arrays the structs point into live in the vectors beside them;
// Simulation points the structs at them when it is built, so a Setup may be copied or moved freely before.
struct Setup {
    g3d_grid grid{};
    g3d_params params{};
    std::vector<double> zeta, ynode;
    std::vector<g3d_bunch> bunches;
    bool plasma_on = false;
    g3d_plasma plasma{};
    std::vector<double> z_points, z_values;
    std::vector<g3d_ion> ions;
    std::vector<std::vector<double>> ion_ip;
    std::vector<g3d_grid_laser> lasers;
    std::vector<g3d_undulator> undulators;
    std::vector<g3d_magnet> magnets;
    std::vector<double> ktab;
    std::vector<g3d_chicane> chicanes;
    int precision = G3D_PREC_FP64;
};

inline void check(int rc, const g3d_ctx* ctx, const char* what) {
    if (rc != G3D_OK) throw std::runtime_error(std::string(what) + ": " + g3d_last_error(ctx));
}

class Simulation {
public:
    explicit Simulation(Setup s) : s_(std::move(s)) {
        g3d_grid g = s_.grid;
        g.zeta = s_.zeta.data();
        g.ynode = s_.ynode.empty() ? nullptr : s_.ynode.data();
        g.nzeta = int32_t(s_.zeta.size());
        check(g3d_create(&g, &s_.params, &ctx_), nullptr, "g3d_create");
        try {
            check(g3d_set_precision(ctx_, s_.precision), ctx_, "g3d_set_precision");
            if (s_.plasma_on) {
                g3d_plasma p = s_.plasma;
                p.z_points = s_.z_points.data(); p.z_values = s_.z_values.data(); p.n_z = int32_t(s_.z_points.size());
                std::vector<g3d_ion> ions = s_.ions;
                for (size_t k = 0; k < ions.size(); ++k) {
                    ions[k].ip_eV = s_.ion_ip[k].data();
                    ions[k].n_ip = int32_t(s_.ion_ip[k].size());
                }
                check(g3d_set_plasma(ctx_, &p, ions.data(), int32_t(ions.size())), ctx_, "g3d_set_plasma");
            }
            for (const g3d_grid_laser& L : s_.lasers) check(g3d_add_grid_laser(ctx_, &L), ctx_, "g3d_add_grid_laser");
            if (!s_.undulators.empty() || !s_.magnets.empty())
                check(g3d_set_external(ctx_, s_.undulators.data(), int32_t(s_.undulators.size()), s_.magnets.data(),
                                       int32_t(s_.magnets.size()), s_.ktab.data(), int32_t(s_.ktab.size())),
                      ctx_, "g3d_set_external");
            if (!s_.chicanes.empty())
                check(g3d_set_chicanes(ctx_, s_.chicanes.data(), int32_t(s_.chicanes.size())), ctx_, "g3d_set_chicanes");
        } catch (...) {
            g3d_destroy(ctx_);
            throw;
        }
    }
    ~Simulation() { g3d_destroy(ctx_); }
    Simulation(const Simulation&) = delete;
    Simulation& operator=(const Simulation&) = delete;

    // Simulation::init (src/sim_setup.cpp:178-197): the bunches of the deck, then the start fields
    void init() {
        load_bunch();
        check(g3d_init(ctx_), ctx_, "init");
    }
    void load_bunch() {
        check(g3d_load_bunches(ctx_, s_.bunches.data(), int32_t(s_.bunches.size())), ctx_, "load_bunch");
    }
    void step() { check(g3d_step(ctx_), ctx_, "step"); }
    bool finished() const { return status().stop != 0; }
    void solve_fields(double D) { check(g3d_solve_fields(ctx_, D), ctx_, "solve_fields"); }
    void currents() { check(g3d_currents(ctx_), ctx_, "currents"); }
    void march(double D) { check(g3d_march(ctx_, D), ctx_, "march"); }
    void sponge_and_real_fields() { check(g3d_sponge_and_real_fields(ctx_), ctx_, "sponge_and_real_fields"); }
    void push(double s0, double s1) { check(g3d_push(ctx_, s0, s1), ctx_, "push"); }
    void shift_window(int nxs, int nys) { check(g3d_shift_window(ctx_, nxs, nys), ctx_, "shift_window"); }
    void write_checkpoint(const std::string& path) { check(g3d_write_checkpoint(ctx_, path.c_str()), ctx_, "write_checkpoint"); }
    void read_checkpoint(const std::string& path) { check(g3d_read_checkpoint(ctx_, path.c_str()), ctx_, "read_checkpoint"); }
    // the same file written by the library's host thread while the run goes on; checkpoint_wait returns when it is done
    void write_checkpoint_async(const std::string& path) {
        check(g3d_write_checkpoint_async(ctx_, path.c_str()), ctx_, "write_checkpoint_async");
    }
    void checkpoint_wait() { check(g3d_checkpoint_wait(ctx_), ctx_, "checkpoint_wait"); }
    std::vector<g3d_particle> host_particles() {
        const int64_t n = status().np;
        std::vector<g3d_particle> v(size_t(n > 0 ? n : 0));
        int64_t got = 0;
        check(g3d_get_particles(ctx_, v.data(), n, &got), ctx_, "host_particles");
        v.resize(size_t(got));
        return v;
    }
    void set_particles(const std::vector<g3d_particle>& v) {
        check(g3d_set_particles(ctx_, v.data(), int64_t(v.size())), ctx_, "set_particles");
    }
    // the 19 weighted sums of Simulation::diagnostics (src/sim_output.cpp:10-26); sets the stop flag of the laser
    std::vector<double> diagnostics_sums() {
        std::vector<double> S(19, 0.0);
        check(g3d_diagnostics(ctx_, S.data()), ctx_, "diagnostics");
        return S;
    }
    // the first and the centred second moments of the beam species (bunches.txt), [group][8] each
    void beam_moments(std::vector<double>& s1, std::vector<double>& s2) {
        s1.assign(16 * 8, 0.0); s2.assign(16 * 8, 0.0);
        int32_t G = 0;
        check(g3d_beam_moments(ctx_, 16, s1.data(), s2.data(), &G), ctx_, "beam_moments");
        s1.resize(size_t(G) * 8); s2.resize(size_t(G) * 8);
    }
    // a real array of the reference layout (jw, the density lines rho_lines / rho_lines_i) as doubles
    std::vector<double> real_array(int32_t which) {
        size_t n = 0, eb = 0;
        check(g3d_array_info(ctx_, which, &n, &eb), ctx_, "array_info");
        if (eb != sizeof(double)) throw std::runtime_error("real_array: not an array of doubles");
        std::vector<double> v(n);
        check(g3d_get_array(ctx_, which, v.data(), n), ctx_, "get_array");
        return v;
    }
    g3d_status status() const {
        g3d_status st{};
        check(g3d_get_status(ctx_, &st), ctx_, "status");
        return st;
    }
    const Setup& setup() const { return s_; }
    g3d_ctx* ctx() { return ctx_; }

private:
    Setup s_;
    g3d_ctx* ctx_ = nullptr;
};

}  // namespace g3dshim
