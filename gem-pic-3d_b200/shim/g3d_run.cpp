// g3d_run: the reference's command line (src/main.cpp:26-121) with the march on the B200. It reads a GEM-PIC-3D
// deck with the reference's own deck and Config layers, maps it onto libg3d (setup_from), and runs init and the
// s-steps through g3dshim::Simulation:
//
//   g3d_run deck [--check] [--restart latest|STEP] [--precision fp64|mixed] [block.key=value ...]
//
// Written to output.dir: diag.txt and bunches.txt (the reference's columns, every output.every steps and the last;
// the beam moments from the device), checkpoints
// every output.checkpoint_every steps in the reference's layout and name (checkpoint_NNNNNN_r0000.bin, with the streaming
// plasma's state; written by the library's host thread while the next steps run, the last one waited for before
// "done"), and
// "done: N steps, X s" on stdout. With loaded ions diag.txt has the reference's last column, the largest ion charge
// density on the axis (from the library's density lines). Field files, particle dumps, frames, openPMD and the other
// output groups of the reference are not written. A deck key the library does not run stops it before any device
// work; exit codes as the reference's: 0 done, 2 error.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include "params_from.hpp"
#include "sim.hpp"

namespace {
constexpr double kC = 299792458.0, kE = 1.602176634e-19, kMe = 9.1093837015e-31, kEps0 = 8.8541878128e-12;

// The table keeps the lines of steps up to `step` on a restart (-1: a new table).
FILE* open_table(const std::string& file, long step) {
    if (step < 0) return std::fopen(file.c_str(), "w");
    std::ifstream in(file);
    std::string keep, line;
    while (std::getline(in, line)) {
        std::istringstream is(line);
        long st = 0;
        if (line.empty() || line[0] == '#' || ((is >> st) && st <= step)) keep += line + "\n";
    }
    FILE* f = std::fopen(file.c_str(), "w");
    if (f) std::fputs(keep.c_str(), f);
    return f;
}

// One line of diag.txt from the 19 sums of the library (the columns of the reference's table: moments in um, the
// laser's position in FWHM, field and kinetic energy in J, the trapped charge in pC).
void diag_line(FILE* f, const Config& c, g3dshim::Simulation& sim, bool header) {
    if (header)
        for (FILE* out : {f, stdout})
            if (out) std::fprintf(out, "# step  z[mm]  N_alive  <x>[um] <y>[um] <zeta>[um]  rms_x rms_y rms_zeta[um]  <px> <py> "
                                       "<pz> <gamma> <p.khat>  rms_pz  eta_rel[FWHM] a_env  W_field[J] W_kin[J]  N_trapped "
                                       "Q_trapped[pC]%s\n", c.mobile_ions() ? "  max_Zni/n0(axis)" : "");
    const std::vector<double> S = sim.diagnostics_sums();
    const g3d_status st = sim.status();
    const double w = S[0] > 0 ? S[0] : 1;
    auto mean = [&](int k) { return S[k] / w; };
    auto spread = [&](int k, int k2) { return std::sqrt(std::max(0.0, mean(k2) - mean(k) * mean(k))); };
    const double um = c.Lu * 1e6;
    double eta_rel = 0, a_env = 0;
    if (c.laser_on) {
        const double xi = mean(13) - c.start_fwhm * c.tau;
        eta_rel = xi / c.tau;
        a_env = c.a0 * std::exp(-2 * std::log(2.0) * xi * xi / (c.tau * c.tau));
    }
    const double Eu = kMe * kC * kC / (c.Lu * kE);             // field unit [V/m]
    const double W_field = S[15] * kEps0 * Eu * Eu * std::pow(c.Lu, 3);
    const double W_kin = (S[10] - S[0]) * c.nc * std::pow(c.Lu, 3) * kMe * kC * kC;
    const double Q_tr = S[18] * c.nc * std::pow(c.Lu, 3) * kE * 1e12;
    char line[600];
    std::snprintf(line, sizeof line,
                  "%6ld %10.5f %8ld %10.4f %10.4f %10.4f %9.4f %9.4f %9.4f %12.6e %12.6e %14.8e %14.8e %14.8e %11.4e %8.4f "
                  "%8.4f %11.4e %11.4e %8ld %11.4e\n",
                  long(st.istep), st.s * c.Lu * 1e3, long(S[14]), mean(1) * um, mean(2) * um, mean(3) * um,
                  spread(1, 4) * um, spread(2, 5) * um, spread(3, 6) * um, mean(7), mean(8), mean(9), mean(10), mean(11),
                  spread(9, 12), eta_rel, a_env, W_field, W_kin, long(S[17]), Q_tr);
    if (c.mobile_ions()) {             // the largest ion charge density on the axis (src/sim_output.cpp:44-51)
        const std::vector<double> rl = sim.real_array(G3D_A_RHO_I);
        const int nx = c.nx, ny = c.ny, N = int(rl.size() / size_t(nx + ny));
        const int i0 = ((int(std::lround(-st.X0 / (c.Lx / nx))) % nx) + nx) % nx;
        double mx = 0;
        for (int n = 0; n + 1 < N; ++n) mx = std::max(mx, rl[size_t(n) * size_t(nx + ny) + size_t(i0)] / c.n0);
        const size_t l = std::strlen(line);
        std::snprintf(line + l - 1, sizeof line - l + 1, " %11.4e\n", mx);
    }
    for (FILE* out : {f, stdout})
        if (out) { std::fputs(line, out); std::fflush(out); }
}

// bunches.txt: per output step one line per beam species (the reference's columns: N, Q [pC], E [MeV], dE/E,
// sig_x, sig_y, eps_nx, eps_ny [um], <zeta>, sig_z [um], <x>, <y> [um]) from the device moments
void bunches_lines(FILE* f, const Config& c, g3dshim::Simulation& sim, bool header) {
    if (!f) return;
    if (header)
        std::fprintf(f, "# step  z[mm]  bunch  N  Q[pC]  E[MeV]  dE/E(rms)  sig_x[um]  sig_y[um]  eps_nx[um]  eps_ny[um]  "
                        "<zeta>[um]  sig_z[um]  <x>[um]  <y>[um]    (trapped = self-injected plasma electrons, inj_<ion> "
                        "= from field ionization)\n");
    std::vector<double> s1, s2;
    sim.beam_moments(s1, s2);
    const g3d_status st = sim.status();
    const double pC = c.nc * std::pow(c.Lu, 3) * kE * 1e12, um = c.Lu * 1e6;
    const std::vector<std::string> names = c.beam_names();
    for (size_t g = 0; g < names.size() && 8 * g < s1.size(); ++g) {
        const double* a = &s1[8 * g];
        const double* b = &s2[8 * g];
        const double w = a[0];
        auto mean = [&](int k) { return w > 0 ? a[2 + k] / w : 0.0; };
        auto var = [&](int k) { return w > 0 ? b[k] / w : 0.0; };
        const double gm = mean(5);
        const double ex = std::sqrt(std::max(0.0, var(0) * var(3) - var(5) * var(5)));
        const double ey = std::sqrt(std::max(0.0, var(1) * var(4) - var(6) * var(6)));
        std::fprintf(f, "%6ld %10.5f %-12s", long(st.istep), st.s * c.Lu * 1e3, names[g].c_str());
        std::fprintf(f, " %10ld %12.6f %13.6f %10.3e %10.5f %10.5f %10.5f %10.5f %11.4f %10.4f %11.5f %11.5f\n", long(a[1]),
                     w * pC, w > 0 ? (gm - 1) * 0.51099895 : 0.0, gm > 0 ? std::sqrt(var(7)) / gm : 0.0,
                     std::sqrt(var(0)) * um, std::sqrt(var(1)) * um, ex * um, ey * um, mean(2) * um, std::sqrt(var(2)) * um,
                     mean(0) * um, mean(1) * um);
    }
    std::fflush(f);
}

std::string checkpoint_name(const std::string& dir, long step) {
    char fn[64];
    std::snprintf(fn, sizeof fn, "/checkpoint_%06ld_r0000.bin", step);
    return dir + fn;
}
long latest_checkpoint(const std::string& dir) {
    long best = -1;
    if (!std::filesystem::is_directory(dir)) return best;
    for (const auto& e : std::filesystem::directory_iterator(dir)) {
        long st = 0; int r = 0;
        if (std::sscanf(e.path().filename().string().c_str(), "checkpoint_%ld_r%d.bin", &st, &r) == 2 && r == 0 && st > best)
            best = st;
    }
    return best;
}
}  // namespace

int main(int argc, char** argv) {
    try {
        if (argc < 2)
            throw std::runtime_error("usage: g3d_run deck [--check] [--restart latest|STEP] [--precision fp64|mixed] "
                                     "[block.key=value ...]");
        Deck d = Deck::read(argv[1]);
        bool check = false;
        long restart = -2;                                  // -2: none, -1: the latest checkpoint
        int precision = G3D_PREC_FP64;
        for (int i = 2; i < argc; ++i) {
            if (!std::strcmp(argv[i], "--check")) check = true;
            else if (!std::strcmp(argv[i], "--restart")) {
                if (i + 1 >= argc) throw std::runtime_error("--restart needs latest or a step");
                restart = !std::strcmp(argv[++i], "latest") ? -1 : std::stol(argv[i]);
            } else if (!std::strcmp(argv[i], "--precision")) {
                if (i + 1 >= argc) throw std::runtime_error("--precision needs fp64 or mixed");
                const std::string v = argv[++i];
                if (v == "mixed") precision = G3D_PREC_MIXED;
                else if (v != "fp64") throw std::runtime_error("--precision: fp64 or mixed, not " + v);
            } else d.override_from(argv[i]);
        }
        const Config c = Config::from_deck(d);
        g3dshim::Setup setup = g3dshim::setup_from(c);        // refuses what the library does not run
        setup.precision = precision;
        c.summary(stdout, 1);
        std::printf("  march: %s, %s form\n", g3d_version(), precision == G3D_PREC_MIXED ? "mixed" : "FP64");
        if (check) return 0;
        std::filesystem::create_directories(c.dir);
        g3dshim::Simulation sim(setup);
        long rs = -1;
        if (restart != -2) {
            rs = restart == -1 ? latest_checkpoint(c.dir) : restart;
            if (rs < 0) throw std::runtime_error("--restart latest: no checkpoint in " + c.dir);
            sim.read_checkpoint(checkpoint_name(c.dir, rs));
            std::printf("restart after step %ld\n", rs);
        } else {
            sim.init();
        }
        FILE* f = open_table(c.dir + "/diag.txt", rs);
        if (!f) throw std::runtime_error("cannot write " + c.dir + "/diag.txt");
        FILE* fb = open_table(c.dir + "/bunches.txt", rs);
        if (rs < 0) { diag_line(f, c, sim, true); bunches_lines(fb, c, sim, true); }
        const auto t0 = std::chrono::steady_clock::now();
        long steps = 0;
        long istep = sim.status().istep;
        while (!sim.finished()) {
            sim.step();
            ++steps; ++istep;
            if (c.every > 0 && istep % c.every == 0) { diag_line(f, c, sim, false); bunches_lines(fb, c, sim, false); }
            if (c.checkpoint_every > 0 && istep % c.checkpoint_every == 0)
                sim.write_checkpoint_async(checkpoint_name(c.dir, istep));
        }
        sim.checkpoint_wait();
        if (c.every <= 0 || istep % c.every) { diag_line(f, c, sim, false); bunches_lines(fb, c, sim, false); }
        std::fclose(f);
        if (fb) std::fclose(fb);
        const double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::printf("done: %ld steps, %.1f s\n", istep, sec);
        (void)steps;
        return 0;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 2;
    }
}
