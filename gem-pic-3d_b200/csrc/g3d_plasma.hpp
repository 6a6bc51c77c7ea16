// State of the streaming plasma (one rank): the device structs of k_plasma.cu and the host-side state of
// Simulation's plasma members (src/sim.hpp:292-311).
#pragma once
#include <functional>
#include <memory>
#include <vector>
#include "g3d_ctx.hpp"

namespace g3d {

// species codes of the reference (src/sim.hpp:29)
constexpr int SP_TRAPPED = 1, SP_PLASMA = 2, SP_ION = 3, SP_FREED = 50, SP_INJECTED = 100;

// one ADK level in code units (reference AdkLevel, src/ionization.hpp:197)
struct AdkDev { double logpre, power, expo, Epeak, Emin; };
// an ion species on the device (reference IonDev, src/sim.hpp:27)
struct IonDevC { double mass; int mobile, ionizing, Zmax, off; double Emin; };

// streaming particles as structure of arrays
struct StrmDev {
    double *x, *y, *zeta, *px, *py, *pz, *w, *z, *q, *qm;
    int32_t *alive, *sp;
    uint64_t* id;
};

// The values of a march that change from step to step. The kernels read them from device memory, so the graph
// of the slice loop, captured once, stays valid for every step.
struct StepVals {
    double s1, sTrap, X0, Y0;
    uint64_t key_step;         // ion_key_step(seed, istep)
    int i0, j0;                // the box column and row through the axis x = 0, y = 0 (the density lines)
};

struct StreamArgs {
    const float* __restrict__ F;
    Geo g;
    LaserDev laser;
    const StepVals* sv;
    double zc, Delta, vz_beam;
    double ylo, yhi;           // free-hand y: a particle beyond these (within a cell of a wall) is lost
    int n, pass;
    double* J;                 // jsr: jx, jy, jz, rho-, rho+ of the half-cell (real planes)
    float* Jf;                 // the same planes in FP32 (the mixed form)
    const IonDevC* ions;
    const AdkDev* adk;
    const StrmDev* sd;         // on the device: [0] the streaming particles, [1] the freed electrons (read at run
                               // time, so that the slice loop's graph outlives a move of either list)
    int* bcnt;
    int bcap;
    int dry;                   // a predictor pass: deposit and ionize, keep the particles as they were
    const void* Fmid;          // Fourier y: the six fields half-way between slices n and n+1, interleaved per point
                               // (FP32: 8 floats, FP64: 6 doubles per point), or null
    ExtDev ext;                // external magnetic elements (none: nu = nm = 0)
    double inv_dx, inv_dy;     // 1/dx, 1/dy (the mixed form's FP32 gathers and deposit)
    double dep_norm;           // 1 / (Delta h_n dx): the deposit factor of half-cell n per unit of q w dt (the mixed form's FP32 deposit)
    const double* Fd;          // exact fields (FP64 form, Fourier y, no ionization, no analytic wave): the F planes in FP64 for
                               // the gather of a particle that starts inside the half-cell (null: the float planes F)
    const struct RecDev* recd; // the same variant, recording for the adjoint: the state of every particle entering half-cell n
                               // (pass 0) into the record (null: none)
    double* rl[2];             // the last pass: the charge of the negative [0] and the positive [1] particles on the lines
                               // through the axis of half-cell n (row j0: nx values, column i0: ny values), or null
};

// The adjoint's record of one march, written by the recording slice loop (device pointers; rs the stride of a particle
// column): x the streaming particles' states (x, y, zeta, z, p_x, p_y, p_z) entering half-cell n at slot n + 1 and
// after the last half-cell at slot 0 (7 rs each); a their states alive at the same slots (rs each); q their q w (0 for a
// fixed ion, which carries no current) and q/m (2 rs); f the exact real fields of slice l after pass p (6 planes of nk
// at 6 nk (P l + p)).
struct RecDev {
    double* x;
    double* f;
    int32_t* a;
    double* q;
    long rs;
};

struct PlasmaPtrs {
    long nkh;
    void *jkx, *jky, *jkz;     // the window's jk: complex128, or complex64 in the mixed form
    cpx *js0x, *js0y, *js0z, *jsn, *sin_, *si0, *pin, *tmp, *dl;
};

struct IonSpec {
    double mass, atoms;
    int Z0, Zmax, mobile, ionization;
    std::vector<double> ip_eV;
    bool loaded() const { return mobile || ionization; }
};

// The fresh plasma lattice of a march (Simulation::load_plasma, src/sim_plasma.cpp:43-90) as the device builds it:
// lattice point L runs over the rows j0 .. j0 + nrows - 1, cells i, sub-cells b2, a2 (a2 fastest); a point of
// positive density gives m particles, the electron first (when free electrons are loaded), then one per loaded ion
// species in order. Every product, quotient and sum below is the host's, in the host's order, so the particles
// (and whether a point has any) are bit for bit those of the reference's loader.
constexpr int LAT_MAXION = 8;
struct LatticeArgs {
    int nx, px, py, j0, electrons, nion;
    long m;
    double dx, dy, X0, Y0, Delta, zf, s0;
    const double* yn;                          // free-hand y: the node positions (null: rows j dy, height dy)
    double f, n0, rmax2, depth, rc2;           // density n0 f g(r) for r^2 < rmax2, g = 1 + depth r^2 / rc2
    int parabolic;
    double ion_atoms[LAT_MAXION], ion_q[LAT_MAXION], ion_qm[LAT_MAXION];
    int ion_sp[LAT_MAXION];
    uint64_t id0;
};

// A DevBuf-backed structure of arrays of streaming particles.
struct StrmBuf {
    DevBuf<double> d;          // 10 columns
    DevBuf<int32_t> i;         // 2 columns
    DevBuf<uint64_t> u;        // ids
    StrmDev v{};
    long cap = 0;
    void alloc(long n, cudaStream_t s);
};

struct PlasmaState {
    g3d_plasma cfg{};
    std::vector<double> zpts, zvals;
    std::vector<IonSpec> ions;
    bool box_mean = true;
    bool any_ionizing = false;                 // some ion species ionizes (the streaming kernel's ADK path)
    // spectra of the streaming current: level s0 per half-cell (the prediction of the next step), the current
    // of one half-cell (jsr real, jsn spectra), the parts of jk held as predictions, backups
    DevBuf<cpx> js0x, js0y, js0z;              // ns+1 half planes
    DevBuf<double> jsr;                        // 5 real planes
    DevBuf<float> jsrf;                        // the same in FP32 (the mixed form)
    DevBuf<double> fmid;                       // the fields half-way through the half-cell, interleaved per point
    // the charge of the streaming particles of every half-cell n on the lines through the axis [N][nx + ny] (row j0,
    // column i0), deposited by the last pass: the negative particles, then (ion_lines) the positive ones
    DevBuf<double> rhol;
    bool ion_lines = false;                    // some ion species is loaded (mobile or ionizing)
    DevBuf<cpx> jsn, jsin, jpred, jtmp, jsi0, dlt, tsp;   // 3 half planes each
    DevBuf<cpx> bk;                            // 4 half planes: R_x, R_y, E_z, B_z of the slice
    StrmBuf s, bn;                             // streaming particles, the freed electrons
    StrmDev strm{}, born{};
    StrmDev sdh[2]{};                          // strm and born as the kernels of the slice loop read them (sdev)
    DevBuf<StrmDev> sdev;
    long nstrm = 0;                            // host copy (exact at the start of the march)
    long born_cap = 0, fresh_last = 0, trapped_total = 0, restreamed_total = 0;
    DevBuf<long> nstrm_dev;
    DevBuf<int> bcnt, flags;
    DevBuf<int> tally;                         // count of particles in a given state (count_state)
    DevBuf<IonDevC> ion_dev;
    DevBuf<AdkDev> adk_dev;
    std::vector<g3d_particle> joining;         // join the next march at their zeta (from the host: restreamed)
    StrmBuf jb;                                // the same on the device: the slow trapped particles of the last march
    long njb = 0;
    DevBuf<unsigned long long> ucount;
    // scratch of the lattice build and of the compaction of trapped particles: flags and their exclusive sums
    // (one entry more than the items), the scan's temporary storage, the trapped particles that join the beam
    DevBuf<int> cflag, coff;
    DevBuf<unsigned char> ctmp;
    StrmBuf tr;
    // the slice loop of a march as CUDA graphs, keyed by what they hold by value (two alternate: the j0 / jk
    // buffers swap every step); captured again only when a buffer moved
    struct LoopGraph { uint64_t key; cudaGraphExec_t exec; long launches; };
    std::vector<LoopGraph> loops;
    // the reverse of a march (the adjoint, k_adj_plasma.cu) as a CUDA graph, keyed like the loops
    struct AdjGraph { uint64_t key = 0; cudaGraphExec_t exec = nullptr; } adjg;
    DevBuf<StepVals> stepv;
    // recording for the adjoint march: when rec_on, march_plasma calls rec_step(nstrm, fresh) after loading its plasma
    // (it points recd at this march's record, or returns false: no record for this march) and the slice loop writes the
    // record through recd (RecDev), so one graph serves every march
    bool rec_on = false;
    std::function<bool(long, long)> rec_step;
    DevBuf<RecDev> recd;
    PlasmaPtrs ptrs(const Ctx& c) const;
    PlasmaState() = default;
    PlasmaState(const PlasmaState&) = delete;
    PlasmaState& operator=(const PlasmaState&) = delete;
    ~PlasmaState() {
        for (auto& l : loops) cudaGraphExecDestroy(l.exec);
        if (adjg.exec) cudaGraphExecDestroy(adjg.exec);
    }
};

// The adjoint of one march (k_adj_plasma.cu). The values of a step its kernels read from device memory:
struct AdjStepDev {
    const double* Fprev;       // the exact real fields of level s0
    double sTrap;
    long np;                   // the streaming particles of the march
    RecDev rec;                // the march's record
};
// The adjoint arrays of the window (device, half spectra):
struct AdjPlasmaPtrs {
    long nkh;
    cpx* lS[6];                // the spectra {R_x, R_y, E_z, B_z, L_x, L_y}, ns planes
    cpx* lj0[2];               // j0 x, y (ns + 1 planes)
    cpx* ljk[3];               // the beam current's jk x, y, z (ns + 1 planes)
    cpx* ljs0[3];              // js0 (ns + 1 planes)
    cpx* lsl[6];               // one slice: the adjoint of its values in one pass (one plane each)
    cpx *lold, *ljsnA, *ljsn, *ldl;      // 4, 3, 3, 3 planes
    cpx* lsi0[2];              // 3 planes each, by the parity of the half-cell
};
// ... and its scratch: the march's record (rec, np streaming particles, fresh of them the fresh plasma, the rest joining)
struct AdjPlasmaWs {
    long np, fresh;
    RecDev rec;
    double *lFup[2], *lFcur;   // 6 real planes each: the adjoints of a slice's real fields
    double* ljsr;              // 3 real planes: the adjoint of a pass's streaming deposit
    double* lam;               // 7 rec.rs: the adjoint of the streaming particles' state (x, y, zeta, z, p)
    double* jl;                // 7 rec.rs: the adjoint of the state of the joining particles carried to the step before
    AdjStepDev* stepd;         // the values of the step (device)
    cpx* Wsc[6];               // one plane each of transform scratch
    cpx* Tsc[3];
};
void adjoint_march_plasma(Ctx& c, const AdjPlasmaWs& w, const AdjPlasmaPtrs& a, const double* Fprev, double* lF, double s0,
                          double s1);
// The slow trapped particles of a march (alive 5 after it, v_z below vz_beam) in list order: they join the next march
// after its fresh plasma. launch_join_adjoint_out copies the adjoint of the state of the next march's joining particles
// (lam from index fresh, n of them) to jl; launch_join_adjoint_in puts jl onto those particles of the march recorded in
// rec (np of them; lam, 7 components of stride rec.rs). Both return how many particles they moved.
long launch_join_adjoint_out(Ctx& c, const double* lam, long rs, long fresh, long n, double* jl);
long launch_join_adjoint_in(Ctx& c, const RecDev& rec, long np, const double* jl, long njl, double* lam);
void launch_d2f(Ctx& c, const double* a, float* b, long n);     // b = float(a)
void launch_f2d(Ctx& c, const float* a, double* b, long n);     // b = double(a)

// launchers (k_plasma.cu)
void launch_record_particles(Ctx& c, int n);     // the adjoint's record of the particles entering half-cell n (-1: after)
void launch_record_fields(Ctx& c, int l, int p); // ... of the exact real fields of slice l after pass p
void launch_stream(Ctx& c, const StreamArgs& a);
void launch_slice_prologue(Ctx& c, int n, int pred_m, int copy_in, int backup);
void launch_pass_prologue(Ctx& c, int n, int restore);
void launch_stream_spectra(Ctx& c);
// Fourier y: the rows of the streaming current's spectra, then the fused column work of a pass (the current's
// y transforms and filters, the replace and march of slice n, the y transforms of slice n's fields into W)
void launch_stream_spectra_rows(Ctx& c);
void launch_pass_cols(Ctx& c, double D, int n, int extrap, double w, int restore);
void launch_replace(Ctx& c, int m, cpx* old, const cpx* nw);
void launch_replace_pred(Ctx& c, int n, int extrap, double w);
void launch_correct(Ctx& c, int n, double q, int own);
void launch_correct_prologue(Ctx& c, int n, double q, int own, int pred_m, int backup);
void launch_march_slice(Ctx& c, double D, int n);
void launch_born_append(Ctx& c);
// number of particles with alive == state among n (n_dev: the count on the device instead, when not null)
long count_state(Ctx& c, const int32_t* alive, long n, const long* n_dev, int state);
void launch_real_fields_slice(Ctx& c, int l, FmidOut fm = FmidOut(), bool cols = true);     // cols false: rows only (W given)
// the lattice points of positive density among npts (their running count into P.coff); returns how many
long launch_lattice_count(Ctx& c, const LatticeArgs& a, long npts);
// the fresh particles of those points into S[0 .. count m)
void launch_lattice_fill(Ctx& c, const LatticeArgs& a, long npts, StrmDev S);
// the trapped particles after a march: the slow ones appended to the device joining list (P.jb), the fast ones into
// P.tr; returns how many fast ones
long launch_trapped_split(Ctx& c, double s1);
// the freed-electron capacity the device joining list needs (ionizing ions); its x, y moved with the window
long launch_join_cap(Ctx& c);
void launch_join_shift(Ctx& c, double sx, double sy);

}  // namespace g3d
