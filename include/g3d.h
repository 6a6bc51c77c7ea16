/*
 * g3d.h -- C-ABI of the B200-native per-zeta-slice march of GEM-PIC-3D.
 *
 * The library (libg3d.so, hand-written sm_100a CUDA) replaces from below the reference's
 * `class Simulation` (src/sim.hpp:222-360) for the hot path: push, current deposit,
 * zeta filter, transverse FFTs, per-mode march, sponge, real fields, window shift and the
 * diagnostics reductions. Every entry point is `extern "C"`, takes plain pointers and
 * sizes, and returns an int status (G3D_OK = 0). A non-zero status leaves a message in
 * g3d_last_error(). Calls are synchronous at the ABI: they return after the work queued on
 * the context's own CUDA stream has finished, unless the name ends in `_async`.
 * One context = one GPU = one host thread (the reference runs one host thread per rank). A context keeps the
 * device that was current at g3d_create and makes it current at the start of every call that takes the context,
 * so a caller may switch devices between calls.
 *
 * Units are the reference's code units (README.md:43-45): c = 1, lengths 1/k0, times
 * 1/omega0, momenta m c, fields m c omega0 / e, densities n_c.
 */
#ifndef G3D_H
#define G3D_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Opaque context: one march on one GPU. */
struct g3d_ctx;
typedef struct g3d_ctx g3d_ctx;

/* ------------------------------------------------------------------ status codes */
#define G3D_OK            0
#define G3D_ERR_CUDA      1   /* a CUDA call failed (reference: gpu_check, src/portable.hpp:43-49) */
#define G3D_ERR_TIMEOUT   2   /* a bounded device-side wait gave up */
#define G3D_ERR_CAPACITY  3   /* a fixed-capacity list overflowed (the list of electrons freed by ionization is
                                 sized for every level of every ion; the environment variable
                                 G3D_BORN_CAPACITY_LIMIT = n > 0 caps it at n to exercise this check) */
#define G3D_ERR_ARG       4   /* an invalid argument (sizes, grid, unknown array id) */
#define G3D_ERR_STATE     5   /* an entry point called in the wrong state */
#define G3D_ERR_IO        6   /* checkpoint file missing, truncated or not a checkpoint */
#define G3D_ERR_NODEV     7   /* no CUDA device visible to this process */

/* ------------------------------------------------------------------ forms */
#define G3D_FP64   0          /* plain form: FP64 throughout, float F as in the reference */
#define G3D_MIXED  1          /* mixed FP32/FP64 form */

/* laser envelope of the analytic plane wave */
#define G3D_ENV_GAUSSIAN 0    /* reference Laser::envelope, src/sim.hpp:195 */
#define G3D_ENV_FLATTOP  1    /* flat top with sin^2 ramps (no counterpart in the reference) */

/* polarisation of the analytic plane wave (reference Laser::pol, src/sim.hpp:192) */
#define G3D_POL_S        0    /* E along y */
#define G3D_POL_P        1    /* E in the x-z plane */
#define G3D_POL_CIRCULAR 2

/* ------------------------------------------------------------------ records */
/* One macro-particle, byte for byte the reference's `struct Particle` (src/sim.hpp:217, 104 B):
 * this is the layout of checkpoints and of g3d_set/get_particles. On the device the library
 * keeps the particles as structure-of-arrays. */
typedef struct g3d_particle {
    double x, y, zeta, px, py, pz, w, rem, z, q, qm;
    int32_t alive, sp;
    uint64_t id;
} g3d_particle;

/* Grid (reference Config grid fields, src/sim.hpp:38-44). */
typedef struct g3d_grid {
    int32_t nx, ny, nzeta;
    int32_t y_fourier;          /* 1: Fourier y (periodic); 0: free-hand y between walls (table ynode) */
    double Lx, Ly;
    const double* zeta;         /* nzeta slice positions, zeta[0] = 0 (rear) ... zeta[nzeta-1] = window */
    const double* ynode;        /* ny+1 node positions of the free-hand y grid, NULL for Fourier y */
} g3d_grid;

/* Run parameters (reference Config, src/sim.hpp:36-187, the subset on the march path). */
typedef struct g3d_params {
    double lambda0;             /* reference wavelength [m] (sets the unit of length 1/k0) */
    double dz, dz_push, z_end;  /* s-step, longest particle sub-step, end of the run */
    double sponge, sponge_y, sponge_rate;
    int32_t move_x, move_y, window_lag;
    int32_t self_fields, zeta_filter, k_filter;
    double push_phase;          /* rad of laser phase per RK4 sub-step */
    /* analytic plane-wave laser (reference Laser, src/sim.hpp:191-210) */
    int32_t laser_on, laser_pol, laser_envelope, reserved0;
    double a0, kL, theta, tau, cep;
    double eta_c;               /* pulse centre in eta (reference: start_fwhm * tau, sim_setup.cpp:54) */
    double stop_fwhm;           /* stop when <eta> - eta_c > stop_fwhm * tau (0: never) */
    double flat_length, ramp_length;   /* G3D_ENV_FLATTOP: plateau length and sin^2 ramp length */
    double zeta_center;         /* zeta of the bunch centre (time origin of the push, PushCtx.zc) */
    int32_t freeze_bunch, start_relax, box_mean, precision;
} g3d_params;

/* A Gaussian or flat-top bunch block (reference Config::Bunch, src/sim.hpp:61-81, the built-in
 * profiles of sim_bunches.cpp:151-158; shot_noise = random). */
typedef struct g3d_bunch {
    double charge_C;            /* |charge| [C] */
    double gamma, sigx, sigy, sigz, length;   /* length > 0: flat top in z instead of sigz */
    double emitx, emity, espread, zeta_center, x0, y0;
    double q;                   /* charge number: -1 electrons, +1 positrons */
    int64_t nmacro;
    uint64_t seed;
    /* shot noise: beamlet <= 1 random (the default); beamlet = M >= 3: Fawley's beamlets (Phys. Rev. ST Accel.
     * Beams 5, 070701 (2002); deck shot_noise = fawley): nmacro / M groups of M particles spread evenly over
     * noise_lambda, displaced so that their bunching at the harmonics h < M/2 is that of the real electrons */
    int32_t beamlet, reserved;
    double noise_lambda;
} g3d_bunch;

/* Streaming plasma (reference Config plasma keys, src/sim.hpp:103-116 and 129): a regular lattice of
 * ppc_x x ppc_y electrons per transverse cell, loaded at the front of the window every s-step, with the ions
 * of the ion blocks at the same points; n = n0 f(z) g(r) for r < r_max. */
typedef struct g3d_plasma {
    double n0;                  /* density [n_c] */
    double r_max;               /* plasma only where r < r_max (1e300: everywhere) */
    double channel_depth, r_channel;   /* parabolic: g(r) = 1 + channel_depth r^2 / r_channel^2 */
    double smooth_length;       /* smoothing 1 / (1 + a^2 k_perp^2) of the streaming current (0: none) */
    double vz_min, vz_beam, trap_advance;
    const double* z_points;     /* longitudinal profile f(z): n_z points, linear between, constant beyond */
    const double* z_values;
    int32_t n_z, ppc_x, ppc_y, iterations;
    int32_t predictor_extrapolate, free_electrons, parabolic, box_mean;
    uint64_t seed;              /* random numbers of the ionization (reference: the first bunch block's seed) */
} g3d_plasma;

/* An ion species (reference Config::IonSpecies, src/sim.hpp:118-127). */
typedef struct g3d_ion {
    double mass;                /* [m_e] */
    double atoms;               /* n_atom / n_e of the plasma profile */
    const double* ip_eV;        /* ionization energies [eV]: ip_eV[k] of k -> k+1, n_ip entries */
    int32_t n_ip, Z0, Zmax, mobile, ionization, reserved;
} g3d_ion;

/* A Gaussian laser on the grid (reference Config::GridLaser, src/sim.hpp:95-101, type = gaussian):
 * R = 2 E_perp of a paraxial beam focused at z_focus, added at the start (Simulation::add_grid_lasers). */
typedef struct g3d_grid_laser {
    double a0, kL, waist, tau, zeta_c, z_focus, cep, pol_angle;
    int32_t circular, helicity;
} g3d_grid_laser;

/* External magnetic elements acting on the particles (reference struct Undulator / Magnet, src/external.hpp:15-30; the
 * deck blocks undulator, quadrupole, plasma_lens, solenoid, as Config::parse_external builds them,
 * src/sim_external.cpp:5-85). Code units: B in m omega0 / e, lengths 1/k0, z the lab position. Undulator: B0 = K k_u,
 * linear ramps of `ramp` at both ends between z0 and z1; planar (B_y, with natural focusing B_y cosh, B_z sinh) or
 * helical (B_x, B_y); nk > 0: a taper, B0(z0 + j dzk) = ktab[koff + j]. Magnet kind 0 quadrupole (gradient g),
 * 1 plasma lens (gradient g inside radius R), 2 solenoid (field g, linear fringes of `ramp`); dsmax the longest push
 * sub-step inside it. */
typedef struct g3d_undulator {
    int32_t helical, focusing;
    double ku, B0, z0, z1, ramp;
    int32_t nk, koff;
    double dzk;
} g3d_undulator;
typedef struct g3d_magnet {
    int32_t kind, reserved;
    double z0, z1, g, R, ramp, dsmax;
} g3d_magnet;

/* A thin chicane at the lab position z (reference Config::Chicane, src/sim.hpp; deck block chicane, code units): every
 * beam particle moves in zeta by r56 (gamma / gamma_ref - 1) - delay. */
typedef struct g3d_chicane {
    double z, r56, delay, gamma_ref;
} g3d_chicane;

/* Scalars of the run (reference members s, istep, X0, Y0, beta_b, gm2_b, np, lost_total). */
typedef struct g3d_status {
    double s, X0, Y0, beta_b, gm2_b, field_energy;
    int64_t istep, np, lost, stop;
} g3d_status;

/* Array ids for g3d_array_info / g3d_get_array / g3d_set_array / g3d_device_ptr.
 * Layouts are the reference's (src/sim.hpp:265-301): spectra [l][j][ix] complex128
 * (l = slice 0..N-1 or half-cell plane 0..N), jw [comp][hw][j][ix] double (3 x (N+3) planes),
 * F [comp][fl][j][ix] float (6 x (N+2) planes). The density lines rho_lines and rho_lines_i
 * (src/sim.hpp:299-301) are [n][nx + ny] double: the charge of the negative (RHO_E) and of the
 * positive (RHO_I) streaming particles of half-cell n in its last pass on the row through the axis
 * (nx values) and on the column through it (ny values); 0 elements without a plasma, and RHO_I
 * without a loaded ion species. */
#define G3D_A_RX   0
#define G3D_A_RY   1
#define G3D_A_EZ   2
#define G3D_A_BZ   3
#define G3D_A_LX   4
#define G3D_A_LY   5
#define G3D_A_J0X  6
#define G3D_A_J0Y  7
#define G3D_A_JKX  8
#define G3D_A_JKY  9
#define G3D_A_JKZ  10
#define G3D_A_JW   11
#define G3D_A_F    12
#define G3D_A_RHO_E 13
#define G3D_A_RHO_I 14
#define G3D_A_COUNT 15

/* ------------------------------------------------------------------ lifetime */
/* Creates a context on the current CUDA device: device buffers of the reference layouts,
 * k-tables, zeta weights. Replaces Simulation::Simulation (src/sim_setup.cpp:5-60). Transverse
 * sizes: nx a power of two in 8..512 or three times one in 24..384; ny the same (from 4) with
 * Fourier y, 3..512 with free-hand y; any other size is G3D_ERR_ARG. */
int g3d_create(const g3d_grid* grid, const g3d_params* params, struct g3d_ctx** out);
void g3d_destroy(struct g3d_ctx* ctx);
/* Message of the last failed call on this context (or of the last failed g3d_create when
 * ctx is NULL). Never NULL. */
const char* g3d_last_error(const struct g3d_ctx* ctx);
/* Library version string. */
const char* g3d_version(void);

/* ------------------------------------------------------------------ particles */
/* Replaces Simulation::set_particles / host_particles (src/sim_setup.cpp:166-175). */
int g3d_set_particles(struct g3d_ctx* ctx, const g3d_particle* parts, int64_t n);
int g3d_get_particles(struct g3d_ctx* ctx, g3d_particle* out, int64_t capacity, int64_t* n);
/* Bunch loading on the host with the reference's random sequence (std::mt19937_64 with
 * std::normal_distribution, src/sim_bunches.cpp:92-217), then uploaded. Sets X0, Y0. */
int g3d_load_bunches(struct g3d_ctx* ctx, const g3d_bunch* bunches, int32_t count);
/* The same sampling without a context or a device: fills `out` (capacity records) with the loaded
 * particles, `n` their count, `lost` those outside the window, X0/Y0 the box origin. The message of a
 * failure is g3d_last_error(NULL). */
int g3d_sample_bunches(const g3d_grid* grid, const g3d_params* params, const g3d_bunch* bunches, int32_t count,
                       g3d_particle* out, int64_t capacity, int64_t* n, int64_t* lost, double* X0, double* Y0);

/* Plasma and ion species (before g3d_init; the ion tables are built here, src/sim_ions.cpp:68-87). */
int g3d_set_plasma(struct g3d_ctx* ctx, const g3d_plasma* plasma, const g3d_ion* ions, int32_t nions);
/* A grid laser, added to R by g3d_init (Simulation::add_grid_lasers, src/sim_fields.cpp:321-374). */
int g3d_add_grid_laser(struct g3d_ctx* ctx, const g3d_grid_laser* laser);
/* The external elements of the run (replaces any set before; nu = nm = 0 removes them). Their fields are added to the
 * gathered fields of the beam push and of the streaming push at the lab position, and the beam push's sub-steps end on
 * their breakpoints (reference add_external / external_step, src/external.hpp:40-92, used at
 * src/sim_kernels.hpp:88 and :126-133 and src/sim_stream.hpp:133). The adjoint march rejects a run with them. */
int g3d_set_external(struct g3d_ctx* ctx, const g3d_undulator* undulators, int32_t nu, const g3d_magnet* magnets,
                     int32_t nm, const double* ktab, int32_t nktab);
/* The thin chicanes of the run (replaces any set before; n = 0 removes them). A step that passes one (s0 < z <= s1)
 * ends with it (reference Simulation::apply_chicanes, src/sim_external.cpp:108-151): the beam's co-moving field of
 * the old positions is taken out of R and that of the new positions put in (vacuum at the chicane; the radiation in
 * the window stays), particles leaving the window are lost, and E_z, B_z, L and the real fields follow from R as at
 * the start. */
int g3d_set_chicanes(struct g3d_ctx* ctx, const g3d_chicane* chicanes, int32_t n);

/* ------------------------------------------------------------------ sharded runs (zeta slabs over ranks)
 * The reference's MPI zeta decomposition (Simulation::Simulation, src/sim_setup.cpp:9-15; Comm, src/comm.hpp:11-46)
 * with its march over the ranks replaced by a transpose: rank r of `world` holds the slices [a, b) of the window
 * (the reference's split: N / world each, the first N % world ranks one more, at least 4) and its beam particles
 * (zeta >= zeta[a + 1] below the next rank's bound; rank 0 everything below), and pushes, deposits, transforms,
 * sponges and turns into real fields only those. The march and the co-moving solve, serial in zeta but independent
 * per mode, run on mode pencils: before them an all-to-all moves the slab's planes of the modes [m0, m1) of every
 * rank to that rank, which then holds all N slices of its modes; after them a second all-to-all moves the results
 * back. Between neighbours, as in the reference: the three top raw current half-cells go up (sim_particles.cpp:
 * 108-119), the filtered j_z ghost half-cells both ways (:210-226), the two lowest real-field slices down
 * (sim_fields.cpp:295-306), and the particles that crossed below zeta[a + 1] down, which finish their push there
 * (sim_particles.cpp:28-48). Sums over the ranks: the deposit's bound (its fixed-point scale is then global, so the
 * current planes are those of one rank holding every particle), the beta sums, the centroid, the diagnostics (the
 * field energy of the slabs and the particles lost in the exchange included) and the beam moments.
 *
 * The library does no communication itself: it calls the caller's `comm` function on the context's thread, its stream
 * synchronized, with DEVICE buffers (G3D_COMM_SUM: `count` values at `data` replaced by their sum over the ranks,
 * `kind` G3D_SUM_F64 or G3D_SUM_I64; G3D_COMM_ALLTOALL: `send` holds world blocks of send_bytes[q] bytes, the q-th for
 * rank q, and `recv` receives world blocks of recv_bytes[r] bytes, the r-th from rank r; host count arrays). It
 * returns 0, or non-zero to fail the call with G3D_ERR_CUDA. Every rank makes the same calls in the same order, so
 * the library's collectives match. g3d_set_ranks comes after g3d_create and before particles are loaded; the run
 * must be FP64 with Fourier y and without plasma, chicanes, checkpoints or the adjoint march (G3D_ERR_STATE). What
 * stays this rank's own: the arrays of g3d_get_array (this slab's planes), g3d_get_particles, g3d_set_particles (the
 * caller gives this rank's particles), g3d_get_status and g3d_beam_beta_sums_static. */
#define G3D_COMM_SUM 0
#define G3D_COMM_ALLTOALL 1
#define G3D_SUM_F64 0
#define G3D_SUM_I64 1
typedef struct g3d_comm_op {
    int32_t op, kind;                            /* G3D_COMM_*, G3D_SUM_* */
    int64_t count;                               /* G3D_COMM_SUM: values at data */
    void* data;
    const void* send;                            /* G3D_COMM_ALLTOALL */
    const int64_t* send_bytes;                   /* [world] */
    void* recv;
    const int64_t* recv_bytes;                   /* [world] */
} g3d_comm_op;
typedef int (*g3d_comm_fn)(void* user, const g3d_comm_op* op);
int g3d_set_ranks(struct g3d_ctx* ctx, int32_t rank, int32_t world, g3d_comm_fn comm, void* user);
/* The partition, host arithmetic only: out = {a, b, m0, m1}, the slab [a, b) of the nzeta slices and the pencil
 * [m0, m1) of the nkh = ny (nx/2 + 1) stored modes of rank `rank` of `world` (G3D_ERR_ARG below 4 slices a rank). */
int g3d_shard_layout(int32_t nzeta, int64_t nkh, int32_t rank, int32_t world, int64_t out[4]);
/* One copy of a transpose: `rows` rows of `cols` elements from src (row stride src_stride) to dst (dst_stride),
 * offsets in elements; an array index of -1 is the send (pack) or receive (unpack) buffer, else the index into the
 * list of arrays given to g3d_shard_transpose_plan. */
typedef struct g3d_block {
    int64_t src, dst, rows, cols, src_stride, dst_stride;
    int32_t src_array, dst_array;
} g3d_block;
#define G3D_SLAB_NODES 0                          /* a slab array of ns planes (slices a .. b-1) */
#define G3D_SLAB_HALF 1                           /* of ns + 1 half-cell planes (a - 1/2 .. b - 1/2) */
/* The plan of the slab -> pencil transpose (to_pencil = 1) or back (0) of `narrays` arrays of the given kinds, on rank
 * `rank`: the copies into the send buffer (pack), the copies out of the receive buffer (unpack) and the byte counts of
 * the all-to-all for an element of elem_bytes. A pencil array holds N (nodes) or N + 1 (half cells) planes of m1 - m0
 * modes. A plan with more blocks than the capacity fails with G3D_ERR_CAPACITY and sets the counts. */
int g3d_shard_transpose_plan(int32_t nzeta, int64_t nkh, int32_t rank, int32_t world, const int32_t* kinds, int32_t narrays,
                             int32_t to_pencil, int64_t elem_bytes, g3d_block* pack, int32_t pack_cap, int32_t* npack,
                             g3d_block* unpack, int32_t unpack_cap, int32_t* nunpack, int64_t* send_bytes,
                             int64_t* recv_bytes);

/* ------------------------------------------------------------------ the march path */
int g3d_init(struct g3d_ctx* ctx);                  /* Simulation::init, sim_setup.cpp:178-197 (after loading) */
int g3d_step(struct g3d_ctx* ctx);                  /* Simulation::step, sim_setup.cpp:199-217 */
int g3d_step_async(struct g3d_ctx* ctx);            /* the same, without the final stream synchronisation */
int g3d_solve_fields(struct g3d_ctx* ctx, double D);/* Simulation::solve_fields, sim_fields.cpp:309-317 */
int g3d_currents(struct g3d_ctx* ctx);              /* Simulation::currents, sim_particles.cpp:56-207 */
int g3d_march(struct g3d_ctx* ctx, double D);       /* Simulation::march, sim_fields.cpp:7-39 */
int g3d_sponge_and_real_fields(struct g3d_ctx* ctx);/* sim_fields.cpp:156-307 */
int g3d_push(struct g3d_ctx* ctx, double s0, double s1);   /* Simulation::push, sim_particles.cpp:6-24 */
int g3d_comoving_field(struct g3d_ctx* ctx);        /* Simulation::comoving_field, sim_fields.cpp:44-151 */
int g3d_relax_start_field(struct g3d_ctx* ctx);     /* sim_fields.cpp:384-410 */

/* Arithmetic of the march. G3D_PREC_FP64 (default): FP64 throughout, the reference's arithmetic.
 * G3D_PREC_MIXED: no counterpart in the reference (FP64 only) - deposit (FP32 atomics), zeta filter (compensated
 * FP32 sums), transverse FFTs, the E_z/B_z/L march, the sponge and the real fields in FP32 / complex64, with FP64
 * kept for the s-level accumulator R_x, R_y and for the particles (with streaming plasma: FP32 gathers and
 * streaming deposit, FP64 particle state and Boris pushes). Set before g3d_init (G3D_ERR_STATE after it). Arrays
 * keep the reference layouts and types at the boundary (g3d_get_array widens, g3d_set_array rounds). */
#define G3D_PREC_FP64  0
#define G3D_PREC_MIXED 1
int g3d_set_precision(struct g3d_ctx* ctx, int32_t mode);

/* Largest particle count g3d_beam_beta_sums_static accepts (its scratch: 2 doubles per particle, 16 MiB). */
#define G3D_BETA_STATIC_MAX 1048576
/* No counterpart in the reference: an added entry point that allocates no device memory. out[0] = sum of w v_z,
 * out[1] = sum of w over the alive particles, in index order: the sums g3d_comoving_field takes the bunch's beta
 * from (beta = out[0] / out[1]; reference sim_fields.cpp:45-51), bit for bit. Its scratch is a static device
 * array of the library instead of a per-call buffer (g3d_comoving_field allocates 16 bytes per particle per call),
 * for callers that must not allocate: a window state that fills the device, or an allocator the caller owns. More than
 * G3D_BETA_STATIC_MAX particles: G3D_ERR_CAPACITY, nothing launched. The scratch is shared by every context of
 * the process on one device, so calls on one device must not overlap in time (they would race on it). The first
 * call on a device may load the library's device code (the address lookup of the scratch), so make it once
 * before any stream capture. Synchronous: returns after the sums have reached `out`. */
int g3d_beam_beta_sums_static(struct g3d_ctx* ctx, double out[2]);
int g3d_shift_window(struct g3d_ctx* ctx, int32_t nxs, int32_t nys);  /* sim_setup.cpp:249-281 */
/* The march of a step with streaming plasma (Simulation::march_plasma, src/sim_plasma.cpp:228-470), after
 * g3d_currents of level s1; g3d_step calls it when a plasma is set. */
int g3d_march_plasma(struct g3d_ctx* ctx, double s0, double s1);
/* Streaming particles of the last march (the reference's `strm`, 104-byte records). */
int g3d_get_streaming(struct g3d_ctx* ctx, g3d_particle* out, int64_t capacity, int64_t* n);

/* ------------------------------------------------------------------ diagnostics */
/* The 19 weighted sums of Simulation::diagnostics (src/sim_output.cpp:10-26) before the
 * rank reduction: S[0..13] weighted moments of the alive bunch particles (1, X, Y, zeta, X^2,
 * Y^2, zeta^2, px, py, pz, gamma, p.khat, pz^2, eta), S[14] their count, S[15] field energy
 * (code units), S[16] lost particles, S[17] count and S[18] charge of trapped particles. */
int g3d_diagnostics(struct g3d_ctx* ctx, double out[19]);
/* Moments of the beam species for bunches.txt (Simulation::write_bunches, src/sim_bunch_diag.cpp:42-80), on the
 * device in a fixed order, two passes (the second moments centred on the first's means). Groups g: the bunch blocks
 * 0 .. nbunch-1, then the trapped plasma electrons, then the electrons injected from each ion species (the reference's
 * beam_index); *ngroups = their number, at most 16 (G3D_ERR_CAPACITY if above `capacity`). Per group, of the alive
 * particles with v = (x, y, zeta, u_x, u_y, gamma), x and y physical: s1[8 g ..] = sum w, count, sum w v[0..5];
 * s2[8 g ..] = sum w d0^2, w d1^2, w d2^2, w d3^2, w d4^2, w d0 d3, w d1 d4, w d5^2 with d = v - mean. */
int g3d_beam_moments(struct g3d_ctx* ctx, int32_t capacity, double* s1, double* s2, int32_t* ngroups);
/* Field energy of the slices in code units (Simulation::local_field_energy, sim_output.cpp:55-77). */
int g3d_field_energy(struct g3d_ctx* ctx, double* out);
int g3d_get_status(const struct g3d_ctx* ctx, g3d_status* out);

/* ------------------------------------------------------------------ arrays (reference layouts) */
int g3d_array_info(const struct g3d_ctx* ctx, int32_t which, size_t* count, size_t* elem_bytes);
int g3d_get_array(struct g3d_ctx* ctx, int32_t which, void* host, size_t count);
int g3d_set_array(struct g3d_ctx* ctx, int32_t which, const void* host, size_t count);
/* Device pointer of an array (valid until the next call that reallocates; j0/jk swap each step). */
void* g3d_device_ptr(struct g3d_ctx* ctx, int32_t which);

/* ------------------------------------------------------------------ checkpoints */
/* Binary checkpoint of the reference (src/sim_checkpoint.cpp:9-58), one rank, bit-compatible. */
int g3d_write_checkpoint(struct g3d_ctx* ctx, const char* path);
int g3d_read_checkpoint(struct g3d_ctx* ctx, const char* path);
/* Asynchronous checkpoint, the same file as g3d_write_checkpoint (no counterpart in the reference, whose checkpoint
 * stops the run while it is written): the state is copied on the device on the context's stream, so the calls that
 * follow (g3d_step ...) may change it at once, and a host thread of the library brings the copy to the host and writes
 * the file (path + ".tmp", renamed to path when complete) while the march goes on. The copy takes device memory of about
 * the state's size, kept for the next checkpoint. One at a time per context: a second call, g3d_write_checkpoint,
 * g3d_read_checkpoint and g3d_checkpoint_wait wait for the one in flight; g3d_checkpoint_wait (and the next of these
 * calls) returns its outcome (G3D_ERR_IO if the file could not be written); g3d_destroy waits for it too. */
int g3d_write_checkpoint_async(struct g3d_ctx* ctx, const char* path);
int g3d_checkpoint_wait(struct g3d_ctx* ctx);

/* ------------------------------------------------------------------ stream, timing */
/* The context's CUDA stream (a cudaStream_t) on which every kernel is launched. */
void* g3d_stream(struct g3d_ctx* ctx);
int g3d_synchronize(struct g3d_ctx* ctx);
/* Per-kernel timing with CUDA events on the context stream: enable (1) / disable (0) and reset. */
int g3d_profile_enable(struct g3d_ctx* ctx, int32_t on);
/* Number of kernels timed so far; name, launches and total milliseconds of kernel k. */
int32_t g3d_profile_count(const struct g3d_ctx* ctx);
int g3d_profile_get(struct g3d_ctx* ctx, int32_t k, const char** name, int64_t* launches, double* total_ms);
/* Kernel launches issued on this context since creation (all kernels, profiled or not). */
int64_t g3d_launch_count(const struct g3d_ctx* ctx);

/* ------------------------------------------------------------------ adjoint march (no reference counterpart) */
/* Laser mode coefficients: every grid laser's R spectrum added at init (Simulation::add_grid_lasers,
 * src/sim_fields.cpp:321-373) is multiplied per stored mode by a(j, kx) = coef[2 (j H + kx)] + i coef[2 (j H + kx) + 1]
 * (ky index j = 0..ny-1, kx = 0..nx/2, H = nx/2 + 1); NULL sets every a to 1. Takes effect at the next g3d_init. */
int g3d_set_laser_modes(struct g3d_ctx* ctx, const double* coef);
/* Exact fields (1) or not (0): the real fields are kept in FP64 beside the float F and the beam push gathers
 * from them (and, with a streaming plasma on the Fourier y grid, the streaming push: its midpoint fields and the
 * gathers of particles joining inside a half-cell); the differentiable forward of which central differences are
 * taken. FP64 form; takes effect at the next g3d_init. */
int g3d_set_exact_fields(struct g3d_ctx* ctx, int32_t on);
/* What grad_p of g3d_adjoint differentiates (no counterpart in the reference). G3D_ADJ_THROUGH_START (the default):
 * the momenta as loaded, before g3d_init, so the derivative runs through the start field the bunch makes (its
 * currents, its beta, the relaxation) as well as through the s-steps. G3D_ADJ_AFTER_START: the momenta right after
 * g3d_init with the start field held, i.e. through the s-steps alone. Any other mode: G3D_ERR_ARG. */
#define G3D_ADJ_THROUGH_START 0
#define G3D_ADJ_AFTER_START   1
int g3d_set_adjoint_momenta(struct g3d_ctx* ctx, int32_t mode);
/* The adjoint march, right after g3d_init (Fourier y, beam and grid lasers, sponge 0, fixed window):
 * nsteps s-steps forward with per-level checkpoints of the beam and the real fields, J = sum w p_z / sum w over
 * the live beam, then the reverse sweep. With a streaming plasma (the FP64 form with exact fields or the mixed form; no
 * ionization, no analytic laser): the levels also keep the spectra, j0, js0 and the particles waiting to join the
 * plasma, each march is recorded (its particles entering every half-cell, the slices' fields after every pass) and
 * transposed; the records of all steps are kept when they fit in half the free device memory, else (or with the
 * environment variable G3D_ADJ_RECOMPUTE set) each step is run again from its level in the reverse sweep (the FP64
 * form only: the mixed form then gives G3D_ERR_CAPACITY). Trapping is kept as
 * the forward took it (slow trapped electrons joining later marches are differentiated); a forward in which a
 * particle joins the beam (fast trapped or restreamed) gives G3D_ERR_STATE. Out: *objective = J; grad_modes (NULL: skipped; needs
 * g3d_set_laser_modes) = dJ/d Re a + i dJ/d Im a per stored mode, 2 ny H doubles; grad_p (NULL: skipped) =
 * dJ/d(p_x, p_y, p_z) of every particle at s = 0, 3 np doubles [particle][component], through the s-steps and
 * (unless g3d_set_adjoint_momenta chose G3D_ADJ_AFTER_START) through the start field the bunch made at g3d_init
 * (its currents, its beta, the relaxation). The run is left at
 * s = nsteps dz; g3d_set_particles + g3d_init start the next evaluation on the same context (the checkpoint
 * workspace is kept between calls). */
int g3d_adjoint(struct g3d_ctx* ctx, int32_t nsteps, double* objective, double* grad_modes, double* grad_p);

#ifdef __cplusplus
}
#endif
#endif /* G3D_H */
