"""Benchmark of the march: particle-pushes/s including the field solve, mixed FP32/FP64 form against the FP64
form, one B200 per rank, with the error of the mixed form stated against the FP64 form.

Workload (default, 3): laser wakefield with streaming plasma, 256 x 256 Fourier modes, 2048 zeta slices (h = 0.2),
plasma 0.002 n_c with 2 x 2 electrons per cell and mobile H+ ions (596,496 streaming particles per step, each
pushed through all 2,047 half-cells, two passes), Gaussian grid laser a0 = 2, w0 = 20, FWHM 30, and a witness bunch
of 4,194,304 macro-electrons; s-step 10. One step = push of the bunch (RK4) + deposit + zeta filter + FFT pair +
the half-cell-by-half-cell plasma march (Boris push, deposit, spectra, prediction, march and real fields of each
slice, correction) + sponge + real fields: Simulation::step of the reference. Pushes per step = beam particles +
streaming particles. The state (about 12 GB in FP64) is larger than L2.
Workload 2: the oblique plane wave on a dense bunch (128 x 128 x 1024, 1,048,576 macro-electrons, no plasma).
Workload 5: ionization injection on free-hand y and zeta grids (256 Fourier modes x 193 graded y nodes between walls,
4096 graded slices, neutral H2 + 1 % N with ADK over every level, 16,440,320 streaming macro-particles per step).

    python bench.py [--gpus N --steps K --warmup W] [--impl g3d|reference] [--workload 1|2|3|5]

Both forms are timed on the same inputs; value is the mixed form, fp64_form the FP64 form, mixed_error the
relative L2 of F and the relative <p_z> of the mixed form against the FP64 form after the same steps. At N = 1
the key adjoint holds the adjoint march's cost against the forward and its agreement with central differences on
workload 4 without its plasma (--no-adjoint skips it).
Under torchrun (N > 1), workloads 3 and 5 (streaming plasma: one serial chain of half-cells) run an independent
replica per rank (scaling weak); workloads 1 and 2 (no plasma) run ONE window sharded over the ranks in zeta slabs,
the march on mode pencils through NCCL all-to-alls (FP64 form, scaling strong; --replicas keeps replicas). Timed on
the device, max over ranks; value = pushes of all ranks / that time.
--impl reference times the reference GEM-PIC-3D CPU/OpenMP build (oracle/_ref) on the host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "gem-pic-3d_b200"))

METRIC = "particle-pushes/s incl. field solve, mixed vs FP64 form, 1 B200, stated error"
UNIT = "pushes/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="g3d", choices=["g3d", "reference"])
    ap.add_argument("--workload", type=int, default=3, choices=[1, 2, 3, 5])
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint march check on workload 4")
    ap.add_argument("--no-error-growth", action="store_true", help="skip the mixed form's error by s-steps")
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"],
                    help="both: time the FP64 form, then the mixed form (the headline) and its error against FP64")
    ap.add_argument("--nzeta", type=int, default=None, help="profiling case: fewer slices (same window)")
    ap.add_argument("--particles", type=int, default=None, help="profiling case: fewer macro-particles")
    ap.add_argument("--replicas", action="store_true", help="N > 1 on workloads 1-2: replicas instead of one sharded run")
    ap.add_argument("--adjoint-plasma", type=int, default=0, metavar="K",
                    help="profiling case: only one adjoint evaluation of workload 4 with its plasma over K s-steps (after "
                         "one untimed evaluation), printing its device time")
    return ap.parse_args()


def sharded(a, world):
    """One window over the ranks (zeta slabs, mode pencils): workloads without plasma on more than one GPU."""
    return world > 1 and a.workload in (1, 2) and not a.replicas


def workload(k, nzeta=None, particles=None):
    from g3d import configs
    kw = {}
    if nzeta:
        kw["nzeta"] = nzeta
    if particles:
        kw["ppc" if k == 5 else "nmacro"] = particles
    return configs.baseline(k, **kw)


def lattice_particles(cfg):
    """Streaming macro-particles loaded per step: the lattice points of the cells (inside the walls on the free-hand
    y grid) times the species (electrons when free, and every ion species)."""
    if cfg.plasma is None:
        return 0
    from g3d import configs
    pd = configs.default_plasma()
    pd.update(cfg.plasma)
    rows = cfg.ny if cfg.ynode is None else cfg.ny - 2
    species = (1 if pd["free_electrons"] else 0) + len(cfg.ions)
    return cfg.nx * rows * pd["ppc_x"] * pd["ppc_y"] * species


def config_json(cfg, k, form="fp64", parallelism="replicas"):
    what = (f"{cfg.particles} macro-electrons" if cfg.particles else
            f"{lattice_particles(cfg)} streaming macro-particles per step")
    return {"workload": f"{k}: {cfg.name}, {cfg.nx}x{cfg.ny} modes x {cfg.nzeta} slices, "
                        f"{what}, {'mixed FP32/FP64' if form == 'mixed' else 'FP64'} form",
            "form": form,
            "nx": cfg.nx, "ny": cfg.ny, "nzeta": cfg.nzeta, "particles": cfg.particles,
            "grid_points": cfg.grid_points, "dz": cfg.params["dz"], "sponge": cfg.params.get("sponge", 0),
            "laser_envelope": "flattop" if cfg.params.get("laser_envelope") == 1 else "gaussian",
            "l2": f"inputs larger than L2 (field state {state_bytes(cfg) / 1e9:.2f} GB, F {f_bytes(cfg) / 1e9:.2f} GB)",
            "parallelism": parallelism}


def state_bytes(cfg):
    """Device bytes of the spectral state: six fields and five current planes, half spectra of complex128."""
    gh = (cfg.nzeta - 1) * cfg.ny * (cfg.nx // 2 + 1)
    return 11 * 16 * gh


def f_bytes(cfg):
    return 6 * (cfg.nzeta + 1) * cfg.nx * cfg.ny * 4


# ------------------------------------------------------------------ algorithmic bytes per launch (FP64)
def algorithmic_bytes(name, cfg, mixed=False, S=0):
    """Per-launch algorithmic bytes of each kernel: what it must read and write once, in the layout this build keeps.

    G = grid points (slices x nx x ny; F carries 6 floats = 24 B, the raw currents 3 values = 24 B in FP64, 12 B
    in the mixed form); Gh = half-spectrum points of a slice set (slices x ny x (nx/2 + 1)); a spectrum costs
    16 B per Gh as complex128 and 8 B as complex64 (the mixed form keeps R in complex128 and the rest in
    complex64). The spectra of real fields are Hermitian, so the kept half is the minimum a transform pass has to
    move. P = beam particles: the push reads x, y, zeta, px, py, pz, z, w (64 B) and writes 48 B (both forms);
    the deposit reads 56 B.
    The per-half-cell kernels of the plasma march work on one slice: nk = nx ny points, nkh = ny (nx/2 + 1) modes,
    S = streaming particles, each read (80 B) and written (64 B) once per half-cell pass (the per-unit figure of
    the streaming push), with the midpoint fields it gathers from (6 doubles or 8 floats per point) and the three
    deposit planes."""
    ns = cfg.nzeta - 1
    nk = cfg.nx * cfg.ny
    G = ns * nk
    Gh = ns * cfg.ny * (cfg.nx // 2 + 1)
    Gc = (ns + 1) * cfg.ny * (cfg.nx // 2 + 1)      # current planes carry one more half-cell
    P = cfg.particles
    nkh = cfg.ny * (cfg.nx // 2 + 1)
    cz = 8 if mixed else 16                          # bytes of a stored spectrum value other than R
    cr = 4 if mixed else 8                           # bytes of a raw current value
    fm = 32 if mixed else 48                         # bytes of the midpoint fields per point
    march_slice = (4 * 16 + 10 * cz + 6 * cz) * nkh + (2 * 16 + 4 * cz) * nkh
    # jsn, sin, js0 (2), dl, pin read; jk (2 half-cells) read and written; sin, pin written (3 components each)
    replace_pred = (6 * 48 + 2 * 3 * cz) * nkh + (2 * 3 * cz + 2 * 48) * nkh
    slice_prologue = (48 + 96 + 48 + 2 * 3 * cz + 48 + 32 + 2 * cz + 64) * nkh
    correct = (48 + 32 + 32 + 48 + 32 + 48 + 48) * nkh  # jsn, si0, R, js0 read; R, dl, js0 written
    plasma = {
        "stream": 144 * S + fm * nk + 3 * cr * nk,
        # Fourier y: the rows alone: the deposit planes read and cleared (FP32: (jx, jy, jz, 0) per point), three
        # complex128 half rows written
        "stream_spectra": 2 * (16 if mixed else 24) * nk + 48 * nkh,
        # the fused column work of a pass: the half rows read, jsn written, the replace and march of the slice
        # (less its read of jsn), the six column transforms of the slice's fields written (their inputs stay in
        # shared memory)
        "pass_cols": 48 * nkh + 48 * nkh + replace_pred + march_slice - 48 * nkh + 6 * cz * nkh,
        "march_slice": march_slice,
        "real_cols_slice": (2 * 16 + 4 * cz + 6 * cz) * nkh,
        # six column transforms read, F written; the other F plane read and the midpoint fields written
        "real_rows_slice": 6 * cz * nkh + 24 * nk + (24 + fm) * nk,
        "replace_pred": replace_pred,
        "slice_prologue": slice_prologue,
        "correct_prologue": correct + slice_prologue,
        "pass_prologue": 3 * cr * nk + 64 * nkh,
    }
    if name in plasma:
        return plasma[name] if S else None
    if not mixed:
        table = {
            "push": 112 * P + 24 * G,          # particles read 64 + written 48; F read 24 per grid point
            "deposit": 56 * P + 24 * G,        # particles read 56; raw currents written 24 per grid point
            "cur_rows": 24 * G + 48 * Gc,      # raw currents read 24; three complex planes written
            "cur_cols": 48 * Gc + 48 * Gc,     # three complex planes read and written (jkx, jky, jkz)
            "march": (9 + 6) * 16 * Gh,        # R, E_z, B_z, j0 (2), jk (3) read; R, E_z, B_z, L written
            "sponge_cols_inv": (2 + 1 + 3) * 16 * Gh,   # R read, j_z read; U, V, psi written
            "sponge_rows": 4 * 16 * Gh,        # U, V read and written
            "sponge_cols_fwd": (3 + 2) * 16 * Gh,       # U, V, psi read; R written
            "real_cols": 12 * 16 * Gh,         # six spectra read, six column transforms written
            "real_rows": 6 * 16 * Gh + 24 * G,  # six column transforms read; F written
        }
    else:
        table = {
            "push": 112 * P + 24 * G,
            "deposit": 56 * P + 12 * G,        # FP32 raw currents
            "cur_rows": 12 * G + 24 * Gc,
            "cur_cols": 24 * Gc + 24 * Gc,
            "march": (7 * 8 + 2 * 16) * Gh + (4 * 8 + 2 * 16) * Gh,   # E_z, B_z, j read, R read; E, B, L and R written
            "sponge_cols_inv": (2 * 16 + 8 + 2 * 8) * Gh,   # R, j_z read; U, V written
            "sponge_rows": 4 * 8 * Gh,
            "sponge_cols_fwd": (2 * 8 + 4 * 16) * Gh,        # U, V read; R read and written (R + dR)
            "real_cols": (2 * 16 + 4 * 8 + 6 * 8) * Gh,      # R, L, E_z, B_z read; six column transforms written
            "real_rows": 6 * 8 * Gh + 24 * G,
        }
    return table.get(name)


# ------------------------------------------------------------------ clocks during the timed region
class ClockSampler:
    def __init__(self, bus_id=None):
        self.bus_id = (bus_id or "").lower()
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        q = ("pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        rows = self.rows
        if self.bus_id:
            mine = [r for r in rows if r and self.bus_id.endswith(r[0].lower()[-12:])]
            rows = mine or rows
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 4 + k and r[4 + k].lower() in ("active", "1"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ CPU baseline: the reference build
def reference_config(cfg):
    from g3d import abi
    if cfg.params.get("laser_envelope") == abi.G3D_ENV_FLATTOP:
        # the reference has only the Gaussian envelope: same pulse centre, FWHM = the plateau length
        import copy
        cfg = copy.deepcopy(cfg)
        cfg.params.update(laser_envelope=abi.G3D_ENV_GAUSSIAN, tau=cfg.params.get("flat_length", 60.0))
    return cfg


SAMPLE_SLICES = (256, 512)      # the reference's sample windows of a plasma workload, at the workload's own h


def sample_config(cfg, k, n):
    """The plasma workload k (configured as cfg) on a window of n slices at cfg's slice step h: the transverse grid,
    plasma, ions, laser and witness unchanged, a shorter window."""
    from g3d import configs
    if k != 3:
        raise ValueError(f"no sampled window for workload {k}")
    return configs.config3(nzeta=n, h=cfg.h, nmacro=cfg.particles)


def reference_rate(cfg, steps, threads, k=None, warmup=0):
    """Reference CPU/OpenMP build on `threads` host threads: (pushes/s, description of the sample, ms per step)
    or (None, why, None).

    Without plasma: init and `warmup` s-steps (untimed), then `steps` s-steps of the full workload. With plasma one
    step of the full window takes minutes on a host (about 5 min on 8 cores for 2048 slices), so the sample is the
    same workload on two shorter windows at the workload's own slice step h (SAMPLE_SLICES slices; the transverse
    grid, plasma, ions, laser and witness are the workload's): init and `warmup` s-steps untimed, then `steps` timed
    s-steps per window. The step time is t(N) = a + b N in the slice count N (the beam push and deposit of the
    witness and the per-step set-up in a; the half-cell march of the streaming plasma, the same work per slice at a
    fixed h, in b), fitted through the two windows and evaluated at the workload's nzeta. A fit that is not
    increasing in N, or a non-positive step time, returns (None, why, None) rather than a number. Pushes per step =
    beam particles + the streaming particles of the last step (loaded per step from the transverse lattice, the same
    count at any window length)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import ref
    if not ref.available():
        return None, "oracle/_ref/libg3dref.so not built", None
    if cfg.plasma is None:
        r = ref.RefSimulation(reference_config(cfg), threads=threads)
        r.load_bunch()
        r.init_fields()
        for _ in range(warmup):
            r.step()
        t0 = time.perf_counter()
        for _ in range(steps):
            r.step()
        dt = time.perf_counter() - t0
        r.close()
        return cfg.particles * steps / dt, (f"the full workload, init and {warmup} s-steps untimed, then {steps} "
                                            f"timed s-steps, OpenMP on {threads} threads"), dt / steps * 1e3
    if k == 5:
        return reference_rate_lattice(cfg, steps, threads, warmup)
    if k is None or cfg.nzeta <= SAMPLE_SLICES[-1]:
        return None, "no sampled windows for this workload", None
    pts = []
    S = 0
    for nz in SAMPLE_SLICES:
        c2 = reference_config(sample_config(cfg, k, nz))
        if c2.particles != cfg.particles or abs(c2.h - cfg.h) > 1e-12 * cfg.h:
            return None, f"sample window of {nz} slices does not keep the workload's h and particles", None
        r = ref.RefSimulation(c2, threads=threads)
        r.init()
        for _ in range(warmup):
            r.step()
        t0 = time.perf_counter()
        for _ in range(steps):
            r.step()
        pts.append((nz, (time.perf_counter() - t0) / steps))
        S = len(r.streaming_particles())
        r.close()
    (n1, t1), (n2, t2) = pts
    b = (t2 - t1) / (n2 - n1)
    t_full = t1 + b * (cfg.nzeta - n1)
    if not (b > 0) or not (t_full > 0):
        return None, (f"reference sample not increasing in the slice count ({n1}: {t1:.2f} s, {n2}: {t2:.2f} s per "
                      f"step); no extrapolation"), None
    return (cfg.particles + S) / t_full, (
        f"{steps} timed s-step(s) per window after an untimed init and {warmup} untimed s-step(s), on windows of "
        f"{n1} and {n2} slices at the workload's h = {cfg.h:g} (same 256x256 transverse grid, plasma, ions, laser and "
        f"witness; {t1:.2f} s and {t2:.2f} s per step), t = a + b N fitted through them and evaluated at N = "
        f"{cfg.nzeta} ({t_full:.1f} s per step); pushes = {cfg.particles} beam + {S} streaming particles; OpenMP on "
        f"{threads} threads"), t_full * 1e3


LATTICE_SAMPLE = (256, (1, 2))    # workload 5's reference sample: slices, and lattice points per cell along x, y


def reference_rate_lattice(cfg, steps, threads, warmup):
    """Workload 5 on the reference: its 16.4 M streaming macro-particles a step through 4,096 slices would take the
    reference hours a step. The sample is the workload's grids and gas on a window of 256 graded slices with 1 x 1 and
    2 x 2 lattice points per cell: the step time is t = a + b S in the streaming particles S of a step (the lattice and
    the electrons freed from it; the field work of the 256 slices in a, the streaming push in b), fitted through the
    two; the full step is then (a + b S_full) x (nzeta - 1) / 255, the work of every term growing with the half-cells
    a particle crosses, S_full the full lattice with the same share of freed electrons as the larger sample. A fit that
    is not increasing in S returns (None, why, None)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import ref
    from g3d import configs
    if not ref.available():
        return None, "oracle/_ref/libg3dref.so not built", None
    n_s, ppcs = LATTICE_SAMPLE
    pts = []
    for ppc in ppcs:
        c2 = configs.config5(nzeta=n_s, ppc=ppc)
        r = ref.RefSimulation(c2, threads=threads)
        r.init()
        for _ in range(warmup):
            r.step()
        t0 = time.perf_counter()
        for _ in range(steps):
            r.step()
        dt = (time.perf_counter() - t0) / steps
        pts.append((len(r.streaming_particles()), dt, lattice_particles(c2)))
        r.close()
    (s1, t1, _), (s2, t2, l2) = pts
    b = (t2 - t1) / (s2 - s1)
    S = lattice_particles(cfg) * s2 / l2          # the lattice and the electrons the gas frees, as in the sample
    t_full = (t1 + b * (S - s1)) * (cfg.nzeta - 1) / (n_s - 1)
    if not (b > 0) or not (t_full > 0):
        return None, f"reference sample not increasing in the particle count ({t1:.2f} s, {t2:.2f} s)", None
    return S / t_full, (
        f"{steps} timed s-step(s) per sample after an untimed init and {warmup} untimed s-step(s), on a window of "
        f"{n_s} graded slices of the workload's grids with {s1} and {s2} streaming particles a step (1 x 1 and 2 x 2 per "
        f"cell; {t1:.2f} s and {t2:.2f} s per step), t = a + b S fitted and scaled to {S:.0f} particles and "
        f"{cfg.nzeta} slices ({t_full:.0f} s per step); OpenMP on {threads} threads"), t_full * 1e3


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ------------------------------------------------------------------ rank aggregation
def max_over_ranks(value, dist=None):
    """Largest value over the ranks (device time of the slowest replica). NCCL needs a CUDA tensor,
    gloo a CPU one."""
    if dist is None or not dist.is_initialized():
        return float(value)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, steps, world, ms_max):
    """Whole-job throughput: the units every rank advanced, over the slowest rank's time."""
    return units_per_rank * steps * world / (ms_max * 1e-3)


# ------------------------------------------------------------------ the reference arm
def run_reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cfg = workload(a.workload, a.nzeta, a.particles)
    cores = host_cores()
    # per sample window: at most 1 warm-up and 2 timed s-steps, so that the arm ends in a few minutes (a 512-slice
    # step of the laser-plasma workload takes ~45 s on 16 host cores)
    steps = max(1, min(a.steps, 2))
    warm = max(0, min(a.warmup, 1))
    v, why, ms = reference_rate(cfg, steps, cores, a.workload, warmup=warm)
    if v is None:
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return
    sample = why
    if cfg.params.get("laser_envelope") == 1:
        sample += " (Gaussian envelope of FWHM 60 in place of the flat top, which the reference lacks)"
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": a.gpus,
                      "steps": steps, "warmup": warm, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                      "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded bunch sampler of the reference)",
                      "config": config_json(cfg, a.workload),
                      "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
                      "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


# ------------------------------------------------------------------ our arm
def min_warmup(a):
    """Warm-up s-steps: at least 3 (the benchmark's rule); workload 5, whose full step runs for minutes, at least 1."""
    return max(a.warmup, 1 if a.workload == 5 else 3)


def time_form(cfg, precision, a, world, dist, local):
    """Init, warm-up, then K device-timed steps of one form; per-kernel event times on the context stream."""
    import torch
    import g3d
    comm = None
    if sharded(a, world):
        from g3d import shard
        comm = shard.RankComm(device=f"cuda:{local}")
    sim = g3d.Simulation(cfg, precision=precision, comm=comm)
    sim.init()
    stream = torch.cuda.ExternalStream(sim.stream_ptr())
    for _ in range(min_warmup(a)):
        sim.step()
    # pushes per step: the beam list, plus with plasma the streaming particles that cross the window in one march
    S = sim.streaming_count() if cfg.plasma is not None else 0
    P = int(sim.status().np) + S
    if comm is not None:                       # a sharded run: the pushes of all ranks, as one replica's
        t = torch.tensor([float(P)], device=f"cuda:{local}")
        dist.all_reduce(t)
        P = int(t.item())
    props = torch.cuda.get_device_properties(local)
    bus = getattr(props, "pci_bus_id", None)
    bus = f"{bus:02x}:00.0" if isinstance(bus, int) else None
    clocks = ClockSampler(bus)
    l0 = sim.launch_count()
    clocks.start()
    time.sleep(0.6)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sim.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(a.steps):
        sim.step_async()
    e1.record(stream)
    e1.synchronize()
    sim.synchronize()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    clk = clocks.stop()
    launches = sim.launch_count() - l0
    # per-kernel CUDA events in a separate pass: events around every kernel add gaps, and the plasma march is
    # launched as one graph only when no events are recorded
    sim.profile(True)
    for _ in range(max(1, min(a.steps, 5))):
        sim.step_async()
    sim.synchronize()
    prof = sim.profile_results()
    sim.profile(False)
    mixed = precision == "mixed"
    kernels = {k: {"launches": n, "avg_ms": round(t / max(1, n), 5), "share": round(t / sum(v[1] for v in prof.values()), 4),
                   "GB/s": (round(algorithmic_bytes(k, cfg, mixed, S) / (t / max(1, n) * 1e-3) / 1e9, 1)
                            if algorithmic_bytes(k, cfg, mixed, S) else None)}
               for k, (n, t) in sorted(prof.items(), key=lambda kv: -kv[1][1])}
    reps = 1 if comm is not None else world
    out = {"sim": sim, "P": P, "stream": stream, "ms": ms, "value": job_rate(P, a.steps, reps, ms), "clk": clk,
           "launches": launches, "prof": prof, "kernels": kernels, "reps": reps}
    if comm is not None:
        out["comm_calls"] = comm.calls
    if S:
        from g3d import configs
        pd = configs.default_plasma()
        pd.update(cfg.plasma)
        it = int(pd["iterations"])
        out["streaming"] = {"particles_per_step": S, "beam_particles": P - S,
                            "half_cell_updates_per_s": S * (cfg.nzeta - 1) * it * a.steps * world / (ms * 1e-3)}
    return out


def roofline(form, cfg, workload, mixed):
    import json as _json
    peaks_path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak, peak_src = float(_json.load(open(peaks_path))["hbm_gbs"]), "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    name, (n_launch, tot_ms) = max(form["prof"].items(), key=lambda kv: kv[1][1])
    avg_ms = tot_ms / max(1, n_launch)
    ab = algorithmic_bytes(name, cfg, mixed, (form.get("streaming") or {}).get("particles_per_step", 0))
    achieved = ab / (avg_ms * 1e-3) / 1e9 if ab else None
    traffic = None
    tpath = os.path.join(REPO, "profiles", "traffic.json")
    if os.path.exists(tpath):
        traffic = _json.load(open(tpath)).get(f"{workload}:{'mixed:' if mixed else ''}{name}")
    return {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak if achieved else None, "traffic": traffic, "peak_source": peak_src,
            "algorithmic_bytes_per_launch": ab, "avg_launch_ms": avg_ms}


def end_to_end(form, a, world, dist):
    """The same metric through the C-ABI with host buffers: every step uploads the particle records from pinned
    host memory (g3d_set_particles), steps (g3d_step) and reads the records and the diagnostics back."""
    import ctypes
    import torch
    import g3d
    sim, P, stream = form["sim"], form["P"], form["stream"]
    Pb = int(sim.status().np)                  # beam records crossing the boundary (P adds the streaming plasma)
    nb = Pb * g3d.PARTICLE_DTYPE.itemsize
    cap = Pb + Pb // 8 + 1024                  # trapped plasma electrons join the beam list
    host = torch.empty(cap * g3d.PARTICLE_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True)
    parts = host.numpy().view(g3d.PARTICLE_DTYPE)
    parts[:Pb] = sim.host_particles()
    out = torch.empty(cap * g3d.PARTICLE_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True)
    outp = out.numpy().view(g3d.PARTICLE_DTYPE)
    n = Pb
    lib, ctx = sim.lib, sim.ctx
    diag = (ctypes.c_double * 19)()
    got = ctypes.c_int64()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    x0 = torch.cuda.Event(enable_timing=True)
    x1 = torch.cuda.Event(enable_timing=True)
    x0.record(stream)
    for _ in range(a.e2e_steps):
        sim._c(lib.g3d_set_particles(ctx, parts.ctypes.data, n))          # inputs: H2D from pinned memory
        sim._c(lib.g3d_step(ctx))
        sim._c(lib.g3d_get_particles(ctx, outp.ctypes.data, cap, ctypes.byref(got)))  # result: D2H
        sim._c(lib.g3d_diagnostics(ctx, diag))
        n = got.value
        parts, outp = outp, parts
    x1.record(stream)
    x1.synchronize()
    wall = time.perf_counter() - t0
    ems = max_over_ranks(max(x0.elapsed_time(x1), wall * 1e3), dist)
    return {"value": job_rate(P, a.e2e_steps, form.get("reps", world), ems), "unit": UNIT,
            "h2d_bytes_per_step": nb, "d2h_bytes_per_step": nb + 19 * 8, "steps": a.e2e_steps,
            "path": "g3d_set_particles (pinned host records) -> g3d_step -> g3d_get_particles + g3d_diagnostics"}


def run_g3d(a):
    import numpy as np
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    cfg = workload(a.workload, a.nzeta, a.particles)
    forms = ["fp64", "mixed"] if a.precision == "both" else [a.precision]
    if sharded(a, world):
        forms = ["fp64"]                        # a sharded run is FP64
    res = {}
    ref_state = None
    err = None
    for prec in forms:
        f = time_form(cfg, prec, a, world, dist, local)
        # the state after warm-up + K steps, for the error of the mixed form against the FP64 form
        F = f["sim"].array("F") if len(forms) > 1 else None
        d = f["sim"].diagnostics_sums()
        if prec == "fp64":
            ref_state = (F, d)
        elif ref_state is not None:
            F0, d0 = ref_state
            rl = lambda x, y: float(np.linalg.norm(x.astype(np.float64) - y) / np.linalg.norm(y.astype(np.float64)))
            err = {"F": rl(F, F0), "<p_z>": abs(d[9] / d[0] - d0[9] / d0[0]) / abs(d0[9] / d0[0]),
                   "field_energy": abs(f["sim"].field_energy() - ref_state_energy) / abs(ref_state_energy),
                   "after_steps": min_warmup(a) + a.steps + max(1, min(a.steps, 5)),   # warm-up, timed, profiled
                   "note": "relative L2 of the float F (all six components) and relative <p_z>, mixed vs FP64 form on the same "
                           "inputs, same GPU"}
        if prec == "fp64":
            ref_state_energy = f["sim"].field_energy()
        if prec == forms[-1] and a.e2e_steps > 0:
            f["e2e"] = end_to_end(f, a, world, dist)
        f["sim"].close()
        res[prec] = f
    head = forms[-1]
    H = res[head]
    mixed = head == "mixed"

    # ---------------- CPU baseline on rank 0 at N = 1
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cores = host_cores()
        # the reference arm's sample with one warm-up and one timed s-step per window (about 2-3 min of host time
        # for the laser-plasma workload on 16 cores; 3 steps of the full workload without plasma)
        v, why, _ = reference_rate(cfg, 1 if cfg.plasma is not None else 3, cores, a.workload, warmup=1)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "reference", "sample": "reference OpenMP build: " + why}

    if dist:
        dist.barrier()
    if rank == 0:
        line = {"metric": METRIC, "value": H["value"], "unit": UNIT, "n_gpus": world, "steps": a.steps,
                "warmup": min_warmup(a), "ms_per_step": H["ms"] / a.steps, "higher_is_better": True,
                "scaling": "strong" if sharded(a, world) else "weak",
                "vs_baseline": None, "dtype": "f32+f64 (mixed form)" if mixed else "f64",
                "data": "synthetic (seeded bunch sampler of the reference)",
                "config": config_json(cfg, a.workload, head,
                                      f"zeta slabs x mode pencils over {world} ranks (NCCL all-to-all)"
                                      if sharded(a, world) else "replicas"),
                "roofline": roofline(H, cfg, a.workload, mixed),
                "kernels": H["kernels"], "e2e": H.get("e2e"), "gpu_launches": H["launches"], "clocks": H["clk"],
                "cpu_baseline": cpu}
        if "streaming" in H:
            line["streaming"] = H["streaming"]
        if world == 1 and not a.no_adjoint:
            line["adjoint"] = adjoint_check()
        if world == 1 and mixed and "fp64" in res and not a.no_error_growth:
            line["mixed_error_growth"] = error_growth(cfg)
        if "fp64" in res and mixed:
            F64 = res["fp64"]
            line["fp64_form"] = {"value": F64["value"], "ms_per_step": F64["ms"] / a.steps, "dtype": "f64",
                                 "roofline": roofline(F64, cfg, a.workload, False), "kernels": F64["kernels"],
                                 "gpu_launches": F64["launches"], "clocks": F64["clk"]}
            line["mixed_over_fp64"] = H["value"] / F64["value"]
            line["mixed_error"] = err
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def error_growth(cfg, checkpoints=(1, 2, 4, 8)):
    """The mixed form's distance from the FP64 form after 1, 2, 4, 8 s-steps from the same start, and the distance
    between two FP64 runs (their deposits add in a different order) after the last: a laser-driven plasma is
    chaotic, so a difference at rounding level grows from step to step in either form."""
    import numpy as np
    import g3d
    sims = {k: g3d.Simulation(cfg, precision=("mixed" if k == "mixed" else "fp64")) for k in ("fp64", "fp64_rerun", "mixed")}
    for sm in sims.values():
        sm.init()
    rl = lambda x, y: float(np.linalg.norm((x.astype(np.float64) - y).ravel()) / np.linalg.norm(y.astype(np.float64).ravel()))
    out = {"F_mixed_vs_fp64": {}, "<p_z>_mixed_vs_fp64": {}}
    done = 0
    for k in checkpoints:
        for _ in range(k - done):
            for sm in sims.values():
                sm.step()
        done = k
        F0 = sims["fp64"].array("F")
        d0 = sims["fp64"].diagnostics_sums()
        out["F_mixed_vs_fp64"][k] = rl(sims["mixed"].array("F"), F0)
        d = sims["mixed"].diagnostics_sums()
        out["<p_z>_mixed_vs_fp64"][k] = abs(d[9] / d[0] - d0[9] / d0[0]) / abs(d0[9] / d0[0])
        if k == checkpoints[-1]:
            out["F_fp64_rerun_vs_fp64"] = {k: rl(sims["fp64_rerun"].array("F"), F0)}
    for sm in sims.values():
        sm.close()
    out["note"] = ("relative L2 of the float F (six components) by s-steps from the same start; the FP64 rerun differs from "
                   "the FP64 run only in the order of its atomic adds")
    return out


def adjoint_check(eps=1e-6):
    """The adjoint march on workload 4 without its plasma (64 x 64 x 512, 65,536 electrons, 40 s-steps): the cost
    of one evaluation of J = mean p_z with its gradient against one forward run of the same steps (device time on
    the context stream, the third of three repetitions on one context), and the adjoint's directional
    derivatives (seeded random directions over the laser mode coefficients and the beam momenta) against
    central differences of the FP64 forward with exact fields, for the FP64 and the mixed adjoint."""
    import numpy as np
    import torch
    from g3d import Simulation, configs
    cfg = configs.config4()
    K = cfg.steps
    H = cfg.nx // 2 + 1

    def timed(sim, fn):
        st = torch.cuda.ExternalStream(sim.stream_ptr())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sim.synchronize()
        e0.record(st)
        out = fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    def final(coef=None, dp=None, through_start=True):
        sim = Simulation(cfg)
        sim.load_bunch()

        def perturb():
            p = sim.host_particles()
            p["px"] += dp[:, 0]; p["py"] += dp[:, 1]; p["pz"] += dp[:, 2]
            sim.set_particles(p)
        if dp is not None and through_start:      # the momenta as loaded: before the start field the bunch makes
            perturb()
        sim.set_laser_modes(coef)
        sim.set_exact_fields(True)
        sim.init_fields()
        if dp is not None and not through_start:  # right after init, the start field held
            perturb()
        for _ in range(K):
            sim.step_async()
        p = sim.host_particles()
        sim.close()
        return p

    def central(pp, pm, e=eps):
        a = pp["alive"] == 1
        return float(np.sum(pp["w"][a] * (pp["pz"][a] - pm["pz"][a])) / np.sum(pp["w"][a]) / (2 * e))

    out = {"workload": f"4 without plasma: {cfg.name}, {cfg.nx}x{cfg.ny} modes x {cfg.nzeta} slices, {cfg.particles} "
                       f"macro-electrons, {K} s-steps", "objective": "mean p_z of the live beam"}
    grads = {}
    for form in ["fp64", "mixed"]:
        sim = Simulation(cfg, precision=form)
        sim.load_bunch()
        p0 = sim.host_particles()
        sim.set_laser_modes(None)
        if form == "fp64":
            sim.set_exact_fields(True)
        tf = ta = None
        for _ in range(3):
            sim.set_particles(p0); sim.init_fields()
            tf, _ = timed(sim, lambda: [sim.step_async() for _ in range(K)])
        for _ in range(3):
            sim.set_particles(p0); sim.init_fields()
            ta, g = timed(sim, lambda: sim.adjoint(K))
        sim.set_particles(p0); sim.init_fields()
        grads[form] = g + (sim.adjoint(K, modes=False, through_start=False)[2],)
        sim.close()
        out[form] = {"forward_ms": tf, "adjoint_ms": ta, "adjoint_over_forward": ta / tf,
                     "note": "adjoint_ms: the forward with per-level checkpoints, J, and the reverse sweep"}
    rng = np.random.default_rng(11)
    d = rng.standard_normal((cfg.ny, H)) + 1j * rng.standard_normal((cfg.ny, H))
    D = np.random.default_rng(12).standard_normal(grads["fp64"][2].shape)
    fl = central(final(coef=1 + eps * d), final(coef=1 - eps * d))
    fa = central(final(dp=eps * D, through_start=False), final(dp=-eps * D, through_start=False))
    e4 = 1e-4
    fm = central(final(dp=e4 * D), final(dp=-e4 * D), e4)
    for form in ["fp64", "mixed"]:
        J, gm, gp, ga = grads[form]
        al, am, aa = float(np.real(np.sum(np.conj(gm) * d))), float(np.sum(gp * D)), float(np.sum(ga * D))
        out[form].update({"J": J, "laser_modes_rel_err": abs(al - fl) / abs(fl), "momenta_rel_err": abs(am - fm) / abs(fm),
                          "momenta_after_start_rel_err": abs(aa - fa) / abs(fa)})
    out["central_differences"] = {
        "eps": eps, "laser_modes": fl, "momenta_after_start": fa, "momenta": fm, "eps_momenta": e4,
        "forward": "FP64 form with exact (FP64) real fields",
        "note": "momenta: as loaded, through the start field (timed adjoint); momenta_after_start: right after init "
                "with the start field held. The first takes eps = 1e-4: the bunch's beta, bit for bit the "
                "reference's sum of w p_z / gamma, rounds at ~1e-14, which a step of 1e-6 does not clear"}
    out["with_plasma"] = plasma_adjoint_check(eps, timed, central)
    return out


def plasma_adjoint_check(eps, timed, central):
    """Workload 4 as specified, with its streaming plasma (0.005 n_c, 2 x 2 per cell, two passes): the adjoint's cost
    against the forward (FP64 form with exact fields; the march records kept from the forward, and with every step run
    again from its level checkpoint), the trapped plasma electrons of the forward, and the directional derivatives
    against central differences of the forward."""
    import os
    import numpy as np
    from g3d import Simulation, configs
    cfg = configs.config4(plasma=True)
    K = cfg.steps
    H = cfg.nx // 2 + 1
    sim = Simulation(cfg)
    sim.load_bunch()
    p0 = sim.host_particles()
    sim.set_laser_modes(None)
    sim.set_exact_fields(True)
    trapped = []
    for _ in range(3):
        sim.set_particles(p0); sim.init_fields()
        tf, _ = timed(sim, lambda: [sim.step_async() for _ in range(K)])
    sim.set_particles(p0); sim.init_fields()
    for _ in range(K):
        sim.step()
        trapped.append(int(np.sum(sim.streaming_particles()["alive"] == 5)))
    times = {}
    for mode in ("stored", "recompute"):
        if mode == "recompute":
            os.environ["G3D_ADJ_RECOMPUTE"] = "1"
        try:
            for _ in range(2):
                sim.set_particles(p0); sim.init_fields()
                ta, g = timed(sim, lambda: sim.adjoint(K))
        finally:
            os.environ.pop("G3D_ADJ_RECOMPUTE", None)
        times[mode] = ta
        if mode == "stored":
            grads = g
    sim.set_particles(p0); sim.init_fields()
    ga = sim.adjoint(K, modes=False, through_start=False)[2]
    sim.close()
    # the mixed form: its own forward (float F, FP32 streaming gathers and deposit) and adjoint (records kept)
    sim = Simulation(cfg, precision="mixed")
    sim.set_particles(p0)
    sim.set_laser_modes(None)
    for _ in range(3):
        sim.set_particles(p0); sim.init_fields()
        tfm, _ = timed(sim, lambda: [sim.step_async() for _ in range(K)])
    for _ in range(2):
        sim.set_particles(p0); sim.init_fields()
        tam, gmix = timed(sim, lambda: sim.adjoint(K))
    sim.close()

    def final(coef=None, dp=None, through_start=True):
        s = Simulation(cfg)
        s.load_bunch()

        def perturb():
            p = s.host_particles()
            p["px"] += dp[:, 0]; p["py"] += dp[:, 1]; p["pz"] += dp[:, 2]
            s.set_particles(p)
        if dp is not None and through_start:
            perturb()
        s.set_laser_modes(coef)
        s.set_exact_fields(True)
        s.init_fields()
        if dp is not None and not through_start:
            perturb()
        for _ in range(K):
            s.step_async()
        p = s.host_particles()
        s.close()
        return p
    J, gm, gp = grads
    d = np.random.default_rng(11).standard_normal((cfg.ny, H)) + 1j * np.random.default_rng(12).standard_normal((cfg.ny, H))
    D = np.random.default_rng(13).standard_normal(gp.shape)
    fl = central(final(coef=1 + eps * d), final(coef=1 - eps * d))
    fa = central(final(dp=eps * D, through_start=False), final(dp=-eps * D, through_start=False))
    e4 = 1e-4
    fm = central(final(dp=e4 * D), final(dp=-e4 * D), e4)
    al, am, aa = float(np.real(np.sum(np.conj(gm) * d))), float(np.sum(gp * D)), float(np.sum(ga * D))
    bl, bm = float(np.real(np.sum(np.conj(gmix[1]) * d))), float(np.sum(gmix[2] * D))
    mixed = {"forward_ms": tfm, "adjoint_ms": tam, "adjoint_over_forward": tam / tfm, "J": gmix[0],
             "laser_modes_rel_err": abs(bl - fl) / abs(fl), "momenta_rel_err": abs(bm - fm) / abs(fm),
             "note": "the mixed forward linearised (records widened, reverse sweep in FP64) against the FP64 forward's central "
                     "differences"}
    return {"mixed": mixed,"workload": f"4: {cfg.name}, {cfg.nx}x{cfg.ny} modes x {cfg.nzeta} slices, {cfg.particles} macro-electrons, "
                        f"plasma n0 0.005 n_c at 2x2 per cell, {K} s-steps", "form": "fp64 (exact fields)",
            "forward_ms": tf, "adjoint_ms": times["stored"], "adjoint_over_forward": times["stored"] / tf,
            "adjoint_recompute_ms": times["recompute"], "adjoint_recompute_over_forward": times["recompute"] / tf,
            "trapped_plasma_electrons_per_step": {"max": max(trapped), "total": sum(trapped)},
            "J": J, "laser_modes_rel_err": abs(al - fl) / abs(fl), "momenta_rel_err": abs(am - fm) / abs(fm),
            "momenta_after_start_rel_err": abs(aa - fa) / abs(fa),
            "central_differences": {"laser_modes": fl, "momenta": fm, "momenta_after_start": fa, "eps": eps, "eps_momenta": e4},
            "note": "adjoint_ms: the forward keeping each march's record, J and the reverse sweep; adjoint_recompute_ms: "
                    "the forward with level checkpoints only, each step run again in the reverse sweep"}


def adjoint_plasma_case(K):
    """One evaluation of the plasma adjoint on workload 4 (64 x 64 x 512, 65,536 electrons, plasma 0.005 n_c at 2 x 2 per
    cell) over K s-steps, after an untimed one on the same context: a case for the profiler."""
    import torch
    from g3d import Simulation, configs
    cfg = configs.config4(plasma=True, steps=K)
    sim = Simulation(cfg)
    sim.load_bunch()
    p0 = sim.host_particles()
    sim.set_laser_modes(None)
    sim.set_exact_fields(True)
    st = torch.cuda.ExternalStream(sim.stream_ptr())
    for rep in range(2):
        sim.set_particles(p0)
        sim.init_fields()
        sim.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        J, _, _ = sim.adjoint(K)
        e1.record(st)
        torch.cuda.synchronize()
    sim.close()
    print(json.dumps({"case": f"plasma adjoint, workload 4, {K} s-steps", "J": J, "adjoint_ms": e0.elapsed_time(e1)}))


def main():
    a = parse()
    if a.adjoint_plasma:
        adjoint_plasma_case(a.adjoint_plasma)
    elif a.impl == "reference":
        run_reference_arm(a)
    else:
        run_g3d(a)


if __name__ == "__main__":
    main()
