"""Host-side mirror of the reference's `class Simulation` (src/sim.hpp:222-360) over the C-ABI.

Same method names, argument meaning and error behaviour: a failing call raises G3DError (a
RuntimeError, as the reference throws std::runtime_error), carrying the C-ABI status code.
Arrays come back in the reference layouts (spectra [l][j][ix] complex128, F [comp][fl][j][ix] float32,
particles as the 104-byte records of PARTICLE_DTYPE).
"""
import ctypes as C

import numpy as np

from . import abi


class G3DError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"g3d error {code}: {msg}")
        self.code = code


def _check(lib, ctx, rc):
    if rc != abi.G3D_OK:
        raise G3DError(rc, lib.g3d_last_error(ctx).decode(errors="replace"))


def sample_bunches(cfg, lib=None):
    """The bunch of the configuration as the reference loads it (src/sim_bunches.cpp:92-217), sampled on
    the host without a device. Returns (particles, lost, X0, Y0)."""
    lib = lib or abi.load_library()
    g, z = cfg.grid_struct()
    p = cfg.params_struct()
    b, nb = cfg.bunch_structs()
    cap = max(1, cfg.particles)
    out = np.zeros(cap, dtype=abi.PARTICLE_DTYPE)
    n, lost, x0, y0 = C.c_int64(), C.c_int64(), C.c_double(), C.c_double()
    rc = lib.g3d_sample_bunches(C.byref(g), C.byref(p), b, nb, out.ctypes.data, cap, C.byref(n), C.byref(lost),
                                C.byref(x0), C.byref(y0))
    if rc != abi.G3D_OK:
        raise G3DError(rc, lib.g3d_last_error(None).decode(errors="replace"))
    return out[: n.value], lost.value, x0.value, y0.value


class Simulation:
    """One march context on the current CUDA device. precision: "fp64" (the reference's arithmetic) or "mixed"
    (FP32 transforms, currents, gathers and E_z/B_z/L storage with the FP64 accumulator R and FP64 particles)."""

    def __init__(self, cfg, lib=None, precision="fp64", comm=None):
        """comm: a shard.RankComm for a run sharded over the ranks of a process group (zeta slabs; FP64, Fourier y,
        no plasma), or None for the whole window on this device."""
        if precision not in ("fp64", "mixed"):
            raise ValueError(f"precision must be 'fp64' or 'mixed', not {precision!r}")
        self.lib = lib or abi.load_library()
        self.cfg = cfg
        g, self._zeta = cfg.grid_struct()
        p = cfg.params_struct()
        h = C.c_void_p()
        rc = self.lib.g3d_create(C.byref(g), C.byref(p), C.byref(h))
        if rc != abi.G3D_OK:
            raise G3DError(rc, self.lib.g3d_last_error(None).decode(errors="replace"))
        self.ctx = h
        self.precision = precision
        self.comm = comm
        self.a = 0
        self.ns = cfg.nzeta
        if comm is not None:
            self._c(self.lib.g3d_set_ranks(self.ctx, comm.rank, comm.world, comm.fn, None))
            from . import shard
            self.a, b, _, _ = shard.layout(cfg.nzeta, cfg.ny * (cfg.nx // 2 + 1), comm.rank, comm.world, self.lib)
            self.ns = b - self.a
        if precision == "mixed":
            self._c(self.lib.g3d_set_precision(self.ctx, abi.G3D_PREC_MIXED))
        ps = cfg.plasma_structs()
        if ps is not None:
            P, ions, nions, self._keep = ps
            self._c(self.lib.g3d_set_plasma(self.ctx, C.byref(P), ions, nions))
        for L in cfg.glaser_structs():
            self._c(self.lib.g3d_add_grid_laser(self.ctx, C.byref(L)))
        if getattr(cfg, "undulators", None) or getattr(cfg, "magnets", None):
            self.set_external(cfg.undulators, cfg.magnets, getattr(cfg, "ktab", None))
        self.N, self.nx, self.ny = cfg.nzeta, cfg.nx, cfg.ny
        self.nk = cfg.nx * cfg.ny

    def set_external(self, undulators=(), magnets=(), ktab=None):
        """External magnetic elements (dicts of the g3d_undulator / g3d_magnet fields, code units; ktab: the taper
        table of the undulators); none removes them (reference src/external.hpp)."""
        U = (abi.Undulator * max(1, len(undulators)))()
        for k, u in enumerate(undulators):
            for f, v in u.items():
                setattr(U[k], f, v)
        M = (abi.Magnet * max(1, len(magnets)))()
        for k, m in enumerate(magnets):
            for f, v in m.items():
                setattr(M[k], f, v)
        kt = np.ascontiguousarray(ktab if ktab is not None else [], dtype=np.float64)
        self._c(self.lib.g3d_set_external(self.ctx, U, len(undulators), M, len(magnets),
                                          kt.ctypes.data_as(C.POINTER(C.c_double)), len(kt)))

    def set_chicanes(self, chicanes=()):
        """Thin chicanes: dicts of z, r56, delay, gamma_ref (code units); none removes them."""
        A = (abi.Chicane * max(1, len(chicanes)))()
        for k, ch in enumerate(chicanes):
            for f, v in ch.items():
                setattr(A[k], f, v)
        self._c(self.lib.g3d_set_chicanes(self.ctx, A, len(chicanes)))

    def close(self):
        if getattr(self, "ctx", None):
            self.lib.g3d_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, rc):
        if rc != abi.G3D_OK and getattr(self, "comm", None) is not None and self.comm.error is not None:
            err, self.comm.error = self.comm.error, None
            raise G3DError(rc, f"{self.lib.g3d_last_error(self.ctx).decode(errors='replace')}: {err!r}") from err
        _check(self.lib, self.ctx, rc)

    # ------------------------------------------------------------ particles
    def load_bunch(self):
        arr, n = self.cfg.bunch_structs()
        self._c(self.lib.g3d_load_bunches(self.ctx, arr, n))

    def set_particles(self, parts):
        parts = np.ascontiguousarray(parts, dtype=abi.PARTICLE_DTYPE)
        self._c(self.lib.g3d_set_particles(self.ctx, parts.ctypes.data, len(parts)))

    def host_particles(self):
        n = self.status().np
        out = np.zeros(n, dtype=abi.PARTICLE_DTYPE)
        got = C.c_int64()
        self._c(self.lib.g3d_get_particles(self.ctx, out.ctypes.data, n, C.byref(got)))
        return out

    # ------------------------------------------------------------ the march path
    def init(self):
        """Simulation::init: the bunch of the configuration, then the start fields."""
        self.load_bunch()
        self.init_fields()

    def init_fields(self):
        self._c(self.lib.g3d_init(self.ctx))

    def step(self):
        self._c(self.lib.g3d_step(self.ctx))

    def step_async(self):
        self._c(self.lib.g3d_step_async(self.ctx))

    def solve_fields(self, D):
        self._c(self.lib.g3d_solve_fields(self.ctx, D))

    def currents(self):
        self._c(self.lib.g3d_currents(self.ctx))

    def march(self, D):
        self._c(self.lib.g3d_march(self.ctx, D))

    def sponge_and_real_fields(self):
        self._c(self.lib.g3d_sponge_and_real_fields(self.ctx))

    def push(self, s0, s1):
        self._c(self.lib.g3d_push(self.ctx, s0, s1))

    def march_plasma(self, s0, s1):
        self._c(self.lib.g3d_march_plasma(self.ctx, s0, s1))

    def streaming_count(self):
        """Number of streaming particles of the last march (plasma electrons and ions, no copy)."""
        n = C.c_int64()
        rc = self.lib.g3d_get_streaming(self.ctx, None, 0, C.byref(n))
        if rc not in (abi.G3D_OK, abi.G3D_ERR_CAPACITY):
            self._c(rc)
        return n.value

    def streaming_particles(self):
        n = C.c_int64(self.streaming_count())
        out = np.zeros(n.value, dtype=abi.PARTICLE_DTYPE)
        self._c(self.lib.g3d_get_streaming(self.ctx, out.ctypes.data, n.value, C.byref(n)))
        return out[: n.value]

    def comoving_field(self):
        self._c(self.lib.g3d_comoving_field(self.ctx))

    def relax_start_field(self):
        self._c(self.lib.g3d_relax_start_field(self.ctx))

    def shift_window(self, nxs, nys):
        self._c(self.lib.g3d_shift_window(self.ctx, nxs, nys))

    # ------------------------------------------------------------ diagnostics
    def diagnostics_sums(self):
        out = (C.c_double * 19)()
        self._c(self.lib.g3d_diagnostics(self.ctx, out))
        return np.array(out[:], dtype=np.float64)

    def beam_moments(self):
        """(s1, s2): per beam species [G, 8] the first sums and the centred second sums of bunches.txt."""
        cap = 16
        s1 = (C.c_double * (8 * cap))()
        s2 = (C.c_double * (8 * cap))()
        G = C.c_int32()
        self._c(self.lib.g3d_beam_moments(self.ctx, cap, s1, s2, C.byref(G)))
        n = 8 * G.value
        return np.array(s1[:n]).reshape(-1, 8), np.array(s2[:n]).reshape(-1, 8)

    def field_energy(self):
        v = C.c_double()
        self._c(self.lib.g3d_field_energy(self.ctx, C.byref(v)))
        return v.value

    def status(self):
        st = abi.Status()
        self._c(self.lib.g3d_get_status(self.ctx, C.byref(st)))
        return st

    @property
    def s(self):
        return self.status().s

    @property
    def istep(self):
        return self.status().istep

    def finished(self):
        return bool(self.status().stop)

    # ------------------------------------------------------------ arrays
    def array_info(self, name):
        n, eb = C.c_size_t(), C.c_size_t()
        self._c(self.lib.g3d_array_info(self.ctx, abi.ARRAYS[name], C.byref(n), C.byref(eb)))
        return n.value, eb.value

    def array(self, name):
        n, eb = self.array_info(name)
        dt = {16: np.complex128, 8: np.float64, 4: np.float32}[eb]
        out = np.empty(n, dtype=dt)
        self._c(self.lib.g3d_get_array(self.ctx, abi.ARRAYS[name], out.ctypes.data, n))
        return out

    def set_array(self, name, values):
        n, eb = self.array_info(name)
        dt = {16: np.complex128, 8: np.float64, 4: np.float32}[eb]
        v = np.ascontiguousarray(values, dtype=dt).ravel()
        if v.size != n:
            raise ValueError(f"{name}: {v.size} values for an array of {n}")
        self._c(self.lib.g3d_set_array(self.ctx, abi.ARRAYS[name], v.ctypes.data, n))

    def device_ptr(self, name):
        return self.lib.g3d_device_ptr(self.ctx, abi.ARRAYS[name])

    # ------------------------------------------------------------ checkpoints
    def write_checkpoint(self, path):
        self._c(self.lib.g3d_write_checkpoint(self.ctx, str(path).encode()))

    def read_checkpoint(self, path):
        self._c(self.lib.g3d_read_checkpoint(self.ctx, str(path).encode()))

    def write_checkpoint_async(self, path):
        """The checkpoint of write_checkpoint, written by a host thread of the library while the run goes on (the
        state copied on the device first); checkpoint_wait() returns when the file is complete."""
        self._c(self.lib.g3d_write_checkpoint_async(self.ctx, str(path).encode()))

    def checkpoint_wait(self):
        self._c(self.lib.g3d_checkpoint_wait(self.ctx))

    # ------------------------------------------------------------ stream, timing
    def stream_ptr(self):
        return self.lib.g3d_stream(self.ctx)

    def synchronize(self):
        self._c(self.lib.g3d_synchronize(self.ctx))

    def profile(self, on=True):
        self._c(self.lib.g3d_profile_enable(self.ctx, 1 if on else 0))

    def profile_results(self):
        out = {}
        for k in range(self.lib.g3d_profile_count(self.ctx)):
            name, n, ms = C.c_char_p(), C.c_int64(), C.c_double()
            self._c(self.lib.g3d_profile_get(self.ctx, k, C.byref(name), C.byref(n), C.byref(ms)))
            out[name.value.decode()] = (n.value, ms.value)
        return out

    def launch_count(self):
        return self.lib.g3d_launch_count(self.ctx)

    # ---------------------------------------------------------------- adjoint march
    def set_laser_modes(self, coef=None):
        """Laser mode coefficients a[j, kx] (complex, ny x (nx/2 + 1)) multiplying the grid lasers' spectra at
        init; None: all ones. Before init."""
        if coef is None:
            self._c(self.lib.g3d_set_laser_modes(self.ctx, None))
            return
        a = np.ascontiguousarray(np.asarray(coef, dtype=np.complex128).reshape(self.ny, self.nx // 2 + 1))
        self._c(self.lib.g3d_set_laser_modes(self.ctx, a.ctypes.data))

    def set_exact_fields(self, on=True):
        """Keep the real fields in FP64 as well and gather the beam push from them. Before init."""
        self._c(self.lib.g3d_set_exact_fields(self.ctx, 1 if on else 0))

    def adjoint(self, nsteps, modes=True, momenta=True, through_start=True):
        """From the start field: nsteps s-steps and the reverse sweep. Returns (J, dJ/da [ny, nx/2+1] complex
        or None, dJ/dp [np, 3] or None) with J = mean p_z of the live beam and dJ/dp taken at load time, through
        the start field the bunch makes as well as through the s-steps (through_start=False: with the start
        field held, through the s-steps alone)."""
        self._c(self.lib.g3d_set_adjoint_momenta(self.ctx, 0 if through_start else 1))
        J = C.c_double()
        gm = np.zeros((self.ny, self.nx // 2 + 1), dtype=np.complex128) if modes else None
        n = self.status().np
        gp = np.zeros((n, 3)) if momenta else None
        self._c(self.lib.g3d_adjoint(self.ctx, int(nsteps), C.byref(J), gm.ctypes.data if modes else None,
                                     gp.ctypes.data if momenta else None))
        return J.value, gm, gp
