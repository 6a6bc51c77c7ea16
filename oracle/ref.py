"""Test infrastructure only: Python binding of oracle/_ref/libg3dref.so, the reference GEM-PIC-3D CPU/OpenMP
build driven by oracle/ref_driver.cpp. Used by tests/ as the parity checker and by bench.py's CPU
baseline; never by the product. Method names match g3d.Simulation so both sides run one script.
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(REPO, "gem-pic-3d_b200"))
from g3d import abi  # noqa: E402  (struct definitions shared with the product's header)

REF_LIB = os.path.join(HERE, "_ref", "libg3dref.so")
REF_BIN = os.path.join(HERE, "_ref", "gempic3d")

_P, _D, _I, _L = C.c_void_p, C.c_double, C.c_int, C.c_long
_SIGS = [
    ("ref_last_error", C.c_char_p, []),
    ("ref_set_threads", _I, [_I]),
    ("ref_create", _I, [C.POINTER(abi.Grid), C.POINTER(abi.Params), C.POINTER(abi.Bunch), _I, C.POINTER(_P)]),
    ("ref_create2", _I, [C.POINTER(abi.Grid), C.POINTER(abi.Params), C.POINTER(abi.Bunch), _I, C.POINTER(abi.Plasma),
                         C.POINTER(abi.Ion), _I, C.POINTER(abi.GridLaser), _I, C.POINTER(_P)]),
    ("ref_get_streaming", _I, [_P, _P, _L, C.POINTER(_L)]),
    ("ref_march_plasma", _I, [_P, _D, _D]),
    ("ref_element", _I, [C.c_char_p, C.POINTER(_D), C.POINTER(_D), _I]),
    ("ref_destroy", None, [_P]),
    ("ref_load_bunches", _I, [_P]),
    ("ref_init", _I, [_P]),
    ("ref_init_fields", _I, [_P]),
    ("ref_step", _I, [_P]),
    ("ref_solve_fields", _I, [_P, _D]),
    ("ref_currents", _I, [_P]),
    ("ref_march", _I, [_P, _D]),
    ("ref_sponge_and_real_fields", _I, [_P]),
    ("ref_push", _I, [_P, _D, _D]),
    ("ref_comoving_field", _I, [_P]),
    ("ref_relax_start_field", _I, [_P]),
    ("ref_shift_window", _I, [_P, _I, _I]),
    ("ref_set_starting", _I, [_P, _I]),
    ("ref_set_origin", _I, [_P, _D, _D]),
    ("ref_set_particles", _I, [_P, _P, _L]),
    ("ref_num_particles", _L, [_P]),
    ("ref_get_particles", _I, [_P, _P, _L]),
    ("ref_get_status", _I, [_P, C.POINTER(abi.Status)]),
    ("ref_array_info", _I, [_P, _I, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    ("ref_get_array", _I, [_P, _I, _P, C.c_size_t]),
    ("ref_set_array", _I, [_P, _I, _P, C.c_size_t]),
    ("ref_field_energy", _D, [_P]),
    ("ref_diagnostics", _I, [_P, C.POINTER(_D)]),
    ("ref_write_checkpoint", _I, [_P, C.c_char_p]),
    ("ref_read_checkpoint", _I, [_P, C.c_char_p, _L]),
]

_lib = None


def element(symbol):
    """(mass [u], ionization energies [eV]) of an element in the reference's table."""
    lib = load()
    m = C.c_double()
    ip = (C.c_double * 120)()
    z = lib.ref_element(symbol.encode(), C.byref(m), ip, 120)
    if z < 0:
        raise KeyError(symbol)
    return m.value, list(ip[:z])


def available():
    return os.path.exists(REF_LIB)


def load():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"{REF_LIB} is not built (make -C oracle)")
        lib = C.CDLL(REF_LIB)
        for name, res, args in _SIGS:
            f = getattr(lib, name)
            f.restype, f.argtypes = res, args
        _lib = lib
    return _lib


class RefSimulation:
    """The reference Simulation (CPU), driven through ref_driver.cpp."""

    def __init__(self, cfg, threads=1):
        self.lib = load()
        self.lib.ref_set_threads(threads)
        self.cfg = cfg
        g, self._z = cfg.grid_struct()
        p = cfg.params_struct()
        b, nb = cfg.bunch_structs()
        h = C.c_void_p()
        ps = cfg.plasma_structs()
        gls = cfg.glaser_structs()
        if ps is None and not gls:
            self._c(self.lib.ref_create(C.byref(g), C.byref(p), b, nb, C.byref(h)))
        else:
            garr = (abi.GridLaser * max(1, len(gls)))(*gls) if gls else (abi.GridLaser * 1)()
            if ps is None:
                self._c(self.lib.ref_create2(C.byref(g), C.byref(p), b, nb, None, None, 0, garr, len(gls), C.byref(h)))
            else:
                P, ions, nions, self._keep = ps
                self._c(self.lib.ref_create2(C.byref(g), C.byref(p), b, nb, C.byref(P), ions, nions, garr, len(gls),
                                             C.byref(h)))
        self.h = h

    def _c(self, rc):
        if rc != 0:
            raise RuntimeError(f"reference error {rc}: {self.lib.ref_last_error().decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.lib.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_bunch(self):
        self._c(self.lib.ref_load_bunches(self.h))

    def init(self):
        self._c(self.lib.ref_init(self.h))

    def init_fields(self):
        self._c(self.lib.ref_init_fields(self.h))

    def step(self):
        self._c(self.lib.ref_step(self.h))

    def solve_fields(self, D):
        self._c(self.lib.ref_solve_fields(self.h, D))

    def currents(self):
        self._c(self.lib.ref_currents(self.h))

    def march(self, D):
        self._c(self.lib.ref_march(self.h, D))

    def sponge_and_real_fields(self):
        self._c(self.lib.ref_sponge_and_real_fields(self.h))

    def push(self, s0, s1):
        self._c(self.lib.ref_push(self.h, s0, s1))

    def comoving_field(self):
        self._c(self.lib.ref_comoving_field(self.h))

    def relax_start_field(self):
        self._c(self.lib.ref_relax_start_field(self.h))

    def shift_window(self, nxs, nys):
        self._c(self.lib.ref_shift_window(self.h, nxs, nys))

    def march_plasma(self, s0, s1):
        self._c(self.lib.ref_march_plasma(self.h, s0, s1))

    def streaming_particles(self):
        n = C.c_long()
        cap = 1 << 24
        out = np.zeros(cap, dtype=abi.PARTICLE_DTYPE)
        self._c(self.lib.ref_get_streaming(self.h, out.ctypes.data, cap, C.byref(n)))
        return out[: n.value].copy()

    def set_starting(self, v):
        self._c(self.lib.ref_set_starting(self.h, 1 if v else 0))

    def set_origin(self, X0, Y0):
        self._c(self.lib.ref_set_origin(self.h, X0, Y0))

    def set_particles(self, parts):
        parts = np.ascontiguousarray(parts, dtype=abi.PARTICLE_DTYPE)
        self._c(self.lib.ref_set_particles(self.h, parts.ctypes.data, len(parts)))

    def host_particles(self):
        n = self.lib.ref_num_particles(self.h)
        out = np.zeros(n, dtype=abi.PARTICLE_DTYPE)
        self._c(self.lib.ref_get_particles(self.h, out.ctypes.data, n))
        return out

    def status(self):
        st = abi.Status()
        self._c(self.lib.ref_get_status(self.h, C.byref(st)))
        return st

    def array(self, name):
        n, eb = C.c_size_t(), C.c_size_t()
        self._c(self.lib.ref_array_info(self.h, abi.ARRAYS[name], C.byref(n), C.byref(eb)))
        dt = {16: np.complex128, 8: np.float64, 4: np.float32}[eb.value]
        out = np.empty(n.value, dtype=dt)
        self._c(self.lib.ref_get_array(self.h, abi.ARRAYS[name], out.ctypes.data, n.value))
        return out

    def set_array(self, name, values):
        n, eb = C.c_size_t(), C.c_size_t()
        self._c(self.lib.ref_array_info(self.h, abi.ARRAYS[name], C.byref(n), C.byref(eb)))
        dt = {16: np.complex128, 8: np.float64, 4: np.float32}[eb.value]
        v = np.ascontiguousarray(values, dtype=dt).ravel()
        self._c(self.lib.ref_set_array(self.h, abi.ARRAYS[name], v.ctypes.data, n.value))

    def field_energy(self):
        return self.lib.ref_field_energy(self.h)

    def diagnostics_sums(self):
        out = (C.c_double * 19)()
        self._c(self.lib.ref_diagnostics(self.h, out))
        return np.array(out[:])

    def write_checkpoint(self, directory):
        self._c(self.lib.ref_write_checkpoint(self.h, str(directory).encode()))

    def read_checkpoint(self, directory, step):
        self._c(self.lib.ref_read_checkpoint(self.h, str(directory).encode(), step))
