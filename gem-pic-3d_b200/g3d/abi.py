"""ctypes binding of the C-ABI in include/g3d.h (libg3d.so, the sm_100a march library).

The structs mirror the header field for field; PARTICLE_DTYPE is the reference's 104-byte
`struct Particle` (src/sim.hpp:217) as a numpy structured dtype.
"""
import ctypes as C
import os

import numpy as np

G3D_OK, G3D_ERR_CUDA, G3D_ERR_TIMEOUT, G3D_ERR_CAPACITY, G3D_ERR_ARG, G3D_ERR_STATE, G3D_ERR_IO, G3D_ERR_NODEV = range(8)
G3D_FP64, G3D_MIXED = 0, 1
G3D_ENV_GAUSSIAN, G3D_ENV_FLATTOP = 0, 1
G3D_PREC_FP64, G3D_PREC_MIXED = 0, 1
G3D_POL_S, G3D_POL_P, G3D_POL_CIRCULAR = 0, 1, 2

ARRAYS = {"Rx": 0, "Ry": 1, "Ez": 2, "Bz": 3, "Lx": 4, "Ly": 5, "j0x": 6, "j0y": 7,
          "jkx": 8, "jky": 9, "jkz": 10, "jw": 11, "F": 12, "rho_lines": 13, "rho_lines_i": 14}

PARTICLE_DTYPE = np.dtype([("x", "<f8"), ("y", "<f8"), ("zeta", "<f8"), ("px", "<f8"), ("py", "<f8"),
                           ("pz", "<f8"), ("w", "<f8"), ("rem", "<f8"), ("z", "<f8"), ("q", "<f8"),
                           ("qm", "<f8"), ("alive", "<i4"), ("sp", "<i4"), ("id", "<u8")])
assert PARTICLE_DTYPE.itemsize == 104


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nzeta", C.c_int32), ("y_fourier", C.c_int32),
                ("Lx", C.c_double), ("Ly", C.c_double),
                ("zeta", C.POINTER(C.c_double)), ("ynode", C.POINTER(C.c_double))]


class Params(C.Structure):
    _fields_ = [("lambda0", C.c_double), ("dz", C.c_double), ("dz_push", C.c_double), ("z_end", C.c_double),
                ("sponge", C.c_double), ("sponge_y", C.c_double), ("sponge_rate", C.c_double),
                ("move_x", C.c_int32), ("move_y", C.c_int32), ("window_lag", C.c_int32),
                ("self_fields", C.c_int32), ("zeta_filter", C.c_int32), ("k_filter", C.c_int32),
                ("push_phase", C.c_double),
                ("laser_on", C.c_int32), ("laser_pol", C.c_int32), ("laser_envelope", C.c_int32),
                ("reserved0", C.c_int32),
                ("a0", C.c_double), ("kL", C.c_double), ("theta", C.c_double), ("tau", C.c_double),
                ("cep", C.c_double), ("eta_c", C.c_double), ("stop_fwhm", C.c_double),
                ("flat_length", C.c_double), ("ramp_length", C.c_double), ("zeta_center", C.c_double),
                ("freeze_bunch", C.c_int32), ("start_relax", C.c_int32), ("box_mean", C.c_int32),
                ("precision", C.c_int32)]


class Bunch(C.Structure):
    _fields_ = [("charge_C", C.c_double), ("gamma", C.c_double), ("sigx", C.c_double), ("sigy", C.c_double),
                ("sigz", C.c_double), ("length", C.c_double), ("emitx", C.c_double), ("emity", C.c_double),
                ("espread", C.c_double), ("zeta_center", C.c_double), ("x0", C.c_double), ("y0", C.c_double),
                ("q", C.c_double), ("nmacro", C.c_int64), ("seed", C.c_uint64), ("beamlet", C.c_int32),
                ("reserved", C.c_int32), ("noise_lambda", C.c_double)]


class Status(C.Structure):
    _fields_ = [("s", C.c_double), ("X0", C.c_double), ("Y0", C.c_double), ("beta_b", C.c_double),
                ("gm2_b", C.c_double), ("field_energy", C.c_double),
                ("istep", C.c_int64), ("np", C.c_int64), ("lost", C.c_int64), ("stop", C.c_int64)]


class Plasma(C.Structure):
    _fields_ = [("n0", C.c_double), ("r_max", C.c_double), ("channel_depth", C.c_double), ("r_channel", C.c_double),
                ("smooth_length", C.c_double), ("vz_min", C.c_double), ("vz_beam", C.c_double),
                ("trap_advance", C.c_double), ("z_points", C.POINTER(C.c_double)), ("z_values", C.POINTER(C.c_double)),
                ("n_z", C.c_int32), ("ppc_x", C.c_int32), ("ppc_y", C.c_int32), ("iterations", C.c_int32),
                ("predictor_extrapolate", C.c_int32), ("free_electrons", C.c_int32), ("parabolic", C.c_int32),
                ("box_mean", C.c_int32), ("seed", C.c_uint64)]


class Ion(C.Structure):
    _fields_ = [("mass", C.c_double), ("atoms", C.c_double), ("ip_eV", C.POINTER(C.c_double)), ("n_ip", C.c_int32),
                ("Z0", C.c_int32), ("Zmax", C.c_int32), ("mobile", C.c_int32), ("ionization", C.c_int32),
                ("reserved", C.c_int32)]


class GridLaser(C.Structure):
    _fields_ = [("a0", C.c_double), ("kL", C.c_double), ("waist", C.c_double), ("tau", C.c_double),
                ("zeta_c", C.c_double), ("z_focus", C.c_double), ("cep", C.c_double), ("pol_angle", C.c_double),
                ("circular", C.c_int32), ("helicity", C.c_int32)]


class Undulator(C.Structure):
    _fields_ = [("helical", C.c_int32), ("focusing", C.c_int32), ("ku", C.c_double), ("B0", C.c_double), ("z0", C.c_double),
                ("z1", C.c_double), ("ramp", C.c_double), ("nk", C.c_int32), ("koff", C.c_int32), ("dzk", C.c_double)]


class Magnet(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reserved", C.c_int32), ("z0", C.c_double), ("z1", C.c_double), ("g", C.c_double),
                ("R", C.c_double), ("ramp", C.c_double), ("dsmax", C.c_double)]


assert C.sizeof(Plasma) == 120 and C.sizeof(Ion) == 48 and C.sizeof(GridLaser) == 72
class Chicane(C.Structure):
    _fields_ = [("z", C.c_double), ("r56", C.c_double), ("delay", C.c_double), ("gamma_ref", C.c_double)]


class CommOp(C.Structure):
    """struct g3d_comm_op: one collective the library asks of the caller (a sharded run)."""
    _fields_ = [("op", C.c_int32), ("kind", C.c_int32), ("count", C.c_int64), ("data", C.c_void_p),
                ("send", C.c_void_p), ("send_bytes", C.POINTER(C.c_int64)), ("recv", C.c_void_p),
                ("recv_bytes", C.POINTER(C.c_int64))]


class Block(C.Structure):
    """struct g3d_block: one copy of a slab <-> pencil transpose."""
    _fields_ = [("src", C.c_int64), ("dst", C.c_int64), ("rows", C.c_int64), ("cols", C.c_int64),
                ("src_stride", C.c_int64), ("dst_stride", C.c_int64), ("src_array", C.c_int32), ("dst_array", C.c_int32)]


G3D_COMM_SUM, G3D_COMM_ALLTOALL = 0, 1
G3D_SUM_F64, G3D_SUM_I64 = 0, 1
G3D_SLAB_NODES, G3D_SLAB_HALF = 0, 1
COMM_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(CommOp))

assert C.sizeof(CommOp) == 56 and C.sizeof(Block) == 56
assert C.sizeof(Undulator) == 64 and C.sizeof(Magnet) == 56 and C.sizeof(Chicane) == 32
assert C.sizeof(Grid) == 48 and C.sizeof(Params) == 200 and C.sizeof(Bunch) == 136 and C.sizeof(Status) == 80

_P = C.c_void_p
_D = C.c_double
_I = C.c_int
_I32 = C.c_int32
_I64 = C.c_int64
_S = C.c_size_t

# (name, restype, argtypes) of every entry point declared in include/g3d.h
SIGNATURES = [
    ("g3d_create", _I, [C.POINTER(Grid), C.POINTER(Params), C.POINTER(_P)]),
    ("g3d_destroy", None, [_P]),
    ("g3d_last_error", C.c_char_p, [_P]),
    ("g3d_version", C.c_char_p, []),
    ("g3d_set_particles", _I, [_P, _P, _I64]),
    ("g3d_get_particles", _I, [_P, _P, _I64, C.POINTER(_I64)]),
    ("g3d_load_bunches", _I, [_P, C.POINTER(Bunch), _I32]),
    ("g3d_sample_bunches", _I, [C.POINTER(Grid), C.POINTER(Params), C.POINTER(Bunch), _I32, _P, _I64,
                                C.POINTER(_I64), C.POINTER(_I64), C.POINTER(_D), C.POINTER(_D)]),
    ("g3d_set_plasma", _I, [_P, C.POINTER(Plasma), C.POINTER(Ion), _I32]),
    ("g3d_add_grid_laser", _I, [_P, C.POINTER(GridLaser)]),
    ("g3d_set_external", _I, [_P, C.POINTER(Undulator), _I32, C.POINTER(Magnet), _I32, C.POINTER(_D), _I32]),
    ("g3d_set_chicanes", _I, [_P, C.POINTER(Chicane), _I32]),
    ("g3d_set_ranks", _I, [_P, _I32, _I32, COMM_FN, _P]),
    ("g3d_shard_layout", _I, [_I32, _I64, _I32, _I32, C.POINTER(_I64)]),
    ("g3d_shard_transpose_plan", _I, [_I32, _I64, _I32, _I32, C.POINTER(_I32), _I32, _I32, _I64, C.POINTER(Block), _I32,
                                      C.POINTER(_I32), C.POINTER(Block), _I32, C.POINTER(_I32), C.POINTER(_I64),
                                      C.POINTER(_I64)]),
    ("g3d_march_plasma", _I, [_P, _D, _D]),
    ("g3d_get_streaming", _I, [_P, _P, _I64, C.POINTER(_I64)]),
    ("g3d_init", _I, [_P]),
    ("g3d_step", _I, [_P]),
    ("g3d_step_async", _I, [_P]),
    ("g3d_solve_fields", _I, [_P, _D]),
    ("g3d_currents", _I, [_P]),
    ("g3d_march", _I, [_P, _D]),
    ("g3d_sponge_and_real_fields", _I, [_P]),
    ("g3d_push", _I, [_P, _D, _D]),
    ("g3d_comoving_field", _I, [_P]),
    ("g3d_relax_start_field", _I, [_P]),
    ("g3d_shift_window", _I, [_P, _I32, _I32]),
    ("g3d_diagnostics", _I, [_P, C.POINTER(_D)]),
    ("g3d_field_energy", _I, [_P, C.POINTER(_D)]),
    ("g3d_beam_moments", _I, [_P, _I32, C.POINTER(_D), C.POINTER(_D), C.POINTER(_I32)]),
    ("g3d_beam_beta_sums_static", _I, [_P, C.POINTER(_D)]),
    ("g3d_set_precision", _I, [_P, _I]),
    ("g3d_get_status", _I, [_P, C.POINTER(Status)]),
    ("g3d_array_info", _I, [_P, _I32, C.POINTER(_S), C.POINTER(_S)]),
    ("g3d_get_array", _I, [_P, _I32, _P, _S]),
    ("g3d_set_array", _I, [_P, _I32, _P, _S]),
    ("g3d_device_ptr", _P, [_P, _I32]),
    ("g3d_write_checkpoint", _I, [_P, C.c_char_p]),
    ("g3d_read_checkpoint", _I, [_P, C.c_char_p]),
    ("g3d_write_checkpoint_async", _I, [_P, C.c_char_p]),
    ("g3d_checkpoint_wait", _I, [_P]),
    ("g3d_stream", _P, [_P]),
    ("g3d_synchronize", _I, [_P]),
    ("g3d_profile_enable", _I, [_P, _I32]),
    ("g3d_profile_count", _I32, [_P]),
    ("g3d_profile_get", _I, [_P, _I32, C.POINTER(C.c_char_p), C.POINTER(_I64), C.POINTER(_D)]),
    ("g3d_launch_count", _I64, [_P]),
    ("g3d_set_laser_modes", _I, [_P, _P]),
    ("g3d_set_exact_fields", _I, [_P, _I32]),
    ("g3d_set_adjoint_momenta", _I, [_P, _I32]),
    ("g3d_adjoint", _I, [_P, _I32, C.POINTER(_D), _P, _P]),
]

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libg3d.so")

_lib = None


def load_library(path=None):
    """Load libg3d.so (built in-tree by __graft_entry__.build()). Fails loudly when it is missing:
    there is no fallback implementation of the march."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"libg3d.so not found at {p}: build it with `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = C.CDLL(p)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib
