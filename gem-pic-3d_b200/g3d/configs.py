"""Run configurations in code units (the reference's deck keys, docs/input_deck.md, set in code the way
the reference's tests do with `base()`, tests/test_util.hpp:36-43).

`baseline(k)` builds the benchmark workloads of this project by their sizes:
  1  frozen-bunch wake in vacuum: 64x64 modes, 256 slices (h = 0.5), 262,144 macro-electrons, 10 s-steps
  2  oblique plane wave on a bunch: 128x128 modes, 1024 slices (h = 0.1), 1,048,576 macro-electrons,
     a0 = 0.5, p polarisation, 20 mrad, flat top 60 with sin^2 ramps 10, 100 s-steps of 2
  3  laser wakefield with streaming plasma: 256x256 modes, 2048 slices, H+ ions, a grid laser, a witness bunch
Every size can be reduced with keyword overrides for tests. `freehand_small` builds a bunch on the free-hand y grid
(a graded table of nodes between conducting walls).
"""
import math
from dataclasses import dataclass, field

import numpy as np

from . import abi

C_SI, E_SI, ME_SI, EPS0 = 299792458.0, 1.602176634e-19, 9.1093837015e-31, 8.8541878128e-12


def units(lambda0):
    """Unit of length Lu = lambda0 / 2 pi [m] and the critical density n_c [m^-3] (sim_config.cpp:5-11)."""
    Lu = lambda0 / (2 * math.pi)
    w0 = C_SI / Lu
    nc = EPS0 * ME_SI * w0 * w0 / (E_SI * E_SI)
    return Lu, nc


def charge_for_peak_density(n_peak, sigx, sigy, sigz, lambda0):
    """|charge| [C] of a Gaussian bunch with the peak density n_peak (units of n_c), sizes in 1/k0."""
    Lu, nc = units(lambda0)
    ne = n_peak * (2 * math.pi) ** 1.5 * sigx * sigy * sigz * nc * Lu ** 3
    return ne * E_SI


@dataclass
class RunConfig:
    name: str
    nx: int
    ny: int
    nzeta: int
    Lx: float
    Ly: float
    h: float                       # uniform slice step
    params: dict = field(default_factory=dict)
    bunches: list = field(default_factory=list)
    steps: int = 10
    plasma: dict = None              # streaming plasma (g3d_plasma keys), None: vacuum
    ions: list = field(default_factory=list)
    glasers: list = field(default_factory=list)
    ynode: np.ndarray = None         # free-hand y: the ny + 1 nodes (walls at the ends); None: Fourier y
    zeta_table: np.ndarray = None    # free-hand zeta: the nzeta slice positions; None: uniform steps h

    @property
    def zeta(self):
        if self.zeta_table is not None:
            return np.asarray(self.zeta_table, dtype=np.float64)
        return np.arange(self.nzeta, dtype=np.float64) * self.h

    def grid_struct(self):
        z = np.ascontiguousarray(self.zeta)
        if self.ynode is None:
            g = abi.Grid(self.nx, self.ny, self.nzeta, 1, self.Lx, self.Ly,
                         z.ctypes.data_as(abi.C.POINTER(abi.C.c_double)), None)
            return g, z        # keep z alive while g is used
        y = np.ascontiguousarray(self.ynode, dtype=np.float64)
        g = abi.Grid(self.nx, self.ny, self.nzeta, 0, self.Lx, float(y[-1] - y[0]),
                     z.ctypes.data_as(abi.C.POINTER(abi.C.c_double)), y.ctypes.data_as(abi.C.POINTER(abi.C.c_double)))
        return g, (z, y)

    def params_struct(self):
        p = abi.Params()
        d = default_params()
        d.update(self.params)
        for k, v in d.items():
            setattr(p, k, v)
        return p

    def bunch_structs(self):
        arr = (abi.Bunch * max(1, len(self.bunches)))()
        for i, b in enumerate(self.bunches):
            d = default_bunch()
            d.update(b)
            for k, v in d.items():
                setattr(arr[i], k, v)
        return arr, len(self.bunches)

    def plasma_structs(self):
        """(Plasma, Ion array, count, keep-alive list) or None without plasma."""
        if self.plasma is None:
            return None
        d = default_plasma()
        d.update(self.plasma)
        keep = []
        zp = np.ascontiguousarray(d.pop("z_points", []), dtype=np.float64)
        zv = np.ascontiguousarray(d.pop("z_values", []), dtype=np.float64)
        keep += [zp, zv]
        P = abi.Plasma()
        for k, v in d.items():
            setattr(P, k, v)
        P.n_z = len(zp)
        P.z_points = zp.ctypes.data_as(abi.C.POINTER(abi.C.c_double))
        P.z_values = zv.ctypes.data_as(abi.C.POINTER(abi.C.c_double))
        arr = (abi.Ion * max(1, len(self.ions)))()
        for i, ion in enumerate(self.ions):
            ip = np.ascontiguousarray(ion.get("ip_eV", []), dtype=np.float64)
            keep.append(ip)
            for k in ("mass", "atoms", "Z0", "Zmax", "mobile", "ionization"):
                setattr(arr[i], k, ion[k])
            arr[i].n_ip = len(ip)
            arr[i].ip_eV = ip.ctypes.data_as(abi.C.POINTER(abi.C.c_double))
        return P, arr, len(self.ions), keep

    def glaser_structs(self):
        out = []
        for g in self.glasers:
            d = dict(a0=1.0, kL=1.0, waist=10.0, tau=10.0, zeta_c=0.0, z_focus=0.0, cep=0.0, pol_angle=0.0,
                     circular=0, helicity=1)
            d.update(g)
            L = abi.GridLaser()
            for k, v in d.items():
                setattr(L, k, v)
            out.append(L)
        return out

    @property
    def grid_points(self):
        return self.nx * self.ny * self.nzeta

    @property
    def particles(self):
        return sum(int(b.get("nmacro", 0)) for b in self.bunches)


def default_params():
    """Deck defaults of the reference (sim_config.cpp:69-343) for the keys of g3d_params."""
    return dict(lambda0=0.8e-6, dz=1.0, dz_push=1.0, z_end=10.0, sponge=0.0, sponge_y=0.0, sponge_rate=0.1,
                move_x=1, move_y=1, window_lag=4, self_fields=1, zeta_filter=1, k_filter=1, push_phase=0.05,
                laser_on=0, laser_pol=abi.G3D_POL_S, laser_envelope=abi.G3D_ENV_GAUSSIAN, reserved0=0,
                a0=0.0, kL=1.0, theta=0.0, tau=1.0, cep=0.0, eta_c=0.0, stop_fwhm=0.0,
                flat_length=0.0, ramp_length=0.0, zeta_center=0.0,
                freeze_bunch=0, start_relax=1, box_mean=1, precision=abi.G3D_FP64)


def default_plasma():
    """Deck defaults of the plasma and numerics keys (sim_config.cpp:167-208)."""
    return dict(n0=0.0, r_max=1e300, channel_depth=0.0, r_channel=1.0, smooth_length=0.0, vz_min=0.8, vz_beam=0.9,
                trap_advance=1.0, ppc_x=2, ppc_y=2, iterations=2, predictor_extrapolate=1, free_electrons=1,
                parabolic=0, box_mean=1, seed=1)


# Elements used by the workloads: standard atomic mass [u] and ionization energies [eV] of every charge state,
# NIST Atomic Spectra Database (tests/test_oracle.py compares them with the reference build's table).
ELEMENTS = {
    "H": (1.008, [13.598434599702]),
    "N": (14.007, [14.53413, 29.60125, 47.4453, 77.4735, 97.8901, 552.06741, 667.0461377]),
}
M_U_KG = 1.66053906660e-27


def ion_species(symbol, Z0, atoms, ionization=False, mobile=True, Zmax=None):
    mass_u, ip = ELEMENTS[symbol]
    Zmax = (len(ip) if ionization else Z0) if Zmax is None else Zmax
    return dict(mass=mass_u * M_U_KG / ME_SI, atoms=atoms, Z0=Z0, Zmax=Zmax, mobile=1 if mobile else 0,
                ionization=1 if ionization else 0, ip_eV=list(ip))


def default_bunch():
    return dict(charge_C=0.0, gamma=2.0, sigx=1.0, sigy=1.0, sigz=1.0, length=0.0, emitx=0.0, emity=0.0,
                espread=0.0, zeta_center=0.0, x0=0.0, y0=0.0, q=-1.0, nmacro=0, seed=1, beamlet=0, noise_lambda=0.0)


def config1(nx=64, ny=64, nzeta=256, nmacro=262144, steps=10):
    """Plain FP64 frozen-bunch wake in vacuum (the CPU-runnable case)."""
    lam = 0.8e-6
    h = 0.5 * (255 / (nzeta - 1))       # keeps the 127.5 window when nzeta is reduced
    dz = 5.0
    sig, sigz = 2.0, 4.0
    q = charge_for_peak_density(0.01, sig, sig, sigz, lam)
    b = dict(charge_C=q, gamma=math.sqrt(1 + 1000.0 ** 2), sigx=sig, sigy=sig, sigz=sigz,
             emitx=0.2, emity=0.2, espread=0.0, zeta_center=64.0, nmacro=nmacro, seed=1)
    p = dict(lambda0=lam, dz=dz, dz_push=dz, z_end=dz * steps, sponge=0.0, sponge_y=0.0,
             move_x=0, move_y=0, zeta_center=64.0)
    return RunConfig("frozen-bunch wake, vacuum", nx, ny, nzeta, 40.0, 40.0, h, p, [b], steps)


def config2(nx=128, ny=128, nzeta=1024, nmacro=1048576, steps=100, envelope=abi.G3D_ENV_FLATTOP):
    """Plain FP64 oblique plane wave on a dense bunch (the headline single-GPU workload)."""
    lam = 0.8e-6
    h = 0.1 * (1023 / (nzeta - 1))
    dz = 2.0
    L = 60.0
    sig, sigz = 3.0, 6.0
    q = charge_for_peak_density(0.05, sig, sig, sigz, lam)
    window = h * (nzeta - 1)
    zc = 0.75 * window                  # reference default bunch.zeta_center (sim_bunches.cpp:49)
    b = dict(charge_C=q, gamma=500.0, sigx=sig, sigy=sig, sigz=sigz, emitx=1.0, emity=1.0, espread=1e-3,
             zeta_center=zc, nmacro=nmacro, seed=1)
    p = dict(lambda0=lam, dz=dz, dz_push=dz, z_end=dz * steps, sponge=0.1 * L, sponge_y=0.1 * L,
             zeta_center=zc, laser_on=1, laser_pol=abi.G3D_POL_P, a0=0.5, kL=1.0, theta=0.02, cep=0.0)
    if envelope == abi.G3D_ENV_FLATTOP:
        # plateau 60, sin^2 ramps 10; the bunch sits in the plateau (eta_c = 0)
        p.update(laser_envelope=abi.G3D_ENV_FLATTOP, flat_length=60.0, ramp_length=10.0, tau=60.0, eta_c=0.0,
                 stop_fwhm=0.0)
    else:
        # the reference's Gaussian envelope with the same intensity FWHM, centred on the bunch
        p.update(laser_envelope=abi.G3D_ENV_GAUSSIAN, tau=60.0, eta_c=0.0, stop_fwhm=0.0)
    return RunConfig("oblique plane wave on a bunch", nx, ny, nzeta, L, L, h, p, [b], steps)


def config3(nx=256, ny=256, nzeta=2048, nmacro=4194304, steps=200, charge_pC=10.0, h=None):
    """Laser wakefield with streaming plasma: 256x256 modes, 2048 slices (h = 0.2), n0 = 0.002 n_c with 2x2 electrons
    per cell and mobile H+ ions, Gaussian grid laser a0 = 2, w0 = 20, tau_FWHM = 30 (1/omega0), focus at s = 0,
    a witness bunch of 4,194,304 electrons (gamma 200, sigma_perp 1, sigma_zeta 2) 60 behind the laser peak,
    200 s-steps of 10.

    h None: fewer slices keep the window of 409.4 (a coarser h). h given (0.2: the workload's own step): a window of
    h (nzeta - 1), shorter with fewer slices; the laser peak then sits min(0.8 window, window - 20) from the rear and
    the witness min(60, 0.6 x that) behind it, which is the full workload's placement at 2048 slices."""
    lam = 0.8e-6
    if h is None:
        h = 0.2 * (2047 / (nzeta - 1))
    dz = 10.0
    L = 80.0
    window = h * (nzeta - 1)
    zl = min(0.8 * window, window - 20.0)  # laser peak
    zb = zl - min(60.0, 0.6 * zl)          # witness centre
    b = dict(charge_C=charge_pC * 1e-12, gamma=200.0, sigx=1.0, sigy=1.0, sigz=2.0, emitx=0.0, emity=0.0,
             espread=0.0, zeta_center=zb, nmacro=nmacro, seed=1)
    p = dict(lambda0=lam, dz=dz, dz_push=dz, z_end=dz * steps, sponge=0.1 * L, sponge_y=0.1 * L, zeta_center=zb,
             move_x=0, move_y=0)
    plasma = dict(n0=0.002, ppc_x=2, ppc_y=2, seed=1)
    ions = [ion_species("H", 1, 1.0)]
    gl = [dict(a0=2.0, kL=1.0, waist=20.0, tau=30.0, zeta_c=zl, z_focus=0.0)]
    return RunConfig("laser wakefield with plasma", nx, ny, nzeta, L, L, h, p, [b], steps, plasma, ions, gl)


def lwfa_small(nx=16, ny=16, nzeta=64, nmacro=600, steps=2, ions=True, a0=1.0, n0=0.01, ppc=2, passes=2,
               extrapolate=1, smooth=0.0):
    """A small laser wakefield (the structure of workload 3 at test sizes): streaming plasma with mobile H+ ions,
    a Gaussian grid laser and a witness bunch."""
    lam = 0.8e-6
    L = 24.0
    h = 0.4 * (63 / (nzeta - 1))
    window = h * (nzeta - 1)
    zl = 0.7 * window
    zb = zl - 10.0
    b = dict(charge_C=0.05e-12, gamma=50.0, sigx=1.0, sigy=1.0, sigz=1.5, emitx=0.05, emity=0.05, espread=0.0,
             zeta_center=zb, nmacro=nmacro, seed=3)
    p = dict(lambda0=lam, dz=2.0, dz_push=2.0, z_end=2.0 * steps, sponge=2.4, sponge_y=2.4, zeta_center=zb,
             move_x=0, move_y=0)
    plasma = dict(n0=n0, ppc_x=ppc, ppc_y=ppc, iterations=passes, predictor_extrapolate=extrapolate,
                  smooth_length=smooth, seed=3)
    ion_list = [ion_species("H", 1, 1.0)] if ions else []
    gl = [dict(a0=a0, kL=1.0, waist=6.0, tau=6.0, zeta_c=zl, z_focus=2.0)]
    return RunConfig("small laser wakefield", nx, ny, nzeta, L, L, h, p, [b], steps, plasma, ion_list, gl)


def ionization_small(nx=16, ny=16, nzeta=64, steps=2, a0=2.5):
    """Small ionization injection (the structure of workload 5 on a Fourier grid): neutral gas of atomic H (the
    H2 of the workload at twice the density) and 1 % N, ADK ionization of every level, a grid laser."""
    lam = 0.8e-6
    L = 24.0
    h = 0.4 * (63 / (nzeta - 1))
    window = h * (nzeta - 1)
    zl = 0.7 * window
    p = dict(lambda0=lam, dz=2.0, dz_push=2.0, z_end=2.0 * steps, sponge=2.4, sponge_y=2.4, zeta_center=0.0,
             move_x=0, move_y=0)
    plasma = dict(n0=0.002, ppc_x=1, ppc_y=1, free_electrons=0, seed=7)
    ion_list = [ion_species("H", 0, 2 * 0.99, ionization=True), ion_species("N", 0, 0.01, ionization=True)]
    gl = [dict(a0=a0, kL=1.0, waist=6.0, tau=6.0, zeta_c=zl, z_focus=0.0)]
    return RunConfig("small ionization injection", nx, ny, nzeta, L, L, h, p, [], steps, plasma, ion_list, gl)


def adjoint_small(nx=16, ny=16, nzeta=64, nmacro=2000, steps=3, gamma=10.0, a0=1.0, charge_pC=0.01):
    """The structure of the adjoint workload at test size: a witness bunch inside a Gaussian grid laser in vacuum
    (no sponge, fixed window), h = 0.25."""
    lam = 0.8e-6
    L = 24.0
    h = 0.25 * (63 / (nzeta - 1))
    window = h * (nzeta - 1)
    zl = 0.5 * window
    b = dict(charge_C=charge_pC * 1e-12, gamma=gamma, sigx=1.0, sigy=1.0, sigz=1.0, emitx=0.05, emity=0.05, espread=0.0,
             zeta_center=zl, nmacro=nmacro, seed=4)
    p = dict(lambda0=lam, dz=1.0, dz_push=1.0, z_end=1.0 * steps, sponge=0.0, sponge_y=0.0, zeta_center=zl,
             move_x=0, move_y=0)
    gl = [dict(a0=a0, kL=1.0, waist=6.0, tau=4.0, zeta_c=zl, z_focus=0.0)]
    return RunConfig("adjoint: witness bunch in a grid laser", nx, ny, nzeta, L, L, h, p, [b], steps, None, [], gl)


def adjoint_plasma_small(nx=16, ny=16, nzeta=64, nmacro=2000, steps=3, gamma=10.0, a0=0.5, charge_pC=0.01, n0=0.01,
                         passes=2, extrapolate=1, smooth=0.0, ions=True):
    """The adjoint test case with a streaming plasma (the structure of workload 4): the witness bunch inside a Gaussian
    grid laser in a plasma of n0 at 2 x 2 per cell, mobile H+ ions, no sponge, fixed window. a0 = 0.5 keeps every plasma
    electron streaming (at a0 = 1 and dz = 1 about 130 a step advance a whole step in z inside the window and are
    trapped, an event the adjoint does not differentiate)."""
    cfg = adjoint_small(nx, ny, nzeta, nmacro, steps, gamma, a0, charge_pC)
    cfg.name = "adjoint: witness bunch in a grid laser and a streaming plasma"
    cfg.plasma = dict(n0=n0, ppc_x=2, ppc_y=2, iterations=passes, predictor_extrapolate=extrapolate,
                      smooth_length=smooth, seed=3)
    cfg.ions = [ion_species("H", 1, 1.0)] if ions else []
    return cfg


def config4(nx=64, ny=64, nzeta=512, nmacro=65536, steps=40, gamma=100.0, a0=1.0, charge_pC=1.0, plasma=False):
    """Workload 4 without its plasma: a Gaussian grid laser (a0 1, waist 10, tau 10) and a bunch of 65,536
    electrons (gamma 100, sigma_perp 1, sigma_zeta 1) inside the pulse, 64 x 64 modes over 40 x 40, 512 slices
    with h = 0.25, 40 s-steps of dz = 2: the frozen-bunch/laser march the adjoint differentiates."""
    lam = 0.8e-6
    L = 40.0
    h = 0.25 * (511 / (nzeta - 1))
    window = h * (nzeta - 1)
    zl = 0.5 * window
    b = dict(charge_C=charge_pC * 1e-12, gamma=gamma, sigx=1.0, sigy=1.0, sigz=1.0, emitx=0.1, emity=0.1, espread=0.0,
             zeta_center=zl, nmacro=nmacro, seed=4)
    p = dict(lambda0=lam, dz=2.0, dz_push=2.0, z_end=2.0 * steps, sponge=0.0, sponge_y=0.0, zeta_center=zl,
             move_x=0, move_y=0)
    gl = [dict(a0=a0, kL=1.0, waist=10.0, tau=10.0, zeta_c=zl, z_focus=0.0)]
    if plasma:        # workload 4 as specified: a streaming plasma of 0.005 n_c at 2 x 2 per cell
        pl = dict(n0=0.005, ppc_x=2, ppc_y=2, iterations=2, predictor_extrapolate=1, seed=4)
        return RunConfig("frozen-bunch/laser march with a streaming plasma (workload 4)", nx, ny, nzeta, L, L, h, p, [b], steps,
                         pl, [], gl)
    return RunConfig("frozen-bunch/laser march (workload 4 without plasma)", nx, ny, nzeta, L, L, h, p, [b], steps, None,
                     [], gl)


def walled_ynode(half, dy0, core, grow, wall):
    """Nodes of a free-hand y grid between conducting walls at -wall and +wall, symmetric about 0, `half` cells a
    side: cells of dy0 for |y| < core, then cells growing by a constant ratio <= grow up to a size d, then cells of
    d out to the wall. d (and the ratio) are found so that the cells end exactly at the wall."""
    n_core = int(round(core / dy0))

    def side(d):
        ng = max(1, math.ceil(math.log(d / dy0) / math.log(grow) - 1e-12)) if d > dy0 else 0
        r = (d / dy0) ** (1.0 / ng) if ng else 1.0
        cells = [dy0] * n_core + [dy0 * r ** k for k in range(1, ng + 1)]
        cells += [d] * (half - len(cells))
        return cells[:half]
    lo, hi = dy0, wall
    for _ in range(200):                      # the outer cell size d that lands on the wall
        mid = 0.5 * (lo + hi)
        if sum(side(mid)) < wall:
            lo = mid
        else:
            hi = mid
    cells = np.array(side(hi))
    cells *= wall / cells.sum()               # the last rounding: exactly at the wall
    pos = np.concatenate([[0.0], np.cumsum(cells)])
    return np.concatenate([-pos[:0:-1], pos])


def stepped_zeta(nzeta, h_fine, h_coarse, ratio, fine_frac=0.2, front_frac=0.25):
    """Slice positions of a free-hand zeta grid with nzeta slices: from the rear, coarse steps h_coarse, steps
    shrinking by `ratio` down to h_fine, a fine region of fine_frac of the slices, steps growing back by `ratio`, and
    coarse steps to the front (front_frac of the coarse slices in front of the fine region). Returns (zeta, start
    and end of the fine region)."""
    ramp = [h_fine * ratio ** k for k in range(1, 1 + math.ceil(math.log(h_coarse / h_fine) / math.log(ratio)))]
    ramp = [min(h, h_coarse) for h in ramp]
    n_steps = nzeta - 1
    n_fine = max(1, int(fine_frac * n_steps))
    n_coarse = n_steps - n_fine - 2 * len(ramp)
    if n_coarse < 2:
        raise ValueError("too few slices for the graded zeta grid")
    n_front = max(1, int(front_frac * n_coarse))
    steps = [h_coarse] * (n_coarse - n_front) + ramp[::-1] + [h_fine] * n_fine + ramp + [h_coarse] * n_front
    z = np.concatenate([[0.0], np.cumsum(steps)])
    f0 = n_coarse - n_front + len(ramp)
    return z, float(z[f0]), float(z[f0 + n_fine])


def config5(nx=256, half=96, nzeta=4096, ppc=13, steps=100, a0=2.5):
    """Ionization injection on free-hand grids: x of 256 Fourier modes over 80; y a table between conducting walls at
    +-40, cells of 0.1 for |y| < 4 growing by <= 15 % a cell to the outer size (2 x 96 cells, 193 nodes); zeta a table
    of 4096 slices, h = 0.05 in the injection region (a fifth of the slices, behind the laser) grading by 5 % a slice
    to h = 0.5 elsewhere. The gas is 99 % H2 (as atomic H at twice the density) and 1 % N, neutral, ionized by ADK
    over all levels (NIST energies), n0 = 0.001 n_c, no free electrons; a Gaussian grid laser a0 = 2.5, w0 = 15,
    FWHM 30, focus at s = 0, 30 behind the window front; 100 s-steps of 10. The macro-particles of a step are the
    lattice points of the 256 x 190 cells inside the walls times ppc x ppc per cell times the two species:
    16,440,320 at ppc = 13 (the workload's 16,777,216 rounded down to a square lattice)."""
    lam = 0.8e-6
    L = 80.0
    y = walled_ynode(half, 0.1, 4.0, 1.15, 40.0)
    z, f0, f1 = stepped_zeta(nzeta, 0.05, 0.5, 1.05)
    window = float(z[-1])
    zl = window - 30.0
    p = dict(lambda0=lam, dz=10.0, dz_push=10.0, z_end=10.0 * steps, sponge=0.1 * L, sponge_y=4.0,
             zeta_center=0.5 * (f0 + f1), move_x=0, move_y=0)
    plasma = dict(n0=0.001, ppc_x=ppc, ppc_y=ppc, free_electrons=0, seed=5)
    ion_list = [ion_species("H", 0, 2 * 0.99, ionization=True), ion_species("N", 0, 0.01, ionization=True)]
    gl = [dict(a0=a0, kL=1.0, waist=15.0, tau=30.0, zeta_c=zl, z_focus=0.0)]
    cfg = RunConfig("ionization injection on free-hand y and zeta grids", nx, 2 * half, nzeta, L, float(y[-1] - y[0]),
                    0.05, p, [], steps, plasma, ion_list, gl)
    cfg.ynode = y
    cfg.zeta_table = z
    return cfg


def baseline(k, **kw):
    if k == 1:
        return config1(**kw)
    if k == 2:
        return config2(**kw)
    if k == 3:
        return config3(**kw)
    if k == 5:
        return config5(**kw)
    raise NotImplementedError(f"workload {k} is not built by this release")


def graded_ynode(half, dy0, grow, core):
    """Nodes of a free-hand y grid symmetric about 0: cells of dy0 for |y| < core, each further cell `grow` times
    the previous one, `half` cells on each side (the walls at the ends)."""
    pos = [0.0]
    d = dy0
    for _ in range(half):
        if pos[-1] >= core:
            d *= grow
        pos.append(pos[-1] + d)
    pos = np.array(pos)
    return np.concatenate([-pos[:0:-1], pos])


def on_freehand_y(cfg, half=14, dy0=0.5, grow=1.15, core=2.5):
    """The same run on a free-hand y grid between walls: 2 x `half` graded cells (dy0 for |y| < core, each further
    cell `grow` times the previous one)."""
    y = graded_ynode(half, dy0, grow, core)
    cfg.ynode = y
    cfg.ny = 2 * half
    cfg.Ly = float(y[-1] - y[0])
    cfg.name += " on the free-hand y grid"
    return cfg


def graded_zeta(window, center, h_fine, h_coarse, grow, core):
    """Slice positions 0 .. >= window: steps of h_fine within `core` of `center`, each further step `grow` times
    the previous one up to h_coarse."""
    def side(length):
        pos, d, x = [0.0], h_fine, 0.0
        while x < length:
            if x >= core:
                d = min(h_coarse, d * grow)
            x += d
            pos.append(x)
        return np.array(pos)
    back = center - side(center)[::-1]          # down to <= 0
    front = center + side(window - center)[1:]   # up to >= window
    z = np.concatenate([back, front])
    return z - z[0]


def on_graded_zeta(cfg, fine=0.5, coarse=2.0, grow=1.15, core=3.0):
    """The same run on a free-hand zeta grid: steps of fine * h within `core` of the first bunch's centre (of the
    laser's, without a bunch), growing by `grow` per slice up to coarse * h; bunch and laser keep their distance
    from the window front."""
    z0 = cfg.zeta
    window = float(z0[-1])
    c = cfg.bunches[0]["zeta_center"] if cfg.bunches else cfg.glasers[0]["zeta_c"]
    z = graded_zeta(window, c, fine * cfg.h, coarse * cfg.h, grow, core)
    d = z[-1] - window                          # keep every position's distance from the front
    for b in cfg.bunches:
        b["zeta_center"] += d
    for g in cfg.glasers:
        g["zeta_c"] += d
    if "zeta_center" in cfg.params:
        cfg.params["zeta_center"] += d
    cfg.zeta_table = z
    cfg.nzeta = len(z)
    cfg.name += " on a graded zeta grid"
    return cfg


def freehand_small(nx=16, half=12, nzeta=32, nmacro=3000, steps=2, sponge=1.5, zeta_filter=1, k_filter=1):
    """A frozen-bunch wake on the free-hand y grid (the structure of workload 5's y grid at test sizes): 16 Fourier
    modes in x, 2 x 12 graded cells in y between walls (0.5 near the axis, growing by 12 % per cell beyond 2.5)."""
    lam = 0.8e-6
    y = graded_ynode(half, 0.5, 1.12, 2.5)
    Lx = 12.0
    h = 0.5 * (31 / (nzeta - 1))
    window = h * (nzeta - 1)
    zc = 0.6 * window
    b = dict(charge_C=0.2e-12, gamma=200.0, sigx=1.0, sigy=1.0, sigz=2.0, emitx=0.1, emity=0.1, espread=1e-3,
             zeta_center=zc, nmacro=nmacro, seed=5)
    p = dict(lambda0=lam, dz=3.0, dz_push=3.0, z_end=3.0 * steps, sponge=sponge, sponge_y=sponge, zeta_center=zc,
             zeta_filter=zeta_filter, k_filter=k_filter, move_x=0, move_y=0)
    cfg = RunConfig("frozen bunch on the free-hand y grid", nx, 2 * half, nzeta, Lx, float(y[-1] - y[0]), h, p, [b], steps)
    cfg.ynode = y
    return cfg
