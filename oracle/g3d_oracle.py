"""Test infrastructure only: a numpy restatement of the reference GEM-PIC-3D FP64 march for Fourier y (the
checker of the CUDA path; never called by the product). Pinned against the reference build
(oracle/_ref, oracle/ref.py) and the golden fixtures in tests/test_oracle.py.

Each function cites the reference code it restates (paths inside the reference project). Vectorised over
particles and modes; loops over slices where the reference's recurrence is serial. Particles come in as the
104-byte records (the sampler is the reference's own, reproduced bit for bit by the product's host loader).
The flat-top envelope (no counterpart in the reference) is restated here from its definition in
include/g3d.h, so it is pinned only by this restatement.
"""
import math

import numpy as np

C_SI, E_SI, ME_SI, EPS0 = 299792458.0, 1.602176634e-19, 9.1093837015e-31, 8.8541878128e-12


class Oracle:
    """State and steps of one rank (a = 0, b = N) with Fourier y."""

    # ------------------------------------------------------------------ set-up: sim_setup.cpp:5-82, 148-164
    def __init__(self, cfg):
        self.cfg = cfg
        p = dict(cfg.params)
        self.P = p
        self.nx, self.ny, self.N = cfg.nx, cfg.ny, cfg.nzeta
        self.nk = self.nx * self.ny
        self.ns = self.N
        self.Lx, self.Ly = cfg.Lx, cfg.Ly
        self.dx, self.dy = cfg.Lx / cfg.nx, cfg.Ly / cfg.ny
        nx, ny, N = self.nx, self.ny, self.N
        rate = p.get("sponge_rate", 0.1)

        def prof(dd, w):
            if w <= 0 or dd >= w:
                return 1.0
            r = 1 - dd / w
            return 1 - rate * r * r

        kf = p.get("k_filter", 1)
        mx = np.where(np.arange(nx) <= nx // 2, np.arange(nx), np.arange(nx) - nx)
        self.kxs = 2 * math.pi * mx / cfg.Lx
        self.kxd = np.where(2 * np.arange(nx) == nx, 0.0, self.kxs)
        self.filt = np.cos(0.5 * self.kxs * self.dx) ** 2 if kf else np.ones(nx)
        self.filt[2 * np.arange(nx) == nx] = 0
        self.maskx = np.array([prof(min(i * self.dx, cfg.Lx - i * self.dx), p.get("sponge", 0.0)) for i in range(nx)])
        my = np.where(np.arange(ny) <= ny // 2, np.arange(ny), np.arange(ny) - ny)
        self.kys = 2 * math.pi * my / cfg.Ly
        self.kyd = np.where(2 * np.arange(ny) == ny, 0.0, self.kys)
        self.filty = np.cos(0.5 * self.kys * self.dy) ** 2 if kf else np.ones(ny)
        self.filty[2 * np.arange(ny) == ny] = 0
        self.masky = np.array([prof(min(j * self.dy, cfg.Ly - j * self.dy), p.get("sponge_y", 0.0)) for j in range(ny)])
        # zeta (setup_zeta)
        Z = cfg.zeta
        self.zeta = Z
        hh = np.diff(Z)
        self.uniform = bool(np.all(hh == hh[0]))
        if self.uniform:
            hh = np.full(N - 1, Z[-1] / (N - 1))
        self.hh = hh
        g = np.array([hh[min(max(m, 0), N - 2)] for m in range(-2, N + 1)])
        self.hcg = g                                        # hcg[m + 2] = h_m
        hm, hp = g[1:N + 1], g[2:N + 2]
        self.wlo, self.whi = hp / (hm + hp), hm / (hm + hp)
        self.wsl = 0.5 * (np.concatenate([[0.0], hh]) + np.concatenate([hh, [0.0]]))
        self.ih = 1 / hh[0]
        self.hmin = float(np.min(np.diff(Z)))
        # state (reference layouts as [plane, j, ix])
        c = np.complex128
        self.Rx, self.Ry, self.Ez, self.Bz, self.Lx_, self.Ly_ = (np.zeros((N, ny, nx), c) for _ in range(6))
        self.j0x, self.j0y, self.jkx, self.jky, self.jkz = (np.zeros((N + 1, ny, nx), c) for _ in range(5))
        self.jw = np.zeros((3, N + 3, ny, nx))
        self.F = np.zeros((6, N + 2, ny, nx), np.float32)
        self.parts = None
        self.s, self.istep, self.X0, self.Y0 = 0.0, 0, 0.0, 0.0
        self.beta_b, self.gm2_b = 1.0, 0.0
        self.starting = False
        self.cent = []
        # laser (sim_setup.cpp:51-54)
        self.laser = dict(on=p.get("laser_on", 0), pol=p.get("laser_pol", 0), env=p.get("laser_envelope", 0),
                          a0=p.get("a0", 0.0), kL=p.get("kL", 1.0), tau=p.get("tau", 1.0), cep=p.get("cep", 0.0),
                          eta_c=p.get("eta_c", 0.0), kx=math.sin(p.get("theta", 0.0)), kz=math.cos(p.get("theta", 0.0)),
                          flat=p.get("flat_length", 0.0), ramp=p.get("ramp_length", 0.0))

    # ------------------------------------------------------------------ helpers
    def locate(self, x):
        """Axis::locate (grid.hpp:329-340) on the zeta slices; arrays."""
        x = np.asarray(x, dtype=np.float64)
        if self.uniform:
            t = (x - 0.0) * self.ih
            i = np.floor(t).astype(np.int64)
            return i, t - i
        Z = self.zeta
        i = np.searchsorted(Z, x, side="right") - 1
        f = np.empty_like(x)
        lo = x < Z[0]
        hi = x >= Z[-1]
        mid = ~(lo | hi)
        t = (x[lo] - Z[0]) / (Z[1] - Z[0])
        i[lo] = np.floor(t).astype(np.int64)
        f[lo] = t - i[lo]
        t = (x[hi] - Z[-1]) / (Z[-1] - Z[-2])
        k = np.floor(t).astype(np.int64)
        i[hi] = self.N - 1 + k
        f[hi] = t - k
        im = i[mid]
        f[mid] = (x[mid] - Z[im]) / (Z[im + 1] - Z[im])
        return i, f

    @staticmethod
    def tsc(x, d, n):
        """tsc / tsc_index (sim_kernels.hpp:21-31): 3 indices (wrapped) and weights, shape (..., 3)."""
        xi = x / d
        i0 = np.floor(xi + 0.5).astype(np.int64)
        f = xi - i0
        w = np.stack([0.5 * (0.5 - f) ** 2, 0.75 - f * f, 0.5 * (0.5 + f) ** 2], axis=-1)
        idx = np.stack([i0 - 1, i0, i0 + 1], axis=-1) % n
        return idx, w

    def set_particles(self, parts):
        self.parts = np.array(parts, copy=True)

    def host_particles(self):
        return self.parts.copy()

    def set_origin(self, X0, Y0):
        self.X0, self.Y0 = X0, Y0

    # ------------------------------------------------------------------ currents: sim_particles.cpp:56-156
    def currents(self):
        nx, ny, N, nk = self.nx, self.ny, self.N, self.nk
        nh = N + 3
        J = np.zeros((3, nh, ny, nx))
        P = self.parts
        al = P["alive"] == 1
        m, fz = self.locate(P["zeta"])
        hw = m + 2
        ok = al & (hw >= 0) & (hw < nh) & (m >= 0) & (m <= N - 2)
        q = P[ok]
        m, hw = m[ok], hw[ok]
        g = np.sqrt(1 + q["px"] ** 2 + q["py"] ** 2 + q["pz"] ** 2)
        vx, vy, vz = q["px"] / g, q["py"] / g, q["pz"] / g
        f = q["q"] * q["w"] / (self.hcg[m + 2] * self.dx)
        ix, wx = self.tsc(q["x"], self.dx, nx)
        jn, wn = self.tsc(q["y"], self.dy, ny)
        ia0 = 1 / self.dy
        for v in range(3):
            for u in range(3):
                w = f * wx[:, u] * wn[:, v] * ia0
                np.add.at(J[0], (hw, jn[:, v], ix[:, u]), w * vx / vz)
                np.add.at(J[1], (hw, jn[:, v], ix[:, u]), w * vy / vz)
                np.add.at(J[2], (hw, jn[:, v], ix[:, u]), w)
        self.jw = J
        # zeta filter on the half-cell charges into the half-cells a-1 .. b-1 (hk = 0..ns)
        zf = self.P.get("zeta_filter", 1)
        v = np.zeros((3, N + 1, ny, nx))
        for hk in range(N + 1):
            hc = hk - 1
            w_ = hk + 1
            if hc < 0 or hc > N - 2:
                continue
            if zf and self.uniform:
                v[:, hk] = 0.25 * J[:, w_ - 1] + 0.5 * J[:, w_] + 0.25 * J[:, w_ + 1]
            elif zf:
                hg = self.hcg
                v[:, hk] = (0.25 * hg[hc + 1] * J[:, w_ - 1] + 0.5 * hg[hc + 2] * J[:, w_] +
                            0.25 * hg[hc + 3] * J[:, w_ + 1]) / hg[hc + 2]
            else:
                v[:, hk] = J[:, w_]
        s1 = np.fft.fft2(v[0] + 1j * v[1], axes=(-2, -1))
        jz = np.fft.fft2(v[2] + 0j, axes=(-2, -1))
        # unpack the pair and apply the transverse filters (Fourier y)
        zm = np.conj(np.roll(np.flip(s1, axis=(-2, -1)), 1, axis=(-2, -1)))
        keep0 = False
        f = self.filty[:, None] * self.filt[None, :]
        f = f.copy()
        if not keep0:
            f[0, 0] = 0.0
        self.jkx = f * (0.5 * (s1 + zm))
        d = s1 - zm
        self.jky = f * (0.5 * (d.imag - 1j * d.real))
        self.jkz = f * jz
        self.jk_alias = False

    # ------------------------------------------------------------------ march: sim_kernels.hpp:173-210
    def march(self, D):
        N = self.N
        KX = self.kxd[None, :] * np.ones((self.ny, 1))
        KY = self.kyd[:, None] * np.ones((1, self.nx))
        k2 = KX ** 2 + KY ** 2
        a, b = 1j * KX, 1j * KY
        p = None
        for n in range(N - 1, -1, -1):
            wl, wu = self.wlo[n], self.whi[n]
            Jx = wl * (self.j0x[n] + self.jkx[n]) + wu * (self.j0x[n + 1] + self.jkx[n + 1])
            Jy = wl * (self.j0y[n] + self.jky[n]) + wu * (self.j0y[n + 1] + self.jky[n + 1])
            Rsx = self.Rx[n] + D * (a * self.Ez[n] + b * self.Bz[n]) - D * Jx
            Rsy = self.Ry[n] + D * (b * self.Ez[n] - a * self.Bz[n]) - D * Jy
            if n == N - 1:
                self.Rx[n], self.Ry[n] = Rsx, Rsy
                z = np.zeros_like(Rsx)
                self.Ez[n], self.Bz[n], self.Lx_[n], self.Ly_[n] = z, z.copy(), z.copy(), z.copy()
                continue
            pRx, pRy, pEz, pBz, pLx, pLy = (A[n + 1] for A in (self.Rx, self.Ry, self.Ez, self.Bz, self.Lx_, self.Ly_))
            h = self.hcg[n + 2]
            upx, upy, upz = self.jkx[n + 1], self.jky[n + 1], self.jkz[n + 1]
            Lsx = pLx - 0.25 * h * (a * pEz - b * pBz) - 0.5 * h * upx
            Lsy = pLy - 0.25 * h * (a * pBz + b * pEz) - 0.5 * h * upy
            Cp = 0.5 * (a * (pRy + pLy) - b * (pRx + pLx))
            Qp = -0.5 * (a * (pRx - pLx)) + 0.5 * (b * (pLy - pRy))
            SB = a * Rsy + a * Lsy - b * Rsx - b * Lsx
            SE = -(a * Rsx) + a * Lsx + b * Lsy - b * Rsy
            den = 1 + 0.25 * h * (D + 0.25 * h) * k2
            Bzn = (pBz - 0.5 * h * Cp - 0.25 * h * SB) / den
            Ezn = (pEz - 0.5 * h * Qp - 0.25 * h * SE - h * upz) / den
            self.Ez[n], self.Bz[n] = Ezn, Bzn
            self.Rx[n] = Rsx + D * (a * Ezn + b * Bzn)
            self.Ry[n] = Rsy + D * (b * Ezn - a * Bzn)
            self.Lx_[n] = Lsx - 0.25 * h * (a * Ezn - b * Bzn)
            self.Ly_[n] = Lsy - 0.25 * h * (a * Bzn + b * Ezn)

    # ------------------------------------------------------------------ sponge and real fields: sim_fields.cpp:156-293
    def sponge_and_real_fields(self):
        N, nk = self.N, self.nk
        KX = self.kxd[None, :] * np.ones((self.ny, 1))
        KY = self.kyd[:, None] * np.ones((1, self.nx))
        k2 = KX ** 2 + KY ** 2
        if self.P.get("sponge", 0) > 0 or self.P.get("sponge_y", 0) > 0:
            g2, opb = self.gm2_b, 1 + self.beta_b
            jz = self.jkz                                  # half-cells 0..N; ghosts (a-2, b) are zero on one rank

            def half(hk):
                if hk < 0 or hk > N:
                    return np.zeros_like(jz[0])
                return jz[hk]

            def rho_at(n):
                if n < 0 or n > N - 1:
                    return np.zeros_like(jz[0])
                return self.wlo[n] * half(n) + self.whi[n] * half(n + 1)

            mask = self.masky[:, None] * self.maskx[None, :]
            for n in range(N):
                hm, hp = self.hcg[n + 1], self.hcg[n + 2]
                cm, cp = 2 / ((hm + hp) * hm), 2 / ((hm + hp) * hp)
                with np.errstate(divide="ignore", invalid="ignore"):
                    d2 = g2 * (cp * rho_at(n + 1) - (cm + cp) * rho_at(n) + cm * rho_at(n - 1))
                    psi = np.where(k2 > 0, (rho_at(n) + d2 / k2) / k2, 0)
                bx, by = -opb * (1j * KX * psi), -opb * (1j * KY * psi)
                u, v = self.Rx[n] - bx, self.Ry[n] - by
                s = np.fft.ifft2(u + 1j * v)
                s = mask * s.real + 1j * mask * s.imag
                z = np.fft.fft2(s)
                zm = np.conj(np.roll(np.flip(z, axis=(-2, -1)), 1, axis=(-2, -1)))
                d = z - zm
                self.Rx[n] = 0.5 * (z + zm) - opb * (1j * KX * psi)
                self.Ry[n] = 0.5 * (d.imag - 1j * d.real) - opb * (1j * KY * psi)
        s1 = np.fft.ifft2(self.Rx + 1j * self.Ry, axes=(-2, -1))
        s2 = np.fft.ifft2(self.Lx_ + 1j * self.Ly_, axes=(-2, -1))
        s3 = np.fft.ifft2(self.Ez + 1j * self.Bz, axes=(-2, -1))
        r1, r2, l1, l2 = s1.real, s1.imag, s2.real, s2.imag
        F = self.F
        F[0, :N] = (0.5 * (r1 + l1)).astype(np.float32)
        F[1, :N] = (0.5 * (r2 + l2)).astype(np.float32)
        F[3, :N] = (0.5 * (l2 - r2)).astype(np.float32)
        F[4, :N] = (0.5 * (r1 - l1)).astype(np.float32)
        F[2, :N] = s3.real.astype(np.float32)
        F[5, :N] = s3.imag.astype(np.float32)

    def j0_from_jk(self):
        self.j0x, self.j0y = self.jkx.copy(), self.jky.copy()

    def solve_fields(self, D):
        self.currents()
        self.march(D)
        self.sponge_and_real_fields()
        self.j0_from_jk()

    # ------------------------------------------------------------------ co-moving field: sim_fields.cpp:44-151
    def comoving_field(self, comoving_c=False):
        P = self.parts
        al = P["alive"] == 1
        g = np.sqrt(1 + P["px"][al] ** 2 + P["py"][al] ** 2 + P["pz"][al] ** 2)
        s0, s1 = float(np.sum(P["w"][al] * P["pz"][al] / g)), float(np.sum(P["w"][al]))
        beta = 1.0 if comoving_c else (s0 / s1 if s1 > 0 else 1.0)
        gm2 = 1 - beta * beta
        if not comoving_c:
            self.beta_b, self.gm2_b = beta, gm2
        N = self.N
        KX = self.kxd[None, :] * np.ones((self.ny, 1))
        KY = self.kyd[:, None] * np.ones((1, self.nx))
        ev = KY ** 2
        cprev = np.zeros(KX.shape)
        dprev = np.zeros(KX.shape, np.complex128)
        cp = np.zeros((N,) + KX.shape)
        dp = np.zeros((N,) + KX.shape, np.complex128)
        for n in range(N):
            hm, hp = self.hcg[n + 1], self.hcg[n + 2]
            lo, up = -gm2 * 2 / ((hm + hp) * hm), -gm2 * 2 / ((hm + hp) * hp)
            dg = KX ** 2 + ev + gm2 * 2 / (hm * hp)
            live = dg != 0
            rhs = (1 / beta) * (self.wlo[n] * self.jkz[n] + self.whi[n] * self.jkz[n + 1])
            if n == 0:
                cprev[:] = 0
                dprev[:] = 0
            with np.errstate(divide="ignore", invalid="ignore"):
                den = dg - lo * cprev
                c_ = np.where(live, up / den, 0.0)
                d_ = np.where(live, (rhs - lo * dprev) / den, 0.0)
            cp[n], dp[n] = c_, d_
            cprev = np.where(live, c_, cprev)
            dprev = np.where(live, d_, dprev)
        nxt = np.zeros(KX.shape, np.complex128)
        for n in range(N - 1, -1, -1):
            nxt = dp[n] - cp[n] * nxt
            dp[n] = nxt
        opb = 1 + beta
        self.Rx = -opb * (1j * KX * dp)
        self.Ry = -opb * (1j * KY * dp)
        self.Ez = np.zeros_like(self.Rx)
        self.Bz = np.zeros_like(self.Rx)

    def relax_start_field(self):
        """sim_fields.cpp:384-410."""
        dx, dy = self.Rx.copy(), self.Ry.copy()
        self.comoving_field(comoving_c=True)
        dx, dy = dx - self.Rx, dy - self.Ry
        D = 100 * self.P["dz"]
        for _ in range(3):
            self.Ez[:] = 0
            self.Bz[:] = 0
            self.j0x[:] = 0
            self.j0y[:] = 0
            self.march(D)
        self.Rx = self.Rx + dx
        self.Ry = self.Ry + dy

    def init_fields(self):
        """Simulation::init after the bunch load (sim_setup.cpp:180-196), one bunch, no grid lasers."""
        self.s, self.istep = 0.0, 0
        if self.P.get("self_fields", 1):
            self.starting = True
            self.currents()
            self.comoving_field()
            if self.P.get("start_relax", 1):
                self.relax_start_field()
            self.march(0.0)
            self.starting = False
            self.sponge_and_real_fields()
            self.j0_from_jk()
        self.window_shift_post()

    # ------------------------------------------------------------------ push: sim_kernels.hpp:44-149
    def laser_field(self, x, z, t):
        L = self.laser
        E = np.zeros((3,) + np.shape(x))
        B = np.zeros_like(E)
        if not L["on"]:
            return E, B
        xi = t - L["kx"] * x - L["kz"] * z - L["eta_c"]
        if L["env"] == 0:
            live = np.abs(xi) <= 5 * L["tau"]
            g = np.exp(-1.3862943611198906 * xi * xi / (L["tau"] * L["tau"]))
            gp = -2.7725887222397811 * xi / (L["tau"] * L["tau"]) * g
        else:
            ax, hf, rp = np.abs(xi), 0.5 * L["flat"], L["ramp"]
            u = (hf + rp - ax) / rp
            sn, cs = np.sin(0.5 * math.pi * u), np.cos(0.5 * math.pi * u)
            plateau = ax <= hf
            live = ax < hf + rp
            g = np.where(plateau, 1.0, sn * sn)
            gp = np.where(plateau, 0.0, np.where(xi > 0, -1.0, 1.0) * (math.pi / rp) * sn * cs)
        ph = L["kL"] * xi + L["cep"]
        c, s = np.cos(ph), np.sin(ph)
        d1 = np.where(live, L["a0"] * (gp * c - L["kL"] * g * s), 0.0)
        d2 = np.where(live, L["a0"] * (gp * s + L["kL"] * g * c), 0.0)
        if L["pol"] == 0:
            E[1] = -d1
        elif L["pol"] == 1:
            E[0] = -d1 * L["kz"]
            E[2] = d1 * L["kx"]
        else:
            E[0] = -d1 * L["kz"]
            E[2] = d1 * L["kx"]
            E[1] = -d2
        B[0] = -L["kz"] * E[1]
        B[1] = L["kz"] * E[0] - L["kx"] * E[2]
        B[2] = L["kx"] * E[1]
        return E, B

    def gather(self, x, y, zeta):
        E = np.zeros((3,) + x.shape)
        B = np.zeros_like(E)
        if not self.P.get("self_fields", 1):
            return E, B
        n, fz = self.locate(zeta)
        fix = (n == -1) & (fz > 1 - 1e-9)
        n = np.where(fix, 0, n)
        fz = np.where(fix, 0.0, fz)
        ok = (n >= 0) & (n <= self.ns)
        nn = np.clip(n, 0, self.ns)
        ix, wx = self.tsc(x, self.dx, self.nx)
        jn, wn = self.tsc(y, self.dy, self.ny)
        F = self.F.astype(np.float64)
        for comp in range(6):
            v = np.zeros(x.shape)
            for j in range(3):
                for i in range(3):
                    p0 = F[comp, nn, jn[:, j], ix[:, i]]
                    p1 = F[comp, nn + 1, jn[:, j], ix[:, i]]
                    v += wx[:, i] * wn[:, j] * ((1 - fz) * p0 + fz * p1)
            v = np.where(ok, v, 0.0)
            if comp < 3:
                E[comp] = v
            else:
                B[comp - 3] = v
        return E, B

    def rhs(self, Y, z, qm):
        x, y, zeta, px, py, pz = Y
        g = np.sqrt(1 + px * px + py * py + pz * pz)
        ok = ~(pz < 0.3 * g)
        gm = (1 + px * px + py * py) / (g + pz)
        E, B = self.gather(np.fmod(np.fmod(x, self.Lx) + self.Lx, self.Lx), np.fmod(np.fmod(y, self.Ly) + self.Ly, self.Ly),
                           zeta)
        Ee, Be = self.laser_field(x + self.X0, z, z - (zeta - self.P.get("zeta_center", 0.0)))
        E, B = E + Ee, B + Be
        ip = 1 / pz
        d = np.stack([px * ip, py * ip, -gm * ip,
                      qm * (g * E[0] + py * B[2] - pz * B[1]) * ip,
                      qm * (g * E[1] + pz * B[0] - px * B[2]) * ip,
                      qm * (g * E[2] + px * B[1] - py * B[0]) * ip])
        return d, ok

    def push(self, s0, s1):
        """RK4 of every alive particle from s0 to s1 (push_one); one rank, no plasma, no externals."""
        P = self.parts
        idx = np.nonzero(P["alive"] == 1)[0]
        q = P[idx]
        Y = np.stack([q["x"], q["y"], q["zeta"], q["px"], q["py"], q["pz"]])
        qm = q["qm"]
        z = np.full(len(idx), float(s0))
        active = np.ones(len(idx), bool)
        dead = np.zeros(len(idx), bool)
        L = self.laser
        dzp, pphase = self.P["dz_push"], self.P.get("push_phase", 0.05)
        while True:
            active &= (z < s1 - 1e-12 * abs(s1)) & ~dead
            if not active.any():
                break
            a = np.nonzero(active)[0]
            Ya, za = Y[:, a], z[a]
            px, py, pz = Ya[3], Ya[4], Ya[5]
            ds = np.where(dzp < s1 - za, dzp, s1 - za)
            g = np.sqrt(1 + px * px + py * py + pz * pz)
            lz = 0.5 * self.hmin * pz * (g + pz) / (1 + px * px + py * py)
            ds = np.where(lz < ds, (s1 - za) / np.ceil((s1 - za) / lz), ds)
            if L["on"]:
                hl = g - px * L["kx"] - pz * L["kz"]
                lim = pphase * pz / (L["kL"] * np.maximum(hl, 1e-12))
                ds = np.where(lim < ds, (s1 - za) / np.ceil((s1 - za) / lim), ds)
            qa = qm[a]
            k1, o1 = self.rhs(Ya, za, qa)
            k2, o2 = self.rhs(Ya + 0.5 * ds * k1, za + 0.5 * ds, qa)
            k3, o3 = self.rhs(Ya + 0.5 * ds * k2, za + 0.5 * ds, qa)
            k4, o4 = self.rhs(Ya + ds * k3, za + ds, qa)
            ok = o1 & o2 & o3 & o4
            w = ds / 6
            Yn = Ya + w * (k1 + 2 * k2 + 2 * k3 + k4)
            Y[:, a] = np.where(ok, Yn, Ya)
            z[a] = np.where(ok, za + ds, za)
            dead[a] |= ~ok
        zmax = self.zeta[-1]
        out = P[idx]
        # a particle whose RK4 stage failed (p_z < 0.3 gamma) is lost with the record of the start of the push
        for k, f in enumerate(["x", "y", "zeta", "px", "py", "pz"]):
            out[f] = np.where(dead, out[f], Y[k])
        out["z"] = np.where(dead, out["z"], s1)
        lost = (Y[2] < 0) | (Y[2] >= zmax)
        out["alive"] = np.where(dead | lost, 0, 1)
        P[idx] = out

    # ------------------------------------------------------------------ window, step, diagnostics
    def window_shift_post(self):
        p = self.P
        if not p.get("move_x", 1) and not p.get("move_y", 1):
            return
        P = self.parts
        m = (P["alive"] == 1) & (P["sp"] <= 0)
        w = P["w"][m]
        self.cent.append((float(np.sum(w * (P["x"][m] + self.X0))), float(np.sum(w * (P["y"][m] + self.Y0))),
                          float(np.sum(w))))

    def window_shift_start(self):
        p = self.P
        if not p.get("move_x", 1) and not p.get("move_y", 1):
            return
        if len(self.cent) < p.get("window_lag", 4):
            return
        c = self.cent.pop(0)
        if c[2] <= 0:
            return
        nxs = int(round_half_away(((c[0] / c[2]) - (self.X0 + 0.5 * self.Lx)) / self.dx)) if p.get("move_x", 1) else 0
        nys = int(round_half_away(((c[1] / c[2]) - (self.Y0 + 0.5 * self.Ly)) / self.dy)) if p.get("move_y", 1) else 0
        if abs(nxs) >= 2 or abs(nys) >= 2:
            self.shift_window(nxs, nys)

    def shift_window(self, nxs, nys):
        """sim_setup.cpp:249-281."""
        self.X0 += nxs * self.dx
        self.Y0 += nys * self.dy
        sx, sy = nxs * self.dx, nys * self.dy
        self.parts["x"] -= sx
        self.parts["y"] -= sy
        ph = self.kxs[None, :] * sx + (self.kys[:, None] * sy if nys else 0.0)
        rot = np.cos(ph) + 1j * np.sin(ph)
        for nm in ("Rx", "Ry", "Ez", "Bz", "j0x", "j0y"):
            setattr(self, nm, getattr(self, nm) * rot)
        self.F = np.roll(self.F, shift=(-nys, -nxs), axis=(-2, -1))

    def step(self):
        self.window_shift_start()
        self.push(self.s, self.s + self.P["dz"])
        self.s += self.P["dz"]
        self.istep += 1
        if self.P.get("self_fields", 1):
            self.solve_fields(0.5 * self.P["dz"])
        self.window_shift_post()

    def field_energy(self):
        """local_field_energy (sim_output.cpp:55-77), Fourier y: dual-cell weight dy for every component."""
        F = self.F[:, :self.N].astype(np.float64)
        w = self.wsl[:, None, None]
        e = 0.0
        for comp in range(6):
            e += np.sum(0.5 * w * self.dy * F[comp] * F[comp])
        return e * self.dx

    def diagnostics_sums(self):
        """The 19 sums of Simulation::diagnostics (sim_output.cpp:10-26)."""
        S = np.zeros(19)
        P = self.parts
        al = P["alive"] == 1
        tr = al & (P["sp"] > 0)
        S[17] = np.count_nonzero(tr)
        S[18] = np.sum(P["q"][tr] * P["w"][tr])
        b = P[al & (P["sp"] <= 0)]
        g = np.sqrt(1 + b["px"] ** 2 + b["py"] ** 2 + b["pz"] ** 2)
        X, Y = b["x"] + self.X0, b["y"] + self.Y0
        L = self.laser
        t = self.s - (b["zeta"] - self.P.get("zeta_center", 0.0))
        et = t - L["kx"] * X - L["kz"] * self.s
        vals = [np.ones_like(X), X, Y, b["zeta"], X * X, Y * Y, b["zeta"] ** 2, b["px"], b["py"], b["pz"], g,
                b["px"] * L["kx"] + b["pz"] * L["kz"], b["pz"] ** 2, et]
        for k, v in enumerate(vals):
            S[k] = np.sum(b["w"] * v)
        S[14] = len(b)
        S[15] = self.field_energy() if self.P.get("self_fields", 1) else 0.0
        return S

    def array(self, name):
        m = {"Rx": self.Rx, "Ry": self.Ry, "Ez": self.Ez, "Bz": self.Bz, "Lx": self.Lx_, "Ly": self.Ly_,
             "j0x": self.j0x, "j0y": self.j0y, "jkx": self.jkx, "jky": self.jky, "jkz": self.jkz,
             "jw": self.jw, "F": self.F}
        return np.ascontiguousarray(m[name]).ravel()

    def set_array(self, name, values):
        cur = self.array(name)
        v = np.asarray(values, dtype=cur.dtype).reshape(self._shape(name))
        attr = {"Lx": "Lx_", "Ly": "Ly_"}.get(name, name)
        setattr(self, attr, v.copy())

    def _shape(self, name):
        N, ny, nx = self.N, self.ny, self.nx
        if name in ("Rx", "Ry", "Ez", "Bz", "Lx", "Ly"):
            return (N, ny, nx)
        if name in ("j0x", "j0y", "jkx", "jky", "jkz"):
            return (N + 1, ny, nx)
        if name == "jw":
            return (3, N + 3, ny, nx)
        return (6, N + 2, ny, nx)


def round_half_away(x):
    """std::lround: nearest integer, halves away from zero."""
    return math.floor(x + 0.5) if x >= 0 else -math.floor(-x + 0.5)
