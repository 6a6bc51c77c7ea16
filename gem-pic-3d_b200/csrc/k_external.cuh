// External magnetic elements in the lab frame, acting on the particles at their lab position (x, y, z): the fields
// are added to the gathered self-fields of the beam and streaming pushes; the field solver does not see them (reference
// src/external.hpp:1-92; the deck blocks undulator, quadrupole, plasma_lens, solenoid). Code units: B in m omega0/e.
//   undulator  psi = k_u (z - z_start), b = B0 g(z) with g the trapezoid of the linear ramps (0 outside), or with a
//              taper b = g(z) B0(z) linear in its table. Planar: B_y = b cosh(k_u y) cos psi, B_z = -b sinh(k_u y)
//              sin psi (natural focusing in y), or B_y = b cos psi without it; helical: B_x = b cos psi, B_y = b sin psi
//   quadrupole B_x = -G y, B_y = -G x (G > 0 focuses electrons in x)
//   plasma lens B_phi = -G r inside the radius R, -G R^2 / r outside
//   solenoid   B_z = B f(z), B_r = -(r/2) B f'(z), f the trapezoid of linear fringes
// The push's sub-steps stay below lambda_u / 32 inside an undulator (RK4 then follows the slippage) and below the
// element's dsmax inside a magnet, and end on every breakpoint (entrance, ends of the ramps, exit), where the field or
// its derivative jumps.
#pragma once
#include "g3d_ctx.hpp"

namespace g3d {

// the trapezoid of an element from a to b with ramps of length r at both ends: 0 outside, its slope on the ramps
__device__ __forceinline__ double ext_trapezoid(double z, double a, double b, double r) {
    if (z <= a || z >= b) return 0.0;
    if (r <= 0) return 1.0;
    return fmin(1.0, fmin((z - a) / r, (b - z) / r));
}

__device__ __forceinline__ void add_external(const ExtDev& X, double x, double y, double z, double B[3]) {
    for (int k = 0; k < X.nu; ++k) {
        const g3d_undulator& U = X.u[k];
        const double g = ext_trapezoid(z, U.z0, U.z1, U.ramp);
        if (g == 0) continue;
        double b = U.B0 * g;
        if (U.nk > 0) {                                      // taper: B0(z) linear between its table points
            const double t = (z - U.z0) / U.dzk;
            const int j = t < double(U.nk - 2) ? int(t) : U.nk - 2;
            const double w = t - j;
            b = g * ((1 - w) * X.kt[U.koff + j] + w * X.kt[U.koff + j + 1]);
        }
        const double psi = U.ku * (z - U.z0), cp = cos(psi), sp = sin(psi);
        if (U.helical) {
            B[0] += b * cp; B[1] += b * sp;
        } else if (U.focusing) {
            B[1] += b * cosh(U.ku * y) * cp; B[2] -= b * sinh(U.ku * y) * sp;
        } else {
            B[1] += b * cp;
        }
    }
    for (int k = 0; k < X.nm; ++k) {
        const g3d_magnet& M = X.m[k];
        if (z < M.z0 || z >= M.z1) continue;
        switch (M.kind) {
        case 0:                                              // quadrupole
            B[0] -= M.g * y; B[1] -= M.g * x;
            break;
        case 1: {                                            // plasma lens
            const double r2 = x * x + y * y, R2 = M.R * M.R;
            const double gr = r2 <= R2 ? M.g : M.g * R2 / r2;
            B[0] += gr * y; B[1] -= gr * x;
            break;
        }
        default: {                                           // solenoid with linear fringes
            double f = 1, df = 0;
            if (M.ramp > 0) {
                if (z - M.z0 < M.ramp) { f = (z - M.z0) / M.ramp; df = 1 / M.ramp; }
                else if (M.z1 - z < M.ramp) { f = (M.z1 - z) / M.ramp; df = -1 / M.ramp; }
            }
            B[2] += M.g * f; B[0] -= 0.5 * x * M.g * df; B[1] -= 0.5 * y * M.g * df;
        }
        }
    }
}

// the longest sub-step from z: ds, shortened inside the elements and to the next breakpoint within reach
__device__ __forceinline__ double external_step(const ExtDev& X, double z, double ds) {
    auto stop_at = [&](double b) { if (b > z + 1e-9 && b < z + ds) ds = b - z; };
    for (int k = 0; k < X.nu; ++k) {
        const g3d_undulator& U = X.u[k];
        if (z >= U.z0 - 1e-9 && z < U.z1) ds = fmin(ds, 6.283185307179586 / (32 * U.ku));
        stop_at(U.z0); stop_at(U.z0 + U.ramp); stop_at(U.z1 - U.ramp); stop_at(U.z1);
    }
    for (int k = 0; k < X.nm; ++k) {
        const g3d_magnet& M = X.m[k];
        if (z >= M.z0 - 1e-9 && z < M.z1) ds = fmin(ds, M.dsmax);
        stop_at(M.z0); stop_at(M.z0 + M.ramp); stop_at(M.z1 - M.ramp); stop_at(M.z1);
    }
    return ds;
}

}  // namespace g3d
