// Run-time dispatch of a power-of-two transform length onto the compile-time FFT kernels.
#pragma once

#define G3D_CASE_N(VAL, NAME, ...) \
    case VAL: {                    \
        constexpr int NAME = VAL;  \
        __VA_ARGS__;               \
    } break;

#define G3D_DISPATCH_N(n, NAME, ...)                                                                   \
    switch (n) {                                                                                       \
        G3D_CASE_N(4, NAME, __VA_ARGS__)                                                               \
        G3D_CASE_N(8, NAME, __VA_ARGS__)                                                               \
        G3D_CASE_N(16, NAME, __VA_ARGS__)                                                              \
        G3D_CASE_N(32, NAME, __VA_ARGS__)                                                              \
        G3D_CASE_N(64, NAME, __VA_ARGS__)                                                              \
        G3D_CASE_N(128, NAME, __VA_ARGS__)                                                             \
        G3D_CASE_N(256, NAME, __VA_ARGS__)                                                             \
        G3D_CASE_N(512, NAME, __VA_ARGS__)                                                             \
        default: throw ::g3d::Error(G3D_ERR_ARG, "transverse sizes must be powers of two in 4..512"); \
    }
