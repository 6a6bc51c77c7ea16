// Run-time dispatch of a transform length (a power of two in 4..512, or three times one in 24..384) onto the
// compile-time FFT kernels.
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
        G3D_CASE_N(24, NAME, __VA_ARGS__)                                                              \
        G3D_CASE_N(48, NAME, __VA_ARGS__)                                                              \
        G3D_CASE_N(96, NAME, __VA_ARGS__)                                                              \
        G3D_CASE_N(192, NAME, __VA_ARGS__)                                                             \
        G3D_CASE_N(384, NAME, __VA_ARGS__)                                                             \
        default: throw ::g3d::Error(G3D_ERR_ARG, "transverse sizes must be powers of two in 4..512 or three times one in 24..384"); \
    }
