// Compile-time dimension dispatch: the kernels are instantiated for the point
// dimensions the library supports (the reference is fixed at 100,
// src/Constants.hpp:23; 64 and 128 cover the other request shapes).
#pragma once

#define KNNG_DISPATCH_D(dval, ...)                                             \
    switch (dval) {                                                            \
        case 64: {                                                             \
            constexpr int D = 64;                                              \
            __VA_ARGS__;                                                       \
            break;                                                             \
        }                                                                      \
        case 100: {                                                            \
            constexpr int D = 100;                                             \
            __VA_ARGS__;                                                       \
            break;                                                             \
        }                                                                      \
        case 128: {                                                            \
            constexpr int D = 128;                                             \
            __VA_ARGS__;                                                       \
            break;                                                             \
        }                                                                      \
        default:                                                               \
            ::knng::fail(KNNG_ERR_UNSUPPORTED, "dimension must be 64, 100 or 128"); \
    }
