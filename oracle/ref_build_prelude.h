// Force-included when compiling the reference sources as a checker
// (oracle/build_ref.py).
//  * glibc's M_1_PIf32 / M_2_PIf32 are _Float32 literals, which nvcc 12.9
//    rejects in device code ("unsupported float variant"); they are redefined
//    as plain float literals of the same decimal constants, which round to the
//    same float values.
//  * <cstdint> is included because the reference relies on it arriving
//    transitively (rasterizer_impl.h:24, :41), which this toolchain does not do.
#pragma once
#include <cstdint>
#include <stdint.h>
#include <math.h>
#undef M_1_PIf32
#define M_1_PIf32 0.318309886183790671537767526745028724f
#undef M_2_PIf32
#define M_2_PIf32 0.636619772367581343075535053490057448f
