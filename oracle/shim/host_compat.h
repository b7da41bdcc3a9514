/* Forced include for the host-CPU build of the reference sources. Under nvcc the reference
 * sees the CUDA vector types (float2/float3, make_float2/3) through <curand_kernel.h>, and
 * unqualified math calls on float arguments (sqrt, sin, cos, isinf) resolve to the float
 * overloads of CUDA's device math. A host C++ compiler needs both provided explicitly:
 * without the using-declarations below, sqrt(float) would bind to the C library's
 * sqrt(double) and round differently from the device build. */
#pragma once
#include <cmath>
#include <cuda_runtime.h>
using std::cos;
using std::isinf;
using std::isnan;
using std::sin;
using std::sqrt;
