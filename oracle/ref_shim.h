// ref_shim.h -- lets the reference's CUDA C kernel sources compile as host C++ (oracle/_ref only).
//
// The reference kernels (namgpu/kernels/phys_rrtm_*.cu) are plain one-thread-per-column SIMT code: no
// shared memory, no warp intrinsics.  With the launch coordinates held in thread-local variables and the
// CUDA qualifiers mapped to host C++, each kernel is an ordinary function that the driver calls once per
// (block, thread) -- the reference's own arithmetic, statement for statement, on the CPU.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>

struct ref_dim3 {
    unsigned int x = 1, y = 1, z = 1;
};
extern thread_local ref_dim3 threadIdx, blockIdx;
extern thread_local ref_dim3 blockDim, gridDim;

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline
#define __constant__

inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline long long min(long long a, long long b) { return a < b ? a : b; }
inline long long max(long long a, long long b) { return a > b ? a : b; }
inline unsigned int min(unsigned int a, unsigned int b) { return a < b ? a : b; }
inline float __int_as_float(int i)
{
    float f;
    std::memcpy(&f, &i, 4);
    return f;
}
inline float __uint_as_float(unsigned int i)
{
    float f;
    std::memcpy(&f, &i, 4);
    return f;
}
#include <math.h>
