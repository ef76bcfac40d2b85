// Host stand-ins for the CUDA qualifiers and intrinsics that the column
// kernels use, so that their source compiles as plain C++ (g++
// -ffp-contract=off, the no-contraction setting of the GPU build).  One
// "thread" of a kernel is one call with blockIdx / threadIdx set; the warp
// intrinsics of the column-ordering kernels are never called on the host.
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#define __device__
#define __host__
#define __global__
#define __noinline__ __attribute__((noinline))
#define __forceinline__ inline
#define __launch_bounds__(...)
#define __shared__ static
typedef void *cudaStream_t;
struct U3 { unsigned x, y, z; };
static U3 blockIdx, threadIdx, blockDim, gridDim;
using std::isnan; using std::isfinite; using std::isinf; using std::sqrt; using std::fabs; using std::round;
using std::ldexp; using std::frexp; using std::signbit;
inline long long __double_as_longlong(double x) { long long r; std::memcpy(&r, &x, 8); return r; }
inline double __longlong_as_double(long long x) { double r; std::memcpy(&r, &x, 8); return r; }
inline double __dmul_rn(double a, double b) { return a * b; }
inline double __dadd_rn(double a, double b) { return a + b; }
inline double __dsub_rn(double a, double b) { return a - b; }
inline double __fma_rn(double a, double b, double c) { return std::fma(a, b, c); }
inline float __fdividef(float a, float b) { return a / b; }
inline float __frcp_rn(float a) { return 1.0f / a; }
inline unsigned __match_any_sync(unsigned, int) { return 1u; }
inline unsigned __activemask() { return 1u; }
inline int __ffs(unsigned x) { return __builtin_ffs((int)x); }
inline int __popc(unsigned x) { return __builtin_popcount(x); }
inline unsigned __shfl_sync(unsigned, unsigned v, int) { return v; }
inline unsigned atomicAdd(unsigned *a, unsigned v) { unsigned o = *a; *a += v; return o; }
inline void __syncthreads() {}
inline int cudaMemsetAsync(void *, int, size_t, cudaStream_t) { return 0; }
#include "vphys_kernels.cuh"
#include "vphys_device.cuh"
