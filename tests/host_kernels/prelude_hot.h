// Host stand-ins for the plain FP64 kernels of the step (EOS, assembly,
// smoothing, momentum, tracers): prelude.h plus the read-only loads, the L2
// residency hints and the launch-shape types those kernels use.  The PTX
// versions of the hints are renamed out of the way before vphys_device.cuh is
// read, so that only these host versions are called (a load or store that
// ignores the policy, which is what the hint leaves of the result).
#define l2_policy_evict_last l2_policy_evict_last_ptx
#define l2_policy_evict_normal l2_policy_evict_normal_ptx
#define l2_policy_evict_first l2_policy_evict_first_ptx
#define ld_hint ld_hint_ptx
#define st_hint st_hint_ptx
#define rcp_nr rcp_nr_ptx
template <class T>
inline T __ldg(const T *p) { return *p; }
struct dim3 {
    unsigned x, y, z;
    dim3(unsigned a = 1, unsigned b = 1, unsigned c = 1) : x(a), y(b), z(c) {}
};
inline unsigned long long atomicAdd(unsigned long long *a, unsigned long long v)
{
    unsigned long long o = *a;
    *a += v;
    return o;
}
#include "prelude.h"
#include "vphys_faces.cuh"
#undef l2_policy_evict_last
#undef l2_policy_evict_normal
#undef l2_policy_evict_first
#undef ld_hint
#undef st_hint
#undef rcp_nr
namespace vphys {
inline unsigned long long l2_policy_evict_last() { return 0; }
inline unsigned long long l2_policy_evict_normal() { return 0; }
inline unsigned long long l2_policy_evict_first() { return 0; }
inline double ld_hint(const double *ptr, unsigned long long) { return *ptr; }
inline void st_hint(double *ptr, double v, unsigned long long) { *ptr = v; }
inline double rcp_nr(double b) { return 1.0 / b; }   // mixed solves only; never reached by the plain kernels
// the dynamic shared memory the kernels declare `extern`: the driver hands
// each thread its own rows instead, so this is never indexed
double smem[1];
}  // namespace vphys
inline void __syncwarp(unsigned = 0xffffffffu) {}
// a host "warp" is one thread: the union of its lanes' live spans is its own
// (the span union only sets which levels a warp walks; each lane's work is
// gated by its own span)
inline int __reduce_min_sync(unsigned, int v) { return v; }
inline int __reduce_max_sync(unsigned, int v) { return v; }
// CUDA's integer min / max
inline int min(int a, int b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
