// Host definitions of the CUDA built-ins that the device header and the
// generated model code use, so that the same text compiles with g++ and the
// generated functions (model_amp, model_adj_*, model_columns, model_kin,
// model_genbod) run on the host.  Test infrastructure: it checks the code
// generator's arithmetic on CPU; nothing in the library uses it.
//
// Only functions that the harness calls are emitted; the warp-shuffle and
// bulk-copy helpers of the device header are never instantiated here, so
// their stand-ins below exist only to let the text parse.
#include <cmath>
#include <cstdint>
#include <math.h>

#define __device__
#define __host__
#define __forceinline__ inline
#define __ldg(p) (*(p))

struct uint4 { unsigned x, y, z, w; };
struct uint2 { unsigned x, y; };
struct double2 { double x, y; };
static inline uint4 make_uint4(unsigned a, unsigned b, unsigned c, unsigned d) { return {a, b, c, d}; }
static inline uint2 make_uint2(unsigned a, unsigned b) { return {a, b}; }
static inline double2 make_double2(double a, double b) { return {a, b}; }
// high 32 bits of the 64-bit product (exact integer arithmetic)
static inline unsigned __umulhi(unsigned a, unsigned b) {
  return (unsigned)(((unsigned long long)a * b) >> 32);
}
template <typename T>
static inline T __shfl_xor_sync(unsigned, T v, int) { return v; }
static inline unsigned long long __cvta_generic_to_shared(const void*) { return 0; }

// one "thread" per event: the per-thread stash has stride 1
#define PWA_TPB 1
