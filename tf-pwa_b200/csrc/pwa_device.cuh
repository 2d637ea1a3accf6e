// Device-side building blocks of the amplitude kernels (hand-written).
//
// This header is prepended, as text, to the model code generated from a
// decay model and compiled at plan-creation time with NVRTC for sm_100a.
// It therefore includes nothing and uses only CUDA built-ins.
//
// Formulas follow the reference package TF-PWA:
//   * Wigner d via sin/cos powers of beta/2 ....... tf_pwa/dfun.py:146-173
//   * conjugated D = e^{i m1 a} d e^{i m2 g} ........ tf_pwa/dfun.py:196-218
//   * q, q^2 ......................................... tf_pwa/amp/core.py:311-334
//   * Blatt-Weisskopf B'(q^2) ........................ tf_pwa/breit_wigner.py:268-277
//   * running-width Breit-Wigner ..................... tf_pwa/breit_wigner.py:74-91,231-245
//   * clip_log ....................................... tf_pwa/model/model.py:283-292
#pragma once

// ---------------------------------------------------------------- complex
template <typename R>
struct cpx {
  R re, im;
};

template <typename R>
__device__ __forceinline__ cpx<R> cmk(R a, R b) {
  cpx<R> z;
  z.re = a;
  z.im = b;
  return z;
}
template <typename R>
__device__ __forceinline__ cpx<R> cadd(cpx<R> a, cpx<R> b) {
  return cmk<R>(a.re + b.re, a.im + b.im);
}
template <typename R>
__device__ __forceinline__ cpx<R> cmul(cpx<R> a, cpx<R> b) {
  return cmk<R>(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
// a * conj(b)
template <typename R>
__device__ __forceinline__ cpx<R> cmulc(cpx<R> a, cpx<R> b) {
  return cmk<R>(a.re * b.re + a.im * b.im, a.im * b.re - a.re * b.im);
}
template <typename R>
__device__ __forceinline__ cpx<R> cscale(cpx<R> a, R s) {
  return cmk<R>(a.re * s, a.im * s);
}
// acc += s * a
template <typename R>
__device__ __forceinline__ void cfma(cpx<R>& acc, R s, cpx<R> a) {
  acc.re = fma(s, a.re, acc.re);
  acc.im = fma(s, a.im, acc.im);
}
// acc += a * b
template <typename R>
__device__ __forceinline__ void cfmac(cpx<R>& acc, cpx<R> a, cpx<R> b) {
  acc.re = fma(a.re, b.re, fma(-a.im, b.im, acc.re));
  acc.im = fma(a.re, b.im, fma(a.im, b.re, acc.im));
}
template <typename R>
__device__ __forceinline__ cpx<R> cconj(cpx<R> a) {
  return cmk<R>(a.re, -a.im);
}
template <typename R>
__device__ __forceinline__ R cabs2(cpx<R> a) {
  return a.re * a.re + a.im * a.im;
}

// ------------------------------------------------------ precision helpers
__device__ __forceinline__ void psincos(double x, double* s, double* c) { sincos(x, s, c); }
__device__ __forceinline__ void psincos(float x, float* s, float* c) { sincosf(x, s, c); }
__device__ __forceinline__ double psqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float psqrt(float x) { return sqrtf(x); }

// e^{i n x/2} for n = -N..N from one sincos of x/2: out[n+N].
template <typename R, int N>
__device__ __forceinline__ void half_angle_powers(R x, cpx<R>* out) {
  R s, c;
  psincos(R(0.5) * x, &s, &c);
  const cpx<R> e1 = cmk<R>(c, s);
  out[N] = cmk<R>(R(1), R(0));
  cpx<R> p = e1;
#pragma unroll
  for (int n = 1; n <= N; ++n) {
    out[N + n] = p;
    out[N - n] = cconj(p);
    p = cmul(p, e1);
  }
}

// sin^l(b/2), cos^l(b/2) for l = 0..N
template <typename R, int N>
__device__ __forceinline__ void half_angle_sc_powers(R b, R* sp, R* cp) {
  R s, c;
  psincos(R(0.5) * b, &s, &c);
  sp[0] = R(1);
  cp[0] = R(1);
#pragma unroll
  for (int l = 1; l <= N; ++l) {
    sp[l] = sp[l - 1] * s;
    cp[l] = cp[l - 1] * c;
  }
}

// The same powers from a given (sin, cos) of the half angle.
template <typename R, int N>
__device__ __forceinline__ void half_angle_powers_sc(R s, R c, cpx<R>* out) {
  const cpx<R> e1 = cmk<R>(c, s);
  out[N] = cmk<R>(R(1), R(0));
  cpx<R> p = e1;
#pragma unroll
  for (int n = 1; n <= N; ++n) {
    out[N + n] = p;
    out[N - n] = cconj(p);
    p = cmul(p, e1);
  }
}
template <typename R, int N>
__device__ __forceinline__ void sc_powers(R s, R c, R* sp, R* cp) {
  sp[0] = R(1);
  cp[0] = R(1);
#pragma unroll
  for (int l = 1; l <= N; ++l) {
    sp[l] = sp[l - 1] * s;
    cp[l] = cp[l - 1] * c;
  }
}

// q^2 of m0 -> m1 m2 (unclamped)
template <typename R>
__device__ __forceinline__ R rel_p2(R m0, R m1, R m2) {
  const R s = m1 + m2, d = m1 - m2;
  const R p = (m0 - s) * (m0 + s) * (m0 - d) * (m0 + d);
  const R t = R(2) * m0;
  return p / (t * t);
}

// |q| of m0 -> m1 m2 with m0 clamped at threshold
template <typename R>
__device__ __forceinline__ R rel_p(R m0, R m1, R m2) {
  const R s = m1 + m2, d = m1 - m2;
  const R me = m0 > s ? m0 : s;
  const R p = (me - s) * (me + s) * (me - d) * (me + d);
  return psqrt(p) / (R(2) * me);
}

// ------------------------------------------------------------ reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Reduce-scatter across a warp by recursive halving.  Every lane holds P
// values (P a multiple of 32); at the step with lane offset O, a lane keeps
// the half of its C live values selected by its lane bit O and adds the
// partner's copy of that half.  After the five steps lane l holds in
// v[0 .. P/32) the warp sums of entries P/32 * l .. P/32 * l + P/32 - 1.
// P - 1 shuffles per lane instead of 5 P for one warp_sum per value.
template <int C, int O, int P>
__device__ __forceinline__ void warp_rs_step(float (&v)[P], int lane) {
  if constexpr (O > 0) {
    const bool up = (lane & O) != 0;
#pragma unroll
    for (int j = 0; j < C / 2; ++j) {
      const float lo = v[j], hi = v[j + C / 2];
      const float keep = up ? hi : lo, send = up ? lo : hi;
      v[j] = keep + __shfl_xor_sync(0xffffffffu, send, O);
    }
    warp_rs_step<C / 2, O / 2, P>(v, lane);
  }
}

template <int P>
__device__ __forceinline__ void warp_reduce_scatter(float (&v)[P], int lane) {
  static_assert(P % 32 == 0, "warp_reduce_scatter: P must be a multiple of 32");
  warp_rs_step<P, 16, P>(v, lane);
}

// clip_log and its derivative in FP64
__device__ __forceinline__ double clip_log(double x, double* dx) {
  const double eps = 1e-6;
  if (x > eps) {
    *dx = 1.0 / x;
    return log(x);
  }
  const double t = (x - eps) / eps;
  *dx = 1.0 / eps - (x - eps) / (eps * eps);
  return -13.815510557964274 + t - 0.5 * t * t;  // log(1e-6) + t - t^2/2
}

// ------------------------------------------------- mbarrier / bulk copies
// Shared-memory barriers with transaction counts and 1-D bulk copies
// (cp.async.bulk, no multicast) for streaming kernels.  Waits are bounded:
// after `limit` polls the caller gets false and must record an error.
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// global -> shared bulk copy completing on `bar`; dst, src 16-byte aligned,
// bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes,
                                         unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity,
                                          unsigned limit) {
  for (unsigned it = 0; it < limit; ++it) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}" : "=r"(ok) : "r"(smem_addr(bar)), "r"(parity) : "memory");
    if (ok) return true;
  }
  return false;
}
