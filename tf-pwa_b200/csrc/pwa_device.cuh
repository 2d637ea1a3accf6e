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
// Products with FP64 constants (couplings, CG and Wigner-d coefficients,
// barrier and lineshape normalisations).  In the FP32 kernels the constant
// is split into FP32 hi + lo parts, so its rounding to FP32 -- the same for
// every event, which would shift the NLL like a parameter change -- leaves
// only per-event rounding of the product.  In FP64 they are plain products.
template <typename R>
__device__ __forceinline__ R mulk(R x, double c) {
  if constexpr (sizeof(R) == 4) {
    const float hi = (float)c;
    return fmaf(x, hi, x * (float)(c - (double)hi));
  } else {
    return x * c;
  }
}
// acc += s * (re + i im)
template <typename R>
__device__ __forceinline__ void cfmak(cpx<R>& acc, R s, double re, double im) {
  if constexpr (sizeof(R) == 4) {
    const float rh = (float)re, ih = (float)im;
    acc.re = fmaf(s, rh, fmaf(s, (float)(re - (double)rh), acc.re));
    acc.im = fmaf(s, ih, fmaf(s, (float)(im - (double)ih), acc.im));
  } else {
    acc.re = fma(s, re, acc.re);
    acc.im = fma(s, im, acc.im);
  }
}
// (re + i im) * z
template <typename R>
__device__ __forceinline__ cpx<R> cmulk(double re, double im, cpx<R> z) {
  if constexpr (sizeof(R) == 4) {
    const float rh = (float)re, ih = (float)im;
    const float rl = (float)(re - (double)rh), il = (float)(im - (double)ih);
    const cpx<float> a = cmul(cmk<float>(rh, ih), z), b = cmul(cmk<float>(rl, il), z);
    return cmk<float>(a.re + b.re, a.im + b.im);
  } else {
    return cmul(cmk<double>(re, im), z);
  }
}

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
// Per-thread asynchronous 8-byte copies global -> shared (cp.async, no
// barrier object: a thread waits for its own copies with cp_async_wait_all,
// which the hardware completes; nothing to time out).
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src)
               : "memory");
}
// 16 bytes through L2 only (streamed data: no L1 allocation)
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src)
               : "memory");
}
// every group of this thread but the most recent one complete
__device__ __forceinline__ void cp_async_wait_prior() {
  asm volatile("cp.async.wait_group 1;" ::: "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_group 0;" ::: "memory");
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
// one arrival (count 1) on `bar`, release semantics at CTA scope
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
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

// ------------------------------------------------ tensor memory / tcgen05
// Fifth-generation tensor-core primitives (sm_100a): tensor-memory
// allocation, MMA issue from shared-memory descriptors, completion through
// an mbarrier, and loads of the accumulator back into registers.
__device__ __forceinline__ void tmem_alloc(unsigned* dst_smem, unsigned ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_addr(dst_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(unsigned taddr, unsigned ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
               : "memory");
}
// Shared-memory matrix descriptor, K-major, no swizzle: core matrices of 8
// rows x 16 bytes stored contiguously; `sbo` = bytes between core matrices
// adjacent in the M/N direction, `lbo` = bytes between the two 16-byte K
// halves of one 32-byte K step; version field 1 (sm_100).
__device__ __forceinline__ unsigned long long umma_desc(const void* p, unsigned lbo, unsigned sbo) {
  const unsigned long long a = (smem_addr(p) >> 4) & 0x3FFFu;
  return a | ((unsigned long long)((lbo >> 4) & 0x3FFFu) << 16) |
         ((unsigned long long)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::i8: signed A and B, S32 accumulator, both
// operands K-major, M (64 or 128) and N (multiple of 16 up to 256).
__host__ __device__ constexpr unsigned umma_idesc_s8(int m, int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((unsigned)(n >> 3) << 17) |
         ((unsigned)(m >> 4) << 24);
}
// D[tmem] (+)= A . B^T with int8 operands from shared memory (one thread).
__device__ __forceinline__ void umma_s8(unsigned d_tmem, unsigned long long a_desc,
                                        unsigned long long b_desc, unsigned idesc, bool accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"((unsigned)accumulate)
      : "memory");
}
// arrive on `bar` once every MMA this thread issued so far has completed
__device__ __forceinline__ void umma_commit(unsigned long long* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// 16 consecutive 32-bit accumulator columns of this thread's lane
__device__ __forceinline__ void tmem_ld16(unsigned taddr, int (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]),
        "=r"(v[14]), "=r"(v[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ------------------------------------------------------------ kinematics
// FP64 four-vector algebra for the dataset step (four-momenta -> masses,
// helicity and alignment angles), restating tf_pwa/angle.py
// (LorentzVector.rest_vector, Vector3.cross_unit / angle_from,
// EulerAngle.angle_zx_z_getx, SU2M) one event per thread.
struct LV {
  double t, x, y, z;
};
struct V3 {
  double x, y, z;
};
struct SU2 {  // [[a, b], [c, d]], complex entries as (re, im)
  double2 a, b, c, d;
};

__device__ __forceinline__ LV lv_add(LV p, LV q) { return {p.t + q.t, p.x + q.x, p.y + q.y, p.z + q.z}; }
__device__ __forceinline__ V3 lv_vec(LV p) { return {p.x, p.y, p.z}; }
__device__ __forceinline__ double v3_dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 v3_cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ V3 v3_unit(V3 a) {
  const double n = sqrt(v3_dot(a, a));
  return {a.x / n, a.y / n, a.z / n};
}
// unit(a x b); for (anti)parallel a, b the reference falls back to a x (b + 1)
__device__ __forceinline__ V3 kin_cross_unit(V3 a, V3 b) {
  V3 c = v3_cross(a, b);
  if (sqrt(v3_dot(c, c)) < 1e-14) c = v3_cross(a, V3{b.x + 1.0, b.y + 1.0, b.z + 1.0});
  return v3_unit(c);
}
__device__ __forceinline__ double kin_angle_from(V3 v, V3 x, V3 y) {
  return atan2(v3_dot(v, y), v3_dot(v, x));
}
// Euler angles (alpha, beta; gamma = 0) from frame (z1, x1) to axis z2, and
// the x axis of the new frame
__device__ __forceinline__ void kin_angle_zx_z_getx(V3 z1, V3 x1, V3 z2, double* alpha,
                                                    double* beta, V3* x2) {
  const V3 u_z1 = v3_unit(z1), u_z2 = v3_unit(z2);
  const V3 u_y1 = kin_cross_unit(z1, x1);
  const V3 u_x1 = kin_cross_unit(u_y1, z1);
  const V3 u_yr = kin_cross_unit(z1, z2);
  const V3 u_xr = kin_cross_unit(u_yr, z1);
  *alpha = kin_angle_from(u_xr, u_x1, u_y1);
  *beta = kin_angle_from(u_z2, u_z1, u_xr);
  *x2 = kin_cross_unit(u_yr, u_z2);
}
// alpha folded into [bias, bias + 2 pi)
__device__ __forceinline__ double kin_fold(double a, double bias) {
  const double tp = 2.0 * 3.141592653589793, x = a - bias;
  return x - tp * floor(x / tp) + bias;
}
// `o` boosted into the rest frame of `p`
__device__ __forceinline__ LV kin_rest_vector(LV p, LV o) {
  const V3 pb = {-p.x / p.t, -p.y / p.t, -p.z / p.t};
  const double beta2 = v3_dot(pb, pb);
  const double gamma = 1.0 / sqrt(1.0 - beta2);
  const double bp = v3_dot(pb, lv_vec(o));
  const double gamma2 = beta2 > 1e-14 ? (gamma - 1.0) / beta2 : 0.0;
  const double s = gamma2 * bp + gamma * o.t;
  return {gamma * (o.t + bp), o.x + s * pb.x, o.y + s * pb.y, o.z + s * pb.z};
}
__device__ __forceinline__ double kin_inv_mass(LV p) {
  return sqrt(fabs(p.t * p.t - (p.x * p.x + p.y * p.y + p.z * p.z)));
}

__device__ __forceinline__ double2 c2mul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 c2add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ SU2 su2_mul(const SU2& p, const SU2& q) {
  return {c2add(c2mul(p.a, q.a), c2mul(p.b, q.c)), c2add(c2mul(p.a, q.b), c2mul(p.b, q.d)),
          c2add(c2mul(p.c, q.a), c2mul(p.d, q.c)), c2add(c2mul(p.c, q.b), c2mul(p.d, q.d))};
}
__device__ __forceinline__ SU2 su2_inv(const SU2& p) {
  return {p.d, make_double2(-p.b.x, -p.b.y), make_double2(-p.c.x, -p.c.y), p.a};
}
// R_y(beta) R_z(alpha)
__device__ __forceinline__ SU2 su2_rot_yz(double beta, double alpha) {
  double s, c, sa, ca;
  sincos(0.5 * beta, &s, &c);
  sincos(0.5 * alpha, &sa, &ca);
  const double2 em = make_double2(ca, -sa), ep = make_double2(ca, sa);
  return {make_double2(c * em.x, c * em.y), make_double2(-s * ep.x, -s * ep.y),
          make_double2(s * em.x, s * em.y), make_double2(c * ep.x, c * ep.y)};
}
// boost along z to the frame where `p` is at rest: diag(e^-w/2, e^w/2)
__device__ __forceinline__ SU2 su2_boost_z_from_p(LV p) {
  const V3 pb = {p.x / p.t, p.y / p.t, p.z / p.t};
  double beta2 = v3_dot(pb, pb);
  beta2 = beta2 < 1.0 ? beta2 : 0.0;
  const double a = exp(0.5 * acosh(1.0 / sqrt(1.0 - beta2)));
  return {make_double2(1.0 / a, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0),
          make_double2(a, 0.0)};
}
__device__ __forceinline__ void su2_euler(const SU2& m, double* alpha, double* beta,
                                          double* gamma) {
  double cb = c2mul(m.a, m.d).x + c2mul(m.b, m.c).x;
  cb = cb < -1.0 ? -1.0 : (cb > 1.0 ? 1.0 : cb);
  *beta = acos(cb);
  const double apg = atan2(m.d.y, m.d.x), amg = -atan2(m.c.y, m.c.x);
  *alpha = apg + amg;
  *gamma = apg - amg;
}

// two-body breakup momentum of a -> b c (0 below threshold)
__device__ __forceinline__ double kin_pdk(double a, double b, double c) {
  const double x = (a - b - c) * (a + b + c) * (a - b + c) * (a + b - c);
  return sqrt(x > 0.0 ? x : 0.0) / (2.0 * a);
}
// boost p by velocity beta
__device__ __forceinline__ LV kin_boost(LV p, V3 beta) {
  const double b2 = v3_dot(beta, beta);
  const double g = 1.0 / sqrt(1.0 - b2);
  const double bp = v3_dot(beta, lv_vec(p));
  const double g2 = b2 > 0.0 ? (g - 1.0) / b2 : 0.0;
  const double s = g2 * bp + g * p.t;
  return {g * (p.t + bp), p.x + s * beta.x, p.y + s * beta.y, p.z + s * beta.z};
}

// ------------------------------------------------------------ random numbers
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11): ten rounds of two
// 32x32->64 multiplies with the published multipliers and Weyl key
// increments.  Counter = (event index, draw number), key = seed, so any
// event can be regenerated from its index alone.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k.x += 0x9E3779B9u;
      k.y += 0xBB67AE85u;
    }
    const unsigned lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    const unsigned lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
  }
  return c;
}
// 53-bit uniform double in [0, 1) from two 32-bit words
__device__ __forceinline__ double u01_53(unsigned a, unsigned b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}
// n uniform doubles of event `i` under `seed` (draw j uses counter word 2 = j/2)
template <int N>
__device__ __forceinline__ void event_uniforms(unsigned long long seed, unsigned long long i,
                                               double (&u)[N]) {
  const uint2 key = make_uint2((unsigned)seed, (unsigned)(seed >> 32));
#pragma unroll
  for (int j = 0; j < (N + 1) / 2; ++j) {
    const uint4 r = philox4x32_10(make_uint4((unsigned)i, (unsigned)(i >> 32), (unsigned)j, 0u), key);
    u[2 * j] = u01_53(r.x, r.y);
    if (2 * j + 1 < N) u[2 * j + 1] = u01_53(r.z, r.w);
  }
}
