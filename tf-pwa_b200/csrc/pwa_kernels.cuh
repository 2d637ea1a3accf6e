// Kernels around the generated ``model_amp`` / ``model_adj`` /
// ``model_columns`` functions and ``model_f`` / ``model_seed`` (sum |A|^2,
// density-matrix weighted for a polarised parent, and the adjoint seed).
//
// Compiled together with the model code by NVRTC (sm_100a).  Events live in
// HBM as structure-of-arrays columns: XM[n_mass][ld] (FP64 invariant
// masses), XA[n_angle][ld] (angles, FP64 or FP32), W[ld] (FP64 weights);
// data events occupy [0, n_data), MC events [n_data, n_all).
//
// pwa_eval_*  one persistent launch over data and MC: blocks
//             [0, blocks_data) walk the data events, the rest the MC events
//             (grid-stride).  Every thread accumulates in FP64
//               data:  sum w clip_log(f),  sum w clip_log'(f) G_k, ... d-shape
//               MC:    sum w f,            sum w G_k,             ... d-shape
//             (the NLL of tf_pwa/model/model.py:407-449 and its gradient
//             pieces), reduces them with warp shuffles and one shared-memory
//             stage, and writes one row of block partials.
// pwa_reduce  sums the block partials in a fixed order (one warp per
//             accumulator), so results are bitwise reproducible.
// pwa_pdf_*   per-event sum |A|^2 (the forward amplitude, AbsPDF.__call__).
// pwa_columns_f64  per-event partial-wave columns F_k for the Gram cache.
// pwa_gram_f64     block partials of M_kl = sum_i w_i sum_o conj(F_ik,o) F_il,o.
#pragma once

#ifndef PWA_TPB
#define PWA_TPB 128
#endif
// polls of an mbarrier before a wait gives up (the kernel then reports an
// error instead of hanging)
#ifndef PWA_WAIT_LIMIT
#define PWA_WAIT_LIMIT (1u << 22)
#endif

template <typename R>
__device__ __forceinline__ void eval_body(const Consts& C, const R* __restrict__ XA,
                                          const double* __restrict__ XM,
                                          const double* __restrict__ W, long long n_data,
                                          long long n_all, long long ld, int blocks_data,
                                          double* __restrict__ partials) {
  const bool is_data = (int)blockIdx.x < blocks_data;
  const long long beg = is_data ? 0 : n_data;
  const long long end = is_data ? n_data : n_all;
  const int nb = is_data ? blocks_data : (int)gridDim.x - blocks_data;
  const int b = is_data ? (int)blockIdx.x : (int)blockIdx.x - blocks_data;
  double acc[PWA_NACC];
#pragma unroll
  for (int j = 0; j < PWA_NACC; ++j) acc[j] = 0.0;
#if PWA_USE_STASH
  // per-thread half-angle sin/cos kept between the forward and adjoint pass
  __shared__ R stash[PWA_NSTASH * PWA_TPB];
  R* st = stash + threadIdx.x;
#endif
  for (long long i = beg + (long long)b * PWA_TPB + threadIdx.x; i < end;
       i += (long long)nb * PWA_TPB) {
    cpx<R> A[PWA_NOUT];
#if PWA_USE_STASH
    model_amp<R, true>(C, XA, XM, ld, i, A, st);
#else
    model_amp<R, false>(C, XA, XM, ld, i, A, nullptr);
#endif
    const double f = model_f<R>(C, A);
    const double w = __ldg(W + i);
    double fac;
    if (is_data) {
      double dl;
      const double cl = clip_log(f, &dl);
      acc[0] = fma(w, cl, acc[0]);
      fac = w * dl;
    } else {
      acc[0] = fma(w, f, acc[0]);
      fac = w;
    }
    cpx<R> Ab[PWA_NOUT];
    model_seed<R>(C, A, fac, Ab, acc + 1 + 2 * PWA_NCOL + PWA_NSHAPE);
#if PWA_USE_STASH
    model_adj_stash<R>(C, XA, XM, ld, i, Ab, acc + 1, acc + 1 + 2 * PWA_NCOL, st);
#else
    model_adj_recompute<R>(C, XA, XM, ld, i, Ab, acc + 1, acc + 1 + 2 * PWA_NCOL);
#endif
  }
  __shared__ double red[PWA_TPB / 32][PWA_NACC];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < PWA_NACC; ++j) {
    const double v = warp_sum(acc[j]);
    if (lane == 0) red[warp][j] = v;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < PWA_NACC; j += PWA_TPB) {
    double s = 0.0;
#pragma unroll
    for (int w2 = 0; w2 < PWA_TPB / 32; ++w2) s += red[w2][j];
    partials[(long long)blockIdx.x * PWA_NACC + j] = s;
  }
}

// Blocks per SM the plain kernels are compiled for (register cap 65536 /
// (128 x MINB)).  Measured on B200 (2.1e6 events): the FP32 form runs
// 7-13 % faster at 4 than at 3 (Lambda_c 424 vs 454 us, four-body 3.94 vs
// 4.52 ms); the FP64 form is faster at 4 for Lambda_c (651 vs 724 us) but
// slower for the four-body model, whose FP64 state already spills at 3
// (6.77 vs 5.95 ms): the model source sets PWA_EVAL_MINB by its size (3
// when it does not).
#ifndef PWA_EVAL_MINB
#define PWA_EVAL_MINB 3
#endif
#ifndef PWA_EVAL_MINB_F32
#define PWA_EVAL_MINB_F32 4
#endif
extern "C" __global__ void __launch_bounds__(PWA_TPB, PWA_EVAL_MINB)
    pwa_eval_f64(const Consts C, const double* __restrict__ XA, const double* __restrict__ XM,
                 const double* __restrict__ W, long long n_data, long long n_all, long long ld,
                 int blocks_data, double* __restrict__ partials) {
  eval_body<double>(C, XA, XM, W, n_data, n_all, ld, blocks_data, partials);
}

extern "C" __global__ void __launch_bounds__(PWA_TPB, PWA_EVAL_MINB_F32)
    pwa_eval_f32(const Consts C, const float* __restrict__ XA, const double* __restrict__ XM,
                 const double* __restrict__ W, long long n_data, long long n_all, long long ld,
                 int blocks_data, double* __restrict__ partials) {
  eval_body<float>(C, XA, XM, W, n_data, n_all, ld, blocks_data, partials);
}

// out[0..nacc) = data sums, out[nacc..2 nacc) = MC sums.  One warp per
// accumulator; each lane strides over the blocks, then a fixed shuffle tree.
// With seq_out set (out in mapped host memory), the call number seq is
// written there last, after a system-scope fence that orders every warp's
// out[] writes (observed through the block barrier) before it.
extern "C" __global__ void pwa_reduce(const double* __restrict__ partials, int nacc,
                                      int blocks_data, int nblocks, double* __restrict__ out,
                                      double* __restrict__ seq_out, double seq) {
  const int lane = threadIdx.x & 31;
  const int warps = blockDim.x >> 5;
  for (int j = (int)(threadIdx.x >> 5); j < 2 * nacc; j += warps) {
    const int which = j / nacc, jj = j % nacc;
    const int b0 = which ? blocks_data : 0, b1 = which ? nblocks : blocks_data;
    double s = 0.0;
    for (int b = b0 + lane; b < b1; b += 32) s += partials[(long long)b * nacc + jj];
    s = warp_sum(s);
    if (lane == 0) out[j] = s;
  }
  if (seq_out) {
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence_system();
      *seq_out = seq;
    }
  }
}

template <typename R>
__device__ __forceinline__ void pdf_body(const Consts& C, const R* __restrict__ XA,
                                         const double* __restrict__ XM, long long beg,
                                         long long end, long long ld, double* __restrict__ out) {
  for (long long i = beg + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < end;
       i += (long long)gridDim.x * blockDim.x) {
    cpx<R> A[PWA_NOUT];
    model_amp<R, false>(C, XA, XM, ld, i, A, nullptr);
    out[i - beg] = model_f<R>(C, A);
  }
}

extern "C" __global__ void __launch_bounds__(PWA_TPB)
    pwa_pdf_f64(const Consts C, const double* __restrict__ XA, const double* __restrict__ XM,
                long long beg, long long end, long long ld, double* __restrict__ out) {
  pdf_body<double>(C, XA, XM, beg, end, ld, out);
}

extern "C" __global__ void __launch_bounds__(PWA_TPB)
    pwa_pdf_f32(const Consts C, const float* __restrict__ XA, const double* __restrict__ XM,
                long long beg, long long end, long long ld, double* __restrict__ out) {
  pdf_body<float>(C, XA, XM, beg, end, ld, out);
}

// Per-event columns F[i][k][o] (complex128 as re,im pairs), event range
// [beg, end) written densely from row 0.
extern "C" __global__ void __launch_bounds__(PWA_TPB)
    pwa_columns_f64(const Consts C, const double* __restrict__ XA,
                    const double* __restrict__ XM, long long beg, long long end, long long ld,
                    double* __restrict__ F) {
  for (long long i = beg + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < end;
       i += (long long)gridDim.x * blockDim.x) {
    cpx<double> Fk[PWA_NCOL * PWA_NOUT];
    model_columns<double>(C, XA, XM, ld, i, Fk);
    double* row = F + (i - beg) * (2LL * PWA_NCOL * PWA_NOUT);
#pragma unroll
    for (int k = 0; k < PWA_NCOL * PWA_NOUT; ++k) {
      row[2 * k] = Fk[k].re;
      row[2 * k + 1] = Fk[k].im;
    }
  }
}

// Block partials of the weighted Gram matrix over rows of F (n rows of
// NCOL*NOUT complex).  Each thread owns (k,l) pairs; events are staged
// through shared memory in tiles of PWA_TPB rows.
extern "C" __global__ void __launch_bounds__(PWA_TPB)
    pwa_gram_f64(const double* __restrict__ F, const double* __restrict__ W, long long n,
                 double* __restrict__ partials) {
  constexpr int NC = PWA_NCOL, NO = PWA_NOUT, ROW = 2 * NC * NO;
  constexpr int TILE = (PWA_TPB * 8 + ROW - 1) / ROW > 0 ? (PWA_TPB * 8 + ROW - 1) / ROW : 1;
  __shared__ double tile[TILE * ROW];
  __shared__ double wt[TILE];
  double accr[(NC * NC + PWA_TPB - 1) / PWA_TPB];
  double acci[(NC * NC + PWA_TPB - 1) / PWA_TPB];
  constexpr int PER = (NC * NC + PWA_TPB - 1) / PWA_TPB;
#pragma unroll
  for (int p = 0; p < PER; ++p) accr[p] = acci[p] = 0.0;
  for (long long t0 = (long long)blockIdx.x * TILE; t0 < n; t0 += (long long)gridDim.x * TILE) {
    const int rows = (int)((n - t0) < TILE ? (n - t0) : TILE);
    __syncthreads();
    for (int j = threadIdx.x; j < rows * ROW; j += PWA_TPB) tile[j] = F[t0 * ROW + j];
    for (int j = threadIdx.x; j < rows; j += PWA_TPB) wt[j] = W[t0 + j];
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int kl = threadIdx.x + p * PWA_TPB;
      if (kl < NC * NC) {
        const int k = kl / NC, l = kl % NC;
        double sr = 0.0, si = 0.0;
        for (int r = 0; r < rows; ++r) {
          double tr = 0.0, ti = 0.0;
#pragma unroll
          for (int o = 0; o < NO; ++o) {
            const double ar = tile[r * ROW + 2 * (k * NO + o)], ai = tile[r * ROW + 2 * (k * NO + o) + 1];
            const double br = tile[r * ROW + 2 * (l * NO + o)], bi = tile[r * ROW + 2 * (l * NO + o) + 1];
            // conj(a) * b
            tr += ar * br + ai * bi;
            ti += ar * bi - ai * br;
          }
          sr = fma(wt[r], tr, sr);
          si = fma(wt[r], ti, si);
        }
        accr[p] += sr;
        acci[p] += si;
      }
    }
  }
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int kl = threadIdx.x + p * PWA_TPB;
    if (kl < NC * NC) {
      partials[(long long)blockIdx.x * 2 * NC * NC + 2 * kl] = accr[p];
      partials[(long long)blockIdx.x * 2 * NC * NC + 2 * kl + 1] = acci[p];
    }
  }
}

// Column-wise deterministic sum of nrows rows of width ncols.
extern "C" __global__ void pwa_sum_rows(const double* __restrict__ in, int nrows, int ncols,
                                        double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const int warps = blockDim.x >> 5;
  for (int j = (int)(blockIdx.x * warps + (threadIdx.x >> 5)); j < ncols; j += gridDim.x * warps) {
    double s = 0.0;
    for (int r = lane; r < nrows; r += 32) s += in[(long long)r * ncols + j];
    s = warp_sum(s);
    if (lane == 0) out[j] = s;
  }
}

// ---------------------------------------------------------------------------
// Gram matrix on the tensor cores, exact-integer sliced products (the Ozaki
// scheme: Ozaki, Ogita, Oishi, Rump, Numer. Algorithms 59 (2012); integer
// tensor cores as in Ootomo, Ozaki, Yokota, IJHPCA 38 (2024)).
//
// Rows r = (event i, helicity o) of X[r][c] = Re F_ic,o (c < NCOL) or
// Im F_i(c-NCOL),o and of Y = w_i X; G = X^T Y (KC x KC real, KC = 2 NCOL)
// holds Re M = G_RR + G_II and Im M = G_RI - G_IR.  Column c of X is scaled
// by 2^-eA_c (max |X_c| < 2^eA_c * 127/128) and split into PWA_OZ_S int8
// slices a_s (weights 2^-7s, |a_1| <= 127, |a_s| <= 64 after): x =
// 2^eA (sum_s a_s 2^-7s) + O(2^(eA-7S-1)), every step exact in FP64.  The
// products a_s b_t with s + t = g <= S + 1 accumulate exactly in int32 in
// the tensor memory (one accumulator per g, KC x CP columns, rows >= KC of
// the M = 128 tile zero), flushed to FP64 registers every PWA_OZ_FLUSH
// rows (int32 cannot overflow: rows x sum |a_s b_t| < 2^31), and
// G_cd = 2^(eA_c + eB_d) sum_g D_g 2^-7g.  Truncation error ~2^-49 of the
// column maxima per product: FP64-level.
#define PWA_OZ_S 7
#define PWA_OZ_KC (2 * PWA_NCOL)
#define PWA_OZ_CP ((PWA_OZ_KC + 15) / 16 * 16)
#define PWA_OZ_KB 64                       // rows per shared-memory stage
#define PWA_OZ_FLUSH 16384                 // rows between accumulator flushes
#define PWA_OZ_ABYTES (128 * PWA_OZ_KB)    // one A slice: M = 128 rows x KB
#define PWA_OZ_BBYTES (PWA_OZ_CP * PWA_OZ_KB)
#define PWA_OZ_STAGE (PWA_OZ_S * (PWA_OZ_ABYTES + PWA_OZ_BBYTES))
#define PWA_OZ_TCOLS (PWA_OZ_S * PWA_OZ_CP <= 32 ? 32 : PWA_OZ_S * PWA_OZ_CP <= 64 ? 64 \
                      : PWA_OZ_S * PWA_OZ_CP <= 128 ? 128 : PWA_OZ_S * PWA_OZ_CP <= 256 ? 256 : 512)
#define PWA_OZ_OK (PWA_OZ_KC <= 64)

// Column maxima of |X| and |w X| over n events of F (rows of NCOL*NOUT
// complex): mx[c] and mx[KC + c] as FP64 bit patterns (non-negative
// doubles order like their bits), combined with atomicMax.
extern "C" __global__ void __launch_bounds__(PWA_TPB)
    pwa_gram_colmax(const double* __restrict__ F, const double* __restrict__ W, long long n,
                    unsigned long long* __restrict__ mx) {
  constexpr int KC = PWA_OZ_KC, NO = PWA_NOUT;
  for (int c = 0; c < KC; ++c) {
    double ma = 0.0, mb = 0.0;
    const int k = c % PWA_NCOL, im = c / PWA_NCOL;
    for (long long i = (long long)blockIdx.x * PWA_TPB + threadIdx.x; i < n;
         i += (long long)gridDim.x * PWA_TPB) {
      const double w = fabs(W[i]);
#pragma unroll
      for (int o = 0; o < NO; ++o) {
        const double x = fabs(F[i * (2LL * PWA_NCOL * NO) + 2 * (k * NO + o) + im]);
        ma = fmax(ma, x);
        mb = fmax(mb, w * x);
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      ma = fmax(ma, __shfl_xor_sync(0xffffffffu, ma, off));
      mb = fmax(mb, __shfl_xor_sync(0xffffffffu, mb, off));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMax(mx + c, (unsigned long long)__double_as_longlong(ma));
      atomicMax(mx + KC + c, (unsigned long long)__double_as_longlong(mb));
    }
  }
}

// exponent e with max < 2^e * 127/128 (0 for an all-zero column)
__device__ __forceinline__ int oz_exponent(double mx) {
  if (!(mx > 0.0)) return 0;
  int e;
  const double m = frexp(mx, &e);  // mx = m 2^e, m in [0.5, 1)
  return m * 128.0 <= 127.0 ? e : e + 1;
}

// int8 slices of 16 consecutive rows of one column, x 2^-e: word[s][q]
// byte j = slice s of value 4 q + j (16 bytes per slice: one core-matrix
// row of a K-major operand)
__device__ __forceinline__ void oz_slices16(const double (&x)[16], int e,
                                            unsigned (&word)[PWA_OZ_S][4]) {
#pragma unroll
  for (int s = 0; s < PWA_OZ_S; ++s)
#pragma unroll
    for (int q = 0; q < 4; ++q) word[s][q] = 0u;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    double v = ldexp(x[j], 7 - e);  // first slice's scale: |v| < 127
#pragma unroll
    for (int s = 0; s < PWA_OZ_S; ++s) {
      const double a = rint(v);
      word[s][j >> 2] |= ((unsigned)(int)a & 0xFFu) << (8 * (j & 3));
      v = (v - a) * 128.0;  // exact: the fraction of v, then 7 more bits
    }
  }
}

// One block of PWA_OZ_THREADS threads per SM; dynamic shared memory: two
// stages of PWA_OZ_STAGE bytes (1024-aligned) and the FP64 accumulators.
// Block b takes a contiguous run of the rows; it writes partial[b][c][d]
// (KC x KC FP64) for an ordered sum.  e8[2 KC]: column maxima
// (pwa_gram_colmax) as FP64 bits.  err[0] is set when a wait on the tensor
// cores gives up.  The stage fill gives each thread 16 rows of one column
// (FP64 loads, exact slicing, one 16-byte store per slice); thread 0 issues
// the MMAs of a filled stage while the others fill the next one.
#define PWA_OZ_THREADS 512
#define PWA_OZ_ACCLD (PWA_OZ_CP + 1)  // padded row of the shared accumulators
extern "C" __global__ void __launch_bounds__(PWA_OZ_THREADS, 1)
    pwa_gram_tc(const double* __restrict__ F, const double* __restrict__ W, long long n,
                const unsigned long long* __restrict__ e8, double* __restrict__ partial,
                unsigned int* __restrict__ err) {
#if PWA_OZ_OK
  constexpr int KC = PWA_OZ_KC, CP = PWA_OZ_CP, S = PWA_OZ_S, KB = PWA_OZ_KB;
  constexpr int NO = PWA_NOUT, NK16 = KB / 16;  // 16-row groups per stage
  constexpr int NT = PWA_OZ_THREADS;
  constexpr unsigned IDESC = umma_idesc_s8(128, CP);
  extern __shared__ __align__(1024) unsigned char oz_smem[];
  __shared__ __align__(8) unsigned long long done[2];
  __shared__ unsigned s_tmem;
  __shared__ int s_e[2 * KC];
  __shared__ int s_err;
  const int tid = threadIdx.x, warp = tid >> 5;
  unsigned char* base = (unsigned char*)(((size_t)oz_smem + 1023) & ~(size_t)1023);
  double* s_acc = (double*)(base + 2 * PWA_OZ_STAGE);  // [KC][PWA_OZ_ACCLD]
  // zero both stages (A rows >= KC stay zero), accumulators, exponents,
  // barriers, TMEM
  for (int j = tid; j < 2 * PWA_OZ_STAGE / 4; j += NT) ((unsigned*)base)[j] = 0u;
  for (int j = tid; j < KC * PWA_OZ_ACCLD; j += NT) s_acc[j] = 0.0;
  for (int c = tid; c < 2 * KC; c += NT) s_e[c] = oz_exponent(__longlong_as_double((long long)e8[c]));
  if (tid == 0) {
    s_err = 0;
    mbar_init(&done[0], 1);
    mbar_init(&done[1], 1);
    mbar_fence_init();
  }
  __syncwarp();
  if (warp == 0) tmem_alloc(&s_tmem, PWA_OZ_TCOLS);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = s_tmem;
  const long long R = n * NO;
  const long long r0 = (long long)blockIdx.x * R / gridDim.x;
  const long long r1 = (long long)(blockIdx.x + 1) * R / gridDim.x;
  int uses[2] = {0, 0};
  bool fresh = true;  // next MMA of each accumulator starts it from zero
  int stage = 0;
  long long since_flush = 0;
  for (long long rb = r0; rb < r1 || since_flush > 0; rb += KB) {
    const bool have = rb < r1;
    const bool flush = !have || since_flush + KB > PWA_OZ_FLUSH;
    if (flush && since_flush > 0) {
      // wait for every MMA issued so far, then add the accumulators to FP64
      for (int st = 0; st < 2; ++st)
        if (uses[st] && !mbar_wait(&done[st], (unsigned)((uses[st] - 1) & 1), PWA_WAIT_LIMIT))
          s_err = 1;
      tc_fence_after();
      __syncwarp();  // tcgen05.ld is warp-collective: reconverge first
      if (warp < 2) {  // TMEM lanes 0..63 = rows c of the accumulators
        const int c = tid;
#pragma unroll 1
        for (int g = 0; g < S; ++g) {
          const double sc = ldexp(1.0, -7 * (g + 2));
#pragma unroll
          for (int q = 0; q < CP / 16; ++q) {
            int v[16];
            tmem_ld16(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)(g * CP + 16 * q), v);
            tmem_wait_ld();
            if (c < KC) {
#pragma unroll
              for (int j = 0; j < 16; ++j) {
                double* a = s_acc + c * PWA_OZ_ACCLD + 16 * q + j;
                *a = fma((double)v[j], sc, *a);
              }
            }
          }
        }
      }
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
      fresh = true;
      since_flush = 0;
      if (!have) break;
    }
    if (s_err) break;
    // refill `stage`: its previous MMAs must be complete
    if (uses[stage] && !mbar_wait(&done[stage], (unsigned)((uses[stage] - 1) & 1), PWA_WAIT_LIMIT))
      s_err = 1;
    unsigned char* A = base + (size_t)stage * PWA_OZ_STAGE;
    unsigned char* B = A + (size_t)S * PWA_OZ_ABYTES;
    for (int item = tid; item < 2 * KC * NK16; item += NT) {
      const bool isb = item >= KC * NK16;
      const int it = isb ? item - KC * NK16 : item;
      const int c = it % KC, k16 = it / KC;
      const int k = c % PWA_NCOL, im = c / PWA_NCOL;
      double x[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        const long long r = rb + 16 * k16 + j;
        x[j] = 0.0;
        if (r < r1) {
          const long long i = r / NO;
          const int o = (int)(r - i * NO);
          x[j] = __ldg(F + i * (2LL * PWA_NCOL * NO) + 2 * (k * NO + o) + im);
          if (isb) x[j] *= __ldg(W + i);
        }
      }
      unsigned word[S][4];
      oz_slices16(x, s_e[(isb ? KC : 0) + c], word);
      // K-major core-matrix layout: byte (row m, k) = (k/16)*(M/8*128) +
      // (m/8)*128 + (m%8)*16 + k%16 with M = 128 (A) or CP (B)
      const int mrows = isb ? CP : 128;
      const int off = k16 * (mrows / 8 * 128) + (c / 8) * 128 + (c % 8) * 16;
      unsigned char* dst = isb ? B : A;
      const int sbytes = isb ? PWA_OZ_BBYTES : PWA_OZ_ABYTES;
#pragma unroll
      for (int s = 0; s < S; ++s)
        *(uint4*)(dst + s * sbytes + off) = make_uint4(word[s][0], word[s][1], word[s][2], word[s][3]);
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll 1
      for (int q = 0; q < KB / 32; ++q) {
#pragma unroll 1
        for (int g = 2; g <= S + 1; ++g) {
          bool first = fresh && q == 0;
          for (int s = g - S > 1 ? g - S : 1; s <= S && s < g; ++s) {
            const int t = g - s;
            const unsigned long long ad =
                umma_desc(A + (size_t)(s - 1) * PWA_OZ_ABYTES + 2 * q * (128 / 8 * 128),
                          128 / 8 * 128, 128);
            const unsigned long long bd =
                umma_desc(B + (size_t)(t - 1) * PWA_OZ_BBYTES + 2 * q * (CP / 8 * 128), CP / 8 * 128,
                          128);
            umma_s8(tmem + (unsigned)((g - 2) * CP), ad, bd, IDESC, !first);
            first = false;
          }
        }
      }
      umma_commit(&done[stage]);
    }
    __syncwarp();
    // no barrier here: the other threads go on to fill the other stage
    // while thread 0 issues; a stage is refilled only after its commit
    uses[stage]++;
    fresh = false;
    since_flush += KB;
    stage ^= 1;
  }
  if (s_err && tid == 0) atomicOr(err, 1u);
  // wait (bounded) for any MMA still running before the tensor memory goes
  for (int st = 0; st < 2; ++st)
    if (uses[st]) mbar_wait(&done[st], (unsigned)((uses[st] - 1) & 1), PWA_WAIT_LIMIT);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  __syncwarp();
  if (warp == 0) tmem_dealloc(tmem, PWA_OZ_TCOLS);
  for (int j = tid; j < KC * KC; j += NT) {
    const int c = j / KC, d = j % KC;
    partial[(long long)blockIdx.x * KC * KC + j] =
        ldexp(s_acc[c * PWA_OZ_ACCLD + d], s_e[c] + s_e[KC + d]);
  }
#endif
}

// Peak FMA throughput of the CUDA cores, the roofline of the compute-bound
// amplitude kernels: every thread runs eight independent chains of `iters`
// fused multiply-adds (FP64 or FP32) and stores their sum, so nothing is
// eliminated.  Work: 2 * 8 * iters flops per thread.
template <typename R>
__device__ __forceinline__ void fma_chains(long long iters, R* __restrict__ out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  R a[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) a[j] = R(1) + R(t % 7) * R(0.001) + R(j) * R(0.01);
  const R b = R(0.9999999), c = R(1e-7);
#pragma unroll 1
  for (long long i = 0; i < iters; i += 4) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
#pragma unroll
      for (int j = 0; j < 8; ++j) a[j] = fma(a[j], b, c);
    }
  }
  R s = R(0);
#pragma unroll
  for (int j = 0; j < 8; ++j) s += a[j];
  out[t] = s;
}
extern "C" __global__ void pwa_fma_peak_f64(long long iters, double* __restrict__ out) {
  fma_chains<double>(iters, out);
}
extern "C" __global__ void pwa_fma_peak_f32(long long iters, float* __restrict__ out) {
  fma_chains<float>(iters, out);
}

// FP64 -> FP32 copy of the angle columns for the mixed-precision kernels.
extern "C" __global__ void pwa_to_f32(const double* __restrict__ in, float* __restrict__ out,
                                      long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

// ---------------------------------------------------------------------------
// Cached partial-wave columns (masses and widths fixed).
//
// Layout (tile-major, PWA_TPB events per tile, zero-padded last tile):
//   Fc[(t * PWA_NF + j) * PWA_TPB + e]  float2 (re, im) of pair j of event
//                                       t*PWA_TPB + e, j over the structurally
//                                       non-zero (column k, helicity o) pairs;
//   Wc[t * PWA_TPB + e]                 FP64 weight (0 for padding).
// A tile is one contiguous block, so one bulk copy moves it to shared memory.
// Values are computed in FP64 and rounded to FP32 once per stored value
// (unbiased per-event rounding, no systematic bias in sums over events).
extern "C" __global__ void __launch_bounds__(PWA_TPB)
    pwa_cache_f32(const Consts C, const double* __restrict__ XA, const double* __restrict__ XM,
                  const double* __restrict__ W, long long n, long long ntiles, long long ld,
                  float2* __restrict__ Fc, double* __restrict__ Wc) {
  const long long total = ntiles * PWA_TPB;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long t = i / PWA_TPB, e = i % PWA_TPB;
    if (i < n) {
      cpx<double> F[PWA_NCOL * PWA_NOUT];
      model_columns<double>(C, XA, XM, ld, i, F);
#pragma unroll
      for (int j = 0; j < PWA_NF; ++j) {
        const cpx<double> v = F[pwa_fk[j] * PWA_NOUT + pwa_fo[j]];
        Fc[(t * PWA_NF + j) * PWA_TPB + e] = make_float2((float)v.re, (float)v.im);
      }
      Wc[i] = W[i];
    } else {
#pragma unroll
      for (int j = 0; j < PWA_NF; ++j) Fc[(t * PWA_NF + j) * PWA_TPB + e] = make_float2(0.f, 0.f);
      Wc[i] = 0.0;
    }
  }
}

// ---------------------------------------------------------------------------
// Floating-shape column cache.  With one pass (no identical-particle swaps),
// no polarised parent and no CP-violating totals (PWA_SHAPE_CACHE_OK), a
// column factorises as
//   F_k,o(event) = r_k BW_ch(k)(m; shapes) Fhat_k,o(event):
// Fhat is the column without its chain's lineshapes (model_columns_ns, in
// FP64 at the shape setting of the cache, stored FP32 in the tile layout of
// the cached kernels, for data and MC events), BW the product of the
// chain's lineshapes from the event's masses (model_shapes, FP64), and r_k
// the ratio of the column's barrier normalisations (sqrt(Pz0_l) norm_l per
// vertex) now and at the cache's setting (host).  An evaluation reads the
// columns and the masses and produces the sums of pwa_eval_f64 -- S0, the
// column sums and the lineshape sums (tf_pwa/model/model.py:407-449 with
// the derivatives of the lineshapes, tf_pwa/breit_wigner.py:56-91) -- so
// the host's chain rule is the plain form's.
extern "C" __global__ void __launch_bounds__(PWA_TPB)
    pwa_cache_ns_f32(const Consts C, const double* __restrict__ XA, const double* __restrict__ XM,
                     long long n, long long ntiles, long long ld, float2* __restrict__ Fc) {
  const long long total = ntiles * PWA_TPB;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long t = i / PWA_TPB, e = i % PWA_TPB;
    if (i < n) {
      cpx<double> F[PWA_NCOL * PWA_NOUT];
      model_columns_ns<double>(C, XA, XM, ld, i, F);
#pragma unroll
      for (int j = 0; j < PWA_NF; ++j) {
        const cpx<double> v = F[pwa_fk[j] * PWA_NOUT + pwa_fo[j]];
        Fc[(t * PWA_NF + j) * PWA_TPB + e] = make_float2((float)v.re, (float)v.im);
      }
    } else {
#pragma unroll
      for (int j = 0; j < PWA_NF; ++j) Fc[(t * PWA_NF + j) * PWA_TPB + e] = make_float2(0.f, 0.f);
    }
  }
}

struct CRatio {
  double v[PWA_NCOL];  // r_k: barrier normalisations now / at the cache's setting
};

#ifndef PWA_SC_MINB
#define PWA_SC_MINB 2
#endif
// PWA_SC_STAGES 2 (set by the model source where the buffers fit): each warp
// copies its next 32 events' cached pairs, masses and weights into shared
// memory (16-byte cp.async, through L2) while it computes the current ones,
// so the loads in flight do not depend on how many warps the registers
// allow; 0: direct loads.
#ifndef PWA_SC_STAGES
#define PWA_SC_STAGES 0
#endif
#define PWA_SC_NM (PWA_NFIELD_MASS > 0 ? PWA_NFIELD_MASS : 1)
// doubles (a float2 pair is one) of one stage: pairs, masses, weights
#define PWA_SC_STAGE ((PWA_NF + PWA_SC_NM + 1) * PWA_TPB)

// Copies of the 32 events from s (a multiple of 32, s < n_all) into stage
// buffer d: lane l moves 16 bytes (two events) of rows l / 16, l / 16 + 2, ...
__device__ __forceinline__ void sc_issue(double* __restrict__ d, const float2* __restrict__ Fc,
                                         const double* __restrict__ XM,
                                         const double* __restrict__ W, long long ld, long long s,
                                         int warp, int lane) {
  const long long t = s / PWA_TPB, e0 = s % PWA_TPB;
  const int half = lane >> 4, c2 = 2 * (lane & 15), col = 32 * warp + c2;
#pragma unroll
  for (int j = half; j < PWA_NF; j += 2)
    cp_async16(d + j * PWA_TPB + col, Fc + (t * PWA_NF + j) * PWA_TPB + e0 + c2);
#pragma unroll
  for (int m = half; m < PWA_NFIELD_MASS; m += 2)
    cp_async16(d + (PWA_NF + m) * PWA_TPB + col, XM + (long long)m * ld + s + c2);
  if (half == 0) cp_async16(d + (PWA_NF + PWA_SC_NM) * PWA_TPB + col, W + s + c2);
}

// Ends with the ordered two-level reduction of pwa_eval_cached (grouped_sum,
// declared below): block rows of 2 * PWA_NACC (a data block's sums in the
// first half, an MC block's in the second); the last block writes the data
// and MC sums to out[0 .. 2 PWA_NACC), the error flag and the call number
// seq (publish_result); out may be mapped host memory.
__device__ __forceinline__ bool grouped_sum(double* __restrict__ partials,
                                            unsigned int* __restrict__ ticket, int na,
                                            double* __restrict__ out, int* s_flag);
__device__ __forceinline__ void publish_result(unsigned int* __restrict__ ticket, int na,
                                               double* __restrict__ out, double seq);

extern "C" __global__ void __launch_bounds__(PWA_TPB, PWA_SC_MINB)
    pwa_eval_shapecache(const Consts C, const CRatio rk, const float2* __restrict__ Fc,
                        const double* __restrict__ XM, const double* __restrict__ W,
                        long long n_data, long long n_all, long long ld, int blocks_data,
                        double* __restrict__ partials, int smem_bytes,
                        unsigned int* __restrict__ ticket, double* __restrict__ out, double seq) {
  constexpr int K = PWA_NCOL, NS = PWA_NSRES > 0 ? PWA_NSRES : 1;
  const bool is_data = (int)blockIdx.x < blocks_data;
  const long long beg = is_data ? 0 : n_data;
  const long long end = is_data ? n_data : n_all;
  const int nb = is_data ? blocks_data : (int)gridDim.x - blocks_data;
  const int b = is_data ? (int)blockIdx.x : (int)blockIdx.x - blocks_data;
  double acc[PWA_NACC];
#pragma unroll
  for (int j = 0; j < PWA_NACC; ++j) acc[j] = 0.0;
#if PWA_SC_STAGES > 0
  extern __shared__ __align__(16) double sc_smem[];
  // launched without the staging buffers: no event is read, the sums are NaN
  const bool staged = smem_bytes >= 2 * PWA_SC_STAGE * (int)sizeof(double);
  if (!staged) acc[0] = __longlong_as_double(0x7ff8000000000000LL);
  const int lane_s = threadIdx.x & 31, warp_s = threadIdx.x >> 5;
  const long long stride = (long long)nb * PWA_TPB;
  // segments of 32 events from a multiple of 32 at or below beg (events
  // outside [beg, end) are computed but not summed)
  long long s = staged ? (beg & ~31LL) + (long long)b * PWA_TPB + 32 * warp_s : end;
  if (s < end) sc_issue(sc_smem, Fc, XM, W, ld, s, warp_s, lane_s);
  cp_async_commit();
  for (int it = 0; s < end; s += stride, ++it) {
    double* cur = sc_smem + (it & 1) * PWA_SC_STAGE;
    double* nxt = sc_smem + ((it & 1) ^ 1) * PWA_SC_STAGE;
    __syncwarp();  // every lane has read the other stage (last segment)
    if (s + stride < end) sc_issue(nxt, Fc, XM, W, ld, s + stride, warp_s, lane_s);
    cp_async_commit();
    cp_async_wait_prior();  // this lane's copies of the current segment landed
    __syncwarp();           // ... and every lane's
    const long long i = s + lane_s;
    const bool valid = i >= beg && i < end;
    const int col = 32 * warp_s + lane_s;
    // the pairs are read from shared memory where used (both passes), not
    // held in registers
    const float2* vs = reinterpret_cast<const float2*>(cur) + col;
#define PWA_SC_V(j) vs[(j) * PWA_TPB]
    cpx<double> BW[PWA_NCHAIN], DM[NS], DG[NS];
    model_shapes<double, false>(C, cur + PWA_NF * PWA_TPB, PWA_TPB, col, BW, DM, DG);
    const double w = valid ? cur[(PWA_NF + PWA_SC_NM) * PWA_TPB + col] : 0.0;
#else
  (void)smem_bytes;
  for (long long i = beg + (long long)b * PWA_TPB + threadIdx.x; i < end;
       i += (long long)nb * PWA_TPB) {
    const long long t = i / PWA_TPB, e = i % PWA_TPB;
    constexpr bool valid = true;
    float2 v[PWA_NF];
#pragma unroll
    for (int j = 0; j < PWA_NF; ++j) v[j] = __ldcs(Fc + (t * PWA_NF + j) * PWA_TPB + e);
#define PWA_SC_V(j) v[j]
    cpx<double> BW[PWA_NCHAIN], DM[NS], DG[NS];
    model_shapes<double>(C, XM, ld, i, BW, DM, DG);
    const double w = __ldg(W + i);
#endif
    // F = s_k Fhat with s_k = r_k BW_ch(k); A_o = sum_k c_k s_k Fhat_k,o
    double ar[PWA_NOUT], ai[PWA_NOUT];
#pragma unroll
    for (int o = 0; o < PWA_NOUT; ++o) ar[o] = ai[o] = 0.0;
#pragma unroll
    for (int j = 0; j < PWA_NF; ++j) {
      const int k = pwa_fk[j], o = pwa_fo[j];
      const cpx<double> bw = BW[pwa_col_chain[k]];
      const cpx<double> cs = cmul(cmk<double>(C.v[2 * k], C.v[2 * k + 1]),
                                  cmk<double>(rk.v[k] * bw.re, rk.v[k] * bw.im));
      const float2 vj = PWA_SC_V(j);
      const double x = (double)vj.x, y = (double)vj.y;
      ar[o] = fma(cs.re, x, fma(-cs.im, y, ar[o]));
      ai[o] = fma(cs.re, y, fma(cs.im, x, ai[o]));
    }
    double f = 0.0;
#pragma unroll
    for (int o = 0; o < PWA_NOUT; ++o) f = fma(ar[o], ar[o], fma(ai[o], ai[o], f));
    double fac;
    if (is_data) {
      double dl;
      const double cl = clip_log(f, &dl);
      acc[0] = valid ? fma(w, cl, acc[0]) : acc[0];
      fac = w * dl;
    } else {
      acc[0] = valid ? fma(w, f, acc[0]) : acc[0];
      fac = w;
    }
    // g_k = fac s_k sum_o conj(A_o) Fhat_k,o (the pairs j run column by
    // column);  SR_s = sum over the columns of the chains holding shape s of
    // c_k g_k
    cpx<double> SR[NS];
#pragma unroll
    for (int q = 0; q < NS; ++q) SR[q] = cmk<double>(0.0, 0.0);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      cpx<double> hk = cmk<double>(0.0, 0.0);
#pragma unroll
      for (int j = 0; j < PWA_NF; ++j) {
        if (pwa_fk[j] != k) continue;
        const int o = pwa_fo[j];
        const float2 vj = PWA_SC_V(j);
        const double x = (double)vj.x, y = (double)vj.y;
        hk.re = fma(ar[o], x, fma(ai[o], y, hk.re));
        hk.im = fma(ar[o], y, fma(-ai[o], x, hk.im));
      }
      const cpx<double> bw = BW[pwa_col_chain[k]];
      cpx<double> g = cscale(cmul(cmk<double>(rk.v[k] * bw.re, rk.v[k] * bw.im), hk), fac);
      g.re = valid ? g.re : 0.0;  // events outside the set (garbage inputs: select, not scale)
      g.im = valid ? g.im : 0.0;
      acc[1 + 2 * k] += g.re;
      acc[2 + 2 * k] += g.im;
      const cpx<double> cg = cmul(cmk<double>(C.v[2 * k], C.v[2 * k + 1]), g);
#pragma unroll
      for (int q = 0; q < PWA_NSRES; ++q)
        if (pwa_sres_chain[q][pwa_col_chain[k]]) {
          SR[q].re += cg.re;
          SR[q].im += cg.im;
        }
    }
#pragma unroll
    for (int q = 0; q < PWA_NSRES; ++q) {
      const double dm = 2.0 * cmul(SR[q], DM[q]).re, dg = 2.0 * cmul(SR[q], DG[q]).re;
      acc[1 + 2 * K + 2 * q] += valid ? dm : 0.0;
      acc[2 + 2 * K + 2 * q] += valid ? dg : 0.0;
    }
  }
#if PWA_SC_STAGES > 0
  cp_async_wait_all();  // (nothing is in flight here: the last group is empty)
#endif
#undef PWA_SC_V
  __shared__ double red[PWA_TPB / 32][PWA_NACC];
  __shared__ int s_last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < PWA_NACC; ++j) {
    const double vv = warp_sum(acc[j]);
    if (lane == 0) red[warp][j] = vv;
  }
  __syncthreads();
  constexpr int NA2 = 2 * PWA_NACC;
  for (int j = threadIdx.x; j < NA2; j += PWA_TPB) {
    const int jj = j - (is_data ? 0 : PWA_NACC);
    double sacc = 0.0;
    if (jj >= 0 && jj < PWA_NACC) {
#pragma unroll
      for (int w2 = 0; w2 < PWA_TPB / 32; ++w2) sacc += red[w2][jj];
    }
    partials[(long long)blockIdx.x * NA2 + j] = sacc;
  }
  __threadfence();
  __syncthreads();
  if (!grouped_sum(partials, ticket, NA2, out, &s_last)) return;
  publish_result(ticket, NA2, out, seq);
}

struct CCoup {
  double v[2 * PWA_NCOL];  // column couplings c_k, (re, im) pairs
};

// Couplings from the parameter block to shared memory with constant
// indices only (an index that depends on the thread would make the
// compiler copy the whole parameter block to local memory).
__device__ __forceinline__ void stage_couplings(const CCoup& c, double* s_c) {
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < 2 * PWA_NCOL; ++j) s_c[j] = c.v[j];
  }
}

#ifndef PWA_STAGES
#define PWA_STAGES 3
#endif
#define PWA_CACHE_NA (1 + 2 * PWA_NCOL)
// Blocks per group of the two-level partial reduction, and the most groups
// a launch may have (the ticket buffer holds 2 + PWA_MAX_GROUPS counters).
#define PWA_GROUP 16
#define PWA_MAX_GROUPS 4096

// Sum of the block partials (rows of `na` doubles, one per block) by the
// last block to finish: thread j owns accumulators j, j + PWA_TPB, ...,
// reads the rows in order (a warp reads consecutive accumulators of a row:
// coalesced) with four interleaved partial sums, so many loads are in
// flight.  The order depends only on the row count: reproducible.
__device__ __forceinline__ void last_block_sum(const double* __restrict__ partials, int nrows,
                                               int na, double* __restrict__ out) {
  for (int j = threadIdx.x; j < na; j += PWA_TPB) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int b = 0;
#pragma unroll 4
    for (; b + 4 <= nrows; b += 4) {
      s0 += __ldcg(partials + (long long)b * na + j);
      s1 += __ldcg(partials + (long long)(b + 1) * na + j);
      s2 += __ldcg(partials + (long long)(b + 2) * na + j);
      s3 += __ldcg(partials + (long long)(b + 3) * na + j);
    }
    for (; b < nrows; ++b) s0 += __ldcg(partials + (long long)b * na + j);
    out[j] = (s0 + s1) + (s2 + s3);
  }
}

// Result publication by the block that wrote out[0 .. na): after the
// block barrier, thread 0 writes the error flag, issues one system-scope
// fence (cumulative: it orders the block's out[] writes, observed through
// the barrier, before what follows) and writes the call number `seq` last,
// so a host that sees out[na + 1] == seq (mapped memory) may read
// everything before it.  Resets the counters for the next launch.
__device__ __forceinline__ void publish_result(unsigned int* __restrict__ ticket, int na,
                                               double* __restrict__ out, double seq) {
  __syncthreads();
  if (threadIdx.x == 0) {
    out[na] = (double)atomicOr((unsigned int*)(ticket + 1), 0u);
    ticket[0] = 0u;
    ticket[1] = 0u;
    __threadfence_system();
    out[na + 1] = seq;
  }
}

// Ordered two-level reduction of the block partials (row b = block b's
// `na` sums, written and fenced by every block before the call).  The last
// block of each group of PWA_GROUP consecutive blocks (ticket[2 + g])
// sums the group's rows in block order into group row g (stored after the
// block rows); the last group (ticket[0]) sums the group rows in order into
// out.  Returns true in that one block.  Counters are reset for the next
// launch; the order depends only on the grid size, so results are
// bitwise reproducible.  *s_flag is a __shared__ int of the caller.
__device__ __forceinline__ bool grouped_sum(double* __restrict__ partials,
                                            unsigned int* __restrict__ ticket, int na,
                                            double* __restrict__ out, int* s_flag) {
  const int nb = (int)gridDim.x, g = (int)blockIdx.x / PWA_GROUP;
  const int ng = (nb + PWA_GROUP - 1) / PWA_GROUP;
  const int gs = min(PWA_GROUP, nb - g * PWA_GROUP);
  double* grows = partials + (long long)nb * na;
  if (threadIdx.x == 0) *s_flag = (atomicAdd(ticket + 2 + g, 1u) == (unsigned)gs - 1);
  __syncthreads();
  if (!*s_flag) return false;
  __threadfence();
  for (int j = threadIdx.x; j < na; j += PWA_TPB) {
    double s[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int r = 0; r < PWA_GROUP; ++r)
      if (r < gs) s[r & 3] += __ldcg(partials + (long long)(g * PWA_GROUP + r) * na + j);
    grows[(long long)g * na + j] = (s[0] + s[1]) + (s[2] + s[3]);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    ticket[2 + g] = 0u;
    *s_flag = (atomicAdd(ticket, 1u) == (unsigned)ng - 1);
  }
  __syncthreads();
  if (!*s_flag) return false;
  __threadfence();
  last_block_sum(grows, ng, na, out);
  return true;
}

// Persistent streaming kernel over the column cache.  Thread 0 keeps
// PWA_STAGES tiles in flight with cp.async.bulk into a shared-memory ring
// (full-barrier per stage with transaction bytes); every thread evaluates
// one event of the current tile from shared memory in FP64; a block
// barrier frees the stage for the next copy.  Block partials go to
// `partials`; the last block to finish (atomic ticket) sums them in a fixed
// order and writes out[0 .. NA), out[NA] = error flag (0 = ok, 1 = a
// barrier wait gave up) and out[NA+1] = seq (the caller's call number, to
// detect a stale result); `out` may be mapped host memory.
extern "C" __global__ void __launch_bounds__(PWA_TPB)
    pwa_eval_cached(const CCoup c, const float2* __restrict__ Fc, const double* __restrict__ Wc,
                    long long ntiles, double* __restrict__ partials,
                    unsigned int* __restrict__ ticket, double* __restrict__ out, double seq) {
  constexpr int NA = PWA_CACHE_NA;
  constexpr unsigned TILE_F = PWA_NF * PWA_TPB * sizeof(float2);
  constexpr unsigned TILE_W = PWA_TPB * sizeof(double);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float2* sF = (float2*)smem_raw;                                    // [STAGES][NF][TPB]
  double* sW = (double*)(smem_raw + PWA_STAGES * TILE_F);            // [STAGES][TPB]
  __shared__ __align__(8) unsigned long long full[PWA_STAGES];
  __shared__ double red[PWA_TPB / 32][NA];
  __shared__ int s_last, s_err;
  const int tid = threadIdx.x;
  if (tid == 0) {
    s_err = 0;
    for (int st = 0; st < PWA_STAGES; ++st) mbar_init(&full[st], 1);
    mbar_fence_init();
  }
  __syncthreads();
  const long long G = gridDim.x, b0 = blockIdx.x;
  if (tid == 0) {
    for (int st = 0; st < PWA_STAGES; ++st) {
      const long long t = b0 + st * G;
      if (t < ntiles) {
        mbar_expect_tx(&full[st], TILE_F + TILE_W);
        bulk_g2s(sF + (long long)st * PWA_NF * PWA_TPB, Fc + t * PWA_NF * PWA_TPB, TILE_F, &full[st]);
        bulk_g2s(sW + st * PWA_TPB, Wc + t * PWA_TPB, TILE_W, &full[st]);
      }
    }
  }
  double acc[NA];
#pragma unroll
  for (int j = 0; j < NA; ++j) acc[j] = 0.0;
  int it = 0;
  for (long long t = b0; t < ntiles; t += G, ++it) {
    const int st = it % PWA_STAGES;
    const unsigned par = (unsigned)((it / PWA_STAGES) & 1);
    if (!mbar_wait(&full[st], par, PWA_WAIT_LIMIT)) {
      s_err = 1;  // benign race: any thread may set it
    }
    __syncthreads();
    if (s_err) break;
    const float2* F = sF + (long long)st * PWA_NF * PWA_TPB;
    const double w = sW[st * PWA_TPB + tid];
    double ar[PWA_NOUT], ai[PWA_NOUT];
#pragma unroll
    for (int o = 0; o < PWA_NOUT; ++o) ar[o] = ai[o] = 0.0;
#pragma unroll
    for (int j = 0; j < PWA_NF; ++j) {
      const int k = pwa_fk[j], o = pwa_fo[j];
      const float2 v = F[j * PWA_TPB + tid];
      const double fr = v.x, fi = v.y;
      const double cr = c.v[2 * k], ci = c.v[2 * k + 1];
      ar[o] = fma(cr, fr, fma(-ci, fi, ar[o]));
      ai[o] = fma(cr, fi, fma(ci, fr, ai[o]));
    }
    double f = 0.0;
#pragma unroll
    for (int o = 0; o < PWA_NOUT; ++o) f = fma(ar[o], ar[o], fma(ai[o], ai[o], f));
    double dl;
    const double cl = clip_log(f, &dl);
    acc[0] = fma(w, cl, acc[0]);
    const double fac = w * dl;
#pragma unroll
    for (int o = 0; o < PWA_NOUT; ++o) {
      ar[o] *= fac;
      ai[o] *= -fac;
    }
#pragma unroll
    for (int j = 0; j < PWA_NF; ++j) {
      const int k = pwa_fk[j], o = pwa_fo[j];
      const float2 v = F[j * PWA_TPB + tid];
      const double fr = v.x, fi = v.y;
      acc[1 + 2 * k] = fma(ar[o], fr, fma(-ai[o], fi, acc[1 + 2 * k]));
      acc[2 + 2 * k] = fma(ar[o], fi, fma(ai[o], fr, acc[2 + 2 * k]));
    }
    __syncthreads();  // stage st fully consumed
    if (tid == 0) {
      const long long tn = t + (long long)PWA_STAGES * G;
      if (tn < ntiles) {
        fence_proxy_async_smem();
        mbar_expect_tx(&full[st], TILE_F + TILE_W);
        bulk_g2s(sF + (long long)st * PWA_NF * PWA_TPB, Fc + tn * PWA_NF * PWA_TPB, TILE_F,
                 &full[st]);
        bulk_g2s(sW + st * PWA_TPB, Wc + tn * PWA_TPB, TILE_W, &full[st]);
      }
    }
  }
  if (s_err) {
    // drain: wait (bounded) for every copy this block issued before exiting
    const int issued = it + PWA_STAGES;
    if (tid == 0)
      for (int k2 = it; k2 < issued; ++k2) {
        const long long t2 = b0 + (long long)k2 * G;
        if (t2 < ntiles) mbar_wait(&full[k2 % PWA_STAGES], (unsigned)((k2 / PWA_STAGES) & 1), PWA_WAIT_LIMIT);
      }
  }
  const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
  for (int j = 0; j < NA; ++j) {
    const double v = warp_sum(acc[j]);
    if (lane == 0) red[warp][j] = v;
  }
  __syncthreads();
  for (int j = tid; j < NA; j += PWA_TPB) {
    double s = 0.0;
#pragma unroll
    for (int w2 = 0; w2 < PWA_TPB / 32; ++w2) s += red[w2][j];
    partials[(long long)blockIdx.x * NA + j] = s;
  }
  if (tid == 0 && s_err) atomicOr((unsigned int*)(ticket + 1), 1u);
  __threadfence();
  __syncthreads();
  if (!grouped_sum(partials, ticket, NA, out, &s_last)) return;
  publish_result(ticket, NA, out, seq);
}

// Direct-load variant of pwa_eval_cached: no shared-memory staging; each
// thread loads its event's pairs straight from the tile-major cache (a warp
// reads 256 contiguous bytes per pair) and the register budget is capped so
// that four blocks (16 warps) share an SM.  A, f, log and all cross-event
// sums in FP64; the per-event sensitivities G_k in FP32 (per-event rounding
// only, summed in FP64).  Same outputs and protocol as pwa_eval_cached.
extern "C" __global__ void __launch_bounds__(PWA_TPB, 4)
    pwa_eval_cached_direct(const CCoup c, const float2* __restrict__ Fc,
                           const double* __restrict__ Wc, long long ntiles,
                           double* __restrict__ partials, unsigned int* __restrict__ ticket,
                           double* __restrict__ out, double seq) {
  constexpr int NA = PWA_CACHE_NA;
  __shared__ double red[PWA_TPB / 32][NA];
  __shared__ int s_last;
  const int tid = threadIdx.x;
  double acc0 = 0.0;
  double accg[2 * PWA_NCOL];
#pragma unroll
  for (int j = 0; j < 2 * PWA_NCOL; ++j) accg[j] = 0.0;
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const float2* F = Fc + t * PWA_NF * PWA_TPB + tid;
    float2 v[PWA_NF];
#pragma unroll
    for (int j = 0; j < PWA_NF; ++j) v[j] = __ldcs(F + j * PWA_TPB);
    const double w = __ldcs(Wc + t * PWA_TPB + tid);
    double ar[PWA_NOUT], ai[PWA_NOUT];
#pragma unroll
    for (int o = 0; o < PWA_NOUT; ++o) ar[o] = ai[o] = 0.0;
#pragma unroll
    for (int j = 0; j < PWA_NF; ++j) {
      const int k = pwa_fk[j], o = pwa_fo[j];
      const double cr = c.v[2 * k], ci = c.v[2 * k + 1];
      ar[o] = fma(cr, (double)v[j].x, fma(-ci, (double)v[j].y, ar[o]));
      ai[o] = fma(cr, (double)v[j].y, fma(ci, (double)v[j].x, ai[o]));
    }
    double f = 0.0;
#pragma unroll
    for (int o = 0; o < PWA_NOUT; ++o) f = fma(ar[o], ar[o], fma(ai[o], ai[o], f));
    double dl;
    const double cl = clip_log(f, &dl);
    acc0 = fma(w, cl, acc0);
    const double fac = w * dl;
    float br[PWA_NOUT], bi[PWA_NOUT];
#pragma unroll
    for (int o = 0; o < PWA_NOUT; ++o) {
      br[o] = (float)(fac * ar[o]);
      bi[o] = (float)(-fac * ai[o]);
    }
    float gr[PWA_NCOL], gi[PWA_NCOL];
#pragma unroll
    for (int k = 0; k < PWA_NCOL; ++k) gr[k] = gi[k] = 0.f;
#pragma unroll
    for (int j = 0; j < PWA_NF; ++j) {
      const int k = pwa_fk[j], o = pwa_fo[j];
      gr[k] = fmaf(br[o], v[j].x, fmaf(-bi[o], v[j].y, gr[k]));
      gi[k] = fmaf(br[o], v[j].y, fmaf(bi[o], v[j].x, gi[k]));
    }
#pragma unroll
    for (int k = 0; k < PWA_NCOL; ++k) {
      accg[2 * k] += (double)gr[k];
      accg[2 * k + 1] += (double)gi[k];
    }
  }
  const int lane = tid & 31, warp = tid >> 5;
  {
    const double v0 = warp_sum(acc0);
    if (lane == 0) red[warp][0] = v0;
  }
#pragma unroll
  for (int j = 0; j < 2 * PWA_NCOL; ++j) {
    const double v2 = warp_sum(accg[j]);
    if (lane == 0) red[warp][1 + j] = v2;
  }
  __syncthreads();
  for (int j = tid; j < NA; j += PWA_TPB) {
    double s2 = 0.0;
#pragma unroll
    for (int w2 = 0; w2 < PWA_TPB / 32; ++w2) s2 += red[w2][j];
    partials[(long long)blockIdx.x * NA + j] = s2;
  }
  __threadfence();
  __syncthreads();
  if (!grouped_sum(partials, ticket, NA, out, &s_last)) return;
  publish_result(ticket, NA, out, seq);
}

// ---------------------------------------------------------------------------
// Column sensitivities summed over a warp before they reach FP64.  The
// per-event terms are those of pwa_eval_cached_direct; the FP32 values
// fac * conj(A) F_k of the warp's 32 events are summed by a reduce-scatter
// (lane l ends with entries PWA_GPAD / 32 * l ..), so each lane carries
// PWA_GPAD / 32 FP64 accumulators across tiles instead of 2 * PWA_NCOL:
// the register footprint no longer grows with the number of columns.
#define PWA_GPAD ((2 * PWA_NCOL + 31) / 32 * 32)
// With 2 * PWA_NCOL <= 16 the sensitivities form one group of 16 values:
// four halving steps leave lanes 2i and 2i + 1 with halves of entry i, one
// more shuffle gives both the warp sum (16 shuffles instead of 31).
// Otherwise PWA_GPAD / 32 groups of 32: lane l holds entry 32 m + l of group m.
#define PWA_RS16 (2 * PWA_NCOL <= 16)
#define PWA_MG (PWA_RS16 ? 1 : PWA_GPAD / 32)
__device__ __forceinline__ int rs_entry(int m, int lane) {
  return PWA_RS16 ? (lane >> 1) : 32 * m + lane;
}
__device__ __forceinline__ bool rs_owner(int lane) { return PWA_RS16 ? !(lane & 1) : true; }

struct CoupParam {  // couplings from the kernel's parameter block
  const CCoup& c;
  __device__ __forceinline__ double operator()(int i) const { return c.v[i]; }
};
struct CoupShared {  // couplings staged in shared memory (read per event, not hoisted)
  const double* c;
  __device__ __forceinline__ double operator()(int i) const { return c[i]; }
};
struct CoupGlobal {  // couplings from global memory (one row per request)
  const double* __restrict__ c;
  __device__ __forceinline__ double operator()(int i) const { return __ldg(c + i); }
};

// One event of a column tile: returns w * clip_log(f) and adds to g (entries
// 2k, 2k + 1 = re, im of fac * conj(A) F_k; the caller zeroes g).  The
// amplitude sums run in two interleaved FP64 partial sums per output to
// halve the dependent-FMA chain.
template <class Coup>
__device__ __forceinline__ double cached_event(const float2 (&v)[PWA_NF], double w,
                                               const Coup& cp, float (&g)[PWA_GPAD]) {
  double ar[PWA_NOUT], ai[PWA_NOUT], br2[PWA_NOUT], bi2[PWA_NOUT];
#pragma unroll
  for (int o = 0; o < PWA_NOUT; ++o) ar[o] = ai[o] = br2[o] = bi2[o] = 0.0;
#pragma unroll
  for (int j = 0; j < PWA_NF; ++j) {
    const int k = pwa_fk[j], o = pwa_fo[j];
    const double cr = cp(2 * k), ci = cp(2 * k + 1);
    if (j & 1) {
      br2[o] = fma(cr, (double)v[j].x, fma(-ci, (double)v[j].y, br2[o]));
      bi2[o] = fma(cr, (double)v[j].y, fma(ci, (double)v[j].x, bi2[o]));
    } else {
      ar[o] = fma(cr, (double)v[j].x, fma(-ci, (double)v[j].y, ar[o]));
      ai[o] = fma(cr, (double)v[j].y, fma(ci, (double)v[j].x, ai[o]));
    }
  }
  double f = 0.0;
#pragma unroll
  for (int o = 0; o < PWA_NOUT; ++o) {
    ar[o] += br2[o];
    ai[o] += bi2[o];
    f = fma(ar[o], ar[o], fma(ai[o], ai[o], f));
  }
  double dl;
  const double cl = clip_log(f, &dl);
  const double fac = w * dl;
  float br[PWA_NOUT], bi[PWA_NOUT];
#pragma unroll
  for (int o = 0; o < PWA_NOUT; ++o) {
    br[o] = (float)(fac * ar[o]);
    bi[o] = (float)(-fac * ai[o]);
  }
#pragma unroll
  for (int j = 0; j < PWA_NF; ++j) {
    const int k = pwa_fk[j], o = pwa_fo[j];
    g[2 * k] = fmaf(br[o], v[j].x, fmaf(-bi[o], v[j].y, g[2 * k]));
    g[2 * k + 1] = fmaf(br[o], v[j].y, fmaf(bi[o], v[j].x, g[2 * k + 1]));
  }
  return w * cl;
}

// four blocks per SM (128 registers)
#ifndef PWA_WRED_MINB
#define PWA_WRED_MINB 4
#endif

// One event of a tile (its columns v[j] loaded once): returns
// w * clip_log(f).  The sensitivities of the warp's 32 events are formed 16
// complex columns at a time and reduce-scattered: gs[m] receives on each
// lane the warp sum of entry 32 m + lane (entries 2k, 2k + 1 = re, im of
// fac * conj(A) F_k).  Every lane of the warp must call it (shuffles).
template <class Coup>
__device__ __forceinline__ double cached_event_rs(const float2 (&v)[PWA_NF], double w,
                                                  const Coup& cp, int lane,
                                                  float (&gs)[PWA_MG]) {
  double ar[PWA_NOUT], ai[PWA_NOUT], br2[PWA_NOUT], bi2[PWA_NOUT];
#pragma unroll
  for (int o = 0; o < PWA_NOUT; ++o) ar[o] = ai[o] = br2[o] = bi2[o] = 0.0;
#pragma unroll
  for (int j = 0; j < PWA_NF; ++j) {
    const int k = pwa_fk[j], o = pwa_fo[j];
    const double cr = cp(2 * k), ci = cp(2 * k + 1);
    if (j & 1) {
      br2[o] = fma(cr, (double)v[j].x, fma(-ci, (double)v[j].y, br2[o]));
      bi2[o] = fma(cr, (double)v[j].y, fma(ci, (double)v[j].x, bi2[o]));
    } else {
      ar[o] = fma(cr, (double)v[j].x, fma(-ci, (double)v[j].y, ar[o]));
      ai[o] = fma(cr, (double)v[j].y, fma(ci, (double)v[j].x, ai[o]));
    }
  }
  double f = 0.0;
#pragma unroll
  for (int o = 0; o < PWA_NOUT; ++o) {
    ar[o] += br2[o];
    ai[o] += bi2[o];
    f = fma(ar[o], ar[o], fma(ai[o], ai[o], f));
  }
  double dl;
  const double cl = clip_log(f, &dl);
  const double fac = w * dl;
  float br[PWA_NOUT], bi[PWA_NOUT];
#pragma unroll
  for (int o = 0; o < PWA_NOUT; ++o) {
    br[o] = (float)(fac * ar[o]);
    bi[o] = (float)(-fac * ai[o]);
  }
#if PWA_RS16
  {
    float g[16];
#pragma unroll
    for (int q = 0; q < 16; ++q) g[q] = 0.f;
#pragma unroll
    for (int j = 0; j < PWA_NF; ++j) {
      const int k = pwa_fk[j], o = pwa_fo[j];
      g[2 * k] = fmaf(br[o], v[j].x, fmaf(-bi[o], v[j].y, g[2 * k]));
      g[2 * k + 1] = fmaf(br[o], v[j].y, fmaf(bi[o], v[j].x, g[2 * k + 1]));
    }
    warp_rs_step<16, 16, 16>(g, lane);
    gs[0] = g[0] + __shfl_xor_sync(0xffffffffu, g[0], 1);
  }
#else
#pragma unroll
  for (int m = 0; m < PWA_GPAD / 32; ++m) {
    float g[32];
#pragma unroll
    for (int q = 0; q < 32; ++q) g[q] = 0.f;
#pragma unroll
    for (int j = 0; j < PWA_NF; ++j) {
      const int k = pwa_fk[j], o = pwa_fo[j];
      if (k >= 16 * m && k < 16 * m + 16) {
        const int q = 2 * (k - 16 * m);
        g[q] = fmaf(br[o], v[j].x, fmaf(-bi[o], v[j].y, g[q]));
        g[q + 1] = fmaf(br[o], v[j].y, fmaf(bi[o], v[j].x, g[q + 1]));
      }
    }
    warp_reduce_scatter<32>(g, lane);
    gs[m] = g[0];
  }
#endif
  return w * cl;
}

extern "C" __global__ void __launch_bounds__(PWA_TPB, PWA_WRED_MINB)
    pwa_eval_cached_wred(const CCoup c, const float2* __restrict__ Fc,
                         const double* __restrict__ Wc, long long ntiles,
                         double* __restrict__ partials, unsigned int* __restrict__ ticket,
                         double* __restrict__ out, double seq) {
  constexpr int NA = PWA_CACHE_NA;
  constexpr int NG = 2 * PWA_NCOL, MG = PWA_MG;
  __shared__ double red[PWA_TPB / 32][NA];
  __shared__ int s_last;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  __shared__ double s_c[2 * PWA_NCOL];
  stage_couplings(c, s_c);
  __syncthreads();
  const CoupShared cp{s_c};
  double acc0 = 0.0;
  double accg[MG];
#pragma unroll
  for (int j = 0; j < MG; ++j) accg[j] = 0.0;
#pragma unroll 1
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const float2* F = Fc + t * PWA_NF * PWA_TPB + tid;
    float2 v[PWA_NF];
#pragma unroll
    for (int j = 0; j < PWA_NF; ++j) v[j] = __ldcs(F + j * PWA_TPB);
    const double w = __ldcs(Wc + t * PWA_TPB + tid);
    float gs[MG];
    acc0 += cached_event_rs(v, w, cp, lane, gs);
#pragma unroll
    for (int m = 0; m < MG; ++m) accg[m] += (double)gs[m];
  }
  {
    const double v0 = warp_sum(acc0);
    if (lane == 0) red[warp][0] = v0;
  }
#pragma unroll
  for (int m = 0; m < MG; ++m) {
    const int idx = rs_entry(m, lane);
    if (rs_owner(lane) && idx < NG) red[warp][1 + idx] = accg[m];
  }
  __syncthreads();
  for (int j = tid; j < NA; j += PWA_TPB) {
    double s2 = 0.0;
#pragma unroll
    for (int w2 = 0; w2 < PWA_TPB / 32; ++w2) s2 += red[w2][j];
    partials[(long long)blockIdx.x * NA + j] = s2;
  }
  __threadfence();
  __syncthreads();
  if (!grouped_sum(partials, ticket, NA, out, &s_last)) return;
  publish_result(ticket, NA, out, seq);
}

// ---------------------------------------------------------------------------
// Shared-memory ring with register-light consumers.  Thread 0 keeps
// PWA_RSTAGES tiles of the column cache in flight with cp.async.bulk (as in
// pwa_eval_cached); every thread evaluates its event of the current tile
// reading its columns from shared memory (FP64 amplitude), then forms the
// column sensitivities 16 complex columns at a time and reduce-scatters each
// group of 32 FP32 values across the warp, so a lane carries PWA_GPAD / 32
// FP64 accumulators.  The bytes in flight are the ring's, not registers, so
// the kernel keeps HBM busy at low occupancy.  Same outputs and protocol as
// pwa_eval_cached.
#ifndef PWA_RSTAGES
#define PWA_RSTAGES 2
#endif
extern "C" __global__ void __launch_bounds__(PWA_TPB)
    pwa_eval_cached_ring2(const CCoup c, const float2* __restrict__ Fc,
                          const double* __restrict__ Wc, long long ntiles,
                          double* __restrict__ partials, unsigned int* __restrict__ ticket,
                          double* __restrict__ out, double seq) {
  constexpr int NA = PWA_CACHE_NA;
  constexpr int NG = 2 * PWA_NCOL, MG = PWA_GPAD / 32;
  constexpr unsigned TILE_F = PWA_NF * PWA_TPB * sizeof(float2);
  constexpr unsigned TILE_W = PWA_TPB * sizeof(double);
  extern __shared__ __align__(128) unsigned char smem_raw[];
  float2* sF = (float2*)smem_raw;                                    // [RSTAGES][NF][TPB]
  double* sW = (double*)(smem_raw + PWA_RSTAGES * TILE_F);           // [RSTAGES][TPB]
  __shared__ __align__(8) unsigned long long full[PWA_RSTAGES];
  __shared__ double red[PWA_TPB / 32][NA];
  __shared__ int s_last, s_err;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) {
    s_err = 0;
    for (int st = 0; st < PWA_RSTAGES; ++st) mbar_init(&full[st], 1);
    mbar_fence_init();
  }
  __syncthreads();
  const long long G = gridDim.x, b0 = blockIdx.x;
  if (tid == 0) {
    for (int st = 0; st < PWA_RSTAGES; ++st) {
      const long long t = b0 + st * G;
      if (t < ntiles) {
        mbar_expect_tx(&full[st], TILE_F + TILE_W);
        bulk_g2s(sF + (long long)st * PWA_NF * PWA_TPB, Fc + t * PWA_NF * PWA_TPB, TILE_F, &full[st]);
        bulk_g2s(sW + st * PWA_TPB, Wc + t * PWA_TPB, TILE_W, &full[st]);
      }
    }
  }
  const CoupParam cp{c};
  double acc0 = 0.0;
  double accg[MG];
#pragma unroll
  for (int j = 0; j < MG; ++j) accg[j] = 0.0;
  int it = 0;
  for (long long t = b0; t < ntiles; t += G, ++it) {
    const int st = it % PWA_RSTAGES;
    const unsigned par = (unsigned)((it / PWA_RSTAGES) & 1);
    if (!mbar_wait(&full[st], par, PWA_WAIT_LIMIT)) {
      s_err = 1;  // benign race: any thread may set it
    }
    __syncthreads();
    if (s_err) break;
    const float2* F = sF + (long long)st * PWA_NF * PWA_TPB + tid;
    const double w = sW[st * PWA_TPB + tid];
    double ar[PWA_NOUT], ai[PWA_NOUT];
#pragma unroll
    for (int o = 0; o < PWA_NOUT; ++o) ar[o] = ai[o] = 0.0;
#pragma unroll
    for (int j = 0; j < PWA_NF; ++j) {
      const int k = pwa_fk[j], o = pwa_fo[j];
      const float2 v = F[j * PWA_TPB];
      const double cr = cp(2 * k), ci = cp(2 * k + 1);
      ar[o] = fma(cr, (double)v.x, fma(-ci, (double)v.y, ar[o]));
      ai[o] = fma(cr, (double)v.y, fma(ci, (double)v.x, ai[o]));
    }
    double f = 0.0;
#pragma unroll
    for (int o = 0; o < PWA_NOUT; ++o) f = fma(ar[o], ar[o], fma(ai[o], ai[o], f));
    double dl;
    const double cl = clip_log(f, &dl);
    acc0 = fma(w, cl, acc0);
    const double fac = w * dl;
    float br[PWA_NOUT], bi[PWA_NOUT];
#pragma unroll
    for (int o = 0; o < PWA_NOUT; ++o) {
      br[o] = (float)(fac * ar[o]);
      bi[o] = (float)(-fac * ai[o]);
    }
#pragma unroll
    for (int m = 0; m < MG; ++m) {
      float g[32];
#pragma unroll
      for (int q = 0; q < 32; ++q) g[q] = 0.f;
#pragma unroll
      for (int j = 0; j < PWA_NF; ++j) {
        const int k = pwa_fk[j], o = pwa_fo[j];
        if (k >= 16 * m && k < 16 * m + 16) {
          const float2 v = F[j * PWA_TPB];
          const int q = 2 * (k - 16 * m);
          g[q] = fmaf(br[o], v.x, fmaf(-bi[o], v.y, g[q]));
          g[q + 1] = fmaf(br[o], v.y, fmaf(bi[o], v.x, g[q + 1]));
        }
      }
      warp_reduce_scatter<32>(g, lane);
      accg[m] += (double)g[0];
    }
    __syncthreads();  // stage st fully consumed
    if (tid == 0) {
      const long long tn = t + (long long)PWA_RSTAGES * G;
      if (tn < ntiles) {
        fence_proxy_async_smem();
        mbar_expect_tx(&full[st], TILE_F + TILE_W);
        bulk_g2s(sF + (long long)st * PWA_NF * PWA_TPB, Fc + tn * PWA_NF * PWA_TPB, TILE_F,
                 &full[st]);
        bulk_g2s(sW + st * PWA_TPB, Wc + tn * PWA_TPB, TILE_W, &full[st]);
      }
    }
  }
  if (s_err) {
    // drain: wait (bounded) for every copy this block issued before exiting
    const int issued = it + PWA_RSTAGES;
    if (tid == 0)
      for (int k2 = it; k2 < issued; ++k2) {
        const long long t2 = b0 + (long long)k2 * G;
        if (t2 < ntiles) mbar_wait(&full[k2 % PWA_RSTAGES], (unsigned)((k2 / PWA_RSTAGES) & 1), PWA_WAIT_LIMIT);
      }
  }
  {
    const double v0 = warp_sum(acc0);
    if (lane == 0) red[warp][0] = v0;
  }
#pragma unroll
  for (int m = 0; m < MG; ++m) {
    const int idx = 32 * m + lane;  // entry `lane` of column group m
    if (idx < NG) red[warp][1 + idx] = accg[m];
  }
  __syncthreads();
  for (int j = tid; j < NA; j += PWA_TPB) {
    double s2 = 0.0;
#pragma unroll
    for (int w2 = 0; w2 < PWA_TPB / 32; ++w2) s2 += red[w2][j];
    partials[(long long)blockIdx.x * NA + j] = s2;
  }
  if (tid == 0 && s_err) atomicOr((unsigned int*)(ticket + 1), 1u);
  __threadfence();
  __syncthreads();
  if (!grouped_sum(partials, ticket, NA, out, &s_last)) return;
  publish_result(ticket, NA, out, seq);
}

// ---------------------------------------------------------------------------
// Check of the bounded waits and of the error protocol of the cached
// kernels (one block, PWA_TPB threads).  Thread 0 arms barrier `never`
// for one tile of bytes that no copy will bring, and barrier `real` for
// one bulk copy of `src` that it does issue; it waits on `never` for
// `polls` polls (the wait gives up), then waits (bounded) on `real`, so no
// copy is in flight when the block exits, and publishes zero sums with
// the error flag set -- what a stalled ring kernel reports.
extern "C" __global__ void __launch_bounds__(PWA_TPB)
    pwa_wait_check(const double* __restrict__ src, unsigned polls,
                   unsigned int* __restrict__ ticket, double* __restrict__ out, double seq,
                   int na) {
  __shared__ __align__(128) double buf[PWA_TPB];
  __shared__ __align__(8) unsigned long long never, real;
  if (threadIdx.x == 0) {
    mbar_init(&never, 1);
    mbar_init(&real, 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    mbar_expect_tx(&never, (unsigned)sizeof(buf));
    mbar_expect_tx(&real, (unsigned)sizeof(buf));
    bulk_g2s(buf, src, (unsigned)sizeof(buf), &real);
    const bool ok = mbar_wait(&never, 0u, polls);
    mbar_wait(&real, 0u, PWA_WAIT_LIMIT);
    if (!ok) atomicOr((unsigned int*)(ticket + 1), 1u);
  }
  for (int j = threadIdx.x; j < na; j += PWA_TPB) out[j] = 0.0;
  publish_result(ticket, na, out, seq);
}

// ---------------------------------------------------------------------------
// Kernels with one block per SM.  Their block partials are few (one row per
// SM), so a single ordered level replaces the two-level reduction: every
// block writes its row and fences it, the last block to take ticket[0] sums
// all rows.  Its threads form `slices` = blockDim / na groups; slice s sums
// rows s, s + slices, ... in order (two interleaved chains), then thread j
// adds the slices' values in order.  The order depends only on the grid:
// bitwise reproducible.  scratch: __shared__, at least blockDim doubles.
__device__ __forceinline__ bool flat_sum(const double* __restrict__ partials,
                                         unsigned int* __restrict__ ticket, int na,
                                         double* __restrict__ out, double* scratch,
                                         int* s_flag) {
  const int nrows = (int)gridDim.x, nt = (int)blockDim.x, t = (int)threadIdx.x;
  if (t == 0) *s_flag = (atomicAdd(ticket, 1u) == (unsigned)nrows - 1);
  __syncthreads();
  if (!*s_flag) return false;
  __threadfence();
  const int slices = nt / na;
  if (slices == 0) {
    for (int j = t; j < na; j += nt) {
      double a0 = 0.0, a1 = 0.0;
      int r = 0;
      for (; r + 1 < nrows; r += 2) {
        a0 += __ldcg(partials + (long long)r * na + j);
        a1 += __ldcg(partials + (long long)(r + 1) * na + j);
      }
      if (r < nrows) a0 += __ldcg(partials + (long long)r * na + j);
      out[j] = a0 + a1;
    }
    return true;
  }
  if (t < slices * na) {
    const int j = t % na, s = t / na;
    double a0 = 0.0, a1 = 0.0;
    int r = s;
    for (; r + slices < nrows; r += 2 * slices) {
      a0 += __ldcg(partials + (long long)r * na + j);
      a1 += __ldcg(partials + (long long)(r + slices) * na + j);
    }
    if (r < nrows) a0 += __ldcg(partials + (long long)r * na + j);
    scratch[s * na + j] = a0 + a1;
  }
  __syncthreads();
  for (int j = t; j < na; j += nt) {
    double a = 0.0;
    for (int s = 0; s < slices; ++s) a += scratch[s * na + j];
    out[j] = a;
  }
  return true;
}

// Warp sums of one block (acc0 on every lane, column group m's entry on
// lane l = value 32 m + l) into red[warp][.], then the block's row of
// partials in warp order.  All threads of the block call it.
template <int NW>
__device__ __forceinline__ void cached_block_row(double acc0, const double* accg,
                                                 double (*red)[PWA_CACHE_NA], int warp, int lane,
                                                 bool active, double* __restrict__ partials) {
  constexpr int NA = PWA_CACHE_NA, NG = 2 * PWA_NCOL, MG = PWA_MG;
  if (active) {
    const double v0 = warp_sum(acc0);
    if (lane == 0) red[warp][0] = v0;
#pragma unroll
    for (int m = 0; m < MG; ++m) {
      const int idx = rs_entry(m, lane);
      if (rs_owner(lane) && idx < NG) red[warp][1 + idx] = accg[m];
    }
  }
  __syncthreads();
  for (int j = (int)threadIdx.x; j < NA; j += (int)blockDim.x) {
    double s = 0.0;
#pragma unroll
    for (int w2 = 0; w2 < NW; ++w2) s += red[w2][j];
    partials[(long long)blockIdx.x * NA + j] = s;
  }
  __threadfence();
  __syncthreads();
}

// Variant 4: one block of PWA_WIDE_WARPS warps per SM.  Each warp streams a
// contiguous run of 32-event units (a quarter of a 128-event tile: 256
// contiguous bytes per cached pair) with the register-held columns and the
// warp reduce-scatter of pwa_eval_cached_wred; contiguous runs keep every
// warp's addresses within a few pages and balance the work to one unit.
#ifndef PWA_WIDE_WARPS
#define PWA_WIDE_WARPS 16
#endif
extern "C" __global__ void __launch_bounds__(PWA_WIDE_WARPS * 32, 1)
    pwa_eval_cached_wide(const CCoup c, const float2* __restrict__ Fc,
                         const double* __restrict__ Wc, long long ntiles,
                         double* __restrict__ partials, unsigned int* __restrict__ ticket,
                         double* __restrict__ out, double seq) {
  constexpr int NA = PWA_CACHE_NA, MG = PWA_MG;
  constexpr int NW = PWA_WIDE_WARPS, UPT = PWA_TPB / 32;
  __shared__ double red[NW][NA];
  __shared__ double s_c[2 * PWA_NCOL];
  __shared__ double scratch[NW * 32];
  __shared__ int s_last;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  stage_couplings(c, s_c);
  __syncthreads();
  const CoupShared cp{s_c};
  const long long U = ntiles * UPT, W = (long long)gridDim.x * NW;
  const long long gw = (long long)blockIdx.x * NW + warp;
  const long long u0 = gw * U / W, u1 = (gw + 1) * U / W;
  double acc0 = 0.0;
  double accg[MG];
#pragma unroll
  for (int m = 0; m < MG; ++m) accg[m] = 0.0;
#pragma unroll 1
  for (long long u = u0; u < u1; ++u) {
    const long long t = u / UPT;
    const int e = (int)(u - t * UPT) * 32 + lane;
    const float2* F = Fc + t * PWA_NF * PWA_TPB + e;
    float2 v[PWA_NF];
#pragma unroll
    for (int j = 0; j < PWA_NF; ++j) v[j] = __ldcs(F + j * PWA_TPB);
    const double w = __ldcs(Wc + t * PWA_TPB + e);
    float gs[MG];
    acc0 += cached_event_rs(v, w, cp, lane, gs);
#pragma unroll
    for (int m = 0; m < MG; ++m) accg[m] += (double)gs[m];
  }
  cached_block_row<NW>(acc0, accg, red, warp, lane, true, partials);
  if (!flat_sum(partials, ticket, NA, out, scratch, &s_last)) return;
  publish_result(ticket, NA, out, seq);
}

// Variant 5: warp-specialised ring, one block per SM.  One producer lane
// keeps up to `stages` (<= PWA_TMA_MAXST) whole 128-event tiles in flight
// with cp.async.bulk (no multicast) into a shared-memory ring; a stage has
// a full barrier (transaction bytes) and an empty barrier (one arrival per
// consumer warp of the group that reads it).  PWA_TMA_GROUPS groups of
// PWA_TPB / 32 consumer warps take the block's tiles in turn; a consumer
// warp copies its 32 events' columns to registers, releases the stage at
// once, then evaluates them as pwa_eval_cached_wred does.  The block's tiles
// are one contiguous run.  Waits are bounded: a wait that gives up sets the
// error flag, the producer waits (bounded) for every copy it issued, and
// the host sees out[NA] != 0.  The ring depth must be a multiple of
// PWA_TMA_GROUPS: then every stage is read by one consumer group only, in
// iteration order, so no group ever waits on a barrier phase two ahead of
// the current one (a parity wait for that phase would return at once).
// Any other depth is refused with the error flag before any barrier use.
#ifndef PWA_TMA_GROUPS
#define PWA_TMA_GROUPS 2
#endif
#define PWA_TMA_MAXST 8
#define PWA_TMA_THREADS ((PWA_TMA_GROUPS * (PWA_TPB / 32) + 1) * 32)
extern "C" __global__ void __launch_bounds__(PWA_TMA_THREADS, 1)
    pwa_eval_cached_tma(const CCoup c, const float2* __restrict__ Fc,
                        const double* __restrict__ Wc, long long ntiles,
                        double* __restrict__ partials, unsigned int* __restrict__ ticket,
                        double* __restrict__ out, double seq, int stages) {
  constexpr int NA = PWA_CACHE_NA, MG = PWA_MG;
  constexpr int UPT = PWA_TPB / 32, NCW = PWA_TMA_GROUPS * UPT;
  constexpr unsigned TILE_F = PWA_NF * PWA_TPB * sizeof(float2);
  constexpr unsigned TILE_W = PWA_TPB * sizeof(double);
  constexpr unsigned STAGE = TILE_F + TILE_W;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(8) unsigned long long full[PWA_TMA_MAXST], empty[PWA_TMA_MAXST];
  __shared__ double red[NCW][NA];
  __shared__ double s_c[2 * PWA_NCOL];
  __shared__ double scratch[PWA_TMA_THREADS];
  __shared__ int s_last;
  __shared__ volatile int s_err;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (stages < PWA_TMA_GROUPS || stages > PWA_TMA_MAXST || stages % PWA_TMA_GROUPS) {
    // refused depth: report it like a stalled ring (zero sums, error flag)
    if (tid == 0) atomicOr((unsigned int*)(ticket + 1), 1u);
    for (int j = tid; j < NA; j += PWA_TMA_THREADS) partials[(long long)blockIdx.x * NA + j] = 0.0;
    __threadfence();
    __syncthreads();
    if (!flat_sum(partials, ticket, NA, out, scratch, &s_last)) return;
    publish_result(ticket, NA, out, seq);
    return;
  }
  if (tid == 0) {
    s_err = 0;
    for (int st = 0; st < stages; ++st) {
      mbar_init(&full[st], 1);
      mbar_init(&empty[st], UPT);
    }
    mbar_fence_init();
  }
  stage_couplings(c, s_c);
  __syncthreads();
  const long long B = gridDim.x, b = blockIdx.x;
  const long long t0 = b * ntiles / B, t1 = (b + 1) * ntiles / B;
  const int n_it = (int)(t1 - t0);
  double acc0 = 0.0;
  double accg[MG];
#pragma unroll
  for (int m = 0; m < MG; ++m) accg[m] = 0.0;
  int issued = 0;
  if (warp == NCW) {
    if (lane == 0) {
      for (int it = 0; it < n_it; ++it) {
        const int st = it % stages;
        if (it >= stages &&
            !mbar_wait(&empty[st], (unsigned)((it / stages - 1) & 1), PWA_WAIT_LIMIT)) {
          s_err = 1;
          break;
        }
        if (s_err) break;
        fence_proxy_async_smem();
        unsigned char* dst = smem_raw + (size_t)st * STAGE;
        mbar_expect_tx(&full[st], STAGE);
        bulk_g2s(dst, Fc + (t0 + it) * PWA_NF * PWA_TPB, TILE_F, &full[st]);
        bulk_g2s(dst + TILE_F, Wc + (t0 + it) * PWA_TPB, TILE_W, &full[st]);
        issued = it + 1;
      }
    }
  } else {
    const int g = warp / UPT, q = warp % UPT;
    const CoupShared cp{s_c};
    for (int it = g; it < n_it; it += PWA_TMA_GROUPS) {
      const int st = it % stages;
      if (!mbar_wait(&full[st], (unsigned)((it / stages) & 1), PWA_WAIT_LIMIT)) s_err = 1;
      if (s_err) break;
      const unsigned char* src = smem_raw + (size_t)st * STAGE;
      const float2* F = (const float2*)src + q * 32 + lane;
      float2 v[PWA_NF];
#pragma unroll
      for (int j = 0; j < PWA_NF; ++j) v[j] = F[j * PWA_TPB];
      const double w = ((const double*)(src + TILE_F))[q * 32 + lane];
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[st]);
      float gs[MG];
      acc0 += cached_event_rs(v, w, cp, lane, gs);
#pragma unroll
      for (int m = 0; m < MG; ++m) accg[m] += (double)gs[m];
    }
  }
  __syncthreads();
  if (s_err && warp == NCW && lane == 0) {
    // no copy may still be writing shared memory when the block exits: wait
    // (bounded) for the last phase of every stage that received a copy
    for (int it = issued - stages > 0 ? issued - stages : 0; it < issued; ++it)
      mbar_wait(&full[it % stages], (unsigned)((it / stages) & 1), PWA_WAIT_LIMIT);
    atomicOr((unsigned int*)(ticket + 1), 1u);
  }
  cached_block_row<NCW>(acc0, accg, red, warp, lane, warp < NCW, partials);
  if (!flat_sum(partials, ticket, NA, out, scratch, &s_last)) return;
  publish_result(ticket, NA, out, seq);
}

// ---------------------------------------------------------------------------
// Many parameter points in one pass over the column cache (Hessian stencils,
// line-search trials, likelihood scans).  One block of PWA_PTS_WARPS warps
// per SM; each warp takes a contiguous run of 32-event units, holds the
// unit's columns in registers and evaluates every point m of the launch on
// them: A_o = sum_k c_mk F_ko in FP32 (couplings staged as FP32 in shared
// memory), f = sum_o |A_o|^2, w * log f (FP32 log, summed in FP64) and the
// sensitivities fac * conj(A) F_k (fac = w clip_log'(f), FP32, reduce-
// scattered across the warp, FP64 accumulation).  Per-warp FP64 rows of
// (point, accumulator) live in shared memory; the block writes its row of
// n_pts * NA sums and the last block sums the rows in a fixed order into
// out[n_pts][NA].  FP32 amplitudes keep the gradient to ~1e-6 relative:
// the differenced Hessian needs no more (the centre point of a stencil is
// evaluated by the FP64-amplitude kernel).
#ifndef PWA_PTS_WARPS
#define PWA_PTS_WARPS 16
#endif
__device__ __forceinline__ float clip_logf(float x, float* dx) {
  const float eps = 1e-6f;
  if (x > eps) {
    *dx = 1.0f / x;
    return logf(x);
  }
  const float t = (x - eps) / eps;
  *dx = 1.0f / eps - (x - eps) / (eps * eps);
  return -13.815510557964274f + t - 0.5f * t * t;  // log(1e-6) + t - t^2/2
}

extern "C" __global__ void __launch_bounds__(PWA_PTS_WARPS * 32, 1)
    pwa_eval_cached_points(const double* __restrict__ ck, int n_pts,
                           const float2* __restrict__ Fc, const double* __restrict__ Wc,
                           long long ntiles, double* __restrict__ partials,
                           unsigned int* __restrict__ ticket, double* __restrict__ out) {
  constexpr int NA = PWA_CACHE_NA, NG = 2 * PWA_NCOL;
  constexpr int NW = PWA_PTS_WARPS, UPT = PWA_TPB / 32;
  extern __shared__ __align__(16) double pts_smem[];
  double* s_acc = pts_smem;                                   // [NW][n_pts][NA]
  float* s_c = (float*)(pts_smem + (size_t)NW * n_pts * NA);  // [n_pts][2 NCOL]
  __shared__ int s_last;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int j = tid; j < NW * n_pts * NA; j += NW * 32) s_acc[j] = 0.0;
  for (int j = tid; j < n_pts * NG; j += NW * 32) s_c[j] = (float)ck[j];
  __syncthreads();
  const long long U = ntiles * UPT, W = (long long)gridDim.x * NW;
  const long long gw = (long long)blockIdx.x * NW + warp;
  const long long u0 = gw * U / W, u1 = (gw + 1) * U / W;
  double* my = s_acc + (size_t)warp * n_pts * NA;
#pragma unroll 1
  for (long long u = u0; u < u1; ++u) {
    const long long t = u / UPT;
    const int e = (int)(u - t * UPT) * 32 + lane;
    const float2* F = Fc + t * PWA_NF * PWA_TPB + e;
    float2 v[PWA_NF];
#pragma unroll
    for (int j = 0; j < PWA_NF; ++j) v[j] = __ldcs(F + j * PWA_TPB);
    const float w = (float)__ldcs(Wc + t * PWA_TPB + e);
#pragma unroll 1
    for (int m = 0; m < n_pts; ++m) {
      const float* c = s_c + m * NG;
      float ar[PWA_NOUT], ai[PWA_NOUT];
#pragma unroll
      for (int o = 0; o < PWA_NOUT; ++o) ar[o] = ai[o] = 0.f;
#pragma unroll
      for (int j = 0; j < PWA_NF; ++j) {
        const int k = pwa_fk[j], o = pwa_fo[j];
        const float cr = c[2 * k], ci = c[2 * k + 1];
        ar[o] = fmaf(cr, v[j].x, fmaf(-ci, v[j].y, ar[o]));
        ai[o] = fmaf(cr, v[j].y, fmaf(ci, v[j].x, ai[o]));
      }
      float f = 0.f;
#pragma unroll
      for (int o = 0; o < PWA_NOUT; ++o) f = fmaf(ar[o], ar[o], fmaf(ai[o], ai[o], f));
      float dl;
      const float cl = clip_logf(f, &dl);
      const float fac = w * dl;
      float br[PWA_NOUT], bi[PWA_NOUT];
#pragma unroll
      for (int o = 0; o < PWA_NOUT; ++o) {
        br[o] = fac * ar[o];
        bi[o] = -fac * ai[o];
      }
      const double s0 = warp_sum((double)(w * cl));
      if (lane == 0) my[m * NA] += s0;
#if PWA_RS16
      float g[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) g[q] = 0.f;
#pragma unroll
      for (int j = 0; j < PWA_NF; ++j) {
        const int k = pwa_fk[j], o = pwa_fo[j];
        g[2 * k] = fmaf(br[o], v[j].x, fmaf(-bi[o], v[j].y, g[2 * k]));
        g[2 * k + 1] = fmaf(br[o], v[j].y, fmaf(bi[o], v[j].x, g[2 * k + 1]));
      }
      warp_rs_step<16, 16, 16>(g, lane);
      const float gs = g[0] + __shfl_xor_sync(0xffffffffu, g[0], 1);
      const int idx = lane >> 1;
      if (!(lane & 1) && idx < NG) my[m * NA + 1 + idx] += (double)gs;
#else
#pragma unroll
      for (int mg = 0; mg < PWA_GPAD / 32; ++mg) {
        float g[32];
#pragma unroll
        for (int q = 0; q < 32; ++q) g[q] = 0.f;
#pragma unroll
        for (int j = 0; j < PWA_NF; ++j) {
          const int k = pwa_fk[j], o = pwa_fo[j];
          if (k >= 16 * mg && k < 16 * mg + 16) {
            const int q = 2 * (k - 16 * mg);
            g[q] = fmaf(br[o], v[j].x, fmaf(-bi[o], v[j].y, g[q]));
            g[q + 1] = fmaf(br[o], v[j].y, fmaf(bi[o], v[j].x, g[q + 1]));
          }
        }
        warp_reduce_scatter<32>(g, lane);
        const int idx = 32 * mg + lane;
        if (idx < NG) my[m * NA + 1 + idx] += (double)g[0];
      }
#endif
    }
  }
  __syncthreads();
  // block row: the warps' rows summed in warp order
  const int tot = n_pts * NA;
  for (int j = tid; j < tot; j += NW * 32) {
    double a = 0.0;
    for (int w2 = 0; w2 < NW; ++w2) a += s_acc[(size_t)w2 * tot + j];
    partials[(long long)blockIdx.x * tot + j] = a;
  }
  __threadfence();
  __syncthreads();
  if (tid == 0) s_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  for (int j = tid; j < tot; j += NW * 32) {
    double a0 = 0.0, a1 = 0.0;
    int r = 0;
    for (; r + 1 < (int)gridDim.x; r += 2) {
      a0 += __ldcg(partials + (long long)r * tot + j);
      a1 += __ldcg(partials + (long long)(r + 1) * tot + j);
    }
    if (r < (int)gridDim.x) a0 += __ldcg(partials + (long long)r * tot + j);
    out[j] = a0 + a1;
  }
  if (tid == 0) ticket[0] = 0u;
}

// ---------------------------------------------------------------------------
// Exact second derivatives in the couplings from the column cache (masses
// and widths fixed).  With A_o = sum_k c_k F_ko, f = sum_o |A_o|^2 and
// G_k = sum_o conj(A_o) F_ko, the data term -sum w t(f) (t = clip_log) has
// second derivatives in the couplings built from
//   H1 = sum w t'(f) Q,  Q_lk = sum_o conj(F_lo) F_ko   (K x K Hermitian)
//   H2 = sum w t''(f) g g^T,  g = (Re G, -Im G)         (2K x 2K)
// and the gradient pieces S0 = sum w t(f), S1 = sum w t'(f) G; the host
// combines them with the derivatives of the column couplings and the MC
// Gram matrix (the reference obtains the same matrix by nested tapes,
// tf_pwa/model/model.py:513-561).  Both matrices are weighted sums of
// outer products of rows: H1 from X1 rows (helicity o, event e) =
// (Re F_.o, Im F_.o) with weight w t'(f) (Re Q = X_RR + X_II, Im Q = X_RI -
// X_IR), H2 from X2 rows (event e) = g with weight w t''(f).
//
// A block walks a contiguous run of 128-event tiles.  Per tile, thread e
// computes its event's A (FP64), f, t, t', t'' and G (FP32) and writes its
// rows of X1 and X2 to shared memory; then each thread accumulates its
// items -- (matrix, PWA_HBS x PWA_HBS block of the upper triangle, split s
// of the rows: every sp-th row from s) -- over the tile in FP32 and adds
// them to FP64 registers.  While it
// does, the next tile's columns of its own event are already on their way
// into a shared-memory stage (per-thread cp.async of 8-byte values, the
// tile's own layout), so the loads overlap the outer products.  The
// block row of partials is [S0, S1 (re, im per column), H1 upper entries,
// H2 upper entries] (upper entry (p, q), p <= q, at p W - p (p - 1) / 2 +
// q - p); rows of several splits of one block are added in split order, so
// the result does not depend on scheduling.
#define PWA_HW (2 * PWA_NCOL)
#define PWA_HBS (PWA_HW % 4 == 0 ? 4 : 2)
#define PWA_HNB (PWA_HW / PWA_HBS)
#define PWA_HUP (PWA_HNB * (PWA_HNB + 1) / 2)
#define PWA_HTRI (PWA_HW * (PWA_HW + 1) / 2)
#define PWA_HNA (1 + PWA_HW + 2 * PWA_HTRI)
// row splits: X1 has PWA_NOUT times the rows of X2, so it gets PWA_NOUT
// times the splits and every item walks about the same number of rows
#define PWA_HSP2 (PWA_HUP * (PWA_NOUT + 1) >= PWA_TPB ? 1 : PWA_TPB / (PWA_HUP * (PWA_NOUT + 1)))
#define PWA_HSP1 (PWA_HSP2 * PWA_NOUT)
#define PWA_HN1 (PWA_HUP * PWA_HSP1)
#define PWA_HITEMS (PWA_HN1 + PWA_HUP * PWA_HSP2)
#define PWA_HIPT ((PWA_HITEMS + PWA_TPB - 1) / PWA_TPB)
// row stride of X1 / X2 in floats: a multiple of 4 (16-byte rows, float4
// stores) that is 4 mod 8, so eight consecutive rows start in eight
// different bank quads (conflict-free 16-byte stores of consecutive events)
#define PWA_HLD4 ((PWA_HW + 3) / 4 * 4)
#define PWA_HLD (PWA_HLD4 % 8 == 0 ? PWA_HLD4 + 4 : PWA_HLD4)

__device__ __forceinline__ int hess_upper(int p, int q) {
  return p * PWA_HW - p * (p - 1) / 2 + (q - p);
}

// one row of W values (zero-padded to PWA_HLD4) as 16-byte stores
__device__ __forceinline__ void hess_store_row(float* dst, const float (&row)[PWA_HLD4]) {
#pragma unroll
  for (int q = 0; q < PWA_HLD4 / 4; ++q)
    *(float4*)(dst + 4 * q) = make_float4(row[4 * q], row[4 * q + 1], row[4 * q + 2], row[4 * q + 3]);
}

#ifndef PWA_HESS_MINB
#define PWA_HESS_MINB 3
#endif
// 1: the next tile is staged by cp.async while the outer products run (the
// host reserves the stage when the model source defines this to 1)
#ifndef PWA_HESS_STAGE
#define PWA_HESS_STAGE 0
#endif
extern "C" __global__ void __launch_bounds__(PWA_TPB, PWA_HESS_MINB)
    pwa_hess_cached(const CCoup c, const float2* __restrict__ Fc,
                    const double* __restrict__ Wc, long long ntiles,
                    double* __restrict__ partials) {
  constexpr int K = PWA_NCOL, W = PWA_HW, BS = PWA_HBS, LD = PWA_HLD;
  constexpr int R1 = PWA_NOUT * PWA_TPB;
  // rows region (X1, X2; the final row buffer reuses it), then s1, s2 and
  // the stage of the next tile
  constexpr unsigned ROWS_B = (R1 + PWA_TPB) * LD * 4;
  constexpr unsigned NA_B = (PWA_HNA * 8 + 15) / 16 * 16;
  constexpr unsigned REG_B = ROWS_B > NA_B ? ROWS_B : NA_B;
  extern __shared__ __align__(16) unsigned char hess_smem[];
  float* X1 = (float*)hess_smem;                                          // [R1][LD]
  float* X2 = X1 + R1 * LD;                                               // [TPB][LD]
  float* s1 = (float*)(hess_smem + REG_B);                                // [TPB]
  float* s2 = s1 + PWA_TPB;                                               // [TPB]
  float2* stF = (float2*)(s2 + PWA_TPB);                                  // [NF][TPB]
  double* stW = (double*)(stF + PWA_NF * PWA_TPB);                        // [TPB]
  double* row_acc = (double*)hess_smem;  // [PWA_HNA], over X1 / X2 after the last tile
  __shared__ double s_c[2 * PWA_NCOL];
  __shared__ double s_red[PWA_TPB / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  stage_couplings(c, s_c);
  __syncthreads();
  // this thread's items (matrix, split, upper block bi <= bj), ordered so
  // that neighbouring threads share the matrix and the rows
  int it_m[PWA_HIPT], it_s[PWA_HIPT], it_bi[PWA_HIPT], it_bj[PWA_HIPT];
  double hacc[PWA_HIPT][BS][BS];
#pragma unroll
  for (int q = 0; q < PWA_HIPT; ++q) {
    const int it = tid + q * PWA_TPB;
    const int m = it < PWA_HN1 ? 0 : 1, r = it < PWA_HN1 ? it : it - PWA_HN1;
    int blk = r % PWA_HUP, bi = 0;
    while (blk >= PWA_HNB - bi) blk -= PWA_HNB - bi++;
    it_m[q] = it < PWA_HITEMS ? m : -1;
    it_s[q] = r / PWA_HUP;
    it_bi[q] = bi;
    it_bj[q] = bi + blk;
#pragma unroll
    for (int i = 0; i < BS; ++i)
#pragma unroll
      for (int j = 0; j < BS; ++j) hacc[q][i][j] = 0.0;
  }
  // S1 as in the evaluation kernels: each event's w t'(f) G (entries 2k,
  // 2k + 1 = re, im of column k) reduce-scattered across the warp in FP32,
  // the lane's entries accumulated in FP64
  double acc_s0 = 0.0, acc_s1[PWA_MG];
#pragma unroll
  for (int q = 0; q < PWA_MG; ++q) acc_s1[q] = 0.0;
  const long long B = gridDim.x, b = blockIdx.x;
  const long long t0 = b * ntiles / B, t1 = (b + 1) * ntiles / B;
#if PWA_HESS_STAGE
  auto stage = [&](long long t) {  // this thread's event of tile t -> stage
    const float2* F = Fc + t * PWA_NF * PWA_TPB + tid;
#pragma unroll
    for (int j = 0; j < PWA_NF; ++j) cp_async8(stF + j * PWA_TPB + tid, F + j * PWA_TPB);
    cp_async8(stW + tid, Wc + t * PWA_TPB + tid);
    cp_async_commit();
  };
  if (t0 < t1) stage(t0);
#endif
#pragma unroll 1
  for (long long t = t0; t < t1; ++t) {
    {  // this thread's event: amplitude, clip_log derivatives, G, rows
      float2 v[PWA_NF];
#if PWA_HESS_STAGE
      cp_async_wait_all();
#pragma unroll
      for (int j = 0; j < PWA_NF; ++j) v[j] = stF[j * PWA_TPB + tid];
      const double w = stW[tid];
#else
      const float2* F = Fc + t * PWA_NF * PWA_TPB + tid;
#pragma unroll
      for (int j = 0; j < PWA_NF; ++j) v[j] = __ldcs(F + j * PWA_TPB);
      const double w = __ldcs(Wc + t * PWA_TPB + tid);
#endif
      double ar[PWA_NOUT], ai[PWA_NOUT];
#pragma unroll
      for (int o = 0; o < PWA_NOUT; ++o) ar[o] = ai[o] = 0.0;
#pragma unroll
      for (int j = 0; j < PWA_NF; ++j) {
        const int k = pwa_fk[j], o = pwa_fo[j];
        const double cr = s_c[2 * k], ci = s_c[2 * k + 1];
        ar[o] = fma(cr, (double)v[j].x, fma(-ci, (double)v[j].y, ar[o]));
        ai[o] = fma(cr, (double)v[j].y, fma(ci, (double)v[j].x, ai[o]));
      }
      double f = 0.0;
#pragma unroll
      for (int o = 0; o < PWA_NOUT; ++o) f = fma(ar[o], ar[o], fma(ai[o], ai[o], f));
      double d1;
      const double cl = clip_log(f, &d1);
      const double d2 = f > 1e-6 ? -d1 * d1 : -1e12;  // clip_log'': -1/eps^2 below eps
      acc_s0 = fma(w, cl, acc_s0);
      float row[PWA_HLD4];
#pragma unroll
      for (int q = 0; q < PWA_HLD4; ++q) row[q] = 0.f;
#pragma unroll
      for (int j = 0; j < PWA_NF; ++j) {  // X2 row: (Re G, -Im G)
        const int k = pwa_fk[j], o = pwa_fo[j];
        const float xr = (float)ar[o], xi = (float)ai[o];
        row[k] = fmaf(xr, v[j].x, fmaf(xi, v[j].y, row[k]));
        row[K + k] = fmaf(xi, v[j].x, fmaf(-xr, v[j].y, row[K + k]));
      }
      hess_store_row(X2 + tid * LD, row);
      {
        const float f1 = (float)(w * d1);
#if PWA_RS16
        float gq[16];
#pragma unroll
        for (int q = 0; q < 16; ++q)
          gq[q] = q < W ? ((q & 1) ? -f1 * row[K + (q >> 1)] : f1 * row[q >> 1]) : 0.f;
        warp_rs_step<16, 16, 16>(gq, lane);
        acc_s1[0] += (double)(gq[0] + __shfl_xor_sync(0xffffffffu, gq[0], 1));
#else
#pragma unroll
        for (int m = 0; m < PWA_GPAD / 32; ++m) {
          float gq[32];
#pragma unroll
          for (int q = 0; q < 32; ++q) {
            const int e = 32 * m + q;
            gq[q] = e < W ? ((e & 1) ? -f1 * row[K + (e >> 1)] : f1 * row[e >> 1]) : 0.f;
          }
          warp_reduce_scatter<32>(gq, lane);
          acc_s1[m] += (double)gq[0];
        }
#endif
      }
#pragma unroll
      for (int o = 0; o < PWA_NOUT; ++o) {  // X1 rows: (Re F_.o, Im F_.o)
#pragma unroll
        for (int q = 0; q < PWA_HLD4; ++q) row[q] = 0.f;
#pragma unroll
        for (int j = 0; j < PWA_NF; ++j)
          if (pwa_fo[j] == o) {
            row[pwa_fk[j]] = v[j].x;
            row[K + pwa_fk[j]] = v[j].y;
          }
        hess_store_row(X1 + (o * PWA_TPB + tid) * LD, row);
      }
      s1[tid] = (float)(w * d1);
      s2[tid] = (float)(w * d2);
    }
    __syncthreads();
#if PWA_HESS_STAGE
    if (t + 1 < t1) stage(t + 1);  // this thread's stage slots are read
#endif
#pragma unroll
    for (int q = 0; q < PWA_HIPT; ++q) {
      if (it_m[q] < 0) continue;
      const float* X = it_m[q] == 0 ? X1 : X2;
      const float* sw = it_m[q] == 0 ? s1 : s2;
      // split s takes rows s, s + sp, s + 2 sp, ...: the splits sharing a
      // warp read neighbouring rows, which start in different bank quads
      const int R = it_m[q] == 0 ? R1 : PWA_TPB, sp = it_m[q] == 0 ? PWA_HSP1 : PWA_HSP2;
      const int cp = it_bi[q] * BS, cq = it_bj[q] * BS;
      float a[BS][BS];
#pragma unroll
      for (int i = 0; i < BS; ++i)
#pragma unroll
        for (int j = 0; j < BS; ++j) a[i][j] = 0.f;
#pragma unroll 4
      for (int r = it_s[q]; r < R; r += sp) {
        const float* x = X + r * LD;
        const float sc = sw[r % PWA_TPB];
        float xp[BS], xq[BS];
#pragma unroll
        for (int i = 0; i < BS; ++i) {
          xp[i] = sc * x[cp + i];
          xq[i] = x[cq + i];
        }
#pragma unroll
        for (int i = 0; i < BS; ++i)
#pragma unroll
          for (int j = 0; j < BS; ++j) a[i][j] = fmaf(xp[i], xq[j], a[i][j]);
      }
#pragma unroll
      for (int i = 0; i < BS; ++i)
#pragma unroll
        for (int j = 0; j < BS; ++j) hacc[q][i][j] += (double)a[i][j];
    }
    __syncthreads();
  }
  // the block row: S0, S1, then the items' blocks added in split order
  for (int j = tid; j < PWA_HNA; j += PWA_TPB) row_acc[j] = 0.0;
  const double v0 = warp_sum(acc_s0);
  if (lane == 0) s_red[warp] = v0;
  __syncthreads();
  if (tid == 0) {
    double a = 0.0;
#pragma unroll
    for (int w2 = 0; w2 < PWA_TPB / 32; ++w2) a += s_red[w2];
    row_acc[0] = a;
  }
  for (int w2 = 0; w2 < PWA_TPB / 32; ++w2) {  // the warps' S1 entries in warp order
    __syncthreads();
    if (warp == w2) {
#pragma unroll
      for (int m = 0; m < PWA_MG; ++m) {
        const int idx = rs_entry(m, lane);
        if (rs_owner(lane) && idx < W) row_acc[1 + idx] += acc_s1[m];
      }
    }
  }
  for (int spl = 0; spl < PWA_HSP1; ++spl) {
    __syncthreads();
#pragma unroll
    for (int q = 0; q < PWA_HIPT; ++q) {
      if (it_m[q] < 0 || it_s[q] != spl) continue;
      double* dst = row_acc + 1 + W + it_m[q] * PWA_HTRI;
#pragma unroll
      for (int i = 0; i < BS; ++i)
#pragma unroll
        for (int j = 0; j < BS; ++j) {
          const int p = it_bi[q] * BS + i, pq = it_bj[q] * BS + j;
          if (p <= pq) dst[hess_upper(p, pq)] += hacc[q][i][j];
        }
    }
  }
  __syncthreads();
  for (int j = tid; j < PWA_HNA; j += PWA_TPB)
    partials[(long long)blockIdx.x * PWA_HNA + j] = row_acc[j];
}

// ---------------------------------------------------------------------------
// Many fits in one launch (serving).  Each fit's data-event column cache is a
// run of tiles in a shared pool (same tile layout as above).  The launch gets
// a work list of (request, pool tile) pairs covering the tiles of every fit
// with a pending evaluation; each block evaluates work tiles with that
// request's couplings and writes one row of per-tile sums.  pwa_reduce_multi
// then sums each request's rows in the fit's own tile order, so a fit's
// result does not depend on which other fits share the launch.  Per-tile
// column sums use the warp reduce-scatter of pwa_eval_cached_wred.
extern "C" __global__ void __launch_bounds__(PWA_TPB, PWA_WRED_MINB)
    pwa_eval_multi(const double* __restrict__ ck, const int* __restrict__ work_req,
                   const long long* __restrict__ work_tile, long long n_work,
                   const float2* __restrict__ Fc, const double* __restrict__ Wc,
                   double* __restrict__ tile_part) {
  constexpr int NA = PWA_CACHE_NA;
  constexpr int NG = 2 * PWA_NCOL;
  __shared__ double red[PWA_TPB / 32][NA];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (long long wi = blockIdx.x; wi < n_work; wi += gridDim.x) {
    const int r = work_req[wi];
    const long long t = work_tile[wi];
    const CoupGlobal cp{ck + (long long)r * 2 * PWA_NCOL};
    const float2* F = Fc + t * PWA_NF * PWA_TPB + tid;
    float2 v[PWA_NF];
#pragma unroll
    for (int j = 0; j < PWA_NF; ++j) v[j] = __ldcs(F + j * PWA_TPB);
    const double w = __ldcs(Wc + t * PWA_TPB + tid);
    float gs[PWA_MG];
    const double s0 = warp_sum(cached_event_rs(v, w, cp, lane, gs));
    if (lane == 0) red[warp][0] = s0;
#pragma unroll
    for (int m = 0; m < PWA_MG; ++m) {
      const int idx = rs_entry(m, lane);
      if (rs_owner(lane) && idx < NG) red[warp][1 + idx] = (double)gs[m];
    }
    __syncthreads();
    for (int j = tid; j < NA; j += PWA_TPB) {
      double s = 0.0;
#pragma unroll
      for (int w2 = 0; w2 < PWA_TPB / 32; ++w2) s += red[w2][j];
      tile_part[wi * NA + j] = s;
    }
    __syncthreads();
  }
}

// out[r * NA + j] = sum over rows [row_beg[r], row_beg[r+1]) of tile_part,
// in row order (one warp per (request, accumulator), lanes strided, fixed
// shuffle tree).
extern "C" __global__ void pwa_reduce_multi(const double* __restrict__ tile_part,
                                            const long long* __restrict__ row_beg, int n_req,
                                            double* __restrict__ out) {
  constexpr int NA = PWA_CACHE_NA;
  const int lane = threadIdx.x & 31;
  const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long q = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
       q < (long long)n_req * NA; q += warps) {
    const int r = (int)(q / NA), j = (int)(q % NA);
    double s = 0.0;
    for (long long row = row_beg[r] + lane; row < row_beg[r + 1]; row += 32) s += tile_part[row * NA + j];
    s = warp_sum(s);
    if (lane == 0) out[q] = s;
  }
}

// ---------------------------------------------------------------------------
// Dataset step on the device (model_kin / model_genbod are generated per
// model).  One event per thread, grid-stride, FP64.
//
// pwa_fields_from_p4: final-state momenta, rows (4 f + c) of P4 with stride
// ld_in (c = E, px, py, pz; finals in dat_order; parent rest frame) -> every
// plan field, row j of OUT with stride ld_out (plan order).
extern "C" __global__ void __launch_bounds__(PWA_TPB)
    pwa_fields_from_p4(const double* __restrict__ P4, long long n, long long ld_in,
                       double* __restrict__ out, long long ld_out) {
  for (long long i = (long long)blockIdx.x * PWA_TPB + threadIdx.x; i < n;
       i += (long long)gridDim.x * PWA_TPB) {
    LV P[PWA_NFIN];
#pragma unroll
    for (int f = 0; f < PWA_NFIN; ++f)
      P[f] = LV{__ldg(P4 + (4LL * f) * ld_in + i), __ldg(P4 + (4LL * f + 1) * ld_in + i),
                __ldg(P4 + (4LL * f + 2) * ld_in + i), __ldg(P4 + (4LL * f + 3) * ld_in + i)};
    double F[PWA_NFIELD];
    model_kin(P, F);
#pragma unroll
    for (int j = 0; j < PWA_NFIELD; ++j) out[(long long)j * ld_out + i] = F[j];
  }
}

// Toy selection.  Candidate event e = first + i is drawn from the Philox
// stream (seed, e): a GENBOD phase-space event accepted with probability
// weight / max weight; for signal (flat = 0) its fields are formed in shared
// memory and sum |A|^2 evaluated (FP64); with fmax > 0 the candidate is kept
// if u fmax < sum |A|^2 (the accept-reject of tf_pwa/applications.py:
// 428-453).  out[i] = sum |A|^2 of a kept signal candidate, 1 for a kept
// flat one, -1 otherwise.  fmax <= 0 applies the phase-space step only
// (a first pass that finds the maximum).
extern "C" __global__ void __launch_bounds__(PWA_TPB)
    pwa_toy_select(const Consts C, unsigned long long seed, long long first, long long n,
                   double fmax, int flat, double* __restrict__ out) {
  extern __shared__ double sfield[];  // [PWA_NFIELD][PWA_TPB]: XM rows, then XA rows
  constexpr int NM = PWA_NFIELD_MASS;
  double* sXM = sfield;
  double* sXA = sfield + NM * PWA_TPB;
  const int tid = threadIdx.x;
  for (long long i = (long long)blockIdx.x * PWA_TPB + tid; i < n;
       i += (long long)gridDim.x * PWA_TPB) {
    double U[PWA_NDRAW];
    event_uniforms(seed, (unsigned long long)(first + i), U);
    LV P[PWA_NFIN];
    const double wps = model_genbod(U, P);
    double res = -1.0;
    if (U[PWA_NDRAW - 2] < wps) {
      if (flat) {
        res = 1.0;
      } else {
        double F[PWA_NFIELD];
        model_kin(P, F);
#pragma unroll
        for (int j = 0; j < PWA_NFIELD; ++j)
          (pwa_field_mass[j] ? sXM : sXA)[pwa_field_slot[j] * PWA_TPB + tid] = F[j];
        cpx<double> A[PWA_NOUT];
        model_amp<double, false, false>(C, sXA, sXM, PWA_TPB, tid, A, nullptr);
        const double f = model_f<double>(C, A);
        res = (fmax <= 0.0 || U[PWA_NDRAW - 1] * fmax < f) ? f : -1.0;
      }
    }
    out[i] = res;
  }
}

// Fields (and optionally momenta) of selected candidates, regenerated from
// their event numbers idx[i]: row j of OUT (stride ld_out) in plan order,
// P4 rows (4 f + c) with stride ld_p4 when P4 is not null.
extern "C" __global__ void __launch_bounds__(PWA_TPB)
    pwa_toy_fields(unsigned long long seed, const long long* __restrict__ idx, long long n,
                   double* __restrict__ out, long long ld_out, double* __restrict__ P4,
                   long long ld_p4) {
  for (long long i = (long long)blockIdx.x * PWA_TPB + threadIdx.x; i < n;
       i += (long long)gridDim.x * PWA_TPB) {
    double U[PWA_NDRAW];
    event_uniforms(seed, (unsigned long long)__ldg(idx + i), U);
    LV P[PWA_NFIN];
    model_genbod(U, P);
    double F[PWA_NFIELD];
    model_kin(P, F);
#pragma unroll
    for (int j = 0; j < PWA_NFIELD; ++j) out[(long long)j * ld_out + i] = F[j];
    if (P4) {
#pragma unroll
      for (int f = 0; f < PWA_NFIN; ++f) {
        P4[(4LL * f) * ld_p4 + i] = P[f].t;
        P4[(4LL * f + 1) * ld_p4 + i] = P[f].x;
        P4[(4LL * f + 2) * ld_p4 + i] = P[f].y;
        P4[(4LL * f + 3) * ld_p4 + i] = P[f].z;
      }
    }
  }
}
