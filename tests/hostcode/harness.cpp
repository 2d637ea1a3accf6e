// Host loops around the generated model functions, one event at a time,
// mirroring the per-event bodies of the CUDA kernels:
//   hx_sums     -- pwa_eval_f64 / pwa_eval_f32 (forward, clip_log or MC
//                  weight, adjoint with or without the stash), summed in
//                  event order
//   hx_amp      -- model_amp: the PWA_NOUT helicity amplitudes per event
//   hx_columns  -- model_columns: the PWA_NCOL x PWA_NOUT column values
//   hx_kin      -- pwa_fields_from_p4: momenta -> plan fields
//   hx_toy      -- pwa_toy_select / pwa_toy_fields: Philox uniforms,
//                  GENBOD, kinematics and sum |A|^2 of candidate events
// This file is appended to the device header and the generated model source
// (after the shim) and compiled with g++ by the tests.
#include <vector>

template <typename R, bool STASH>
static void sums_t(const Consts& C, const R* XA, const double* XM, const double* W,
                   long long beg, long long end, long long ld, bool is_data, double* acc) {
  for (int j = 0; j < PWA_NACC; ++j) acc[j] = 0.0;
  R st[PWA_NSTASH > 0 ? PWA_NSTASH : 1];
  for (long long i = beg; i < end; ++i) {
    cpx<R> A[PWA_NOUT];
    model_amp<R, STASH, false>(C, XA, XM, ld, i, A, st);
    const double f = model_f<R>(C, A);
    const double w = W[i];
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
    if (STASH)
      model_adj_stash<R, false>(C, XA, XM, ld, i, Ab, acc + 1, acc + 1 + 2 * PWA_NCOL, st);
    else
      model_adj_recompute<R, false>(C, XA, XM, ld, i, Ab, acc + 1, acc + 1 + 2 * PWA_NCOL);
  }
}

// out[0 .. PWA_NACC): data sums, out[PWA_NACC .. 2 PWA_NACC): MC sums.
// XA holds FP64 angles; with f32 != 0 they are rounded to FP32 first (the
// FP32-recompute form stores its angle fields as FP32).
// the constant block as the library packs it: FP64 values, then each
// one's FP32 rounding and the FP32 rounding of the rest
static void fill_consts(Consts& C, const double* Cv) {
  for (int j = 0; j < PWA_NCONST; ++j) {
    C.v[j] = Cv[j];
    C.h[j] = (float)Cv[j];
    C.l[j] = (float)(Cv[j] - (double)C.h[j]);
  }
}

extern "C" int hx_sums(const double* Cv, const double* XM, const double* XA, const double* W,
                       long long n_data, long long n_all, long long ld, int f32, int stash,
                       double* out) {
  Consts C;
  fill_consts(C, Cv);
  if (f32) {
    std::vector<float> xa((size_t)PWA_NANGLE_ROWS * ld);
    for (size_t j = 0; j < xa.size(); ++j) xa[j] = (float)XA[j];
    if (stash) {
      sums_t<float, true>(C, xa.data(), XM, W, 0, n_data, ld, true, out);
      sums_t<float, true>(C, xa.data(), XM, W, n_data, n_all, ld, false, out + PWA_NACC);
    } else {
      sums_t<float, false>(C, xa.data(), XM, W, 0, n_data, ld, true, out);
      sums_t<float, false>(C, xa.data(), XM, W, n_data, n_all, ld, false, out + PWA_NACC);
    }
  } else if (stash) {
    sums_t<double, true>(C, XA, XM, W, 0, n_data, ld, true, out);
    sums_t<double, true>(C, XA, XM, W, n_data, n_all, ld, false, out + PWA_NACC);
  } else {
    sums_t<double, false>(C, XA, XM, W, 0, n_data, ld, true, out);
    sums_t<double, false>(C, XA, XM, W, n_data, n_all, ld, false, out + PWA_NACC);
  }
  return PWA_NACC;
}

template <typename R>
static void amp_t(const Consts& C, const R* XA, const double* XM, long long n, long long ld,
                  double* out) {
  for (long long i = 0; i < n; ++i) {
    cpx<R> A[PWA_NOUT];
    model_amp<R, false, false>(C, XA, XM, ld, i, A, nullptr);
    for (int o = 0; o < PWA_NOUT; ++o) {
      out[2 * (i * PWA_NOUT + o)] = double(A[o].re);
      out[2 * (i * PWA_NOUT + o) + 1] = double(A[o].im);
    }
  }
}

// A[i * PWA_NOUT + o] as (re, im) pairs; f32 != 0: the FP32 form (angles
// rounded to FP32, amplitude arithmetic in FP32)
extern "C" int hx_amp(const double* Cv, const double* XM, const double* XA, long long n,
                      long long ld, int f32, double* out) {
  Consts C;
  fill_consts(C, Cv);
  if (f32) {
    std::vector<float> xa((size_t)PWA_NANGLE_ROWS * ld);
    for (size_t j = 0; j < xa.size(); ++j) xa[j] = (float)XA[j];
    amp_t<float>(C, xa.data(), XM, n, ld, out);
  } else {
    amp_t<double>(C, XA, XM, n, ld, out);
  }
  return PWA_NOUT;
}

// F[(i * PWA_NCOL + k) * PWA_NOUT + o] as (re, im) pairs
extern "C" int hx_columns(const double* Cv, const double* XM, const double* XA, long long n,
                          long long ld, double* out) {
  Consts C;
  fill_consts(C, Cv);
  for (long long i = 0; i < n; ++i) {
    cpx<double> F[PWA_NCOL * PWA_NOUT];
    model_columns<double, false>(C, XA, XM, ld, i, F);
    for (int j = 0; j < PWA_NCOL * PWA_NOUT; ++j) {
      out[2 * (i * PWA_NCOL * PWA_NOUT + j)] = F[j].re;
      out[2 * (i * PWA_NCOL * PWA_NOUT + j) + 1] = F[j].im;
    }
  }
  return PWA_NCOL;
}

// columns without their chains' lineshapes, layout of hx_columns
extern "C" int hx_columns_ns(const double* Cv, const double* XM, const double* XA, long long n,
                             long long ld, double* out) {
  Consts C;
  fill_consts(C, Cv);
  for (long long i = 0; i < n; ++i) {
    cpx<double> F[PWA_NCOL * PWA_NOUT];
    model_columns_ns<double, false>(C, XA, XM, ld, i, F);
    for (int j = 0; j < PWA_NCOL * PWA_NOUT; ++j) {
      out[2 * (i * PWA_NCOL * PWA_NOUT + j)] = F[j].re;
      out[2 * (i * PWA_NCOL * PWA_NOUT + j) + 1] = F[j].im;
    }
  }
  return PWA_NCOL;
}

// per event: chain lineshape products BW[PWA_NCHAIN], then the log-derivative
// factors DM, DG [PWA_NSRES] of each floating lineshape, as (re, im) pairs
extern "C" int hx_shapes(const double* Cv, const double* XM, long long n, long long ld,
                         double* out) {
  Consts C;
  fill_consts(C, Cv);
  constexpr int NS = PWA_NSRES > 0 ? PWA_NSRES : 1, W = PWA_NCHAIN + 2 * NS;
  for (long long i = 0; i < n; ++i) {
    cpx<double> BW[PWA_NCHAIN], DM[NS], DG[NS];
    for (int q = 0; q < NS; ++q) DM[q] = DG[q] = cmk<double>(0.0, 0.0);
    model_shapes<double, false>(C, XM, ld, i, BW, DM, DG);
    double* o = out + 2 * i * W;
    for (int c = 0; c < PWA_NCHAIN; ++c) o[2 * c] = BW[c].re, o[2 * c + 1] = BW[c].im;
    for (int q = 0; q < NS; ++q) {
      o[2 * (PWA_NCHAIN + q)] = DM[q].re, o[2 * (PWA_NCHAIN + q) + 1] = DM[q].im;
      o[2 * (PWA_NCHAIN + NS + q)] = DG[q].re, o[2 * (PWA_NCHAIN + NS + q) + 1] = DG[q].im;
    }
  }
  return W;
}

// P4 rows (4 f + c), stride n -> fields rows j (plan order), stride n
extern "C" int hx_kin(const double* P4, long long n, double* out) {
  for (long long i = 0; i < n; ++i) {
    LV P[PWA_NFIN];
    for (int f = 0; f < PWA_NFIN; ++f)
      P[f] = LV{P4[(4LL * f) * n + i], P4[(4LL * f + 1) * n + i], P4[(4LL * f + 2) * n + i],
                P4[(4LL * f + 3) * n + i]};
    double F[PWA_NFIELD];
    model_kin(P, F);
    for (int j = 0; j < PWA_NFIELD; ++j) out[(long long)j * n + i] = F[j];
  }
  return PWA_NFIELD;
}

#if PWA_HAS_GENBOD
// candidates first .. first + n - 1 of (seed): phase-space weight, the two
// acceptance uniforms, sum |A|^2 (FP64) and the momenta (rows 4 f + c,
// stride n) and fields (rows j, stride n)
extern "C" int hx_toy(const double* Cv, unsigned long long seed, long long first, long long n,
                      double* wps, double* u_ps, double* u_amp, double* f_out, double* P4,
                      double* fields) {
  Consts C;
  fill_consts(C, Cv);
  for (long long i = 0; i < n; ++i) {
    double U[PWA_NDRAW];
    event_uniforms(seed, (unsigned long long)(first + i), U);
    LV P[PWA_NFIN];
    wps[i] = model_genbod(U, P);
    u_ps[i] = U[PWA_NDRAW - 2];
    u_amp[i] = U[PWA_NDRAW - 1];
    double F[PWA_NFIELD];
    model_kin(P, F);
    double sXM[PWA_NFIELD_MASS > 0 ? PWA_NFIELD_MASS : 1];
    double sXA[PWA_NFIELD];
    for (int j = 0; j < PWA_NFIELD; ++j) {
      (pwa_field_mass[j] ? sXM : sXA)[pwa_field_slot[j]] = F[j];
      fields[(long long)j * n + i] = F[j];
    }
    cpx<double> A[PWA_NOUT];
    model_amp<double, false, false>(C, sXA, sXM, 1, 0, A, nullptr);
    f_out[i] = model_f<double>(C, A);
    for (int fi = 0; fi < PWA_NFIN; ++fi) {
      P4[(4LL * fi) * n + i] = P[fi].t;
      P4[(4LL * fi + 1) * n + i] = P[fi].x;
      P4[(4LL * fi + 2) * n + i] = P[fi].y;
      P4[(4LL * fi + 3) * n + i] = P[fi].z;
    }
  }
  return PWA_NDRAW;
}
#endif
