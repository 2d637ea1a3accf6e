/*
 * C ABI of the B200 amplitude-fit engine (libpwa_b200.so).
 *
 * The reference package (TF-PWA) is pure Python/TensorFlow and has no FFI of
 * its own; these entry points sit under the Python classes that replace the
 * reference's hot path, one for each piece of work that path does:
 *
 *   pwa_plan_create    compile a decay model          tf_pwa/amp/amp.py:43-64
 *                      (AbsPDF construction / init_params of the amplitude)
 *   pwa_upload_events  keep data + MC events resident  tf_pwa/model/model.py:1126-1164
 *                      (FCN.__init__: weights, batches, MC weights)
 *   pwa_eval           NLL + gradient sums             tf_pwa/model/model.py:407-449,1207-1229
 *                      (BaseModel.nll_grad_batch / FCN.nll_grad)
 *   pwa_eval_pdf       per-event sum |A|^2             tf_pwa/amp/amp.py:120-129
 *                      (AbsPDF.__call__ -> DecayGroup.sum_amp, core.py:1919-1931)
 *   pwa_build_gram     cached MC integral matrix       tf_pwa/model/opt_int.py:128-296
 *                      (ModelCachedInt.build_cached_int)
 *   pwa_fields_from_p4 momenta -> masses and angles    tf_pwa/cal_angle.py:262-490
 *                      (cal_angle_from_momentum at data load)
 *   pwa_toy_select /   flat phase space and toy        tf_pwa/phasespace.py:31-254,
 *   pwa_toy_fields     accept-reject on sum |A|^2      tf_pwa/applications.py:394-487
 *   pwa_hostprog_* /   constants, Jacobian, chain rule tf_pwa/model/model.py:407-449,1223-1229
 *   pwa_nll_grad_vars  from the variables (host side   tf_pwa/amp/core.py:349-418,1072-1104
 *                      of FCN.nll_grad)
 *   pwa_hessian_cached Hessian (differenced adjoint)   tf_pwa/model/model.py:513-561
 *   pwa_hessian_cached_exact  (closed form, one pass)  tf_pwa/model/model.py:513-561
 *   pwa_read_dat       text momentum files             tf_pwa/data.py:300-365
 *   pwa_server_*       many fits, each a BFGS driver   tf_pwa/fit.py:189-419 (one per fit)
 *   pwa_compile_only / pwa_precompile / pwa_last_error / pwa_plan_info / pwa_plan_destroy
 *                      build check and bookkeeping (no reference counterpart)
 *
 * Conventions: plain pointers and sizes only; every call returns 0 on success
 * or a PWA_ERR_* code, with a message in pwa_last_error().  Nothing throws
 * across the ABI.  Calls on one handle must not overlap; different handles
 * are independent.  `stream` is a cudaStream_t (0 = legacy default stream).
 */
#ifndef PWA_B200_H
#define PWA_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pwa_plan pwa_plan;
typedef struct pwa_server pwa_server;
typedef struct pwa_hostprog pwa_hostprog;

enum {
  PWA_OK = 0,
  PWA_ERR_ARG = 1,      /* invalid argument / size */
  PWA_ERR_COMPILE = 2,  /* NVRTC compilation or module load failed */
  PWA_ERR_CUDA = 3,     /* CUDA runtime error */
  PWA_ERR_STATE = 4,    /* call order (e.g. eval before upload) */
  PWA_ERR_OOM = 5       /* device allocation failed */
};

enum { PWA_PLAIN_F64 = 0, PWA_MIXED_F32 = 1 };

/* Compile a model.  `src` is the generated model source (model_event /
 * model_columns and the Consts layout); the library prepends its device
 * headers and compiles for sm_100a on the current device.
 * n_mass / n_angle: number of FP64 mass / angle columns of an event;
 * ncol, nout, nshape, nconst, nf: model sizes matching the source (nf =
 * structurally non-zero (column, helicity) pairs, PWA_NF of the source;
 * nshape = every accumulator past the 2*ncol column sums: lineshape,
 * polarisation and charge -1 column sums, so that 1 + 2*ncol + nshape equals
 * the source's PWA_NACC, else PWA_ERR_ARG).
 * tpb: threads per block of the fused kernels (32..1024, multiple of 32). */
int pwa_plan_create(const char* src, size_t src_len, int n_mass, int n_angle, int ncol, int nout,
                    int nshape, int nconst, int nf, int tpb, pwa_plan** out);

int pwa_plan_destroy(pwa_plan* h);

/* Compile the model module for `arch` (e.g. "sm_100a") without a device and
 * return the NVRTC/ptxas log (register and spill report) in log_buf.  Used
 * by the build step to check generated models on a machine without a GPU. */
int pwa_compile_only(const char* src, size_t src_len, int tpb, const char* arch, char* log_buf,
                     size_t log_len);

/* Compile the model module for `arch` without a device and store the cubin
 * in the on-disk cache (PWA_CUBIN_CACHE=<dir>), where pwa_plan_create on a
 * device of that architecture finds it instead of compiling: ahead-of-time
 * builds of known models.  PWA_ERR_STATE when the variable is not set;
 * NVRTC errors as PWA_ERR_COMPILE with the log in log_buf. */
int pwa_precompile(const char* src, size_t src_len, int tpb, const char* arch, char* log_buf,
                   size_t log_len);

/* Events: xm[n_mass][n_data+n_mc], xa[n_angle][n_data+n_mc], w[n_data+n_mc]
 * (row-major; data rows first, then MC).  Data weights are the final
 * (alpha-scaled) weights; MC weights are normalised to sum 1 by the caller.
 * `on_device` = 1 when the pointers are device memory. */
int pwa_upload_events(pwa_plan* h, const double* xm, const double* xa, const double* w,
                      long long n_data, long long n_mc, int on_device, void* stream);

/* One evaluation.  consts[nconst] per the model's Consts layout.
 * out[2*nacc] (host): data sums then MC sums, nacc = 1 + 2*ncol + nshape:
 *   [0] sum w clip_log(f) (data) / sum w f (MC)
 *   [1+2k], [2+2k]  Re/Im sum fac * G_k,   G_k = sum_o conj(A_o) F_k,o
 *   [1+2ncol+s]     sum fac * d f / d shape_s
 * fac = w * clip_log'(f) for data, w for MC.  precision: PWA_PLAIN_F64 or
 * PWA_MIXED_F32 (FP32 amplitudes, FP64 sums).  mc = 0 skips the MC set. */
int pwa_eval(pwa_plan* h, const double* consts, int precision, int mc, void* stream, double* out);

/* The device work of pwa_eval (fused kernel + fixed-order reduction) only,
 * enqueued on `stream` without waiting; the sums stay on the device.  For
 * timing the kernels and for capture into larger asynchronous pipelines. */
int pwa_eval_enqueue(pwa_plan* h, const double* consts, int precision, int mc, void* stream);

/* Per-event sum |A|^2 of events [beg, end) of the uploaded set into
 * out_dev (device, end-beg doubles). */
int pwa_eval_pdf(pwa_plan* h, const double* consts, int precision, long long beg, long long end,
                 double* out_dev, void* stream);

/* Dataset step on the device: final-state four-momenta -> every event field
 * of the model (invariant masses, helicity angles, alignment angles), as
 * tf_pwa/cal_angle.py:262-490 (cal_angle_from_momentum) computes them at
 * data-load time.  p4: device, rows (4 f + c) with stride ld_in (c = E, px,
 * py, pz; finals in dat_order; parent rest frame); out: device, one row per
 * field in plan order with stride ld_out.  Enqueued on `stream`. */
int pwa_fields_from_p4(pwa_plan* h, const double* p4, long long n, long long ld_in, double* out,
                       long long ld_out, void* stream);

/* Toy / MC generation on the device (tf_pwa/phasespace.py:31-254 flat phase
 * space; tf_pwa/applications.py:394-487 accept-reject on sum |A|^2).
 * Candidate e = first + i is drawn from a Philox4x32-10 stream keyed by
 * `seed`; out[i] (device, n doubles) = sum |A|^2 of a kept signal candidate
 * (flat = 0; kept when u * fmax < sum |A|^2, or when fmax <= 0 after the
 * phase-space step alone), 1 for a kept flat candidate (flat = 1; consts
 * may be null), -1 for a rejected one.  Enqueued on `stream`. */
int pwa_toy_select(pwa_plan* h, const double* consts, unsigned long long seed, long long first,
                   long long n, double fmax, int flat, double* out, void* stream);

/* Fields (out: rows in plan order, stride ld_out) and, if p4 is not null,
 * momenta (rows 4 f + c, stride ld_p4) of candidates idx[0..n) (device
 * event numbers as passed to pwa_toy_select), regenerated from the same
 * random stream.  Enqueued on `stream`. */
int pwa_toy_fields(pwa_plan* h, unsigned long long seed, const long long* idx, long long n,
                   double* out, long long ld_out, double* p4, long long ld_p4, void* stream);

/* ---- floating masses/widths: shape-free column cache -------------------
 * For models whose columns factorise as (lineshapes of the chain) x
 * (shape-free column) -- one pass, no polarised parent, no CP-violating
 * totals -- pwa_shape_cache computes, at the shape setting in consts, every
 * event's (data and MC) columns without their lineshapes (FP64, stored
 * FP32).  pwa_eval_shapecache then evaluates at any setting: lineshapes from
 * the resident masses, the column couplings times ratio[ncol] (each
 * column's barrier normalisations now over at the cache's setting), and
 * returns the sums of pwa_eval (out[2 * nacc]: data, MC), so the chain rule
 * of the plain form applies.  The reference recomputes the whole amplitude
 * per evaluation when shapes float (tf_pwa/model/model.py:407-449,
 * tf_pwa/amp/core.py:1392-1445); PWA_ERR_STATE for models that do not
 * factorise. */
int pwa_shape_cache(pwa_plan* h, const double* consts, void* stream);
int pwa_eval_shapecache(pwa_plan* h, const double* consts, const double* ratio, void* stream,
                        double* out);
/* The same launches without the copy back (results in device memory, for
 * timing or chaining on the stream). */
int pwa_eval_shapecache_enqueue(pwa_plan* h, const double* consts, const double* ratio,
                                void* stream);

/* Hessian of the cached-form NLL with respect to the trainable parameters
 * (tf_pwa/model/model.py:513-561, BaseModel.nll_grad_hessian; errors via
 * tf_pwa/applications.py:280-309): central 4-point differences of the
 * adjoint gradient, h_i = step * max(|x_i|, 1e-2), symmetrised; also the
 * NLL and gradient at vars.  out_hess: n_train x n_train, row-major.
 * Needs pwa_cache_data, pwa_build_gram and pwa_set_param_layout first. */
int pwa_hessian_cached(pwa_plan* h, const double* vars, double sum_w, double step, void* stream,
                       double* out_nll, double* out_grad, double* out_hess);

/* Exact Hessian of the cached-form NLL in the trainable coupling parts
 * (what tf_pwa/model/model.py:513-561 computes by nested GradientTape), in
 * one pass over the column cache: the kernel sums, over the data events,
 * S0 = sum w t(f), S1 = sum w t'(f) G, H1 = sum w t'(f) Q and
 * H2 = sum w t''(f) g g^T (t = clip_log, Q_lk = sum_o conj(F_lo) F_ko,
 * G_k = sum_o conj(A_o) F_ko, g = (Re G, -Im G)); the host adds the MC
 * term from the Gram matrix and applies the first and second derivatives
 * of the column couplings.  Also the NLL and gradient at vars.  out_hess:
 * n_train x n_train, row-major, symmetric.  Needs pwa_cache_data,
 * pwa_build_gram and pwa_set_param_layout first; every trainable variable
 * must be a coupling part (masses and widths fixed). */
int pwa_hessian_cached_exact(pwa_plan* h, const double* vars, double sum_w, void* stream,
                             double* out_nll, double* out_grad, double* out_hess);

/* The data sums of pwa_hessian_cached_exact at vars (host out, 1 + 2K +
 * 2K(2K + 1) doubles for K = ncol): S0, S1 (re, im per column), then the
 * upper triangles (p <= q, row-major) of the 2K x 2K sums
 * sum w t'(f) X X^T over rows X = (Re F_.o, Im F_.o) and sum w t''(f) g g^T.
 * Sums of event shards add (multi-GPU: all-reduce them). */
int pwa_hess_sums_cached(pwa_plan* h, const double* vars, void* stream, double* out);

/* Momentum file ingest (tf_pwa/data.py:300-365, load_dat_file): all
 * whitespace- or comma-separated numbers of a text file ('#' starts a
 * comment), parsed on all host cores, in file order, into out (host,
 * capacity cap); *n_values = their count.  With out = NULL only the count is
 * returned.  No plan handle: failures are reported by pwa_last_error(NULL). */
int pwa_read_dat(const char* path, double* out, long long cap, long long* n_values);

/* Gram matrix of the MC set, M_kl = sum_i w_i sum_o conj(F_ik,o) F_il,o,
 * to FP64 accuracy; out[2*ncol*ncol] host, (re, im) row-major. */
int pwa_build_gram(pwa_plan* h, const double* consts, void* stream, double* out);

/* How pwa_build_gram contracts the columns (tf_pwa/model/opt_int.py:128-296
 * builds the same matrix with a TF einsum): 0 = FP64 on the CUDA cores,
 * 1 = tensor cores (tcgen05 int8 MMAs on seven exact slices of every value,
 * exact int32 accumulation, FP64 recombination; models with at most 32
 * columns, others use 0), -1 = automatic (0: at the shipped models' column
 * counts the slicing costs more than the FP64 products it replaces).  The
 * error flag of the tensor-core kernel turns into PWA_ERR_CUDA. */
int pwa_set_gram_method(pwa_plan* h, int method);

/* ---- fixed masses/widths: cached partial-wave columns -------------------
 * The reference's cached-integral / cached-amplitude modes
 * (tf_pwa/model/opt_int.py:128-558) keep per-event amplitude factors while
 * masses and widths are fixed.  pwa_cache_data evaluates the columns
 * F_k,o of all data events once (FP64) and keeps them as FP32 complex;
 * pwa_build_gram (above) keeps the MC Gram matrix.  Each evaluation then
 * streams the column cache once with FP64 arithmetic. */
int pwa_cache_data(pwa_plan* h, const double* consts, void* stream);

/* Kernel used for the cached data term: 0 = shared-memory ring fed by bulk
 * copies, 1 = direct loads with four blocks per SM and per-thread FP64
 * column sums, 2 = direct loads with the column sums of each warp's 32
 * events reduce-scattered in FP32 before FP64 accumulation (register use
 * independent of the column count), 3 = shared-memory ring (two stages)
 * whose consumers read their columns from shared memory and reduce-scatter
 * the column sums, 4 = one block of 16 warps per SM, each warp a
 * contiguous run of events, single-level ordered reduction, 5 = one block
 * per SM with a producer warp keeping a deep ring of bulk copies in flight
 * for 8 consumer warps, -1 = automatic (default: 2). */
int pwa_set_cached_variant(pwa_plan* h, int variant);

/* Autotuner of the cached data-term kernel (no counterpart in the
 * reference, which has no kernels): times every configuration -- variant
 * 2 at each block count per SM the occupancy allows, variants 1 and 4,
 * variant 5 at every even ring depth from 4 stages to the shared-memory
 * limit (its two consumer groups need an even depth),
 * variants 0 and 3 -- with CUDA events around each of `reps` launches on
 * the plan's column cache and couplings ck, every launch after a write of
 * a 256 MB buffer (L2 flushed; the buffer is allocated for the call and
 * freed), and keeps the fastest.
 * out[i] = mean microseconds per launch of configuration i (at most 32),
 * *n_cand their count.  pwa_cached_config reads the configuration in use
 * (variant, ring depth, blocks per SM of variant 2); pwa_set_cached_config
 * sets one (0 = keep the default for that field). */
int pwa_autotune_cached(pwa_plan* h, const double* ck, int reps, void* stream, int* n_cand,
                        double* out);
int pwa_cached_config(pwa_plan* h, int* out);
int pwa_set_cached_config(pwa_plan* h, int variant, int stages, int bps);

/* Data-term kernels on the cache with column couplings ck[2*ncol]
 * (re, im); sums (1 + 2*ncol doubles) stay on the device. */
int pwa_eval_cached_enqueue(pwa_plan* h, const double* ck, void* stream);

/* Parameter layout for the C-side chain rule (fit parameter vector of
 * n_vars reals, tf_pwa/variable.py order): coupling j is the complex number
 * (vars[coup_r[j]], vars[coup_i[j]]), polar (r e^{i phi}) when
 * coup_polar[j]; column k is the product of couplings col_fac[k*nfac+f]
 * (-1 = unused slot); the gradient is taken w.r.t. vars[train_idx[t]]. */
int pwa_set_param_layout(pwa_plan* h, int n_vars, int n_coup, const int* coup_r,
                         const int* coup_i, const int* coup_polar, int nfac, const int* col_fac,
                         int n_train, const int* train_idx);

/* This device's NLL pieces from the cache + Gram: out[3 + 2*n_train] =
 * [S_data, S_mc*mc_share, sw, g_data[n_train], g_mc*mc_share[n_train]];
 * summing the vectors of several devices and forming
 * NLL = -S_d + sw ln S_m, grad = -g_d + sw g_m / S_m gives the NLL of the
 * union of their events (tf_pwa/model/model.py:433-449).  sw = sum of the
 * final data weights. */
int pwa_pieces_cached(pwa_plan* h, const double* vars, double sw, double mc_share, void* stream,
                      double* out);

/* NLL and gradient (FCN.nll_grad, tf_pwa/model/model.py:1223-1229) on one
 * device from the cache: vars[n_vars] in, *out_nll and out_grad[n_train]. */
/* Many parameter points in one pass over the column cache (the reference
 * evaluates each point of a Hessian stencil, line search or likelihood scan
 * separately, tf_pwa/model/model.py:513-561): vars holds n_pts rows of
 * n_vars values; out n_pts rows of the piece vector of pwa_pieces_cached.
 * Each warp holds its events' columns in registers and evaluates every
 * point on them with FP32 amplitudes and FP32 log (FP64 sums), so
 * gradients are good to ~1e-6 relative and the NLL to ~1e-4 absolute at
 * 1e6 events; pwa_hessian_cached uses it for its 4 n_train stencil
 * points.  Points beyond what one launch's shared memory holds (about 100
 * for 8 columns, 25 for 30) go in further launches. */
int pwa_pieces_points(pwa_plan* h, int n_pts, const double* vars, double sw, double mc_share,
                      void* stream, double* out);
int pwa_nll_grad_cached(pwa_plan* h, const double* vars, double sw, void* stream,
                        double* out_nll, double* out_grad);

/* ---- evaluations from the variable vector (host program) ---------------
 * The host side of one evaluation in native code: the reference builds the
 * couplings, lineshape and barrier constants from its variables and applies
 * the chain rule per evaluation (tf_pwa/model/model.py:407-449,
 * tf_pwa/amp/core.py:349-418,1072-1104, tf_pwa/variable.py:1715-1765).  A
 * host program holds, for one model and one variable layout, what that
 * takes; it needs no device and runs on the host alone.
 *
 * Format: ip (int) and dp (double) arrays read in order
 *   ip: 0x50574850, 2, ncol, nconst, nshape (all sums past the column
 *       sums, as pwa_plan_create), n_vars, n_train, n_coup, nfac,
 *       coup_r[n_coup], coup_i[n_coup], coup_polar[n_coup] (the couplings'
 *       variable indices, polar r e^{i phi} or r + i phi),
 *       col_fac[ncol*nfac] (column k = product of couplings, -1 unused),
 *       train_idx[n_train],
 *       n_vg, n_vg x (coupling, re slot, im slot) (vertex couplings and
 *       chain totals in the constant block),
 *       n_m, m_var[n_m] (variable of each listed mass, -1 fixed),
 *       n_vt, per vertex: ia, ib, ic (mass indices of a -> b c), no_q0,
 *         n_e, per entry: l, has_bprime, norm, Pz0 slot, norm slot, n_coef,
 *       n_ls, per lineshape: kind (0 BW, 1 BWR, 2 BWR2), m0, mb, mc (mass
 *         indices), L, width variable (-1 fixed), slots m0sq, K, useq, y,
 *         iq02, wn, kappa_m, inv_g0 (-1 absent), n_coef,
 *       n_sel, n_sel x (variable, shape sum) (d f / d variable through
 *         that sum of the kernels),
 *       n_mj, per resonance mass with barrier factors: variable, mass
 *         index, n_verts, verts[], n_c, n_c x (column, vertex, entry),
 *       n_rt, n_rt x (column, slot, sqrt) (barrier normalisations of each
 *         column),
 *       n_rho, rho_re[n_rho], rho_im[n_rho] (density matrix slots of a
 *         polarised parent, 0 entries otherwise), pol_off (its sums after
 *         the lineshape sums), n_pol, pol_var[n_pol],
 *       n_cp, n_cp x (coupling, deltar variable, deltai variable, charge -1
 *         re slot, im slot) (CP-violating totals),
 *       n_cpc, n_cpc x (column, charge -1 coupling re slot, im slot),
 *       cp_off (charge -1 column sums among the extra sums, -1 none),
 *       0x50574850
 *   dp: m_base[n_m] (masses of the fixed entries), per vertex d and per
 *       entry coef[n_coef] (B' polynomial, highest power first), per
 *       lineshape d, default width, coef[n_coef]; rho = rho0 + sum_q p_q G_q:
 *       rho0 and per polarisation variable G_q as n_rho (re, im) pairs.
 * PWA_ERR_ARG (message in pwa_last_error(NULL)) for a malformed program. */
int pwa_hostprog_create(const int* ip, long long n_ip, const double* dp, long long n_dp,
                        pwa_hostprog** out);
int pwa_hostprog_destroy(pwa_hostprog* p);
/* The constant block (nconst doubles) of the kernels at vars[n_vars]. */
int pwa_hostprog_consts(pwa_hostprog* p, const double* vars, double* out);
/* J[2*(t*ncol + k)] (re, im): d c_k / d vars[train_idx[t]];
 * Jm[2*(t*n_cpc + q)]: d c_q^- / d vars[train_idx[t]] of the CP columns'
 * charge -1 couplings (may be NULL when there are none);
 * D[t*nshape + j]: its selector of the kernels' extra sum j (lineshape
 * sums, then the parent-helicity products of a polarised parent). */
int pwa_hostprog_jacobian(pwa_hostprog* p, const double* vars, double* J, double* D,
                          double* Jm);
/* Piece vector (pwa_pieces_cached layout) from the kernels' data and MC
 * sums sd, sm (1 + 2*ncol + nshape each). */
int pwa_hostprog_pieces(pwa_hostprog* p, const double* vars, const double* sd, const double* sm,
                        double sw, double mc_share, double* out);
/* Each column's product of its barrier normalisations in a constant block
 * (PWA_ERR_ARG where one is not positive). */
int pwa_hostprog_column_rho(const pwa_hostprog* p, const double* consts, double* out);

enum { PWA_FORM_PLAIN_F64 = 0, PWA_FORM_MIXED_F32 = 1, PWA_FORM_SHAPE_CACHE = 2 };

/* A copy of p for this plan's evaluations (sizes must match the plan). */
int pwa_set_host_program(pwa_plan* h, const pwa_hostprog* p);
/* Piece vector of one evaluation at vars: constants and Jacobian from the
 * plan's host program, the kernels of `form` (FP64, FP32 amplitudes, or the
 * floating-shape column cache of pwa_shape_cache, which falls back to FP32
 * amplitudes at a point where a barrier normalisation is not positive), the
 * chain rule.  BaseModel.nll_grad_batch, tf_pwa/model/model.py:739-759. */
int pwa_pieces_vars(pwa_plan* h, const double* vars, int form, double sw, double mc_share,
                    void* stream, double* out);
/* NLL and gradient of one device's events (FCN.nll_grad,
 * tf_pwa/model/model.py:1223-1229). */
int pwa_nll_grad_vars(pwa_plan* h, const double* vars, int form, double sw, void* stream,
                      double* out_nll, double* out_grad);

/* ---- many concurrent fits (serving) ------------------------------------
 * A pool of column-cache tiles (PWA_TPB events each) holds the data events
 * of many fits at once; each fit owns one run of tiles.  The fits share the
 * model, the MC sample and therefore the Gram matrix built by
 * pwa_build_gram; each has its own couplings.  There is no counterpart in the
 * reference (which runs one fit per process); these calls serve the
 * reference's FCN.nll_grad for many fits in one launch. */
int pwa_pool_reserve(pwa_plan* h, long long n_tiles);
/* First-fit run of ceil(n_events / tile) tiles; PWA_ERR_OOM when no free run
 * is large enough (the caller's admission control waits and retries). */
int pwa_pool_alloc(pwa_plan* h, long long n_events, long long* first_tile, long long* n_tiles);
int pwa_pool_free(pwa_plan* h, long long first_tile);
/* Columns of a fit's n data events (device columns as pwa_upload_events,
 * leading dimension ld, final weights w) into its tile run. */
int pwa_pool_fill(pwa_plan* h, long long first_tile, const double* consts, const double* xm,
                  const double* xa, const double* w, long long n, long long ld, void* stream);
/* One launch for n_req pending evaluations: request r uses tiles
 * [first_tile[r], first_tile[r] + n_tiles[r]) and the parameter vector
 * vars[r * n_vars ...]; out[r * (3 + 2*n_train) ...] receives its piece
 * vector (see pwa_pieces_cached) with data weight sum sw[r].  A request's
 * result does not depend on the other requests in the launch. */
int pwa_pieces_multi(pwa_plan* h, int n_req, const long long* first_tile, const long long* n_tiles,
                     const double* vars, const double* sw, double mc_share, void* stream,
                     double* out);

/* Allocation-free variant of pwa_eval's device work (plain FP64 kernels),
 * with no counterpart in the reference.  For callers that cannot call
 * cudaMalloc while they run: a host framework that owns every device byte
 * through its own arena and forbids plug-ins from allocating, or a loop
 * that must not take the allocator's locks.  The caller passes device inputs xm
 * [n_mass][ld], xa [n_angle][ld], w [ld] (data rows first, then MC, same
 * meaning as pwa_upload_events) and a device output out[2*nacc] (data sums,
 * then MC sums, as pwa_eval).  Block partials live in a fixed device array
 * inside the library (1184 blocks x 256 accumulators of FP64, 2.4 MB held
 * by every GPU that loads the library until exit); models with more than
 * 256 accumulators are rejected with PWA_ERR_ARG.  Allocates nothing and
 * does not wait.  The first call on a device looks up the array's device
 * address; make that first call before any stream capture.  The address is
 * kept for the life of the process: a cudaDeviceReset in between is not
 * supported.  The current device must be the plan's (else PWA_ERR_STATE).
 * The array is built as sm_100a code: this call needs a compute capability
 * 10.0 GPU.  Calls share the array: calls that overlap on the GPU race. */
int pwa_eval_noalloc(pwa_plan* h, const double* consts, const double* xm, const double* xa,
                     const double* w, long long n_data, long long n_mc, long long ld,
                     double* out, void* stream);

/* Check of the failure detection of the cached evaluation, with no
 * counterpart in the reference (its fit loop reports a failed evaluation,
 * tf_pwa/fit.py:13-15,257-260).  mode 0 launches a one-block kernel whose
 * barrier wait gives up after `polls` polls (the bytes it waits for are
 * never sent; the one copy it did issue is drained before it exits) and
 * publishes the error flag as a stalled cached kernel would; mode 1
 * launches nothing, so the host's poll of the mapped result gives up after
 * host_limit_s seconds.  Returns what an evaluation would: PWA_ERR_CUDA
 * with "a barrier wait timed out" (mode 0) or "stale result" (mode 1) in
 * pwa_last_error.  The plan stays usable.  ticket memory (>= 1 KB) is the
 * copy's source. */
int pwa_wait_check(pwa_plan* h, int mode, unsigned polls, double host_limit_s, void* stream);

/* Peak FMA throughput of the CUDA cores (*out, flop/s), the roofline of the
 * compute-bound amplitude kernels (no counterpart in the reference):
 * precision PWA_PLAIN_F64 or PWA_MIXED_F32 (FP32 FMAs); 8 blocks of 256
 * threads per SM, each thread eight independent chains of `iters` (a
 * multiple of 4) FMAs, timed with CUDA events after one warm-up launch. */
int pwa_fma_peak(pwa_plan* h, int precision, long long iters, void* stream, double* out);

/* info[0..7]: registers/thread of eval_f64, eval_f32, local bytes f64, f32,
 * blocks, blocks_data, nacc, threads per block. */
int pwa_plan_info(pwa_plan* h, long long* info);

const char* pwa_last_error(pwa_plan* h);

/* Native fit server: many concurrent fits of one model (toy, pull and
 * significance studies, tf_pwa/fit.py:189-419 per fit) sharing the plan's
 * MC Gram matrix.  Each fit is a BFGS state machine (inverse-Hessian
 * update, backtracking Armijo line search; converged at max|g| < gtol,
 * stopped when a step lowers the NLL by less than 1e-14 relative, after 20
 * backtracks or at maxiter iterations); one scheduler thread admits fits into the plan's tile pool
 * (pwa_pool_reserve first) and evaluates the pending point of every active
 * fit in one multi-request launch per round.  base_vars: all variables
 * (fixed values); consts: the constant block for the column caches.  While
 * a server runs, no other thread may use its plan. */
int pwa_server_create(pwa_plan* h, const double* base_vars, const double* consts, int max_active,
                      double gtol, int maxiter, pwa_server** out);
/* Queue a fit: x0 = its trainable start values; xm, xa, w = its events'
 * mass/angle columns and weights on the device (stride ld), which must stay
 * valid until its result is final. */
int pwa_server_submit(pwa_server* s, const double* x0, const double* xm, const double* xa,
                      const double* w, long long n, long long ld, long long* fit_id);
/* Result of a fit (wait != 0: block until it is final).  status: 0 running,
 * 1 converged, 2 stopped (iteration limit or line search), 3 failed;
 * latency_s = finish - submission. */
int pwa_server_result(pwa_server* s, long long fit_id, int wait, int* status, double* x,
                      double* nll, int* n_eval, int* n_iter, double* latency_s);
/* out[5]: rounds (launches), requests, seconds inside the launches, active
 * fits, queued fits. */
int pwa_server_stats(pwa_server* s, double* out);
/* The service's own tuning of its multi-request launch (no counterpart in
 * the reference): its first rounds with at least 16 tiles per SM of work
 * try each block count per SM the occupancy allows (up to four), three
 * rounds each, timing seconds per work tile, and keep the fastest.
 * out[9]: [0] the block count chosen (0 while tuning), then per candidate
 * (block count, median seconds per tile). */
int pwa_server_tuning(pwa_server* s, double* out);
/* Stop the scheduler (unfinished fits end as failed) and free the server. */
int pwa_server_destroy(pwa_server* s);

#ifdef __cplusplus
}
#endif

#endif /* PWA_B200_H */
