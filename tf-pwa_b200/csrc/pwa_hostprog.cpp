// Host program of one model (pwa_hostprog.h): the constant block, the
// Jacobian of the column couplings and the chain rule in native code.
//
// The formulas follow the engine's Python host code line for line, with the
// same order of operations, so that the constant block agrees with it to
// rounding: rel_p / rel_p2 (tf_pwa/amp/core.py:311-334), the
// Blatt-Weisskopf polynomials of tf_pwa/breit_wigner.py:319-390 evaluated by
// Horner's rule, the lineshape constants of BW (K = m0 Gamma0), BWR
// (K = m0^2 Gamma0 B(q0) / q0^(2L+1), q0 clamped at threshold) and BWR2
// (K = m0^2 Gamma0 B(q0^2), q0^2 unclamped; tf_pwa/breit_wigner.py:56-91,
// 193-265,280-306).  Derivatives in a mass are taken by a complex step of
// 1e-20 (exact to rounding: no difference is formed).
#include "pwa_hostprog.h"

#include <cmath>

namespace pwa_host {
namespace {

using cd = std::complex<double>;
constexpr double kStep = 1e-20;

inline double re(double x) { return x; }
inline double re(const cd& x) { return x.real(); }
inline double im(double) { return 0.0; }
inline double im(const cd& x) { return x.imag(); }

// x^n for a small integer n >= 0: the C library's pow for reals, binary
// powering (products from the low bit up) for complex numbers
inline double ipow(double x, int n) { return std::pow(x, (double)n); }
inline cd ipow(const cd& x, int n) {
  cd r(1.0, 0.0), p = x;
  for (unsigned m = 1; m > 0 && (unsigned)n >= m; m <<= 1) {
    if (n & m) r = r * p;
    p = p * p;
  }
  return r;
}

template <class T>
T rel_p2(T m0, T m1, T m2) {
  const T s = m1 + m2, d = m1 - m2;
  return (m0 - s) * (m0 + s) * (m0 - d) * (m0 + d) / ipow(2.0 * m0, 2);
}

template <class T>
T rel_p(T m0, T m1, T m2) {
  const T s = m1 + m2, d = m1 - m2;
  const T me = re(m0) > re(s) ? m0 : s;
  const T p = (me - s) * (me + s) * (me - d) * (me + d);
  return std::sqrt(p) / (2.0 * me);
}

template <class T>
T horner(const std::vector<double>& coef, T z) {
  T r = T(0.0);
  for (double c : coef) r = r * z + c;
  return r;
}

// 1 / |q0^2|^(l/2); for a complex q0^2, 1 / sqrt(q0^2 q0^2)^(l/2)
inline double inv_norm(double q02, int l) { return 1.0 / std::pow(std::fabs(q02), l / 2.0); }
inline cd inv_norm(const cd& q02, int l) {
  const cd a = std::sqrt(q02 * q02);
  const cd p = (l % 2 == 0) ? ipow(a, l / 2) : std::pow(a, l / 2.0);
  return 1.0 / p;
}

template <class T>
void entry_values(T q02, double d, const pwa_hostprog::VEntry& e, T* pz, T* nrm) {
  const T z = q02 * d * d;
  *pz = e.bp ? horner(e.coef, z) : T(1.0);
  *nrm = e.bn ? inv_norm(q02, e.l) : T(1.0);
}

template <class T>
T vertex_q02(const std::vector<T>& M, const pwa_hostprog::VRow& r) {
  if (r.noq0) return T(1.0);
  return rel_p2(M[r.ia], M[r.ib], M[r.ic]);
}

// (K, useq, q0^2) of one lineshape at parent mass m0
template <class T>
void row_values(const pwa_hostprog::LRow& r, T m0, double g0, T mb, T mc, T* K, double* useq,
                T* q02) {
  *useq = 1.0;
  *q02 = T(0.0);
  if (r.kind == 0) {  // BW
    *K = m0 * g0;
    return;
  }
  if (r.kind == 2) {  // BWR2
    *q02 = rel_p2(m0, mb, mc);
    const T z = *q02 * r.d * r.d;
    *K = m0 * m0 * g0 * horner(r.coef, z);
    return;
  }
  const T q0 = rel_p(m0, mb, mc);  // BWR
  const T z = ipow(q0 * r.d, 2);
  const T b = horner(r.coef, z);
  if (re(q0) > 1e-15) {
    *K = m0 * m0 * g0 * b / ipow(q0, 2 * r.L + 1);
  } else {
    *K = m0 * m0 * g0 * b;
    *useq = 0.0;
  }
}

void mass_list(const pwa_hostprog* p, const double* vars, std::vector<double>* M) {
  *M = p->m_base;
  for (size_t i = 0; i < M->size(); ++i)
    if (p->m_var[i] >= 0) (*M)[i] = vars[p->m_var[i]];
}

// Lineshape and barrier constants into C (the rest of C untouched) and the
// barrier rows of every resonance mass.
void shape_part(pwa_hostprog* p, const double* vars, double* C) {
  std::vector<double> M;
  mass_list(p, vars, &M);
  for (const auto& r : p->vt) {
    const double q02 = vertex_q02(M, r);
    for (const auto& e : r.e) {
      double pz, nrm;
      entry_values(q02, r.d, e, &pz, &nrm);
      if (e.s_pz >= 0) C[e.s_pz] = pz;
      if (e.s_norm >= 0) C[e.s_norm] = nrm;
    }
  }
  for (const auto& r : p->ls) {
    const double m0 = M[r.im], mb = M[r.ib], mc = M[r.ic];
    const double g0 = r.g_var >= 0 ? vars[r.g_var] : r.g_def;
    C[r.s_m0sq] = m0 * m0;
    double K, useq, q02;
    row_values(r, m0, g0, mb, mc, &K, &useq, &q02);
    if (r.kind == 1) {
      C[r.s_k] = K;
      C[r.s_useq] = useq;
    } else if (r.kind == 2) {
      C[r.s_k] = K;
      C[r.s_iq] = 1.0 / q02;
    } else {
      C[r.s_y] = K;
    }
    if (r.s_wn >= 0) C[r.s_wn] = g0;
    if (r.s_kap >= 0) {
      // kappa = d ln(m0 Gamma) / d m0; for BWR2 m0 Gamma2 = K r^(L+1/2) / (m B)
      // gives d ln K - (L + 1/2) d ln q0^2
      cd Kc, qc;
      double uc;
      row_values(r, cd(m0, kStep), g0, cd(mb), cd(mc), &Kc, &uc, &qc);
      double kap = K != 0.0 ? Kc.imag() / kStep / K : 0.0;
      if (r.kind == 2) kap -= (r.L + 0.5) * qc.imag() / kStep / q02;
      C[r.s_kap] = kap;
      C[r.s_ig] = g0 != 0.0 ? 1.0 / g0 : 0.0;
    }
  }
  // barrier rows: d ln(bf_l) / dm with bf_l ~ sqrt(Pz0_l) norm_l per vertex
  // entry, summed over each column's entries
  p->kap.assign(p->mj.size(), std::vector<double>(p->ncol, 0.0));
  for (size_t q = 0; q < p->mj.size(); ++q) {
    const auto& mj = p->mj[q];
    std::vector<cd> Mc(M.begin(), M.end());
    Mc[mj.qi] = cd(M[mj.qi], kStep);
    std::vector<std::vector<double>> dlog(p->vt.size());
    for (int v : mj.verts) {
      const auto& r = p->vt[v];
      const double q0r = vertex_q02(M, r);
      const cd q0c = vertex_q02(Mc, r);
      dlog[v].resize(r.e.size());
      for (size_t j = 0; j < r.e.size(); ++j) {
        double pz0, n0;
        cd pzc, nc;
        entry_values(q0r, r.d, r.e[j], &pz0, &n0);
        entry_values(q0c, r.d, r.e[j], &pzc, &nc);
        double t = 0.0;
        if (r.e[j].bp) t += 0.5 * pzc.imag() / kStep / pz0;
        if (r.e[j].bn) t += nc.imag() / kStep / n0;
        dlog[v][j] = t;
      }
    }
    for (size_t c = 0; c < mj.c_col.size(); ++c)
      p->kap[q][mj.c_col[c]] += dlog[mj.c_row[c]][mj.c_ent[c]];
  }
}

// the cursor of parse(): bounds-checked reads of the two arrays
struct Reader {
  const int* ip;
  long long n_ip, i = 0;
  const double* dp;
  long long n_dp, j = 0;
  bool ok = true;
  int next() {
    if (i >= n_ip) {
      ok = false;
      return 0;
    }
    return ip[i++];
  }
  double dnext() {
    if (j >= n_dp) {
      ok = false;
      return 0.0;
    }
    return dp[j++];
  }
  // a non-negative count of at most cap, and of at most the ints left (every
  // counted item reads at least one), so a malformed program cannot make
  // parse() allocate more than its own size
  int count(int cap) {
    const int n = next();
    if (n < 0 || n > cap || n > n_ip - i) ok = false;
    return ok ? n : 0;
  }
  int value(int cap) {  // a non-negative size of at most cap (not a list length)
    const int n = next();
    if (n < 0 || n > cap) ok = false;
    return ok ? n : 0;
  }
};

}  // namespace

bool parse(const int* ip, long long n_ip, const double* dp, long long n_dp, pwa_hostprog* p,
           std::string* err) {
  Reader rd{ip, n_ip, 0, dp, n_dp};
  constexpr int kMagic = 0x50574850, kVersion = 2, kCap = 1 << 20;
  auto fail = [&](const std::string& m) {
    *err = "host program: " + m;
    return false;
  };
  if (!ip || n_ip <= 0 || (n_dp > 0 && !dp)) return fail("empty program");
  if (rd.next() != kMagic || rd.next() != kVersion) return fail("bad magic or version");
  p->ncol = rd.value(kCap);
  p->nconst = rd.value(kCap);
  p->nshape = rd.value(kCap);
  p->n_vars = rd.value(kCap);
  p->n_train = rd.value(kCap);
  p->n_coup = rd.value(kCap);
  p->nfac = rd.value(64);
  if (!rd.ok || p->ncol <= 0 || p->nconst < 2 * p->ncol || p->n_coup <= 0 || p->nfac <= 0)
    return fail("bad header");
  auto ints = [&](std::vector<int>* v, long long n) {
    if (n < 0 || n > rd.n_ip - rd.i) {
      rd.ok = false;
      n = 0;
    }
    v->resize(n);
    for (long long q = 0; q < n; ++q) (*v)[q] = rd.next();
  };
  ints(&p->coup_r, p->n_coup);
  ints(&p->coup_i, p->n_coup);
  ints(&p->coup_polar, p->n_coup);
  ints(&p->col_fac, (long long)p->ncol * p->nfac);
  ints(&p->train_idx, p->n_train);
  const int n_vg = rd.count(kCap);
  p->vg_src.resize(n_vg);
  p->vg_re.resize(n_vg);
  p->vg_im.resize(n_vg);
  for (int q = 0; q < n_vg; ++q) {
    p->vg_src[q] = rd.next();
    p->vg_re[q] = rd.next();
    p->vg_im[q] = rd.next();
  }
  const int n_m = rd.count(kCap);
  ints(&p->m_var, n_m);
  p->m_base.resize(n_m);
  for (int q = 0; q < n_m; ++q) p->m_base[q] = rd.dnext();
  const int n_vt = rd.count(kCap);
  p->vt.assign(n_vt, {});
  for (auto& r : p->vt) {
    r.ia = rd.next();
    r.ib = rd.next();
    r.ic = rd.next();
    r.noq0 = rd.next();
    r.e.resize(rd.count(64));
    r.d = rd.dnext();
    for (auto& e : r.e) {
      e.l = rd.next();
      e.bp = rd.next();
      e.bn = rd.next();
      e.s_pz = rd.next();
      e.s_norm = rd.next();
      e.coef.resize(rd.value(64));  // doubles: not a count of ints
      for (auto& c : e.coef) c = rd.dnext();
    }
  }
  const int n_ls = rd.count(kCap);
  p->ls.assign(n_ls, {});
  for (auto& r : p->ls) {
    r.kind = rd.next();
    r.im = rd.next();
    r.ib = rd.next();
    r.ic = rd.next();
    r.L = rd.next();
    r.g_var = rd.next();
    r.s_m0sq = rd.next();
    r.s_k = rd.next();
    r.s_useq = rd.next();
    r.s_y = rd.next();
    r.s_iq = rd.next();
    r.s_wn = rd.next();
    r.s_kap = rd.next();
    r.s_ig = rd.next();
    r.coef.resize(rd.value(64));
    r.d = rd.dnext();
    r.g_def = rd.dnext();
    for (auto& c : r.coef) c = rd.dnext();
  }
  const int n_sel = rd.count(kCap);
  p->sel_var.resize(n_sel);
  p->sel_slot.resize(n_sel);
  for (int q = 0; q < n_sel; ++q) {
    p->sel_var[q] = rd.next();
    p->sel_slot[q] = rd.next();
  }
  const int n_mj = rd.count(kCap);
  p->mj.assign(n_mj, {});
  for (auto& m : p->mj) {
    m.var = rd.next();
    m.qi = rd.next();
    ints(&m.verts, rd.count(kCap));
    const int nc = rd.count(kCap);
    m.c_col.resize(nc);
    m.c_row.resize(nc);
    m.c_ent.resize(nc);
    for (int q = 0; q < nc; ++q) {
      m.c_col[q] = rd.next();
      m.c_row[q] = rd.next();
      m.c_ent[q] = rd.next();
    }
  }
  const int n_rt = rd.count(kCap);
  p->rt_col.resize(n_rt);
  p->rt_slot.resize(n_rt);
  p->rt_sqrt.resize(n_rt);
  for (int q = 0; q < n_rt; ++q) {
    p->rt_col[q] = rd.next();
    p->rt_slot[q] = rd.next();
    p->rt_sqrt[q] = rd.next();
  }
  p->n_rho = rd.count(64 * 64);
  ints(&p->rho_re, p->n_rho);
  ints(&p->rho_im, p->n_rho);
  p->pol_off = rd.next();
  ints(&p->pol_var, rd.count(kCap));
  p->rho0.resize(2 * p->n_rho);
  for (auto& x : p->rho0) x = rd.dnext();
  p->rho_g.assign(p->pol_var.size(), std::vector<double>(2 * p->n_rho));
  for (auto& g : p->rho_g)
    for (auto& x : g) x = rd.dnext();
  const int n_cp = rd.count(kCap);
  p->cp_coup.resize(n_cp);
  p->cp_dr.resize(n_cp);
  p->cp_di.resize(n_cp);
  p->cp_t_re.resize(n_cp);
  p->cp_t_im.resize(n_cp);
  for (int q = 0; q < n_cp; ++q) {
    p->cp_coup[q] = rd.next();
    p->cp_dr[q] = rd.next();
    p->cp_di[q] = rd.next();
    p->cp_t_re[q] = rd.next();
    p->cp_t_im[q] = rd.next();
  }
  const int n_cpc = rd.count(kCap);
  p->cp_col.resize(n_cpc);
  p->cp_c_re.resize(n_cpc);
  p->cp_c_im.resize(n_cpc);
  for (int q = 0; q < n_cpc; ++q) {
    p->cp_col[q] = rd.next();
    p->cp_c_re[q] = rd.next();
    p->cp_c_im[q] = rd.next();
  }
  p->cp_off = rd.next();
  if (rd.next() != kMagic || !rd.ok) return fail("truncated program");
  if (rd.i != n_ip || rd.j != n_dp) return fail("trailing entries");

  // ranges of every index
  const int V = p->n_vars, S = p->nconst, K = p->ncol;
  auto in = [](int x, int lo, int hi) { return x >= lo && x < hi; };
  auto slot = [&](int x) { return x == -1 || in(x, 0, S); };
  for (int q = 0; q < p->n_coup; ++q)
    if (!in(p->coup_r[q], 0, V) || !in(p->coup_i[q], 0, V)) return fail("coupling index");
  for (int x : p->col_fac)
    if (!in(x, -1, p->n_coup)) return fail("column factor index");
  for (int x : p->train_idx)
    if (!in(x, 0, V)) return fail("trainable index");
  for (int q = 0; q < n_vg; ++q)
    if (!in(p->vg_src[q], 0, p->n_coup) || !in(p->vg_re[q], 0, S) || !in(p->vg_im[q], 0, S))
      return fail("vertex coupling slot");
  for (int x : p->m_var)
    if (!in(x, -1, V)) return fail("mass variable index");
  for (const auto& r : p->vt) {
    if (!in(r.ia, 0, n_m) || !in(r.ib, 0, n_m) || !in(r.ic, 0, n_m)) return fail("vertex mass");
    for (const auto& e : r.e)
      if (!slot(e.s_pz) || !slot(e.s_norm) || e.l < 0) return fail("vertex entry");
  }
  for (const auto& r : p->ls) {
    if (!in(r.kind, 0, 3) || !in(r.im, 0, n_m) || !in(r.ib, 0, n_m) || !in(r.ic, 0, n_m) ||
        !in(r.g_var, -1, V) || !in(r.s_m0sq, 0, S) || !slot(r.s_k) || !slot(r.s_useq) ||
        !slot(r.s_y) || !slot(r.s_iq) || !slot(r.s_wn) || !slot(r.s_kap) || !slot(r.s_ig) ||
        r.L < 0)
      return fail("lineshape row");
    if ((r.kind == 1 && (r.s_k < 0 || r.s_useq < 0)) || (r.kind == 2 && (r.s_k < 0 || r.s_iq < 0)) ||
        (r.kind == 0 && r.s_y < 0) || ((r.s_kap < 0) != (r.s_ig < 0)))
      return fail("lineshape slots");
  }
  for (int q = 0; q < n_sel; ++q)
    if (!in(p->sel_var[q], 0, V) || !in(p->sel_slot[q], 0, p->nshape)) return fail("selector");
  for (const auto& m : p->mj) {
    if (!in(m.var, 0, V) || !in(m.qi, 0, n_m)) return fail("barrier row");
    for (int v : m.verts)
      if (!in(v, 0, n_vt)) return fail("barrier row vertex");
    for (size_t q = 0; q < m.c_col.size(); ++q) {
      if (!in(m.c_col[q], 0, K) || !in(m.c_row[q], 0, n_vt) ||
          !in(m.c_ent[q], 0, (int)p->vt[m.c_row[q]].e.size()))
        return fail("barrier row entry");
      bool listed = false;
      for (int v : m.verts) listed |= v == m.c_row[q];
      if (!listed) return fail("barrier row entry outside its vertices");
    }
  }
  for (int q = 0; q < n_rt; ++q)
    if (!in(p->rt_col[q], 0, K) || !in(p->rt_slot[q], 0, S)) return fail("normalisation term");
  for (int e = 0; e < p->n_rho; ++e)
    if (!in(p->rho_re[e], 0, S) || !in(p->rho_im[e], 0, S)) return fail("density matrix slot");
  if (p->n_rho && (p->pol_off < 0 || p->pol_off + 2 * p->n_rho > p->nshape))
    return fail("polarisation sums outside the extra sums");
  for (int v : p->pol_var)
    if (!in(v, 0, V) || !p->n_rho) return fail("polarisation variable");
  for (int q = 0; q < n_cp; ++q)
    if (!in(p->cp_coup[q], 0, p->n_coup) || !in(p->cp_dr[q], 0, V) || !in(p->cp_di[q], 0, V) ||
        !in(p->cp_t_re[q], 0, S) || !in(p->cp_t_im[q], 0, S))
      return fail("CP total");
  for (int q = 0; q < n_cpc; ++q)
    if (!in(p->cp_col[q], 0, K) || !in(p->cp_c_re[q], 0, S) || !in(p->cp_c_im[q], 0, S))
      return fail("CP column");
  if (p->cp_off != -1 && (p->cp_off < 0 || p->cp_off + 2 * n_cpc > p->nshape))
    return fail("charge -1 sums outside the extra sums");

  // roles of the trainable variables and the inputs of the shape part
  p->coup_cp.assign(p->n_coup, -1);
  for (int q = 0; q < n_cp; ++q) p->coup_cp[p->cp_coup[q]] = q;
  p->t_coup.assign(p->n_train, -1);
  p->t_comp.assign(p->n_train, 0);
  p->t_sel.assign(p->n_train, -1);
  p->t_mj.assign(p->n_train, -1);
  p->t_pol.assign(p->n_train, -1);
  for (int t = 0; t < p->n_train; ++t) {
    const int v = p->train_idx[t];
    for (int q = 0; q < p->n_coup && p->t_coup[t] < 0; ++q) {
      if (p->coup_r[q] == v) p->t_coup[t] = q, p->t_comp[t] = 0;
      else if (p->coup_i[q] == v) p->t_coup[t] = q, p->t_comp[t] = 1;
    }
    for (int q = 0; q < n_cp && p->t_coup[t] < 0; ++q) {
      if (p->cp_dr[q] == v) p->t_coup[t] = p->cp_coup[q], p->t_comp[t] = 2;
      else if (p->cp_di[q] == v) p->t_coup[t] = p->cp_coup[q], p->t_comp[t] = 3;
    }
    for (size_t q = 0; q < p->pol_var.size(); ++q)
      if (p->pol_var[q] == v) p->t_pol[t] = (int)q;
    for (int q = 0; q < n_sel; ++q)
      if (p->sel_var[q] == v) p->t_sel[t] = p->sel_slot[q];
    for (int q = 0; q < n_mj; ++q)
      if (p->mj[q].var == v) p->t_mj[t] = q;
  }
  p->key_var.clear();
  auto add_key = [&](int v) {
    if (v < 0) return;
    for (int x : p->key_var)
      if (x == v) return;
    p->key_var.push_back(v);
  };
  for (int x : p->m_var) add_key(x);
  for (const auto& r : p->ls) add_key(r.g_var);
  p->have_shape = false;
  return true;
}

void consts(pwa_hostprog* p, const double* vars, double* C, std::vector<cd>* z,
            std::vector<double>* ck) {
  // shape part: recomputed when a mass or width it reads changed
  bool same = p->have_shape && p->key.size() == p->key_var.size();
  for (size_t q = 0; same && q < p->key_var.size(); ++q) same = p->key[q] == vars[p->key_var[q]];
  if (!same) {
    p->cshape.assign(p->nconst, 0.0);
    shape_part(p, vars, p->cshape.data());
    p->key.resize(p->key_var.size());
    for (size_t q = 0; q < p->key_var.size(); ++q) p->key[q] = vars[p->key_var[q]];
    p->have_shape = true;
  }
  for (int q = 0; q < p->nconst; ++q) C[q] = p->cshape[q];
  // couplings: r e^{i phi} (polar) or r + i phi, columns their products;
  // a CP total at (r + dr, i + di), its charge -1 value at (r - dr, i - di)
  auto value = [](int polar, double r, double ph) {
    return polar ? cd(r * std::cos(ph), r * std::sin(ph)) : cd(r, ph);
  };
  z->resize(p->n_coup);
  p->zm.resize(p->n_coup);
  for (int j = 0; j < p->n_coup; ++j) {
    double r = vars[p->coup_r[j]], ph = vars[p->coup_i[j]];
    const int q = p->coup_cp[j];
    if (q >= 0) {
      const double dr = vars[p->cp_dr[q]], di = vars[p->cp_di[q]];
      p->zm[j] = value(p->coup_polar[j], r - dr, ph - di);
      r += dr;
      ph += di;
      (*z)[j] = value(p->coup_polar[j], r, ph);
    } else {
      (*z)[j] = p->zm[j] = value(p->coup_polar[j], r, ph);
    }
  }
  auto column = [&](int k, const std::vector<cd>& zz) {
    cd c(1.0, 0.0);
    for (int f = 0; f < p->nfac; ++f) {
      const int j = p->col_fac[k * p->nfac + f];
      if (j >= 0) c = c * zz[j];
    }
    return c;
  };
  ck->resize(2 * p->ncol);
  for (int k = 0; k < p->ncol; ++k) {
    const cd c = column(k, *z);
    (*ck)[2 * k] = C[2 * k] = c.real();
    (*ck)[2 * k + 1] = C[2 * k + 1] = c.imag();
  }
  for (size_t q = 0; q < p->vg_src.size(); ++q) {
    C[p->vg_re[q]] = (*z)[p->vg_src[q]].real();
    C[p->vg_im[q]] = (*z)[p->vg_src[q]].imag();
  }
  for (size_t q = 0; q < p->cp_coup.size(); ++q) {
    C[p->cp_t_re[q]] = p->zm[p->cp_coup[q]].real();
    C[p->cp_t_im[q]] = p->zm[p->cp_coup[q]].imag();
  }
  p->ckm.resize(2 * p->cp_col.size());
  for (size_t q = 0; q < p->cp_col.size(); ++q) {
    const cd c = column(p->cp_col[q], p->zm);
    p->ckm[2 * q] = C[p->cp_c_re[q]] = c.real();
    p->ckm[2 * q + 1] = C[p->cp_c_im[q]] = c.imag();
  }
  // parent density matrix, linear in the polarisation variables
  for (int e = 0; e < p->n_rho; ++e) {
    cd r(p->rho0[2 * e], p->rho0[2 * e + 1]);
    for (size_t q = 0; q < p->pol_var.size(); ++q)
      r += vars[p->pol_var[q]] * cd(p->rho_g[q][2 * e], p->rho_g[q][2 * e + 1]);
    C[p->rho_re[e]] = r.real();
    C[p->rho_im[e]] = r.imag();
  }
}

void jacobian(pwa_hostprog* p, const double* vars, const std::vector<cd>& z,
              const std::vector<double>& ck, cd* J, cd* Jm, double* D) {
  const int K = p->ncol, P = p->n_train, NS = p->nshape, NC = (int)p->cp_col.size();
  for (long long q = 0; q < (long long)P * K; ++q) J[q] = cd(0.0, 0.0);
  if (Jm)
    for (long long q = 0; q < (long long)P * NC; ++q) Jm[q] = cd(0.0, 0.0);
  for (long long q = 0; q < (long long)P * NS; ++q) D[q] = 0.0;
  // d(prod of column k's factors)/dz_j with the factors zz (each occurrence
  // of j in turn, the others kept), times dz
  auto prod_rule = [&](int k, int j, const std::vector<cd>& zz, cd dz) {
    int cnt = 0;
    cd others(1.0, 0.0);
    for (int f = 0; f < p->nfac; ++f) {
      const int q = p->col_fac[k * p->nfac + f];
      if (q < 0) continue;
      if (q == j && cnt++ == 0) continue;
      others = others * zz[q];
    }
    return cnt ? (double)cnt * others * dz : cd(0.0, 0.0);
  };
  for (int t = 0; t < P; ++t) {
    cd* Jt = J + (long long)t * K;
    cd* Jmt = Jm ? Jm + (long long)t * NC : nullptr;
    const int j = p->t_coup[t];
    if (j >= 0) {
      // z = a e^{i phi}: dz/da = e^{i phi}, dz/dphi = i z (polar); 1, i
      // (Cartesian); at the charge's own (a, phi); deltar / deltai enter
      // charge -1 with a minus sign
      const int role = p->t_comp[t], q = p->coup_cp[j];
      const bool is_i = role == 1 || role == 3;
      auto dz_at = [&](double ph, const cd& zv) {
        if (p->coup_polar[j]) return is_i ? cd(0.0, 1.0) * zv : cd(std::cos(ph), std::sin(ph));
        return is_i ? cd(0.0, 1.0) : cd(1.0, 0.0);
      };
      double ph_p = vars[p->coup_i[j]], ph_m = ph_p;
      if (q >= 0) {
        ph_p += vars[p->cp_di[q]];
        ph_m -= vars[p->cp_di[q]];
      }
      const cd dzp = dz_at(ph_p, z[j]);
      const cd dzm = (role >= 2 ? -1.0 : 1.0) * dz_at(ph_m, p->zm[j]);
      for (int k = 0; k < K; ++k) Jt[k] = prod_rule(k, j, z, dzp);
      if (Jmt)
        for (int c = 0; c < NC; ++c) Jmt[c] = prod_rule(p->cp_col[c], j, p->zm, dzm);
    }
    if (p->t_mj[t] >= 0) {
      const auto& kap = p->kap[p->t_mj[t]];
      for (int k = 0; k < K; ++k) Jt[k] += cd(ck[2 * k], ck[2 * k + 1]) * kap[k];
      if (Jmt)
        for (int c = 0; c < NC; ++c)
          Jmt[c] += cd(p->ckm[2 * c], p->ckm[2 * c + 1]) * kap[p->cp_col[c]];
    }
    double* Dt = D + (long long)t * NS;
    if (p->t_sel[t] >= 0) Dt[p->t_sel[t]] = 1.0;
    if (p->t_pol[t] >= 0) {
      // d f / d p = Re sum_e T_e G_e with the kernels' T sums as (re, im):
      // Re(T G) = T.re G.re - T.im G.im
      const auto& g = p->rho_g[p->t_pol[t]];
      for (int e = 0; e < p->n_rho; ++e) {
        Dt[p->pol_off + 2 * e] = g[2 * e];
        Dt[p->pol_off + 2 * e + 1] = -g[2 * e + 1];
      }
    }
  }
}

void grad_from_sums(const pwa_hostprog* p, const cd* J, const cd* Jm, const double* D,
                    const double* s, double* g) {
  const int K = p->ncol, NS = p->nshape, NC = (int)p->cp_col.size();
  for (int t = 0; t < p->n_train; ++t) {
    const cd* Jt = J + (long long)t * K;
    double acc = 0.0;
    for (int k = 0; k < K; ++k) acc += Jt[k].real() * s[1 + 2 * k] - Jt[k].imag() * s[2 + 2 * k];
    if (Jm && p->cp_off >= 0) {
      // charge -1 column sums of the CP columns
      const cd* Jmt = Jm + (long long)t * NC;
      const double* sm = s + 1 + 2 * K + p->cp_off;
      for (int c = 0; c < NC; ++c) acc += Jmt[c].real() * sm[2 * c] - Jmt[c].imag() * sm[2 * c + 1];
    }
    acc *= 2.0;
    for (int q = 0; q < NS; ++q) acc += D[(long long)t * NS + q] * s[1 + 2 * K + q];
    g[t] = acc;
  }
}

bool column_rho(const pwa_hostprog* p, const double* C, double* rho) {
  for (int k = 0; k < p->ncol; ++k) rho[k] = 1.0;
  for (size_t q = 0; q < p->rt_col.size(); ++q) {
    const double v = C[p->rt_slot[q]];
    if (!(v > 0.0)) return false;
    rho[p->rt_col[q]] *= p->rt_sqrt[q] ? std::sqrt(v) : v;
  }
  return true;
}

}  // namespace pwa_host
