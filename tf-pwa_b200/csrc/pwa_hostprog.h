// Host program of one model: everything an evaluation computes on the host
// from the fit-parameter vector, in native code.
//
//  * the constant block of the generated kernels: column couplings, vertex
//    couplings and chain totals (tf_pwa/variable.py:1715-1765,
//    tf_pwa/amp/core.py:764-773,1325-1329), barrier constants sqrt(P_l(q0^2
//    d^2)) and 1/|q0^2|^(l/2) per vertex (tf_pwa/amp/core.py:1072-1104,
//    tf_pwa/breit_wigner.py:268-277,332-355), lineshape constants of BW,
//    BWR and BWR2 (tf_pwa/breit_wigner.py:56-91,193-265,280-306) and the
//    mass derivative of ln(m0 Gamma(m)) by a complex step;
//  * the chain rule from the kernels' sums to the trainable variables
//    (tf_pwa/model/model.py:407-449): coupling rows by the product rule,
//    lineshape rows through the kernels' shape sums, barrier rows of a
//    resonance mass as d ln(prod of the column's barrier factors) / dm by a
//    complex step;
//  * the barrier-normalisation product of each column, the factor between
//    the floating-shape column cache's columns and the model's.
//
// The program is built once per model and variable layout (flat int and
// double arrays, format in include/pwa_b200.h) and holds a cache of the
// shape part keyed by the mass and width values it reads.
#pragma once

#include <complex>
#include <string>
#include <vector>

struct pwa_hostprog {
  struct VEntry {
    int l = 0, bp = 0, bn = 0, s_pz = -1, s_norm = -1;
    std::vector<double> coef;  // B' polynomial in z = q0^2 d^2, highest power first
  };
  struct VRow {
    int ia = 0, ib = 0, ic = 0, noq0 = 0;
    double d = 0.0;
    std::vector<VEntry> e;
  };
  struct LRow {
    int kind = 0, im = 0, ib = 0, ic = 0, L = 0, g_var = -1;
    int s_m0sq = -1, s_k = -1, s_useq = -1, s_y = -1, s_iq = -1, s_wn = -1, s_kap = -1,
        s_ig = -1;
    double d = 0.0, g_def = 0.0;
    std::vector<double> coef;
  };
  struct MJac {  // barrier rows of one resonance mass
    int var = 0, qi = 0;
    std::vector<int> verts;              // vertex rows it enters
    std::vector<int> c_col, c_row, c_ent;  // (column, vertex row, entry) summed per column
  };
  int ncol = 0, nconst = 0, nshape = 0, n_vars = 0, n_train = 0, n_coup = 0, nfac = 0;
  std::vector<int> coup_r, coup_i, coup_polar, col_fac, train_idx;
  std::vector<int> vg_src, vg_re, vg_im;
  std::vector<double> m_base;
  std::vector<int> m_var;
  std::vector<VRow> vt;
  std::vector<LRow> ls;
  std::vector<int> sel_var, sel_slot;
  std::vector<MJac> mj;
  std::vector<int> rt_col, rt_slot, rt_sqrt;
  // polarised parent: rho = rho0 + sum_q p_q G_q into the slots rho_re /
  // rho_im (n_rho entries); p_q acts through the kernels' parent-helicity
  // sums from pol_off on (d f / d p_q = Re sum_e T_e G_q,e)
  int n_rho = 0, pol_off = 0;
  std::vector<int> rho_re, rho_im, pol_var;
  std::vector<double> rho0;                 // (re, im) per entry
  std::vector<std::vector<double>> rho_g;   // per polarisation variable
  // CP-violating chain totals: charge +1 takes (r + dr, i + di), charge -1
  // (r - dr, i - di) (tf_pwa/variable.py:199-235); the minus-charge totals
  // and the CP columns' minus-charge couplings go to their slots, the
  // kernels' charge -1 column sums start at cp_off (-1: the data carry no
  // charge, no such sums)
  std::vector<int> cp_coup, cp_dr, cp_di, cp_t_re, cp_t_im;  // per CP total
  std::vector<int> cp_col, cp_c_re, cp_c_im;                 // per CP column
  int cp_off = -1;
  std::vector<int> key_var;
  // per coupling: its CP total entry or -1
  std::vector<int> coup_cp;
  // per trainable variable: coupling index or -1 with its role (0 r, 1 i,
  // 2 deltar, 3 deltai), shape selector slot or -1, barrier-row entry of mj
  // or -1, polarisation entry or -1
  std::vector<int> t_coup, t_comp, t_sel, t_mj, t_pol;
  // couplings and CP columns' couplings of the last consts() call, charge -1
  std::vector<std::complex<double>> zm;
  std::vector<double> ckm;
  // cache of the shape part
  bool have_shape = false;
  std::vector<double> key, cshape;
  std::vector<std::vector<double>> kap;  // per mj entry, per column
  std::string err;
};

namespace pwa_host {

// Parse the flat arrays into *p; false with *err set on a malformed program.
bool parse(const int* ip, long long n_ip, const double* dp, long long n_dp, pwa_hostprog* p,
           std::string* err);
// Constant block (nconst doubles) at vars; z (n_coup couplings) and ck
// (2*ncol, re/im) are filled on the way.
void consts(pwa_hostprog* p, const double* vars, double* C, std::vector<std::complex<double>>* z,
            std::vector<double>* ck);
// Jacobian of the column couplings, J[t*ncol + k] (complex), of the CP
// columns' charge -1 couplings, Jm[t*ncp_col + q] (may be null without CP
// columns), and the selectors D[t*nshape + j] of the kernels' extra sums of
// every trainable variable (after consts()).
void jacobian(pwa_hostprog* p, const double* vars, const std::vector<std::complex<double>>& z,
              const std::vector<double>& ck, std::complex<double>* J, std::complex<double>* Jm,
              double* D);
// d(sum)/d(trainable) of one event set's sums s (1 + 2*ncol + nshape).
void grad_from_sums(const pwa_hostprog* p, const std::complex<double>* J,
                    const std::complex<double>* Jm, const double* D, const double* s, double* g);
// Barrier-normalisation product of each column (ncol) in the constant
// block C; false where a factor is not positive (the columns do not
// factorise at this setting).
bool column_rho(const pwa_hostprog* p, const double* C, double* rho);

}  // namespace pwa_host
