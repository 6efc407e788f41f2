// TEST INFRASTRUCTURE ONLY. The product's generated fit-step adjoint
// (mkfit_b200/csrc/generated_adjoint.cuh) instantiated in double precision
// on the host. The CPU tests compare its gradient with central finite
// differences of the independent FP64 restatement (restate.c, rs_fit with
// shift_rphi / shift_z / mat_scale), which checks the derivation itself
// without a GPU; the GPU tests then compare the FP32 device gradient with
// the same finite differences.
#include "../mkfit_b200/csrc/adjoint_step.cuh"

#include <vector>

using namespace mkfg::adj;

extern "C" void adj_f64_fit_grad(int n, int n_steps, const float* par, const float* err,
                                 const int* chg, const float* hit_pos, const float* hit_err,
                                 const double* theta, const float* rl, const float* xi,
                                 int material, double* chi2_sum, double* grad) {
  const MatGrid mat{material ? rl : nullptr, material ? xi : nullptr};
  double total = 0;
  for (int j = 0; j < 3 * n_steps; ++j) grad[j] = 0;
  std::vector<double> ck((size_t)n_steps * 27);
  for (int i = 0; i < n; ++i) {
    double p[6], e[21];
    for (int k = 0; k < 6; ++k) p[k] = par[k * n + i];
    for (int k = 0; k < 21; ++k) e[k] = err[k * n + i];
    const double kk = chg[i] * 100.0 / (-0.299792458 * 3.8112);
    auto hit = [&](int s, double (&m)[3], double (&me)[6]) {
      for (int k = 0; k < 3; ++k) m[k] = hit_pos[((size_t)s * 3 + k) * n + i];
      for (int k = 0; k < 6; ++k) me[k] = hit_err[((size_t)s * 6 + k) * n + i];
    };
    for (int s = 0; s < n_steps; ++s) {
      for (int k = 0; k < 6; ++k) ck[s * 27 + k] = p[k];
      for (int k = 0; k < 21; ++k) ck[s * 27 + 6 + k] = e[k];
      double m[3], me[6], op[6], oe[21], c2;
      hit(s, m, me);
      if (material)
        barrel_step_fwd_mat(p, e, m, me, theta[3 * s], theta[3 * s + 1], theta[3 * s + 2], kk,
                            mat, op, oe, c2);
      else
        barrel_step_fwd_nomat(p, e, m, me, theta[3 * s], theta[3 * s + 1], theta[3 * s + 2], kk,
                              mat, op, oe, c2);
      for (int k = 0; k < 6; ++k) p[k] = op[k];
      for (int k = 0; k < 21; ++k) e[k] = oe[k];
      total += c2;
    }
    double pb[6] = {0}, eb[21] = {0};
    for (int s = n_steps - 1; s >= 0; --s) {
      double cp[6], ce[21], m[3], me[6], npb[6], neb[21], ga, gb, gc;
      for (int k = 0; k < 6; ++k) cp[k] = ck[s * 27 + k];
      for (int k = 0; k < 21; ++k) ce[k] = ck[s * 27 + 6 + k];
      hit(s, m, me);
      if (material)
        barrel_step_rev_mat(cp, ce, m, me, theta[3 * s], theta[3 * s + 1], theta[3 * s + 2], kk,
                            mat, pb, eb, 1.0, npb, neb, ga, gb, gc);
      else
        barrel_step_rev_nomat(cp, ce, m, me, theta[3 * s], theta[3 * s + 1], theta[3 * s + 2],
                              kk, mat, pb, eb, 1.0, npb, neb, ga, gb, gc);
      for (int k = 0; k < 6; ++k) pb[k] = npb[k];
      for (int k = 0; k < 21; ++k) eb[k] = neb[k];
      grad[3 * s] += ga;
      grad[3 * s + 1] += gb;
      grad[3 * s + 2] += gc;
    }
  }
  *chi2_sum = total;
}
