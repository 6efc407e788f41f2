/*
 * FP64 restatement of the reference's Kalman-fit arithmetic. See restate.h.
 * TEST INFRASTRUCTURE ONLY (the oracle); never part of the product.
 *
 * Each routine evaluates the same algorithm as the cited reference routine
 * (same iteration count, same 4th-order half-angle polynomial, same
 * material model), with every intermediate in double precision.
 */
#include "restate.h"

#include <math.h>
#include <string.h>

#define RS_PI 3.14159265358979323846
#define RS_SOL 0.299792458
#define RS_B 3.8112
#define RS_NITER 5

static int sym(int i, int j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

static double hipo(double x, double y) { return sqrt(x * x + y * y); }

/* Config.h:434-437 */
static double bfield_zr(double z, double r) {
  return (-3.94991e-06 * z * z + 7.53701e-06 * z + 3.8114) * (2.43878e-11 * r * r + 1.0);
}

/* Matrix.h:48-56 */
static void sincos4(double x, double* s, double* c) {
  const double x2 = x * x;
  *c = 1.0 - 0.5 * x2 + 0.04166667 * x2 * x2;
  *s = x - 0.16666667 * x * x2;
}

static double squash_phi(double phi) {
  if (phi >= RS_PI) phi -= 2 * RS_PI;
  if (phi < -RS_PI) phi += 2 * RS_PI;
  return phi;
}

/* C = J * E * J^T with E packed symmetric (dense 6x6 in double). */
static void similarity(const double J[36], const double E[21], double out[21]) {
  double T[36];
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      double s = 0;
      for (int k = 0; k < 6; ++k) s += J[i * 6 + k] * E[sym(k, j)];
      T[i * 6 + j] = s;
    }
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j <= i; ++j) {
      double s = 0;
      for (int k = 0; k < 6; ++k) s += T[i * 6 + k] * J[j * 6 + k];
      out[sym(i, j)] = s;
    }
}

/* mkFit/PropagationMPlex.icc:5-246 */
static int helix_to_r(const double in[6], int chg, double r, int param_b, double out[6],
                      double J[36]) {
  memset(J, 0, sizeof(double) * 36);
  int fail = 0;
  double r0 = hipo(in[0], in[1]);
  const double bf = param_b ? bfield_zr(in[2], r0) : RS_B;
  const double k = chg * 100.0 / (-RS_SOL * bf);
  const double xin = in[0], yin = in[1], ipt = in[3], phiin = in[4], theta = in[5];
  const double kinv = 1.0 / k, pt = 1.0 / ipt;
  double D = 0, cosa = 0, sina = 0, cosah = 0, sinah = 0, id = 0;
  double cosP = cos(phiin), sinP = sin(phiin);
  double pxin = cosP * pt, pyin = sinP * pt;
  double dDdx = r0 > 0 ? -xin / r0 : 0, dDdy = r0 > 0 ? -yin / r0 : 0, dDdipt = 0, dDdphi = 0;
  double ox = in[0], oy = in[1];
  for (int it = 0; it < RS_NITER; ++it) {
    r0 = hipo(ox, oy);
    const double oodotp = r0 * pt / (pxin * ox + pyin * oy);
    if (oodotp > 5.0 || oodotp < 0) {
      id = 0;
      fail = 1;
    } else {
      id = (r - r0) * oodotp;
    }
    D += id;
    sincos4(id * ipt * kinv * 0.5, &sinah, &cosah);
    cosa = 1 - 2 * sinah * sinah;
    sina = 2 * sinah * cosah;
    if (it + 1 != RS_NITER) {
      const double x = ox, y = oy;
      const double oor0 = (r0 > 0 && fabs(r - r0) < 0.0001) ? 1.0 / r0 : 0.0;
      const double dadipt = id * kinv;
      const double dadx = -x * ipt * kinv * oor0, dady = -y * ipt * kinv * oor0;
      const double pxca = pxin * cosa, pxsa = pxin * sina, pyca = pyin * cosa, pysa = pyin * sina;
      double tmp = k * dadx;
      dDdx -= (x * (1 + tmp * (pxca - pysa)) + y * tmp * (pyca + pxsa)) * oor0;
      tmp = k * dady;
      dDdy -= (x * tmp * (pxca - pysa) + y * (1 + tmp * (pyca + pxsa))) * oor0;
      tmp = dadipt * ipt;
      dDdipt -= k * (x * (pxca * tmp - pysa * tmp - pyca - pxsa + pyin) +
                     y * (pyca * tmp + pxsa * tmp - pysa + pxca - pxin)) * pt * oor0;
      dDdphi += k * (x * (pysa - pxin + pxca) - y * (pxsa - pyin + pyca)) * oor0;
    }
    ox += 2 * k * sinah * (pxin * cosah - pyin * sinah);
    oy += 2 * k * sinah * (pyin * cosah + pxin * sinah);
    const double pxo = pxin;
    pxin = pxin * cosa - pyin * sina;
    pyin = pyin * cosa + pxo * sina;
  }
  const double alpha = D * ipt * kinv;
  const double dadx = dDdx * ipt * kinv, dady = dDdy * ipt * kinv;
  const double dadipt = (ipt * dDdipt + D) * kinv, dadphi = dDdphi * ipt * kinv;
  sincos4(alpha, &sina, &cosa);
  J[0] = 1 + k * dadx * (cosP * cosa - sinP * sina) * pt;
  J[1] = k * dady * (cosP * cosa - sinP * sina) * pt;
  J[3] = k * (cosP * (ipt * dadipt * cosa - sina) + sinP * ((1 - cosa) - ipt * dadipt * sina)) * pt * pt;
  J[4] = k * (cosP * dadphi * cosa - sinP * dadphi * sina - sinP * sina + cosP * cosa - cosP) * pt;
  J[6] = k * dadx * (sinP * cosa + cosP * sina) * pt;
  J[7] = 1 + k * dady * (sinP * cosa + cosP * sina) * pt;
  J[9] = k * (sinP * (ipt * dadipt * cosa - sina) + cosP * (ipt * dadipt * sina - (1 - cosa))) * pt * pt;
  J[10] = k * (sinP * dadphi * cosa + cosP * dadphi * sina + sinP * cosa + cosP * sina - sinP) * pt;
  const double cosT = cos(theta), isinT = 1.0 / sin(theta);
  out[0] = ox;
  out[1] = oy;
  out[2] = in[2] + k * alpha * cosT * pt * isinT;
  out[3] = ipt;
  out[4] = in[4] + alpha;
  out[5] = theta;
  J[12] = k * cosT * dadx * pt * isinT;
  J[13] = k * cosT * dady * pt * isinT;
  J[14] = 1;
  J[15] = k * cosT * (ipt * dadipt - alpha) * pt * pt * isinT;
  J[16] = k * dadphi * cosT * pt * isinT;
  J[17] = -k * alpha * pt * isinT * isinT;
  J[21] = 1;
  J[24] = dadx;
  J[25] = dady;
  J[27] = dadipt;
  J[28] = 1 + dadphi;
  J[35] = 1;
  return fail;
}

/* mkFit/PropagationMPlex.cc:604-712 */
static void helix_to_z(const double in[6], int chg, double zout, int param_b, double out[6],
                       double J[36]) {
  memset(J, 0, sizeof(double) * 36);
  J[0] = J[7] = J[21] = J[28] = J[35] = 1;
  const double zin = in[2], ipt = in[3], phiin = in[4], theta = in[5];
  const double bf = param_b ? bfield_zr(zin, hipo(in[0], in[1])) : RS_B;
  const double k = chg * 100.0 / (-RS_SOL * bf), kinv = 1.0 / k, pt = 1.0 / ipt;
  const double cosP = cos(phiin), sinP = sin(phiin), cosT = cos(theta), sinT = sin(theta);
  const double tanT = sinT / cosT, icos2T = 1.0 / (cosT * cosT);
  const double pxin = cosP * pt, pyin = sinP * pt;
  const double deltaZ = zout - zin, alpha = deltaZ * tanT * ipt * kinv;
  double sinah, cosah;
  sincos4(alpha * 0.5, &sinah, &cosah);
  const double cosa = 1 - 2 * sinah * sinah, sina = 2 * sinah * cosah;
  out[0] = in[0] + 2 * k * sinah * (pxin * cosah - pyin * sinah);
  out[1] = in[1] + 2 * k * sinah * (pyin * cosah + pxin * sinah);
  out[2] = zout;
  out[3] = in[3];
  out[4] = phiin + alpha;
  out[5] = in[5];
  const double a = pxin * cosa - pyin * sina, b = pyin * cosa + pxin * sina;
  J[2] = -tanT * ipt * a;
  J[3] = k * pt * pt * (cosP * (alpha * cosa - sina) + sinP * 2 * sinah * (sinah - alpha * cosah));
  J[4] = -2 * k * pt * sinah * (sinP * cosah + cosP * sinah);
  J[5] = deltaZ * ipt * a * icos2T;
  J[8] = -tanT * ipt * b;
  J[9] = k * pt * pt * (sinP * (alpha * cosa - sina) - cosP * 2 * sinah * (sinah - alpha * cosah));
  J[10] = 2 * k * pt * sinah * (cosP * cosah - sinP * sinah);
  J[11] = deltaZ * ipt * b * icos2T;
  J[26] = -ipt * tanT * kinv;
  J[27] = tanT * deltaZ * kinv;
  J[29] = ipt * deltaZ * kinv * icos2T;
}

/* mkFit/PropagationMPlex.cc:716-767 */
static void material_effects(double radL, double xi, double sign, int barrel, double C[21],
                             double par[6]) {
  if (radL < 1e-13) return;
  const double theta = par[5], pt = 1.0 / par[3], p = pt / sin(theta), p2 = p * p;
  const double mpi = 0.140, mpi2 = mpi * mpi;
  const double beta2 = p2 / (p2 + mpi2), beta = sqrt(beta2);
  const double invCos = barrel ? p / pt : 1.0 / fabs(cos(theta));
  radL *= invCos;
  if (radL < 1e-13) return;
  const double tms = 0.0136 * (1 + 0.038 * log(radL)) / (beta * p);
  const double tms2 = tms * tms * radL;
  C[14] += tms2;
  C[20] += tms2;
  const double gamma2 = (p2 + mpi2) / mpi2, gamma = sqrt(gamma2);
  const double me = 0.0005;
  const double wmax = 2 * me * beta2 * gamma2 / (1 + 2 * gamma * me / mpi + me * me / (mpi * mpi));
  const double I = 16.0e-9 * 10.75;
  const double dh = log(28.816e-9 * sqrt(2.33 * 0.498) / I) + log(beta * gamma) - 0.5;
  const double dEdx = beta < 1 ? (2 * (xi * invCos * (0.5 * log(2 * me * beta2 * gamma2 * wmax / (I * I)) - beta2 - dh) / beta2)) : 0;
  const double dP = sign * dEdx / beta;
  par[3] = p / (fmax(p + dP, 0.001) * pt);
  C[9] += dP * dP / (p2 * pt * pt);
}

static void mat_lookup(const rs_material* m, double z, double r, double scale, double* rl, double* xi) {
  *rl = 0;
  *xi = 0;
  if (!m || !m->rl) return;
  const int zb = (int)((float)(fabs(z) * 300.0) / 300.0f);
  const int rb = (int)((float)(r * 120.0) / 120.0f);
  if (zb >= 0 && zb < 300 && rb >= 0 && rb < 120) {
    *rl = m->rl[zb * 120 + rb] * scale;
    *xi = m->xi[zb * 120 + rb] * scale;
  }
}

static int propagate_r_scaled(const double in_par[6], const double in_err[21], int chg, double r,
                              unsigned pflags, const rs_material* mat, double scale,
                              double out_par[6], double out_err[21]) {
  double J[36], p[6], C[21];
  const int fail = helix_to_r(in_par, chg, r, pflags & 1u, p, J);
  memcpy(C, in_err, sizeof(C));
  if (pflags & 2u) {
    double rl = 0, xi = 0;
    if (!fail) mat_lookup(mat, p[2], r, scale, &rl, &xi);
    const double sign = r > hipo(in_par[0], in_par[1]) ? 1.0 : -1.0;
    material_effects(rl, xi, sign, 1, C, p);
  }
  p[4] = squash_phi(p[4]);
  if (fail) {
    memcpy(out_par, in_par, sizeof(double) * 6);
    memcpy(out_err, in_err, sizeof(double) * 21);
  } else {
    memcpy(out_par, p, sizeof(double) * 6);
    similarity(J, C, out_err);
  }
  return fail;
}

int rs_propagate_to_r(const double in_par[6], const double in_err[21], int chg, double r,
                      unsigned pflags, const rs_material* mat, double out_par[6],
                      double out_err[21]) {
  return propagate_r_scaled(in_par, in_err, chg, r, pflags, mat, 1.0, out_par, out_err);
}

static void propagate_z_scaled(const double in_par[6], const double in_err[21], int chg, double z,
                               unsigned pflags, const rs_material* mat, double scale,
                               double out_par[6], double out_err[21]) {
  double J[36], p[6], C[21];
  helix_to_z(in_par, chg, z, pflags & 1u, p, J);
  memcpy(C, in_err, sizeof(C));
  if (pflags & 2u) {
    double rl = 0, xi = 0;
    mat_lookup(mat, z, hipo(p[0], p[1]), scale, &rl, &xi);
    const double sign = fabs(z) > fabs(in_par[2]) ? 1.0 : -1.0;
    material_effects(rl, xi, sign, 0, C, p);
  }
  p[4] = squash_phi(p[4]);
  memcpy(out_par, p, sizeof(double) * 6);
  similarity(J, C, out_err);
}

void rs_propagate_to_z(const double in_par[6], const double in_err[21], int chg, double z,
                       unsigned pflags, const rs_material* mat, double out_par[6],
                       double out_err[21]) {
  propagate_z_scaled(in_par, in_err, chg, z, pflags, mat, 1.0, out_par, out_err);
}

/* Shared tail: gain K (6x2) from the local 2x2 inverse and the projector
 * rows (hx, hy, hz) of the two local coordinates. */
static void kalman_apply(const double par[6], const double err[21], const double H[2][3],
                         const double Sinv[3], const double res[2], double out_par[6],
                         double out_err[21]) {
  double PHt[6][2];
  for (int i = 0; i < 6; ++i)
    for (int a = 0; a < 2; ++a) {
      double s = 0;
      for (int c = 0; c < 3; ++c) s += err[sym(i, c)] * H[a][c];
      PHt[i][a] = s;
    }
  double K[6][2];
  for (int i = 0; i < 6; ++i) {
    K[i][0] = PHt[i][0] * Sinv[0] + PHt[i][1] * Sinv[1];
    K[i][1] = PHt[i][0] * Sinv[1] + PHt[i][1] * Sinv[2];
  }
  for (int i = 0; i < 6; ++i) out_par[i] = par[i] + K[i][0] * res[0] + K[i][1] * res[1];
  out_par[4] = squash_phi(out_par[4]);
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j <= i; ++j)
      out_err[sym(i, j)] = err[sym(i, j)] - (K[i][0] * PHt[j][0] + K[i][1] * PHt[j][1]);
}

/* mkFit/KalmanUtilsMPlex.cc:548-681 */
double rs_kalman_barrel(const double par[6], const double err[21], const double mpos[3],
                        const double merr[6], double out_par[6], double out_err[21]) {
  const double r = hipo(mpos[0], mpos[1]);
  const double r00 = -(mpos[1] + par[1]) / (2 * r), r01 = (mpos[0] + par[0]) / (2 * r);
  const double H[2][3] = {{r00, r01, 0}, {0, 0, 1}};
  const double rg[3] = {mpos[0] - par[0], mpos[1] - par[1], mpos[2] - par[2]};
  const double res[2] = {r00 * rg[0] + r01 * rg[1], rg[2]};
  double S[3] = {0, 0, 0};
  for (int a = 0; a < 2; ++a)
    for (int b = 0; b <= a; ++b) {
      double s = 0;
      for (int c = 0; c < 3; ++c)
        for (int d = 0; d < 3; ++d) s += H[a][c] * (err[sym(c, d)] + merr[sym(c, d)]) * H[b][d];
      S[a * (a + 1) / 2 + b] = s;
    }
  const double det = S[0] * S[2] - S[1] * S[1];
  const double Si[3] = {S[2] / det, -S[1] / det, S[0] / det};
  const double chi2 = Si[0] * res[0] * res[0] + Si[2] * res[1] * res[1] + 2 * Si[1] * res[0] * res[1];
  if (out_par) kalman_apply(par, err, H, Si, res, out_par, out_err);
  return chi2;
}

/* mkFit/KalmanUtilsMPlex.cc:774-888 */
double rs_kalman_endcap(const double par[6], const double err[21], const double mpos[3],
                        const double merr[6], double out_par[6], double out_err[21]) {
  const double H[2][3] = {{1, 0, 0}, {0, 1, 0}};
  const double res[2] = {mpos[0] - par[0], mpos[1] - par[1]};
  const double S[3] = {err[0] + merr[0], err[1] + merr[1], err[2] + merr[2]};
  const double det = S[0] * S[2] - S[1] * S[1];
  const double Si[3] = {S[2] / det, -S[1] / det, S[0] / det};
  const double chi2 = Si[0] * res[0] * res[0] + Si[2] * res[1] * res[1] + 2 * Si[1] * res[0] * res[1];
  if (out_par) kalman_apply(par, err, H, Si, res, out_par, out_err);
  return chi2;
}

void rs_fit(int n, int n_steps, const float* par, const float* err, const int* chg,
            const float* hit_pos, const float* hit_err, unsigned long long endcap_mask,
            unsigned pflags, const rs_material* mat, const double* shift_rphi,
            const double* shift_z, const double* mat_scale, double* out_par, double* out_err,
            double* out_chi2) {
  for (int i = 0; i < n; ++i) {
    double p[6], e[21], pp[6], pe[21];
    for (int k = 0; k < 6; ++k) p[k] = par[k * n + i];
    for (int k = 0; k < 21; ++k) e[k] = err[k * n + i];
    double chi2 = 0;
    for (int s = 0; s < n_steps; ++s) {
      const float* hp = hit_pos + (size_t)s * 3 * n;
      const float* he = hit_err + (size_t)s * 6 * n;
      double m[3] = {hp[i], hp[n + i], hp[2 * n + i]}, me[6];
      for (int k = 0; k < 6; ++k) me[k] = he[k * n + i];
      if (shift_rphi || shift_z) {
        const double rh = hipo(m[0], m[1]);
        const double a = shift_rphi ? shift_rphi[s] : 0.0, b = shift_z ? shift_z[s] : 0.0;
        const double tx = -m[1] / rh, ty = m[0] / rh;
        m[0] += a * tx;
        m[1] += a * ty;
        m[2] += b;
      }
      const double scale = mat_scale ? mat_scale[s] : 1.0;
      if (!((endcap_mask >> s) & 1ull)) {
        propagate_r_scaled(p, e, chg[i], hipo(m[0], m[1]), pflags, mat, scale, pp, pe);
        chi2 += rs_kalman_barrel(pp, pe, m, me, p, e);
      } else {
        propagate_z_scaled(p, e, chg[i], m[2], pflags, mat, scale, pp, pe);
        chi2 += rs_kalman_endcap(pp, pe, m, me, p, e);
      }
    }
    for (int k = 0; k < 6; ++k) out_par[k * n + i] = p[k];
    for (int k = 0; k < 21; ++k) out_err[k * n + i] = e[k];
    if (out_chi2) out_chi2[i] = chi2;
  }
}

/* Clone-engine candidates replayed in double precision from their seed
 * state along their hit-on-track lists, with the arithmetic of the
 * reference's finding steps:
 *  - chi2 of a hit (MkFinder::FindCandidatesCloneEngine with
 *    finding_requires_propagation_to_hit_pos, mkFit/MkFinder.cc:1116-1240,
 *    KalmanUtilsMPlex.cc:518-544, 744-770): the candidate propagated to the
 *    layer (inter-layer flags, r or z of the layer), then to the hit
 *    (intra-layer flags), |chi2|;
 *  - update (MkFinder::UpdateWithLastHit, mkFit/MkFinder.cc:1291-1308,
 *    KalmanUtilsMPlex.cc:471-505, 697-731): the candidate propagated to the
 *    last hit added on the layer (inter-layer flags) and updated with it;
 *    a negative 1/pT flips the charge;
 *  - a layer with no hit (a hole node) leaves the state as it is.
 * The first skip[i] nodes (the seed's own hits) are not replayed. */
void rs_replay_cands(int n, const float* seed_par, const float* seed_err, const int* seed_chg,
                     const int* n_nodes, const int* node_hit, const int* node_layer,
                     int node_stride, const int* skip, const float* hit_pos,
                     const float* hit_err, int hit_stride, const int* layer_begin,
                     const int* layer_is_barrel, const float* layer_prop_to,
                     unsigned inter_pflags, unsigned intra_pflags, const rs_material* mat,
                     double* out_par, double* out_err, int* out_chg, double* out_chi2) {
  for (int i = 0; i < n; ++i) {
    double p[6], e[21];
    for (int k = 0; k < 6; ++k) p[k] = seed_par[i * 6 + k];
    for (int k = 0; k < 21; ++k) e[k] = seed_err[i * 21 + k];
    int chg = seed_chg[i];
    double chi2 = 0;
    const int* hits = node_hit + (size_t)i * node_stride;
    const int* lays = node_layer + (size_t)i * node_stride;
    int k = skip[i];
    while (k < n_nodes[i]) {
      const int lyr = lays[k];
      int end = k;
      while (end < n_nodes[i] && lays[end] == lyr) ++end;
      int last = -1;
      for (int j = k; j < end; ++j)
        if (hits[j] >= 0) last = j;
      if (last >= 0) {
        const int barrel = layer_is_barrel[lyr];
        double lp[6], le[21];
        if (barrel)
          propagate_r_scaled(p, e, chg, layer_prop_to[lyr], inter_pflags, mat, 1.0, lp, le);
        else
          propagate_z_scaled(p, e, chg, layer_prop_to[lyr], inter_pflags, mat, 1.0, lp, le);
        for (int j = k; j < end; ++j) {
          if (hits[j] < 0) continue;
          const int g = layer_begin[lyr] + hits[j];
          double m[3], me[6], hp[6], he[21];
          for (int c = 0; c < 3; ++c) m[c] = hit_pos[(size_t)c * hit_stride + g];
          for (int c = 0; c < 6; ++c) me[c] = hit_err[(size_t)c * hit_stride + g];
          if (barrel) {
            propagate_r_scaled(lp, le, chg, hipo(m[0], m[1]), intra_pflags, mat, 1.0, hp, he);
            chi2 += fabs(rs_kalman_barrel(hp, he, m, me, NULL, NULL));
          } else {
            propagate_z_scaled(lp, le, chg, m[2], intra_pflags, mat, 1.0, hp, he);
            chi2 += fabs(rs_kalman_endcap(hp, he, m, me, NULL, NULL));
          }
        }
        const int g = layer_begin[lyr] + hits[last];
        double m[3], me[6], hp[6], he[21];
        for (int c = 0; c < 3; ++c) m[c] = hit_pos[(size_t)c * hit_stride + g];
        for (int c = 0; c < 6; ++c) me[c] = hit_err[(size_t)c * hit_stride + g];
        if (barrel) {
          propagate_r_scaled(p, e, chg, hipo(m[0], m[1]), inter_pflags, mat, 1.0, hp, he);
          rs_kalman_barrel(hp, he, m, me, p, e);
        } else {
          propagate_z_scaled(p, e, chg, m[2], inter_pflags, mat, 1.0, hp, he);
          rs_kalman_endcap(hp, he, m, me, p, e);
        }
        if (p[3] < 0) {
          chg = -chg;
          p[3] = -p[3];
        }
      }
      k = end;
    }
    for (int c = 0; c < 6; ++c) out_par[i * 6 + c] = p[c];
    for (int c = 0; c < 21; ++c) out_err[i * 21 + c] = e[c];
    out_chg[i] = chg;
    out_chi2[i] = chi2;
  }
}
