/*
 * FP64 restatement of the reference's Kalman-fit arithmetic (trackreco/mkFit).
 *
 * TEST INFRASTRUCTURE ONLY (the oracle): used by tests/ and bench.py's CPU
 * baseline leg to state the error of the FP32 results against the same
 * algorithm evaluated in double precision, and for finite-difference checks
 * of the adjoint. Never linked into the product.
 *
 * Parity pin: tests/test_oracle.py checks this restatement against the
 * reference's own compiled CPU path (oracle/_ref) on identical inputs.
 *
 * Layouts as in include/mkfit_b200.h: par[6], err[21] packed lower triangle.
 */
#ifndef MKFG_RESTATE_H
#define MKFG_RESTATE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Material grid (300 x 120) used by the propagation; NULL disables lookups. */
typedef struct {
  const float* rl;
  const float* xi;
} rs_material;

/* Helix propagation to radius r (mkFit/PropagationMPlex.cc:408-505).
 * Returns the fail flag; on failure out = in. */
int rs_propagate_to_r(const double in_par[6], const double in_err[21], int chg, double r,
                      unsigned pflags, const rs_material* mat, double out_par[6],
                      double out_err[21]);

/* Helix propagation to plane z (mkFit/PropagationMPlex.cc:510-601). */
void rs_propagate_to_z(const double in_par[6], const double in_err[21], int chg, double z,
                       unsigned pflags, const rs_material* mat, double out_par[6],
                       double out_err[21]);

/* Barrel / endcap Kalman operation (mkFit/KalmanUtilsMPlex.cc:548-681,
 * 774-888). Returns chi2; writes the update when out_par != NULL. */
double rs_kalman_barrel(const double par[6], const double err[21], const double mpos[3],
                        const double merr[6], double out_par[6], double out_err[21]);
double rs_kalman_endcap(const double par[6], const double err[21], const double mpos[3],
                        const double merr[6], double out_par[6], double out_err[21]);

/* Whole fit of n tracks over n_steps barrel/endcap steps, SoA in/out as in
 * mkfg_fit: par[6][n], err[21][n], hit_pos[step][3][n], hit_err[step][6][n].
 * Optional per-layer alignment shifts (r-phi, z) applied to the hit
 * positions and per-layer material-thickness scales applied to rl/xi
 * (arrays of n_steps or NULL). out_chi2[n] (optional) = summed chi2. */
void rs_fit(int n, int n_steps, const float* par, const float* err, const int* chg,
            const float* hit_pos, const float* hit_err, unsigned long long endcap_mask,
            unsigned pflags, const rs_material* mat, const double* shift_rphi,
            const double* shift_z, const double* mat_scale, double* out_par, double* out_err,
            double* out_chi2);

/* Clone-engine candidates replayed from their seed state along their
 * hit-on-track lists in double precision (the arithmetic of the reference's
 * FindCandidatesCloneEngine chi2 and UpdateWithLastHit steps): n candidates
 * with seed_par[n][6], seed_err[n][21], seed_chg[n]; nodes
 * node_hit/node_layer[n][node_stride] (index within the layer, negative =
 * hole), n_nodes[n], skip[n] seed nodes; hits hit_pos[3][hit_stride],
 * hit_err[6][hit_stride] with layer l at [layer_begin[l], layer_begin[l+1]);
 * per layer: barrel flag and the r or z the finding propagates to. Outputs
 * the final state (out_par[n][6], out_err[n][21], out_chg[n]) and the sum
 * of the hits' chi2 (out_chi2[n]). */
void rs_replay_cands(int n, const float* seed_par, const float* seed_err, const int* seed_chg,
                     const int* n_nodes, const int* node_hit, const int* node_layer,
                     int node_stride, const int* skip, const float* hit_pos,
                     const float* hit_err, int hit_stride, const int* layer_begin,
                     const int* layer_is_barrel, const float* layer_prop_to,
                     unsigned inter_pflags, unsigned intra_pflags, const rs_material* mat,
                     double* out_par, double* out_err, int* out_chg, double* out_chi2);

#ifdef __cplusplus
}
#endif
#endif
