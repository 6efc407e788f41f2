/*
 * mkfit_b200 -- C ABI of the B200-native Kalman-filter tracking hot path.
 *
 * Plain C types only: pointers, sizes and POD structs. Every entry point
 * returns an int status (MKFG_OK = 0), never aborts, and records a message
 * retrievable with mkfg_last_error(). All device work is enqueued on the
 * stream of the context (or the stream the caller passes), so calls from
 * different host threads on different contexts are independent.
 *
 * Data layout (the reference's Matriplex layout, Matriplex/Matriplex.h:63-68,
 * widened to a whole batch): structure of arrays, lane fastest. Element e of
 * item i lives at base[e * stride + i]. Track parameters are the reference's
 * CCS coordinates (x, y, z, 1/pT, phi, theta); covariances are 21 floats in
 * packed lower-triangle order (Matriplex/MatriplexSym.h:15-22); hit
 * covariances are 6 floats in the same order.
 */
#ifndef MKFIT_B200_H
#define MKFIT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum {
  MKFG_OK = 0,
  MKFG_ERR_BAD_INPUT = 1, /* invalid argument, size or pointer */
  MKFG_ERR_CUDA = 2,      /* a CUDA runtime call failed */
  MKFG_ERR_OVERFLOW = 3,  /* a device capacity was exceeded (results truncated) */
  MKFG_ERR_TIMEOUT = 4,   /* a bounded device wait gave up */
  MKFG_ERR_NO_DEVICE = 5  /* no usable sm_100 device */
};

/* Propagation flag bits (reference PropagationFlagsEnum, Config.h:17-23). */
enum { MKFG_PF_NONE = 0, MKFG_PF_PARAM_BFIELD = 0x1, MKFG_PF_MATERIAL = 0x2 };

/* Copies the calling thread's last error message (NUL-terminated). */
void mkfg_last_error(char* buf, size_t len);

/* Library version string, e.g. "mkfit_b200 0.1 sm_100a". */
const char* mkfg_version(void);

/* --------------------------------------------------------------- context */
/* A context binds one CUDA device and one stream and owns the device copies
 * of the material map, the detector geometry and scratch buffers for the
 * host-buffer entry points. Replaces the reference's per-thread worker pools
 * (mkFit/Pool.h:15-58, mkFit/MkBuilder.h:34-49). */
typedef struct mkfg_context mkfg_context;

int mkfg_context_create(int device, mkfg_context** out);
int mkfg_context_destroy(mkfg_context* ctx);
/* The cudaStream_t used by the context, as an opaque pointer. */
void* mkfg_context_stream(mkfg_context* ctx);
/* Makes the context enqueue its work on the caller's stream (a
 * cudaStream_t of the context's device, as an opaque pointer; NULL: back
 * to the stream the context created). Waits for the work already enqueued
 * on the current stream first. The caller keeps the stream alive while the
 * context uses it. */
int mkfg_context_set_stream(mkfg_context* ctx, void* stream);
int mkfg_context_synchronize(mkfg_context* ctx);

/* Upload the (z, r) material grid, 300 x 120 floats each, row = z bin
 * (reference Config::RlgridME / XigridME, Config.h:123-165, filled there by
 * fillZRgridME, MaterialEffects.h:277-290). Host pointers. */
int mkfg_set_material(mkfg_context* ctx, const float* rl_grid, const float* xi_grid);

/* Measures the device's FP32 FMA throughput (TFLOP/s) with a register-only
 * kernel: the roofline denominator of this library's kernels, which run on
 * the FP32 CUDA cores. No reference counterpart (measurement utility). */
int mkfg_probe_fp32_peak(mkfg_context* ctx, int iters, double* tflops);

/* ------------------------------------------------------------ track SoA */
typedef struct {
  float* par;   /* [6][stride]  */
  float* err;   /* [21][stride] */
  int32_t* chg; /* [stride]     */
  int32_t n;    /* number of tracks */
  int32_t stride;
} mkfg_tracks;

/* Hits of an event: all layers in one SoA buffer, layer l occupying items
 * [layer_begin[l], layer_begin[l+1]). Reference: std::vector<HitVec>
 * (Event.h) / Hit (Hit.h:185-304). */
typedef struct {
  const float* pos;          /* [3][stride] x, y, z */
  const float* err;          /* [6][stride] packed symmetric */
  const int32_t* layer_begin;/* [n_layers + 1], device pointer */
  int32_t n_layers;
  int32_t stride;
} mkfg_hits;

/* ------------------------------------------------------------------ fit */
/* Kalman fit over a fixed sequence of hits per track: for each layer step
 * l, propagate to the hit's radius (barrel) or z (endcap) and update.
 * Replaces MkFitter::InputTracksForFit + FitTracksWithInterSlurp +
 * OutputFittedTracks (mkFit/MkFitter.cc:286-363, 505-522) and the steered
 * form FitTracksSteered (mkFit/MkFitter.cc:473-503).
 *
 *   hot_index [n_steps][hot_stride]: index of track i's hit within layer
 *     hit_layer[l]; a negative index uses the layer's hit 0, as the
 *     reference's packer does (mkFit/MkFitter.cc:344-348).
 *   hit_layer [n_steps]: host array, layer of each step.
 *   endcap_mask: bit l set -> step l is an endcap (z) step.
 *   out_chi2 (optional, [n]): sum over steps of the predicted-residual chi2
 *     (kalmanOperation with KFO_Calculate_Chi2|KFO_Update_Params).
 * All array pointers are device pointers; in and out may alias. */
typedef struct {
  mkfg_tracks in;
  mkfg_tracks out;
  mkfg_hits hits;
  const int32_t* hot_index;
  int32_t hot_stride;
  int32_t n_steps;
  const int32_t* hit_layer; /* host */
  uint64_t endcap_mask;
  uint32_t pflags;
  float* out_chi2;
} mkfg_fit_args;

int mkfg_fit(mkfg_context* ctx, const mkfg_fit_args* args);

/* ----------------------------------------------------------- operators */
/* The finding's operator table (FindingFoos, mkFit/FindingFoos.h:10-38,
 * FindingFoos.cc:7-8) as plain calls on n states, endcap = 0 for the
 * barrel member of the table and 1 for the endcap one. Arrays are
 * lane-fastest with element stride `stride` >= n (element e of state i at
 * e * stride + i: a Matriplex's storage with stride NN); only lanes
 * [0, n) are read and written. Host pointers; the context's material map;
 * pflags: PropagationFlags bits (1 B field, 2 material). Synchronize.
 *
 * mkfg_op_propagate <- MkBase::PropagateTracksToR / PropagateTracksToZ
 *   (mkFit/MkBase.h:35-75): propagation to target[i] (r or z).
 * mkfg_op_propagate_chi2 <- kalmanPropagateAndComputeChi2[Endcap]
 *   (mkFit/KalmanUtilsMPlex.cc:524-544, 751-770): propagation to the hit's
 *   radius / z, chi2 of the hit (not its absolute value), the propagated
 *   parameters.
 * mkfg_op_propagate_update <- kalmanPropagateAndUpdate[Endcap]
 *   (:471-505, 697-731): propagation to the hit, update, charge flip of a
 *   negative 1/pT; out_chg may alias chg. */
int mkfg_op_propagate(mkfg_context* ctx, int32_t endcap, int32_t n, int32_t stride,
                      const float* par, const float* err, const int32_t* chg, const float* target,
                      uint32_t pflags, float* out_par, float* out_err);
int mkfg_op_propagate_chi2(mkfg_context* ctx, int32_t endcap, int32_t n, int32_t stride,
                           const float* par, const float* err, const int32_t* chg,
                           const float* hit_pos, const float* hit_err, uint32_t pflags,
                           float* out_chi2, float* out_prop_par);
int mkfg_op_propagate_update(mkfg_context* ctx, int32_t endcap, int32_t n, int32_t stride,
                             const float* par, const float* err, const int32_t* chg,
                             const float* hit_pos, const float* hit_err, uint32_t pflags,
                             float* out_par, float* out_err, int32_t* out_chg);

/* Same fit from HOST buffers: copies inputs to device scratch owned by the
 * context, fits, copies outputs back, synchronizes. The pointers inside
 * args (including hits.layer_begin) are host pointers here. */
int mkfg_fit_host(mkfg_context* ctx, const mkfg_fit_args* args);

/* Same fit from HOST buffers without allocating anything: inputs and
 * outputs are staged through a fixed 16 MiB device array compiled into the
 * library (a file-scope __device__ array) instead of the context's
 * grow-only scratch; no cudaMalloc / cudaFree or allocating library call is
 * made. Inputs whose staging exceeds 16 MiB (e.g. more than ~16k tracks x
 * 10 layers) are rejected with MKFG_ERR_BAD_INPUT and a message giving the
 * size; use mkfg_fit_host for them. Nothing in the array needs to start at
 * zero. The array is shared by all callers on a device: calls on the same
 * device must not overlap (other threads, other contexts), or they race on
 * it. The first call on a device resolves the array's address there
 * (cudaGetSymbolAddress, which may load the module); the call synchronizes
 * its stream before returning. No reference counterpart. */
int mkfg_fit_host_static(mkfg_context* ctx, const mkfg_fit_args* args);


/* ------------------------------------------------------ differentiable fit */
/* Summed chi2 of a barrel fit as a function of per-step alignment and
 * material parameters, and its gradient (hand-derived reverse mode through
 * the Kalman update, the covariance transport, the material effects and the
 * iterative helix propagation). No reference counterpart: the reference fit
 * (mkFit/MkFitter.cc:505-522) is not differentiable.
 *
 *   fit: as for mkfg_fit (device pointers); barrel steps only
 *     (endcap_mask 0), pflags 0 or material (2). out tracks may be NULL;
 *     out_chi2 (optional) receives each track's chi2 sum.
 *   theta [n_steps][3] (device): per step a = hit shift along the
 *     transverse tangent (r-phi, cm), b = hit shift in z (cm), c = scale of
 *     the layer's radiation length and xi (1 = nominal).
 *   checkpoint [n_steps][27][n] (device): state entering each step, written
 *     by the forward call and read by the backward call.
 *   chi2_sum (device, one double): L = sum over tracks and steps of chi2. */
typedef struct {
  mkfg_fit_args fit;
  const float* theta;
  float* checkpoint;
  double* chi2_sum;
} mkfg_align_args;

int mkfg_align_chi2_forward(mkfg_context* ctx, const mkfg_align_args* args);
/* grad_theta [n_steps][3] (device, double) = grad_out * dL/dtheta, for the
 * checkpoints of the last forward call with the same args; grad_out is a
 * device scalar (the incoming adjoint of L). */
int mkfg_align_chi2_backward(mkfg_context* ctx, const mkfg_align_args* args,
                             const float* grad_out, double* grad_theta);

/* ------------------------------------------------------------- finding */
/* Detector geometry + finding iteration configuration. Replaces the
 * reference's TrackerInfo / IterationConfig as consumed by MkBuilder
 * (TrackerInfo.h:35-147, mkFit/IterationConfig.h:44-124,
 * mkFit/SteeringParams.h:36-163). Host pointers; copied by the call.
 *
 * layer_desc: n_layers rows of 32 floats:
 *   0 is_barrel, 1 rin, 2 rout, 3 zmin, 4 zmax, 5 propagate_to, 6 q_bin
 *   (> 0 bin width, < 0 number of bins), 7 has_r_hole, 8 hole_rmin,
 *   9 hole_rmax, 10 is_pixel, 11 is_stereo, 12-15 min/max dphi, min/max dq,
 *   16-19 c_dp_{sf,0,1,2}, 20-23 c_dq_{sf,0,1,2}, 24-27 c_c2_{sf,0,1,2},
 *   28 layer type, 29 is_seed, 30-31 unused.
 * plans: n_regions rows of max_plan layer ids (-1 padded); the forward
 * search starts after plan position pickup[r]. */
typedef struct {
  int32_t n_layers;
  const float* layer_desc;
  int32_t n_regions;
  int32_t max_plan;
  const int32_t* plans;
  const int32_t* plan_len;
  const int32_t* pickup;
  int32_t max_cands_per_seed; /* <= 8 */
  int32_t max_holes_per_cand;
  int32_t max_consec_holes;
  float chi2_cut_min;
  float chi2_cut_overlap;
  float pt_cut_overlap;
  uint32_t inter_layer_pflags; /* Config::finding_inter_layer_pflags */
  uint32_t intra_layer_pflags; /* Config::finding_intra_layer_pflags */
  int32_t requires_prop_to_hit; /* Config::finding_requires_propagation_to_hit_pos; must be 1 */
  /* IterationConfig::m_requires_seed_hit_sorting: the upload sorts every
   * seed's hits by layer (Track::sortHitsByLayer, a stable sort) before it
   * orders the seeds, as run_OneIteration does (pixelLessStep, tobTecStep). */
  int32_t sort_seed_hits;
} mkfg_find_config;

/* The finder takes a copy of the context's material map (mkfg_set_material)
 * here: a later mkfg_set_material on the same context (e.g. for a fit on
 * another detector) does not change what the finding propagates through;
 * call mkfg_finder_setup again to take the new map. Events uploaded
 * before a setup are dropped: upload again before the next run. */
int mkfg_finder_setup(mkfg_context* ctx, const mkfg_find_config* cfg);

/* ---- memoryFile event files (DataFile / Event::write_out / read_in,
 * Event.cc:123-444; header Event.h:74-127) ---------------------------------
 * Host-only: no context or device needed. The reader indexes the event
 * records at open and reads any event by number into this library's SoA
 * layout; the writer produces files the reference reads (format version 6,
 * x86-64 struct layout: Track 160 B, Hit 44 B, HitOnTrack 4 B). */
#define MKFG_MF_SIM_TRACK_STATES 0x1 /* DataFile::ES_SimTrackStates */
#define MKFG_MF_SEEDS 0x2            /* ES_Seeds */
#define MKFG_MF_CMSSW_TRACKS 0x4     /* ES_CmsswTracks */
#define MKFG_MF_HIT_ITER_MASKS 0x8   /* ES_HitIterMasks */
#define MKFG_MF_BEAM_SPOT 0x10       /* ES_BeamSpot */

typedef struct {
  int32_t format_version;
  int32_t n_layers;
  int32_t n_events; /* complete event records found */
  int32_t extra_sections;
} mkfg_mf_header;

/* A track vector (Track fields; hits of track i at [hits_begin[i],
 * hits_begin[i+1]) of hit_index / hit_layer, HitOnTrack order). On write,
 * null valid / chi2 / score / status / label / nfound take the defaults
 * (1, 0, 0, 0, -1, counted from the hits as Track::addHitIdx does). */
typedef struct {
  int32_t n;
  const float* par;        /* [6][n] */
  const float* err;        /* [21][n] packed symmetric */
  const int32_t* charge;
  const uint8_t* valid;
  const float* chi2;
  const float* score;
  const uint32_t* status;  /* Track::Status raw bits */
  const int32_t* label;
  const int32_t* nfound;
  const int32_t* hits_begin; /* [n+1] */
  const int32_t* hit_index;
  const int32_t* hit_layer;
} mkfg_mf_tracks;

/* One event. Hits of layer l at [layer_begin[l], layer_begin[l+1]).
 * hit_packed: Hit::PackedData raw bits (detid 12 | charge-per-cm code 8 |
 * span rows 3 | span cols 3). mc_info: [n_mc][4] MCHitInfo (track, layer,
 * ith layer hit, mcHitID). beam_spot: 8 floats (x, y, z, sigmaZ,
 * beamWidthX, beamWidthY, dxdz, dydz); null on write = BeamSpot defaults. */
typedef struct {
  int32_t n_layers;
  const int32_t* layer_begin;
  const float* hit_pos;      /* [3][n_hits] */
  const float* hit_err;      /* [6][n_hits] */
  const int32_t* hit_mcid;   /* Hit::mcHitID */
  const uint32_t* hit_packed;
  const uint64_t* hit_masks; /* [n_hits] iteration masks, or null */
  int32_t n_mc;
  const int32_t* mc_info;
  mkfg_mf_tracks sim;
  mkfg_mf_tracks seeds;
  mkfg_mf_tracks cmssw;
  int32_t n_sim_states;
  const float* sim_state_par;  /* [6][n_sim_states] */
  const float* sim_state_err;  /* [21][n_sim_states] */
  const int32_t* sim_state_charge;
  const float* beam_spot;
} mkfg_mf_event;

typedef struct mkfg_mf_reader mkfg_mf_reader;
/* DataFile::OpenRead: checks magic, version (4..6), struct sizes and layer
 * count, then indexes the event records. On a truncated file the reader is
 * still returned (with the complete events) together with an error. */
int mkfg_mf_open(const char* path, mkfg_mf_reader** out, mkfg_mf_header* hdr);
/* Event::read_in of event number `event`; out's arrays belong to the
 * reader and stay valid until its next read or close. */
int mkfg_mf_read_event(mkfg_mf_reader* r, int32_t event, mkfg_mf_event* out);
void mkfg_mf_close(mkfg_mf_reader* r);
/* DataFile::OpenWrite + Event::write_out of every event + CloseWrite. */
int mkfg_mf_write(const char* path, int32_t n_layers, int32_t extra_sections, int32_t n_events,
                  const mkfg_mf_event* events);
/* The finder's per-hit detid / charge-per-cm and [n_seeds][max_seed_hits]
 * seed hits (mkfg_event fields) from a read event; any output may be null.
 * MKFG_ERR_OVERFLOW if a seed has more than max_seed_hits hits. */
int mkfg_mf_finder_event(const mkfg_mf_event* ev, int32_t* detid, int32_t* cpcm,
                         int32_t max_seed_hits, int32_t* seed_nhits, int32_t* seed_hit_layer,
                         int32_t* seed_hit_index);

/* Seed cleaning (StdSeq::clean_cms_seedtracks_iter, mkFit/MkStdSeqs.cc:115-311):
 * the iteration's window parameters (IterationParams c_ptthr_hpt, c_dzmax_*,
 * c_drmax_*, mkFit/IterationConfig.h:107-116; set_seed_cleaning_params order)
 * and the beam spot (BeamSpot x, y, Hit.h:340). */
typedef struct {
  float pt_thr;
  float dzmax_bh, drmax_bh;
  float dzmax_bl, drmax_bl;
  float dzmax_eh, drmax_eh;
  float dzmax_el, drmax_el;
  float beam_x, beam_y;
} mkfg_seed_clean_params;

/* Cleans the seeds of n_events events (event e's seeds at
 * [event_seed_begin[e], event_seed_begin[e+1]), the reference's seed order
 * within an event). Host pointers. seed_par [6][n] (CCS), seed_chg [n],
 * seed_nhits [n] with hits [n][in_hits] (layer, index). keep[n]: 1 for the
 * seeds the reference keeps; out_nhits / out_hit_layer / out_hit_index
 * ([n][max_hits], max_hits >= 15): the kept seeds' hit lists after the merge
 * of the dropped seeds' hits (sorted by layer where hits were added).
 * MKFG_ERR_OVERFLOW if more than 4096 overlapping pairs fall in one event.
 * Replaces the call in MkBuilder's run_OneIteration (mkFit/buildtestMPlex.cc:
 * 660-665). */
int mkfg_clean_seeds(mkfg_context* ctx, const mkfg_seed_clean_params* p, int32_t n_events,
                     const int32_t* event_seed_begin, const float* seed_par,
                     const int32_t* seed_chg, const int32_t* seed_nhits,
                     const int32_t* seed_hit_layer, const int32_t* seed_hit_index,
                     int32_t in_hits, int32_t max_hits, int32_t* keep, int32_t* out_nhits,
                     int32_t* out_hit_layer, int32_t* out_hit_index);

/* One event: hits (layer l at [layer_begin[l], layer_begin[l+1])) and seeds.
 * Host pointers. cpcm: strip charge per cm as given to Hit::setupAsStrip,
 * negative for pixel hits (Hit.h:285-300); detid: 12-bit module id in the
 * layer. Seed hits: [n_seeds][seed_hit_stride] (layer, index within
 * layer), seed_nhits of them valid; seed_hit_stride 0 means 4, at most
 * MKFG_MAX_SEED_HITS (seeds merged by the seed cleaning carry up to 15). */
#define MKFG_MAX_SEED_HITS 16
typedef struct {
  int32_t n_layers;
  const int32_t* layer_begin;
  const float* pos; /* [3][n_hits] */
  const float* err; /* [6][n_hits] */
  const int32_t* detid;
  const int32_t* cpcm;
  int32_t n_seeds;
  const float* seed_par; /* [6][n_seeds] */
  const float* seed_err; /* [21][n_seeds] */
  const int32_t* seed_chg;
  const int32_t* seed_nhits;
  const int32_t* seed_hit_layer;
  const int32_t* seed_hit_index;
  int32_t seed_hit_stride;
  /* Hits that earlier iterations used, which the search skips
   * (IterationMaskIfc: one flag per hit, layer by layer in the order of
   * pos; 1 = masked), or NULL. */
  const uint8_t* hit_mask;
} mkfg_event;

/* Finding output, indexed by input seed; m = max_cands_per_seed slots per
 * seed, best first (after MergeCandsAndBestShortOne). Host pointers; any
 * may be NULL to skip. Hit lists: [n_seeds*m][64] (index, layer), unused
 * entries -100. */
typedef struct {
  int32_t* n_cands;
  int32_t* region;
  float* par;  /* [n_seeds*m][6] */
  float* err;  /* [n_seeds*m][21] */
  int32_t* chg;
  float* chi2;
  float* score;
  int32_t* nfound;
  int32_t* ntot;
  int32_t* noverlap;
  int32_t* ninside;
  int32_t* ntail;
  int32_t* hit_idx;
  int32_t* hit_lyr;
} mkfg_find_out;

/* Plain form, the drop-in for MkBuilder::find_tracks_load_seeds +
 * FindTracksCloneEngine (mkFit/MkBuilder.cc:1491-1501, 1847-2058) on one
 * event: upload (host hit-index build as LayerOfHits::SuckInHits and seed
 * partition as import_seeds), run (one launch sequence per layer step),
 * download (export of all candidates, as TrackCand::exportTrack). */
int mkfg_find_upload(mkfg_context* ctx, const mkfg_event* ev);
/* Batched form: n_events events uploaded together and found by the same
 * launches (or graph replay); mkfg_find_download then returns the seeds of
 * all events concatenated in event order (n_seeds = the total). No
 * reference counterpart: the reference runs events in separate threads
 * (mkFit/mkFit.cc:308-425). */
int mkfg_find_upload_batch(mkfg_context* ctx, const mkfg_event* evs, int32_t n_events);
int mkfg_find_run(mkfg_context* ctx);
/* The same sequence captured once per upload into a CUDA graph and
 * replayed (one graph launch per call). No reference counterpart. */
int mkfg_find_run_graph(mkfg_context* ctx);
/* The plain run with a CUDA event after every launch: kernel_ms[7]
 * receives the device time of each kernel class summed over the layer
 * steps (0 reset, 1 activate, 2 propagate, 3 chi2, 4 clone, 5 update,
 * 6 merge). For per-kernel rooflines. No reference counterpart. */
int mkfg_find_run_timed(mkfg_context* ctx, float* kernel_ms);
/* Per layer-plan step of the last run: launch_ms[max_steps][5] the device
 * time of each step launch of the last mkfg_find_run_timed (activate,
 * propagate, chi2, clone, update), counts[max_steps][7] the work of the
 * last run of any form that fills them (plain, graph, timed): active
 * candidates in barrel / endcap layers, (candidate, hit) pairs barrel /
 * endcap, Kalman updates barrel / endcap, seeds finding. Either pointer may
 * be null. No reference counterpart (diagnostics). */
int mkfg_find_step_profile(mkfg_context* ctx, float* launch_ms, int32_t* counts);
/* Fused form of the same run: one launch in which every thread block carries
 * seeds_per_block consecutive seeds (4, 8 or 16; 0 = the value chosen by
 * mkfg_find_autotune, 16 before any tuning) through all layer steps and the
 * final merge, with the step scratch in shared memory. Same candidates and
 * hit lists as mkfg_find_run; candidate states agree to FP32 rounding (the
 * shared step code may be contracted into FMAs differently). No reference
 * counterpart. */
int mkfg_find_run_fused(mkfg_context* ctx, int32_t seeds_per_block);
/* Times mkfg_find_run_fused on the uploaded events for every supported
 * seeds_per_block, keeps the fastest for later calls with 0, and returns it
 * with its time per run in milliseconds (either pointer may be NULL).
 * Leaves the outputs of a completed run. No reference counterpart. */
int mkfg_find_autotune(mkfg_context* ctx, int32_t* seeds_per_block, float* ms_per_run);
/* Backward fit of every seed's best candidate after a run (plain, graph or
 * fused): from the last layer of the seed's region plan down to plan
 * position bkfit_last[region] (host array, NULL = 0), refit over the
 * candidate's hits with the covariance scaled by 100, chi2 summed;
 * parameters, covariance, chi2 and score of candidate 0 are replaced
 * (mkfg_find_download returns them), its charge is kept. Replaces
 * MkBuilder::BackwardFit / fit_cands (mkFit/MkBuilder.cc:2153-2253) and
 * MkFinder::BkFitInputTracks / BkFitFitTracks / BkFitOutputTracks
 * (mkFit/MkFinder.cc:1368-1452, 1573-1742). pflags: Config::
 * backward_fit_pflags. group_width: the reference's Matriplex width NN
 * (8 for its AVX2 build, 16 for AVX-512; 0 = 8) -- seeds are fitted in
 * groups of that many, whose members share layer skips and stand-in
 * measurements as in the reference. Synchronizes the context stream. */
int mkfg_find_backward_fit(mkfg_context* ctx, const int32_t* bkfit_last, uint32_t pflags,
                           int32_t group_width);
/* Backward search after mkfg_find_backward_fit (run_OneIteration with
 * m_backward_search, mkFit/buildtestMPlex.cc:700-714):
 * CompactifyHitStorageForBestCand without dropping seed hits + BeginBkwSearch
 * (mkFit/HitStructures.cc:554-674), FindTracksCloneEngine(IT_BkwSearch)
 * over each region's plan positions bksearch_pickup[region] .. 0 in reverse
 * (SteeringParams::set_iterator_limits third argument; -1 = no backward
 * plan, seeds left alone), then EndBkwSearch (:676-702) on the best
 * candidate, which mkfg_find_download / _download_best then return with the
 * hits found inward first. The low-pT looper stop does not apply (it is a
 * forward-search rule). Synchronizes the context stream. */
int mkfg_find_backward_search(mkfg_context* ctx, const int32_t* bksearch_pickup);
/* IterationParams of a search (the fields of mkFit/IterationConfig.h:96-104
 * the clone engine reads). */
typedef struct {
  int32_t max_cands_per_seed, max_holes_per_cand, max_consec_holes;
  float chi2_cut_min, chi2_cut_overlap, pt_cut_overlap;
} mkfg_search_params;
/* mkfg_find_backward_search with the iteration's own backward-search
 * parameters (IterationConfig::m_backward_params: pixelLessStep and
 * tobTecStep allow holes there, mkFit/Geoms/CMS-2017.cc
 * SetupBackwardSearch_Iter7/8); NULL = the forward parameters. Seed hits
 * are kept (m_backward_drop_seed_hits off, as in every CMS-2017
 * iteration). */
int mkfg_find_backward_search_with(mkfg_context* ctx, const int32_t* bksearch_pickup,
                                   const mkfg_search_params* params);
/* Output selection of run_OneIteration after a run (and backward fit):
 * every seed's best candidate is dropped if its covariance has a negative
 * diagonal or a non-finite element (StdSeq::qfilter_nan_n_silly with
 * filter_comb_cands, mkFit/MkBuilder.cc:279-314), the rest are compared in
 * pairs within their event and the lower-score track of a duplicate pair
 * is dropped (StdSeq::find_duplicates_sharedhits_pixelseed,
 * mkFit/MkStdSeqs.cc:510-603, used by find_and_remove_duplicates for
 * iterations with m_requires_dupclean_tight). keep[n_seeds] (host, by
 * input seed) receives 1 for the survivors. The config holds the
 * iteration's duplicate parameters (IterationConfig::set_dupl_params) and
 * the reference's window constants (Config::maxd1pt, maxdphi, maxdcth,
 * maxcth_ob, maxcth_fw). */
typedef struct {
  float frac_shared_hits;
  float drth_central, drth_obarrel, drth_forward;
  float max_d_invpt, max_d_phi, max_d_cottheta;
  float max_cottheta_obarrel, max_cottheta_forward;
  /* Which duplicate removal runs (the branch find_and_remove_duplicates
   * takes, mkFit/MkStdSeqs.cc:605-630): MKFG_DUP_PIXELSEED (iterations with
   * m_requires_dupclean_tight), MKFG_DUP_SHAREDHITS
   * (find_duplicates_sharedhits, :456-508: quality-filtered iterations
   * without it; frac_shared_hits only), MKFG_DUP_ETA_PHI (find_duplicates +
   * remove_duplicates, :334-429: the other iterations) or MKFG_DUP_NONE
   * (run_OneIteration's do_remove_duplicates off). */
  int32_t mode;
  /* TrackBase algorithm code of the seeds (find_duplicates leaves tracks of
   * algorithms 9 and 10 alone). */
  int32_t algorithm;
  /* find_duplicates windows: Config::maxdPt (on 1/pT), maxdPhi, maxdEta,
   * maxdR, minFracHitsShared, useHitsForDuplicates (Config.cc:86-91). */
  float ep_max_d_pt, ep_max_d_phi, ep_max_d_eta, ep_max_dr, ep_min_frac_hits_shared;
  int32_t ep_use_hits;
} mkfg_select_config;

#define MKFG_DUP_PIXELSEED 0
#define MKFG_DUP_SHAREDHITS 1
#define MKFG_DUP_ETA_PHI 2
#define MKFG_DUP_NONE 3

int mkfg_find_select(mkfg_context* ctx, const mkfg_select_config* cfg, int32_t n_seeds,
                     int32_t* keep);
/* A quality filter of run_OneIteration on every seed's best candidate, as
 * MkBuilder::filter_comb_cands (mkFit/MkBuilder.cc:279-318) applies it
 * (mkFit/buildtestMPlex.cc:676-724): the StdSeq filter `kind`
 * (mkFit/MkStdSeqs.h:39-148) with min_hits for the hit-count filters and
 * the beam spot for the d0 cuts. pass[n_seeds] (host, by input seed; may be
 * NULL): 1 pass, 0 fail, -1 the seed has no candidate. With `remove`, a
 * failing seed loses its comb candidate: the backward fit (whose seed groups
 * are then formed over the remaining seeds, as in the reference's compacted
 * candidate vector), the backward search, the selection and the downloads
 * see it as empty. A run restores every seed. Synchronizes the stream. */
#define MKFG_QF_NAN_N_SILLY 0       /* qfilter_nan_n_silly */
#define MKFG_QF_N_HITS 1            /* qfilter_n_hits(min_hits) */
#define MKFG_QF_N_HITS_PIXSEED 2    /* qfilter_n_hits_pixseed(min_hits) */
#define MKFG_QF_N_LAYERS 3          /* qfilter_n_layers */
#define MKFG_QF_N_LAYERS_PIXELLESS 4 /* qfilter_n_layers_pixelLess */
#define MKFG_QF_PIXELLESS_FWD 5     /* qfilter_pixelLessFwd */
#define MKFG_QF_PIXELLESS_BKWD 6    /* qfilter_pixelLessBkwd */
typedef struct {
  int32_t kind;
  int32_t min_hits;
  float beam_spot_x, beam_spot_y;
} mkfg_qfilter_config;

int mkfg_find_filter(mkfg_context* ctx, const mkfg_qfilter_config* cfg, int32_t n_seeds,
                     int32_t remove, int32_t* pass);
/* MkFinder::SelectHitIndices (mkFit/MkFinder.cc:227-684) as a plain worker
 * call on the uploaded event `event`: for n states already propagated to
 * layer `layer` (par[6][n], err[21][n], as MkFinder's Par[iP] / Err[iP]),
 * the window from the position covariance and the layer's (dynamic)
 * limits, the sensitive-region test and the bin scan. xhit_size[n]
 * (XHitSize: hits found, at most 16; -1 when the state is outside the
 * layer), xhit_idx[n][16] (XHitArr: hit indices within the layer in scan
 * order, -1 after the last), wsr[n] (may be NULL: 0 inside, 1 edge,
 * 2 outside). Synchronizes the stream. */
int mkfg_find_select_hit_indices(mkfg_context* ctx, int32_t event, int32_t layer, int32_t n,
                                 const float* par, const float* err, int32_t* xhit_size,
                                 int32_t* xhit_idx, int32_t* wsr);

/* Counters of the candidates a per-layer worker call takes: the TrackCand
 * fields MkFinder::copy_in loads (mkFit/MkFinder.h:269-289). Host arrays
 * of n entries. */
typedef struct {
  const int32_t* nfound;  /* nFoundHits */
  const int32_t* nover;   /* nOverlapHits */
  const int32_t* ninside; /* nInsideMinusOneHits */
  const int32_t* ntail;   /* nTailMinusOneHits */
  const float* chi2;      /* chi2 */
} mkfg_cand_counts;

/* Records a candidate can hand to the cloner on one layer: up to 16 hits
 * and one hole. */
#define MKFG_REC_PER_CAND 17

/* IdxChi2List records (Track.h:28-42) of one worker call, [n][17] each,
 * entries past n[i] zero. hit: index within the layer, or the hole code
 * (-1 hole, -2 stop, -3 edge); module: the hit's detIDinLayer (-1 for the
 * hole); chi2: chi2_hit; score: getScoreStruct of the record. */
typedef struct {
  int32_t* n;
  int32_t* hit;
  int32_t* module;
  float* chi2;
  float* score;
} mkfg_ce_records;

/* MkFinder::FindCandidatesCloneEngine (mkFit/MkFinder.cc:1116-1284) as a
 * plain worker call on uploaded event `event`: for n candidates whose
 * states are propagated to layer `layer` (par[6][n], err[21][n], chg[n], as
 * Par[iP] / Err[iP]) with their counters, and the hit lists
 * mkfg_find_select_hit_indices gave for them (xhit_size[n],
 * xhit_idx[n][16], wsr[n]), the records each candidate hands to the
 * cloner, in the order it hands them: its accepted hits in xhit_idx order
 * (chi2 of kalmanPropagateAndComputeChi2 under the dynamic cut, strip
 * compatibility and charge, the pixel same-layer check), then the hole
 * record unless wsr says outside. seed_hot_layers[n][3] (may be NULL: no
 * pixel check): layers of the comb candidate's first three hit-on-track
 * nodes, -1 where it has none. The inactive-module code -7 is never
 * produced (no module is inactive). Host arrays; a hit index outside the
 * layer is refused with MKFG_ERR_BAD_INPUT. Synchronizes the stream. */
int mkfg_find_candidates_clone_engine(mkfg_context* ctx, int32_t event, int32_t layer, int32_t n,
                                      const float* par, const float* err, const int32_t* chg,
                                      const mkfg_cand_counts* counts,
                                      const int32_t* seed_hot_layers, const int32_t* xhit_size,
                                      const int32_t* xhit_idx, const int32_t* wsr,
                                      mkfg_ce_records* out);

/* MkFinder::UpdateWithLastHit + CopyOutParErr (mkFit/MkFinder.cc:
 * 1291-1335) as a plain worker call on uploaded event `event`: n states
 * (par[6][n], err[21][n], chg[n], as Par[iP]) propagated to their hit on
 * layer `layer` (hit_idx[n], index within the layer) with the finding's
 * inter-layer flags and updated (kalmanPropagateAndUpdate[Endcap]), the
 * charge flipped where 1/pT turns negative. Host arrays; in and out may
 * alias. Synchronizes the stream. */
int mkfg_find_update_with_last_hit(mkfg_context* ctx, int32_t event, int32_t layer, int32_t n,
                                   const float* par, const float* err, const int32_t* chg,
                                   const int32_t* hit_idx, float* out_par, float* out_err,
                                   int32_t* out_chg);

/* Hit index of a new candidate that added no hit of its own (a held-back
 * copy). */
#define MKFG_NO_HIT (-100000)

/* Seeds in Finding state at one layer, as CandCloner::ProcessSeedRange
 * takes them. Candidate slot k = 8 * seed + c, c < n_cands[seed] (at most
 * the finder's maxCandsPerSeed); arrays of 8 * n_seeds entries
 * ([6][8 n_seeds] and [21][8 n_seeds] for par / err), records
 * [8 n_seeds][17] in the mkfg_ce_records layout, at most 16 hits and one
 * hole per candidate. held_back: 0 searched on this layer, 1 held
 * back as it is, 2 held back with a stop (-2) node added
 * (MkBuilder::find_tracks_handle_missed_layers, mkFit/MkBuilder.cc:
 * 1568-1637). A best short candidate exists where bshort_valid is set,
 * with score bshort_score. Host arrays. */
typedef struct {
  int32_t n_seeds;
  const int32_t* n_cands;
  const float* par;
  const float* err;
  const int32_t* chg;
  const float* chi2;
  const float* score;
  const int32_t* nfound;
  const int32_t* nmiss;
  const int32_t* nover;
  const int32_t* ninside;
  const int32_t* ntail;
  const int32_t* held_back;
  const int32_t* n_rec;
  const int32_t* rec_hit;
  const int32_t* rec_module;
  const float* rec_chi2;
  const float* rec_score;
  const int32_t* bshort_valid;
  const float* bshort_score;
} mkfg_clone_in;

/* The seeds after the clone step: n_cands, and per new candidate slot
 * (same layout as the input) its state and counters, parent (input slot c
 * it was made from), hit (the hit or hole code it added, MKFG_NO_HIT for
 * a held-back copy), overlap_hit (the overlap hit it added, -1 none),
 * update_hit (the hit UpdateWithLastHit must use, -1 when it takes no
 * update); slots past n_cands hold parent -1. The best short candidate per
 * seed: valid flag, score (-1e16, getScoreWorstPossible, when not valid),
 * found hits and chi2. */
typedef struct {
  int32_t* n_cands;
  float* par;
  float* err;
  int32_t* chg;
  float* chi2;
  float* score;
  int32_t* nfound;
  int32_t* nmiss;
  int32_t* nover;
  int32_t* ninside;
  int32_t* ntail;
  int32_t* parent;
  int32_t* hit;
  int32_t* overlap_hit;
  int32_t* update_hit;
  int32_t* bshort_valid; /* [n_seeds] */
  float* bshort_score;   /* -1e16 (getScoreWorstPossible) when not valid */
  int32_t* bshort_nfound;
  float* bshort_chi2;
} mkfg_clone_out;

/* CandCloner::ProcessSeedRange (mkFit/CandCloner.cc:36-189) as a plain
 * worker call for layer `layer`, with the configured finder's cuts
 * (maxCandsPerSeed, chi2CutOverlap, pTCutOverlap): per seed the records
 * ranked by score, the top maxCandsPerSeed taken, stop (-2) records
 * offered to the best short candidate, held-back candidates merged in by
 * score, the overlap hit of the parent's best pair appended (pT above the
 * cut), the update list formed. Exact score ties are ranked by record
 * position (candidate, then hand-over order), the order std::sort leaves
 * when it keeps them. Needs mkfg_finder_setup, no event. Synchronizes. */
int mkfg_find_clone_seeds(mkfg_context* ctx, int32_t layer, const mkfg_clone_in* in,
                          mkfg_clone_out* out);
/* The hit index the upload built on the device for uploaded event `event`
 * (LayerOfHits after SuckInHits / EndRegistrationOfHits,
 * mkFit/HitStructures.cc:77-338): bins in the layout of
 * mkfg_prepare_event_host, and srank for the event's hits; either may be
 * NULL. For checking the device build against the host one. */
int mkfg_find_hit_index(mkfg_context* ctx, int32_t event, uint32_t* bins, int32_t* srank);
/* Work done by the last run (for FLOP accounting): candidate propagations
 * to a layer, (candidate, hit) chi2 evaluations, Kalman updates, and the
 * number of layer-plan steps. No reference counterpart. */
int mkfg_find_work(mkfg_context* ctx, int64_t* active_cands, int64_t* hit_pairs,
                   int64_t* updates, int32_t* steps);
/* Diagnostics of the last mkfg_find_work call: chi2 evaluations counted by
 * the chi2 kernel, seed-steps handled by the clone kernel. */
int mkfg_find_work_detail(mkfg_context* ctx, int64_t* chi2_evals, int64_t* seeds_cloned);

/* Hit-on-track arena of the following uploads: nodes_per_seed nodes per
 * seed (at least MKFG_MAX_SEED_HITS + 2), or 0 to size it for the
 * configured plans (the default, which no run exceeds). A search that
 * needs more nodes than the arena holds keeps the nodes it has, drops the
 * rest and makes the next download return MKFG_ERR_OVERFLOW, with every
 * output still written; the reference's CcPool throws std::bad_alloc
 * instead (mkFit/HitStructures.h:428-435). */
int mkfg_find_set_arena_capacity(mkfg_context* ctx, int32_t nodes_per_seed);

/* Where the following uploads import the seeds (MkBuilder::import_seeds
 * with the CMS-2017 partition, mkFit/MkBuilder.cc:214-275, and
 * CombCandidate::ImportSeed): on_host = 0 (the default) on the device --
 * region, eta order and initial candidates computed there, so the host
 * only copies the seeds as given -- or 1 on the host's worker threads.
 * Both give the same candidates. The upload uses the host whatever the
 * setting for iterations that sort seed hits first (pixelLessStep), for an
 * event of more than 16384 seeds, and for a seed whose last hit is not
 * one of its event's hits. */
int mkfg_find_set_seed_import(mkfg_context* ctx, int32_t on_host);

/* on = 1: the propagation kernel of the following runs copies, per chunk
 * of 256 active candidates, the (q bin, phi bin) table of the chunk's
 * first (event, layer) into shared memory with one bulk copy (TMA,
 * cp.async.bulk + mbarrier) and scans it there; 0 (the default): every
 * candidate reads the table from global memory. Same results either way
 * (LayerOfHits::m_phi_bin_infos, mkFit/HitStructures.h:152-159; the bin
 * loop of MkFinder::SelectHitIndices, mkFit/MkFinder.cc:464-466). No
 * reference counterpart. */
int mkfg_find_set_bin_staging(mkfg_context* ctx, int32_t on);

/* Launch configuration of the graph form's list-driven kernels: grid of
 * the propagation, chi2, clone and update kernels as a multiple of the
 * blocks the device keeps resident for each (grid_mult[4]), and the bin
 * staging of mkfg_find_set_bin_staging. ms_before / ms_after: the step
 * time (sum of the per-launch device times of one run) before and after
 * a tuning. No reference counterpart. */
typedef struct {
  int32_t grid_mult[4];
  int32_t stage_bins;
  float ms_before;
  float ms_after;
} mkfg_graph_tuning;

/* Tunes the launch configuration on the uploaded batch: each kernel's
 * grid multiple in turn over 1 .. 16 by its own device time (each setting
 * timed `reps` times, the minimum kept), then the bin staging by the
 * propagation kernel's time; the choice stays with the context for its
 * following runs and is returned in *out (may be NULL). The results of a
 * run do not depend on these settings. */
int mkfg_find_autotune_graph(mkfg_context* ctx, int32_t reps, mkfg_graph_tuning* out);
/* Sets or reads the launch configuration (e.g. one a caller kept from an
 * earlier tuning). */
int mkfg_find_set_graph_tuning(mkfg_context* ctx, const mkfg_graph_tuning* t);
int mkfg_find_get_graph_tuning(mkfg_context* ctx, mkfg_graph_tuning* t);

/* Clone-step counters of the last mkfg_find_work call: the records
 * (IdxChi2List entries, hits and holes) present when the seeds were ranked
 * and the new candidates written. Counted by the eager run (mkfg_find_run)
 * only; zero after a graph replay. Diagnostic; no reference counterpart
 * (the reference's CandCloner keeps no such totals). */
int mkfg_find_work_clone(mkfg_context* ctx, int64_t* records, int64_t* new_cands);
int mkfg_find_download(mkfg_context* ctx, int32_t n_seeds, mkfg_find_out* out);
/* The same export for the best candidate of every seed only (m = 1 slot
 * per seed in every output array; n_cands[s] = 1 when the seed has a
 * candidate): replaces MkBuilder::export_best_comb_cands
 * (mkFit/MkBuilder.cc:348-362, called by run_OneIteration,
 * mkFit/buildtestMPlex.cc:734). Hit lists keep the missing-hit entries
 * (negative indices), as exportTrack(false); a caller that wants
 * remove_missing_hits drops them. */
int mkfg_find_download_best(mkfg_context* ctx, int32_t n_seeds, mkfg_find_out* out);
int mkfg_find_event(mkfg_context* ctx, const mkfg_event* ev, mkfg_find_out* out);

/* Host-only (no device needed): the hit-index build and seed ordering that
 * mkfg_find_upload performs, for inspection and tests. bins: all layers'
 * (q bin x 256 phi bin) entries (first | last << 16), layer after layer;
 * *n_bins receives the count (pass bins = NULL to query it). srank[n_hits]:
 * per sorted position (layer by layer) the hit's index within its layer
 * (LayerOfHits::GetOriginalHitIndex). seed_order[n_seeds]: input seed at
 * each sorted position; seed_region[n_seeds]: eta region per input seed. */
int mkfg_prepare_event_host(const mkfg_find_config* cfg, const mkfg_event* ev, uint32_t* bins,
                            int32_t* n_bins, int32_t* srank, int32_t* seed_order,
                            int32_t* seed_region);

#ifdef __cplusplus
}
#endif

#endif /* MKFIT_B200_H */
