/*
 * drmppi.h — C ABI of the B200-native MPPI / PR-MPPI control step for the
 * drone-race StratRace environment.
 *
 * This is the drop-in boundary for the reference's controller layer:
 *   class Controller { virtual void getControl(const SimState&, float* outAction) = 0; ... }
 *   (reference: include/controllers.h:12-21), with the two concrete controllers
 *   MPPIController  (include/controllers.h:23-111, src/mppi_controller.cu:15-514) and
 *   PRMPPIController (include/controllers.h:114-179, src/prmppi_controller.cu:14-349).
 *
 * Every entry point returns an int status (DR_OK == 0) and never throws. Pointers are
 * host pointers unless a name ends in `_dev`. Nothing here takes a torch type.
 *
 * Compile-time sizes of the reference (N_OPP, N_TRUE_MODELS, USE_SPLINES, ...) are
 * runtime fields here; supported combinations are listed in dr_supported().
 * The model has one parameter factor (reference N_MODEL_FACTORS = 1,
 * include/environments/env_stratrace_defs.h:17), so the number of branch plans is
 * n_theta + 1 (reference N_BRANCH_PLANS = BRANCH_SIZE(0)).
 */
#ifndef DRMPPI_H
#define DRMPPI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DR_ABI_VERSION 2

#define DR_DIM 2             /* reference EnvStratRace::DIM == ACTION_DIM (env_stratrace_defs.h:9,15) */
#define DR_MAX_OPP 3         /* reference N_OPP (compile-time 1, env_stratrace_defs.h:10) */
#define DR_MAX_AGENTS 4      /* N_OPP + 1 */
#define DR_MAX_THETA 8       /* reference N_TRUE_MODELS (compile-time 2) */
#define DR_MAX_KNOTS 64      /* reference MAX_N_KNOTS = 60 (include/config.h:27) */
#define DR_MAX_T 256         /* longest horizon accepted (dense mode: nKnots = nTimesteps) */
#define DR_GRAD_MAX_STEPS 8  /* gradient steps of the refinement (dr_mppi_set_grad_refine) */
#define DR_GRAD_WEIGHTS 6    /* cost weights the gradient path differentiates (dr_mppi_nominal_grad) */
#define DR_N_TRACK_SAMPLES 512 /* reference N_TRACK_SAMPLES (env_stratrace_defs.h:11) */

/* Status codes. */
enum dr_status
{
    DR_OK = 0,
    DR_ERR_INVALID_ARG = 1,  /* bad pointer, size or config value (reference throws std::runtime_error) */
    DR_ERR_UNSUPPORTED = 2,  /* (n_opp, n_theta) combination not compiled in */
    DR_ERR_CUDA = 3,         /* a CUDA runtime call failed; dr_last_error() has the text */
    DR_ERR_OOM = 4,          /* device allocation failed */
    DR_ERR_NO_DEVICE = 5,    /* no usable CUDA device */
    DR_ERR_TIMEOUT = 6,      /* a bounded device-side wait gave up */
    DR_ERR_STATE = 7,        /* call out of order (e.g. engine not set) */
};

/* Per-hypothesis opponent policy parameters (reference OppConfig,
 * env_stratrace_defs.h:42-50). Arrays are indexed by opponent 0..n_opp-1. */
typedef struct dr_opp_config
{
    float s1[DR_MAX_OPP];
    float s2[DR_MAX_OPP];
    float s3[DR_MAX_OPP];
    float speed_scale[DR_MAX_OPP];
    float action_noise[DR_MAX_OPP];
} dr_opp_config;

/* Environment (reference EnvironmentConfig, env_stratrace_defs.h:53-86; wire order of
 * src/environments/env_stratrace.cpp:135-226). Agent 0 is the controlled (ego) agent.
 * The four track grids are HOST pointers to DR_N_TRACK_SAMPLES samples each
 * ([512][2] for p/dp/t, [512] for kappa); they are copied at create time. */
typedef struct dr_env_config
{
    int32_t n_opp;   /* 1..DR_MAX_OPP */
    int32_t n_theta; /* 1..DR_MAX_THETA */
    float arena_min[DR_DIM];
    float arena_max[DR_DIM];
    float dt;
    int32_t send_states;
    float drone_radius;
    float pos_noise_level;
    float speed_noise_level;
    float action_noise_level;
    float max_speed[DR_MAX_AGENTS];
    float max_accel[DR_MAX_AGENTS];
    float track_width;
    int32_t n_win_laps;
    float init_belief[DR_MAX_THETA];
    dr_opp_config opp_configs[DR_MAX_THETA];
    float kP;
    float kV;
    float max_opp_lat_dist_fact;
    float track_length;
    const float* p_grid;
    const float* dp_grid;
    const float* t_grid;
    const float* kappa_grid;
} dr_env_config;

/* Simulation state (reference SimState, env_stratrace_defs.h:88-96). Only the first
 * n_opp + 1 agents are used. */
typedef struct dr_sim_state
{
    float pos[DR_MAX_AGENTS * DR_DIM];
    float vel[DR_MAX_AGENTS * DR_DIM];
    float S[DR_MAX_AGENTS];
    float lat_dist[DR_MAX_AGENTS];
    int32_t laps[DR_MAX_AGENTS];
} dr_sim_state;

/* MPPI configuration (reference MPPIConfig, include/config.h:116-154; wire order of
 * src/config.cpp:5-53). Fields after max_verif_eps are extensions. */
typedef struct dr_mppi_config
{
    int32_t n_samples;
    int32_t n_timesteps;
    int32_t n_knots;                /* spline mode: M knots; dense mode: ignored (M = T) */
    int32_t knots[DR_MAX_KNOTS];    /* tau_i, strictly increasing, tau_{M-1} <= T-2 */
    int32_t use_splines;            /* reference compile-time USE_SPLINES (include/config.h:25) */
    float inv_temperature;          /* used as a temperature: w = exp(-(c-min)/inv_temperature) */
    float sampling_noise;           /* stddev of the control perturbation */
    float gate_traversal_margin;    /* carried for wire compatibility; unused by the model */
    float coll_dist_factor;
    float boundary_cost;
    float boundary_threshold_factor;
    float outside_cost;
    float win_cost;
    float opp_win_cost;
    float final_adv_weight;
    float final_opp_adv_weight;
    float min_confidence;
    int32_t n_verif_samples;
    float beta;
    int32_t verif_horizon;          /* must be <= n_timesteps */
    float max_verif_eps;
    /* extensions (not in the reference; defaults keep reference behaviour) */
    float sampling_noise_dim[DR_DIM]; /* per-dimension stddev; 0 => use sampling_noise */
    float min_nu;                   /* reference MPPIController::min_nu = 0.0005 (controllers.h:47) */
    float max_nu;                   /* reference MPPIController::max_nu = 0.001 (controllers.h:48) */
    int32_t verify;                 /* 1 (reference) = run plan verification; 0 = always use the new plan */
} dr_mppi_config;

/* PR-MPPI configuration (reference PRMPPIConfig, include/config.h:157-192; wire order
 * of src/config.cpp:55-84). */
typedef struct dr_prmppi_config
{
    int32_t n_samples;
    int32_t n_timesteps;
    float inv_temperature;
    float sampling_noise;
    float gate_traversal_margin;
    float coll_dist_factor;
    float boundary_cost;
    float boundary_threshold_factor;
    float win_cost;
    float opp_win_cost;
    float final_adv_weight;
    float final_opp_adv_weight;
    float safety_weight;
    float min_safe_dist;
    float delta;
    int32_t P;                      /* number of sampled hypotheses */
    /* extensions */
    float sampling_noise_dim[DR_DIM];
    float min_nu;
    float max_nu;
} dr_prmppi_config;

/* Per-step outputs of an MPPI controller; mirrors the public fields the reference
 * engine reads (src/engine.cpp:75-117). */
typedef struct dr_mppi_info
{
    uint32_t fail_count_total;   /* sum of the chosen plan's failCount (engine.cpp:77) */
    int32_t use_new_plan;
    double epsilon;
    double epsilon_partial;
    double certified_loss;
    int32_t branch_idx;          /* branch whose first action was sent */
    float min_cost;              /* minCosts[branch_idx][0] */
    float nu;                    /* nu[branch_idx] */
    float inv_temperature;       /* temperature after this step's adaptation */
    int32_t nonfinite_costs;     /* number of samples whose cost was not finite */
    int32_t verif_timeouts;      /* CTAs (rollout or verification) whose bounded staging wait gave up;
                                    the step then returns DR_ERR_TIMEOUT */
    /* gradient refinement (dr_mppi_set_grad_refine; no counterpart in the reference) */
    float grad_cost_plain;       /* objective of the plain MPPI update */
    float grad_cost_refined;     /* objective of the plan kept (<= grad_cost_plain) */
    int32_t grad_best_step;      /* gradient steps in the plan kept (0: the plain update), -1 when off */
} dr_mppi_info;

/* Per-step outputs of a PR-MPPI controller (src/engine.cpp:171-212). */
typedef struct dr_prmppi_info
{
    int32_t use_nom_plan;
    int32_t reset_nom;
    float cand_cost[2];          /* averaged full cost of cand1 / cand2 */
    float min_costs[3];          /* nom_full, rob_full, rob_safe */
    float nu[3];
    float inv_temperature[3];    /* after this step's adaptation */
    int32_t nonfinite_costs;
} dr_prmppi_info;

typedef struct dr_mppi dr_mppi;
typedef struct dr_prmppi dr_prmppi;
typedef struct dr_mppi_batch dr_mppi_batch;
typedef struct dr_prmppi_batch dr_prmppi_batch;

/* ---- library ------------------------------------------------------------------ */
int dr_abi_version(void);
/* 1 if (n_opp, n_theta) is compiled in. */
int dr_supported(int n_opp, int n_theta);
/* Text of the last error on this thread ("" if none). */
const char* dr_last_error(void);
const char* dr_status_string(int status);

/* ---- MPPI controller (reference MPPIController) --------------------------------- */
/* nominal: n_theta+1 branch plans x n_timesteps x DR_DIM, or NULL for zeros
 * (controllers.h:26-29; mppi_controller.cu:25-34). stream: cudaStream_t or NULL for a
 * stream owned by the controller. */
int dr_mppi_create(const dr_env_config* env, const dr_mppi_config* cfg, uint64_t seed, const float* nominal, int device, void* stream,
                   dr_mppi** out);
int dr_mppi_destroy(dr_mppi* h);
/* One control step (reference MPPIController::getControl, mppi_controller.cu:250-466).
 * belief: n_theta floats. out_action: DR_DIM floats. info may be NULL. Blocks until done. */
int dr_mppi_step(dr_mppi* h, const dr_sim_state* state, const float* belief, float* out_action, dr_mppi_info* info);
/* Host mirror of the dense nominal (reference h_nominal, (n_theta+1) x T x DR_DIM). */
int dr_mppi_get_nominal(const dr_mppi* h, float* out, size_t n);
/* Spline knots currently on the device ((n_theta+1) x M x DR_DIM; dense mode: x T). */
int dr_mppi_get_knots(dr_mppi* h, float* out, size_t n);
/* failCount arrays of the last step (n_timesteps each): new plan, previous plan, chosen. */
int dr_mppi_get_fail_counts(const dr_mppi* h, uint32_t* fc_new, uint32_t* fc_old, uint32_t* fc_chosen, size_t n);
float dr_mppi_get_temperature(const dr_mppi* h);
int dr_mppi_set_temperature(dr_mppi* h, float inv_temperature);
/* Control-step counter (it keys the Philox streams); settable for deterministic replay. */
uint64_t dr_mppi_get_step(const dr_mppi* h);
/* Bytes copied host->device and device->host by one dr_mppi_step of this controller. */
int dr_mppi_io_bytes(const dr_mppi* h, size_t* h2d, size_t* d2h);
int dr_mppi_set_step(dr_mppi* h, uint64_t step);
/* Per-kernel device time (ms) of the last step, measured with CUDA events on the
 * controller's stream when profiling is on. names/ms arrays of capacity n. */
int dr_mppi_set_profiling(dr_mppi* h, int on);
/* Average per-kernel ms over the steps recorded since profiling was switched on. */
int dr_mppi_get_kernel_times(dr_mppi* h, const char** names, float* ms, int n, int* count);

/* Batched step: n controllers on one device advanced by one launch sequence
 * (all agents x samples in one grid). states: n; beliefs: n x DR_MAX_THETA;
 * out_actions: n x DR_DIM; infos: n or NULL. */
int dr_mppi_batch_create(dr_mppi* const* hs, int n, void* stream, dr_mppi_batch** out);
int dr_mppi_batch_destroy(dr_mppi_batch* b);
int dr_mppi_batch_step(dr_mppi_batch* b, const dr_sim_state* states, const float* beliefs, float* out_actions, dr_mppi_info* infos);
/* Device-resident variant for throughput measurement: states/beliefs already on the
 * device (n records), results stay on the device; no host synchronisation. */
int dr_mppi_batch_step_dev(dr_mppi_batch* b, const dr_sim_state* states_dev, const float* beliefs_dev);
int dr_mppi_batch_set_graph(dr_mppi_batch* b, int use_graph);
/* Fully device-resident control step: the host tail of getControl (mppi_controller.cu:
 * 363-456: Clopper-Pearson certification, plan choice, epsilon, branch, temperature,
 * warm-start shift) runs on the device too. states_dev (n dr_sim_state, or n
 * dr_gate_state for a gate-race batch) and beliefs_dev (n x DR_MAX_THETA) are read from
 * device memory; actions_dev (n x DR_DIM) and infos_dev (n) are written to device memory.
 * Enqueued on the batch's stream without waiting; replayed from a CUDA graph while the
 * four pointers stay the same. The controller state carried from step to step stays on
 * the device; the host mirrors (dr_mppi_get_nominal, fail counts) are not refreshed by
 * it. A later host step (dr_mppi_batch_step, dr_mppi_step) first copies that state back. */
int dr_mppi_batch_step_device(dr_mppi_batch* b, const void* states_dev, const float* beliefs_dev, float* actions_dev, dr_mppi_info* infos_dev);
/* True-dynamics step of every controller's race on the device (engine dynStep,
 * engine.cpp:286-312): states_dev (n dr_sim_state, or n dr_gate_state for a gate-race
 * batch) and beliefs_dev (as above) advanced in place with actions_dev under
 * true_theta_dev (n); terms_dev (n) receives the terminal type. The noise is the Philox
 * stream that dr_env_step / dr_gate_env_step (seed, step) draw, at each controller's step
 * counter (its number of control steps so far). After a dr_mppi_batch_step_device; no
 * host synchronisation. */
int dr_mppi_batch_env_step_device(dr_mppi_batch* b, const int32_t* true_theta_dev, const float* actions_dev, void* states_dev, float* beliefs_dev,
                                  int update_belief, uint64_t seed, int32_t* terms_dev);
/* Per-kernel device time of the batch's steps (CUDA events on its stream), averaged
 * over the steps recorded since profiling was switched on (also for *_step_dev). */
int dr_mppi_batch_set_profiling(dr_mppi_batch* b, int on);
/* 1 (default): the previous plan's verification runs on a second stream concurrently
 * with the rollout and the update; 0: everything in order on the batch's stream. */
int dr_mppi_batch_set_overlap(dr_mppi_batch* b, int on);
/* 1 (default): the step's critical path runs on an internal stream of the device's highest
 * priority and the side verification on one of the lowest; 0: both at the batch stream's
 * and the side stream's default priorities (for measurement). */
int dr_mppi_batch_set_priority(dr_mppi_batch* b, int on);
/* Launch shape of the rollout and the verification (strategic race batches). 0 (default):
 * one CTA per tile. n > 0: a persistent launch of n CTAs per SM that take tiles from a
 * device work queue until every controller's tiles are done; -1: as many CTAs per SM as
 * fit. rollout_lockstep 1: the rollout threads of a CTA take a barrier every step (the
 * verification always does). The tile tables list the longest tiles first in both shapes;
 * results are the same in every shape. verify_ctas_per_sm applies to the new plan's
 * verification (and to both plans when they run in one launch); the previous plan's beside
 * the rollout has its own shape (dr_mppi_batch_set_side_verify). A gate-race batch accepts
 * only 0, 0, 0
 * (DR_ERR_UNSUPPORTED otherwise). No counterpart in the reference, which launches one
 * controller's kernels at a time. */
int dr_mppi_batch_set_persistent(dr_mppi_batch* b, int rollout_ctas_per_sm, int verify_ctas_per_sm, int rollout_lockstep);
/* Shape of the previous plan's verification when it runs beside the rollout and the update
 * (dr_mppi_batch_set_overlap 1): 0 (default) one CTA per tile; n > 0 a persistent grid of n
 * CTAs per SM fed by the device work queue, which leaves room on every SM for the step's
 * critical path but verifies more slowly; -1 as many as fit. Results are the same.
 * Strategic race batches (a gate-race batch accepts only 0). No counterpart in the
 * reference. */
int dr_mppi_batch_set_side_verify(dr_mppi_batch* b, int ctas_per_sm);
/* 1: the update and the new plan's verification are launched as programmatic dependents
 * of the kernel before them (their CTAs are dispatched as SM slots free up and wait in the
 * kernel for its results); 0 (default): plain launches. Results are the same. No
 * counterpart in the reference. */
int dr_mppi_batch_set_pdl(dr_mppi_batch* b, int on);
#define DR_TUNE_MAX_CANDIDATES 12
/* What dr_mppi_batch_autotune measured and chose. Candidate values: CTAs per SM of a
 * persistent launch (0 = one CTA per tile) for the rollout and the verification; the
 * adjoint's checkpoint stride for the gradient refinement (0 = the default policy). */
typedef struct dr_tune_report
{
    int rollout_ctas_per_sm; /* chosen */
    int rollout_lockstep;    /* chosen */
    int verify_ctas_per_sm;  /* chosen */
    int grad_ckpt;           /* chosen (0 when no controller of the batch refines) */
    int n_rollout, n_verify, n_grad;
    int rollout_cand[DR_TUNE_MAX_CANDIDATES];
    int rollout_lock[DR_TUNE_MAX_CANDIDATES];
    float rollout_ms[DR_TUNE_MAX_CANDIDATES]; /* median device time of one launch */
    int verify_cand[DR_TUNE_MAX_CANDIDATES];
    float verify_ms[DR_TUNE_MAX_CANDIDATES];
    int grad_cand[DR_TUNE_MAX_CANDIDATES];
    float grad_ms[DR_TUNE_MAX_CANDIDATES];
} dr_tune_report;
/* Times the launch-shape candidates of this batch on its current inputs (`reps` timed
 * launches each after one untimed one, CUDA events on the batch stream) and keeps the
 * fastest: rollout grid (one CTA per tile, or the fullest persistent grids) with and
 * without lockstep, verification grid (one CTA per tile, or 1..max persistent CTAs per
 * SM) and, for controllers with gradient refinement, the checkpoint stride (every state
 * kept when it fits, ceil(sqrt T), 2 ceil(sqrt T)). A candidate replaces the default (timed
 * first) only when it is more than 2 % faster. None of the choices changes a result.
 * The timed launches write only per-step scratch (costs, failure histograms, gradient
 * statistics), which the next step overwrites; the controllers' plans and state are not
 * touched. Needs one completed step of the batch (DR_ERR_STATE before). `out` may be NULL.
 * No counterpart in the reference. */
int dr_mppi_batch_autotune(dr_mppi_batch* b, int reps, dr_tune_report* out);
int dr_mppi_batch_get_kernel_times(dr_mppi_batch* b, const char** names, float* ms, int n, int* count);
/* The schedule of the recorded steps: for each timed kernel (the critical-path stream's
 * and the previous-plan verification stream's), its start and end in ms after the start
 * of the step (CUDA events; averages over the recorded steps). Kernels of the two
 * streams overlap where the device ran them concurrently. No counterpart in the reference. */
int dr_mppi_batch_get_kernel_timeline(dr_mppi_batch* b, const char** names, float* start_ms, float* end_ms, int n, int* count);

/* ---- gradient path (no counterpart in the reference) -----------------------------
 * The objective of an MPPI controller's noise-free rollout of the control sequence U
 * (the spline knots, or the dense controls; (n_theta+1) x M x DR_DIM floats), rolled out
 * as fullRolloutKernel does (kernels.cu:34-171: branch plans switched on the belief
 * threshold, DECAY-discounted stateCost plus finalCost, costs.cuh:7-39) with every noise
 * source off, under each hypothesis compatible with the current commitment, averaged
 * with the belief weights as aggregateBranchCostsKernel averages (kernels.cu:175-217).
 * Strategic race only.
 *
 * dr_mppi_nominal_grad: for n start points knots_dev [n][(n_theta+1)][M][DR_DIM] and
 * cost weights weights_dev [n][DR_GRAD_WEIGHTS] (NULL: the controller's), in the order
 * boundary_cost, outside_cost, win_cost, opp_win_cost, final_adv_weight,
 * final_opp_adv_weight, writes cost_dev [n], and, where not NULL, the gradients
 * d_knots_dev [n][(n_theta+1)][M][DR_DIM] and d_weights_dev [n][DR_GRAD_WEIGHTS]. All
 * arrays are device memory; the work is enqueued on `stream` (NULL: legacy default)
 * and the call returns without waiting. The adjoint sweep keeps the rollout state every
 * ckpt_stride steps and recomputes between them (1: every state kept, no recomputation;
 * 0: 1 when the states fit in shared memory, else ceil(sqrt(n_timesteps))); the result
 * does not depend on it. Calls on one controller must not run concurrently on different
 * streams. */
int dr_mppi_nominal_grad(dr_mppi* h, const dr_sim_state* state, const float* belief, int n, const float* knots_dev, const float* weights_dev,
                         float* cost_dev, float* d_knots_dev, float* d_weights_dev, int ckpt_stride, void* stream);
/* Gradient-refined MPPI: after each MPPI update, `steps` projected gradient steps on the
 * objective above (each control moves by at most step_size x the ego's max_accel, then
 * the per-knot acceleration clamp); the plan with the lowest objective among the plain
 * update and the gradient iterates is kept. steps = 0 (the default) turns it off;
 * 0 <= steps <= DR_GRAD_MAX_STEPS. ckpt_stride as above. Set it before creating a
 * batch of this controller. */
int dr_mppi_set_grad_refine(dr_mppi* h, int steps, float step_size, int ckpt_stride);

/* ---- sample sharding of one controller across processes (one per GPU) -----------
 * No counterpart in the reference. Process `rank` of `world` rolls out the samples
 * [rank K / world, (rank+1) K / world) and verifies [rank V / world, (rank+1) V / world),
 * with every random stream keyed by the global sample index, so the union over the
 * processes is the single-process workload. Each process reduces its share with its own
 * minimum cost m_r; one all-gather exchanges these partials, and every process merges them
 * the same way, rescaling process r's weighted sums by exp(-(m_r - m) / lambda) to the
 * global minimum m. A step is three calls with two collectives of the caller (e.g.
 * torch.distributed over NCCL, on the controller's stream) in between, on device buffers
 * it owns:
 *   dr_mppi_shard_begin   prologue, previous-plan verification, rollout, and this
 *                         process's partial -> partial_dev (dr_mppi_shard_words words:
 *                         per (branch plan, knot) its masked minimum and its sums
 *                         (w coeff eps0, w coeff eps1, w coeff) with that minimum, then the
 *                         previous plan's failure histogram, T u32)
 *                                         caller: all-gather -> gathered_dev [world][words]
 *   dr_mppi_shard_update  the merge, the update (interpolation, clamp, gradient refinement
 *                         if set), the new-plan verification -> hist_dev (T u32)
 *                                         caller: all-reduce SUM of hist_dev
 *   dr_mppi_shard_finish  the host tail on the summed histograms -> action, info
 * Begin and update only enqueue work on the controller's stream (the caller's
 * collectives must follow it on that stream); finish synchronises. The minima equal the
 * single-process step's; the updated controls agree with it to FP32 rounding (the
 * rescaling rounds differently); every process computes identical results.
 * dr_mppi_step is refused on a sharded controller. */
int dr_mppi_set_shard(dr_mppi* h, int rank, int world);
int dr_mppi_shard_words(const dr_mppi* h, size_t* words);
int dr_mppi_shard_begin(dr_mppi* h, const dr_sim_state* state, const float* belief, float* partial_dev);
int dr_mppi_shard_update(dr_mppi* h, const float* gathered_dev, int world, uint32_t* hist_dev);
int dr_mppi_shard_finish(dr_mppi* h, const uint32_t* hist_dev, const float* belief, float* out_action, dr_mppi_info* info);

/* Sample sharding of one PR-MPPI controller across processes (the reference's
 * PRMPPIController::getControl, prmppi_controller.cu:180-346, split at its reductions).
 * dr_prmppi_set_shard gives process `rank` the samples [rank K / world, (rank+1) K / world)
 * of every hypothesis (all P hypotheses of a sample stay together, so the per-sample
 * averaging over hypotheses is local). Per step, one exchange:
 *   dr_prmppi_shard_begin   prologue (hypotheses drawn alike on every process), rollout of
 *                           this process's samples, its three minima (nominal + full cost,
 *                           robust + full cost, robust + safety) and its weighted sums of
 *                           the absolute controls with them -> partial_dev
 *                           (dr_prmppi_shard_words = 3 + 3 x T x 3 floats)
 *                                         caller: all-gather -> gathered_dev [world][words]
 *   dr_prmppi_shard_finish  the merge (as for MPPI), the weighted averages, the
 *                           candidates' re-check and choice (replicated on every process)
 *                           and the host tail -> action, info
 * Begin only enqueues work on the controller's stream; finish synchronises. The minima
 * equal the single-process step's, the plans agree with it to FP32 rounding;
 * info->nonfinite_costs counts this process's samples. dr_prmppi_step is refused on a
 * sharded controller. */
int dr_prmppi_set_shard(dr_prmppi* h, int rank, int world);
int dr_prmppi_shard_words(const dr_prmppi* h, size_t* words);
int dr_prmppi_shard_begin(dr_prmppi* h, const dr_sim_state* state, const float* belief, float* partial_dev);
int dr_prmppi_shard_finish(dr_prmppi* h, const float* gathered_dev, int world, float* out_action, dr_prmppi_info* info);

/* ---- MPPI test hooks (component parity against the reference kernels) ----------- */
/* Clopper-Pearson bounds (state.h:134-151) of n counts k out of N at level alpha, as the
 * device tail evaluates them (dr_debug_cp) and as the host tail does (dr_debug_cp_host);
 * upper != 0: the upper bound. */
int dr_debug_cp(const uint32_t* k, int n, uint32_t N, double alpha, int upper, double* out);
int dr_debug_cp_host(const uint32_t* k, int n, uint32_t N, double alpha, int upper, double* out);
/* Control perturbation the next step will draw, in the reference layout
 * noise[(n_theta+1)][M][K][DR_DIM] (kernels.cu:28). */
int dr_mppi_debug_noise(dr_mppi* h, float* noise, size_t n);
/* Rollout of the next step on the current knots/nominal (kernels.cu:34-171): costsTrue
 * [n_theta][K], branchUsed/branchTime [n_theta][K], costs [n_theta+1][K] (kernels.cu:175-217). */
int dr_mppi_debug_rollout(dr_mppi* h, const dr_sim_state* state, const float* belief, float* costs_true, int32_t* branch_used,
                          int32_t* branch_time, float* costs);
/* Update only (kernels.cu:221-456) on the given rollout outputs: replaces the device knots
 * (spline mode) or dense nominal and writes the new dense nominal, minCosts
 * [(n_theta+1)][M] and nu [(n_theta+1)]. Uses the same noise as the next step. */
int dr_mppi_debug_update(dr_mppi* h, const float* belief, const float* costs_true, const int32_t* branch_used, const int32_t* branch_time,
                         float* dense_nominal, float* min_costs, float* nu);
/* Verification of a dense plan ((n_theta+1) x T x DR_DIM) from `state`: failCount[T]
 * (kernels.cu:488-551). plan selects the Philox stream (0 new, 1 previous).
 * fail_time (optional, V entries): per-sample failure time or -1. thetas (optional): V. */
int dr_mppi_debug_verify(dr_mppi* h, const dr_sim_state* state, const float* belief, const float* dense_plan, int plan,
                         uint32_t* fail_count, int32_t* fail_time, int32_t* thetas);
/* Arithmetic flavour of this controller's Monte-Carlo verification (no counterpart in the
 * reference, whose verifyNominalFailureKernel, kernels.cu:488-551, draws its hypotheses and
 * noise from curand, so that its failure counts are reproducible only in distribution).
 * on = 0 (the default): the fast flavour, with the hardware's approximate division, square
 * root and exponential and Box-Muller normals; on = 1: the exact flavour, the reference's
 * IEEE arithmetic and the library's inverse-CDF normals, whose per-sample failure times
 * equal the CPU oracle's. Controllers of one batch need the same flavour, so set it before
 * batching the controller. */
int dr_mppi_set_verify_exact(dr_mppi* h, int on);
/* Whether the fast verification reads the ego's moves from the shared ego tables (on = 1,
 * the default) or moves the ego in every sample (on = 0). The tables hold, per plan, the
 * ego's trajectory without branching and for every branch and branching step; they are
 * built only when no environment noise moves the ego and both plans' tables fit in 16 MiB
 * (the library's build-time DR_EGO_TABLE_MAX_BYTES). The failure times are the same
 * either way; off is slower. Set it before batching the controller. No counterpart in the
 * reference. */
int dr_mppi_set_ego_table(dr_mppi* h, int on);
/* Test switch for the bounded device waits (no counterpart in the reference, whose
 * kernels have no device-side wait): while `on` is set, the rollout and verification CTAs
 * of this controller's own steps (dr_mppi_step, the dr_mppi_debug_* hooks) announce their
 * staging bytes but issue no copy, so each staging wait gives up after `polls` polls (<= 0:
 * the default limit) with nothing in flight; the step then returns DR_ERR_TIMEOUT and
 * info->verif_timeouts counts the CTAs that gave up. Batches the controller joined later
 * keep their own copy of its settings. */
int dr_mppi_debug_stage_timeout(dr_mppi* h, int on, int polls);

/* ---- PR-MPPI controller (reference PRMPPIController) ---------------------------- */
/* nominal: n_timesteps x DR_DIM or NULL (prmppi_controller.cu:24-37). */
int dr_prmppi_create(const dr_env_config* env, const dr_prmppi_config* cfg, uint64_t seed, const float* nominal, int device, void* stream,
                     dr_prmppi** out);
int dr_prmppi_destroy(dr_prmppi* h);
/* One control step (prmppi_controller.cu:142-349). */
int dr_prmppi_step(dr_prmppi* h, const dr_sim_state* state, const float* belief, float* out_action, dr_prmppi_info* info);
/* Host mirrors h_nom_nominal / h_rob_nominal (T x DR_DIM each). */
int dr_prmppi_get_nominals(const dr_prmppi* h, float* nom, float* rob, size_t n);
uint64_t dr_prmppi_get_step(const dr_prmppi* h);
int dr_prmppi_io_bytes(const dr_prmppi* h, size_t* h2d, size_t* d2h);
int dr_prmppi_set_step(dr_prmppi* h, uint64_t step);
int dr_prmppi_set_profiling(dr_prmppi* h, int on);
int dr_prmppi_get_kernel_times(dr_prmppi* h, const char** names, float* ms, int n, int* count);
int dr_prmppi_batch_create(dr_prmppi* const* hs, int n, void* stream, dr_prmppi_batch** out);
int dr_prmppi_batch_destroy(dr_prmppi_batch* b);
int dr_prmppi_batch_step(dr_prmppi_batch* b, const dr_sim_state* states, const float* beliefs, float* out_actions, dr_prmppi_info* infos);
int dr_prmppi_batch_step_dev(dr_prmppi_batch* b, const dr_sim_state* states_dev, const float* beliefs_dev);
int dr_prmppi_batch_set_profiling(dr_prmppi_batch* b, int on);
int dr_prmppi_batch_get_kernel_times(dr_prmppi_batch* b, const char** names, float* ms, int n, int* count);
/* Hypothesis slots per thread of the batch's PR-MPPI rollout (1, the default, 2 or 4):
 * with several, a thread rolls out that many of a sample's hypothesis slots side by side
 * and moves the ego once for them (the ego's motion depends only on its own perturbed
 * plan, which the slots share). Costs are bit-identical for every choice; it takes effect
 * only where no environment noise moves the ego and P is a multiple of it (else 1).
 * Strategic race batches. No counterpart in the reference. Measured on the 4-agent
 * P 8 x K 2048 x H 64 workload: the rollout takes 0.59 / 0.60 / 0.93 ms at 1 / 2 / 4 (the
 * ego's moves are a small share of a step, fewer warps hide less latency), so 1 stays
 * the default. */
int dr_prmppi_batch_set_rollout_slots(dr_prmppi_batch* b, int slots);

/* ---- PR-MPPI test hooks ---------------------------------------------------------- */
/* noise[T][K][DR_DIM] (prmppi_kernels.cu:17) and thetas[P] (prmppi_kernels.cu:23-51) of the next step. */
int dr_prmppi_debug_noise(dr_prmppi* h, const float* belief, float* noise, size_t n, int32_t* thetas);
/* Rollout of the next step (prmppi_kernels.cu:55-130): cost_nom/cost_rob [P][K][2]
 * (running cost, safety cost), before averaging. The nominals are the shifted ones. */
int dr_prmppi_debug_rollout(dr_prmppi* h, const dr_sim_state* state, const float* belief, float* cost_nom, float* cost_rob);

/* ---- prediction streaming (the engine's sendState, src/engine.cpp:55-264) --------
 * After each closed-loop step the reference engine re-simulates the controller's plan on
 * the host, with noise off, and streams the predicted trajectories in MSG_STATE. These
 * entry points run that re-simulation on the device. Output rows (one per hypothesis for
 * MPPI; for PR-MPPI one per hypothesis with the nominal plan, then the robust plan under
 * the last hypothesis) hold, with T the horizon (or t_stride):
 *   positions [rows][T][(n_opp + 1) * DR_DIM]  every agent's position after each step,
 *                                              the last one repeated after a terminal step
 *                                              (Env::pushPredictions, env_stratrace.cpp:70-78)
 *   actions   [rows][T][DR_DIM]                the ego actions taken, zero after the stop
 *   records   [rows][DR_PREDICT_RECORD]        initial branch, branching time, branch (MPPI;
 *                                              0, -1, 0 for PR-MPPI), stop reason (EventType:
 *                                              0 outside, 1 winner, 2 opponent winner,
 *                                              3 truncated), stop time (-1: none)
 *   costs     [rows]                           MPPI: the discounted running + terminal cost
 *                                              (engine.cpp:131-141); PR-MPPI: running +
 *                                              terminal + safety weight if unsafe, on the
 *                                              predicted states (the engine prints these,
 *                                              evaluated on the current state, 221-222). */
#define DR_PREDICT_RECORD 5
/* MPPI (engine.cpp:73-166): from `state` (the state after the step) and `belief`, under
 * every hypothesis, the controller's plan as the engine holds it (the chosen plan with the
 * warm-start shift of the sent branch), belief update and branching on. Host buffers. */
int dr_mppi_predict(dr_mppi* h, const dr_sim_state* state, const float* belief, float* positions, float* actions, int32_t* records, float* costs);
/* The same for every controller of a batch stepped on the device (dr_mppi_batch_step_device,
 * which leaves each controller's pending shift in the batch's device records), from device
 * states and beliefs (DR_MAX_THETA per controller) into device outputs: controller i's rows
 * start at row i * n_theta, each of t_stride steps (at least every controller's horizon).
 * Enqueued on the batch's stream. DR_ERR_STATE before the first device step. */
int dr_mppi_batch_predict_device(dr_mppi_batch* b, const void* states_dev, const float* beliefs_dev, float* positions_dev, float* actions_dev,
                                 int32_t* records_dev, float* costs_dev, int t_stride);
/* PR-MPPI (engine.cpp:167-240): from `prev_state` (the state before the step), the new
 * nominal plan under every hypothesis and the robust plan under the last one. */
int dr_prmppi_predict(dr_prmppi* h, const dr_sim_state* prev_state, float* positions, float* actions, int32_t* records, float* costs);

/* ---- allocation-free rollout ------------------------------------------------------
 * No counterpart in the reference: an entry point for callers that cannot call
 * cudaMalloc (code where the device allocator is off limits, e.g. a real-time control
 * loop or a memory-pool owner that forbids allocation, or a host framework that hands
 * the library only buffers it owns). It runs the same fused rollout + per-branch cost
 * aggregation as dr_mppi_debug_rollout, for the controls knots_dev and the Philox
 * stream (seed, step), and writes costs_dev ((n_theta+1) x n_samples, device memory).
 * knots_dev: (n_theta+1) x M x DR_DIM floats on the device, M = n_knots (spline mode)
 * or n_timesteps (dense mode). Allocates nothing: its scratch is one static device
 * array of DR_NOALLOC_SCRATCH_BYTES per GPU, held until the process exits; a problem
 * that does not fit (roughly 8 x n_theta x n_samples bytes plus the track and the
 * controls) is rejected with DR_ERR_INVALID_ARG. All calls share that array: calls
 * whose GPU work overlaps race on it. The first call on a device (and the first after
 * the device's context was reset) looks the array up (cudaGetSymbolAddress) with that
 * device current, so make it before any stream capture. The call is synchronous: it
 * returns after the work on `stream` (NULL: legacy default) has completed. Samples whose
 * cost is not finite keep that value in costs_dev; a rollout CTA whose bounded staging
 * wait gave up makes the call return DR_ERR_TIMEOUT. */
#define DR_NOALLOC_SCRATCH_BYTES (4u << 20)
int dr_mppi_rollout_costs_noalloc(const dr_env_config* env, const dr_mppi_config* cfg, uint64_t seed, uint64_t step, const dr_sim_state* state,
                                  const float* belief, const float* knots_dev, float* costs_dev, void* stream);

/* Natural-cubic-spline basis B (T x M, row-major) of the knots tau_0..tau_{M-1}: the
 * reference's MPPIController::buildSplineMatrix (src/mppi_controller.cu:56-141). */
int dr_spline_matrix(int T, int M, const int32_t* knots, float* out);

/* ---- track preprocessing on the device (python-src/utils.py:390-427) -------------
 * The StratRace track grids of n_tracks tracks from their track functions sampled at
 * DR_N_TRACK_SAMPLES points (q: n_tracks x 512 x 2, host): the cumulative chord length as
 * the spline parameter, periodic cubic splines x(s), y(s) (the reference's scipy
 * CubicSpline, bc_type="periodic"), evaluated at 512 uniform arc lengths. Outputs (host)
 * per track: p_grid and dp_grid (512 x 2), t_grid (512 x 2, unit tangent), kappa_grid (512),
 * track_length (1); computed in double precision, stored as float32. */
int dr_track_grids(const double* q, int n_tracks, float* p_grid, float* dp_grid, float* t_grid, float* kappa_grid, float* track_length);

/* ---- environment step on the device (reference engine dynStep, engine.cpp:286-312) */
/* Advances `state` in place by one true-dynamics step for the ego action, with the
 * given true hypothesis; updates belief (n_theta) in place. Returns the terminal type
 * (0 none, 1 lose, 2 win, 3 opponent win) in *term. Noise is drawn from the Philox
 * stream (seed, step). */
int dr_env_step(const dr_env_config* env, int true_theta, const float* action, dr_sim_state* state, float* belief, int update_belief,
                uint64_t seed, uint64_t step, int* term);

/* Test hook: the projection onto the centreline (fastProjectOnTrack, env_stratrace.h:88-162)
 * of n points xy[n][2], each from its previous arc length prev_s[n], as the kernels run it:
 * mode 0 the verification's fast flavour (certified local search of the window, with the
 * full window scan where the search cannot certify its sample), 1 the fast flavour with
 * the full window scan only, 2 the exact flavour (the rollout's: the same search on the
 * unrounded distances), 3 the exact flavour with the full window scan only (the
 * reference's algorithm as written). Writes the arc length, the signed lateral distance
 * and the track sample index of the arc length. */
int dr_debug_project(const dr_env_config* env, const float* xy, const float* prev_s, int n, int mode, float* s_out, float* lat_out, int32_t* idx_out);
/* The squared radii cert[512] of the fast projection's local search for the centreline
 * p_grid[512][2] (host only, no GPU): within cert[c] of sample c, a point at which c is a
 * local minimum of the squared distances to the samples is nearer to c than to every other
 * sample of any window holding c, by more than 1e-3 m^2; negative where nothing is
 * certified. Part of the packed track the kernels read. */
int dr_projection_certificate(const float* p_grid, float* cert);

/* ==== gate race (the reference's EnvDroneRace, include/environments/env_dronerace.h) ====
 * Two agents (the MPPI ego at index i_mppi, one PID opponent), gates crossed in order,
 * laps counted at the last gate, PID opponents following racelines. The reference fixes
 * N_GATES, N_RACELINES and the obstacle counts at compile time (env_dronerace_defs.h:
 * 2 gates, 2 racelines, no obstacles); here gates and obstacles are runtime counts up to
 * the maxima below, the racelines stay 2. */
#define DR_GATE_AGENTS 2        /* reference EnvDroneRace::N_AGENTS (env_dronerace_defs.h:8) */
#define DR_GATE_RACELINES 2     /* reference N_RACELINES (env_dronerace_defs.h:17); fixed */
#define DR_GATE_MAX_GATES 16
#define DR_GATE_MAX_OBSTACLES 4 /* rectangle and round obstacles each */

/* Opponent PID controller (reference PIDConfig, env_dronerace_defs.h:44-56; wire order of
 * env_dronerace.cpp:104-121). */
typedef struct dr_pid_config
{
    float kp;
    float kd;
    float repulsion_factor;
    float repulsion_power;
    float repulsion_dist_fact;
    int32_t raceline_index;
    float action_noise;
} dr_pid_config;

/* Gate-race environment (reference EnvDroneRace::EnvironmentConfig,
 * env_dronerace_defs.h:60-93). track_points is a HOST pointer to
 * DR_GATE_RACELINES x DR_N_TRACK_SAMPLES x 2 floats (the racelines, one after the other). */
typedef struct dr_gate_env_config
{
    int32_t n_theta;            /* PID hypotheses (reference N_TRUE_MODELS) */
    float arena_min[DR_DIM];
    float arena_max[DR_DIM];
    float dt;
    int32_t send_states;
    float drone_radius;
    float pos_noise_level;
    float speed_noise_level;
    float action_noise_level;
    float max_speed[DR_GATE_AGENTS];
    float max_accel[DR_GATE_AGENTS];
    int32_t n_win_laps;
    float target_distance;      /* PID look-ahead along the raceline (fraction of a lap) */
    int32_t n_gates;
    float gate_centers[DR_GATE_MAX_GATES * DR_DIM];
    float gate_vectors[DR_GATE_MAX_GATES * DR_DIM];
    float gate_radius[DR_GATE_MAX_GATES];
    int32_t n_obstacles;        /* rectangles [xmin, ymin, xmax, ymax] */
    float obstacles[DR_GATE_MAX_OBSTACLES * DR_DIM * 2];
    int32_t n_round_obstacles;
    float round_obs_centers[DR_GATE_MAX_OBSTACLES * DR_DIM];
    float round_obs_radius[DR_GATE_MAX_OBSTACLES];
    const float* track_points;  /* host, [DR_GATE_RACELINES][DR_N_TRACK_SAMPLES][2] */
    float init_belief[DR_MAX_THETA];
    dr_pid_config opp_pid[DR_MAX_THETA];
    int32_t i_mppi;             /* index of the ego agent (0 or 1) */
} dr_gate_env_config;

/* Gate-race state (reference EnvDroneRace::SimState, env_dronerace_defs.h:95-103).
 * S[agent * DR_GATE_RACELINES + r] is the arc-length fraction on raceline r; a negative
 * S of an agent means "not tracked" (the reference sets the ego's to -1 on load,
 * env_dronerace.cpp:96-97, and never projects it). */
typedef struct dr_gate_state
{
    float pos[DR_GATE_AGENTS * DR_DIM];
    float vel[DR_GATE_AGENTS * DR_DIM];
    float S[DR_GATE_AGENTS * DR_GATE_RACELINES];
    int32_t laps[DR_GATE_AGENTS];
    int32_t gates[DR_GATE_AGENTS];
} dr_gate_state;

/* An MPPI controller on the gate race (the reference's MPPIController compiled with
 * USE_ENV_DRONERACE). The handle is a dr_mppi: destroy, nominals, knots, fail counts,
 * temperature, profiling and batching work as for the strategic race; a batch holds
 * controllers of one environment kind (for a gate-race batch, dr_mppi_batch_step_dev
 * takes dr_gate_state records). Step it with dr_gate_mppi_step. */
int dr_gate_mppi_create(const dr_gate_env_config* env, const dr_mppi_config* cfg, uint64_t seed, const float* nominal, int device, void* stream,
                        dr_mppi** out);
/* MPPIController::getControl (src/mppi_controller.cu:250-466) on the gate race. */
int dr_gate_mppi_step(dr_mppi* h, const dr_gate_state* state, const float* belief, float* out_action, dr_mppi_info* info);
/* PR-MPPI on the gate race: the reference's PRMPPIController built with USE_ENV_DRONERACE
 * (its PR-MPPI kernels and cost functions over the gate race's environment,
 * include/environments/env_dronerace.h). Same configuration, results and info as the
 * strategic race's; the state is a dr_gate_state and the ego is env->i_mppi.
 * dr_prmppi_step refuses a gate-race controller and dr_gate_prmppi_step a strategic one. */
int dr_gate_prmppi_create(const dr_gate_env_config* env, const dr_prmppi_config* cfg, uint64_t seed, const float* nominal, int device, void* stream,
                          dr_prmppi** out);
int dr_gate_prmppi_step(dr_prmppi* h, const dr_gate_state* state, const float* belief, float* out_action, dr_prmppi_info* info);
/* Test hook: as dr_prmppi_debug_rollout, on the gate race. */
int dr_gate_prmppi_debug_rollout(dr_prmppi* h, const dr_gate_state* state, const float* belief, float* cost_nom, float* cost_rob);
int dr_gate_mppi_batch_step(dr_mppi_batch* b, const dr_gate_state* states, const float* beliefs, float* out_actions, dr_mppi_info* infos);
/* Test hooks, as dr_mppi_debug_rollout / dr_mppi_debug_verify (same outputs). */
int dr_gate_mppi_debug_rollout(dr_mppi* h, const dr_gate_state* state, const float* belief, float* costs_true, int32_t* branch_used,
                               int32_t* branch_time, float* costs);
int dr_gate_mppi_debug_verify(dr_mppi* h, const dr_gate_state* state, const float* belief, const float* dense_plan, int plan,
                              uint32_t* fail_counts, int32_t* fail_time, int32_t* theta);
/* One gate-race environment step on the device (environmentStep, env_dronerace.h:
 * 546-680, with noise on, as the engine's dynStep), like dr_env_step. */
int dr_gate_env_step(const dr_gate_env_config* env, int true_theta, const float* action, dr_gate_state* state, float* belief, int update_belief,
                     uint64_t seed, uint64_t step, int* term);

#ifdef __cplusplus
}
#endif

#endif /* DRMPPI_H */
