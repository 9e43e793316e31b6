/*
 * cls_b200.h -- C ABI of the B200 differentiable soft-robot simulation step.
 *
 * The reference (erizmr/Complex-locomotion-skill-learning-via-differentiable-
 * physics) has no foreign-function boundary: its trainer drives Taichi kernels
 * through duck-typed Python objects.  Each entry point below replaces one
 * step of that protocol; the reference interface it stands in for is cited
 * beside it (paths relative to the reference root).
 *
 * Conventions
 *   - every function returns CLS_OK (0) or a negative CLS_ERR_* code; the
 *     message of the last failure is available from cls_last_error();
 *   - host arrays are float64 and row-major, in the reference's field layouts
 *     ([t][env][i] for trajectory fields, [env][vertex][3] for states);
 *   - environments are numbered in the order given to cls_create; internally
 *     they are grouped by robot, which callers never see;
 *   - a handle is bound to one CUDA stream (cls_set_stream) and is not
 *     thread-safe; distinct handles may be used concurrently;
 *   - all work is asynchronous on the handle's stream except functions that
 *     return host data, which synchronise that stream.
 */
#ifndef CLS_B200_H_
#define CLS_B200_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CLS_OK 0
#define CLS_ERR_INVALID (-1)   /* bad argument or configuration */
#define CLS_ERR_CUDA (-2)      /* CUDA runtime error */
#define CLS_ERR_OOM (-3)       /* device allocation failed */
#define CLS_ERR_NONFINITE (-4) /* NaN/Inf detected in the simulated state */
#define CLS_ERR_STATE (-5)     /* call out of order (e.g. backward before forward) */
#define CLS_ERR_TIMEOUT (-6)   /* a kernel's bounded wait ran out (reported by cls_synchronize) */

#define CLS_ACT_SIN 0
#define CLS_ACT_TANH 1

#define CLS_LOSS_VELOCITY 1
#define CLS_LOSS_HEIGHT 2
#define CLS_LOSS_POSE 4
#define CLS_LOSS_ACTUATION 8
#define CLS_LOSS_ROTATION 16
#define CLS_LOSS_CRAWL 32

#define CLS_MAX_HIDDEN 4

typedef struct cls_sim cls_sim;

/* One robot type: geometry plus its controller shape.
 * Replaces config["robot"]{objects, springs} produced by
 * RobotDesignMassSpring3D.build (multitask/robot_design.py:572-591, rows of
 * add_spring :344-349) and the Model shape (multitask/nn.py:79-109). */
typedef struct {
  int32_t n_vertices;
  int32_t n_springs;
  const double* objects;        /* [n_vertices][3] initial positions */
  const double* springs;        /* [n_springs][5]: a, b, rest length, stiffness, actuation */
  int32_t robot_id;             /* 100: heading from vertices 45, 46, 34, 36 */
  int32_t n_outputs;            /* MLP outputs; 0 = one per spring (reference) */
  const int32_t* spring_output; /* [n_springs] output feeding each spring or -1; NULL = identity */
  int32_t n_hidden_layers;      /* 1..CLS_MAX_HIDDEN (reference: 1) */
  int32_t hidden[CLS_MAX_HIDDEN];
} cls_robot_desc;

/* Simulation / controller / optimiser constants: the cfg3d JSON schema after
 * ConfigSim._add_adaptive_configs (multitask/config_sim.py:103-147). */
typedef struct {
  int32_t max_steps;            /* process.max_steps: trajectory length T */
  double dt;                    /* process.dt */
  double gravity;               /* simulator.gravity */
  double ground_height;         /* simulator.ground_height */
  double drag_damping;          /* simulator.drag_damping */
  double dashpot_damping;       /* simulator.dashpot_damping */
  double friction;              /* 0.4 in the reference (solver_mass_spring.py:136) */
  double stiffness_scale;       /* 0.1 in the reference (solver_mass_spring.py:64) */
  int32_t run_period, turn_period, jump_period;
  double spring_omega;          /* process.spring_omega */
  int32_t n_sin_waves, duplicate_v, duplicate_h, duplicate_c;
  int32_t activation_hidden;    /* CLS_ACT_SIN (reference) or CLS_ACT_TANH */
  int32_t activation_output;
  int32_t loss_mask;            /* CLS_LOSS_* bits (reference 3D: velocity | rotation) */
  int32_t precision;            /* 32 or 64 */
  int32_t checkpoint_every;     /* substeps per checkpoint segment (K) */
  double max_speed, max_height; /* process.max_speed / max_height */
  double adam_b1, adam_b2, learning_rate;
  int32_t threads_per_block;    /* 0: choose automatically */
  int32_t keep_trajectory;      /* 1: keep x[t] for every t (cls_get_trajectory, mesh export)
                                   even when no rotation or pose loss needs it; 0: only then */
} cls_sim_params;

/* Fills *p with the reference's defaults for cfg3d/sim_quad.json. */
void cls_default_params(cls_sim_params* p);

/* Allocates a batch of n_envs environments; env_robot[e] selects the robot type
 * of env e.  Replaces TaichiEnv.__init__ + SolverMassSpring.__init__ +
 * Model.__init__ (multitask/taichi_env.py:22-147, solver_mass_spring.py:8-56,
 * nn.py:79-109) and SolverMassSpring.initialize_robot (:58-67). */
int cls_create(const cls_robot_desc* robots, int32_t n_robots, const int32_t* env_robot,
               int32_t n_envs, const cls_sim_params* params, cls_sim** out);
int cls_destroy(cls_sim* sim);

/* Message of the last failure on this handle (NULL handle: last cls_create
 * failure of the calling thread). */
const char* cls_last_error(const cls_sim* sim);

/* Binds the handle to a cudaStream_t (NULL: legacy default stream). */
int cls_set_stream(cls_sim* sim, void* stream);

/* Sizes of the packed layouts. */
int cls_get_sizes(const cls_sim* sim, int32_t* n_envs, int32_t* n_vertices_total,
                  int32_t* max_steps);
/* Width of weight layer `layer` of `robot` in the reference layout
 * (rows = outputs, cols = inputs; layer 0 cols = n_input_states). */
int cls_get_layer_shape(const cls_sim* sim, int32_t robot, int32_t layer, int32_t* rows,
                        int32_t* cols);

/* x[0], v[0] of every env ([n_vertices_total][3], envs in creation order).
 * Replaces TaichiEnv.setup_robot / reset_robot / copy_robot
 * (multitask/taichi_env.py:487-510). */
int cls_set_state(cls_sim* sim, const double* x0, const double* v0);

/* target_v [T][n_envs][3], target_h [T][n_envs], target_c [T][n_envs].
 * Replaces initialize_train / initialize_validate / initialize_script
 * (multitask/taichi_env.py:333-469) when targets come from the caller. */
int cls_set_targets(cls_sim* sim, const double* target_v, const double* target_h,
                    const double* target_c);

/* The targets as the device holds them (same layouts as cls_set_targets;
 * any pointer may be NULL): the fields TaichiEnv.initialize_train writes
 * (multitask/taichi_env.py:385-447), read back after cls_initialize_train. */
int cls_get_targets(cls_sim* sim, double* target_v, double* target_h, double* target_c);

/* Reference-layout weights W [rows][cols], b [rows] of one layer; layer 0 is
 * weights1/bias1 (multitask/nn.py:31-43).  Replaces Model.load_weights. */
int cls_set_weights(cls_sim* sim, int32_t robot, int32_t layer, const double* W, const double* b);
int cls_get_weights(cls_sim* sim, int32_t robot, int32_t layer, double* W, double* b);
/* Gradient of the loss w.r.t. the same (after cls_backward). */
int cls_get_grads(cls_sim* sim, int32_t robot, int32_t layer, double* gW, double* gb);

/* Training rollout of `steps` substeps (t in [0, steps-2], the loop of
 * DiffPhyTrainer.simulate, multitask/diffphy_trainer.py:231-255), saving a
 * checkpoint every K substeps and the per-step observables. */
int cls_forward(cls_sim* sim, int32_t steps);
/* Forward-only evaluation rollout (t in [0, steps], diffphy_trainer.py:257-268). */
int cls_forward_eval(cls_sim* sim, int32_t steps);
/* Loss of the last rollout (TaichiEnv.get_loss, multitask/taichi_env.py:304-331).
 * loss_terms[8] = total, velocity, height, pose, rotation, weight, actuation,
 * crawl; loss_env [8][n_envs] the per-env losses (loss_batch fields, scaled by
 * B as the reference does); either may be NULL. */
int cls_loss(cls_sim* sim, double* loss_terms, double* loss_env);
/* Selects the losses of the following rollouts (CLS_LOSS_* bits): the
 * loss_enable set that DiffPhyTrainer passes to TaichiEnv.get_loss
 * (multitask/taichi_env.py:304-317).  Rotation and pose need the trajectory
 * (created with one of them or keep_trajectory), actuation its record
 * (created with it); CLS_ERR_INVALID otherwise.  A CUDA graph captured
 * earlier keeps the set it was captured with.  The next cls_backward needs a
 * new cls_forward. */
int cls_set_loss_mask(cls_sim* sim, int32_t mask);
/* Reverse pass (ti.ad.Tape exit, diffphy_trainer.py:246): recompute each
 * segment from its checkpoint and run the hand-written adjoints. */
int cls_backward(cls_sim* sim);
/* forward + loss + backward in one call; returns the total loss. */
int cls_simulate(cls_sim* sim, int32_t steps, double* loss);
/* Same rollout, but every env runs in its own launch (one robot per launch). */
int cls_simulate_per_env(cls_sim* sim, int32_t steps, double* loss);
/* Adam step on all weights (Model.gradient_update, multitask/nn.py:163-171,
 * 184-191) with bias correction for iteration `iter`; *tns receives the
 * squared gradient norm (Model.get_TNS, :173-182) if non-NULL. */
int cls_adam_step(cls_sim* sim, int32_t iter, double* tns);
/* Device buffers of the weight and bias gradients of every robot type (in
 * the library's packed layout, elem_bytes = 4 or 8 by precision), which
 * cls_backward writes and cls_adam_step reads; valid until cls_destroy.
 * Ranks holding identically created handles (the same robot types, each
 * with a share of one controller's envs) all-reduce them in place between
 * cls_backward and cls_adam_step to train one shared controller
 * data-parallel, each having set the total env count with
 * cls_set_loss_envs.  No reference counterpart: the reference trains one
 * batch on one device. */
int cls_grad_buffers(cls_sim* sim, void** weight_grads, int64_t* n_weight, void** bias_grads,
                     int64_t* n_bias, int32_t* elem_bytes);
/* The env count B that robot type `robot`'s loss terms are divided by
 * (multitask/taichi_env.py:185-293 divide by the batch size); default: the
 * handle's own env count of the type.  A rank holding one shard of a
 * controller's envs sets the total over all ranks, so that its loss and
 * gradients are its shard's share of the whole batch's and the all-reduced
 * sum is the whole batch's.  n_envs must be at least the handle's count.
 * The next cls_backward needs a new cls_forward; a CUDA graph captured
 * earlier reads the new value when it is replayed (the robot table lives in
 * device memory).  No reference counterpart. */
int cls_set_loss_envs(cls_sim* sim, int32_t robot, int32_t n_envs);
/* zero the Adam moments (Model.clear_adam, multitask/nn.py:111-114) */
int cls_clear_adam(cls_sim* sim);

/* Observables of the last rollout: center [T][n_envs][3], height, upper
 * height, rotation [T][n_envs] (solver fields of the same names). */
int cls_get_observables(cls_sim* sim, double* center, double* height, double* upper_height,
                        double* rotation);
/* Positions x[t] for all t ([T][n_vertices_total][3]); only available when a
 * rotation or pose loss is enabled or params.keep_trajectory is set (the
 * trajectory is then kept). */
int cls_get_trajectory(cls_sim* sim, double* x);
/* State after the last processed substep ([n_vertices_total][3]). */
int cls_get_final_state(cls_sim* sim, double* x, double* v);
/* d loss / d x[0], d v[0] after cls_backward ([n_vertices_total][3]). */
int cls_get_state_grads(cls_sim* sim, double* gx0, double* gv0);

/* Waits for the handle's stream; returns CLS_ERR_NONFINITE if a kernel saw
 * NaN/Inf state, CLS_ERR_TIMEOUT if a tensor-core tile's bounded wait ran out,
 * since the last check (then clears the status). */
int cls_synchronize(cls_sim* sim);

/* Self-test of the tensor-core tiles' bounded waits (batched controller path
 * and weight-gradient tiles): with starve = 1 every tile issues no bulk
 * copies and no MMAs, so its wait for operands runs out after wait_limit
 * polls (0: the built-in limit) with nothing in flight; the tile then frees
 * its tensor memory, skips its epilogue and sets the status that
 * cls_synchronize reports as CLS_ERR_TIMEOUT.  Results are invalid while
 * starved; starve = 0 restores normal operation.  No reference
 * counterpart. */
int cls_debug_gemm_starve(cls_sim* sim, int32_t starve, uint32_t wait_limit);

/* Model.weights_init (multitask/nn.py:59-67) on the device:
 * W = (u * 2 - 1) * sqrt(6 / fan_in) with u from a counter-based generator
 * seeded by `seed` (the reference draws from ti.random); biases unchanged. */
int cls_weights_init(cls_sim* sim, uint64_t seed);
/* TaichiEnv.initialize_train (multitask/taichi_env.py:385-447, 3D branch) on
 * the device for t < steps, drawing the task pool from (seed, iter). */
int cls_initialize_train(cls_sim* sim, int32_t iter, int32_t steps, uint64_t seed,
                         double max_speed);

/* Per-kernel profile: when enabled, every launch is bracketed by CUDA events
 * on the handle's stream.  cls_profile_read returns, per launch category
 * (0 first-pass forward, 1 segment recompute, 2 reverse, 3 weight-gradient
 * products, 4 loss, 5 optimiser/packing, 6 other, 7 batched controller GEMMs
 * of the forward passes, 8 batched controller GEMMs of the reverse pass), the
 * summed device time in ms and the number of launches; launches are counted
 * even when disabled. */
#define CLS_PROFILE_KINDS 9
int cls_profile_enable(cls_sim* sim, int32_t on);
int cls_profile_read(cls_sim* sim, double* ms, int64_t* launches, int32_t reset);
/* Per-phase clock totals of the fused kernels, out[32] (clock64 cycles summed
 * over CTAs; forward: 10 observables and controller input, 13 controller,
 * 16 springs and advance; reverse: 3 advance and spring adjoints up to the
 * output layer's dz, 6 controller adjoint, 8 input / centre / height
 * adjoints).  Written only by a library built with -DCLS_PHASE_TIMERS; zeros
 * otherwise.  No reference counterpart. */
int cls_phase_read(cls_sim* sim, unsigned long long* out);

/* Captures one training iteration (forward + loss + backward, optionally the
 * Adam step) into a CUDA graph and replays it; cls_graph_launch replays. */
int cls_graph_capture(cls_sim* sim, int32_t steps, int32_t with_adam);
int cls_graph_launch(cls_sim* sim, int32_t iter);

/* Controller path.  The reference evaluates Model.forward per env and
 * substep (multitask/nn.py:130-146, called from diffphy_trainer.py:246-256);
 * here the fused segment kernels run it per env (CLS_CONTROLLER_PER_ENV),
 * while the batched path splits each substep at the controller and runs each
 * layer as one GEMM over all envs of a robot type (FP32: tensor cores,
 * tcgen05 with a 3xTF32 split, FP32 accumulate; FP64: SIMT), with the same
 * results within rounding.  CLS_CONTROLLER_AUTO (the default at creation)
 * takes the batched path when every robot type has at least 256 envs.  No
 * reference counterpart: a layout choice of this implementation.  Serving
 * windows (cls_serve_*) and per-env launches always use the fused kernels. */
#define CLS_CONTROLLER_AUTO 0
#define CLS_CONTROLLER_PER_ENV 1
#define CLS_CONTROLLER_BATCHED 2
int cls_set_controller_path(cls_sim* sim, int32_t path);
/* *on = 1 when the batched path is active. */
int cls_controller_batched(const cls_sim* sim, int32_t* on);

/* Launch shape of the fused segment kernels: threads per CTA (64..1024, a
 * multiple of 32; up to 256, up to 512 and up to 1024 select kernel
 * instances compiled for 255, 128 and 64 registers per thread), the CTAs per
 * SM that the persistent grid is sized for (grid = min(envs, SMs x
 * ctas_per_sm); CTAs take envs from a work queue, largest first), and where
 * the kernels read the controller: weights_shared = 1 copies each env's
 * weights and biases into shared memory once per work item (the robot's
 * controller must fit beside the kernels' own shared memory), 0 reads them
 * from global memory every substep, -1 (the default at creation) chooses 1
 * when it fits without fewer resident CTAs.  Results do not depend on
 * ctas_per_sm or weights_shared, and depend on threads_per_block only through
 * the rounding of block-wide reductions.  No reference counterpart: Taichi
 * chose its own block sizes per kernel (ti.loop_config).  A CUDA graph
 * captured earlier keeps the shape it was captured with.  CLS_ERR_INVALID
 * when a robot's shared memory does not fit the instance or no CTA of that
 * size can be resident.  cls_get_launch_shape reports weights_shared as the
 * applied 0 or 1 (the pointer may be NULL). */
int cls_set_launch_shape(cls_sim* sim, int32_t threads_per_block, int32_t ctas_per_sm,
                         int32_t weights_shared);
int cls_get_launch_shape(const cls_sim* sim, int32_t* threads_per_block, int32_t* ctas_per_sm,
                         int32_t* weights_shared);

/* Per-spring tables of the fused and step kernels: each spring's impulse
 * (forward) and adjoint terms (fused reverse) evaluated once into shared
 * memory and gathered per vertex, instead of evaluated from both of its
 * endpoints.  mode -1 (the default at creation): on when the largest robot's
 * table fits (<= 3072 springs in FP32); 0 off; 1 on (CLS_ERR_INVALID when it
 * does not fit).  The same results (each spring is evaluated in the same
 * argument order either way and gathered in the same order).  No reference
 * counterpart. */
int cls_set_spring_tables(cls_sim* sim, int32_t mode);
int cls_spring_tables(const cls_sim* sim, int32_t* on);

/* One timed candidate of cls_autotune. */
typedef struct cls_launch_shape {
  int32_t controller_path;    /* CLS_CONTROLLER_PER_ENV or CLS_CONTROLLER_BATCHED */
  int32_t threads_per_block;  /* fused kernels (per-env path) */
  int32_t ctas_per_sm;
  int32_t weights_shared;     /* 0 or 1 */
  float ms;                   /* one forward + loss + backward over the tuning horizon */
} cls_launch_shape;

/* Autotuner: times one training rollout (cls_forward + the loss + cls_backward,
 * CUDA events on the handle's stream, `repeats` runs after one untimed run) of
 * `steps` substeps (<= 0: min(max_steps, 2 K + 1, 101)) for every feasible
 * launch shape -- threads per CTA in {128, 256, 512, 1024} x controller in
 * global or shared memory x CTAs per SM from 1 to what can be resident (at
 * most 4) -- and, when every robot type has at
 * least 32 envs, for the batched controller path, then applies the fastest.
 * Needs the state, targets and weights set (it runs the caller's workload);
 * leaves the weights unchanged and the rollout, loss and gradient buffers as
 * after a training rollout.  Up to max_entries candidates are written to
 * `table`; *n_entries = the number timed.  Profiling must be off.  No
 * reference counterpart. */
int cls_autotune(cls_sim* sim, int32_t steps, int32_t repeats, cls_launch_shape* table,
                 int32_t max_entries, int32_t* n_entries);

/* ---------------------------------------------------------------------------
 * Serving: one handle as a pool of env slots at different times of their own
 * episodes.  The reference has no serving path; these calls let a request
 * loop (serving.py) fold rollout requests into a running batch: a slot is
 * (re)started with cls_serve_reset_env, and every launch advances each slot
 * through its own window.  Each slot needs a robot (controller) of its own,
 * so that its weight gradients are its own.
 *
 * windows: [n_envs][4] int32 in user env order, {t_begin, t_end, checkpoint,
 * first}: the env runs steps [t_begin, t_end) of its episode from checkpoint
 * `checkpoint` (t_begin = checkpoint * checkpoint_every, t_end <= steps - 1;
 * a reverse window spans one checkpoint segment); t_begin >= t_end leaves the
 * env idle.  `first` marks the first (last-in-time) reverse segment of an
 * env's reverse pass.
 * steps: [n_envs] episode steps of each env (the `steps` of cls_forward).
 * --------------------------------------------------------------------------- */
/* Initial state x0 (v0 may be NULL: zero) [n_v][3] and targets tv [T][3],
 * th [T], tc [T] (NULL: zero) of one env; clears its observables. */
int cls_serve_reset_env(cls_sim* sim, int32_t env, const double* x0, const double* v0, const double* tv,
                        const double* th, const double* tc);
/* First-pass substeps of every env's window (checkpoints at window ends). */
int cls_serve_forward(cls_sim* sim, const int32_t* windows, const int32_t* steps);
/* One reverse segment per env window (recompute + adjoint + weight
 * gradients); an env's robot gradients restart at its `first` segment. */
int cls_serve_backward(cls_sim* sim, const int32_t* windows, const int32_t* steps);
/* Per-env losses [8][n_envs] (cls_loss's loss_env layout) with per-env steps;
 * envs with steps <= 0 are skipped (zeros). */
int cls_serve_loss(cls_sim* sim, const int32_t* steps, double* loss_env);
/* State at the end of the env's last forward window, [n_v][3] each. */
int cls_serve_env_state(cls_sim* sim, int32_t env, double* x, double* v);

/* ---------------------------------------------------------------------------
 * Admission and polling (continuous batching in the library).  No reference
 * counterpart: the reference trains one batch at a time
 * (multitask/diffphy_trainer.py:219-256); serving.Server is the Python form
 * of the same scheduler.  Every env of the handle is a slot with a robot
 * entry (controller) of its own.  A request runs on a free slot of the robot
 * class of slot `robot` (slots whose robot entries have the same geometry,
 * spring table, output map and layer widths); cls_admit restarts that slot
 * alone (cls_serve_reset_env) when the request's HBM footprint (state,
 * checkpoints, trajectory, observables, targets, controller; reverse records
 * for gradient queries) fits beside the admitted requests' in bytes_budget
 * (< 0: no limit), else *slot = -1 and nothing changes.  cls_poll waits for
 * the tick in flight, applies it (losses at the end of a first pass, the
 * reverse pass of gradient queries, counted down one checkpoint segment per
 * round) and issues the next tick: one forward window of tick_segments x
 * checkpoint_every substeps for every slot in its first pass, then
 * tick_segments reverse segments for every slot in its reverse pass; it
 * reports the ids of finished requests (at most `capacity`; the rest at the
 * next call) and the number of slots still running.  A finished request keeps
 * its slot -- loss terms, final positions and, for gradient queries, the
 * slot's weight gradients (cls_get_grads with robot = its slot) -- until
 * cls_serve_release.  Requests admitted between polls join the next tick.
 * Invalid ids, steps outside [2, max_steps], a duplicate id or a gradient
 * query on a slot whose robot entry other envs share fail with
 * CLS_ERR_INVALID; a non-finite state or GEMM timeout seen at a tick's end
 * is reported by cls_poll as by cls_synchronize.
 * --------------------------------------------------------------------------- */
typedef struct cls_request {
  uint64_t id;              /* caller's request id (unique among admitted ones) */
  int32_t robot;            /* a slot whose robot class the request runs on */
  int32_t steps;            /* episode steps (cls_forward's `steps`) */
  int32_t grad;             /* 1: forward + adjoint (weight gradients); 0: forward only */
  const double* x0;         /* [n_v][3] initial positions; NULL: the robot's objects */
  const double* target_v;   /* [max_steps][3]; NULL: zeros */
  const double* target_h;   /* [max_steps]; NULL: zeros */
  const double* target_c;   /* [max_steps]; NULL: zeros */
} cls_request;
/* Checkpoint segments a tick advances every request by (default 1); only
 * with no tick in flight. */
int cls_serve_tick(cls_sim* sim, int32_t tick_segments);
int cls_admit(cls_sim* sim, const cls_request* req, int64_t bytes_budget, int32_t* slot);
int cls_poll(cls_sim* sim, uint64_t* done, int32_t capacity, int32_t* n_done, int32_t* n_active);
/* Slot, loss terms [8] (total, velocity, height, pose, rotation, weight,
 * actuation, crawl; NULL: skipped) and final positions [n_v][3] (NULL:
 * skipped) of a finished request. */
int cls_serve_result(cls_sim* sim, uint64_t id, int32_t* slot, double* loss_terms, double* final_x);
int cls_serve_release(cls_sim* sim, uint64_t id);

/* Targets of one env for t in [t_from, max_steps) (rows tv [T - t_from][3],
 * th, tc [T - t_from]; NULL leaves that field), other times and envs
 * untouched: an interactive client changing its goal while its episode runs
 * (TaichiEnv.initialize_interactive, multitask/taichi_env.py:333-338, as
 * interactive_3d.py:13-28 calls it on key presses). */
int cls_serve_set_targets(cls_sim* sim, int32_t env, int32_t t_from, const double* tv, const double* th,
                          const double* tc);

/* One substep of every env with controller outputs chosen by the caller (an
 * external policy in place of the embedded controller): MassSpringEnv.step
 * (multitask/mass_spring_env.py:55-93) -- pass_actuation, apply_spring_force
 * and advance_toi of substep t - 1, then compute_center, compute_height and
 * nn_input of t.  outputs: [n_envs][omax] (omax = the largest robot's output
 * count; a robot without an output map has one output per spring, as the
 * reference's actuation field); NULL with t = 0 observes the state set by
 * cls_set_state (MassSpringEnv.reset, :207-224).  observation: [n_envs][imax]
 * rows in the reference's input layout (imax = the largest n_input_states);
 * center_height: [n_envs][4] = centre and height of t.  The state stays on
 * the device between calls; the observables of t are kept as a rollout's
 * (cls_get_observables).  No reference counterpart as a C function. */
int cls_env_step(cls_sim* sim, int32_t t, const double* outputs, double* observation, double* center_height);

/* ---------------------------------------------------------------------------
 * Differentiable MLS-MPM (multitask/solver_mpm.py).  The reference's solver is
 * 2D (fixed-corotated, actuation along y) and unreachable from its env
 * (taichi_env.py:136 constructs it without its config); these entry points run
 * its algorithm in 2D or 3D, with per-particle fibre directions and a
 * neo-Hookean option, and add the checkpointed reverse pass.
 * --------------------------------------------------------------------------- */
#define CLS_MPM_FIXED_COROTATED 0 /* reference model, 2D only */
#define CLS_MPM_NEO_HOOKEAN 1

typedef struct cls_mpm cls_mpm;

/* Particle body: RobotDesignMPM.build output (multitask/robot_design.py:38-110):
 * positions, actuator id per particle (-1 passive); fibre directions are new
 * (NULL: the reference's e_y). */
typedef struct {
  int32_t dim;                  /* 2 or 3 */
  int32_t n_particles;
  const double* positions;      /* [n_particles][dim], inside the unit box */
  const int32_t* muscle;        /* [n_particles] actuator index or -1 (NULL: all -1) */
  const double* fibre;          /* [n_particles][dim] unit directions or NULL */
  int32_t n_muscles;
} cls_mpm_body;

/* SolverMPM constants (multitask/solver_mpm.py:8-52, config_sim.py:123-129). */
typedef struct {
  int32_t max_steps;            /* trajectory length T */
  int32_t n_grid;               /* simulator.mpm.n_grid (dx = 1 / n_grid) */
  int32_t bound;                /* simulator.bound: sticky layer width in cells */
  int32_t material;             /* CLS_MPM_* */
  int32_t precision;            /* 32 or 64 */
  int32_t checkpoint_every;     /* K */
  double dt, gravity, p_vol, mu, la, act_strength, mass;
  int32_t tile_nodes;           /* > 0: warp-private shared-memory tiles of this many grid
                                   nodes (at most 1024) for the gathers and scatters; 0
                                   (default) or < 0: gathers through L1 and 16-byte vector
                                   reductions straight to the grid */
  int32_t particle_order;       /* internal particle order (results are the same up to the
                                   order of FP additions): CLS_MPM_ORDER_CELLS (0) or
                                   CLS_MPM_ORDER_BASE_RUNS (1, cls_mpm_default_params) */
} cls_mpm_params;

/* CLS_MPM_ORDER_CELLS: Morton order of the initial cells with the 32 lanes of
 * a warp in 32 different cells (every lane's reductions on distinct nodes).
 * CLS_MPM_ORDER_BASE_RUNS: particles sorted by the base cell of their stencil
 * (floor(x / dx - 0.5)) at creation, so that lanes of a warp form runs that
 * scatter to the same 27 nodes; in the forward P2G each run's contributions
 * are summed by warp shuffles and its first lane issues one 16-byte reduction
 * per node (runs are found every substep from the current positions, so any
 * motion stays exact); the adjoint's scatter reduces per lane.  tile_nodes
 * must be <= 0. */
#define CLS_MPM_ORDER_CELLS 0
#define CLS_MPM_ORDER_BASE_RUNS 1

/* Fills *p with the reference's 2D MPM constants (dt 1e-3, gravity -10,
 * n_grid 32, bound 3, p_vol 1, mu = la = 40, act_strength 4, mass 1), no
 * tiles and the base-cell particle order. */
void cls_mpm_default_params(cls_mpm_params* p);
/* Replaces SolverMPM.__init__ + initialize_robot (solver_mpm.py:7-58). */
int cls_mpm_create(const cls_mpm_body* body, const cls_mpm_params* params, int32_t n_envs,
                   cls_mpm** out);
int cls_mpm_destroy(cls_mpm* sim);
const char* cls_mpm_last_error(const cls_mpm* sim);
int cls_mpm_set_stream(cls_mpm* sim, void* stream);
/* x[0], v[0] ([n_envs][n_particles][dim]); C = 0 and F = I as clear_states
 * does (solver_mpm.py:60-71). */
int cls_mpm_set_state(cls_mpm* sim, const double* x0, const double* v0);
/* actuation [T][n_envs][n_muscles] (the solver's actuation field). */
int cls_mpm_set_actuation(cls_mpm* sim, const double* act);
/* Centre-tracking loss sum_t w_t sum_env |c_t - target_t|^2 with c the
 * particle-weighted centre: w [T+1], target [T+1][n_envs][dim], particle
 * weights [n_particles] (NULL: uniform = compute_center, solver_mpm.py:167-173). */
int cls_mpm_set_loss(cls_mpm* sim, const double* w, const double* target, const double* pw);
/* steps x advance_core (clear_grid, p2g, grid_op, g2p; solver_mpm.py:175-180). */
int cls_mpm_forward(cls_mpm* sim, int32_t steps);
int cls_mpm_loss(cls_mpm* sim, double* loss);
/* Reverse pass (advance_core_grad, solver_mpm.py:182-190, over checkpointed
 * segments). */
int cls_mpm_backward(cls_mpm* sim);
int cls_mpm_get_final_state(cls_mpm* sim, double* x, double* v, double* C, double* F);
/* d loss / d actuation [T][n_envs][n_muscles] and / d initial x, v, C, F. */
int cls_mpm_get_grads(cls_mpm* sim, double* gact, double* gx0, double* gv0, double* gC0,
                      double* gF0);
/* centres [T+1][n_envs][dim] of the last rollout. */
int cls_mpm_get_centers(cls_mpm* sim, double* centers);
/* forward + backward of `steps` captured into a CUDA graph; replay. */
int cls_mpm_graph_capture(cls_mpm* sim, int32_t steps);
int cls_mpm_graph_launch(cls_mpm* sim);
/* Per-kernel CUDA-event timing on the handle's stream (no counterpart in the
 * reference).  Categories: 0 particle kernel of the first pass (G2P of step f
 * fused with P2G of step f+1), 1 the same kernel in the reverse pass's
 * recompute, 2 grid update, 3 particle adjoint (P2G^T of step f fused with
 * G2P^T of step f-1), 4 grid adjoint, 5 other (centre and actuation-gradient
 * reductions, list resets).  ms / launches have CLS_MPM_PROFILE_KINDS entries. */
/* Measured throughput (operations/s, *ops_per_s) of the particle kernels'
 * scatter instruction -- 16-byte vector reductions into an n_nodes x 16-byte
 * buffer (pass the kernels' grid size: an L2-resident grid measures the L2
 * reduction rate), each warp's lanes on distinct nodes of one 1 KB block --
 * over about n_ops reductions; the denominator of the MPM scatter roofline.
 * Allocates its own buffer on the current device.  No reference
 * counterpart. */
int cls_mpm_reduction_peak(int64_t n_nodes, int64_t n_ops, double* ops_per_s);
#define CLS_MPM_PROFILE_KINDS 6
int cls_mpm_profile_enable(cls_mpm* sim, int32_t on);
int cls_mpm_profile_read(cls_mpm* sim, double* ms, int64_t* launches, int32_t reset);

/* ---------------------------------------------------------------------------
 * Mass-spring substeps without any allocation.  This entry point has no
 * counterpart in the reference; it exists for callers that may not allocate
 * device memory (a host runtime that owns a fixed device-memory budget or pool,
 * or code that must not allocate while a surrounding system captures work) and
 * therefore cannot create a cls_sim, whose buffers come from cudaMalloc.
 *
 * Runs n_substeps of spring forces (atomic scatter into a velocity increment)
 * followed by the damped, ground-contact advance, in place on the caller's x
 * and v.  All pointers are device pointers owned by the caller; the call
 * allocates nothing (no cudaMalloc, no library allocator) and keeps its only
 * scratch -- the velocity increment, n_envs * n_vertices * 3 floats -- in a
 * fixed 2^21-float (8 MiB) array inside the library that every GPU loading the
 * library holds until exit.  Larger problems are rejected with
 * CLS_ERR_INVALID and a message.  All calls share that array: calls that
 * overlap on the GPU race and must be serialised by the caller.  Each call
 * clears the part it uses first.  The array's device address belongs to a CUDA
 * context: the first call in each context (a device's primary context, or one
 * the caller created with the driver API and made current) resolves it with
 * that context current; make that first call before any stream capture in that
 * context.  Spring endpoints must lie in [0, n_vertices); springs whose
 * endpoints do not are skipped.  A CUDA error already pending when the call
 * starts is left pending and reported as CLS_ERR_CUDA, with nothing launched.
 * --------------------------------------------------------------------------- */
typedef struct {
  int32_t n_envs, n_vertices, n_springs, n_substeps;
  const int32_t* spring_a;      /* [n_springs] first endpoint, in [0, n_vertices) */
  const int32_t* spring_b;      /* [n_springs] second endpoint, in [0, n_vertices) */
  const float* rest_length;     /* [n_springs] */
  const float* stiffness;       /* [n_springs] as applied (after any scaling) */
  const float* actuation_coef;  /* [n_springs] */
  const float* actuation;       /* [n_envs][n_springs], held for all substeps */
  float* x;                     /* [n_envs][n_vertices][3], advanced in place */
  float* v;                     /* [n_envs][n_vertices][3], advanced in place */
  float dt, gravity, ground_height, drag_damping, dashpot_damping, friction;
  char* error_message;          /* optional buffer for a failure message */
  int32_t error_capacity;
} cls_noalloc_advance;

int cls_ms_advance_noalloc(const cls_noalloc_advance* args, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CLS_B200_H_ */
