/*
 * ms_oracle.c -- FP64 CPU oracle for the differentiable mass-spring substep.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker the CUDA path is compared
 * against; it is never linked into, called by, or shipped with the product
 * library.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load it.
 *
 * It restates, loop for loop, the Taichi kernels of the reference
 * (erizmr/Complex-locomotion-skill-learning-via-differentiable-physics) over
 * full-trajectory fields laid out [t][env][i] exactly as the reference places
 * them (multitask/solver_mass_spring.py:25-56, multitask/nn.py:97-105,
 * multitask/taichi_env.py:123-129).  The reverse pass is written by hand and
 * follows Taichi's reverse-mode rules for the same statements (ti.ad.Tape in
 * multitask/diffphy_trainer.py:246): every kernel's adjoint accumulates into the
 * .grad of what it read, kernels are replayed in reverse launch order, branch
 * conditions are re-evaluated on the recorded values, and min/max route the
 * adjoint to the first operand only when it is strictly selected (ties go to the
 * second operand).
 *
 * Generalisations beyond the reference, all defaulting to the reference:
 *   - the MLP may have 1..4 hidden layers (reference: 1, multitask/nn.py:130-146);
 *   - hidden / output activation may be sin (reference) or tanh;
 *   - the MLP output may feed every spring (reference: n_output = n_springs,
 *     multitask/diffphy_trainer.py:178-185) or only actuated springs (out_index);
 *   - friction coefficient is a parameter (reference hard-codes 0.4,
 *     multitask/solver_mass_spring.py:136);
 *   - the env count B that the loss terms are divided by may be set apart
 *     from the batch's own (loss_envs), for a batch that is one shard of a
 *     larger batch.
 *
 * Precision: double throughout, as the reference (multitask/utils.py:12).
 * Parallelism: OpenMP over environments (independent in every kernel).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAX_LAYERS 5

enum { ORC_ACT_SIN = 0, ORC_ACT_TANH = 1 };
enum {
  ORC_LOSS_VELOCITY = 1, ORC_LOSS_HEIGHT = 2, ORC_LOSS_POSE = 4,
  ORC_LOSS_ACTUATION = 8, ORC_LOSS_ROTATION = 16, ORC_LOSS_CRAWL = 32
};
/* slots of the loss vector: total followed by the reference's loss_dict order
 * (multitask/taichi_env.py:82-88) */
enum { L_TOTAL = 0, L_VEL = 1, L_HEIGHT = 2, L_POSE = 3, L_ROT = 4, L_WEIGHT = 5,
       L_ACT = 6, L_CRAWL = 7, L_COUNT = 8 };

typedef struct {
  int B, N, S, T;
  int n_sin, dup_v, dup_h, dup_c, n_in, n_out;
  int n_layers;                    /* weight layers = hidden layers + 1 */
  int width[ORC_MAX_LAYERS + 1];   /* width[0] = n_in ... width[n_layers] = n_out */
  int act_hidden, act_out;
  int run_period, turn_period, jump_period, robot_id;
  int loss_mask;
  int n_threads;                   /* 0: OpenMP default */
  int loss_envs;                   /* B of the loss normalisation; 0: the batch's B (reference) */
  double dt, gravity, ground, drag, dashpot, friction, spring_omega;
  double max_speed, max_height;
  /* robot */
  const int *sa, *sb, *out_index;
  const double *len, *stiff, *coef; /* stiff already divided by 10 (initialize_robot) */
  const double *init_obj;           /* [N][3] initial_objects, for the pose loss */
  /* MLP: W[l] is [width[l+1]][width[l]], b[l] is [width[l+1]] */
  double *W[ORC_MAX_LAYERS], *b[ORC_MAX_LAYERS], *gW[ORC_MAX_LAYERS], *gb[ORC_MAX_LAYERS];
  /* trajectory fields */
  double *x, *v, *v_inc;            /* [T][B][N][3] */
  double *center;                   /* [T][B][3] */
  double *height, *upper, *rotation;/* [T][B] */
  double *act;                      /* [T][B][S] solver.actuation */
  double *input;                    /* [T][B][n_in] */
  double *z[ORC_MAX_LAYERS];        /* [T][B][width[l+1]] pre-bias accumulators */
  double *tv, *th, *tc;             /* [T][B][3], [T][B], [T][B] */
  /* adjoints */
  double *gx, *gv, *gv_inc, *gcenter, *gheight, *gupper, *gact, *ginput;
  double *gz[ORC_MAX_LAYERS];
  /* losses */
  double *loss;                     /* [L_COUNT] */
  double *loss_batch;               /* [L_COUNT][B] */
  double *current_max_height;       /* [1] */
} orc_ms;

/* ---------------------------------------------------------------- helpers */
#define IX3(p, t, k, i) (((((size_t)(t) * (p)->B + (k)) * (p)->N) + (i)) * 3)

/* Precision-study hooks, compiled only into libms_oracle_study.so
 * (-DORC_STUDY; tests/study_fp32_state.py drives them).  They model an
 * implementation that computes in FP64 but stores chosen fields in FP32
 * (ST_* bits of st_round: the value written is rounded to the nearest float),
 * optionally keeps the positions exactly while every reader sees the rounded
 * copy (ST_X_EXACT: a compensated position update), and records or forces
 * the contact decisions of advance_toi.  Without ORC_STUDY every hook is the
 * identity and the oracle is the plain FP64 restatement. */
enum { ST_X = 1, ST_V = 2, ST_VINC = 4, ST_MLP = 8, ST_INPUT = 16, ST_ADJ = 32, ST_WSUM = 64,
       ST_X_EXACT = 128 };
#ifdef ORC_STUDY
static int st_round = 0;
static unsigned char* st_flags = NULL; /* [T][B][N] contact decisions */
static int st_flag_mode = 0;           /* 1: record, 2: force */
static double* st_xe = NULL;           /* [T][B][N][3] exact positions (ST_X_EXACT) */
void orc_study_set(int round_bits, unsigned char* flags, int flag_mode, double* x_exact) {
  st_round = round_bits;
  st_flags = flags;
  st_flag_mode = flags ? flag_mode : 0;
  st_xe = x_exact;
}
#define ST_ROUND(bit, v) ((st_round & (bit)) ? (double)(float)(v) : (v))
static int st_contact(const orc_ms* p, int t, int k, int i, int hit, int forward) {
  size_t f = ((size_t)t * p->B + k) * p->N + i;
  if (st_flag_mode == 2 || (st_flag_mode == 1 && !forward)) return st_flags[f];
  if (st_flag_mode == 1) st_flags[f] = (unsigned char)hit;
  return hit;
}
#define ST_XE(p, t, k, i) ((st_round & ST_X_EXACT) ? st_xe + IX3(p, t, k, i) : p->x + IX3(p, t, k, i))
#else
#define ST_ROUND(bit, v) (v)
#define st_contact(p, t, k, i, hit, fw) (hit)
#define ST_XE(p, t, k, i) (p->x + IX3(p, t, k, i))
#endif
#define IC3(p, t, k) ((((size_t)(t) * (p)->B) + (k)) * 3)
#define IB(p, t, k) (((size_t)(t) * (p)->B) + (k))
#define IS(p, t, k, s) ((((size_t)(t) * (p)->B + (k)) * (p)->S) + (s))
#define IIN(p, t, k, j) ((((size_t)(t) * (p)->B + (k)) * (p)->n_in) + (j))
#define IZ(p, l, t, k, i) ((((size_t)(t) * (p)->B + (k)) * (p)->width[(l) + 1]) + (i))

static double actf(int kind, double x) { return kind == ORC_ACT_TANH ? tanh(x) : sin(x); }
static double actd(int kind, double x) {
  if (kind == ORC_ACT_TANH) { double y = tanh(x); return 1.0 - y * y; }
  return cos(x);
}

static void set_threads(const orc_ms* p) {
#ifdef _OPENMP
  if (p->n_threads > 0) omp_set_num_threads(p->n_threads);
#else
  (void)p;
#endif
}

/* ================================================================ forward */

/* compute_center: multitask/solver_mass_spring.py:150-156 */
static void k_center(const orc_ms* p, int t, int k) {
  double* c = p->center + IC3(p, t, k);
  c[0] = c[1] = c[2] = 0.0;
  for (int i = 0; i < p->N; ++i)
    for (int d = 0; d < 3; ++d) c[d] += p->x[IX3(p, t, k, i) + d] / p->N;
  for (int d = 0; d < 3; ++d) c[d] = ST_ROUND(ST_INPUT, c[d]);
}

/* compute_height: multitask/solver_mass_spring.py:158-173 */
static void k_height(const orc_ms* p, int t, int k) {
  double h = 10.0;
  for (int i = 0; i < p->N; ++i) h = fmin(h, p->x[IX3(p, t, k, i) + 1]);
  if (t % p->jump_period == 0) p->height[IB(p, t, k)] = h;
  else p->height[IB(p, t, k)] = fmax(p->height[IB(p, t - 1, k)], h);
  double u = -10.0;
  for (int i = 0; i < p->N; ++i) u = fmax(u, p->x[IX3(p, t, k, i) + 1]);
  p->upper[IB(p, t, k)] = u;
}

/* compute_rotation: multitask/solver_mass_spring.py:175-192 (forward only: no
 * loss of the reference reads the rotation field) */
static void k_rotation(const orc_ms* p, int t, int k) {
  double dir[3];
  if (p->robot_id == 100) {
    for (int d = 0; d < 3; ++d)
      dir[d] = p->x[IX3(p, t, k, 45) + d] + p->x[IX3(p, t, k, 46) + d] -
               p->x[IX3(p, t, k, 34) + d] - p->x[IX3(p, t, k, 36) + d];
  } else {
    double hc[3] = {0, 0, 0}, tc[3] = {0, 0, 0}, hn = 0, tn = 0;
    for (int i = 0; i < p->N; ++i) {
      const double* xi = p->x + IX3(p, t, k, i);
      if (p->x[IX3(p, 0, k, i)] < p->center[IC3(p, 0, k)]) {
        for (int d = 0; d < 3; ++d) hc[d] += xi[d];
        hn += 1.0;
      } else {
        for (int d = 0; d < 3; ++d) tc[d] += xi[d];
        tn += 1.0;
      }
    }
    for (int d = 0; d < 3; ++d) dir[d] = -hc[d] * tn + tc[d] * hn;
  }
  p->rotation[IB(p, t, k)] = atan2(dir[2], dir[0]);
}

/* nn_input: multitask/taichi_env.py:149-183 (3D branch) */
static void k_nn_input(const orc_ms* p, int t, int k, int offset) {
  double* in = p->input + IIN(p, t, k, 0);
  for (int j = 0; j < p->n_sin; ++j)
    in[j] = sin(p->spring_omega * (double)(t + offset) * p->dt +
                2.0 * M_PI / p->n_sin * (double)j);
  const double* c = p->center + IC3(p, t, k);
  for (int j = 0; j < p->N; ++j) {
    const double* xj = p->x + IX3(p, t, k, j);
    for (int d = 0; d < 3; ++d) {
      in[j * 6 + p->n_sin + d] = ST_ROUND(ST_INPUT, (xj[d] - c[d]) / 0.2);
      in[j * 6 + p->n_sin + 3 + d] = 0.0;
    }
  }
  int base = p->N * 6 + p->n_sin;
  for (int j = 0; j < p->dup_v; ++j) {
    in[base + j * 2] = p->tv[IC3(p, t, k) + 0] / p->max_speed;
    in[base + j * 2 + 1] = p->tv[IC3(p, t, k) + 2] / p->max_speed;
  }
  base += p->dup_v * 2;
  for (int j = 0; j < p->dup_h; ++j) in[base + j] = p->th[IB(p, t, k)];
  base += p->dup_h;
  for (int j = 0; j < p->dup_c; ++j) in[base + j] = p->tc[IB(p, t, k)];
}

/* Model.nn1 / nn2 generalised to n_layers: multitask/nn.py:130-146.
 * z = W a_prev (accumulated from zero, nn.py:116-121), a = act(z + b). */
static void k_mlp(const orc_ms* p, int t, int k, double* scratch_a, double* scratch_b) {
  const double* a_prev = p->input + IIN(p, t, k, 0);
  for (int l = 0; l < p->n_layers; ++l) {
    int nin = p->width[l], nout = p->width[l + 1];
    double* z = p->z[l] + IZ(p, l, t, k, 0);
    double* a_next = (l & 1) ? scratch_b : scratch_a;
    int last = (l == p->n_layers - 1);
    for (int i = 0; i < nout; ++i) {
      double s = 0.0;
      const double* w = p->W[l] + (size_t)i * nin;
      for (int j = 0; j < nin; ++j) s += w[j] * a_prev[j];
      z[i] = ST_ROUND(ST_MLP, s);
      a_next[i] = ST_ROUND(ST_MLP, actf(last ? p->act_out : p->act_hidden, z[i] + p->b[l][i]));
    }
    a_prev = a_next;
  }
  /* output_act is the solver's actuation field (diffphy_trainer.py:178-185) */
  double* act = p->act + IS(p, t, k, 0);
  for (int s = 0; s < p->S; ++s) {
    int o = p->out_index[s];
    act[s] = (o >= 0) ? a_prev[o] : 0.0;
  }
}

/* apply_spring_force: multitask/solver_mass_spring.py:86-105 */
static void k_spring(const orc_ms* p, int t, int k) {
  for (int i = 0; i < p->S; ++i) {
    int a = p->sa[i], b = p->sb[i];
    const double* xa = p->x + IX3(p, t, k, a);
    const double* xb = p->x + IX3(p, t, k, b);
    const double* va = p->v + IX3(p, t, k, a);
    const double* vb = p->v + IX3(p, t, k, b);
    double dist[3], n2 = 0.0;
    for (int d = 0; d < 3; ++d) { dist[d] = xa[d] - xb[d]; n2 += dist[d] * dist[d]; }
    double length = sqrt(n2 + 1e-8) + 1e-4;
    double target = p->len[i] * (1.0 + p->coef[i] * p->act[IS(p, t, k, i)]);
    double sc = p->dt * (length - target) * p->stiff[i] / length;
    double invlen = 1.0 / sqrt(n2);             /* normalized(): 1/(norm()+0) */
    double dn[3], vrel = 0.0;
    for (int d = 0; d < 3; ++d) { dn[d] = dist[d] * invlen; vrel += (va[d] - vb[d]) * dn[d]; }
    double* ia = p->v_inc + IX3(p, t, k, a);
    double* ib = p->v_inc + IX3(p, t, k, b);
    for (int d = 0; d < 3; ++d) {
      double imp = sc * dist[d] + p->dashpot * vrel * dn[d];
      ia[d] -= imp;
      ib[d] += imp;
    }
  }
#ifdef ORC_STUDY
  if (st_round & ST_VINC)
    for (int i = 0; i < 3 * p->N; ++i) p->v_inc[IX3(p, t, k, 0) + i] = ST_ROUND(ST_VINC, p->v_inc[IX3(p, t, k, 0) + i]);
#endif
}

/* advance_toi: multitask/solver_mass_spring.py:117-148; writes step t from t-1 */
static void k_advance(const orc_ms* p, int t, int k) {
  double s = exp(-p->dt * p->drag);
  for (int i = 0; i < p->N; ++i) {
    const double* v0 = p->v + IX3(p, t - 1, k, i);
    const double* x0 = ST_XE(p, t - 1, k, i);
    const double* vi = p->v_inc + IX3(p, t - 1, k, i);
    double ov[3], nv[3], nx[3];
    for (int d = 0; d < 3; ++d) ov[d] = s * v0[d] + (d == 1 ? p->dt * p->gravity : 0.0) + vi[d];
    double toi = 0.0;
    for (int d = 0; d < 3; ++d) nv[d] = ov[d];
    double nx1 = x0[1] + p->dt * ov[1];
    if (st_contact(p, t, k, i, nx1 < p->ground && ov[1] < -1e-4, 1)) {
      toi = -(x0[1] - p->ground) / ov[1];
      double f = p->friction * (-ov[1]);
      nv[1] = 0.0;
      nv[0] = (ov[0] < 0) ? fmin(0.0, ov[0] + f) : fmax(0.0, ov[0] - f);
      nv[2] = (ov[2] < 0) ? fmin(0.0, ov[2] + f) : fmax(0.0, ov[2] - f);
    }
    for (int d = 0; d < 3; ++d) nx[d] = x0[d] + toi * ov[d] + (p->dt - toi) * nv[d];
    double* v1 = p->v + IX3(p, t, k, i);
    double* x1 = p->x + IX3(p, t, k, i);
    for (int d = 0; d < 3; ++d) { v1[d] = ST_ROUND(ST_V, nv[d]); x1[d] = ST_ROUND(ST_X, nx[d]); }
#ifdef ORC_STUDY
    if (st_round & ST_X_EXACT)
      for (int d = 0; d < 3; ++d) { st_xe[IX3(p, t, k, i) + d] = nx[d]; x1[d] = (double)(float)nx[d]; }
#endif
  }
}

/* One training rollout: the loop of DiffPhyTrainer.simulate,
 * multitask/diffphy_trainer.py:231-255 (clear_states, nn.clear, then
 * t in [0, steps-2]: pre_advance, nn_input, forward, advance).  x[0], v[0] and the
 * targets are inputs.  Fields at t = steps-1 that pre_advance/forward never write
 * (center, height, upper, rotation, actuation) stay zero, as in the reference. */
static int forward_impl(const orc_ms* p, int steps, int eval_mode) {
  /* training: t in [0, steps-2] (diffphy_trainer.py:248); evaluation:
   * t in [0, steps] (diffphy_trainer.py:258), which writes x[steps+1] */
  int last = eval_mode ? steps : steps - 2;
  if (eval_mode) {
    if (steps < 0 || steps + 1 >= p->T) return -1;
  } else if (steps < 2 || steps > p->T) {
    return -1;
  }
  set_threads(p);
  int maxw = 0;
  for (int l = 0; l <= p->n_layers; ++l) if (p->width[l] > maxw) maxw = p->width[l];
#pragma omp parallel
  {
    double* sa = (double*)malloc(sizeof(double) * maxw);
    double* sb = (double*)malloc(sizeof(double) * maxw);
#pragma omp for schedule(dynamic, 1)
    for (int k = 0; k < p->B; ++k) {
      /* clear_states: v_inc := 0 for all t (solver_mass_spring.py:69-84) */
      for (int t = 0; t <= last; ++t)
        memset(p->v_inc + IX3(p, t, k, 0), 0, sizeof(double) * 3 * p->N);
      for (int t = 0; t <= last; ++t) {
        k_center(p, t, k);
        k_height(p, t, k);
        k_rotation(p, t, k);
        k_nn_input(p, t, k, 0);
        k_mlp(p, t, k, sa, sb);
        k_spring(p, t, k);
        k_advance(p, t + 1, k);
      }
    }
    free(sa);
    free(sb);
  }
  return 0;
}

int orc_ms_forward(const orc_ms* p, int steps) { return forward_impl(p, steps, 0); }

/* forward-only evaluation rollout (DiffPhyTrainer.simulate(train=False)) */
int orc_ms_forward_eval(const orc_ms* p, int steps) { return forward_impl(p, steps, 1); }

/* ================================================================= losses */

/* get_loss: multitask/taichi_env.py:185-331 (3D branches).  Terms whose time
 * index would be read past the end of the fields (t == steps in the pose / crawl
 * loops) are skipped. */
int orc_ms_loss(const orc_ms* p, int steps) {
  const int B = p->B, rp = p->run_period, tp = p->turn_period, jp = p->jump_period;
  const double LB = p->loss_envs > 0 ? p->loss_envs : B;
  memset(p->loss, 0, sizeof(double) * L_COUNT);
  memset(p->loss_batch, 0, sizeof(double) * L_COUNT * B);
  double cmh = p->current_max_height ? p->current_max_height[0] : 0.0;
  for (int k = 0; k < B; ++k) {
    if (p->loss_mask & ORC_LOSS_VELOCITY) {           /* taichi_env.py:185-211 */
      for (int t = rp; t <= steps && t < p->T; ++t) {
        if (t % tp > rp) {
          const double* c1 = p->center + IC3(p, t, k);
          const double* c0 = p->center + IC3(p, t - rp, k);
          const double* tv = p->tv + IC3(p, t - rp, k);
          double ex = c1[0] - c0[0] - tv[0], ez = c1[2] - c0[2] - tv[2];
          double lx = ex * ex / LB / steps * 100, lz = ez * ez / LB / steps * 100;
          p->loss[L_VEL] += lx + lz;
          p->loss_batch[L_VEL * B + k] += (lx + lz) * LB;
        }
      }
    }
    if (p->loss_mask & ORC_LOSS_HEIGHT) {             /* taichi_env.py:213-222 */
      for (int t = 1; t <= steps && t < p->T; ++t) {
        if (t % jp == jp - 1 && p->th[IB(p, t, k)] > 0.1 + 1e-6) {
          double e = p->height[IB(p, t, k)] - p->th[IB(p, t, k)];
          double lh = e * e / LB / (steps / jp) * 100;
          p->loss[L_HEIGHT] += lh;
          p->loss_batch[L_HEIGHT * B + k] += lh * LB;
          if (p->height[IB(p, t, k)] > cmh) cmh = p->height[IB(p, t, k)];
        }
      }
    }
    if (p->loss_mask & ORC_LOSS_POSE) {               /* taichi_env.py:224-233 */
      for (int t = 1; t <= steps && t < p->T; ++t) {
        if (t % jp == 0) {
          for (int i = 0; i < p->N; ++i) {
            double d2 = 0.0;
            for (int d = 0; d < 3; ++d) {
              double e = p->x[IX3(p, t, k, i) + d] - p->init_obj[i * 3 + d];
              d2 += e * e;
            }
            double lp = d2 / LB / (steps / jp);
            p->loss[L_POSE] += lp;
            p->loss_batch[L_POSE * B + k] += lp * LB;
          }
        }
      }
    }
    if (p->loss_mask & ORC_LOSS_ACTUATION) {          /* taichi_env.py:276-285 */
      for (int t = 0; t < steps; ++t) {
        if (p->th[IB(p, t, k)] < 0.1 + 1e-4) {
          double lim = pow(fabs(p->tv[IC3(p, t, k)]) / 0.08, 0.5);
          for (int i = 0; i < p->S; ++i) {
            double la = fmax(fabs(p->act[IS(p, t, k, i)]) - lim, 0.0) / p->S / LB / steps * 10;
            p->loss[L_ACT] += la;
            p->loss_batch[L_ACT * B + k] += la * LB;
          }
        }
      }
    }
    if (p->loss_mask & ORC_LOSS_ROTATION) {           /* taichi_env.py:235-252 */
      for (int t = 1; t <= steps && t < p->T; ++t) {
        if (t % tp > rp) {
          double ang = p->th[IB(p, t - rp, k)] * 72. / 180. * 3.1415926535;
          double ca = cos(ang), sn = sin(ang);
          const double* c1 = p->center + IC3(p, t, k);
          const double* c0 = p->center + IC3(p, t - rp, k);
          for (int i = 0; i < p->N; ++i) {
            const double* x1 = p->x + IX3(p, t, k, i);
            const double* x0 = p->x + IX3(p, t - rp, k, i);
            double t0[3], t1[3], t2[3];
            for (int d = 0; d < 3; ++d) { t0[d] = x1[d] - c1[d]; t1[d] = x0[d] - c0[d]; }
            t2[0] = ca * t1[0] - sn * t1[2];
            t2[1] = t1[1];
            t2[2] = sn * t1[0] + ca * t1[2];
            double n2 = 0.0;
            for (int d = 0; d < 3; ++d) n2 += (t0[d] - t2[d]) * (t0[d] - t2[d]);
            double lr = n2 / steps / 40;
            p->loss[L_ROT] += lr;
            p->loss_batch[L_ROT * B + k] += lr * LB;
          }
        }
      }
    }
    if (p->loss_mask & ORC_LOSS_CRAWL) {              /* taichi_env.py:287-293 */
      for (int t = 1; t <= steps && t < p->T; ++t) {
        if (p->tc[IB(p, t, k)] > 1 - 1e-4) {
          double e = fmax(p->upper[IB(p, t, k)] - 0.1, 0.0);
          double lc = e * e / LB / steps * 5.;
          p->loss[L_CRAWL] += lc;
          p->loss_batch[L_CRAWL * B + k] += lc * LB;
        }
      }
    }
  }
  /* compute_loss_final / _batch: taichi_env.py:295-331 */
  for (int l = 1; l < L_COUNT; ++l) p->loss[L_TOTAL] += p->loss[l];
  for (int k = 0; k < B; ++k)
    for (int l = 1; l < L_COUNT; ++l) p->loss_batch[L_TOTAL * B + k] += p->loss_batch[l * B + k];
  if (p->current_max_height) p->current_max_height[0] = cmh;
  return 0;
}

/* ================================================================ reverse */

/* adjoint of the loss kernels with loss.grad = 1 (Tape seeding) */
static void a_loss(const orc_ms* p, int steps, int k) {
  const int rp = p->run_period, tp = p->turn_period, jp = p->jump_period;
  const double B = p->loss_envs > 0 ? p->loss_envs : p->B;
  if (p->loss_mask & ORC_LOSS_VELOCITY) {
    for (int t = rp; t <= steps && t < p->T; ++t) {
      if (t % tp > rp) {
        const double* c1 = p->center + IC3(p, t, k);
        const double* c0 = p->center + IC3(p, t - rp, k);
        const double* tv = p->tv + IC3(p, t - rp, k);
        double g = 100.0 / steps / B * 2.0;
        double ex = (c1[0] - c0[0] - tv[0]) * g, ez = (c1[2] - c0[2] - tv[2]) * g;
        p->gcenter[IC3(p, t, k) + 0] += ex;
        p->gcenter[IC3(p, t - rp, k) + 0] -= ex;
        p->gcenter[IC3(p, t, k) + 2] += ez;
        p->gcenter[IC3(p, t - rp, k) + 2] -= ez;
      }
    }
  }
  if (p->loss_mask & ORC_LOSS_HEIGHT) {
    for (int t = 1; t <= steps && t < p->T; ++t) {
      if (t % jp == jp - 1 && p->th[IB(p, t, k)] > 0.1 + 1e-6) {
        double e = p->height[IB(p, t, k)] - p->th[IB(p, t, k)];
        p->gheight[IB(p, t, k)] += 2.0 * e * 100.0 / (steps / jp) / B;
      }
    }
  }
  if (p->loss_mask & ORC_LOSS_POSE) {
    for (int t = 1; t <= steps && t < p->T; ++t) {
      if (t % jp == 0) {
        for (int i = 0; i < p->N; ++i)
          for (int d = 0; d < 3; ++d) {
            double e = p->x[IX3(p, t, k, i) + d] - p->init_obj[i * 3 + d];
            p->gx[IX3(p, t, k, i) + d] += 2.0 * e / (steps / jp) / B;
          }
      }
    }
  }
  if (p->loss_mask & ORC_LOSS_ACTUATION) {
    for (int t = 0; t < steps; ++t) {
      if (p->th[IB(p, t, k)] < 0.1 + 1e-4) {
        double lim = pow(fabs(p->tv[IC3(p, t, k)]) / 0.08, 0.5);
        for (int i = 0; i < p->S; ++i) {
          double a = p->act[IS(p, t, k, i)];
          double arg = fabs(a) - lim;
          if (0.0 < arg) {   /* max(arg, 0): adjoint to arg only when strictly larger */
            double sg = (a > 0) - (a < 0);
            p->gact[IS(p, t, k, i)] += sg * 10.0 / steps / B / p->S;
          }
        }
      }
    }
  }
  if (p->loss_mask & ORC_LOSS_ROTATION) {
    for (int t = 1; t <= steps && t < p->T; ++t) {
      if (t % tp > rp) {
        double ang = p->th[IB(p, t - rp, k)] * 72. / 180. * 3.1415926535;
        double ca = cos(ang), sn = sin(ang);
        const double* c1 = p->center + IC3(p, t, k);
        const double* c0 = p->center + IC3(p, t - rp, k);
        double gc1[3] = {0, 0, 0}, gc0[3] = {0, 0, 0};
        for (int i = 0; i < p->N; ++i) {
          const double* x1 = p->x + IX3(p, t, k, i);
          const double* x0 = p->x + IX3(p, t - rp, k, i);
          double t0[3], t1[3], t2[3], g0[3], g2[3], g1[3];
          for (int d = 0; d < 3; ++d) { t0[d] = x1[d] - c1[d]; t1[d] = x0[d] - c0[d]; }
          t2[0] = ca * t1[0] - sn * t1[2];
          t2[1] = t1[1];
          t2[2] = sn * t1[0] + ca * t1[2];
          for (int d = 0; d < 3; ++d) { g0[d] = 2.0 * (t0[d] - t2[d]) / 40.0 / steps; g2[d] = -g0[d]; }
          g1[0] = ca * g2[0] + sn * g2[2];
          g1[1] = g2[1];
          g1[2] = -sn * g2[0] + ca * g2[2];
          for (int d = 0; d < 3; ++d) {
            p->gx[IX3(p, t, k, i) + d] += g0[d];
            gc1[d] -= g0[d];
            p->gx[IX3(p, t - rp, k, i) + d] += g1[d];
            gc0[d] -= g1[d];
          }
        }
        for (int d = 0; d < 3; ++d) {
          p->gcenter[IC3(p, t, k) + d] += gc1[d];
          p->gcenter[IC3(p, t - rp, k) + d] += gc0[d];
        }
      }
    }
  }
  if (p->loss_mask & ORC_LOSS_CRAWL) {
    for (int t = 1; t <= steps && t < p->T; ++t) {
      if (p->tc[IB(p, t, k)] > 1 - 1e-4) {
        double e = p->upper[IB(p, t, k)] - 0.1;
        if (0.0 < e) p->gupper[IB(p, t, k)] += 2.0 * e * 5.0 / steps / B;
      }
    }
  }
}

/* adjoint of advance_toi(t): reads x,v,v_inc[t-1], writes grads of them */
static void a_advance(const orc_ms* p, int t, int k) {
  double s = exp(-p->dt * p->drag);
  for (int i = 0; i < p->N; ++i) {
    const double* v0 = p->v + IX3(p, t - 1, k, i);
    const double* x0 = p->x + IX3(p, t - 1, k, i);
    const double* vi = p->v_inc + IX3(p, t - 1, k, i);
    double* gv1 = p->gv + IX3(p, t, k, i);
    double* gx1 = p->gx + IX3(p, t, k, i);
    double ov[3], nv[3];
    for (int d = 0; d < 3; ++d) ov[d] = s * v0[d] + (d == 1 ? p->dt * p->gravity : 0.0) + vi[d];
    double toi = 0.0;
    for (int d = 0; d < 3; ++d) nv[d] = ov[d];
    double nx1 = x0[1] + p->dt * ov[1];
    int hit = st_contact(p, t, k, i, nx1 < p->ground && ov[1] < -1e-4, 0);
    double f = 0.0;
    if (hit) {
      toi = -(x0[1] - p->ground) / ov[1];
      f = p->friction * (-ov[1]);
      nv[1] = 0.0;
      nv[0] = (ov[0] < 0) ? fmin(0.0, ov[0] + f) : fmax(0.0, ov[0] - f);
      nv[2] = (ov[2] < 0) ? fmin(0.0, ov[2] + f) : fmax(0.0, ov[2] - f);
    }
    /* new_x = old_x + toi*old_v + (dt - toi)*new_v ; v[t] = new_v */
    double gox[3], gov[3], gnv[3], gtoi = 0.0;
    for (int d = 0; d < 3; ++d) {
      gox[d] = gx1[d];
      gov[d] = toi * gx1[d];
      gnv[d] = (p->dt - toi) * gx1[d] + gv1[d];
      gtoi += gx1[d] * ov[d] - gx1[d] * nv[d];
    }
    if (hit) {
      double gf = 0.0;
      /* x component: min(0, ov0 + f) or max(0, ov0 - f) */
      if (ov[0] < 0) {
        if (!(0.0 < ov[0] + f)) { gov[0] += gnv[0]; gf += gnv[0]; }
      } else {
        if (!(ov[0] - f < 0.0)) { gov[0] += gnv[0]; gf -= gnv[0]; }
      }
      if (ov[2] < 0) {
        if (!(0.0 < ov[2] + f)) { gov[2] += gnv[2]; gf += gnv[2]; }
      } else {
        if (!(ov[2] - f < 0.0)) { gov[2] += gnv[2]; gf -= gnv[2]; }
      }
      /* f = friction * (-ov1) */
      gov[1] += -p->friction * gf;
      /* toi = -(x0_1 - ground) / ov1 */
      gox[1] += -gtoi / ov[1];
      gov[1] += gtoi * (x0[1] - p->ground) / (ov[1] * ov[1]);
    } else {
      for (int d = 0; d < 3; ++d) gov[d] += gnv[d];
    }
    double* gv0 = p->gv + IX3(p, t - 1, k, i);
    double* gx0 = p->gx + IX3(p, t - 1, k, i);
    double* gvi = p->gv_inc + IX3(p, t - 1, k, i);
    for (int d = 0; d < 3; ++d) {
      gx0[d] += gox[d];
      gv0[d] += s * gov[d];
      gvi[d] += gov[d];
    }
  }
}

/* adjoint of apply_spring_force(t) */
static void a_spring(const orc_ms* p, int t, int k) {
  for (int i = 0; i < p->S; ++i) {
    int a = p->sa[i], b = p->sb[i];
    const double* xa = p->x + IX3(p, t, k, a);
    const double* xb = p->x + IX3(p, t, k, b);
    const double* va = p->v + IX3(p, t, k, a);
    const double* vb = p->v + IX3(p, t, k, b);
    double dist[3], n2 = 0.0;
    for (int d = 0; d < 3; ++d) { dist[d] = xa[d] - xb[d]; n2 += dist[d] * dist[d]; }
    double r8 = sqrt(n2 + 1e-8);
    double length = r8 + 1e-4;
    double target = p->len[i] * (1.0 + p->coef[i] * p->act[IS(p, t, k, i)]);
    double sc = p->dt * (length - target) * p->stiff[i] / length;
    double r = sqrt(n2), invlen = 1.0 / r;
    double dn[3], dv[3], vrel = 0.0;
    for (int d = 0; d < 3; ++d) {
      dn[d] = dist[d] * invlen;
      dv[d] = va[d] - vb[d];
      vrel += dv[d] * dn[d];
    }
    double gimp[3];
    for (int d = 0; d < 3; ++d)
      gimp[d] = p->gv_inc[IX3(p, t, k, b) + d] - p->gv_inc[IX3(p, t, k, a) + d];
    /* imp = sc*dist + dashpot*vrel*dn */
    double gdist[3], gsc = 0.0, gvrel = 0.0, gdn[3];
    for (int d = 0; d < 3; ++d) {
      gdist[d] = sc * gimp[d];
      gsc += gimp[d] * dist[d];
      gvrel += p->dashpot * gimp[d] * dn[d];
      gdn[d] = p->dashpot * vrel * gimp[d];
    }
    /* vrel = dv . dn */
    for (int d = 0; d < 3; ++d) gdn[d] += gvrel * dv[d];
    double* gva = p->gv + IX3(p, t, k, a);
    double* gvb = p->gv + IX3(p, t, k, b);
    for (int d = 0; d < 3; ++d) { gva[d] += gvrel * dn[d]; gvb[d] -= gvrel * dn[d]; }
    /* dn = dist * invlen, invlen = 1/r, r = |dist| */
    double ginv = 0.0;
    for (int d = 0; d < 3; ++d) { gdist[d] += invlen * gdn[d]; ginv += gdn[d] * dist[d]; }
    double gr = -ginv / (r * r);
    for (int d = 0; d < 3; ++d) gdist[d] += gr * dist[d] / r;
    /* sc = dt*(length - target)*stiff/length */
    double glen = gsc * p->dt * p->stiff[i] * target / (length * length);
    double gtarget = -gsc * p->dt * p->stiff[i] / length;
    for (int d = 0; d < 3; ++d) gdist[d] += glen * dist[d] / r8;
    p->gact[IS(p, t, k, i)] += gtarget * p->len[i] * p->coef[i];
    double* gxa = p->gx + IX3(p, t, k, a);
    double* gxb = p->gx + IX3(p, t, k, b);
    for (int d = 0; d < 3; ++d) { gxa[d] += gdist[d]; gxb[d] -= gdist[d]; }
  }
}

/* adjoint of the MLP at step t; weight grads accumulate into per-thread
 * buffers gWt/gbt (summed after the parallel region) */
static void a_mlp(const orc_ms* p, int t, int k, double** gWt, double** gbt,
                  double* ga_cur, double* ga_prev, double* abuf) {
  int L = p->n_layers;
  /* actuation -> output activation grad */
  int nout = p->width[L];
  for (int o = 0; o < nout; ++o) ga_cur[o] = 0.0;
  for (int s = 0; s < p->S; ++s) {
    int o = p->out_index[s];
    if (o >= 0) ga_cur[o] += p->gact[IS(p, t, k, s)];
  }
  for (int l = L - 1; l >= 0; --l) {
    int nin = p->width[l], nou = p->width[l + 1];
    const double* z = p->z[l] + IZ(p, l, t, k, 0);
    int last = (l == L - 1);
    /* previous activation a_{l} (input of layer l) */
    const double* aprev;
    if (l == 0) {
      aprev = p->input + IIN(p, t, k, 0);
    } else {
      const double* zp = p->z[l - 1] + IZ(p, l - 1, t, k, 0);
      for (int j = 0; j < nin; ++j) abuf[j] = actf(p->act_hidden, zp[j] + p->b[l - 1][j]);
      aprev = abuf;
    }
    for (int j = 0; j < nin; ++j) ga_prev[j] = 0.0;
    for (int i = 0; i < nou; ++i) {
      double gz = ga_cur[i] * actd(last ? p->act_out : p->act_hidden, z[i] + p->b[l][i]);
      p->gz[l][IZ(p, l, t, k, i)] += gz;
      gbt[l][i] += gz;
      const double* w = p->W[l] + (size_t)i * nin;
      double* gw = gWt[l] + (size_t)i * nin;
      for (int j = 0; j < nin; ++j) {
        gw[j] += gz * aprev[j];
        ga_prev[j] += gz * w[j];
      }
    }
    for (int j = 0; j < nin; ++j) ga_cur[j] = ga_prev[j];
  }
  double* gin = p->ginput + IIN(p, t, k, 0);
  for (int j = 0; j < p->n_in; ++j) gin[j] += ga_cur[j];
}

/* adjoint of nn_input(t): only the position slots depend on simulation state */
static void a_nn_input(const orc_ms* p, int t, int k) {
  const double* gin = p->ginput + IIN(p, t, k, 0);
  double* gc = p->gcenter + IC3(p, t, k);
  for (int j = 0; j < p->N; ++j)
    for (int d = 0; d < 3; ++d) {
      double g = gin[j * 6 + p->n_sin + d] / 0.2;
      p->gx[IX3(p, t, k, j) + d] += g;
      gc[d] -= g;
    }
}

/* adjoint of compute_height(t) (running max of the lowest point) and of the
 * upper height (highest point) */
static void a_height(const orc_ms* p, int t, int k) {
  double gh = p->gheight[IB(p, t, k)];
  if (gh != 0.0) {
    /* h = min over the unrolled loop starting from 10.0: adjoint lands on the
     * last vertex that attains the minimum */
    int arg = -1;
    double h = 10.0;
    for (int i = 0; i < p->N; ++i) {
      double y = p->x[IX3(p, t, k, i) + 1];
      if (!(h < y)) arg = i;
      h = fmin(h, y);
    }
    double gmin = 0.0;
    if (t % p->jump_period == 0) gmin = gh;
    else {
      double prev = p->height[IB(p, t - 1, k)];
      if (h < prev) p->gheight[IB(p, t - 1, k)] += gh;  /* max(prev, h): first operand strictly larger */
      else gmin = gh;
    }
    if (arg >= 0) p->gx[IX3(p, t, k, arg) + 1] += gmin;
  }
  double gu = p->gupper[IB(p, t, k)];
  if (gu != 0.0) {
    int arg = -1;
    double u = -10.0;
    for (int i = 0; i < p->N; ++i) {
      double y = p->x[IX3(p, t, k, i) + 1];
      if (!(y < u)) arg = i;
      u = fmax(u, y);
    }
    if (arg >= 0) p->gx[IX3(p, t, k, arg) + 1] += gu;
  }
}

/* adjoint of compute_center(t) */
static void a_center(const orc_ms* p, int t, int k) {
  const double* gc = p->gcenter + IC3(p, t, k);
  for (int i = 0; i < p->N; ++i)
    for (int d = 0; d < 3; ++d) p->gx[IX3(p, t, k, i) + d] += gc[d] / p->N;
}

/* Reverse pass of the training rollout with loss.grad = 1.  All grad arrays must
 * be zero on entry (Tape clears them).  Weight grads are summed over envs in a
 * fixed order, so the result is deterministic. */
int orc_ms_backward(const orc_ms* p, int steps) {
  if (steps < 2 || steps > p->T) return -1;
  set_threads(p);
  int L = p->n_layers, maxw = 0;
  for (int l = 0; l <= L; ++l) if (p->width[l] > maxw) maxw = p->width[l];
  /* per-env weight-grad buffers, reduced in env order afterwards */
  size_t wsz = 0, bsz = 0;
  for (int l = 0; l < L; ++l) {
    wsz += (size_t)p->width[l + 1] * p->width[l];
    bsz += (size_t)p->width[l + 1];
  }
  double* gw_env = (double*)calloc((size_t)p->B * (wsz + bsz), sizeof(double));
  if (!gw_env) return -2;
#pragma omp parallel
  {
    double* ga_cur = (double*)malloc(sizeof(double) * maxw);
    double* ga_prev = (double*)malloc(sizeof(double) * maxw);
    double* abuf = (double*)malloc(sizeof(double) * maxw);
#pragma omp for schedule(dynamic, 1)
    for (int k = 0; k < p->B; ++k) {
      double* base = gw_env + (size_t)k * (wsz + bsz);
      double* gWt[ORC_MAX_LAYERS];
      double* gbt[ORC_MAX_LAYERS];
      size_t off = 0;
      for (int l = 0; l < L; ++l) { gWt[l] = base + off; off += (size_t)p->width[l + 1] * p->width[l]; }
      for (int l = 0; l < L; ++l) { gbt[l] = base + off; off += (size_t)p->width[l + 1]; }
      a_loss(p, steps, k);
      for (int t = steps - 2; t >= 0; --t) {
        a_advance(p, t + 1, k);
        a_spring(p, t, k);
        a_mlp(p, t, k, gWt, gbt, ga_cur, ga_prev, abuf);
        a_nn_input(p, t, k);
        a_height(p, t, k);
        a_center(p, t, k);
#ifdef ORC_STUDY
        if (st_round & ST_ADJ)
          for (int i = 0; i < 3 * p->N; ++i) {
            size_t o = IX3(p, t, k, 0) + i;
            p->gx[o] = ST_ROUND(ST_ADJ, p->gx[o]);
            p->gv[o] = ST_ROUND(ST_ADJ, p->gv[o]);
            p->gv_inc[o] = ST_ROUND(ST_ADJ, p->gv_inc[o]);
          }
        if (st_round & ST_WSUM)
          for (int l = 0; l < L; ++l) {
            size_t n = (size_t)p->width[l + 1] * p->width[l];
            for (size_t e = 0; e < n; ++e) gWt[l][e] = ST_ROUND(ST_WSUM, gWt[l][e]);
            for (int e = 0; e < p->width[l + 1]; ++e) gbt[l][e] = ST_ROUND(ST_WSUM, gbt[l][e]);
          }
#endif
      }
    }
    free(ga_cur);
    free(ga_prev);
    free(abuf);
  }
  for (int k = 0; k < p->B; ++k) {
    double* base = gw_env + (size_t)k * (wsz + bsz);
    size_t off = 0;
    for (int l = 0; l < L; ++l) {
      size_t n = (size_t)p->width[l + 1] * p->width[l];
      for (size_t e = 0; e < n; ++e) p->gW[l][e] += base[off + e];
      off += n;
    }
    for (int l = 0; l < L; ++l) {
      size_t n = (size_t)p->width[l + 1];
      for (size_t e = 0; e < n; ++e) p->gb[l][e] += base[off + e];
      off += n;
    }
  }
  free(gw_env);
  return 0;
}

/* ============================================================== optimiser */

/* Model.adam_update: multitask/nn.py:184-191 */
void orc_adam(double* w, const double* g, double* m, double* v, long n, double lr,
              double b1, double b2, int iter) {
  for (long i = 0; i < n; ++i) {
    m[i] = b1 * m[i] + (1 - b1) * g[i];
    v[i] = b2 * v[i] + (1 - b2) * g[i] * g[i];
    double mc = m[i] / (1 - pow(b1, iter + 1));
    double vc = v[i] / (1 - pow(b2, iter + 1));
    w[i] -= (lr * mc) / (sqrt(vc) + 1e-8);
  }
}

/* Model.compute_TNS: multitask/nn.py:179-182 */
double orc_tns(const double* g, long n) {
  double s = 0.0;
  for (long i = 0; i < n; ++i) s += g[i] * g[i];
  return s;
}

/* Model.weights_init with a caller-supplied uniform stream in [0,1):
 * multitask/nn.py:59-67 (the reference draws from ti.random) */
void orc_weights_init(double* w, long rows, long cols, const double* u01) {
  double q = sqrt(6.0 / cols);
  for (long i = 0; i < rows * cols; ++i) w[i] = (u01[i] * 2 - 1) * q;
}

int orc_abi_version(void) { return 1; }
