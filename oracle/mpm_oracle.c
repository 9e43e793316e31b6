/*
 * mpm_oracle.c -- FP64 CPU oracle for the differentiable MLS-MPM substep.
 *
 * TEST INFRASTRUCTURE ONLY: the checker the CUDA MPM path is compared
 * against; never linked into or shipped with the product library.
 *
 * Restates multitask/solver_mpm.py of the reference
 * (erizmr/Complex-locomotion-skill-learning-via-differentiable-physics):
 *   p2g      :83-124  (quadratic B-spline weights, F' = (I + dt C) F, stress,
 *                      APIC affine momentum, scatter to the 3^D neighbours)
 *   grid_op  :126-144 (momentum -> velocity, gravity, sticky walls: every
 *                      component zeroed within `bound` cells of any wall)
 *   g2p      :146-165 (gather v and C, x' = x + dt v')
 *   advance_core / advance_core_grad :175-190 (the reverse pass recomputes the
 *                      grid of each step from the particle state, then runs the
 *                      adjoints of g2p, grid_op and p2g)
 * The reference is 2D with the fixed-corotated model and actuation along the
 * material y axis.  Generalisations, defaulting to the reference: dim 2 or 3;
 * fibre direction per particle (actuation stress a * (F f)(F f)^T, the
 * reference's being f = e_y); compressible neo-Hookean Kirchhoff stress
 * mu (F F^T - I) + lambda ln(J) I (the textbook form) in addition to
 * fixed-corotated (2D only; its polar decomposition is the closed form
 * R = [[c, -s], [s, c]], c, s from (F00 + F11, F10 - F01)).  Solid particles
 * only (the reference fills particle_type with 1).
 *
 * The training loss here is a centre-tracking loss (the reference's MPM path
 * never reaches a loss):  L = sum_t w_t sum_k sum_d (c_tkd - target_tkd)^2,
 * c = sum_p pw_p x_p / sum_p pw_p (pw = 1: the mean particle position).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { MPM_FIXED_COROTATED = 0, MPM_NEO_HOOKEAN = 1 };

typedef struct {
  int dim, n_grid, B, P, T, M, material, bound;
  double dx, inv_dx, dt, p_vol, mu, la, act_strength, gravity, mass;
  const int* muscle;        /* [P] actuator index or -1 */
  const double* fibre;      /* [P][dim] */
  /* trajectory [T+1][B][P][...] */
  double *x, *v, *C, *F;    /* x, v: dim; C, F: dim*dim */
  const double* act;        /* [T][B][M] */
  const double* loss_w;     /* [T+1] */
  const double* loss_pw;    /* [P] particle weights of the tracked centre */
  const double* target;     /* [T+1][B][dim] */
  /* adjoints */
  double *gx0, *gv0, *gC0, *gF0; /* [B][P][...] of the initial state */
  double* gact;             /* [T][B][M] */
  double* loss;             /* [1] */
} orc_mpm;

#define D_ (p->dim)
#define IP(p, t, k, i) ((((size_t)(t) * (p)->B + (k)) * (p)->P + (i)))

static int ipow3(int d) { return d == 2 ? 9 : 27; }

static size_t grid_cells(const orc_mpm* p) {
  size_t n = (size_t)p->n_grid;
  return p->dim == 2 ? n * n : n * n * n;
}

static void weights(const orc_mpm* p, const double* xp, int base[3], double fx[3], double w[3][3],
                    double dw[3][3]) {
  for (int d = 0; d < p->dim; ++d) {
    base[d] = (int)(xp[d] * p->inv_dx - 0.5);
    fx[d] = xp[d] * p->inv_dx - (double)base[d];
    w[0][d] = 0.5 * (1.5 - fx[d]) * (1.5 - fx[d]);
    w[1][d] = 0.75 - (fx[d] - 1.0) * (fx[d] - 1.0);
    w[2][d] = 0.5 * (fx[d] - 0.5) * (fx[d] - 0.5);
    dw[0][d] = -(1.5 - fx[d]);
    dw[1][d] = -2.0 * (fx[d] - 1.0);
    dw[2][d] = fx[d] - 0.5;
  }
}

static void offs(int dim, int q, int o[3]) {
  o[0] = q % 3;
  o[1] = (q / 3) % 3;
  o[2] = dim == 3 ? q / 9 : 0;
}

static size_t cell(const orc_mpm* p, const int base[3], const int o[3]) {
  size_t n = (size_t)p->n_grid;
  size_t idx = 0;
  for (int d = 0; d < p->dim; ++d) idx = idx * n + (size_t)(base[d] + o[d]);
  return idx;
}

static double det(int dim, const double* A) {
  if (dim == 2) return A[0] * A[3] - A[1] * A[2];
  return A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
         A[2] * (A[3] * A[7] - A[4] * A[6]);
}

/* cofactor matrix: d det / d A */
static void cof(int dim, const double* A, double* c) {
  if (dim == 2) {
    c[0] = A[3]; c[1] = -A[2]; c[2] = -A[1]; c[3] = A[0];
    return;
  }
  c[0] = A[4] * A[8] - A[5] * A[7];
  c[1] = A[5] * A[6] - A[3] * A[8];
  c[2] = A[3] * A[7] - A[4] * A[6];
  c[3] = A[2] * A[7] - A[1] * A[8];
  c[4] = A[0] * A[8] - A[2] * A[6];
  c[5] = A[1] * A[6] - A[0] * A[7];
  c[6] = A[1] * A[5] - A[2] * A[4];
  c[7] = A[2] * A[3] - A[0] * A[5];
  c[8] = A[0] * A[4] - A[1] * A[3];
}

/* Kirchhoff-type stress tau(F) incl. actuation (p2g, solver_mpm.py:89-115) */
static void stress(const orc_mpm* p, const double* nF, int k, int pi, int t, double* tau) {
  const int D = p->dim;
  double J = det(D, nF);
  memset(tau, 0, sizeof(double) * 9);
  if (p->material == MPM_FIXED_COROTATED) {
    double xx = nF[0] + nF[3], yy = nF[2] - nF[1];
    double sc = 1.0 / sqrt(xx * xx + yy * yy);
    double c = xx * sc, s = yy * sc;
    double R[4] = {c, -s, s, c};
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) {
        double acc = 0;
        for (int q = 0; q < 2; ++q) acc += (nF[i * 2 + q] - R[i * 2 + q]) * nF[j * 2 + q];
        tau[i * 2 + j] = 2 * p->mu * acc;
      }
    for (int i = 0; i < 2; ++i) tau[i * 2 + i] += p->la * (J - 1) * J;
  } else {
    for (int i = 0; i < D; ++i)
      for (int j = 0; j < D; ++j) {
        double acc = 0;
        for (int q = 0; q < D; ++q) acc += nF[i * D + q] * nF[j * D + q];
        tau[i * D + j] = p->mu * (acc - (i == j ? 1.0 : 0.0));
      }
    for (int i = 0; i < D; ++i) tau[i * D + i] += p->la * log(J);
  }
  int m = p->muscle[pi];
  if (m >= 0) {
    double a = p->act[((size_t)t * p->B + k) * p->M + m] * p->act_strength;
    double u[3] = {0, 0, 0};
    for (int i = 0; i < D; ++i)
      for (int q = 0; q < D; ++q) u[i] += nF[i * D + q] * p->fibre[(size_t)pi * D + q];
    for (int i = 0; i < D; ++i)
      for (int j = 0; j < D; ++j) tau[i * D + j] += a * u[i] * u[j];
  }
}

/* P2G + grid_op for env k at step t into grid (mass, momentum -> velocity) */
static void build_grid(const orc_mpm* p, int t, int k, double* gm, double* gv, double* gvo) {
  const int D = p->dim, nn = ipow3(D);
  size_t cells = grid_cells(p);
  memset(gm, 0, sizeof(double) * cells);
  memset(gv, 0, sizeof(double) * cells * D);
  const double ks = p->dt * p->p_vol * 4 * p->inv_dx * p->inv_dx;
  for (int pi = 0; pi < p->P; ++pi) {
    const double* xp = p->x + IP(p, t, k, pi) * D;
    const double* vp = p->v + IP(p, t, k, pi) * D;
    const double* Cp = p->C + IP(p, t, k, pi) * D * D;
    const double* Fp = p->F + IP(p, t, k, pi) * D * D;
    int base[3]; double fx[3], w[3][3], dw[3][3];
    weights(p, xp, base, fx, w, dw);
    double nF[9], tau[9], aff[9];
    for (int i = 0; i < D; ++i)
      for (int j = 0; j < D; ++j) {
        double acc = 0;
        for (int q = 0; q < D; ++q) acc += ((i == q ? 1.0 : 0.0) + p->dt * Cp[i * D + q]) * Fp[q * D + j];
        nF[i * D + j] = acc;
      }
    stress(p, nF, k, pi, t, tau);
    for (int e = 0; e < D * D; ++e) aff[e] = -ks * tau[e] + p->mass * Cp[e];
    for (int q = 0; q < nn; ++q) {
      int o[3]; offs(D, q, o);
      double wt = 1, dpos[3];
      for (int d = 0; d < D; ++d) { wt *= w[o[d]][d]; dpos[d] = ((double)o[d] - fx[d]) * p->dx; }
      size_t c = cell(p, base, o);
      for (int i = 0; i < D; ++i) {
        double mom = p->mass * vp[i];
        for (int j = 0; j < D; ++j) mom += aff[i * D + j] * dpos[j];
        gv[c * D + i] += wt * mom;
      }
      gm[c] += wt * p->mass;
    }
  }
  /* grid_op */
  for (size_t c = 0; c < cells; ++c) {
    int I[3];
    size_t r = c;
    for (int d = D - 1; d >= 0; --d) { I[d] = (int)(r % p->n_grid); r /= p->n_grid; }
    double inv_m = 1.0 / (gm[c] + 1e-10);
    int wall = 0;
    for (int d = 0; d < D; ++d)
      if (I[d] < p->bound || I[d] > p->n_grid - p->bound) wall = 1;
    for (int i = 0; i < D; ++i) {
      double vo = inv_m * gv[c * D + i];
      if (i == 1) vo += p->dt * p->gravity;
      gvo[c * D + i] = wall ? 0.0 : vo;
    }
  }
}

static void g2p(const orc_mpm* p, int t, int k, const double* gvo) {
  const int D = p->dim, nn = ipow3(D);
  for (int pi = 0; pi < p->P; ++pi) {
    const double* xp = p->x + IP(p, t, k, pi) * D;
    const double* Cp = p->C + IP(p, t, k, pi) * D * D;
    const double* Fp = p->F + IP(p, t, k, pi) * D * D;
    int base[3]; double fx[3], w[3][3], dw[3][3];
    weights(p, xp, base, fx, w, dw);
    double nv[3] = {0, 0, 0}, nC[9] = {0};
    for (int q = 0; q < nn; ++q) {
      int o[3]; offs(D, q, o);
      double wt = 1, dpos[3];
      for (int d = 0; d < D; ++d) { wt *= w[o[d]][d]; dpos[d] = (double)o[d] - fx[d]; }
      size_t c = cell(p, base, o);
      for (int i = 0; i < D; ++i) {
        nv[i] += wt * gvo[c * D + i];
        for (int j = 0; j < D; ++j) nC[i * D + j] += 4 * wt * gvo[c * D + i] * dpos[j] * p->inv_dx;
      }
    }
    double* x1 = p->x + IP(p, t + 1, k, pi) * D;
    double* v1 = p->v + IP(p, t + 1, k, pi) * D;
    double* C1 = p->C + IP(p, t + 1, k, pi) * D * D;
    double* F1 = p->F + IP(p, t + 1, k, pi) * D * D;
    for (int i = 0; i < D; ++i) { v1[i] = nv[i]; x1[i] = xp[i] + p->dt * nv[i]; }
    for (int e = 0; e < D * D; ++e) C1[e] = nC[e];
    for (int i = 0; i < D; ++i)
      for (int j = 0; j < D; ++j) {
        double acc = 0;
        for (int q = 0; q < D; ++q) acc += ((i == q ? 1.0 : 0.0) + p->dt * Cp[i * D + q]) * Fp[q * D + j];
        F1[i * D + j] = acc;
      }
  }
}

int orc_mpm_forward(const orc_mpm* p, int steps) {
  if (steps < 0 || steps > p->T) return -1;
  size_t cells = grid_cells(p);
#pragma omp parallel for schedule(dynamic, 1)
  for (int k = 0; k < p->B; ++k) {
    double* gm = (double*)malloc(sizeof(double) * cells);
    double* gv = (double*)malloc(sizeof(double) * cells * p->dim);
    double* gvo = (double*)malloc(sizeof(double) * cells * p->dim);
    for (int t = 0; t < steps; ++t) {
      build_grid(p, t, k, gm, gv, gvo);
      g2p(p, t, k, gvo);
    }
    free(gm); free(gv); free(gvo);
  }
  return 0;
}

static double pw_sum(const orc_mpm* p) {
  double s = 0;
  for (int pi = 0; pi < p->P; ++pi) s += p->loss_pw[pi];
  return s;
}

static void center_of(const orc_mpm* p, int t, int k, double c[3]) {
  c[0] = c[1] = c[2] = 0;
  const double sw = pw_sum(p);
  for (int pi = 0; pi < p->P; ++pi)
    for (int d = 0; d < p->dim; ++d) c[d] += p->loss_pw[pi] * p->x[IP(p, t, k, pi) * p->dim + d];
  for (int d = 0; d < p->dim; ++d) c[d] /= sw;
}

double orc_mpm_loss(const orc_mpm* p, int steps) {
  double L = 0;
  for (int t = 0; t <= steps; ++t) {
    if (p->loss_w[t] == 0.0) continue;
    for (int k = 0; k < p->B; ++k) {
      double c[3];
      center_of(p, t, k, c);
      for (int d = 0; d < p->dim; ++d) {
        double e = c[d] - p->target[((size_t)t * p->B + k) * p->dim + d];
        L += p->loss_w[t] * e * e;
      }
    }
  }
  if (p->loss) p->loss[0] = L;
  return L;
}

/* adjoint of stress(): g_tau -> g_nF (accumulated), g_act */
static void stress_adj(const orc_mpm* p, const double* nF, int k, int pi, int t, const double* gt,
                       double* gF, double* gact) {
  const int D = p->dim;
  double J = det(D, nF), cf[9];
  cof(D, nF, cf);
  double tr = 0;
  for (int i = 0; i < D; ++i) tr += gt[i * D + i];
  if (p->material == MPM_FIXED_COROTATED) {
    double xx = nF[0] + nF[3], yy = nF[2] - nF[1];
    double r2 = xx * xx + yy * yy, r = sqrt(r2), r3 = r2 * r;
    double sc = 1.0 / r, c = xx * sc, s = yy * sc;
    double R[4] = {c, -s, s, c};
    /* tau = 2 mu (F F^T - R F^T) + la (J^2 - J) I */
    for (int i = 0; i < 2; ++i)
      for (int q = 0; q < 2; ++q) {
        double acc = 0, acc2 = 0;
        for (int j = 0; j < 2; ++j) {
          acc += (gt[i * 2 + j] + gt[j * 2 + i]) * nF[j * 2 + q];
          acc2 += gt[j * 2 + i] * R[j * 2 + q];
        }
        gF[i * 2 + q] += 2 * p->mu * acc - 2 * p->mu * acc2;
      }
    double gR[4];
    for (int i = 0; i < 2; ++i)
      for (int q = 0; q < 2; ++q) {
        double acc = 0;
        for (int j = 0; j < 2; ++j) acc += gt[i * 2 + j] * nF[j * 2 + q];
        gR[i * 2 + q] = -2 * p->mu * acc;
      }
    double gc = gR[0] + gR[3], gs = -gR[1] + gR[2];
    double gxx = gc * yy * yy / r3 - gs * xx * yy / r3;
    double gyy = -gc * xx * yy / r3 + gs * xx * xx / r3;
    gF[0] += gxx; gF[3] += gxx; gF[2] += gyy; gF[1] -= gyy;
    double gJ = p->la * (2 * J - 1) * tr;
    for (int e = 0; e < 4; ++e) gF[e] += gJ * cf[e];
  } else {
    for (int i = 0; i < D; ++i)
      for (int q = 0; q < D; ++q) {
        double acc = 0;
        for (int j = 0; j < D; ++j) acc += (gt[i * D + j] + gt[j * D + i]) * nF[j * D + q];
        gF[i * D + q] += p->mu * acc;
      }
    double gJ = p->la * tr / J;
    for (int e = 0; e < D * D; ++e) gF[e] += gJ * cf[e];
  }
  int m = p->muscle[pi];
  if (m >= 0) {
    double a = p->act[((size_t)t * p->B + k) * p->M + m] * p->act_strength;
    const double* f = p->fibre + (size_t)pi * D;
    double u[3] = {0, 0, 0};
    for (int i = 0; i < D; ++i)
      for (int q = 0; q < D; ++q) u[i] += nF[i * D + q] * f[q];
    double ga = 0, gu[3] = {0, 0, 0};
    for (int i = 0; i < D; ++i)
      for (int j = 0; j < D; ++j) {
        ga += gt[i * D + j] * u[i] * u[j];
        gu[i] += a * (gt[i * D + j] + gt[j * D + i]) * u[j];
      }
    for (int i = 0; i < D; ++i)
      for (int q = 0; q < D; ++q) gF[i * D + q] += gu[i] * f[q];
    gact[((size_t)t * p->B + k) * p->M + m] += ga * p->act_strength;
  }
}

/* Reverse pass.  gact must be zero on entry; initial-state grads are written. */
int orc_mpm_backward(const orc_mpm* p, int steps) {
  const int D = p->dim, nn = ipow3(D);
  size_t cells = grid_cells(p);
  const double ks = p->dt * p->p_vol * 4 * p->inv_dx * p->inv_dx;
#pragma omp parallel for schedule(dynamic, 1)
  for (int k = 0; k < p->B; ++k) {
    double* gm = (double*)malloc(sizeof(double) * cells);
    double* gv = (double*)malloc(sizeof(double) * cells * D);
    double* gvo = (double*)malloc(sizeof(double) * cells * D);
    double* g_gvo = (double*)malloc(sizeof(double) * cells * D);
    double* g_gv = (double*)malloc(sizeof(double) * cells * D);
    double* g_gm = (double*)malloc(sizeof(double) * cells);
    size_t psz = (size_t)p->P;
    double* ax = (double*)calloc(psz * D, sizeof(double));
    double* av = (double*)calloc(psz * D, sizeof(double));
    double* aC = (double*)calloc(psz * D * D, sizeof(double));
    double* aF = (double*)calloc(psz * D * D, sizeof(double));
    /* loss seeds at t = steps */
    for (int t = steps; t >= 0; --t) {
      if (p->loss_w[t] != 0.0) {
        double c[3];
        center_of(p, t, k, c);
        const double sw = pw_sum(p);
        for (int pi = 0; pi < p->P; ++pi)
          for (int d = 0; d < D; ++d)
            ax[pi * D + d] += 2 * p->loss_w[t] * (c[d] - p->target[((size_t)t * p->B + k) * D + d]) *
                              p->loss_pw[pi] / sw;
      }
      if (t == 0) break;
      const int f = t - 1;   /* step f -> f + 1 = t */
      build_grid(p, f, k, gm, gv, gvo);
      memset(g_gvo, 0, sizeof(double) * cells * D);
      /* g2p adjoint */
      double* nx = (double*)calloc(psz * D, sizeof(double));
      double* nv = (double*)calloc(psz * D, sizeof(double));
      double* nC = (double*)calloc(psz * D * D, sizeof(double));
      double* nF = (double*)calloc(psz * D * D, sizeof(double));
      for (int pi = 0; pi < p->P; ++pi) {
        const double* xp = p->x + IP(p, f, k, pi) * D;
        int base[3]; double fx[3], w[3][3], dw[3][3];
        weights(p, xp, base, fx, w, dw);
        double gvt[3];
        for (int i = 0; i < D; ++i) { nx[pi * D + i] += ax[pi * D + i]; gvt[i] = av[pi * D + i] + p->dt * ax[pi * D + i]; }
        const double* gC1 = aC + (size_t)pi * D * D;
        double gfx[3] = {0, 0, 0};
        for (int q = 0; q < nn; ++q) {
          int o[3]; offs(D, q, o);
          double wt = 1, dpos[3], dwt[3];
          for (int d = 0; d < D; ++d) { wt *= w[o[d]][d]; dpos[d] = (double)o[d] - fx[d]; }
          for (int d = 0; d < D; ++d) {
            dwt[d] = dw[o[d]][d];
            for (int e = 0; e < D; ++e) if (e != d) dwt[d] *= w[o[e]][e];
          }
          size_t c = cell(p, base, o);
          const double* g = gvo + c * D;
          double gw = 0;
          for (int i = 0; i < D; ++i) {
            double gGC = 0;
            for (int j = 0; j < D; ++j) gGC += gC1[i * D + j] * dpos[j];
            g_gvo[c * D + i] += wt * gvt[i] + 4 * p->inv_dx * wt * gGC;
            gw += gvt[i] * g[i] + 4 * p->inv_dx * g[i] * gGC;
          }
          for (int j = 0; j < D; ++j) {
            double acc = 0;
            for (int i = 0; i < D; ++i) acc += gC1[i * D + j] * g[i];
            gfx[j] -= 4 * p->inv_dx * wt * acc;
          }
          for (int d = 0; d < D; ++d) gfx[d] += gw * dwt[d];
        }
        for (int d = 0; d < D; ++d) nx[pi * D + d] += gfx[d] * p->inv_dx;
        /* F' = (I + dt C) F: adjoint carried into the p2g adjoint below */
      }
      /* grid_op adjoint */
      memset(g_gv, 0, sizeof(double) * cells * D);
      memset(g_gm, 0, sizeof(double) * cells);
      for (size_t c = 0; c < cells; ++c) {
        int I[3];
        size_t r = c;
        for (int d = D - 1; d >= 0; --d) { I[d] = (int)(r % p->n_grid); r /= p->n_grid; }
        int wall = 0;
        for (int d = 0; d < D; ++d)
          if (I[d] < p->bound || I[d] > p->n_grid - p->bound) wall = 1;
        if (wall) continue;
        double inv_m = 1.0 / (gm[c] + 1e-10);
        for (int i = 0; i < D; ++i) {
          g_gv[c * D + i] = g_gvo[c * D + i] * inv_m;
          g_gm[c] -= g_gvo[c * D + i] * gv[c * D + i] * inv_m * inv_m;
        }
      }
      /* p2g adjoint (and the F' adjoint) */
      for (int pi = 0; pi < p->P; ++pi) {
        const double* xp = p->x + IP(p, f, k, pi) * D;
        const double* vp = p->v + IP(p, f, k, pi) * D;
        const double* Cp = p->C + IP(p, f, k, pi) * D * D;
        const double* Fp = p->F + IP(p, f, k, pi) * D * D;
        int base[3]; double fx[3], w[3][3], dw[3][3];
        weights(p, xp, base, fx, w, dw);
        double nFm[9], tau[9], aff[9];
        for (int i = 0; i < D; ++i)
          for (int j = 0; j < D; ++j) {
            double acc = 0;
            for (int q = 0; q < D; ++q) acc += ((i == q ? 1.0 : 0.0) + p->dt * Cp[i * D + q]) * Fp[q * D + j];
            nFm[i * D + j] = acc;
          }
        stress(p, nFm, k, pi, f, tau);
        for (int e = 0; e < D * D; ++e) aff[e] = -ks * tau[e] + p->mass * Cp[e];
        double gaff[9] = {0}, gfx[3] = {0, 0, 0};
        for (int q = 0; q < nn; ++q) {
          int o[3]; offs(D, q, o);
          double wt = 1, dpos[3], dwt[3];
          for (int d = 0; d < D; ++d) { wt *= w[o[d]][d]; dpos[d] = ((double)o[d] - fx[d]) * p->dx; }
          for (int d = 0; d < D; ++d) {
            dwt[d] = dw[o[d]][d];
            for (int e = 0; e < D; ++e) if (e != d) dwt[d] *= w[o[e]][e];
          }
          size_t c = cell(p, base, o);
          const double* gg = g_gv + c * D;
          double gw = g_gm[c] * p->mass;
          for (int i = 0; i < D; ++i) {
            double mom = p->mass * vp[i];
            for (int j = 0; j < D; ++j) mom += aff[i * D + j] * dpos[j];
            gw += gg[i] * mom;
            nv[pi * D + i] += wt * p->mass * gg[i];
            for (int j = 0; j < D; ++j) gaff[i * D + j] += wt * gg[i] * dpos[j];
          }
          for (int j = 0; j < D; ++j) {
            double acc = 0;
            for (int i = 0; i < D; ++i) acc += aff[i * D + j] * gg[i];
            gfx[j] -= wt * acc * p->dx;
          }
          for (int d = 0; d < D; ++d) gfx[d] += gw * dwt[d];
        }
        for (int d = 0; d < D; ++d) nx[pi * D + d] += gfx[d] * p->inv_dx;
        double gtau[9], gnF[9];
        for (int e = 0; e < D * D; ++e) {
          nC[(size_t)pi * D * D + e] += p->mass * gaff[e];
          gtau[e] = -ks * gaff[e];
          gnF[e] = aF[(size_t)pi * D * D + e];   /* F_{f+1} = new_F */
        }
        stress_adj(p, nFm, k, pi, f, gtau, gnF, p->gact);
        /* new_F = (I + dt C) F */
        for (int i = 0; i < D; ++i)
          for (int q = 0; q < D; ++q) {
            double accC = 0, accF = 0;
            for (int j = 0; j < D; ++j) {
              accC += gnF[i * D + j] * Fp[q * D + j];
              accF += ((j == i ? 1.0 : 0.0) + p->dt * Cp[j * D + i]) * gnF[j * D + q];
            }
            nC[(size_t)pi * D * D + i * D + q] += p->dt * accC;
            nF[(size_t)pi * D * D + i * D + q] += accF;
          }
      }
      memcpy(ax, nx, sizeof(double) * psz * D);
      memcpy(av, nv, sizeof(double) * psz * D);
      memcpy(aC, nC, sizeof(double) * psz * D * D);
      memcpy(aF, nF, sizeof(double) * psz * D * D);
      free(nx); free(nv); free(nC); free(nF);
    }
    memcpy(p->gx0 + (size_t)k * psz * D, ax, sizeof(double) * psz * D);
    memcpy(p->gv0 + (size_t)k * psz * D, av, sizeof(double) * psz * D);
    memcpy(p->gC0 + (size_t)k * psz * D * D, aC, sizeof(double) * psz * D * D);
    memcpy(p->gF0 + (size_t)k * psz * D * D, aF, sizeof(double) * psz * D * D);
    free(ax); free(av); free(aC); free(aF);
    free(gm); free(gv); free(gvo); free(g_gvo); free(g_gv); free(g_gm);
  }
  return 0;
}
