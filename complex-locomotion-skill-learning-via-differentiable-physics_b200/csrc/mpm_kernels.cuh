// mpm_kernels.cuh -- differentiable MLS-MPM substep (P2G, grid update, G2P)
// and its hand-written adjoint, dimension-templated (2D / 3D).
//
// Follows the reference's multitask/solver_mpm.py (2D): p2g :83-124, grid_op
// :126-144, g2p :146-165, advance_core_grad :182-190 (the adjoint of a step
// rebuilds that step's grid from the particle state, then runs g2p^T,
// grid_op^T, p2g^T).  Generalised to 3D, per-particle fibre directions
// (actuation stress a * (F f)(F f)^T; the reference's is f = e_y) and the
// compressible neo-Hookean Kirchhoff stress mu (F F^T - I) + lambda ln(J) I
// next to the reference's fixed-corotated model (2D only, closed-form polar
// decomposition).
#pragma once
#include "cls_common.cuh"

namespace cls {
namespace mpm {

enum Material : int { FIXED_COROTATED = 0, NEO_HOOKEAN = 1 };

template <typename R>
struct Args {
  int n_envs, P, M, n_grid, bound, material;
  long long cells;                       // n_grid^D per env
  R dx, inv_dx, dt, ks, mu, la, act_strength, gravity, mass;   // ks = dt p_vol 4 inv_dx^2
  const int* muscle;                     // [P]
  const R* fibre;                        // [P][D]
  // state at step f and f + 1, [E][P][D] and [E][P][D][D]
  const R* x; const R* v; const R* C; const R* F;
  R* x1; R* v1; R* C1; R* F1;
  const R* act;                          // [E][M] of step f
  R* gm; R* gmv; R* gvo;                 // grid [E][cells], [E][cells][D] x 2
  // adjoints of state f + 1 (a*) and of state f (n*)
  const R* ax; const R* av; const R* aC; const R* aF;
  R* nx; R* nv; R* nC; R* nF;
  R* g_gvo; R* g_gv; R* g_gm;            // grid adjoints
  R* gact;                               // [E][M] of step f
};

template <typename R, int D>
struct Kern {
  static constexpr int NN = D == 2 ? 9 : 27;

  // quadratic B-spline weights of the 3^D stencil.  The base cell is clamped
  // into [0, n_grid - 3] so that a particle that has left the domain can never
  // address memory outside its env's grid (the reference does not check);
  // for particles inside the domain the clamp has no effect.
  __device__ static void weights(const R* xp, R inv_dx, int n_grid, int base[D], R fx[D], R w[3][D],
                                 R dw[3][D]) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
      base[d] = (int)(xp[d] * inv_dx - R(0.5));
      base[d] = base[d] < 0 ? 0 : (base[d] > n_grid - 3 ? n_grid - 3 : base[d]);
      fx[d] = xp[d] * inv_dx - (R)base[d];
      w[0][d] = R(0.5) * (R(1.5) - fx[d]) * (R(1.5) - fx[d]);
      w[1][d] = R(0.75) - (fx[d] - R(1)) * (fx[d] - R(1));
      w[2][d] = R(0.5) * (fx[d] - R(0.5)) * (fx[d] - R(0.5));
      dw[0][d] = -(R(1.5) - fx[d]);
      dw[1][d] = R(-2) * (fx[d] - R(1));
      dw[2][d] = fx[d] - R(0.5);
    }
  }

  __device__ static void offs(int q, int o[D]) {
    o[0] = q % 3;
    o[1] = (q / 3) % 3;
    if (D == 3) o[D - 1] = q / 9;
  }

  __device__ static long long cell(int n, const int base[D], const int o[D]) {
    long long idx = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) idx = idx * n + (base[d] + o[d]);
    return idx;
  }

  __device__ static R det(const R* A) {
    if (D == 2) return A[0] * A[3] - A[1] * A[2];
    return A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) +
           A[2] * (A[3] * A[7] - A[4] * A[6]);
  }

  __device__ static void cof(const R* A, R* c) {
    if (D == 2) {
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

  // new_F = (I + dt C) F   (solver_mpm.py:89)
  __device__ static void new_F(const R* C, const R* F, R dt, R* nF) {
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) {
        R acc = 0;
#pragma unroll
        for (int q = 0; q < D; ++q) acc += ((i == q ? R(1) : R(0)) + dt * C[i * D + q]) * F[q * D + j];
        nF[i * D + j] = acc;
      }
  }

  // Kirchhoff stress incl. actuation (solver_mpm.py:96-115)
  __device__ static void stress(const Args<R>& a, const R* nF, int pidx, R act, R* tau) {
    const R J = det(nF);
    if (D == 2 && a.material == FIXED_COROTATED) {
      const R xx = nF[0] + nF[3], yy = nF[2] - nF[1];
      const R sc = R(1) / dsqrt<R>(xx * xx + yy * yy);
      const R c = xx * sc, s = yy * sc;
      const R Rm[4] = {c, -s, s, c};
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          R acc = 0;
#pragma unroll
          for (int q = 0; q < 2; ++q) acc += (nF[i * 2 + q] - Rm[i * 2 + q]) * nF[j * 2 + q];
          tau[i * D + j] = R(2) * a.mu * acc;
        }
#pragma unroll
      for (int i = 0; i < 2; ++i) tau[i * D + i] += a.la * (J - R(1)) * J;
    } else {
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) {
          R acc = 0;
#pragma unroll
          for (int q = 0; q < D; ++q) acc += nF[i * D + q] * nF[j * D + q];
          tau[i * D + j] = a.mu * (acc - (i == j ? R(1) : R(0)));
        }
#pragma unroll
      for (int i = 0; i < D; ++i) tau[i * D + i] += a.la * log(J);
    }
    if (a.muscle[pidx] >= 0) {
      const R am = act * a.act_strength;
      const R* f = a.fibre + (size_t)pidx * D;
      R u[D];
#pragma unroll
      for (int i = 0; i < D; ++i) {
        u[i] = 0;
#pragma unroll
        for (int q = 0; q < D; ++q) u[i] += nF[i * D + q] * f[q];
      }
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) tau[i * D + j] += am * u[i] * u[j];
    }
  }

  // d tau / d nF (accumulated into gF) and d actuation (returned)
  __device__ static R stress_adj(const Args<R>& a, const R* nF, int pidx, R act, const R* gt, R* gF) {
    const R J = det(nF);
    R cf[D * D];
    cof(nF, cf);
    R tr = 0;
#pragma unroll
    for (int i = 0; i < D; ++i) tr += gt[i * D + i];
    if (D == 2 && a.material == FIXED_COROTATED) {
      const R xx = nF[0] + nF[3], yy = nF[2] - nF[1];
      const R r2 = xx * xx + yy * yy, r = dsqrt<R>(r2), r3 = r2 * r;
      const R c = xx / r, s = yy / r;
      const R Rm[4] = {c, -s, s, c};
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          R acc = 0, acc2 = 0;
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            acc += (gt[i * 2 + j] + gt[j * 2 + i]) * nF[j * 2 + q];
            acc2 += gt[j * 2 + i] * Rm[j * 2 + q];
          }
          gF[i * 2 + q] += R(2) * a.mu * acc - R(2) * a.mu * acc2;
        }
      R gR[4];
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          R acc = 0;
#pragma unroll
          for (int j = 0; j < 2; ++j) acc += gt[i * 2 + j] * nF[j * 2 + q];
          gR[i * 2 + q] = R(-2) * a.mu * acc;
        }
      const R gc = gR[0] + gR[3], gs = -gR[1] + gR[2];
      const R gxx = gc * yy * yy / r3 - gs * xx * yy / r3;
      const R gyy = -gc * xx * yy / r3 + gs * xx * xx / r3;
      gF[0] += gxx; gF[3] += gxx; gF[2] += gyy; gF[1] -= gyy;
      const R gJ = a.la * (R(2) * J - R(1)) * tr;
#pragma unroll
      for (int e = 0; e < 4; ++e) gF[e] += gJ * cf[e];
    } else {
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int q = 0; q < D; ++q) {
          R acc = 0;
#pragma unroll
          for (int j = 0; j < D; ++j) acc += (gt[i * D + j] + gt[j * D + i]) * nF[j * D + q];
          gF[i * D + q] += a.mu * acc;
        }
      const R gJ = a.la * tr / J;
#pragma unroll
      for (int e = 0; e < D * D; ++e) gF[e] += gJ * cf[e];
    }
    R gact = 0;
    if (a.muscle[pidx] >= 0) {
      const R am = act * a.act_strength;
      const R* f = a.fibre + (size_t)pidx * D;
      R u[D];
#pragma unroll
      for (int i = 0; i < D; ++i) {
        u[i] = 0;
#pragma unroll
        for (int q = 0; q < D; ++q) u[i] += nF[i * D + q] * f[q];
      }
      R ga = 0, gu[D];
#pragma unroll
      for (int i = 0; i < D; ++i) gu[i] = 0;
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int j = 0; j < D; ++j) {
          ga += gt[i * D + j] * u[i] * u[j];
          gu[i] += am * (gt[i * D + j] + gt[j * D + i]) * u[j];
        }
#pragma unroll
      for (int i = 0; i < D; ++i)
#pragma unroll
        for (int q = 0; q < D; ++q) gF[i * D + q] += gu[i] * f[q];
      gact = ga * a.act_strength;
    }
    return gact;
  }
};

// ------------------------------------------------------------------ forward
// P2G (solver_mpm.py:83-124): scatter mass and APIC momentum with atomics;
// optionally store F_{f+1}.
template <typename R, int D>
__global__ void p2g_kernel(Args<R> a, int write_F) {
  using K = Kern<R, D>;
  const long long total = (long long)a.n_envs * a.P;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(q / a.P), p = (int)(q % a.P);
    const R* xp = a.x + q * D;
    const R* vp = a.v + q * D;
    const R* Cp = a.C + q * D * D;
    const R* Fp = a.F + q * D * D;
    int base[D]; R fx[D], w[3][D], dw[3][D];
    K::weights(xp, a.inv_dx, a.n_grid, base, fx, w, dw);
    R nF[D * D], tau[D * D], aff[D * D];
    K::new_F(Cp, Fp, a.dt, nF);
    const int m = a.muscle[p];
    const R act = m >= 0 ? a.act[(size_t)e * a.M + m] : R(0);
    K::stress(a, nF, p, act, tau);
#pragma unroll
    for (int i = 0; i < D * D; ++i) aff[i] = -a.ks * tau[i] + a.mass * Cp[i];
    if (write_F) {
#pragma unroll
      for (int i = 0; i < D * D; ++i) a.F1[q * D * D + i] = nF[i];
    }
    R* gm = a.gm + (size_t)e * a.cells;
    R* gmv = a.gmv + (size_t)e * a.cells * D;
#pragma unroll 1
    for (int nq = 0; nq < K::NN; ++nq) {
      int o[D];
      K::offs(nq, o);
      R wt = 1, dpos[D];
#pragma unroll
      for (int d = 0; d < D; ++d) { wt *= w[o[d]][d]; dpos[d] = ((R)o[d] - fx[d]) * a.dx; }
      const long long c = K::cell(a.n_grid, base, o);
#pragma unroll
      for (int i = 0; i < D; ++i) {
        R mom = a.mass * vp[i];
#pragma unroll
        for (int j = 0; j < D; ++j) mom += aff[i * D + j] * dpos[j];
        atomicAdd(gmv + c * D + i, wt * mom);
      }
      atomicAdd(gm + c, wt * a.mass);
    }
  }
}

// grid_op (solver_mpm.py:126-144): velocity, gravity on axis 1, sticky walls
template <typename R, int D>
__global__ void grid_op_kernel(Args<R> a) {
  const long long total = (long long)a.n_envs * a.cells;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    long long r = q % a.cells;
    bool wall = false;
#pragma unroll
    for (int d = D - 1; d >= 0; --d) {
      const int I = (int)(r % a.n_grid);
      r /= a.n_grid;
      wall |= (I < a.bound || I > a.n_grid - a.bound);
    }
    const R inv_m = R(1) / (a.gm[q] + R(1e-10));
#pragma unroll
    for (int i = 0; i < D; ++i) {
      R vo = inv_m * a.gmv[q * D + i];
      if (i == 1) vo += a.dt * a.gravity;
      a.gvo[q * D + i] = wall ? R(0) : vo;
    }
  }
}

// G2P (solver_mpm.py:146-165)
template <typename R, int D>
__global__ void g2p_kernel(Args<R> a) {
  using K = Kern<R, D>;
  const long long total = (long long)a.n_envs * a.P;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(q / a.P);
    const R* xp = a.x + q * D;
    int base[D]; R fx[D], w[3][D], dw[3][D];
    K::weights(xp, a.inv_dx, a.n_grid, base, fx, w, dw);
    R nv[D], nC[D * D];
#pragma unroll
    for (int i = 0; i < D; ++i) nv[i] = 0;
#pragma unroll
    for (int i = 0; i < D * D; ++i) nC[i] = 0;
    const R* gvo = a.gvo + (size_t)e * a.cells * D;
#pragma unroll 1
    for (int nq = 0; nq < K::NN; ++nq) {
      int o[D];
      K::offs(nq, o);
      R wt = 1, dpos[D];
#pragma unroll
      for (int d = 0; d < D; ++d) { wt *= w[o[d]][d]; dpos[d] = (R)o[d] - fx[d]; }
      const long long c = K::cell(a.n_grid, base, o);
#pragma unroll
      for (int i = 0; i < D; ++i) {
        const R g = gvo[c * D + i];
        nv[i] += wt * g;
#pragma unroll
        for (int j = 0; j < D; ++j) nC[i * D + j] += R(4) * wt * g * dpos[j] * a.inv_dx;
      }
    }
#pragma unroll
    for (int i = 0; i < D; ++i) {
      a.v1[q * D + i] = nv[i];
      a.x1[q * D + i] = xp[i] + a.dt * nv[i];
    }
#pragma unroll
    for (int i = 0; i < D * D; ++i) a.C1[q * D * D + i] = nC[i];
  }
}

// ------------------------------------------------------------------ adjoint
// G2P^T: scatter d grid velocity (atomics); write the x, v-independent parts
// of the state-f adjoint (n* are overwritten here, accumulated by P2G^T).
template <typename R, int D>
__global__ void g2p_adj_kernel(Args<R> a) {
  using K = Kern<R, D>;
  const long long total = (long long)a.n_envs * a.P;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(q / a.P);
    const R* xp = a.x + q * D;
    int base[D]; R fx[D], w[3][D], dw[3][D];
    K::weights(xp, a.inv_dx, a.n_grid, base, fx, w, dw);
    R gvt[D], gfx[D];
#pragma unroll
    for (int i = 0; i < D; ++i) {
      gvt[i] = a.av[q * D + i] + a.dt * a.ax[q * D + i];
      gfx[i] = 0;
    }
    const R* gC1 = a.aC + q * D * D;
    const R* gvo = a.gvo + (size_t)e * a.cells * D;
    R* ggvo = a.g_gvo + (size_t)e * a.cells * D;
#pragma unroll 1
    for (int nq = 0; nq < K::NN; ++nq) {
      int o[D];
      K::offs(nq, o);
      R wt = 1, dpos[D], dwt[D];
#pragma unroll
      for (int d = 0; d < D; ++d) { wt *= w[o[d]][d]; dpos[d] = (R)o[d] - fx[d]; }
#pragma unroll
      for (int d = 0; d < D; ++d) {
        dwt[d] = dw[o[d]][d];
#pragma unroll
        for (int f = 0; f < D; ++f)
          if (f != d) dwt[d] *= w[o[f]][f];
      }
      const long long c = K::cell(a.n_grid, base, o);
      R gw = 0;
#pragma unroll
      for (int i = 0; i < D; ++i) {
        R gGC = 0;
#pragma unroll
        for (int j = 0; j < D; ++j) gGC += gC1[i * D + j] * dpos[j];
        const R g = gvo[c * D + i];
        atomicAdd(ggvo + c * D + i, wt * gvt[i] + R(4) * a.inv_dx * wt * gGC);
        gw += gvt[i] * g + R(4) * a.inv_dx * g * gGC;
      }
#pragma unroll
      for (int j = 0; j < D; ++j) {
        R acc = 0;
#pragma unroll
        for (int i = 0; i < D; ++i) acc += gC1[i * D + j] * gvo[c * D + i];
        gfx[j] -= R(4) * a.inv_dx * wt * acc;
      }
#pragma unroll
      for (int d = 0; d < D; ++d) gfx[d] += gw * dwt[d];
    }
#pragma unroll
    for (int d = 0; d < D; ++d) a.nx[q * D + d] = a.ax[q * D + d] + gfx[d] * a.inv_dx;
  }
}

// grid_op^T
template <typename R, int D>
__global__ void grid_op_adj_kernel(Args<R> a) {
  const long long total = (long long)a.n_envs * a.cells;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    long long r = q % a.cells;
    bool wall = false;
#pragma unroll
    for (int d = D - 1; d >= 0; --d) {
      const int I = (int)(r % a.n_grid);
      r /= a.n_grid;
      wall |= (I < a.bound || I > a.n_grid - a.bound);
    }
    R gmass = 0;
    const R inv_m = R(1) / (a.gm[q] + R(1e-10));
#pragma unroll
    for (int i = 0; i < D; ++i) {
      const R g = wall ? R(0) : a.g_gvo[q * D + i];
      a.g_gv[q * D + i] = g * inv_m;
      gmass -= g * a.gmv[q * D + i] * inv_m * inv_m;
    }
    a.g_gm[q] = gmass;
  }
}

// P2G^T (and the adjoint of F_{f+1} = (I + dt C) F): gather grid adjoints,
// finish the state-f adjoint, accumulate d actuation.
template <typename R, int D>
__global__ void p2g_adj_kernel(Args<R> a) {
  using K = Kern<R, D>;
  const long long total = (long long)a.n_envs * a.P;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(q / a.P), p = (int)(q % a.P);
    const R* xp = a.x + q * D;
    const R* vp = a.v + q * D;
    const R* Cp = a.C + q * D * D;
    const R* Fp = a.F + q * D * D;
    int base[D]; R fx[D], w[3][D], dw[3][D];
    K::weights(xp, a.inv_dx, a.n_grid, base, fx, w, dw);
    R nFm[D * D], tau[D * D], aff[D * D];
    K::new_F(Cp, Fp, a.dt, nFm);
    const int m = a.muscle[p];
    const R act = m >= 0 ? a.act[(size_t)e * a.M + m] : R(0);
    K::stress(a, nFm, p, act, tau);
#pragma unroll
    for (int i = 0; i < D * D; ++i) aff[i] = -a.ks * tau[i] + a.mass * Cp[i];
    R gaff[D * D], gfx[D], gvp[D];
#pragma unroll
    for (int i = 0; i < D * D; ++i) gaff[i] = 0;
#pragma unroll
    for (int i = 0; i < D; ++i) { gfx[i] = 0; gvp[i] = 0; }
    const R* ggv = a.g_gv + (size_t)e * a.cells * D;
    const R* ggm = a.g_gm + (size_t)e * a.cells;
#pragma unroll 1
    for (int nq = 0; nq < K::NN; ++nq) {
      int o[D];
      K::offs(nq, o);
      R wt = 1, dpos[D], dwt[D];
#pragma unroll
      for (int d = 0; d < D; ++d) { wt *= w[o[d]][d]; dpos[d] = ((R)o[d] - fx[d]) * a.dx; }
#pragma unroll
      for (int d = 0; d < D; ++d) {
        dwt[d] = dw[o[d]][d];
#pragma unroll
        for (int f = 0; f < D; ++f)
          if (f != d) dwt[d] *= w[o[f]][f];
      }
      const long long c = K::cell(a.n_grid, base, o);
      R gg[D];
#pragma unroll
      for (int i = 0; i < D; ++i) gg[i] = ggv[c * D + i];
      R gw = ggm[c] * a.mass;
#pragma unroll
      for (int i = 0; i < D; ++i) {
        R mom = a.mass * vp[i];
#pragma unroll
        for (int j = 0; j < D; ++j) mom += aff[i * D + j] * dpos[j];
        gw += gg[i] * mom;
        gvp[i] += wt * a.mass * gg[i];
#pragma unroll
        for (int j = 0; j < D; ++j) gaff[i * D + j] += wt * gg[i] * dpos[j];
      }
#pragma unroll
      for (int j = 0; j < D; ++j) {
        R acc = 0;
#pragma unroll
        for (int i = 0; i < D; ++i) acc += aff[i * D + j] * gg[i];
        gfx[j] -= wt * acc * a.dx;
      }
#pragma unroll
      for (int d = 0; d < D; ++d) gfx[d] += gw * dwt[d];
    }
    R gtau[D * D], gnF[D * D];
#pragma unroll
    for (int i = 0; i < D * D; ++i) {
      gtau[i] = -a.ks * gaff[i];
      gnF[i] = a.aF[q * D * D + i];
    }
    const R ga = K::stress_adj(a, nFm, p, act, gtau, gnF);
    if (m >= 0 && ga != R(0)) atomicAdd(a.gact + (size_t)e * a.M + m, ga);
    // state-f adjoint: x (nx already holds the G2P^T part), v, C, F
#pragma unroll
    for (int d = 0; d < D; ++d) {
      a.nx[q * D + d] += gfx[d] * a.inv_dx;
      a.nv[q * D + d] = gvp[d];
    }
#pragma unroll
    for (int i = 0; i < D; ++i)
#pragma unroll
      for (int j = 0; j < D; ++j) {
        R accC = 0, accF = 0;
#pragma unroll
        for (int k = 0; k < D; ++k) {
          accC += gnF[i * D + k] * Fp[j * D + k];
          accF += ((k == i ? R(1) : R(0)) + a.dt * Cp[k * D + i]) * gnF[k * D + j];
        }
        a.nC[q * D * D + i * D + j] = a.mass * gaff[i * D + j] + a.dt * accC;
        a.nF[q * D * D + i * D + j] = accF;
      }
  }
}

// weighted centre of every env: c = sum pw x / sum pw  (one block per env)
template <typename R, int D>
__global__ void center_kernel(const R* __restrict__ x, const R* __restrict__ pw, R pw_sum, int P,
                              R* __restrict__ out) {
  __shared__ R red[32 * 3];
  const int e = blockIdx.x;
  R s[3] = {0, 0, 0};
  for (int p = threadIdx.x; p < P; p += blockDim.x) {
    const R wgt = pw[p];
#pragma unroll
    for (int d = 0; d < D; ++d) s[d] += wgt * x[((size_t)e * P + p) * D + d];
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int d = 0; d < D; ++d)
    for (int o = 16; o > 0; o >>= 1) s[d] += __shfl_xor_sync(0xffffffffu, s[d], o);
  if (lane == 0)
    for (int d = 0; d < D; ++d) red[d * 32 + wid] = s[d];
  __syncthreads();
  if (threadIdx.x < D) {
    R acc = 0;
    for (int w2 = 0; w2 < nw; ++w2) acc += red[threadIdx.x * 32 + w2];
    out[(size_t)e * D + threadIdx.x] = acc / pw_sum;
  }
}

// loss seed at step t: a_x += 2 w (c - target) pw / sum pw
template <typename R, int D>
__global__ void seed_kernel(R* __restrict__ ax, const R* __restrict__ center, const R* __restrict__ target,
                            const R* __restrict__ pw, R weight, R pw_sum, int n_envs, int P) {
  const long long total = (long long)n_envs * P;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    const int e = (int)(q / P), p = (int)(q % P);
#pragma unroll
    for (int d = 0; d < D; ++d)
      ax[q * D + d] += R(2) * weight * (center[(size_t)e * D + d] - target[(size_t)e * D + d]) * pw[p] / pw_sum;
  }
}

}  // namespace mpm
}  // namespace cls
