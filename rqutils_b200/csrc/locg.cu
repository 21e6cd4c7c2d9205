// Single-vector LOCG/LOBPCG on the device: ground_locg (ground_locg.py:128-162) and
// _ground_locg_callable (:188-423), with _project_out (:426-464), eigenpair_2x2 (:467-478) and
// eigenpair_3x3 (:481-514).
//
// Every BLAS-1 step of an iteration is one pass of a fused kernel k_lc: up to two outputs that
// are linear combinations of up to MAXS input vectors (coefficients read from device memory),
// plus up to MAXD inner products of inputs/outputs, reduced deterministically (per-block
// partials, last block sums them in a fixed order).  The last block then runs the scalar step
// that follows in the algorithm (normalisation factors, the 2x2/3x3 Rayleigh-Ritz solve, the
// convergence test) on one thread and writes the next pass's coefficients, so an iteration has
// no host synchronisation.  With an sqd operator as the matvec the whole while-loop is one
// CUDA graph with a conditional WHILE node whose condition the convergence step sets.
//
// Inner products always accumulate in FP64 (also for FP32 vectors).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cooperative_groups.h>

#include "internal.cuh"
#include "dispatch.cuh"
#include "accum.cuh"

#include <tuple>

namespace sqd {
namespace {

constexpr int LC_THREADS = 256;
constexpr int kMaxOrth = 8;

enum Post : int {
  P_NONE = 0,
  P_INV_NORM,        // coef[0][0] = 1/|v| (no zero guard: xinit /= norm)
  P_THETA0,          // theta = Re <x|ax>; coef (1, -theta) for (ax, x)
  P_R0NORM,          // rnorm; coef[0][0] = 1/rnorm
  P_RR2,             // 2x2 Rayleigh-Ritz -> theta, kappa; coefs of t, u over (x, p)
  P_TU_NORM,         // coefs x = u/|u|, y = t/|t| over (u, t); then r coef (1, -theta)
  P_PROJ_IPS,        // coef (1, -<x|v>, -<y|v>) over (v, x, y)
  P_PROJ_NORM_IPS,   // s = 1/|v| (0 -> 1): coef (s, -s<x|v>, -s<y|v>)
  P_PROJ_MASK,       // keep = |v| >= 0.99
  P_RR3,             // 3x3 Rayleigh-Ritz -> theta, kappa; coef of s over (x, y, p)
  P_SNORM,           // |s| -> coefs of u (out0) and t (out1) over (x, y, p)
  P_XY_NORM,         // coefs x/|u|, y/|t| over (x, y)
  P_CONV,            // residual test (red0 = |r|^2, red1 = |Ax|^2)
  P_CONV_SPLIT,      // residual test with |Ax|^2 stored earlier (orth path)
  P_STORE_AX,        // store |Ax|^2
  P_ORTH_IPS,        // coef (1, -<o_k|v>...) over (v, o_0, ...)
  P_ORTH_NORM,       // s = 1/|v| (0 -> 1)
  P_SET_R_COEF,      // coef (1, -theta) for r = ax - theta x
  P_THETA_ONLY,      // theta = Re <x|ax> (refinement bookkeeping)
  P_RESET,           // clear done/converged/stall tracking (restart of a loop)
  P_GRAM_IMPLICIT,   // fast variant: Gram of {x, y, p} with p unnormalised -> RR3, update coefs
  P_UPDATE_NORMS,    // fast variant: |u|, |t| -> scaling + residual coefs
  P_CONV_PROJ,       // fast variant: residual test + first projection coefs for the next step
  P_CHECK0           // reference residual test on (|r|^2, |Ax|^2) without counting an iteration
};

struct LocgDev {
  double red[16][2];     // reduction results of the last pass
  double coef[6][10][2]; // coefficients of the next pass (output x source)
  double theta;
  double theta_prev;
  double kappa[3][2];
  double rnorm;
  double axnorm2;
  double tol;
  double nscale;         // 10 * n (reltol factor)
  double inner_rtol;     // > 0: converge on |r| < inner_rtol |theta| (FP32 inner sweeps)
  double etol;           // > 0: also stop when |dtheta| <= etol |theta|
  double best_r;
  int best_it;
  int niter;
  int maxiter;
  int converged;
  int done;
  int keep;              // project_out mask result
  int rzero;
  int stall;             // stop after this many iterations without improving |r| (0 = never)
  // Per-iteration record (the reference's log_level <= DEBUG prints, ground_locg.py:330-331,
  // 377-378): rows of kHistCols doubles written by the convergence step while hist_n <
  // hist_cap; hist == nullptr records nothing.
  double* hist;
  int hist_cap;
  int hist_n;
  int hist_phase;        // first column of every row: 0 = FP64 iteration, 1 = FP32 sweep
};

static_assert(sizeof(LocgDev) % sizeof(long long) == 0, "LocgDev is copied in 8-byte words");

// Columns of a history row: phase, iteration, theta, |r|, reltol ((|Ax| - theta) * 10 N; the
// FP32 sweeps store their stopping threshold inner_rtol * |theta| there), converged.
constexpr int kHistCols = 6;

enum Gate : int { G_NONE = 0, G_DONE = 1, G_KEEP = 2 };

template <int MAXS, int MAXD, int MAXO>
struct LCArgs {
  int64_t n;
  const void* src[MAXS];
  void* out[MAXO];
  int nsrc, nout, ndot, post, gate, use_cond;
  signed char da[MAXD], db[MAXD];
  LocgDev* dev;
  double* partials;
  unsigned* counter;
  cudaGraphConditionalHandle cond;
};

// ----------------------------------------------------------------------------- small solvers
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
  const double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 cscale(double2 a, double s) {
  return make_double2(a.x * s, a.y * s);
}

// eigenpair_2x2 (ground_locg.py:467-478); m is Hermitian, row-major.
__device__ void eig2(const double2 m[2][2], double* val, double2 vec[2]) {
  const double d0 = m[0][0].x, d1 = m[1][1].x;
  const double det = d0 * d1 - cabs2(m[1][0]);
  const double tr = d0 + d1;
  // tr^2 - 4 det = (d0 - d1)^2 + 4 |m10|^2 >= 0; rounding can take it just below 0 for a
  // (near-)degenerate pair, where the reference's sqrt returns NaN: clamped at 0.
  const double ev = (tr - sqrt(fmax(tr * tr - 4.0 * det, 0.0))) * 0.5;
  const double2 num = make_double2(d1 - ev + m[1][0].x, -m[1][0].y);
  const double2 den = make_double2(d0 - ev + m[1][0].x, m[1][0].y);
  double2 v0 = cdiv(num, den);
  const double nrm = sqrt(v0.x * v0.x + v0.y * v0.y + 1.0);
  vec[0] = cscale(v0, 1.0 / nrm);
  vec[1] = make_double2(-1.0 / nrm, 0.0);
  *val = ev;
}

// eigenpair_3x3 (ground_locg.py:481-514): Cardano's method after J. Kopp, Int. J. Mod. Phys. C
// 19, 523 (2008), lowest eigenvalue, eigenvector from the cross product of two columns of
// (m - lambda).
__device__ void eig3(const double2 m[3][3], double* val, double2 vec[3]) {
  const double d0 = m[0][0].x, d1 = m[1][1].x, d2 = m[2][2].x;
  const double mo0 = cabs2(m[1][0]), mo1 = cabs2(m[2][0]), mo2 = cabs2(m[2][1]);
  const double c2 = -(d0 + d1 + d2);
  const double c1 = (d0 * d2 + d1 * d0 + d2 * d1) - (mo0 + mo1 + mo2);
  double c0 = d0 * mo2 + d1 * mo1 + d2 * mo0;
  c0 -= d0 * d1 * d2;
  c0 -= 2.0 * cmul(cmul(m[0][2], m[1][0]), m[2][1]).x;
  const double p = c2 * c2 - 3.0 * c1;
  const double q = -13.5 * c0 - c2 * c2 * c2 + 4.5 * c2 * c1;
  // 27 (c1^2 (p - c1) / 4 + c0 (q + 27 c0 / 4)) is 27 times the discriminant term of the
  // characteristic cubic, >= 0 for a Hermitian matrix; rounding (and FMA contraction) can take
  // it just below 0 for (near-)degenerate eigenvalues, where the reference's sqrt returns NaN.
  // Clamped at 0, as are p (>= 0 likewise) below.
  const double phi =
      atan2(sqrt(fmax(27.0 * (0.25 * c1 * c1 * (p - c1) + c0 * (q + 6.75 * c0)), 0.0)), q) /
      3.0;
  const double cphi = cos(phi), sphi = sin(phi);
  const double s3 = sqrt(3.0);
  const double xmin = fmin(fmin(2.0 * cphi, -cphi - s3 * sphi), -cphi + s3 * sphi);
  const double ev = sqrt(fmax(p, 0.0)) / 3.0 * xmin - c2 / 3.0;
  double2 a[3] = {m[0][1], m[1][1], m[2][1]};
  double2 b[3] = {m[0][2], m[1][2], m[2][2]};
  a[1].x -= ev;
  b[2].x -= ev;
  double2 cr[3];
  cr[0] = cconj(csub(cmul(a[1], b[2]), cmul(a[2], b[1])));
  cr[1] = cconj(csub(cmul(a[2], b[0]), cmul(a[0], b[2])));
  cr[2] = cconj(csub(cmul(a[0], b[1]), cmul(a[1], b[0])));
  const double nrm = sqrt(cr[0].x * cr[0].x + cr[1].x * cr[1].x + cr[2].x * cr[2].x +
                          cr[0].y * cr[0].y + cr[1].y * cr[1].y + cr[2].y * cr[2].y);
  for (int k = 0; k < 3; ++k) vec[k] = cscale(cr[k], 1.0 / nrm);
  *val = ev;
}

__device__ __forceinline__ double2 red_c(const LocgDev* d, int k) {
  return make_double2(d->red[k][0], d->red[k][1]);
}
__device__ __forceinline__ void set_coef(LocgDev* d, int o, int k, double2 c) {
  d->coef[o][k][0] = c.x;
  d->coef[o][k][1] = c.y;
}
__device__ __forceinline__ void set_coef_r(LocgDev* d, int o, int k, double c) {
  d->coef[o][k][0] = c;
  d->coef[o][k][1] = 0.0;
}

// Convergence test after an iteration (ground_locg.py:371-376), or the FP32 inner criterion.
__device__ void conv_step(LocgDev* d, double ax2, int use_cond, cudaGraphConditionalHandle cond) {
  const double r = sqrt(d->red[0][0]);
  d->rnorm = r;
  d->niter += 1;
  bool conv;
  double reltol;
  if (d->inner_rtol > 0.0) {
    reltol = d->inner_rtol * fabs(d->theta);
    conv = r < reltol;
    if (r < 0.5 * d->best_r) {
      d->best_r = r;
      d->best_it = d->niter;
    }
    if (d->stall > 0 && d->niter - d->best_it > d->stall) conv = true;
  } else {
    reltol = (sqrt(ax2) - d->theta) * d->nscale;
    conv = r < d->tol * reltol;
  }
  if (d->etol > 0.0 && d->niter >= 2 && fabs(d->theta - d->theta_prev) <= d->etol * fabs(d->theta))
    conv = true;
  if (d->hist != nullptr && d->hist_n < d->hist_cap) {
    double* row = d->hist + static_cast<int64_t>(d->hist_n) * kHistCols;
    row[0] = d->hist_phase;
    row[1] = d->niter;
    row[2] = d->theta;
    row[3] = r;
    row[4] = reltol;
    row[5] = conv ? 1.0 : 0.0;
    d->hist_n += 1;
  }
  d->converged = conv;
  d->done = conv || d->niter >= d->maxiter;
  if (use_cond) cudaGraphSetConditional(cond, d->done ? 0u : 1u);
}

__device__ void run_post(LocgDev* d, int post, int nsrc, int use_cond,
                         cudaGraphConditionalHandle cond) {
  switch (post) {
    case P_NONE: break;
    case P_INV_NORM: set_coef_r(d, 0, 0, 1.0 / sqrt(d->red[0][0])); break;
    case P_THETA0: {
      d->theta = d->red[0][0];
      set_coef_r(d, 0, 0, 1.0);
      set_coef_r(d, 0, 1, -d->theta);
    } break;
    case P_R0NORM: {
      d->rnorm = sqrt(d->red[0][0]);
      d->rzero = d->rnorm == 0.0;
      set_coef_r(d, 0, 0, 1.0 / d->rnorm);
      // The start vector is an exact eigenvector.  The reference carries on into its loop body
      // and divides 0/0 (|s| = 0, ground_locg.py:336-338), returning NaN; here the exact
      // eigenpair is returned instead.
      if (d->rzero) {
        d->converged = 1;
        d->done = 1;
      }
    } break;
    case P_RR2: {
      double2 m[2][2];
      m[0][0] = red_c(d, 0);
      m[1][0] = red_c(d, 1);
      m[0][1] = cconj(m[1][0]);
      m[1][1] = red_c(d, 2);
      double ev;
      double2 k[2];
      eig2(m, &ev, k);
      d->theta = ev;
      // t = p k0 - x k1 ; u = x k0 + p k1   (sources x, p)
      set_coef(d, 0, 0, make_double2(-k[1].x, -k[1].y));
      set_coef(d, 0, 1, k[0]);
      set_coef(d, 1, 0, k[0]);
      set_coef(d, 1, 1, k[1]);
    } break;
    case P_TU_NORM: {
      // red0 = |t|^2, red1 = |u|^2 ; sources (u, t): x = u/|u|, y = t/|t|
      set_coef_r(d, 0, 0, 1.0 / sqrt(d->red[1][0]));
      set_coef_r(d, 0, 1, 0.0);
      set_coef_r(d, 1, 0, 0.0);
      set_coef_r(d, 1, 1, 1.0 / sqrt(d->red[0][0]));
    } break;
    case P_PROJ_IPS: {
      set_coef_r(d, 0, 0, 1.0);
      set_coef(d, 0, 1, make_double2(-d->red[0][0], -d->red[0][1]));
      set_coef(d, 0, 2, make_double2(-d->red[1][0], -d->red[1][1]));
    } break;
    case P_PROJ_NORM_IPS: {
      const double nv = sqrt(d->red[0][0]);
      const double s = nv == 0.0 ? 1.0 : 1.0 / nv;
      set_coef_r(d, 0, 0, s);
      set_coef(d, 0, 1, make_double2(-s * d->red[1][0], -s * d->red[1][1]));
      set_coef(d, 0, 2, make_double2(-s * d->red[2][0], -s * d->red[2][1]));
    } break;
    case P_PROJ_MASK: {
      d->keep = sqrt(d->red[0][0]) >= 0.99;
      set_coef_r(d, 0, 0, d->keep ? 1.0 : 0.0);
    } break;
    case P_RR3: {
      double2 m[3][3];
      m[0][0] = red_c(d, 0);
      m[1][1] = red_c(d, 1);
      m[2][2] = red_c(d, 2);
      m[1][0] = red_c(d, 3);
      m[2][0] = red_c(d, 4);
      m[2][1] = red_c(d, 5);
      m[0][1] = cconj(m[1][0]);
      m[0][2] = cconj(m[2][0]);
      m[1][2] = cconj(m[2][1]);
      double ev;
      double2 k[3];
      eig3(m, &ev, k);
      d->theta_prev = d->theta;
      d->theta = ev;
      for (int i = 0; i < 3; ++i) {
        d->kappa[i][0] = k[i].x;
        d->kappa[i][1] = k[i].y;
      }
      set_coef_r(d, 0, 0, 0.0);
      set_coef(d, 0, 1, k[1]);
      set_coef(d, 0, 2, k[2]);
    } break;
    case P_SNORM: {
      const double ns = sqrt(d->red[0][0]);
      const double2 k0 = make_double2(d->kappa[0][0], d->kappa[0][1]);
      const double2 k1 = make_double2(d->kappa[1][0], d->kappa[1][1]);
      const double2 k2 = make_double2(d->kappa[2][0], d->kappa[2][1]);
      // u = k0 x + k1 y + k2 p
      set_coef(d, 0, 0, k0);
      set_coef(d, 0, 1, k1);
      set_coef(d, 0, 2, k2);
      // t = (k0/ns)(k1 y + k2 p) - ns x
      const double2 f = cscale(k0, 1.0 / ns);
      set_coef_r(d, 1, 0, -ns);
      set_coef(d, 1, 1, cmul(k1, f));
      set_coef(d, 1, 2, cmul(k2, f));
    } break;
    case P_XY_NORM: {
      set_coef_r(d, 0, 0, 1.0 / sqrt(d->red[0][0]));
      set_coef_r(d, 0, 1, 0.0);
      set_coef_r(d, 1, 0, 0.0);
      set_coef_r(d, 1, 1, 1.0 / sqrt(d->red[1][0]));
    } break;
    case P_CONV:
    case P_CONV_SPLIT:
      conv_step(d, post == P_CONV ? d->red[1][0] : d->axnorm2, use_cond, cond);
      break;
    case P_STORE_AX: d->axnorm2 = d->red[0][0]; break;
    case P_ORTH_IPS: {
      set_coef_r(d, 0, 0, 1.0);
      for (int k = 1; k < nsrc; ++k)
        set_coef(d, 0, k, make_double2(-d->red[k - 1][0], -d->red[k - 1][1]));
    } break;
    case P_ORTH_NORM: {
      const double nv = sqrt(d->red[0][0]);
      set_coef_r(d, 0, 0, nv == 0.0 ? 1.0 : 1.0 / nv);
    } break;
    case P_SET_R_COEF: {
      set_coef_r(d, 0, 0, 1.0);
      set_coef_r(d, 0, 1, -d->theta);
    } break;
    case P_THETA_ONLY: d->theta = d->red[0][0]; break;
    case P_RESET: {
      d->done = 0;
      d->converged = 0;
      d->best_r = 1e300;
      d->best_it = d->niter;
    } break;
    case P_CHECK0: {
      const double r = sqrt(d->red[0][0]);
      d->rnorm = r;
      const double reltol = (sqrt(d->red[1][0]) - d->theta) * d->nscale;
      d->converged = r < d->tol * reltol;
      d->done = d->converged;
    } break;
    case P_GRAM_IMPLICIT: {
      // red: 0 <x|Ax> 1 <y|Ay> 2 <p|Ap> 3 <y|Ax> 4 <p|Ax> 5 <p|Ay> 6 <p|p> 7 <y|p>
      const double pp = d->red[6][0];
      if (!(pp > 0.0)) {  // r already in span{x, y}: nothing left to improve
        d->converged = 1;
        d->done = 1;
        if (use_cond) cudaGraphSetConditional(cond, 0u);
        break;
      }
      const double s1 = 1.0 / sqrt(pp);
      double2 m[3][3];
      m[0][0] = red_c(d, 0);
      m[1][1] = red_c(d, 1);
      m[2][2] = cscale(red_c(d, 2), s1 * s1);
      m[1][0] = red_c(d, 3);
      m[2][0] = cscale(red_c(d, 4), s1);
      m[2][1] = cscale(red_c(d, 5), s1);
      m[0][1] = cconj(m[1][0]);
      m[0][2] = cconj(m[2][0]);
      m[1][2] = cconj(m[2][1]);
      double ev;
      double2 k[3];
      eig3(m, &ev, k);
      d->theta_prev = d->theta;
      d->theta = ev;
      const double2 k2 = cscale(k[2], s1);  // coefficient on the unnormalised p
      // |s|^2 for s = k1 y + k2 p_hat, y and p_hat normalised, <y|p_hat> = red7 s1
      const double2 yp = cscale(red_c(d, 7), s1);
      const double ns = sqrt(fmax(cabs2(k[1]) + cabs2(k[2]) + 2.0 * cmul(cconj(k[1]), cmul(k[2], yp)).x, 1e-300));
      const double2 f = cscale(k[0], 1.0 / ns);
      for (int o = 0; o < 4; ++o)
        for (int q = 0; q < 6; ++q) set_coef_r(d, o, q, 0.0);
      // u (x), t (y) over (x, y, p); A u (ax), A t (ay) over (ax, ay, ap)
      set_coef(d, 0, 0, k[0]);
      set_coef(d, 0, 1, k[1]);
      set_coef(d, 0, 2, k2);
      set_coef_r(d, 1, 0, -ns);
      set_coef(d, 1, 1, cmul(k[1], f));
      set_coef(d, 1, 2, cmul(k2, f));
      set_coef(d, 2, 3, k[0]);
      set_coef(d, 2, 4, k[1]);
      set_coef(d, 2, 5, k2);
      set_coef_r(d, 3, 3, -ns);
      set_coef(d, 3, 4, cmul(k[1], f));
      set_coef(d, 3, 5, cmul(k2, f));
    } break;
    case P_UPDATE_NORMS: {
      // red: 0 |u|^2, 1 |t|^2 ; next pass sources (x=u, y=t, ax=Au, ay=At)
      const double cu = 1.0 / sqrt(d->red[0][0]);
      const double ct = 1.0 / sqrt(d->red[1][0]);
      for (int o = 0; o < 5; ++o)
        for (int q = 0; q < 4; ++q) set_coef_r(d, o, q, 0.0);
      set_coef_r(d, 0, 0, cu);
      set_coef_r(d, 1, 1, ct);
      set_coef_r(d, 2, 2, cu);
      set_coef_r(d, 3, 3, ct);
      set_coef_r(d, 4, 0, -d->theta * cu);
      set_coef_r(d, 4, 2, cu);
    } break;
    case P_CONV_PROJ: {
      // red: 0 |r|^2, 1 |Ax|^2, 2 <x|r>, 3 <y|r>
      conv_step(d, d->red[1][0], use_cond, cond);
      for (int q = 0; q < 3; ++q) {
        d->coef[0][q][0] = 0.0;
        d->coef[0][q][1] = 0.0;
      }
      set_coef_r(d, 0, 0, 1.0);
      set_coef(d, 0, 1, make_double2(-d->red[2][0], -d->red[2][1]));
      set_coef(d, 0, 2, make_double2(-d->red[3][0], -d->red[3][1]));
    } break;
    default: break;
  }
}

// Last block of a pass: sums the per-block partials (gridDim.x rows of STRIDE doubles, the
// first nv of each used) into dev->red.  Thread t adds blocks t, t + blockDim.x, ... in order,
// then warps and the block reduce in a fixed order, so the result is deterministic; the loads
// of all values are independent and in flight together (the former one-thread-per-value loop
// over all blocks took ~40 us per pass at 1,024 blocks).
template <int STRIDE>
__device__ __forceinline__ void final_reduce(const double* partials, int nv, LocgDev* dev) {
  __shared__ double wsum[STRIDE][LC_THREADS / 32];
  double t[STRIDE];
#pragma unroll
  for (int q = 0; q < STRIDE; ++q) t[q] = 0.0;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
    const double* row = partials + static_cast<int64_t>(b) * STRIDE;
#pragma unroll
    for (int q = 0; q < STRIDE; ++q)
      if (q < nv) t[q] += __ldcg(row + q);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < STRIDE; ++q) {
    if (q < nv) {
      const double w = warp_sum(t[q]);
      if (lane == 0) wsum[q][warp] = w;
    }
  }
  __syncthreads();
  if (threadIdx.x < nv) {
    double v = 0.0;
    for (int w = 0; w < LC_THREADS / 32; ++w) v += wsum[threadIdx.x][w];
    dev->red[threadIdx.x >> 1][threadIdx.x & 1] = v;
  }
}

// ----------------------------------------------------------------------------- fused pass
template <typename R, int NC, int MAXS, int MAXD, int MAXO>
__global__ void __launch_bounds__(LC_THREADS) k_lc(LCArgs<MAXS, MAXD, MAXO> a) {
  LocgDev* dev = a.dev;
  if ((a.gate & G_DONE) && *(volatile int*)&dev->done) return;
  if ((a.gate & G_KEEP) && *(volatile int*)&dev->keep) return;
  __shared__ double2 sc[MAXO][MAXS];
  for (int t = threadIdx.x; t < MAXO * MAXS; t += blockDim.x)
    sc[t / MAXS][t % MAXS] = make_double2(dev->coef[t / MAXS][t % MAXS][0],
                                          dev->coef[t / MAXS][t % MAXS][1]);
  __syncthreads();
  double acc[MAXD][2];
#pragma unroll
  for (int d = 0; d < MAXD; ++d) acc[d][0] = acc[d][1] = 0.0;

  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < a.n; i += stride) {
    double2 s[MAXS];
#pragma unroll
    for (int k = 0; k < MAXS; ++k) {
      s[k] = make_double2(0.0, 0.0);
      if (k < a.nsrc) {
        const Cx<R> v = ld_elem_rw<R, NC>(static_cast<const R*>(a.src[k]), i);
        s[k] = make_double2(double(v.re), double(v.im));
      }
    }
    double2 o[MAXO];
#pragma unroll
    for (int q = 0; q < MAXO; ++q) {
      o[q] = make_double2(0.0, 0.0);
      if (q < a.nout) {
#pragma unroll
        for (int k = 0; k < MAXS; ++k)
          if (k < a.nsrc) o[q] = cadd(o[q], cmul(sc[q][k], s[k]));
        if constexpr (NC == 1) o[q].y = 0.0;
      }
    }
#pragma unroll
    for (int d = 0; d < MAXD; ++d) {
      if (d < a.ndot) {
        double2 x = make_double2(0.0, 0.0), y = make_double2(0.0, 0.0);
        const int ca = a.da[d], cb = a.db[d];
#pragma unroll
        for (int k = 0; k < MAXS; ++k) {
          if (ca == k) x = s[k];
          if (cb == k) y = s[k];
        }
#pragma unroll
        for (int q = 0; q < MAXO; ++q) {
          if (ca == 100 + q) x = o[q];
          if (cb == 100 + q) y = o[q];
        }
        // conj(x) * y
        acc[d][0] += x.x * y.x + x.y * y.y;
        acc[d][1] += x.x * y.y - x.y * y.x;
      }
    }
#pragma unroll
    for (int q = 0; q < MAXO; ++q)
      if (q < a.nout && a.out[q] != nullptr)
        st_elem<R, NC>(static_cast<R*>(a.out[q]), i, cx_make<R>(R(o[q].x), R(o[q].y)));
  }

  if (a.ndot == 0 && a.post == P_NONE) return;
  // Block reduction of the dot accumulators.
  __shared__ double sred[MAXD * 2][LC_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < MAXD; ++d) {
    if (d < a.ndot) {
      const double v0 = warp_sum(acc[d][0]);
      const double v1 = warp_sum(acc[d][1]);
      if (lane == 0) {
        sred[2 * d][warp] = v0;
        sred[2 * d + 1][warp] = v1;
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < 2 * a.ndot) {
    double t = 0.0;
    for (int w = 0; w < LC_THREADS / 32; ++w) t += sred[threadIdx.x][w];
    a.partials[static_cast<int64_t>(blockIdx.x) * (2 * MAXD) + threadIdx.x] = t;
  }
  __threadfence();
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(a.counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  final_reduce<2 * MAXD>(a.partials, 2 * a.ndot, dev);
  __syncthreads();
  if (threadIdx.x == 0) {
    run_post(dev, a.post, a.nsrc, a.use_cond, a.cond);
    *a.counter = 0u;
  }
}

// A pass whose shape is known at compile time: NS sources, NO outputs and the dots' operand
// codes (k < NS: source k; 100 + q: output q).  The generic k_lc reads these from its
// arguments and predicates every unrolled step and operand choice on them, which makes its
// widest form instruction-bound; the hot passes of the LOCG iterations run through this
// specialisation instead (same arguments, same post-op, same deterministic reduction).
template <int NS_, int NO_, int... D>
struct PassShape {
  static constexpr int NS = NS_, NO = NO_, ND = int(sizeof...(D)) / 2;
  static constexpr int codes[sizeof...(D) + 2] = {D..., 0, 0};
};

template <int C, int NO>
__device__ __forceinline__ double2 operand(const double2* s, const double2* o) {
  if constexpr (C >= 100) return o[C - 100];
  else return s[C];
}

template <typename S, int I, int END>
struct DotLoop {
  __device__ __forceinline__ static void run(double (*acc)[2], const double2* s, const double2* o) {
    if constexpr (I < END) {
      const double2 x = operand<S::codes[2 * I], S::NO>(s, o);
      const double2 y = operand<S::codes[2 * I + 1], S::NO>(s, o);
      acc[I][0] += x.x * y.x + x.y * y.y;   // conj(x) * y
      acc[I][1] += x.x * y.y - x.y * y.x;
      DotLoop<S, I + 1, END>::run(acc, s, o);
    }
  }
};

// A complex value in a pass's arithmetic type T: float in the FP32 sweeps of the persistent
// iteration (their outputs are rounded to float, and FP64 arithmetic runs at a fraction of the
// FP32 rate), double otherwise.  Dots always accumulate in FP64 (a product of two floats is
// exact in double).
template <typename T>
struct C2 {
  T x, y;
};

template <int C, typename T>
__device__ __forceinline__ C2<T> operand_t(const C2<T>* s, const C2<T>* o) {
  if constexpr (C >= 100) return o[C - 100];
  else return s[C];
}

template <typename S, int I, int END>
struct DotLoopT {
  template <typename T>
  __device__ __forceinline__ static void run(double (*acc)[2], const C2<T>* s, const C2<T>* o) {
    if constexpr (I < END) {
      const C2<T> xa = operand_t<S::codes[2 * I]>(s, o);
      const C2<T> ya = operand_t<S::codes[2 * I + 1]>(s, o);
      const double xr = xa.x, xi = xa.y, yr = ya.x, yi = ya.y;
      acc[I][0] += xr * yr + xi * yi;   // conj(x) * y
      acc[I][1] += xr * yi - xi * yr;
      DotLoopT<S, I + 1, END>::run(acc, s, o);
    }
  }
};

template <typename R, int NC, typename S>
__global__ void __launch_bounds__(LC_THREADS) k_lcs(LCArgs<6, 10, 5> a) {
  constexpr int NS = S::NS, NO = S::NO, ND = S::ND;
  constexpr int NOA = NO > 0 ? NO : 1, NDA = ND > 0 ? ND : 1;
  LocgDev* dev = a.dev;
  if ((a.gate & G_DONE) && *(volatile int*)&dev->done) return;
  if ((a.gate & G_KEEP) && *(volatile int*)&dev->keep) return;
  __shared__ double2 sc[NOA][NS];
  for (int t = threadIdx.x; t < NO * NS; t += blockDim.x)
    sc[t / NS][t % NS] = make_double2(dev->coef[t / NS][t % NS][0], dev->coef[t / NS][t % NS][1]);
  __syncthreads();
  double acc[NDA][2];
#pragma unroll
  for (int d = 0; d < NDA; ++d) acc[d][0] = acc[d][1] = 0.0;
  // One element per thread per step (U > 1 makes the compiler keep every coefficient of the
  // wide shapes in registers; they then spill).  Once this step's loads are issued, the sources
  // of the thread's next element are prefetched into L2, so two steps' reads are in flight at
  // the register cost of one.
  constexpr int U = 1;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  constexpr int64_t EB = int64_t(sizeof(R)) * NC;  // bytes per vector element
  for (int64_t i0 = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i0 < a.n; i0 += U * stride) {
    Cx<R> raw[U][NS];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = i0 + u * stride;
#pragma unroll
      for (int k = 0; k < NS; ++k)
        raw[u][k] = i < a.n ? ld_elem_rw<R, NC>(static_cast<const R*>(a.src[k]), i)
                            : cx_make<R>(R(0), R(0));
    }
    if (i0 + U * stride < a.n) {
#pragma unroll
      for (int k = 0; k < NS; ++k)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(static_cast<const char*>(a.src[k]) +
                                                       (i0 + U * stride) * EB));
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int64_t i = i0 + u * stride;
      double2 sv[NS];
#pragma unroll
      for (int k = 0; k < NS; ++k) sv[k] = make_double2(double(raw[u][k].re), double(raw[u][k].im));
      double2 ov[NOA];
#pragma unroll
      for (int q = 0; q < NO; ++q) {
        double2 t = make_double2(0.0, 0.0);
#pragma unroll
        for (int k = 0; k < NS; ++k) t = cadd(t, cmul(sc[q][k], sv[k]));
        if constexpr (NC == 1) t.y = 0.0;
        ov[q] = t;
      }
      if (i < a.n) {
        DotLoop<S, 0, ND>::run(acc, sv, ov);
#pragma unroll
        for (int q = 0; q < NO; ++q)
          if (a.out[q] != nullptr)
            st_elem<R, NC>(static_cast<R*>(a.out[q]), i, cx_make<R>(R(ov[q].x), R(ov[q].y)));
      }
    }
  }
  if (ND == 0 && a.post == P_NONE) return;
  __shared__ double sred[NDA * 2][LC_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    const double v0 = warp_sum(acc[d][0]);
    const double v1 = warp_sum(acc[d][1]);
    if (lane == 0) {
      sred[2 * d][warp] = v0;
      sred[2 * d + 1][warp] = v1;
    }
  }
  __syncthreads();
  if (threadIdx.x < 2 * ND) {
    double t = 0.0;
    for (int w = 0; w < LC_THREADS / 32; ++w) t += sred[threadIdx.x][w];
    a.partials[static_cast<int64_t>(blockIdx.x) * (2 * 10) + threadIdx.x] = t;
  }
  __threadfence();
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(a.counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  final_reduce<2 * 10>(a.partials, 2 * ND, dev);
  __syncthreads();
  if (threadIdx.x == 0) {
    run_post(dev, a.post, a.nsrc, a.use_cond, a.cond);
    *a.counter = 0u;
  }
}

// The pass shapes of the LOCG iterations (reference body, fast implicit body, start/refresh).
using ShapeList = std::tuple<
    PassShape<3, 1, 100, 100, 1, 100, 2, 100>,               // project + normalise + ips
    PassShape<3, 1>,                                         // p = combination of (p, x, y)
    PassShape<6, 0, 0, 3, 1, 4, 2, 5, 1, 3, 2, 3, 2, 4, 2, 2, 1, 2>,  // implicit Gram
    PassShape<6, 4, 100, 100, 101, 101>,                     // x, y, Ax, Ay and norms
    PassShape<4, 5, 104, 104, 102, 102, 100, 104, 101, 104>, // scale, residual, next ips
    PassShape<3, 0, 1, 0, 2, 0>,                             // <x|r>, <y|r>
    PassShape<3, 1, 1, 100, 2, 100>,
    PassShape<3, 1, 100, 100>,
    PassShape<1, 1>,
    PassShape<6, 0, 0, 3, 1, 4, 2, 5, 1, 3, 2, 3, 2, 4>,     // reference Gram (3x3)
    PassShape<3, 2, 100, 100, 101, 101>,
    PassShape<2, 2>,
    PassShape<2, 1, 100, 100, 0, 0>,                         // residual + convergence
    PassShape<2, 1, 0, 0>,
    PassShape<1, 0, 0, 0>,
    PassShape<2, 0, 1, 0>,
    PassShape<2, 1, 100, 100>,
    PassShape<4, 0, 0, 2, 1, 2, 1, 3>,
    PassShape<2, 2, 100, 100, 101, 101>>;

template <typename S>
bool shape_matches(const LCArgs<6, 10, 5>& a) {
  if (a.nsrc != S::NS || a.nout != S::NO || a.ndot != S::ND) return false;
  for (int d = 0; d < S::ND; ++d)
    if (a.da[d] != S::codes[2 * d] || a.db[d] != S::codes[2 * d + 1]) return false;
  return true;
}

// Launches the specialised pass for a's shape; false when no listed shape matches.
template <typename R, int NC, size_t I = 0>
bool launch_shaped(const LCArgs<6, 10, 5>& a, unsigned blocks, cudaStream_t st) {
  if constexpr (I < std::tuple_size<ShapeList>::value) {
    using S = std::tuple_element_t<I, ShapeList>;
    if (shape_matches<S>(a)) {
      k_lcs<R, NC, S><<<blocks, LC_THREADS, 0, st>>>(a);
      return true;
    }
    return launch_shaped<R, NC, I + 1>(a, blocks, st);
  } else {
    return false;
  }
}

template <typename R, int NC>
__global__ void k_onehot(R* x, int64_t n, int64_t idx) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    st_elem<R, NC>(x, i, cx_make<R>(R(i == idx ? 1 : 0), R(0)));
}

template <typename RO, typename RI, int NC>
__global__ void k_convert(const RI* in, RO* out, int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const Cx<RI> v = ld_elem_rw<RI, NC>(in, i);
    st_elem<RO, NC>(out, i, cx_make<RO>(RO(v.re), RO(v.im)));
  }
}

// ------------------------------------------------------------- persistent implicit iteration
// The fast implicit iteration (5 fused passes + 1 cached CSR matvec) as ONE cooperative launch
// that loops until the convergence step sets `done`.  On small operators the graph form is
// bound by its ~6 dependent launches per iteration, each a few microseconds of launch and
// drain; here the iteration is three phases separated by grid barriers: the first projection
// round, the second round fused with the matvec and the Gram dots (persist_gram_matvec), and
// the update with the residual and the convergence dots (PShapeU).  The last block to reach a
// barrier sums the dot partials of all blocks (fixed order) before it releases the others;
// every block then runs the scalar step on its own shared-memory copy of the solver state from
// the same sums, so all blocks hold bit-identical coefficients without a second barrier;
// block 0 writes the history rows and, at the end, the state back.
// Vectors written within the launch are read through L2 (ld.global.cg).
struct PersistArgs {
  // ps[0]: first projection round; ps[2]: the Gram dots' sources (x, y, p, A x, A y, A p);
  // ps[3]: the update pass (PShapeU).  ps[1] and ps[4] are not used: the second projection
  // round is folded into the Gram-matvec phase and the normalisation into the scales.
  LCArgs<6, 10, 5> ps[5];
  const int64_t* row_ptr;      // cached CSR operator
  const uint32_t* cols;
  const void* vals;            // FP64 or FP32 elements, as the vectors
  const void* mv_in;           // p
  void* mv_out;                // A p
  int64_t n;
  LocgDev* dev;
  double* partials;            // gridDim.x x 20 doubles: per-block dot partials
  double* red;                 // 20 doubles: the sums, from the last block of a barrier
  unsigned* bar;               // [0] arrivals, [1] generation, [2] fault (zeroed per launch)
  int max_iter;
};

constexpr long long kBarrierSpinLimit = 1ll << 25;   // most with >= 64 ns sleeps: > 2 s

// Grid barrier for a cooperative launch (all blocks co-resident).  Bounded: a block that
// waits too long, or sees another block's fault, records the fault and returns false, and the
// kernel returns; the host reports it.  When `part` is given, the last block to arrive sums the
// nv per-block partials (in block order, as final_reduce does) into red_g before it releases
// the others, which then read the nv sums; the sums end up in sd.red in every block.
__device__ __forceinline__ bool persist_barrier(unsigned* bar, unsigned& gen,
                                                const double* part = nullptr, int nv = 0,
                                                double* red_g = nullptr, LocgDev* sd = nullptr) {
  __shared__ int last_s, ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last_s = gridDim.x == 1 || atomicAdd(&bar[0], 1u) == gridDim.x - 1;
    ok_s = 1;
  }
  __syncthreads();
  if (last_s) {
    if (part != nullptr) {
      final_reduce<20>(part, nv, sd);
      __syncthreads();
      if (threadIdx.x < nv) red_g[threadIdx.x] = sd->red[threadIdx.x >> 1][threadIdx.x & 1];
    }
    __syncthreads();
    if (threadIdx.x == 0 && gridDim.x > 1) {
      atomicExch(&bar[0], 0u);
      __threadfence();
      atomicAdd(&bar[1], 1u);
    }
  } else if (threadIdx.x == 0) {
    long long spins = 0;
    while (*reinterpret_cast<volatile unsigned*>(&bar[1]) == gen) {
      if (*reinterpret_cast<volatile unsigned*>(&bar[2]) != 0u || ++spins > kBarrierSpinLimit) {
        atomicExch(&bar[2], 1u);
        ok_s = 0;
        break;
      }
      if (spins > 4096) __nanosleep(64);   // poll back to back first: most waits are short
    }
    __threadfence();
  }
  __syncthreads();
  ++gen;
  if (!ok_s) return false;
  if (part != nullptr && !last_s) {
    if (threadIdx.x < nv) sd->red[threadIdx.x >> 1][threadIdx.x & 1] = __ldcg(red_g + threadIdx.x);
    __syncthreads();
  }
  return true;
}

// Sync of all blocks at the end of a phase.  CLU (the grid is one thread-block cluster): the
// hardware cluster barrier (release/acquire at cluster scope); otherwise the bounded grid
// barrier above.
template <bool CLU>
__device__ __forceinline__ bool persist_sync(const PersistArgs& pa, unsigned& gen) {
  if constexpr (CLU) {
    __threadfence();
    cooperative_groups::this_cluster().sync();
    return true;
  } else {
    return persist_barrier(pa.bar, gen);
  }
}

// End of a phase: the block's dot partials (acc: ND complex sums), then the barrier, after
// which every block holds the sums in sd.red.  cpart (CLU only): the kernel's shared [2][20]
// partials, alternating per dot phase; every block sums the blocks' partials through
// distributed shared memory in rank order.
template <int ND, bool CLU>
__device__ __forceinline__ bool persist_finish(double (*acc)[2], LocgDev& sd,
                                               const PersistArgs& pa, unsigned& gen,
                                               double* cpart, int& buf) {
  constexpr int NDA = ND > 0 ? ND : 1;
  double* part = pa.partials;
  if constexpr (ND > 0) {
    __shared__ double sred[NDA * 2][LC_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      const double v0 = warp_sum(acc[d][0]);
      const double v1 = warp_sum(acc[d][1]);
      if (lane == 0) {
        sred[2 * d][warp] = v0;
        sred[2 * d + 1][warp] = v1;
      }
    }
    __syncthreads();
    if (threadIdx.x < 2 * ND) {
      double t = 0.0;
      for (int w = 0; w < LC_THREADS / 32; ++w) t += sred[threadIdx.x][w];
      if constexpr (CLU) cpart[buf * 20 + threadIdx.x] = t;
      else part[static_cast<int64_t>(blockIdx.x) * 20 + threadIdx.x] = t;
    }
  }
  if constexpr (CLU) {
    persist_sync<true>(pa, gen);
    if constexpr (ND > 0) {
      if (threadIdx.x < 2 * ND) {
        cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
        double v = 0.0;
        for (unsigned b = 0; b < cl.num_blocks(); ++b)
          v += cl.map_shared_rank(cpart + buf * 20, b)[threadIdx.x];
        sd.red[threadIdx.x >> 1][threadIdx.x & 1] = v;
      }
      buf ^= 1;
      __syncthreads();
    }
    return true;
  } else if constexpr (ND > 0) {
    return persist_barrier(pa.bar, gen, part, 2 * ND, pa.red, &sd);
  } else {
    return persist_barrier(pa.bar, gen);
  }
}

// A thread step's share of a vector: two elements (8 bytes for float, 16 for complex64 or
// double), or one complex128 element (16 bytes).
template <typename R, int NC>
struct VChunk {
  static constexpr int EB = static_cast<int>(sizeof(R)) * NC;   // bytes per element
  static constexpr int VW = EB >= 16 ? 1 : 2;
  static constexpr int BYTES = VW * EB;
  using Raw = std::conditional_t<BYTES == 16, double2, unsigned long long>;
  R v[VW * NC];
  __device__ __forceinline__ double2 elem(int e) const {
    if constexpr (NC == 2) return make_double2(double(v[2 * e]), double(v[2 * e + 1]));
    else return make_double2(double(v[e]), 0.0);
  }
  __device__ __forceinline__ void set(int e, double2 t) {
    if constexpr (NC == 2) {
      v[2 * e] = R(t.x);
      v[2 * e + 1] = R(t.y);
    } else {
      v[e] = R(t.x);
    }
  }
  __device__ __forceinline__ C2<R> elem_t(int e, R scale) const {
    if constexpr (NC == 2) return C2<R>{v[2 * e] * scale, v[2 * e + 1] * scale};
    else return C2<R>{v[e] * scale, R(0)};
  }
  __device__ __forceinline__ void set_t(int e, C2<R> t) {
    if constexpr (NC == 2) {
      v[2 * e] = t.x;
      v[2 * e + 1] = t.y;
    } else {
      v[e] = t.x;
    }
  }
};
static_assert(sizeof(VChunk<float, 2>) == 16 && sizeof(VChunk<float, 1>) == 8 &&
              sizeof(VChunk<double, 1>) == 16 && sizeof(VChunk<double, 2>) == 16, "chunks");

template <typename R, int NC>
__device__ __forceinline__ VChunk<R, NC> ld_chunk_cg(const R* p, int64_t j) {
  using Raw = typename VChunk<R, NC>::Raw;
  const Raw raw = __ldcg(reinterpret_cast<const Raw*>(p) + j);
  VChunk<R, NC> c;
  memcpy(&c, &raw, sizeof(Raw));
  return c;
}

template <typename R, int NC>
__device__ __forceinline__ void st_chunk(R* p, int64_t j, const VChunk<R, NC>& c) {
  using Raw = typename VChunk<R, NC>::Raw;
  Raw raw;
  memcpy(&raw, &c, sizeof(Raw));
  reinterpret_cast<Raw*>(p)[j] = raw;
}

// One elementwise pass: every element's NO outputs as combinations of its NS sources (each
// times its scale sc[k], see k_locg_persist) with the coefficients in sd.coef, in the vectors'
// precision, the ND dots in FP64, then the phase end and the post step.  Each thread step moves two elements of every vector
// (one complex128; 16 bytes for complex64), which puts twice the bytes in flight per load as
// one element at a time; the vectors are 16-byte aligned (the host checks), an odd last
// element is done on its own.
template <typename R, int NC, typename S, bool CLU>
__device__ __forceinline__ bool persist_pass(const LCArgs<6, 10, 5>& a, LocgDev& sd,
                                             const PersistArgs& pa, unsigned& gen,
                                             double* cpart, int& buf, const double* sc) {
  constexpr int NS = S::NS, NO = S::NO, ND = S::ND;
  constexpr int NOA = NO > 0 ? NO : 1, NDA = ND > 0 ? ND : 1;
  constexpr int VW = VChunk<R, NC>::VW;
  using T = R;   // the combinations' arithmetic type (C2 above)
  __shared__ C2<T> co[NOA][NS];
  for (int t = threadIdx.x; t < NO * NS; t += blockDim.x)
    co[t / NS][t % NS] = C2<T>{T(sd.coef[t / NS][t % NS][0]), T(sd.coef[t / NS][t % NS][1])};
  T scl[NS];
#pragma unroll
  for (int k = 0; k < NS; ++k) scl[k] = T(sc[k]);
  __syncthreads();
  double acc[NDA][2];
#pragma unroll
  for (int d = 0; d < NDA; ++d) acc[d][0] = acc[d][1] = 0.0;
  auto combine = [&](const C2<T>* sv, C2<T>* ov) {
#pragma unroll
    for (int q = 0; q < NO; ++q) {
      C2<T> t{T(0), T(0)};
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        const C2<T> c = co[q][k];
        t.x += c.x * sv[k].x - c.y * sv[k].y;
        t.y += c.x * sv[k].y + c.y * sv[k].x;
      }
      if constexpr (NC == 1) t.y = T(0);
      ov[q] = t;
    }
    DotLoopT<S, 0, ND>::run(acc, sv, ov);
  };
  const int64_t tid = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  const int64_t nvec = a.n / VW;
  for (int64_t j = tid; j < nvec; j += stride) {
    VChunk<R, NC> raw[NS];
#pragma unroll
    for (int k = 0; k < NS; ++k) raw[k] = ld_chunk_cg<R, NC>(static_cast<const R*>(a.src[k]), j);
    if (j + stride < nvec) {
#pragma unroll
      for (int k = 0; k < NS; ++k)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(static_cast<const char*>(a.src[k]) +
                                                       (j + stride) * VChunk<R, NC>::BYTES));
    }
    VChunk<R, NC> res[NOA];
#pragma unroll
    for (int e = 0; e < VW; ++e) {
      C2<T> sv[NS], ov[NOA];
#pragma unroll
      for (int k = 0; k < NS; ++k) sv[k] = raw[k].elem_t(e, scl[k]);
      combine(sv, ov);
#pragma unroll
      for (int q = 0; q < NO; ++q) res[q].set_t(e, ov[q]);
    }
#pragma unroll
    for (int q = 0; q < NO; ++q)
      if (a.out[q] != nullptr) st_chunk<R, NC>(static_cast<R*>(a.out[q]), j, res[q]);
  }
  if constexpr (VW > 1) {
    for (int64_t i = nvec * VW + tid; i < a.n; i += stride) {
      C2<T> sv[NS], ov[NOA];
#pragma unroll
      for (int k = 0; k < NS; ++k) {
        const Cx<R> v = ld_elem_cg<R, NC>(static_cast<const R*>(a.src[k]), i);
        sv[k] = C2<T>{v.re * scl[k], v.im * scl[k]};
      }
      combine(sv, ov);
#pragma unroll
      for (int q = 0; q < NO; ++q)
        if (a.out[q] != nullptr)
          st_elem<R, NC>(static_cast<R*>(a.out[q]), i, cx_make<R>(ov[q].x, ov[q].y));
    }
  }
  if (!persist_finish<ND, CLU>(acc, sd, pa, gen, cpart, buf)) return false;
  if (threadIdx.x == 0 && a.post != P_NONE) run_post(&sd, a.post, a.nsrc, 0, 0);
  __syncthreads();
  return true;
}

using PShape0 = PassShape<3, 1, 100, 100, 1, 100, 2, 100>;
using PShape2 = PassShape<6, 0, 0, 3, 1, 4, 2, 5, 1, 3, 2, 3, 2, 4, 2, 2, 1, 2>;
// The update pass of the persistent iteration: u, t, A u, A t and r' = A u - theta u from
// (x, y, p0, A x, A y, A p0), unnormalised, with |u|^2, |t|^2, |r'|^2, |A u|^2, <u|r'>, <t|r'>.
// body_fast normalises in a pass of its own (x, y, A x, A y read and written once more, r
// written); here the norms become the scales the next passes apply as they load.
using PShapeU = PassShape<6, 5, 100, 100, 101, 101, 104, 104, 102, 102, 100, 104, 101, 104>;

// x[i] *= s, in place (the final normalisation of a persistent loop).
template <typename R, int NC>
struct PersistNorm {
  R* p;
  double s;
  __device__ __forceinline__ void apply(int64_t i) const {
    const Cx<R> v = ld_elem_cg<R, NC>(p, i);
    st_elem<R, NC>(p, i, cx_make<R>(R(double(v.re) * s), R(double(v.im) * s)));
  }
};

// The second projection round of p, the matvec and the Gram pass of the fast iteration
// (body_fast's passes 2 and 3 and its matvec) as ONE phase.  The second round forms
// p = c0 p0 + c1 x + c2 y from the first round's p0 with the coefficients c of the first
// round's post step; since A p = c0 A p0 + c1 A x + c2 A y and A x, A y are carried, the phase
// gathers p0 (complete since the last barrier) for A p0, stores A p0 where A p would go, forms
// p and A p of its own rows in registers for the Gram dots, and once the Rayleigh-Ritz step has
// set the update pass's coefficients over (x, y, p, A x, A y, A p), folds c into them so that
// the update pass reads p0 and A p0 instead.  Relative to c0, c1 and c2 are the second round's
// corrections, of the order of the first round's rounding error, so the carried A x, A y enter
// with that weight.  This saves two grid barriers and four vector streams per iteration.
// Rows: LPR lanes per row (the row's elementwise operands are loaded by its first lane before
// the row's pair loads are issued); with LPR = 1 (rows of about one stored pair, such as
// near-diagonal operators) a thread takes two or four consecutive rows per step.
template <typename R, int NC, int NCA, int LPR, bool CLU>
__device__ __forceinline__ bool persist_gram_matvec(const PersistArgs& pa, LocgDev& sd,
                                                    unsigned& gen, double* cpart, int& buf,
                                                    const double* vs) {
  using S = PShape2;   // sources x, y, p, A x, A y, A p; eight dots
  constexpr int ND = S::ND;
  const LCArgs<6, 10, 5>& g = pa.ps[2];
  const R* xs = static_cast<const R*>(g.src[0]);
  const R* ys = static_cast<const R*>(g.src[1]);
  const R* p0 = static_cast<const R*>(pa.mv_in);
  const R* axs = static_cast<const R*>(g.src[3]);
  const R* ays = static_cast<const R*>(g.src[4]);
  const R* vals = static_cast<const R*>(pa.vals);
  R* ap0 = static_cast<R*>(pa.mv_out);
  const double2 c0 = make_double2(sd.coef[0][0][0], sd.coef[0][0][1]);
  const double2 c1 = make_double2(sd.coef[0][1][0], sd.coef[0][1][1]);
  const double2 c2 = make_double2(sd.coef[0][2][0], sd.coef[0][2][1]);
  const double sx = vs[0], sy = vs[1];   // stored x, A x and y, A y times these
  double acc[ND][2];
#pragma unroll
  for (int d = 0; d < ND; ++d) acc[d][0] = acc[d][1] = 0.0;
  auto d2 = [](Cx<R> v) { return make_double2(double(v.re), double(v.im)); };
  // A p0 of the row is m; x..ay its elementwise operands.
  auto finish = [&](int64_t row, const CAcc<R, NC, NCA>& m, Cx<R> x, Cx<R> y, Cx<R> p,
                    Cx<R> ax, Cx<R> ay) {
    const Cx<R> a0 = cx_make<R>(m.re.value(), m.im.value());
    st_elem<R, NC>(ap0, row, a0);
    double2 sv[6];
    sv[0] = cscale(d2(x), sx);
    sv[1] = cscale(d2(y), sy);
    sv[3] = cscale(d2(ax), sx);
    sv[4] = cscale(d2(ay), sy);
    sv[2] = cadd(cmul(c0, d2(p)), cadd(cmul(c1, sv[0]), cmul(c2, sv[1])));
    sv[5] = cadd(cmul(c0, d2(a0)), cadd(cmul(c1, sv[3]), cmul(c2, sv[4])));
    if constexpr (NC == 1) sv[2].y = sv[5].y = 0.0;
    DotLoop<S, 0, ND>::run(acc, sv, sv);
  };
  const Cx<R> zero = cx_make<R>(R(0), R(0));
  if constexpr (LPR == 1) {
    // ROWS consecutive rows per thread step (one 16-byte chunk of every vector for complex64,
    // two for complex128): their pair chains are in flight together and their elementwise
    // operands arrive as chunk loads.
    constexpr int VW = VChunk<R, NC>::VW;
    constexpr int ROWS = VW > 2 ? VW : 2;
    constexpr int NCH = ROWS / VW;
    const int64_t tid = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    const int64_t T = int64_t(gridDim.x) * blockDim.x;
    const int64_t nsteps = pa.n / ROWS;
    for (int64_t j = tid; j < nsteps; j += T) {
      const int64_t row0 = j * ROWS;
      VChunk<R, NC> cx[NCH], cy[NCH], cp[NCH], cax[NCH], cay[NCH];
#pragma unroll
      for (int h = 0; h < NCH; ++h) {
        cx[h] = ld_chunk_cg<R, NC>(xs, j * NCH + h);
        cy[h] = ld_chunk_cg<R, NC>(ys, j * NCH + h);
        cp[h] = ld_chunk_cg<R, NC>(p0, j * NCH + h);
        cax[h] = ld_chunk_cg<R, NC>(axs, j * NCH + h);
        cay[h] = ld_chunk_cg<R, NC>(ays, j * NCH + h);
      }
      int64_t bnd[ROWS + 1];
#pragma unroll
      for (int u = 0; u <= ROWS; ++u) bnd[u] = __ldg(pa.row_ptr + row0 + u);
      uint32_t c[ROWS];
#pragma unroll
      for (int u = 0; u < ROWS; ++u) c[u] = bnd[u] < bnd[u + 1] ? __ldg(pa.cols + bnd[u]) : 0u;
      CAcc<R, NC, NCA> m[ROWS];
#pragma unroll
      for (int u = 0; u < ROWS; ++u)
        if (bnd[u] < bnd[u + 1])
          m[u].add(ld_elem<R, NCA>(vals, bnd[u]), ld_elem_cg<R, NC>(p0, c[u]));
#pragma unroll
      for (int u = 0; u < ROWS; ++u)
        if (bnd[u] + 1 < bnd[u + 1])
          csr_row_dot<R, NC, NCA, 1, true>(pa.cols, vals, p0, bnd[u] + 1, bnd[u + 1], m[u]);
      VChunk<R, NC> ca[NCH];
#pragma unroll
      for (int u = 0; u < ROWS; ++u) {
        const Cx<R> a0 = cx_make<R>(m[u].re.value(), m[u].im.value());
        ca[u / VW].set(u % VW, d2(a0));
        double2 sv[6];
        sv[0] = cscale(cx[u / VW].elem(u % VW), sx);
        sv[1] = cscale(cy[u / VW].elem(u % VW), sy);
        sv[3] = cscale(cax[u / VW].elem(u % VW), sx);
        sv[4] = cscale(cay[u / VW].elem(u % VW), sy);
        sv[2] = cadd(cmul(c0, cp[u / VW].elem(u % VW)), cadd(cmul(c1, sv[0]), cmul(c2, sv[1])));
        sv[5] = cadd(cmul(c0, d2(a0)), cadd(cmul(c1, sv[3]), cmul(c2, sv[4])));
        if constexpr (NC == 1) sv[2].y = sv[5].y = 0.0;
        DotLoop<S, 0, ND>::run(acc, sv, sv);
      }
#pragma unroll
      for (int h = 0; h < NCH; ++h) st_chunk<R, NC>(ap0, j * NCH + h, ca[h]);
    }
    for (int64_t row = nsteps * ROWS + tid; row < pa.n; row += T) {
      CAcc<R, NC, NCA> m;
      csr_row_dot<R, NC, NCA, 1, true>(pa.cols, vals, p0, __ldg(pa.row_ptr + row),
                                       __ldg(pa.row_ptr + row + 1), m);
      finish(row, m, ld_elem_cg<R, NC>(xs, row), ld_elem_cg<R, NC>(ys, row),
             ld_elem_cg<R, NC>(p0, row), ld_elem_cg<R, NC>(axs, row), ld_elem_cg<R, NC>(ays, row));
    }
  } else {
    constexpr int RPW = 32 / LPR;
    const int lane = threadIdx.x & 31;
    const int sub = lane % LPR, slot = lane / LPR;
    const int64_t w0 = (blockIdx.x * int64_t(blockDim.x) + threadIdx.x) >> 5;
    const int64_t nw = (int64_t(gridDim.x) * blockDim.x) >> 5;
    for (int64_t rb = w0 * RPW; rb < pa.n; rb += nw * RPW) {
      const int64_t row = rb + slot;
      const bool live = row < pa.n, lead = live && sub == 0;
      const Cx<R> ex = lead ? ld_elem_cg<R, NC>(xs, row) : zero;
      const Cx<R> ey = lead ? ld_elem_cg<R, NC>(ys, row) : zero;
      const Cx<R> ep = lead ? ld_elem_cg<R, NC>(p0, row) : zero;
      const Cx<R> eax = lead ? ld_elem_cg<R, NC>(axs, row) : zero;
      const Cx<R> eay = lead ? ld_elem_cg<R, NC>(ays, row) : zero;
      CAcc<R, NC, NCA> m;
      if (live) {
        const int64_t b = __ldg(pa.row_ptr + row), e = __ldg(pa.row_ptr + row + 1);
        csr_row_dot<R, NC, NCA, LPR, true>(pa.cols, vals, p0, b + sub, e, m);
      }
      m.merge(LPR);
      if (lead) finish(row, m, ex, ey, ep, eax, eay);
    }
  }
  if (!persist_finish<ND, CLU>(acc, sd, pa, gen, cpart, buf)) return false;
  if (threadIdx.x == 0) {
    run_post(&sd, g.post, g.nsrc, 0, 0);
    if (!sd.done) {
      // update pass: x, y over sources (x, y, p) = columns 0-2, A x, A y over columns 3-5
      for (int o = 0; o < 4; ++o) {
        const int q0 = o < 2 ? 0 : 3;
        const double2 k = make_double2(sd.coef[o][q0 + 2][0], sd.coef[o][q0 + 2][1]);
        const double2 a = cadd(make_double2(sd.coef[o][q0][0], sd.coef[o][q0][1]), cmul(k, c1));
        const double2 b = cadd(make_double2(sd.coef[o][q0 + 1][0], sd.coef[o][q0 + 1][1]),
                               cmul(k, c2));
        const double2 f = cmul(k, c0);
        sd.coef[o][q0][0] = a.x;
        sd.coef[o][q0][1] = a.y;
        sd.coef[o][q0 + 1][0] = b.x;
        sd.coef[o][q0 + 1][1] = b.y;
        sd.coef[o][q0 + 2][0] = f.x;
        sd.coef[o][q0 + 2][1] = f.y;
      }
      // fifth output of the update pass: r' = A u - theta u (the residual times |u|)
      for (int q = 0; q < 6; ++q) {
        sd.coef[4][q][0] = q < 3 ? -sd.theta * sd.coef[0][q][0] : sd.coef[2][q][0];
        sd.coef[4][q][1] = q < 3 ? -sd.theta * sd.coef[0][q][1] : sd.coef[2][q][1];
      }
    }
  }
  __syncthreads();
  return true;
}

// Two blocks per SM: the FP32 passes' 16-byte steps and the Gram phase's eight FP64 dot sums
// need up to 128 registers a thread (with three blocks per SM, 85, they spilled 0.5-1 KB).
template <typename R, int NC, int NCA, int LPR, bool CLU>
__global__ void __launch_bounds__(LC_THREADS, 2) k_locg_persist(PersistArgs pa) {
  __shared__ LocgDev sd;
  __shared__ double cpart[2 * 20];
  {
    const long long* src = reinterpret_cast<const long long*>(pa.dev);
    long long* dst = reinterpret_cast<long long*>(&sd);
    for (int i = threadIdx.x; i < int(sizeof(LocgDev) / sizeof(long long)); i += blockDim.x)
      dst[i] = __ldcg(src + i);
  }
  // vs: the stored x, A x, r times vs[0] and y, A y times vs[1] are the iteration's (normalised)
  // vectors; sc0, scu: the per-source scales of the first projection and the update pass.
  __shared__ double vs[2], sc0[3], scu[6];
  if (threadIdx.x < 6) {
    scu[threadIdx.x] = 1.0;
    if (threadIdx.x < 3) sc0[threadIdx.x] = 1.0;
    if (threadIdx.x < 2) vs[threadIdx.x] = 1.0;
  }
  __syncthreads();
  if (blockIdx.x != 0 && threadIdx.x == 0) sd.hist = nullptr;   // block 0 records
  __syncthreads();
  unsigned gen = 0;
  int buf = 0;
  for (int it = 0; it < pa.max_iter && !sd.done; ++it) {
    if (!persist_pass<R, NC, PShape0, CLU>(pa.ps[0], sd, pa, gen, cpart, buf, sc0)) return;
    if (!persist_gram_matvec<R, NC, NCA, LPR, CLU>(pa, sd, gen, cpart, buf, vs)) return;
    if (sd.done) break;   // the Rayleigh-Ritz step found nothing left to improve
    if (!persist_pass<R, NC, PShapeU, CLU>(pa.ps[3], sd, pa, gen, cpart, buf, scu)) return;
    if (threadIdx.x == 0) {
      // red: |u|^2, |t|^2, |r'|^2, |A u|^2, <u|r'>, <t|r'> of the stored (unnormalised) update;
      // the convergence step wants |r|^2, |A x|^2, <x|r>, <y|r> of x = u/|u|, y = t/|t|,
      // r = r'/|u|.
      const double cu = 1.0 / sqrt(sd.red[0][0]), ct = 1.0 / sqrt(sd.red[1][0]);
      const double rr = cu * cu * sd.red[2][0], axax = cu * cu * sd.red[3][0];
      const double xr0 = cu * cu * sd.red[4][0], xr1 = cu * cu * sd.red[4][1];
      const double yr0 = cu * ct * sd.red[5][0], yr1 = cu * ct * sd.red[5][1];
      sd.red[0][0] = rr;
      sd.red[0][1] = 0.0;
      sd.red[1][0] = axax;
      sd.red[1][1] = 0.0;
      sd.red[2][0] = xr0;
      sd.red[2][1] = xr1;
      sd.red[3][0] = yr0;
      sd.red[3][1] = yr1;
      run_post(&sd, P_CONV_PROJ, 4, 0, 0);
      vs[0] = cu;
      vs[1] = ct;
      sc0[0] = cu;   // r
      sc0[1] = cu;   // x
      sc0[2] = ct;   // y
      scu[0] = cu;   // x
      scu[1] = ct;   // y
      scu[3] = cu;   // A x
      scu[4] = ct;   // A y
    }
    __syncthreads();
  }
  // Leave the vectors normalised for the host (all blocks are past the last phase's barrier).
  {
    const PersistNorm<R, NC> nx{static_cast<R*>(const_cast<void*>(pa.ps[3].src[0])), vs[0]};
    const PersistNorm<R, NC> ny{static_cast<R*>(const_cast<void*>(pa.ps[3].src[1])), vs[1]};
    const PersistNorm<R, NC> nax{static_cast<R*>(const_cast<void*>(pa.ps[3].src[3])), vs[0]};
    const PersistNorm<R, NC> nay{static_cast<R*>(const_cast<void*>(pa.ps[3].src[4])), vs[1]};
    const PersistNorm<R, NC> nr{static_cast<R*>(pa.ps[3].out[4]), vs[0]};
    const int64_t tid = blockIdx.x * int64_t(blockDim.x) + threadIdx.x;
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = tid; i < pa.n; i += stride) {
      nx.apply(i);
      ny.apply(i);
      nax.apply(i);
      nay.apply(i);
      nr.apply(i);
    }
  }
  if constexpr (CLU) persist_sync<true>(pa, gen);   // no block leaves while others read its smem
  if (blockIdx.x == 0) {
    const long long* src = reinterpret_cast<const long long*>(&sd);
    long long* dst = reinterpret_cast<long long*>(pa.dev);
    for (int i = threadIdx.x; i < int(sizeof(LocgDev) / sizeof(long long)); i += blockDim.x)
      dst[i] = src[i];
  }
}

// ----------------------------------------------------------------------------- host driver
struct Vec {
  void* p = nullptr;
};

template <typename R, int NC>
class Locg {
 public:
  using Tiny = LCArgs<3, 3, 2>;
  using Wide = LCArgs<6, 10, 5>;
  using Orth = LCArgs<kMaxOrth + 1, kMaxOrth, 2>;

  Locg(int64_t n, sqd_matvec_fn fn, void* ctx, cudaStream_t st)
      : n_(n), fn_(fn), ctx_(ctx), st_(st), cur_(st) {
    for (auto* b : {&x_, &y_, &r_, &p_, &ax_, &ay_, &ap_, &t0_})
      b->alloc(static_cast<size_t>(n) * NC, st);
    blocks_ = static_cast<unsigned>(
        std::max<int64_t>(1, std::min<int64_t>((n + LC_THREADS - 1) / LC_THREADS,
                                               8 * num_sms())));
    partials_.alloc(static_cast<size_t>(blocks_) * 2 * 16, st);
    counter_.alloc(1, st);
    dev_.alloc(1, st);
    SQD_CUDA(cudaMemsetAsync(counter_.ptr, 0, sizeof(unsigned), st));
    SQD_CUDA(cudaMemsetAsync(dev_.ptr, 0, sizeof(LocgDev), st));
    SQD_CUDA(cudaMallocHost(reinterpret_cast<void**>(&host_), sizeof(LocgDev)));
  }
  ~Locg() {
    for (int v = 0; v < 2; ++v) {
      if (exec_[v]) cudaGraphExecDestroy(exec_[v]);
      if (graph_[v]) cudaGraphDestroy(graph_[v]);
    }
    if (host_) cudaFreeHost(host_);
  }

  R* x() { return x_.ptr; }
  LocgDev* dev() { return dev_.ptr; }
  // A cached solver serving a later call on another stream (its previous work has finished:
  // every solve ends with a stream synchronisation).
  void set_stream(cudaStream_t st) { st_ = cur_ = st; }

  // Where the next solve records its iterations (nullptr: nothing); takes effect at
  // set_params.
  void set_history(double* rows, int cap, int phase) {
    hist_ = rows;
    hist_cap_ = cap;
    hist_phase_ = phase;
  }

  void set_params(double tol, double nscale, int maxiter, double inner_rtol, double etol,
                  int stall) {
    LocgDev h{};
    h.hist = hist_;
    h.hist_cap = hist_cap_;
    h.hist_phase = hist_phase_;
    h.tol = tol;
    h.nscale = nscale;
    h.maxiter = maxiter;
    h.inner_rtol = inner_rtol;
    h.etol = etol;
    h.stall = stall;
    h.best_r = 1e300;
    // Copy only the parameter block; counters are reset here too.
    SQD_CUDA(cudaMemcpyAsync(dev_.ptr, &h, sizeof(LocgDev), cudaMemcpyHostToDevice, st_));
    SQD_CUDA(cudaStreamSynchronize(st_));
  }

  // ---- one fused pass
  void lc(std::initializer_list<const void*> srcs, std::initializer_list<void*> outs,
          std::initializer_list<std::pair<int, int>> dots, int post, int gate = G_NONE) {
    if (srcs.size() <= 6 && dots.size() <= 10 && outs.size() <= 5) {
      Wide w{};
      fill(w, srcs, outs, dots, post, gate);
      if (launch_shaped<R, NC>(w, blocks_, cur_)) {
        SQD_CHECK_LAUNCH();
        return;
      }
    }
    if (srcs.size() <= 3 && dots.size() <= 3 && outs.size() <= 2) {
      Tiny a{};
      fill(a, srcs, outs, dots, post, gate);
      k_lc<R, NC, 3, 3, 2><<<blocks_, LC_THREADS, 0, cur_>>>(a);
    } else if (srcs.size() <= 6 && dots.size() <= 10 && outs.size() <= 5) {
      Wide a{};
      fill(a, srcs, outs, dots, post, gate);
      k_lc<R, NC, 6, 10, 5><<<blocks_, LC_THREADS, 0, cur_>>>(a);
    } else {
      SQD_REQUIRE(srcs.size() <= kMaxOrth + 1 && dots.size() <= kMaxOrth && outs.size() <= 2,
                  "fused pass too wide");
      Orth a{};
      fill(a, srcs, outs, dots, post, gate);
      k_lc<R, NC, kMaxOrth + 1, kMaxOrth, 2><<<blocks_, LC_THREADS, 0, cur_>>>(a);
    }
    SQD_CHECK_LAUNCH();
  }

  // Runs only the scalar step `post` (one thread).
  void post_only(int post, int gate = G_NONE) {
    Tiny a{};
    fill(a, {}, {}, {}, post, gate);
    a.n = 0;
    k_lc<R, NC, 3, 3, 2><<<1, LC_THREADS, 0, cur_>>>(a);
    SQD_CHECK_LAUNCH();
  }

  void matvec(const void* in, void* out) {
    const int rc = fn_(ctx_, in, out, cur_);
    if (rc != SQD_OK) throw Error(rc, std::string("matvec callback failed: ") + last_msg());
  }

  void read_host() {
    SQD_CUDA(cudaMemcpyAsync(host_, dev_.ptr, sizeof(LocgDev), cudaMemcpyDeviceToHost, st_));
    SQD_CUDA(cudaStreamSynchronize(st_));
  }
  const LocgDev& host() const { return *host_; }

  // project_out(orth, v, normalize) with n_orth basis vectors (ground_locg.py:426-464).
  void project_orth(const std::vector<const void*>& orth, void* v, bool normalize, int gate) {
    if (orth.empty()) return;
    for (int round = 0; round < 4; ++round) {
      std::vector<std::pair<int, int>> dd;
      for (size_t k = 0; k < orth.size(); ++k) dd.push_back({static_cast<int>(k + 1), 0});
      lc_vec(orth, v, {}, dd, P_ORTH_IPS, gate);
      const bool norm_now = normalize && round < 2;
      lc_vec(orth, v, {v}, norm_now ? std::vector<std::pair<int, int>>{{100, 100}}
                                     : std::vector<std::pair<int, int>>{},
             norm_now ? P_ORTH_NORM : P_NONE, gate);
      if (norm_now) lc({v}, {v}, {}, P_NONE, gate);
    }
    if (normalize) {
      lc({v}, {}, {{0, 0}}, P_PROJ_MASK, gate);
      lc({v}, {v}, {}, P_NONE, gate | G_KEEP);
    }
  }

  // ---------------------------------------------------------------- the faithful algorithm
  // Start: x already holds xinit (unnormalised).  Returns after iter0 and iter1.
  void start(const std::vector<const void*>& orth) {
    R* x = x_.ptr;
    lc({x}, {}, {{0, 0}}, P_INV_NORM);
    lc({x}, {x}, {}, P_NONE);
    // body_iter0 (:280-291)
    matvec(x, ax_.ptr);
    project_orth(orth, ax_.ptr, false, G_NONE);
    lc({ax_.ptr, x}, {}, {{1, 0}}, P_THETA0);
    lc({ax_.ptr, x}, {r_.ptr}, {{100, 100}}, P_R0NORM);
    read_host();
    if (host_->rzero) {
      SQD_CUDA(cudaMemsetAsync(y_.ptr, 0, sizeof(R) * NC * n_, st_));
      return;
    }
    // body_iter1 (:293-322)
    lc({r_.ptr}, {p_.ptr}, {}, P_NONE);
    matvec(x, ax_.ptr);
    matvec(p_.ptr, ap_.ptr);
    lc({x, p_.ptr, ax_.ptr, ap_.ptr}, {}, {{0, 2}, {1, 2}, {1, 3}}, P_RR2);
    lc({x, p_.ptr}, {t0_.ptr, ay_.ptr}, {{100, 100}, {101, 101}}, P_TU_NORM);  // t, u
    lc({ay_.ptr, t0_.ptr}, {x, y_.ptr}, {}, P_NONE);
    project_orth(orth, x, true, G_NONE);
    matvec(x, ax_.ptr);
    post_only(P_SET_R_COEF);
    lc({ax_.ptr, x}, {r_.ptr}, {}, P_NONE);
    project_orth(orth, r_.ptr, false, G_NONE);
  }

  // One body iteration (:324-383).  All passes are gated on `done`.
  void body(const std::vector<const void*>& orth) {
    R *x = x_.ptr, *y = y_.ptr, *r = r_.ptr, *p = p_.ptr;
    const int g = G_DONE;
    // p = project_out((x, y), r): 4 rounds, normalising in the first two.
    lc({r, x, y}, {}, {{1, 0}, {2, 0}}, P_PROJ_IPS, g);
    lc({r, x, y}, {p}, {{100, 100}, {1, 100}, {2, 100}}, P_PROJ_NORM_IPS, g);
    lc({p, x, y}, {p}, {{100, 100}, {1, 100}, {2, 100}}, P_PROJ_NORM_IPS, g);
    lc({p, x, y}, {p}, {{1, 100}, {2, 100}}, P_PROJ_IPS, g);
    lc({p, x, y}, {p}, {{100, 100}}, P_PROJ_MASK, g);
    lc({p}, {p}, {}, P_NONE, g | G_KEEP);
    // Rayleigh-Ritz on {x, y, p}
    matvec(x, ax_.ptr);
    matvec(y, ay_.ptr);
    matvec(p, ap_.ptr);
    lc({x, y, p, ax_.ptr, ay_.ptr, ap_.ptr}, {}, {{0, 3}, {1, 4}, {2, 5}, {1, 3}, {2, 3}, {2, 4}},
       P_RR3, g);
    // s = k1 y + k2 p (virtual), |s|
    lc({x, y, p}, {nullptr}, {{100, 100}}, P_SNORM, g);
    // u -> x, t -> y (in place), norms
    lc({x, y, p}, {x, y}, {{100, 100}, {101, 101}}, P_XY_NORM, g);
    lc({x, y}, {x, y}, {}, orth.empty() ? P_SET_R_COEF : P_NONE, g);
    project_orth(orth, x, true, g);
    matvec(x, ax_.ptr);
    if (!orth.empty()) post_only(P_SET_R_COEF, g);
    if (orth.empty()) {
      lc({ax_.ptr, x}, {r}, {{100, 100}, {0, 0}}, P_CONV, g);
    } else {
      lc({ax_.ptr, x}, {r}, {{0, 0}}, P_STORE_AX, g);
      project_orth(orth, r, false, g);
      lc({r}, {}, {{0, 0}}, P_CONV_SPLIT, g);
    }
  }

  // ------------------------------------------------------ implicit-product variant (FP32)
  // Same Rayleigh-Ritz recurrence, but A x and A y are carried along as the same linear
  // combinations as x and y, so an iteration needs one matvec (A p).  Used for the FP32
  // sweeps of the mixed-precision solver; refresh() recomputes A x and A y to cancel drift.
  void start_implicit(const std::vector<const void*>& orth = {}) {
    R* x = x_.ptr;
    lc({x}, {}, {{0, 0}}, P_INV_NORM);
    lc({x}, {x}, {}, P_NONE);
    matvec(x, ax_.ptr);
    lc({ax_.ptr, x}, {}, {{1, 0}}, P_THETA0);
    lc({ax_.ptr, x}, {r_.ptr}, {{100, 100}}, P_R0NORM);
    read_host();
    if (host_->rzero) {
      SQD_CUDA(cudaMemsetAsync(y_.ptr, 0, sizeof(R) * NC * n_, st_));
      SQD_CUDA(cudaMemsetAsync(ay_.ptr, 0, sizeof(R) * NC * n_, st_));
      return;
    }
    lc({r_.ptr}, {p_.ptr}, {}, P_NONE);
    project_orth(orth, p_.ptr, false, G_NONE);
    matvec(p_.ptr, ap_.ptr);
    lc({x, p_.ptr, ax_.ptr, ap_.ptr}, {}, {{0, 2}, {1, 2}, {1, 3}}, P_RR2);
    lc({ax_.ptr, ap_.ptr}, {ay_.ptr, ax_.ptr}, {}, P_NONE);          // A t, A u
    lc({x, p_.ptr}, {y_.ptr, x}, {{100, 100}, {101, 101}}, P_TU_NORM);  // t, u
    lc({x, y_.ptr}, {x, y_.ptr}, {}, P_NONE);
    lc({ax_.ptr, ay_.ptr}, {ax_.ptr, ay_.ptr}, {}, P_SET_R_COEF);
    lc({ax_.ptr, x}, {r_.ptr}, {{100, 100}, {0, 0}}, P_CONV);
  }

  // First projection coefficients of the fast variant, from the current r, x, y.
  void proj_ips() { lc({r_.ptr, x_.ptr, y_.ptr}, {}, {{1, 0}, {2, 0}}, P_PROJ_IPS); }

  // Fast implicit iteration: 5 fused passes + 1 matvec.  p is projected out of {x, y} in two
  // rounds (the second unnormalised: its norm enters the Rayleigh-Ritz step analytically),
  // the Gram matrix of {x, y, p} comes from the carried A x, A y and the new A p, and
  // x, y, A x, A y, r and the next step's first projection coefficients are produced in two
  // passes.
  void body_fast(const std::vector<const void*>& orth) {
    R *x = x_.ptr, *y = y_.ptr, *r = r_.ptr, *p = p_.ptr;
    R *ax = ax_.ptr, *ay = ay_.ptr, *ap = ap_.ptr;
    const int g = G_DONE;
    lc({r, x, y}, {p}, {{100, 100}, {1, 100}, {2, 100}}, P_PROJ_NORM_IPS, g);
    lc({p, x, y}, {p}, {}, P_NONE, g);
    // Orthogonality constraints (excited states): the search direction leaves their span;
    // the Gram pass measures |p| afresh.
    project_orth(orth, p, false, g);
    matvec(p, ap);
    lc({x, y, p, ax, ay, ap}, {},
       {{0, 3}, {1, 4}, {2, 5}, {1, 3}, {2, 3}, {2, 4}, {2, 2}, {1, 2}}, P_GRAM_IMPLICIT, g);
    lc({x, y, p, ax, ay, ap}, {x, y, ax, ay}, {{100, 100}, {101, 101}}, P_UPDATE_NORMS, g);
    lc({x, y, ax, ay}, {x, y, ax, ay, r}, {{104, 104}, {102, 102}, {100, 104}, {101, 104}},
       P_CONV_PROJ, g);
  }

  // Recompute A x, A y and the residual explicitly; re-runs the convergence test.
  void refresh() {
    post_only(P_RESET);
    matvec(x_.ptr, ax_.ptr);
    matvec(y_.ptr, ay_.ptr);
    lc({ax_.ptr, x_.ptr}, {}, {{1, 0}}, P_THETA0);
    lc({ax_.ptr, x_.ptr}, {r_.ptr}, {{100, 100}, {0, 0}}, P_CONV);
    proj_ips();
    read_host();
  }

  // Reference iteration 0 plus the reference residual test (no iteration counted).
  void check0() {
    R* x = x_.ptr;
    lc({x}, {}, {{0, 0}}, P_INV_NORM);
    lc({x}, {x}, {}, P_NONE);
    matvec(x, ax_.ptr);
    lc({ax_.ptr, x}, {}, {{1, 0}}, P_THETA0);
    lc({ax_.ptr, x}, {r_.ptr}, {{100, 100}, {0, 0}}, P_CHECK0);
    read_host();
  }

  // Runs the while-loop.  use_graph: one CUDA graph with a conditional WHILE node.
  void loop(const std::vector<const void*>& orth, int maxiter, bool use_graph,
            bool fast = false) {
    read_host();
    if (maxiter <= 0 || host_->done) return;
    if (fast && use_graph && orth.empty() && persist_op_ != nullptr && persist_aligned()) {
      loop_persistent(maxiter);
      return;
    }
    auto run_body = [&] {
      if (fast) body_fast(orth);
      else body(orth);
    };
    if (!use_graph) {
      for (;;) {
        run_body();
        read_host();
        if (host_->done) break;
      }
      return;
    }
    const int v = fast ? 1 : 0;
    if (!exec_[v]) {
      // One graph per body variant, built on first use and relaunched afterwards: a conditional
      // WHILE node whose body is one iteration captured from a private stream (the legacy
      // default stream cannot be captured).
      SQD_CUDA(cudaGraphCreate(&graph_[v], 0));
      SQD_CUDA(cudaGraphConditionalHandleCreate(&cond_[v], graph_[v], 1,
                                                cudaGraphCondAssignDefault));
      cudaGraphNodeParams cp{};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = cond_[v];
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      cudaGraphNode_t node;
      SQD_CUDA(cudaGraphAddNode(&node, graph_[v], nullptr, 0, &cp));
      cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
      cudaStream_t cap = nullptr;
      SQD_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
      cur_ = cap;
      use_cond_ = 1;
      cond_cur_ = cond_[v];
      auto restore = [&] {
        cur_ = st_;
        use_cond_ = 0;
        cudaStreamDestroy(cap);
      };
      cudaError_t cerr = cudaStreamBeginCaptureToGraph(cap, bodyg, nullptr, nullptr, 0,
                                                       cudaStreamCaptureModeThreadLocal);
      if (cerr != cudaSuccess) {
        restore();
        SQD_CUDA(cerr);
      }
      try {
        run_body();
      } catch (...) {
        cudaGraph_t dummy;
        cudaStreamEndCapture(cap, &dummy);
        restore();
        throw;
      }
      cerr = cudaStreamEndCapture(cap, &bodyg);
      restore();
      SQD_CUDA(cerr);
      SQD_CUDA(cudaGraphInstantiate(&exec_[v], graph_[v], 0));
    }
    SQD_CUDA(cudaGraphLaunch(exec_[v], st_));
    read_host();
  }

  DevBuf<R> x_, y_, r_, p_, ax_, ay_, ap_, t0_;

 private:
  template <typename A>
  void fill(A& a, std::initializer_list<const void*> srcs, std::initializer_list<void*> outs,
            std::initializer_list<std::pair<int, int>> dots, int post, int gate) {
    a.n = n_;
    int k = 0;
    for (auto s : srcs) a.src[k++] = s;
    a.nsrc = k;
    k = 0;
    for (auto o : outs) a.out[k++] = o;
    a.nout = k;
    k = 0;
    for (auto d : dots) {
      a.da[k] = static_cast<signed char>(d.first);
      a.db[k] = static_cast<signed char>(d.second);
      ++k;
    }
    a.ndot = k;
    a.post = post;
    a.gate = gate;
    a.dev = dev_.ptr;
    a.partials = partials_.ptr;
    a.counter = counter_.ptr;
    a.use_cond = use_cond_;
    a.cond = cond_cur_;
  }
  // Variant for the orth projection: sources (v, o_0, ..., o_{m-1}).
  void lc_vec(const std::vector<const void*>& orth, void* v, std::vector<void*> outs,
              const std::vector<std::pair<int, int>>& dots, int post, int gate) {
    Orth a{};
    a.n = n_;
    a.src[0] = v;
    for (size_t k = 0; k < orth.size(); ++k) a.src[k + 1] = orth[k];
    a.nsrc = static_cast<int>(orth.size() + 1);
    a.nout = static_cast<int>(outs.size());
    for (size_t k = 0; k < outs.size(); ++k) a.out[k] = outs[k];
    a.ndot = static_cast<int>(dots.size());
    for (size_t k = 0; k < dots.size(); ++k) {
      a.da[k] = static_cast<signed char>(dots[k].first);
      a.db[k] = static_cast<signed char>(dots[k].second);
    }
    a.post = post;
    a.gate = gate;
    a.dev = dev_.ptr;
    a.partials = partials_.ptr;
    a.counter = counter_.ptr;
    a.use_cond = use_cond_;
    a.cond = cond_cur_;
    k_lc<R, NC, kMaxOrth + 1, kMaxOrth, 2><<<blocks_, LC_THREADS, 0, cur_>>>(a);
    SQD_CHECK_LAUNCH();
  }
  static std::string last_msg() {
    const char* m = sqd_last_error();
    return m ? m : "";
  }

 public:
  // The fast iteration may run as one persistent launch (k_locg_persist) when the matvec is
  // this cached operator's CSR kernel; nullptr keeps the graph form.
  void set_persistent_op(sqd_op_s* op) { persist_op_ = op; }
  // The persistent passes move 16 bytes of every vector per thread step.
  bool persist_aligned() const {
    const R* vecs[] = {x_.ptr, y_.ptr, r_.ptr, p_.ptr, ax_.ptr, ay_.ptr, ap_.ptr};
    for (const R* v : vecs)
      if (reinterpret_cast<uintptr_t>(v) % 16 != 0) return false;
    return true;
  }

 private:
  // Small vectors (at most kClusterMax blocks' worth): the grid is one thread-block cluster,
  // synchronised by the hardware cluster barrier with the partials exchanged through
  // distributed shared memory.  Larger: a cooperative launch with the bounded grid barrier.
  static constexpr int kClusterMax = 16;

  template <int NCA, int LPR>
  void launch_persistent(PersistArgs& pa) {
    const int64_t want = (n_ + LC_THREADS - 1) / LC_THREADS;
    if (persist_grid_ == 0) {
      if (want <= kClusterMax) {
        persist_cluster_ = true;
        persist_grid_ = static_cast<unsigned>(std::max<int64_t>(1, want));
      } else {
        int per_sm = 0;
        SQD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, k_locg_persist<R, NC, NCA, LPR, false>, LC_THREADS, 0));
        if (const char* e = std::getenv("SQD_LOCG_PERSIST_BLOCKS"))   // per SM (tuning)
          per_sm = std::min(per_sm, std::max(1, std::atoi(e)));
        const int64_t cap = static_cast<int64_t>(std::max(per_sm, 1)) * num_sms();
        persist_grid_ = static_cast<unsigned>(std::max<int64_t>(1, std::min(want, cap)));
      }
      ppart_.alloc(static_cast<size_t>(persist_grid_) * 20 + 20, st_);
      bar_.alloc(4, st_);
    }
    pa.partials = ppart_.ptr;
    pa.red = ppart_.ptr + static_cast<size_t>(persist_grid_) * 20;
    pa.bar = bar_.ptr;
    SQD_CUDA(cudaMemsetAsync(bar_.ptr, 0, 4 * sizeof(unsigned), st_));
    if (persist_cluster_) {
      auto kern = k_locg_persist<R, NC, NCA, LPR, true>;
      if (persist_grid_ > 8)
        SQD_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = dim3(persist_grid_);
      cfg.blockDim = dim3(LC_THREADS);
      cfg.stream = st_;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = persist_grid_;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      SQD_CUDA(cudaLaunchKernelEx(&cfg, kern, pa));
    } else {
      auto kern = k_locg_persist<R, NC, NCA, LPR, false>;
      void* args[] = {&pa};
      SQD_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kern), persist_grid_,
                                           LC_THREADS, args, 0, st_));
    }
  }

  // loop(fast) as one cooperative launch: the body_fast passes and the CSR matvec, phases
  // separated by grid barriers, until the convergence step sets `done`.
  void loop_persistent(int maxiter) {
    sqd_op_s* op = persist_op_;
    R *x = x_.ptr, *y = y_.ptr, *r = r_.ptr, *p = p_.ptr;
    R *ax = ax_.ptr, *ay = ay_.ptr, *ap = ap_.ptr;
    PersistArgs pa{};
    fill(pa.ps[0], {r, x, y}, {p}, {{100, 100}, {1, 100}, {2, 100}}, P_PROJ_NORM_IPS, G_NONE);
    fill(pa.ps[2], {x, y, p, ax, ay, ap}, {},
         {{0, 3}, {1, 4}, {2, 5}, {1, 3}, {2, 3}, {2, 4}, {2, 2}, {1, 2}}, P_GRAM_IMPLICIT,
         G_NONE);
    // update pass (PShapeU): unnormalised u, t, A u, A t, r'; the kernel applies the norms
    fill(pa.ps[3], {x, y, p, ax, ay, ap}, {x, y, ax, ay, r},
         {{100, 100}, {101, 101}, {104, 104}, {102, 102}, {100, 104}, {101, 104}}, P_NONE,
         G_NONE);
    pa.row_ptr = op->row_ptr.ptr;
    pa.cols = op->cols.ptr;
    if constexpr (sizeof(R) == 8) pa.vals = op->values.ptr;
    else pa.vals = op->values32.ptr;
    pa.mv_in = p;
    pa.mv_out = ap;
    pa.n = n_;
    pa.dev = dev_.ptr;
    pa.max_iter = maxiter + 1;
    // Lanes per row from the mean row length, not the standalone matvec's tuned value: inside
    // the persistent launch the grid is small and a row's lanes should not exceed its pairs.
    const double avg = n_ > 0 ? static_cast<double>(op->nnz) / static_cast<double>(n_) : 0.0;
    const int lpr = avg >= 96 ? 32 : avg >= 40 ? 16 : avg >= 16 ? 8 : avg >= 6 ? 4
                  : avg >= 2 ? 2 : 1;
    const auto t_launch = std::chrono::steady_clock::now();
    dispatch_lpr(lpr, [&](auto lpr_t) {
      constexpr int LPR = decltype(lpr_t)::value;
      if constexpr (NC == 2) {
        if (op->value_complex) launch_persistent<2, LPR>(pa);
        else launch_persistent<1, LPR>(pa);
      } else {
        launch_persistent<1, LPR>(pa);
      }
    });
    read_host();
    unsigned fault = 0;
    SQD_CUDA(cudaMemcpyAsync(&fault, bar_.ptr + 2, sizeof(unsigned), cudaMemcpyDeviceToHost,
                             st_));
    SQD_CUDA(cudaStreamSynchronize(st_));
    if (std::getenv("SQD_LOCG_TRACE"))
      std::fprintf(stderr, "[sqd_locg persistent] %s, %u blocks (%s), %d iterations, %.3f ms\n",
                   sizeof(R) == 4 ? "fp32" : "fp64", persist_grid_,
                   persist_cluster_ ? "cluster" : "cooperative", host_->niter,
                   std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() -
                                                             t_launch).count());
    if (fault)
      throw Error(SQD_ERR_DEVICE, "persistent LOCG iteration: a grid barrier timed out");
  }

  int64_t n_;
  sqd_matvec_fn fn_;
  void* ctx_;
  cudaStream_t st_;
  cudaStream_t cur_;  // launch stream: st_, or the private capture stream while capturing
  double* hist_ = nullptr;
  int hist_cap_ = 0;
  int hist_phase_ = 0;
  sqd_op_s* persist_op_ = nullptr;
  unsigned persist_grid_ = 0;
  bool persist_cluster_ = false;
  DevBuf<double> ppart_;
  DevBuf<unsigned> bar_;
  unsigned blocks_ = 1;
  DevBuf<double> partials_;
  DevBuf<unsigned> counter_;
  DevBuf<LocgDev> dev_;
  LocgDev* host_ = nullptr;
  int use_cond_ = 0;
  cudaGraphConditionalHandle cond_cur_ = 0;
  cudaGraphConditionalHandle cond_[2] = {0, 0};
  cudaGraph_t graph_[2] = {nullptr, nullptr};
  cudaGraphExec_t exec_[2] = {nullptr, nullptr};
};

// Matvec adapter for the FP32 phase of the mixed solver.
struct OpCtx32 {
  sqd_op_s* op;
  int dtype;
};
int op_cb32(void* ctx, const void* x, void* y, void* stream) {
  auto* c = static_cast<OpCtx32*>(ctx);
  return guarded([&] { op_matvec(c->op, x, y, c->dtype, as_stream(stream)); });
}
struct OpCtx64 {
  sqd_op_s* op;
  int dtype;
};
int op_cb64(void* ctx, const void* x, void* y, void* stream) {
  auto* c = static_cast<OpCtx64*>(ctx);
  return guarded([&] { op_matvec(c->op, x, y, c->dtype, as_stream(stream)); });
}

// Solver objects kept on the operator between solves: the work vectors and the instantiated
// graphs of the iteration loops are reused instead of allocated and captured again (the first
// FP64 phase after the FP32 sweeps otherwise waits for the pool to map 8 new vectors).
// Valid while n, the vector kind and the operator's matvec schedule stay the same; only solves
// without orthogonality constraints use it (a captured graph holds the constraint vectors).
template <int NC>
struct SolverCache final : LocgCacheBase {
  int64_t n = 0;
  uint64_t version = 0;
  OpCtx32 c32{};
  OpCtx64 c64{};
  std::unique_ptr<Locg<float, NC>> l32;
  std::unique_ptr<Locg<double, NC>> l64;
};

template <int NC>
SolverCache<NC>* solver_cache(sqd_op_s* op, int64_t n) {
  auto* c = dynamic_cast<SolverCache<NC>*>(op->locg_cache.get());
  if (!c || c->n != n || c->version != op->schedule_version) {
    op->locg_cache.reset();  // frees the stale objects first
    auto fresh = std::make_unique<SolverCache<NC>>();
    fresh->n = n;
    fresh->version = op->schedule_version;
    fresh->c32 = OpCtx32{op, NC == 2 ? SQD_C64 : SQD_F32};
    fresh->c64 = OpCtx64{op, NC == 2 ? SQD_C128 : SQD_F64};
    c = fresh.get();
    op->locg_cache = std::move(fresh);
  }
  return c;
}

// Iteration record requested by sqd_locg_record for the next sqd_locg call on this thread.
struct HistRequest {
  double* rows_host = nullptr;
  int64_t max_rows = 0;
  int64_t* count_host = nullptr;
};
thread_local HistRequest g_hist_request;

// Device rows for one solver object; copied to the caller's host rows after the solve.
struct HistRecorder {
  HistRequest req;
  DevBuf<double> rows[2];   // [0] FP64, [1] FP32
  void arm(int phase, cudaStream_t st) {
    rows[phase].alloc(static_cast<size_t>(req.max_rows) * kHistCols, st);
  }
  // Copies FP32 rows (they come first in time) then FP64 rows, up to max_rows in total.
  template <class L64, class L32>
  void finish(L64* l64, L32* l32, cudaStream_t st) {
    int64_t written = 0;
    auto take = [&](auto* l, int phase) {
      if (!l || !rows[phase].ptr) return;
      l->read_host();
      const int64_t n = std::min<int64_t>(l->host().hist_n, req.max_rows - written);
      if (n > 0)
        SQD_CUDA(cudaMemcpyAsync(req.rows_host + written * kHistCols, rows[phase].ptr,
                                 sizeof(double) * kHistCols * n, cudaMemcpyDeviceToHost, st));
      written += std::max<int64_t>(n, 0);
      l->set_history(nullptr, 0, 0);
    };
    take(l32, 1);
    take(l64, 0);
    SQD_CUDA(cudaStreamSynchronize(st));
    if (req.count_host) *req.count_host = written;
  }
};

// cache_op: the sqd operator behind fn (NULL for a caller's own matvec), whose solver cache
// the FP64 path may use.
template <int NC>
void run_locg(int64_t n, int dtype, sqd_matvec_fn fn, void* ctx, sqd_op_s* cache_op,
              const void* xinit, int64_t xinit_index, const std::vector<const void*>& orth,
              double tol, int maxiter, int mode, bool use_graph, cudaStream_t st,
              double* eigval, void* eigvec, int* niter, double* residual) {
  const double eps64 = 2.220446049250313e-16;
  const double nscale = 10.0 * static_cast<double>(n);
  const unsigned G = grid_for(n, 256, 8192);
  if (mode == SQD_LOCG_FP64) {
    std::unique_ptr<Locg<double, NC>> own;
    Locg<double, NC>* lp = nullptr;
    if (cache_op && orth.empty()) {
      auto* cache = solver_cache<NC>(cache_op, n);
      if (!cache->l64) cache->l64 = std::make_unique<Locg<double, NC>>(n, op_cb64, &cache->c64, st);
      lp = cache->l64.get();
      lp->set_stream(st);
    } else {
      own = std::make_unique<Locg<double, NC>>(n, fn, ctx, st);
      lp = own.get();
    }
    Locg<double, NC>& L = *lp;
    HistRecorder rec{g_hist_request};
    g_hist_request = HistRequest{};
    if (rec.req.rows_host) rec.arm(0, st);
    // always set: a cached solver must not keep a previous solve's (freed) record buffer
    L.set_history(rec.rows[0].ptr, static_cast<int>(rec.req.max_rows), 0);
    L.set_params(tol < 0 ? eps64 : tol, nscale, maxiter, 0.0, 0.0, 0);
    if (xinit)
      SQD_CUDA(cudaMemcpyAsync(L.x(), xinit, sizeof(double) * NC * n, cudaMemcpyDeviceToDevice,
                               st));
    else
      k_onehot<double, NC><<<G, 256, 0, st>>>(L.x(), n, xinit_index);
    SQD_CHECK_LAUNCH();
    if (!xinit) L.project_orth(orth, L.x(), true, G_NONE);
    L.start(orth);
    L.loop(orth, maxiter, use_graph);
    const LocgDev& h = L.host();
    *eigval = h.theta;
    *niter = h.niter;
    if (residual) *residual = h.rnorm;
    SQD_CUDA(cudaMemcpyAsync(eigvec, L.x(), sizeof(double) * NC * n, cudaMemcpyDeviceToDevice,
                             st));
    SQD_CUDA(cudaStreamSynchronize(st));
    if (rec.req.rows_host) rec.finish(&L, static_cast<Locg<float, NC>*>(nullptr), st);
    return;
  }
  // Mixed precision.
  //  1. FP32 sweeps: complex64/f32 vectors, FP32 matrix elements with the compensated matvec,
  //     FP64 inner products, implicit products (one matvec per iteration), until
  //     |r| < kInnerRtol |theta| or the residual stops improving; A x and A y are then
  //     recomputed explicitly and the test repeated (restarts cancel recurrence drift).
  //  2. FP64 check: the vector is promoted, A x, theta and r are recomputed in FP64 and the
  //     reference's residual test (ground_locg.py:371-376) is applied.
  //  3. Only if it fails: FP64 iterations of the reference algorithm from that vector.
  SQD_REQUIRE(fn == sqd_op_matvec_cb, "mixed precision needs an sqd operator as the matvec");
  auto* op = static_cast<sqd_op_s*>(ctx);
  op_ensure_values32(op, st);
  // Orthogonality constraints (excited states): FP32 copies for the sweeps, fresh solver
  // objects (a cached graph would hold the vectors).
  std::vector<DevBuf<float>> orth32_bufs;
  std::vector<const void*> orth32;
  for (const void* o : orth) {
    DevBuf<float> b;
    b.alloc(static_cast<size_t>(n) * NC, st);
    k_convert<float, double, NC><<<G, 256, 0, st>>>(static_cast<const double*>(o), b.ptr, n);
    SQD_CHECK_LAUNCH();
    orth32.push_back(b.ptr);
    orth32_bufs.push_back(std::move(b));
  }
  OpCtx32 own_c32{op, NC == 2 ? SQD_C64 : SQD_F32};
  OpCtx64 own_c64{op, NC == 2 ? SQD_C128 : SQD_F64};
  std::unique_ptr<Locg<float, NC>> own32;
  std::unique_ptr<Locg<double, NC>> own64;
  Locg<float, NC>* l32 = nullptr;
  Locg<double, NC>* l64 = nullptr;
  if (orth.empty()) {
    SolverCache<NC>* cache = solver_cache<NC>(op, n);
    if (!cache->l64) cache->l64 = std::make_unique<Locg<double, NC>>(n, op_cb64, &cache->c64, st);
    if (!cache->l32) cache->l32 = std::make_unique<Locg<float, NC>>(n, op_cb32, &cache->c32, st);
    l32 = cache->l32.get();
    l64 = cache->l64.get();
  } else {
    own64 = std::make_unique<Locg<double, NC>>(n, op_cb64, &own_c64, st);
    own32 = std::make_unique<Locg<float, NC>>(n, op_cb32, &own_c32, st);
    l32 = own32.get();
    l64 = own64.get();
  }
  // Phase timing on stderr when SQD_LOCG_TRACE is set (like the reference's debug prints).
  const bool trace = std::getenv("SQD_LOCG_TRACE") != nullptr;
  cudaEvent_t ev[5] = {};
  if (trace)
    for (auto& e : ev) SQD_CUDA(cudaEventCreate(&e));
  // host clock at each mark too: a wait outside this stream's work shows as a gap between the
  // two clocks
  std::chrono::steady_clock::time_point th[5];
  auto mark = [&](int k) {
    if (trace) {
      SQD_CUDA(cudaEventRecord(ev[k], st));
      th[k] = std::chrono::steady_clock::now();
    }
  };
  mark(0);
  constexpr double kInnerRtol = 2e-7;
  constexpr int kStall = 25;
  constexpr int kRestarts = 6;
  int it32 = 0;
  Locg<double, NC>& L = *l64;
  L.set_stream(st);
  HistRecorder rec{g_hist_request};
  g_hist_request = HistRequest{};
  if (rec.req.rows_host) {
    rec.arm(0, st);
    rec.arm(1, st);
  }
  // always set: a cached solver must not keep a previous solve's (freed) record buffer
  L.set_history(rec.rows[0].ptr, static_cast<int>(rec.req.max_rows), 0);
  l32->set_history(rec.rows[1].ptr, static_cast<int>(rec.req.max_rows), 1);
  // Persistent iterations (one cooperative launch per loop) where the matvec is the cached
  // CSR kernel and the operator is small enough that launch latency, not bandwidth, bounds the
  // graph form: up to 4 Mi rows and 64 Mi stored pairs (a large matvec runs better as its own
  // kernel at full occupancy).  SQD_LOCG_PERSISTENT=0 disables, =1 forces.
  {
    const char* env = std::getenv("SQD_LOCG_PERSISTENT");
    const bool on = env ? std::atoi(env) != 0
                        : n <= (int64_t(4) << 20) && op->nnz <= (int64_t(64) << 20);
    auto csr = [&](int prec) {
      return op->x_cache == 1 && op->z_cache == 2 &&
             (!op->prod.built || op->layout[prec] == SQD_LAYOUT_CSR);
    };
    l32->set_persistent_op(on && csr(1) ? op : nullptr);
    L.set_persistent_op(on && csr(0) ? op : nullptr);
  }
  {
    Locg<float, NC>& L32 = *l32;
    L32.set_stream(st);
    L32.set_params(0.0, nscale, maxiter, kInnerRtol, 0.0, kStall);
    if (xinit) {
      k_convert<float, double, NC><<<G, 256, 0, st>>>(static_cast<const double*>(xinit),
                                                     L32.x(), n);
    } else {
      k_onehot<float, NC><<<G, 256, 0, st>>>(L32.x(), n, xinit_index);
    }
    SQD_CHECK_LAUNCH();
    if (!xinit) L32.project_orth(orth32, L32.x(), true, G_NONE);
    L32.start_implicit(orth32);
    L32.proj_ips();
    for (int k = 0; k < kRestarts; ++k) {
      L32.loop(orth32, maxiter, use_graph, true);
      if (L32.host().niter >= maxiter || L32.host().rzero) break;
      L32.refresh();
      if (L32.host().converged || L32.host().niter >= maxiter) break;
    }
    it32 = L32.host().niter;
    k_convert<double, float, NC><<<G, 256, 0, st>>>(L32.x(), L.x(), n);
    SQD_CHECK_LAUNCH();
    mark(1);
  }
  mark(2);
  const int left = std::max(1, maxiter - it32);
  L.set_params(tol < 0 ? eps64 : tol, nscale, left, 0.0, 0.0, 0);
  if (orth.empty()) {
    // FP64 polish: fast implicit iterations (one FP64 matvec each) with the reference's
    // residual test; in FP64 the carried products drift by O(eps) only.
    L.start_implicit();
    L.proj_ips();
    mark(3);
    L.loop(orth, left, use_graph, true);
  } else {
    // With constraints: the reference iteration from the FP32 vector, which projects every
    // residual against the constraint vectors in FP64.
    L.start(orth);
    mark(3);
    L.loop(orth, left, use_graph);
  }
  const int it64 = L.host().niter;
  mark(4);
  if (trace) {
    SQD_CUDA(cudaEventSynchronize(ev[4]));
    float t[4];
    for (int k = 0; k < 4; ++k) SQD_CUDA(cudaEventElapsedTime(&t[k], ev[k], ev[k + 1]));
    auto ms = [](std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
      return std::chrono::duration<double, std::milli>(b - a).count();
    };
    std::fprintf(stderr,
                 "[sqd_locg mixed] fp32 sweeps %d it %.3f ms | phase switch %.3f ms | "
                 "fp64 start %.3f ms | fp64 iterations %d it %.3f ms | host %.3f %.3f %.3f "
                 "%.3f ms\n",
                 it32, t[0], t[1], t[2], it64, t[3], ms(th[0], th[1]), ms(th[1], th[2]),
                 ms(th[2], th[3]), ms(th[3], th[4]));
    for (auto& e : ev) cudaEventDestroy(e);
  }
  const LocgDev& h = L.host();
  *eigval = h.theta;
  *niter = it32 + it64;
  if (residual) *residual = h.rnorm;
  SQD_CUDA(cudaMemcpyAsync(eigvec, L.x(), sizeof(double) * NC * n, cudaMemcpyDeviceToDevice,
                           st));
  SQD_CUDA(cudaStreamSynchronize(st));
  if (rec.req.rows_host) rec.finish(&L, l32, st);
}

}  // namespace
}  // namespace sqd

// ============================================================================================
// Batched instances: many independent operators solved together.
//
// The instances' stored pairs are concatenated into one block-diagonal CSR.  Rows are cut
// into tiles that never cross an instance boundary; every kernel walks the tile list (a
// per-instance work queue) and skips the tiles of instances that have converged.  Inner
// products are reduced per tile and then per instance (one warp per instance, tiles in fixed
// order, so results are deterministic), after which that warp runs the instance's scalar step
// (Rayleigh-Ritz, normalisations, convergence) on its own coefficient bank.  A whole batched
// iteration is one CUDA graph body; the WHILE condition is "some instance still active".
// ============================================================================================
struct sqd_batch_s {
  int n = 0;
  int value_complex = 0;
  int64_t total_rows = 0;
  int64_t total_nnz = 0;
  std::vector<int64_t> row0;          // host [n + 1]
  sqd::DevBuf<int64_t> row_ptr;       // [total_rows + 1]
  sqd::DevBuf<uint32_t> cols;         // [total_nnz] global source rows
  sqd::DevBuf<double> values;         // [total_nnz * nca]
  sqd::DevBuf<float> values32;        // FP32 copy
  int n_tiles = 0;
  sqd::DevBuf<int32_t> tile_inst;     // [n_tiles]
  sqd::DevBuf<int64_t> tile_row0;     // [n_tiles + 1]
  std::vector<int32_t> inst_tile0;    // host [n + 1]
  sqd::DevBuf<int32_t> inst_tile0_d;  // [n + 1]
  int lanes[2] = {8, 8};
};

namespace sqd {
namespace {

constexpr int64_t kTileRows = 2048;

template <typename R, int NCV, int NCA, int LPR>
__global__ void __launch_bounds__(256)
k_bmv_csr(const int64_t* __restrict__ row_ptr, const uint32_t* __restrict__ cols,
          const R* __restrict__ vals, const R* __restrict__ v, R* __restrict__ out,
          const int32_t* __restrict__ tile_inst, const int64_t* __restrict__ tile_row0,
          int n_tiles, const LocgDev* dev) {
  constexpr int RPW = 32 / LPR;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sub = lane % LPR, slot = lane / LPR;
  const int nwarps = blockDim.x >> 5;
  for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    if (*(volatile const int*)&dev[tile_inst[t]].done) continue;
    const int64_t r0 = tile_row0[t], r1 = tile_row0[t + 1];
    for (int64_t rb = r0 + int64_t(warp) * RPW; rb < r1; rb += int64_t(nwarps) * RPW) {
      const int64_t row = rb + slot;
      CAcc<R, NCV, NCA> acc;
      if (row < r1) {
        const int64_t b = __ldg(row_ptr + row), e = __ldg(row_ptr + row + 1);
        csr_row_dot<R, NCV, NCA, LPR>(cols, vals, v, b + sub, e, acc);
      }
      acc.merge(LPR);
      if (sub == 0 && row < r1)
        st_elem<R, NCV>(out, row, cx_make<R>(acc.re.value(), acc.im.value()));
    }
  }
}

template <int MAXS, int MAXD, int MAXO>
struct BLCArgs {
  const void* src[MAXS];
  void* out[MAXO];
  int nsrc, nout, ndot, gate;
  signed char da[MAXD], db[MAXD];
  LocgDev* dev;
  double* partials;
  const int32_t* tile_inst;
  const int64_t* tile_row0;
  int n_tiles;
};

template <typename R, int NC, int MAXS, int MAXD, int MAXO>
__global__ void __launch_bounds__(LC_THREADS) k_blc(BLCArgs<MAXS, MAXD, MAXO> a) {
  __shared__ double2 sc[MAXO][MAXS];
  __shared__ double sred[MAXD * 2][LC_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int t = blockIdx.x; t < a.n_tiles; t += gridDim.x) {
    const LocgDev* dev = a.dev + a.tile_inst[t];
    __syncthreads();
    const bool skip = ((a.gate & G_DONE) && *(volatile const int*)&dev->done) ||
                      ((a.gate & G_KEEP) && *(volatile const int*)&dev->keep);
    if (skip) {
      if (threadIdx.x < 2 * a.ndot)
        a.partials[static_cast<int64_t>(t) * (2 * MAXD) + threadIdx.x] = 0.0;
      continue;
    }
    for (int q = threadIdx.x; q < MAXO * MAXS; q += blockDim.x)
      sc[q / MAXS][q % MAXS] = make_double2(dev->coef[q / MAXS][q % MAXS][0],
                                            dev->coef[q / MAXS][q % MAXS][1]);
    __syncthreads();
    double acc[MAXD][2];
#pragma unroll
    for (int d = 0; d < MAXD; ++d) acc[d][0] = acc[d][1] = 0.0;
    const int64_t e = a.tile_row0[t + 1];
    for (int64_t i = a.tile_row0[t] + threadIdx.x; i < e; i += blockDim.x) {
      double2 s[MAXS];
#pragma unroll
      for (int k = 0; k < MAXS; ++k) {
        s[k] = make_double2(0.0, 0.0);
        if (k < a.nsrc) {
          const Cx<R> v = ld_elem_rw<R, NC>(static_cast<const R*>(a.src[k]), i);
          s[k] = make_double2(double(v.re), double(v.im));
        }
      }
      double2 o[MAXO];
#pragma unroll
      for (int q = 0; q < MAXO; ++q) {
        o[q] = make_double2(0.0, 0.0);
        if (q < a.nout) {
#pragma unroll
          for (int k = 0; k < MAXS; ++k)
            if (k < a.nsrc) o[q] = cadd(o[q], cmul(sc[q][k], s[k]));
          if constexpr (NC == 1) o[q].y = 0.0;
        }
      }
#pragma unroll
      for (int d = 0; d < MAXD; ++d) {
        if (d < a.ndot) {
          double2 x = make_double2(0.0, 0.0), y = make_double2(0.0, 0.0);
          const int ca = a.da[d], cb = a.db[d];
#pragma unroll
          for (int k = 0; k < MAXS; ++k) {
            if (ca == k) x = s[k];
            if (cb == k) y = s[k];
          }
#pragma unroll
          for (int q = 0; q < MAXO; ++q) {
            if (ca == 100 + q) x = o[q];
            if (cb == 100 + q) y = o[q];
          }
          acc[d][0] += x.x * y.x + x.y * y.y;
          acc[d][1] += x.x * y.y - x.y * y.x;
        }
      }
#pragma unroll
      for (int q = 0; q < MAXO; ++q)
        if (q < a.nout && a.out[q] != nullptr)
          st_elem<R, NC>(static_cast<R*>(a.out[q]), i, cx_make<R>(R(o[q].x), R(o[q].y)));
    }
    if (a.ndot > 0) {
#pragma unroll
      for (int d = 0; d < MAXD; ++d) {
        if (d < a.ndot) {
          const double v0 = warp_sum(acc[d][0]);
          const double v1 = warp_sum(acc[d][1]);
          if (lane == 0) {
            sred[2 * d][warp] = v0;
            sred[2 * d + 1][warp] = v1;
          }
        }
      }
      __syncthreads();
      if (threadIdx.x < 2 * a.ndot) {
        double v = 0.0;
        for (int w = 0; w < LC_THREADS / 32; ++w) v += sred[threadIdx.x][w];
        a.partials[static_cast<int64_t>(t) * (2 * MAXD) + threadIdx.x] = v;
      }
    }
  }
}

// One warp per instance: sum its tiles' partials in order, then run its scalar step.
__global__ void k_bpost(const double* partials, int stride, const int32_t* inst_tile0, int n,
                        LocgDev* dev, int ndot, int nsrc, int post, int gate) {
  const int inst = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (inst >= n) return;
  LocgDev* d = dev + inst;
  if ((gate & G_DONE) && d->done) return;
  if (lane < 2 * ndot) {
    double v = 0.0;
    for (int t = inst_tile0[inst]; t < inst_tile0[inst + 1]; ++t)
      v += partials[static_cast<int64_t>(t) * stride + lane];
    d->red[lane >> 1][lane & 1] = v;
  }
  __syncwarp();
  if (lane == 0) run_post(d, post, nsrc, 0, 0);
}

// Counts the active instances and sets the WHILE condition.
__global__ void k_bactive(const LocgDev* dev, int n, int use_cond,
                          cudaGraphConditionalHandle cond, int* active) {
  __shared__ int cnt;
  if (threadIdx.x == 0) cnt = 0;
  __syncthreads();
  int c = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) c += dev[i].done ? 0 : 1;
  atomicAdd(&cnt, c);
  __syncthreads();
  if (threadIdx.x == 0) {
    *active = cnt;
    if (use_cond) cudaGraphSetConditional(cond, cnt > 0 ? 1u : 0u);
  }
}

template <typename R, int NC>
__global__ void k_bonehot(R* x, const int32_t* tile_inst, const int64_t* tile_row0, int n_tiles,
                          const int64_t* row0, const int64_t* idx) {
  for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
    const int inst = tile_inst[t];
    const int64_t hot = row0[inst] + idx[inst];
    for (int64_t i = tile_row0[t] + threadIdx.x; i < tile_row0[t + 1]; i += blockDim.x)
      st_elem<R, NC>(x, i, cx_make<R>(R(i == hot ? 1 : 0), R(0)));
  }
}

template <typename R, int NC>
class BLocg {
 public:
  using Tiny = BLCArgs<3, 3, 2>;
  using Wide = BLCArgs<6, 10, 5>;

  BLocg(sqd_batch_s* b, cudaStream_t st) : b_(b), st_(st), cur_(st) {
    const int64_t n = b->total_rows;
    for (auto* v : {&x_, &y_, &r_, &p_, &ax_, &ay_, &ap_}) v->alloc(static_cast<size_t>(n) * NC, st);
    dev_.alloc(b->n, st);
    partials_.alloc(static_cast<size_t>(b->n_tiles) * 20, st);
    active_.alloc(1, st);
    SQD_CUDA(cudaMemsetAsync(dev_.ptr, 0, sizeof(LocgDev) * b->n, st));
    SQD_CUDA(cudaMallocHost(reinterpret_cast<void**>(&host_), sizeof(LocgDev) * b->n));
    blocks_ = static_cast<unsigned>(std::max(1, std::min(b->n_tiles, 8 * num_sms())));
  }
  ~BLocg() {
    if (exec_) cudaGraphExecDestroy(exec_);
    if (graph_) cudaGraphDestroy(graph_);
    if (host_) cudaFreeHost(host_);
  }
  R* x() { return x_.ptr; }
  const LocgDev& host(int i) const { return host_[i]; }

  void set_params(double tol, int maxiter, double inner_rtol, double etol, int stall) {
    std::vector<LocgDev> h(b_->n);
    for (int i = 0; i < b_->n; ++i) {
      h[i] = LocgDev{};
      h[i].tol = tol;
      h[i].nscale = 10.0 * static_cast<double>(b_->row0[i + 1] - b_->row0[i]);
      h[i].maxiter = maxiter;
      h[i].inner_rtol = inner_rtol;
      h[i].etol = etol;
      h[i].stall = stall;
      h[i].best_r = 1e300;
    }
    SQD_CUDA(cudaMemcpyAsync(dev_.ptr, h.data(), sizeof(LocgDev) * b_->n,
                             cudaMemcpyHostToDevice, st_));
    SQD_CUDA(cudaStreamSynchronize(st_));
  }

  void lc(std::initializer_list<const void*> srcs, std::initializer_list<void*> outs,
          std::initializer_list<std::pair<int, int>> dots, int post, int gate = G_NONE) {
    if (srcs.size() <= 3 && dots.size() <= 3 && outs.size() <= 2) {
      Tiny a{};
      fill(a, srcs, outs, dots, gate);
      if (srcs.size() > 0) k_blc<R, NC, 3, 3, 2><<<blocks_, LC_THREADS, 0, cur_>>>(a);
      SQD_CHECK_LAUNCH();
      posts(a.nsrc, static_cast<int>(dots.size()), 6, post, gate);
    } else {
      SQD_REQUIRE(srcs.size() <= 6 && dots.size() <= 10 && outs.size() <= 5, "pass too wide");
      Wide a{};
      fill(a, srcs, outs, dots, gate);
      k_blc<R, NC, 6, 10, 5><<<blocks_, LC_THREADS, 0, cur_>>>(a);
      SQD_CHECK_LAUNCH();
      posts(a.nsrc, static_cast<int>(dots.size()), 20, post, gate);
    }
  }
  void post_only(int post, int gate = G_NONE) { posts(0, 0, 6, post, gate); }

  void matvec(const R* in, R* out) {
    const int prec = sizeof(R) == 8 ? 0 : 1;
    const R* vals;
    if constexpr (sizeof(R) == 8) vals = b_->values.ptr;
    else vals = b_->values32.ptr;
    auto launch = [&](auto nca_t) {
      constexpr int NCA = decltype(nca_t)::value;
      dispatch_lpr(b_->lanes[prec], [&](auto lpr_t) {
        constexpr int LPR = decltype(lpr_t)::value;
        const unsigned G = static_cast<unsigned>(std::max(1, std::min(b_->n_tiles, 16 * num_sms())));
        k_bmv_csr<R, NC, NCA, LPR><<<G, 256, 0, cur_>>>(b_->row_ptr.ptr, b_->cols.ptr, vals, in,
                                                        out, b_->tile_inst.ptr,
                                                        b_->tile_row0.ptr, b_->n_tiles, dev_.ptr);
      });
    };
    if constexpr (NC == 2) {
      if (b_->value_complex) launch(IntTag<2>{});
      else launch(IntTag<1>{});
    } else {
      launch(IntTag<1>{});
    }
    SQD_CHECK_LAUNCH();
  }

  void read_host() {
    SQD_CUDA(cudaMemcpyAsync(host_, dev_.ptr, sizeof(LocgDev) * b_->n, cudaMemcpyDeviceToHost,
                             st_));
    SQD_CUDA(cudaStreamSynchronize(st_));
  }
  int active() {
    int h = 0;
    k_bactive<<<1, 256, 0, st_>>>(dev_.ptr, b_->n, 0, 0, active_.ptr);
    SQD_CHECK_LAUNCH();
    copy_to_host(&h, active_.ptr, 1, st_);
    return h;
  }

  void onehot(const int64_t* idx_host) {
    DevBuf<int64_t> row0, idx;
    row0.alloc(b_->n + 1, st_);
    idx.alloc(b_->n, st_);
    SQD_CUDA(cudaMemcpyAsync(row0.ptr, b_->row0.data(), sizeof(int64_t) * (b_->n + 1),
                             cudaMemcpyHostToDevice, st_));
    SQD_CUDA(cudaMemcpyAsync(idx.ptr, idx_host, sizeof(int64_t) * b_->n, cudaMemcpyHostToDevice,
                             st_));
    k_bonehot<R, NC><<<blocks_, 256, 0, st_>>>(x_.ptr, b_->tile_inst.ptr, b_->tile_row0.ptr,
                                               b_->n_tiles, row0.ptr, idx.ptr);
    SQD_CHECK_LAUNCH();
    SQD_CUDA(cudaStreamSynchronize(st_));
  }

  // Same sequence as Locg::start_implicit, every pass after the first residual gated so that
  // instances whose start vector is exact stop there.
  void start_implicit() {
    R *x = x_.ptr, *y = y_.ptr, *r = r_.ptr, *p = p_.ptr, *ax = ax_.ptr, *ay = ay_.ptr,
      *ap = ap_.ptr;
    const int g = G_DONE;
    lc({x}, {}, {{0, 0}}, P_INV_NORM);
    lc({x}, {x}, {}, P_NONE);
    matvec(x, ax);
    lc({ax, x}, {}, {{1, 0}}, P_THETA0);
    lc({ax, x}, {r}, {{100, 100}}, P_R0NORM);
    SQD_CUDA(cudaMemsetAsync(y, 0, sizeof(R) * NC * b_->total_rows, cur_));
    SQD_CUDA(cudaMemsetAsync(ay, 0, sizeof(R) * NC * b_->total_rows, cur_));
    lc({r}, {p}, {}, P_NONE, g);
    matvec(p, ap);
    lc({x, p, ax, ap}, {}, {{0, 2}, {1, 2}, {1, 3}}, P_RR2, g);
    lc({ax, ap}, {ay, ax}, {}, P_NONE, g);
    lc({x, p}, {y, x}, {{100, 100}, {101, 101}}, P_TU_NORM, g);
    lc({x, y}, {x, y}, {}, P_NONE, g);
    lc({ax, ay}, {ax, ay}, {}, P_SET_R_COEF, g);
    lc({ax, x}, {r}, {{100, 100}, {0, 0}}, P_CONV, g);
    lc({r, x, y}, {}, {{1, 0}, {2, 0}}, P_PROJ_IPS, g);
  }

  void body_fast() {
    R *x = x_.ptr, *y = y_.ptr, *r = r_.ptr, *p = p_.ptr, *ax = ax_.ptr, *ay = ay_.ptr,
      *ap = ap_.ptr;
    const int g = G_DONE;
    lc({r, x, y}, {p}, {{100, 100}, {1, 100}, {2, 100}}, P_PROJ_NORM_IPS, g);
    lc({p, x, y}, {p}, {}, P_NONE, g);
    matvec(p, ap);
    lc({x, y, p, ax, ay, ap}, {},
       {{0, 3}, {1, 4}, {2, 5}, {1, 3}, {2, 3}, {2, 4}, {2, 2}, {1, 2}}, P_GRAM_IMPLICIT, g);
    lc({x, y, p, ax, ay, ap}, {x, y, ax, ay}, {{100, 100}, {101, 101}}, P_UPDATE_NORMS, g);
    lc({x, y, ax, ay}, {x, y, ax, ay, r}, {{104, 104}, {102, 102}, {100, 104}, {101, 104}},
       P_CONV_PROJ, g);
    k_bactive<<<1, 256, 0, cur_>>>(dev_.ptr, b_->n, use_cond_, cond_, active_.ptr);
    SQD_CHECK_LAUNCH();
  }

  // Explicit A x, A y, residual and convergence test for every instance (drift check).
  void refresh() {
    post_only(P_RESET);
    matvec(x_.ptr, ax_.ptr);
    matvec(y_.ptr, ay_.ptr);
    lc({ax_.ptr, x_.ptr}, {}, {{1, 0}}, P_THETA0);
    lc({ax_.ptr, x_.ptr}, {r_.ptr}, {{100, 100}, {0, 0}}, P_CONV);
    lc({r_.ptr, x_.ptr, y_.ptr}, {}, {{1, 0}, {2, 0}}, P_PROJ_IPS);
  }

  void loop(bool use_graph) {
    if (active() == 0) return;
    if (!use_graph) {
      for (;;) {
        body_fast();
        if (active() == 0) break;
      }
      return;
    }
    if (!exec_) {
      SQD_CUDA(cudaGraphCreate(&graph_, 0));
      SQD_CUDA(cudaGraphConditionalHandleCreate(&cond_, graph_, 1, cudaGraphCondAssignDefault));
      cudaGraphNodeParams cp{};
      cp.type = cudaGraphNodeTypeConditional;
      cp.conditional.handle = cond_;
      cp.conditional.type = cudaGraphCondTypeWhile;
      cp.conditional.size = 1;
      cudaGraphNode_t node;
      SQD_CUDA(cudaGraphAddNode(&node, graph_, nullptr, 0, &cp));
      cudaGraph_t bodyg = cp.conditional.phGraph_out[0];
      cudaStream_t cap = nullptr;
      SQD_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
      cur_ = cap;
      use_cond_ = 1;
      auto restore = [&] {
        cur_ = st_;
        use_cond_ = 0;
        cudaStreamDestroy(cap);
      };
      cudaError_t cerr = cudaStreamBeginCaptureToGraph(cap, bodyg, nullptr, nullptr, 0,
                                                       cudaStreamCaptureModeThreadLocal);
      if (cerr != cudaSuccess) {
        restore();
        SQD_CUDA(cerr);
      }
      try {
        body_fast();
      } catch (...) {
        cudaGraph_t dummy;
        cudaStreamEndCapture(cap, &dummy);
        restore();
        throw;
      }
      cerr = cudaStreamEndCapture(cap, &bodyg);
      restore();
      SQD_CUDA(cerr);
      SQD_CUDA(cudaGraphInstantiate(&exec_, graph_, 0));
    }
    SQD_CUDA(cudaGraphLaunch(exec_, st_));
    SQD_CUDA(cudaStreamSynchronize(st_));
  }

  DevBuf<R> x_, y_, r_, p_, ax_, ay_, ap_;

 private:
  template <typename A>
  void fill(A& a, std::initializer_list<const void*> srcs, std::initializer_list<void*> outs,
            std::initializer_list<std::pair<int, int>> dots, int gate) {
    int k = 0;
    for (auto s : srcs) a.src[k++] = s;
    a.nsrc = k;
    k = 0;
    for (auto o : outs) a.out[k++] = o;
    a.nout = k;
    k = 0;
    for (auto d : dots) {
      a.da[k] = static_cast<signed char>(d.first);
      a.db[k] = static_cast<signed char>(d.second);
      ++k;
    }
    a.ndot = k;
    a.gate = gate;
    a.dev = dev_.ptr;
    a.partials = partials_.ptr;
    a.tile_inst = b_->tile_inst.ptr;
    a.tile_row0 = b_->tile_row0.ptr;
    a.n_tiles = b_->n_tiles;
  }
  void posts(int nsrc, int ndot, int stride, int post, int gate) {
    if (post == P_NONE && ndot == 0) return;
    const unsigned G = grid_for(static_cast<int64_t>(b_->n) * 32, 256);
    k_bpost<<<G, 256, 0, cur_>>>(partials_.ptr, stride, b_->inst_tile0_d.ptr, b_->n, dev_.ptr,
                                 ndot, nsrc, post, gate);
    SQD_CHECK_LAUNCH();
  }

  sqd_batch_s* b_;
  cudaStream_t st_, cur_;
  unsigned blocks_ = 1;
  DevBuf<LocgDev> dev_;
  DevBuf<double> partials_;
  DevBuf<int> active_;
  LocgDev* host_ = nullptr;
  int use_cond_ = 0;
  cudaGraphConditionalHandle cond_ = 0;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t exec_ = nullptr;
};

template <int NC>
void run_batch(sqd_batch_s* b, const double* xinit, const int64_t* xidx, double tol, int maxiter,
               bool use_graph, cudaStream_t st, double* eig, double* vecs, int* niter,
               double* resid) {
  constexpr double kInnerRtol = 2e-7;
  constexpr int kStall = 25;
  constexpr int kRestarts = 6;
  const double eps64 = 2.220446049250313e-16;
  const int64_t n = b->total_rows;
  const unsigned G = grid_for(n, 256, 8192);
  std::vector<int> it32(b->n, 0);
  DevBuf<double> x64;
  x64.alloc(static_cast<size_t>(n) * NC, st);
  {
    BLocg<float, NC> L(b, st);
    L.set_params(0.0, maxiter, kInnerRtol, 0.0, kStall);
    if (xinit)
      k_convert<float, double, NC><<<G, 256, 0, st>>>(xinit, L.x(), n);
    else
      L.onehot(xidx);
    SQD_CHECK_LAUNCH();
    L.start_implicit();
    for (int k = 0; k < kRestarts; ++k) {
      L.loop(use_graph);
      L.refresh();
      if (L.active() == 0) break;
    }
    L.read_host();
    for (int i = 0; i < b->n; ++i) it32[i] = L.host(i).niter;
    k_convert<double, float, NC><<<G, 256, 0, st>>>(L.x(), x64.ptr, n);
    SQD_CHECK_LAUNCH();
  }
  BLocg<double, NC> L(b, st);
  L.set_params(tol < 0 ? eps64 : tol, maxiter, 0.0, 0.0, 0);
  SQD_CUDA(cudaMemcpyAsync(L.x(), x64.ptr, sizeof(double) * NC * n, cudaMemcpyDeviceToDevice, st));
  L.start_implicit();
  L.loop(use_graph);
  L.read_host();
  for (int i = 0; i < b->n; ++i) {
    eig[i] = L.host(i).theta;
    niter[i] = it32[i] + L.host(i).niter;
    if (resid) resid[i] = L.host(i).rnorm;
  }
  SQD_CUDA(cudaMemcpyAsync(vecs, L.x(), sizeof(double) * NC * n, cudaMemcpyDeviceToDevice, st));
  SQD_CUDA(cudaStreamSynchronize(st));
}

__global__ void k_add_i64(const int64_t* in, int64_t* out, int64_t n, int64_t add) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    out[i] = in[i] + add;
}
__global__ void k_add_u32(const uint32_t* in, uint32_t* out, int64_t n, uint32_t add) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    out[i] = in[i] + add;
}

}  // namespace
}  // namespace sqd

using namespace sqd;

extern "C" int sqd_op_matvec_cb(void* ctx, const void* x, void* y, void* stream) {
  return guarded([&] {
    SQD_REQUIRE(ctx != nullptr, "NULL operator");
    auto* op = static_cast<sqd_op_s*>(ctx);
    // Applies the operator to complex128 vectors (sqd_locg substitutes its own dtype).
    op_matvec(op, x, y, SQD_C128, as_stream(stream));
  });
}

// Operator callback with an explicit dtype (used by the FP64 solver).
namespace {
struct OpDtypeCtx {
  sqd_op_s* op;
  int dtype;
};
int op_dtype_cb(void* ctx, const void* x, void* y, void* stream) {
  auto* c = static_cast<OpDtypeCtx*>(ctx);
  return guarded([&] { op_matvec(c->op, x, y, c->dtype, as_stream(stream)); });
}
}  // namespace

extern "C" int sqd_locg_record(double* rows_host, int64_t max_rows, int64_t* count_host) {
  return guarded([&] {
    SQD_REQUIRE(max_rows >= 0 && max_rows <= (1 << 24), "max_rows must be in [0, 2^24]");
    g_hist_request = HistRequest{};
    if (rows_host == nullptr || max_rows == 0) return;
    g_hist_request = HistRequest{rows_host, max_rows, count_host};
    if (count_host) *count_host = 0;
  });
}

extern "C" int sqd_locg(int64_t n, int dtype, sqd_matvec_fn fn, void* ctx, const void* xinit,
                        int64_t xinit_index, const void* const* orth, int n_orth, double tol,
                        int maxiter, int mode, int use_graph, void* stream, double* eigval_host,
                        void* eigvec, int* niter_host, double* residual_host) {
  return guarded([&] {
    SQD_REQUIRE(n >= 1, "empty vector space");
    SQD_REQUIRE(dtype == SQD_F64 || dtype == SQD_C128, "LOCG result dtype must be F64 or C128");
    SQD_REQUIRE(fn != nullptr, "NULL matvec");
    SQD_REQUIRE(eigval_host && eigvec && niter_host, "NULL output");
    SQD_REQUIRE(n_orth >= 0 && n_orth <= kMaxOrth, "at most 8 orth vectors");
    SQD_REQUIRE(mode == SQD_LOCG_FP64 || mode == SQD_LOCG_MIXED, "bad LOCG mode");
    SQD_REQUIRE(xinit != nullptr || (xinit_index >= 0 && xinit_index < n),
                "xinit index out of range");
    cudaStream_t st = as_stream(stream);
    std::vector<const void*> ov;
    for (int k = 0; k < n_orth; ++k) ov.push_back(orth[k]);
    OpDtypeCtx octx{nullptr, dtype};
    sqd_matvec_fn f = fn;
    void* c = ctx;
    bool graph = use_graph != 0;
    if (fn == sqd_op_matvec_cb) {
      octx.op = static_cast<sqd_op_s*>(ctx);
      SQD_REQUIRE(octx.op->s->states_size == n, "vector size differs from the operator size");
      SQD_REQUIRE(dtype == SQD_C128 || !octx.op->value_complex,
                  "a complex Hamiltonian needs complex vectors");
      if (mode == SQD_LOCG_FP64) {
        f = op_dtype_cb;
        c = &octx;
      }
    } else {
      graph = false;  // foreign callbacks may synchronise; no capture
    }
    if (dtype == SQD_C128)
      run_locg<2>(n, dtype, f, c, octx.op, xinit, xinit_index, ov, tol, maxiter, mode, graph,
                  st, eigval_host, eigvec, niter_host, residual_host);
    else
      run_locg<1>(n, dtype, f, c, octx.op, xinit, xinit_index, ov, tol, maxiter, mode, graph,
                  st, eigval_host, eigvec, niter_host, residual_host);
  });
}

// ---------------------------------------------------------------------------- batched C ABI
extern "C" int sqd_batch_create(const sqd_op_t* ops, int n_ops, void* stream,
                                sqd_batch_t* out) {
  return guarded([&] {
    SQD_REQUIRE(out != nullptr, "out handle is NULL");
    *out = nullptr;
    SQD_REQUIRE(ops != nullptr && n_ops >= 1, "no operators");
    cudaStream_t st = as_stream(stream);
    auto b = std::make_unique<sqd_batch_s>();
    b->n = n_ops;
    b->value_complex = ops[0]->value_complex;
    b->row0.assign(n_ops + 1, 0);
    std::vector<int64_t> nnz0(n_ops + 1, 0);
    for (int i = 0; i < n_ops; ++i) {
      const sqd_op_s* op = ops[i];
      SQD_REQUIRE(op != nullptr, "NULL operator");
      SQD_REQUIRE(op->x_cache == 1 && op->z_cache == 2,
                  "batched operators need cache_strategy (1, 2)");
      SQD_REQUIRE(op->value_complex == b->value_complex,
                  "batched operators must all be real or all complex");
      b->row0[i + 1] = b->row0[i] + op->s->states_size;
      nnz0[i + 1] = nnz0[i] + op->nnz;
    }
    b->total_rows = b->row0[n_ops];
    b->total_nnz = nnz0[n_ops];
    SQD_REQUIRE(b->total_rows < (int64_t(1) << 32), "batch limited to 2^32 rows");
    const int nca = b->value_complex ? 2 : 1;
    b->row_ptr.alloc(b->total_rows + 1, st);
    b->cols.alloc(std::max<int64_t>(b->total_nnz, 1), st);
    b->values.alloc(std::max<int64_t>(b->total_nnz, 1) * nca, st);
    for (int i = 0; i < n_ops; ++i) {
      const sqd_op_s* op = ops[i];
      const int64_t rows = op->s->states_size;
      k_add_i64<<<grid_for(rows, 256, 4096), 256, 0, st>>>(op->row_ptr.ptr,
                                                            b->row_ptr.ptr + b->row0[i], rows,
                                                            nnz0[i]);
      if (op->nnz > 0) {
        k_add_u32<<<grid_for(op->nnz, 256, 8192), 256, 0, st>>>(
            op->cols.ptr, b->cols.ptr + nnz0[i], op->nnz, static_cast<uint32_t>(b->row0[i]));
        SQD_CUDA(cudaMemcpyAsync(b->values.ptr + nnz0[i] * nca, op->values.ptr,
                                 sizeof(double) * op->nnz * nca, cudaMemcpyDeviceToDevice, st));
      }
      SQD_CHECK_LAUNCH();
    }
    SQD_CUDA(cudaMemcpyAsync(b->row_ptr.ptr + b->total_rows, &b->total_nnz, sizeof(int64_t),
                             cudaMemcpyHostToDevice, st));
    const size_t nv = static_cast<size_t>(std::max<int64_t>(b->total_nnz, 1)) * nca;
    b->values32.alloc(nv, st);
    k_convert<float, double, 1><<<grid_for(nv, 256, 16384), 256, 0, st>>>(b->values.ptr,
                                                                         b->values32.ptr, nv);
    SQD_CHECK_LAUNCH();
    // tiles
    std::vector<int32_t> ti;
    std::vector<int64_t> tr;
    b->inst_tile0.assign(n_ops + 1, 0);
    for (int i = 0; i < n_ops; ++i) {
      b->inst_tile0[i] = static_cast<int32_t>(ti.size());
      for (int64_t r = b->row0[i]; r < b->row0[i + 1]; r += kTileRows) {
        ti.push_back(i);
        tr.push_back(r);
      }
    }
    b->inst_tile0[n_ops] = static_cast<int32_t>(ti.size());
    tr.push_back(b->total_rows);
    b->n_tiles = static_cast<int>(ti.size());
    b->tile_inst.alloc(ti.size(), st);
    b->tile_row0.alloc(tr.size(), st);
    b->inst_tile0_d.alloc(n_ops + 1, st);
    SQD_CUDA(cudaMemcpyAsync(b->tile_inst.ptr, ti.data(), sizeof(int32_t) * ti.size(),
                             cudaMemcpyHostToDevice, st));
    SQD_CUDA(cudaMemcpyAsync(b->tile_row0.ptr, tr.data(), sizeof(int64_t) * tr.size(),
                             cudaMemcpyHostToDevice, st));
    SQD_CUDA(cudaMemcpyAsync(b->inst_tile0_d.ptr, b->inst_tile0.data(),
                             sizeof(int32_t) * (n_ops + 1), cudaMemcpyHostToDevice, st));
    const double avg = b->total_rows > 0 ? double(b->total_nnz) / double(b->total_rows) : 0.0;
    const int lpr = avg >= 96 ? 32 : avg >= 40 ? 16 : avg >= 16 ? 8 : avg >= 6 ? 4
                  : avg >= 2 ? 2 : 1;
    b->lanes[0] = b->lanes[1] = lpr;
    SQD_CUDA(cudaStreamSynchronize(st));
    *out = b.release();
  });
}

extern "C" int sqd_batch_info(sqd_batch_t b, int64_t* total_rows, int64_t* total_pairs) {
  return guarded([&] {
    SQD_REQUIRE(b != nullptr, "NULL batch");
    if (total_rows) *total_rows = b->total_rows;
    if (total_pairs) *total_pairs = b->total_nnz;
  });
}

extern "C" int sqd_batch_set_lanes(sqd_batch_t b, int precision, int lanes_per_row) {
  return guarded([&] {
    SQD_REQUIRE(b != nullptr, "NULL batch");
    SQD_REQUIRE(precision == 0 || precision == 1, "precision must be 0 (FP64) or 1 (FP32)");
    dispatch_lpr(lanes_per_row, [](auto) {});
    b->lanes[precision] = lanes_per_row;
  });
}

extern "C" int sqd_batch_locg(sqd_batch_t b, int dtype, const void* xinit,
                              const int64_t* xinit_index_host, double tol, int maxiter,
                              int use_graph, void* stream, double* eigvals_host, void* eigvecs,
                              int* niters_host, double* residuals_host) {
  return guarded([&] {
    SQD_REQUIRE(b != nullptr && eigvals_host && eigvecs && niters_host, "NULL argument");
    SQD_REQUIRE(dtype == SQD_F64 || dtype == SQD_C128, "batched LOCG dtype must be F64 or C128");
    SQD_REQUIRE(dtype == SQD_C128 || !b->value_complex,
                "a complex Hamiltonian needs complex vectors");
    SQD_REQUIRE(xinit != nullptr || xinit_index_host != nullptr, "no start vectors");
    if (!xinit)
      for (int i = 0; i < b->n; ++i)
        SQD_REQUIRE(xinit_index_host[i] >= 0 &&
                        xinit_index_host[i] < b->row0[i + 1] - b->row0[i],
                    "start index out of range");
    SQD_REQUIRE(maxiter >= 1, "maxiter must be positive");
    cudaStream_t st = as_stream(stream);
    if (dtype == SQD_C128)
      run_batch<2>(b, static_cast<const double*>(xinit), xinit_index_host, tol, maxiter,
                   use_graph != 0, st, eigvals_host, static_cast<double*>(eigvecs), niters_host,
                   residuals_host);
    else
      run_batch<1>(b, static_cast<const double*>(xinit), xinit_index_host, tol, maxiter,
                   use_graph != 0, st, eigvals_host, static_cast<double*>(eigvecs), niters_host,
                   residuals_host);
  });
}

extern "C" void sqd_batch_destroy(sqd_batch_t b) { delete b; }

// ----------------------------------------------------------------------------- small eigenpairs
// eigenpair_2x2 / eigenpair_3x3 (ground_locg.py:467-514) on a batch of Hermitian matrices, one
// thread per matrix: the same device functions the Rayleigh-Ritz steps of the solver call.
namespace sqd {
namespace {
__global__ void k_eigenpair_small(const double2* __restrict__ mats, int64_t count, int dim,
                                  double* __restrict__ vals, double2* __restrict__ vecs) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  const double2* m = mats + i * dim * dim;
  if (dim == 2) {
    double2 a[2][2] = {{m[0], m[1]}, {m[2], m[3]}};
    double2 v[2];
    eig2(a, &vals[i], v);
    vecs[i * 2] = v[0];
    vecs[i * 2 + 1] = v[1];
  } else {
    double2 a[3][3] = {{m[0], m[1], m[2]}, {m[3], m[4], m[5]}, {m[6], m[7], m[8]}};
    double2 v[3];
    eig3(a, &vals[i], v);
    for (int k = 0; k < 3; ++k) vecs[i * 3 + k] = v[k];
  }
}
}  // namespace
}  // namespace sqd

extern "C" int sqd_eigenpair_small(const void* mats, int64_t count, int dim, double* vals,
                                   void* vecs, void* stream) {
  return guarded([&] {
    SQD_REQUIRE(dim == 2 || dim == 3, "dim must be 2 or 3");
    SQD_REQUIRE(count >= 0, "negative count");
    if (count == 0) return;
    SQD_REQUIRE(mats != nullptr && vals != nullptr && vecs != nullptr, "NULL array");
    const int threads = 128;
    const int64_t blocks = (count + threads - 1) / threads;
    SQD_REQUIRE(blocks <= 0x7fffffff, "count too large");
    k_eigenpair_small<<<(unsigned)blocks, threads, 0, as_stream(stream)>>>(
        static_cast<const double2*>(mats), count, dim, vals, static_cast<double2*>(vecs));
    SQD_CHECK_LAUNCH();
  });
}
