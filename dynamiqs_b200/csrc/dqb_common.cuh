// Shared device code for the mesolve kernels: Runge-Kutta tableaux, dense-output
// weights, the integral step-size controller, complex helpers and block reductions.
//
// The RK engine re-creates what dynamiqs obtains from diffrax (diffrax_integrator.py:
// 59-133): Tsit5 (Tsitouras 2011) and Dopri5 (Dormand & Prince 1980) with FSAL, the
// embedded error estimate (Dopri5 with the alternative fourth-order embedded weights
// 1951/21600, 0, 22642/50085, 451/720, -12231/42400, 649/6300, 1/60), an RMS error norm
// over every complex entry of e / (atol + rtol * max(|y0|, |y1|)), an integral
// controller with exponent 1/5 and the Hairer-Norsett-Wanner starting step with
// exponent 1/4 in its last stage.  These choices reproduce the step counts the
// reference prints for its README, mesolve-docstring and Dopri5 workflow examples
// (40/40/0, 9/9/0, 56/48/8).  Time, step size, the error-norm
// accumulation and the controller run in FP64; the state and the stages in FP32
// complex (complex64, the reference's default dtype).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/dqb200.h"

#include <cstring>

namespace dqb {

// ------------------------------------------------------------------------------------
// tableaux (index 0 = Tsit5, 1 = Dopri5); a is 7x7 row-major, row 6 = b (FSAL)
// ------------------------------------------------------------------------------------
struct Tableau {
  double c[7];
  double a[7][7];
  double b[7];
  double btilde[7];  // b - bhat
  double cmid[7];    // Dopri5 midpoint weights (Shampine); unused for Tsit5
};

static __constant__ Tableau c_tab[2] = {
    // Tsit5 (Tsitouras 2011)
    {{0.0, 0.161, 0.327, 0.9, 0.9800255409045097, 1.0, 1.0},
     {{0, 0, 0, 0, 0, 0, 0},
      {0.161, 0, 0, 0, 0, 0, 0},
      {-0.008480655492356989, 0.335480655492357, 0, 0, 0, 0, 0},
      {2.897153057105493, -6.359448489975075, 4.3622954328695815, 0, 0, 0, 0},
      {5.325864828439257, -11.748883564062828, 7.4955393428898365, -0.09249506636175525, 0, 0, 0},
      {5.86145544294642, -12.92096931784711, 8.159367898576159, -0.071584973281401,
       -0.028269050394068383, 0, 0},
      {0.09646076681806523, 0.01, 0.4798896504144996, 1.379008574103742, -3.290069515436081,
       2.324710524099774, 0}},
     {0.09646076681806523, 0.01, 0.4798896504144996, 1.379008574103742, -3.290069515436081,
      2.324710524099774, 0.0},
     {-0.001780011052226, -0.000816434459657, 0.007880878010262, -0.144711007173263,
      0.582357165452555, -0.458082105929187, 1.0 / 66.0},
     {0, 0, 0, 0, 0, 0, 0}},
    // Dopri5 (Dormand & Prince 1980; error weights b - bhat with the alternative bhat)
    {{0.0, 0.2, 0.3, 0.8, 8.0 / 9.0, 1.0, 1.0},
     {{0, 0, 0, 0, 0, 0, 0},
      {0.2, 0, 0, 0, 0, 0, 0},
      {3.0 / 40.0, 9.0 / 40.0, 0, 0, 0, 0, 0},
      {44.0 / 45.0, -56.0 / 15.0, 32.0 / 9.0, 0, 0, 0, 0},
      {19372.0 / 6561.0, -25360.0 / 2187.0, 64448.0 / 6561.0, -212.0 / 729.0, 0, 0, 0},
      {9017.0 / 3168.0, -355.0 / 33.0, 46732.0 / 5247.0, 49.0 / 176.0, -5103.0 / 18656.0, 0, 0},
      {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0, 0}},
     {35.0 / 384.0, 0.0, 500.0 / 1113.0, 125.0 / 192.0, -2187.0 / 6784.0, 11.0 / 84.0, 0.0},
     {35.0 / 384.0 - 1951.0 / 21600.0, 0.0, 500.0 / 1113.0 - 22642.0 / 50085.0,
      125.0 / 192.0 - 451.0 / 720.0, -2187.0 / 6784.0 + 12231.0 / 42400.0,
      11.0 / 84.0 - 649.0 / 6300.0, -1.0 / 60.0},
     {6025192743.0 / 30085553152.0 / 2.0, 0.0, 51252292925.0 / 65400821598.0 / 2.0,
      -2691868925.0 / 45128329728.0 / 2.0, 187940372067.0 / 1594534317056.0 / 2.0,
      -1776094331.0 / 19743644256.0 / 2.0, 11237099.0 / 235043384.0 / 2.0}},
};

// Dense-output weights w_i(theta): y(t + theta h) = y + h * sum_i w_i k_i.
// Tsit5: Tsitouras' continuous extension.  Dopri5: the quartic through y0, y1,
// h k1, h k7 and Shampine's midpoint y_mid = y0 + h sum cmid_i k_i, which gives
//   w_i = b_i (-5t^2 + 14t^3 - 8t^4) + cmid_i (16t^2 - 32t^3 + 16t^4)
//         + [i=1] (t - 4t^2 + 5t^3 - 2t^4) + [i=7] (t^2 - 3t^3 + 2t^4).
__device__ __forceinline__ void dense_weights(int method, double t, double w[7]) {
  const double t2 = t * t;
  if (method == DQB_METHOD_TSIT5) {
    w[0] = -1.0530884977290216 * t * (t - 1.3299890189751412) *
           (t2 - 1.4364028541716351 * t + 0.7139816917074209);
    w[1] = 0.1017 * t2 * (t2 - 2.1966568338249754 * t + 1.2949852507374631);
    w[2] = 2.490627285651252793 * t2 * (t2 - 2.38535645472061657 * t + 1.57803468208092486);
    w[3] = -16.54810288924490272 * (t - 1.21712927295533244) * (t - 0.61620406037800089) * t2;
    w[4] = 47.37952196281928122 * (t - 1.203071208372362603) * (t - 0.658047292653547382) * t2;
    w[5] = -34.87065786149660974 * (t - 1.2) * (t - 0.666666666666666667) * t2;
    w[6] = 2.5 * (t - 1.0) * (t - 0.6) * t2;
  } else {
    const double t3 = t2 * t, t4 = t3 * t;
    const double pb = -5.0 * t2 + 14.0 * t3 - 8.0 * t4;
    const double pm = 16.0 * t2 - 32.0 * t3 + 16.0 * t4;
    const Tableau& T = c_tab[1];
    for (int i = 0; i < 7; ++i) w[i] = T.b[i] * pb + T.cmid[i] * pm;
    w[0] += t - 4.0 * t2 + 5.0 * t3 - 2.0 * t4;
    w[6] += t2 - 3.0 * t3 + 2.0 * t4;
  }
}

// ------------------------------------------------------------------------------------
// controller (one thread)
// ------------------------------------------------------------------------------------
struct CtrlOpts {
  int method, form;
  double rtol, atol, safety, factormin, factormax;
  long long max_steps;
  double t0;
  int save_states, check_hermitian;
};

__host__ inline CtrlOpts make_ctrl(const dqb_ode_options& o) {
  CtrlOpts c;
  c.method = o.method;
  c.form = o.form;
  c.rtol = o.rtol;
  c.atol = o.atol;
  c.safety = o.safety;
  c.factormin = o.factormin;
  c.factormax = o.factormax;
  c.max_steps = o.max_steps;
  c.t0 = o.t0;
  c.save_states = o.save_states;
  c.check_hermitian = o.check_hermitian;
  return c;
}

// Integral controller: factor = clip(safety * err^(-1/5), fmin, factormax) with
// fmin = 1 on an accepted step (an accepted step never shrinks the next one) and
// factormin on a rejected one.  A zero error gives factormax.
__device__ __forceinline__ double step_factor(const CtrlOpts& o, double err, bool keep) {
  const double fmin = keep ? 1.0 : o.factormin;
  double f;
  if (err == 0.0) {
    f = o.factormax;
  } else if (!(err < INFINITY)) {  // inf or nan
    f = fmin;
  } else {
    f = o.safety * pow(err, -0.2);
  }
  f = fmin > f ? fmin : f;
  f = f > o.factormax ? o.factormax : f;
  return f;
}

// Next trial end time after a step from `t` (the new current time): clipped to t1,
// and snapped to t1 when within 1e-10 of it (half of what is left after a rejection).
__device__ __forceinline__ double next_tend(double t, double dt, double t1, bool keep) {
  double tn = t + dt;
  if (tn > t1 - 1e-10) tn = keep ? t1 : t + 0.5 * (t1 - t);
  return tn < t1 ? tn : t1;
}

// ------------------------------------------------------------------------------------
// complex helpers
// ------------------------------------------------------------------------------------
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ void cmac(float2& acc, float2 a, float2 b) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(a.y, b.x, acc.y);
}
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 acc) {  // acc + a b
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(a.y, b.x, acc.y);
  return acc;
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 caxpy(float s, float2 x, float2 y) {  // y + s x
  return make_float2(fmaf(s, x.x, y.x), fmaf(s, x.y, y.y));
}
__device__ __forceinline__ float cabs2f(float2 a) { return fmaf(a.x, a.x, a.y * a.y); }
__device__ __forceinline__ float cabsf(float2 a) { return sqrtf(cabs2f(a)); }

// ------------------------------------------------------------------------------------
// block reductions (blockDim.x multiple of 32, <= 1024)
// ------------------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Sum of `v` over the block; every thread gets the result.  `red` holds >= 33 doubles.
__device__ __forceinline__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (wid == 0) {
    double x = lane < nw ? red[lane] : 0.0;
    x = warp_sum(x);
    if (lane == 0) red[32] = x;
  }
  __syncthreads();
  return red[32];
}

// Sums of `a` and `b` over the block at once; every thread gets both.  `red` holds >= 66
// doubles.
__device__ __forceinline__ double2 block_sum2(double a, double b, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  a = warp_sum(a);
  b = warp_sum(b);
  __syncthreads();
  if (lane == 0) red[wid] = a, red[32 + wid] = b;
  __syncthreads();
  if (wid == 0) {
    double x = lane < nw ? red[lane] : 0.0, y = lane < nw ? red[32 + lane] : 0.0;
    x = warp_sum(x);
    y = warp_sum(y);
    if (lane == 0) red[64] = x, red[65] = y;
  }
  __syncthreads();
  return make_double2(red[64], red[65]);
}

// One time-dependent term of H (dqb_td_term), by value in the kernel arguments.
struct TdTerm {
  int kind, n_times;
  const double* times;
  const double2* values;
  const int* vidx;
  double amp_re, amp_im, omega, phase, t_center, sigma, t_start, t_end;
};

// c_m(t) of term T for instance `inst`.
__device__ __forceinline__ double2 td_coef(const TdTerm& T, long long inst, double t) {
  if (T.kind == DQB_TD_CONST) return make_double2(1.0, 0.0);
  if (T.kind == DQB_TD_PWC) {
    const int nt = T.n_times;
    if (!(t >= T.times[0]) || !(t < T.times[nt - 1])) return make_double2(0.0, 0.0);
    int lo = 0, hi = nt - 1;  // times[lo] <= t < times[hi]
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (T.times[mid] <= t) lo = mid; else hi = mid;
    }
    const long long set = T.vidx ? T.vidx[inst] : 0;
    return T.values[set * (nt - 1) + lo];
  }
  if (!(t >= T.t_start) || !(t < T.t_end)) return make_double2(0.0, 0.0);
  double f = cos(T.omega * t + T.phase);
  if (T.sigma > 0.0) {
    const double d = (t - T.t_center) / T.sigma;
    f *= exp(-0.5 * d * d);
  }
  return make_double2(T.amp_re * f, T.amp_im * f);
}

// The time-dependent terms of H for the large-problem steppers, by value in the kernel
// arguments: ops_m in the layout of the path (dense [M, n, n] or DIA diagonals on H's
// offsets [M, h_nd, n]).
struct TdOps {
  int M;
  const float2* ops;
  TdTerm term[DQB_TD_MAX_TERMS];
};

// One dqb_td_term as a TdTerm (host side); DQB_ERR_INVALID_ARGUMENT on a malformed one.
inline int td_term_from(const dqb_td_term& a, TdTerm* T) {
  if (a.kind != DQB_TD_PWC && a.kind != DQB_TD_WAVE && a.kind != DQB_TD_CONST) return DQB_ERR_INVALID_ARGUMENT;
  if (a.kind == DQB_TD_PWC && (a.n_times < 2 || !a.times || !a.values)) return DQB_ERR_INVALID_ARGUMENT;
  T->kind = a.kind;
  T->n_times = a.n_times;
  T->times = a.times;
  T->values = (const double2*)a.values;
  T->vidx = a.value_index;
  T->amp_re = a.amp_re;
  T->amp_im = a.amp_im;
  T->omega = a.omega;
  T->phase = a.phase;
  T->t_center = a.t_center;
  T->sigma = a.sigma;
  T->t_start = a.t_start;
  T->t_end = a.t_end;
  return DQB_OK;
}

// TdOps of a dqb_td_hamiltonian (host side); DQB_ERR_INVALID_ARGUMENT on a malformed one.
inline int td_ops_from(const dqb_td_hamiltonian* u, TdOps* out) {
  std::memset(out, 0, sizeof(*out));
  if (u->n_terms < 0 || u->n_terms > DQB_TD_MAX_TERMS || u->n_jump_ts < 0) return DQB_ERR_INVALID_ARGUMENT;
  if ((u->n_terms > 0 && (!u->ops || !u->terms)) || (u->n_jump_ts > 0 && !u->jump_ts)) return DQB_ERR_INVALID_ARGUMENT;
  out->M = u->n_terms;
  out->ops = (const float2*)u->ops;
  for (int m = 0; m < out->M; ++m)
    if (int rc = td_term_from(u->terms[m], &out->term[m])) return rc;
  return DQB_OK;
}

// First discontinuity strictly after t (or +inf).
__device__ __forceinline__ double next_jump(const double* jts, int nj, double t) {
  int lo = 0, hi = nj;  // first index with jts[idx] > t
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (jts[mid] <= t) lo = mid + 1; else hi = mid;
  }
  return lo < nj ? jts[lo] : INFINITY;
}

// Next trial end time from t for a step dt: clipped just before the next discontinuity
// (made_jump), then clipped to t1 as next_tend does.
__device__ __forceinline__ double next_trial(const double* jts, int nj, double t, double dt, double t1, bool keep,
                                             int& made_jump) {
  double tn = t + dt;
  made_jump = 0;
  if (nj > 0) {
    const double J = next_jump(jts, nj, t);
    if (tn >= J) {
      tn = nextafter(J, -INFINITY);
      made_jump = 1;
    }
  }
  if (tn > t1 - 1e-10) tn = keep ? t1 : t + 0.5 * (t1 - t);
  return tn < t1 ? tn : t1;
}

// Zero a few words on a stream with a kernel (a memset would order itself against the
// work of every other stream).
static __global__ void zero_words_kernel(unsigned int* p, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = 0u;
}

// Every kernel of the library asks for the largest shared-memory carveout, so that kernels
// of different entry points can share an SM without reconfiguring it (a carveout switch
// serialises concurrent streams).
template <class Kern>
__host__ inline void prefer_max_shared(Kern kern) {
  cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
}

}  // namespace dqb
