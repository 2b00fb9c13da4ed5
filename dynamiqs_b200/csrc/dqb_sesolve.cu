// Batched linear ODEs d y/dt = A y on the same Runge-Kutta engine as the master-equation
// kernels (the Tsit5 / Dopri5 tableaux, starting step, FP64 error norm, integral
// controller and dense output of dqb_common.cuh), in two forms:
//   * the Schroedinger equation d psi/dt = -i H psi (dynamiqs/integrators/core/
//     diffrax_integrator.py:221-228, sesolve.py), y = psi, expectation values
//     <psi|E|psi>;
//   * the vectorized master equation d vec(rho)/dt = S vec(rho) with the Lindbladian
//     superoperator S (diffrax_integrator.py:325-327, utils/vectorization.py:213-259),
//     y = vec(rho) (columns stacked), expectation values tr(E rho) = sum_ij E[i][j]
//     rho[j][i], a dot product of y with E read row by row.
//
// One warp solves one instance at a time and takes the next one from an atomic counter
// when it finishes (a persistent kernel, W warps per CTA).  Lane l owns the entries
// i = l + 32 r (r < R) of psi and of the seven stages, in registers; H lives in the warp's
// own shared-memory tile (rows padded to an odd stride of float2, so that the 32 lanes
// reading one column of 32 rows hit 16 distinct bank pairs); the stage input is staged in
// a small per-warp shared vector that every lane reads by broadcast.  Everything a warp
// decides -- error norm, accept or reject, next step, save points -- is computed by all
// of its lanes from the same warp-reduced values, so the lanes never diverge.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "dqb_common.cuh"

namespace dqb {

namespace se {

constexpr int kThreads = 256;  // 8 warps

enum Mode { kSchrodinger = 0, kLinear = 1 };

struct Args {
  int n, nE, ntsave;  // n: length of y (the Hilbert dimension, or its square when vectorized)
  int mode;           // Mode
  const float2* AT;   // kLinear: A transposed, complex64 [*, n, n] (A[i][m] at AT[m * n + i])
  long long batch;
  const float2* H;
  const float2* psi0;
  const float2* E;
  const double* tsave;
  const int* Hidx;
  const int* pidx;
  float2* states;
  float2* expects;
  int* infos;
  int* status;
  unsigned int* counter;
  CtrlOpts o;
};

template <int R>
struct Warp {
  static constexpr int NP = 32 * R;   // padded dimension
  static constexpr int LD = NP + 1;   // H row stride (float2)
  static constexpr int H_FLOATS = NP * LD;
  static constexpr int BYTES = (H_FLOATS + NP) * 8;  // H tile + stage-input vector
};

__device__ __forceinline__ double wsum(double v) { return warp_sum(v); }

// The operator of an instance: in the warp's shared-memory tile (row i at i * LD), or
// in global memory as A^T (A[i][m] at AT[m * n + i]: the 32 lanes reading one column of
// 32 consecutive rows read 256 consecutive bytes).
struct Op {
  const float2* s;
  const float2* g;
  int mode;
};

// out_r = (A x)_r for the lane's rows (times -i for the Schroedinger form), x staged in sx.
template <int R, bool G>
__device__ __forceinline__ void matvec(const Op& A, const float2* __restrict__ sx, int n, float2 (&out)[R]) {
  const int lane = threadIdx.x & 31;
  float2 acc[R];
#pragma unroll
  for (int r = 0; r < R; ++r) acc[r] = make_float2(0.f, 0.f);
#pragma unroll 4
  for (int m = 0; m < n; ++m) {
    const float2 xm = sx[m];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int i = lane + 32 * r;
      const float2 a = G ? (i < n ? __ldg(A.g + (long long)m * n + i) : make_float2(0.f, 0.f))
                         : A.s[i * Warp<R>::LD + m];
      cmac(acc[r], a, xm);
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r)
    out[r] = A.mode == kSchrodinger ? make_float2(acc[r].y, -acc[r].x) : acc[r];
}

// Stage the vector x (lane's entries) and evaluate f(x).
template <int R, bool G>
__device__ __forceinline__ void rhs(const Op& A, float2* sx, int n, const float2 (&x)[R], float2 (&out)[R]) {
  const int lane = threadIdx.x & 31;
  __syncwarp();
#pragma unroll
  for (int r = 0; r < R; ++r) sx[lane + 32 * r] = x[r];
  __syncwarp();
  matvec<R, G>(A, sx, n, out);
}

// State at save index `sidx` (entries v, lane's rows) and its expectation values
// <psi|E_m|psi> = sum_ij conj(psi_i) E_m[i][j] psi_j (FP64 sums); v is staged in sx.
template <int R>
__device__ void save_point(const Args& a, long long inst, int sidx, float2* sx, const float2 (&v)[R]) {
  const int lane = threadIdx.x & 31, n = a.n;
  __syncwarp();
#pragma unroll
  for (int r = 0; r < R; ++r) sx[lane + 32 * r] = v[r];
  __syncwarp();
  if (a.o.save_states) {
    float2* dst = a.states + (inst * a.ntsave + sidx) * (long long)n;
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (lane + 32 * r < n) dst[lane + 32 * r] = v[r];
  }
  for (int m = 0; m < a.nE; ++m) {
    double er = 0.0, ei = 0.0;
    if (a.mode == kLinear) {
      // tr(E rho) = sum_k E_k y_k with E read row by row (k = i * sqrt(n) + j)
      const float2* Em = a.E + (long long)m * n;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int k = lane + 32 * r;
        if (k >= n) continue;
        const float2 e = Em[k];
        er += (double)e.x * v[r].x - (double)e.y * v[r].y;
        ei += (double)e.x * v[r].y + (double)e.y * v[r].x;
      }
    } else {
      const float2* Em = a.E + (long long)m * n * n;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int j = lane + 32 * r;
        if (j >= n) continue;
        float2 acc = make_float2(0.f, 0.f);  // sum_i conj(psi_i) E[i][j]
        for (int i = 0; i < n; ++i) cmac(acc, cconj(sx[i]), Em[(long long)i * n + j]);
        er += (double)acc.x * v[r].x - (double)acc.y * v[r].y;
        ei += (double)acc.x * v[r].y + (double)acc.y * v[r].x;
      }
    }
    er = wsum(er);
    ei = wsum(ei);
    if (lane == 0) a.expects[(inst * a.nE + m) * a.ntsave + sidx] = make_float2((float)er, (float)ei);
  }
}

// Fill the warp's tile with the instance's operator (H row-major, or A from A^T).
template <int R>
__device__ void load_tile(const Args& a, long long hi, float2* sH) {
  const int lane = threadIdx.x & 31, n = a.n;
  const float2* src = (a.mode == kLinear ? a.AT : a.H) + hi * (long long)n * n;
  for (int e = lane; e < Warp<R>::NP * Warp<R>::NP; e += 32) {
    const int p = e / Warp<R>::NP, q = e % Warp<R>::NP;  // source row p, column q
    const float2 v = (p < n && q < n) ? src[(long long)p * n + q] : make_float2(0.f, 0.f);
    if (a.mode == kLinear) sH[q * Warp<R>::LD + p] = v;  // A[q][p] = AT[p][q]
    else sH[p * Warp<R>::LD + q] = v;
  }
}

template <int R, bool G>
__device__ void solve_instance(const Args& a, long long inst, float2* sH, float2* sx) {
  const int lane = threadIdx.x & 31, n = a.n;
  const CtrlOpts& o = a.o;
  const Tableau& T = c_tab[o.method];
  const double inv_n = 1.0 / (double)n;
  const long long hi = a.Hidx ? a.Hidx[inst] : inst;
  const long long pi = a.pidx ? a.pidx[inst] : inst;
  __syncwarp();
  Op A{sH, nullptr, a.mode};
  if (G) A.g = a.AT + hi * (long long)n * n;
  else load_tile<R>(a, hi, sH);
  float2 y[R], k[7][R], y1[R], x[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = lane + 32 * r;
    y[r] = i < n ? a.psi0[pi * n + i] : make_float2(0.f, 0.f);
  }
  __syncwarp();

  // ---- starting step (Hairer-Norsett-Wanner, RMS norm) --------------------------------
  rhs<R, G>(A, sx, n, y, k[0]);
  double s0 = 0.0, s1 = 0.0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const double sc = o.atol + o.rtol * (double)cabsf(y[r]);
    s0 += (double)cabs2f(y[r]) / (sc * sc);
    s1 += (double)cabs2f(k[0][r]) / (sc * sc);
  }
  s0 = wsum(s0);
  s1 = wsum(s1);
  const double d0 = sqrt(s0 * inv_n), d1 = sqrt(s1 * inv_n);
  const double h0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : 0.01 * d0 / d1;
#pragma unroll
  for (int r = 0; r < R; ++r) x[r] = caxpy((float)h0, k[0][r], y[r]);
  rhs<R, G>(A, sx, n, x, k[1]);
  double s2 = 0.0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const double sc = o.atol + o.rtol * (double)cabsf(y[r]);
    const double dx = (double)k[1][r].x - (double)k[0][r].x, dy = (double)k[1][r].y - (double)k[0][r].y;
    s2 += (dx * dx + dy * dy) / (sc * sc);
  }
  s2 = wsum(s2);
  const double t1 = a.tsave[a.ntsave - 1];
  double t = o.t0, tnext;
  {
    const double d2 = sqrt(s2 * inv_n) / h0;
    const double md = d1 > d2 ? d1 : d2;
    const double h1 = md <= 1e-15 ? fmax(1e-6, h0 * 1e-3) : pow(0.01 / md, 0.25);
    const double dt = fmin(100.0 * h0, h1);
    double tn = t + dt;
    if (tn > t1 - 1e-10) tn = t1;
    tnext = tn < t1 ? tn : t1;
  }
  long long nsteps = 0, nacc = 0, nrej = 0;
  int status = DQB_INST_OK, sidx = 0;
  bool run = t < t1;

  // ---- main loop ----------------------------------------------------------------------
  while (run) {
    if (nsteps >= o.max_steps) {
      status = DQB_INST_MAX_STEPS;
      break;
    }
    const double h = tnext - t;
#pragma unroll
    for (int s = 1; s < 7; ++s) {
      float cf[6];
#pragma unroll
      for (int j = 0; j < 6; ++j) cf[j] = (float)(h * T.a[s][j]);
#pragma unroll
      for (int r = 0; r < R; ++r) {
        float2 v = y[r];
#pragma unroll
        for (int j = 0; j < 6; ++j)
          if (j < s) v = caxpy(cf[j], k[j][r], v);
        x[r] = v;
      }
      if (s == 6) {
#pragma unroll
        for (int r = 0; r < R; ++r) y1[r] = x[r];  // row 6 of a is b (FSAL)
      }
      rhs<R, G>(A, sx, n, x, k[s]);  // (the unrolled stage loop keeps k[] in registers)
    }
    double se = 0.0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      double ex = 0.0, ey = 0.0;
#pragma unroll
      for (int j = 0; j < 7; ++j) {
        const double cb = h * T.btilde[j];
        ex = fma(cb, (double)k[j][r].x, ex);
        ey = fma(cb, (double)k[j][r].y, ey);
      }
      const float ya = cabsf(y[r]), y1a = cabsf(y1[r]);
      const double sc = o.atol + o.rtol * (double)(ya > y1a ? ya : y1a);
      if (lane + 32 * r < a.n) se += (ex * ex + ey * ey) / (sc * sc);
    }
    se = wsum(se);
    const double err = sqrt(se * inv_n);
    nsteps += 1;
    if (!(err < INFINITY)) {
      status = DQB_INST_NONFINITE;
      nrej += 1;
      break;
    }
    const bool keep = err < 1.0;
    const double dtnew = h * step_factor(o, err, keep);
    if (keep) {
      nacc += 1;
      while (sidx < a.ntsave && a.tsave[sidx] <= tnext) {
        double w[7];
        const double theta = h > 0.0 ? (a.tsave[sidx] - t) / h : 1.0;
        dense_weights(o.method, theta, w);
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
          v[r] = y[r];
#pragma unroll
          for (int j = 0; j < 7; ++j) v[r] = caxpy((float)(h * w[j]), k[j][r], v[r]);
        }
        save_point<R>(a, inst, sidx, sx, v);
        ++sidx;
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        y[r] = y1[r];
        k[0][r] = k[6][r];
      }
      t = tnext;
    } else {
      nrej += 1;
    }
    tnext = next_tend(t, dtnew, t1, keep);
    run = t < t1;
  }
  // saves left over (t1 <= t0: every save is the initial state)
  if (status == DQB_INST_OK) {
    while (sidx < a.ntsave && a.tsave[sidx] <= t) {
      save_point<R>(a, inst, sidx, sx, y);
      ++sidx;
    }
  }
  if (!o.save_states) {
    float2* dst = a.states + inst * (long long)n;
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (lane + 32 * r < n) dst[lane + 32 * r] = y[r];
  }
  __threadfence();
  __syncwarp();
  if (lane == 0) {
    a.infos[inst * 3 + 0] = (int)nsteps;
    a.infos[inst * 3 + 1] = (int)nacc;
    a.infos[inst * 3 + 2] = (int)nrej;
    __threadfence_system();
    a.status[inst] = status;
  }
}

// Shared memory of one warp: the operator tile and the stage-input vector, or the vector
// alone when the operator is read from global memory (G).
template <int R, bool G>
constexpr int warp_bytes() {
  return G ? Warp<R>::NP * 8 : Warp<R>::BYTES;
}

template <int R, bool G>
__global__ void __launch_bounds__(kThreads) sesolve_kernel(Args a, int warps) {
  extern __shared__ float4 se_smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp >= warps) return;  // warps beyond the shared memory's room take no work
  float2* base = reinterpret_cast<float2*>(reinterpret_cast<char*>(se_smem) + (size_t)warp * warp_bytes<R, G>());
  float2* sH = G ? nullptr : base;
  float2* sx = G ? base : base + Warp<R>::H_FLOATS;
  for (;;) {
    unsigned int v = 0;
    if (lane == 0) v = atomicAdd(a.counter, 1u);
    const long long inst = (long long)__shfl_sync(0xffffffffu, v, 0);
    if (inst >= a.batch) break;
    solve_instance<R, G>(a, inst, sH, sx);
  }
}

// One right-hand side -i H psi per instance (no RK loop), one warp per instance.
template <int R>
__global__ void __launch_bounds__(32) schrodinger_rhs_kernel(Args a, const float2* psi, float2* out) {
  extern __shared__ float4 se_smem[];
  float2* sH = reinterpret_cast<float2*>(se_smem);
  float2* sx = sH + Warp<R>::H_FLOATS;
  const long long b = blockIdx.x;
  const int lane = threadIdx.x, n = a.n;
  load_tile<R>(a, a.Hidx ? a.Hidx[b] : b, sH);
  float2 x[R], y[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int i = lane + 32 * r;
    x[r] = i < n ? psi[b * n + i] : make_float2(0.f, 0.f);
  }
  const Op A{sH, nullptr, a.mode};
  rhs<R, false>(A, sx, n, x, y);
#pragma unroll
  for (int r = 0; r < R; ++r)
    if (lane + 32 * r < n) out[b * n + lane + 32 * r] = y[r];
}

int rows_per_lane(int n) { return n <= 32 ? 1 : (n <= 64 ? 2 : (n <= 128 ? 4 : (n <= 256 ? 8 : 0))); }

size_t max_optin_smem() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return v > 0 ? (size_t)v : (size_t)232448;
}

template <int R, bool G>
int launch(const Args& a, cudaStream_t s) {
  static std::once_flag once;
  const size_t cap = max_optin_smem();
  std::call_once(once, [cap] {
    cudaFuncSetAttribute(sesolve_kernel<R, G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cap);
    prefer_max_shared(sesolve_kernel<R, G>);
  });
  const int warps = (int)std::min<size_t>(kThreads / 32, cap / warp_bytes<R, G>());
  if (warps < 1) return DQB_ERR_UNSUPPORTED;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long per_cta = warps;
  long long grid = std::min<long long>(sms, (a.batch + per_cta - 1) / per_cta);
  if (grid < 1) grid = 1;
  zero_words_kernel<<<1, 64, 0, s>>>(a.counter, 64);
  sesolve_kernel<R, G><<<(unsigned)grid, kThreads, (size_t)warps * warp_bytes<R, G>(), s>>>(a, warps);
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}

template <int R>
int launch_rhs(const Args& a, const float2* psi, float2* out, cudaStream_t s) {
  static std::once_flag once;
  std::call_once(once, [] {
    cudaFuncSetAttribute(schrodinger_rhs_kernel<R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         Warp<R>::BYTES);
  });
  schrodinger_rhs_kernel<R><<<(unsigned)a.batch, 32, Warp<R>::BYTES, s>>>(a, psi, out);
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}

int check(const dqb_dense_problem* p, int max_n) {
  if (!p) return DQB_ERR_INVALID_ARGUMENT;
  if (p->n < 1 || p->n_jumps != 0 || p->n_exp < 0 || p->n_tsave < 1 || p->batch < 0) return DQB_ERR_INVALID_ARGUMENT;
  if (p->batch >= (int64_t)0x7fffffff) return DQB_ERR_INVALID_ARGUMENT;
  if (!p->H || !p->rho0 || !p->tsave || (p->n_exp > 0 && !p->E)) return DQB_ERR_INVALID_ARGUMENT;
  if (p->n > max_n) return DQB_ERR_UNSUPPORTED;
  return DQB_OK;
}

int check_run(const dqb_dense_problem* p, const dqb_ode_options* o, const dqb_outputs* out, int max_n) {
  int rc = check(p, max_n);
  if (rc) return rc;
  if (!o || !out || !out->states || !out->infos || !out->status || (p->n_exp > 0 && !out->expects))
    return DQB_ERR_INVALID_ARGUMENT;
  if (o->method != DQB_METHOD_TSIT5 && o->method != DQB_METHOD_DOPRI5) return DQB_ERR_INVALID_ARGUMENT;
  if (!(o->rtol >= 0) || !(o->atol >= 0) || o->max_steps < 0) return DQB_ERR_INVALID_ARGUMENT;
  return DQB_OK;
}

Args make(const dqb_dense_problem* p) {
  Args a;
  a.mode = kSchrodinger;
  a.AT = nullptr;
  a.n = p->n;
  a.nE = p->n_exp;
  a.ntsave = p->n_tsave;
  a.batch = p->batch;
  a.H = (const float2*)p->H;
  a.psi0 = (const float2*)p->rho0;
  a.E = (const float2*)p->E;
  a.tsave = p->tsave;
  a.Hidx = p->H_index;
  a.pidx = p->rho0_index;
  a.states = a.expects = nullptr;
  a.infos = a.status = nullptr;
  a.counter = nullptr;
  return a;
}

}  // namespace se
}  // namespace dqb

using namespace dqb;

extern "C" size_t dqb_sesolve_dense_workspace_size(void) { return 256; }

static int run(se::Args& a, const dqb_dense_problem* p, const dqb_ode_options* o, const dqb_outputs* out,
               void* workspace, size_t workspace_bytes, cudaStream_t s) {
  if (p->batch == 0) return DQB_OK;
  if (!workspace || workspace_bytes < 256) return DQB_ERR_WORKSPACE_TOO_SMALL;
  a.states = (float2*)out->states;
  a.expects = (float2*)out->expects;
  a.infos = out->infos;
  a.status = out->status;
  a.counter = (unsigned int*)workspace;
  a.o = make_ctrl(*o);
  switch (se::rows_per_lane(p->n)) {
    case 1: return se::launch<1, false>(a, s);
    case 2: return se::launch<2, false>(a, s);
    case 4: return se::launch<4, false>(a, s);
    default: return se::launch<8, true>(a, s);
  }
}

extern "C" int dqb_sesolve_dense(const dqb_dense_problem* p, const dqb_ode_options* o, const dqb_outputs* out,
                                 void* workspace, size_t workspace_bytes, void* stream) {
  int rc = se::check_run(p, o, out, 128);
  if (rc) return rc;
  se::Args a = se::make(p);
  return run(a, p, o, out, workspace, workspace_bytes, (cudaStream_t)stream);
}

extern "C" int dqb_mesolve_vectorized(const dqb_dense_problem* p, const void* superop_t, const dqb_ode_options* o,
                                      const dqb_outputs* out, void* workspace, size_t workspace_bytes,
                                      void* stream) {
  int rc = se::check_run(p, o, out, 256);
  if (rc) return rc;
  if (!superop_t) return DQB_ERR_INVALID_ARGUMENT;
  se::Args a = se::make(p);
  a.mode = se::kLinear;
  a.AT = (const float2*)superop_t;
  return run(a, p, o, out, workspace, workspace_bytes, (cudaStream_t)stream);
}

extern "C" int dqb_schrodinger_rhs_dense(const dqb_dense_problem* p, const void* psi, void* outp, void* stream) {
  int rc = se::check(p, 128);
  if (rc) return rc;
  if (!psi || !outp) return DQB_ERR_INVALID_ARGUMENT;
  if (p->batch == 0) return DQB_OK;
  se::Args a = se::make(p);
  cudaStream_t s = (cudaStream_t)stream;
  switch (se::rows_per_lane(p->n)) {
    case 1: return se::launch_rhs<1>(a, (const float2*)psi, (float2*)outp, s);
    case 2: return se::launch_rhs<2>(a, (const float2*)psi, (float2*)outp, s);
    default: return se::launch_rhs<4>(a, (const float2*)psi, (float2*)outp, s);
  }
}
