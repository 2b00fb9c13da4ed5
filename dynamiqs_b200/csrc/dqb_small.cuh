// The per-instance adaptive Runge-Kutta solve of the persistent n <= 64 kernels, shared by
// the CUDA-core kernel (dqb_dense_small.cu) and the tensor-core kernel
// (dqb_dense_small_tc.cu).  The two differ only in how one right-hand side is evaluated,
// which they supply as an "engine":
//
//   struct Engine {
//     // Operators of the instance into shared memory (Hnh = -iH - 1/2 sum L^+L built
//     // there); ends with a barrier.
//     __device__ void load(const InstView& a);
//     // X[e] = x_of(e) for every e = i * NP + j (i, j < NP); when `also` is not null,
//     // also[e] = X[e]; then out[e] = f(t, X)[e] for every e (zero outside n x n).
//     // Every thread of the block calls it; it ends with a barrier.
//     template <class F> __device__ void rhs(F x_of, float2* also, float2* out, double t);
//     // True once a bounded wait has run out (the tensor-core engine); the instance then
//     // ends with DQB_INST_NONFINITE and the kernel stops taking new instances.
//     __device__ bool failed() const;
//     // Compile-time features: discontinuity times in the controller (time-dependent H),
//     // and the gradient tape; solves without them carry none of their code.
//     static constexpr bool kJumps, kTape;
//   };
//
// The loop follows what dynamiqs obtains from diffrax (dynamiqs/integrators/core/
// diffrax_integrator.py:59-147): starting step, Tsit5 / Dopri5 stages with FSAL, FP64
// embedded-error norm, integral controller, dense output at every tsave point crossed
// by an accepted step, SaveAt(t1=True) when only the final state is kept.
#pragma once

#include "dqb_common.cuh"

namespace dqb {

constexpr int kSmallThreads = 256;
constexpr int kSlotMats = 9;  // y, y1, k1..k7

// Time-dependent part of H (dqb_td_hamiltonian), by value in the kernel arguments (the
// terms and the discontinuity helpers are in dqb_common.cuh).
struct TdArgs {
  int M;                 // number of terms (0: constant H)
  const float2* ops;     // [M, n, n]
  TdTerm term[DQB_TD_MAX_TERMS];
  int n_jump;
  const double* jump_ts;
};

struct DenseSmallArgs {
  int n, K, nE, ntsave;
  long long batch;
  const float2* H;
  const float2* L;
  const float2* rho0;
  const float2* E;
  int rho0_is_ket;
  const double* tsave;
  const int* Hidx;
  const int* Lidx;
  const int* ridx;
  float2* states;
  float2* expects;
  int* infos;
  int* status;
  float2* slots;
  unsigned int* counter;
  const int* order;  // start order of the instances, or null (0, 1, 2, ...)
  CtrlOpts o;
  TdArgs td;
  // gradient tape (or null): per instance, the start time, size and starting state of
  // every accepted step, at most tape_cap of them
  double* tape_t;
  double* tape_h;
  float2* tape_y;
  int tape_cap;
};

struct Ctrl {
  double t, tnext, h, t1, dtnew, dt_prop;
  int made_jump;
  float w[7];
  int keep, run, status, save_idx;
  long long nsteps, nacc, nrej;
  long long inst;
  int sy, sy1, sk[7];
};

// Everything one instance's solve reads and writes (pointers at the instance's own data).
struct InstView {
  int n, K, nE, ntsave, is_ket, save_states;
  double t0;
  const float2* H;     // n x n
  const float2* L;     // K x n x n
  const float2* rho0;  // n x n, or n x 1 when is_ket
  const float2* E;     // nE x n x n
  const double* tsave;
  float2* states;      // nsave x n x n
  float2* expects;     // nE x ntsave
  int* infos;          // 3
  int* status;         // 1
  const volatile int* cancel;  // nonzero: stop (ragged launches), or null
  long long inst;      // index of the instance in its batch
  int n_jump;          // discontinuity times (the controller's jump_ts)
  const double* jump_ts;
  double* tape_t;      // gradient tape of the instance (null: none)
  double* tape_h;
  float2* tape_y;      // the batch's tape states: [batch, tape_cap, NP, NP]
  int tape_cap;
};

__device__ __forceinline__ InstView view_of(const DenseSmallArgs& a, long long inst) {
  InstView v;
  v.inst = inst;
  v.cancel = nullptr;
  v.n_jump = a.td.n_jump;
  v.jump_ts = a.td.jump_ts;
  v.tape_cap = a.tape_cap;
  v.tape_t = a.tape_t ? a.tape_t + inst * a.tape_cap : nullptr;
  v.tape_h = a.tape_h ? a.tape_h + inst * a.tape_cap : nullptr;
  v.tape_y = a.tape_y;  // the whole tape: solve_one offsets it by inst * tape_cap * NP^2
  const int n = a.n;
  const long long nn = (long long)n * n;
  const long long hi = a.Hidx ? a.Hidx[inst] : inst;
  const long long li = a.Lidx ? a.Lidx[inst] : inst;
  const long long ri = a.ridx ? a.ridx[inst] : inst;
  v.n = n;
  v.K = a.K;
  v.nE = a.nE;
  v.ntsave = a.ntsave;
  v.is_ket = a.rho0_is_ket;
  v.save_states = a.o.save_states;
  v.t0 = a.o.t0;
  v.H = a.H + hi * nn;
  v.L = a.L + li * a.K * nn;
  v.rho0 = a.rho0 + ri * (a.rho0_is_ket ? (long long)n : nn);
  v.E = a.E;
  v.tsave = a.tsave;
  v.states = a.states ? a.states + inst * (a.o.save_states ? a.ntsave : 1) * nn : nullptr;
  v.expects = a.expects ? a.expects + inst * a.nE * a.ntsave : nullptr;
  v.infos = a.infos ? a.infos + inst * 3 : nullptr;
  v.status = a.status ? a.status + inst : nullptr;
  return v;
}

// Write the state at save index `sidx` (y + sum_q cw[q] k_q when `interp`, else y)
// and its expectation values tr(E_m rho) = sum_ij E_m[j][i] rho[i][j] (FP64 sums).
template <int NP>
__device__ void save_point(const InstView& v, int sidx, const float2* __restrict__ yv,
                           float2* const (&kk)[7], const float (&cw)[7], bool interp, double* red) {
  constexpr int NN = NP * NP;
  const int n = v.n;
  for (int m0 = 0; m0 == 0 || m0 < v.nE; m0 += 8) {
    const int mc = v.nE - m0 < 8 ? v.nE - m0 : 8;
    double er[8], ei[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) er[m] = ei[m] = 0.0;
    for (int e = threadIdx.x; e < NN; e += blockDim.x) {
      const int i = e / NP, j = e % NP;
      if (i >= n || j >= n) continue;
      float2 val = yv[e];
      if (interp) {
#pragma unroll
        for (int q = 0; q < 7; ++q) val = caxpy(cw[q], kk[q][e], val);
      }
      if (m0 == 0 && v.save_states) v.states[((long long)sidx * n + i) * n + j] = val;
#pragma unroll
      for (int m = 0; m < 8; ++m) {
        if (m < mc) {
          const float2 ev = v.E[((long long)(m0 + m) * n + j) * n + i];
          er[m] += (double)ev.x * val.x - (double)ev.y * val.y;
          ei[m] += (double)ev.x * val.y + (double)ev.y * val.x;
        }
      }
    }
    for (int m = 0; m < mc; ++m) {
      const double sr = block_sum(er[m], red);
      const double si = block_sum(ei[m], red);
      if (threadIdx.x == 0) v.expects[(m0 + m) * v.ntsave + sidx] = make_float2((float)sr, (float)si);
    }
  }
}

// One instance's whole solve; `slot` holds kSlotMats NP x NP complex64 matrices.
template <int NP, class Engine>
__device__ void solve_one(Engine& eng, const InstView& a, const CtrlOpts& o, float2* slot, double* red,
                          Ctrl& ctl) {
  constexpr int NN = NP * NP;
  const int tid = threadIdx.x;
  const int n = a.n;
  const Tableau& T = c_tab[o.method];
  const double inv_nn = 1.0 / (double(n) * double(n));

  // ---- operators ------------------------------------------------------------------
  eng.load(a);

  // ---- initial state (todm for kets) and hermiticity check (rtol = atol = 1e-5) ----
  if (tid == 0) {
    ctl.sy = 0;
    ctl.sy1 = 1;
    for (int j = 0; j < 7; ++j) ctl.sk[j] = 2 + j;
    ctl.status = DQB_INST_OK;
    ctl.nsteps = ctl.nacc = ctl.nrej = 0;
    ctl.save_idx = 0;
  }
  __syncthreads();
  float2* y = slot + ctl.sy * NN;
  int bad = 0;
  for (int e = tid; e < NN; e += blockDim.x) {
    const int i = e / NP, j = e % NP;
    float2 v = make_float2(0.f, 0.f);
    if (i < n && j < n) {
      if (a.is_ket) {
        const float2* psi = a.rho0;
        v = cmul(psi[i], cconj(psi[j]));
      } else {
        const float2* r0 = a.rho0;
        v = r0[i * n + j];
        if (o.check_hermitian) {
          const float2 u = cconj(r0[j * n + i]);
          const float d = cabsf(make_float2(v.x - u.x, v.y - u.y));
          if (!(d <= 1e-5f + 1e-5f * cabsf(u))) bad = 1;
        }
      }
    }
    y[e] = v;
  }
  bad = __syncthreads_or(bad);
  if (bad) {
    if (tid == 0) {
      a.infos[0] = a.infos[1] = a.infos[2] = 0;
      __threadfence_system();  // status last: a caller may poll it from the host
      a.status[0] = DQB_INST_NOT_HERMITIAN;
    }
    return;
  }

  // ---- starting step (Hairer-Norsett-Wanner, RMS norm) --------------------------------
  const double t1 = a.tsave[a.ntsave - 1];
  float2* k1 = slot + ctl.sk[0] * NN;
  float2* kscr = slot + ctl.sk[1] * NN;
  eng.rhs([&](int e) { return y[e]; }, nullptr, k1, a.t0);
  double s0 = 0.0, s1 = 0.0;
  for (int e = tid; e < NN; e += blockDim.x) {
    const float2 yv = y[e], fv = k1[e];
    const double sc = o.atol + o.rtol * (double)cabsf(yv);
    s0 += (double)cabs2f(yv) / (sc * sc);
    s1 += (double)cabs2f(fv) / (sc * sc);
  }
  s0 = block_sum(s0, red);
  s1 = block_sum(s1, red);
  const double d0 = sqrt(s0 * inv_nn), d1 = sqrt(s1 * inv_nn);
  const double h0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : 0.01 * d0 / d1;
  const float h0f = (float)h0;
  eng.rhs([&](int e) { return caxpy(h0f, k1[e], y[e]); }, nullptr, kscr, a.t0 + h0);
  double s2 = 0.0;
  for (int e = tid; e < NN; e += blockDim.x) {
    const float2 yv = y[e], f0 = k1[e], f1 = kscr[e];
    const double sc = o.atol + o.rtol * (double)cabsf(yv);
    const double dx = (double)f1.x - (double)f0.x, dy = (double)f1.y - (double)f0.y;
    s2 += (dx * dx + dy * dy) / (sc * sc);
  }
  s2 = block_sum(s2, red);
  if (tid == 0) {
    const double d2 = sqrt(s2 * inv_nn) / h0;
    const double md = d1 > d2 ? d1 : d2;
    const double h1 = md <= 1e-15 ? fmax(1e-6, h0 * 1e-3) : pow(0.01 / md, 0.25);
    const double dt = fmin(100.0 * h0, h1);
    ctl.t = a.t0;
    ctl.t1 = t1;
    ctl.dt_prop = dt;
    ctl.made_jump = 0;
    if constexpr (Engine::kJumps) {
      ctl.tnext = next_trial(a.jump_ts, a.n_jump, a.t0, dt, t1, true, ctl.made_jump);
    } else {
      double tn = a.t0 + dt;
      if (tn > t1 - 1e-10) tn = t1;
      ctl.tnext = tn < t1 ? tn : t1;
    }
    ctl.run = a.t0 < t1;
    if (eng.failed()) {
      ctl.status = DQB_INST_NONFINITE;
      ctl.run = 0;
    }
  }
  __syncthreads();

  // ---- main loop ----------------------------------------------------------------------
  // (a degenerate interval t1 <= t0 never enters it; the save loop after it then writes
  // the initial state at every save point)
  while (ctl.run) {
    if (ctl.nsteps >= o.max_steps) {
      if (tid == 0) ctl.status = DQB_INST_MAX_STEPS;
      break;
    }
    if (a.cancel != nullptr && (ctl.nsteps & 15) == 0) {  // a caller's stop request
      __syncthreads();  // every thread has read ctl before thread 0 may change it
      if (tid == 0 && *a.cancel != 0) ctl.status = DQB_INST_CANCELLED;
      __syncthreads();
      if (ctl.status == DQB_INST_CANCELLED) break;
    }
    const double h = ctl.tnext - ctl.t;
    float2* yv = slot + ctl.sy * NN;
    float2* y1 = slot + ctl.sy1 * NN;
    float2* kk[7];
#pragma unroll
    for (int j = 0; j < 7; ++j) kk[j] = slot + ctl.sk[j] * NN;

    // stages 2..6
    for (int s = 1; s < 6; ++s) {
      float cf[5];
#pragma unroll
      for (int j = 0; j < 5; ++j) cf[j] = (float)(h * T.a[s][j]);
      eng.rhs(
          [&](int e) {
            float2 x = yv[e];
#pragma unroll
            for (int j = 0; j < 5; ++j)
              if (j < s) x = caxpy(cf[j], kk[j][e], x);
            return x;
          },
          nullptr, kk[s], ctl.t + T.c[s] * h);
    }
    // y1 (FSAL stage input) and k7
    {
      float cf[6];
#pragma unroll
      for (int j = 0; j < 6; ++j) cf[j] = (float)(h * T.b[j]);
      eng.rhs(
          [&](int e) {
            float2 x = yv[e];
#pragma unroll
            for (int j = 0; j < 6; ++j) x = caxpy(cf[j], kk[j][e], x);
            return x;
          },
          y1, kk[6], ctl.tnext);
    }
    // embedded error, FP64 accumulation
    double se = 0.0;
    {
      double cb[7];
#pragma unroll
      for (int j = 0; j < 7; ++j) cb[j] = h * T.btilde[j];
#pragma unroll 4
      for (int e = tid; e < NN; e += blockDim.x) {
        double ex = 0.0, ey = 0.0;
#pragma unroll
        for (int j = 0; j < 7; ++j) {
          const float2 kv = kk[j][e];
          ex = fma(cb[j], (double)kv.x, ex);
          ey = fma(cb[j], (double)kv.y, ey);
        }
        const float ya = cabsf(yv[e]), y1a = cabsf(y1[e]);
        const double sc = o.atol + o.rtol * (double)(ya > y1a ? ya : y1a);
        se += (ex * ex + ey * ey) / (sc * sc);
      }
    }
    se = block_sum(se, red);
    if (tid == 0) {
      const double err = eng.failed() ? (double)NAN : sqrt(se * inv_nn);
      ctl.nsteps += 1;
      if (!(err < INFINITY)) {
        ctl.status = DQB_INST_NONFINITE;
        ctl.nrej += 1;
        ctl.run = 0;
        ctl.keep = 0;
      } else {
        const bool keep = err < 1.0;
        ctl.keep = keep;
        if (keep) ctl.nacc += 1; else ctl.nrej += 1;
        // after a step clipped at a discontinuity the controller scales its proposal
        const double base = (Engine::kJumps && ctl.made_jump) ? ctl.dt_prop : h;
        ctl.dtnew = base * step_factor(o, err, keep);
      }
    }
    __syncthreads();
    if (ctl.status != DQB_INST_OK) break;

    if (ctl.keep) {
      // gradient tape: the accepted step's start time, size and starting state
      if (Engine::kTape && a.tape_y && ctl.nacc <= a.tape_cap) {
        const long long idx = ctl.nacc - 1;
        if (tid == 0) {
          a.tape_t[idx] = ctl.t;
          a.tape_h[idx] = h;
        }
        float2* dst = a.tape_y + (a.inst * (long long)a.tape_cap + idx) * NN;
        for (int e = tid; e < NN; e += blockDim.x) dst[e] = yv[e];
      }
      // dense output at every save time in (t, tnext]
      while (ctl.save_idx < a.ntsave && a.tsave[ctl.save_idx] <= ctl.tnext) {
        if (tid == 0) {
          double w[7];
          const double theta = h > 0.0 ? (a.tsave[ctl.save_idx] - ctl.t) / h : 1.0;
          dense_weights(o.method, theta, w);
          for (int j = 0; j < 7; ++j) ctl.w[j] = (float)(h * w[j]);
        }
        __syncthreads();
        float cw[7];
#pragma unroll
        for (int j = 0; j < 7; ++j) cw[j] = ctl.w[j];
        save_point<NP>(a, ctl.save_idx, yv, kk, cw, true, red);
        __syncthreads();
        if (tid == 0) ctl.save_idx += 1;
        __syncthreads();
      }
      if (tid == 0) {
        int tmp = ctl.sy;
        ctl.sy = ctl.sy1;
        ctl.sy1 = tmp;
        tmp = ctl.sk[0];
        ctl.sk[0] = ctl.sk[6];
        ctl.sk[6] = tmp;
        // a step that ended just before a discontinuity: the next starts on it
        ctl.t = (Engine::kJumps && ctl.made_jump) ? nextafter(ctl.tnext, INFINITY) : ctl.tnext;
      }
      if constexpr (Engine::kJumps) {
        __syncthreads();
        if (ctl.made_jump && ctl.t < ctl.t1) {  // first stage re-evaluated across the jump
          const float2* yn = slot + ctl.sy * NN;
          eng.rhs([&](int e) { return yn[e]; }, nullptr, slot + ctl.sk[0] * NN, ctl.t);
        }
      }
    }
    __syncthreads();
    if (tid == 0) {
      if constexpr (Engine::kJumps) {
        ctl.dt_prop = ctl.dtnew;
        ctl.tnext = next_trial(a.jump_ts, a.n_jump, ctl.t, ctl.dtnew, ctl.t1, ctl.keep, ctl.made_jump);
      } else {
        ctl.tnext = next_tend(ctl.t, ctl.dtnew, ctl.t1, ctl.keep);
      }
      ctl.run = ctl.t < ctl.t1;
    }
    __syncthreads();
  }
  __syncthreads();

  // saves left over (t1 <= t0: every save is the initial state)
  if (ctl.status == DQB_INST_OK) {
    const float2* yv = slot + ctl.sy * NN;
    while (ctl.save_idx < a.ntsave && a.tsave[ctl.save_idx] <= ctl.t) {
      float2* kk[7];
      float cw[7];
#pragma unroll
      for (int j = 0; j < 7; ++j) {
        kk[j] = slot + ctl.sk[j] * NN;
        cw[j] = 0.f;
      }
      save_point<NP>(a, ctl.save_idx, yv, kk, cw, false, red);
      __syncthreads();
      if (tid == 0) ctl.save_idx += 1;
      __syncthreads();
    }
  }
  // final state when only the last state is kept (SubSaveAt(t1=True))
  if (!a.save_states) {
    const float2* yv = slot + ctl.sy * NN;
    for (int e = tid; e < NN; e += blockDim.x) {
      const int i = e / NP, j = e % NP;
      if (i < n && j < n) a.states[(long long)i * n + j] = yv[e];
    }
  }
  // Every output of the instance is written before its status, with a system-scope fence
  // in between, so that a caller polling the status word in host-mapped memory (the
  // serving loop) can hand the result out as soon as the word changes.
  __threadfence();
  __syncthreads();
  if (tid == 0) {
    a.infos[0] = (int)ctl.nsteps;
    a.infos[1] = (int)ctl.nacc;
    a.infos[2] = (int)ctl.nrej;
    __threadfence_system();
    a.status[0] = ctl.status;
  }
}

}  // namespace dqb
