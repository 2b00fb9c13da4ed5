// Batched RK stepper for problems too large for one CTA (n > 64 dense, or sparse DIA).
//
// One RK step of every running instance is a fixed sequence of grid-wide kernels:
//   for s = 2..6:  combine  X   = y + h sum_{j<s} a_sj k_j        (elementwise)
//                  rhs      k_s = f(X)                            (DIA stencil or GEMMs)
//                  combine  y1  = y + h sum_{j<7} b_j k_j ; rhs k7 = f(y1)
//                  error    acc += |h sum_j btilde_j k_j|^2 / sc^2 (FP64 atomics)
//                  control  (one thread per instance, FP64): accept / reject, save range
//                  save     dense output at the tsave points crossed, tr(E rho) sums
//                  commit   swap y <-> y1 and k1 <-> k7 on accept, next trial step
// The sequence is the body of a CUDA-graph WHILE node whose condition the commit kernel
// sets to "some instance is still running", so a whole batched solve is one graph launch
// with no host round trip.  Every instance keeps its own t, dt, accept/reject state and
// step counters; finished instances are skipped by every kernel.  The loop ends because
// every iteration advances each running instance's attempted-step counter, which is
// bounded by max_steps, and the commit kernel also stops after max_steps + 2 iterations.
#pragma once

#include <cuda_runtime.h>

#include "dqb_common.cuh"

namespace dqb {
namespace big {

constexpr int kSlots = 10;  // y, y1, k1..k7, X
constexpr int kInactive = 99;  // status of a capacity slot beyond the wave's instance count
constexpr int kX = 9;
constexpr int kElemThreads = 256;

struct Inst {
  double t, tnext, h, dtnew, t1, h0;
  double acc[3];  // error / starting-step norm accumulators
  int status, run, keep, save_idx, save_lo, save_hi, herm_bad, retired;
  long long nsteps, nacc, nrej;
  int sy, sy1, sk[7];
  // Krylov form (kry_* kernels): sk[q - 1] holds u_q = (tau L)^q y for q = 1..7, except
  // that the true u_1 is sig1 times the stored one; kvalid = how many of u_0..u_7 are
  // current; sf = the slot that receives tau L y1 (the next step's u_1)
  double tau, sig1;
  int kvalid, sf;
  // discontinuities (time-dependent H): dt_prop = the controller's proposal that the last
  // trial step was clipped from; made_jump = that step ends just before a discontinuity;
  // refresh = the accepted step crossed one, so the first stage must be re-evaluated
  double dt_prop;
  int made_jump, refresh;
  // the instance's own problem data and outputs (shared arrays or a ragged descriptor)
  int nts, nE, save_states, is_ket;
  const double* ts;
  const float2* rho0;
  const float2* E;
  float2* states;
  float2* expects;
  double2* eacc;
  int* infos;
  int* status_out;
  const volatile int* cancel;  // ragged launches: the caller's stop word, or null
};

struct Common {
  int n;
  long long nn;  // n * n
  int B, nE, ntsave, form, save_states, rho0_is_ket;
  CtrlOpts o;
  const double* tsave;
  Inst* inst;
  float2* mats;    // [B][kSlots][nn]
  double2* eacc;   // [B][nE][ntsave]
  float2* states;  // [B][nsave][n][n]
  float2* expects; // [B][nE][ntsave]
  int* infos;
  int* status;
  const float2* E;  // [nE][n][n]
  const float2* rho0;
  const int* ridx;
  long long* iter;  // graph-loop iteration counter
  const dqb_ragged_instance* rag;  // per-instance descriptors, or null
  long long eacc_stride;           // expectation accumulators per instance (ragged)
  const int* count_dev;            // live instances (<= B) read at run time, or null
  int n_jump;                      // discontinuity times of a time-dependent H (jump_ts)
  const double* jump_ts;           // device float64 [n_jump], ascending
};

__device__ __forceinline__ float2* slot(const Common& c, int b, int s) {
  return c.mats + ((long long)b * kSlots + s) * c.nn;
}

__device__ __forceinline__ void block_atomic_add(double v, double* dst, double* red) {
  v = block_sum(v, red);
  if (threadIdx.x == 0) atomicAdd(dst, v);
}

// Time at which instance I evaluates the right-hand side `which` of a time-dependent H,
// or false when it evaluates none: 1..5 the stage input x_s at t + c_s h, 6 y1 at the
// step's end, 7 the first stage re-evaluated after a discontinuity (refresh set), 8 the
// first stage at the start, 9 the starting-step probe at t + h0.
__device__ __forceinline__ bool td_stage_time(const Common& c, const Inst& I, int which, double* t) {
  if (which >= 8 ? I.status != DQB_INST_OK : (!I.run || (which == 7 && !I.refresh))) return false;
  const Tableau& T = c_tab[c.o.method];
  *t = which <= 5 ? I.t + T.c[which] * I.h : (which == 6 ? I.tnext : (which == 9 ? I.t + I.h0 : I.t));
  return true;
}

// ------------------------------------------------------------------------------------
// set-up
// ------------------------------------------------------------------------------------

// One thread per instance.
static __global__ void setup_kernel(Common c) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b == 0) *c.iter = 0;
  if (b >= c.B) return;
  Inst& I = c.inst[b];
  if (c.count_dev && b >= *c.count_dev) {  // unused capacity: every kernel skips it
    I.status = kInactive;
    I.retired = 0;
    I.run = 0;
    I.nts = I.nE = 0;
    I.save_idx = I.save_lo = I.save_hi = 0;
    I.herm_bad = 0;
    I.nsteps = I.nacc = I.nrej = 0;
    return;
  }
  if (c.rag) {
    const dqb_ragged_instance& r = c.rag[b];
    I.nts = r.n_tsave;
    I.nE = r.n_exp;
    I.save_states = r.save_states;
    I.is_ket = r.rho0_is_ket;
    I.ts = r.tsave;
    I.rho0 = (const float2*)r.rho0;
    I.E = (const float2*)r.E;
    I.states = (float2*)r.states;
    I.expects = (float2*)r.expects;
    I.eacc = c.eacc + (long long)b * c.eacc_stride;
    I.infos = r.infos;
    I.status_out = r.status;
    I.cancel = r.cancel;
    I.t = r.t0;
  } else {
    I.cancel = nullptr;
    const long long ri = c.ridx ? c.ridx[b] : b;
    I.nts = c.ntsave;
    I.nE = c.nE;
    I.save_states = c.save_states;
    I.is_ket = c.rho0_is_ket;
    I.ts = c.tsave;
    I.rho0 = c.rho0 + ri * (c.rho0_is_ket ? (long long)c.n : c.nn);
    I.E = c.E;
    I.states = c.states + (long long)b * (c.save_states ? c.ntsave : 1) * c.nn;
    I.expects = c.expects + (long long)b * c.nE * c.ntsave;
    I.eacc = c.eacc + (long long)b * c.nE * c.ntsave;
    I.infos = c.infos + 3 * b;
    I.status_out = c.status + b;
    I.t = c.o.t0;
  }
  I.t1 = I.ts[I.nts - 1];
  I.tnext = I.t1;
  I.h = I.dtnew = I.h0 = 0.0;
  I.acc[0] = I.acc[1] = I.acc[2] = 0.0;
  I.status = DQB_INST_OK;
  I.run = 0;
  I.keep = 0;
  I.save_idx = I.save_lo = I.save_hi = 0;
  I.herm_bad = 0;
  I.retired = 0;
  I.nsteps = I.nacc = I.nrej = 0;
  I.sy = 0;
  I.sy1 = 1;
  for (int j = 0; j < 7; ++j) I.sk[j] = 2 + j;
  I.tau = I.sig1 = 1.0;
  I.kvalid = 0;
  I.sf = kX;
  I.dt_prop = 0.0;
  I.made_jump = I.refresh = 0;
}

// grid (tiles, B): rho0 (or psi psi^+) into y, hermiticity check, expects sums zeroed.
static __global__ void load_rho0_kernel(Common c) {
  const int b = blockIdx.y;
  Inst& I = c.inst[b];
  if (I.status == kInactive) return;
  const int n = c.n;
  float2* y = slot(c, b, 0);
  int bad = 0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < c.nn;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e / n), j = (int)(e % n);
    float2 v;
    if (I.is_ket) {
      const float2* psi = I.rho0;
      v = cmul(psi[i], cconj(psi[j]));
    } else {
      const float2* r0 = I.rho0;
      v = r0[e];
      if (c.o.check_hermitian) {
        const float2 u = cconj(r0[(long long)j * n + i]);
        const float d = cabsf(make_float2(v.x - u.x, v.y - u.y));
        if (!(d <= 1e-5f + 1e-5f * cabsf(u))) bad = 1;
      }
    }
    y[e] = v;
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) I.herm_bad = 1;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)I.nE * I.nts;
       e += (long long)gridDim.x * blockDim.x)
    I.eacc[e] = make_double2(0.0, 0.0);
}

// ------------------------------------------------------------------------------------
// elementwise kernels: grid (tiles, B)
// ------------------------------------------------------------------------------------

// mode 0..4: X = y + h sum_{j<=mode} a[mode+1][j] k_j    (stage mode+2 input)
// mode 5:    y1 = y + h sum_{j<6} b_j k_j
// mode 6:    X = y + h0 k1                              (starting-step probe)
static __global__ void combine_kernel(Common c, int mode) {
  const int b = blockIdx.y;
  const Inst& I = c.inst[b];
  if (mode == 6) {
    if (I.status != DQB_INST_OK) return;
  } else if (!I.run) {
    return;
  }
  const Tableau& T = c_tab[c.o.method];
  float cf[6];
  int nterm;
  if (mode == 6) {
    cf[0] = (float)I.h0;
    nterm = 1;
  } else if (mode == 5) {
    for (int j = 0; j < 6; ++j) cf[j] = (float)(I.h * T.b[j]);
    nterm = 6;
  } else {
    for (int j = 0; j < 6; ++j) cf[j] = (float)(I.h * T.a[mode + 1][j]);
    nterm = mode + 1;
  }
  const float2* y = slot(c, b, I.sy);
  const float2* k[6];
  for (int j = 0; j < 6; ++j) k[j] = slot(c, b, I.sk[j]);
  float2* out = slot(c, b, mode == 5 ? I.sy1 : kX);
  if ((c.nn & 1) == 0 && (reinterpret_cast<uintptr_t>(c.mats) & 15) == 0) {
    // two complex values per 16-byte access (every slot starts on a 16-byte boundary when
    // the slot array does and n^2 is even): half the load instructions, twice the bytes in
    // flight per request
    const long long nn2 = c.nn >> 1;
    const float4* y4 = reinterpret_cast<const float4*>(y);
    float4* o4 = reinterpret_cast<float4*>(out);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn2;
         e += (long long)gridDim.x * blockDim.x) {
      float4 x = y4[e];
#pragma unroll
      for (int j = 0; j < 6; ++j)
        if (j < nterm) {
          const float4 v = reinterpret_cast<const float4*>(k[j])[e];
          x.x = fmaf(cf[j], v.x, x.x);
          x.y = fmaf(cf[j], v.y, x.y);
          x.z = fmaf(cf[j], v.z, x.z);
          x.w = fmaf(cf[j], v.w, x.w);
        }
      o4[e] = x;
    }
    return;
  }
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < c.nn;
       e += (long long)gridDim.x * blockDim.x) {
    float2 x = y[e];
#pragma unroll
    for (int j = 0; j < 6; ++j)
      if (j < nterm) x = caxpy(cf[j], k[j][e], x);
    out[e] = x;
  }
}

// Embedded-error accumulation: acc[0] += sum |h sum_j btilde_j k_j|^2 / sc^2.
static __global__ void error_kernel(Common c) {
  __shared__ double red[40];
  const int b = blockIdx.y;
  Inst& I = c.inst[b];
  if (!I.run) return;
  const Tableau& T = c_tab[c.o.method];
  double cb[7];
  for (int j = 0; j < 7; ++j) cb[j] = I.h * T.btilde[j];
  const float2* y = slot(c, b, I.sy);
  const float2* y1 = slot(c, b, I.sy1);
  const float2* k[7];
  for (int j = 0; j < 7; ++j) k[j] = slot(c, b, I.sk[j]);
  double s = 0.0;
  auto term = [&](float2 kv0, float2 kv1, float2 kv2, float2 kv3, float2 kv4, float2 kv5, float2 kv6,
                  float2 yv, float2 y1v) {
    const float2 kv[7] = {kv0, kv1, kv2, kv3, kv4, kv5, kv6};
    double ex = 0.0, ey = 0.0;
#pragma unroll
    for (int j = 0; j < 7; ++j) {
      ex = fma(cb[j], (double)kv[j].x, ex);
      ey = fma(cb[j], (double)kv[j].y, ey);
    }
    const float ya = cabsf(yv), y1a = cabsf(y1v);
    const double sc = c.o.atol + c.o.rtol * (double)(ya > y1a ? ya : y1a);
    return (ex * ex + ey * ey) / (sc * sc);
  };
  if ((c.nn & 1) == 0 && (reinterpret_cast<uintptr_t>(c.mats) & 15) == 0) {
    // two complex values per 16-byte access, as in combine_kernel
    const long long nn2 = c.nn >> 1;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn2;
         e += (long long)gridDim.x * blockDim.x) {
      float4 kv[7];
#pragma unroll
      for (int j = 0; j < 7; ++j) kv[j] = reinterpret_cast<const float4*>(k[j])[e];
      const float4 yv = reinterpret_cast<const float4*>(y)[e];
      const float4 y1v = reinterpret_cast<const float4*>(y1)[e];
#define DQB_LO(v) make_float2(v.x, v.y)
#define DQB_HI(v) make_float2(v.z, v.w)
      s += term(DQB_LO(kv[0]), DQB_LO(kv[1]), DQB_LO(kv[2]), DQB_LO(kv[3]), DQB_LO(kv[4]), DQB_LO(kv[5]),
                DQB_LO(kv[6]), DQB_LO(yv), DQB_LO(y1v));
      s += term(DQB_HI(kv[0]), DQB_HI(kv[1]), DQB_HI(kv[2]), DQB_HI(kv[3]), DQB_HI(kv[4]), DQB_HI(kv[5]),
                DQB_HI(kv[6]), DQB_HI(yv), DQB_HI(y1v));
#undef DQB_LO
#undef DQB_HI
    }
  } else {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < c.nn;
         e += (long long)gridDim.x * blockDim.x)
      s += term(k[0][e], k[1][e], k[2][e], k[3][e], k[4][e], k[5][e], k[6][e], y[e], y1[e]);
  }
  block_atomic_add(s, &I.acc[0], red);
}

// ------------------------------------------------------------------------------------
// hermitian-form elementwise kernels: upper-triangle tiles, mirrored writes
// ------------------------------------------------------------------------------------
//
// In the hermitian form every matrix the stepper combines -- y, the stages k_j (the
// right-hand sides write exactly hermitian outputs), the stage inputs, y1 and the Krylov
// basis -- is hermitian, so an elementwise pass needs to read only the tiles on and above
// the diagonal: each CTA takes one 32 x 32 tile (ti <= tj), computes it, writes it, and for
// ti < tj writes its conjugate transpose to tile (tj, ti) through shared memory (rows of 32
// contiguous values both ways).  Reads fall to a little over half; writes are unchanged.
// Diagonal tiles are computed whole and not mirrored.  Sums over all elements (the error
// norm) weight an off-diagonal tile twice: its mirror has the same magnitudes.
// grid (T (T + 1) / 2, B) with T = ceil(n / 32), 256 threads (32 x 8, 4 rows each).

constexpr int kHT = 32;

__device__ __forceinline__ int herm_row_start(int r, int T) { return r * T - r * (r - 1) / 2; }

__device__ __forceinline__ void herm_tile(int t, int T, int& ti, int& tj) {
  // t-th upper tile in row-major order of the upper triangle: row r holds T - r tiles and
  // starts at r T - r (r - 1) / 2; the root of that quadratic, then exact integer fix-ups
  const float b = 2.f * T + 1.f;
  int r = (int)((b - sqrtf(fmaxf(b * b - 8.f * t, 0.f))) * 0.5f);
  r = r < 0 ? 0 : (r > T - 1 ? T - 1 : r);
  while (r > 0 && herm_row_start(r, T) > t) --r;
  while (r < T - 1 && herm_row_start(r + 1, T) <= t) ++r;
  ti = r;
  tj = r + (t - herm_row_start(r, T));
}

// A thread's four elements of a 32 x 32 tile.  VEC = false: rows ly + 8q (ly = tid / 32),
// column tid % 32.  VEC = true (n even): rows ly + 16q (ly = tid / 16, q < 2), columns
// 2 (tid % 16) and the next, read and written as one 16-byte access per row; element
// 2q + p is row q, column p.
template <bool VEC>
struct HTile {
  int lx, ly;
  __device__ __forceinline__ HTile() : lx(VEC ? threadIdx.x & 15 : threadIdx.x & 31),
                                       ly(VEC ? threadIdx.x >> 4 : threadIdx.x >> 5) {}
  __device__ __forceinline__ int row(int q) const { return VEC ? ly + 16 * (q >> 1) : ly + 8 * q; }
  __device__ __forceinline__ int col(int q) const { return VEC ? 2 * lx + (q & 1) : lx; }
};

// Loads the thread's four elements of tile (ti, tj) of M (zeros outside the matrix).
template <bool VEC>
__device__ __forceinline__ void htile_load(const float2* __restrict__ M, int n, int ti, int tj, float2 (&v)[4]) {
  const HTile<VEC> t;
  if (VEC) {
#pragma unroll
    for (int q = 0; q < 4; q += 2) {
      const int r = ti * kHT + t.row(q), c0 = tj * kHT + t.col(q);
      float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
      if (r < n && c0 < n) x = *reinterpret_cast<const float4*>(M + (long long)r * n + c0);
      v[q] = make_float2(x.x, x.y);
      v[q + 1] = make_float2(x.z, x.w);
    }
  } else {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = ti * kHT + t.row(q), c = tj * kHT + t.col(q);
      v[q] = (r < n && c < n) ? M[(long long)r * n + c] : make_float2(0.f, 0.f);
    }
  }
}

// Whether the thread's element q lies inside the matrix.
template <bool VEC>
__device__ __forceinline__ bool htile_in(int n, int ti, int tj, int q) {
  const HTile<VEC> t;
  return ti * kHT + t.row(q) < n && tj * kHT + t.col(q) < n;
}

// Writes v at tile (ti, tj) and, for ti < tj, its conjugate transpose at (tj, ti) through
// the 32 x 33 shared tile `sh`.
template <bool VEC>
__device__ __forceinline__ void herm_store(float2* __restrict__ out, int n, int ti, int tj, const float2 (&v)[4],
                                           float2 (*sh)[kHT + 1]) {
  const HTile<VEC> t;
  if (VEC) {
#pragma unroll
    for (int q = 0; q < 4; q += 2) {
      const int r = ti * kHT + t.row(q), c0 = tj * kHT + t.col(q);
      if (r < n && c0 < n)
        *reinterpret_cast<float4*>(out + (long long)r * n + c0) = make_float4(v[q].x, v[q].y, v[q + 1].x, v[q + 1].y);
    }
  } else {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = ti * kHT + t.row(q), c = tj * kHT + t.col(q);
      if (r < n && c < n) out[(long long)r * n + c] = v[q];
    }
  }
  if (ti == tj) return;  // uniform over the block
  __syncthreads();       // the tile is free (a previous use has been read)
#pragma unroll
  for (int q = 0; q < 4; ++q) sh[t.row(q)][t.col(q)] = v[q];
  __syncthreads();
  // output row tj*32 + a, column ti*32 + b takes the conjugate of the tile's (b, a)
  if (VEC) {
#pragma unroll
    for (int q = 0; q < 4; q += 2) {
      const int a = t.row(q), b0 = t.col(q);
      const int r = tj * kHT + a, c0 = ti * kHT + b0;
      if (r < n && c0 < n) {
        const float2 w0 = cconj(sh[b0][a]), w1 = cconj(sh[b0 + 1][a]);
        *reinterpret_cast<float4*>(out + (long long)r * n + c0) = make_float4(w0.x, w0.y, w1.x, w1.y);
      }
    }
  } else {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int a = t.row(q), b = t.col(q);
      const int r = tj * kHT + a, c = ti * kHT + b;
      if (r < n && c < n) out[(long long)r * n + c] = cconj(sh[b][a]);
    }
  }
}

// combine_kernel for the hermitian form (same modes).
template <bool VEC>
static __global__ void combine_h_kernel(Common c, int mode) {
  __shared__ float2 sh[kHT][kHT + 1];
  const int b = blockIdx.y;
  const Inst& I = c.inst[b];
  if (mode == 6) {
    if (I.status != DQB_INST_OK) return;
  } else if (!I.run) {
    return;
  }
  const Tableau& Tb = c_tab[c.o.method];
  float cf[6];
  int nterm;
  if (mode == 6) {
    cf[0] = (float)I.h0;
    nterm = 1;
  } else if (mode == 5) {
    for (int j = 0; j < 6; ++j) cf[j] = (float)(I.h * Tb.b[j]);
    nterm = 6;
  } else {
    for (int j = 0; j < 6; ++j) cf[j] = (float)(I.h * Tb.a[mode + 1][j]);
    nterm = mode + 1;
  }
  const int n = c.n, T = (n + kHT - 1) / kHT;
  int ti, tj;
  herm_tile(blockIdx.x, T, ti, tj);
  float2 v[4], w[4];
  htile_load<VEC>(slot(c, b, I.sy), n, ti, tj, v);
#pragma unroll
  for (int j = 0; j < 6; ++j)
    if (j < nterm) {
      htile_load<VEC>(slot(c, b, I.sk[j]), n, ti, tj, w);
#pragma unroll
      for (int q = 0; q < 4; ++q) v[q] = caxpy(cf[j], w[q], v[q]);
    }
  herm_store<VEC>(slot(c, b, mode == 5 ? I.sy1 : kX), n, ti, tj, v, sh);
}

// error_kernel for the hermitian form: the same FP64 sum, off-diagonal tiles counted twice.
template <bool VEC>
static __global__ void error_h_kernel(Common c) {
  __shared__ double red[40];
  const int b = blockIdx.y;
  Inst& I = c.inst[b];
  if (!I.run) return;
  const Tableau& Tb = c_tab[c.o.method];
  const int n = c.n, T = (n + kHT - 1) / kHT;
  int ti, tj;
  herm_tile(blockIdx.x, T, ti, tj);
  double ex[4] = {0, 0, 0, 0}, ey[4] = {0, 0, 0, 0};
  float2 w[4];
#pragma unroll
  for (int j = 0; j < 7; ++j) {
    const double cb = I.h * Tb.btilde[j];
    htile_load<VEC>(slot(c, b, I.sk[j]), n, ti, tj, w);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      ex[q] = fma(cb, (double)w[q].x, ex[q]);
      ey[q] = fma(cb, (double)w[q].y, ey[q]);
    }
  }
  float2 yv[4], y1v[4];
  htile_load<VEC>(slot(c, b, I.sy), n, ti, tj, yv);
  htile_load<VEC>(slot(c, b, I.sy1), n, ti, tj, y1v);
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    if (htile_in<VEC>(n, ti, tj, q)) {
      const float ya = cabsf(yv[q]), y1a = cabsf(y1v[q]);
      const double sc = c.o.atol + c.o.rtol * (double)(ya > y1a ? ya : y1a);
      s += (ex[q] * ex[q] + ey[q] * ey[q]) / (sc * sc);
    }
  }
  if (ti != tj) s *= 2.0;
  block_atomic_add(s, &I.acc[0], red);
}

// Starting-step norms.  phase 0: acc[0] += |y/sc|^2, acc[1] += |k1/sc|^2;
// phase 1: acc[2] += |(k2 - k1)/sc|^2 (k2 = f(y + h0 k1));
// phase 2 (Krylov form, k2 holding L k1): acc[2] += |h0 L k1 / sc|^2, the same quantity
// for a linear right-hand side.
static __global__ void init_norm_kernel(Common c, int phase) {
  __shared__ double red[40];
  const int b = blockIdx.y;
  Inst& I = c.inst[b];
  if (I.status != DQB_INST_OK) return;
  const float2* y = slot(c, b, I.sy);
  const float2* k1 = slot(c, b, I.sk[0]);
  const float2* k2 = slot(c, b, I.sk[1]);
  double s0 = 0.0, s1 = 0.0;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < c.nn;
       e += (long long)gridDim.x * blockDim.x) {
    const float2 yv = y[e];
    const double sc = c.o.atol + c.o.rtol * (double)cabsf(yv);
    const float2 f0 = k1[e];
    if (phase == 0) {
      s0 += (double)cabs2f(yv) / (sc * sc);
      s1 += (double)cabs2f(f0) / (sc * sc);
    } else if (phase == 1) {
      const float2 f1 = k2[e];
      const double dx = (double)f1.x - f0.x, dy = (double)f1.y - f0.y;
      s0 += (dx * dx + dy * dy) / (sc * sc);
    } else {
      const float2 f1 = k2[e];
      const double dx = I.h0 * f1.x, dy = I.h0 * f1.y;
      s0 += (dx * dx + dy * dy) / (sc * sc);
    }
  }
  if (phase == 0) {
    block_atomic_add(s0, &I.acc[0], red);
    block_atomic_add(s1, &I.acc[1], red);
  } else {
    block_atomic_add(s0, &I.acc[2], red);
  }
}

// One thread per instance.  phase 0: hermiticity verdict and h0 from d0, d1.
// phase 1: first trial step (Hairer-Norsett-Wanner).
static __global__ void init_ctrl_kernel(Common c, int phase) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= c.B) return;
  Inst& I = c.inst[b];
  const double inv_nn = 1.0 / (double)c.nn;
  if (I.status == kInactive) return;
  if (phase == 0) {
    if (I.herm_bad) I.status = DQB_INST_NOT_HERMITIAN;
    const double d0 = sqrt(I.acc[0] * inv_nn), d1 = sqrt(I.acc[1] * inv_nn);
    I.h0 = (d0 < 1e-5 || d1 < 1e-5) ? 1e-6 : 0.01 * d0 / d1;
    I.acc[0] = d0;
    I.acc[1] = d1;
    I.acc[2] = 0.0;
  } else {
    if (I.status != DQB_INST_OK) {
      I.run = 0;
      return;
    }
    const double d1 = I.acc[1];
    const double d2 = sqrt(I.acc[2] * inv_nn) / I.h0;
    const double md = d1 > d2 ? d1 : d2;
    const double h1 = md <= 1e-15 ? fmax(1e-6, I.h0 * 1e-3) : pow(0.01 / md, 0.25);
    const double dt = fmin(100.0 * I.h0, h1);
    I.dt_prop = dt;
    I.tnext = next_trial(c.jump_ts, c.n_jump, I.t, dt, I.t1, true, I.made_jump);
    I.h = I.tnext - I.t;
    I.run = I.t < I.t1;
    I.acc[0] = I.acc[1] = I.acc[2] = 0.0;
    // Krylov form: the basis of the first step is scaled by its trial step, and the stored
    // u_1 is L y (sk[0], from the starting-step probe)
    I.tau = I.h;
    I.sig1 = I.h;
    I.kvalid = 2;
  }
}

// One thread per instance: accept / reject and the range of saves the step crosses.
static __global__ void control_kernel(Common c) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= c.B) return;
  Inst& I = c.inst[b];
  I.keep = 0;
  I.save_lo = I.save_hi = I.save_idx;
  if (!I.run) return;
  if (I.nsteps >= c.o.max_steps) {
    I.status = DQB_INST_MAX_STEPS;
    I.run = 0;
    return;
  }
  if (I.cancel != nullptr && *I.cancel != 0) {  // a caller's stop request
    I.status = DQB_INST_CANCELLED;
    I.run = 0;
    return;
  }
  const double err = sqrt(I.acc[0] / (double)c.nn);
  I.acc[0] = 0.0;
  I.nsteps += 1;
  if (!(err < INFINITY)) {
    I.status = DQB_INST_NONFINITE;
    I.nrej += 1;
    I.run = 0;
    return;
  }
  const bool keep = err < 1.0;
  I.keep = keep;
  if (keep) I.nacc += 1; else I.nrej += 1;
  // after a step clipped at a discontinuity the controller scales its proposal
  I.dtnew = (I.made_jump ? I.dt_prop : I.h) * step_factor(c.o, err, keep);
  if (keep) {
    int hi = I.save_idx;
    while (hi < I.nts && I.ts[hi] <= I.tnext) ++hi;
    I.save_hi = hi;
  }
}

// ------------------------------------------------------------------------------------
// Krylov form of the step, for a linear right-hand side with constant operators
// ------------------------------------------------------------------------------------
//
// For dy/dt = L y with L linear and constant, every quantity of an explicit RK step is a
// polynomial in hL applied to y.  With the basis u_q = (tau L)^q y (q = 0..7; tau = the
// step the basis was built for, r = h / tau):
//   h k_j   = sum_{q=1}^{j} alpha_{j,q-1} r^q u_q,
//             alpha_{j,0} = 1,  alpha_{j,m} = sum_{l<j} a_{jl} alpha_{l,m-1}
//   y1      = sum_q beta_q r^q u_q,          beta_0 = 1,  beta_q = sum_j b_j alpha_{j,q-1}
//   error   = sum_q eps_q r^q u_q,           eps_q = sum_j btilde_j alpha_{j,q-1}
//   y(theta)= sum_q delta_q(theta) r^q u_q,  delta_q = sum_j w_j(theta) alpha_{j,q-1}
//   tau L y1 = sum_{q<7} beta_q r^q u_{q+1}  (the next step's first stage, FSAL)
// -- the same numbers as the stage-by-stage form in exact arithmetic (a_7j = b_j for both
// tableaux, so stage 7 is L y1).  The basis costs six pure right-hand sides u_{q+1} =
// tau L u_q per accepted step, and y1, the error and the next first stage are one
// streaming pass over u_0..u_7: 22 passes over the state per attempted step instead of 54.
// A rejected step keeps its basis (only r changes), so a retry is that one pass alone.
// The error needs no cancellation either: eps_q = 0 for q up to the embedded order, so
// the estimate is a sum of the O(h^5) terms themselves.

// alpha_{j,m} of the method (j = stage 0..6, m = power 0..6).
__device__ inline void kry_alpha(int method, double al[7][7]) {
  const Tableau& T = c_tab[method];
  for (int j = 0; j < 7; ++j) {
    al[j][0] = 1.0;
    for (int m = 1; m < 7; ++m) {
      double v = 0.0;
      for (int l = 0; l < j; ++l) v += T.a[j][l] * al[l][m - 1];
      al[j][m] = v;
    }
  }
}

// Coefficients of u_0..u_7 in y1 (cy), the error (ce) and tau L y1 (cs) for r = h / tau;
// the stored u_1 is scaled by sig1.
__device__ inline void kry_step_coefs(int method, double r, double sig1, float cy[8], float ce[8], float cs[8]) {
  const Tableau& T = c_tab[method];
  double al[7][7];
  kry_alpha(method, al);
  double beta[8], eps[8], rp[8];
  rp[0] = 1.0;
  for (int q = 1; q < 8; ++q) rp[q] = rp[q - 1] * r;
  beta[0] = 1.0;
  eps[0] = 0.0;
  for (int q = 1; q < 8; ++q) {
    double bq = 0.0, eq = 0.0;
    for (int j = 0; j < 7; ++j) {
      bq += T.b[j] * al[j][q - 1];
      eq += T.btilde[j] * al[j][q - 1];
    }
    beta[q] = bq;
    eps[q] = eq;
  }
  for (int q = 0; q < 8; ++q) {
    const double s = q == 1 ? sig1 : 1.0;
    cy[q] = (float)(beta[q] * rp[q] * s);
    ce[q] = (float)(eps[q] * rp[q] * s);
    cs[q] = q == 0 ? 0.f : (float)(beta[q - 1] * rp[q - 1] * s);
  }
}

// Coefficients of u_0..u_7 in the dense output at theta (same scaling rules).
__device__ inline void kry_dense_coefs(int method, double theta, double r, double sig1, float cw[8]) {
  double al[7][7], w[7];
  kry_alpha(method, al);
  dense_weights(method, theta, w);
  double rp = 1.0;
  cw[0] = 1.f;
  for (int q = 1; q < 8; ++q) {
    rp *= r;
    double d = 0.0;
    for (int j = 0; j < 7; ++j) d += w[j] * al[j][q - 1];
    cw[q] = (float)(d * rp * (q == 1 ? sig1 : 1.0));
  }
}

__device__ __forceinline__ double kry_ratio(const Inst& I) { return I.tau > 0.0 ? I.h / I.tau : 0.0; }

// grid (tiles, B): states and tr(E rho) at the saves an accepted step crossed, up to
// kSaveChunk save points per pass over the inputs (one pass for the usual one or few).
// mode 0: y itself (the saves left over after the loop: t1 <= t0, or a stopped instance);
// mode 1: the dense output y + h sum_j w_j(theta) k_j of the stage form;
// mode 2: the dense output sum_q delta_q(theta) r^q u_q of the Krylov form.
constexpr int kSaveChunk = 4;

static __global__ void save_kernel(Common c, int mode) {
  __shared__ double red[40];
  __shared__ float cws[kSaveChunk][8];
  const int b = blockIdx.y;
  const Inst& I = c.inst[b];
  const int lo = I.save_lo, hi = I.save_hi;
  if (hi <= lo) return;
  const float2* p[8];
  p[0] = slot(c, b, I.sy);
  for (int q = 1; q < 8; ++q) p[q] = slot(c, b, I.sk[q - 1]);
  const int nq = mode == 0 ? 1 : 8;
  const int n = c.n;
  const bool herm = c.form == DQB_FORM_HERMITIAN;
  for (int s0 = lo; s0 < hi; s0 += kSaveChunk) {
    const int ns = hi - s0 < kSaveChunk ? hi - s0 : kSaveChunk;
    __syncthreads();  // the previous chunk's weights are no longer read
    if (threadIdx.x < ns) {
      float* cw = cws[threadIdx.x];
      const double theta = I.h > 0.0 ? (I.ts[s0 + threadIdx.x] - I.t) / I.h : 1.0;
      if (mode == 2) {
        kry_dense_coefs(c.o.method, theta, kry_ratio(I), I.sig1, cw);
      } else {
        double w[7];
        dense_weights(c.o.method, theta, w);
        cw[0] = 1.f;
        for (int j = 0; j < 7; ++j) cw[j + 1] = mode == 0 ? 0.f : (float)(I.h * w[j]);
      }
    }
    __syncthreads();
    for (int m0 = 0; m0 == 0 || m0 < I.nE; m0 += 2) {
      const int mc = I.nE - m0 < 2 ? I.nE - m0 : 2;
      double er[kSaveChunk][2], ei[kSaveChunk][2];
#pragma unroll
      for (int si = 0; si < kSaveChunk; ++si) er[si][0] = er[si][1] = ei[si][0] = ei[si][1] = 0.0;
      for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < c.nn;
           e += (long long)gridDim.x * blockDim.x) {
        float2 x[8], xt[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) x[q] = q < nq ? p[q][e] : make_float2(0.f, 0.f);
        long long et = e;
        if (mc > 0 && !herm) {
          const int i = (int)(e / n), j = (int)(e % n);
          et = (long long)j * n + i;
#pragma unroll
          for (int q = 0; q < 8; ++q) xt[q] = q < nq ? p[q][et] : make_float2(0.f, 0.f);
        }
        float2 ev[2] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
#pragma unroll
        for (int m = 0; m < 2; ++m)
          if (m < mc) ev[m] = I.E[(long long)(m0 + m) * c.nn + e];
#pragma unroll
        for (int si = 0; si < kSaveChunk; ++si) {
          if (si < ns) {
            float2 v = make_float2(0.f, 0.f);
#pragma unroll
            for (int q = 0; q < 8; ++q) v = caxpy(cws[si][q], x[q], v);
            if (m0 == 0 && I.save_states) I.states[(long long)(s0 + si) * c.nn + e] = v;
            if (mc > 0) {
              // tr(E rho) = sum_ij E_ij rho_ji; rho_ji = conj(rho_ij) when rho is hermitian
              float2 rt;
              if (herm) {
                rt = cconj(v);
              } else {
                rt = make_float2(0.f, 0.f);
#pragma unroll
                for (int q = 0; q < 8; ++q) rt = caxpy(cws[si][q], xt[q], rt);
              }
#pragma unroll
              for (int m = 0; m < 2; ++m) {
                if (m < mc) {
                  er[si][m] += (double)ev[m].x * rt.x - (double)ev[m].y * rt.y;
                  ei[si][m] += (double)ev[m].x * rt.y + (double)ev[m].y * rt.x;
                }
              }
            }
          }
        }
      }
#pragma unroll
      for (int si = 0; si < kSaveChunk; ++si)
#pragma unroll
        for (int m = 0; m < 2; ++m) {
          if (si < ns && m < mc) {  // uniform over the block
            double2* acc = I.eacc + (long long)(m0 + m) * I.nts + s0 + si;
            const double sr = block_sum(er[si][m], red);
            const double sim = block_sum(ei[si][m], red);
            if (threadIdx.x == 0) {
              atomicAdd(&acc->x, sr);
              atomicAdd(&acc->y, sim);
            }
          }
        }
    }
  }
}

// save_kernel for the hermitian form: one 32 x 32 tile of the upper triangle per block
// (grid (T (T + 1) / 2, B), 256 threads), so every input is read on its upper tiles only
// -- half the bytes, and a stage slot that holds only those tiles is enough -- and each
// saved state is written with its mirror (herm_store).  For hermitian rho,
// tr(E rho) = sum_ij E_ij conj(rho_ij): a diagonal tile adds its own elements, an
// off-diagonal one E_ij conj(rho_ij) + E_ji rho_ij for each of its elements.  The states
// are the same FP32 sums in the same order as save_kernel's.  The mirror tile of E is
// staged through shared memory (row-wise loads), and the two parts of each trace are
// reduced together.
template <bool VEC>
static __global__ void save_h_kernel(Common c, int mode) {
  __shared__ double red[72];
  __shared__ float cws[kSaveChunk][8];
  __shared__ float2 sh[kHT][kHT + 1];
  __shared__ float2 shE[kHT][kHT + 1];
  const int b = blockIdx.y;
  const Inst& I = c.inst[b];
  const int lo = I.save_lo, hi = I.save_hi;
  if (hi <= lo) return;
  const int n = c.n, T = (n + kHT - 1) / kHT;
  int ti, tj;
  herm_tile(blockIdx.x, T, ti, tj);
  const int nq = mode == 0 ? 1 : 8;
  const HTile<VEC> t;
  for (int s0 = lo; s0 < hi; s0 += kSaveChunk) {
    const int ns = hi - s0 < kSaveChunk ? hi - s0 : kSaveChunk;
    __syncthreads();  // the previous chunk's weights are no longer read
    if (threadIdx.x < ns) {
      float* cw = cws[threadIdx.x];
      const double theta = I.h > 0.0 ? (I.ts[s0 + threadIdx.x] - I.t) / I.h : 1.0;
      if (mode == 2) {
        kry_dense_coefs(c.o.method, theta, kry_ratio(I), I.sig1, cw);
      } else {
        double w[7];
        dense_weights(c.o.method, theta, w);
        cw[0] = 1.f;
        for (int j = 0; j < 7; ++j) cw[j + 1] = mode == 0 ? 0.f : (float)(I.h * w[j]);
      }
    }
    __syncthreads();
    float2 vs[kSaveChunk][4];
#pragma unroll
    for (int si = 0; si < kSaveChunk; ++si)
#pragma unroll
      for (int e = 0; e < 4; ++e) vs[si][e] = make_float2(0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      if (q < nq) {
        float2 x[4];
        htile_load<VEC>(slot(c, b, q == 0 ? I.sy : I.sk[q - 1]), n, ti, tj, x);
#pragma unroll
        for (int si = 0; si < kSaveChunk; ++si)
          if (si < ns) {
            const float w = cws[si][q];
#pragma unroll
            for (int e = 0; e < 4; ++e) vs[si][e] = caxpy(w, x[e], vs[si][e]);
          }
      }
    }
#pragma unroll
    for (int si = 0; si < kSaveChunk; ++si) {
      if (si >= ns) break;  // uniform over the block
      const float2(&v)[4] = vs[si];
      if (I.save_states) herm_store<VEC>(I.states + (long long)(s0 + si) * c.nn, n, ti, tj, v, sh);
      for (int m = 0; m < I.nE; ++m) {
        const float2* E = I.E + (long long)m * c.nn;
        if (ti != tj) {  // uniform over the block: E's tile (tj, ti) into shE
          __syncthreads();  // the previous operator's tile has been read
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int r = tj * kHT + t.row(e), cc = ti * kHT + t.col(e);
            shE[t.row(e)][t.col(e)] = (r < n && cc < n) ? E[(long long)r * n + cc] : make_float2(0.f, 0.f);
          }
          __syncthreads();
        }
        double sr = 0.0, sim = 0.0;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          if (htile_in<VEC>(n, ti, tj, e)) {
            const long long r = ti * kHT + t.row(e), cc = tj * kHT + t.col(e);
            const float2 a = E[r * n + cc];
            sr += (double)a.x * v[e].x + (double)a.y * v[e].y;
            sim += (double)a.y * v[e].x - (double)a.x * v[e].y;
            if (ti != tj) {
              const float2 a2 = shE[t.col(e)][t.row(e)];  // E_ji
              sr += (double)a2.x * v[e].x - (double)a2.y * v[e].y;
              sim += (double)a2.x * v[e].y + (double)a2.y * v[e].x;
            }
          }
        }
        const double2 tot = block_sum2(sr, sim, red);
        if (threadIdx.x == 0) {
          double2* acc = I.eacc + (long long)m * I.nts + s0 + si;
          atomicAdd(&acc->x, tot.x);
          atomicAdd(&acc->y, tot.y);
        }
      }
    }
  }
}

// One block: per-instance commit, then the WHILE-node condition (or, when the loop is
// driven from the host, the same condition written to `flag`).
static __global__ void commit_kernel(Common c, cudaGraphConditionalHandle handle, int* flag) {
  int any = 0;
  for (int b = threadIdx.x; b < c.B; b += blockDim.x) {
    Inst& I = c.inst[b];
    if (I.run) {
      I.refresh = 0;
      if (I.keep) {
        int tmp = I.sy;
        I.sy = I.sy1;
        I.sy1 = tmp;
        tmp = I.sk[0];
        I.sk[0] = I.sk[6];
        I.sk[6] = tmp;
        // a step that ended just before a discontinuity: the next starts on it, with its
        // first stage re-evaluated there (refresh)
        I.t = I.made_jump ? nextafter(I.tnext, INFINITY) : I.tnext;
        I.refresh = I.made_jump && I.t < I.t1;
        I.save_idx = I.save_hi;
      }
      I.dt_prop = I.dtnew;
      I.tnext = next_trial(c.jump_ts, c.n_jump, I.t, I.dtnew, I.t1, I.keep, I.made_jump);
      I.h = I.tnext - I.t;
      I.run = I.t < I.t1;
    }
    I.save_lo = I.save_hi = I.save_idx;
    any |= I.run;
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) {
    const long long it = ++(*c.iter);
    const bool more = any && it < c.o.max_steps + 2;
    if (flag)
      *flag = more ? 1 : 0;
    else
      cudaGraphSetConditional(handle, more ? 1u : 0u);
  }
}

// grid (tiles, B): y1, tau L y1 and the error sum of the trial step from u_0..u_7, for
// every running instance (a retried step included).
static __global__ void kry_combine_kernel(Common c) {
  __shared__ double red[40];
  __shared__ float cf[3][8];
  const int b = blockIdx.y;
  Inst& I = c.inst[b];
  if (!I.run) return;
  if (threadIdx.x == 0) kry_step_coefs(c.o.method, kry_ratio(I), I.sig1, cf[0], cf[1], cf[2]);
  __syncthreads();
  float cy[8], ce[8], cs[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) cy[q] = cf[0][q], ce[q] = cf[1][q], cs[q] = cf[2][q];
  const float2* u[8];
  u[0] = slot(c, b, I.sy);
#pragma unroll
  for (int q = 1; q < 8; ++q) u[q] = slot(c, b, I.sk[q - 1]);
  float2* y1 = slot(c, b, I.sy1);
  float2* s1 = slot(c, b, I.sf);
  const double atol = c.o.atol, rtol = c.o.rtol;
  double s = 0.0;
  auto one = [&](const float2 (&v)[8], float2& oy, float2& os) {
    float2 a = make_float2(0.f, 0.f), e = make_float2(0.f, 0.f), f = make_float2(0.f, 0.f);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      a = caxpy(cy[q], v[q], a);
      e = caxpy(ce[q], v[q], e);
      f = caxpy(cs[q], v[q], f);
    }
    oy = a;
    os = f;
    const float ya = cabsf(v[0]), y1a = cabsf(a);
    const double sc = atol + rtol * (double)(ya > y1a ? ya : y1a);
    const double ex = e.x, ey = e.y;
    s += (ex * ex + ey * ey) / (sc * sc);
  };
  if ((c.nn & 1) == 0 && (reinterpret_cast<uintptr_t>(c.mats) & 15) == 0) {
    // two complex values per 16-byte access, as in combine_kernel
    const long long nn2 = c.nn >> 1;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn2;
         e += (long long)gridDim.x * blockDim.x) {
      float4 v4[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) v4[q] = reinterpret_cast<const float4*>(u[q])[e];
      float2 lo[8], hi[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) lo[q] = make_float2(v4[q].x, v4[q].y), hi[q] = make_float2(v4[q].z, v4[q].w);
      float2 ya, sa, yb, sb;
      one(lo, ya, sa);
      one(hi, yb, sb);
      reinterpret_cast<float4*>(y1)[e] = make_float4(ya.x, ya.y, yb.x, yb.y);
      reinterpret_cast<float4*>(s1)[e] = make_float4(sa.x, sa.y, sb.x, sb.y);
    }
  } else {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < c.nn;
         e += (long long)gridDim.x * blockDim.x) {
      float2 v[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) v[q] = u[q][e];
      one(v, y1[e], s1[e]);
    }
  }
  block_atomic_add(s, &I.acc[0], red);
}

// kry_combine_kernel for the hermitian form (upper-triangle tiles, mirrored writes).
template <bool VEC>
static __global__ void kry_combine_h_kernel(Common c) {
  __shared__ double red[40];
  __shared__ float cf[3][8];
  __shared__ float2 sh[kHT][kHT + 1];
  const int b = blockIdx.y;
  Inst& I = c.inst[b];
  if (!I.run) return;
  if (threadIdx.x == 0) kry_step_coefs(c.o.method, kry_ratio(I), I.sig1, cf[0], cf[1], cf[2]);
  __syncthreads();
  const int n = c.n, T = (n + kHT - 1) / kHT;
  int ti, tj;
  herm_tile(blockIdx.x, T, ti, tj);
  float2 u0[4], vy[4], ve[4], vs[4], w[4];
  htile_load<VEC>(slot(c, b, I.sy), n, ti, tj, u0);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    vy[q] = make_float2(cf[0][0] * u0[q].x, cf[0][0] * u0[q].y);
    ve[q] = make_float2(0.f, 0.f);
    vs[q] = make_float2(0.f, 0.f);
  }
#pragma unroll
  for (int k = 1; k < 8; ++k) {
    htile_load<VEC>(slot(c, b, I.sk[k - 1]), n, ti, tj, w);
    const float a = cf[0][k], e = cf[1][k], f = cf[2][k];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      vy[q] = caxpy(a, w[q], vy[q]);
      ve[q] = caxpy(e, w[q], ve[q]);
      vs[q] = caxpy(f, w[q], vs[q]);
    }
  }
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    if (htile_in<VEC>(n, ti, tj, q)) {
      const float ya = cabsf(u0[q]), y1a = cabsf(vy[q]);
      const double sc = c.o.atol + c.o.rtol * (double)(ya > y1a ? ya : y1a);
      const double ex = ve[q].x, ey = ve[q].y;
      s += (ex * ex + ey * ey) / (sc * sc);
    }
  }
  if (ti != tj) s *= 2.0;
  herm_store<VEC>(slot(c, b, I.sy1), n, ti, tj, vy, sh);
  herm_store<VEC>(slot(c, b, I.sf), n, ti, tj, vs, sh);
  block_atomic_add(s, &I.acc[0], red);
}

// One block: per-instance commit of the Krylov form, then the WHILE-node condition (as
// commit_kernel).  An accepted step makes y1 the new u_0 and tau L y1 the new (scaled)
// u_1, and rebuilds the basis for the next trial step; a rejected one keeps the basis.
static __global__ void kry_commit_kernel(Common c, cudaGraphConditionalHandle handle, int* flag) {
  int any = 0;
  for (int b = threadIdx.x; b < c.B; b += blockDim.x) {
    Inst& I = c.inst[b];
    if (I.run) {
      if (I.keep) {
        int tmp = I.sy;
        I.sy = I.sy1;
        I.sy1 = tmp;
        tmp = I.sk[0];
        I.sk[0] = I.sf;
        I.sf = tmp;
        I.t = I.tnext;
        I.save_idx = I.save_hi;
      }
      I.tnext = next_tend(I.t, I.dtnew, I.t1, I.keep);
      I.h = I.tnext - I.t;
      if (I.keep) {
        I.sig1 = I.tau > 0.0 ? I.h / I.tau : 1.0;
        I.tau = I.h;
        I.kvalid = 2;
      } else {
        I.kvalid = 8;
      }
      I.run = I.t < I.t1;
    }
    I.save_lo = I.save_hi = I.save_idx;
    any |= I.run;
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) {
    const long long it = ++(*c.iter);
    const bool more = any && it < c.o.max_steps + 2;
    if (flag)
      *flag = more ? 1 : 0;
    else
      cudaGraphSetConditional(handle, more ? 1u : 0u);
  }
}

// ------------------------------------------------------------------------------------
// launch helpers: the hermitian-half elementwise kernels in the hermitian form
// ------------------------------------------------------------------------------------
inline dim3 herm_grid(int n, int B) {
  const int T = (n + kHT - 1) / kHT;
  return dim3((unsigned)(T * (T + 1) / 2), (unsigned)B);
}
// 16-byte accesses when every row starts on a 16-byte boundary (n even, slots aligned).
inline bool herm_vec(const Common& c) { return (c.n % 2) == 0 && (reinterpret_cast<uintptr_t>(c.mats) & 15) == 0; }
inline void launch_combine(cudaStream_t s, const Common& c, dim3 ge, int mode) {
  if (c.form != DQB_FORM_HERMITIAN)
    combine_kernel<<<ge, kElemThreads, 0, s>>>(c, mode);
  else if (herm_vec(c))
    combine_h_kernel<true><<<herm_grid(c.n, c.B), 256, 0, s>>>(c, mode);
  else
    combine_h_kernel<false><<<herm_grid(c.n, c.B), 256, 0, s>>>(c, mode);
}
inline void launch_error(cudaStream_t s, const Common& c, dim3 ge) {
  if (c.form != DQB_FORM_HERMITIAN)
    error_kernel<<<ge, kElemThreads, 0, s>>>(c);
  else if (herm_vec(c))
    error_h_kernel<true><<<herm_grid(c.n, c.B), 256, 0, s>>>(c);
  else
    error_h_kernel<false><<<herm_grid(c.n, c.B), 256, 0, s>>>(c);
}
// Saves of an accepted step (or the leftovers, mode 0); the hermitian form reads the
// upper tiles of its inputs only.
inline void launch_save(cudaStream_t s, const Common& c, dim3 ge, int mode) {
  if (c.form != DQB_FORM_HERMITIAN)
    save_kernel<<<ge, kElemThreads, 0, s>>>(c, mode);
  else if (herm_vec(c))
    save_h_kernel<true><<<herm_grid(c.n, c.B), 256, 0, s>>>(c, mode);
  else
    save_h_kernel<false><<<herm_grid(c.n, c.B), 256, 0, s>>>(c, mode);
}
inline void launch_kry_combine(cudaStream_t s, const Common& c, dim3 ge) {
  if (c.form != DQB_FORM_HERMITIAN)
    kry_combine_kernel<<<ge, kElemThreads, 0, s>>>(c);
  else if (herm_vec(c))
    kry_combine_h_kernel<true><<<herm_grid(c.n, c.B), 256, 0, s>>>(c);
  else
    kry_combine_h_kernel<false><<<herm_grid(c.n, c.B), 256, 0, s>>>(c);
}

// One block per instance after the loop: the saves left over (t1 <= t0, or a
// stopped instance), final state when only it is kept, expects, infos, status.
static __global__ void pre_finalize_kernel(Common c) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= c.B) return;
  Inst& I = c.inst[b];
  I.save_lo = I.save_idx;
  I.save_hi = I.save_idx;
  if (I.status == DQB_INST_OK) {
    int hi = I.save_idx;
    while (hi < I.nts && I.ts[hi] <= I.t) ++hi;
    I.save_hi = hi;
  }
}

// grid (B), inside the RK loop of ragged launches, after the commit: hands out each
// instance that finished normally in this iteration (every save written) without waiting
// for the rest of the batch -- final state (when only it is kept), expectation values,
// infos, then, after a system-scope fence, the status word, which a serving loop may poll
// in host-mapped memory.  finalize_kernel later writes the same values again.
static __global__ void retire_kernel(Common c) {
  const int b = blockIdx.x;
  Inst& I = c.inst[b];
  if (I.retired || I.run) return;
  if (!(I.status == DQB_INST_OK && I.save_idx >= I.nts) && I.status != DQB_INST_CANCELLED) return;
  if (!I.save_states) {
    const float2* y = slot(c, b, I.sy);
    for (long long e = threadIdx.x; e < c.nn; e += blockDim.x) I.states[e] = y[e];
  }
  for (int e = threadIdx.x; e < I.nE * I.nts; e += blockDim.x) {
    const double2 v = I.eacc[e];
    I.expects[e] = make_float2((float)v.x, (float)v.y);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    I.infos[0] = (int)I.nsteps;
    I.infos[1] = (int)I.nacc;
    I.infos[2] = (int)I.nrej;
    __threadfence_system();
    I.status_out[0] = I.status;
    I.retired = 1;
  }
}

static __global__ void finalize_kernel(Common c) {
  const int b = blockIdx.y;
  Inst& I = c.inst[b];
  if (I.status == kInactive) return;
  if (!I.save_states) {
    const float2* y = slot(c, b, I.sy);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < c.nn;
         e += (long long)gridDim.x * blockDim.x)
      I.states[e] = y[e];
  }
  if (blockIdx.x == 0) {
    for (int e = threadIdx.x; e < I.nE * I.nts; e += blockDim.x) {
      const double2 v = I.eacc[e];
      I.expects[e] = make_float2((float)v.x, (float)v.y);
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      I.infos[0] = (int)I.nsteps;
      I.infos[1] = (int)I.nacc;
      I.infos[2] = (int)I.nrej;
      __threadfence_system();
      I.status_out[0] = I.status;
    }
  }
}

}  // namespace big
}  // namespace dqb
