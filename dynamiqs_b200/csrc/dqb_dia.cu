// Sparse-DIA mesolve for large n (e.g. two 64-level modes, n = 4096, rho = 128 MiB).
//
// Right-hand side, element by element, from the DIA diagonals (column-indexed:
// A[c - k][c] = diag_k[c]; dynamiqs/qarrays/sparsedia_primitives.py:232-261):
//   (Hnh X)[i][j]   = sum_d hnh_d[i + k_d] X[i + k_d][j]                 (row shifts)
//   (X Hnh^+)[i][j] = sum_d conj(hnh_d[j + k_d]) X[i][j + k_d]           (column shifts)
//   (L X L^+)[i][j] = sum_{p,q} l_p[i + q_p] conj(l_q[j + q_q]) X[i + q_p][j + q_q]
// and f(X) = Hnh X + X Hnh^+ + sum_k L_k X L_k^+.  For a hermitian X this equals the
// reference's hermitian form tmp + tmp^+ with tmp = Hnh X + 1/2 sum L X L^+
// (diffrax_integrator.py:319-323) and it is the standard form (:312-317) for any X, so
// one stencil serves both.  Every term is a shifted, coalesced read of X (algorithmic
// traffic: read X once, write f(X) once; the shifted re-reads come from L1/L2 or shared
// memory).  Three kernels compute it -- generic, tiled (coefficient tables in shared
// memory) and staged (the rows of X the offsets touch in shared memory) -- and the
// autotuner keeps the fastest per problem shape (dqb_ode_options.tile).
//
// Hnh's diagonals are built once per instance on the device (the reference rebuilds
// them with matmul_sparsedia_sparsedia + add_sparsedia_sparsedia on every RHS,
// sparsedia_primitives.py:172-229).  The RK loop is the stepper of dqb_big.cuh run as a
// CUDA graph WHILE node.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <set>
#include <vector>

#include "dqb_big.cuh"
#include "dqb_graph.cuh"
#include "dqb_tc.cuh"

namespace dqb {

struct DiaOps {
  int n;
  int nh;                             // diagonals of Hnh
  int hoff[DQB_DIA_MAX_HNH_DIAGS];
  int hmap[DQB_DIA_MAX_HNH_DIAGS];    // index of the same offset in H, or -1
  int h_nd;                           // diagonals of H
  int K;
  int nl;                             // sum of jump diagonals
  int lstart[DQB_DIA_MAX_JUMPS + 1];
  int loff[DQB_DIA_MAX_JUMP_DIAGS];
  // (p, s) pairs of diagonals of the same jump operator: the terms
  // l_p[i + q_p] conj(l_s[j + q_s]) X[i + q_p][j + q_s] of L X L^+ (up to 64 recorded)
  int npair;
  int pair_p[64];
  int pair_s[64];
  const float2* H;                    // [*, h_nd, n]
  const float2* L;                    // [*, nl, n]
  const int* Hidx;
  const int* Lidx;
  float2* hnh;                        // [B, nh, n]
  float2* hnh0;                       // [B, nh, n]: the constant part of Hnh when H depends
                                      // on time (hnh then holds Hnh at the stage time)
  // time-dependent jump operators: L above points to the per-instance copies c_k(t) L_k
  // ([B, nl, n], Lidx null) that the stencils read; L0 / L0idx are the given diagonals
  const float2* L0;
  const int* L0idx;
};

// Prefactors c_k(t) of the jump operators (time-dependent jump operators), by value.
struct DiaJumpTd {
  int on;
  TdTerm term[DQB_DIA_MAX_JUMPS];
};


namespace {

// One thread per (column c, instance b): Hnh diagonals of instance b.
__global__ void hnh_dia_kernel(DiaOps d, int B) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (c >= d.n || b >= B) return;
  const int n = d.n;
  const long long hi = d.Hidx ? d.Hidx[b] : b;
  const long long li = d.Lidx ? d.Lidx[b] : b;
  const float2* H = d.H + hi * d.h_nd * n;
  const float2* L = d.L + li * d.nl * n;
  float2* out = d.hnh + (long long)b * d.nh * n;
  for (int q = 0; q < d.nh; ++q) {
    const int k = d.hoff[q];
    float2 v = make_float2(0.f, 0.f);
    if (c - k >= 0 && c - k < n) {
      if (d.hmap[q] >= 0) {
        const float2 h = H[d.hmap[q] * n + c];
        v = make_float2(h.y, -h.x);  // -i h
      }
      for (int jk = 0; jk < d.K; ++jk) {
        for (int p = d.lstart[jk]; p < d.lstart[jk + 1]; ++p) {
          for (int r = d.lstart[jk]; r < d.lstart[jk + 1]; ++r) {
            if (d.loff[r] - d.loff[p] != k) continue;
            // (L^+ L)[c - k][c] += conj(l_p[c - k]) l_r[c]
            const float2 t = cmul(cconj(L[p * n + (c - k)]), L[r * n + c]);
            v.x -= 0.5f * t.x;
            v.y -= 0.5f * t.y;
          }
        }
      }
    }
    out[q * n + c] = v;
  }
}

// Hnh at the time of a right-hand side (big::td_stage_time), for every instance that
// evaluates it: hnh = hnh0 - i sum_m c_m(t) ops_m on H's diagonals (ops_m given by its
// diagonals on H's offsets, [M, h_nd, n]; the jump terms are in hnh0).  grid (ceil(n / 256), B).
__global__ void hnh_td_kernel(big::Common c, DiaOps d, TdOps td, int which) {
  __shared__ float2 cm[DQB_TD_MAX_TERMS];
  const int b = blockIdx.y;
  double t;
  if (!big::td_stage_time(c, c.inst[b], which, &t)) return;
  if (threadIdx.x < td.M) {
    const double2 v = td_coef(td.term[threadIdx.x], b, t);
    cm[threadIdx.x] = make_float2((float)v.x, (float)v.y);
  }
  __syncthreads();
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = d.n;
  if (col >= n) return;
  const float2* h0 = d.hnh0 + (long long)b * d.nh * n;
  float2* out = d.hnh + (long long)b * d.nh * n;
  for (int q = 0; q < d.nh; ++q) {
    float2 v = h0[q * n + col];
    const int k = d.hoff[q];
    if (d.hmap[q] >= 0 && col - k >= 0 && col - k < n) {
      float2 a = make_float2(0.f, 0.f);
      for (int m = 0; m < td.M; ++m) a = cfma(cm[m], td.ops[((long long)m * d.h_nd + d.hmap[q]) * n + col], a);
      v.x += a.y;  // -i a
      v.y -= a.x;
    }
    out[q * n + col] = v;
  }
}

// Time-dependent jump operators L_k(t) = c_k(t) L_k (and H(t) as hnh_td_kernel): at the
// time of a right-hand side (big::td_stage_time) every instance that evaluates it gets
//   L(t)   = c_k(t) L_k on jump k's diagonals (the copies the stencils read), and
//   Hnh(t) = -i (H + sum_m c_m(t) ops_m) - 1/2 sum_k |c_k(t)|^2 L_k^+ L_k
// on Hnh's diagonals, the L^+ L products formed from the given diagonals as
// hnh_dia_kernel does.  grid (ceil(n / 256), B).
__global__ void hnh_td_jump_kernel(big::Common c, DiaOps d, TdOps td, DiaJumpTd jt, int which) {
  __shared__ float2 cm[DQB_TD_MAX_TERMS];
  __shared__ float2 ck[DQB_DIA_MAX_JUMPS];
  __shared__ float wk[DQB_DIA_MAX_JUMPS];
  const int b = blockIdx.y;
  double t;
  if (!big::td_stage_time(c, c.inst[b], which, &t)) return;
  if (threadIdx.x < td.M) {
    const double2 v = td_coef(td.term[threadIdx.x], b, t);
    cm[threadIdx.x] = make_float2((float)v.x, (float)v.y);
  }
  if (threadIdx.x < d.K) {
    const double2 v = td_coef(jt.term[threadIdx.x], b, t);
    ck[threadIdx.x] = make_float2((float)v.x, (float)v.y);
    wk[threadIdx.x] = (float)(v.x * v.x + v.y * v.y);
  }
  __syncthreads();
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  const int n = d.n;
  if (col >= n) return;
  const long long hi = d.Hidx ? d.Hidx[b] : b;
  const long long li = d.L0idx ? d.L0idx[b] : b;
  const float2* H = d.H + hi * d.h_nd * n;
  const float2* L = d.L0 + li * d.nl * n;
  float2* Lt = const_cast<float2*>(d.L) + (long long)b * d.nl * n;
  for (int k = 0; k < d.K; ++k)
    for (int p = d.lstart[k]; p < d.lstart[k + 1]; ++p) Lt[(long long)p * n + col] = cmul(ck[k], L[(long long)p * n + col]);
  float2* out = d.hnh + (long long)b * d.nh * n;
  for (int q = 0; q < d.nh; ++q) {
    const int k = d.hoff[q];
    float2 v = make_float2(0.f, 0.f);
    if (col - k >= 0 && col - k < n) {
      if (d.hmap[q] >= 0) {
        float2 h = H[d.hmap[q] * n + col];
        for (int m = 0; m < td.M; ++m) h = cfma(cm[m], td.ops[((long long)m * d.h_nd + d.hmap[q]) * n + col], h);
        v = make_float2(h.y, -h.x);  // -i h
      }
      for (int jk = 0; jk < d.K; ++jk) {
        for (int p = d.lstart[jk]; p < d.lstart[jk + 1]; ++p) {
          for (int r = d.lstart[jk]; r < d.lstart[jk + 1]; ++r) {
            if (d.loff[r] - d.loff[p] != k) continue;
            // |c_k|^2 (L^+ L)[col - k][col] += conj(l_p[col - k]) l_r[col]
            const float2 u = cmul(cconj(L[p * n + (col - k)]), L[r * n + col]);
            v.x -= 0.5f * wk[jk] * u.x;
            v.y -= 0.5f * wk[jk] * u.y;
          }
        }
      }
    }
    out[q * n + col] = v;
  }
}

constexpr int kRhsCols = 128;
constexpr int kRhsRows = 8;

// Input, output and output scale of one instance's right-hand side inside a solve.
// kry = 0: k[out_k] = f(input) with input 0 = y, 1 = y1, 2 = X, 3 = k1, for the running
// instances (need_run = 1), those with status OK (need_run = 0), or the running ones whose
// first stage is re-evaluated after a discontinuity (need_run = 2).  kry = q in 1..6 (the
// Krylov form): u_{q+1} = tau L u_q for the running instances whose basis lacks it, with
// the stored u_1 scaled by sig1.  Returns false when the instance has nothing to do.
struct RhsIo {
  const float2* X;
  float2* out;
  float scale;
};
__device__ __forceinline__ bool rhs_io(const big::Common& c, int b, int in_sel, int out_k, int need_run, int kry,
                                       RhsIo& io) {
  const big::Inst& I = c.inst[b];
  io.scale = 1.f;
  if (kry > 0) {
    if (!I.run || I.kvalid >= kry + 2) return false;
    io.X = big::slot(c, b, I.sk[kry - 1]);
    io.out = big::slot(c, b, I.sk[kry]);
    io.scale = (float)(kry == 1 ? I.tau * I.sig1 : I.tau);
    return true;
  }
  if (need_run == 2 ? !(I.run && I.refresh) : (need_run ? !I.run : I.status != DQB_INST_OK)) return false;
  io.X = big::slot(c, b, in_sel == 0 ? I.sy : (in_sel == 1 ? I.sy1 : (in_sel == 3 ? I.sk[0] : big::kX)));
  io.out = big::slot(c, b, I.sk[out_k]);
  return true;
}

__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// Generic f(X) for DIA operators (any number of diagonals).  grid (n / 128, n / 8, B),
// block 128: each thread owns one column and 8 consecutive rows.
// in_sel: 0 = y, 1 = y1, 2 = X.  need_run: 1 = running instances, 0 = status OK.
__global__ void __launch_bounds__(kRhsCols) rhs_dia_generic_kernel(big::Common c, DiaOps d, int in_sel, int out_k,
                                                                   int need_run, int kry, const float2* ext_in,
                                                                   float2* ext_out) {
  const int b = blockIdx.z;
  const float2* X;
  float2* out;
  float scale = 1.f;
  const float2* L;
  if (ext_in) {  // stand-alone evaluation (dqb_lindblad_rhs_dia)
    X = ext_in + (long long)b * d.n * d.n;
    out = ext_out + (long long)b * d.n * d.n;
  } else {
    RhsIo io;
    if (!rhs_io(c, b, in_sel, out_k, need_run, kry, io)) return;
    X = io.X;
    out = io.out;
    scale = io.scale;
  }
  const long long li = d.Lidx ? d.Lidx[b] : b;
  L = d.L + li * d.nl * d.n;
  const float2* hnh = d.hnh + (long long)b * d.nh * d.n;
  const int n = d.n;
  const int j = blockIdx.x * kRhsCols + threadIdx.x;
  if (j >= n) return;
  const int i0 = blockIdx.y * kRhsRows;
  for (int r = 0; r < kRhsRows; ++r) {
    const int i = i0 + r;
    if (i >= n) break;
    float2 acc = make_float2(0.f, 0.f);
    for (int q = 0; q < d.nh; ++q) {
      const int k = d.hoff[q];
      float2 pair = make_float2(0.f, 0.f);
      const int ik = i + k, jk = j + k;
      if (ik >= 0 && ik < n) pair = cmul(__ldg(&hnh[q * n + ik]), __ldg(&X[(long long)ik * n + j]));
      if (jk >= 0 && jk < n) {
        const float2 t = cmul(cconj(__ldg(&hnh[q * n + jk])), __ldg(&X[(long long)i * n + jk]));
        pair = cadd(pair, t);
      }
      acc = cadd(acc, pair);
    }
    for (int jk = 0; jk < d.K; ++jk) {
      for (int p = d.lstart[jk]; p < d.lstart[jk + 1]; ++p) {
        const int ip = i + d.loff[p];
        if (ip < 0 || ip >= n) continue;
        const float2 lp = __ldg(&L[p * n + ip]);
        for (int s = d.lstart[jk]; s < d.lstart[jk + 1]; ++s) {
          const int jq = j + d.loff[s];
          if (jq < 0 || jq >= n) continue;
          const float2 coef = cmul(lp, cconj(__ldg(&L[s * n + jq])));
          acc = cadd(acc, cmul(coef, __ldg(&X[(long long)ip * n + jq])));
        }
      }
    }
    out[(long long)i * n + j] = cscale(acc, scale);
  }
}

// Tiled f(X): every coefficient in shared memory, the inner loops over the diagonals read
// one 16-byte table entry per term.  grid (n / 128, n / R, B), block 128: each thread owns
// one column j and R consecutive rows.  Per CTA, for the diagonal terms t (the nh diagonals
// of Hnh, then the npair (p, s) jump-diagonal pairs):
//   row table  [t][r]:   the row factor (hnh_q[i + k_q] or l_p[i + q_p], 0 outside the
//                        matrix) and the clamped source row of that term for row i0 + r;
//   col table  [t][tid]: the column factor (conj(hnh_q[j + k_q]) or conj(l_s[j + q_s])) and
//                        the clamped source column for this thread's column.
// Then out[i][j] = sum_q (hrow_q(i) X[ri_q(i)][j] + hcol_q(j) X[i][cj_q(j)])
//                + sum_pairs prow_t(i) pcol_t(j) X[ri_t(i)][cj_t(j)],
// the same terms as the generic kernel.  Occupancy stays high (few registers; the tables
// are (nh + npair) (R + 128) 16 bytes), which the load latency of the shifted reads needs.
struct __align__(16) DiaCoef {
  float2 f;  // factor
  int idx;   // clamped source row times n (row table) or clamped source column (column table)
  int pad;
};
constexpr int kTiledMaxTerms = 20;

template <int R>
__global__ void __launch_bounds__(kRhsCols) rhs_dia_tiled_kernel(big::Common c, DiaOps d, int in_sel, int out_k,
                                                                int need_run, int kry, const float2* ext_in,
                                                                float2* ext_out) {
  extern __shared__ DiaCoef dia_tab[];
  const int b = blockIdx.z;
  const float2* X;
  float2* out;
  float scale = 1.f;
  if (ext_in) {  // stand-alone evaluation (dqb_lindblad_rhs_dia)
    X = ext_in + (long long)b * d.n * d.n;
    out = ext_out + (long long)b * d.n * d.n;
  } else {
    RhsIo io;
    if (!rhs_io(c, b, in_sel, out_k, need_run, kry, io)) return;
    X = io.X;
    out = io.out;
    scale = io.scale;
  }
  const int n = d.n, nh = d.nh, np = d.npair, nt = nh + np;
  const long long li = d.Lidx ? d.Lidx[b] : b;
  const float2* L = d.L + li * d.nl * n;
  const float2* hnh = d.hnh + (long long)b * nh * n;
  const int i0 = blockIdx.y * R;
  const int j0 = blockIdx.x * kRhsCols;
  DiaCoef* rowt = dia_tab;          // [nt][R]
  DiaCoef* colt = dia_tab + nt * R;  // [nt][kRhsCols]

  for (int e = threadIdx.x; e < nt * R; e += blockDim.x) {
    const int t = e / R, r = e % R, i = i0 + r;
    int off;
    const float2* diag;
    if (t < nh) {
      off = d.hoff[t];
      diag = hnh + t * n;
    } else {
      const int p = d.pair_p[t - nh];
      off = d.loff[p];
      diag = L + p * n;
    }
    const int src = i + off;
    const bool in = i < n && src >= 0 && src < n;
    DiaCoef v;
    v.f = in ? __ldg(&diag[src]) : make_float2(0.f, 0.f);
    v.idx = (src < 0 ? 0 : (src >= n ? n - 1 : src)) * n;  // element offset of the source row
    v.pad = 0;
    rowt[e] = v;
  }
  {
    const int j = j0 + threadIdx.x;
    for (int t = 0; t < nt; ++t) {
      int off;
      const float2* diag;
      if (t < nh) {
        off = d.hoff[t];
        diag = hnh + t * n;
      } else {
        const int sd = d.pair_s[t - nh];
        off = d.loff[sd];
        diag = L + sd * n;
      }
      const int src = j + off;
      const bool in = j < n && src >= 0 && src < n;
      DiaCoef v;
      v.f = in ? cconj(__ldg(&diag[src])) : make_float2(0.f, 0.f);
      v.idx = src < 0 ? 0 : (src >= n ? n - 1 : src);
      v.pad = 0;
      colt[t * kRhsCols + threadIdx.x] = v;
    }
  }
  __syncthreads();
  const int j = j0 + threadIdx.x;
  if (j >= n) return;
  const int rows = min(R, n - i0);
  for (int r = 0; r < rows; ++r) {
    const int i = i0 + r;
    const float2* Xi = X + (long long)i * n;
    float2 acc = make_float2(0.f, 0.f);
    // unrolled so that several terms' loads are in flight at once
#pragma unroll 4
    for (int q = 0; q < nh; ++q) {
      const DiaCoef rc = rowt[q * R + r];
      const DiaCoef cc = colt[q * kRhsCols + threadIdx.x];
      acc = cfma(rc.f, __ldg(&X[rc.idx + j]), acc);
      acc = cfma(cc.f, __ldg(&Xi[cc.idx]), acc);
    }
#pragma unroll 2
    for (int t = nh; t < nt; ++t) {
      const DiaCoef rc = rowt[t * R + r];
      const DiaCoef cc = colt[t * kRhsCols + threadIdx.x];
      acc = cfma(cmul(rc.f, cc.f), __ldg(&X[rc.idx + cc.idx]), acc);
    }
    out[(long long)i * n + j] = cscale(acc, scale);
  }
}

// Staged f(X): the few groups of rows of X that the diagonals touch, with their column
// halos, are copied into shared memory once per CTA; every term then reads shared memory.
// Every read of the stencil is X[i + ro][j + co] for a (row offset, column offset) pair of
// its term: (k_q, 0) for the row term of Hnh diagonal q, (0, k_q) for its column term, and
// (q_p, q_s) for a jump-diagonal pair.  The host groups the distinct row offsets that lie
// within R of each other (DiaStage): group g stages rows i0 + rlo_g .. i0 + R - 1 + rhi_g and
// columns j0 + clo_g .. j0 + 127 + chi_g of X (zeros outside the matrix).  For the coupled
// Kerr operators (row offsets -64, -63, 0, 1, 63, 64) that is three groups of R + 1 rows, so
// each element of X leaves L2 about 5 times per right-hand side instead of ~12.
constexpr int kStageMaxGroups = 8;
constexpr int kStageMaxTerms = 24;
constexpr size_t kStageMaxSmem = 200 * 1024;  // dynamic shared memory of one CTA

struct DiaStage {
  int ngroup;
  int g_rlo[kStageMaxGroups];   // smallest row offset of the group
  int g_rows[kStageMaxGroups];  // staged rows: R + (rhi - rlo)
  int g_clo[kStageMaxGroups];   // smallest column offset of the group's reads
  int g_cols[kStageMaxGroups];  // staged columns: 128 + (chi - clo)
  int g_off[kStageMaxGroups];   // start of the group in the staged array (complex values)
  int n0, n1, n2;               // row terms, column terms, pair terms, in this order
  int t_diag[kStageMaxTerms];   // Hnh diagonal (row / column terms) or pair index (pairs)
  int t_base[kStageMaxTerms];   // staged index of (row 0 of the tile, column 0 of the tile)
  int t_stride[kStageMaxTerms]; // row stride of the term's group
  int staged;                   // complex values staged per CTA
};

template <int R>
__global__ void __launch_bounds__(kRhsCols) rhs_dia_staged_kernel(big::Common c, DiaOps d, DiaStage st, int in_sel,
                                                                 int out_k, int need_run, int kry,
                                                                 const float2* ext_in, float2* ext_out) {
  extern __shared__ float4 dia_stage_raw[];
  const int b = blockIdx.z;
  const float2* X;
  float2* out;
  float scale = 1.f;
  if (ext_in) {  // stand-alone evaluation (dqb_lindblad_rhs_dia)
    X = ext_in + (long long)b * d.n * d.n;
    out = ext_out + (long long)b * d.n * d.n;
  } else {
    RhsIo io;
    if (!rhs_io(c, b, in_sel, out_k, need_run, kry, io)) return;
    X = io.X;
    out = io.out;
    scale = io.scale;
  }
  const int n = d.n, nt = st.n0 + st.n1 + st.n2, tid = threadIdx.x;
  const long long li = d.Lidx ? d.Lidx[b] : b;
  const float2* L = d.L + li * d.nl * n;
  const float2* hnh = d.hnh + (long long)b * d.nh * n;
  const int i0 = blockIdx.y * R, j0 = blockIdx.x * kRhsCols;
  float2* S = reinterpret_cast<float2*>(dia_stage_raw);
  float2* rowc = S + st.staged;    // [nt][R]
  float2* colc = rowc + nt * R;    // [nt][128]

  // stage with asynchronous 8-byte copies (zero-filled outside the matrix), all in flight
  // while the coefficient tables are computed
  for (int g = 0; g < st.ngroup; ++g) {
    const int gr0 = i0 + st.g_rlo[g], gc0 = j0 + st.g_clo[g], cols = st.g_cols[g];
    float2* dst = S + st.g_off[g];
    for (int rr = 0; rr < st.g_rows[g]; ++rr) {
      const int gr = gr0 + rr;
      const bool rin = gr >= 0 && gr < n;
      const float2* src = X + (long long)(rin ? gr : 0) * n;
      for (int cc = tid; cc < cols; cc += kRhsCols) {
        const int gc = gc0 + cc;
        const bool in = rin && gc >= 0 && gc < n;
        const uint32_t sa = static_cast<uint32_t>(__cvta_generic_to_shared(dst + rr * cols + cc));
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(sa), "l"(in ? src + gc : X),
                     "r"(in ? 8 : 0)
                     : "memory");
      }
    }
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
  for (int e = tid; e < nt * R; e += kRhsCols) {
    const int t = e / R, i = i0 + e % R;
    float2 v = make_float2(0.f, 0.f);
    if (i < n) {
      if (t < st.n0) {
        const int q = st.t_diag[t], src = i + d.hoff[q];
        if (src >= 0 && src < n) v = __ldg(&hnh[q * n + src]);
      } else if (t < st.n0 + st.n1) {
        v = make_float2(1.f, 0.f);
      } else {
        const int p = d.pair_p[st.t_diag[t]], src = i + d.loff[p];
        if (src >= 0 && src < n) v = __ldg(&L[p * n + src]);
      }
    }
    rowc[e] = v;
  }
  {
    const int j = j0 + tid;
    for (int t = 0; t < nt; ++t) {
      float2 v = make_float2(0.f, 0.f);
      if (j < n) {
        if (t < st.n0) {
          v = make_float2(1.f, 0.f);
        } else if (t < st.n0 + st.n1) {
          const int q = st.t_diag[t], src = j + d.hoff[q];
          if (src >= 0 && src < n) v = cconj(__ldg(&hnh[q * n + src]));
        } else {
          const int sd = d.pair_s[st.t_diag[t]], src = j + d.loff[sd];
          if (src >= 0 && src < n) v = cconj(__ldg(&L[sd * n + src]));
        }
      }
      colc[t * kRhsCols + tid] = v;
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
  __syncthreads();
  const int j = j0 + tid;
  if (j >= n) return;
  const int rows = min(R, n - i0);
  const int e0 = st.n0, e1 = st.n0 + st.n1;
  for (int r = 0; r < rows; ++r) {
    float2 acc = make_float2(0.f, 0.f);
#pragma unroll 4
    for (int t = 0; t < e0; ++t)
      acc = cfma(rowc[t * R + r], S[st.t_base[t] + r * st.t_stride[t] + tid], acc);
#pragma unroll 4
    for (int t = e0; t < e1; ++t)
      acc = cfma(colc[t * kRhsCols + tid], S[st.t_base[t] + r * st.t_stride[t] + tid], acc);
#pragma unroll 2
    for (int t = e1; t < nt; ++t)
      acc = cfma(cmul(rowc[t * R + r], colc[t * kRhsCols + tid]), S[st.t_base[t] + r * st.t_stride[t] + tid],
                 acc);
    out[(long long)(i0 + r) * n + j] = cscale(acc, scale);
  }
}

// Wide f(X): C = 2 or 4 consecutive columns per thread, walked down R rows per CTA.  Every
// read of the stencil is C adjacent values X[i + ro][j + co .. j + co + C - 1]: 16-byte
// loads when j + co is even (j is a multiple of C, so that is when co is even), 8-byte
// loads at the odd ends otherwise.  The column factors of the thread's columns stay in
// registers for the whole walk (they do not depend on the row); the row factors of the
// CTA's R rows are a shared-memory table, as in the tiled kernel.  Terms (the host's
// DiaWide):
//   center   X[i][j]             hnh_0[i] + conj(hnh_0[j])       (row and column term of
//                                                                  Hnh's diagonal 0 at once)
//   row      X[i + k][j]         hnh_k[i + k]                     for Hnh's offsets k != 0
//   column   X[i][j + k]         conj(hnh_k[j + k])
//   pair     X[i + q_p][j + q_s] l_p[i + q_p] conj(l_s[j + q_s])
// -- the generic kernel's terms with fewer instructions per element: one load per two
// elements for most terms, and the column factors loaded once per thread instead of once
// per element.  Needs n to be a multiple of C (16-byte aligned rows); NR and NP are the
// numbers of row (= column) terms and pairs, padded by zero terms.
constexpr int kWideMaxNR = 8;
constexpr int kWideMaxNP = 4;

struct DiaWide {
  int has0, q0;                 // Hnh has diagonal 0, at index q0
  int nr;                       // real row / column terms (<= NR)
  int rq[kWideMaxNR];           // Hnh diagonal of each
  int rk[kWideMaxNR];           // its offset
  int np;                       // real pairs (<= NP)
  int pp[kWideMaxNP], ps[kWideMaxNP];    // jump diagonals p, s
  int pro[kWideMaxNP], pco[kWideMaxNP];  // their offsets
};

struct __align__(16) WideRow {
  float2 f;   // row factor
  int off;    // clamped source row times n
  int pad;
};

// C values X[row][col .. col + C - 1] (row pointer given); `inb`: all C columns inside the
// matrix (else every column is clamped: its factor is zero, the read only has to be a
// valid entry).
template <int C>
__device__ __forceinline__ void wide_load(const float2* __restrict__ rp, int col, bool inb, int n, float2 (&v)[C]) {
  if (inb) {
    if ((col & 1) == 0) {
#pragma unroll
      for (int h = 0; h < C / 2; ++h) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(rp + col + 2 * h));
        v[2 * h] = make_float2(a.x, a.y), v[2 * h + 1] = make_float2(a.z, a.w);
      }
    } else {
      v[0] = __ldg(rp + col);
#pragma unroll
      for (int h = 0; h < C / 2 - 1; ++h) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(rp + col + 1 + 2 * h));
        v[1 + 2 * h] = make_float2(a.x, a.y), v[2 + 2 * h] = make_float2(a.z, a.w);
      }
      v[C - 1] = __ldg(rp + col + C - 1);
    }
  } else {
#pragma unroll
    for (int q = 0; q < C; ++q) {
      const int cc = col + q;
      v[q] = __ldg(rp + (cc < 0 ? 0 : (cc >= n ? n - 1 : cc)));
    }
  }
}

// HERM (the hermitian form, X hermitian): f(X) is hermitian, so only the elements on and
// above the diagonal are computed -- a CTA whose tile lies below the diagonal exits at
// once -- and each strictly-upper element is also written, conjugated, at its mirror
// position, through a shared-memory strip of the CTA's R x (128 C) outputs so that the
// mirrored rows leave as contiguous R-value segments.  About half the stencil work, and
// the output is hermitian to the last bit.  `half` (HERM only): write the 32 x 32 tiles on
// and above the diagonal and nothing else -- every element (i, j) with j >= 32 floor(i / 32),
// the set the hermitian-half elementwise kernels read -- and no mirror, for a stage slot
// that only those kernels consume.
template <int R, int NR, int NP, int C, bool HERM, int U = 1, int MB = 4>
__global__ void __launch_bounds__(kRhsCols, MB) rhs_dia_wide_kernel(big::Common c, DiaOps d, DiaWide w, int in_sel,
                                                                  int out_k, int need_run, int kry,
                                                                  const float2* ext_in, float2* ext_out,
                                                                  int half) {
  constexpr int NT = 1 + NR + NP;  // row-table terms: center, rows, pairs
  constexpr int W = kRhsCols * C;  // columns of the CTA's tile
  constexpr int SW = W + 1;        // row stride of the strip (the mirror reads down columns)
  __shared__ WideRow rowt[NT][R];
  extern __shared__ float2 strip[];  // [R][SW] when HERM
  const int i0 = blockIdx.y * R;
  const int j0 = blockIdx.x * W;
  const int hmask = half ? ~31 : ~0;      // R divides 32: one diagonal tile row per CTA
  if (HERM && j0 + W - 1 < (i0 & hmask)) return;  // the whole tile is below the diagonal
  const int b = blockIdx.z;
  const float2* X;
  float2* out;
  float scale = 1.f;
  if (ext_in) {  // stand-alone evaluation (dqb_lindblad_rhs_dia)
    X = ext_in + (long long)b * d.n * d.n;
    out = ext_out + (long long)b * d.n * d.n;
  } else {
    RhsIo io;
    if (!rhs_io(c, b, in_sel, out_k, need_run, kry, io)) return;
    X = io.X;
    out = io.out;
    scale = io.scale;
  }
  const int n = d.n;
  const long long li = d.Lidx ? d.Lidx[b] : b;
  const float2* L = d.L + li * d.nl * n;
  const float2* hnh = d.hnh + (long long)b * d.nh * n;
  const int j = j0 + threadIdx.x * C;

  // row factors of the CTA's R rows
  for (int e = threadIdx.x; e < NT * R; e += blockDim.x) {
    const int t = e / R, r = e % R, i = i0 + r;
    int off = 0;
    const float2* diag = nullptr;
    if (t == 0) {
      if (w.has0) diag = hnh + w.q0 * n;
    } else if (t <= NR) {
      if (t - 1 < w.nr) off = w.rk[t - 1], diag = hnh + w.rq[t - 1] * n;
    } else {
      if (t - 1 - NR < w.np) off = w.pro[t - 1 - NR], diag = L + w.pp[t - 1 - NR] * n;
    }
    const int src = i + off;
    const bool in = diag != nullptr && i < n && src >= 0 && src < n;
    WideRow v;
    v.f = in ? __ldg(&diag[src]) : make_float2(0.f, 0.f);
    v.off = (src < 0 ? 0 : (src >= n ? n - 1 : src)) * n;
    v.pad = 0;
    rowt[t][r] = v;
  }
  __syncthreads();
  const bool active = j < n;  // n is a multiple of C: all C columns or none
  const int rows = min(R, n - i0);
  if (!HERM && !active) return;
  if (active) {
  // column factors of the thread's C columns
  float2 cc0[C], ccol[NR][C], cpair[NP][C];
  unsigned inb_col = 0, inb_pair = 0;
#pragma unroll
  for (int q = 0; q < C; ++q) cc0[q] = w.has0 ? cconj(__ldg(&hnh[w.q0 * n + j + q])) : make_float2(0.f, 0.f);
#pragma unroll
  for (int t = 0; t < NR; ++t) {
    const int k = t < w.nr ? w.rk[t] : 0;
    if (j + k >= 0 && j + k + C - 1 < n) inb_col |= 1u << t;
#pragma unroll
    for (int q = 0; q < C; ++q) {
      const int src = j + q + k;
      ccol[t][q] = (t < w.nr && src >= 0 && src < n) ? cconj(__ldg(&hnh[w.rq[t] * n + src])) : make_float2(0.f, 0.f);
    }
  }
#pragma unroll
  for (int t = 0; t < NP; ++t) {
    const int k = t < w.np ? w.pco[t] : 0;
    if (j + k >= 0 && j + k + C - 1 < n) inb_pair |= 1u << t;
#pragma unroll
    for (int q = 0; q < C; ++q) {
      const int src = j + q + k;
      cpair[t][q] = (t < w.np && src >= 0 && src < n) ? cconj(__ldg(&L[w.ps[t] * n + src])) : make_float2(0.f, 0.f);
    }
  }

#pragma unroll U  // U = 2: two rows' loads in flight per thread
  for (int r = 0; r < rows; ++r) {
    const int i = i0 + r;
    const int ilim = i & hmask;              // first column written in row i
    if (HERM && j + C - 1 < ilim) break;  // this and the later rows lie below the diagonal
    const float2* Xi = X + (long long)i * n;
    float2 acc[C];
    float2 v[C];
    {
      const WideRow rc = rowt[0][r];
      wide_load<C>(Xi, j, true, n, v);
#pragma unroll
      for (int q = 0; q < C; ++q) acc[q] = cmul(cadd(rc.f, cc0[q]), v[q]);
    }
#pragma unroll
    for (int t = 0; t < NR; ++t) {
      const WideRow rc = rowt[1 + t][r];
      wide_load<C>(X + rc.off, j, true, n, v);
#pragma unroll
      for (int q = 0; q < C; ++q) acc[q] = cfma(rc.f, v[q], acc[q]);
      const int k = t < w.nr ? w.rk[t] : 0;
      wide_load<C>(Xi, j + k, (inb_col >> t) & 1u, n, v);
#pragma unroll
      for (int q = 0; q < C; ++q) acc[q] = cfma(ccol[t][q], v[q], acc[q]);
    }
#pragma unroll
    for (int t = 0; t < NP; ++t) {
      const WideRow rc = rowt[1 + NR + t][r];
      const int k = t < w.np ? w.pco[t] : 0;
      wide_load<C>(X + rc.off, j + k, (inb_pair >> t) & 1u, n, v);
#pragma unroll
      for (int q = 0; q < C; ++q) acc[q] = cfma(cmul(rc.f, cpair[t][q]), v[q], acc[q]);
    }
#pragma unroll
    for (int q = 0; q < C; ++q) acc[q] = make_float2(acc[q].x * scale, acc[q].y * scale);
    if (HERM && j <= i && i < j + C) acc[i - j].y = 0.f;  // a hermitian matrix's diagonal is real
    float2* orow = out + (long long)i * n + j;
    if (!HERM || j >= ilim) {  // every column on or above the diagonal (its tile)
#pragma unroll
      for (int h = 0; h < C / 2; ++h)
        reinterpret_cast<float4*>(orow)[h] = make_float4(acc[2 * h].x, acc[2 * h].y, acc[2 * h + 1].x, acc[2 * h + 1].y);
    } else {
#pragma unroll
      for (int q = 0; q < C; ++q)
        if (j + q >= i) orow[q] = acc[q];
    }
    if (HERM && !half) {
#pragma unroll
      for (int q = 0; q < C; ++q) strip[r * SW + threadIdx.x * C + q] = acc[q];
    }
  }
  }  // active
  if (HERM && !half) {
    // mirror: out[jj][i0 + r] = conj(f[i0 + r][jj]) for jj > i0 + r, R contiguous values per
    // target row (R threads per row, one value each)
    __syncthreads();
    for (int e = threadIdx.x; e < W * R; e += kRhsCols) {
      const int r = e % R, cj = e / R;
      const int i = i0 + r, jj = j0 + cj;
      if (r < rows && jj < n && jj > i) out[(long long)jj * n + i] = cconj(strip[r * SW + cj]);
    }
  }
}

// Bulk-staged f(X), hermitian form: the rows of X a CTA's stencil reads are copied into
// shared memory by the bulk-copy (TMA) engine, one copy per staged row, two stages in
// flight, and every term then reads shared memory at its shifted position.  A CTA owns
// 256 columns (one per thread) and a band of kBulkBand rows, walked in stages of R rows;
// per stage it stages each group of row offsets that lie close together (DiaBulk: R +
// span rows of the group, its column halo included), so every row of X leaves L2 about
// three times instead of once per term, and no load of the stencil waits on L2.  Tiles
// below the diagonal are skipped and the strictly-upper elements mirrored, as in the wide
// kernel's hermitian half.  Rows and columns outside the matrix are zero in shared
// memory (zero-filled by the threads; the copies are clipped to the matrix).  Every wait
// is bounded; a wait that runs out makes the CTA drain its copies and write nothing.
constexpr int kBulkW = 256;      // columns per CTA (threads)
constexpr unsigned long long kBulkWaitNs = 200000000ull;  // 0.2 s: a stage's copies take microseconds
constexpr int kBulkBand = 256;   // rows per CTA
constexpr int kBulkMaxGroups = 4;
constexpr int kBulkMaxTerms = 1 + 2 * kWideMaxNR + kWideMaxNP;

struct DiaBulk {
  int ngroup;
  int g_rlo[kBulkMaxGroups];   // row offset of the group's first staged row
  int g_rows[kBulkMaxGroups];  // staged rows per stage: R + span of the group's row offsets
  int g_clo[kBulkMaxGroups];   // column offset of the first staged column (even)
  int g_cols[kBulkMaxGroups];  // staged columns (even)
  int g_off[kBulkMaxGroups];   // offset of the group in a stage buffer (complex values, even)
  int r_lo, r_hi, c_lo, c_hi;  // extreme row and column offsets staged (interior test)
  int stage;                   // complex values per stage buffer (even)
  // terms: 0 = center, 1..NR = row terms, NR+1..2NR = column terms, then the pairs
  int t_base[kBulkMaxTerms];   // stage offset of (row 0 of the stage, thread 0)
  int t_stride[kBulkMaxTerms]; // row stride of the term's group
};

template <int R, int NR, int NP>
__global__ void __launch_bounds__(kBulkW, 1) rhs_dia_bulk_kernel(big::Common c, DiaOps d, DiaWide w, DiaBulk pl,
                                                                int in_sel, int out_k, int need_run, int kry,
                                                                const float2* ext_in, float2* ext_out) {
  constexpr int NT = 1 + NR + NP;  // row-table terms: center, rows, pairs
  extern __shared__ float4 bulk_raw[];
  __shared__ uint64_t bars[2];
  __shared__ WideRow rowt[NT][R];
  __shared__ int fail_sh;
  const int j0 = blockIdx.x * kBulkW, I0 = blockIdx.y * kBulkBand;
  if (j0 + kBulkW - 1 < I0) return;  // the whole band is below the diagonal
  const int b = blockIdx.z;
  const float2* X;
  float2* out;
  float scale = 1.f;
  if (ext_in) {
    X = ext_in + (long long)b * d.n * d.n;
    out = ext_out + (long long)b * d.n * d.n;
  } else {
    RhsIo io;
    if (!rhs_io(c, b, in_sel, out_k, need_run, kry, io)) return;
    X = io.X;
    out = io.out;
    scale = io.scale;
  }
  const int n = d.n, tid = threadIdx.x;
  const long long li = d.Lidx ? d.Lidx[b] : b;
  const float2* L = d.L + li * d.nl * n;
  const float2* hnh = d.hnh + (long long)b * d.nh * n;
  float2* buf[2];
  buf[0] = reinterpret_cast<float2*>(bulk_raw);
  buf[1] = buf[0] + pl.stage;
  float2* strip = buf[1] + pl.stage;  // [R][kBulkW + 1]
  const uint32_t bar[2] = {tc::smem_u32(&bars[0]), tc::smem_u32(&bars[1])};
  // stages of this CTA: rows I0 .. I0 + kBulkBand - 1 inside the matrix, up to the last
  // stage that reaches the diagonal of the CTA's columns
  const int band_rows = min(kBulkBand, n - I0);
  int nst = (band_rows + R - 1) / R;
  nst = min(nst, (j0 + kBulkW - 1 - I0) / R + 1);
  if (tid == 0) {
    tc::mbar_init(bar[0], 1);
    tc::mbar_init(bar[1], 1);
    tc::fence_mbar_init();
    fail_sh = 0;
  }
  __syncthreads();

  // column factors of this thread's column
  const int j = j0 + tid;
  const bool jin = j < n;
  float2 ccen = make_float2(0.f, 0.f), ccol[NR], cpair[NP];
  if (jin && w.has0) ccen = cconj(__ldg(&hnh[w.q0 * n + j]));
#pragma unroll
  for (int t = 0; t < NR; ++t) {
    const int src = j + (t < w.nr ? w.rk[t] : 0);
    ccol[t] = (jin && t < w.nr && src >= 0 && src < n) ? cconj(__ldg(&hnh[w.rq[t] * n + src])) : make_float2(0.f, 0.f);
  }
#pragma unroll
  for (int t = 0; t < NP; ++t) {
    const int src = j + (t < w.np ? w.pco[t] : 0);
    cpair[t] = (jin && t < w.np && src >= 0 && src < n) ? cconj(__ldg(&L[w.ps[t] * n + src])) : make_float2(0.f, 0.f);
  }

  // stage st into buffer st & 1: the threads zero what the copies do not cover, then one
  // thread issues the copies (their bytes announced on the stage's barrier first)
  auto prep = [&](int st) {
    float2* B = buf[st & 1];
    const int is = I0 + st * R;
    const bool rows_in = is + pl.r_lo >= 0 && is + R - 1 + pl.r_hi < n;
    const bool cols_in = j0 + pl.c_lo >= 0 && j0 + kBulkW - 1 + pl.c_hi < n;
    if (!(rows_in && cols_in)) {
      for (int g = 0; g < pl.ngroup; ++g) {
        const int gr0 = is + pl.g_rlo[g], gc0 = j0 + pl.g_clo[g], cols = pl.g_cols[g];
        for (int e = tid; e < pl.g_rows[g] * cols; e += kBulkW) {
          const int rr = e / cols, cc = e % cols;
          const int gr = gr0 + rr, gc = gc0 + cc;
          if (gr < 0 || gr >= n || gc < 0 || gc >= n) B[pl.g_off[g] + e] = make_float2(0.f, 0.f);
        }
      }
    }
    if (tid == 0) {
      uint32_t bytes = 0;
      for (int g = 0; g < pl.ngroup; ++g) {
        const int gc0 = j0 + pl.g_clo[g];
        const int c_a = max(gc0, 0), c_b = min(gc0 + pl.g_cols[g], n);
        if (c_b <= c_a) continue;
        for (int rr = 0; rr < pl.g_rows[g]; ++rr) {
          const int gr = is + pl.g_rlo[g] + rr;
          if (gr >= 0 && gr < n) bytes += (uint32_t)(c_b - c_a) * 8u;
        }
      }
      tc::mbar_arrive_expect_tx(bar[st & 1], bytes);
      for (int g = 0; g < pl.ngroup; ++g) {
        const int gc0 = j0 + pl.g_clo[g];
        const int c_a = max(gc0, 0), c_b = min(gc0 + pl.g_cols[g], n);
        if (c_b <= c_a) continue;
        for (int rr = 0; rr < pl.g_rows[g]; ++rr) {
          const int gr = is + pl.g_rlo[g] + rr;
          if (gr < 0 || gr >= n) continue;
          float2* dst = B + pl.g_off[g] + rr * pl.g_cols[g] + (c_a - gc0);
          tc::bulk_copy_g2s(tc::smem_u32(dst), X + (long long)gr * n + c_a, (uint32_t)(c_b - c_a) * 8u,
                            bar[st & 1]);
        }
      }
    }
  };

  if (nst > 0) prep(0);
  int st = 0;
  for (; st < nst; ++st) {
    if (st + 1 < nst) prep(st + 1);
    const int is = I0 + st * R;
    // row factors of the stage's rows
    for (int e = tid; e < NT * R; e += kBulkW) {
      const int t = e / R, r = e % R, i = is + r;
      int off = 0;
      const float2* diag = nullptr;
      if (t == 0) {
        if (w.has0) diag = hnh + w.q0 * n;
      } else if (t <= NR) {
        if (t - 1 < w.nr) off = w.rk[t - 1], diag = hnh + w.rq[t - 1] * n;
      } else {
        if (t - 1 - NR < w.np) off = w.pro[t - 1 - NR], diag = L + w.pp[t - 1 - NR] * n;
      }
      const int src = i + off;
      WideRow v;
      v.f = (diag != nullptr && i < n && src >= 0 && src < n) ? __ldg(&diag[src]) : make_float2(0.f, 0.f);
      v.off = 0;
      v.pad = 0;
      rowt[t][r] = v;
    }
    __syncthreads();  // row table and this stage's zero-fill visible
    const bool ok = tc::mbar_wait_for(bar[st & 1], (uint32_t)((st >> 1) & 1), kBulkWaitNs);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) fail_sh = 1;
      break;
    }
    const float2* B = buf[st & 1];
    const int rows = min(R, n - is);
#pragma unroll 1
    for (int r = 0; r < rows; ++r) {
      const int i = is + r;
      if (!jin || j < i) continue;  // outside the matrix or below the diagonal
      float2 acc = cmul(cadd(rowt[0][r].f, ccen), B[pl.t_base[0] + r * pl.t_stride[0] + tid]);
#pragma unroll
      for (int t = 0; t < NR; ++t) {
        acc = cfma(rowt[1 + t][r].f, B[pl.t_base[1 + t] + r * pl.t_stride[1 + t] + tid], acc);
        acc = cfma(ccol[t], B[pl.t_base[1 + NR + t] + r * pl.t_stride[1 + NR + t] + tid], acc);
      }
#pragma unroll
      for (int t = 0; t < NP; ++t)
        acc = cfma(cmul(rowt[1 + NR + t][r].f, cpair[t]),
                   B[pl.t_base[1 + 2 * NR + t] + r * pl.t_stride[1 + 2 * NR + t] + tid], acc);
      acc = make_float2(acc.x * scale, i == j ? 0.f : acc.y * scale);  // a hermitian diagonal is real
      out[(long long)i * n + j] = acc;
      strip[r * (kBulkW + 1) + tid] = acc;
    }
    __syncthreads();
    // mirror: out[jj][i] = conj(f[i][jj]) for jj > i, R contiguous values per target row
    for (int e = tid; e < kBulkW * R; e += kBulkW) {
      const int r = e % R, cj = e / R;
      const int i = is + r, jj = j0 + cj;
      if (r < rows && jj < n && jj > i) out[(long long)jj * n + i] = cconj(strip[r * (kBulkW + 1) + cj]);
    }
    __syncthreads();  // strip, row table and buffer st & 1 are free again
  }
  if (fail_sh) {
    // drain (bounded): the failed stage's copies and the next stage's may still be in flight
    tc::mbar_wait_for(bar[st & 1], (uint32_t)((st >> 1) & 1), kBulkWaitNs);
    if (st + 1 < nst) tc::mbar_wait_for(bar[(st + 1) & 1], (uint32_t)(((st + 1) >> 1) & 1), kBulkWaitNs);
  }
}

// ------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------

size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

struct DiaLayout {
  size_t off_iter, off_inst, off_eacc, off_hnh, off_hnh0, off_lt, off_mats, total;
};

int build_ops(const dqb_dia_problem* p, DiaOps* d) {
  std::memset(d, 0, sizeof(*d));
  if (p->h_ndiag < 0 || p->h_ndiag > DQB_DIA_MAX_HNH_DIAGS) return DQB_ERR_UNSUPPORTED;
  if (p->n_jumps < 0 || p->n_jumps > DQB_DIA_MAX_JUMPS) return DQB_ERR_UNSUPPORTED;
  if (p->h_ndiag > 0 && !p->h_offsets) return DQB_ERR_INVALID_ARGUMENT;
  if (p->n_jumps > 0 && (!p->l_ndiag || !p->l_offsets)) return DQB_ERR_INVALID_ARGUMENT;
  d->n = p->n;
  d->h_nd = p->h_ndiag;
  d->K = p->n_jumps;
  int nl = 0;
  d->lstart[0] = 0;
  for (int k = 0; k < p->n_jumps; ++k) {
    if (p->l_ndiag[k] < 0) return DQB_ERR_INVALID_ARGUMENT;
    nl += p->l_ndiag[k];
    if (nl > DQB_DIA_MAX_JUMP_DIAGS) return DQB_ERR_UNSUPPORTED;
    d->lstart[k + 1] = nl;
  }
  d->nl = nl;
  std::set<int> offs;
  for (int q = 0; q < p->h_ndiag; ++q) {
    const int k = p->h_offsets[q];
    if (k <= -p->n || k >= p->n) return DQB_ERR_INVALID_ARGUMENT;
    offs.insert(k);
  }
  d->npair = 0;
  for (int k = 0; k < p->n_jumps; ++k)
    for (int a = d->lstart[k]; a < d->lstart[k + 1]; ++a)
      for (int b = d->lstart[k]; b < d->lstart[k + 1]; ++b) {
        if (d->npair < 64) {
          d->pair_p[d->npair] = a;
          d->pair_s[d->npair] = b;
        }
        d->npair++;  // counts past 64 too: the fast kernel is then not used
      }
  for (int q = 0; q < nl; ++q) {
    d->loff[q] = p->l_offsets[q];
    if (d->loff[q] <= -p->n || d->loff[q] >= p->n) return DQB_ERR_INVALID_ARGUMENT;
  }
  for (int k = 0; k < p->n_jumps; ++k)
    for (int a = d->lstart[k]; a < d->lstart[k + 1]; ++a)
      for (int c = d->lstart[k]; c < d->lstart[k + 1]; ++c) {
        const int o = d->loff[c] - d->loff[a];
        if (o > -p->n && o < p->n) offs.insert(o);
      }
  if ((int)offs.size() > DQB_DIA_MAX_HNH_DIAGS) return DQB_ERR_UNSUPPORTED;
  d->nh = 0;
  for (int o : offs) {
    d->hoff[d->nh] = o;
    d->hmap[d->nh] = -1;
    for (int q = 0; q < p->h_ndiag; ++q)
      if (p->h_offsets[q] == o) d->hmap[d->nh] = q;
    d->nh++;
  }
  d->H = (const float2*)p->h_diags;
  d->L = (const float2*)p->l_diags;
  d->Hidx = p->H_index;
  d->Lidx = p->L_index;
  return DQB_OK;
}

DiaLayout layout_for(const dqb_dia_problem* p, int nh) {
  DiaLayout l;
  const size_t B = (size_t)p->batch, n = (size_t)p->n;
  l.off_iter = 0;
  l.off_inst = 256;
  l.off_eacc = align_up(l.off_inst + B * sizeof(big::Inst));
  l.off_hnh = align_up(l.off_eacc + B * (size_t)p->n_exp * p->n_tsave * sizeof(double2));
  l.off_hnh0 = align_up(l.off_hnh + B * (size_t)nh * n * sizeof(float2));
  size_t nl = 0;
  for (int k = 0; k < p->n_jumps; ++k) nl += (size_t)p->l_ndiag[k];
  l.off_lt = align_up(l.off_hnh0 + B * (size_t)nh * n * sizeof(float2));
  l.off_mats = align_up(l.off_lt + B * nl * n * sizeof(float2));
  l.total = l.off_mats + B * big::kSlots * n * n * sizeof(float2);
  return l;
}

// Operator fields (what a right-hand side needs).
int check_ops(const dqb_dia_problem* p) {
  if (!p) return DQB_ERR_INVALID_ARGUMENT;
  if (p->n < 2 || p->n_jumps < 0 || p->batch < 0) return DQB_ERR_INVALID_ARGUMENT;
  if (p->batch > 65535) return DQB_ERR_UNSUPPORTED;
  if ((p->h_ndiag > 0 && !p->h_diags) || (p->n_jumps > 0 && !p->l_diags)) return DQB_ERR_INVALID_ARGUMENT;
  return DQB_OK;
}

// Everything a solve needs.
int check_problem(const dqb_dia_problem* p) {
  int rc = check_ops(p);
  if (rc) return rc;
  if (p->n_exp < 0 || p->n_tsave < 1 || !p->rho0 || !p->tsave) return DQB_ERR_INVALID_ARGUMENT;
  if (p->n_exp > 0 && !p->E) return DQB_ERR_INVALID_ARGUMENT;
  return DQB_OK;
}

bool fast_ok(const DiaOps& d) {  // row offsets i * n held in int32
  return d.npair <= 64 && d.nh + d.npair <= kTiledMaxTerms && d.n <= 46340;
}

size_t tiled_smem(const DiaOps& d, int rows) {
  return (size_t)(d.nh + d.npair) * (rows + kRhsCols) * sizeof(DiaCoef);
}

// Staging plan of rhs_dia_staged_kernel<R> (see DiaStage); false when the operators need
// more groups, terms or shared memory than it allows.
bool plan_stage(const DiaOps& d, int R, DiaStage* st, size_t* smem) {
  std::memset(st, 0, sizeof(*st));
  if (d.n > 46340 || d.npair > 64) return false;
  const int nt = 2 * d.nh + d.npair;
  if (nt > kStageMaxTerms) return false;
  int ro[kStageMaxTerms], co[kStageMaxTerms], diag[kStageMaxTerms];
  int t = 0;
  for (int q = 0; q < d.nh; ++q, ++t) ro[t] = d.hoff[q], co[t] = 0, diag[t] = q;
  for (int q = 0; q < d.nh; ++q, ++t) ro[t] = 0, co[t] = d.hoff[q], diag[t] = q;
  for (int k = 0; k < d.npair; ++k, ++t) ro[t] = d.loff[d.pair_p[k]], co[t] = d.loff[d.pair_s[k]], diag[t] = k;
  std::vector<int> rs(ro, ro + nt);
  std::sort(rs.begin(), rs.end());
  rs.erase(std::unique(rs.begin(), rs.end()), rs.end());
  int glo[kStageMaxGroups], ghi[kStageMaxGroups], ng = 0;
  for (int v : rs) {
    if (ng > 0 && v - ghi[ng - 1] <= R) {
      ghi[ng - 1] = v;
    } else {
      if (ng == kStageMaxGroups) return false;
      glo[ng] = ghi[ng] = v;
      ++ng;
    }
  }
  st->ngroup = ng;
  int total = 0;
  for (int g = 0; g < ng; ++g) {
    int clo = 1 << 30, chi = -(1 << 30);
    for (int k = 0; k < nt; ++k)
      if (ro[k] >= glo[g] && ro[k] <= ghi[g]) clo = std::min(clo, co[k]), chi = std::max(chi, co[k]);
    st->g_rlo[g] = glo[g];
    st->g_rows[g] = R + ghi[g] - glo[g];
    st->g_clo[g] = clo;
    st->g_cols[g] = kRhsCols + chi - clo;
    st->g_off[g] = total;
    total += st->g_rows[g] * st->g_cols[g];
  }
  st->staged = total;
  st->n0 = d.nh;
  st->n1 = d.nh;
  st->n2 = d.npair;
  for (int k = 0; k < nt; ++k) {
    int g = 0;
    while (!(ro[k] >= glo[g] && ro[k] <= ghi[g])) ++g;
    st->t_diag[k] = diag[k];
    st->t_stride[k] = st->g_cols[g];
    st->t_base[k] = st->g_off[g] + (ro[k] - glo[g]) * st->g_cols[g] + (co[k] - st->g_clo[g]);
  }
  *smem = ((size_t)total + (size_t)nt * (R + kRhsCols)) * sizeof(float2);
  return *smem <= kStageMaxSmem;
}

// Terms of the wide kernel (see rhs_dia_wide_kernel); false when the operators have more
// row / column or pair terms than it holds, or rows it cannot address.
bool plan_wide(const DiaOps& d, int C, DiaWide* w) {
  std::memset(w, 0, sizeof(*w));
  if (d.n % C != 0 || d.n > 46340 || d.npair > kWideMaxNP) return false;
  w->q0 = 0;
  for (int q = 0; q < d.nh; ++q) {
    if (d.hoff[q] == 0) {
      w->has0 = 1;
      w->q0 = q;
    } else {
      if (w->nr == kWideMaxNR) return false;
      w->rq[w->nr] = q;
      w->rk[w->nr] = d.hoff[q];
      w->nr++;
    }
  }
  w->np = d.npair;
  for (int t = 0; t < d.npair; ++t) {
    w->pp[t] = d.pair_p[t];
    w->ps[t] = d.pair_s[t];
    w->pro[t] = d.loff[d.pair_p[t]];
    w->pco[t] = d.loff[d.pair_s[t]];
  }
  return true;
}

// Staging plan of rhs_dia_bulk_kernel<R> (see DiaBulk) from the wide kernel's terms; false
// when the groups or the shared memory do not fit.
bool plan_bulk(const DiaOps& d, const DiaWide& w, int R, int NR, int NP, DiaBulk* pl, size_t* smem) {
  std::memset(pl, 0, sizeof(*pl));
  if (d.n % 2 != 0 || d.n > 46340) return false;
  const int nt = 1 + 2 * NR + NP;
  int ro[kBulkMaxTerms], co[kBulkMaxTerms];
  ro[0] = co[0] = 0;
  for (int t = 0; t < NR; ++t) {
    const int k = t < w.nr ? w.rk[t] : 0;
    ro[1 + t] = k, co[1 + t] = 0;
    ro[1 + NR + t] = 0, co[1 + NR + t] = k;
  }
  for (int t = 0; t < NP; ++t) {
    ro[1 + 2 * NR + t] = t < w.np ? w.pro[t] : 0;
    co[1 + 2 * NR + t] = t < w.np ? w.pco[t] : 0;
  }
  std::vector<int> rs(ro, ro + nt);
  std::sort(rs.begin(), rs.end());
  rs.erase(std::unique(rs.begin(), rs.end()), rs.end());
  int glo[kBulkMaxGroups], ghi[kBulkMaxGroups], ng = 0;
  for (int v : rs) {
    if (ng > 0 && v - ghi[ng - 1] <= R) {
      ghi[ng - 1] = v;
    } else {
      if (ng == kBulkMaxGroups) return false;
      glo[ng] = ghi[ng] = v;
      ++ng;
    }
  }
  pl->ngroup = ng;
  int total = 0;
  pl->r_lo = pl->c_lo = 1 << 30;
  pl->r_hi = pl->c_hi = -(1 << 30);
  for (int g = 0; g < ng; ++g) {
    int clo = 1 << 30, chi = -(1 << 30);
    for (int t = 0; t < nt; ++t)
      if (ro[t] >= glo[g] && ro[t] <= ghi[g]) clo = std::min(clo, co[t]), chi = std::max(chi, co[t]);
    const int clo_e = clo - (((clo % 2) + 2) % 2);  // even (16-byte aligned copies)
    int cols = kBulkW + chi - clo_e;
    cols += cols % 2;
    pl->g_rlo[g] = glo[g];
    pl->g_rows[g] = R + ghi[g] - glo[g];
    pl->g_clo[g] = clo_e;
    pl->g_cols[g] = cols;
    pl->g_off[g] = total;
    total += pl->g_rows[g] * cols;
    pl->r_lo = std::min(pl->r_lo, glo[g]);
    pl->r_hi = std::max(pl->r_hi, ghi[g]);
    pl->c_lo = std::min(pl->c_lo, clo_e);
    pl->c_hi = std::max(pl->c_hi, clo_e + cols - kBulkW);
  }
  pl->stage = total;
  for (int t = 0; t < nt; ++t) {
    int g = 0;
    while (!(ro[t] >= glo[g] && ro[t] <= ghi[g])) ++g;
    pl->t_stride[t] = pl->g_cols[g];
    pl->t_base[t] = pl->g_off[g] + (ro[t] - glo[g]) * pl->g_cols[g] + (co[t] - pl->g_clo[g]);
  }
  *smem = (2 * (size_t)total + (size_t)R * (kBulkW + 1)) * sizeof(float2);
  return *smem <= kStageMaxSmem;
}

// Compile-time term counts of the wide kernel's instances: NR in {4, 8}, NP in {2, 4},
// padded by zero terms.
int wide_nr(int nr) { return nr <= 4 ? 4 : 8; }
int wide_np(int np) { return np <= 2 ? 2 : 4; }

// Shape codes of the wide kernel: 200 + R (C = 4 columns per thread) or 300 + R (C = 2),
// R = 8 or 16 rows per CTA; 408 / 508: 8 rows, two rows' loads in flight per thread;
// 708: 8 rows with C = 2, registers capped for 6 resident CTAs per SM (instead of 4) so
// that more warps hide the shifted loads' latency (C = 4 capped for 5 CTAs spills).
bool is_wide(int rows) {
  return rows == 208 || rows == 216 || rows == 308 || rows == 316 || rows == 408 || rows == 508 ||
         rows == 708;
}
bool is_bulk(int rows) { return rows == 604 || rows == 608; }
int wide_c(int rows) { return (rows / 100) % 2 == 1 ? 2 : 4; }  // 2xx, 4xx: 4; 3xx, 5xx, 7xx: 2
int wide_r(int rows) { return rows % 100; }

// Launch shape of the stencil from `tile`: 4, 8 or 16 = the tiled kernel with that many rows
// per thread (when the operators have at most kTiledMaxTerms diagonal terms); 108 or 116 =
// the staged kernel with 8 or 16 rows per CTA (when its plan fits); 208 or 216 (4 columns
// per thread), 308 or 316 (2 columns) = the wide kernel with 8 or 16 rows per CTA, 408 /
// 508 = 8 rows with two rows in flight per thread, 708 = 8 rows (2 columns) with registers
// capped for more resident CTAs (when its plan fits); anything else (0 =
// default, 1) = the generic kernel.  The autotuner picks among them per problem shape.
// Returns the shape code (1 = generic).
int rows_for(const DiaOps& d, int tile) {
  if (is_bulk(tile)) {
    DiaWide w;
    DiaBulk pl;
    size_t sm;
    if (plan_wide(d, 2, &w) && plan_bulk(d, w, tile - 600, wide_nr(w.nr), wide_np(w.np), &pl, &sm)) return tile;
  }
  if (is_wide(tile)) {
    DiaWide w;
    if (plan_wide(d, wide_c(tile), &w)) return tile;
  }
  if (tile == 108 || tile == 116) {
    DiaStage st;
    size_t sm;
    if (plan_stage(d, tile - 100, &st, &sm)) return tile;
  }
  if (!fast_ok(d)) return 1;
  return (tile == 4 || tile == 8 || tile == 16) ? tile : 1;
}

dim3 rhs_grid(const DiaOps& d, int rows, int B) {
  if (is_bulk(rows)) return dim3((d.n + kBulkW - 1) / kBulkW, (d.n + kBulkBand - 1) / kBulkBand, B);
  if (is_wide(rows)) {
    const int r = wide_r(rows), cols = kRhsCols * wide_c(rows);
    return dim3((d.n + cols - 1) / cols, (d.n + r - 1) / r, B);
  }
  const int r = rows == 1 ? kRhsRows : (rows > 100 ? rows - 100 : rows);
  return dim3((d.n + kRhsCols - 1) / kRhsCols, (d.n + r - 1) / r, B);
}

template <int R, int C, bool HERM, int U, int MB>
void launch_wide_form(cudaStream_t s, dim3 g, const big::Common& c, const DiaOps& d, const DiaWide& w,
                      int in_sel, int out_k, int need_run, int kry, const float2* ext_in, float2* ext_out,
                      int half) {
  const int nr = wide_nr(w.nr), np = wide_np(w.np);
  const size_t sm = HERM && !half ? (size_t)R * (kRhsCols * C + 1) * sizeof(float2) : 0;
  if (nr == 4 && np == 2)
    rhs_dia_wide_kernel<R, 4, 2, C, HERM, U, MB><<<g, kRhsCols, sm, s>>>(c, d, w, in_sel, out_k, need_run, kry,
                                                                    ext_in, ext_out, half);
  else if (nr == 4)
    rhs_dia_wide_kernel<R, 4, 4, C, HERM, U, MB><<<g, kRhsCols, sm, s>>>(c, d, w, in_sel, out_k, need_run, kry,
                                                                    ext_in, ext_out, half);
  else if (np == 2)
    rhs_dia_wide_kernel<R, 8, 2, C, HERM, U, MB><<<g, kRhsCols, sm, s>>>(c, d, w, in_sel, out_k, need_run, kry,
                                                                    ext_in, ext_out, half);
  else
    rhs_dia_wide_kernel<R, 8, 4, C, HERM, U, MB><<<g, kRhsCols, sm, s>>>(c, d, w, in_sel, out_k, need_run, kry,
                                                                    ext_in, ext_out, half);
}

template <int R>
void launch_bulk(cudaStream_t s, dim3 g, const big::Common& c, const DiaOps& d, const DiaWide& w, int in_sel,
                 int out_k, int need_run, int kry, const float2* ext_in, float2* ext_out) {
  const int nr = wide_nr(w.nr), np = wide_np(w.np);
  DiaBulk pl;
  size_t sm = 0;
  plan_bulk(d, w, R, nr, np, &pl, &sm);  // rows_for checked that it fits
  if (nr == 4 && np == 2)
    rhs_dia_bulk_kernel<R, 4, 2><<<g, kBulkW, sm, s>>>(c, d, w, pl, in_sel, out_k, need_run, kry, ext_in, ext_out);
  else if (nr == 4)
    rhs_dia_bulk_kernel<R, 4, 4><<<g, kBulkW, sm, s>>>(c, d, w, pl, in_sel, out_k, need_run, kry, ext_in, ext_out);
  else if (np == 2)
    rhs_dia_bulk_kernel<R, 8, 2><<<g, kBulkW, sm, s>>>(c, d, w, pl, in_sel, out_k, need_run, kry, ext_in, ext_out);
  else
    rhs_dia_bulk_kernel<R, 8, 4><<<g, kBulkW, sm, s>>>(c, d, w, pl, in_sel, out_k, need_run, kry, ext_in, ext_out);
}

template <int R, int C, int U = 1, int MB = 4>
void launch_wide(cudaStream_t s, dim3 g, const big::Common& c, const DiaOps& d, const DiaWide& w, int in_sel,
                 int out_k, int need_run, int kry, const float2* ext_in, float2* ext_out, bool herm, bool half) {
  if (herm)
    launch_wide_form<R, C, true, U, MB>(s, g, c, d, w, in_sel, out_k, need_run, kry, ext_in, ext_out, half ? 1 : 0);
  else
    launch_wide_form<R, C, false, U, MB>(s, g, c, d, w, in_sel, out_k, need_run, kry, ext_in, ext_out, 0);
}

// One right-hand side of every instance: k[out_k] = f(input), through the kernel the shape
// code `rows` selects (rows_for).  `half` (hermitian form): the output only has to hold the
// 32 x 32 tiles on and above the diagonal (a stage slot read by the hermitian-half
// elementwise kernels alone); the wide kernels then write nothing else, the others write
// the whole matrix all the same.
void launch_rhs_dia(cudaStream_t s, const big::Common& c, const DiaOps& d, int B, int rows, int in_sel,
                    int out_k, int need_run, const float2* ext_in, float2* ext_out, int kry = 0,
                    bool herm = false, bool half = false) {
  if (is_bulk(rows) && !herm) rows = 308;  // the bulk kernel is hermitian-only
  const dim3 g = rhs_grid(d, rows, B);
  if (is_bulk(rows)) {
    DiaWide w;
    plan_wide(d, 2, &w);
    if (rows == 604)
      launch_bulk<4>(s, g, c, d, w, in_sel, out_k, need_run, kry, ext_in, ext_out);
    else
      launch_bulk<8>(s, g, c, d, w, in_sel, out_k, need_run, kry, ext_in, ext_out);
    return;
  }
  if (is_wide(rows)) {
    DiaWide w;
    plan_wide(d, wide_c(rows), &w);  // rows_for checked that it fits
    switch (rows) {
      case 208: launch_wide<8, 4>(s, g, c, d, w, in_sel, out_k, need_run, kry, ext_in, ext_out, herm, half); break;
      case 216: launch_wide<16, 4>(s, g, c, d, w, in_sel, out_k, need_run, kry, ext_in, ext_out, herm, half); break;
      case 308: launch_wide<8, 2>(s, g, c, d, w, in_sel, out_k, need_run, kry, ext_in, ext_out, herm, half); break;
      case 408: launch_wide<8, 4, 2>(s, g, c, d, w, in_sel, out_k, need_run, kry, ext_in, ext_out, herm, half); break;
      case 508: launch_wide<8, 2, 2>(s, g, c, d, w, in_sel, out_k, need_run, kry, ext_in, ext_out, herm, half); break;
      case 708: launch_wide<8, 2, 1, 6>(s, g, c, d, w, in_sel, out_k, need_run, kry, ext_in, ext_out, herm, half); break;
      default: launch_wide<16, 2>(s, g, c, d, w, in_sel, out_k, need_run, kry, ext_in, ext_out, herm, half);
    }
    return;
  }
  if (rows > 100) {
    DiaStage st;
    size_t sm = 0;
    plan_stage(d, rows - 100, &st, &sm);  // rows_for checked that it fits
    if (rows == 116)
      rhs_dia_staged_kernel<16><<<g, kRhsCols, sm, s>>>(c, d, st, in_sel, out_k, need_run, kry, ext_in, ext_out);
    else
      rhs_dia_staged_kernel<8><<<g, kRhsCols, sm, s>>>(c, d, st, in_sel, out_k, need_run, kry, ext_in, ext_out);
    return;
  }
  const size_t sm = tiled_smem(d, rows);
  if (rows == 4) {
    rhs_dia_tiled_kernel<4><<<g, kRhsCols, sm, s>>>(c, d, in_sel, out_k, need_run, kry, ext_in, ext_out);
  } else if (rows == 8) {
    rhs_dia_tiled_kernel<8><<<g, kRhsCols, sm, s>>>(c, d, in_sel, out_k, need_run, kry, ext_in, ext_out);
  } else if (rows == 16) {
    rhs_dia_tiled_kernel<16><<<g, kRhsCols, sm, s>>>(c, d, in_sel, out_k, need_run, kry, ext_in, ext_out);
  } else {
    rhs_dia_generic_kernel<<<g, kRhsCols, 0, s>>>(c, d, in_sel, out_k, need_run, kry, ext_in, ext_out);
  }
}

GraphCache g_cache;

struct LaunchKey {
  big::Common c;
  DiaOps d;
  TdOps td;
  DiaJumpTd jt;
  int grid_e, grid_r_x, grid_r_y, krylov;
};

}  // namespace
}  // namespace dqb

using namespace dqb;

// One-time: every kernel of this file asks for the same (largest) shared-memory carveout.
static void init_carveouts() {
  static std::once_flag once;
  std::call_once(once, [] {
    prefer_max_shared(big::setup_kernel);
    prefer_max_shared(big::load_rho0_kernel);
    prefer_max_shared(big::combine_kernel);
    prefer_max_shared(big::error_kernel);
    prefer_max_shared(big::init_norm_kernel);
    prefer_max_shared(big::init_ctrl_kernel);
    prefer_max_shared(big::control_kernel);
    prefer_max_shared(big::save_kernel);
    prefer_max_shared(big::save_h_kernel<true>);
    prefer_max_shared(big::save_h_kernel<false>);
    prefer_max_shared(big::commit_kernel);
    prefer_max_shared(big::kry_combine_kernel);
    prefer_max_shared(big::combine_h_kernel<true>);
    prefer_max_shared(big::combine_h_kernel<false>);
    prefer_max_shared(big::error_h_kernel<true>);
    prefer_max_shared(big::error_h_kernel<false>);
    prefer_max_shared(big::kry_combine_h_kernel<true>);
    prefer_max_shared(big::kry_combine_h_kernel<false>);
    prefer_max_shared(big::kry_commit_kernel);
    prefer_max_shared(big::pre_finalize_kernel);
    prefer_max_shared(big::finalize_kernel);
    prefer_max_shared(zero_words_kernel);
    prefer_max_shared(hnh_dia_kernel);
    prefer_max_shared(hnh_td_kernel);
    prefer_max_shared(hnh_td_jump_kernel);
    prefer_max_shared(rhs_dia_generic_kernel);
    prefer_max_shared(rhs_dia_tiled_kernel<4>);
    prefer_max_shared(rhs_dia_tiled_kernel<8>);
    prefer_max_shared(rhs_dia_tiled_kernel<16>);
    prefer_max_shared(rhs_dia_staged_kernel<8>);
    prefer_max_shared(rhs_dia_staged_kernel<16>);
    auto herm_attr = [](auto kern) {
      prefer_max_shared(kern);
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           16 * (kRhsCols * 4 + 1) * (int)sizeof(float2));
    };
    auto bulk_attr = [](auto kern) {
      prefer_max_shared(kern);
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStageMaxSmem);
    };
    bulk_attr(rhs_dia_bulk_kernel<4, 4, 2>);
    bulk_attr(rhs_dia_bulk_kernel<4, 4, 4>);
    bulk_attr(rhs_dia_bulk_kernel<4, 8, 2>);
    bulk_attr(rhs_dia_bulk_kernel<4, 8, 4>);
    bulk_attr(rhs_dia_bulk_kernel<8, 4, 2>);
    bulk_attr(rhs_dia_bulk_kernel<8, 4, 4>);
    bulk_attr(rhs_dia_bulk_kernel<8, 8, 2>);
    bulk_attr(rhs_dia_bulk_kernel<8, 8, 4>);
    herm_attr(rhs_dia_wide_kernel<16, 4, 2, 4, true>);
    herm_attr(rhs_dia_wide_kernel<16, 4, 4, 4, true>);
    herm_attr(rhs_dia_wide_kernel<16, 8, 2, 4, true>);
    herm_attr(rhs_dia_wide_kernel<16, 8, 4, 4, true>);
    cudaFuncSetAttribute(rhs_dia_staged_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStageMaxSmem);
    cudaFuncSetAttribute(rhs_dia_staged_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kStageMaxSmem);
  });
}

extern "C" size_t dqb_mesolve_dia_workspace_size(const dqb_dia_problem* p) {
  if (check_problem(p)) return 0;
  DiaOps d;
  if (build_ops(p, &d)) return 0;
  return layout_for(p, d.nh).total;
}

extern "C" int dqb_lindblad_rhs_dia(const dqb_dia_problem* p, int32_t form, const void* rho, void* outp,
                                    void* workspace, size_t workspace_bytes, void* stream) {
  return dqb_lindblad_rhs_dia_tiled(p, form, 0, rho, outp, workspace, workspace_bytes, stream);
}

extern "C" int dqb_lindblad_rhs_dia_tiled(const dqb_dia_problem* p, int32_t form, int32_t tile, const void* rho,
                                          void* outp, void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_ops(p);
  if (rc) return rc;
  if (!rho || !outp) return DQB_ERR_INVALID_ARGUMENT;
  if (form != DQB_FORM_HERMITIAN && form != DQB_FORM_STANDARD && form != DQB_FORM_HERMITIAN_UPPER)
    return DQB_ERR_INVALID_ARGUMENT;
  if (p->batch == 0) return DQB_OK;
  DiaOps d;
  rc = build_ops(p, &d);
  if (rc) return rc;
  const size_t need = (size_t)p->batch * d.nh * p->n * sizeof(float2);
  if (!workspace || workspace_bytes < need) return DQB_ERR_WORKSPACE_TOO_SMALL;
  d.hnh = (float2*)workspace;
  cudaStream_t s = (cudaStream_t)stream;
  init_carveouts();
  hnh_dia_kernel<<<dim3((p->n + 255) / 256, (unsigned)p->batch), 256, 0, s>>>(d, (int)p->batch);
  big::Common c;
  std::memset(&c, 0, sizeof(c));
  int rows = rows_for(d, tile);
  if ((is_wide(rows) || is_bulk(rows)) &&
      ((reinterpret_cast<uintptr_t>(rho) | reinterpret_cast<uintptr_t>(outp)) & 15))
    rows = 1;
  launch_rhs_dia(s, c, d, (int)p->batch, rows, 2, 0, 0, (const float2*)rho, (float2*)outp, 0,
                 form != DQB_FORM_STANDARD, form == DQB_FORM_HERMITIAN_UPPER);
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}

// The solve; `tdh` (or null) adds the time-dependent terms of H and the discontinuity
// times of the controller.
static int solve_dia(const dqb_dia_problem* p, const dqb_td_hamiltonian* tdh, const dqb_ode_options* o,
                     const dqb_outputs* out, void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_problem(p);
  if (rc) return rc;
  if (!o || !out || !out->states || !out->infos || !out->status || (p->n_exp > 0 && !out->expects))
    return DQB_ERR_INVALID_ARGUMENT;
  if (o->method != DQB_METHOD_TSIT5 && o->method != DQB_METHOD_DOPRI5) return DQB_ERR_INVALID_ARGUMENT;
  if (o->form != DQB_FORM_HERMITIAN && o->form != DQB_FORM_STANDARD) return DQB_ERR_INVALID_ARGUMENT;
  if (!(o->rtol >= 0) || !(o->atol >= 0) || o->max_steps < 0) return DQB_ERR_INVALID_ARGUMENT;
  if (o->stepper < DQB_STEPPER_AUTO || o->stepper > DQB_STEPPER_KRYLOV) return DQB_ERR_INVALID_ARGUMENT;
  TdOps td;
  std::memset(&td, 0, sizeof(td));
  DiaJumpTd jt;
  std::memset(&jt, 0, sizeof(jt));
  if (tdh) {
    // the Krylov form needs a constant right-hand side
    if (o->stepper == DQB_STEPPER_KRYLOV) return DQB_ERR_UNSUPPORTED;
    if (int tr = td_ops_from(tdh, &td)) return tr;
    if (tdh->jump_terms) {
      jt.on = 1;
      for (int k = 0; k < p->n_jumps; ++k)
        if (int tr = td_term_from(tdh->jump_terms[k], &jt.term[k])) return tr;
    }
  }
  if (p->batch == 0) return DQB_OK;
  DiaOps d;
  rc = build_ops(p, &d);
  if (rc) return rc;
  const DiaLayout lay = layout_for(p, d.nh);
  if (!workspace || workspace_bytes < lay.total) return DQB_ERR_WORKSPACE_TOO_SMALL;
  char* ws = (char*)workspace;
  d.hnh = (float2*)(ws + lay.off_hnh);
  d.hnh0 = (float2*)(ws + lay.off_hnh0);
  const bool timedep = tdh != nullptr;
  if (jt.on) {  // the stencils read the per-instance copies c_k(t) L_k
    d.L0 = d.L;
    d.L0idx = d.Lidx;
    d.L = (const float2*)(ws + lay.off_lt);
    d.Lidx = nullptr;
  }

  big::Common c;
  std::memset(&c, 0, sizeof(c));
  c.n = p->n;
  c.nn = (long long)p->n * p->n;
  c.B = (int)p->batch;
  c.nE = p->n_exp;
  c.ntsave = p->n_tsave;
  c.form = o->form;
  c.save_states = o->save_states;
  c.rho0_is_ket = p->rho0_is_ket;
  c.o = make_ctrl(*o);
  c.tsave = p->tsave;
  c.inst = (big::Inst*)(ws + lay.off_inst);
  c.mats = (float2*)(ws + lay.off_mats);
  c.eacc = (double2*)(ws + lay.off_eacc);
  c.states = (float2*)out->states;
  c.expects = (float2*)out->expects;
  c.infos = out->infos;
  c.status = out->status;
  c.E = (const float2*)p->E;
  c.rho0 = (const float2*)p->rho0;
  c.ridx = p->rho0_index;
  c.iter = (long long*)(ws + lay.off_iter);
  if (timedep) {
    c.n_jump = tdh->n_jump_ts;
    c.jump_ts = tdh->jump_ts;
  }

  cudaStream_t s = (cudaStream_t)stream;
  const int B = c.B;
  const long long nn = c.nn;
  int grid_e = (int)std::min<long long>((nn + big::kElemThreads - 1) / big::kElemThreads, 1184);
  if (grid_e < 1) grid_e = 1;
  const dim3 ge(grid_e, B);
  int rows = rows_for(d, o->tile);
  if ((is_wide(rows) || is_bulk(rows)) && (reinterpret_cast<uintptr_t>(c.mats) & 15)) rows = 1;
  const bool krylov = o->stepper == DQB_STEPPER_KRYLOV;
  const bool herm = o->form == DQB_FORM_HERMITIAN;
  const dim3 gi((B + 127) / 128);
  const int T = big::kElemThreads;

  // ---- set-up and starting step (outside the graph) ----------------------------------
  init_carveouts();
  big::setup_kernel<<<gi, 128, 0, s>>>(c);
  if (!jt.on) {  // (with time-dependent jump operators every Hnh is formed at its time)
    DiaOps d0 = d;  // the constant Hnh: into hnh, or into hnh0 when H depends on time
    if (timedep) d0.hnh = d.hnh0;
    hnh_dia_kernel<<<dim3((p->n + 255) / 256, B), 256, 0, s>>>(d0, B);
  }
  const dim3 gh((p->n + 255) / 256, B);
  // Hnh (and the jump operators) at the time of the next right-hand side (time-dependent
  // operators only)
  auto at_time = [&](cudaStream_t cs, int which) {
    if (jt.on)
      hnh_td_jump_kernel<<<gh, 256, 0, cs>>>(c, d, td, jt, which);
    else if (timedep)
      hnh_td_kernel<<<gh, 256, 0, cs>>>(c, d, td, which);
  };
  big::load_rho0_kernel<<<ge, T, 0, s>>>(c);
  at_time(s, 8);
  launch_rhs_dia(s, c, d, B, rows, 0, 0, 0, nullptr, nullptr, 0, herm);
  big::init_norm_kernel<<<ge, T, 0, s>>>(c, 0);
  big::init_ctrl_kernel<<<gi, 128, 0, s>>>(c, 0);
  if (krylov) {
    // the probe f(y + h0 k1) - f(y) of the starting step is h0 L k1 for a linear f
    launch_rhs_dia(s, c, d, B, rows, 3, 1, 0, nullptr, nullptr, 0, herm);
    big::init_norm_kernel<<<ge, T, 0, s>>>(c, 2);
  } else {
    big::launch_combine(s, c, ge, 6);
    at_time(s, 9);
    launch_rhs_dia(s, c, d, B, rows, 2, 1, 0, nullptr, nullptr, 0, herm);
    big::init_norm_kernel<<<ge, T, 0, s>>>(c, 1);
  }
  big::init_ctrl_kernel<<<gi, 128, 0, s>>>(c, 1);
  if (cudaGetLastError() != cudaSuccess) return DQB_ERR_CUDA;

  // ---- the RK loop: graph with a WHILE node ------------------------------------------
  auto body = [&](cudaStream_t cs, cudaGraphConditionalHandle h, int* flag) {
    if (krylov) {
      for (int q = 1; q <= 6; ++q) launch_rhs_dia(cs, c, d, B, rows, 0, 0, 1, nullptr, nullptr, q, herm);
      big::launch_kry_combine(cs, c, ge);
      big::control_kernel<<<gi, 128, 0, cs>>>(c);
      big::launch_save(cs, c, ge, 2);
      big::kry_commit_kernel<<<1, 1024, 0, cs>>>(c, h, flag);
      return;
    }
    for (int st = 0; st < 5; ++st) {
      big::launch_combine(cs, c, ge, st);
      at_time(cs, st + 1);
      launch_rhs_dia(cs, c, d, B, rows, 2, st + 1, 1, nullptr, nullptr, 0, herm, herm);
    }
    big::launch_combine(cs, c, ge, 5);
    at_time(cs, 6);
    launch_rhs_dia(cs, c, d, B, rows, 1, 6, 1, nullptr, nullptr, 0, herm, herm);
    big::launch_error(cs, c, ge);
    big::control_kernel<<<gi, 128, 0, cs>>>(c);
    big::launch_save(cs, c, ge, 1);
    big::commit_kernel<<<1, 1024, 0, cs>>>(c, h, flag);
    if (timedep) {  // the first stage of a step that starts on a discontinuity
      at_time(cs, 7);
      launch_rhs_dia(cs, c, d, B, rows, 0, 0, 2, nullptr, nullptr, 0, herm, herm);
    }
  };
  if (host_loop_requested()) {
    if (run_host_loop(body, (int*)(c.iter + 1), s) != cudaSuccess) return DQB_ERR_CUDA;
  } else {
    LaunchKey key;
    std::memset(&key, 0, sizeof(key));
    key.c = c;
    key.d = d;
    key.td = td;
    key.jt = jt;
    key.grid_e = grid_e;
    key.grid_r_x = rows;
    key.grid_r_y = fast_ok(d);
    key.krylov = krylov;
    cudaGraphExec_t exec = g_cache.find(&key, sizeof(key));
    if (!exec) {
      if (build_while_graph(body, &exec) != cudaSuccess) return DQB_ERR_CUDA;
      g_cache.insert(&key, sizeof(key), exec, s);
    } else {
      g_cache.touch(&key, sizeof(key), s);
    }
    if (cudaGraphLaunch(exec, s) != cudaSuccess) return DQB_ERR_CUDA;
  }

  // ---- leftovers and outputs -----------------------------------------------------------
  big::pre_finalize_kernel<<<gi, 128, 0, s>>>(c);
  big::launch_save(s, c, ge, 0);
  big::finalize_kernel<<<ge, T, 0, s>>>(c);
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}

extern "C" int dqb_mesolve_dia(const dqb_dia_problem* p, const dqb_ode_options* o, const dqb_outputs* out,
                               void* workspace, size_t workspace_bytes, void* stream) {
  return solve_dia(p, nullptr, o, out, workspace, workspace_bytes, stream);
}

extern "C" int dqb_mesolve_dia_td(const dqb_dia_problem* p, const dqb_td_hamiltonian* td, const dqb_ode_options* o,
                                  const dqb_outputs* out, void* workspace, size_t workspace_bytes, void* stream) {
  if (!td) return DQB_ERR_INVALID_ARGUMENT;
  return solve_dia(p, td, o, out, workspace, workspace_bytes, stream);
}
