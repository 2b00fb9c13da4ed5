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

constexpr int kRhsCols = 128;
constexpr int kRhsRows = 8;

// Generic f(X) for DIA operators (any number of diagonals).  grid (n / 128, n / 8, B),
// block 128: each thread owns one column and 8 consecutive rows.
// in_sel: 0 = y, 1 = y1, 2 = X.  need_run: 1 = running instances, 0 = status OK.
__global__ void __launch_bounds__(kRhsCols) rhs_dia_generic_kernel(big::Common c, DiaOps d, int in_sel, int out_k,
                                                                   int need_run, const float2* ext_in,
                                                                   float2* ext_out) {
  const int b = blockIdx.z;
  const float2* X;
  float2* out;
  const float2* L;
  if (ext_in) {  // stand-alone evaluation (dqb_lindblad_rhs_dia)
    X = ext_in + (long long)b * d.n * d.n;
    out = ext_out + (long long)b * d.n * d.n;
  } else {
    const big::Inst& I = c.inst[b];
    if (need_run ? !I.run : I.status != DQB_INST_OK) return;
    X = big::slot(c, b, in_sel == 0 ? I.sy : (in_sel == 1 ? I.sy1 : big::kX));
    out = big::slot(c, b, I.sk[out_k]);
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
    out[(long long)i * n + j] = acc;
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
                                                                int need_run, const float2* ext_in,
                                                                float2* ext_out) {
  extern __shared__ DiaCoef dia_tab[];
  const int b = blockIdx.z;
  const float2* X;
  float2* out;
  if (ext_in) {  // stand-alone evaluation (dqb_lindblad_rhs_dia)
    X = ext_in + (long long)b * d.n * d.n;
    out = ext_out + (long long)b * d.n * d.n;
  } else {
    const big::Inst& I = c.inst[b];
    if (need_run ? !I.run : I.status != DQB_INST_OK) return;
    X = big::slot(c, b, in_sel == 0 ? I.sy : (in_sel == 1 ? I.sy1 : big::kX));
    out = big::slot(c, b, I.sk[out_k]);
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
    out[(long long)i * n + j] = acc;
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
                                                                 int out_k, int need_run, const float2* ext_in,
                                                                 float2* ext_out) {
  extern __shared__ float4 dia_stage_raw[];
  const int b = blockIdx.z;
  const float2* X;
  float2* out;
  if (ext_in) {  // stand-alone evaluation (dqb_lindblad_rhs_dia)
    X = ext_in + (long long)b * d.n * d.n;
    out = ext_out + (long long)b * d.n * d.n;
  } else {
    const big::Inst& I = c.inst[b];
    if (need_run ? !I.run : I.status != DQB_INST_OK) return;
    X = big::slot(c, b, in_sel == 0 ? I.sy : (in_sel == 1 ? I.sy1 : big::kX));
    out = big::slot(c, b, I.sk[out_k]);
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
    out[(long long)(i0 + r) * n + j] = acc;
  }
}

// ------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------

size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

struct DiaLayout {
  size_t off_iter, off_inst, off_eacc, off_hnh, off_mats, total;
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
  l.off_mats = align_up(l.off_hnh + B * (size_t)nh * n * sizeof(float2));
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

// Launch shape of the stencil from `tile`: 4, 8 or 16 = the tiled kernel with that many rows
// per thread (when the operators have at most kTiledMaxTerms diagonal terms); 108 or 116 =
// the staged kernel with 8 or 16 rows per CTA (when its plan fits); anything else (0 =
// default, 1) = the generic kernel.  The autotuner picks among them per problem shape.
// Returns the shape code (1 = generic).
int rows_for(const DiaOps& d, int tile) {
  if (tile == 108 || tile == 116) {
    DiaStage st;
    size_t sm;
    if (plan_stage(d, tile - 100, &st, &sm)) return tile;
  }
  if (!fast_ok(d)) return 1;
  return (tile == 4 || tile == 8 || tile == 16) ? tile : 1;
}

dim3 rhs_grid(const DiaOps& d, int rows, int B) {
  const int r = rows == 1 ? kRhsRows : (rows > 100 ? rows - 100 : rows);
  return dim3((d.n + kRhsCols - 1) / kRhsCols, (d.n + r - 1) / r, B);
}

// One right-hand side of every instance: k[out_k] = f(input), through the kernel the shape
// code `rows` selects (rows_for).
void launch_rhs_dia(cudaStream_t s, const big::Common& c, const DiaOps& d, int B, int rows, int in_sel,
                    int out_k, int need_run, const float2* ext_in, float2* ext_out) {
  const dim3 g = rhs_grid(d, rows, B);
  if (rows > 100) {
    DiaStage st;
    size_t sm = 0;
    plan_stage(d, rows - 100, &st, &sm);  // rows_for checked that it fits
    if (rows == 116)
      rhs_dia_staged_kernel<16><<<g, kRhsCols, sm, s>>>(c, d, st, in_sel, out_k, need_run, ext_in, ext_out);
    else
      rhs_dia_staged_kernel<8><<<g, kRhsCols, sm, s>>>(c, d, st, in_sel, out_k, need_run, ext_in, ext_out);
    return;
  }
  const size_t sm = tiled_smem(d, rows);
  if (rows == 4) {
    rhs_dia_tiled_kernel<4><<<g, kRhsCols, sm, s>>>(c, d, in_sel, out_k, need_run, ext_in, ext_out);
  } else if (rows == 8) {
    rhs_dia_tiled_kernel<8><<<g, kRhsCols, sm, s>>>(c, d, in_sel, out_k, need_run, ext_in, ext_out);
  } else if (rows == 16) {
    rhs_dia_tiled_kernel<16><<<g, kRhsCols, sm, s>>>(c, d, in_sel, out_k, need_run, ext_in, ext_out);
  } else {
    rhs_dia_generic_kernel<<<g, kRhsCols, 0, s>>>(c, d, in_sel, out_k, need_run, ext_in, ext_out);
  }
}

GraphCache g_cache;

struct LaunchKey {
  big::Common c;
  DiaOps d;
  int grid_e, grid_r_x, grid_r_y;
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
    prefer_max_shared(big::commit_kernel);
    prefer_max_shared(big::pre_finalize_kernel);
    prefer_max_shared(big::finalize_kernel);
    prefer_max_shared(zero_words_kernel);
    prefer_max_shared(hnh_dia_kernel);
    prefer_max_shared(rhs_dia_generic_kernel);
    prefer_max_shared(rhs_dia_tiled_kernel<4>);
    prefer_max_shared(rhs_dia_tiled_kernel<8>);
    prefer_max_shared(rhs_dia_tiled_kernel<16>);
    prefer_max_shared(rhs_dia_staged_kernel<8>);
    prefer_max_shared(rhs_dia_staged_kernel<16>);
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
  if (form != DQB_FORM_HERMITIAN && form != DQB_FORM_STANDARD) return DQB_ERR_INVALID_ARGUMENT;
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
  launch_rhs_dia(s, c, d, (int)p->batch, rows_for(d, tile), 2, 0, 0, (const float2*)rho, (float2*)outp);
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}

extern "C" int dqb_mesolve_dia(const dqb_dia_problem* p, const dqb_ode_options* o, const dqb_outputs* out,
                               void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_problem(p);
  if (rc) return rc;
  if (!o || !out || !out->states || !out->infos || !out->status || (p->n_exp > 0 && !out->expects))
    return DQB_ERR_INVALID_ARGUMENT;
  if (o->method != DQB_METHOD_TSIT5 && o->method != DQB_METHOD_DOPRI5) return DQB_ERR_INVALID_ARGUMENT;
  if (o->form != DQB_FORM_HERMITIAN && o->form != DQB_FORM_STANDARD) return DQB_ERR_INVALID_ARGUMENT;
  if (!(o->rtol >= 0) || !(o->atol >= 0) || o->max_steps < 0) return DQB_ERR_INVALID_ARGUMENT;
  if (p->batch == 0) return DQB_OK;
  DiaOps d;
  rc = build_ops(p, &d);
  if (rc) return rc;
  const DiaLayout lay = layout_for(p, d.nh);
  if (!workspace || workspace_bytes < lay.total) return DQB_ERR_WORKSPACE_TOO_SMALL;
  char* ws = (char*)workspace;
  d.hnh = (float2*)(ws + lay.off_hnh);

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

  cudaStream_t s = (cudaStream_t)stream;
  const int B = c.B;
  const long long nn = c.nn;
  int grid_e = (int)std::min<long long>((nn + big::kElemThreads - 1) / big::kElemThreads, 1184);
  if (grid_e < 1) grid_e = 1;
  const dim3 ge(grid_e, B);
  const int rows = rows_for(d, o->tile);
  const dim3 gi((B + 127) / 128);
  const int T = big::kElemThreads;

  // ---- set-up and starting step (outside the graph) ----------------------------------
  init_carveouts();
  big::setup_kernel<<<gi, 128, 0, s>>>(c);
  hnh_dia_kernel<<<dim3((p->n + 255) / 256, B), 256, 0, s>>>(d, B);
  big::load_rho0_kernel<<<ge, T, 0, s>>>(c);
  launch_rhs_dia(s, c, d, B, rows, 0, 0, 0, nullptr, nullptr);
  big::init_norm_kernel<<<ge, T, 0, s>>>(c, 0);
  big::init_ctrl_kernel<<<gi, 128, 0, s>>>(c, 0);
  big::combine_kernel<<<ge, T, 0, s>>>(c, 6);
  launch_rhs_dia(s, c, d, B, rows, 2, 1, 0, nullptr, nullptr);
  big::init_norm_kernel<<<ge, T, 0, s>>>(c, 1);
  big::init_ctrl_kernel<<<gi, 128, 0, s>>>(c, 1);
  if (cudaGetLastError() != cudaSuccess) return DQB_ERR_CUDA;

  // ---- the RK loop: graph with a WHILE node ------------------------------------------
  auto body = [&](cudaStream_t cs, cudaGraphConditionalHandle h, int* flag) {
    for (int st = 0; st < 5; ++st) {
      big::combine_kernel<<<ge, T, 0, cs>>>(c, st);
      launch_rhs_dia(cs, c, d, B, rows, 2, st + 1, 1, nullptr, nullptr);
    }
    big::combine_kernel<<<ge, T, 0, cs>>>(c, 5);
    launch_rhs_dia(cs, c, d, B, rows, 1, 6, 1, nullptr, nullptr);
    big::error_kernel<<<ge, T, 0, cs>>>(c);
    big::control_kernel<<<gi, 128, 0, cs>>>(c);
    big::save_kernel<<<ge, T, 0, cs>>>(c, 1);
    big::commit_kernel<<<1, 1024, 0, cs>>>(c, h, flag);
  };
  if (host_loop_requested()) {
    if (run_host_loop(body, (int*)(c.iter + 1), s) != cudaSuccess) return DQB_ERR_CUDA;
  } else {
    LaunchKey key;
    std::memset(&key, 0, sizeof(key));
    key.c = c;
    key.d = d;
    key.grid_e = grid_e;
    key.grid_r_x = rows;
    key.grid_r_y = fast_ok(d);
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
  big::save_kernel<<<ge, T, 0, s>>>(c, 0);
  big::finalize_kernel<<<ge, T, 0, s>>>(c);
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}
