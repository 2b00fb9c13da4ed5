// Dense mesolve for n > 64 (e.g. transmon x cavity, n = 256, 256 instances).
//
// Per right-hand side of every running instance (dynamiqs/integrators/core/
// diffrax_integrator.py:312-323):
//   T_k  = s L_k X                       (batched complex GEMM, s = 1/2 hermitian, 1 standard)
//   tmp  = Hnh X + sum_k T_k L_k^+  [+ X Hnh^+ in the standard form]   (one GEMM, summed terms)
//   k    = tmp + tmp^+ (hermitian form; exact hermitian by construction) or tmp (standard)
// Hnh = -iH - 1/2 sum L^+L is computed once per instance by the same GEMM.  The RK loop is
// the stepper of dqb_big.cuh run as a CUDA-graph WHILE node.
//
// GEMM: 64 x 64 output tile per CTA, K-slices of 16 staged in shared memory (A stored
// k-major so both operands are read as rows), 256 threads x (4 x 4) complex outputs,
// FP32 FMA; each K-slice is read from global memory into registers (coalesced along the
// operand's rows, transposed on the way into shared memory when the operand is a ^+).
// Any n (edges zero-filled).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "dqb_big.cuh"
#include "dqb_graph.cuh"

namespace dqb {
namespace {

enum Src : int { SRC_IN = 0, SRC_HNH = 1, SRC_L = 2, SRC_T = 3, SRC_TMP = 4, SRC_H = 5 };

struct Term {
  int srcA, kA, opA;  // opA: 0 = A, 1 = A^+
  int srcB, kB, opB;
  float alpha;
};

struct LargeOps {
  int n, K;
  const float2* H;  // [*, n, n]
  const float2* L;  // [*, K, n, n]
  const int* Hidx;
  const int* Lidx;
  float2* hnh;  // [B, n, n]
  float2* T;    // [B, K, n, n]
  float2* tmp;  // [B, n, n]
  const dqb_ragged_instance* rag;  // per-instance operators (ragged batches), or null
};

__device__ __forceinline__ int jumps_of(const LargeOps& d, int b) { return d.rag ? d.rag[b].n_jumps : d.K; }

struct GemmJob {
  int nterms;
  Term t[4];
  int dst;       // SRC_T (with kdst), SRC_TMP, SRC_HNH
  int kdst;      // jump index for SRC_T; for GEMMs over all jumps, kdst = -1 (blockIdx.z % K)
  int add_miH;   // epilogue: C += -i H (Hnh set-up)
  int accumulate;  // epilogue: C += result (further terms of a long sum)
  int in_sel;    // 0 = y, 1 = y1, 2 = X
  int need_run;  // 1: running instances, 0: status OK, 2: all (stand-alone)
};

constexpr int BM = 64, BN = 64, BK = 16, NT = 256;

__device__ __forceinline__ const float2* src_ptr(const big::Common& c, const LargeOps& d, int b, int src, int k,
                                                 int in_sel, const float2* ext_in) {
  const long long nn = (long long)d.n * d.n;
  switch (src) {
    case SRC_IN:
      if (ext_in) return ext_in + b * nn;
      {
        const big::Inst& I = c.inst[b];
        return big::slot(c, b, in_sel == 0 ? I.sy : (in_sel == 1 ? I.sy1 : big::kX));
      }
    case SRC_HNH: return d.hnh + b * nn;
    case SRC_L: {
      if (d.rag) return (const float2*)d.rag[b].L + k * nn;
      const long long li = d.Lidx ? d.Lidx[b] : b;
      return d.L + (li * d.K + k) * nn;
    }
    case SRC_T: return d.T + ((long long)b * d.K + k) * nn;
    case SRC_TMP: return d.tmp + b * nn;
    default: {
      if (d.rag) return (const float2*)d.rag[b].H;
      const long long hi = d.Hidx ? d.Hidx[b] : b;
      return d.H + hi * nn;
    }
  }
}

// Load a BK x BM slice of op(M) (rows r0.., k-columns k0..) into S[k][m] (k-major).
// op 0: op(M)[r][k] = M[r][k];  op 1: op(M)[r][k] = conj(M[k][r]).
__device__ __forceinline__ void load_slice(float2 (&reg)[4], const float2* __restrict__ M, int n, int r0, int k0,
                                           int op) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int e = tid + q * NT;  // 0..1023 over (BM x BK)
    int r, k;
    if (op == 0) {  // consecutive threads walk k (contiguous in M's rows)
      r = e / BK;
      k = e % BK;
    } else {        // consecutive threads walk r (contiguous in M's rows k)
      k = e / BM;
      r = e % BM;
    }
    const int gr = r0 + r, gk = k0 + k;
    float2 v = make_float2(0.f, 0.f);
    if (gr < n && gk < n) {
      v = op == 0 ? M[(long long)gr * n + gk] : cconj(M[(long long)gk * n + gr]);
    }
    reg[q] = v;
  }
}

__device__ __forceinline__ void store_slice(float2* S, const float2 (&reg)[4], int op) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int e = tid + q * NT;
    int r, k;
    if (op == 0) {
      r = e / BK;
      k = e % BK;
    } else {
      k = e / BM;
      r = e % BM;
    }
    S[k * (BM + 1) + r] = reg[q];
  }
}

// grid (tiles_n * tiles_n, 1, B * Kz): one 64 x 64 tile of C = sum_terms alpha op(A) op(B).
__global__ void __launch_bounds__(NT) cgemm_kernel(big::Common c, LargeOps d, GemmJob job, const float2* ext_in,
                                                   float2* ext_out) {
  __shared__ float2 As[BK * (BM + 1)];
  __shared__ float2 Bs[BK * (BN + 1)];
  const int n = d.n;
  const int Kz = job.kdst < 0 ? d.K : 1;
  const int b = blockIdx.z / Kz;
  const int kz = job.kdst < 0 ? (int)(blockIdx.z % Kz) : job.kdst;
  if (job.need_run != 2) {
    const big::Inst& I = c.inst[b];
    if (job.need_run == 1 ? !I.run : I.status != DQB_INST_OK) return;
  }
  const int Kb = jumps_of(d, b);
  if (job.kdst < 0 && kz >= Kb) return;  // this instance has fewer jumps
  const int tiles = (n + BM - 1) / BM;
  const int tr = blockIdx.x / tiles, tc = blockIdx.x % tiles;
  const int r0 = tr * BM, c0 = tc * BN;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_float2(0.f, 0.f);

  for (int t = 0; t < job.nterms; ++t) {
    const Term T = job.t[t];
    if ((T.srcA == SRC_T || T.srcA == SRC_L) && T.kA >= Kb) continue;  // missing jump
    const float2* A = src_ptr(c, d, b, T.srcA, T.kA < 0 ? kz : T.kA, job.in_sel, ext_in);
    const float2* B = src_ptr(c, d, b, T.srcB, T.kB < 0 ? kz : T.kB, job.in_sel, ext_in);
    float2 ra[4], rb[4];
    float2 tsum[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) tsum[i][j] = make_float2(0.f, 0.f);
    for (int k0 = 0; k0 < n; k0 += BK) {
      load_slice(ra, A, n, r0, k0, T.opA);
      // op(B)[k][col]: op 0 -> B[k][col]; op 1 -> conj(B[col][k]).  Load into Bs[k][col].
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int e = threadIdx.x + q * NT;
        int col, k;
        if (T.opB == 0) {
          k = e / BN;
          col = e % BN;
        } else {
          col = e / BK;
          k = e % BK;
        }
        const int gc = c0 + col, gk = k0 + k;
        float2 v = make_float2(0.f, 0.f);
        if (gc < n && gk < n) v = T.opB == 0 ? B[(long long)gk * n + gc] : cconj(B[(long long)gc * n + gk]);
        rb[q] = v;
      }
      __syncthreads();
      store_slice(As, ra, T.opA);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int e = threadIdx.x + q * NT;
        int col, k;
        if (T.opB == 0) {
          k = e / BN;
          col = e % BN;
        } else {
          col = e / BK;
          k = e % BK;
        }
        Bs[k * (BN + 1) + col] = rb[q];
      }
      __syncthreads();
#pragma unroll
      for (int k = 0; k < BK; ++k) {
        float2 a[4], bb[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[k * (BM + 1) + ty + 16 * i];
#pragma unroll
        for (int j = 0; j < 4; ++j) bb[j] = Bs[k * (BN + 1) + tx + 16 * j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) cmac(tsum[i][j], a[i], bb[j]);
      }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        acc[i][j].x = fmaf(T.alpha, tsum[i][j].x, acc[i][j].x);
        acc[i][j].y = fmaf(T.alpha, tsum[i][j].y, acc[i][j].y);
      }
  }
  // epilogue
  float2* C;
  if (ext_out) {
    C = ext_out + (long long)b * n * n;
  } else if (job.dst == SRC_T) {
    C = d.T + ((long long)b * d.K + kz) * (long long)n * n;
  } else if (job.dst == SRC_TMP) {
    C = d.tmp + (long long)b * n * n;
  } else {
    C = d.hnh + (long long)b * n * n;
  }
  const float2* Hm = job.add_miH ? src_ptr(c, d, b, SRC_H, 0, 0, nullptr) : nullptr;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int gr = r0 + ty + 16 * i;
    if (gr >= n) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gc = c0 + tx + 16 * j;
      if (gc >= n) continue;
      float2 v = acc[i][j];
      if (job.accumulate) v = cadd(v, C[(long long)gr * n + gc]);
      if (Hm) {
        const float2 h = Hm[(long long)gr * n + gc];
        v.x += h.y;  // -i h
        v.y -= h.x;
      }
      C[(long long)gr * n + gc] = v;
    }
  }
}

// k_out = tmp + tmp^+ (hermitian form) via 32 x 32 shared-memory tile pairs, or a copy.
// grid (tiles32 * tiles32, B).
__global__ void __launch_bounds__(256) symmetrize_kernel(big::Common c, LargeOps d, int out_k, int need_run,
                                                         int herm, float2* ext_out) {
  __shared__ float2 tT[32][33];
  const int b = blockIdx.y;
  float2* out;
  if (ext_out) {
    out = ext_out + (long long)b * d.n * d.n;
  } else {
    const big::Inst& I = c.inst[b];
    if (need_run ? !I.run : I.status != DQB_INST_OK) return;
    out = big::slot(c, b, I.sk[out_k]);
  }
  const int n = d.n;
  const float2* tmp = d.tmp + (long long)b * n * n;
  const int tiles = (n + 31) / 32;
  const int ti = blockIdx.x / tiles, tj = blockIdx.x % tiles;
  const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;  // 32 x 8
  if (herm) {
    // stage tile (tj, ti) transposed
    for (int r = ly; r < 32; r += 8) {
      const int gr = tj * 32 + r, gc = ti * 32 + lx;
      tT[lx][r] = (gr < n && gc < n) ? tmp[(long long)gr * n + gc] : make_float2(0.f, 0.f);
    }
    __syncthreads();
  }
  for (int r = ly; r < 32; r += 8) {
    const int gr = ti * 32 + r, gc = tj * 32 + lx;
    if (gr >= n || gc >= n) continue;
    float2 v = tmp[(long long)gr * n + gc];
    if (herm) v = cadd(v, cconj(tT[r][lx]));
    out[(long long)gr * n + gc] = v;
  }
}

size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

struct LargeLayout {
  size_t off_iter, off_inst, off_eacc, off_hnh, off_T, off_tmp, off_mats, total;
};

LargeLayout large_layout(int n, int K, int nE, int ntsave, long long B) {
  LargeLayout l;
  const size_t nn = (size_t)n * n;
  l.off_iter = 0;
  l.off_inst = 256;
  l.off_eacc = align_up(l.off_inst + B * sizeof(big::Inst));
  l.off_hnh = align_up(l.off_eacc + B * (size_t)nE * ntsave * sizeof(double2));
  l.off_T = align_up(l.off_hnh + B * nn * sizeof(float2));
  l.off_tmp = align_up(l.off_T + B * (size_t)K * nn * sizeof(float2));
  l.off_mats = align_up(l.off_tmp + B * nn * sizeof(float2));
  l.total = l.off_mats + B * (size_t)big::kSlots * nn * sizeof(float2);
  return l;
}

// The three launches of one right-hand side (T_k, tmp, symmetrize).
void launch_rhs(cudaStream_t s, const big::Common& c, const LargeOps& d, int B, int in_sel, int out_k,
                int need_run, int form, const float2* ext_in, float2* ext_out) {
  const int n = d.n;
  const int tiles = (n + BM - 1) / BM;
  const float sc = form == DQB_FORM_HERMITIAN ? 0.5f : 1.0f;
  if (d.K > 0) {
    GemmJob j1;
    std::memset(&j1, 0, sizeof(j1));
    j1.nterms = 1;
    j1.t[0] = Term{SRC_L, -1, 0, SRC_IN, 0, 0, sc};
    j1.dst = SRC_T;
    j1.kdst = -1;
    j1.in_sel = in_sel;
    j1.need_run = need_run;
    cgemm_kernel<<<dim3(tiles * tiles, 1, B * d.K), NT, 0, s>>>(c, d, j1, ext_in, nullptr);
  }
  // tmp = Hnh X + sum_k T_k L_k^+ [+ X Hnh^+]: at most 4 summed terms per launch, the
  // rest accumulated by further launches into tmp
  GemmJob j2;
  std::memset(&j2, 0, sizeof(j2));
  j2.dst = SRC_TMP;
  j2.kdst = 0;
  j2.in_sel = in_sel;
  j2.need_run = need_run;
  int nt = 0;
  j2.t[nt++] = Term{SRC_HNH, 0, 0, SRC_IN, 0, 0, 1.0f};
  if (form == DQB_FORM_STANDARD) j2.t[nt++] = Term{SRC_IN, 0, 0, SRC_HNH, 0, 1, 1.0f};
  int k = 0;
  for (;;) {
    while (k < d.K && nt < 4) j2.t[nt++] = Term{SRC_T, k, 0, SRC_L, k, 1, 1.0f}, ++k;
    j2.nterms = nt;
    cgemm_kernel<<<dim3(tiles * tiles, 1, B), NT, 0, s>>>(c, d, j2, ext_in, nullptr);
    if (k >= d.K) break;
    j2.accumulate = 1;
    nt = 0;
  }
  const int t32 = (n + 31) / 32;
  symmetrize_kernel<<<dim3(t32 * t32, B), 256, 0, s>>>(c, d, out_k, need_run, form == DQB_FORM_HERMITIAN,
                                                       ext_out);
}

int check_dense_large(const dqb_dense_problem* p) {
  if (!p) return DQB_ERR_INVALID_ARGUMENT;
  if (p->n < 2 || p->n_jumps < 0 || p->batch < 0) return DQB_ERR_INVALID_ARGUMENT;
  if (p->batch > 65535 / std::max(1, p->n_jumps)) return DQB_ERR_UNSUPPORTED;
  if (!p->H || (p->n_jumps > 0 && !p->L)) return DQB_ERR_INVALID_ARGUMENT;
  if (p->n_jumps > 16) return DQB_ERR_UNSUPPORTED;
  return DQB_OK;
}

GraphCache g_cache;

struct LaunchKey {
  big::Common c;
  LargeOps d;
  int form;
};

LargeOps make_ops(const dqb_dense_problem* p, char* ws, const LargeLayout& lay) {
  LargeOps d;
  std::memset(&d, 0, sizeof(d));
  d.n = p->n;
  d.K = p->n_jumps;
  d.H = (const float2*)p->H;
  d.L = (const float2*)p->L;
  d.Hidx = p->H_index;
  d.Lidx = p->L_index;
  d.hnh = (float2*)(ws + lay.off_hnh);
  d.T = (float2*)(ws + lay.off_T);
  d.tmp = (float2*)(ws + lay.off_tmp);
  return d;
}

void launch_hnh(cudaStream_t s, const big::Common& c, const LargeOps& d, int B, int need_run) {
  const int tiles = (d.n + BM - 1) / BM;
  GemmJob j;
  std::memset(&j, 0, sizeof(j));
  j.dst = SRC_HNH;
  j.kdst = 0;
  j.add_miH = 1;
  j.need_run = need_run;
  int k = 0;
  do {  // Hnh = -iH - 1/2 sum_k L_k^+ L_k, four jumps per launch
    int nt = 0;
    while (k < d.K && nt < 4) j.t[nt++] = Term{SRC_L, k, 1, SRC_L, k, 0, -0.5f}, ++k;
    j.nterms = nt;
    cgemm_kernel<<<dim3(tiles * tiles, 1, B), NT, 0, s>>>(c, d, j, nullptr, nullptr);
    j.add_miH = 0;
    j.accumulate = 1;
  } while (k < d.K);
}

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
    prefer_max_shared(cgemm_kernel);
    prefer_max_shared(symmetrize_kernel);
  });
}

static int run_large(const big::Common& c, const LargeOps& d, cudaStream_t s) {
  init_carveouts();
  const int B = c.B;
  int grid_e = (int)std::min<long long>((c.nn + big::kElemThreads - 1) / big::kElemThreads, 1184);
  if (grid_e < 1) grid_e = 1;
  const dim3 ge(grid_e, B);
  const dim3 gi((B + 127) / 128);
  const int T = big::kElemThreads;
  const int form = c.form;

  big::setup_kernel<<<gi, 128, 0, s>>>(c);
  big::load_rho0_kernel<<<ge, T, 0, s>>>(c);
  launch_hnh(s, c, d, B, 0);
  launch_rhs(s, c, d, B, 0, 0, 0, form, nullptr, nullptr);
  big::init_norm_kernel<<<ge, T, 0, s>>>(c, 0);
  big::init_ctrl_kernel<<<gi, 128, 0, s>>>(c, 0);
  big::combine_kernel<<<ge, T, 0, s>>>(c, 6);
  launch_rhs(s, c, d, B, 2, 1, 0, form, nullptr, nullptr);
  big::init_norm_kernel<<<ge, T, 0, s>>>(c, 1);
  big::init_ctrl_kernel<<<gi, 128, 0, s>>>(c, 1);
  if (cudaGetLastError() != cudaSuccess) return DQB_ERR_CUDA;

  LaunchKey key;
  std::memset(&key, 0, sizeof(key));
  key.c = c;
  key.d = d;
  key.form = form;
  cudaGraphExec_t exec = g_cache.find(&key, sizeof(key));
  if (!exec) {
    auto body = [&](cudaStream_t cs, cudaGraphConditionalHandle h) {
      for (int st = 0; st < 5; ++st) {
        big::combine_kernel<<<ge, T, 0, cs>>>(c, st);
        launch_rhs(cs, c, d, B, 2, st + 1, 1, form, nullptr, nullptr);
      }
      big::combine_kernel<<<ge, T, 0, cs>>>(c, 5);
      launch_rhs(cs, c, d, B, 1, 6, 1, form, nullptr, nullptr);
      big::error_kernel<<<ge, T, 0, cs>>>(c);
      big::control_kernel<<<gi, 128, 0, cs>>>(c);
      big::save_kernel<<<ge, T, 0, cs>>>(c, 1);
      big::commit_kernel<<<1, 1024, 0, cs>>>(c, h);
    };
    if (build_while_graph(body, &exec) != cudaSuccess) return DQB_ERR_CUDA;
    g_cache.insert(&key, sizeof(key), exec, s);
  } else {
    g_cache.touch(&key, sizeof(key), s);
  }
  if (cudaGraphLaunch(exec, s) != cudaSuccess) return DQB_ERR_CUDA;
  big::pre_finalize_kernel<<<gi, 128, 0, s>>>(c);
  big::save_kernel<<<ge, T, 0, s>>>(c, 0);
  big::finalize_kernel<<<ge, T, 0, s>>>(c);
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}



extern "C" size_t dqb_mesolve_dense_large_workspace_size(int32_t n, int32_t n_jumps, int32_t n_exp,
                                                         int32_t n_tsave, int64_t batch) {
  if (n < 2 || n_jumps < 0 || n_exp < 0 || n_tsave < 1 || batch <= 0) return 0;
  return large_layout(n, n_jumps, n_exp, n_tsave, batch).total;
}

extern "C" int dqb_lindblad_rhs_dense_large(const dqb_dense_problem* p, int32_t form, const void* rho, void* outp,
                                            void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_dense_large(p);
  if (rc) return rc;
  if (!rho || !outp) return DQB_ERR_INVALID_ARGUMENT;
  if (form != DQB_FORM_HERMITIAN && form != DQB_FORM_STANDARD) return DQB_ERR_INVALID_ARGUMENT;
  if (p->batch == 0) return DQB_OK;
  const LargeLayout lay = large_layout(p->n, p->n_jumps, 0, 1, p->batch);
  if (!workspace || workspace_bytes < lay.off_mats) return DQB_ERR_WORKSPACE_TOO_SMALL;
  LargeOps d = make_ops(p, (char*)workspace, lay);
  big::Common c;
  std::memset(&c, 0, sizeof(c));
  cudaStream_t s = (cudaStream_t)stream;
  init_carveouts();
  launch_hnh(s, c, d, (int)p->batch, 2);
  launch_rhs(s, c, d, (int)p->batch, 2, 0, 2, form, (const float2*)rho, (float2*)outp);
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}

extern "C" size_t dqb_mesolve_dense_large_ragged_workspace_size(int32_t n, int32_t max_jumps, int32_t max_exp,
                                                                int32_t max_tsave, int64_t count) {
  return dqb_mesolve_dense_large_workspace_size(n, max_jumps, max_exp, max_tsave, count);
}

extern "C" int dqb_mesolve_dense_large_ragged(const dqb_ragged_instance* instances, int64_t count,
                                              const int32_t* count_device, int32_t n, int32_t max_jumps,
                                              int32_t max_exp, int32_t max_tsave, const dqb_ode_options* o,
                                              void* workspace, size_t workspace_bytes, void* stream) {
  if (!o || count < 0 || n < 2 || max_jumps < 0 || max_jumps > 16 || max_exp < 0 || max_tsave < 1)
    return DQB_ERR_INVALID_ARGUMENT;
  if (count > 65535 / std::max(1, (int)max_jumps)) return DQB_ERR_UNSUPPORTED;
  if (o->method != DQB_METHOD_TSIT5 && o->method != DQB_METHOD_DOPRI5) return DQB_ERR_INVALID_ARGUMENT;
  if (o->form != DQB_FORM_HERMITIAN && o->form != DQB_FORM_STANDARD) return DQB_ERR_INVALID_ARGUMENT;
  if (!(o->rtol >= 0) || !(o->atol >= 0) || o->max_steps < 0) return DQB_ERR_INVALID_ARGUMENT;
  if (count == 0) return DQB_OK;
  if (!instances) return DQB_ERR_INVALID_ARGUMENT;
  const LargeLayout lay = large_layout(n, max_jumps, max_exp, max_tsave, count);
  if (!workspace || workspace_bytes < lay.total) return DQB_ERR_WORKSPACE_TOO_SMALL;
  char* ws = (char*)workspace;
  dqb_dense_problem p;
  std::memset(&p, 0, sizeof(p));
  p.n = n;
  p.n_jumps = max_jumps;
  p.batch = count;
  LargeOps d = make_ops(&p, ws, lay);
  d.rag = instances;
  big::Common c;
  std::memset(&c, 0, sizeof(c));
  c.n = n;
  c.nn = (long long)n * n;
  c.B = (int)count;
  c.form = o->form;
  c.o = make_ctrl(*o);
  c.inst = (big::Inst*)(ws + lay.off_inst);
  c.mats = (float2*)(ws + lay.off_mats);
  c.eacc = (double2*)(ws + lay.off_eacc);
  c.eacc_stride = (long long)max_exp * max_tsave;
  c.iter = (long long*)(ws + lay.off_iter);
  c.rag = instances;
  c.count_dev = count_device;
  return run_large(c, d, (cudaStream_t)stream);
}

extern "C" int dqb_mesolve_dense_large(const dqb_dense_problem* p, const dqb_ode_options* o, const dqb_outputs* out,
                                       void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_dense_large(p);
  if (rc) return rc;
  if (!o || !out || !out->states || !out->infos || !out->status || (p->n_exp > 0 && !out->expects))
    return DQB_ERR_INVALID_ARGUMENT;
  if (p->n_exp < 0 || p->n_tsave < 1 || !p->rho0 || !p->tsave || (p->n_exp > 0 && !p->E))
    return DQB_ERR_INVALID_ARGUMENT;
  if (o->method != DQB_METHOD_TSIT5 && o->method != DQB_METHOD_DOPRI5) return DQB_ERR_INVALID_ARGUMENT;
  if (o->form != DQB_FORM_HERMITIAN && o->form != DQB_FORM_STANDARD) return DQB_ERR_INVALID_ARGUMENT;
  if (!(o->rtol >= 0) || !(o->atol >= 0) || o->max_steps < 0) return DQB_ERR_INVALID_ARGUMENT;
  if (p->batch == 0) return DQB_OK;
  const LargeLayout lay = large_layout(p->n, p->n_jumps, p->n_exp, p->n_tsave, p->batch);
  if (!workspace || workspace_bytes < lay.total) return DQB_ERR_WORKSPACE_TOO_SMALL;
  char* ws = (char*)workspace;
  LargeOps d = make_ops(p, ws, lay);

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

  return run_large(c, d, (cudaStream_t)stream);
}
