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
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "dqb_big.cuh"
#include "dqb_graph.cuh"
#include "dqb_tc.cuh"

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
  int prec;                        // DQB_PREC_*: FP32 CUDA cores or a tensor-core mode
};

__device__ __forceinline__ int jumps_of(const LargeOps& d, int b) { return d.rag ? d.rag[b].n_jumps : d.K; }

struct GemmJob {
  int nterms;
  Term t[4];
  int dst;       // SRC_T (with kdst), SRC_TMP, SRC_HNH
  int kdst;      // jump index for SRC_T; for GEMMs over all jumps, kdst = -1 (blockIdx.z % K)
  int add_miH;   // epilogue: C += -i H (Hnh set-up)
  int accumulate;  // epilogue: C += result (further terms of a long sum)
  int in_sel;    // 0 = y, 1 = y1, 2 = X, 2 + q = k_q (the Krylov form's u_q)
  int need_run;  // 1: running instances, 0: status OK, 2: all (stand-alone), 3: refresh
  int kry;       // q > 0: Krylov basis right-hand side u_{q+1} = tau L u_q (skipped where the
                 // instance's basis already has it)
};

// Whether instance b takes no part in a job (need_run and the Krylov basis state).
__device__ __forceinline__ bool job_skips(const big::Common& c, int b, int need_run, int kry) {
  if (need_run == 2) return false;
  const big::Inst& I = c.inst[b];
  if (need_run == 3) return !(I.run && I.refresh);  // the first stage after a discontinuity
  if (need_run == 1 ? !I.run : I.status != DQB_INST_OK) return true;
  return kry > 0 && I.kvalid >= kry + 2;
}

constexpr int BM = 64, BN = 64, BK = 16, NT = 256;

__device__ __forceinline__ const float2* src_ptr(const big::Common& c, const LargeOps& d, int b, int src, int k,
                                                 int in_sel, const float2* ext_in) {
  const long long nn = (long long)d.n * d.n;
  switch (src) {
    case SRC_IN:
      if (ext_in) return ext_in + b * nn;
      {
        const big::Inst& I = c.inst[b];
        return big::slot(c, b, in_sel == 0 ? I.sy : (in_sel == 1 ? I.sy1 : (in_sel == 2 ? big::kX : I.sk[in_sel - 3])));
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
  if (job_skips(c, b, job.need_run, job.kry)) return;
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

// k_out = tmp + tmp^+ (hermitian form) via 32 x 32 shared-memory tile pairs, or a copy;
// for a Krylov basis right-hand side (kry = q > 0) times tau (and sig1 for q = 1).
// grid (tiles32 * tiles32, B).
__global__ void __launch_bounds__(256) symmetrize_kernel(big::Common c, LargeOps d, int out_k, int need_run,
                                                         int herm, int kry, float2* ext_out) {
  __shared__ float2 tT[32][33];
  const int b = blockIdx.y;
  float2* out;
  float scale = 1.f;
  if (ext_out) {
    out = ext_out + (long long)b * d.n * d.n;
  } else {
    if (job_skips(c, b, need_run, kry)) return;
    const big::Inst& I = c.inst[b];
    out = big::slot(c, b, I.sk[out_k]);
    if (kry > 0) scale = (float)(kry == 1 ? I.tau * I.sig1 : I.tau);
  }
  const int n = d.n;
  const float2* tmp = d.tmp + (long long)b * n * n;
  const int tiles = (n + 31) / 32;
  const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;  // 32 x 8
  if (herm) {
    // one tile pair per block (grid over the upper tiles): k(ti, tj) = tmp(ti, tj) +
    // tmp(tj, ti)^+ written directly, k(tj, ti) its conjugate transpose (mirrored), so
    // every element of tmp is read once
    int ti, tj;
    big::herm_tile(blockIdx.x, tiles, ti, tj);
    for (int r = ly; r < 32; r += 8) {
      const int gr = tj * 32 + r, gc = ti * 32 + lx;
      tT[lx][r] = (gr < n && gc < n) ? tmp[(long long)gr * n + gc] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2 v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int r = ly + 8 * q, gr = ti * 32 + r, gc = tj * 32 + lx;
      float2 x = make_float2(0.f, 0.f);
      if (gr < n && gc < n) x = cadd(tmp[(long long)gr * n + gc], cconj(tT[r][lx]));
      v[q] = make_float2(x.x * scale, x.y * scale);
    }
    big::herm_store<false>(out, n, ti, tj, v, tT);
    return;
  }
  const int ti = blockIdx.x / tiles, tj = blockIdx.x % tiles;
  for (int r = ly; r < 32; r += 8) {
    const int gr = ti * 32 + r, gc = tj * 32 + lx;
    if (gr >= n || gc >= n) continue;
    float2 v = tmp[(long long)gr * n + gc];
    out[(long long)gr * n + gc] = make_float2(v.x * scale, v.y * scale);
  }
}

// ------------------------------------------------------------------------------------
// Tensor-core GEMM (tcgen05): C = alpha sum_t A_t M_t^+ for complex n x n matrices.
// ------------------------------------------------------------------------------------
// Real form.  With complex64 stored interleaved, row i of A is the real row
// A'[i] = (Re A[i][0], Im A[i][0], Re A[i][1], ...) of length 2n, and C = A M^+ is the real
// product C' = A' B' in which C' is C interleaved the same way and B' (2n x 2n) has, in its
// K-major (transposed) form, the rows
//   B'^T[2j]   = M[j]                         -> Re C[i][j] = sum_k Re A Re M + Im A Im M
//   B'^T[2j+1] = (i M)[j] = (-Im M, Re M)     -> Im C[i][j] = sum_k Im A Re M - Re A Im M
// so both operands are read row by row from the complex matrices with no transpose, and the
// real GEMM does exactly the 8 n^3 flops of the complex one.  A hermitian X is its own M
// (X = X^+), which covers every product of the hermitian-form right-hand side:
// L_k X = L_k X^+, Hnh X = Hnh X^+ and T_k L_k^+.
//
// Tile: 128 rows x 128 complex columns of C (MMA M = 128, N = 256 real columns) per CTA.
// The hi*hi products accumulate in one TMEM accumulator (256 columns) and the two small
// cross products hi*lo + lo*hi in a second one, summed in FP32 registers at the end: the
// tensor core's accumulation loses a fraction of an ulp of the accumulator per MMA, so
// adding the small terms into the large accumulator would triple that loss.  The contraction runs in stages of 128 bytes of every
// operand row (16 complex values for TF32, 32 for BF16), two stages in shared memory.
// Eight producer warps load complex64 rows (L2-resident), split each value into hi + lo,
// apply the (-Im, Re) map for the odd B rows and store into the swizzled tiles; one warp
// issues the MMAs (lo*hi + hi*lo + hi*hi with FP32 accumulation in TMEM: 3xTF32 or 3xBF16;
// hi*hi alone in the single-pass TF32 mode); the eight warps then read the accumulator out
// of TMEM (warp w reads lanes 32 (w % 4) .. +31, column half w / 4) and write C.
namespace tcg {
constexpr int kProdWarps = 8;
constexpr int kProd = kProdWarps * 32;
constexpr int kThreads = kProd + 32;
constexpr uint32_t kAccCols = 256;             // one FP32 accumulator: 128 lanes x 256 columns
// Stage geometry for a K-slice of RB bytes of every operand row (RB = 128: 128-byte
// swizzle, two 96 KB stages; RB = 64: 64-byte swizzle, four 48 KB stages).
template <int RB>
struct Cfg {
  static constexpr uint32_t kA = 128 * RB;                // one 128-row operand tile (bytes)
  static constexpr uint32_t kB = 256 * RB;                // one 256-row operand tile
  static constexpr uint32_t kStage = 2 * kA + 2 * kB;     // A hi, A lo, B hi, B lo
  static constexpr int kStages = RB == 128 ? 2 : 4;
  static constexpr int kSmem = kStages * kStage + 1024;   // + alignment slack
  static constexpr int kChunks = RB / 16;                 // 16-byte chunks per tile row
  static constexpr int kJobs = 128 * kChunks / kProd;     // chunks of A (and of M) per producer
  static constexpr int kMma = RB / 32;                    // MMAs (32 bytes of K each) per stage
  // byte offset of chunk c of row r in a swizzled K-major tile
  static __device__ __forceinline__ uint32_t off(uint32_t r, uint32_t c) {
    return RB == 128 ? r * 128 + ((c ^ (r & 7)) << 4) : r * 64 + ((c ^ ((r >> 1) & 3)) << 4);
  }
  static __device__ __forceinline__ uint64_t desc(uint32_t saddr) {
    return RB == 128 ? tc::smem_desc_k128(saddr) : tc::smem_desc_k64(saddr);
  }
};
}  // namespace tcg

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}

__device__ __forceinline__ void st_split_tf32(uint32_t hi_addr, uint32_t lo_addr, float4 v, bool split) {
  float h0, h1, h2, h3, l0, l1, l2, l3;
  tc::split_tf32(v.x, h0, l0);
  tc::split_tf32(v.y, h1, l1);
  tc::split_tf32(v.z, h2, l2);
  tc::split_tf32(v.w, h3, l3);
  st_shared_v4(hi_addr, __float_as_uint(h0), __float_as_uint(h1), __float_as_uint(h2), __float_as_uint(h3));
  if (split)
    st_shared_v4(lo_addr, __float_as_uint(l0), __float_as_uint(l1), __float_as_uint(l2), __float_as_uint(l3));
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
  lo = *reinterpret_cast<const uint32_t*>(&l);
  return *reinterpret_cast<const uint32_t*>(&h);
}

__device__ __forceinline__ void st_split_bf16(uint32_t hi_addr, uint32_t lo_addr, float4 u, float4 v) {
  uint32_t l0, l1, l2, l3;
  const uint32_t h0 = pack_bf16(u.x, u.y, l0);
  const uint32_t h1 = pack_bf16(u.z, u.w, l1);
  const uint32_t h2 = pack_bf16(v.x, v.y, l2);
  const uint32_t h3 = pack_bf16(v.z, v.w, l3);
  st_shared_v4(hi_addr, h0, h1, h2, h3);
  st_shared_v4(lo_addr, l0, l1, l2, l3);
}

// The RB-byte slice [k0, k0 + KC) of this thread's A and M chunks.  Job e = ptid + 256 q
// covers row e / kChunks, 16-byte shared-memory chunk e % kChunks; a chunk is one float4
// (two complex values) for TF32 and two float4 (four complex values) for BF16.
template <int RB, bool BF16>
__device__ __forceinline__ void tc_load_stage(float4 (&v)[(BF16 ? 4 : 2) * tcg::Cfg<RB>::kJobs],
                                              const float2* __restrict__ A, const float2* __restrict__ M, int n,
                                              int row0, int col0, int k0, int ptid) {
  using C = tcg::Cfg<RB>;
  constexpr int PER = BF16 ? 2 : 1;
#pragma unroll
  for (int q = 0; q < C::kJobs; ++q) {
    const int e = ptid + tcg::kProd * q;
    const int r = e / C::kChunks, cc = e % C::kChunks;
    const int gr = row0 + r, gj = col0 + r;
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int k = k0 + (cc * PER + p) * 2;  // n is even, so a float4 is all in or all out
      v[q * PER + p] = (gr < n && k < n) ? __ldg(reinterpret_cast<const float4*>(A + (long long)gr * n + k))
                                         : make_float4(0.f, 0.f, 0.f, 0.f);
      v[C::kJobs * PER + q * PER + p] = (gj < n && k < n)
                                            ? __ldg(reinterpret_cast<const float4*>(M + (long long)gj * n + k))
                                            : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
}

template <int RB, bool BF16, bool SPLIT>
__device__ __forceinline__ void tc_store_stage(const float4 (&v)[(BF16 ? 4 : 2) * tcg::Cfg<RB>::kJobs], uint32_t st,
                                               int ptid) {
  using C = tcg::Cfg<RB>;
  const uint32_t Ahi = st, Alo = st + C::kA, Bhi = st + 2 * C::kA, Blo = st + 2 * C::kA + C::kB;
  constexpr int MJ = (BF16 ? 2 : 1) * C::kJobs;  // first M value in v
#pragma unroll
  for (int q = 0; q < C::kJobs; ++q) {
    const int e = ptid + tcg::kProd * q;
    const uint32_t r = e / C::kChunks, cc = e % C::kChunks;
    const uint32_t oa = C::off(r, cc);
    const uint32_t ob0 = C::off(2 * r, cc);
    const uint32_t ob1 = C::off(2 * r + 1, cc);
    // The (-Im, Re) row of M is the (Re, Im) row's split with its pairs swapped and the
    // first element negated: the hi/lo split commutes with negation, so each value of M is
    // split once.
    if (!BF16) {
      const float4 a = v[q], m = v[MJ + q];
      st_split_tf32(Ahi + oa, Alo + oa, a, SPLIT);
      float h0, h1, h2, h3, l0, l1, l2, l3;
      tc::split_tf32(m.x, h0, l0);
      tc::split_tf32(m.y, h1, l1);
      tc::split_tf32(m.z, h2, l2);
      tc::split_tf32(m.w, h3, l3);
      st_shared_v4(Bhi + ob0, __float_as_uint(h0), __float_as_uint(h1), __float_as_uint(h2), __float_as_uint(h3));
      st_shared_v4(Bhi + ob1, __float_as_uint(-h1), __float_as_uint(h0), __float_as_uint(-h3), __float_as_uint(h2));
      if (SPLIT) {
        st_shared_v4(Blo + ob0, __float_as_uint(l0), __float_as_uint(l1), __float_as_uint(l2), __float_as_uint(l3));
        st_shared_v4(Blo + ob1, __float_as_uint(-l1), __float_as_uint(l0), __float_as_uint(-l3), __float_as_uint(l2));
      }
    } else {
      const float4 a0 = v[2 * q], a1 = v[2 * q + 1], m0 = v[MJ + 2 * q], m1 = v[MJ + 2 * q + 1];
      st_split_bf16(Ahi + oa, Alo + oa, a0, a1);
      uint32_t l0, l1, l2, l3;
      const uint32_t h0 = pack_bf16(m0.x, m0.y, l0);
      const uint32_t h1 = pack_bf16(m0.z, m0.w, l1);
      const uint32_t h2 = pack_bf16(m1.x, m1.y, l2);
      const uint32_t h3 = pack_bf16(m1.z, m1.w, l3);
      st_shared_v4(Bhi + ob0, h0, h1, h2, h3);
      st_shared_v4(Blo + ob0, l0, l1, l2, l3);
      // (re, im) in the low / high halves -> (-im, re)
      auto rot = [](uint32_t x) { return ((x >> 16) ^ 0x8000u) | (x << 16); };
      st_shared_v4(Bhi + ob1, rot(h0), rot(h1), rot(h2), rot(h3));
      st_shared_v4(Blo + ob1, rot(l0), rot(l1), rot(l2), rot(l3));
    }
  }
}

// grid (tiles128^2, 1, B * Kz), kThreads threads, kSmem dynamic shared bytes.  Same job
// semantics as cgemm_kernel, restricted to terms A M^+ (opA = 0; opB = 1, or B = the
// hermitian stage input) with one alpha; on a wait that runs out the tile is written as
// NaN, which the error norm turns into DQB_INST_NONFINITE.
template <int PREC, int RB>
__global__ void __launch_bounds__(tcg::kThreads, 1)
    tc_cgemm_kernel(big::Common c, LargeOps d, GemmJob job, const float2* ext_in, float2* ext_out) {
  using Cf = tcg::Cfg<RB>;
  constexpr bool kBf16 = PREC == DQB_PREC_BF16X3;
  constexpr bool kSplit = PREC != DQB_PREC_TF32;
  constexpr int KC = kBf16 ? RB / 4 : RB / 8;  // complex contraction values per stage
  constexpr int NV = (kBf16 ? 4 : 2) * Cf::kJobs;
  constexpr uint32_t kCols = kSplit ? 2 * tcg::kAccCols : tcg::kAccCols;
  extern __shared__ uint8_t tc_dsm[];
  __shared__ uint64_t bars[2 * Cf::kStages + 1];
  __shared__ uint32_t tmem_sh;
  __shared__ int fail_sh;

  const int n = d.n;
  const int Kz = job.kdst < 0 ? d.K : 1;
  const int b = blockIdx.z / Kz;
  const int kz = job.kdst < 0 ? (int)(blockIdx.z % Kz) : job.kdst;
  if (job_skips(c, b, job.need_run, job.kry)) return;
  const int Kb = jumps_of(d, b);
  if (job.kdst < 0 && kz >= Kb) return;
  const int tiles = (n + 127) >> 7;
  const int row0 = (blockIdx.x / tiles) * 128, col0 = (blockIdx.x % tiles) * 128;

  const float2* Ap[4];
  const float2* Mp[4];
  int nt = 0;
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    if (t >= job.nterms) break;
    const Term T = job.t[t];
    if ((T.srcA == SRC_T || T.srcA == SRC_L) && T.kA >= Kb) continue;  // missing jump
    Ap[nt] = src_ptr(c, d, b, T.srcA, T.kA < 0 ? kz : T.kA, job.in_sel, ext_in);
    Mp[nt] = src_ptr(c, d, b, T.srcB, T.kB < 0 ? kz : T.kB, job.in_sel, ext_in);
    ++nt;
  }
  const int kchunks = (n + KC - 1) / KC;
  const int total = nt * kchunks;

  const uint32_t raw = tc::smem_u32(tc_dsm);
  const uint32_t sbase = (raw + 1023u) & ~1023u;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t bar_full = tc::smem_u32(&bars[0]);
  const uint32_t bar_empty = tc::smem_u32(&bars[Cf::kStages]);
  const uint32_t bar_done = tc::smem_u32(&bars[2 * Cf::kStages]);
  if (warp == tcg::kProdWarps) {
    tc::tmem_alloc(tc::smem_u32(&tmem_sh), kCols);
    tc::tmem_relinquish();
    if (lane == 0) {
      for (int s = 0; s < Cf::kStages; ++s) {
        tc::mbar_init(bar_full + 8 * s, tcg::kProd);
        tc::mbar_init(bar_empty + 8 * s, 1);
      }
      tc::mbar_init(bar_done, 1);
      tc::fence_mbar_init();
      fail_sh = 0;
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = tmem_sh;

  if (warp < tcg::kProdWarps) {
    // ---- producers ----
    // Global loads run PRE stages ahead of the shared-memory stores (as many as the
    // registers hold: two 128-byte TF32 stages or one BF16 stage; twice that for 64 bytes).
    constexpr int PRE = (kBf16 ? 1 : 2) * (128 / RB);
    const int ptid = threadIdx.x;
    float4 buf[PRE + 1][NV];
#pragma unroll
    for (int p = 0; p < PRE; ++p)
      if (p < total)
        tc_load_stage<RB, kBf16>(buf[p], Ap[p / kchunks], Mp[p / kchunks], n, row0, col0, (p % kchunks) * KC,
                                 ptid);
    for (int it = 0; it < total; ++it) {
      const int s = it % Cf::kStages;
      if (it + PRE < total) {
        const int term = (it + PRE) / kchunks;
        tc_load_stage<RB, kBf16>(buf[PRE], Ap[term], Mp[term], n, row0, col0, ((it + PRE) % kchunks) * KC, ptid);
      }
      if (it >= Cf::kStages && !tc::mbar_wait(bar_empty + 8 * s, ((it / Cf::kStages) - 1) & 1)) {
        fail_sh = 1;
        break;
      }
      tc_store_stage<RB, kBf16, kSplit>(buf[0], sbase + s * Cf::kStage, ptid);
      tc::fence_proxy_async_smem();
      tc::mbar_arrive(bar_full + 8 * s);
#pragma unroll
      for (int p = 0; p < PRE; ++p)
#pragma unroll
        for (int i = 0; i < NV; ++i) buf[p][i] = buf[p + 1][i];
    }
  } else if (lane == 0) {
    // ---- MMA issuer ----
    constexpr uint32_t idesc = tc::instr_desc(kBf16 ? 1u : 2u, 128, 256);
    for (int it = 0; it < total; ++it) {
      const int s = it % Cf::kStages;
      if (!tc::mbar_wait(bar_full + 8 * s, (it / Cf::kStages) & 1)) {
        fail_sh = 1;
        break;
      }
      tc::tc_fence_after();
      const uint32_t st = sbase + s * Cf::kStage;
#pragma unroll
      for (int kk = 0; kk < Cf::kMma; ++kk) {
        const uint64_t ah = Cf::desc(st + kk * 32);
        const uint64_t al = Cf::desc(st + Cf::kA + kk * 32);
        const uint64_t bh = Cf::desc(st + 2 * Cf::kA + kk * 32);
        const uint64_t bl = Cf::desc(st + 2 * Cf::kA + Cf::kB + kk * 32);
        const uint32_t acc = (it | kk) ? 1u : 0u;
        const uint32_t small = tmem + tcg::kAccCols;
        if (kBf16) {
          tc::mma_bf16(small, al, bh, idesc, acc);
          tc::mma_bf16(small, ah, bl, idesc, 1u);
          tc::mma_bf16(tmem, ah, bh, idesc, acc);
        } else if (kSplit) {
          tc::mma_tf32(small, al, bh, idesc, acc);
          tc::mma_tf32(small, ah, bl, idesc, 1u);
          tc::mma_tf32(tmem, ah, bh, idesc, acc);
        } else {
          tc::mma_tf32(tmem, ah, bh, idesc, acc);
        }
      }
      tc::mma_commit(bar_empty + 8 * s);
    }
    tc::mma_commit(bar_done);
  }

  if (warp < tcg::kProdWarps) {
    // ---- epilogue: TMEM -> registers -> C ----
    __syncwarp();
    bool got = tc::mbar_wait(bar_done, 0);
    got = __all_sync(0xffffffffu, got);
    tc::tc_fence_after();
    const bool bad = __any_sync(0xffffffffu, !got || fail_sh != 0);
    const int q = warp & 3, h = warp >> 2;
    const int r = row0 + 32 * q + lane;
    float2* C;
    if (ext_out) {
      C = ext_out + (long long)b * n * n;
    } else if (job.dst == SRC_T) {
      C = d.T + ((long long)b * d.K + kz) * (long long)n * n;
    } else {
      C = d.tmp + (long long)b * n * n;
    }
    const float alpha = job.t[0].alpha;
#pragma unroll 1
    for (int ch = 0; ch < 8; ++ch) {
      const int fcol = h * 128 + ch * 16;
      float v[16];
      __syncwarp();
      if (!bad && total > 0) {
        const uint32_t ta = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)fcol;
        tc::tmem_ld16(ta, v);
        if (kSplit) {
          float w[16];
          tc::tmem_ld16(ta + tcg::kAccCols, w);
          tc::tmem_ld_wait();
#pragma unroll
          for (int i = 0; i < 16; ++i) v[i] += w[i];
        } else {
          tc::tmem_ld_wait();
        }
      } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = bad ? __int_as_float(0x7fc00000) : 0.f;
      }
      const int cc0 = col0 + (fcol >> 1);
      if (r >= n || cc0 >= n) continue;
      float2* row = C + (long long)r * n + cc0;
      if (cc0 + 8 <= n) {
#pragma unroll
        for (int j = 0; j < 8; j += 2) {
          float4 o = make_float4(alpha * v[2 * j], alpha * v[2 * j + 1], alpha * v[2 * j + 2], alpha * v[2 * j + 3]);
          if (job.accumulate) {
            const float4 p = *reinterpret_cast<const float4*>(row + j);
            o.x += p.x;
            o.y += p.y;
            o.z += p.z;
            o.w += p.w;
          }
          *reinterpret_cast<float4*>(row + j) = o;
        }
      } else {
        for (int j = 0; j < 8 && cc0 + j < n; ++j) {
          float2 o = make_float2(alpha * v[2 * j], alpha * v[2 * j + 1]);
          if (job.accumulate) o = cadd(o, row[j]);
          row[j] = o;
        }
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == tcg::kProdWarps) {
    __syncwarp();
    tc::tmem_dealloc(tmem, kCols);
  }
}

// The GEMM path's products run on the tensor cores when a precision other than FP32 is
// asked for, the form is hermitian (every product is then A M^+) and n is even (float4
// rows).
bool use_tc(const LargeOps& d, int form) {
  return d.prec != DQB_PREC_FP32 && form == DQB_FORM_HERMITIAN && (d.n % 2) == 0;
}

// K-slice of the tensor-core GEMM's stages: 128 bytes (two 96 KB stages) unless
// DQB_TC_SLICE=64 in the environment (four 48 KB stages), read once.  The 128-byte slice is
// the faster one: 67.3 against 50.4 solves/s on the transmon x cavity workload (n = 256,
// 3xTF32), as the shorter slice doubles the barrier round trips and MMA issues per byte.
inline int tc_slice() {
  static const int rb = [] {
    const char* v = std::getenv("DQB_TC_SLICE");
    return (v != nullptr && std::atoi(v) == 64) ? 64 : 128;
  }();
  return rb;
}

template <int RB>
void launch_tc(cudaStream_t s, dim3 g, const big::Common& c, const LargeOps& d, const GemmJob& j,
               const float2* ext_in, float2* ext_out) {
  constexpr int sm = tcg::Cfg<RB>::kSmem;
  switch (d.prec) {
    case DQB_PREC_TF32X3:
      tc_cgemm_kernel<DQB_PREC_TF32X3, RB><<<g, tcg::kThreads, sm, s>>>(c, d, j, ext_in, ext_out);
      break;
    case DQB_PREC_BF16X3:
      tc_cgemm_kernel<DQB_PREC_BF16X3, RB><<<g, tcg::kThreads, sm, s>>>(c, d, j, ext_in, ext_out);
      break;
    default:
      tc_cgemm_kernel<DQB_PREC_TF32, RB><<<g, tcg::kThreads, sm, s>>>(c, d, j, ext_in, ext_out);
      break;
  }
}

void launch_gemm(cudaStream_t s, const big::Common& c, const LargeOps& d, const GemmJob& j, int zdim,
                 const float2* ext_in, float2* ext_out, bool tcp) {
  if (tcp) {
    const int t = (d.n + 127) / 128;
    const dim3 g(t * t, 1, zdim);
    if (tc_slice() == 128)
      launch_tc<128>(s, g, c, d, j, ext_in, ext_out);
    else
      launch_tc<64>(s, g, c, d, j, ext_in, ext_out);
  } else {
    const int t = (d.n + BM - 1) / BM;
    cgemm_kernel<<<dim3(t * t, 1, zdim), NT, 0, s>>>(c, d, j, ext_in, ext_out);
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
                int need_run, int form, const float2* ext_in, float2* ext_out, int kry = 0) {
  const int n = d.n;
  const bool tcp = use_tc(d, form);
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
    j1.kry = kry;
    launch_gemm(s, c, d, j1, B * d.K, ext_in, nullptr, tcp);
  }
  // tmp = Hnh X + sum_k T_k L_k^+ [+ X Hnh^+]: at most 4 summed terms per launch, the
  // rest accumulated by further launches into tmp
  GemmJob j2;
  std::memset(&j2, 0, sizeof(j2));
  j2.dst = SRC_TMP;
  j2.kdst = 0;
  j2.in_sel = in_sel;
  j2.need_run = need_run;
  j2.kry = kry;
  int nt = 0;
  j2.t[nt++] = Term{SRC_HNH, 0, 0, SRC_IN, 0, 0, 1.0f};
  if (form == DQB_FORM_STANDARD) j2.t[nt++] = Term{SRC_IN, 0, 0, SRC_HNH, 0, 1, 1.0f};
  int k = 0;
  for (;;) {
    while (k < d.K && nt < 4) j2.t[nt++] = Term{SRC_T, k, 0, SRC_L, k, 1, 1.0f}, ++k;
    j2.nterms = nt;
    launch_gemm(s, c, d, j2, B, ext_in, nullptr, tcp);
    if (k >= d.K) break;
    j2.accumulate = 1;
    nt = 0;
  }
  const int t32 = (n + 31) / 32;
  const bool herm = form == DQB_FORM_HERMITIAN;
  symmetrize_kernel<<<herm ? big::herm_grid(n, B) : dim3(t32 * t32, B), 256, 0, s>>>(c, d, out_k, need_run, herm, kry,
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

// Form of the RK step on the GEMM path: the Krylov form when asked for.
bool large_krylov(const dqb_ode_options& o) { return o.stepper == DQB_STEPPER_KRYLOV; }

int check_precision(int prec, int form, int n) {
  if (prec < DQB_PREC_FP32 || prec > DQB_PREC_TF32) return DQB_ERR_INVALID_ARGUMENT;
  if (prec != DQB_PREC_FP32 && (form != DQB_FORM_HERMITIAN || n % 2 != 0)) return DQB_ERR_UNSUPPORTED;
  return DQB_OK;
}

GraphCache g_cache;

// Prefactors c_k(t) of the jump operators (time-dependent jump operators), by value.
struct JumpTd {
  int on;
  TdTerm term[16];
};

struct LaunchKey {
  big::Common c;
  LargeOps d;
  TdOps td;
  JumpTd jt;
  float2* hnh0;
  const float2* L0;
  int form, krylov;
};

// Time-dependent jump operators: the per-instance copies L_k(t) = c_k(t) L_k that the
// products read (L0: the given operators, indexed by L0idx), at the time of a right-hand
// side (big::td_stage_time).  grid (tiles, B).
__global__ void lt_td_dense_kernel(big::Common c, LargeOps d, JumpTd jt, const float2* L0, const int* L0idx,
                                   int which) {
  __shared__ float2 ck[16];
  const int b = blockIdx.y;
  double t;
  if (!big::td_stage_time(c, c.inst[b], which, &t)) return;
  if (threadIdx.x < d.K) {
    const double2 v = td_coef(jt.term[threadIdx.x], b, t);
    ck[threadIdx.x] = make_float2((float)v.x, (float)v.y);
  }
  __syncthreads();
  const long long nn = c.nn;
  const long long li = L0idx ? L0idx[b] : b;
  const float2* src = L0 + li * d.K * nn;
  float2* dst = const_cast<float2*>(d.L) + (long long)b * d.K * nn;
  for (int k = 0; k < d.K; ++k)
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn; e += (long long)gridDim.x * blockDim.x)
      dst[k * nn + e] = cmul(ck[k], src[k * nn + e]);
}

// Hnh at the time of a right-hand side (big::td_stage_time) of a time-dependent H:
// hnh = hnh0 - i sum_m c_m(t) ops_m, ops dense [M, n, n].  grid (tiles, B).
__global__ void hnh_td_dense_kernel(big::Common c, LargeOps d, TdOps td, const float2* hnh0, int which) {
  __shared__ float2 cm[DQB_TD_MAX_TERMS];
  const int b = blockIdx.y;
  double t;
  if (!big::td_stage_time(c, c.inst[b], which, &t)) return;
  if (threadIdx.x < td.M) {
    const double2 v = td_coef(td.term[threadIdx.x], b, t);
    cm[threadIdx.x] = make_float2((float)v.x, (float)v.y);
  }
  __syncthreads();
  const long long nn = c.nn;
  const float2* h0 = hnh0 + (long long)b * nn;
  float2* out = d.hnh + (long long)b * nn;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn; e += (long long)gridDim.x * blockDim.x) {
    float2 a = make_float2(0.f, 0.f);
    for (int m = 0; m < td.M; ++m) a = cfma(cm[m], td.ops[(long long)m * nn + e], a);
    const float2 v = h0[e];
    out[e] = make_float2(v.x + a.y, v.y - a.x);  // hnh0 - i a
  }
}

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
    prefer_max_shared(big::retire_kernel);
    prefer_max_shared(big::pre_finalize_kernel);
    prefer_max_shared(big::finalize_kernel);
    prefer_max_shared(zero_words_kernel);
    prefer_max_shared(cgemm_kernel);
    prefer_max_shared(symmetrize_kernel);
    prefer_max_shared(hnh_td_dense_kernel);
    prefer_max_shared(lt_td_dense_kernel);
    auto tc_attrs = [](auto kern, int smem) {
      prefer_max_shared(kern);
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    };
    tc_attrs(tc_cgemm_kernel<DQB_PREC_TF32X3, 128>, tcg::Cfg<128>::kSmem);
    tc_attrs(tc_cgemm_kernel<DQB_PREC_BF16X3, 128>, tcg::Cfg<128>::kSmem);
    tc_attrs(tc_cgemm_kernel<DQB_PREC_TF32, 128>, tcg::Cfg<128>::kSmem);
    tc_attrs(tc_cgemm_kernel<DQB_PREC_TF32X3, 64>, tcg::Cfg<64>::kSmem);
    tc_attrs(tc_cgemm_kernel<DQB_PREC_BF16X3, 64>, tcg::Cfg<64>::kSmem);
    tc_attrs(tc_cgemm_kernel<DQB_PREC_TF32, 64>, tcg::Cfg<64>::kSmem);
  });
}

// The solve; `td` (or null) with `hnh0` (B n^2 values): the time-dependent terms of H;
// `jt` (or null) with `Lt` (B K n^2 values): time-dependent jump operators, whose copies
// c_k(t) L_k the products then read (and Hnh is formed by the GEMM from them at every
// right-hand side).
static int run_large(const big::Common& c, const LargeOps& d_in, cudaStream_t s, bool krylov,
                     const TdOps* td = nullptr, float2* hnh0 = nullptr, const JumpTd* jt = nullptr,
                     float2* Lt = nullptr) {
  init_carveouts();
  LargeOps d = d_in;
  JumpTd jtv;
  std::memset(&jtv, 0, sizeof(jtv));
  const float2* L0 = d_in.L;
  const int* L0idx = d_in.Lidx;
  if (jt && jt->on) {
    jtv = *jt;
    d.L = Lt;
    d.Lidx = nullptr;
  }
  const int B = c.B;
  int grid_e = (int)std::min<long long>((c.nn + big::kElemThreads - 1) / big::kElemThreads, 1184);
  if (grid_e < 1) grid_e = 1;
  const dim3 ge(grid_e, B);
  const dim3 gi((B + 127) / 128);
  const int T = big::kElemThreads;
  const int form = c.form;

  const bool timedep = td != nullptr;
  TdOps tdv;
  std::memset(&tdv, 0, sizeof(tdv));
  if (timedep) tdv = *td;
  // Hnh (and the jump operators) at the time of the next right-hand side (time-dependent
  // operators only)
  auto at_time = [&](cudaStream_t cs, int which) {
    if (jtv.on) {
      lt_td_dense_kernel<<<ge, T, 0, cs>>>(c, d, jtv, L0, L0idx, which);
      // Hnh = -iH - 1/2 sum L(t)^+ L(t) by the GEMM, for the instances that evaluate it
      launch_hnh(cs, c, d, B, which >= 8 ? 0 : (which == 7 ? 3 : 1));
      if (tdv.M > 0) hnh_td_dense_kernel<<<ge, T, 0, cs>>>(c, d, tdv, d.hnh, which);  // in place
    } else if (timedep) {
      hnh_td_dense_kernel<<<ge, T, 0, cs>>>(c, d, tdv, hnh0, which);
    }
  };

  big::setup_kernel<<<gi, 128, 0, s>>>(c);
  big::load_rho0_kernel<<<ge, T, 0, s>>>(c);
  if (!jtv.on) {  // (with time-dependent jump operators every Hnh is formed at its time)
    LargeOps d0 = d;  // the constant Hnh: into hnh, or into hnh0 when H depends on time
    if (timedep) d0.hnh = hnh0;
    launch_hnh(s, c, d0, B, 0);
  }
  at_time(s, 8);
  launch_rhs(s, c, d, B, 0, 0, 0, form, nullptr, nullptr);
  big::init_norm_kernel<<<ge, T, 0, s>>>(c, 0);
  big::init_ctrl_kernel<<<gi, 128, 0, s>>>(c, 0);
  if (krylov) {
    // the probe f(y + h0 k1) - f(y) of the starting step is h0 L k1 for a linear f
    launch_rhs(s, c, d, B, 3, 1, 0, form, nullptr, nullptr);
    big::init_norm_kernel<<<ge, T, 0, s>>>(c, 2);
  } else {
    big::launch_combine(s, c, ge, 6);
    at_time(s, 9);
    launch_rhs(s, c, d, B, 2, 1, 0, form, nullptr, nullptr);
    big::init_norm_kernel<<<ge, T, 0, s>>>(c, 1);
  }
  big::init_ctrl_kernel<<<gi, 128, 0, s>>>(c, 1);
  if (cudaGetLastError() != cudaSuccess) return DQB_ERR_CUDA;

  auto body = [&](cudaStream_t cs, cudaGraphConditionalHandle h, int* flag) {
    if (krylov) {
      for (int q = 1; q <= 6; ++q) launch_rhs(cs, c, d, B, q + 2, q, 1, form, nullptr, nullptr, q);
      big::launch_kry_combine(cs, c, ge);
      big::control_kernel<<<gi, 128, 0, cs>>>(c);
      big::launch_save(cs, c, ge, 2);
      big::kry_commit_kernel<<<1, 1024, 0, cs>>>(c, h, flag);
      if (c.rag) big::retire_kernel<<<B, 256, 0, cs>>>(c);
      return;
    }
    for (int st = 0; st < 5; ++st) {
      big::launch_combine(cs, c, ge, st);
      at_time(cs, st + 1);
      launch_rhs(cs, c, d, B, 2, st + 1, 1, form, nullptr, nullptr);
    }
    big::launch_combine(cs, c, ge, 5);
    at_time(cs, 6);
    launch_rhs(cs, c, d, B, 1, 6, 1, form, nullptr, nullptr);
    big::launch_error(cs, c, ge);
    big::control_kernel<<<gi, 128, 0, cs>>>(c);
    big::launch_save(cs, c, ge, 1);
    big::commit_kernel<<<1, 1024, 0, cs>>>(c, h, flag);
    if (c.rag) big::retire_kernel<<<B, 256, 0, cs>>>(c);
    if (timedep) {  // the first stage of a step that starts on a discontinuity
      at_time(cs, 7);
      launch_rhs(cs, c, d, B, 0, 0, 3, form, nullptr, nullptr);
    }
  };
  if (host_loop_requested()) {
    if (run_host_loop(body, (int*)(c.iter + 1), s) != cudaSuccess) return DQB_ERR_CUDA;
  } else {
    LaunchKey key;
    std::memset(&key, 0, sizeof(key));
    key.c = c;
    key.d = d;
    key.td = tdv;
    key.jt = jtv;
    key.hnh0 = hnh0;
    key.L0 = L0;
    key.form = form;
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
  big::pre_finalize_kernel<<<gi, 128, 0, s>>>(c);
  big::launch_save(s, c, ge, 0);
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
  return dqb_lindblad_rhs_dense_large_prec(p, form, DQB_PREC_FP32, rho, outp, workspace, workspace_bytes, stream);
}

extern "C" int dqb_lindblad_rhs_dense_large_prec(const dqb_dense_problem* p, int32_t form, int32_t precision,
                                                 const void* rho, void* outp, void* workspace,
                                                 size_t workspace_bytes, void* stream) {
  int rc = check_dense_large(p);
  if (rc) return rc;
  if (!rho || !outp) return DQB_ERR_INVALID_ARGUMENT;
  if (form != DQB_FORM_HERMITIAN && form != DQB_FORM_STANDARD) return DQB_ERR_INVALID_ARGUMENT;
  rc = check_precision(precision, form, p->n);
  if (rc) return rc;
  if (p->batch == 0) return DQB_OK;
  const LargeLayout lay = large_layout(p->n, p->n_jumps, 0, 1, p->batch);
  if (!workspace || workspace_bytes < lay.off_mats) return DQB_ERR_WORKSPACE_TOO_SMALL;
  LargeOps d = make_ops(p, (char*)workspace, lay);
  d.prec = precision;
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
  if (o->stepper < DQB_STEPPER_AUTO || o->stepper > DQB_STEPPER_KRYLOV) return DQB_ERR_INVALID_ARGUMENT;
  if (int prc = check_precision(o->precision, o->form, n)) return prc;
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
  d.prec = o->precision;
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
  return run_large(c, d, (cudaStream_t)stream, large_krylov(*o));
}

static int solve_large(const dqb_dense_problem* p, const dqb_td_hamiltonian* tdh, const dqb_ode_options* o,
                       const dqb_outputs* out, void* workspace, size_t workspace_bytes, void* stream) {
  int rc = check_dense_large(p);
  if (rc) return rc;
  if (!o || !out || !out->states || !out->infos || !out->status || (p->n_exp > 0 && !out->expects))
    return DQB_ERR_INVALID_ARGUMENT;
  if (p->n_exp < 0 || p->n_tsave < 1 || !p->rho0 || !p->tsave || (p->n_exp > 0 && !p->E))
    return DQB_ERR_INVALID_ARGUMENT;
  if (o->method != DQB_METHOD_TSIT5 && o->method != DQB_METHOD_DOPRI5) return DQB_ERR_INVALID_ARGUMENT;
  if (o->form != DQB_FORM_HERMITIAN && o->form != DQB_FORM_STANDARD) return DQB_ERR_INVALID_ARGUMENT;
  if (!(o->rtol >= 0) || !(o->atol >= 0) || o->max_steps < 0) return DQB_ERR_INVALID_ARGUMENT;
  if (o->stepper < DQB_STEPPER_AUTO || o->stepper > DQB_STEPPER_KRYLOV) return DQB_ERR_INVALID_ARGUMENT;
  if (int prc = check_precision(o->precision, o->form, p->n)) return prc;
  TdOps td;
  JumpTd jt;
  std::memset(&jt, 0, sizeof(jt));
  if (tdh) {
    // the Krylov form needs a constant right-hand side
    if (large_krylov(*o)) return DQB_ERR_UNSUPPORTED;
    if (int tr = td_ops_from(tdh, &td)) return tr;
    if (tdh->jump_terms) {
      if (p->n_jumps > 16) return DQB_ERR_UNSUPPORTED;
      jt.on = 1;
      for (int k = 0; k < p->n_jumps; ++k)
        if (int tr = td_term_from(tdh->jump_terms[k], &jt.term[k])) return tr;
    }
  }
  if (p->batch == 0) return DQB_OK;
  const LargeLayout lay = large_layout(p->n, p->n_jumps, p->n_exp, p->n_tsave, p->batch);
  const size_t nnb = (size_t)p->batch * p->n * p->n * sizeof(float2);
  const size_t need = tdh ? align_up(lay.total) + nnb * (1 + std::max(p->n_jumps, 1)) : lay.total;
  if (!workspace || workspace_bytes < need) return DQB_ERR_WORKSPACE_TOO_SMALL;
  char* ws = (char*)workspace;
  LargeOps d = make_ops(p, ws, lay);
  d.prec = o->precision;

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
  if (!tdh) return run_large(c, d, (cudaStream_t)stream, large_krylov(*o));
  c.n_jump = tdh->n_jump_ts;
  c.jump_ts = tdh->jump_ts;
  return run_large(c, d, (cudaStream_t)stream, false, &td, (float2*)(ws + align_up(lay.total)), &jt,
                   (float2*)(ws + align_up(lay.total) + nnb));
}

extern "C" int dqb_mesolve_dense_large(const dqb_dense_problem* p, const dqb_ode_options* o, const dqb_outputs* out,
                                       void* workspace, size_t workspace_bytes, void* stream) {
  return solve_large(p, nullptr, o, out, workspace, workspace_bytes, stream);
}

extern "C" size_t dqb_mesolve_dense_large_td_workspace_size(int32_t n, int32_t n_jumps, int32_t n_exp,
                                                            int32_t n_tsave, int64_t batch) {
  const size_t base = dqb_mesolve_dense_large_workspace_size(n, n_jumps, n_exp, n_tsave, batch);
  return base ? align_up(base) + (size_t)batch * n * n * sizeof(float2) * (1 + std::max(n_jumps, 1)) : 0;
}

extern "C" int dqb_mesolve_dense_large_td(const dqb_dense_problem* p, const dqb_td_hamiltonian* td,
                                          const dqb_ode_options* o, const dqb_outputs* out, void* workspace,
                                          size_t workspace_bytes, void* stream) {
  if (!td) return DQB_ERR_INVALID_ARGUMENT;
  return solve_large(p, td, o, out, workspace, workspace_bytes, stream);
}
