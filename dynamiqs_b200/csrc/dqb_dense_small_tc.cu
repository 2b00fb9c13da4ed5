// Persistent batched mesolve kernel for dense operators with 32 < n <= 64 whose products
// run on the tcgen05 tensor cores (the engine of solve_one, dqb_small.cuh), hermitian form,
// at most two jump operators.
//
// Arithmetic.  Every operand is split into two FP16 values, x * s = hi + lo, after
// scaling the matrix by a power of two s that puts its largest entry just below 2^14
// (so hi never overflows and lo keeps 11 bits down to 2^-24); each real product is then
// hi*hi + hi*lo + lo*hi with FP32 accumulation in tensor memory, ~22 bits per product --
// the accuracy of FP32 CUDA-core products, with FP16 operands at half the shared memory of
// a TF32 split and twice its tensor throughput.  The scales are exact powers of two, so
// they cost no rounding.
//
// Complex products as real ones.  A complex product C = A B is one real MMA of M = 128
// rows, N = 128 columns: the A tile holds Re A in rows 0-63 and Im A in rows 64-127, the B
// tile (stored as B^T, K-major) holds Re B in rows 0-63 and Im B in rows 64-127, so the
// accumulator D holds [[ArBr, ArBi], [AiBr, AiBi]] and Cr = D[i][j] - D[64+i][64+j],
// Ci = D[i][64+j] + D[64+i][j] -- a combination across TMEM lanes i and 64+i, done through
// shared memory in the epilogue.  The right-hand side of the hermitian form
// (dynamiqs/integrators/core/diffrax_integrator.py:319-323) is evaluated as
//   T_k = L_k X                                   (one MMA chain per jump, K = 64)
//   tmp = Hnh X + 1/2 sum_k L_k T_k^+             (two accumulators, K = 64 and 64 K)
//   out = tmp + tmp^+
// where L_k T_k^+ = L_k X^+ L_k^+ stands for the reference's (L_k X) L_k^+: the two differ
// by the anti-hermitian part of X only, which tmp + tmp^+ cancels, so the output is the
// reference's for any X.  Hnh X and the L_k tiles (A operands of both products) stay in
// shared memory for the whole solve; T_k becomes the B operand of the second product.
//
// Shared memory (K jumps): X tile 32 KB, Hnh tile 32 KB, one 32 KB tile per jump, one
// 32 KB T tile per jump (at least one; it doubles as the FP32 staging buffer of the
// epilogues): 192 KB at K = 2, one CTA per SM.  Tensor memory: 512 columns (product
// accumulators of both jumps, Hnh X, sum L T^+).  Every mbarrier wait is bounded by
// tc::kWaitLimitNs; a wait that runs out marks the instance non-finite and ends the kernel.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>

#include "dqb_small.cuh"
#include "dqb_tc.cuh"

namespace dqb {

namespace stc {

constexpr int kTile = 16384;           // one 128-row x 64-value FP16 tile
constexpr uint32_t kTmemCols = 512;
constexpr uint32_t kColD1 = 0;         // T_k accumulators at 128 k
constexpr uint32_t kColA = 256;        // Hnh X
constexpr uint32_t kColB = 384;        // sum_k L_k T_k^+

__host__ __device__ constexpr int t_base(int K) { return 4 * kTile + 2 * kTile * K; }
__host__ __device__ constexpr int smem_bytes(int K) {
  return t_base(K) + 2 * kTile * (K > 0 ? K : 1) + 1024;
}

// Byte offset of the 16-byte chunk c (values 8c..8c+7) of row r in a K-major tile with
// the 128-byte swizzle: 8-row atoms of 1024 bytes, chunk position c ^ (r % 8).
__device__ __forceinline__ uint32_t chunk_off(int r, int c) {
  return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((c ^ (r & 7)) << 4));
}

// Store v[0..7] * s as FP16 hi and lo values (hi = fp16(v s), lo = fp16(v s - hi)).
__device__ __forceinline__ void put_chunk(uint8_t* hi_tile, uint8_t* lo_tile, int r, int c,
                                          const float (&v)[8], float s) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const float a = v[2 * q] * s, b = v[2 * q + 1] * s;
    const __half ha = __float2half_rn(a), hb = __float2half_rn(b);
    const __half la = __float2half_rn(a - __half2float(ha)), lb = __float2half_rn(b - __half2float(hb));
    h[q] = (uint32_t)__half_as_ushort(ha) | ((uint32_t)__half_as_ushort(hb) << 16);
    l[q] = (uint32_t)__half_as_ushort(la) | ((uint32_t)__half_as_ushort(lb) << 16);
  }
  const uint32_t off = chunk_off(r, c);
  *reinterpret_cast<uint4*>(hi_tile + off) = make_uint4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<uint4*>(lo_tile + off) = make_uint4(l[0], l[1], l[2], l[3]);
}

// Exponent of the power-of-two scale that puts the largest magnitude m just below 2^14,
// clamped to [-63, 63] so that products and inverses of scales stay finite floats.
__device__ __forceinline__ int scale_exp(float m) {
  if (!(m > 0.f) || !(m < INFINITY)) return 0;
  int e;
  frexpf(m, &e);  // m = f 2^e, f in [0.5, 1)
  return max(-63, min(63, 14 - e));
}

// Largest value of v over the block (every thread gets it); `red` holds >= 9 floats.
__device__ __forceinline__ float block_max(float v, float* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (wid == 0) {
    float x = lane < nw ? red[lane] : 0.f;
    x = warp_max(x);
    if (lane == 0) red[8] = x;
  }
  __syncthreads();
  return red[8];
}

// FP32 complex 64 x 64 staging matrix with an XOR swizzle on the column (bank spread for
// the column-parallel epilogue writes and the transposed reads of the symmetrisation).
__device__ __forceinline__ int sidx(int i, int j) { return i * 64 + (j ^ (i & 31)); }

// The three products of a split operand pair, accumulating into tmem column `d`.
__device__ __forceinline__ void mma3(uint32_t d, uint32_t a_hi, uint32_t b_hi, uint32_t idesc, uint32_t acc) {
  const uint64_t ah = tc::smem_desc_k128(a_hi), al = tc::smem_desc_k128(a_hi + kTile);
  const uint64_t bh = tc::smem_desc_k128(b_hi), bl = tc::smem_desc_k128(b_hi + kTile);
  tc::mma_bf16(d, ah, bh, idesc, acc);  // kind::f16; the descriptor selects FP16 operands
  tc::mma_bf16(d, ah, bl, idesc, 1u);
  tc::mma_bf16(d, al, bh, idesc, 1u);
}

}  // namespace stc

struct TcEngine {
  static constexpr bool kJumps = false, kTape = false;
  uint8_t* g;        // tile area (generic address, 1024-aligned)
  uint32_t s;        // its shared-window address
  uint32_t tmem;     // tensor-memory base (512 columns)
  uint32_t bar1, bar2;
  uint32_t ph1, ph2; // phases of bar1 / bar2 completed so far
  int n, K;
  int eL[2], eH;     // scale exponents of the operators
  float* redf;       // >= 9 floats of shared scratch
  int* fail;         // shared failure flag
  unsigned long long wait_ns;  // limit of every mbarrier wait

  __device__ uint8_t* x_hi() const { return g; }
  __device__ uint8_t* h_hi() const { return g + 2 * stc::kTile; }
  __device__ uint8_t* l_hi(int k) const { return g + 4 * stc::kTile + 2 * stc::kTile * k; }
  __device__ uint8_t* t_hi(int k) const { return g + stc::t_base(K) + 2 * stc::kTile * k; }
  __device__ uint32_t sa(const uint8_t* p) const { return s + (uint32_t)(p - g); }
  __device__ float2* staging(int k) const { return reinterpret_cast<float2*>(t_hi(k)); }

  __device__ bool failed() const { return *fail != 0; }

  __device__ bool wait(uint32_t bar, uint32_t& ph) {
    // a limit of 1 ns gives up at once (how a test drives this path deterministically)
    bool ok = !failed() && wait_ns > 1 && tc::mbar_wait_for(bar, ph & 1u, wait_ns);
    ok = __syncthreads_and(ok);
    ++ph;
    if (!ok && threadIdx.x == 0) *fail = 1;
    __syncthreads();
    tc::tc_fence_after();
    return ok;
  }

  // Operators: L_k tiles and the Hnh tile, with their scales.
  __device__ void load(const InstView& a) {
    n = a.n;
    K = a.K;
    const int tid = threadIdx.x;
    float2* Ls = staging(0);  // K x 64 x 64 FP32 copy of the jump operators (T region)
    for (int e = tid; e < K * 4096; e += blockDim.x) {
      const int k = e >> 12, r = e & 4095, i = r >> 6, j = r & 63;
      Ls[e] = (i < n && j < n) ? a.L[(long long)k * n * n + i * n + j] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    for (int k = 0; k < K; ++k) {
      float m = 0.f;
      for (int e = tid; e < 4096; e += blockDim.x) {
        const float2 v = Ls[k * 4096 + e];
        m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
      }
      eL[k] = stc::scale_exp(stc::block_max(m, redf));
      const float sc = ldexpf(1.f, eL[k]);
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int t = tid + 256 * u, i = t & 63, c = t >> 6;
        float re[8], im[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const float2 v = Ls[k * 4096 + i * 64 + 8 * c + q];
          re[q] = v.x;
          im[q] = v.y;
        }
        stc::put_chunk(l_hi(k), l_hi(k) + stc::kTile, i, c, re, sc);
        stc::put_chunk(l_hi(k), l_hi(k) + stc::kTile, 64 + i, c, im, sc);
      }
    }
    // Hnh = -iH - 1/2 sum_k L_k^+ L_k, FP32, staged in the X tile area
    float2* Hs = reinterpret_cast<float2*>(x_hi());
    float m = 0.f;
    for (int e = tid; e < 4096; e += blockDim.x) {
      const int i = e >> 6, j = e & 63;
      float2 acc = make_float2(0.f, 0.f);
      for (int k = 0; k < K; ++k)
        for (int q = 0; q < n; ++q) cmac(acc, cconj(Ls[k * 4096 + q * 64 + i]), Ls[k * 4096 + q * 64 + j]);
      const float2 h = (i < n && j < n) ? a.H[i * n + j] : make_float2(0.f, 0.f);
      const float2 v = make_float2(h.y - 0.5f * acc.x, -h.x - 0.5f * acc.y);
      Hs[e] = v;
      m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
    }
    eH = stc::scale_exp(stc::block_max(m, redf));  // (its barriers order the Hs writes)
    const float sc = ldexpf(1.f, eH);
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int t = tid + 256 * u, i = t & 63, c = t >> 6;
      float re[8], im[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const float2 v = Hs[i * 64 + 8 * c + q];
        re[q] = v.x;
        im[q] = v.y;
      }
      stc::put_chunk(h_hi(), h_hi() + stc::kTile, i, c, re, sc);  // (the H tile is not the X area)
      stc::put_chunk(h_hi(), h_hi() + stc::kTile, 64 + i, c, im, sc);
    }
    __syncthreads();
  }

  // One part of a product epilogue: the warp's 32 TMEM lanes of accumulator(s) at `col`
  // (and `col2` with weight f2 when f2 != 0), its 64-column half, into staging S:
  //   low lanes (rows 0-63):   half 0 -> S.re, half 1 -> S.im
  //   high lanes (rows 64-127): half 1 -> S.re with a minus sign, half 0 -> S.im
  // `init` assigns, otherwise adds.
  __device__ void epi_part(uint32_t col, float f, uint32_t col2, float f2, float2* S, bool low, bool init) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int q = warp & 3, half = warp >> 2;
    const int i = 32 * q + lane - (low ? 0 : 64);
    const bool to_re = low ? half == 0 : half == 1;
    const float sg = (low || !to_re) ? 1.f : -1.f;
    float* base = reinterpret_cast<float*>(S);
#pragma unroll 1
    for (int cc = 0; cc < 4; ++cc) {
      const uint32_t c0 = (uint32_t)(half * 64 + 16 * cc);
      const uint32_t ta = tmem + ((uint32_t)(32 * q) << 16);
      float v[16];
      tc::tmem_ld16(ta + col + c0, v);
      if (f2 != 0.f) {
        float w[16];
        tc::tmem_ld16(ta + col2 + c0, w);
        tc::tmem_ld_wait();
#pragma unroll
        for (int c = 0; c < 16; ++c) v[c] = v[c] * f + w[c] * f2;
      } else {
        tc::tmem_ld_wait();
#pragma unroll
        for (int c = 0; c < 16; ++c) v[c] *= f;
      }
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        float* p = base + 2 * stc::sidx(i, 16 * cc + c) + (to_re ? 0 : 1);
        *p = init ? sg * v[c] : *p + sg * v[c];
      }
    }
  }

  template <class F>
  __device__ void rhs(F x_of, float2* also, float2* out, double /*t: constant operators*/) {
    const int tid = threadIdx.x, warp = tid >> 5;
    const int q = warp & 3;
    constexpr uint32_t idesc = tc::instr_desc(0u, 128, 128);  // FP16 x FP16 -> FP32
    // ---- stage input X: two (column j, 8-row chunk c) tasks per thread -------------
    float xr[2][8], xi[2][8];
    float mx = 0.f;
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int t = tid + 256 * u, j = t & 63, c = t >> 6;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int e = (8 * c + r) * 64 + j;
        const float2 x = x_of(e);
        if (also) also[e] = x;
        xr[u][r] = x.x;
        xi[u][r] = x.y;
        mx = fmaxf(mx, fmaxf(fabsf(x.x), fabsf(x.y)));
      }
    }
    const int eX = stc::scale_exp(stc::block_max(mx, redf));
    {
      const float sc = ldexpf(1.f, eX);
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int t = tid + 256 * u, j = t & 63, c = t >> 6;
        // B^T rows: row j = column j of Re X, row 64 + j = column j of Im X
        stc::put_chunk(x_hi(), x_hi() + stc::kTile, j, c, xr[u], sc);
        stc::put_chunk(x_hi(), x_hi() + stc::kTile, 64 + j, c, xi[u], sc);
      }
    }
    tc::fence_proxy_async_smem();
    __syncthreads();
    if (tid == 0 && !failed()) {
      tc::tc_fence_after();
      for (int k = 0; k < K; ++k)
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
          stc::mma3(tmem + stc::kColD1 + 128u * k, sa(l_hi(k)) + 32u * kk, sa(x_hi()) + 32u * kk, idesc,
                    kk > 0 ? 1u : 0u);
      if (K > 0) tc::mma_commit(bar1);
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)
        stc::mma3(tmem + stc::kColA, sa(h_hi()) + 32u * kk, sa(x_hi()) + 32u * kk, idesc, kk > 0 ? 1u : 0u);
      if (K == 0) tc::mma_commit(bar2);
    }

    int eB = 0;
    if (K > 0) {
      // ---- T_k = L_k X: accumulators -> FP32 staging (in T_k's own tile area) -----
      wait(bar1, ph1);
      const float fT0 = ldexpf(1.f, -(eL[0] + eX));
      const float fT1 = K > 1 ? ldexpf(1.f, -(eL[1] + eX)) : 0.f;
      if (K == 2) {
        // both halves of the warps busy: jump 0 from the low lanes, jump 1 from the high
        if (q < 2) epi_part(stc::kColD1, fT0, 0, 0.f, staging(0), true, true);
        else epi_part(stc::kColD1 + 128, fT1, 0, 0.f, staging(1), false, true);
        __syncthreads();
        if (q < 2) epi_part(stc::kColD1 + 128, fT1, 0, 0.f, staging(1), true, false);
        else epi_part(stc::kColD1, fT0, 0, 0.f, staging(0), false, false);
      } else {
        if (q < 2) epi_part(stc::kColD1, fT0, 0, 0.f, staging(0), true, true);
        __syncthreads();
        if (q >= 2) epi_part(stc::kColD1, fT0, 0, 0.f, staging(0), false, false);
      }
      tc::tc_fence_before();
      __syncthreads();
      // ---- B operand of L_k T_k^+: rows j = 1/2 Re T_k row j, rows 64 + j = -1/2 Im T_k
      float tr[2][2][8], ti[2][2][8];
      float p = 0.f;
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        if (k >= K) break;
        const float2* S = staging(k);
        const float w = ldexpf(0.5f, -eL[k]);  // max |1/2 T_k| / s_Lk is what must fit
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int t = tid + 256 * u, i = t & 63, c = t >> 6;
#pragma unroll
          for (int r = 0; r < 8; ++r) {
            const float2 v = S[stc::sidx(i, 8 * c + r)];
            tr[k][u][r] = 0.5f * v.x;
            ti[k][u][r] = -0.5f * v.y;
            p = fmaxf(p, w * fmaxf(fabsf(v.x), fabsf(v.y)));
          }
        }
      }
      eB = stc::scale_exp(stc::block_max(p, redf));  // its barriers end every staging read
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        if (k >= K) break;
        const float sc = ldexpf(1.f, eB - eL[k]);  // s_Tk = s_B / s_Lk
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int t = tid + 256 * u, i = t & 63, c = t >> 6;
          stc::put_chunk(t_hi(k), t_hi(k) + stc::kTile, i, c, tr[k][u], sc);
          stc::put_chunk(t_hi(k), t_hi(k) + stc::kTile, 64 + i, c, ti[k][u], sc);
        }
      }
      tc::fence_proxy_async_smem();
      __syncthreads();
      if (tid == 0 && !failed()) {
        tc::tc_fence_after();
        for (int k = 0; k < K; ++k)
#pragma unroll
          for (int kk = 0; kk < 4; ++kk)
            stc::mma3(tmem + stc::kColB, sa(l_hi(k)) + 32u * kk, sa(t_hi(k)) + 32u * kk, idesc,
                      (k > 0 || kk > 0) ? 1u : 0u);
        tc::mma_commit(bar2);
      }
    }

    // ---- tmp = Hnh X + 1/2 sum_k L_k T_k^+ -> staging, then out = tmp + tmp^+ ---------
    const bool ok = wait(bar2, ph2);
    const float fA = ldexpf(1.f, -(eH + eX));
    const float fB = K > 0 ? ldexpf(1.f, -eB) : 0.f;
    float2* S = staging(0);
    if (q < 2) epi_part(stc::kColA, fA, stc::kColB, fB, S, true, true);
    __syncthreads();
    if (q >= 2) epi_part(stc::kColA, fA, stc::kColB, fB, S, false, false);
    tc::tc_fence_before();
    __syncthreads();
    const float bad = ok ? 0.f : __int_as_float(0x7fc00000);
    for (int e = tid; e < 4096; e += blockDim.x) {
      const int i = e >> 6, j = e & 63;
      const float2 a = S[stc::sidx(i, j)], b = S[stc::sidx(j, i)];
      out[e] = make_float2(a.x + b.x + bad, a.y - b.y + bad);
    }
    __syncthreads();
  }
};

// After a wait has run out, MMAs issued before it may still be in flight: commit them to
// a fresh barrier and wait for them (the default limit) before the tensor memory they write
// is freed.
__device__ void drain_after_failure(uint64_t* bar_exit, int failed) {
  if (failed && threadIdx.x == 0) {
    const uint32_t b = tc::smem_u32(bar_exit);
    tc::mma_commit(b);
    tc::mbar_wait_for(b, 0, tc::kWaitLimitNs);
  }
}

__global__ void __launch_bounds__(kSmallThreads, 1) mesolve_small_tc_kernel(DenseSmallArgs a,
                                                                            unsigned long long wait_ns) {
  extern __shared__ uint8_t stc_dsm[];
  __shared__ double red[40];
  __shared__ float redf[16];
  __shared__ Ctrl ctl;
  __shared__ uint64_t bars[3];
  __shared__ uint32_t tmem_sh;
  __shared__ int fail_sh;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) {
    tc::tmem_alloc(tc::smem_u32(&tmem_sh), stc::kTmemCols);
    tc::tmem_relinquish();
    if (lane == 0) {
      tc::mbar_init(tc::smem_u32(&bars[0]), 1);
      tc::mbar_init(tc::smem_u32(&bars[1]), 1);
      tc::mbar_init(tc::smem_u32(&bars[2]), 1);
      tc::fence_mbar_init();
      fail_sh = 0;
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t raw = tc::smem_u32(stc_dsm);
  const uint32_t pad = ((raw + 1023u) & ~1023u) - raw;
  TcEngine eng;
  eng.g = stc_dsm + pad;
  eng.s = raw + pad;
  eng.tmem = tmem_sh;
  eng.bar1 = tc::smem_u32(&bars[0]);
  eng.bar2 = tc::smem_u32(&bars[1]);
  eng.ph1 = eng.ph2 = 0;
  eng.n = a.n;
  eng.K = a.K;
  eng.redf = redf;
  eng.fail = &fail_sh;
  eng.wait_ns = wait_ns;
  float2* slot = a.slots + (size_t)blockIdx.x * kSlotMats * 4096;
  for (;;) {
    if (threadIdx.x == 0) ctl.inst = (long long)atomicAdd(a.counter, 1u);
    __syncthreads();
    const long long pos = ctl.inst;
    if (pos >= a.batch || fail_sh) break;
    const long long inst = a.order ? (long long)a.order[pos] : pos;
    if (inst < 0 || inst >= a.batch) {
      __syncthreads();
      continue;
    }
    const InstView v = view_of(a, inst);
    solve_one<64>(eng, v, a.o, slot, red, ctl);
    __syncthreads();
  }
  drain_after_failure(&bars[2], fail_sh);
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    __syncwarp();
    tc::tmem_dealloc(eng.tmem, stc::kTmemCols);
  }
}

// One right-hand side per instance (no RK loop), for parity tests: out is [batch, n, n].
__global__ void __launch_bounds__(kSmallThreads, 1) rhs_small_tc_kernel(DenseSmallArgs a, const float2* rho,
                                                                        float2* out) {
  extern __shared__ uint8_t stc_dsm[];
  __shared__ float redf[16];
  __shared__ uint64_t bars[2];
  __shared__ uint32_t tmem_sh;
  __shared__ int fail_sh;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp == 0) {
    tc::tmem_alloc(tc::smem_u32(&tmem_sh), stc::kTmemCols);
    tc::tmem_relinquish();
    if (lane == 0) {
      tc::mbar_init(tc::smem_u32(&bars[0]), 1);
      tc::mbar_init(tc::smem_u32(&bars[1]), 1);
      tc::fence_mbar_init();
      fail_sh = 0;
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t raw = tc::smem_u32(stc_dsm);
  const uint32_t pad = ((raw + 1023u) & ~1023u) - raw;
  TcEngine eng;
  eng.g = stc_dsm + pad;
  eng.s = raw + pad;
  eng.tmem = tmem_sh;
  eng.bar1 = tc::smem_u32(&bars[0]);
  eng.bar2 = tc::smem_u32(&bars[1]);
  eng.ph1 = eng.ph2 = 0;
  eng.redf = redf;
  eng.fail = &fail_sh;
  eng.wait_ns = tc::kWaitLimitNs;
  const long long b = blockIdx.x;
  const int n = a.n;
  InstView v{};
  v.n = n;
  v.K = a.K;
  v.H = a.H + (a.Hidx ? a.Hidx[b] : b) * (long long)n * n;
  v.L = a.L + (a.Lidx ? a.Lidx[b] : b) * (long long)a.K * n * n;
  eng.load(v);
  float2* o = out + b * (long long)n * n;
  const float2* r = rho + b * (long long)n * n;
  // the engine writes a padded 64 x 64 result: into global scratch, then the n x n block out
  float2* full = a.slots + b * 4096;
  eng.rhs([&](int e) {
            const int i = e >> 6, j = e & 63;
            return (i < n && j < n) ? r[i * n + j] : make_float2(0.f, 0.f);
          },
          nullptr, full, 0.0);
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) o[e] = full[(e / n) * 64 + e % n];
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    __syncwarp();
    tc::tmem_dealloc(eng.tmem, stc::kTmemCols);
  }
}

// Limit of the tensor-core kernels' mbarrier waits (dqb_set_tc_wait_limit_ns).
std::atomic<unsigned long long> g_wait_limit_ns{tc::kWaitLimitNs};
unsigned long long tc_wait_limit_ns() { return g_wait_limit_ns.load(); }

// One mbarrier wait that nothing completes, bounded by `limit_ns`: out[0] = 1 if it gave
// up, out[1] = microseconds it waited.
__global__ void bounded_wait_probe_kernel(unsigned long long limit_ns, int* out) {
  __shared__ uint64_t bar;
  if (threadIdx.x != 0) return;
  const uint32_t b = tc::smem_u32(&bar);
  tc::mbar_init(b, 1);
  tc::fence_mbar_init();
  const unsigned long long t0 = tc::globaltimer_ns();
  const bool done = tc::mbar_wait_for(b, 0, limit_ns);
  out[0] = done ? 0 : 1;
  out[1] = (int)((tc::globaltimer_ns() - t0) / 1000ull);
}

static void raise_smem_limit_once() {
  static std::once_flag once;
  std::call_once(once, [] {
    cudaFuncSetAttribute(mesolve_small_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, stc::smem_bytes(2));
    cudaFuncSetAttribute(rhs_small_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, stc::smem_bytes(2));
    prefer_max_shared(mesolve_small_tc_kernel);
    prefer_max_shared(rhs_small_tc_kernel);
  });
}

// Does the tensor-core kernel apply to this problem?  (32 < n <= 64, at most two jump
// operators, hermitian form.)
bool small_tc_applies(int n, int K, int form) {
  return n > 32 && n <= 64 && K >= 0 && K <= 2 && form == DQB_FORM_HERMITIAN;
}

// Launch the persistent tensor-core kernel: one CTA per SM (at most `batch`), the work
// counter at `counter` (zeroed by the caller) and the CTAs' slots at `slots`.
int small_tc_launch(const DenseSmallArgs& a, int max_grid, cudaStream_t s) {
  raise_smem_limit_once();
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  long long g = std::min<long long>(sms, a.batch);
  g = std::min<long long>(g, max_grid);
  if (g < 1) g = 1;
  mesolve_small_tc_kernel<<<(unsigned)g, kSmallThreads, stc::smem_bytes(a.K), s>>>(a, tc_wait_limit_ns());
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}

// One right-hand side per instance on the tensor cores; `scratch` holds batch x 64 x 64
// complex64.
int small_tc_rhs(const DenseSmallArgs& a, const float2* rho, float2* out, float2* scratch, cudaStream_t s) {
  raise_smem_limit_once();
  DenseSmallArgs b = a;
  b.slots = scratch;
  rhs_small_tc_kernel<<<(unsigned)a.batch, kSmallThreads, stc::smem_bytes(a.K), s>>>(b, rho, out);
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}

}  // namespace dqb

extern "C" void dqb_set_tc_wait_limit_ns(uint64_t ns) {
  dqb::g_wait_limit_ns.store(ns ? (unsigned long long)ns : dqb::tc::kWaitLimitNs);
}

extern "C" int dqb_probe_bounded_wait(uint64_t limit_ns, int32_t* result, void* stream) {
  if (!result || limit_ns > 1000000000ull) return DQB_ERR_INVALID_ARGUMENT;
  dqb::bounded_wait_probe_kernel<<<1, 32, 0, (cudaStream_t)stream>>>((unsigned long long)limit_ns, result);
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}
