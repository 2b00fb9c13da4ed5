// Persistent batched mesolve kernel for dense operators with n <= 64.
//
// One CTA solves one instance at a time and fetches the next instance from an atomic
// counter when it finishes, so instances with different step counts never wait for
// each other (the reference vmaps diffrax's while loop, which runs every lane for as
// many iterations as the slowest one: dynamiqs/integrators/apis/mesolve.py:307-336).
//
// Per CTA, shared memory holds Hnh = -iH - 1/2 sum L^+L (built once per instance), the
// jump operators L_k, the current stage input X and a product buffer T, each padded
// to a row stride of NP+1 complex so that row and column (transposed) reads are both
// bank-conflict free.  The seven RK stages, y and y1 live in a per-CTA scratch slot in
// global memory (9 * NP^2 complex64 = 288 KiB at NP = 64; 148 slots = 43 MB, resident
// in the 126 MB L2).  The products run on the FP32 pipes: 256 threads, each owning an
// (NP/16) x (NP/16) tile of the output, complex multiply-accumulate as 4 FFMA.  In the
// hermitian form the hermitian product (L_k X) L_k^+ is computed only on the tile pairs on
// and below the block diagonal (gemm_herm), which tmp + tmp^+ completes exactly.
//
// Right-hand sides (dynamiqs/integrators/core/diffrax_integrator.py:312-323):
//   hermitian: tmp = Hnh X + 1/2 sum_k (L_k X) L_k^+ ;  out = tmp + tmp^+
//   standard : out = Hnh X + X Hnh^+ + sum_k (L_k X) L_k^+
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <utility>
#include <vector>

#include "dqb_small.cuh"

namespace dqb {

bool small_tc_applies(int n, int K, int form);
int small_tc_launch(const DenseSmallArgs& a, int max_grid, cudaStream_t s);
int small_tc_rhs(const DenseSmallArgs& a, const float2* rho, float2* out, float2* scratch, cudaStream_t s);

template <int NP>
struct Small {
  static constexpr int LD = NP + 1;
  static constexpr int R = NP / 16;
  static constexpr int MAT = NP * LD;
  static constexpr int NN = NP * NP;
};

// acc[r][c] += sum_k op(A)[row][k] * op(B)[k][col], rows ty + 16 r, cols tx + 16 c.
// CA: op(A) = A^+, CB: op(B) = B^+ (both read transposed from the padded layout).
template <int NP, bool CA, bool CB>
__device__ __forceinline__ void gemm(float2 (&acc)[NP / 16][NP / 16], const float2* __restrict__ A,
                                     const float2* __restrict__ B, int kn) {
  constexpr int R = NP / 16, LD = NP + 1;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll 8
  for (int k = 0; k < kn; ++k) {
    float2 a[R], b[R];
#pragma unroll
    for (int r = 0; r < R; ++r) a[r] = CA ? cconj(A[k * LD + ty + 16 * r]) : A[(ty + 16 * r) * LD + k];
#pragma unroll
    for (int c = 0; c < R; ++c) b[c] = CB ? cconj(B[(tx + 16 * c) * LD + k]) : B[k * LD + tx + 16 * c];
    // the two FMAs of a real or imaginary part that depend on each other are R*R
    // instructions apart
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int c = 0; c < R; ++c) {
        acc[r][c].x = fmaf(a[r].x, b[c].x, acc[r][c].x);
        acc[r][c].y = fmaf(a[r].x, b[c].y, acc[r][c].y);
      }
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int c = 0; c < R; ++c) {
        acc[r][c].x = fmaf(-a[r].y, b[c].y, acc[r][c].x);
        acc[r][c].y = fmaf(a[r].y, b[c].x, acc[r][c].y);
      }
  }
}

// The hermitian product S = T L^+ (T = L X with X hermitian, so S = L X L^+ is hermitian)
// computed on the tile pairs r >= c only: acc[r][r] += S blocks on the diagonal,
// low[r (r - 1) / 2 + c] += S blocks strictly below it.  The strictly-upper blocks are
// conj(S^T) of these, so the right-hand side only needs S on and below the diagonal blocks:
// (R + 1) R / 2 of the R^2 block pairs (10 of 16 at NP = 64).
template <int NP>
__device__ __forceinline__ void gemm_herm(float2 (&acc)[NP / 16][NP / 16],
                                          float2 (&low)[(NP / 16) * (NP / 16 - 1) / 2 + 1],
                                          const float2* __restrict__ A, const float2* __restrict__ B,
                                          int kn) {
  constexpr int R = NP / 16, LD = NP + 1;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll 8
  for (int k = 0; k < kn; ++k) {
    float2 a[R], b[R];
#pragma unroll
    for (int r = 0; r < R; ++r) a[r] = A[(ty + 16 * r) * LD + k];
#pragma unroll
    for (int c = 0; c < R; ++c) b[c] = cconj(B[(tx + 16 * c) * LD + k]);
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int c = 0; c <= r; ++c) {
        float2& d = r == c ? acc[r][r] : low[r * (r - 1) / 2 + c];
        d.x = fmaf(a[r].x, b[c].x, d.x);
        d.y = fmaf(a[r].x, b[c].y, d.y);
      }
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int c = 0; c <= r; ++c) {
        float2& d = r == c ? acc[r][r] : low[r * (r - 1) / 2 + c];
        d.x = fmaf(-a[r].y, b[c].y, d.x);
        d.y = fmaf(a[r].y, b[c].x, d.y);
      }
  }
}

template <int NP>
__device__ __forceinline__ void zero_tile(float2 (&t)[NP / 16][NP / 16]) {
#pragma unroll
  for (int r = 0; r < NP / 16; ++r)
#pragma unroll
    for (int c = 0; c < NP / 16; ++c) t[r][c] = make_float2(0.f, 0.f);
}

template <int NP>
__device__ __forceinline__ void store_tile(float2* S, const float2 (&t)[NP / 16][NP / 16], float s) {
  constexpr int LD = NP + 1;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
  for (int r = 0; r < NP / 16; ++r)
#pragma unroll
    for (int c = 0; c < NP / 16; ++c)
      S[(ty + 16 * r) * LD + tx + 16 * c] = make_float2(s * t[r][c].x, s * t[r][c].y);
}

// Load an n x n row-major global matrix into a padded NP x (NP+1) shared buffer.
template <int NP>
__device__ __forceinline__ void load_padded(float2* S, const float2* __restrict__ g, int n) {
  for (int e = threadIdx.x; e < NP * NP; e += blockDim.x) {
    const int i = e / NP, j = e % NP;
    S[i * Small<NP>::LD + j] = (i < n && j < n) ? g[i * n + j] : make_float2(0.f, 0.f);
  }
}

// Build Hnh = -iH - 1/2 sum_k L_k^+ L_k in place (sH holds H on entry).
template <int NP>
__device__ void build_hnh(float2* sH, const float2* sL, int n, int K) {
  constexpr int LD = NP + 1;
  float2 acc[NP / 16][NP / 16];
  zero_tile<NP>(acc);
  for (int k = 0; k < K; ++k) gemm<NP, true, false>(acc, sL + k * Small<NP>::MAT, sL + k * Small<NP>::MAT, n);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
  for (int r = 0; r < NP / 16; ++r)
#pragma unroll
    for (int c = 0; c < NP / 16; ++c) {
      const int idx = (ty + 16 * r) * LD + tx + 16 * c;
      const float2 h = sH[idx];
      sH[idx] = make_float2(h.y - 0.5f * acc[r][c].x, -h.x - 0.5f * acc[r][c].y);
    }
}

// out[i * ldo + j] = f(X)[i][j] for i, j < nlim.  Ends without a barrier.
template <int NP>
__device__ void rhs(const float2* sH, const float2* sL, const float2* sX, float2* sT, int n, int K,
                    int form, float2* __restrict__ out, int ldo, int nlim) {
  constexpr int LD = NP + 1;
  float2 acc[NP / 16][NP / 16];
  zero_tile<NP>(acc);
  gemm<NP, false, false>(acc, sH, sX, n);
  if (form == DQB_FORM_STANDARD) gemm<NP, false, true>(acc, sX, sH, n);
  const bool hermf = form == DQB_FORM_HERMITIAN;
  constexpr int R = NP / 16, NLOW = R * (R - 1) / 2 + 1;
  float2 low[NLOW];
#pragma unroll
  for (int q = 0; q < NLOW; ++q) low[q] = make_float2(0.f, 0.f);
  for (int k = 0; k < K; ++k) {
    const float2* Lk = sL + k * Small<NP>::MAT;
    float2 t[NP / 16][NP / 16];
    zero_tile<NP>(t);
    gemm<NP, false, false>(t, Lk, sX, n);
    __syncthreads();  // readers of the previous T are done
    store_tile<NP>(sT, t, hermf ? 0.5f : 1.0f);
    __syncthreads();
    if (hermf)
      gemm_herm<NP>(acc, low, sT, Lk, n);
    else
      gemm<NP, false, true>(acc, sT, Lk, n);
  }
  if (hermf) {
    // tmp = Hnh X + 1/2 S with S's strictly-upper blocks left out and its strictly-lower
    // blocks doubled: tmp + tmp^+ is then Hnh X + (Hnh X)^+ + S, the reference's
    // hermitian form (S hermitian), from 10 of the 16 block products of T L^+
#pragma unroll
    for (int r = 1; r < R; ++r)
#pragma unroll
      for (int c = 0; c < r; ++c) {
        const float2 v = low[r * (r - 1) / 2 + c];
        acc[r][c].x = fmaf(2.f, v.x, acc[r][c].x);
        acc[r][c].y = fmaf(2.f, v.y, acc[r][c].y);
      }
  }
  __syncthreads();
  store_tile<NP>(sT, acc, 1.0f);
  __syncthreads();
  const bool herm = form == DQB_FORM_HERMITIAN;
  for (int e = threadIdx.x; e < NP * NP; e += blockDim.x) {
    const int i = e / NP, j = e % NP;
    if (i < nlim && j < nlim) {
      float2 v = sT[i * LD + j];
      if (herm) v = cadd(v, cconj(sT[j * LD + i]));
      out[i * ldo + j] = v;
    }
  }
}

// The right-hand side on CUDA cores (the engine of solve_one, dqb_small.cuh): Hnh, the
// jump operators, the stage input X and the product buffer T in padded shared memory.
// With a time-dependent H (td->M > 0) the constant part Hnh0 = -iH0 - 1/2 sum L^+L is kept
// in one more padded matrix, and every right-hand side first forms
// Hnh(t) = Hnh0 - i sum_m c_m(t) H_m in sH from the terms' operators in global memory.
template <int NP, int FEAT>
struct SimtEngine {
  static constexpr bool kJumps = (FEAT & 1) != 0, kTape = (FEAT & 2) != 0;
  float2 *sH, *sX, *sT, *sL;
  int n, K, form;
  const TdArgs* td;
  float2* sH0;
  long long inst;

  __device__ void load(const InstView& a) {
    n = a.n;
    K = a.K;
    inst = a.inst;
    load_padded<NP>(sH, a.H, n);
    for (int k = 0; k < K; ++k) load_padded<NP>(sL + k * Small<NP>::MAT, a.L + (long long)k * n * n, n);
    __syncthreads();
    build_hnh<NP>(sH, sL, n, K);
    __syncthreads();
    if constexpr (kJumps) {
      for (int e = threadIdx.x; e < Small<NP>::MAT; e += blockDim.x) sH0[e] = sH[e];
      __syncthreads();
    }
  }

  template <class F>
  __device__ void rhs(F x_of, float2* also, float2* out, double t) {
    constexpr int LD = NP + 1;
    const int M = kJumps ? td->M : 0;
    float2 c[DQB_TD_MAX_TERMS];
#pragma unroll
    for (int m = 0; m < DQB_TD_MAX_TERMS; ++m) {
      c[m] = make_float2(0.f, 0.f);
      if (kJumps && m < M) {
        const double2 v = td_coef(td->term[m], inst, t);
        c[m] = make_float2((float)v.x, (float)v.y);
      }
    }
#pragma unroll 4
    for (int e = threadIdx.x; e < NP * NP; e += blockDim.x) {
      const int i = e / NP, j = e % NP;
      const float2 x = x_of(e);
      sX[i * LD + j] = x;
      if (also) also[e] = x;
      if (kJumps) {
        float2 h = sH0[i * LD + j];
        if (i < n && j < n) {
          float2 acc = make_float2(0.f, 0.f);  // sum_m c_m(t) H_m[i][j]
#pragma unroll
          for (int m = 0; m < DQB_TD_MAX_TERMS; ++m)
            if (m < M) cmac(acc, c[m], td->ops[((long long)m * n + i) * n + j]);
          h = make_float2(h.x + acc.y, h.y - acc.x);  // - i acc
        }
        sH[i * LD + j] = h;
      }
    }
    __syncthreads();
    dqb::rhs<NP>(sH, sL, sX, sT, n, K, form, out, NP, NP);
    __syncthreads();
  }

  __device__ bool failed() const { return false; }
};

// FEAT: 0 = constant operators, 1 = time-dependent H (discontinuity times), 2 = gradient tape.
template <int NP, int FEAT = 0>
__global__ void __launch_bounds__(kSmallThreads, NP == 64 ? 1 : (NP == 32 ? 3 : 4)) mesolve_small_kernel(DenseSmallArgs a) {
  extern __shared__ float4 smem_raw[];
  __shared__ double red[40];
  __shared__ Ctrl ctl;
  float2* sH = reinterpret_cast<float2*>(smem_raw);
  float2* sX = sH + Small<NP>::MAT;
  float2* sT = sX + Small<NP>::MAT;
  float2* sL = sT + Small<NP>::MAT;
  float2* slot = a.slots + (size_t)blockIdx.x * kSlotMats * Small<NP>::NN;
  for (;;) {
    if (threadIdx.x == 0) ctl.inst = (long long)atomicAdd(a.counter, 1u);
    __syncthreads();
    const long long pos = ctl.inst;
    if (pos >= a.batch) break;
    const long long inst = a.order ? (long long)a.order[pos] : pos;
    if (inst < 0 || inst >= a.batch) {  // not a valid instance: skip it
      __syncthreads();                    // every thread has read ctl.inst
      continue;
    }
    const InstView v = view_of(a, inst);
    SimtEngine<NP, FEAT> eng{sH, sX, sT, sL, a.n, a.K, a.o.form, &a.td, sL + a.K * Small<NP>::MAT, inst};
    solve_one<NP>(eng, v, a.o, slot, red, ctl);
    __syncthreads();
  }
}

// One right-hand side per instance (no RK loop); out is [batch, n, n].
template <int NP>
__global__ void __launch_bounds__(kSmallThreads) rhs_small_kernel(DenseSmallArgs a, int form, const float2* rho,
                                                                  float2* out) {
  extern __shared__ float4 smem_raw[];
  float2* sH = reinterpret_cast<float2*>(smem_raw);
  float2* sX = sH + Small<NP>::MAT;
  float2* sT = sX + Small<NP>::MAT;
  float2* sL = sT + Small<NP>::MAT;
  const long long b = blockIdx.x;
  const int n = a.n, K = a.K;
  const long long hi = a.Hidx ? a.Hidx[b] : b;
  const long long li = a.Lidx ? a.Lidx[b] : b;
  load_padded<NP>(sH, a.H + hi * n * n, n);
  for (int k = 0; k < K; ++k) load_padded<NP>(sL + k * Small<NP>::MAT, a.L + (li * K + k) * n * n, n);
  load_padded<NP>(sX, rho + b * n * n, n);
  __syncthreads();
  build_hnh<NP>(sH, sL, n, K);
  __syncthreads();
  rhs<NP>(sH, sL, sX, sT, n, K, form, out + b * n * n, n, n);
}

// ------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------
template <int NP>
static size_t small_smem_bytes(int K) {
  return (size_t)(3 + K) * Small<NP>::MAT * sizeof(float2);
}

static int pick_np(int n) { return n <= 16 ? 16 : (n <= 32 ? 32 : (n <= 64 ? 64 : 0)); }

static size_t max_optin_smem() {
  int dev = 0, v = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  return v > 0 ? (size_t)v : (size_t)232448;
}

static size_t smem_for(int NP, int K) {
  switch (NP) {
    case 16: return small_smem_bytes<16>(K);
    case 32: return small_smem_bytes<32>(K);
    default: return small_smem_bytes<64>(K);
  }
}

// Occupancy of a persistent kernel for a dynamic shared-memory size.  The kernel's
// dynamic shared-memory limit is raised once, to the device maximum, and never lowered:
// the attribute is per-function state shared by every host thread, so per-call values
// could race with another thread's launch.  Results are cached per (kernel, smem).
template <class Kern>
static int resident_ctas(Kern kern, size_t smem) {
  static std::mutex mu;
  static std::vector<std::pair<const void*, size_t>> keys;  // (kernel, smem)
  static std::vector<int> values;
  static std::vector<const void*> raised;
  const void* fn = (const void*)kern;
  std::lock_guard<std::mutex> lock(mu);
  if (std::find(raised.begin(), raised.end(), fn) == raised.end()) {
    cudaFuncAttributes fa;
    cudaFuncGetAttributes(&fa, kern);
    const int limit = (int)max_optin_smem() - (int)fa.sharedSizeBytes;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, limit);
    prefer_max_shared(kern);
    raised.push_back(fn);
  }
  for (size_t i = 0; i < keys.size(); ++i)
    if (keys[i].first == fn && keys[i].second == smem) return values[i];
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kSmallThreads, smem);
  keys.emplace_back(fn, smem);
  values.push_back(per_sm);
  return per_sm;
}

static int sm_count() {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

// Resident CTAs for (NP, K) of the kernel variant FEAT on the current device (raising
// that variant's shared-memory limit); 0 if the shared memory does not fit.
template <int NP, int FEAT = 0>
static int small_grid(int K, long long batch) {
  const size_t smem = small_smem_bytes<NP>(K);
  if (smem + 2048 > max_optin_smem()) return 0;
  const int per_sm = resident_ctas(mesolve_small_kernel<NP, FEAT>, smem);
  if (per_sm < 1) return 0;
  long long g = (long long)per_sm * sm_count();
  if (g > batch) g = batch;
  return (int)std::max<long long>(g, 1);
}

template <int FEAT = 0>
static int grid_for(int NP, int K, long long batch) {
  switch (NP) {
    case 16: return small_grid<16, FEAT>(K, batch);
    case 32: return small_grid<32, FEAT>(K, batch);
    default: return small_grid<64, FEAT>(K, batch);
  }
}

}  // namespace dqb

using namespace dqb;

extern "C" int32_t dqb_dense_small_max_n(int32_t n_jumps) {
  if (n_jumps < 0) return 0;
  const size_t cap = max_optin_smem() - 2048;
  if (smem_for(64, n_jumps) <= cap) return 64;
  if (smem_for(32, n_jumps) <= cap) return 32;
  if (smem_for(16, n_jumps) <= cap) return 16;
  return 0;
}

extern "C" size_t dqb_mesolve_dense_workspace_size(int32_t n, int32_t n_jumps, int64_t batch) {
  const int NP = pick_np(n);
  if (NP == 0 || batch <= 0) return 0;
  const int g = grid_for(NP, n_jumps, batch);
  if (g <= 0) return 0;
  return 256 + (size_t)g * kSlotMats * NP * NP * sizeof(float2);
}

static int validate_dense(const dqb_dense_problem* p, const dqb_ode_options* o) {
  if (!p || !o) return DQB_ERR_INVALID_ARGUMENT;
  if (p->n < 1 || p->n_jumps < 0 || p->n_exp < 0 || p->n_tsave < 1 || p->batch < 0) return DQB_ERR_INVALID_ARGUMENT;
  if (p->batch >= (int64_t)0x7fffffff) return DQB_ERR_INVALID_ARGUMENT;
  if (!p->H || (p->n_jumps > 0 && !p->L) || !p->rho0 || !p->tsave) return DQB_ERR_INVALID_ARGUMENT;
  if (p->n_exp > 0 && !p->E) return DQB_ERR_INVALID_ARGUMENT;
  if (o->method != DQB_METHOD_TSIT5 && o->method != DQB_METHOD_DOPRI5) return DQB_ERR_INVALID_ARGUMENT;
  if (o->form != DQB_FORM_HERMITIAN && o->form != DQB_FORM_STANDARD) return DQB_ERR_INVALID_ARGUMENT;
  if (!(o->rtol >= 0) || !(o->atol >= 0) || o->max_steps < 0) return DQB_ERR_INVALID_ARGUMENT;
  return DQB_OK;
}

static DenseSmallArgs make_args(const dqb_dense_problem* p, const dqb_ode_options* o, const dqb_outputs* out) {
  DenseSmallArgs a;
  a.n = p->n;
  a.K = p->n_jumps;
  a.nE = p->n_exp;
  a.ntsave = p->n_tsave;
  a.batch = p->batch;
  a.H = (const float2*)p->H;
  a.L = (const float2*)p->L;
  a.rho0 = (const float2*)p->rho0;
  a.E = (const float2*)p->E;
  a.rho0_is_ket = p->rho0_is_ket;
  a.tsave = p->tsave;
  a.Hidx = p->H_index;
  a.Lidx = p->L_index;
  a.ridx = p->rho0_index;
  a.order = p->start_order;
  a.states = out ? (float2*)out->states : nullptr;
  a.expects = out ? (float2*)out->expects : nullptr;
  a.infos = out ? out->infos : nullptr;
  a.status = out ? out->status : nullptr;
  a.slots = nullptr;
  a.counter = nullptr;
  if (o) a.o = make_ctrl(*o);
  std::memset(&a.td, 0, sizeof(a.td));
  a.tape_t = a.tape_h = nullptr;
  a.tape_y = nullptr;
  a.tape_cap = 0;
  return a;
}

extern "C" int dqb_mesolve_dense(const dqb_dense_problem* p, const dqb_ode_options* o, const dqb_outputs* out,
                                 void* workspace, size_t workspace_bytes, void* stream) {
  int rc = validate_dense(p, o);
  if (rc) return rc;
  if (!out || !out->states || !out->infos || !out->status || (p->n_exp > 0 && !out->expects))
    return DQB_ERR_INVALID_ARGUMENT;
  if (p->batch == 0) return DQB_OK;
  const int NP = pick_np(p->n);
  if (NP == 0 || dqb_dense_small_max_n(p->n_jumps) < NP) return DQB_ERR_UNSUPPORTED;
  const size_t need = dqb_mesolve_dense_workspace_size(p->n, p->n_jumps, p->batch);
  if (need == 0) return DQB_ERR_UNSUPPORTED;
  if (!workspace || workspace_bytes < need) return DQB_ERR_WORKSPACE_TOO_SMALL;
  const int grid = grid_for(NP, p->n_jumps, p->batch);
  cudaStream_t s = (cudaStream_t)stream;
  DenseSmallArgs a = make_args(p, o, out);
  a.counter = (unsigned int*)workspace;
  a.slots = (float2*)((char*)workspace + 256);
  zero_words_kernel<<<1, 64, 0, s>>>((unsigned int*)workspace, 64);
  if (o->precision == DQB_PREC_F16X3 && small_tc_applies(p->n, p->n_jumps, o->form))
    return small_tc_launch(a, grid, s);
  const size_t smem = smem_for(NP, p->n_jumps);
  switch (NP) {
    case 16: mesolve_small_kernel<16><<<grid, kSmallThreads, smem, s>>>(a); break;
    case 32: mesolve_small_kernel<32><<<grid, kSmallThreads, smem, s>>>(a); break;
    default: mesolve_small_kernel<64><<<grid, kSmallThreads, smem, s>>>(a); break;
  }
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}

extern "C" int dqb_mesolve_dense_td(const dqb_dense_problem* p, const dqb_td_hamiltonian* td,
                                    const dqb_ode_options* o, const dqb_outputs* out, void* workspace,
                                    size_t workspace_bytes, void* stream) {
  int rc = validate_dense(p, o);
  if (rc) return rc;
  if (!out || !out->states || !out->infos || !out->status || (p->n_exp > 0 && !out->expects))
    return DQB_ERR_INVALID_ARGUMENT;
  if (!td || td->n_terms < 0 || td->n_terms > DQB_TD_MAX_TERMS || td->n_jump_ts < 0) return DQB_ERR_INVALID_ARGUMENT;
  if (td->jump_terms) return DQB_ERR_UNSUPPORTED;  // time-dependent jump operators: the DIA path
  if ((td->n_terms > 0 && (!td->ops || !td->terms)) || (td->n_jump_ts > 0 && !td->jump_ts))
    return DQB_ERR_INVALID_ARGUMENT;
  for (int m = 0; m < td->n_terms; ++m) {
    const dqb_td_term& T = td->terms[m];
    if (T.kind == DQB_TD_PWC) {
      if (T.n_times < 2 || !T.times || !T.values) return DQB_ERR_INVALID_ARGUMENT;
    } else if (T.kind != DQB_TD_WAVE) {
      return DQB_ERR_INVALID_ARGUMENT;
    }
  }
  if (p->batch == 0) return DQB_OK;
  const int NP = pick_np(p->n);
  const int Keff = p->n_jumps + 1;  // one more shared-memory matrix: the constant Hnh0
  if (NP == 0 || dqb_dense_small_max_n(Keff) < NP) return DQB_ERR_UNSUPPORTED;
  const size_t need = dqb_mesolve_dense_workspace_size(p->n, Keff, p->batch);
  if (need == 0) return DQB_ERR_UNSUPPORTED;
  if (!workspace || workspace_bytes < need) return DQB_ERR_WORKSPACE_TOO_SMALL;
  const int grid = grid_for<1>(NP, Keff, p->batch);
  cudaStream_t s = (cudaStream_t)stream;
  DenseSmallArgs a = make_args(p, o, out);
  a.counter = (unsigned int*)workspace;
  a.slots = (float2*)((char*)workspace + 256);
  a.td.M = td->n_terms;
  a.td.ops = (const float2*)td->ops;
  for (int m = 0; m < td->n_terms; ++m) {
    const dqb_td_term& T = td->terms[m];
    TdTerm& d = a.td.term[m];
    d.kind = T.kind;
    d.n_times = T.n_times;
    d.times = T.times;
    d.values = (const double2*)T.values;
    d.vidx = T.value_index;
    d.amp_re = T.amp_re;
    d.amp_im = T.amp_im;
    d.omega = T.omega;
    d.phase = T.phase;
    d.t_center = T.t_center;
    d.sigma = T.sigma;
    d.t_start = T.t_start;
    d.t_end = T.t_end;
  }
  a.td.n_jump = td->n_jump_ts;
  a.td.jump_ts = td->jump_ts;
  zero_words_kernel<<<1, 64, 0, s>>>((unsigned int*)workspace, 64);
  const size_t smem = smem_for(NP, Keff);
  switch (NP) {
    case 16: mesolve_small_kernel<16, 1><<<grid, kSmallThreads, smem, s>>>(a); break;
    case 32: mesolve_small_kernel<32, 1><<<grid, kSmallThreads, smem, s>>>(a); break;
    default: mesolve_small_kernel<64, 1><<<grid, kSmallThreads, smem, s>>>(a); break;
  }
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}

extern "C" int dqb_lindblad_rhs_dense(const dqb_dense_problem* p, int32_t form, const void* rho, void* outp,
                                      void* stream) {
  if (!p || !rho || !outp) return DQB_ERR_INVALID_ARGUMENT;
  if (p->n < 1 || p->n_jumps < 0 || p->batch < 0 || !p->H || (p->n_jumps > 0 && !p->L))
    return DQB_ERR_INVALID_ARGUMENT;
  if (form != DQB_FORM_HERMITIAN && form != DQB_FORM_STANDARD) return DQB_ERR_INVALID_ARGUMENT;
  if (p->batch == 0) return DQB_OK;
  const int NP = pick_np(p->n);
  if (NP == 0 || dqb_dense_small_max_n(p->n_jumps) < NP) return DQB_ERR_UNSUPPORTED;
  DenseSmallArgs a = make_args(p, nullptr, nullptr);
  const size_t smem = smem_for(NP, p->n_jumps);
  cudaStream_t s = (cudaStream_t)stream;
  const unsigned grid = (unsigned)p->batch;
  switch (NP) {
    case 16:
      resident_ctas(rhs_small_kernel<16>, smem);
      rhs_small_kernel<16><<<grid, kSmallThreads, smem, s>>>(a, form, (const float2*)rho, (float2*)outp);
      break;
    case 32:
      resident_ctas(rhs_small_kernel<32>, smem);
      rhs_small_kernel<32><<<grid, kSmallThreads, smem, s>>>(a, form, (const float2*)rho, (float2*)outp);
      break;
    default:
      resident_ctas(rhs_small_kernel<64>, smem);
      rhs_small_kernel<64><<<grid, kSmallThreads, smem, s>>>(a, form, (const float2*)rho, (float2*)outp);
      break;
  }
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}

extern "C" int dqb_lindblad_rhs_dense_prec(const dqb_dense_problem* p, int32_t form, int32_t precision,
                                           const void* rho, void* outp, void* workspace, size_t workspace_bytes,
                                           void* stream) {
  if (precision == DQB_PREC_FP32) return dqb_lindblad_rhs_dense(p, form, rho, outp, stream);
  if (precision != DQB_PREC_F16X3) return DQB_ERR_INVALID_ARGUMENT;
  if (!p || !rho || !outp) return DQB_ERR_INVALID_ARGUMENT;
  if (p->n < 1 || p->n_jumps < 0 || p->batch < 0 || !p->H || (p->n_jumps > 0 && !p->L))
    return DQB_ERR_INVALID_ARGUMENT;
  if (form != DQB_FORM_HERMITIAN && form != DQB_FORM_STANDARD) return DQB_ERR_INVALID_ARGUMENT;
  if (!small_tc_applies(p->n, p->n_jumps, form)) return DQB_ERR_UNSUPPORTED;
  if (p->batch == 0) return DQB_OK;
  if (p->batch >= (int64_t)0x7fffffff) return DQB_ERR_INVALID_ARGUMENT;
  if (!workspace || workspace_bytes < (size_t)p->batch * 32768) return DQB_ERR_WORKSPACE_TOO_SMALL;
  DenseSmallArgs a = make_args(p, nullptr, nullptr);
  return small_tc_rhs(a, (const float2*)rho, (float2*)outp, (float2*)workspace, (cudaStream_t)stream);
}

namespace dqb {

// ------------------------------------------------------------------------------------
// gradients: the discrete adjoint of the recorded Runge-Kutta steps
// ------------------------------------------------------------------------------------
//
// Reverse-mode differentiation of the whole solve -- what JAX does through diffrax for the
// reference's Direct / BackwardCheckpointed gradients (dynamiqs/gradient.py:10-110,
// diffrax_integrator.py:88-99): the step sizes are constants (the controller is not
// differentiated), and every accepted step is differentiated exactly.  For a linear
// right-hand side k = S(X) = Hnh X + X Hnh^+ + sum_k L_k X L_k^+ the reverse pass of one
// step, given the cotangent lambda of its end state and the cotangents G_s of the saves it
// made (y_s = y + h sum_j w_j(theta_s) k_j), is
//   kappa_j = h b_j lambda + sum_s h w_j(theta_s) G_s,
//   for j = 7 .. 1: xi_j = S^+(kappa_j),  kappa_l += h a_jl xi_j (l < j),
//   lambda <- lambda + sum_s G_s + sum_j xi_j,
// with S^+(Z) = Hnh^+ Z + Z Hnh + sum_k L_k^+ Z L_k (the same product structure with Hnh
// and L_k replaced by their adjoints, applied in place in shared memory), and the
// operator gradients accumulate, with Zs = kappa_j + kappa_j^+ and X_j hermitian,
//   dH += i Zs X_j,   dL_k += Zs L_k X_j - 1/2 L_k (X_j Zs + Zs X_j)
// (complex gradients in the convention dLoss = Re tr(G^+ dA)).  The stage inputs X_j are
// recomputed from the recorded start state of each step.

constexpr int kAdjMats = 23;  // X_1..7, k_1..6 (+1 spare), kappa_1..7, xi, lambda

struct AdjArgs {
  DenseSmallArgs p;              // operators, indices, E, tsave, method, form, t0
  const int* nacc;               // [batch] accepted steps of each instance (forward infos)
  const float2* gstates;         // [batch, nsave, n, n] cotangents of the saved states, or null
  const float2* gexpects;        // [batch, nE, ntsave] cotangents of the expectation values, or null
  float2* grad_rho0;             // [batch, n, n] (or [batch, n] for kets)
  float2* grad_H;                // [batch, n, n]
  float2* grad_L;                // [batch, K, n, n]
};

// Conjugate-transpose a padded NP x NP matrix in shared memory, in place.
template <int NP>
__device__ void dagger_inplace(float2* S) {
  constexpr int LD = NP + 1;
  for (int e = threadIdx.x; e < NP * NP; e += blockDim.x) {
    const int i = e / NP, j = e % NP;
    if (i < j) {
      const float2 a = S[i * LD + j], b = S[j * LD + i];
      S[i * LD + j] = cconj(b);
      S[j * LD + i] = cconj(a);
    } else if (i == j) {
      S[i * LD + i] = cconj(S[i * LD + i]);
    }
  }
}

// Global NP x NP matrix into a padded shared buffer (all NP^2 entries).
template <int NP>
__device__ __forceinline__ void to_smem(float2* S, const float2* __restrict__ g) {
  for (int e = threadIdx.x; e < NP * NP; e += blockDim.x) S[(e / NP) * (NP + 1) + e % NP] = g[e];
}

// g[e] (+)= s * tile (the 4x4 register tile layout of gemm) for the n x n block.
template <int NP>
__device__ __forceinline__ void add_tile(float2* g, const float2 (&t)[NP / 16][NP / 16], float2 s, int n) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
  for (int r = 0; r < NP / 16; ++r)
#pragma unroll
    for (int c = 0; c < NP / 16; ++c) {
      const int i = ty + 16 * r, j = tx + 16 * c;
      if (i < n && j < n) {
        float2& d = g[i * n + j];
        d = cadd(d, cmul(s, t[r][c]));
      }
    }
}

template <int NP>
__global__ void __launch_bounds__(kSmallThreads, 1) mesolve_adjoint_kernel(AdjArgs A) {
  extern __shared__ float4 smem_raw[];
  __shared__ long long inst_sh;
  constexpr int NN = NP * NP, LD = NP + 1, MAT = Small<NP>::MAT;
  const DenseSmallArgs& a = A.p;
  const int tid = threadIdx.x, n = a.n, K = a.K;
  float2* sH = reinterpret_cast<float2*>(smem_raw);
  float2* sX = sH + MAT;
  float2* sT = sX + MAT;
  float2* sL = sT + MAT;
  float2* sU = sL + K * MAT;  // one more product buffer
  float2* slot = a.slots + (size_t)blockIdx.x * kAdjMats * NN;
  float2* Xs = slot;             // X_1..7
  float2* ks = slot + 7 * NN;    // k_1..6
  float2* kap = slot + 14 * NN;  // kappa_1..7
  float2* xi = slot + 21 * NN;
  float2* lam = slot + 22 * NN;
  const Tableau& T = c_tab[a.o.method];
  for (;;) {
    if (tid == 0) inst_sh = (long long)atomicAdd(a.counter, 1u);
    __syncthreads();
    const long long b = inst_sh;
    if (b >= a.batch) break;
    const InstView v = view_of(a, b);
    const long long nn = (long long)n * n;
    float2* gH = A.grad_H + b * nn;
    float2* gL = A.grad_L + b * K * nn;
    for (long long e = tid; e < nn; e += blockDim.x) gH[e] = make_float2(0.f, 0.f);
    for (long long e = tid; e < K * nn; e += blockDim.x) gL[e] = make_float2(0.f, 0.f);
    load_padded<NP>(sH, v.H, n);
    for (int k = 0; k < K; ++k) load_padded<NP>(sL + k * MAT, v.L + (long long)k * nn, n);
    __syncthreads();
    build_hnh<NP>(sH, sL, n, K);
    __syncthreads();
    const int nsave = a.o.save_states ? a.ntsave : 1;
    // lambda: the final state's cotangent when only it is saved, else zero
    for (int e = tid; e < NN; e += blockDim.x) {
      const int i = e / NP, j = e % NP;
      float2 g = make_float2(0.f, 0.f);
      if (!a.o.save_states && A.gstates && i < n && j < n) g = A.gstates[b * nn + i * n + j];
      lam[e] = g;
    }
    int sp = a.ntsave - 1;  // saves are taken from the last one backwards
    const int N = A.nacc[b];
    for (int st = N - 1; st >= 0; --st) {
      const double t = v.tape_t[st], h = v.tape_h[st];
      const float2* y = a.tape_y + (b * (long long)a.tape_cap + st) * NN;
      // (a) direct cotangents of the stages: the step's end state and its saves
      for (int e = tid; e < NN; e += blockDim.x) {
        const float2 l = lam[e];
#pragma unroll
        for (int j = 0; j < 7; ++j) kap[j * NN + e] = make_float2((float)(h * T.b[j]) * l.x, (float)(h * T.b[j]) * l.y);
      }
      __syncthreads();
      while (sp >= 0 && (st == 0 || a.tsave[sp] > t)) {
        double w[7];
        dense_weights(a.o.method, h > 0.0 ? (a.tsave[sp] - t) / h : 1.0, w);
        for (int e = tid; e < NN; e += blockDim.x) {
          const int i = e / NP, j = e % NP;
          if (i >= n || j >= n) continue;
          float2 g = make_float2(0.f, 0.f);
          if (a.o.save_states && A.gstates) g = A.gstates[(b * nsave + sp) * nn + i * n + j];
          if (A.gexpects)
            for (int m = 0; m < a.nE; ++m) {  // d tr(E rho) / d rho: cotangent ebar E^+
              const float2 eb = A.gexpects[(b * a.nE + m) * a.ntsave + sp];
              g = cfma(eb, cconj(a.E[((long long)m * n + j) * n + i]), g);
            }
#pragma unroll
          for (int q = 0; q < 7; ++q) kap[q * NN + e] = caxpy((float)(h * w[q]), g, kap[q * NN + e]);
          lam[e] = cadd(lam[e], g);
        }
        __syncthreads();
        --sp;
      }
      // (b) the forward stages again: X_1 = y, X_j = y + h sum_{l<j} a_jl k_l, k_j = S(X_j)
      for (int j = 0; j < 7; ++j) {
        float cf[6];
#pragma unroll
        for (int l = 0; l < 6; ++l) cf[l] = (float)(h * T.a[j][l]);
        for (int e = tid; e < NN; e += blockDim.x) {
          float2 x = y[e];
          for (int l = 0; l < j; ++l) x = caxpy(cf[l], ks[l * NN + e], x);
          Xs[j * NN + e] = x;
          sX[(e / NP) * LD + e % NP] = x;
        }
        __syncthreads();
        if (j < 6) dqb::rhs<NP>(sH, sL, sX, sT, n, K, DQB_FORM_STANDARD, ks + j * NN, NP, NP);
        __syncthreads();
      }
      // (c) adjoint operators in place: Hnh -> Hnh^+, L_k -> L_k^+
      dagger_inplace<NP>(sH);
      for (int k = 0; k < K; ++k) dagger_inplace<NP>(sL + k * MAT);
      __syncthreads();
      // (d) stages backwards
      for (int j = 6; j >= 0; --j) {
        to_smem<NP>(sX, kap + j * NN);
        __syncthreads();
        dqb::rhs<NP>(sH, sL, sX, sT, n, K, DQB_FORM_STANDARD, xi, NP, NP);  // xi = S^+(kappa_j)
        __syncthreads();
        for (int e = tid; e < NN; e += blockDim.x) {
          const float2 x = xi[e];
          lam[e] = cadd(lam[e], x);
          for (int l = 0; l < j; ++l) kap[l * NN + e] = caxpy((float)(h * T.a[j][l]), x, kap[l * NN + e]);
        }
        // operator gradients: sT <- Zs = kappa_j + kappa_j^+, sX <- X_j
        for (int e = tid; e < NN; e += blockDim.x) {
          const int i = e / NP, c = e % NP;
          sT[i * LD + c] = cadd(kap[j * NN + e], cconj(kap[j * NN + c * NP + i]));
          sX[i * LD + c] = Xs[j * NN + e];
        }
        __syncthreads();
        float2 acc[NP / 16][NP / 16];
        zero_tile<NP>(acc);
        gemm<NP, false, false>(acc, sT, sX, NP);  // Zs X
        add_tile<NP>(gH, acc, make_float2(0.f, 1.f), n);
        store_tile<NP>(sU, acc, 1.0f);              // sU = Zs X
        __syncthreads();
        for (int k = 0; k < K; ++k) {
          const float2* Lk = sL + k * MAT;  // holds L_k^+; op = ^+ reads L_k back
          // - 1/2 L (Zs X)
          zero_tile<NP>(acc);
          gemm<NP, true, false>(acc, Lk, sU, NP);
          add_tile<NP>(gL + k * nn, acc, make_float2(-0.5f, 0.f), n);
        }
        __syncthreads();
        zero_tile<NP>(acc);
        gemm<NP, false, false>(acc, sX, sT, NP);  // X Zs
        store_tile<NP>(sU, acc, 1.0f);
        __syncthreads();
        for (int k = 0; k < K; ++k) {
          const float2* Lk = sL + k * MAT;
          zero_tile<NP>(acc);
          gemm<NP, true, false>(acc, Lk, sU, NP);  // - 1/2 L (X Zs)
          add_tile<NP>(gL + k * nn, acc, make_float2(-0.5f, 0.f), n);
        }
        for (int k = 0; k < K; ++k) {
          const float2* Lk = sL + k * MAT;
          zero_tile<NP>(acc);
          gemm<NP, false, true>(acc, sT, Lk, NP);  // Zs L
          __syncthreads();
          store_tile<NP>(sU, acc, 1.0f);
          __syncthreads();
          zero_tile<NP>(acc);
          gemm<NP, false, false>(acc, sU, sX, NP);  // (Zs L) X
          add_tile<NP>(gL + k * nn, acc, make_float2(1.f, 0.f), n);
          __syncthreads();
        }
        __syncthreads();
      }
      // (e) operators back
      dagger_inplace<NP>(sH);
      for (int k = 0; k < K; ++k) dagger_inplace<NP>(sL + k * MAT);
      __syncthreads();
    }
    // saves at or before t0 (no step reached them): they read y0 itself
    while (sp >= 0) {
      for (int e = tid; e < NN; e += blockDim.x) {
        const int i = e / NP, j = e % NP;
        if (i >= n || j >= n) continue;
        float2 g = make_float2(0.f, 0.f);
        if (a.o.save_states && A.gstates) g = A.gstates[(b * nsave + sp) * nn + i * n + j];
        if (A.gexpects)
          for (int m = 0; m < a.nE; ++m)
            g = cfma(A.gexpects[(b * a.nE + m) * a.ntsave + sp], cconj(a.E[((long long)m * n + j) * n + i]), g);
        lam[e] = cadd(lam[e], g);
      }
      __syncthreads();
      --sp;
    }
    // rho0 = psi psi^+ for a ket: psibar = (lambda + lambda^+) psi
    __syncthreads();
    if (v.is_ket) {
      for (int i = tid; i < n; i += blockDim.x) {
        float2 acc = make_float2(0.f, 0.f);
        for (int j = 0; j < n; ++j)
          acc = cfma(cadd(lam[i * NP + j], cconj(lam[j * NP + i])), v.rho0[j], acc);
        A.grad_rho0[b * n + i] = acc;
      }
    } else {
      for (long long e = tid; e < nn; e += blockDim.x) A.grad_rho0[b * nn + e] = lam[(e / n) * NP + e % n];
    }
    __syncthreads();
  }
}

template <int NP>
static size_t adjoint_smem_bytes(int K) {
  return (size_t)(4 + K) * Small<NP>::MAT * sizeof(float2);
}

template <int NP>
static int adjoint_launch(const AdjArgs& A, cudaStream_t s, long long max_grid) {
  const size_t smem = adjoint_smem_bytes<NP>(A.p.K);
  if (smem + 2048 > max_optin_smem()) return DQB_ERR_UNSUPPORTED;
  const int per_sm = resident_ctas(mesolve_adjoint_kernel<NP>, smem);
  if (per_sm < 1) return DQB_ERR_UNSUPPORTED;
  long long g = std::min<long long>((long long)per_sm * sm_count(), A.p.batch);
  g = std::min<long long>(g, max_grid);
  mesolve_adjoint_kernel<NP><<<(unsigned)std::max<long long>(g, 1), kSmallThreads, smem, s>>>(A);
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}

}  // namespace dqb

extern "C" size_t dqb_mesolve_dense_tape_bytes(int32_t n, int32_t tape_cap, int64_t batch) {
  const int NP = dqb::pick_np(n);
  if (NP == 0 || tape_cap < 0 || batch < 0) return 0;
  return (size_t)batch * tape_cap * NP * NP * sizeof(float2);
}

extern "C" int dqb_mesolve_dense_taped(const dqb_dense_problem* p, const dqb_ode_options* o,
                                       const dqb_outputs* out, const dqb_tape* tape, void* workspace,
                                       size_t workspace_bytes, void* stream) {
  using namespace dqb;
  int rc = validate_dense(p, o);
  if (rc) return rc;
  if (!out || !out->states || !out->infos || !out->status || (p->n_exp > 0 && !out->expects))
    return DQB_ERR_INVALID_ARGUMENT;
  if (!tape || !tape->t || !tape->h || !tape->y || tape->capacity < 1) return DQB_ERR_INVALID_ARGUMENT;
  if (p->batch == 0) return DQB_OK;
  const int NP = pick_np(p->n);
  if (NP == 0 || dqb_dense_small_max_n(p->n_jumps) < NP) return DQB_ERR_UNSUPPORTED;
  const size_t need = dqb_mesolve_dense_workspace_size(p->n, p->n_jumps, p->batch);
  if (need == 0) return DQB_ERR_UNSUPPORTED;
  if (!workspace || workspace_bytes < need) return DQB_ERR_WORKSPACE_TOO_SMALL;
  const int grid = grid_for<2>(NP, p->n_jumps, p->batch);
  cudaStream_t s = (cudaStream_t)stream;
  DenseSmallArgs a = make_args(p, o, out);
  a.counter = (unsigned int*)workspace;
  a.slots = (float2*)((char*)workspace + 256);
  a.tape_t = tape->t;
  a.tape_h = tape->h;
  a.tape_y = (float2*)tape->y;
  a.tape_cap = tape->capacity;
  zero_words_kernel<<<1, 64, 0, s>>>((unsigned int*)workspace, 64);
  const size_t smem = smem_for(NP, p->n_jumps);
  switch (NP) {
    case 16: mesolve_small_kernel<16, 2><<<grid, kSmallThreads, smem, s>>>(a); break;
    case 32: mesolve_small_kernel<32, 2><<<grid, kSmallThreads, smem, s>>>(a); break;
    default: mesolve_small_kernel<64, 2><<<grid, kSmallThreads, smem, s>>>(a); break;
  }
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}

extern "C" size_t dqb_mesolve_dense_adjoint_workspace_size(int32_t n, int32_t n_jumps, int64_t batch) {
  using namespace dqb;
  const int NP = pick_np(n);
  if (NP == 0 || batch <= 0 || n_jumps < 0) return 0;
  const size_t smem = (size_t)(4 + n_jumps) * (NP + 1) * NP * sizeof(float2);
  if (smem + 2048 > max_optin_smem()) return 0;
  const long long g = std::min<long long>((long long)sm_count(), batch);
  return 256 + (size_t)g * kAdjMats * NP * NP * sizeof(float2);
}

extern "C" int dqb_mesolve_dense_adjoint(const dqb_dense_problem* p, const dqb_ode_options* o,
                                         const dqb_tape* tape, const int32_t* naccepted,
                                         const dqb_cotangents* cot, const dqb_gradients* grads,
                                         void* workspace, size_t workspace_bytes, void* stream) {
  using namespace dqb;
  int rc = validate_dense(p, o);
  if (rc) return rc;
  if (!tape || !tape->t || !tape->h || !tape->y || !naccepted || !cot || !grads) return DQB_ERR_INVALID_ARGUMENT;
  if (!grads->rho0 || !grads->H || (p->n_jumps > 0 && !grads->L)) return DQB_ERR_INVALID_ARGUMENT;
  if (p->n_exp > 0 && cot->expects && !p->E) return DQB_ERR_INVALID_ARGUMENT;
  if (p->batch == 0) return DQB_OK;
  const int NP = pick_np(p->n);
  if (NP == 0) return DQB_ERR_UNSUPPORTED;
  const size_t need = dqb_mesolve_dense_adjoint_workspace_size(p->n, p->n_jumps, p->batch);
  if (need == 0) return DQB_ERR_UNSUPPORTED;
  if (!workspace || workspace_bytes < need) return DQB_ERR_WORKSPACE_TOO_SMALL;
  cudaStream_t s = (cudaStream_t)stream;
  AdjArgs A;
  A.p = make_args(p, o, nullptr);
  A.p.counter = (unsigned int*)workspace;
  A.p.slots = (float2*)((char*)workspace + 256);
  A.p.tape_t = tape->t;
  A.p.tape_h = tape->h;
  A.p.tape_y = (float2*)tape->y;
  A.p.tape_cap = tape->capacity;
  A.nacc = naccepted;
  A.gstates = (const float2*)cot->states;
  A.gexpects = (const float2*)cot->expects;
  A.grad_rho0 = (float2*)grads->rho0;
  A.grad_H = (float2*)grads->H;
  A.grad_L = (float2*)grads->L;
  zero_words_kernel<<<1, 64, 0, s>>>((unsigned int*)workspace, 64);
  const long long max_grid = (long long)((workspace_bytes - 256) / ((size_t)kAdjMats * NP * NP * sizeof(float2)));
  switch (NP) {
    case 16: return adjoint_launch<16>(A, s, max_grid);
    case 32: return adjoint_launch<32>(A, s, max_grid);
    default: return adjoint_launch<64>(A, s, max_grid);
  }
}

extern "C" const char* dqb_version(void) { return "dqb200 0.2 sm_100a"; }

// ------------------------------------------------------------------------------------
// internal helpers for entry points that bring their own scratch (not exported)
// ------------------------------------------------------------------------------------
namespace dqb {

// Bytes of one in-flight instance's scratch slot for dimension n (0 if n > 64).
size_t small_slot_bytes(int n) {
  const int NP = pick_np(n);
  return NP ? (size_t)kSlotMats * NP * NP * sizeof(float2) : 0;
}

// Resident CTAs of the persistent kernel for (n, K, batch) on the current device.
int small_resident_grid(int n, int K, long long batch) {
  const int NP = pick_np(n);
  return NP ? grid_for(NP, K, batch) : 0;
}

// Argument checks of dqb_mesolve_dense, without the workspace.
int small_check_args(const dqb_dense_problem* p, const dqb_ode_options* o, const dqb_outputs* out) {
  int rc = validate_dense(p, o);
  if (rc) return rc;
  if (!out || !out->states || !out->infos || !out->status || (p->n_exp > 0 && !out->expects))
    return DQB_ERR_INVALID_ARGUMENT;
  const int NP = pick_np(p->n);
  if (NP == 0 || dqb_dense_small_max_n(p->n_jumps) < NP) return DQB_ERR_UNSUPPORTED;
  return DQB_OK;
}

// Launch the persistent kernel on `grid` CTAs with a zeroed work counter at `counter`
// and grid * small_slot_bytes(n) bytes of slots at `slots` (both device addresses).
int small_launch_with_scratch(const dqb_dense_problem* p, const dqb_ode_options* o, const dqb_outputs* out,
                              unsigned int* counter, void* slots, int grid, cudaStream_t s) {
  const int NP = pick_np(p->n);
  DenseSmallArgs a = make_args(p, o, out);
  a.counter = counter;
  a.slots = (float2*)slots;
  const size_t smem = smem_for(NP, p->n_jumps);
  switch (NP) {
    case 16: mesolve_small_kernel<16><<<grid, kSmallThreads, smem, s>>>(a); break;
    case 32: mesolve_small_kernel<32><<<grid, kSmallThreads, smem, s>>>(a); break;
    default: mesolve_small_kernel<64><<<grid, kSmallThreads, smem, s>>>(a); break;
  }
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}

}  // namespace dqb

// ------------------------------------------------------------------------------------
// ragged batches: every instance brings its own n, jumps, tsave and output buffers
// ------------------------------------------------------------------------------------
namespace dqb {

template <int NP>
__global__ void __launch_bounds__(kSmallThreads, NP == 64 ? 1 : (NP == 32 ? 3 : 4)) mesolve_ragged_kernel(const dqb_ragged_instance* __restrict__ d,
                                                                       long long count, CtrlOpts o, float2* slots,
                                                                       unsigned int* counter) {
  extern __shared__ float4 smem_raw[];
  __shared__ double red[40];
  __shared__ Ctrl ctl;
  float2* sH = reinterpret_cast<float2*>(smem_raw);
  float2* sX = sH + Small<NP>::MAT;
  float2* sT = sX + Small<NP>::MAT;
  float2* sL = sT + Small<NP>::MAT;
  float2* slot = slots + (size_t)blockIdx.x * kSlotMats * Small<NP>::NN;
  for (;;) {
    if (threadIdx.x == 0) ctl.inst = (long long)atomicAdd(counter, 1u);
    __syncthreads();
    const long long inst = ctl.inst;
    if (inst >= count) break;
    const dqb_ragged_instance& r = d[inst];
    InstView v;
    v.n = r.n;
    v.K = r.n_jumps;
    v.nE = r.n_exp;
    v.ntsave = r.n_tsave;
    v.is_ket = r.rho0_is_ket;
    v.save_states = r.save_states;
    v.t0 = r.t0;
    v.H = (const float2*)r.H;
    v.L = (const float2*)r.L;
    v.rho0 = (const float2*)r.rho0;
    v.E = (const float2*)r.E;
    v.tsave = r.tsave;
    v.states = (float2*)r.states;
    v.expects = (float2*)r.expects;
    v.infos = r.infos;
    v.status = r.status;
    v.cancel = r.cancel;
    v.inst = inst;
    v.n_jump = 0;
    v.jump_ts = nullptr;
    v.tape_t = v.tape_h = nullptr;
    v.tape_y = nullptr;
    v.tape_cap = 0;
    SimtEngine<NP, 0> eng{sH, sX, sT, sL, v.n, v.K, o.form, nullptr, nullptr, inst};
    solve_one<NP>(eng, v, o, slot, red, ctl);
    __syncthreads();
  }
}

template <int NP>
static int ragged_grid(int K, long long count) {
  const size_t smem = small_smem_bytes<NP>(K);
  if (smem + 2048 > max_optin_smem()) return 0;
  const int per_sm = resident_ctas(mesolve_ragged_kernel<NP>, smem);
  if (per_sm < 1) return 0;
  long long g = (long long)per_sm * sm_count();
  if (g > count) g = count;
  return (int)std::max<long long>(g, 1);
}

static int ragged_grid_for(int NP, int K, long long count) {
  switch (NP) {
    case 16: return ragged_grid<16>(K, count);
    case 32: return ragged_grid<32>(K, count);
    default: return ragged_grid<64>(K, count);
  }
}

}  // namespace dqb

extern "C" size_t dqb_mesolve_ragged_workspace_size(int32_t max_n, int32_t max_jumps, int64_t count) {
  const int NP = pick_np(max_n);
  if (NP == 0 || count <= 0 || max_jumps < 0) return 0;
  const int g = ragged_grid_for(NP, max_jumps, count);
  if (g <= 0) return 0;
  return 256 + (size_t)g * kSlotMats * NP * NP * sizeof(float2);
}

extern "C" int dqb_mesolve_ragged(const dqb_ragged_instance* instances, int64_t count, int32_t max_n,
                                  int32_t max_jumps, const dqb_ode_options* o, void* workspace,
                                  size_t workspace_bytes, void* stream) {
  if (!o || count < 0 || max_n < 1 || max_jumps < 0) return DQB_ERR_INVALID_ARGUMENT;
  if (count >= (int64_t)0x7fffffff) return DQB_ERR_INVALID_ARGUMENT;
  if (o->method != DQB_METHOD_TSIT5 && o->method != DQB_METHOD_DOPRI5) return DQB_ERR_INVALID_ARGUMENT;
  if (o->form != DQB_FORM_HERMITIAN && o->form != DQB_FORM_STANDARD) return DQB_ERR_INVALID_ARGUMENT;
  if (!(o->rtol >= 0) || !(o->atol >= 0) || o->max_steps < 0) return DQB_ERR_INVALID_ARGUMENT;
  if (count == 0) return DQB_OK;
  if (!instances) return DQB_ERR_INVALID_ARGUMENT;
  const int NP = pick_np(max_n);
  if (NP == 0 || dqb_dense_small_max_n(max_jumps) < NP) return DQB_ERR_UNSUPPORTED;
  const size_t need = dqb_mesolve_ragged_workspace_size(max_n, max_jumps, count);
  if (need == 0) return DQB_ERR_UNSUPPORTED;
  if (!workspace || workspace_bytes < need) return DQB_ERR_WORKSPACE_TOO_SMALL;
  const int grid = ragged_grid_for(NP, max_jumps, count);
  cudaStream_t s = (cudaStream_t)stream;
  zero_words_kernel<<<1, 64, 0, s>>>((unsigned int*)workspace, 64);
  unsigned int* counter = (unsigned int*)workspace;
  float2* slots = (float2*)((char*)workspace + 256);
  const CtrlOpts c = make_ctrl(*o);
  const size_t smem = smem_for(NP, max_jumps);
  switch (NP) {
    case 16: mesolve_ragged_kernel<16><<<grid, kSmallThreads, smem, s>>>(instances, count, c, slots, counter); break;
    case 32: mesolve_ragged_kernel<32><<<grid, kSmallThreads, smem, s>>>(instances, count, c, slots, counter); break;
    default: mesolve_ragged_kernel<64><<<grid, kSmallThreads, smem, s>>>(instances, count, c, slots, counter); break;
  }
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}
