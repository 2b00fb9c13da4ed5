// Schroedinger equation d psi/dt = -i H psi beyond the warp-per-instance kernel (n > 128,
// dense H, or H in sparse-DIA storage at any n): the batched stepper of dqb_big.cuh with
// state vectors for states -- its slots hold psi, the stage inputs and the seven stages as
// n-vectors (Common.nn = n), and its combination, error, starting-step, control and
// commit kernels are the mesolve ones, elementwise over the n entries (the RMS error norm
// of the reference over psi, dynamiqs/integrators/core/diffrax_integrator.py:221-228).
// What is specific to kets:
//   * the right-hand side -i H x: a batched matrix-vector product (dense: one warp per row,
//     x staged in shared memory; DIA: one thread per row, out_i = -i sum_d
//     diag_d[i + k_d] x[i + k_d] with the reference's column-indexed diagonals);
//   * the save pass: the dense output v at each save point, then <v|E|v> = sum_i
//     conj(v_i) (E v)_i in FP64 (utils/general.py:467-474), one warp per row of E.
// A time-dependent H(t) = H + sum_m c_m(t) ops_m (dqb_td_hamiltonian) is formed per
// instance before every right-hand side, at that stage's time, into a workspace copy that
// the right-hand side then reads; the controller clips its steps at the discontinuities
// (the stepper's jump_ts handling).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "dqb_big.cuh"
#include "dqb_graph.cuh"

namespace dqb {
namespace {

constexpr int kSeThreads = 256;
constexpr int kSeRowsPerBlock = 32;  // dense product and save pass: rows of H / E per block
constexpr int kSeMaxN = 8192;        // x or v staged in shared memory (64 KB)

struct SeOps {
  int n;
  int dia;           // 0: dense H [*, n, n]; 1: DIA diagonals [*, nd, n]
  int nd;
  int off[DQB_DIA_MAX_HNH_DIAGS];
  const float2* H;   // read by the right-hand side (H(t) of instance b at b when time-dependent)
  const int* Hidx;
  float2* Ht;        // time-dependent H: the per-instance copies H points to (workspace)
  const float2* H0;  // time-dependent H: the constant part, indexed by H0idx
  const int* H0idx;
};

// Values of one instance's H: n^2 (dense) or nd n (DIA).
__host__ __device__ __forceinline__ long long h_size(const SeOps& d) {
  return d.dia ? (long long)d.nd * d.n : (long long)d.n * d.n;
}

__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Input and output slots of a right-hand side (in_sel 0 = y, 1 = y1, 2 = X; need_run 1 =
// running instances, 0 = every instance whose status is OK, 2 = the running ones whose
// first stage is re-evaluated after a discontinuity).
__device__ __forceinline__ bool se_io(const big::Common& c, int b, int in_sel, int out_k, int need_run,
                                      const float2*& x, float2*& out) {
  const big::Inst& I = c.inst[b];
  if (need_run == 2 ? !(I.run && I.refresh) : (need_run ? !I.run : I.status != DQB_INST_OK)) return false;
  x = big::slot(c, b, in_sel == 0 ? I.sy : (in_sel == 1 ? I.sy1 : big::kX));
  out = big::slot(c, b, I.sk[out_k]);
  return true;
}

// Dense: grid (ceil(n / 32), B), 256 threads, x in dynamic shared memory (n values).
// Each warp takes 4 rows; a lane sums the columns 2 lane + 64 t and 2 lane + 64 t + 1 (one
// 16-byte load of H per pair when n is even), then the warp reduces.
__global__ void __launch_bounds__(kSeThreads) se_rhs_dense_kernel(big::Common c, SeOps d, int in_sel, int out_k,
                                                                  int need_run) {
  extern __shared__ float2 sx[];
  const int b = blockIdx.y;
  const float2* x;
  float2* out;
  if (!se_io(c, b, in_sel, out_k, need_run, x, out)) return;
  const int n = d.n;
  for (int e = threadIdx.x; e < n; e += blockDim.x) sx[e] = x[e];
  __syncthreads();
  const float2* H = d.H + (d.Hidx ? (long long)d.Hidx[b] : (long long)b) * n * n;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool even = (n & 1) == 0;
  for (int rr = warp; rr < kSeRowsPerBlock; rr += kSeThreads / 32) {
    const int i = blockIdx.x * kSeRowsPerBlock + rr;
    if (i >= n) break;
    const float2* Hi = H + (long long)i * n;
    float2 acc = make_float2(0.f, 0.f);
    if (even) {
#pragma unroll 4  // four 16-byte loads of the row in flight per lane
      for (int j = 2 * lane; j < n; j += 64) {
        const float4 h = __ldg(reinterpret_cast<const float4*>(Hi + j));
        acc = cfma(make_float2(h.x, h.y), sx[j], acc);
        acc = cfma(make_float2(h.z, h.w), sx[j + 1], acc);
      }
    } else {
      for (int j = lane; j < n; j += 32) acc = cfma(__ldg(Hi + j), sx[j], acc);
    }
    acc.x = warp_sumf(acc.x);
    acc.y = warp_sumf(acc.y);
    if (lane == 0) out[i] = make_float2(acc.y, -acc.x);  // -i (H x)_i
  }
}

// DIA: grid (ceil(n / 256), B), one row per thread.
__global__ void __launch_bounds__(kSeThreads) se_rhs_dia_kernel(big::Common c, SeOps d, int in_sel, int out_k,
                                                                int need_run) {
  const int b = blockIdx.y;
  const float2* x;
  float2* out;
  if (!se_io(c, b, in_sel, out_k, need_run, x, out)) return;
  const int n = d.n;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float2* D = d.H + (d.Hidx ? (long long)d.Hidx[b] : (long long)b) * d.nd * n;
  float2 acc = make_float2(0.f, 0.f);
  for (int q = 0; q < d.nd; ++q) {
    const int j = i + d.off[q];  // H[i][j] = diag_q[j]
    if (j >= 0 && j < n) acc = cfma(__ldg(D + (long long)q * n + j), x[j], acc);
  }
  out[i] = make_float2(acc.y, -acc.x);
}

// H(t) of every instance that evaluates the right-hand side `which` (big::td_stage_time):
// d.H[b] = H0[H0idx[b]] + sum_m c_m(t) ops_m, in the layout of the path.  grid (tiles, B).
__global__ void se_h_td_kernel(big::Common c, SeOps d, TdOps td, int which) {
  __shared__ float2 cm[DQB_TD_MAX_TERMS];
  const int b = blockIdx.y;
  double t;
  if (!big::td_stage_time(c, c.inst[b], which, &t)) return;
  if (threadIdx.x < td.M) {
    const double2 v = td_coef(td.term[threadIdx.x], b, t);
    cm[threadIdx.x] = make_float2((float)v.x, (float)v.y);
  }
  __syncthreads();
  const long long hs = h_size(d);
  const float2* h0 = d.H0 + (d.H0idx ? (long long)d.H0idx[b] : (long long)b) * hs;
  float2* out = d.Ht + (long long)b * hs;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < hs; e += (long long)gridDim.x * blockDim.x) {
    float2 v = h0[e];
    for (int m = 0; m < td.M; ++m) v = cfma(cm[m], td.ops[(long long)m * hs + e], v);
    out[e] = v;
  }
}

// grid (tiles, B): psi0 into y, expectation sums zeroed.
__global__ void se_load_kernel(big::Common c) {
  const int b = blockIdx.y;
  big::Inst& I = c.inst[b];
  if (I.status == big::kInactive) return;
  float2* y = big::slot(c, b, I.sy);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < c.nn;
       e += (long long)gridDim.x * blockDim.x)
    y[e] = I.rho0[e];
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)I.nE * I.nts;
       e += (long long)gridDim.x * blockDim.x)
    I.eacc[e] = make_double2(0.0, 0.0);
}

// Saves of the step (mode 1: dense output of the stages; mode 0: y itself, the leftovers
// after the loop).  grid (ceil(n / 32), B), 256 threads, v in dynamic shared memory: every
// block forms the whole v of a save point (the same FP32 sums in the same order as the
// mesolve save pass), writes its 32 rows of the state and adds its rows' share of
// <v|E_m|v> = sum_i conj(v_i) sum_j E_ij v_j, one warp per row, FP64 sums.
__global__ void __launch_bounds__(kSeThreads) se_save_kernel(big::Common c, int mode) {
  extern __shared__ float2 sv[];
  __shared__ double red[72];
  __shared__ float cw[8];
  const int b = blockIdx.y;
  const big::Inst& I = c.inst[b];
  const int lo = I.save_lo, hi = I.save_hi;
  if (hi <= lo) return;
  const int n = c.n;
  const float2* p[8];
  p[0] = big::slot(c, b, I.sy);
  for (int q = 1; q < 8; ++q) p[q] = big::slot(c, b, I.sk[q - 1]);
  const int nq = mode == 0 ? 1 : 8;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int s = lo; s < hi; ++s) {
    __syncthreads();  // the previous save's v and weights are no longer read
    if (threadIdx.x == 0) {
      const double theta = I.h > 0.0 ? (I.ts[s] - I.t) / I.h : 1.0;
      double w[7];
      dense_weights(c.o.method, theta, w);
      cw[0] = 1.f;
      for (int j = 0; j < 7; ++j) cw[j + 1] = mode == 0 ? 0.f : (float)(I.h * w[j]);
    }
    __syncthreads();
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      float2 v = make_float2(0.f, 0.f);
      for (int q = 0; q < nq; ++q) v = caxpy(cw[q], p[q][e], v);
      sv[e] = v;
    }
    __syncthreads();
    const int r0 = blockIdx.x * kSeRowsPerBlock;
    if (I.save_states)
      for (int r = threadIdx.x; r < kSeRowsPerBlock && r0 + r < n; r += blockDim.x)
        I.states[(long long)s * n + r0 + r] = sv[r0 + r];
    for (int m = 0; m < I.nE; ++m) {
      const float2* E = I.E + (long long)m * n * n;
      double sr = 0.0, si = 0.0;
      for (int rr = warp; rr < kSeRowsPerBlock; rr += kSeThreads / 32) {
        const int i = r0 + rr;
        if (i >= n) break;
        const float2* Ei = E + (long long)i * n;
        double ar = 0.0, ai = 0.0;
        for (int j = lane; j < n; j += 32) {
          const float2 e = __ldg(Ei + j), v = sv[j];
          ar += (double)e.x * v.x - (double)e.y * v.y;
          ai += (double)e.x * v.y + (double)e.y * v.x;
        }
        const float2 vi = sv[i];  // conj(v_i) (E v)_i
        sr += (double)vi.x * ar + (double)vi.y * ai;
        si += (double)vi.x * ai - (double)vi.y * ar;
      }
      const double2 tot = block_sum2(sr, si, red);
      if (threadIdx.x == 0) {
        double2* acc = I.eacc + (long long)m * I.nts + s;
        atomicAdd(&acc->x, tot.x);
        atomicAdd(&acc->y, tot.y);
      }
    }
  }
}

struct SeLayout {
  size_t off_iter, off_inst, off_eacc, off_mats, total;
};

size_t se_align(size_t x) { return (x + 255) & ~(size_t)255; }

SeLayout se_layout(int n, int nE, int ntsave, long long B) {
  SeLayout l;
  l.off_iter = 0;
  l.off_inst = 256;
  l.off_eacc = se_align(l.off_inst + B * sizeof(big::Inst));
  l.off_mats = se_align(l.off_eacc + B * (size_t)nE * ntsave * sizeof(double2));
  l.total = l.off_mats + B * (size_t)big::kSlots * n * sizeof(float2);
  return l;
}

GraphCache g_cache;

struct LaunchKey {
  big::Common c;
  SeOps d;
  TdOps td;
};

void launch_rhs(cudaStream_t s, const big::Common& c, const SeOps& d, int in_sel, int out_k, int need_run) {
  if (d.dia) {
    se_rhs_dia_kernel<<<dim3((d.n + kSeThreads - 1) / kSeThreads, c.B), kSeThreads, 0, s>>>(c, d, in_sel, out_k,
                                                                                          need_run);
  } else {
    se_rhs_dense_kernel<<<dim3((d.n + kSeRowsPerBlock - 1) / kSeRowsPerBlock, c.B), kSeThreads,
                          (size_t)d.n * sizeof(float2), s>>>(c, d, in_sel, out_k, need_run);
  }
}

void launch_save(cudaStream_t s, const big::Common& c, int mode) {
  se_save_kernel<<<dim3((c.n + kSeRowsPerBlock - 1) / kSeRowsPerBlock, c.B), kSeThreads,
                   (size_t)c.n * sizeof(float2), s>>>(c, mode);
}

void init_attrs() {
  static std::once_flag once;
  std::call_once(once, [] {
    prefer_max_shared(se_rhs_dense_kernel);
    prefer_max_shared(se_save_kernel);
    prefer_max_shared(se_h_td_kernel);
    cudaFuncSetAttribute(se_rhs_dense_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         kSeMaxN * (int)sizeof(float2));
    cudaFuncSetAttribute(se_save_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSeMaxN * (int)sizeof(float2));
  });
}

int check_opts(const dqb_ode_options* o, const dqb_outputs* out, int n_exp) {
  if (!o || !out || !out->states || !out->infos || !out->status || (n_exp > 0 && !out->expects))
    return DQB_ERR_INVALID_ARGUMENT;
  if (o->method != DQB_METHOD_TSIT5 && o->method != DQB_METHOD_DOPRI5) return DQB_ERR_INVALID_ARGUMENT;
  if (!(o->rtol >= 0) || !(o->atol >= 0) || o->max_steps < 0) return DQB_ERR_INVALID_ARGUMENT;
  return DQB_OK;
}

// The solve, once the operators are described by `d0`; `tdh` (or null): the time-dependent
// terms of H (ops_m in the layout of d0.H) and the discontinuity times.
int run(const SeOps& d0, int nE, int ntsave, long long B, const void* psi0, const int* pidx, const void* E,
        const double* tsave, const dqb_ode_options* o, const dqb_outputs* out, void* workspace,
        size_t workspace_bytes, cudaStream_t s, const dqb_td_hamiltonian* tdh = nullptr) {
  const SeLayout lay = se_layout(d0.n, nE, ntsave, B);
  TdOps td;
  std::memset(&td, 0, sizeof(td));
  if (tdh) {
    if (tdh->jump_terms) return DQB_ERR_UNSUPPORTED;  // the Schroedinger equation has no jumps
    if (int tr = td_ops_from(tdh, &td)) return tr;
  }
  const size_t need = tdh ? se_align(lay.total) + (size_t)B * h_size(d0) * sizeof(float2) : lay.total;
  if (!workspace || workspace_bytes < need) return DQB_ERR_WORKSPACE_TOO_SMALL;
  char* ws = (char*)workspace;
  SeOps d = d0;
  if (tdh) {  // the right-hand side reads H(t), one copy per instance in the workspace
    d.H0 = d0.H;
    d.H0idx = d0.Hidx;
    d.Ht = (float2*)(ws + se_align(lay.total));
    d.H = d.Ht;
    d.Hidx = nullptr;
  }
  big::Common c;
  std::memset(&c, 0, sizeof(c));
  c.n = d.n;
  c.nn = d.n;  // the stepper's elementwise kernels run over the n entries of psi
  c.B = (int)B;
  c.nE = nE;
  c.ntsave = ntsave;
  c.form = DQB_FORM_STANDARD;
  c.save_states = o->save_states;
  c.rho0_is_ket = 0;  // psi0 is copied as it is (se_load_kernel); no psi psi^+
  c.o = make_ctrl(*o);
  c.o.check_hermitian = 0;
  c.tsave = tsave;
  c.inst = (big::Inst*)(ws + lay.off_inst);
  c.mats = (float2*)(ws + lay.off_mats);
  c.eacc = (double2*)(ws + lay.off_eacc);
  c.states = (float2*)out->states;
  c.expects = (float2*)out->expects;
  c.infos = out->infos;
  c.status = out->status;
  c.E = (const float2*)E;
  c.rho0 = (const float2*)psi0;
  c.ridx = pidx;
  c.iter = (long long*)(ws + lay.off_iter);
  if (tdh) {
    c.n_jump = tdh->n_jump_ts;
    c.jump_ts = tdh->jump_ts;
  }

  init_attrs();
  int grid_e = (int)std::min<long long>((c.nn + big::kElemThreads - 1) / big::kElemThreads, 1184);
  if (grid_e < 1) grid_e = 1;
  const dim3 ge(grid_e, c.B);
  const dim3 gi((c.B + 127) / 128);
  const int T = big::kElemThreads;
  const dim3 gh((unsigned)std::min<long long>((h_size(d) + T - 1) / T, 1184), c.B);
  // H at the time of the next right-hand side (time-dependent H only)
  auto at_time = [&](cudaStream_t cs, int which) {
    if (tdh) se_h_td_kernel<<<gh, T, 0, cs>>>(c, d, td, which);
  };

  big::setup_kernel<<<gi, 128, 0, s>>>(c);
  se_load_kernel<<<ge, T, 0, s>>>(c);
  at_time(s, 8);
  launch_rhs(s, c, d, 0, 0, 0);
  big::init_norm_kernel<<<ge, T, 0, s>>>(c, 0);
  big::init_ctrl_kernel<<<gi, 128, 0, s>>>(c, 0);
  big::combine_kernel<<<ge, T, 0, s>>>(c, 6);
  at_time(s, 9);
  launch_rhs(s, c, d, 2, 1, 0);
  big::init_norm_kernel<<<ge, T, 0, s>>>(c, 1);
  big::init_ctrl_kernel<<<gi, 128, 0, s>>>(c, 1);
  if (cudaGetLastError() != cudaSuccess) return DQB_ERR_CUDA;

  auto body = [&](cudaStream_t cs, cudaGraphConditionalHandle h, int* flag) {
    for (int st = 0; st < 5; ++st) {
      big::combine_kernel<<<ge, T, 0, cs>>>(c, st);
      at_time(cs, st + 1);
      launch_rhs(cs, c, d, 2, st + 1, 1);
    }
    big::combine_kernel<<<ge, T, 0, cs>>>(c, 5);
    at_time(cs, 6);
    launch_rhs(cs, c, d, 1, 6, 1);
    big::error_kernel<<<ge, T, 0, cs>>>(c);
    big::control_kernel<<<gi, 128, 0, cs>>>(c);
    launch_save(cs, c, 1);
    big::commit_kernel<<<1, 1024, 0, cs>>>(c, h, flag);
    if (tdh) {  // the first stage of a step that starts on a discontinuity
      at_time(cs, 7);
      launch_rhs(cs, c, d, 0, 0, 2);
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
  launch_save(s, c, 0);
  big::finalize_kernel<<<ge, T, 0, s>>>(c);
  return cudaGetLastError() == cudaSuccess ? DQB_OK : DQB_ERR_CUDA;
}

}  // namespace
}  // namespace dqb

using namespace dqb;

extern "C" size_t dqb_sesolve_large_workspace_size(int32_t n, int32_t n_exp, int32_t n_tsave, int64_t batch) {
  if (n < 1 || n > kSeMaxN || n_exp < 0 || n_tsave < 1 || batch <= 0) return 0;
  return se_layout(n, n_exp, n_tsave, batch).total;
}

extern "C" size_t dqb_sesolve_large_td_workspace_size(int32_t n, int64_t h_values, int32_t n_exp, int32_t n_tsave,
                                                      int64_t batch) {
  const size_t base = dqb_sesolve_large_workspace_size(n, n_exp, n_tsave, batch);
  if (!base || h_values < 1) return 0;
  return se_align(base) + (size_t)batch * h_values * sizeof(float2);
}

static int sesolve_dense_large(const dqb_dense_problem* p, const dqb_td_hamiltonian* td, const dqb_ode_options* o,
                               const dqb_outputs* out, void* workspace, size_t workspace_bytes, void* stream) {
  if (!p) return DQB_ERR_INVALID_ARGUMENT;
  if (p->n < 1 || p->n_jumps != 0 || p->n_exp < 0 || p->n_tsave < 1 || p->batch < 0) return DQB_ERR_INVALID_ARGUMENT;
  if (!p->H || !p->rho0 || !p->tsave || (p->n_exp > 0 && !p->E)) return DQB_ERR_INVALID_ARGUMENT;
  if (p->n > kSeMaxN || p->batch > 65535) return DQB_ERR_UNSUPPORTED;
  int rc = check_opts(o, out, p->n_exp);
  if (rc) return rc;
  if (p->batch == 0) return DQB_OK;
  SeOps d;
  std::memset(&d, 0, sizeof(d));
  d.n = p->n;
  d.dia = 0;
  d.H = (const float2*)p->H;
  d.Hidx = p->H_index;
  return run(d, p->n_exp, p->n_tsave, p->batch, p->rho0, p->rho0_index, p->E, p->tsave, o, out, workspace,
             workspace_bytes, (cudaStream_t)stream, td);
}

extern "C" int dqb_sesolve_dense_large(const dqb_dense_problem* p, const dqb_ode_options* o,
                                       const dqb_outputs* out, void* workspace, size_t workspace_bytes,
                                       void* stream) {
  return sesolve_dense_large(p, nullptr, o, out, workspace, workspace_bytes, stream);
}

extern "C" int dqb_sesolve_dense_large_td(const dqb_dense_problem* p, const dqb_td_hamiltonian* td,
                                          const dqb_ode_options* o, const dqb_outputs* out, void* workspace,
                                          size_t workspace_bytes, void* stream) {
  if (!td) return DQB_ERR_INVALID_ARGUMENT;
  return sesolve_dense_large(p, td, o, out, workspace, workspace_bytes, stream);
}

static int sesolve_dia(const dqb_dia_problem* p, const dqb_td_hamiltonian* td, const dqb_ode_options* o,
                       const dqb_outputs* out, void* workspace, size_t workspace_bytes, void* stream) {
  if (!p) return DQB_ERR_INVALID_ARGUMENT;
  if (p->n < 1 || p->n_jumps != 0 || p->n_exp < 0 || p->n_tsave < 1 || p->batch < 0) return DQB_ERR_INVALID_ARGUMENT;
  if (p->h_ndiag < 0 || (p->h_ndiag > 0 && (!p->h_offsets || !p->h_diags))) return DQB_ERR_INVALID_ARGUMENT;
  if (!p->rho0 || !p->tsave || (p->n_exp > 0 && !p->E)) return DQB_ERR_INVALID_ARGUMENT;
  if (p->n > kSeMaxN || p->batch > 65535 || p->h_ndiag > DQB_DIA_MAX_HNH_DIAGS) return DQB_ERR_UNSUPPORTED;
  int rc = check_opts(o, out, p->n_exp);
  if (rc) return rc;
  if (p->batch == 0) return DQB_OK;
  SeOps d;
  std::memset(&d, 0, sizeof(d));
  d.n = p->n;
  d.dia = 1;
  d.nd = p->h_ndiag;
  for (int q = 0; q < d.nd; ++q) {
    if (p->h_offsets[q] <= -p->n || p->h_offsets[q] >= p->n) return DQB_ERR_INVALID_ARGUMENT;
    d.off[q] = p->h_offsets[q];
  }
  d.H = (const float2*)p->h_diags;
  d.Hidx = p->H_index;
  return run(d, p->n_exp, p->n_tsave, p->batch, p->rho0, p->rho0_index, p->E, p->tsave, o, out, workspace,
             workspace_bytes, (cudaStream_t)stream, td);
}

extern "C" int dqb_sesolve_dia(const dqb_dia_problem* p, const dqb_ode_options* o, const dqb_outputs* out,
                               void* workspace, size_t workspace_bytes, void* stream) {
  return sesolve_dia(p, nullptr, o, out, workspace, workspace_bytes, stream);
}

extern "C" int dqb_sesolve_dia_td(const dqb_dia_problem* p, const dqb_td_hamiltonian* td, const dqb_ode_options* o,
                                  const dqb_outputs* out, void* workspace, size_t workspace_bytes, void* stream) {
  if (!td) return DQB_ERR_INVALID_ARGUMENT;
  return sesolve_dia(p, td, o, out, workspace, workspace_bytes, stream);
}
