// Host helpers shared by the large-problem entry points: the CUDA graph that runs the
// RK loop as a device-side WHILE node, and a small cache of its executables.
#pragma once

#include <cstdlib>

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <vector>

namespace dqb {

// Executable graphs keyed by the bytes of the launch parameters (pointers and sizes):
// a repeated call with the same buffers reuses its executable.  An evicted executable may
// still be running, so it is parked with an event recorded on the stream it was last
// launched on and destroyed once that event has completed (checked without blocking on
// every later insert).
class GraphCache {
 public:
  struct Entry {
    std::vector<unsigned char> key;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t stream = nullptr;
  };
  struct Parked {
    cudaGraphExec_t exec;
    cudaEvent_t done;
  };

  cudaGraphExec_t find(const void* key, size_t len) {
    std::lock_guard<std::mutex> lock(mu_);
    for (auto& e : entries_)
      if (e.key.size() == len && std::memcmp(e.key.data(), key, len) == 0) return e.exec;
    return nullptr;
  }

  void insert(const void* key, size_t len, cudaGraphExec_t exec, cudaStream_t s) {
    std::lock_guard<std::mutex> lock(mu_);
    reap();
    if (entries_.size() >= kMax) {
      Entry& old = entries_.front();
      Parked p{old.exec, nullptr};
      if (cudaEventCreateWithFlags(&p.done, cudaEventDisableTiming) == cudaSuccess &&
          cudaEventRecord(p.done, old.stream) == cudaSuccess) {
        parked_.push_back(p);
      } else {  // no event: wait for the stream instead
        if (p.done) cudaEventDestroy(p.done);
        cudaStreamSynchronize(old.stream);
        cudaGraphExecDestroy(old.exec);
      }
      entries_.erase(entries_.begin());
    }
    Entry e;
    e.key.assign((const unsigned char*)key, (const unsigned char*)key + len);
    e.exec = exec;
    e.stream = s;
    entries_.push_back(std::move(e));
  }

  void touch(const void* key, size_t len, cudaStream_t s) {
    std::lock_guard<std::mutex> lock(mu_);
    for (auto& e : entries_)
      if (e.key.size() == len && std::memcmp(e.key.data(), key, len) == 0) e.stream = s;
  }

 private:
  void reap() {
    for (size_t i = 0; i < parked_.size();) {
      if (cudaEventQuery(parked_[i].done) == cudaSuccess) {
        cudaGraphExecDestroy(parked_[i].exec);
        cudaEventDestroy(parked_[i].done);
        parked_.erase(parked_.begin() + i);
      } else {
        ++i;
      }
    }
  }

  static constexpr size_t kMax = 64;
  std::mutex mu_;
  std::vector<Entry> entries_;
  std::vector<Parked> parked_;
};

// DQB_HOST_LOOP=1 in the environment (read once): run the RK loop from the host, one
// iteration per round trip, instead of as a graph WHILE node.  Same kernels, same
// results; it exists for profilers that cannot see kernels inside conditional graphs.
inline bool host_loop_requested() {
  static const bool on = [] {
    const char* v = std::getenv("DQB_HOST_LOOP");
    return v != nullptr && v[0] == '1';
  }();
  return on;
}

// Host-driven form of "WHILE (cond) { body }": `body(stream, 0, flag)` enqueues one
// iteration whose last kernel writes the condition to the device word `flag`; the call
// returns when it reads 0.  Synchronises `stream` once per iteration.
template <class Body>
cudaError_t run_host_loop(Body body, int* flag, cudaStream_t s) {
  for (;;) {
    body(s, cudaGraphConditionalHandle(0), flag);
    int more = 0;
    cudaError_t err = cudaMemcpyAsync(&more, flag, sizeof(int), cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err == cudaSuccess) err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    if (!more) return cudaSuccess;
  }
}

// Build "WHILE (cond) { body }" where `body(stream, handle, nullptr)` enqueues one loop
// iteration on the capture stream and must end with a kernel that sets the condition.
template <class Body>
cudaError_t build_while_graph(Body body, cudaGraphExec_t* out) {
  cudaGraph_t g = nullptr;
  cudaError_t err = cudaGraphCreate(&g, 0);
  if (err != cudaSuccess) return err;
  cudaGraphConditionalHandle handle;
  err = cudaGraphConditionalHandleCreate(&handle, g, 1, cudaGraphCondAssignDefault);
  if (err == cudaSuccess) {
    cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = handle;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    err = cudaGraphAddNode(&node, g, nullptr, 0, &p);
    if (err == cudaSuccess) {
      cudaGraph_t bodyg = p.conditional.phGraph_out[0];
      cudaStream_t cap;
      err = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
      if (err == cudaSuccess) {
        err = cudaStreamBeginCaptureToGraph(cap, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
        if (err == cudaSuccess) {
          body(cap, handle, (int*)nullptr);
          cudaError_t e2 = cudaStreamEndCapture(cap, &bodyg);
          if (err == cudaSuccess) err = e2;
          if (err == cudaSuccess) err = cudaGetLastError();
        }
        cudaStreamDestroy(cap);
      }
      if (err == cudaSuccess) err = cudaGraphInstantiate(out, g, 0);
    }
  }
  cudaGraphDestroy(g);
  return err;
}

}  // namespace dqb
