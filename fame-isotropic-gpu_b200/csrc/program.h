// A recorded sequence of kernel launches with data-dependent WHILE loops.
//
// The same emit calls either launch directly on a stream with the loops run by
// the host (host-driven mode, the condition is read back after every iteration),
// or build one CUDA graph whose loops are conditional WHILE nodes set from device
// code (graph mode).  The solver records one batch of k-points once and replays
// the instantiated graph for every batch.
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <vector>

#include "state.cuh"

namespace fame {

struct CudaError : std::runtime_error {
  cudaError_t code;
  CudaError(cudaError_t c, const std::string& what) : std::runtime_error(what), code(c) {}
};

#define FAME_CK(call)                                                                      \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      throw ::fame::CudaError(e_, std::string(#call) + ": " + cudaGetErrorString(e_) +     \
                                      " (" + __FILE__ + ":" + std::to_string(__LINE__) + ")"); \
  } while (0)

class Program {
 public:
  Program(cudaStream_t s, bool graph, int* host_flag_buf, int max_host_iters)
      : stream_(s), graph_(graph), hflag_(host_flag_buf), max_iters_(max_host_iters) {
    if (graph_) {
      FAME_CK(cudaGraphCreate(&root_, 0));
      frames_.push_back({root_, nullptr});
    }
  }
  ~Program() {
    if (exec_) cudaGraphExecDestroy(exec_);
    if (root_) cudaGraphDestroy(root_);
  }
  Program(const Program&) = delete;
  Program& operator=(const Program&) = delete;

  bool graph_mode() const { return graph_; }

  template <typename... P, typename... A>
  void launch(void (*k)(P...), dim3 grid, dim3 block, size_t smem, A... args) {
    if (grid.x == 0 || grid.y == 0 || grid.z == 0) return;
    if (!graph_) {
      k<<<grid, block, smem, stream_>>>(args...);
      FAME_CK(cudaGetLastError());
      return;
    }
    auto vals = std::make_shared<std::tuple<P...>>(args...);
    void* ptrs[sizeof...(P) + 1];
    fill_ptrs(*vals, ptrs, std::index_sequence_for<P...>{});
    cudaKernelNodeParams kp = {};
    kp.func = reinterpret_cast<void*>(k);
    kp.gridDim = grid;
    kp.blockDim = block;
    kp.sharedMemBytes = (unsigned)smem;
    kp.kernelParams = ptrs;
    cudaGraphNode_t node;
    Frame& f = frames_.back();
    FAME_CK(cudaGraphAddKernelNode(&node, f.g, f.last ? &f.last : nullptr, f.last ? 1 : 0, &kp));
    f.last = node;
  }

  // Condition object for one WHILE loop; pass it to the kernels that set it.
  // `trips` (2 device ints) and `cap` bound the loop on the device.
  Cond make_cond(int* dflag, int* trips, int cap) {
    Cond c;
    c.flag = dflag;
    c.trips = trips;
    c.cap = cap;
    c.handle = 0;
    if (graph_) FAME_CK(cudaGraphConditionalHandleCreate(&c.handle, root_, 0, 0));
    return c;
  }

  // while (cond) body();  The condition must have been set by an earlier kernel.
  void while_loop(const Cond& c, const std::function<void()>& body) {
    if (!graph_) {
      for (int it = 0;; it++) {
        FAME_CK(cudaMemcpyAsync(hflag_, c.flag, sizeof(int), cudaMemcpyDeviceToHost, stream_));
        FAME_CK(cudaStreamSynchronize(stream_));
        if (!*hflag_) break;
        if (it >= max_iters_) throw std::runtime_error("host-driven loop exceeded its iteration cap");
        body();
      }
      return;
    }
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = c.handle;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    Frame& f = frames_.back();
    cudaGraphNode_t node;
    FAME_CK(cudaGraphAddNode(&node, f.g, f.last ? &f.last : nullptr, f.last ? 1 : 0, &np));
    f.last = node;
    cudaGraph_t body_graph = np.conditional.phGraph_out[0];
    frames_.push_back({body_graph, nullptr});
    body();
    frames_.pop_back();
  }

  void instantiate() {
    if (graph_ && !exec_) FAME_CK(cudaGraphInstantiate(&exec_, root_, 0));
  }
  void run() {
    if (graph_) {
      instantiate();
      FAME_CK(cudaGraphLaunch(exec_, stream_));
    }
  }

 private:
  struct Frame {
    cudaGraph_t g;
    cudaGraphNode_t last;
  };
  template <typename Tup, size_t... I>
  static void fill_ptrs(Tup& t, void** p, std::index_sequence<I...>) {
    ((p[I] = (void*)&std::get<I>(t)), ...);
  }
  cudaStream_t stream_;
  bool graph_;
  int* hflag_;
  int max_iters_;
  cudaGraph_t root_ = nullptr;
  cudaGraphExec_t exec_ = nullptr;
  std::vector<Frame> frames_;
};

}  // namespace fame
