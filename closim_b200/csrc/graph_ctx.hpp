// Building blocks of a graph-captured step: conditional nodes (IF / WHILE)
// whose bodies are captured from streams, nested to any depth.
//
// A step graph is captured once from the solver's stream and replayed; every
// decision the host-driven step takes between launches (accept or halve the
// Armijo step, stop Newton, rebuild the broadphase superset) is taken instead by
// a one-thread kernel that sets a conditional handle (cudaGraphSetConditional),
// so a replay needs no host round trip.
#pragma once
#include <cuda_runtime.h>

#include <stdexcept>
#include <string>
#include <vector>

namespace cs {

struct GraphError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define GCK(x)                                                                                   \
  do {                                                                                           \
    cudaError_t e_ = (x);                                                                        \
    if (e_ != cudaSuccess) throw GraphError(std::string(#x) + ": " + cudaGetErrorString(e_));    \
  } while (0)

class GraphCtx {
 public:
  // The stream captured into at the current nesting depth.
  cudaStream_t cur() const { return stack_.back(); }

  // Begins a capture of the whole step on `s`; returns the graph under construction.
  void begin(cudaStream_t s) {
    stack_.assign(1, s);
    GCK(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
  }
  cudaGraph_t end() {
    cudaGraph_t g = nullptr;
    GCK(cudaStreamEndCapture(stack_.front(), &g));
    stack_.clear();
    return g;
  }

  // A new conditional handle for a node to be added at the current depth.
  cudaGraphConditionalHandle handle(unsigned defaultValue) {
    cudaGraph_t g = graph_here();
    cudaGraphConditionalHandle h;
    GCK(cudaGraphConditionalHandleCreate(&h, g, defaultValue, cudaGraphCondAssignDefault));
    return h;
  }

  // Adds an IF (or WHILE) node after the work captured so far at this depth and
  // continues capturing into its body on a pooled stream; close with pop().
  void push(cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type) {
    cudaStream_t s = cur();
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    GCK(cudaStreamGetCaptureInfo(s, &st, nullptr, &g, &deps, &nd));
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    GCK(cudaGraphAddNode(&node, g, deps, nd, &p));
    GCK(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    cudaStream_t body = pooled(stack_.size());
    GCK(cudaStreamBeginCaptureToGraph(body, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeRelaxed));
    stack_.push_back(body);
  }
  void pop() {
    cudaGraph_t g = nullptr;
    GCK(cudaStreamEndCapture(stack_.back(), &g));
    stack_.pop_back();
  }

  ~GraphCtx() {
    for (cudaStream_t s : pool_) cudaStreamDestroy(s);
  }

 private:
  std::vector<cudaStream_t> stack_;
  std::vector<cudaStream_t> pool_;

  cudaGraph_t graph_here() {
    cudaStreamCaptureStatus st;
    cudaGraph_t g = nullptr;
    GCK(cudaStreamGetCaptureInfo(cur(), &st, nullptr, &g, nullptr, nullptr));
    return g;
  }
  cudaStream_t pooled(size_t depth) {
    while (pool_.size() < depth) {
      cudaStream_t s;
      GCK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      pool_.push_back(s);
    }
    return pool_[depth - 1];
  }
};

}  // namespace cs
