// graph_replay.cuh -- replay of a single-matrix call's launches as a CUDA graph.
//
// After its one host readback (the 1-norm that picks the plan), expm and its
// adjoint only enqueue kernels and look-ahead events on the caller's stream.
// Those launches depend on nothing but the call's configuration (size, plan,
// pointers, stream, the handle's settings), which the caller folds into a key.
// A configuration seen for the first time runs directly; seen again right
// after, it is captured once and replayed from then on (one graph launch
// instead of one launch per kernel and event).
#pragma once

#include <cstdint>
#include <type_traits>

#include "kernels.cuh"

namespace clm {

// The handle's graph slot of each element type.
template <typename T> constexpr int type_slot() {
  return std::is_same<T, float>::value    ? 0
         : std::is_same<T, double>::value ? 1
         : std::is_same<T, float2>::value ? 2
                                          : 3;
}

// FNV-1a over the 64-bit words of a call's configuration.
struct CallKey {
  unsigned long long h = 1469598103934665603ull;
  void mix(unsigned long long v) { h = (h ^ v) * 1099511628211ull; }
  void mix(const void *p) { mix((unsigned long long)reinterpret_cast<std::uintptr_t>(p)); }
};

// Runs `launch` (enqueue only, no host synchronisation) directly, or replays
// the graph held in `g` when `key` matches it. Never while kernel timing is
// on, on the legacy default streams (not capturable) or on a thread that must
// create no CUDA resources (a NoLookAheadScope is open). A failed capture sets
// *enabled to 0, and the call and every later one run directly.
template <typename F>
calamanStatus_t run_or_replay(int *enabled, BatchedGraph &g, cudaStream_t st, unsigned long long key,
                              F &&launch) {
  if (enabled == nullptr || !*enabled || tl_timer != nullptr || tl_no_lookahead || st == nullptr ||
      st == cudaStreamLegacy || st == cudaStreamPerThread)
    return launch();
  if (g.exec != nullptr && g.key == key) {
    cudaError_t e = cudaGraphLaunch(static_cast<cudaGraphExec_t>(g.exec), st);
    if (e != cudaSuccess) return runtime_status(e);
    note_launch(g.launches);
    return ok_status();
  }
  if (g.seen != key) {  // first sighting: run directly
    g.seen = key;
    return launch();
  }
  const unsigned long long before = g_launch_count();
  cudaGraph_t graph = nullptr;
  calamanStatus_t ls = ok_status();
  cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    ls = launch();
    e = cudaStreamEndCapture(st, &graph);
  }
  cudaGraphExec_t exec = nullptr;
  if (e == cudaSuccess && is_ok(ls)) e = cudaGraphInstantiate(&exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (e != cudaSuccess || !is_ok(ls) || exec == nullptr) {  // run directly from now on
    cudaGetLastError();
    *enabled = 0;
    return launch();
  }
  if (g.exec) cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(g.exec));
  g.exec = exec;
  g.key = key;
  g.launches = (unsigned)(g_launch_count() - before);
  e = cudaGraphLaunch(exec, st);
  return e == cudaSuccess ? ok_status() : runtime_status(e);
}

}  // namespace clm
