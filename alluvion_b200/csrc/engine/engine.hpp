// engine.hpp -- host-side engine context: device binding, scratch buffers,
// error reporting.  Shared by the engine's translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <map>
#include <string>
#include <tuple>
#include <unordered_map>
#include <utility>
#include <vector>

#include "alluvion_b200.h"

namespace alb {

// Thread-local message of the last failing call (al_last_error).
void set_error(const std::string& msg);
const std::string& get_error();

// Evaluates a CUDA runtime call; on failure records the message and returns
// AL_ERR_CUDA from the enclosing function.
#define ALB_CUDA(call)                                                          \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      ::alb::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));     \
      return AL_ERR_CUDA;                                                       \
    }                                                                           \
  } while (0)

// Propagates a non-zero al_status.
#define ALB_TRY(expr)          \
  do {                         \
    int s_ = (expr);           \
    if (s_ != AL_OK) return s_; \
  } while (0)

#define ALB_CHECK_ARG(cond, msg)        \
  do {                                  \
    if (!(cond)) {                      \
      ::alb::set_error(msg);            \
      return AL_ERR_INVALID;            \
    }                                   \
  } while (0)

// A named, growable device buffer.  Capacity only grows; contents are not
// preserved across growth.
struct Scratch {
  void* ptr = nullptr;
  size_t bytes = 0;
};

}  // namespace alb

struct al_engine;

namespace alb {
// Records one named launch group (`kernels` launches) on `st`: counts the
// launches and, while profiling is on, brackets them with CUDA events.
struct LaunchScope {
  al_engine* e;
  const char* name;
  cudaStream_t st;
  cudaEvent_t start = nullptr;
  LaunchScope(al_engine* e_, const char* name_, cudaStream_t st_, int kernels);
  ~LaunchScope();
};
}  // namespace alb

#define ALB_LAUNCH(eng, name, nk, st, ...)           \
  do {                                               \
    ::alb::LaunchScope ls_((eng), (name), (st), (nk)); \
    __VA_ARGS__;                                     \
  } while (0)

struct al_engine {
  int device = 0;
  int num_sms = 0;
  std::unordered_map<std::string, alb::Scratch> scratch;
  // launch statistics (al_engine_set_profiling / al_engine_kernel_stat)
  struct Stat {
    double total_ms = 0;
    uint64_t count = 0;
  };
  bool profiling = false;
  uint64_t launches = 0;
  std::vector<std::pair<std::string, Stat>> stats;  // insertion order
  struct Pending {
    const char* name;
    cudaEvent_t start, stop;
  };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> event_pool;
  cudaEvent_t take_event();
  // Accumulates the elapsed times of recorded launches (after a sync).
  int flush_stats();

  // Captured step graphs (al_engine_set_graph_mode).  `generation` counts
  // scratch reallocations; a graph whose key (sizes, caller pointers,
  // generation) no longer matches is recaptured.
  struct Graph {
    std::vector<uint64_t> key;
    cudaGraphExec_t exec = nullptr;
    uint32_t fixed_launches = 0;
  };
  bool graph_mode = true;
  uint64_t generation = 0;
  uint64_t graph_captures = 0, graph_replays = 0;
  std::vector<std::vector<uint64_t>> seen_keys;  // keys run eagerly once
  std::vector<Graph> graphs;
  cudaStream_t capture_stream = nullptr;
  cudaStream_t body_stream = nullptr;
  int capture_streams();  // creates the two capture streams on first use
  void drop_graphs();
  // Batched steps: one capture branch (stream + join event) per scene, a
  // fork event, and the buffer namespace of the scene being prepared or
  // enqueued ("" outside batches).
  std::vector<cudaStream_t> branch_streams;
  std::vector<cudaEvent_t> join_events;
  cudaEvent_t fork_event = nullptr;
  int branches(uint32_t count);  // creates streams / events up to `count`
  std::string ns;
  // Batched steps run fused (one launch per solver pass over all scenes)
  // unless disabled (al_engine_set_batch_fused) or their scenes rule it out;
  // the
  // block -> scene tables last uploaded for a fused batch, with their
  // buffers, and that batch's graph key.
  bool batch_fused = true;
  std::vector<unsigned char> fused_tables;
  std::vector<uint64_t> fused_key;
  // pinned host staging (control readback, reports)
  void* pinned = nullptr;
  size_t pinned_bytes = 0;

  // Launch shapes of the tunable pass groups (al_engine_set_launch_shape):
  // (group, particle-count bucket floor(log2 n), context 0 single / 1 batch)
  // -> (threads per block, threads per particle).  Entries override the
  // defaults; setting one invalidates the captured graphs.
  std::map<std::tuple<std::string, uint32_t, uint32_t>, std::pair<uint32_t, uint32_t>> shapes;
  // The caller's particle_x of the last learned-warm-start step per buffer
  // namespace: a step with other buffers is a new scene and starts its gate
  // afresh.
  std::unordered_map<std::string, const void*> warm_owner;

  // Returns a device buffer of at least `bytes` under `name`.
  int buffer(const char* name, size_t bytes, void** out);
  template <class T>
  int buf(const char* name, size_t count, T** out) {
    return buffer(name, count * sizeof(T), reinterpret_cast<void**>(out));
  }
  // As buf(); *fresh tells whether the buffer was (re)allocated by this call.
  template <class T>
  int buf(const char* name, size_t count, T** out, bool* fresh) {
    const uint64_t g0 = generation;  // buffer() counts every allocation it makes
    const int rc = buffer(name, count * sizeof(T), reinterpret_cast<void**>(out));
    *fresh = rc == AL_OK && generation != g0;
    return rc;
  }
  int host_pinned(size_t bytes, void** out);
  int activate() const;
  ~al_engine();
};
