// capi.cu -- extern "C" entry points declared in include/alluvion_b200.h:
// engine lifecycle, grid sort and the standalone neighbor update.
#include <string>

#include "boundary.cuh"
#include "engine.hpp"
#include "grid.cuh"
#include "neighbors.cuh"

namespace alb {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }
const std::string& get_error() { return g_last_error; }

}  // namespace alb

using namespace alb;

int al_engine::activate() const {
  ALB_CUDA(cudaSetDevice(device));
  return AL_OK;
}

int al_engine::buffer(const char* name, size_t bytes, void** out) {
  Scratch& s = ns.empty() ? scratch[name] : scratch[ns + name];
  if (s.bytes < bytes || s.ptr == nullptr) {
    if (s.ptr) {
      ALB_CUDA(cudaFree(s.ptr));
      s.ptr = nullptr;
      s.bytes = 0;
    }
    size_t want = bytes < 256 ? 256 : bytes;
    cudaError_t err = cudaMalloc(&s.ptr, want);
    if (err != cudaSuccess) {
      s.ptr = nullptr;
      set_error(std::string("cudaMalloc(") + name + ", " + std::to_string(want) +
                " bytes): " + cudaGetErrorString(err));
      return AL_ERR_ALLOC;
    }
    s.bytes = want;
    ++generation;  // captured graphs hold the old pointers
  }
  *out = s.ptr;
  return AL_OK;
}

int al_engine::host_pinned(size_t bytes, void** out) {
  if (pinned_bytes < bytes || pinned == nullptr) {
    if (pinned) ALB_CUDA(cudaFreeHost(pinned));
    pinned = nullptr;
    pinned_bytes = 0;
    ALB_CUDA(cudaMallocHost(&pinned, bytes));
    pinned_bytes = bytes;
    ++generation;
  }
  *out = pinned;
  return AL_OK;
}

cudaEvent_t al_engine::take_event() {
  if (!event_pool.empty()) {
    cudaEvent_t ev = event_pool.back();
    event_pool.pop_back();
    return ev;
  }
  cudaEvent_t ev = nullptr;
  if (cudaEventCreate(&ev) != cudaSuccess) return nullptr;
  return ev;
}

int al_engine::flush_stats() {
  for (Pending& p : pending) {
    float ms = 0;
    cudaError_t err = cudaEventElapsedTime(&ms, p.start, p.stop);
    event_pool.push_back(p.start);
    event_pool.push_back(p.stop);
    if (err != cudaSuccess) continue;
    Stat* s = nullptr;
    for (auto& kv : stats)
      if (kv.first == p.name) s = &kv.second;
    if (!s) {
      stats.emplace_back(p.name, Stat{});
      s = &stats.back().second;
    }
    s->total_ms += ms;
    s->count += 1;
  }
  pending.clear();
  return AL_OK;
}

namespace alb {
LaunchScope::LaunchScope(al_engine* e_, const char* name_, cudaStream_t st_, int kernels)
    : e(e_), name(name_), st(st_) {
  e->launches += uint64_t(kernels);
  if (e->profiling) {
    start = e->take_event();
    if (start) cudaEventRecord(start, st);
  }
}
LaunchScope::~LaunchScope() {
  if (!start) return;
  cudaEvent_t stop = e->take_event();
  if (!stop) return;
  cudaEventRecord(stop, st);
  e->pending.push_back(al_engine::Pending{name, start, stop});
}
}  // namespace alb

int al_engine::capture_streams() {
  if (!capture_stream)
    ALB_CUDA(cudaStreamCreateWithFlags(&capture_stream, cudaStreamNonBlocking));
  if (!body_stream) ALB_CUDA(cudaStreamCreateWithFlags(&body_stream, cudaStreamNonBlocking));
  return AL_OK;
}

int al_engine::branches(uint32_t count) {
  if (!fork_event) ALB_CUDA(cudaEventCreateWithFlags(&fork_event, cudaEventDisableTiming));
  while (branch_streams.size() < count) {
    cudaStream_t s = nullptr;
    ALB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    branch_streams.push_back(s);
    cudaEvent_t ev = nullptr;
    ALB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    join_events.push_back(ev);
  }
  return AL_OK;
}

void al_engine::drop_graphs() {
  for (Graph& g : graphs)
    if (g.exec) cudaGraphExecDestroy(g.exec);
  graphs.clear();
  seen_keys.clear();
}

al_engine::~al_engine() {
  cudaSetDevice(device);
  drop_graphs();
  if (capture_stream) cudaStreamDestroy(capture_stream);
  if (body_stream) cudaStreamDestroy(body_stream);
  for (cudaStream_t s : branch_streams) cudaStreamDestroy(s);
  for (cudaEvent_t ev : join_events) cudaEventDestroy(ev);
  if (fork_event) cudaEventDestroy(fork_event);
  for (auto& kv : scratch)
    if (kv.second.ptr) cudaFree(kv.second.ptr);
  if (pinned) cudaFreeHost(pinned);
  for (Pending& p : pending) {
    cudaEventDestroy(p.start);
    cudaEventDestroy(p.stop);
  }
  for (cudaEvent_t ev : event_pool) cudaEventDestroy(ev);
}

extern "C" {

const char* al_status_string(int status) {
  switch (status) {
    case AL_OK: return "ok";
    case AL_ERR_CUDA: return "CUDA runtime error";
    case AL_ERR_INVALID: return "invalid argument";
    case AL_ERR_OUT_OF_GRID: return "particle outside the grid (grid_anomaly[0])";
    case AL_ERR_CELL_OVERFLOW: return "cell capacity exceeded (grid_anomaly[1])";
    case AL_ERR_NEIGHBOR_OVERFLOW: return "neighbor capacity exceeded (grid_anomaly[2])";
    case AL_ERR_UNSUPPORTED: return "unsupported option";
    case AL_ERR_TIMEOUT: return "bounded device wait timed out";
    case AL_ERR_NO_DEVICE: return "no sm_100 CUDA device";
    case AL_ERR_ALLOC: return "device allocation failed";
    default: return "unknown status";
  }
}

const char* al_last_error(void) { return get_error().c_str(); }

int al_engine_create(int device, al_engine** out) {
  ALB_CHECK_ARG(out != nullptr, "al_engine_create: out is null");
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    set_error("al_engine_create: no CUDA device " + std::to_string(device));
    return AL_ERR_NO_DEVICE;
  }
  cudaDeviceProp prop;
  ALB_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major != 10) {
    set_error("al_engine_create: device " + std::to_string(device) + " is sm_" +
              std::to_string(prop.major) + std::to_string(prop.minor) +
              "; this build targets sm_100a");
    return AL_ERR_NO_DEVICE;
  }
  ALB_CUDA(cudaSetDevice(device));
  ALB_TRY(upload_peirce_tables(nullptr));
  al_engine* e = new al_engine();
  e->device = device;
  e->num_sms = prop.multiProcessorCount;
  *out = e;
  return AL_OK;
}

int al_engine_destroy(al_engine* engine) {
  delete engine;
  return AL_OK;
}

int al_engine_synchronize(al_engine* engine, void* stream) {
  ALB_CHECK_ARG(engine != nullptr, "al_engine_synchronize: engine is null");
  ALB_TRY(engine->activate());
  ALB_CUDA(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  return engine->flush_stats();
}

int al_allocate(al_engine* engine, void** ptr, size_t bytes) {
  ALB_CHECK_ARG(engine && ptr, "al_allocate: null argument");
  *ptr = nullptr;
  if (bytes == 0) return AL_OK;
  ALB_TRY(engine->activate());
  if (cudaMalloc(ptr, bytes) != cudaSuccess) {
    cudaGetLastError();
    *ptr = nullptr;
    set_error("al_allocate: cudaMalloc of " + std::to_string(bytes) + " bytes failed");
    return AL_ERR_ALLOC;
  }
  return AL_OK;
}

int al_free(al_engine* engine, void* ptr) {
  ALB_CHECK_ARG(engine != nullptr, "al_free: engine is null");
  if (!ptr) return AL_OK;
  ALB_TRY(engine->activate());
  ALB_CUDA(cudaFree(ptr));
  return AL_OK;
}

int al_copy(al_engine* engine, void* dst, const void* src, size_t bytes) {
  ALB_CHECK_ARG(engine != nullptr, "al_copy: engine is null");
  if (bytes == 0) return AL_OK;
  ALB_CHECK_ARG(dst && src, "al_copy: null pointer");
  ALB_TRY(engine->activate());
  ALB_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDefault));
  return AL_OK;
}

int al_set(al_engine* engine, void* dst, int value, size_t bytes) {
  ALB_CHECK_ARG(engine != nullptr, "al_set: engine is null");
  if (bytes == 0) return AL_OK;
  ALB_CHECK_ARG(dst != nullptr, "al_set: null pointer");
  ALB_TRY(engine->activate());
  ALB_CUDA(cudaMemset(dst, value, bytes));
  ALB_CUDA(cudaDeviceSynchronize());
  return AL_OK;
}

int al_engine_set_graph_mode(al_engine* engine, int enable) {
  ALB_CHECK_ARG(engine != nullptr, "al_engine_set_graph_mode: engine is null");
  engine->graph_mode = enable != 0;
  return AL_OK;
}

int al_engine_graph_stats(al_engine* engine, uint64_t* captures, uint64_t* replays) {
  ALB_CHECK_ARG(engine && captures && replays, "al_engine_graph_stats: null argument");
  *captures = engine->graph_captures;
  *replays = engine->graph_replays;
  return AL_OK;
}

int al_engine_set_profiling(al_engine* engine, int enable) {
  ALB_CHECK_ARG(engine != nullptr, "al_engine_set_profiling: engine is null");
  engine->profiling = enable != 0;
  return AL_OK;
}

int al_engine_reset_stats(al_engine* engine) {
  ALB_CHECK_ARG(engine != nullptr, "al_engine_reset_stats: engine is null");
  ALB_TRY(engine->activate());
  ALB_CUDA(cudaDeviceSynchronize());
  engine->flush_stats();
  engine->stats.clear();
  engine->launches = 0;
  return AL_OK;
}

int al_engine_launch_count(al_engine* engine, uint64_t* count) {
  ALB_CHECK_ARG(engine && count, "al_engine_launch_count: null argument");
  *count = engine->launches;
  return AL_OK;
}

int al_engine_kernel_stat(al_engine* engine, uint32_t index, char* name, size_t name_len,
                          double* total_ms, uint64_t* count) {
  ALB_CHECK_ARG(engine && name && name_len && total_ms && count,
                "al_engine_kernel_stat: null argument");
  engine->flush_stats();
  if (index >= engine->stats.size()) {
    set_error("al_engine_kernel_stat: index past the last entry");
    return AL_ERR_INVALID;
  }
  const auto& kv = engine->stats[index];
  std::snprintf(name, name_len, "%s", kv.first.c_str());
  *total_ms = kv.second.total_ms;
  *count = kv.second.count;
  return AL_OK;
}

}  // extern "C"

namespace {

// Reads the device anomaly flags after `st` drains and maps them to a status.
int anomaly_status(const uint32_t* flags_dev, cudaStream_t st, uint32_t* host_copy) {
  uint32_t f[4] = {0, 0, 0, 0};
  ALB_CUDA(cudaMemcpyAsync(f, flags_dev, sizeof(f), cudaMemcpyDeviceToHost, st));
  ALB_CUDA(cudaStreamSynchronize(st));
  if (host_copy)
    for (int k = 0; k < 3; ++k) host_copy[k] = f[k];
  if (f[0]) return AL_ERR_OUT_OF_GRID;
  if (f[1]) return AL_ERR_CELL_OVERFLOW;
  if (f[2]) return AL_ERR_NEIGHBOR_OVERFLOW;
  return AL_OK;
}

int check_consti(const al_consti* cni) {
  ALB_CHECK_ARG(cni != nullptr, "consti is null");
  ALB_CHECK_ARG(cni->grid_res[0] > 0 && cni->grid_res[1] > 0 && cni->grid_res[2] > 0,
                "grid_res must be positive");
  ALB_CHECK_ARG(uint64_t(cni->grid_res[0]) * cni->grid_res[1] * cni->grid_res[2] < (1ull << 31),
                "grid has too many cells");
  ALB_CHECK_ARG(cni->max_num_neighbors_per_particle > 0, "max_num_neighbors_per_particle is 0");
  ALB_CHECK_ARG(cni->num_boundaries <= AL_MAX_BOUNDARIES, "too many boundaries");
  return AL_OK;
}

template <class TF, class C>
int grid_sort_impl(al_engine* e, const C* cn, const al_consti* cni, const TF* x, uint32_t n,
                   uint32_t* particle_cell, uint32_t* sorted_to_original, uint32_t* cell_start,
                   uint32_t* pid_length, void* stream) {
  ALB_CHECK_ARG(e && cn && (x || n == 0), "al_grid_sort: null argument");
  ALB_CHECK_ARG(n == 0 || (particle_cell && sorted_to_original), "al_grid_sort: null output");
  ALB_TRY(check_consti(cni));
  ALB_TRY(e->activate());
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  Cn<TF> c = to_cn<TF>(*cn);
  GridDims g = to_dims(*cni);
  vec4<TF>* xs = nullptr;
  uint32_t* flags = nullptr;
  ALB_TRY(e->buf("sorted.x", n, &xs));
  ALB_TRY(e->buf("flags", 4, &flags));
  ALB_CUDA(cudaMemsetAsync(flags, 0, 4 * sizeof(uint32_t), st));
  GridState gs;
  ALB_TRY(grid_build<TF>(e, c, g, x, n, xs, flags, gs, st));
  if (n > 0) {
    ALB_CUDA(
        cudaMemcpyAsync(particle_cell, gs.cell, size_t(n) * 4, cudaMemcpyDeviceToDevice, st));
    ALB_CUDA(cudaMemcpyAsync(sorted_to_original, gs.perm, size_t(n) * 4,
                             cudaMemcpyDeviceToDevice, st));
  }
  if (cell_start)
    ALB_CUDA(cudaMemcpyAsync(cell_start, gs.cell_start, (size_t(g.ncells) + 1) * 4,
                             cudaMemcpyDeviceToDevice, st));
  if (pid_length)
    ALB_CUDA(cudaMemcpyAsync(pid_length, gs.count, size_t(g.ncells) * 4, cudaMemcpyDeviceToDevice,
                             st));
  return anomaly_status(flags, st, nullptr);
}

template <class TF, class C>
int update_neighbors_impl(al_engine* e, const C* cn, const al_consti* cni, const TF* x,
                          uint32_t n, const TF* boundary_kernel, TF* density, uint32_t* num_nbr,
                          TF* neighbors, uint32_t* grid_anomaly, void* stream,
                          double wrap_length = 0) {
  ALB_CHECK_ARG(e && cn && ((x && num_nbr) || n == 0),
                "al_update_particle_neighbors: null argument");
  ALB_TRY(check_consti(cni));
  ALB_CHECK_ARG(cni->num_boundaries == 0 || boundary_kernel != nullptr,
                "al_update_particle_neighbors: boundary kernel required when num_boundaries > 0");
  ALB_TRY(e->activate());
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  Cn<TF> c = to_cn<TF>(*cn);
  if (wrap_length > 0) set_wrap(c, TF(wrap_length));  // update_particle_neighbors<1>
  GridDims g = to_dims(*cni);
  vec4<TF>* xs = nullptr;
  uint32_t *flags = nullptr, *nbr = nullptr, *ncount = nullptr;
  TF* rho = nullptr;
  ALB_TRY(e->buf("sorted.x", size_t(n) + kSortedPad, &xs));
  ALB_TRY(e->buf("flags", 4, &flags));
  ALB_TRY(e->buf("nbr.list", size_t(n) * g.cap_nbr, &nbr));
  ALB_TRY(e->buf("nbr.count", n, &ncount));
  ALB_TRY(e->buf("sorted.rho", n, &rho));
  ALB_CUDA(cudaMemsetAsync(flags, 0, 4 * sizeof(uint32_t), st));
  GridState gs;
  ALB_TRY(grid_build<TF>(e, c, g, x, n, xs, flags, gs, st));
  RefBoundaryKernel<TF> bk{boundary_kernel, gs.perm, n, g.nb};
  ALB_TRY(build_neighbors_density<TF>(c, g, gs, xs, bk, nbr, ncount, rho, nullptr, nullptr, st));
  ALB_TRY(export_neighbors<TF>(c, g, gs, xs, nbr, ncount, rho, neighbors, num_nbr, density, st));
  if (grid_anomaly)
    ALB_CUDA(cudaMemcpyAsync(grid_anomaly, flags, 3 * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                             st));
  return anomaly_status(flags, st, nullptr);
}

}  // namespace

extern "C" {

int al_grid_sort_f32(al_engine* engine, const al_const_f32* cn, const al_consti* cni,
                     const float* particle_x, uint32_t num_particles, uint32_t* particle_cell,
                     uint32_t* sorted_to_original, uint32_t* cell_start, uint32_t* pid_length,
                     void* stream) {
  return grid_sort_impl<float>(engine, cn, cni, particle_x, num_particles, particle_cell,
                               sorted_to_original, cell_start, pid_length, stream);
}
int al_grid_sort_f64(al_engine* engine, const al_const_f64* cn, const al_consti* cni,
                     const double* particle_x, uint32_t num_particles, uint32_t* particle_cell,
                     uint32_t* sorted_to_original, uint32_t* cell_start, uint32_t* pid_length,
                     void* stream) {
  return grid_sort_impl<double>(engine, cn, cni, particle_x, num_particles, particle_cell,
                                sorted_to_original, cell_start, pid_length, stream);
}

int al_update_particle_neighbors_f32(al_engine* engine, const al_const_f32* cn,
                                     const al_consti* cni, const float* particle_x,
                                     uint32_t num_particles,
                                     const float* particle_boundary_kernel,
                                     float* particle_density, uint32_t* particle_num_neighbors,
                                     float* particle_neighbors, uint32_t* grid_anomaly,
                                     void* stream) {
  return update_neighbors_impl<float>(engine, cn, cni, particle_x, num_particles,
                                      particle_boundary_kernel, particle_density,
                                      particle_num_neighbors, particle_neighbors, grid_anomaly,
                                      stream);
}
int al_update_particle_neighbors_f64(al_engine* engine, const al_const_f64* cn,
                                     const al_consti* cni, const double* particle_x,
                                     uint32_t num_particles,
                                     const double* particle_boundary_kernel,
                                     double* particle_density, uint32_t* particle_num_neighbors,
                                     double* particle_neighbors, uint32_t* grid_anomaly,
                                     void* stream) {
  return update_neighbors_impl<double>(engine, cn, cni, particle_x, num_particles,
                                       particle_boundary_kernel, particle_density,
                                       particle_num_neighbors, particle_neighbors, grid_anomaly,
                                       stream);
}

int al_update_particle_neighbors_periodic_f32(al_engine* engine, const al_const_f32* cn,
                                              const al_consti* cni, const float* particle_x,
                                              uint32_t num_particles,
                                              const float* particle_boundary_kernel,
                                              float* particle_density,
                                              uint32_t* particle_num_neighbors,
                                              float* particle_neighbors, uint32_t* grid_anomaly,
                                              double wrap_length, void* stream) {
  ALB_CHECK_ARG(wrap_length > 0, "al_update_particle_neighbors_periodic: wrap_length <= 0");
  return update_neighbors_impl<float>(engine, cn, cni, particle_x, num_particles,
                                      particle_boundary_kernel, particle_density,
                                      particle_num_neighbors, particle_neighbors, grid_anomaly,
                                      stream, wrap_length);
}
int al_update_particle_neighbors_periodic_f64(al_engine* engine, const al_const_f64* cn,
                                              const al_consti* cni, const double* particle_x,
                                              uint32_t num_particles,
                                              const double* particle_boundary_kernel,
                                              double* particle_density,
                                              uint32_t* particle_num_neighbors,
                                              double* particle_neighbors, uint32_t* grid_anomaly,
                                              double wrap_length, void* stream) {
  ALB_CHECK_ARG(wrap_length > 0, "al_update_particle_neighbors_periodic: wrap_length <= 0");
  return update_neighbors_impl<double>(engine, cn, cni, particle_x, num_particles,
                                       particle_boundary_kernel, particle_density,
                                       particle_num_neighbors, particle_neighbors, grid_anomaly,
                                       stream, wrap_length);
}

}  // extern "C"
