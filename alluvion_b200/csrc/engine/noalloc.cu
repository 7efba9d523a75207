// noalloc.cu -- a grid sort that allocates nothing.
//
// Some callers cannot let a library call cudaMalloc: a renderer or game
// engine that owns the device memory budget and forbids plugins from
// allocating behind its back, or a real-time loop that cannot afford the
// implicit device synchronisation a cudaMalloc / cudaFree pair can cause.
// For them this file provides al_grid_sort_noalloc_f32: the same cell hash
// and stable counting sort as al_grid_sort_f32, with all of its scratch in
// one file-scope device array that is sized at compile time.  The caller
// still passes the inputs and the output buffers.
//
// The array is part of the library's device image.  Once the image is
// loaded on a GPU (with CUDA's lazy module loading, at this entry point's
// first call on that GPU) the GPU holds its 12.6 MiB until the process
// exits.  Every call shares it, so two calls that overlap on the GPU
// (different streams, or different host threads with no ordering between
// them) race and corrupt each other; callers must order them.  The array
// keeps the previous call's contents; the call clears what must start at
// zero (cell counts, anomaly flags).  Each call ends by reading the anomaly
// flags back to the host, which synchronises the caller's stream.
#include <mutex>
#include <string>

#include "grid.cuh"

namespace alb {
namespace {

// Largest problem the static scratch holds.
constexpr uint32_t kNoAllocMaxParticles = 1u << 20;  // 1,048,576 particles
constexpr uint32_t kNoAllocMaxCells = 1u << 20;      // 1,048,576 grid cells

constexpr size_t up64(size_t words) { return (words + 63) & ~size_t(63); }
constexpr size_t kScanTileWords = 256 * 8;
constexpr size_t kOffRank = 0;
constexpr size_t kOffCount = kOffRank + up64(kNoAllocMaxParticles);
constexpr size_t kOffStart = kOffCount + up64(size_t(kNoAllocMaxCells) + 1);
constexpr size_t kOffSums = kOffStart + up64(size_t(kNoAllocMaxCells) + 2);
constexpr size_t kOffFlags =
    kOffSums + up64((size_t(kNoAllocMaxCells) + 1 + kScanTileWords - 1) / kScanTileWords);
constexpr size_t kScratchWords = kOffFlags + 64;

// The scratch itself.  In host code its name is only a host-side stand-in,
// not a device address: the kernels receive the address obtained from
// cudaGetSymbolAddress below.
static __device__ __align__(256) uint32_t g_grid_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
uint32_t* g_scratch_addr[kMaxDevices] = {};

// Device address of g_grid_scratch on the current device, looked up once
// per device (with that device current) and cached.
int scratch_address(uint32_t** out) {
  int dev = 0;
  ALB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("al_grid_sort_noalloc: device ordinal out of range");
    return AL_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t err = cudaGetSymbolAddress(&p, g_grid_scratch);
    if (err != cudaSuccess || p == nullptr) {
      set_error(std::string("al_grid_sort_noalloc: cudaGetSymbolAddress failed: ") +
                cudaGetErrorString(err));
      return AL_ERR_CUDA;
    }
    g_scratch_addr[dev] = static_cast<uint32_t*>(p);
  }
  *out = g_scratch_addr[dev];
  return AL_OK;
}

}  // namespace
}  // namespace alb

using namespace alb;

extern "C" int al_grid_sort_noalloc_f32(const al_const_f32* cn, const al_consti* cni,
                                        const float* particle_x, uint32_t num_particles,
                                        uint32_t* particle_cell, uint32_t* sorted_to_original,
                                        uint32_t* cell_start, uint32_t* pid_length,
                                        void* stream) {
  ALB_CHECK_ARG(cn && cni, "al_grid_sort_noalloc: null argument");
  ALB_CHECK_ARG(cni->grid_res[0] > 0 && cni->grid_res[1] > 0 && cni->grid_res[2] > 0,
                "al_grid_sort_noalloc: grid_res must be positive");
  const uint64_t ncells = uint64_t(cni->grid_res[0]) * cni->grid_res[1] * cni->grid_res[2];
  if (num_particles > kNoAllocMaxParticles) {
    set_error("al_grid_sort_noalloc: " + std::to_string(num_particles) +
              " particles exceed the static scratch limit of " +
              std::to_string(kNoAllocMaxParticles));
    return AL_ERR_INVALID;
  }
  if (ncells > kNoAllocMaxCells) {
    set_error("al_grid_sort_noalloc: " + std::to_string(ncells) +
              " grid cells exceed the static scratch limit of " +
              std::to_string(kNoAllocMaxCells));
    return AL_ERR_INVALID;
  }
  ALB_CHECK_ARG(num_particles == 0 || (particle_x && particle_cell && sorted_to_original),
                "al_grid_sort_noalloc: null particle buffer");
  uint32_t* base = nullptr;
  ALB_TRY(scratch_address(&base));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const Cn<float> c = to_cn<float>(*cn);
  const GridDims g = to_dims(*cni);
  GridSortScratch sc{base + kOffRank, base + kOffCount, base + kOffStart, base + kOffSums,
                     base + kOffFlags};
  ALB_TRY(grid_sort_into<float>(c, g, particle_x, num_particles, particle_cell,
                                sorted_to_original, sc, st));
  if (cell_start)
    ALB_CUDA(cudaMemcpyAsync(cell_start, sc.start, (size_t(ncells) + 1) * sizeof(uint32_t),
                             cudaMemcpyDeviceToDevice, st));
  if (pid_length)
    ALB_CUDA(cudaMemcpyAsync(pid_length, sc.count, size_t(ncells) * sizeof(uint32_t),
                             cudaMemcpyDeviceToDevice, st));
  uint32_t f[4] = {0, 0, 0, 0};
  ALB_CUDA(cudaMemcpyAsync(f, sc.flags, sizeof(f), cudaMemcpyDeviceToHost, st));
  ALB_CUDA(cudaStreamSynchronize(st));
  if (f[0]) return AL_ERR_OUT_OF_GRID;
  if (f[1]) return AL_ERR_CELL_OVERFLOW;
  return AL_OK;
}
