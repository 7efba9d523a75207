// warmnet.cu -- tensor-core (tcgen05) inference and training kernels of
// the learned warm start (see warmnet.cuh).
//
// One CTA of 128 threads owns 128-particle tiles: thread r holds row r of
// the tile, which is TMEM lane r of every M = 128 accumulator.  Per layer
// the threads write their BF16 activations into a K-major shared-memory
// operand, one elected thread issues tcgen05.mma (A = activations, B =
// weights, D in TMEM) and commits to an mbarrier, and all threads read
// their row of D back with tcgen05.ld.  Every wait is bounded; a timeout
// raises an error flag, and the CTA stops issuing work, waits (bounded)
// for what it issued, frees its TMEM and returns.
#include <cuda_bf16.h>

#include "tc.cuh"
#include "warmnet.cuh"

namespace alb {

namespace {

inline uint32_t blocks_for(uint32_t n, int block) { return (n + block - 1) / block; }

constexpr uint32_t kTile = 128;              // particles per tile (MMA M)
constexpr long long kWaitCycles = 400000000; // ~0.2 s at 2 GHz
constexpr uint32_t kInferTmemCols = 256;     // D1 [0, 64), D2 [64, 128), D3 [128, 144)

// Shared-memory map of the inference kernel (bytes).
constexpr uint32_t kSmA1 = 0;                                   // [128][16] bf16
constexpr uint32_t kSmA2 = kSmA1 + kTile * kWarmInPad * 2;      // [128][64]
constexpr uint32_t kSmA3 = kSmA2 + kTile * kWarmHidden * 2;     // [128][64]
constexpr uint32_t kSmB1 = kSmA3 + kTile * kWarmHidden * 2;     // W1 [64][16]
constexpr uint32_t kSmB2 = kSmB1 + kWarmHidden * kWarmInPad * 2;   // W2 [64][64]
constexpr uint32_t kSmB3 = kSmB2 + kWarmHidden * kWarmHidden * 2;  // W3 [16][64]
constexpr uint32_t kSmBias = kSmB3 + kWarmOutPad * kWarmHidden * 2;  // b1, b2, b3 f32
constexpr uint32_t kSmBar = kSmBias + 1024;                     // mbarrier (8 B)
constexpr uint32_t kSmTmem = kSmBar + 8;                        // TMEM base (4 B)
constexpr uint32_t kSmUsed = kSmTmem + 8;
// Requested dynamic shared memory: more than a third of the SM's 228 KB,
// so at most two CTAs (2 x 256 TMEM columns of 512) share an SM and a TMEM
// allocation never waits for another CTA.
constexpr uint32_t kInferSmem = 100 * 1024;
static_assert(kSmUsed <= kInferSmem, "shared-memory map");

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// Writes 8 consecutive K values (k0 multiple of 8) of row r of a K-major
// [rows][K] bf16 tile as one 16-byte store.
__device__ __forceinline__ void put8(uint8_t* tile, uint32_t r, uint32_t k0, uint32_t K,
                                     const float* v) {
  uint4 q;
  q.x = pack_bf16(v[0], v[1]);
  q.y = pack_bf16(v[2], v[3]);
  q.z = pack_bf16(v[4], v[5]);
  q.w = pack_bf16(v[6], v[7]);
  *reinterpret_cast<uint4*>(tile + tc::kmajor_offset(r, k0, K)) = q;
}

// Loads a [N][K] weight block (source rows of length ksrc, rows >= nsrc
// and columns >= ksrc zero) into a K-major bf16 tile.  All threads.
__device__ __forceinline__ void load_weights(uint8_t* tile, const float* __restrict__ w,
                                             uint32_t N, uint32_t K, uint32_t nsrc,
                                             uint32_t ksrc) {
  for (uint32_t i = threadIdx.x; i < N * K; i += blockDim.x) {
    const uint32_t n = i / K, k = i % K;
    const float v = (n < nsrc && k < ksrc) ? w[n * ksrc + k] : 0.f;
    *reinterpret_cast<__nv_bfloat16*>(tile + tc::kmajor_offset(n, k, K)) = __float2bfloat16_rn(v);
  }
}

// Issues D (+)= A x B^T over K (multiple of 16) and commits; one thread.
__device__ __forceinline__ void issue_layer(uint32_t d_tmem, const uint8_t* a, const uint8_t* b,
                                            uint32_t K, uint32_t N, uint64_t* bar) {
  const uint32_t sa = tc::smem_u32(a), sb = tc::smem_u32(b);
  const uint32_t idesc = tc::idesc_bf16(kTile, N);
  for (uint32_t k = 0; k < K / 16; ++k)
    tc::mma_bf16(d_tmem, tc::tile_desc(sa, K, k), tc::tile_desc(sb, K, k), idesc, k > 0);
  tc::commit(bar);
}

// Makes the threads' shared-memory operand writes visible to the tensor
// cores and lets thread 0 issue a layer; then everyone waits for it.
// Returns false (in every thread) if any wait timed out.
__device__ __forceinline__ bool run_layer(uint32_t d_tmem, const uint8_t* a, const uint8_t* b,
                                          uint32_t K, uint32_t N, uint64_t* bar,
                                          uint32_t& phase, bool ok) {
  tc::fence_smem_to_async();
  tc::fence_before_sync();
  ok = __syncthreads_and(ok);
  if (!ok) return false;
  if (threadIdx.x == 0) {
    tc::fence_after_sync();
    issue_layer(d_tmem, a, b, K, N, bar);
  }
  ok = tc::mbar_wait(bar, phase, kWaitCycles);
  phase ^= 1u;
  tc::fence_after_sync();
  return __syncthreads_and(ok);
}

__global__ void __launch_bounds__(kTile)
    k_warm_forward(WarmNetDev net, const float* __restrict__ features, uint32_t n,
                   float* __restrict__ out, uint32_t* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t* A1 = sm + kSmA1;
  uint8_t* A2 = sm + kSmA2;
  uint8_t* A3 = sm + kSmA3;
  uint8_t* B1 = sm + kSmB1;
  uint8_t* B2 = sm + kSmB2;
  uint8_t* B3 = sm + kSmB3;
  float* bias = reinterpret_cast<float*>(sm + kSmBias);  // b1[64] b2[64] b3[2]
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kSmBar);
  uint32_t* tbase = reinterpret_cast<uint32_t*>(sm + kSmTmem);
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  const float* P = net.params;
  load_weights(B1, P + kOffW1, kWarmHidden, kWarmInPad, kWarmHidden, kWarmIn);
  load_weights(B2, P + kOffW2, kWarmHidden, kWarmHidden, kWarmHidden, kWarmHidden);
  load_weights(B3, P + kOffW3, kWarmOutPad, kWarmHidden, kWarmOut, kWarmHidden);
  for (uint32_t i = tid; i < 2 * kWarmHidden + kWarmOut; i += kTile)
    bias[i] = i < kWarmHidden ? P[kOffB1 + i]
                              : (i < 2 * kWarmHidden ? P[kOffB2 + i - kWarmHidden]
                                                     : P[kOffB3 + i - 2 * kWarmHidden]);
  if (tid == 0) {
    tc::mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    tc::tmem_alloc(tbase, kInferTmemCols);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tbase;
  const uint32_t lane = (warp * 32u) << 16;  // this warp's TMEM lanes
  const uint32_t ntiles = (n + kTile - 1) / kTile;
  uint32_t phase = 0;
  bool ok = true;
  for (uint32_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const uint32_t p = tile * kTile + tid;
    // ---- layer 1: x (normalised, bf16) x W1^T
    {
      float raw[kWarmIn];
#pragma unroll
      for (int k = 0; k < kWarmIn; ++k) raw[k] = p < n ? features[size_t(p) * kWarmIn + k] : 0.f;
      float x[kWarmInPad];
      warm_normalize(net, raw, x);
      if (p >= n) {
#pragma unroll
        for (int k = 0; k < kWarmInPad; ++k) x[k] = 0.f;
      }
      put8(A1, tid, 0, kWarmInPad, x);
      put8(A1, tid, 8, kWarmInPad, x + 8);
    }
    ok = run_layer(tmem + 0, A1, B1, kWarmInPad, kWarmHidden, bar, phase, ok);
    if (!ok) break;
    // ---- layer 2: gelu(z1 + b1) x W2^T
    {
      float z[kWarmHidden];
      tc::tmem_ld64(tmem + lane + 0, z);
#pragma unroll
      for (int j = 0; j < kWarmHidden; ++j) z[j] = gelu(z[j] + bias[j]);
#pragma unroll
      for (int c = 0; c < kWarmHidden / 8; ++c) put8(A2, tid, 8 * c, kWarmHidden, z + 8 * c);
    }
    ok = run_layer(tmem + 64, A2, B2, kWarmHidden, kWarmHidden, bar, phase, ok);
    if (!ok) break;
    // ---- layer 3: gelu(z2 + b2) x W3^T (N padded to 16)
    {
      float z[kWarmHidden];
      tc::tmem_ld64(tmem + lane + 64, z);
#pragma unroll
      for (int j = 0; j < kWarmHidden; ++j) z[j] = gelu(z[j] + bias[kWarmHidden + j]);
#pragma unroll
      for (int c = 0; c < kWarmHidden / 8; ++c) put8(A3, tid, 8 * c, kWarmHidden, z + 8 * c);
    }
    ok = run_layer(tmem + 128, A3, B3, kWarmHidden, kWarmOutPad, bar, phase, ok);
    if (!ok) break;
    {
      float y[16];
      tc::tmem_ld16(tmem + lane + 128, y);
      if (p < n) {
        out[size_t(p) * 2 + 0] = (y[0] + bias[2 * kWarmHidden + 0]) * net.out_scale[0];
        out[size_t(p) * 2 + 1] = (y[1] + bias[2 * kWarmHidden + 1]) * net.out_scale[1];
      }
    }
    // TMEM reads of this tile are complete before the next tile's MMAs
    tc::fence_before_sync();
    __syncthreads();
  }
  if (!ok) {
    if (tid == 0) atomicOr(err, 1u);
    // a layer may still be in flight: give it one more bounded wait
    tc::mbar_wait(bar, phase ^ 1u, kWaitCycles);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, kInferTmemCols);
  }
}

}  // namespace

int warm_forward(al_engine* e, const WarmNetDev& net, const float* features, uint32_t n,
                 float* out, uint32_t* err, cudaStream_t st) {
  if (n == 0) return AL_OK;
  static bool attr_set[64] = {};
  if (e->device >= 0 && e->device < 64 && !attr_set[e->device]) {
    ALB_CUDA(cudaFuncSetAttribute(k_warm_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(kInferSmem)));
    attr_set[e->device] = true;
  }
  const uint32_t tiles = blocks_for(n, kTile);
  const uint32_t grid = tiles < uint32_t(2 * e->num_sms) ? tiles : uint32_t(2 * e->num_sms);
  k_warm_forward<<<grid, kTile, kInferSmem, st>>>(net, features, n, out, err);
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

}  // namespace alb

using namespace alb;

extern "C" {

int al_warm_net_forward_f32(al_engine* engine, const al_warm_net* net, const float* features,
                            uint32_t n, float* out, void* stream) {
  ALB_CHECK_ARG(engine && net, "al_warm_net_forward_f32: null argument");
  ALB_CHECK_ARG(n == 0 || (net->params && features && out),
                "al_warm_net_forward_f32: null device pointer");
  ALB_TRY(engine->activate());
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  uint32_t* err = nullptr;
  ALB_TRY(engine->buf("warm.err", 1, &err));
  ALB_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), st));
  ALB_LAUNCH(engine, "warm_forward", 1, st,
             ALB_TRY(warm_forward(engine, to_warm_dev(*net), features, n, out, err, st)));
  uint32_t h = 0;
  ALB_CUDA(cudaMemcpyAsync(&h, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  ALB_CUDA(cudaStreamSynchronize(st));
  engine->flush_stats();
  if (h) {
    set_error("al_warm_net_forward_f32: a tensor-core wait timed out");
    return AL_ERR_TIMEOUT;
  }
  return AL_OK;
}

}  // extern "C"
