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

#include <cmath>

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
                   float* __restrict__ out, uint32_t* __restrict__ err,
                   const uint32_t* __restrict__ skip) {
  // the whole grid leaves before any shared-memory or TMEM work when the
  // step's gate says the prediction is not used
  if (skip && *skip) return;
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

// ---------------------------------------------------------------- training
// One CTA per SM runs forward and backward over its 128-row tiles and
// accumulates the weight gradients in TMEM across tiles:
//   D4 = dz2 x W2                      (dh1, backward through layer 2)
//   D5 += [dz2^T; dz1^T] x [h1^T; x^T; 1]^T   -> dW2, db2 (rows 0-63), dW1,
//         db1 (rows 64-127); column 79 is the ones row of B (bias sums)
//   D6 += [h2^T; 1; 0] x [dy^T; 0]^T          -> dW3^T (rows 0-63), db3 (row 64)
// with every gradient operand rounded to BF16 (the oracle rounds at the
// same points).  Partial gradients per CTA are summed in CTA order by
// k_warm_reduce.
constexpr uint32_t kTrainTmemCols = 512;
constexpr uint32_t kTD1 = 0, kTD2 = 64, kTD3 = 128, kTD4 = 160, kTD5 = 256, kTD6 = 352;
constexpr uint32_t kGradN = 80;     // D5 columns: h1 (64) + x (12) + zero pad (3) + ones (1)
constexpr uint32_t kOnesRow = 79;   // row of B5 (and column of D5) holding ones
constexpr uint32_t kSamples = kTile;  // K of the gradient products

constexpr uint32_t kTA1 = 0;                          // x      [128][16]
constexpr uint32_t kTA2 = kTA1 + kTile * 16 * 2;      // h1     [128][64]
constexpr uint32_t kTA3 = kTA2 + kTile * 64 * 2;      // h2     [128][64]
constexpr uint32_t kTA4 = kTA3 + kTile * 64 * 2;      // dz2    [128][64]
constexpr uint32_t kTB1 = kTA4 + kTile * 64 * 2;      // W1     [64][16]
constexpr uint32_t kTB2 = kTB1 + 64 * 16 * 2;         // W2     [64][64]
constexpr uint32_t kTB3 = kTB2 + 64 * 64 * 2;         // W3     [16][64]
constexpr uint32_t kTB2T = kTB3 + 16 * 64 * 2;        // W2^T   [64][64]
constexpr uint32_t kTGA = kTB2T + 64 * 64 * 2;        // [128][128]
constexpr uint32_t kTGB = kTGA + 128 * kSamples * 2;  // [80][128]
constexpr uint32_t kTHA = kTGB + kGradN * kSamples * 2;  // [128][128]
constexpr uint32_t kTHB = kTHA + 128 * kSamples * 2;  // [16][128]
constexpr uint32_t kTF32 = kTHB + 16 * kSamples * 2;  // b1[64] b2[64] b3[2] W3[2][64] f32
constexpr uint32_t kTRed = kTF32 + 2048;              // loss partials, 4 doubles
constexpr uint32_t kTBar = kTRed + 64;
constexpr uint32_t kTTmem = kTBar + 8;
constexpr uint32_t kTUsed = kTTmem + 8;
// over half of the SM's shared memory: one CTA (512 TMEM columns) per SM
constexpr uint32_t kTrainSmem = 168 * 1024;
static_assert(kTUsed <= kTrainSmem, "training shared-memory map");

__device__ __forceinline__ float bf16_round(float v) {
  return __bfloat162float(__float2bfloat16_rn(v));
}
// Element (m, c) of a K-major [rows][128] bf16 tile (c: the sample).
__device__ __forceinline__ void put_t(uint8_t* tile, uint32_t m, uint32_t c, float v) {
  *reinterpret_cast<__nv_bfloat16*>(tile + tc::kmajor_offset(m, c, kSamples)) =
      __float2bfloat16_rn(v);
}

// Issues the two gradient products over the tile's 128 samples and commits.
__device__ __forceinline__ void issue_grads(uint32_t tmem, const uint8_t* ga, const uint8_t* gb,
                                            const uint8_t* ha, const uint8_t* hb, bool first,
                                            uint64_t* bar) {
  const uint32_t i5 = tc::idesc_bf16(kTile, kGradN), i6 = tc::idesc_bf16(kTile, 16);
  const uint32_t sga = tc::smem_u32(ga), sgb = tc::smem_u32(gb);
  const uint32_t sha = tc::smem_u32(ha), shb = tc::smem_u32(hb);
  for (uint32_t k = 0; k < kSamples / 16; ++k) {
    const uint32_t acc = (first && k == 0) ? 0u : 1u;
    tc::mma_bf16(tmem + kTD5, tc::tile_desc(sga, kSamples, k), tc::tile_desc(sgb, kSamples, k),
                 i5, acc);
    tc::mma_bf16(tmem + kTD6, tc::tile_desc(sha, kSamples, k), tc::tile_desc(shb, kSamples, k),
                 i6, acc);
  }
  tc::commit(bar);
}

__global__ void __launch_bounds__(kTile)
    k_warm_train(WarmNetDev net, const float* __restrict__ features,
                 const float* __restrict__ targets, uint32_t n, float inv_n,
                 float* __restrict__ part, double* __restrict__ part_loss,
                 uint32_t* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint8_t *A1 = sm + kTA1, *A2 = sm + kTA2, *A3 = sm + kTA3, *A4 = sm + kTA4;
  uint8_t *B1 = sm + kTB1, *B2 = sm + kTB2, *B3 = sm + kTB3, *B2T = sm + kTB2T;
  uint8_t *GA = sm + kTGA, *GB = sm + kTGB, *HA = sm + kTHA, *HB = sm + kTHB;
  float* f32 = reinterpret_cast<float*>(sm + kTF32);
  float *b1 = f32, *b2 = f32 + 64, *b3 = f32 + 128, *w3 = f32 + 130;  // w3: bf16-rounded
  double* red = reinterpret_cast<double*>(sm + kTRed);
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + kTBar);
  uint32_t* tbase = reinterpret_cast<uint32_t*>(sm + kTTmem);
  const uint32_t tid = threadIdx.x, warp = tid >> 5;
  const float* P = net.params;
  load_weights(B1, P + kOffW1, 64, 16, 64, kWarmIn);
  load_weights(B2, P + kOffW2, 64, 64, 64, 64);
  load_weights(B3, P + kOffW3, 16, 64, kWarmOut, 64);
  for (uint32_t i = tid; i < 64 * 64; i += kTile) {  // W2^T: [j][k] = W2[k][j]
    const uint32_t j = i / 64, k = i % 64;
    *reinterpret_cast<__nv_bfloat16*>(B2T + tc::kmajor_offset(j, k, 64)) =
        __float2bfloat16_rn(P[kOffW2 + k * 64 + j]);
  }
  for (uint32_t i = tid; i < 64; i += kTile) {
    b1[i] = P[kOffB1 + i];
    b2[i] = P[kOffB2 + i];
    w3[i] = bf16_round(P[kOffW3 + i]);
    w3[64 + i] = bf16_round(P[kOffW3 + 64 + i]);
  }
  if (tid < kWarmOut) b3[tid] = P[kOffB3 + tid];
  // constant parts of the gradient operands
  for (uint32_t c = 0; c < kSamples; c += 1) {
    if (tid >= 65) put_t(HA, tid, c, 0.f);       // rows 65-127 of [h2^T; 1; 0]
    if (tid >= 2 && tid < 16) put_t(HB, tid, c, 0.f);  // rows 2-15 of [dy^T; 0]
    if (tid >= 76 && tid < kOnesRow) put_t(GB, tid, c, 0.f);  // x pad rows
  }
  if (tid == 0) {
    tc::mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    tc::tmem_alloc(tbase, kTrainTmemCols);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tbase;
  const uint32_t lane = (warp * 32u) << 16;
  const uint32_t ntiles = (n + kTile - 1) / kTile;
  uint32_t phase = 0;
  bool ok = true, first = true;
  double loss = 0;
  for (uint32_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
    const uint32_t p = tile * kTile + tid;
    const bool valid = p < n;
    // ---- layer 1
    {
      float raw[kWarmIn];
#pragma unroll
      for (int k = 0; k < kWarmIn; ++k) raw[k] = valid ? features[size_t(p) * kWarmIn + k] : 0.f;
      float x[kWarmInPad];
      warm_normalize(net, raw, x);
#pragma unroll
      for (int k = 0; k < kWarmInPad; ++k) x[k] = valid ? x[k] : 0.f;
      put8(A1, tid, 0, 16, x);
      put8(A1, tid, 8, 16, x + 8);
#pragma unroll
      for (int k = 0; k < kWarmIn; ++k) put_t(GB, 64 + k, tid, x[k]);
      put_t(GB, kOnesRow, tid, 1.f);
    }
    ok = run_layer(tmem + kTD1, A1, B1, 16, 64, bar, phase, ok);
    if (!ok) break;
    // ---- layer 2 input h1 (also the B rows 0-63 of the dW2 product)
    {
      float z[64];
      tc::tmem_ld64(tmem + lane + kTD1, z);
#pragma unroll
      for (int j = 0; j < 64; ++j) z[j] = gelu(z[j] + b1[j]);
#pragma unroll
      for (int c = 0; c < 8; ++c) put8(A2, tid, 8 * c, 64, z + 8 * c);
#pragma unroll
      for (int j = 0; j < 64; ++j) put_t(GB, j, tid, z[j]);
    }
    ok = run_layer(tmem + kTD2, A2, B2, 64, 64, bar, phase, ok);
    if (!ok) break;
    // ---- layer 3 input h2 (also the A rows 0-63 of the dW3 product)
    {
      float z[64];
      tc::tmem_ld64(tmem + lane + kTD2, z);
#pragma unroll
      for (int j = 0; j < 64; ++j) z[j] = gelu(z[j] + b2[j]);
#pragma unroll
      for (int c = 0; c < 8; ++c) put8(A3, tid, 8 * c, 64, z + 8 * c);
#pragma unroll
      for (int j = 0; j < 64; ++j) put_t(HA, j, tid, z[j]);
      put_t(HA, 64, tid, 1.f);
    }
    ok = run_layer(tmem + kTD3, A3, B3, 64, 16, bar, phase, ok);
    if (!ok) break;
    // ---- output gradient dy = (y - t) / n and dz2 = (dy W3) * g'(z2)
    {
      float y[16];
      tc::tmem_ld16(tmem + lane + kTD3, y);
      float dy[kWarmOut];
#pragma unroll
      for (int o = 0; o < kWarmOut; ++o) {
        const float t = valid ? targets[size_t(p) * kWarmOut + o] / net.out_scale[o] : 0.f;
        const float d = valid ? (y[o] + b3[o]) - t : 0.f;
        loss += 0.5 * double(d) * double(d);
        dy[o] = d * inv_n;
        put_t(HB, o, tid, dy[o]);
      }
      float z[64];
      tc::tmem_ld64(tmem + lane + kTD2, z);
#pragma unroll
      for (int j = 0; j < 64; ++j) {
        const float dh = dy[0] * w3[j] + dy[1] * w3[64 + j];
        z[j] = dh * gelu_grad(z[j] + b2[j]);
      }
#pragma unroll
      for (int c = 0; c < 8; ++c) put8(A4, tid, 8 * c, 64, z + 8 * c);
#pragma unroll
      for (int j = 0; j < 64; ++j) put_t(GA, j, tid, z[j]);
    }
    ok = run_layer(tmem + kTD4, A4, B2T, 64, 64, bar, phase, ok);
    if (!ok) break;
    // ---- dz1 = (dz2 W2) * g'(z1)
    {
      float dh[64], z[64];
      tc::tmem_ld64(tmem + lane + kTD4, dh);
      tc::tmem_ld64(tmem + lane + kTD1, z);
#pragma unroll
      for (int j = 0; j < 64; ++j) put_t(GA, 64 + j, tid, dh[j] * gelu_grad(z[j] + b1[j]));
    }
    // ---- gradient products, accumulated over this CTA's tiles
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    ok = __syncthreads_and(ok);
    if (!ok) break;
    if (tid == 0) {
      tc::fence_after_sync();
      issue_grads(tmem, GA, GB, HA, HB, first, bar);
    }
    ok = tc::mbar_wait(bar, phase, kWaitCycles);
    phase ^= 1u;
    tc::fence_after_sync();
    ok = __syncthreads_and(ok);
    first = false;
  }
  // ---- this CTA's partial gradients (row tid of D5 and D6) and loss
  float* g = part + size_t(blockIdx.x) * AL_WARM_NUM_PARAMS;
  if (ok && !first) {
    float d5[64], d5b[16], d6[16];
    tc::tmem_ld64(tmem + lane + kTD5, d5);
    tc::tmem_ld16(tmem + lane + kTD5 + 64, d5b);
    tc::tmem_ld16(tmem + lane + kTD6, d6);
    if (tid < 64) {
      for (int j = 0; j < 64; ++j) g[kOffW2 + tid * 64 + j] = d5[j];
      g[kOffB2 + tid] = d5b[kOnesRow - 64];
      g[kOffW3 + tid] = d6[0];
      g[kOffW3 + 64 + tid] = d6[1];
    } else {
      const uint32_t k = tid - 64;
      for (int i = 0; i < kWarmIn; ++i) g[kOffW1 + k * kWarmIn + i] = d5b[i];
      g[kOffB1 + k] = d5b[kOnesRow - 64];
      if (tid == 64) {
        g[kOffB3 + 0] = d6[0];
        g[kOffB3 + 1] = d6[1];
      }
    }
  } else {
    for (uint32_t i = tid; i < AL_WARM_NUM_PARAMS; i += kTile) g[i] = 0.f;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) loss += __shfl_xor_sync(0xffffffffu, loss, o);
  if ((tid & 31) == 0) red[warp] = loss;
  if (!ok) {
    if (tid == 0) atomicOr(err, 1u);
    tc::mbar_wait(bar, phase ^ 1u, kWaitCycles);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (tid == 0) part_loss[blockIdx.x] = red[0] + red[1] + red[2] + red[3];
  if (warp == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, kTrainTmemCols);
  }
}

// grad[i] = sum over CTAs (in CTA order, double) of the partials; loss
// likewise, divided by n.
__global__ void k_warm_reduce(const float* __restrict__ part, const double* __restrict__ part_loss,
                              uint32_t nparts, uint32_t n, float* __restrict__ grad,
                              double* __restrict__ loss) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < AL_WARM_NUM_PARAMS) {
    double s = 0;
    for (uint32_t c = 0; c < nparts; ++c) s += double(part[size_t(c) * AL_WARM_NUM_PARAMS + i]);
    grad[i] = float(s);
  }
  if (i == 0) {
    double s = 0;
    for (uint32_t c = 0; c < nparts; ++c) s += part_loss[c];
    *loss = n ? s / double(n) : 0.0;
  }
}

// Adam (Kingma & Ba 2015) on the FP32 master parameters; omb1 = 1 - beta1
// and omb2 = 1 - beta2 come from the host in double precision.
__global__ void k_warm_adam(float* __restrict__ p, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, uint32_t count,
                            float lr, float beta1, float beta2, float omb1, float omb2, float eps,
                            float c1, float c2) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float gi = g[i];
  const float mi = beta1 * m[i] + omb1 * gi;
  const float vi = beta2 * v[i] + omb2 * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

}  // namespace

int warm_forward(al_engine* e, const WarmNetDev& net, const float* features, uint32_t n,
                 float* out, uint32_t* err, cudaStream_t st, const uint32_t* skip) {
  if (n == 0) return AL_OK;
  static bool attr_set[64] = {};
  if (e->device >= 0 && e->device < 64 && !attr_set[e->device]) {
    ALB_CUDA(cudaFuncSetAttribute(k_warm_forward, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(kInferSmem)));
    attr_set[e->device] = true;
  }
  const uint32_t tiles = blocks_for(n, kTile);
  const uint32_t grid = tiles < uint32_t(2 * e->num_sms) ? tiles : uint32_t(2 * e->num_sms);
  k_warm_forward<<<grid, kTile, kInferSmem, st>>>(net, features, n, out, err, skip);
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

int warm_gradient(al_engine* e, const WarmNetDev& net, const float* features,
                  const float* targets, uint32_t n, float* grad, double* loss, uint32_t* err,
                  cudaStream_t st) {
  static bool attr_set[64] = {};
  if (e->device >= 0 && e->device < 64 && !attr_set[e->device]) {
    ALB_CUDA(cudaFuncSetAttribute(k_warm_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(kTrainSmem)));
    attr_set[e->device] = true;
  }
  const uint32_t tiles = blocks_for(n, kTile);
  uint32_t grid = tiles < uint32_t(e->num_sms) ? tiles : uint32_t(e->num_sms);
  if (grid == 0) grid = 1;
  float* part = nullptr;
  double* part_loss = nullptr;
  ALB_TRY(e->buf("warm.part", size_t(grid) * AL_WARM_NUM_PARAMS, &part));
  ALB_TRY(e->buf("warm.part_loss", grid, &part_loss));
  k_warm_train<<<grid, kTile, kTrainSmem, st>>>(net, features, targets, n,
                                                n ? 1.f / float(n) : 0.f, part, part_loss, err);
  ALB_CUDA(cudaGetLastError());
  k_warm_reduce<<<blocks_for(AL_WARM_NUM_PARAMS, 256), 256, 0, st>>>(part, part_loss, grid, n,
                                                                      grad, loss);
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

int al_warm_net_gradient_f32(al_engine* engine, const al_warm_net* net, const float* features,
                             const float* targets, uint32_t n, float* grad, double* loss,
                             void* stream) {
  ALB_CHECK_ARG(engine && net && grad, "al_warm_net_gradient_f32: null argument");
  ALB_CHECK_ARG(net->params && (n == 0 || (features && targets)),
                "al_warm_net_gradient_f32: null device pointer");
  ALB_TRY(engine->activate());
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  uint32_t* err = nullptr;
  double* dloss = nullptr;
  ALB_TRY(engine->buf("warm.err", 1, &err));
  ALB_TRY(engine->buf("warm.loss", 1, &dloss));
  ALB_CUDA(cudaMemsetAsync(err, 0, sizeof(uint32_t), st));
  ALB_LAUNCH(engine, "warm_gradient", 2, st,
             ALB_TRY(warm_gradient(engine, to_warm_dev(*net), features, targets, n, grad, dloss,
                                   err, st)));
  uint32_t h = 0;
  double l = 0;
  ALB_CUDA(cudaMemcpyAsync(&h, err, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  ALB_CUDA(cudaMemcpyAsync(&l, dloss, sizeof(double), cudaMemcpyDeviceToHost, st));
  ALB_CUDA(cudaStreamSynchronize(st));
  engine->flush_stats();
  if (loss) *loss = l;
  if (h) {
    set_error("al_warm_net_gradient_f32: a tensor-core wait timed out");
    return AL_ERR_TIMEOUT;
  }
  return AL_OK;
}

int al_warm_net_adam_f32(al_engine* engine, float* params, const float* grad, float* m, float* v,
                         uint32_t step, float lr, void* stream) {
  ALB_CHECK_ARG(engine && params && grad && m && v, "al_warm_net_adam_f32: null argument");
  ALB_CHECK_ARG(step >= 1, "al_warm_net_adam_f32: step counts from 1");
  ALB_TRY(engine->activate());
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const double beta1 = 0.9, beta2 = 0.999;
  const float c1 = float(1.0 - std::pow(beta1, double(step)));
  const float c2 = float(1.0 - std::pow(beta2, double(step)));
  ALB_LAUNCH(engine, "warm_adam", 1, st,
             (k_warm_adam<<<blocks_for(AL_WARM_NUM_PARAMS, 256), 256, 0, st>>>(
                 params, grad, m, v, AL_WARM_NUM_PARAMS, lr, float(beta1), float(beta2),
                 float(1.0 - beta1), float(1.0 - beta2), 1e-8f, c1, c2)));
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

}  // extern "C"
