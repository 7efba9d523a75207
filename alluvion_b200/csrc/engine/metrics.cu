// metrics.cu -- the reference's Runner reductions used to score sampled
// fields against targets (runner.hpp:715-744, 4710-4800):
//   al_calculate_se_*           calculate_se: se[i] = |v0[i] - v1[i]|^2
//   al_calculate_se_weighted_*  calculate_se_weighted: sum w[i] |v0[i] - v1[i]|^2
//   al_calculate_se_yz_masked_* calculate_se_yz_masked: sum over mask[i] == 1 of
//                               (v0 - v1).y^2 + (v0 - v1).z^2
//   al_sum_products_*           sum_products: component-wise sum of v0[i] v1[i]
// Each per-element term is formed in the variables' real type with
// correctly rounded operations (no contraction), as the reference's functors
// evaluate it; the sums are taken in double in a fixed order (per-block
// grid-stride partials, then one block over the partials), so a result does
// not depend on the launch.  The reference sums with thrust::transform_reduce
// in the real type, whose order is unspecified.
#include "common.cuh"
#include "engine.hpp"

namespace alb {
namespace {

constexpr int kMetricBlock = 256;

template <class TF>
__device__ __forceinline__ TF sq_diff(const TF* a, const TF* b, uint32_t i, uint32_t dims,
                                      uint32_t from) {
  TF s = 0;
  for (uint32_t k = from; k < dims; ++k) {
    const TF d = sub_rn(a[size_t(i) * dims + k], b[size_t(i) * dims + k]);
    s = k == from ? mul_rn(d, d) : add_rn(s, mul_rn(d, d));
  }
  return s;
}

template <class TF>
__global__ void k_se(const TF* __restrict__ v0, const TF* __restrict__ v1, uint32_t n,
                     uint32_t dims, TF* __restrict__ se) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) se[i] = sq_diff(v0, v1, i, dims, 0);
}

// OP 0: sum w |d|^2; 1: sum over w == 1 of d.y^2 + d.z^2; 2: per-component
// sum of v0 v1 (out[0..dims)).  Per-block partials in `part[block * 4 + k]`.
template <class TF, int OP>
__global__ void __launch_bounds__(kMetricBlock)
    k_metric_partial(const TF* __restrict__ v0, const TF* __restrict__ v1,
                     const TF* __restrict__ w, uint32_t n, uint32_t dims, double* part) {
  __shared__ double red[4][kMetricBlock];
  double acc[4] = {0, 0, 0, 0};
  for (uint32_t i = blockIdx.x * kMetricBlock + threadIdx.x; i < n;
       i += gridDim.x * kMetricBlock) {
    if (OP == 0) {
      acc[0] += double(mul_rn(w[i], sq_diff(v0, v1, i, dims, 0)));
    } else if (OP == 1) {
      if (w[i] == TF(1)) acc[0] += double(sq_diff(v0, v1, i, 3, 1));
    } else {
      for (uint32_t k = 0; k < dims; ++k)
        acc[k] += double(mul_rn(v0[size_t(i) * dims + k], v1[size_t(i) * dims + k]));
    }
  }
  for (int k = 0; k < 4; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int s = kMetricBlock / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x < 4) part[size_t(blockIdx.x) * 4 + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void __launch_bounds__(kMetricBlock)
    k_metric_final(const double* __restrict__ part, uint32_t blocks, double* out) {
  __shared__ double red[4][kMetricBlock];
  double acc[4] = {0, 0, 0, 0};
  for (uint32_t b = threadIdx.x; b < blocks; b += kMetricBlock)
    for (int k = 0; k < 4; ++k) acc[k] += part[size_t(b) * 4 + k];
  for (int k = 0; k < 4; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int s = kMetricBlock / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int k = 0; k < 4; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x < 4) out[threadIdx.x] = red[threadIdx.x][0];
}

template <class TF, int OP>
int metric(al_engine* e, const TF* v0, const TF* v1, const TF* w, uint32_t n, uint32_t dims,
           double* result, uint32_t nres, void* stream) {
  ALB_TRY(e->activate());
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n == 0) {
    for (uint32_t k = 0; k < nres; ++k) result[k] = 0;
    return AL_OK;
  }
  // a fixed grid for a given n: two blocks per SM at most
  const uint32_t want = (n + kMetricBlock - 1) / kMetricBlock;
  const uint32_t cap = uint32_t(e->num_sms) * 2;
  const uint32_t blocks = want < cap ? want : cap;
  double* part = nullptr;
  double* dres = nullptr;
  ALB_TRY(e->buf("metric.partials", size_t(blocks) * 4, &part));
  ALB_TRY(e->buf("metric.result", 4, &dres));
  ALB_LAUNCH(e, "metric", 2, st, {
    k_metric_partial<TF, OP><<<blocks, kMetricBlock, 0, st>>>(v0, v1, w, n, dims, part);
    k_metric_final<<<1, kMetricBlock, 0, st>>>(part, blocks, dres);
  });
  ALB_CUDA(cudaGetLastError());
  double h[4];
  ALB_CUDA(cudaMemcpyAsync(h, dres, sizeof(h), cudaMemcpyDeviceToHost, st));
  ALB_CUDA(cudaStreamSynchronize(st));
  e->flush_stats();
  for (uint32_t k = 0; k < nres; ++k) result[k] = h[k];
  return AL_OK;
}

template <class TF>
int calculate_se(al_engine* e, const TF* v0, const TF* v1, TF* se, uint32_t n, uint32_t dims,
                 void* stream) {
  ALB_CHECK_ARG(e && (n == 0 || (v0 && v1 && se)), "al_calculate_se: null argument");
  ALB_CHECK_ARG(dims >= 1 && dims <= 4, "al_calculate_se: dims must be 1..4");
  ALB_TRY(e->activate());
  if (n == 0) return AL_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  ALB_LAUNCH(e, "calculate_se", 1, st,
             (k_se<TF><<<(n + kMetricBlock - 1) / kMetricBlock, kMetricBlock, 0, st>>>(
                 v0, v1, n, dims, se)));
  ALB_CUDA(cudaGetLastError());
  return AL_OK;
}

template <class TF>
int se_weighted(al_engine* e, const TF* v0, const TF* v1, const TF* w, uint32_t n,
                uint32_t dims, double* result, void* stream) {
  ALB_CHECK_ARG(e && result && (n == 0 || (v0 && v1 && w)),
                "al_calculate_se_weighted: null argument");
  ALB_CHECK_ARG(dims >= 1 && dims <= 4, "al_calculate_se_weighted: dims must be 1..4");
  return metric<TF, 0>(e, v0, v1, w, n, dims, result, 1, stream);
}

template <class TF>
int se_yz_masked(al_engine* e, const TF* v0, const TF* v1, const TF* mask, uint32_t n,
                 double* result, void* stream) {
  ALB_CHECK_ARG(e && result && (n == 0 || (v0 && v1 && mask)),
                "al_calculate_se_yz_masked: null argument");
  return metric<TF, 1>(e, v0, v1, mask, n, 3, result, 1, stream);
}

template <class TF>
int sum_products(al_engine* e, const TF* v0, const TF* v1, uint32_t n, uint32_t dims,
                 double* result, void* stream) {
  ALB_CHECK_ARG(e && result && (n == 0 || (v0 && v1)), "al_sum_products: null argument");
  ALB_CHECK_ARG(dims >= 1 && dims <= 4, "al_sum_products: dims must be 1..4");
  return metric<TF, 2>(e, v0, v1, nullptr, n, dims, result, dims, stream);
}

}  // namespace
}  // namespace alb

using namespace alb;

extern "C" {

int al_calculate_se_f32(al_engine* e, const float* v0, const float* v1, float* se, uint32_t n,
                        uint32_t dims, void* stream) {
  return calculate_se<float>(e, v0, v1, se, n, dims, stream);
}
int al_calculate_se_f64(al_engine* e, const double* v0, const double* v1, double* se, uint32_t n,
                        uint32_t dims, void* stream) {
  return calculate_se<double>(e, v0, v1, se, n, dims, stream);
}
int al_calculate_se_weighted_f32(al_engine* e, const float* v0, const float* v1,
                                 const float* weight, uint32_t n, uint32_t dims, double* result,
                                 void* stream) {
  return se_weighted<float>(e, v0, v1, weight, n, dims, result, stream);
}
int al_calculate_se_weighted_f64(al_engine* e, const double* v0, const double* v1,
                                 const double* weight, uint32_t n, uint32_t dims, double* result,
                                 void* stream) {
  return se_weighted<double>(e, v0, v1, weight, n, dims, result, stream);
}
int al_calculate_se_yz_masked_f32(al_engine* e, const float* v0, const float* v1,
                                  const float* mask, uint32_t n, double* result, void* stream) {
  return se_yz_masked<float>(e, v0, v1, mask, n, result, stream);
}
int al_calculate_se_yz_masked_f64(al_engine* e, const double* v0, const double* v1,
                                  const double* mask, uint32_t n, double* result, void* stream) {
  return se_yz_masked<double>(e, v0, v1, mask, n, result, stream);
}
int al_sum_products_f32(al_engine* e, const float* v0, const float* v1, uint32_t n,
                        uint32_t dims, double* result, void* stream) {
  return sum_products<float>(e, v0, v1, n, dims, result, stream);
}
int al_sum_products_f64(al_engine* e, const double* v0, const double* v1, uint32_t n,
                        uint32_t dims, double* result, void* stream) {
  return sum_products<double>(e, v0, v1, n, dims, result, stream);
}

}  // extern "C"
