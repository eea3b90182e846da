// Huber colour loss of NeuS2 (rendering/volume_render.py:43-54): the mean over n elements of
// d < delta ? 0.5 d^2 / delta : d - 0.5 delta, d = |pred - target|, and in the same pass its
// gradient (1/n) (d < delta ? (pred - target) / delta : sign(pred - target)). One kernel writes the
// gradient and per-block double partials; a one-block kernel sums them in block order.
#include "common.cuh"

namespace vx {

__global__ void __launch_bounds__(256) k_huber(const float* __restrict__ pred, const float* __restrict__ target,
                                               int64_t n, float delta, float inv_n, float* __restrict__ grad,
                                               double* __restrict__ partials) {
  __shared__ double red[8];
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float e = pred[i] - target[i];
    const float d = fabsf(e);
    const bool quad = d < delta;
    acc += (double)(quad ? (0.5f * (d * d)) / delta : d - 0.5f * delta);
    if (grad) {
      const float sg = e > 0.0f ? 1.0f : (e < 0.0f ? -1.0f : 0.0f);
      grad[i] = inv_n * (quad ? e / delta : sg);
    }
  }
  acc = warp_sum_d(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    partials[blockIdx.x] = s;
  }
}

__global__ void k_huber_finalize(const double* __restrict__ partials, int nb, int64_t n, float* __restrict__ loss) {
  __shared__ double red[8];
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partials[b];
  s = warp_sum_d(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    *loss = (float)(t / (double)n);
  }
}

}  // namespace vx

using namespace vx;

extern "C" {

int vx_huber_loss_blocks(int64_t n) { return (int)grid_for(n, 256, 4); }

int vx_huber_loss(const float* pred, const float* target, int64_t n, float delta, float* loss, float* grad,
                  double* partials, int64_t n_partials, void* stream) {
  VX_REQUIRE(n > 0, "empty input");
  VX_REQUIRE(delta > 0.0f, "delta must be > 0");
  VX_REQUIRE(pred && target && loss && partials, "null pointer");
  const int nb = vx_huber_loss_blocks(n);
  VX_REQUIRE(n_partials >= nb, "partials hold %lld doubles, need %d", (long long)n_partials, nb);
  cudaStream_t st = (cudaStream_t)stream;
  k_huber<<<nb, 256, 0, st>>>(pred, target, n, delta, (float)(1.0 / (double)n), grad, partials);
  k_huber_finalize<<<1, 256, 0, st>>>(partials, nb, n, loss);
  count_launches(2);
  return check_launch("huber_loss");
}

}  // extern "C"
