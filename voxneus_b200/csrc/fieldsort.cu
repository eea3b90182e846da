// SDF + Eq.7 gradient/normal queries (models/sdf_grid.py:90-160) of a large batch of scattered
// points, in spatial order. When the grid does not fit in L2 (a 512^3 grid is 512 MiB), a batch of
// random points reads every stencil from a different DRAM row: the plain query of 2^24 random
// points in a 512^3 grid moves ~0.26 TB/s. Here the points are first sorted by the Morton code of
// their grid cell (CUB radix sort of (key, index) pairs), then queried in that order, so a warp's
// 32 points share grid lines; each result is written back at the point's own index. The per-point
// arithmetic is the plain query's (common.cuh), so the outputs are bit-identical to it.
#include <cub/device/device_radix_sort.cuh>

#include "common.cuh"

namespace vx {
namespace {

// the low 10 bits of v, spread to every third bit
__device__ __forceinline__ uint32_t spread3(uint32_t v) {
  v &= 0x3ffu;
  v = (v | (v << 16)) & 0x030000ffu;
  v = (v | (v << 8)) & 0x0300f00fu;
  v = (v | (v << 4)) & 0x030c30c3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

__global__ void __launch_bounds__(256) k_morton_keys(const float* __restrict__ xyz, int64_t n, Grid g, int shift,
                                                     uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float cx = gs_coord(__ldg(xyz + 3 * i), g.lo[0], g.den[0], g.inv_den[0], g.rx);
    const float cy = gs_coord(__ldg(xyz + 3 * i + 1), g.lo[1], g.den[1], g.inv_den[1], g.ry);
    const float cz = gs_coord(__ldg(xyz + 3 * i + 2), g.lo[2], g.den[2], g.inv_den[2], g.rz);
    // cell indices (the clamp of gs_coord keeps them in [0, R-1]; NaN reads as 0)
    const uint32_t x = (uint32_t)cx >> shift, y = (uint32_t)cy >> shift, z = (uint32_t)cz >> shift;
    keys[i] = (spread3(x) << 2) | (spread3(y) << 1) | spread3(z);
    vals[i] = (uint32_t)i;
  }
}

__global__ void __launch_bounds__(256) k_field_query_order(const float* __restrict__ f, Grid g,
                                                           const float* __restrict__ xyz,
                                                           const uint32_t* __restrict__ order, int64_t n,
                                                           float* __restrict__ sdf, float* __restrict__ grad,
                                                           float* __restrict__ normal) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = __ldg(order + j);
    const float px = __ldg(xyz + 3 * i), py = __ldg(xyz + 3 * i + 1), pz = __ldg(xyz + 3 * i + 2);
    if (sdf && !(grad || normal)) sdf[i] = query_sdf(f, g, px, py, pz);
    if (grad || normal) {
      Eq7 e;
      eq7_setup(g, px, py, pz, e);
      float c[8], w[8];
      eq7_load_block(f, g, e, c);
      if (sdf) sdf[i] = query_sdf_block(f, g, px, py, pz, e, c);
      eq7_weights(e, w);
      float gr[3], nn[3], len;
      eq7_gradient_block(f, g, e, w, c, gr);
      if (grad) {
        grad[3 * i] = gr[0];
        grad[3 * i + 1] = gr[1];
        grad[3 * i + 2] = gr[2];
      }
      if (normal) {
        normalize_eps(gr, nn, len);
        normal[3 * i] = nn[0];
        normal[3 * i + 1] = nn[1];
        normal[3 * i + 2] = nn[2];
      }
    }
  }
}

constexpr int64_t kAlign = 256;
inline int64_t align_up(int64_t b) { return (b + kAlign - 1) / kAlign * kAlign; }

// key bits: 3 x the bits of the largest cell index after the shift that keeps it under 2^10
void key_shape(const int32_t res[3], int& shift, int& bits) {
  int r = res[0] > res[1] ? res[0] : res[1];
  r = r > res[2] ? r : res[2];
  int b = 1;
  while ((1 << b) < r) ++b;  // cell indices < 2^b
  shift = b > 10 ? b - 10 : 0;
  bits = 3 * (b - shift);
}

size_t sort_temp_bytes(int64_t n, int bits) {
  size_t temp = 0;
  if (cub::DeviceRadixSort::SortPairs(nullptr, temp, (uint32_t*)nullptr, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                      (uint32_t*)nullptr, (int)n, 0, bits) != cudaSuccess)
    return 0;
  return temp;
}

}  // namespace
}  // namespace vx

using namespace vx;

extern "C" {

int64_t vx_field_query_sorted_workspace(int64_t n, const int32_t res[3]) {
  if (n <= 0 || n > INT32_MAX || !res) return 0;
  int shift, bits;
  key_shape(res, shift, bits);
  const size_t temp = sort_temp_bytes(n, bits);
  if (temp == 0) return 0;
  return 4 * align_up(n * 4) + align_up((int64_t)temp);
}

int vx_field_query_sorted(const float* grid, const int32_t res[3], const float xyz_min[3], const float xyz_max[3],
                          const float* xyz, int64_t n, float* sdf, float* grad, float* normal, void* workspace,
                          int64_t workspace_bytes, void* stream) {
  if (int s = check_grid(res)) return s;
  VX_REQUIRE(n >= 0 && n <= INT32_MAX, "n out of range (0 .. 2^31-1)");
  if (n == 0 || (!sdf && !grad && !normal)) return VX_OK;
  VX_REQUIRE(grid && xyz && xyz_min && xyz_max && workspace, "null pointer");
  const int64_t need = vx_field_query_sorted_workspace(n, res);
  VX_REQUIRE(need > 0, "sort workspace size query failed");
  VX_REQUIRE(workspace_bytes >= need, "workspace holds %lld bytes, need %lld", (long long)workspace_bytes,
             (long long)need);
  VX_REQUIRE(((uintptr_t)workspace & (kAlign - 1)) == 0, "workspace must be 256-byte aligned");
  int shift, bits;
  key_shape(res, shift, bits);
  Grid g = make_grid(res, xyz_min, xyz_max);
  char* w = static_cast<char*>(workspace);
  const int64_t a = align_up(n * 4);
  uint32_t* k_in = reinterpret_cast<uint32_t*>(w);
  uint32_t* k_out = reinterpret_cast<uint32_t*>(w + a);
  uint32_t* v_in = reinterpret_cast<uint32_t*>(w + 2 * a);
  uint32_t* v_out = reinterpret_cast<uint32_t*>(w + 3 * a);
  void* temp = w + 4 * a;
  size_t temp_bytes = (size_t)(workspace_bytes - 4 * a);
  cudaStream_t st = (cudaStream_t)stream;
  k_morton_keys<<<grid_for(n, 256, 8), 256, 0, st>>>(xyz, n, g, shift, k_in, v_in);
  cudaError_t e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, k_in, k_out, v_in, v_out, (int)n, 0, bits, st);
  if (e != cudaSuccess) return set_error(VX_ERR_CUDA, "field_query_sorted: sort: %s", cudaGetErrorString(e));
  k_field_query_order<<<grid_for(n, 256), 256, 0, st>>>(grid, g, xyz, v_out, n, sdf, grad, normal);
  count_launches(2);
  return check_launch("field_query_sorted");
}

}  // extern "C"
