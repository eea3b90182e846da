// Trilinear grid upsampling with align_corners=True (geometry/upsample.py:12-39, the
// F.interpolate call of models/sdf_grid.py:183-195).
//
// Upsampling is write-bound (a 128^3 -> 256^3 pass reads 8 MiB, L2-resident, and writes
// 64 MiB): one thread per 4 consecutive z outputs, 16-byte stores when the row allows.
#include "common.cuh"

namespace vx {

struct Axis {
  float scale;
  int in;
};

// ATen's align_corners source index: src = scale * dst, scale = (in - 1) / (out - 1).
__device__ __forceinline__ void src_index(const Axis& a, int o, int& i0, int& ip, float& l0, float& l1) {
  const float r = a.scale * (float)o;
  i0 = (int)r;
  ip = (i0 < a.in - 1) ? 1 : 0;
  l1 = r - (float)i0;
  l0 = 1.0f - l1;
}

__global__ void __launch_bounds__(256) k_grid_upsample(const float* __restrict__ src, int ix, int iy, int iz,
                                                       float* __restrict__ dst, int ox, int oy, int oz, Axis ax, Axis ay,
                                                       Axis az) {
  const int zq = (oz + 3) / 4;
  const int64_t total = (int64_t)ox * oy * zq;
  const bool vec = (oz % 4) == 0;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
    const int zb = (int)(q % zq) * 4;
    const int64_t r = q / zq;
    const int y = (int)(r % oy);
    const int x = (int)(r / oy);
    int x0, xp, y0, yp;
    float lx0, lx1, ly0, ly1;
    src_index(ax, x, x0, xp, lx0, lx1);
    src_index(ay, y, y0, yp, ly0, ly1);
    const float* r00 = src + ((int64_t)x0 * iy + y0) * iz;
    const float* r01 = src + ((int64_t)x0 * iy + y0 + yp) * iz;
    const float* r10 = src + ((int64_t)(x0 + xp) * iy + y0) * iz;
    const float* r11 = src + ((int64_t)(x0 + xp) * iy + y0 + yp) * iz;
    float v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int z = zb + k;
      if (z >= oz) {
        v[k] = 0.0f;
        continue;
      }
      int z0, zp;
      float lz0, lz1;
      src_index(az, z, z0, zp, lz0, lz1);
      v[k] = lx0 * (ly0 * (lz0 * __ldg(r00 + z0) + lz1 * __ldg(r00 + z0 + zp)) +
                    ly1 * (lz0 * __ldg(r01 + z0) + lz1 * __ldg(r01 + z0 + zp))) +
             lx1 * (ly0 * (lz0 * __ldg(r10 + z0) + lz1 * __ldg(r10 + z0 + zp)) +
                    ly1 * (lz0 * __ldg(r11 + z0) + lz1 * __ldg(r11 + z0 + zp)));
    }
    float* out = dst + ((int64_t)x * oy + y) * oz + zb;
    if (vec) {
      *reinterpret_cast<float4*>(out) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
      for (int k = 0; k < 4 && zb + k < oz; ++k) out[k] = v[k];
    }
  }
}

}  // namespace vx

using namespace vx;

extern "C" {

int vx_grid_upsample(const float* src, const int32_t res_in[3], float* dst, const int32_t res_out[3], void* stream) {
  VX_REQUIRE(res_in && res_out, "null resolution");
  for (int a = 0; a < 3; ++a) VX_REQUIRE(res_in[a] >= 1 && res_out[a] >= 1, "resolutions must be positive");
  VX_REQUIRE((int64_t)res_out[0] * res_out[1] * res_out[2] < (int64_t(1) << 31), "output has 2^31 or more voxels");
  VX_REQUIRE(src && dst, "null pointer");
  VX_REQUIRE(((uintptr_t)dst & 15) == 0, "dst must be 16-byte aligned");
  Axis ax[3];
  for (int a = 0; a < 3; ++a) {
    ax[a].in = res_in[a];
    ax[a].scale = res_out[a] > 1 ? (float)(res_in[a] - 1) / (float)(res_out[a] - 1) : 0.0f;
  }
  const int64_t total = (int64_t)res_out[0] * res_out[1] * ((res_out[2] + 3) / 4);
  k_grid_upsample<<<grid_for(total, 256, 8), 256, 0, (cudaStream_t)stream>>>(
      src, res_in[0], res_in[1], res_in[2], dst, res_out[0], res_out[1], res_out[2], ax[0], ax[1], ax[2]);
  count_launches(1);
  return check_launch("grid_upsample");
}

}  // extern "C"
