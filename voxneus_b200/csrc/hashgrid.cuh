// Multiresolution hash-grid helpers shared by the appearance kernels (models/radiance_hash.py:71-166,
// models/embedder.py:55-87).
#pragma once

#include "common.cuh"

namespace vx {

constexpr int kMaxLevels = 32;

struct HashArgs {
  const float* table;  // (L, T, 2)
  float* table_grad;   // adjoint output, (L, T, 2)
  int L, log2T;
  int res[kMaxLevels];
  float lw[kMaxLevels];  // NeuS2 lambda level weights (0 = skipped level)
  // position source: normalised points (P,3), or world positions o + d * t of (rays, S)
  const float* pts;
  const float* rays_o;
  const float* rays_d;
  const float* mid;
  int S;
  float lo[3], den[3], inv_den[3];
  int64_t P;
  float* out;  // rows of length >= 2L
  int64_t ld;
  const float* d_out;  // adjoint input rows
  int64_t ld_d;
  int sh_col;          // -1: no SH
  const float* dirs;   // per-sample dirs (row stride dir_ss) or per-ray via rays_d when null
  int64_t dir_ss;
  int nrm_col;         // -1: no normal copy
  const float* normals;
  int pad_col;         // -1: none; column set to 0
};

__device__ __forceinline__ void sample_pos(const HashArgs& a, int64_t i, float x[3]) {
  if (a.pts) {
    x[0] = a.pts[3 * i];
    x[1] = a.pts[3 * i + 1];
    x[2] = a.pts[3 * i + 2];
  } else {
    const int64_t r = i / a.S;
    const float t = a.mid[i];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float p = ray_at(__ldg(a.rays_o + 3 * r + c), __ldg(a.rays_d + 3 * r + c), t);
      x[c] = div_den(__fsub_rn(p, a.lo[c]), a.den[c], a.inv_den[c]);
    }
  }
  // RadianceHashGrid.forward clamps to [0, 1] (radiance_hash.py:213)
#pragma unroll
  for (int c = 0; c < 3; ++c) x[c] = fminf(fmaxf(x[c], 0.0f), 1.0f);
}

__device__ __forceinline__ uint32_t hash3(uint32_t x, uint32_t y, uint32_t z, uint32_t mask) {
  return (x * 1u ^ y * 2654435761u ^ z * 805459861u) & mask;
}

struct LevelCell {
  uint32_t h[8];
  float w[8];
  bool xpair;  // the cell's x index is even: corners k and k+4 (x, x+1) are entries h[k], h[k]^1
};

__device__ __forceinline__ void level_cell(const float x[3], int res, uint32_t mask, LevelCell& c) {
  const float fr = (float)res;
  int c0[3];
  float d[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float s = x[k] * fr;
    const float fl = floorf(s);
    c0[k] = (int)fl;
    d[k] = s - fl;
  }
  c.xpair = (c0[0] & 1) == 0;
  const float ox = 1.0f - d[0], oy = 1.0f - d[1], oz = 1.0f - d[2];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t cx = (uint32_t)(c0[0] + ((k >> 2) & 1));
    const uint32_t cy = (uint32_t)(c0[1] + ((k >> 1) & 1));
    const uint32_t cz = (uint32_t)(c0[2] + (k & 1));
    c.h[k] = hash3(cx, cy, cz, mask);
    c.w[k] = ((k & 4) ? d[0] : ox) * ((k & 2) ? d[1] : oy) * ((k & 1) ? d[2] : oz);
  }
}

// Trilinear blend of one level's 2 features, corners in the order 0..7. Corners k < 4 are read
// as the aligned 16-byte pair holding h[k]; when the cell's x index is even that pair also holds
// corner k+4 (hash bit 0 is x's bit 0), else corner k+4 is a separate 8-byte load. Same sums,
// same order as eight 8-byte loads; about a quarter fewer sectors touched.
__device__ __forceinline__ void gather_level(const float2* __restrict__ tab, const LevelCell& c, float& f0,
                                             float& f1) {
  float2 e[8];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(tab) + (c.h[k] >> 1));
    const bool odd = c.h[k] & 1u;
    e[k] = odd ? make_float2(v.z, v.w) : make_float2(v.x, v.y);
    e[k + 4] = odd ? make_float2(v.x, v.y) : make_float2(v.z, v.w);
  }
  if (!c.xpair) {
#pragma unroll
    for (int k = 4; k < 8; ++k) e[k] = __ldg(tab + c.h[k]);
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    f0 = fmaf(c.w[k], e[k].x, f0);
    f1 = fmaf(c.w[k], e[k].y, f1);
  }
}

// Adjoint of gather_level: one 16-byte atomic per x-pair when the cell's x index is even.
__device__ __forceinline__ void scatter_level(float2* __restrict__ tab, const LevelCell& c, float g0, float g1) {
  if (c.xpair) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float a0 = c.w[k] * g0, a1 = c.w[k] * g1, b0 = c.w[k + 4] * g0, b1 = c.w[k + 4] * g1;
      const bool odd = c.h[k] & 1u;
      atomicAdd(reinterpret_cast<float4*>(tab) + (c.h[k] >> 1),
                odd ? make_float4(b0, b1, a0, a1) : make_float4(a0, a1, b0, b1));
    }
  } else {
#pragma unroll
    for (int k = 0; k < 8; ++k) atomicAdd(tab + c.h[k], make_float2(c.w[k] * g0, c.w[k] * g1));
  }
}

// Degree-4 real spherical harmonics of a unit direction (models/embedder.py:55-87), four at a time:
// values 4k .. 4k+3. k is a constant at every call (an unrolled loop), so only that group is built.
// Every product and difference is rounded on its own, left to right as the reference's elementwise
// float32 tensor ops evaluate them (Python constants rounded to float32), so the values are the
// reference's bits in every kernel: no multiply-add is fused, whatever the surrounding code.
__device__ __forceinline__ float4 sh_chunk(float x, float y, float z, int k) {
  const float xx = __fmul_rn(x, x), yy = __fmul_rn(y, y);
  if (k == 0)
    return make_float4((float)0.28209479177387814, __fmul_rn((float)-0.4886025119029199, y),
                       __fmul_rn((float)0.4886025119029199, z), __fmul_rn((float)-0.4886025119029199, x));
  if (k == 1) {
    const float zz2 = __fmul_rn(__fmul_rn(2.0f, z), z);
    return make_float4(__fmul_rn(__fmul_rn((float)1.0925484305920792, x), y),
                       __fmul_rn(__fmul_rn((float)-1.0925484305920792, y), z),
                       __fmul_rn((float)0.31539156525252005, __fsub_rn(__fsub_rn(zz2, xx), yy)),
                       __fmul_rn(__fmul_rn((float)-1.0925484305920792, x), z));
  }
  if (k == 2) {
    const float zz4 = __fmul_rn(__fmul_rn(4.0f, z), z);
    return make_float4(__fmul_rn((float)0.5462742152960396, __fsub_rn(xx, yy)),
                       __fmul_rn(__fmul_rn((float)-0.5900435899266435, y),
                                 __fsub_rn(__fmul_rn(__fmul_rn(3.0f, x), x), yy)),
                       __fmul_rn(__fmul_rn(__fmul_rn((float)2.890611442640554, x), y), z),
                       __fmul_rn(__fmul_rn((float)-0.4570457994644658, y), __fsub_rn(__fsub_rn(zz4, xx), yy)));
  }
  const float zz2 = __fmul_rn(__fmul_rn(2.0f, z), z), zz4 = __fmul_rn(__fmul_rn(4.0f, z), z);
  const float xx3 = __fmul_rn(__fmul_rn(3.0f, x), x), yy3 = __fmul_rn(__fmul_rn(3.0f, y), y);
  return make_float4(__fmul_rn(__fmul_rn((float)0.3731763325901154, z), __fsub_rn(__fsub_rn(zz2, xx3), yy3)),
                     __fmul_rn(__fmul_rn((float)-0.4570457994644658, x), __fsub_rn(__fsub_rn(zz4, xx), yy)),
                     __fmul_rn(__fmul_rn((float)1.445305721320277, z), __fsub_rn(xx, yy)),
                     __fmul_rn(__fmul_rn((float)-0.5900435899266435, x), __fsub_rn(xx, yy3)));
}

__device__ __forceinline__ void sh16(float x, float y, float z, float o[16]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float4 v = sh_chunk(x, y, z, k);
    o[4 * k] = v.x;
    o[4 * k + 1] = v.y;
    o[4 * k + 2] = v.z;
    o[4 * k + 3] = v.w;
  }
}


inline int fill_hash(HashArgs& a, const float* table, int n_levels, int log2_size, int n_features,
                     const int32_t* level_res, const float* level_weights) {
  VX_REQUIRE(n_levels >= 1 && n_levels <= kMaxLevels, "n_levels must be in [1, %d]", kMaxLevels);
  VX_REQUIRE(log2_size >= 1 && log2_size <= 30, "log2 table size must be in [1, 30]");
  VX_REQUIRE(n_features == 2, "only 2 features per level are supported (got %d)", n_features);
  VX_REQUIRE(level_res, "level resolutions are null");
  a.table = table;
  a.L = n_levels;
  a.log2T = log2_size;
  for (int l = 0; l < n_levels; ++l) {
    VX_REQUIRE(level_res[l] >= 1, "level resolution must be >= 1");
    a.res[l] = level_res[l];
    a.lw[l] = level_weights ? level_weights[l] : 1.0f;
  }
  return VX_OK;
}

inline void fill_positions(HashArgs& a, const float* pts_norm, const float* rays_o, const float* rays_d,
                           const float* mid, int S, const float xyz_min[3], const float xyz_max[3]) {
  a.pts = pts_norm;
  a.rays_o = rays_o;
  a.rays_d = rays_d;
  a.mid = mid;
  a.S = S > 0 ? S : 1;
  for (int c = 0; c < 3; ++c) {
    a.lo[c] = xyz_min ? xyz_min[c] : 0.f;
    a.den[c] = xyz_min ? (xyz_max[c] - xyz_min[c]) + 1e-8f : 1.f;
    a.inv_den[c] = pow2_recip(a.den[c]);
  }
}


}  // namespace vx
