// Appearance hand-off: multiresolution hash encoding (models/radiance_hash.py:71-166),
// degree-4 spherical harmonics of the view direction (models/embedder.py:55-87) and the
// copy of the Eq.7 normal, written as one row per sample of the radiance MLP input
// ([hash 32 | SH 16 | normal 3], models/radiance_mlp.py:94-98).
//
// One thread per sample, all levels in a loop: each thread writes its own row, the 8 corner
// features of a level are float2 gathers from the (L, 2^19, 2) table (64 MiB at the default
// size, L2-resident), and the adjoint scatters with float2 atomics (sm_90+ vector atomics).
// Hash indices are computed in uint32 arithmetic: the low log2(T) bits of
// x*1 ^ y*2654435761 ^ z*805459861 equal the reference's int64 value modulo 2^log2(T).
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
  float lo[3], den[3];
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
      x[c] = __fdiv_rn(__fsub_rn(p, a.lo[c]), a.den[c]);
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

__device__ __forceinline__ void sh16(float x, float y, float z, float o[16]) {
  o[0] = 0.28209479177387814f;
  o[1] = -0.4886025119029199f * y;
  o[2] = 0.4886025119029199f * z;
  o[3] = -0.4886025119029199f * x;
  o[4] = 1.0925484305920792f * x * y;
  o[5] = -1.0925484305920792f * y * z;
  o[6] = 0.31539156525252005f * (2.0f * z * z - x * x - y * y);
  o[7] = -1.0925484305920792f * x * z;
  o[8] = 0.5462742152960396f * (x * x - y * y);
  o[9] = -0.5900435899266435f * y * (3.0f * x * x - y * y);
  o[10] = 2.890611442640554f * x * y * z;
  o[11] = -0.4570457994644658f * y * (4.0f * z * z - x * x - y * y);
  o[12] = 0.3731763325901154f * z * (2.0f * z * z - 3.0f * x * x - 3.0f * y * y);
  o[13] = -0.4570457994644658f * x * (4.0f * z * z - x * x - y * y);
  o[14] = 1.445305721320277f * z * (x * x - y * y);
  o[15] = -0.5900435899266435f * x * (x * x - 3.0f * y * y);
}

__global__ void __launch_bounds__(256) k_appearance_fwd(HashArgs a) {
  const uint32_t mask = (1u << a.log2T) - 1u;
  const size_t T = (size_t)1 << a.log2T;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.P; i += (int64_t)gridDim.x * blockDim.x) {
    float* row = a.out + i * a.ld;
    if (a.table) {
      float x[3];
      sample_pos(a, i, x);
#pragma unroll 1
      for (int l = 0; l < a.L; ++l) {
        const float lw = a.lw[l];
        if (lw == 0.0f) {
          row[2 * l] = 0.0f;
          row[2 * l + 1] = 0.0f;
          continue;
        }
        LevelCell c;
        level_cell(x, a.res[l], mask, c);
        const float2* tab = reinterpret_cast<const float2*>(a.table) + (size_t)l * T;
        float f0 = 0.0f, f1 = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const float2 e = __ldg(tab + c.h[k]);
          f0 = fmaf(c.w[k], e.x, f0);
          f1 = fmaf(c.w[k], e.y, f1);
        }
        if (lw < 1.0f) {
          f0 *= lw;
          f1 *= lw;
        }
        row[2 * l] = f0;
        row[2 * l + 1] = f1;
      }
    }
    if (a.sh_col >= 0) {
      float dx, dy, dz;
      if (a.dirs) {
        dx = a.dirs[i * a.dir_ss];
        dy = a.dirs[i * a.dir_ss + 1];
        dz = a.dirs[i * a.dir_ss + 2];
      } else {
        const int64_t r = i / a.S;
        dx = __ldg(a.rays_d + 3 * r);
        dy = __ldg(a.rays_d + 3 * r + 1);
        dz = __ldg(a.rays_d + 3 * r + 2);
      }
      float o[16];
      sh16(dx, dy, dz, o);
#pragma unroll
      for (int k = 0; k < 16; ++k) row[a.sh_col + k] = o[k];
    }
    if (a.nrm_col >= 0) {
      row[a.nrm_col] = a.normals[3 * i];
      row[a.nrm_col + 1] = a.normals[3 * i + 1];
      row[a.nrm_col + 2] = a.normals[3 * i + 2];
    }
    if (a.pad_col >= 0) row[a.pad_col] = 0.0f;
  }
}

__global__ void __launch_bounds__(256) k_hash_bwd(HashArgs a) {
  const uint32_t mask = (1u << a.log2T) - 1u;
  const size_t T = (size_t)1 << a.log2T;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.P; i += (int64_t)gridDim.x * blockDim.x) {
    const float* drow = a.d_out + i * a.ld_d;
    float x[3];
    sample_pos(a, i, x);
#pragma unroll 1
    for (int l = 0; l < a.L; ++l) {
      const float lw = a.lw[l];
      if (lw == 0.0f) continue;
      float g0 = drow[2 * l], g1 = drow[2 * l + 1];
      if (lw < 1.0f) {
        g0 *= lw;
        g1 *= lw;
      }
      if (g0 == 0.0f && g1 == 0.0f) continue;
      LevelCell c;
      level_cell(x, a.res[l], mask, c);
      float2* tab = reinterpret_cast<float2*>(a.table_grad) + (size_t)l * T;
#pragma unroll
      for (int k = 0; k < 8; ++k) atomicAdd(tab + c.h[k], make_float2(c.w[k] * g0, c.w[k] * g1));
    }
  }
}

static int fill_hash(HashArgs& a, const float* table, int n_levels, int log2_size, int n_features,
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

static void fill_positions(HashArgs& a, const float* pts_norm, const float* rays_o, const float* rays_d,
                           const float* mid, int S, const float xyz_min[3], const float xyz_max[3]) {
  a.pts = pts_norm;
  a.rays_o = rays_o;
  a.rays_d = rays_d;
  a.mid = mid;
  a.S = S > 0 ? S : 1;
  for (int c = 0; c < 3; ++c) {
    a.lo[c] = xyz_min ? xyz_min[c] : 0.f;
    a.den[c] = xyz_min ? (xyz_max[c] - xyz_min[c]) + 1e-8f : 1.f;
  }
}

}  // namespace vx

using namespace vx;

extern "C" {

int vx_appearance_forward(const float* table, int n_levels, int log2_size, int n_features, const int32_t* level_res,
                          const float* level_weights, const float* pts_norm, const float* rays_o, const float* rays_d,
                          const float* mid, int n_samples, const float xyz_min[3], const float xyz_max[3],
                          int64_t n_points, float* out, int64_t ld, int sh_col, const float* dirs,
                          int64_t dir_stride, int normal_col, const float* normals, int pad_col, void* stream) {
  HashArgs a{};
  if (table) {
    if (int s = fill_hash(a, table, n_levels, log2_size, n_features, level_res, level_weights)) return s;
  } else {
    a.table = nullptr;
    a.L = 0;
  }
  VX_REQUIRE(n_points >= 0, "n_points < 0");
  if (n_points == 0) return VX_OK;
  VX_REQUIRE(out, "out is null");
  VX_REQUIRE(!table || pts_norm || (rays_o && rays_d && mid && n_samples >= 1 && xyz_min && xyz_max),
             "need normalised points or rays + midpoints + bounds");
  VX_REQUIRE(!table || ld >= 2 * n_levels, "row stride smaller than the hash feature width");
  VX_REQUIRE(sh_col < 0 || (sh_col + 16 <= ld && (dirs || rays_d)), "bad SH column or missing directions");
  VX_REQUIRE(normal_col < 0 || (normal_col + 3 <= ld && normals), "bad normal column or missing normals");
  VX_REQUIRE(pad_col < ld, "bad pad column");
  fill_positions(a, pts_norm, rays_o, rays_d, mid, n_samples, pts_norm ? nullptr : xyz_min, xyz_max);
  a.P = n_points;
  a.out = out;
  a.ld = ld;
  a.sh_col = sh_col;
  a.dirs = dirs;
  a.dir_ss = dir_stride;
  a.nrm_col = normal_col;
  a.normals = normals;
  a.pad_col = pad_col;
  k_appearance_fwd<<<grid_for(n_points, 256), 256, 0, (cudaStream_t)stream>>>(a);
  count_launches(1);
  return check_launch("appearance_forward");
}

int vx_hash_encode_backward(float* table_grad, int n_levels, int log2_size, int n_features, const int32_t* level_res,
                            const float* level_weights, const float* pts_norm, const float* rays_o,
                            const float* rays_d, const float* mid, int n_samples, const float xyz_min[3],
                            const float xyz_max[3], int64_t n_points, const float* d_out, int64_t ld_d,
                            void* stream) {
  HashArgs a{};
  if (int s = fill_hash(a, nullptr, n_levels, log2_size, n_features, level_res, level_weights)) return s;
  VX_REQUIRE(n_points >= 0, "n_points < 0");
  if (n_points == 0) return VX_OK;
  VX_REQUIRE(table_grad && d_out, "null pointer");
  VX_REQUIRE(pts_norm || (rays_o && rays_d && mid && n_samples >= 1 && xyz_min && xyz_max),
             "need normalised points or rays + midpoints + bounds");
  VX_REQUIRE(ld_d >= 2 * n_levels, "gradient row stride smaller than the hash feature width");
  fill_positions(a, pts_norm, rays_o, rays_d, mid, n_samples, pts_norm ? nullptr : xyz_min, xyz_max);
  a.table_grad = table_grad;
  a.P = n_points;
  a.d_out = d_out;
  a.ld_d = ld_d;
  k_hash_bwd<<<grid_for(n_points, 256), 256, 0, (cudaStream_t)stream>>>(a);
  count_launches(1);
  return check_launch("hash_encode_backward");
}

}  // extern "C"
