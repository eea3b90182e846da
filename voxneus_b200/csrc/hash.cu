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
#include "hashgrid.cuh"

namespace vx {

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
        gather_level(tab, c, f0, f1);
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

// Adjoint of the hash encoding, four threads per sample: thread (i, g) scatters levels
// [g*lpt, (g+1)*lpt), lpt = ceil(L/4), loading its d_out values before the first atomic so the
// loads overlap; float4 atomics for the x-pairs of even cells (scatter_level).
__global__ void __launch_bounds__(256) k_hash_bwd(HashArgs a) {
  const uint32_t mask = (1u << a.log2T) - 1u;
  const size_t T = (size_t)1 << a.log2T;
  const int lpt = (a.L + 3) >> 2;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < a.P * 4; e += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = e >> 2;
    const int l0 = (int)(e & 3) * lpt;
    const int l1 = min(l0 + lpt, a.L);
    if (l0 >= l1) continue;
    const float* drow = a.d_out + i * a.ld_d;
    float g[16];  // lpt <= 8 (L <= 32)
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int l = l0 + q;
      g[2 * q] = l < l1 ? drow[2 * l] : 0.0f;
      g[2 * q + 1] = l < l1 ? drow[2 * l + 1] : 0.0f;
    }
    float x[3];
    sample_pos(a, i, x);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int l = l0 + q;
      if (l >= l1) break;
      const float lw = a.lw[l];
      if (lw == 0.0f) continue;
      float g0 = g[2 * q], g1 = g[2 * q + 1];
      if (lw < 1.0f) {
        g0 *= lw;
        g1 *= lw;
      }
      if (g0 == 0.0f && g1 == 0.0f) continue;
      LevelCell c;
      level_cell(x, a.res[l], mask, c);
      float2* tab = reinterpret_cast<float2*>(a.table_grad) + (size_t)l * T;
      scatter_level(tab, c, g0, g1);
    }
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
  // 32 blocks a SM (4 resident): more, shorter blocks keep the atomics' tail short (0.118 ->
  // 0.111 ms at 1M samples against 16)
  k_hash_bwd<<<grid_for(n_points * 4, 256, 32), 256, 0, (cudaStream_t)stream>>>(a);
  count_launches(1);
  return check_launch("hash_encode_backward");
}

}  // extern "C"
