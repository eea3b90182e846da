// Occupancy-grid EMA update (rendering/occupancy_grid.py:62-119), the periodic refresh of the
// bitmask the sampler reads (training/trainer.py:171-173: every 16 steps, a random quarter of
// the 128^3 cells).
//
// The caller draws the cells (three int64 index vectors, torch.randint order x, y, z) so that the
// random stream is the reference's. Two launches:
//   k_occ_eval   per drawn cell: centre point, SDF (trilinear grid query or caller values),
//                logistic density s*sig*(1-sig), near-surface floor, EMA max with the previous
//                density; writes the new value and the cell's linear index to a workspace.
//   k_occ_store  scatters the values into the density grid and the thresholded mask.
// A cell drawn more than once reads the density from before the update in every draw and all
// draws write the same value, which is the result of the reference's gather-then-index_put; one
// fused launch could read a value another draw already wrote. Work per cell: 24 B of indices,
// one 4 B gather of the previous density, 8 SDF corners (the 96^3 grid stays in L2), 8 B
// workspace out and back, 5 B scattered out.
#include "common.cuh"

namespace vx {
namespace {

struct OccArgs {
  const float* sdf_grid;  // dense SDF grid, or null when sdf_values is given
  Grid g;
  const float* sdf_values;  // SDF at the drawn cells (n), used when sdf_grid is null
  int r;                    // occupancy resolution (cubic)
  float lo[3], span[3];     // occupancy bounds: xyz_min, xyz_max - xyz_min
  const int64_t *ix, *iy, *iz;
  int64_t n;
  const float* s_ptr;
  int s_is_variance;
  float s_max;
  float near_thr;       // float32(2 * |(xyz_max - xyz_min) / r|)
  float floor_density;  // float32(2 * threshold)
  float decay;
  int first;
};

// torch.maximum: NaN if either operand is NaN
__device__ __forceinline__ float max_nan(float a, float b) { return (a > b || a != a) ? a : b; }

// (float(i) + 0.5) / r mapped into [lo, lo + span] with the reference's roundings (no FMA)
__device__ __forceinline__ float cell_centre(int64_t i, int r, float lo, float span) {
  const float t = __fdiv_rn(__fadd_rn((float)i, 0.5f), (float)r);
  return __fadd_rn(lo, __fmul_rn(t, span));
}

__device__ __forceinline__ bool valid_cell(const OccArgs& a, int64_t x, int64_t y, int64_t z) {
  return (uint64_t)x < (uint64_t)a.r && (uint64_t)y < (uint64_t)a.r && (uint64_t)z < (uint64_t)a.r;
}

__global__ void __launch_bounds__(256) k_occ_points(OccArgs a, float* __restrict__ pts) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
    pts[3 * i + 0] = cell_centre(__ldg(a.ix + i), a.r, a.lo[0], a.span[0]);
    pts[3 * i + 1] = cell_centre(__ldg(a.iy + i), a.r, a.lo[1], a.span[1]);
    pts[3 * i + 2] = cell_centre(__ldg(a.iz + i), a.r, a.lo[2], a.span[2]);
  }
}

__global__ void __launch_bounds__(256) k_occ_eval(OccArgs a, const float* __restrict__ density,
                                                  float* __restrict__ upd, int32_t* __restrict__ cell,
                                                  unsigned int* __restrict__ n_invalid) {
  const float v = __ldg(a.s_ptr);
  // s = clamp(exp(10 v), 1e-4, s_max) (models/variance.py:38-41) when given the variance parameter
  const float s = a.s_is_variance ? fminf(fmaxf(expf(v * 10.0f), 1e-4f), a.s_max) : v;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
    const int64_t x = __ldg(a.ix + i), y = __ldg(a.iy + i), z = __ldg(a.iz + i);
    if (!valid_cell(a, x, y, z)) {
      cell[i] = -1;
      if (n_invalid) atomicAdd(n_invalid, 1u);
      continue;
    }
    float f;
    if (a.sdf_grid) {
      f = query_sdf(a.sdf_grid, a.g, cell_centre(x, a.r, a.lo[0], a.span[0]), cell_centre(y, a.r, a.lo[1], a.span[1]),
                    cell_centre(z, a.r, a.lo[2], a.span[2]));
    } else {
      f = __ldg(a.sdf_values + i);
    }
    // logistic density (occupancy_grid.py:15-22): (s * sig) * (1 - sig), sig = sigmoid(s * sdf)
    const float sig = sigmoidf_ref(__fmul_rn(s, f));
    const float dens = __fmul_rn(__fmul_rn(s, sig), __fsub_rn(1.0f, sig));
    // near-surface floor (:106-108): near * (2 threshold), near = |sdf| < 2 |voxel step|
    float e = max_nan(dens, fabsf(f) < a.near_thr ? a.floor_density : 0.0f);
    const int32_t c = (int32_t)((x * a.r + y) * a.r + z);
    if (!a.first) e = max_nan(__fmul_rn(__ldg(density + c), a.decay), e);
    upd[i] = e;
    cell[i] = c;
  }
}

__global__ void __launch_bounds__(256) k_occ_store(const float* __restrict__ upd, const int32_t* __restrict__ cell,
                                                   int64_t n, float threshold, float* __restrict__ density,
                                                   uint8_t* __restrict__ mask) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int32_t c = cell[i];
    if (c < 0) continue;
    const float u = upd[i];
    density[c] = u;
    mask[c] = u > threshold ? 1 : 0;
  }
}

__global__ void __launch_bounds__(256) k_occ_query(Occ oc, const float* __restrict__ pts, int64_t n,
                                                   uint8_t* __restrict__ out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = occupied(oc, __ldg(pts + 3 * i), __ldg(pts + 3 * i + 1), __ldg(pts + 3 * i + 2)) ? 1 : 0;
}

int fill_occ(OccArgs& a, int32_t occ_res, const float occ_min[3], const float occ_max[3], const int64_t* ix,
             const int64_t* iy, const int64_t* iz, int64_t n) {
  VX_REQUIRE(occ_res >= 1 && (int64_t)occ_res * occ_res * occ_res < ((int64_t)1 << 31),
             "occupancy resolution %d out of range", occ_res);
  VX_REQUIRE(n >= 0, "n < 0");
  VX_REQUIRE(occ_min && occ_max, "null pointer");
  VX_REQUIRE(n == 0 || (ix && iy && iz), "null pointer");
  a = OccArgs{};
  a.r = occ_res;
  double d2 = 0.0;
  for (int k = 0; k < 3; ++k) {
    a.lo[k] = occ_min[k];
    a.span[k] = occ_max[k] - occ_min[k];
    const float st = a.span[k] / (float)occ_res;
    d2 += (double)st * (double)st;
  }
  // torch.linalg.norm(step) in float32, doubled in double, compared as float32
  a.near_thr = (float)(2.0 * (double)(float)sqrt(d2));
  a.ix = ix;
  a.iy = iy;
  a.iz = iz;
  a.n = n;
  return VX_OK;
}

}  // namespace
}  // namespace vx

using namespace vx;

extern "C" {

int64_t vx_occupancy_workspace(int64_t n) { return n <= 0 ? 0 : ((n * 4 + 15) / 16) * 16 * 2; }

int vx_occupancy_points(int32_t occ_res, const float occ_min[3], const float occ_max[3], const int64_t* idx_x,
                        const int64_t* idx_y, const int64_t* idx_z, int64_t n, float* pts, void* stream) {
  OccArgs a;
  if (int st = fill_occ(a, occ_res, occ_min, occ_max, idx_x, idx_y, idx_z, n)) return st;
  if (n == 0) return VX_OK;
  VX_REQUIRE(pts, "null pointer");
  k_occ_points<<<grid_for(n, 256, 8), 256, 0, (cudaStream_t)stream>>>(a, pts);
  count_launches(1);
  return check_launch("occupancy_points");
}

int vx_occupancy_query(const uint8_t* mask, int32_t occ_res, const float occ_min[3], const float occ_max[3],
                       const float* pts, int64_t n, uint8_t* occupied_out, void* stream) {
  VX_REQUIRE(occ_res >= 1 && (int64_t)occ_res * occ_res * occ_res < ((int64_t)1 << 31),
             "occupancy resolution %d out of range", occ_res);
  VX_REQUIRE(n >= 0, "n < 0");
  if (n == 0) return VX_OK;
  VX_REQUIRE(mask && occ_min && occ_max && pts && occupied_out, "null pointer");
  k_occ_query<<<grid_for(n, 256, 8), 256, 0, (cudaStream_t)stream>>>(make_occ(mask, occ_res, occ_min, occ_max), pts,
                                                                      n, occupied_out);
  count_launches(1);
  return check_launch("occupancy_query");
}

int vx_occupancy_update(const float* sdf_grid, const int32_t res[3], const float sdf_min[3], const float sdf_max[3],
                        const float* sdf_values, int32_t occ_res, const float occ_min[3], const float occ_max[3],
                        const int64_t* idx_x, const int64_t* idx_y, const int64_t* idx_z, int64_t n,
                        const float* s, int s_is_variance, float s_max, int first, float decay, float threshold,
                        float* density, uint8_t* mask, void* workspace, int64_t workspace_bytes,
                        unsigned int* n_invalid, void* stream) {
  OccArgs a;
  if (int st = fill_occ(a, occ_res, occ_min, occ_max, idx_x, idx_y, idx_z, n)) return st;
  VX_REQUIRE((sdf_grid != nullptr) != (sdf_values != nullptr), "exactly one of sdf_grid and sdf_values is required");
  if (sdf_grid) {
    if (int st = check_grid(res)) return st;
    VX_REQUIRE(sdf_min && sdf_max, "null pointer");
    a.sdf_grid = sdf_grid;
    a.g = make_grid(res, sdf_min, sdf_max);
  }
  a.sdf_values = sdf_values;
  if (n == 0) return VX_OK;
  VX_REQUIRE(s && density && mask && workspace, "null pointer");
  VX_REQUIRE(workspace_bytes >= vx_occupancy_workspace(n), "workspace holds %lld bytes, need %lld",
             (long long)workspace_bytes, (long long)vx_occupancy_workspace(n));
  VX_REQUIRE(((uintptr_t)workspace & 15) == 0, "workspace must be 16-byte aligned");
  a.s_ptr = s;
  a.s_is_variance = s_is_variance;
  a.s_max = s_max;
  a.first = first;
  a.decay = decay;
  a.floor_density = (float)((double)threshold * 2.0);
  float* upd = static_cast<float*>(workspace);
  int32_t* cell = reinterpret_cast<int32_t*>(static_cast<char*>(workspace) + vx_occupancy_workspace(n) / 2);
  const unsigned blocks = grid_for(n, 256, 8);
  k_occ_eval<<<blocks, 256, 0, (cudaStream_t)stream>>>(a, density, upd, cell, n_invalid);
  k_occ_store<<<blocks, 256, 0, (cudaStream_t)stream>>>(upd, cell, n, threshold, density, mask);
  count_launches(2);
  return check_launch("occupancy_update");
}

}  // extern "C"
