// SDF-grid field queries: trilinear SDF (S2), Eq.7 interpolated gradients and normals
// (S3/S8), their adjoints, the reference-compatible gradient_interp pair, and the lattice
// query of the large-grid workload.
//
// One thread per point, grid-stride loops over a grid sized to the 148 SMs. The 32-value
// Eq.7 stencil is read through the read-only path; a 256^3 grid (64 MiB) is L2-resident,
// so neighbouring samples of a ray hit L1/L2.
#include "common.cuh"

namespace vx {

__global__ void __launch_bounds__(256) k_gradient_interp_fwd(const float* __restrict__ f, Grid g,
                                                             const float* __restrict__ coords, int64_t n,
                                                             float* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    Eq7 e;
    eq7_setup_grid_coords(g, coords[3 * i], coords[3 * i + 1], coords[3 * i + 2], e);
    float w[8], gr[3];
    eq7_weights(e, w);
    eq7_gradient(f, g, e, w, gr);
    out[3 * i] = gr[0];
    out[3 * i + 1] = gr[1];
    out[3 * i + 2] = gr[2];
  }
}

__global__ void __launch_bounds__(256) k_gradient_interp_bwd(const float* __restrict__ dout,
                                                             const float* __restrict__ coords, int64_t n, Grid g,
                                                             float* __restrict__ gg) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    Eq7 e;
    eq7_setup_grid_coords(g, coords[3 * i], coords[3 * i + 1], coords[3 * i + 2], e);
    float w[8];
    eq7_weights(e, w);
    const float dg[3] = {dout[3 * i], dout[3 * i + 1], dout[3 * i + 2]};
    eq7_scatter(gg, g, e, w, dg);
  }
}

// sdf / grad / normal / corners / weights for world points; every output optional.
__global__ void __launch_bounds__(256) k_field_query(const float* __restrict__ f, Grid g,
                                                     const float* __restrict__ xyz, int64_t n,
                                                     float* __restrict__ sdf, float* __restrict__ grad,
                                                     float* __restrict__ normal, int64_t* __restrict__ corners,
                                                     float* __restrict__ weights) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float px = xyz[3 * i], py = xyz[3 * i + 1], pz = xyz[3 * i + 2];
    if (sdf && !(grad || normal)) sdf[i] = query_sdf(f, g, px, py, pz);
    if (grad || normal || corners || weights) {
      Eq7 e;
      eq7_setup(g, px, py, pz, e);
      float w[8];
      eq7_weights(e, w);
      if (grad || normal) {
        float c[8], gr[3], nn[3], len;  // the cell's corner values, shared by the SDF and the gradient
        eq7_load_block(f, g, e, c);
        if (sdf) sdf[i] = query_sdf_block(f, g, px, py, pz, e, c);
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
      if (corners) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          int64_t* c = corners + (i * 8 + k) * 3;
          c[0] = (k & 4) ? e.x1 : e.x0;
          c[1] = (k & 2) ? e.y1 : e.y0;
          c[2] = (k & 1) ? e.z1 : e.z0;
        }
      }
      if (weights) {
#pragma unroll
        for (int k = 0; k < 8; ++k) weights[i * 8 + k] = w[k];
      }
    }
  }
}

// Adjoint of k_field_query with respect to the grid: d_sdf (n), d_grad (n,3), d_normal (n,3),
// each optional.
__global__ void __launch_bounds__(256, 4) k_field_query_bwd(const float* __restrict__ f, Grid g,
                                                         const float* __restrict__ xyz, int64_t n,
                                                         const float* __restrict__ d_sdf,
                                                         const float* __restrict__ d_grad,
                                                         const float* __restrict__ d_normal,
                                                         float* __restrict__ gg) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float px = xyz[3 * i], py = xyz[3 * i + 1], pz = xyz[3 * i + 2];
    if (d_sdf) {
      Tri t;
      gs_setup(g, px, py, pz, t);
      gs_scatter(gg, g, t, d_sdf[i]);
    }
    if (d_grad || d_normal) {
      Eq7 e;
      eq7_setup(g, px, py, pz, e);
      float w[8];
      eq7_weights(e, w);
      float dg[3] = {0.0f, 0.0f, 0.0f};
      if (d_normal) {
        float gr[3], nn[3], len;
        eq7_gradient(f, g, e, w, gr);
        normalize_eps(gr, nn, len);
        const float dn[3] = {d_normal[3 * i], d_normal[3 * i + 1], d_normal[3 * i + 2]};
        normalize_eps_bwd(gr, len, dn, dg);
      }
      if (d_grad) {
        dg[0] += d_grad[3 * i];
        dg[1] += d_grad[3 * i + 1];
        dg[2] += d_grad[3 * i + 2];
      }
      eq7_scatter(gg, g, e, w, dg);
    }
  }
}

// Lattice value: ATen's linspace split (start + step*i on the first half, end - step*(n-1-i)
// on the second), evaluated without FMA.
__device__ __forceinline__ float lattice_coord(float lo, float hi, int n, int i) {
  if (n <= 1) return lo;
  const float step = (hi - lo) / (float)(n - 1);
  if (i < n / 2) return __fadd_rn(lo, __fmul_rn(step, (float)i));
  return __fsub_rn(hi, __fmul_rn(step, (float)(n - 1 - i)));
}

__global__ void __launch_bounds__(256, 4) k_field_lattice(const float* __restrict__ f, Grid g, int nx, int ny, int nz,
                                                       float lx, float ly, float lz, float hx, float hy, float hz,
                                                       float* __restrict__ sdf, float* __restrict__ normal) {
  const int64_t total = (int64_t)nx * ny * nz;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int k = (int)(i % nz);
    const int64_t r = i / nz;
    const int j = (int)(r % ny);
    const int ii = (int)(r / ny);
    const float px = lattice_coord(lx, hx, nx, ii), py = lattice_coord(ly, hy, ny, j), pz = lattice_coord(lz, hz, nz, k);
    if (sdf && !normal) sdf[i] = query_sdf(f, g, px, py, pz);
    if (normal) {
      Eq7 e;
      eq7_setup(g, px, py, pz, e);
      float c[8], w[8], gr[3], nn[3], len;
      eq7_load_block(f, g, e, c);
      if (sdf) sdf[i] = query_sdf_block(f, g, px, py, pz, e, c);
      eq7_weights(e, w);
      eq7_gradient_block(f, g, e, w, c, gr);
      normalize_eps(gr, nn, len);
      normal[3 * i] = nn[0];
      normal[3 * i + 1] = nn[1];
      normal[3 * i + 2] = nn[2];
    }
  }
}

// Corners and weights at grid-index coordinates (geometry/coordinates.py:55-124).
__global__ void __launch_bounds__(256) k_corners_weights(Grid g, const float* __restrict__ coords, int64_t n,
                                                         int64_t* __restrict__ corners, float* __restrict__ weights) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    Eq7 e;
    eq7_setup_grid_coords(g, coords[3 * i], coords[3 * i + 1], coords[3 * i + 2], e);
    float w[8];
    eq7_weights(e, w);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      if (corners) {
        int64_t* c = corners + (i * 8 + k) * 3;
        c[0] = (k & 4) ? e.x1 : e.x0;
        c[1] = (k & 2) ? e.y1 : e.y0;
        c[2] = (k & 1) ? e.z1 : e.z0;
      }
      if (weights) weights[i * 8 + k] = w[k];
    }
  }
}

static Grid grid_from_eps(const int32_t res[3], const float eps[3]) {
  const float lo[3] = {0.f, 0.f, 0.f}, hi[3] = {1.f, 1.f, 1.f};
  Grid g = make_grid(res, lo, hi);
  for (int a = 0; a < 3; ++a) g.eps[a] = eps[a];
  return g;
}

}  // namespace vx

using namespace vx;

extern "C" {

int vx_gradient_interp_forward(const float* grid, const int32_t res[3], const float* coords, int64_t n,
                               const float eps[3], float* out_grad, void* stream) {
  if (int s = check_grid(res)) return s;
  VX_REQUIRE(n >= 0, "n < 0");
  if (n == 0) return VX_OK;
  VX_REQUIRE(grid && coords && out_grad && eps, "null pointer");
  Grid g = grid_from_eps(res, eps);
  k_gradient_interp_fwd<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(grid, g, coords, n, out_grad);
  count_launches(1);
  return check_launch("gradient_interp_forward");
}

int vx_gradient_interp_backward(const float* grad_out, const float* coords, int64_t n, float* grad_grid,
                                const int32_t res[3], const float eps[3], void* stream) {
  if (int s = check_grid(res)) return s;
  VX_REQUIRE(n >= 0, "n < 0");
  if (n == 0) return VX_OK;
  VX_REQUIRE(grad_out && coords && grad_grid && eps, "null pointer");
  Grid g = grid_from_eps(res, eps);
  k_gradient_interp_bwd<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(grad_out, coords, n, g, grad_grid);
  count_launches(1);
  return check_launch("gradient_interp_backward");
}

int vx_field_query(const float* grid, const int32_t res[3], const float xyz_min[3], const float xyz_max[3],
                   const float* xyz, int64_t n, float* sdf, float* grad, float* normal, int64_t* corners,
                   float* weights, void* stream) {
  if (int s = check_grid(res)) return s;
  VX_REQUIRE(n >= 0, "n < 0");
  if (n == 0) return VX_OK;
  VX_REQUIRE(grid && xyz && xyz_min && xyz_max, "null pointer");
  Grid g = make_grid(res, xyz_min, xyz_max);
  k_field_query<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(grid, g, xyz, n, sdf, grad, normal, corners,
                                                                      weights);
  count_launches(1);
  return check_launch("field_query");
}

int vx_field_query_backward(const float* grid, const int32_t res[3], const float xyz_min[3], const float xyz_max[3],
                            const float* xyz, int64_t n, const float* d_sdf, const float* d_grad,
                            const float* d_normal, float* grad_grid, void* stream) {
  if (int s = check_grid(res)) return s;
  VX_REQUIRE(n >= 0, "n < 0");
  if (n == 0 || (!d_sdf && !d_grad && !d_normal)) return VX_OK;
  VX_REQUIRE(grid && xyz && grad_grid && xyz_min && xyz_max, "null pointer");
  Grid g = make_grid(res, xyz_min, xyz_max);
  k_field_query_bwd<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(grid, g, xyz, n, d_sdf, d_grad, d_normal,
                                                                          grad_grid);
  count_launches(1);
  return check_launch("field_query_backward");
}

int vx_field_query_lattice(const float* grid, const int32_t res[3], const float xyz_min[3], const float xyz_max[3],
                           const int32_t lattice[3], const float lat_min[3], const float lat_max[3], float* sdf,
                           float* normal, void* stream) {
  if (int s = check_grid(res)) return s;
  VX_REQUIRE(lattice && lat_min && lat_max, "null pointer");
  VX_REQUIRE(lattice[0] > 0 && lattice[1] > 0 && lattice[2] > 0, "lattice size must be positive");
  VX_REQUIRE(grid && xyz_min && xyz_max, "null pointer");
  Grid g = make_grid(res, xyz_min, xyz_max);
  const int64_t total = (int64_t)lattice[0] * lattice[1] * lattice[2];
  k_field_lattice<<<grid_for(total, 256), 256, 0, (cudaStream_t)stream>>>(
      grid, g, lattice[0], lattice[1], lattice[2], lat_min[0], lat_min[1], lat_min[2], lat_max[0], lat_max[1],
      lat_max[2], sdf, normal);
  count_launches(1);
  return check_launch("field_query_lattice");
}

int vx_corners_weights(const float* coords, int64_t n, const int32_t res[3], int64_t* corners, float* weights,
                       void* stream) {
  if (int s = check_grid(res)) return s;
  VX_REQUIRE(n >= 0, "n < 0");
  if (n == 0) return VX_OK;
  VX_REQUIRE(coords && (corners || weights), "null pointer");
  const float eps[3] = {1.f, 1.f, 1.f};
  Grid g = grid_from_eps(res, eps);
  k_corners_weights<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(g, coords, n, corners, weights);
  count_launches(1);
  return check_launch("corners_weights");
}

}  // extern "C"
