// Deterministic adjoint scatters: sorted segmented reduction instead of float atomics.
//
// The geometry adjoint (SDF corners + the 48 Eq.7 stencil terms per sample) and the hash-table
// adjoint (8 corners x 2 features per level per sample) emit (destination index, value) pairs
// at fixed slots (sample-major), a stable radix sort groups them by destination, and one thread
// per destination sums its run in slot order and adds it to the gradient. The summation order
// depends only on the inputs, so the result is bitwise reproducible run to run. Pairs whose
// destination is out of range carry the sentinel key `n_dest` and are dropped.
#include <cub/device/device_radix_sort.cuh>

#include "common.cuh"

namespace vx {

constexpr int kGeoPairs = 56;  // 8 grid_sample corners + 8 corners x 6 central-difference taps

__global__ void __launch_bounds__(256) k_geometry_pairs(const float* __restrict__ f, Grid g,
                                                        const float* __restrict__ rays_o,
                                                        const float* __restrict__ rays_d,
                                                        const float* __restrict__ mid, int64_t n, int S,
                                                        const float* __restrict__ d_sdf,
                                                        const float* __restrict__ d_normal,
                                                        const float* __restrict__ d_normal2, int64_t ld2,
                                                        uint32_t* __restrict__ keys, float* __restrict__ vals,
                                                        uint32_t sentinel) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t* K = keys + i * kGeoPairs;
    float* V = vals + i * kGeoPairs;
    const int64_t r = i / S;
    const float t = mid[i];
    const float px = ray_at(__ldg(rays_o + 3 * r), __ldg(rays_d + 3 * r), t);
    const float py = ray_at(__ldg(rays_o + 3 * r + 1), __ldg(rays_d + 3 * r + 1), t);
    const float pz = ray_at(__ldg(rays_o + 3 * r + 2), __ldg(rays_d + 3 * r + 2), t);
    const float ds = d_sdf ? d_sdf[i] : 0.0f;
    Tri tr;
    gs_setup(g, px, py, pz, tr);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const bool ok = (tr.inb >> k) & 1u;
      const int x = tr.x0 + ((k >> 2) & 1), y = tr.y0 + ((k >> 1) & 1), z = tr.z0 + (k & 1);
      K[k] = ok ? (uint32_t)lin3(g, x, y, z) : sentinel;
      V[k] = ok ? tr.w[k] * ds : 0.0f;
    }
    float dn[3] = {0.f, 0.f, 0.f};
    if (d_normal) {
      dn[0] = d_normal[3 * i];
      dn[1] = d_normal[3 * i + 1];
      dn[2] = d_normal[3 * i + 2];
    }
    if (d_normal2) {
      dn[0] += d_normal2[i * ld2];
      dn[1] += d_normal2[i * ld2 + 1];
      dn[2] += d_normal2[i * ld2 + 2];
    }
    Eq7 e;
    eq7_setup(g, px, py, pz, e);
    float w[8], gr[3], nn[3], len, dg[3];
    eq7_weights(e, w);
    eq7_gradient(f, g, e, w, gr);
    normalize_eps(gr, nn, len);
    normalize_eps_bwd(gr, len, dn, dg);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int x = (k & 4) ? e.x1 : e.x0;
      const int y = (k & 2) ? e.y1 : e.y0;
      const int z = (k & 1) ? e.z1 : e.z0;
      const int xp = min(x + 1, g.rx - 1), xm = max(x - 1, 0);
      const int yp = min(y + 1, g.ry - 1), ym = max(y - 1, 0);
      const int zp = min(z + 1, g.rz - 1), zm = max(z - 1, 0);
      const float vx = (w[k] * dg[0]) / fd_den(xp, xm, g.eps[0]);
      const float vy = (w[k] * dg[1]) / fd_den(yp, ym, g.eps[1]);
      const float vz = (w[k] * dg[2]) / fd_den(zp, zm, g.eps[2]);
      uint32_t* KK = K + 8 + 6 * k;
      float* VV = V + 8 + 6 * k;
      KK[0] = lin3(g, xp, y, z);
      VV[0] = vx;
      KK[1] = lin3(g, xm, y, z);
      VV[1] = -vx;
      KK[2] = lin3(g, x, yp, z);
      VV[2] = vy;
      KK[3] = lin3(g, x, ym, z);
      VV[3] = -vy;
      KK[4] = lin3(g, x, y, zp);
      VV[4] = vz;
      KK[5] = lin3(g, x, y, zm);
      VV[5] = -vz;
    }
  }
}

// One thread per run head: sum the run in order and add it to out[key].
__global__ void __launch_bounds__(256) k_segmented_add(const uint32_t* __restrict__ keys,
                                                       const float* __restrict__ vals, int64_t n, uint32_t sentinel,
                                                       float* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t k = keys[i];
    if (k >= sentinel) continue;
    if (i > 0 && keys[i - 1] == k) continue;
    float acc = 0.0f;
    int64_t j = i;
    while (j < n && keys[j] == k) {
      acc += vals[j];
      ++j;
    }
    out[k] += acc;
  }
}

// Hash-table adjoint pairs: destination = float index into the (L, T, 2) table.
__global__ void __launch_bounds__(256) k_hash_pairs(const float* __restrict__ rays_o, const float* __restrict__ rays_d,
                                                    const float* __restrict__ mid, const float* __restrict__ pts, int S,
                                                    float lo0, float lo1, float lo2, float den0, float den1, float den2,
                                                    int L, int log2T, const int* __restrict__ res_d,
                                                    const float* __restrict__ lw_d, int64_t n,
                                                    const float* __restrict__ d_out, int64_t ld_d,
                                                    uint32_t* __restrict__ keys, float* __restrict__ vals,
                                                    uint32_t sentinel) {
  const uint32_t mask = (1u << log2T) - 1u;
  const uint32_t T = 1u << log2T;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float x[3];
    if (pts) {
      x[0] = pts[3 * i];
      x[1] = pts[3 * i + 1];
      x[2] = pts[3 * i + 2];
    } else {
      const int64_t r = i / S;
      const float t = mid[i];
      const float lo[3] = {lo0, lo1, lo2}, den[3] = {den0, den1, den2};
#pragma unroll
      for (int c = 0; c < 3; ++c)
        x[c] = __fdiv_rn(__fsub_rn(ray_at(__ldg(rays_o + 3 * r + c), __ldg(rays_d + 3 * r + c), t), lo[c]), den[c]);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) x[c] = fminf(fmaxf(x[c], 0.0f), 1.0f);
    uint32_t* K = keys + i * (int64_t)L * 16;
    float* V = vals + i * (int64_t)L * 16;
    for (int l = 0; l < L; ++l) {
      const float lw = lw_d[l];
      float g0 = d_out[i * ld_d + 2 * l], g1 = d_out[i * ld_d + 2 * l + 1];
      if (lw < 1.0f) {
        g0 *= lw;
        g1 *= lw;
      }
      const float fr = (float)res_d[l];
      int c0[3];
      float dd[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const float s = x[k] * fr;
        const float fl = floorf(s);
        c0[k] = (int)fl;
        dd[k] = s - fl;
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const uint32_t cx = (uint32_t)(c0[0] + ((k >> 2) & 1));
        const uint32_t cy = (uint32_t)(c0[1] + ((k >> 1) & 1));
        const uint32_t cz = (uint32_t)(c0[2] + (k & 1));
        const uint32_t h = (cx * 1u ^ cy * 2654435761u ^ cz * 805459861u) & mask;
        const float w = ((k & 4) ? dd[0] : 1.0f - dd[0]) * ((k & 2) ? dd[1] : 1.0f - dd[1]) *
                        ((k & 1) ? dd[2] : 1.0f - dd[2]);
        const uint32_t base = ((uint32_t)l * T + h) * 2u;
        const bool on = lw != 0.0f;
        K[l * 16 + 2 * k] = on ? base : sentinel;
        V[l * 16 + 2 * k] = w * g0;
        K[l * 16 + 2 * k + 1] = on ? base + 1u : sentinel;
        V[l * 16 + 2 * k + 1] = w * g1;
      }
    }
  }
}

static int key_bits(uint64_t sentinel) {
  int b = 1;
  while (b < 32 && (uint64_t(1) << b) <= sentinel) ++b;
  return b;
}

struct Workspace {
  uint32_t* k_in;
  uint32_t* k_out;
  float* v_in;
  float* v_out;
  void* temp;
  size_t temp_bytes;
};

static size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

static int carve(void* ws, size_t ws_bytes, int64_t n_pairs, int bits, Workspace& w, size_t* need) {
  size_t temp = 0;
  cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, temp, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                                  (float*)nullptr, (float*)nullptr, (int)n_pairs, 0, bits);
  if (e != cudaSuccess) return set_error(VX_ERR_CUDA, "radix sort sizing: %s", cudaGetErrorString(e));
  const size_t b4 = align256((size_t)n_pairs * 4);
  const size_t total = 4 * b4 + align256(temp);
  if (need) *need = total;
  if (!ws) return VX_OK;
  VX_REQUIRE(ws_bytes >= total, "workspace holds %zu bytes, need %zu", ws_bytes, total);
  char* p = (char*)ws;
  w.k_in = (uint32_t*)p;
  w.k_out = (uint32_t*)(p + b4);
  w.v_in = (float*)(p + 2 * b4);
  w.v_out = (float*)(p + 3 * b4);
  w.temp = p + 4 * b4;
  w.temp_bytes = temp;
  return VX_OK;
}

static int sort_and_add(Workspace& w, int64_t n_pairs, int bits, uint32_t sentinel, float* out, cudaStream_t st) {
  size_t tb = w.temp_bytes;
  cudaError_t e = cub::DeviceRadixSort::SortPairs(w.temp, tb, w.k_in, w.k_out, w.v_in, w.v_out, (int)n_pairs, 0,
                                                  bits, st);
  if (e != cudaSuccess) return set_error(VX_ERR_CUDA, "radix sort: %s", cudaGetErrorString(e));
  k_segmented_add<<<grid_for(n_pairs, 256), 256, 0, st>>>(w.k_out, w.v_out, n_pairs, sentinel, out);
  return VX_OK;
}

}  // namespace vx

using namespace vx;

extern "C" {

size_t vx_geometry_backward_det_workspace(int64_t n_rays, int n_samples, const int32_t res[3]) {
  const int64_t n = n_rays * n_samples * kGeoPairs;
  if (n <= 0 || n >= (int64_t(1) << 31)) return 0;
  const uint64_t nvox = (uint64_t)res[0] * res[1] * res[2];
  Workspace w;
  size_t need = 0;
  if (carve(nullptr, 0, n, key_bits(nvox), w, &need)) return 0;
  return need;
}

int vx_render_geometry_backward_det(const float* grid, const int32_t res[3], const float xyz_min[3],
                                    const float xyz_max[3], const float* rays_o, const float* rays_d, const float* mid,
                                    int64_t n_rays, int n_samples, const float* d_sdf, const float* d_normal,
                                    const float* d_normal2, int64_t ld2, float* grid_grad, void* workspace,
                                    size_t workspace_bytes, void* stream) {
  VX_REQUIRE(res && res[0] >= 2 && res[1] >= 2 && res[2] >= 2, "grid resolution must be >= 2 per axis");
  const uint64_t nvox = (uint64_t)res[0] * res[1] * res[2];
  VX_REQUIRE(nvox < (uint64_t(1) << 31), "grid has 2^31 or more voxels");
  VX_REQUIRE(n_rays >= 0 && n_samples >= 1, "bad sizes");
  VX_REQUIRE(!d_normal2 || ld2 >= 3, "ld2 must be >= 3");
  const int64_t n = n_rays * n_samples;
  if (n == 0) return VX_OK;
  VX_REQUIRE(n * kGeoPairs < (int64_t(1) << 31), "too many samples for one deterministic pass");
  VX_REQUIRE(grid && rays_o && rays_d && mid && grid_grad && xyz_min && xyz_max && workspace, "null pointer");
  const int bits = key_bits(nvox);
  Workspace w;
  if (int s = carve(workspace, workspace_bytes, n * kGeoPairs, bits, w, nullptr)) return s;
  Grid g = make_grid(res, xyz_min, xyz_max);
  cudaStream_t st = (cudaStream_t)stream;
  k_geometry_pairs<<<grid_for(n, 256), 256, 0, st>>>(grid, g, rays_o, rays_d, mid, n, n_samples, d_sdf, d_normal,
                                                      d_normal2, ld2, w.k_in, w.v_in, (uint32_t)nvox);
  if (int s = sort_and_add(w, n * kGeoPairs, bits, (uint32_t)nvox, grid_grad, st)) return s;
  count_launches(3);
  return check_launch("render_geometry_backward_det");
}

size_t vx_hash_backward_det_workspace(int64_t n_points, int n_levels, int log2_size) {
  const int64_t n = n_points * n_levels * 16;
  if (n <= 0 || n >= (int64_t(1) << 31) || log2_size > 26) return 0;
  const uint64_t ndest = (uint64_t)n_levels << (log2_size + 1);
  Workspace w;
  size_t need = 0;
  if (carve(nullptr, 0, n, key_bits(ndest), w, &need)) return 0;
  return need;
}

int vx_hash_encode_backward_det(float* table_grad, int n_levels, int log2_size, int n_features,
                                const int32_t* level_res_dev, const float* level_weights_dev, const float* pts_norm,
                                const float* rays_o, const float* rays_d, const float* mid, int n_samples,
                                const float xyz_min[3], const float xyz_max[3], int64_t n_points, const float* d_out,
                                int64_t ld_d, void* workspace, size_t workspace_bytes, void* stream) {
  VX_REQUIRE(n_levels >= 1 && n_levels <= 32 && log2_size >= 1 && log2_size <= 26, "bad hash configuration");
  VX_REQUIRE(n_features == 2, "only 2 features per level are supported");
  VX_REQUIRE(n_points >= 0, "n_points < 0");
  if (n_points == 0) return VX_OK;
  const int64_t n = n_points * n_levels * 16;
  VX_REQUIRE(n < (int64_t(1) << 31), "too many points for one deterministic pass");
  VX_REQUIRE(table_grad && d_out && level_res_dev && level_weights_dev && workspace, "null pointer");
  VX_REQUIRE(pts_norm || (rays_o && rays_d && mid && n_samples >= 1 && xyz_min && xyz_max),
             "need normalised points or rays + midpoints + bounds");
  VX_REQUIRE(ld_d >= 2 * n_levels, "gradient row stride smaller than the hash feature width");
  const uint64_t ndest = (uint64_t)n_levels << (log2_size + 1);
  const int bits = key_bits(ndest);
  Workspace w;
  if (int s = carve(workspace, workspace_bytes, n, bits, w, nullptr)) return s;
  float lo[3] = {0, 0, 0}, den[3] = {1, 1, 1};
  if (!pts_norm)
    for (int c = 0; c < 3; ++c) {
      lo[c] = xyz_min[c];
      den[c] = (xyz_max[c] - xyz_min[c]) + 1e-8f;
    }
  cudaStream_t st = (cudaStream_t)stream;
  k_hash_pairs<<<grid_for(n_points, 256), 256, 0, st>>>(rays_o, rays_d, mid, pts_norm, n_samples > 0 ? n_samples : 1,
                                                         lo[0], lo[1], lo[2], den[0], den[1], den[2], n_levels,
                                                         log2_size, level_res_dev, level_weights_dev, n_points, d_out,
                                                         ld_d, w.k_in, w.v_in, (uint32_t)ndest);
  if (int s = sort_and_add(w, n, bits, (uint32_t)ndest, table_grad, st)) return s;
  count_launches(3);
  return check_launch("hash_encode_backward_det");
}

}  // extern "C"
