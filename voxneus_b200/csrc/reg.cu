// Closed-form eikonal (Eq.10-11, regularization/eikonal.py:13-171) and Laplacian curvature
// (Eq.12-14, regularization/curvature.py:13-165) gradients written straight into the grid
// gradient.
//
// Two forms:
//  * list form (the reference's kernel interface, eikonal_grad.cu / curvature_grad.cu):
//    one thread per listed vertex, atomics into the gradient, scale 2/|list|;
//  * fused gather form for the training step: one pass over 32x4x4 voxel tiles of the
//    grid, skipping tiles with no active vertex. Each output voxel sums, in registers, the
//    contributions of the <= 7 active interior vertices whose stencil touches it (itself
//    and its 6 face neighbours), reading a halo-2 tile of the SDF from shared memory. No
//    atomics: the result is deterministic. The active set is the V_R bitmap with the relax
//    and narrow-band predicates, and |V_R| comes from the device-side counts.
// Both forms also reduce the monitoring losses (mean over interior vertices) through
// per-block partials and a last-block epilogue.
#include "common.cuh"

namespace vx {

struct RegOut {
  double* partials;       // 3 per block: eikonal sum, curvature sum, interior count
  unsigned int* counter;  // zero before the first launch; reset by the last block
  float* losses;          // [eikonal, curvature]
};

__device__ void reduce_losses(const RegOut& o, double e, double c, double n) {
  __shared__ double s[3][32];
  __shared__ bool is_last;
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int nthreads = blockDim.x * blockDim.y * blockDim.z;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int wl = tid & 31, ww = tid >> 5;
  (void)lane;
  (void)warp;
  e = warp_sum_d(e);
  c = warp_sum_d(c);
  n = warp_sum_d(n);
  if (wl == 0) {
    s[0][ww] = e;
    s[1][ww] = c;
    s[2][ww] = n;
  }
  __syncthreads();
  const unsigned nblocks = gridDim.x * gridDim.y * gridDim.z;
  const unsigned bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
  if (tid == 0) {
    double a = 0, b = 0, k = 0;
    for (int w = 0; w < (nthreads + 31) / 32; ++w) {
      a += s[0][w];
      b += s[1][w];
      k += s[2][w];
    }
    o.partials[3 * bid] = a;
    o.partials[3 * bid + 1] = b;
    o.partials[3 * bid + 2] = k;
    __threadfence();
    is_last = (atomicAdd(o.counter, 1u) == nblocks - 1);
  }
  __syncthreads();
  if (!is_last) return;
  // last block: every thread sums a fixed strided subset, then a fixed-order warp/block tree
  // (deterministic for a given launch shape)
  __threadfence();
  const volatile double* p = o.partials;
  double a = 0, b = 0, k = 0;
  for (unsigned i = tid; i < nblocks; i += nthreads) {
    a += p[3 * i];
    b += p[3 * i + 1];
    k += p[3 * i + 2];
  }
  a = warp_sum_d(a);
  b = warp_sum_d(b);
  k = warp_sum_d(k);
  __syncthreads();
  if (wl == 0) {
    s[0][ww] = a;
    s[1][ww] = b;
    s[2][ww] = k;
  }
  __syncthreads();
  if (tid == 0) {
    a = b = k = 0;
    for (int w = 0; w < (nthreads + 31) / 32; ++w) {
      a += s[0][w];
      b += s[1][w];
      k += s[2][w];
    }
    if (o.losses) {
      o.losses[0] = k > 0 ? (float)(a / k) : 0.0f;
      o.losses[1] = k > 0 ? (float)(b / k) : 0.0f;
    }
    *o.counter = 0u;
  }
}

// ------------------------------------ list form --------------------------------------------

__global__ void __launch_bounds__(256) k_eikonal_list(const float* __restrict__ f, Grid g,
                                                      const int64_t* __restrict__ verts, int64_t nv,
                                                      float* __restrict__ gg, float weight, RegOut o) {
  double e = 0, n = 0;
  const float dx = 2.0f * g.eps[0], dy = 2.0f * g.eps[1], dz = 2.0f * g.eps[2];
  const int nblk = gridDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv; i += (int64_t)nblk * blockDim.x) {
    const int64_t vx_ = verts[3 * i], vy_ = verts[3 * i + 1], vz_ = verts[3 * i + 2];
    if (vx_ <= 0 || vx_ >= g.rx - 1 || vy_ <= 0 || vy_ >= g.ry - 1 || vz_ <= 0 || vz_ >= g.rz - 1) continue;
    const int x = (int)vx_, y = (int)vy_, z = (int)vz_;
    const float nx = (__ldg(f + lin3(g, x + 1, y, z)) - __ldg(f + lin3(g, x - 1, y, z))) / dx;
    const float ny = (__ldg(f + lin3(g, x, y + 1, z)) - __ldg(f + lin3(g, x, y - 1, z))) / dy;
    const float nz = (__ldg(f + lin3(g, x, y, z + 1)) - __ldg(f + lin3(g, x, y, z - 1))) / dz;
    const float len = sqrtf(nx * nx + ny * ny + nz * nz);
    const float scale = (2.0f / (float)nv) * (1.0f - 1.0f / (len + 1e-8f)) * weight;
    const float ax = scale * nx, ay = scale * ny, az = scale * nz;
    if (gg) {
      atomicAdd(gg + lin3(g, x + 1, y, z), ax / dx);
      atomicAdd(gg + lin3(g, x - 1, y, z), -ax / dx);
      atomicAdd(gg + lin3(g, x, y + 1, z), ay / dy);
      atomicAdd(gg + lin3(g, x, y - 1, z), -ay / dy);
      atomicAdd(gg + lin3(g, x, y, z + 1), az / dz);
      atomicAdd(gg + lin3(g, x, y, z - 1), -az / dz);
    }
    const double l = sqrt((double)nx * nx + (double)ny * ny + (double)nz * nz + 1e-16);
    e += (l - 1.0) * (l - 1.0);
    n += 1.0;
  }
  reduce_losses(o, e, 0.0, n);
}

__global__ void __launch_bounds__(256) k_curvature_list(const float* __restrict__ f, Grid g,
                                                        const int64_t* __restrict__ verts, int64_t nv,
                                                        float* __restrict__ gg, float weight, RegOut o) {
  double c = 0, n = 0;
  const float ex2 = g.eps[0] * g.eps[0], ey2 = g.eps[1] * g.eps[1], ez2 = g.eps[2] * g.eps[2];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nv; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t vx_ = verts[3 * i], vy_ = verts[3 * i + 1], vz_ = verts[3 * i + 2];
    if (vx_ <= 0 || vx_ >= g.rx - 1 || vy_ <= 0 || vy_ >= g.ry - 1 || vz_ <= 0 || vz_ >= g.rz - 1) continue;
    const int x = (int)vx_, y = (int)vy_, z = (int)vz_;
    const float fc = __ldg(f + lin3(g, x, y, z));
    const float Lx = (__ldg(f + lin3(g, x + 1, y, z)) + __ldg(f + lin3(g, x - 1, y, z)) - 2.0f * fc) / ex2;
    const float Ly = (__ldg(f + lin3(g, x, y + 1, z)) + __ldg(f + lin3(g, x, y - 1, z)) - 2.0f * fc) / ey2;
    const float Lz = (__ldg(f + lin3(g, x, y, z + 1)) + __ldg(f + lin3(g, x, y, z - 1)) - 2.0f * fc) / ez2;
    const float scale = (2.0f / (float)nv) * weight;
    if (gg) {
      atomicAdd(gg + lin3(g, x, y, z), scale * (-2.0f * Lx / ex2 - 2.0f * Ly / ey2 - 2.0f * Lz / ez2));
      atomicAdd(gg + lin3(g, x + 1, y, z), scale * (Lx / ex2));
      atomicAdd(gg + lin3(g, x - 1, y, z), scale * (Lx / ex2));
      atomicAdd(gg + lin3(g, x, y + 1, z), scale * (Ly / ey2));
      atomicAdd(gg + lin3(g, x, y - 1, z), scale * (Ly / ey2));
      atomicAdd(gg + lin3(g, x, y, z + 1), scale * (Lz / ez2));
      atomicAdd(gg + lin3(g, x, y, z - 1), scale * (Lz / ez2));
    }
    c += (double)Lx * Lx + (double)Ly * Ly + (double)Lz * Lz;
    n += 1.0;
  }
  reduce_losses(o, 0.0, c, n);
}

// ------------------------------------ gather form ------------------------------------------

constexpr int TZ = 32, TY = 4, TX = 4;  // output tile (z fastest)
constexpr int HZ = TZ + 4, HY = TY + 4, HX = TX + 4;  // SDF box, halo 2
constexpr int MZ = TZ + 2, MY = TY + 2, MX = TX + 2;  // vertex box, halo 1
constexpr int NVB = MX * MY * MZ;                      // vertices in the halo-1 box

struct StencilArgs {
  const float* f;
  const uint32_t* fb;  // filtered V_R bitmaps from vx_vr_count: [bits & band | bits & band & relax]
  int64_t nwords;
  Grid g;
  const unsigned long long* counts;  // from vx_vr_count
  float relax_r;
  float w_eik, w_curv;
  float* gg;
  int tiles_z, tiles_y;
};

__device__ __forceinline__ void tile_origin(const StencilArgs& a, int t, int& x0, int& y0, int& z0) {
  const int tz = t % a.tiles_z;
  const int ty = (t / a.tiles_z) % a.tiles_y;
  const int tx = t / (a.tiles_z * a.tiles_y);
  z0 = tz * TZ;
  y0 = ty * TY;
  x0 = tx * TX;
}

// Does the halo-1 box of tile t hold any V_R vertex? Word-level test of the filtered bitmap by
// one warp, one lane per (x, y) row of the box (z range [z0-1, z0+TZ] covers at most 3 words).
__device__ __forceinline__ bool tile_has_bits_warp(const StencilArgs& a, const uint32_t* bm, int t, int lane) {
  int x0, y0, z0;
  tile_origin(a, t, x0, y0, z0);
  bool hit = false;
  for (int r = lane; r < MX * MY; r += 32) {
    const int x = x0 - 1 + r / MY, y = y0 - 1 + r % MY;
    if (x < 0 || x >= a.g.rx || y < 0 || y >= a.g.ry) continue;
    const int zlo = max(z0 - 1, 0), zhi = min(z0 + TZ, a.g.rz - 1);
    const int b0 = lin3(a.g, x, y, zlo), b1 = lin3(a.g, x, y, zhi);
    for (int w = b0 >> 5; w <= (b1 >> 5); ++w) {
      uint32_t m = 0xffffffffu;
      if (w == (b0 >> 5)) m &= 0xffffffffu << (b0 & 31);
      if (w == (b1 >> 5)) m &= 0xffffffffu >> (31 - (b1 & 31));
      hit |= (__ldg(bm + w) & m) != 0u;
    }
  }
  return __any_sync(0xffffffffu, hit);
}

// Persistent grid over 32x4x4 tiles taken 8 at a time; blockDim = (32, 4, 2). Each warp tests one
// tile of the batch against the filtered bitmap, so an empty tile costs one load per lane. For
// an active tile: stage the SDF box (halo 2); evaluate every active interior vertex of the halo-1
// box once, storing the contribution it makes to itself (curvature centre) and to each face
// neighbour (eikonal +-dL/dn_a / 2eps_a plus curvature L_a/eps_a^2, scaled); then every output
// voxel sums the <= 7 terms that land on it. Per-block loss partials; k_reg_finalize reduces them.
__global__ void __launch_bounds__(256) k_reg_stencil(StencilArgs a, double* __restrict__ partials, int ntiles) {
  __shared__ float F[HX][HY][HZ];
  __shared__ float T[7][NVB];  // [0] centre, [1+2a] to v+e_a, [2+2a] to v-e_a
  __shared__ double red[3][8];
  __shared__ int active[8];
  const int tid = threadIdx.x + 32 * (threadIdx.y + 4 * threadIdx.z);
  const bool relax_on = a.relax_r > 0.0f && a.counts[1] > 0;
  const bool band_on = a.counts[2] != a.counts[0] || a.counts[3] != a.counts[1];
  (void)band_on;
  const uint32_t* bm = a.fb + (relax_on ? a.nwords : 0);
  // |V_R| after the filters: counts[1 or 3] (relax) / counts[0 or 2] (no relax); the filtered
  // bitmaps already carry the band, so the band count is the one to use
  const unsigned long long nv = relax_on ? a.counts[3] : a.counts[2];
  const float inv_nv = nv > 0 ? 2.0f / (float)nv : 0.0f;
  const float dx = 2.0f * a.g.eps[0], dy = 2.0f * a.g.eps[1], dz = 2.0f * a.g.eps[2];
  const float ex2 = a.g.eps[0] * a.g.eps[0], ey2 = a.g.eps[1] * a.g.eps[1], ez2 = a.g.eps[2] * a.g.eps[2];
  const float sc = inv_nv * a.w_curv;
  double le = 0, lc = 0, ln = 0;
  for (int tb = blockIdx.x * 8; tb < ntiles; tb += gridDim.x * 8) {
    {
      const int w = tid >> 5;
      const bool hit = (tb + w < ntiles) ? tile_has_bits_warp(a, bm, tb + w, tid & 31) : false;
      if ((tid & 31) == 0) active[w] = hit;
    }
    __syncthreads();
    for (int wt = 0; wt < 8; ++wt) {
      if (!active[wt]) continue;
      int x0, y0, z0;
      tile_origin(a, tb + wt, x0, y0, z0);
      for (int q = tid; q < HX * HY * HZ; q += 256) {
        const int hz = q % HZ, hy = (q / HZ) % HY, hx = q / (HZ * HY);
        const int x = x0 - 2 + hx, y = y0 - 2 + hy, z = z0 - 2 + hz;
        float v = 0.0f;
        if (x >= 0 && x < a.g.rx && y >= 0 && y < a.g.ry && z >= 0 && z < a.g.rz)
          v = __ldg(a.f + lin3(a.g, x, y, z));
        F[hx][hy][hz] = v;
      }
      __syncthreads();
      // per-vertex terms of the halo-1 box
      for (int q = tid; q < NVB; q += 256) {
        const int mz = q % MZ, my = (q / MZ) % MY, mx = q / (MZ * MY);
        const int x = x0 - 1 + mx, y = y0 - 1 + my, z = z0 - 1 + mz;
        bool on = x >= 1 && x <= a.g.rx - 2 && y >= 1 && y <= a.g.ry - 2 && z >= 1 && z <= a.g.rz - 2;
        if (on) {
          const int idx = lin3(a.g, x, y, z);
          on = (__ldg(bm + (idx >> 5)) >> (idx & 31)) & 1u;
        }
        float t0 = 0.f, tpx = 0.f, tmx = 0.f, tpy = 0.f, tmy = 0.f, tpz = 0.f, tmz = 0.f;
        if (on) {
          const int hx = mx + 1, hy = my + 1, hz = mz + 1;
          const float fc = F[hx][hy][hz];
          const float fxp = F[hx + 1][hy][hz], fxm = F[hx - 1][hy][hz];
          const float fyp = F[hx][hy + 1][hz], fym = F[hx][hy - 1][hz];
          const float fzp = F[hx][hy][hz + 1], fzm = F[hx][hy][hz - 1];
          const float Lx = (fxp + fxm - 2.0f * fc) / ex2;
          const float Ly = (fyp + fym - 2.0f * fc) / ey2;
          const float Lz = (fzp + fzm - 2.0f * fc) / ez2;
          const float nx = (fxp - fxm) / dx, ny = (fyp - fym) / dy, nz = (fzp - fzm) / dz;
          const float len = sqrtf(nx * nx + ny * ny + nz * nz);
          // eikonal_grad.cu: scale = 2/|V_R| (1 - 1/(|n| + 1e-8)) w; +-scale*n_a / (2 eps_a)
          const float se = inv_nv * (1.0f - 1.0f / (len + 1e-8f)) * a.w_eik;
          const float ex = (se * nx) / dx, ey = (se * ny) / dy, ez = (se * nz) / dz;
          // curvature_grad.cu: centre scale*(-2 Lx/ex^2 - 2 Ly/ey^2 - 2 Lz/ez^2), neighbours scale*L_a/eps_a^2
          const float cx = sc * (Lx / ex2), cy = sc * (Ly / ey2), cz = sc * (Lz / ez2);
          t0 = sc * (-2.0f * Lx / ex2 - 2.0f * Ly / ey2 - 2.0f * Lz / ez2);
          tpx = ex + cx;
          tmx = -ex + cx;
          tpy = ey + cy;
          tmy = -ey + cy;
          tpz = ez + cz;
          tmz = -ez + cz;
          if (mx >= 1 && mx <= TX && my >= 1 && my <= TY && mz >= 1 && mz <= TZ) {  // owned by this tile
            const double l = sqrt((double)nx * nx + (double)ny * ny + (double)nz * nz + 1e-16);
            le += (l - 1.0) * (l - 1.0);
            lc += (double)Lx * Lx + (double)Ly * Ly + (double)Lz * Lz;
            ln += 1.0;
          }
        }
        T[0][q] = t0;
        T[1][q] = tpx;
        T[2][q] = tmx;
        T[3][q] = tpy;
        T[4][q] = tmy;
        T[5][q] = tpz;
        T[6][q] = tmz;
      }
      __syncthreads();
      const int lz = threadIdx.x, ly = threadIdx.y;
#pragma unroll
      for (int rep = 0; rep < 2; ++rep) {
        const int lx = threadIdx.z + 2 * rep;
        const int x = x0 + lx, y = y0 + ly, z = z0 + lz;
        if (x >= a.g.rx || y >= a.g.ry || z >= a.g.rz) continue;
        const int c = ((lx + 1) * MY + (ly + 1)) * MZ + (lz + 1);  // this voxel in the vertex box
        float acc = T[0][c];
        acc += T[1][c - MY * MZ] + T[2][c + MY * MZ];  // from v - e_x (to v + e_x) and v + e_x (to v - e_x)
        acc += T[3][c - MZ] + T[4][c + MZ];
        acc += T[5][c - 1] + T[6][c + 1];
        if (acc != 0.0f) {
          float* p = a.gg + lin3(a.g, x, y, z);
          *p += acc;
        }
      }
      __syncthreads();  // F and T are rewritten by the next tile
    }
    __syncthreads();  // active[] is rewritten by the next batch
  }
  le = warp_sum_d(le);
  lc = warp_sum_d(lc);
  ln = warp_sum_d(ln);
  const int wl = tid & 31, ww = tid >> 5;
  if (wl == 0) {
    red[0][ww] = le;
    red[1][ww] = lc;
    red[2][ww] = ln;
  }
  __syncthreads();
  if (tid == 0) {
    double s0 = 0, s1 = 0, s2 = 0;
    for (int w = 0; w < 8; ++w) {
      s0 += red[0][w];
      s1 += red[1][w];
      s2 += red[2][w];
    }
    partials[3 * blockIdx.x] = s0;
    partials[3 * blockIdx.x + 1] = s1;
    partials[3 * blockIdx.x + 2] = s2;
  }
}

// Mean losses over interior vertices from the per-block partials, fixed reduction order.
__global__ void __launch_bounds__(256) k_reg_finalize(const double* __restrict__ partials, int nblocks,
                                                      float* __restrict__ losses) {
  __shared__ double red[3][8];
  double a = 0, b = 0, k = 0;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
    a += partials[3 * i];
    b += partials[3 * i + 1];
    k += partials[3 * i + 2];
  }
  a = warp_sum_d(a);
  b = warp_sum_d(b);
  k = warp_sum_d(k);
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = a;
    red[1][threadIdx.x >> 5] = b;
    red[2][threadIdx.x >> 5] = k;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    a = b = k = 0;
    for (int w = 0; w < 8; ++w) {
      a += red[0][w];
      b += red[1][w];
      k += red[2][w];
    }
    losses[0] = k > 0 ? (float)(a / k) : 0.0f;
    losses[1] = k > 0 ? (float)(b / k) : 0.0f;
  }
}

static int check_reg(const int32_t res[3]) {
  VX_REQUIRE(res && res[0] >= 3 && res[1] >= 3 && res[2] >= 3, "grid resolution must be >= 3 per axis");
  VX_REQUIRE((int64_t)res[0] * res[1] * res[2] < (int64_t(1) << 31), "grid has 2^31 or more voxels");
  return VX_OK;
}

static Grid grid_eps(const int32_t res[3], const float eps[3]) {
  const float lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
  Grid g = make_grid(res, lo, hi);
  for (int a = 0; a < 3; ++a) g.eps[a] = eps[a];
  return g;
}

}  // namespace vx

using namespace vx;

extern "C" {

int vx_reg_list_blocks(int64_t n_verts) { return (int)grid_for(n_verts, 256, 4); }

int vx_eikonal_grad(const float* grid, const int32_t res[3], const int64_t* verts, int64_t n_verts, float* grad_grid,
                    const float eps[3], float weight, double* partials, int n_partials, unsigned int* counter,
                    float* losses, void* stream) {
  if (int s = check_reg(res)) return s;
  VX_REQUIRE(n_verts >= 0, "n_verts < 0");
  if (n_verts == 0) return VX_OK;
  VX_REQUIRE(grid && verts && eps && partials && counter, "null pointer");
  const int blocks = vx_reg_list_blocks(n_verts);
  VX_REQUIRE(n_partials >= 3 * blocks, "partials buffer too small (%d < %d)", n_partials, 3 * blocks);
  RegOut o{partials, counter, losses};
  k_eikonal_list<<<blocks, 256, 0, (cudaStream_t)stream>>>(grid, grid_eps(res, eps), verts, n_verts, grad_grid,
                                                            weight, o);
  count_launches(1);
  return check_launch("eikonal_grad");
}

int vx_curvature_grad(const float* grid, const int32_t res[3], const int64_t* verts, int64_t n_verts,
                      float* grad_grid, const float eps[3], float weight, double* partials, int n_partials,
                      unsigned int* counter, float* losses, void* stream) {
  if (int s = check_reg(res)) return s;
  VX_REQUIRE(n_verts >= 0, "n_verts < 0");
  if (n_verts == 0) return VX_OK;
  VX_REQUIRE(grid && verts && eps && partials && counter, "null pointer");
  const int blocks = vx_reg_list_blocks(n_verts);
  VX_REQUIRE(n_partials >= 3 * blocks, "partials buffer too small (%d < %d)", n_partials, 3 * blocks);
  RegOut o{partials, counter, losses};
  k_curvature_list<<<blocks, 256, 0, (cudaStream_t)stream>>>(grid, grid_eps(res, eps), verts, n_verts, grad_grid,
                                                              weight, o);
  count_launches(1);
  return check_launch("curvature_grad");
}

static int64_t stencil_tiles(const int32_t res[3]) {
  return (int64_t)((res[2] + TZ - 1) / TZ) * ((res[1] + TY - 1) / TY) * ((res[0] + TX - 1) / TX);
}

int64_t vx_reg_stencil_blocks(const int32_t res[3]) {
  const int64_t t = (stencil_tiles(res) + 7) / 8;  // tiles are taken 8 per block iteration
  const int64_t cap = (int64_t)kSMs * 4;
  return t < cap ? t : cap;
}

int vx_reg_stencil(const float* grid, const uint32_t* bitmap, const int32_t res[3], const float xyz_min[3],
                   const float xyz_max[3], float relax_radius, float band, const unsigned long long* counts,
                   float w_eik, float w_curv, float* grad_grid, double* partials, int64_t n_partials,
                   unsigned int* counter, float* losses, void* stream) {
  if (int s = check_reg(res)) return s;
  VX_REQUIRE(grid && bitmap && counts && grad_grid && partials && xyz_min && xyz_max, "null pointer");
  const int64_t nb = vx_reg_stencil_blocks(res);
  VX_REQUIRE(nb < (int64_t(1) << 31), "grid too large");
  VX_REQUIRE(n_partials >= 3 * nb, "partials buffer too small (%lld < %lld)", (long long)n_partials,
             (long long)(3 * nb));
  StencilArgs a;
  a.f = grid;
  a.fb = bitmap;
  a.nwords = ((int64_t)res[0] * res[1] * res[2] + 31) / 32;
  a.g = make_grid(res, xyz_min, xyz_max);
  a.counts = counts;
  a.relax_r = relax_radius;
  (void)band;
  a.w_eik = w_eik;
  a.w_curv = w_curv;
  a.gg = grad_grid;
  a.tiles_z = (res[2] + TZ - 1) / TZ;
  a.tiles_y = (res[1] + TY - 1) / TY;
  (void)counter;
  const int64_t ntiles = stencil_tiles(res);
  k_reg_stencil<<<(unsigned)nb, dim3(32, 4, 2), 0, (cudaStream_t)stream>>>(a, partials, (int)ntiles);
  if (losses) k_reg_finalize<<<1, 256, 0, (cudaStream_t)stream>>>(partials, (int)nb, losses);
  count_launches(losses ? 2 : 1);
  return check_launch("reg_stencil");
}

}  // extern "C"
