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
constexpr int MY = TY + 2, MX = TX + 2;  // halo-1 box extents in y and x

struct StencilArgs {
  const float* f;
  const uint32_t* fb;  // filtered V_R bitmaps from vx_vr_count: [bits & band | bits & band & relax]
  int64_t nwords;
  Grid g;
  const unsigned long long* counts;  // from vx_vr_count
  float relax_r;
  float w_eik, w_curv;
  float* gg;
  int tiles_z, tiles_y, tiles_x;
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

struct StencilConsts {
  float inv_nv, dx, dy, dz, ex2, ey2, ez2, sc, w_eik;
};

// What active vertex (x, y, z) adds to itself (t0: curvature centre) and to its face neighbours
// (tp[a] to v + e_a, tm[a] to v - e_a: eikonal +-scale n_a / (2 eps_a) plus curvature scale L_a /
// eps_a^2), with scale = 2/|V_R| (1 - 1/(|n| + 1e-8)) w_eik and sc = 2/|V_R| w_curv
// (eikonal_grad.cu, curvature_grad.cu); also its two loss terms.
__device__ __forceinline__ void vertex_terms(const StencilArgs& a, const StencilConsts& k, int x, int y, int z,
                                             float& t0, float tp[3], float tm[3], double* loss) {
  const float* f = a.f;
  const int c = lin3(a.g, x, y, z);
  const int sx = a.g.ry * a.g.rz, sy = a.g.rz;
  const float fc = __ldg(f + c);
  const float fxp = __ldg(f + c + sx), fxm = __ldg(f + c - sx);
  const float fyp = __ldg(f + c + sy), fym = __ldg(f + c - sy);
  const float fzp = __ldg(f + c + 1), fzm = __ldg(f + c - 1);
  const float Lx = (fxp + fxm - 2.0f * fc) / k.ex2;
  const float Ly = (fyp + fym - 2.0f * fc) / k.ey2;
  const float Lz = (fzp + fzm - 2.0f * fc) / k.ez2;
  const float nx = (fxp - fxm) / k.dx, ny = (fyp - fym) / k.dy, nz = (fzp - fzm) / k.dz;
  const float len = sqrtf(nx * nx + ny * ny + nz * nz);
  const float se = k.inv_nv * (1.0f - 1.0f / (len + 1e-8f)) * k.w_eik;
  const float ex = (se * nx) / k.dx, ey = (se * ny) / k.dy, ez = (se * nz) / k.dz;
  const float cx = k.sc * (Lx / k.ex2), cy = k.sc * (Ly / k.ey2), cz = k.sc * (Lz / k.ez2);
  t0 = k.sc * (-2.0f * Lx / k.ex2 - 2.0f * Ly / k.ey2 - 2.0f * Lz / k.ez2);
  tp[0] = ex + cx;
  tm[0] = -ex + cx;
  tp[1] = ey + cy;
  tm[1] = -ey + cy;
  tp[2] = ez + cz;
  tm[2] = -ez + cz;
  if (loss) {
    const double l = sqrt((double)nx * nx + (double)ny * ny + (double)nz * nz + 1e-16);
    loss[0] += (l - 1.0) * (l - 1.0);
    loss[1] += (double)Lx * Lx + (double)Ly * Ly + (double)Lz * Lz;
    loss[2] += 1.0;
  }
}

// V_R bits of the vertices (x, y, z0 - 1 .. z0 + 32) of one grid column as bits 0..33 of a word
// pair (vertices outside the interior read 0).
__device__ __forceinline__ uint64_t column_window(const StencilArgs& a, const uint32_t* __restrict__ bm, int x, int y,
                                                  int z0) {
  if (x < 1 || x > a.g.rx - 2 || y < 1 || y > a.g.ry - 2) return 0ull;
  const int64_t b = (int64_t)lin3(a.g, x, y, z0) - 1;  // bit of vertex z0 - 1 (may precede the column)
  const int64_t w0 = b >> 5;
  const int s = (int)(b & 31);
  const uint32_t u0 = (w0 >= 0 && w0 < a.nwords) ? __ldg(bm + w0) : 0u;
  const uint32_t u1 = (w0 + 1 < a.nwords) ? __ldg(bm + w0 + 1) : 0u;
  const uint32_t u2 = (s > 0 && w0 + 2 < a.nwords) ? __ldg(bm + w0 + 2) : 0u;
  uint64_t v = ((uint64_t)u1 << 32 | u0) >> s;
  if (s > 0) v |= (uint64_t)u2 << (64 - s);
  // keep interior z only: z = z0 - 1 + k in [1, rz - 2]
  const int klo = max(0, 2 - z0), khi = min(33, a.g.rz - 1 - z0);
  if (khi < klo) return 0ull;
  const uint64_t keep = ((khi >= 63 ? ~0ull : ((1ull << (khi + 1)) - 1ull))) & ~((1ull << klo) - 1ull);
  return v & keep;
}

__device__ __forceinline__ uint64_t shfl_u64(uint64_t v, int src) {
  const uint32_t lo = __shfl_sync(0xffffffffu, (uint32_t)v, src);
  const uint32_t hi = __shfl_sync(0xffffffffu, (uint32_t)(v >> 32), src);
  return (uint64_t)hi << 32 | lo;
}

// Does tile t own a vertex of the filtered V_R set? One thread per tile (its own voxels, no halo).
__global__ void __launch_bounds__(256) k_tile_flags(StencilArgs a, int ntiles, uint8_t* __restrict__ flags) {
  const bool relax_on = a.relax_r > 0.0f && a.counts[1] > 0;
  const uint32_t* bm = a.fb + (relax_on ? a.nwords : 0);
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) {
    int x0, y0, z0;
    tile_origin(a, t, x0, y0, z0);
    bool hit = false;
    const int z1 = min(z0 + TZ, a.g.rz) - 1;
    for (int q = 0; q < TX * TY && !hit; ++q) {
      const int x = x0 + q / TY, y = y0 + q % TY;
      if (x >= a.g.rx || y >= a.g.ry) continue;
      const int b0 = lin3(a.g, x, y, z0), b1 = lin3(a.g, x, y, z1);
      for (int w = b0 >> 5; w <= (b1 >> 5); ++w) {
        uint32_t m = 0xffffffffu;
        if (w == (b0 >> 5)) m &= 0xffffffffu << (b0 & 31);
        if (w == (b1 >> 5)) m &= 0xffffffffu >> (31 - (b1 & 31));
        hit |= (__ldg(bm + w) & m) != 0u;
      }
    }
    flags[t] = hit ? 1 : 0;
  }
}

// Fused eikonal + curvature gradient in gather form over 32x4x4 tiles. Warp w of the grid owns
// tiles w, w + W, w + 2W, ... (W warps); its lanes test 32 of them at once against the flags of the
// 3x3x3 tiles around each (a tile's outputs need the vertices of its halo), and the warp then
// works through the tiles that need it, one at a time, lane = z offset. Lane c < 36 loads the V_R
// window of column (x0 - 1 + c / 6, y0 - 1 + c % 6) of the tile's halo; each output voxel reads its
// 7 neighbour bits from those windows (warp shuffles of a uniform column) and sums, in a fixed
// order, the terms of the active ones, each evaluated from the SDF through L1 — V_R is a thin
// band, so few vertices are active. No atomics, no shared staging; per-block loss partials
// (fixed assignment and order) for k_reg_finalize.
__global__ void __launch_bounds__(256) k_reg_stencil(StencilArgs a, const uint8_t* __restrict__ flags,
                                                     double* __restrict__ partials, int ntiles) {
  __shared__ double red[3][8];
  __shared__ uint16_t vlist_all[8][MX * MY * (TZ + 2)];  // per warp: active vertices of the halo box
  __shared__ float acc_all[8][TX * TY * TZ];             // per warp: the tile's output sums
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint16_t* vlist = vlist_all[warp];
  float* acc_s = acc_all[warp];
  for (int o = lane; o < TX * TY * TZ; o += 32) acc_s[o] = 0.0f;
  __syncwarp();
  const bool relax_on = a.relax_r > 0.0f && a.counts[1] > 0;
  const uint32_t* bm = a.fb + (relax_on ? a.nwords : 0);
  // |V_R| after the filters: counts[3] (relax) / counts[2] (no relax); the filtered bitmaps
  // already carry the band, so the band count is the one to use
  const unsigned long long nv = relax_on ? a.counts[3] : a.counts[2];
  StencilConsts k;
  k.inv_nv = nv > 0 ? 2.0f / (float)nv : 0.0f;
  k.dx = 2.0f * a.g.eps[0];
  k.dy = 2.0f * a.g.eps[1];
  k.dz = 2.0f * a.g.eps[2];
  k.ex2 = a.g.eps[0] * a.g.eps[0];
  k.ey2 = a.g.eps[1] * a.g.eps[1];
  k.ez2 = a.g.eps[2] * a.g.eps[2];
  k.sc = k.inv_nv * a.w_curv;
  k.w_eik = a.w_eik;
  double loss[3] = {0.0, 0.0, 0.0};
  const int gw = blockIdx.x * 8 + warp, nw = gridDim.x * 8;
  for (int base = 0; gw + base * nw < ntiles; base += 32) {
    const int tl = gw + (base + lane) * nw;
    bool need = false;
    if (tl < ntiles) {
      const int tz = tl % a.tiles_z, ty = (tl / a.tiles_z) % a.tiles_y, tx = tl / (a.tiles_z * a.tiles_y);
      for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dz = -1; dz <= 1; ++dz) {
            const int nx = tx + dx, ny = ty + dy, nz = tz + dz;
            if (nx < 0 || nx >= a.tiles_x || ny < 0 || ny >= a.tiles_y || nz < 0 || nz >= a.tiles_z) continue;
            need |= __ldg(flags + ((int64_t)nx * a.tiles_y + ny) * a.tiles_z + nz) != 0;
          }
    }
    unsigned todo = __ballot_sync(0xffffffffu, need);
    while (todo) {
      const int b = __ffs(todo) - 1;
      todo &= todo - 1;
      const int t = gw + (base + b) * nw;
      int x0, y0, z0;
      tile_origin(a, t, x0, y0, z0);
      const uint64_t w0 = column_window(a, bm, x0 - 1 + lane / 6, y0 - 1 + lane % 6, z0);
      const uint64_t w1 =
          lane < 4 ? column_window(a, bm, x0 - 1 + (lane + 32) / 6, y0 - 1 + (lane + 32) % 6, z0) : 0ull;
      const int cnt0 = __popcll(w0), cnt1 = __popcll(w1);
      int incl = cnt0 + cnt1;  // inclusive warp prefix of the vertex counts (column order)
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      if (total == 0) continue;
      // compact the active vertices of the halo box: code = column * 34 + window bit
      int pos = incl - cnt0 - cnt1;
      for (uint64_t m = w0; m; m &= m - 1) vlist[pos++] = (uint16_t)(lane * 34 + __ffsll((long long)m) - 1);
      for (uint64_t m = w1; m; m &= m - 1) vlist[pos++] = (uint16_t)((lane + 32) * 34 + __ffsll((long long)m) - 1);
      __syncwarp();
      // evaluate each vertex once and add its 7 terms into the tile's accumulators in 7 ordered
      // passes (two vertices never share a target within a pass)
      for (int base = 0; base < total; base += 32) {
        const int idx = base + lane;
        float t0 = 0.0f, tp[3] = {0.0f, 0.0f, 0.0f}, tm[3] = {0.0f, 0.0f, 0.0f};
        int vx = 0, vy = 0, vz = 0;
        const bool mine = idx < total;
        if (mine) {
          const int code = vlist[idx], col = code / 34, kb = code - 34 * col;
          vx = x0 - 1 + col / MY;
          vy = y0 - 1 + col % MY;
          vz = z0 - 1 + kb;
          const bool owned = vx >= x0 && vx < x0 + TX && vy >= y0 && vy < y0 + TY && vz >= z0 && vz < z0 + TZ;
          vertex_terms(a, k, vx, vy, vz, t0, tp, tm, owned ? loss : nullptr);
        }
#pragma unroll
        for (int p = 0; p < 7; ++p) {
          const int ax = p == 1 ? 1 : (p == 2 ? -1 : 0), ay = p == 3 ? 1 : (p == 4 ? -1 : 0);
          const int az = p == 5 ? 1 : (p == 6 ? -1 : 0);
          const float term = p == 0 ? t0 : (p & 1) ? tp[(p - 1) >> 1] : tm[(p - 1) >> 1];
          const int ox = vx + ax - x0, oy = vy + ay - y0, oz = vz + az - z0;
          if (mine && ox >= 0 && ox < TX && oy >= 0 && oy < TY && oz >= 0 && oz < TZ)
            acc_s[(ox * TY + oy) * TZ + oz] += term;
          __syncwarp();
        }
      }
      // add the tile's sums to the gradient (z-contiguous lanes) and clear the accumulators
#pragma unroll 1
      for (int o = lane; o < TX * TY * TZ; o += 32) {
        const float v = acc_s[o];
        if (v != 0.0f) {
          const int ox = o / (TY * TZ), oy = (o / TZ) % TY, oz = o % TZ;
          a.gg[lin3(a.g, x0 + ox, y0 + oy, z0 + oz)] += v;
          acc_s[o] = 0.0f;
        }
      }
      __syncwarp();
    }
  }
  double le = warp_sum_d(loss[0]), lc = warp_sum_d(loss[1]), ln = warp_sum_d(loss[2]);
  if (lane == 0) {
    red[0][warp] = le;
    red[1][warp] = lc;
    red[2][warp] = ln;
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

// Mean losses over interior vertices from the per-block partials, fixed reduction order; and
// |V_R| after the filters (relax sphere when it keeps any vertex, band) for n_active.
__global__ void __launch_bounds__(256) k_reg_finalize(const double* __restrict__ partials, int nblocks,
                                                      float* __restrict__ losses,
                                                      const unsigned long long* __restrict__ counts, int relax,
                                                      int band, long long* __restrict__ n_active) {
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
    if (losses) {
      losses[0] = k > 0 ? (float)(a / k) : 0.0f;
      losses[1] = k > 0 ? (float)(b / k) : 0.0f;
    }
    if (n_active) {
      const bool relax_on = relax && counts[1] > 0;
      *n_active = (long long)(band ? (relax_on ? counts[3] : counts[2]) : (relax_on ? counts[1] : counts[0]));
    }
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
  const int64_t t = (stencil_tiles(res) + 7) / 8;  // at least one tile per warp
  const int64_t cap = (int64_t)kSMs * 4;
  return t < cap ? t : cap;
}

int64_t vx_reg_stencil_workspace(const int32_t res[3]) {
  // 3 loss doubles per block, then one flag byte per tile
  return 3 * vx_reg_stencil_blocks(res) + (stencil_tiles(res) + 7) / 8;
}

int vx_reg_stencil(const float* grid, const uint32_t* bitmap, const int32_t res[3], const float xyz_min[3],
                   const float xyz_max[3], float relax_radius, float band, const unsigned long long* counts,
                   float w_eik, float w_curv, float* grad_grid, double* partials, int64_t n_partials,
                   unsigned int* counter, float* losses, int64_t* n_active, void* stream) {
  if (int s = check_reg(res)) return s;
  VX_REQUIRE(grid && bitmap && counts && grad_grid && partials && xyz_min && xyz_max, "null pointer");
  const int64_t nb = vx_reg_stencil_blocks(res);
  const int64_t need = vx_reg_stencil_workspace(res);
  VX_REQUIRE(n_partials >= need, "workspace too small (%lld < %lld doubles)", (long long)n_partials,
             (long long)need);
  StencilArgs a;
  a.f = grid;
  a.fb = bitmap;
  a.nwords = ((int64_t)res[0] * res[1] * res[2] + 31) / 32;
  a.g = make_grid(res, xyz_min, xyz_max);
  a.counts = counts;
  a.relax_r = relax_radius;
  a.w_eik = w_eik;
  a.w_curv = w_curv;
  a.gg = grad_grid;
  a.tiles_z = (res[2] + TZ - 1) / TZ;
  a.tiles_y = (res[1] + TY - 1) / TY;
  a.tiles_x = (res[0] + TX - 1) / TX;
  (void)counter;
  const int64_t ntiles = stencil_tiles(res);
  uint8_t* flags = reinterpret_cast<uint8_t*>(partials + 3 * nb);
  cudaStream_t st = (cudaStream_t)stream;
  k_tile_flags<<<grid_for(ntiles, 256), 256, 0, st>>>(a, (int)ntiles, flags);
  k_reg_stencil<<<(unsigned)nb, 256, 0, st>>>(a, flags, partials, (int)ntiles);
  if (losses || n_active)
    k_reg_finalize<<<1, 256, 0, st>>>(partials, (int)nb, losses, counts, relax_radius > 0.0f ? 1 : 0,
                                      band > 0.0f ? 1 : 0, reinterpret_cast<long long*>(n_active));
  count_launches(losses || n_active ? 3 : 2);
  return check_launch("reg_stencil");
}

}  // extern "C"
