// Shared device helpers for the VoxNeuS sm_100a library.
//
// Data layout in HBM: the SDF grid is a dense row-major float32 volume (X, Y, Z) with z
// fastest, linear index = (x * Y + y) * Z + z (the reference's `(1,1,X,Y,Z)` parameter
// storage, models/sdf_grid.py:51). Every index is int32: the host rejects grids with
// 2^31 or more voxels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

#include "../../include/voxneus_b200.h"

namespace vx {

// ---------------------------------------------------------------------------------------
// Error state and launch accounting (host side, defined in capi.cu)
// ---------------------------------------------------------------------------------------
int set_error(int code, const char* fmt, ...);
int check_launch(const char* what);
void count_launches(int n);

#define VX_REQUIRE(cond, ...)                                         \
  do {                                                                \
    if (!(cond)) return ::vx::set_error(VX_ERR_INVALID, __VA_ARGS__); \
  } while (0)

constexpr int kSMs = 148;  // B200: 2 dies x 74 SMs

inline unsigned grid_for(int64_t n, int threads, int per_sm = 16) {
  int64_t b = (n + threads - 1) / threads;
  int64_t cap = (int64_t)kSMs * per_sm;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (unsigned)b;
}

// ---------------------------------------------------------------------------------------
// Grid description passed by value to kernels
// ---------------------------------------------------------------------------------------
struct Grid {
  int rx, ry, rz;
  float lo[3];   // xyz_min
  float den[3];  // (xyz_max - xyz_min) + 1e-8f, the reference's normalisation denominator
  float inv_den[3];  // 1 / den when den is a power of two (exact), else 0
  float eps[3];  // voxel size (xyz_max - xyz_min) / (res - 1)
  float hi_clamp[3];  // float32(res - 1.0001): Eq.7 coordinate clamp (coordinates.py:73-75)
};

// 1 / d when d is a power of two (then x / d == x * (1 / d) exactly for every float x), else 0.
__host__ inline float pow2_recip(float d) {
  int e = 0;
  const float m = std::frexp(d, &e);
  const float r = 1.0f / d;
  return (d > 0.0f && m == 0.5f && std::isnormal(r)) ? r : 0.0f;
}

// x / den with IEEE rounding; a multiplication when den is a power of two (inv = pow2_recip(den)).
__device__ __forceinline__ float div_den(float x, float den, float inv) {
  return inv != 0.0f ? __fmul_rn(x, inv) : __fdiv_rn(x, den);
}

__host__ inline Grid make_grid(const int32_t res[3], const float lo[3], const float hi[3]) {
  Grid g;
  g.rx = res[0];
  g.ry = res[1];
  g.rz = res[2];
  for (int a = 0; a < 3; ++a) {
    g.lo[a] = lo[a];
    float span = hi[a] - lo[a];
    g.den[a] = span + 1e-8f;
    g.inv_den[a] = pow2_recip(g.den[a]);
    g.eps[a] = span / ((float)res[a] - 1.0f);
    g.hi_clamp[a] = (float)((double)res[a] - 1.0001);
  }
  return g;
}

// Host check of a dense grid resolution: >= 2 per axis, fewer than 2^31 voxels (int32 indexing).
inline int check_grid(const int32_t res[3]) {
  VX_REQUIRE(res != nullptr, "res is null");
  VX_REQUIRE(res[0] >= 2 && res[1] >= 2 && res[2] >= 2, "grid resolution must be >= 2 per axis (got %d,%d,%d)",
             res[0], res[1], res[2]);
  VX_REQUIRE((int64_t)res[0] * res[1] * res[2] < (int64_t(1) << 31), "grid has 2^31 or more voxels");
  return VX_OK;
}

__device__ __forceinline__ int lin3(const Grid& g, int x, int y, int z) { return (x * g.ry + y) * g.rz + z; }
__device__ __forceinline__ int gdim(const Grid& g, int a) { return a == 0 ? g.rx : (a == 1 ? g.ry : g.rz); }

// Position along a ray with the reference's rounding: o + (d * t), two roundings, no FMA
// (voxneus.py:229-230, sampler.py:183).
__device__ __forceinline__ float ray_at(float o, float d, float t) { return __fadd_rn(o, __fmul_rn(d, t)); }

// ---------------------------------------------------------------------------------------
// Trilinear SDF with F.grid_sample semantics (bilinear 5-D, padding="border",
// align_corners=True) after the world -> [-1, 1] map of models/sdf_grid.py:105-118.
// ---------------------------------------------------------------------------------------
struct Tri {
  int x0, y0, z0;       // lower corner (may be R-1; the +1 corner is then out of bounds)
  float w[8];           // weights in corner order 000,001,...,111 (x slowest)
  unsigned inb;         // bit k set when corner k is inside the grid
};

__device__ __forceinline__ float gs_coord(float p, float lo, float den, float inv, int R) {
  float n = div_den(__fsub_rn(p, lo), den, inv);
  float g = __fsub_rn(__fmul_rn(n, 2.0f), 1.0f);
  // (g + 1) / 2 as a multiply by 0.5: dividing by a power of two is exact scaling, so the two give
  // the same bits (a rounded division costs a multi-instruction sequence per axis)
  float c = __fmul_rn(__fmul_rn(__fadd_rn(g, 1.0f), 0.5f), (float)(R - 1));
  c = fminf((float)(R - 1), fmaxf(c, 0.0f));
  return c;
}

__device__ __forceinline__ void gs_setup(const Grid& g, float px, float py, float pz, Tri& t) {
  const float cx = gs_coord(px, g.lo[0], g.den[0], g.inv_den[0], g.rx);
  const float cy = gs_coord(py, g.lo[1], g.den[1], g.inv_den[1], g.ry);
  const float cz = gs_coord(pz, g.lo[2], g.den[2], g.inv_den[2], g.rz);
  t.x0 = (int)floorf(cx);
  t.y0 = (int)floorf(cy);
  t.z0 = (int)floorf(cz);
  const float x1 = (float)(t.x0 + 1), y1 = (float)(t.y0 + 1), z1 = (float)(t.z0 + 1);
  const float fx0 = (float)t.x0, fy0 = (float)t.y0, fz0 = (float)t.z0;
  // ATen's grid_sampler_3d weight expressions, written in (x,y,z) = (D,H,W) order:
  // each weight is (W-term * H-term) * D-term.
  const float zl = z1 - cz, zh = cz - fz0;
  const float yl = y1 - cy, yh = cy - fy0;
  const float xl = x1 - cx, xh = cx - fx0;
  t.w[0] = (zl * yl) * xl;
  t.w[1] = (zh * yl) * xl;
  t.w[2] = (zl * yh) * xl;
  t.w[3] = (zh * yh) * xl;
  t.w[4] = (zl * yl) * xh;
  t.w[5] = (zh * yl) * xh;
  t.w[6] = (zl * yh) * xh;
  t.w[7] = (zh * yh) * xh;
  const bool bx1 = t.x0 + 1 < g.rx, by1 = t.y0 + 1 < g.ry, bz1 = t.z0 + 1 < g.rz;
  unsigned m = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    bool ok = (!(k & 4) || bx1) && (!(k & 2) || by1) && (!(k & 1) || bz1);
    m |= (ok ? 1u : 0u) << k;
  }
  t.inb = m;
}

__device__ __forceinline__ float gs_sample(const float* __restrict__ f, const Grid& g, const Tri& t) {
  float acc = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if (t.inb & (1u << k)) {
      const int x = t.x0 + ((k >> 2) & 1), y = t.y0 + ((k >> 1) & 1), z = t.z0 + (k & 1);
      acc = fmaf(__ldg(f + lin3(g, x, y, z)), t.w[k], acc);
    }
  }
  return acc;
}

__device__ __forceinline__ float query_sdf(const float* __restrict__ f, const Grid& g, float px, float py, float pz) {
  Tri t;
  gs_setup(g, px, py, pz, t);
  return gs_sample(f, g, t);
}

// ---------------------------------------------------------------------------------------
// Eq.7 interpolated gradient (geometry/coordinates.py:55-124 corners and weights,
// geometry/gradients.py:59-139 per-corner central differences, one-sided at the border).
// ---------------------------------------------------------------------------------------
struct Eq7 {
  int x0, y0, z0;  // lower corner, x0 <= R-2 (the clamp keeps coordinates below R-1)
  int x1, y1, z1;  // upper corner, clamped to R-1
  float dx, dy, dz;
};

__device__ __forceinline__ float eq7_coord(float p, float lo, float den, float inv, int R) {
  return __fmul_rn(div_den(__fsub_rn(p, lo), den, inv), (float)R - 1.0f);
}

__device__ __forceinline__ void eq7_setup_grid_coords(const Grid& g, float cx, float cy, float cz, Eq7& e) {
  // torch.clamp(x, 0, hi) == min(max(x, 0), hi)
  cx = fminf(fmaxf(cx, 0.0f), g.hi_clamp[0]);
  cy = fminf(fmaxf(cy, 0.0f), g.hi_clamp[1]);
  cz = fminf(fmaxf(cz, 0.0f), g.hi_clamp[2]);
  int x0 = (int)floorf(cx), y0 = (int)floorf(cy), z0 = (int)floorf(cz);
  x0 = min(max(x0, 0), g.rx - 1);
  y0 = min(max(y0, 0), g.ry - 1);
  z0 = min(max(z0, 0), g.rz - 1);
  e.x0 = x0;
  e.y0 = y0;
  e.z0 = z0;
  e.x1 = min(x0 + 1, g.rx - 1);
  e.y1 = min(y0 + 1, g.ry - 1);
  e.z1 = min(z0 + 1, g.rz - 1);
  e.dx = cx - (float)x0;
  e.dy = cy - (float)y0;
  e.dz = cz - (float)z0;
}

__device__ __forceinline__ void eq7_setup(const Grid& g, float px, float py, float pz, Eq7& e) {
  eq7_setup_grid_coords(g, eq7_coord(px, g.lo[0], g.den[0], g.inv_den[0], g.rx),
                        eq7_coord(py, g.lo[1], g.den[1], g.inv_den[1], g.ry),
                        eq7_coord(pz, g.lo[2], g.den[2], g.inv_den[2], g.rz), e);
}

__device__ __forceinline__ void eq7_weights(const Eq7& e, float w[8]) {
  const float ox = 1.0f - e.dx, oy = 1.0f - e.dy, oz = 1.0f - e.dz;
  w[0] = ox * oy * oz;
  w[1] = ox * oy * e.dz;
  w[2] = ox * e.dy * oz;
  w[3] = ox * e.dy * e.dz;
  w[4] = e.dx * oy * oz;
  w[5] = e.dx * oy * e.dz;
  w[6] = e.dx * e.dy * oz;
  w[7] = e.dx * e.dy * e.dz;
}

// One-sided-at-border difference denominators: max((p - m) * eps, eps).
__device__ __forceinline__ float fd_den(int p, int m, float eps) { return fmaxf((float)(p - m) * eps, eps); }

// Interpolated gradient g = sum_k w_k n[c_k].
// The 2x2x2 block of corner values (corner k: x bit 4, y bit 2, z bit 1).
__device__ __forceinline__ void eq7_load_block(const float* __restrict__ f, const Grid& g, const Eq7& e, float c[8]) {
#pragma unroll
  for (int k = 0; k < 8; ++k)
    c[k] = __ldg(f + lin3(g, (k & 4) ? e.x1 : e.x0, (k & 2) ? e.y1 : e.y0, (k & 1) ? e.z1 : e.z0));
}

// Eq.7 gradient from the corner block c: per corner the central differences of Eq.6 (indices
// clamped, one-sided at the border) blended with the corner weights. A corner's neighbour towards
// the other side of the cell is a block value (the lower corner's +1 neighbour is the upper corner by
// definition; the upper corner's -1 neighbour is the lower one unless the cell is degenerate at the
// border, then it is loaded), so a point loads 8 + 24 values instead of 48; the arithmetic and its
// order are those of the per-corner formula (geometry/gradients.py:59-139).
__device__ __forceinline__ void eq7_gradient_block(const float* __restrict__ f, const Grid& g, const Eq7& e,
                                                   const float w[8], const float c[8], float out[3]) {
  float gx = 0.0f, gy = 0.0f, gz = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int x = (k & 4) ? e.x1 : e.x0;
    const int y = (k & 2) ? e.y1 : e.y0;
    const int z = (k & 1) ? e.z1 : e.z0;
    const int xp = min(x + 1, g.rx - 1), xm = max(x - 1, 0);
    const int yp = min(y + 1, g.ry - 1), ym = max(y - 1, 0);
    const int zp = min(z + 1, g.rz - 1), zm = max(z - 1, 0);
    float fxp, fxm, fyp, fym, fzp, fzm;
    if (k & 4) {
      fxp = __ldg(f + lin3(g, xp, y, z));
      fxm = xm == e.x0 ? c[k ^ 4] : __ldg(f + lin3(g, xm, y, z));
    } else {
      fxp = c[k ^ 4];  // xp == e.x1
      fxm = __ldg(f + lin3(g, xm, y, z));
    }
    if (k & 2) {
      fyp = __ldg(f + lin3(g, x, yp, z));
      fym = ym == e.y0 ? c[k ^ 2] : __ldg(f + lin3(g, x, ym, z));
    } else {
      fyp = c[k ^ 2];  // yp == e.y1
      fym = __ldg(f + lin3(g, x, ym, z));
    }
    if (k & 1) {
      fzp = __ldg(f + lin3(g, x, y, zp));
      fzm = zm == e.z0 ? c[k ^ 1] : __ldg(f + lin3(g, x, y, zm));
    } else {
      fzp = c[k ^ 1];  // zp == e.z1
      fzm = __ldg(f + lin3(g, x, y, zm));
    }
    const float nx = (fxp - fxm) / fd_den(xp, xm, g.eps[0]);
    const float ny = (fyp - fym) / fd_den(yp, ym, g.eps[1]);
    const float nz = (fzp - fzm) / fd_den(zp, zm, g.eps[2]);
    gx = fmaf(w[k], nx, gx);
    gy = fmaf(w[k], ny, gy);
    gz = fmaf(w[k], nz, gz);
  }
  out[0] = gx;
  out[1] = gy;
  out[2] = gz;
}

__device__ __forceinline__ void eq7_gradient(const float* __restrict__ f, const Grid& g, const Eq7& e,
                                             const float w[8], float out[3]) {
  float c[8];
  eq7_load_block(f, g, e, c);
  eq7_gradient_block(f, g, e, w, c, out);
}

// query_sdf reusing an Eq.7 corner block: when grid_sample's cell is the same cell with all eight
// corners inside the grid (interior points), its corner values are c (same accumulation order);
// otherwise the corners are loaded.
__device__ __forceinline__ float query_sdf_block(const float* __restrict__ f, const Grid& g, float px, float py,
                                                 float pz, const Eq7& e, const float c[8]) {
  Tri t;
  gs_setup(g, px, py, pz, t);
  if (t.inb != 0xffu || t.x0 != e.x0 || t.y0 != e.y0 || t.z0 != e.z0) return gs_sample(f, g, t);
  float acc = 0.0f;
#pragma unroll
  for (int k = 0; k < 8; ++k) acc = fmaf(c[k], t.w[k], acc);
  return acc;
}

__device__ __forceinline__ float norm3(float x, float y, float z) { return sqrtf(x * x + y * y + z * z); }

// normal = g / (|g| + 1e-8)  (gradients.py:136-137)
__device__ __forceinline__ void normalize_eps(const float gr[3], float n[3], float& len) {
  len = norm3(gr[0], gr[1], gr[2]);
  const float d = len + 1e-8f;
  n[0] = gr[0] / d;
  n[1] = gr[1] / d;
  n[2] = gr[2] / d;
}

// Adjoint of normal = g / (|g| + 1e-8): returns dL/dg given dL/dn.
__device__ __forceinline__ void normalize_eps_bwd(const float gr[3], float len, const float dn[3], float dg[3]) {
  const float d = len + 1e-8f;
  dg[0] = dn[0] / d;
  dg[1] = dn[1] / d;
  dg[2] = dn[2] / d;
  if (len > 0.0f) {
    const float dot = gr[0] * dn[0] + gr[1] * dn[1] + gr[2] * dn[2];
    const float c = dot / (d * d * len);
    dg[0] -= c * gr[0];
    dg[1] -= c * gr[1];
    dg[2] -= c * gr[2];
  }
}

// Scatter of dL/dg into the 32-value Eq.7 stencil: grid[c_k +- e_a] += +-w_k dL/dg_a / den.
// Adjoint of eq7_gradient: dL/dg scattered into the Eq.6 differences. Contributions that land on
// the cell's own corners are summed in acc (which may already hold other terms for those corners,
// e.g. the SDF's) and added with one atomic per corner; the 24 outer face neighbours take one each:
// 32 atomics per point instead of 48 (the atomic order is unspecified either way).
__device__ __forceinline__ void eq7_scatter_acc(float* __restrict__ gg, const Grid& g, const Eq7& e,
                                                const float w[8], const float dg[3], float acc[8]) {
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
    if (k & 4) {
      atomicAdd(gg + lin3(g, xp, y, z), vx);
      if (xm == e.x0) acc[k ^ 4] -= vx; else atomicAdd(gg + lin3(g, xm, y, z), -vx);
    } else {
      acc[k ^ 4] += vx;  // xp == e.x1
      atomicAdd(gg + lin3(g, xm, y, z), -vx);
    }
    if (k & 2) {
      atomicAdd(gg + lin3(g, x, yp, z), vy);
      if (ym == e.y0) acc[k ^ 2] -= vy; else atomicAdd(gg + lin3(g, x, ym, z), -vy);
    } else {
      acc[k ^ 2] += vy;  // yp == e.y1
      atomicAdd(gg + lin3(g, x, ym, z), -vy);
    }
    if (k & 1) {
      atomicAdd(gg + lin3(g, x, y, zp), vz);
      if (zm == e.z0) acc[k ^ 1] -= vz; else atomicAdd(gg + lin3(g, x, y, zm), -vz);
    } else {
      acc[k ^ 1] += vz;  // zp == e.z1
      atomicAdd(gg + lin3(g, x, y, zm), -vz);
    }
  }
#pragma unroll
  for (int k = 0; k < 8; ++k)
    if (acc[k] != 0.0f)
      atomicAdd(gg + lin3(g, (k & 4) ? e.x1 : e.x0, (k & 2) ? e.y1 : e.y0, (k & 1) ? e.z1 : e.z0), acc[k]);
}

__device__ __forceinline__ void eq7_scatter(float* __restrict__ gg, const Grid& g, const Eq7& e, const float w[8],
                                            const float dg[3]) {
  float acc[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
  eq7_scatter_acc(gg, g, e, w, dg, acc);
}

// Scatter of dL/dsdf into the grid_sample corners.
__device__ __forceinline__ void gs_scatter(float* __restrict__ gg, const Grid& g, const Tri& t, float ds) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if (t.inb & (1u << k)) {
      const int x = t.x0 + ((k >> 2) & 1), y = t.y0 + ((k >> 1) & 1), z = t.z0 + (k & 1);
      atomicAdd(gg + lin3(g, x, y, z), t.w[k] * ds);
    }
  }
}

// Mark the 8 Eq.7 corners of a sample in a V_R bitmap (bit = linear index), skipping the

// ---------------------------------------------------------------------------------------
// Occupancy mask lookup, OccupancyGrid.is_occupied (rendering/occupancy_grid.py:122-147):
// n = (p - min) / (max - min + 1e-8); occupied iff n in [0, 1] on every axis and
// mask[int(clamp(n * R, 0, R - 1.0001))] is set.
// ---------------------------------------------------------------------------------------
struct Occ {
  const uint8_t* mask;  // (R,R,R) bool, or nullptr for no modulation
  int r;
  float lo[3], den[3], inv_den[3];
};

__device__ __forceinline__ bool occupied(const Occ& oc, float px, float py, float pz) {
  const float p[3] = {px, py, pz};
  int c[3];
  bool inb = true;
  const float hi = (float)((double)oc.r - 1.0001);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float n = div_den(__fsub_rn(p[a], oc.lo[a]), oc.den[a], oc.inv_den[a]);
    inb = inb && (n >= 0.0f) && (n <= 1.0f);
    const float s = fminf(fmaxf(__fmul_rn(n, (float)oc.r), 0.0f), hi);
    c[a] = (int)s;
  }
  return inb && oc.mask[(c[0] * oc.r + c[1]) * oc.r + c[2]] != 0;
}

inline Occ make_occ(const uint8_t* mask, int r, const float lo[3], const float hi[3]) {
  Occ oc;
  oc.mask = mask;
  oc.r = r;
  for (int a = 0; a < 3; ++a) {
    oc.lo[a] = mask ? lo[a] : 0.f;
    oc.den[a] = mask ? (hi[a] - lo[a]) + 1e-8f : 1.f;
    oc.inv_den[a] = pow2_recip(oc.den[a]);
  }
  return oc;
}

// atomic when the bit is already set.
__device__ __forceinline__ void mark_corners(uint32_t* __restrict__ bm, const Grid& g, const Eq7& e) {
#pragma unroll
  for (int k = 0; k < 8; k += 2) {
    const int x = (k & 4) ? e.x1 : e.x0;
    const int y = (k & 2) ? e.y1 : e.y0;
    const int i0 = lin3(g, x, y, e.z0);
    const int i1 = lin3(g, x, y, e.z1);
    const int w0 = i0 >> 5, w1 = i1 >> 5;
    const uint32_t b0 = 1u << (i0 & 31), b1 = 1u << (i1 & 31);
    if (w0 == w1) {
      const uint32_t m = b0 | b1;
      if ((__ldcg(bm + w0) & m) != m) atomicOr(bm + w0, m);
    } else {
      if (!(__ldcg(bm + w0) & b0)) atomicOr(bm + w0, b0);
      if (!(__ldcg(bm + w1) & b1)) atomicOr(bm + w1, b1);
    }
  }
}

__device__ __forceinline__ float sigmoidf_ref(float x) { return 1.0f / (1.0f + expf(-x)); }

// Warp helpers
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Inclusive scans across the 32 lanes
__device__ __forceinline__ float warp_incl_sum(float v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    float t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}
__device__ __forceinline__ float warp_incl_prod(float v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    float t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v *= t;
  }
  return v;
}

__device__ __forceinline__ double warp_incl_sum_d(double v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    double t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}
__device__ __forceinline__ double warp_incl_prod_d(double v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    double t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v *= t;
  }
  return v;
}

}  // namespace vx
