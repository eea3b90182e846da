// Active vertex set V_R (regularization/active_vertices.py:12-50 plus the trainer's
// relax filter, training/trainer.py:262-266) as a bitmap over the grid.
//
// Bit b of word w marks linear voxel index 32 w + b. Corners are marked by the render
// geometry kernel (or from an explicit corner list here); a counting pass evaluates the
// relax predicate |xyz_min + idx*eps| < radius and the optional narrow band |f| < band per
// set bit; compaction walks the words in order, so the list comes out sorted ascending,
// exactly torch.unique's order.
//
// counts[0] = |bits|, counts[1] = |bits & relax|, counts[2] = |bits & band|,
// counts[3] = |bits & relax & band|. The relax filter applies only when counts[1] > 0
// (the reference keeps all vertices when none passes).
#include <mutex>

#include "common.cuh"

namespace vx {

struct VrArgs {
  const uint32_t* bm;
  Grid g;
  const float* f;  // grid values (band predicate)
  float relax_r;   // <= 0: no relax predicate
  float band;      // <= 0: no band predicate; else |f| < band
  int64_t nwords;
  int64_t nvox;
};

__device__ __forceinline__ void vox_xyz(const Grid& g, int idx, int& x, int& y, int& z) {
  z = idx % g.rz;
  const int rem = idx / g.rz;
  y = rem % g.ry;
  x = rem / g.ry;
}

__device__ __forceinline__ bool relax_ok(const VrArgs& a, int x, int y, int z) {
  if (a.relax_r <= 0.0f) return true;
  const float wx = __fadd_rn(a.g.lo[0], __fmul_rn((float)x, a.g.eps[0]));
  const float wy = __fadd_rn(a.g.lo[1], __fmul_rn((float)y, a.g.eps[1]));
  const float wz = __fadd_rn(a.g.lo[2], __fmul_rn((float)z, a.g.eps[2]));
  // |w| with the squares accumulated by fused multiply-adds, x first: the rounding of the
  // reference's float32 torch.linalg.norm on the host for all but a fraction of a percent of
  // vectors (each of which differs by one ulp, deciding membership only within an ulp of the radius)
  const float n = sqrtf(__fmaf_rn(wz, wz, __fmaf_rn(wy, wy, __fmul_rn(wx, wx))));
  return n < a.relax_r;
}

__device__ __forceinline__ bool band_ok(const VrArgs& a, int idx) {
  if (a.band <= 0.0f) return true;
  return fabsf(__ldg(a.f + idx)) < a.band;
}

// membership of voxel idx (bit known set) in the final set for a given relax mode
__device__ __forceinline__ bool in_final(const VrArgs& a, int idx, bool relax_on) {
  int x, y, z;
  vox_xyz(a.g, idx, x, y, z);
  if (relax_on && !relax_ok(a, x, y, z)) return false;
  return band_ok(a, idx);
}

__global__ void k_vr_mark_list(const int64_t* __restrict__ corners, int64_t n, Grid g, uint32_t* __restrict__ bm) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t cx = corners[3 * i], cy = corners[3 * i + 1], cz = corners[3 * i + 2];
    const int x = (int)min(max(cx, (int64_t)0), (int64_t)g.rx - 1);
    const int y = (int)min(max(cy, (int64_t)0), (int64_t)g.ry - 1);
    const int z = (int)min(max(cz, (int64_t)0), (int64_t)g.rz - 1);
    const int idx = lin3(g, x, y, z);
    const uint32_t b = 1u << (idx & 31);
    if (!(__ldcg(bm + (idx >> 5)) & b)) atomicOr(bm + (idx >> 5), b);
  }
}

// Counts, and (when `filtered` is given) the filtered bitmaps: filtered[w] = bits & band,
// filtered[nwords + w] = bits & band & relax.
__global__ void __launch_bounds__(256) k_vr_count(VrArgs a, unsigned long long* __restrict__ counts,
                                                  uint32_t* __restrict__ filtered) {
  unsigned long long c[4] = {0, 0, 0, 0};
  for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < a.nwords; w += (int64_t)gridDim.x * blockDim.x) {
    uint32_t bits = a.bm[w];
    uint32_t f_band = 0, f_both = 0;
    while (bits) {
      const int b = __ffs(bits) - 1;
      bits &= bits - 1;
      const int idx = (int)(w * 32 + b);
      if (idx >= a.nvox) break;
      int x, y, z;
      vox_xyz(a.g, idx, x, y, z);
      const bool r = relax_ok(a, x, y, z);
      const bool bd = band_ok(a, idx);
      c[0] += 1;
      c[1] += r;
      c[2] += bd;
      c[3] += (r && bd);
      f_band |= (bd ? 1u : 0u) << b;
      f_both |= ((r && bd) ? 1u : 0u) << b;
    }
    if (filtered) {
      filtered[w] = f_band;
      filtered[a.nwords + w] = f_both;
    }
  }
  __shared__ unsigned long long sc[4][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    unsigned long long v = c[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sc[k][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    unsigned long long v = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += sc[threadIdx.x][w];
    if (v) atomicAdd(counts + threadIdx.x, v);
  }
}

// The same counts and filtered bitmaps when every word lies inside one z row (Z % 32 == 0) and
// the grid is 16-byte aligned: the 32 voxels of word w share (x, y) and have z = z0..z0+31, so
// their SDF values are one 128-byte line (eight float4 loads, all in flight together) and the
// relax distance needs x^2 + y^2 once; every bit of a nonzero word is evaluated without branches.
__global__ void __launch_bounds__(256) k_vr_count_rows(VrArgs a, unsigned long long* __restrict__ counts,
                                                       uint32_t* __restrict__ filtered) {
  unsigned long long c[4] = {0, 0, 0, 0};
  for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < a.nwords; w += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t bits = a.bm[w];
    uint32_t rmask = 0xffffffffu, bmask = 0xffffffffu;
    if (bits) {
      int x, y, z0;
      vox_xyz(a.g, (int)(w * 32), x, y, z0);
      if (a.relax_r > 0.0f) {
        const float wx = __fadd_rn(a.g.lo[0], __fmul_rn((float)x, a.g.eps[0]));
        const float wy = __fadd_rn(a.g.lo[1], __fmul_rn((float)y, a.g.eps[1]));
        const float xy = __fadd_rn(__fmul_rn(wx, wx), __fmul_rn(wy, wy));
        rmask = 0;
#pragma unroll
        for (int b = 0; b < 32; ++b) {
          const float wz = __fadd_rn(a.g.lo[2], __fmul_rn((float)(z0 + b), a.g.eps[2]));
          rmask |= (sqrtf(__fadd_rn(xy, __fmul_rn(wz, wz))) < a.relax_r ? 1u : 0u) << b;
        }
      }
      if (a.band > 0.0f) {
        const float4* f4 = reinterpret_cast<const float4*>(a.f + w * 32);
        float4 v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = __ldg(f4 + k);
        bmask = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          bmask |= (fabsf(v[k].x) < a.band ? 1u : 0u) << (4 * k);
          bmask |= (fabsf(v[k].y) < a.band ? 1u : 0u) << (4 * k + 1);
          bmask |= (fabsf(v[k].z) < a.band ? 1u : 0u) << (4 * k + 2);
          bmask |= (fabsf(v[k].w) < a.band ? 1u : 0u) << (4 * k + 3);
        }
      }
      c[0] += __popc(bits);
      c[1] += __popc(bits & rmask);
      c[2] += __popc(bits & bmask);
      c[3] += __popc(bits & rmask & bmask);
    }
    if (filtered) {
      filtered[w] = bits & bmask;
      filtered[a.nwords + w] = bits & bmask & rmask;
    }
  }
  __shared__ unsigned long long sc[4][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    unsigned long long v = c[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sc[k][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    unsigned long long v = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += sc[threadIdx.x][w];
    if (v) atomicAdd(counts + threadIdx.x, v);
  }
}

__device__ __forceinline__ bool relax_mode(const unsigned long long* counts, float relax_r) {
  return relax_r > 0.0f && counts[1] > 0;
}

// Per-thread word chunk for compaction: each thread owns kWordsPerThread consecutive words.
constexpr int kWordsPerThread = 4;
constexpr int kCompactThreads = 256;
constexpr int64_t kWordsPerBlock = (int64_t)kWordsPerThread * kCompactThreads;

__device__ __forceinline__ int count_chunk(const VrArgs& a, int64_t w0, bool relax_on) {
  int c = 0;
  for (int k = 0; k < kWordsPerThread; ++k) {
    const int64_t w = w0 + k;
    if (w >= a.nwords) break;
    uint32_t bits = a.bm[w];
    while (bits) {
      const int b = __ffs(bits) - 1;
      bits &= bits - 1;
      const int idx = (int)(w * 32 + b);
      if (idx >= a.nvox) break;
      c += in_final(a, idx, relax_on);
    }
  }
  return c;
}

__device__ __forceinline__ int block_excl_scan(int v, int* tmp, int& total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) tmp[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    int x = (lane < (int)(blockDim.x >> 5)) ? tmp[lane] : 0;
    int xi = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, xi, o);
      if (lane >= o) xi += t;
    }
    if (lane < (int)(blockDim.x >> 5)) tmp[lane] = xi - x;
    if (lane == 31) tmp[32] = xi;
  }
  __syncthreads();
  total = tmp[32];
  const int r = tmp[warp] + inc - v;
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kCompactThreads) k_vr_block_counts(VrArgs a, const unsigned long long* counts,
                                                                      int* __restrict__ block_counts) {
  __shared__ int tmp[33];
  const bool relax_on = relax_mode(counts, a.relax_r);
  const int64_t w0 = blockIdx.x * kWordsPerBlock + (int64_t)threadIdx.x * kWordsPerThread;
  int total;
  block_excl_scan(count_chunk(a, w0, relax_on), tmp, total);
  if (threadIdx.x == 0) block_counts[blockIdx.x] = total;
}

// Single-block exclusive scan of the block counts (in place).
__global__ void __launch_bounds__(1024) k_vr_scan(int* __restrict__ block_counts, int nb) {
  __shared__ int tmp[33];
  int carry = 0;
  for (int base = 0; base < nb; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int v = (i < nb) ? block_counts[i] : 0;
    int total;
    const int ex = block_excl_scan(v, tmp, total);
    if (i < nb) block_counts[i] = carry + ex;
    carry += total;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kCompactThreads) k_vr_write(VrArgs a, const unsigned long long* counts,
                                                               const int* __restrict__ block_offsets,
                                                               int64_t* __restrict__ verts, int64_t* __restrict__ linear,
                                                               int64_t capacity) {
  __shared__ int tmp[33];
  const bool relax_on = relax_mode(counts, a.relax_r);
  const int64_t w0 = blockIdx.x * kWordsPerBlock + (int64_t)threadIdx.x * kWordsPerThread;
  int total;
  int64_t pos = block_offsets[blockIdx.x] + block_excl_scan(count_chunk(a, w0, relax_on), tmp, total);
  for (int k = 0; k < kWordsPerThread; ++k) {
    const int64_t w = w0 + k;
    if (w >= a.nwords) break;
    uint32_t bits = a.bm[w];
    while (bits) {
      const int b = __ffs(bits) - 1;
      bits &= bits - 1;
      const int idx = (int)(w * 32 + b);
      if (idx >= a.nvox) break;
      if (!in_final(a, idx, relax_on)) continue;
      if (pos < capacity) {
        if (linear) linear[pos] = idx;
        if (verts) {
          int x, y, z;
          vox_xyz(a.g, idx, x, y, z);
          verts[3 * pos] = x;
          verts[3 * pos + 1] = y;
          verts[3 * pos + 2] = z;
        }
      }
      ++pos;
    }
  }
}

static int make_vr(VrArgs& a, const uint32_t* bitmap, const float* grid, const int32_t res[3], const float lo[3],
                   const float hi[3], float relax_radius, float band) {
  VX_REQUIRE(res && res[0] >= 1 && res[1] >= 1 && res[2] >= 1, "bad resolution");
  VX_REQUIRE((int64_t)res[0] * res[1] * res[2] < (int64_t(1) << 31), "grid has 2^31 or more voxels");
  VX_REQUIRE(bitmap && lo && hi, "null pointer");
  VX_REQUIRE(band <= 0.0f || grid, "band predicate needs the grid values");
  a.bm = bitmap;
  a.g = make_grid(res, lo, hi);
  a.f = grid;
  a.relax_r = relax_radius;
  a.band = band;
  a.nvox = (int64_t)res[0] * res[1] * res[2];
  a.nwords = (a.nvox + 31) / 32;
  return VX_OK;
}

// Scratch of the allocation-free compaction entry point: per-block offsets in a file-scope
// device array. 4096 entries (16 KiB) cover grids of up to 4096 * 32768 = 2^27 voxels
// (512^3). Every GPU that loads the library holds this array until the process exits.
constexpr int64_t kNoAllocMaxBlocks = 4096;
static __device__ __align__(256) int g_vr_block_offsets[kNoAllocMaxBlocks];

// Device address of g_vr_block_offsets, looked up once per device with that device
// current (a host-side reference to the symbol is not a device address) and kept for the life
// of the process: valid while the device's primary context lives (a cudaDeviceReset would
// reload the module and could move the array).
static int noalloc_offsets(int** out) {
  static std::mutex mu;
  static int* addr[64] = {nullptr};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_error(VX_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return set_error(VX_ERR_INVALID, "device index %d out of range", dev);
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_vr_block_offsets);
    if (e != cudaSuccess) return set_error(VX_ERR_CUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
    addr[dev] = static_cast<int*>(p);
  }
  *out = addr[dev];
  return VX_OK;
}

}  // namespace vx

using namespace vx;

extern "C" {

int vx_vr_compact_noalloc(const uint32_t* bitmap, const float* grid, const int32_t res[3], const float xyz_min[3],
                          const float xyz_max[3], float relax_radius, float band, const unsigned long long* counts,
                          int64_t* verts_out, int64_t* linear_out, int64_t capacity, void* stream) {
  VrArgs a;
  if (int s = make_vr(a, bitmap, grid, res, xyz_min, xyz_max, relax_radius, band)) return s;
  VX_REQUIRE(counts, "counts is null");
  const int64_t nb = (a.nwords + kWordsPerBlock - 1) / kWordsPerBlock;
  VX_REQUIRE(nb <= kNoAllocMaxBlocks,
             "grid of %lld voxels needs %lld compaction blocks; the allocation-free entry point holds %lld "
             "(grids up to 2^27 voxels); use vx_vr_compact with caller scratch",
             (long long)a.nvox, (long long)nb, (long long)kNoAllocMaxBlocks);
  int* offsets = nullptr;
  if (int s = noalloc_offsets(&offsets)) return s;
  // every offset the write pass reads is produced by the count pass of this call: nothing in
  // the array has to start at zero
  cudaStream_t st = (cudaStream_t)stream;
  k_vr_block_counts<<<(unsigned)nb, kCompactThreads, 0, st>>>(a, counts, offsets);
  k_vr_scan<<<1, 1024, 0, st>>>(offsets, (int)nb);
  k_vr_write<<<(unsigned)nb, kCompactThreads, 0, st>>>(a, counts, offsets, verts_out, linear_out, capacity);
  count_launches(3);
  return check_launch("vr_compact_noalloc");
}

int64_t vx_vr_bitmap_words(const int32_t res[3]) {
  return ((int64_t)res[0] * res[1] * res[2] + 31) / 32;
}

int64_t vx_vr_compact_blocks(const int32_t res[3]) {
  return (vx_vr_bitmap_words(res) + kWordsPerBlock - 1) / kWordsPerBlock;
}

int vx_vr_mark_corners(const int64_t* corners, int64_t n_corners, const int32_t res[3], uint32_t* bitmap,
                       void* stream) {
  VX_REQUIRE(res && res[0] >= 1 && res[1] >= 1 && res[2] >= 1, "bad resolution");
  VX_REQUIRE((int64_t)res[0] * res[1] * res[2] < (int64_t(1) << 31), "grid has 2^31 or more voxels");
  VX_REQUIRE(n_corners >= 0, "n < 0");
  if (n_corners == 0) return VX_OK;
  VX_REQUIRE(corners && bitmap, "null pointer");
  const float lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
  Grid g = make_grid(res, lo, hi);
  k_vr_mark_list<<<grid_for(n_corners, 256), 256, 0, (cudaStream_t)stream>>>(corners, n_corners, g, bitmap);
  count_launches(1);
  return check_launch("vr_mark_corners");
}

int vx_vr_count(const uint32_t* bitmap, const float* grid, const int32_t res[3], const float xyz_min[3],
                const float xyz_max[3], float relax_radius, float band, unsigned long long* counts,
                uint32_t* filtered, void* stream) {
  VrArgs a;
  if (int s = make_vr(a, bitmap, grid, res, xyz_min, xyz_max, relax_radius, band)) return s;
  VX_REQUIRE(counts, "counts is null");
  if (a.g.rz % 32 == 0 && (a.band <= 0.0f || ((uintptr_t)grid & 15) == 0))
    k_vr_count_rows<<<grid_for(a.nwords, 256, 8), 256, 0, (cudaStream_t)stream>>>(a, counts, filtered);
  else
    k_vr_count<<<grid_for(a.nwords, 256, 8), 256, 0, (cudaStream_t)stream>>>(a, counts, filtered);
  count_launches(1);
  return check_launch("vr_count");
}

int vx_vr_compact(const uint32_t* bitmap, const float* grid, const int32_t res[3], const float xyz_min[3],
                  const float xyz_max[3], float relax_radius, float band, const unsigned long long* counts,
                  int* block_scratch, int64_t n_block_scratch, int64_t* verts_out, int64_t* linear_out,
                  int64_t capacity, void* stream) {
  VrArgs a;
  if (int s = make_vr(a, bitmap, grid, res, xyz_min, xyz_max, relax_radius, band)) return s;
  VX_REQUIRE(counts && block_scratch, "null pointer");
  const int64_t nb = (a.nwords + kWordsPerBlock - 1) / kWordsPerBlock;
  VX_REQUIRE(n_block_scratch >= nb, "block scratch holds %lld entries, need %lld", (long long)n_block_scratch,
             (long long)nb);
  VX_REQUIRE(nb < (int64_t(1) << 31), "grid too large");
  cudaStream_t st = (cudaStream_t)stream;
  k_vr_block_counts<<<(unsigned)nb, kCompactThreads, 0, st>>>(a, counts, block_scratch);
  k_vr_scan<<<1, 1024, 0, st>>>(block_scratch, (int)nb);
  k_vr_write<<<(unsigned)nb, kCompactThreads, 0, st>>>(a, counts, block_scratch, verts_out, linear_out, capacity);
  count_launches(3);
  return check_launch("vr_compact");
}

}  // extern "C"
