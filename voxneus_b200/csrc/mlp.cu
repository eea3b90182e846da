// Radiance MLP [hash 32 | SH 16 | normal 3] -> 64 ReLU -> 3 Sigmoid (models/radiance_mlp.py:42-53,
// 81-98) on the 5th-generation tensor cores (tcgen05, kind::tf32, accumulators in TMEM).
//
// Accuracy: every product runs as a 3-term split x = hi + lo (hi, lo tf32), a*b ~ ah*bh + ah*bl +
// al*bh, accumulated in f32 — about 21 bits per product, the FP32 parity bar (colours 1e-5, weight
// gradients 1e-4 of their scale) holds where a single tf32 pass (11 bits) would not.
//
// Operands are K-major canonical no-swizzle layouts (tc.cuh; kind::tf32 with an MN-major operand
// writes nothing on this part, so every operand is staged with its contraction dimension
// contiguous). A 16-byte chunk holds 4 consecutive K elements of one row:
//   X    (128 sample rows, K = features): chunk (m, 4f..4f+3) at (f*16 + m/8)*128 + (m%8)*16
//   W0   [hi; lo] (128 rows: hidden unit n's hi part in row n, its lo part in row 64 + n, K =
//        features): element (r, k) at ((k/4)*16 + r/8)*128 + (r%8)*16 + (k%4)*4
//   W0^T [hi; lo] (128 feature rows, K = hidden), DZ (128 sample rows, K = hidden), and X^T [hi; lo]
//   / DZ^T [hi; lo] (128 rows, K = the tile's samples) likewise.
// The stacked hi/lo operands let one N = 128 MMA form two of the three products:
//   Z   = X W0^T   A = X_hi, B = [W_hi; W_lo] (N = 128) + A = X_lo, B = W_hi (N = 64), K = 56 in 7
//                  steps; Z = columns [0, 64) + [64, 128)
//   dX  = DZ W0    the same with A = DZ_hi / DZ_lo, B = W0^T [hi; lo], K = 64 in 8 steps
//   dW0 = [DZh;DZl]^T X   A = DZ^T [hi; lo], B = X^T [hi; lo] (N = 128), K = 128 samples in 16 steps
// The forward writes the colours (and, for the adjoint, the input rows: 52 floats, or the compact
// 36-float rows of the fused appearance path); the adjoint recomputes Z with the identical MMA
// sequence, writes dL/d(hash) and dL/d(normal), accumulates dW0 (and db0 through a ones column) in
// TMEM across its tiles and dW1 in TMEM / db1 in registers, and writes per-block partials that
// k_mlp_wgrad_reduce sums in a fixed order (deterministic). The folded variant (compact rows whose
// tiles each lie inside one ray) contracts K = 40 features [hash | normal | one] in 5 steps, with
// SH(d) as a per-ray bias of the hidden layer and the SH columns of dW0 taken from each tile's
// column sum of dL/dz.
#include "hashgrid.cuh"
#include "tc.cuh"

namespace vx {

constexpr int KIN = 51;  // input features
constexpr int KP = 52;   // row width of the input rows (column 51 is padding)
// Compact rows of the fused appearance path: [hash 32 | normal 3 | pad], 144 bytes. The 16 SH(d)
// features (columns 32..47 of a full row) depend on the ray only. When a ray's samples fill whole
// 128-row tiles the folded MLP (fold_col, fold_bias below) adds them as a per-ray hidden bias;
// otherwise the MLP kernels rebuild them from the ray's direction while they stage a tile, the same
// function on the same operands as the row writer, so that both layouts give the same bits.
constexpr int KC = 36;
constexpr int NH = 64;   // hidden units
constexpr int NO = 3;    // colours
constexpr int TM = 128;  // samples per tile (TMEM lanes)
constexpr int WG = NH * KP + NO * NH + NH + NO;  // per-block weight-gradient partial size
constexpr uint32_t kWaitLimit = 1u << 22;       // default mbarrier polls before a tile gives up
// After a block gives up on a wait, the copy or MMA it waited for may still be running: the
// block waits for it (at most this many polls) before it frees tensor memory and exits, so no
// asynchronous write lands in memory that another block owns next.
constexpr uint32_t kDrainLimit = 1u << 22;

constexpr uint32_t kXBytes = 16 * 16 * 128;  // one tf32 part of X (or DZ)
constexpr uint32_t kWBytes = 16 * 16 * 128;  // W0 (or W0^T) as [hi; lo]

__device__ int g_tc_timeouts = 0;

// The wait policy of the MMA kernels: polls per mbarrier wait, and a caller's device status word
// (nullable) that every block which gave up increments.
struct TcGuard {
  int* status;
  uint32_t limit;
};

// The guard the host launchers of this thread pass (vx_tc_guard).
thread_local TcGuard t_guard{nullptr, kWaitLimit};

// Whether this thread's launches take the caller's poll limit (a kernel variant that reads it) or
// the default (a compile-time bound, which keeps the waits' loops as tight as before).
inline bool custom_wait() { return t_guard.limit != kWaitLimit; }

__device__ __forceinline__ void report_timeout(int* status) {
  atomicAdd(&g_tc_timeouts, 1);
  if (status) atomicAdd(status, 1);
}

// Where a kernel's full rows come from: rays_d == nullptr, rows of KP floats; otherwise compact
// rows of KC floats whose SH features are recomputed from rays_d of the sample's ray (i / S; the
// entry points keep the sample count below 2^32).
struct RowSrc {
  const float* rays_d;
  int64_t S;
};

// Feature chunk c = (hh ? 7 : 0) + j (0..12, four features each) of a staged sample: chunks 0..7
// the hash features, 8..11 SH(d), 12 the normal and the pad column. j is a constant of the
// unrolled staging loop, so each SH group is built only where it is stored.
template <bool kCompact>
__device__ __forceinline__ float4 x_chunk(const float4* rrow, bool hh, int j, float3 dir) {
  if (kCompact && hh) {
    if (j == 0) return rrow[7];
    if (j <= 4) return sh_chunk(dir.x, dir.y, dir.z, j - 1);
    return rrow[8];
  }
  return rrow[(hh ? 7 : 0) + j];
}

// The ray direction of sample i, for the thread that stages the sample's chunks 7..12.
template <bool kCompact>
__device__ __forceinline__ float3 stage_dir(const RowSrc& src, int64_t i, bool need) {
  float3 d = make_float3(0.0f, 0.0f, 0.0f);
  if (kCompact && need) {
    const uint32_t r = (uint32_t)i / (uint32_t)src.S;
    d = make_float3(__ldg(src.rays_d + 3 * (size_t)r), __ldg(src.rays_d + 3 * (size_t)r + 1),
                    __ldg(src.rays_d + 3 * (size_t)r + 2));
  }
  return d;
}

struct MlpW {
  const float* W0;  // (64, 51)
  const float* b0;  // (64)
  const float* W1;  // (3, 64)
  const float* b1;  // (3)
};

// The folded MLP (compact rows whose 128-row tiles each lie inside one ray, so SH(d) is constant
// over a tile): the 16 SH columns leave the contraction and become a per-ray bias of the hidden
// layer, b0 + W0[:, 32:48] SH(d). Its input features are [hash 32 | normal 3 | one | 0 x 4], K = 40.
// Folded feature k comes from column fold_col(k) of W0 (-1: none).
__device__ __forceinline__ int fold_col(int k) { return k < 32 ? k : (k < 35 ? 48 + (k - 32) : -1); }

// The per-ray bias of hidden unit n: b0[n] + sum_k W0[n, 32 + k] sh[k], k = 0..15 in order (the
// forward and the adjoint evaluate it identically, so the adjoint's recomputed hidden layer has
// the forward's bits).
__device__ __forceinline__ float fold_bias(const MlpW& w, int n, const float sh[16]) {
  float b = __ldg(w.b0 + n);
#pragma unroll
  for (int k = 0; k < 16; ++k) b = fmaf(__ldg(w.W0 + n * KIN + 32 + k), sh[k], b);
  return b;
}

// SH(d) of ray r.
__device__ __forceinline__ void ray_sh(const float* __restrict__ rays_d, int64_t r, float sh[16]) {
  sh16(__ldg(rays_d + 3 * r), __ldg(rays_d + 3 * r + 1), __ldg(rays_d + 3 * r + 2), sh);
}

__device__ __forceinline__ uint32_t x_off(int f, int m) { return (uint32_t)((f * 16 + (m >> 3)) * 128 + (m & 7) * 16); }
// row r of [W_hi; W_lo] (r < 64: hi of hidden unit r, else lo of hidden unit r - 64), feature k
__device__ __forceinline__ uint32_t w_off(int r, int k) {
  return (uint32_t)(((k >> 2) * 16 + (r >> 3)) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

__device__ __forceinline__ void st_split4(uint8_t* hi, uint8_t* lo, uint32_t off, float a, float b, float c, float d) {
  float4 h, l;
  tc::split_tf32(a, h.x, l.x);
  tc::split_tf32(b, h.y, l.y);
  tc::split_tf32(c, h.z, l.z);
  tc::split_tf32(d, h.w, l.w);
  *reinterpret_cast<float4*>(hi + off) = h;
  *reinterpret_cast<float4*>(lo + off) = l;
}

// W0 as [hi; lo] tf32 (features 51..63 zero), b0, W1, b1; X feature chunks 13..15 (columns 52..63,
// never written by the tiles) zeroed.
__device__ void stage_weights(const MlpW& w, uint8_t* W2, uint8_t* XH, uint8_t* XL, float* B0, float* W1s, float* B1,
                              int tid, int nt) {
  for (int e = tid; e < NH * 64; e += nt) {
    const int n = e >> 6, k = e & 63;
    float h, l;
    tc::split_tf32(k < KIN ? w.W0[n * KIN + k] : 0.0f, h, l);
    *reinterpret_cast<float*>(W2 + w_off(n, k)) = h;
    *reinterpret_cast<float*>(W2 + w_off(NH + n, k)) = l;
  }
  for (int e = tid; e < 3 * TM; e += nt) {
    const uint32_t off = x_off(13 + e / TM, e % TM);
    *reinterpret_cast<float4*>(XH + off) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    *reinterpret_cast<float4*>(XL + off) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
  for (int i = tid; i < NH; i += nt) B0[i] = w.b0[i];
  for (int i = tid; i < NO * NH; i += nt) W1s[i] = w.W1[i];
  if (tid < NO) B1[tid] = w.b1[tid];
}

// Row chunks of sample m of the tile at m0 into registers: thread (m, hh) takes the 16-byte
// chunks 0..6 (hh = 0) or 7..12 (hh = 1, v[6] unused). Rows past P read as 0.
__device__ __forceinline__ void load_row_chunks(const float* __restrict__ X, int64_t ldx, bool vec, int64_t P,
                                                int64_t m0, int m, int hh, float4 v[7]) {
  const bool ok = m0 + m < P;
  const float* row = X + (m0 + m) * ldx;
  const int c0 = hh ? 7 : 0;
#pragma unroll
  for (int j = 0; j < 7; ++j) {
    const int c = c0 + j;
    v[j] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (ok && c < 13) {
      if (vec) {
        v[j] = __ldg(reinterpret_cast<const float4*>(row) + c);
      } else {
        v[j].x = __ldg(row + 4 * c);
        v[j].y = __ldg(row + 4 * c + 1);
        v[j].z = __ldg(row + 4 * c + 2);
        v[j].w = 4 * c + 3 < KIN ? __ldg(row + 4 * c + 3) : 0.0f;
      }
    }
  }
}

// The chunks of load_row_chunks into the X buffers (hi/lo tf32); column 51 becomes `one` on
// real rows.
__device__ __forceinline__ void store_row_chunks(const float4 v[7], bool valid, uint8_t* XH, uint8_t* XL, int m,
                                                 int hh, float one) {
  const int c0 = hh ? 7 : 0;
#pragma unroll
  for (int j = 0; j < 7; ++j) {
    const int c = c0 + j;
    if (c < 13) {
      float4 u = v[j];
      if (c == 12 && valid) u.w = one;
      st_split4(XH, XL, x_off(c, m), u.x, u.y, u.z, u.w);
    }
  }
}

constexpr uint32_t kId128 = tc::idesc_tf32(TM, 2 * NH, false, false);
constexpr uint32_t kId64 = tc::idesc_tf32(TM, NH, false, false);

// A [hi | lo] K-major operand times a stacked [hi; lo] B: columns [t, t + 64) receive
// A_hi B_hi + A_lo B_hi and [t + 64, t + 128) receive A_hi B_lo (one N = 128 and one N = 64 MMA per
// 8-wide K step; the result is the sum of the two column halves). Issued by one thread.
__device__ __forceinline__ void issue_split(uint32_t t, uint32_t ah0, uint32_t al0, uint32_t b0, int ksteps) {
#pragma unroll 1
  for (int ks = 0; ks < ksteps; ++ks) {
    const uint64_t ah = tc::sdesc(ah0 + ks * 4096, 2048, 128), al = tc::sdesc(al0 + ks * 4096, 2048, 128);
    const uint64_t b = tc::sdesc(b0 + ks * 4096, 2048, 128);
    tc::mma_tf32(t, ah, b, kId128, ks > 0);
    tc::mma_tf32(t, al, b, kId64, true);
  }
}

// issue_split with the A hi part in tensor memory: A_hi's K elements in columns ah_tmem + 8*ks of the
// sample lanes (the same products in the same order as issue_split).
__device__ __forceinline__ void issue_split_ts(uint32_t t, uint32_t ah_tmem, uint32_t al0, uint32_t b0, int ksteps) {
#pragma unroll 1
  for (int ks = 0; ks < ksteps; ++ks) {
    const uint64_t al = tc::sdesc(al0 + ks * 4096, 2048, 128);
    const uint64_t b = tc::sdesc(b0 + ks * 4096, 2048, 128);
    tc::mma_tf32_ts(t, ah_tmem + 8 * ks, b, kId128, ks > 0);
    tc::mma_tf32(t, al, b, kId64, true);
  }
}

// Z = X W0^T into TMEM columns [tz, tz + 128) as two halves to add (same sequence in both passes).
__device__ __forceinline__ void issue_z(uint32_t tz, uint32_t xh, uint32_t xl, uint32_t w2) {
  issue_split(tz, xh, xl, w2, 7);
}

// 32 columns of a split result: TMEM columns [col, col + 32) + [col + 64, col + 96) of this warp's lanes
__device__ __forceinline__ void tmem_ld_sum32(uint32_t taddr, float v[32]) {
  float u[32];
  tc::tmem_ld32(taddr, v);
  tc::tmem_ld32(taddr + 64, u);
  tc::tmem_wait_ld();
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] += u[j];
}

// This thread's half of the colour pre-activation: hidden units 32*hh..32*hh+31 of sample lane.
__device__ __forceinline__ void colour_partial(const float z[32], int hh, const float* B0, const float* W1s,
                                               float& p0, float& p1, float& p2) {
  p0 = p1 = p2 = 0.0f;
#pragma unroll
  for (int j4 = 0; j4 < 8; ++j4) {
    const int n = 32 * hh + 4 * j4;
    const float4 b = *reinterpret_cast<const float4*>(B0 + n);
    const float4 u0 = *reinterpret_cast<const float4*>(W1s + n);
    const float4 u1 = *reinterpret_cast<const float4*>(W1s + NH + n);
    const float4 u2 = *reinterpret_cast<const float4*>(W1s + 2 * NH + n);
    const float bb[4] = {b.x, b.y, b.z, b.w}, w0[4] = {u0.x, u0.y, u0.z, u0.w};
    const float w1[4] = {u1.x, u1.y, u1.z, u1.w}, w2[4] = {u2.x, u2.y, u2.z, u2.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const float h = fmaxf(z[4 * j4 + i] + bb[i], 0.0f);
      p0 = fmaf(w0[i], h, p0);
      p1 = fmaf(w1[i], h, p1);
      p2 = fmaf(w2[i], h, p2);
    }
  }
}

// Forward. kHashIn: the 51 features of a tile are built in place (two threads per sample, 8 hash
// levels each; SH of the view direction; the normal); else they are read from rows X. kRowsOut
// also writes the rows for the adjoint. 256 threads: warp w reads TMEM lanes 32*(w%4).. and
// hidden columns 32*(w/4)..; the two column halves meet in shared memory.
template <bool kHashIn, bool kRowsOut, bool kCustomWait>
__global__ void __launch_bounds__(256, 2) k_mlp_fwd_tc(HashArgs a, const float* __restrict__ X, int64_t ldx, int xvec,
                                                       int64_t P, MlpW w, float* __restrict__ colors,
                                                       TcGuard g) {
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t wait_limit = kCustomWait ? g.limit : kWaitLimit;  // a constant bound unless a caller set one
  uint8_t* XH = smem;
  uint8_t* XL = XH + kXBytes;
  uint8_t* W2 = XL + kXBytes;
  float* B0 = reinterpret_cast<float*>(W2 + kWBytes);
  float* W1s = B0 + NH;
  float* B1 = W1s + NO * NH;
  float* RED = B1 + 4;  // [2][TM][4]
  uint64_t* bar = reinterpret_cast<uint64_t*>(RED + 2 * TM * 4);
  uint32_t* s_taddr = reinterpret_cast<uint32_t*>(bar + 1);
  const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31, q = wid & 3, hh = wid >> 2;
  stage_weights(w, W2, XH, XL, B0, W1s, B1, tid, blockDim.x);
  if (tid == 0) tc::mbar_init(bar, 1);
  if (wid == 0) tc::tmem_alloc(s_taddr, 128);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *s_taddr;
  const uint32_t xh = tc::smem_u32(XH), xl = tc::smem_u32(XL), w2 = tc::smem_u32(W2);
  const uint32_t mask = (1u << a.log2T) - 1u;
  const size_t T = (size_t)1 << a.log2T;
  uint32_t phase = 0;
  const int64_t ntiles = (P + TM - 1) / TM;
  float4 pre[7];
  if (!kHashIn && (int64_t)blockIdx.x < ntiles)
    load_row_chunks(X, ldx, xvec != 0, P, (int64_t)blockIdx.x * TM, tid & (TM - 1), tid >> 7, pre);
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t m0 = t * TM;
    if (kHashIn) {
      const int m = tid & (TM - 1), half = tid >> 7;
      const int64_t i = m0 + m;
      float feat[16], extra[16];
      if (i < P) {
        float x[3];
        sample_pos(a, i, x);
#pragma unroll
        for (int qq = 0; qq < 8; ++qq) {
          const int l = 8 * half + qq;
          const float lw = a.lw[l];
          float f0 = 0.0f, f1 = 0.0f;
          if (lw != 0.0f) {
            LevelCell c;
            level_cell(x, a.res[l], mask, c);
            const float2* tab = reinterpret_cast<const float2*>(a.table) + (size_t)l * T;
            gather_level(tab, c, f0, f1);
            if (lw < 1.0f) {
              f0 *= lw;
              f1 *= lw;
            }
          }
          feat[2 * qq] = f0;
          feat[2 * qq + 1] = f1;
        }
        if (half == 0) {
          const int64_t r = i / a.S;
          sh16(__ldg(a.rays_d + 3 * r), __ldg(a.rays_d + 3 * r + 1), __ldg(a.rays_d + 3 * r + 2), extra);
        } else {
          extra[0] = a.normals[3 * i];
          extra[1] = a.normals[3 * i + 1];
          extra[2] = a.normals[3 * i + 2];
          extra[3] = 0.0f;
        }
      } else {
#pragma unroll
        for (int qq = 0; qq < 16; ++qq) feat[qq] = extra[qq] = 0.0f;
      }
#pragma unroll
      for (int c = 0; c < 4; ++c)
        st_split4(XH, XL, x_off(4 * half + c, m), feat[4 * c], feat[4 * c + 1], feat[4 * c + 2], feat[4 * c + 3]);
      if (half == 0) {
#pragma unroll
        for (int c = 0; c < 4; ++c)
          st_split4(XH, XL, x_off(8 + c, m), extra[4 * c], extra[4 * c + 1], extra[4 * c + 2], extra[4 * c + 3]);
      } else {
        st_split4(XH, XL, x_off(12, m), extra[0], extra[1], extra[2], extra[3]);
      }
      if (kRowsOut && i < P) {
        float4* row = reinterpret_cast<float4*>(a.out + i * a.ld);
#pragma unroll
        for (int c = 0; c < 4; ++c)
          row[4 * half + c] = make_float4(feat[4 * c], feat[4 * c + 1], feat[4 * c + 2], feat[4 * c + 3]);
        if (half == 0) {
#pragma unroll
          for (int c = 0; c < 4; ++c)
            row[8 + c] = make_float4(extra[4 * c], extra[4 * c + 1], extra[4 * c + 2], extra[4 * c + 3]);
        } else {
          row[12] = make_float4(extra[0], extra[1], extra[2], extra[3]);
        }
      }
    } else {
      store_row_chunks(pre, m0 + (tid & (TM - 1)) < P, XH, XL, tid & (TM - 1), tid >> 7, 0.0f);
    }
    tc::fence_smem_to_async();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      issue_z(tbase, xh, xl, w2);
      tc::commit(bar);
    }
    if (!kHashIn && t + gridDim.x < ntiles)  // next tile's rows fly during the MMA and the epilogue
      load_row_chunks(X, ldx, xvec != 0, P, (t + gridDim.x) * TM, tid & (TM - 1), tid >> 7, pre);
    const bool ok = tc::mbar_wait(bar, phase, wait_limit);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
      if (tid == 0) {
        if (!ok) tc::mbar_wait(bar, phase ^ 1u, kDrainLimit);  // this tile's Z MMA, before TMEM is freed
        report_timeout(g.status);
      }
      break;
    }
    tc::fence_after_sync();
    float z[32];
    tmem_ld_sum32(tbase + ((uint32_t)(32 * q) << 16) + 32 * hh, z);
    float p0, p1, p2;
    colour_partial(z, hh, B0, W1s, p0, p1, p2);
    float* r = RED + (hh * TM + 32 * q + lane) * 4;
    r[0] = p0;
    r[1] = p1;
    r[2] = p2;
    tc::fence_before_sync();
    __syncthreads();
    if (tid < TM && m0 + tid < P) {
#pragma unroll
      for (int c = 0; c < NO; ++c) {
        const float o = (B1[c] + RED[tid * 4 + c]) + RED[(TM + tid) * 4 + c];
        colors[(m0 + tid) * NO + c] = sigmoidf_ref(o);
      }
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (wid == 0) tc::tmem_dealloc(tbase, 128);
}

constexpr size_t kFwdSmem = 2 * kXBytes + kWBytes + sizeof(float) * (NH + NO * NH + 4 + 2 * TM * 4) + 16;

// Forward on contiguous 52-float rows (ldx = 52, 16-byte aligned): one CTA of 512 threads per SM
// holding two independent tile slots of 256 threads (slot s = threads 256 s ..), which share the
// stacked weights and alternate on the tensor core. Each slot has its own X operand (the lo part in
// shared memory, the hi part in TMEM columns 256 + 64 s, sample lanes, written with tcgen05.st),
// its own 128 accumulator columns, and a row buffer that the next tile's rows reach by one bulk
// copy, issued as soon as the slot has staged its current tile; a slot synchronises on its own
// named barrier, so one slot's MMA wait overlaps the other's staging and epilogue. Row prefetch
// through registers (the general kernel above) left every warp stalled on its 16-byte loads of 32
// rows at a time.
constexpr uint32_t kFwdSlotBytes = kXBytes + TM * KP * 4 + 2 * TM * 4 * 4;  // XL, rows, RED
// shared head: W0 [hi; lo], b0, W1, b1, barriers, TMEM address, fail flags; slots from a 1 KB boundary
constexpr size_t kFwd2Head =
    1024 * ((kWBytes + sizeof(float) * (NH + NO * NH + 4) + 64 + 2 * NH * sizeof(float) + 1023) / 1024);
// the folded MLP's per-ray hidden bias of each slot's tile: the last 2 x 64 floats of the head
constexpr size_t kFwd2Beta = kFwd2Head - 2 * NH * sizeof(float);
static_assert(kFwd2Beta >= kWBytes + sizeof(float) * (NH + NO * NH + 4) + 64, "forward head overlaps its bias");
constexpr size_t kFwd2Smem = kFwd2Head + 2 * (size_t)kFwdSlotBytes;
// one CTA per SM (it allocates all 512 TMEM columns): two would need <= 116 KB each
static_assert(kFwd2Smem > 116 * 1024, "two forward CTAs would fit on an SM and contend for TMEM");

__device__ __forceinline__ void slot_sync(int slot) {
  asm volatile("bar.sync %0, 256;" ::"r"(1 + slot) : "memory");
}

template <bool kCustomWait, bool kCompact, bool kFold>
__global__ void __launch_bounds__(512, 1) k_mlp_fwd_rows2(const float* __restrict__ X, int64_t P, MlpW w,
                                                         float* __restrict__ colors, TcGuard g, RowSrc src) {
  static_assert(!kFold || kCompact, "the folded MLP reads compact rows");
  constexpr int kLd = kCompact ? KC : KP;  // floats per row in global memory
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t wait_limit = kCustomWait ? g.limit : kWaitLimit;
  uint8_t* W2 = smem;
  float* B0 = reinterpret_cast<float*>(W2 + kWBytes);
  float* W1s = B0 + NH;
  float* B1 = W1s + NO * NH;
  uint64_t* bars = reinterpret_cast<uint64_t*>(B1 + 4);  // [slot][mma, rows]
  uint32_t* s_taddr = reinterpret_cast<uint32_t*>(bars + 4);
  int* s_fail = reinterpret_cast<int*>(s_taddr + 1);  // [2]
  const int tid = threadIdx.x, slot = tid >> 8, stid = tid & 255;
  const int wid = stid >> 5, lane = tid & 31, q = wid & 3, hh = wid >> 2;
  const int m = 32 * q + lane;  // this thread's sample in its slot's tile
  uint8_t* SL = smem + kFwd2Head + (size_t)slot * kFwdSlotBytes;
  float* BETA = reinterpret_cast<float*>(smem + kFwd2Beta) + NH * slot;  // kFold: this slot's tile's bias
  uint8_t* XL = SL;
  uint8_t* ROWS = XL + kXBytes;
  float* RED = reinterpret_cast<float*>(ROWS + TM * KP * 4);  // [2][TM][4]
  uint64_t* bar = bars + 2 * slot;
  uint64_t* bar_rows = bar + 1;
  // weights and each slot's X_lo feature chunks 13..15 (zero), by all 512 threads
  for (int e = tid; e < NH * 64; e += blockDim.x) {
    const int n = e >> 6, k = e & 63;
    const int col = kFold ? fold_col(k) : (k < KIN ? k : -1);
    float h, l;
    tc::split_tf32(col >= 0 ? w.W0[n * KIN + col] : 0.0f, h, l);
    *reinterpret_cast<float*>(W2 + w_off(n, k)) = h;
    *reinterpret_cast<float*>(W2 + w_off(NH + n, k)) = l;
  }
  for (int e = stid; e < 3 * TM; e += 256)
    *reinterpret_cast<float4*>(XL + x_off(13 + e / TM, e % TM)) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  for (int i = tid; i < NH; i += blockDim.x) B0[i] = w.b0[i];
  for (int i = tid; i < NO * NH; i += blockDim.x) W1s[i] = w.W1[i];
  if (tid < NO) B1[tid] = w.b1[tid];
  if (stid == 0) {
    tc::mbar_init(bar, 1);
    tc::mbar_init(bar_rows, 1);
    s_fail[slot] = 0;
  }
  if (tid < 32) tc::tmem_alloc(s_taddr, 512);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tcol = *s_taddr + 128 * slot;       // Z accumulator (two halves)
  const uint32_t acol = *s_taddr + 256 + 64 * slot;  // X_hi: feature f in column acol + f
  const uint32_t lane_base = (uint32_t)(32 * q) << 16;
  const uint32_t xl = tc::smem_u32(XL), w2 = tc::smem_u32(W2);
  const int64_t ntiles = (P + TM - 1) / TM;
  const int64_t t0 = 2 * (int64_t)blockIdx.x + slot, tstride = 2 * (int64_t)gridDim.x;
  auto fetch_rows = [&](int64_t t) {
    const int64_t m0 = t * TM;
    const uint32_t bytes = (uint32_t)(P - m0 < TM ? P - m0 : TM) * (uint32_t)(kLd * 4);
    tc::mbar_arrive_expect_tx(bar_rows, bytes);
    tc::bulk_g2s(ROWS, X + m0 * kLd, bytes, bar_rows);
  };
  // slot thread 0's bookkeeping for a give-up: a rows copy in flight and the mbarrier parity it
  // completes, and whether its own wait on the slot's MMA gave up
  bool rows_pending = false, mma_pending = false;
  uint32_t rows_parity = 0;
  if (stid == 0 && t0 < ntiles) {
    fetch_rows(t0);
    rows_pending = true;
  }
  uint32_t phase = 0, rphase = 0;
  float dnx = 0.0f, dny = 0.0f, dnz = 0.0f;  // kFold, threads 0..63: this tile's ray direction
  if (kFold && stid < NH && t0 < ntiles) {
    const int64_t r = t0 * TM / src.S;
    dnx = __ldg(src.rays_d + 3 * r);
    dny = __ldg(src.rays_d + 3 * r + 1);
    dnz = __ldg(src.rays_d + 3 * r + 2);
  }
  for (int64_t t = t0; t < ntiles; t += tstride) {
    const int64_t m0 = t * TM;
    const bool valid = m0 + m < P;
    const bool got = tc::mbar_wait(bar_rows, rphase, wait_limit);
    rphase ^= 1u;
    if (!got) s_fail[slot] = 1;
    slot_sync(slot);
    if (s_fail[slot]) break;
    if (stid == 0) rows_pending = false;
    if constexpr (kFold) {  // rows -> X_hi / X_lo: [hash 32 | normal 3 | 0 | 0 x 4]
      const float4* rrow = reinterpret_cast<const float4*>(ROWS + m * (kLd * 4));
      const int c0 = hh ? 5 : 0;
      float xh[20];  // features 4*c0 .. 4*c0 + 19
#pragma unroll
      for (int j = 0; j < 5; ++j) {
        const int c = c0 + j;
        float4 u = (valid && c < 9) ? rrow[c] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (c == 8) u.w = 0.0f;
        const float v[4] = {u.x, u.y, u.z, u.w};
        float lo[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) tc::split_tf32(v[i], xh[4 * j + i], lo[i]);
        *reinterpret_cast<float4*>(XL + x_off(c, m)) = make_float4(lo[0], lo[1], lo[2], lo[3]);
      }
      const uint32_t ta = acol + lane_base + 4 * c0;  // stores aligned to their widths
      if (hh == 0) {
        tc::tmem_st16(ta, xh);
        tc::tmem_st4(ta + 16, xh + 16);
      } else {
        tc::tmem_st4(ta, xh);
        tc::tmem_st8(ta + 4, xh + 4);
        tc::tmem_st8(ta + 12, xh + 12);
      }
      tc::tmem_wait_st();
    } else {  // rows -> X_hi (TMEM) and X_lo (sample rows); column 51 zero (the padding column may hold anything)
      const float4* rrow = reinterpret_cast<const float4*>(ROWS + m * (kLd * 4));
      const int c0 = hh ? 7 : 0;
      const float3 dir = stage_dir<kCompact>(src, m0 + m, valid && hh);
      float xh[28];  // features 4*c0 .. 4*c0 + 27 (hh = 1: 28..55, with 52..55 the zero chunk 13)
#pragma unroll
      for (int j = 0; j < 7; ++j) {
        const int c = c0 + j;
        if (c < 13) {
          float4 u = valid ? x_chunk<kCompact>(rrow, hh, j, dir) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          if (c == 12) u.w = 0.0f;
          const float v[4] = {u.x, u.y, u.z, u.w};
          float lo[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) tc::split_tf32(v[i], xh[4 * j + i], lo[i]);
          *reinterpret_cast<float4*>(XL + x_off(c, m)) = make_float4(lo[0], lo[1], lo[2], lo[3]);
        } else {
#pragma unroll
          for (int i = 0; i < 4; ++i) xh[4 * j + i] = 0.0f;
        }
      }
      // stores aligned to their widths (the column base is a multiple of 64)
      const uint32_t ta = acol + lane_base + 4 * c0;
      if (hh == 0) {
        tc::tmem_st16(ta, xh);
        tc::tmem_st8(ta + 16, xh + 16);
        tc::tmem_st4(ta + 24, xh + 24);
      } else {
        tc::tmem_st4(ta, xh);
        tc::tmem_st16(ta + 4, xh + 4);
        tc::tmem_st8(ta + 20, xh + 20);
      }
      tc::tmem_wait_st();
    }
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    slot_sync(slot);
    if (stid == 0) {
      tc::fence_after_sync();
      issue_split_ts(tcol, acol, xl, w2, kFold ? 5 : 7);
      tc::commit(bar);
      if (t + tstride < ntiles) {  // ROWS has been read: bring this slot's next tile
        fetch_rows(t + tstride);
        rows_pending = true;
        rows_parity = rphase;
      }
    }
    if (kFold && stid < NH) {  // the tile's hidden bias, while its MMA runs (read after the wait)
      float sh[16];
      sh16(dnx, dny, dnz, sh);
      if (t + tstride < ntiles) {  // the direction of the slot's next tile's ray, a tile ahead
        const int64_t r = (t + tstride) * TM / src.S;
        dnx = __ldg(src.rays_d + 3 * r);
        dny = __ldg(src.rays_d + 3 * r + 1);
        dnz = __ldg(src.rays_d + 3 * r + 2);
      }
      BETA[stid] = fold_bias(w, stid, sh);
    }
    const bool ok = tc::mbar_wait(bar, phase, wait_limit);
    phase ^= 1u;
    if (!ok) {
      s_fail[slot] = 1;
      mma_pending = true;  // read by slot thread 0 only
    }
    slot_sync(slot);
    if (s_fail[slot]) break;
    tc::fence_after_sync();
    float z[32];
    tmem_ld_sum32(tcol + lane_base + 32 * hh, z);
    float p0, p1, p2;
    colour_partial(z, hh, kFold ? BETA : B0, W1s, p0, p1, p2);
    float* r = RED + (hh * TM + m) * 4;
    r[0] = p0;
    r[1] = p1;
    r[2] = p2;
    tc::fence_before_sync();
    slot_sync(slot);
    if (stid < TM && m0 + stid < P) {
#pragma unroll
      for (int c = 0; c < NO; ++c) {
        const float o = (B1[c] + RED[stid * 4 + c]) + RED[(TM + stid) * 4 + c];
        colors[(m0 + stid) * NO + c] = sigmoidf_ref(o);
      }
    }
  }
  if (stid == 0 && s_fail[slot]) {
    // this slot's MMA and a rows copy into its buffer may still run: let them finish (bounded)
    // before TMEM and shared memory are released
    if (mma_pending) tc::mbar_wait(bar, phase ^ 1u, kDrainLimit);
    if (rows_pending) tc::mbar_wait(bar_rows, rows_parity, kDrainLimit);
    report_timeout(g.status);
  }
  tc::fence_before_sync();
  __syncthreads();
  if (tid < 32) tc::tmem_dealloc(*s_taddr, 512);
}

// Adjoint. d_out (P,3) -> d_hash (P,32), d_normal (P,3), per-block weight-gradient partials
// [dW0 (64 x 52) | dW1 (3 x 64) | db0 (64) | db1 (3)]. tcgen05 kind::tf32 takes K-major operands
// only here, so the sample contraction of dW0 reads transposed copies: X^T (written as the rows
// are staged) and DZ^T, whose scalar stores are bank-conflict free because their 16-byte K chunks
// of 4 samples sit 1040 / 2064 bytes apart (one 16-byte pad per chunk slab).
// Per tile: stage rows -> Z MMA -> epilogue (colours, dO, dW1 in registers, DZ) -> dX MMA ->
// DZ^T -> dW0 MMA (overlapping the dX readout). TMEM columns: Z, then dX, in [0,128) (two halves
// each); dW0 = [DZ_hi | DZ_lo]^T X_hi in [128,192) and x X_lo in [192,256); dW1 sums in
// [256,448); the hi part of the Z and dX MMAs' A operand (X_hi, then DZ_hi; sample lanes, K along
// the columns) in [448,512), written by the threads with tcgen05.st, so it takes no shared-memory
// stores or operand reads (the lo parts stay in R1).
constexpr uint32_t kXtSlab = 16 * 128 + 16;   // X^T: 4 samples x 128 rows (features hi | features lo)
constexpr uint32_t kDztSlab = 16 * 128 + 16;  // DZ^T: 4 samples x 128 rows (hidden hi | hidden lo)
constexpr uint32_t kXtBytes = 32 * kXtSlab;
constexpr uint32_t kR1Bytes = 66560;          // X (hi, lo) -> DZ (hi, lo) -> DZ^T, one at a time
constexpr uint32_t kRowBytes = KP * 4;        // one 52-float input row
constexpr uint32_t kRowsBytes = TM * kRowBytes;  // the next tile's rows, brought in by a bulk copy
constexpr uint32_t kAhiCol = 448;                // TMEM column of A_hi (X_hi, then DZ_hi)

__device__ __forceinline__ uint32_t xt_off(int f, int m) {
  return (uint32_t)((m >> 2) * kXtSlab + (f >> 3) * 128 + (f & 7) * 16 + (m & 3) * 4);
}
__device__ __forceinline__ uint32_t dzt_off(int r, int m) {
  return (uint32_t)((m >> 2) * kDztSlab + (r >> 3) * 128 + (r & 7) * 16 + (m & 3) * 4);
}
// W0^T [hi; lo] (row f < 64: hi of feature f, else lo of feature f - 64; hidden K): element (f, n)
// at (n/4)*2048 + (f/8)*128 + (f%8)*16 + (n%4)*4
__device__ __forceinline__ uint32_t wt_off(int f, int n) {
  return (uint32_t)((n >> 2) * 2048 + (f >> 3) * 128 + (f & 7) * 16 + (n & 3) * 4);
}

// kBulk: the rows are contiguous 52-float rows (ldx = 52, 16-byte aligned); each tile's rows reach
// shared memory through one bulk copy issued as soon as the previous tile has been staged, so no
// registers or load instructions are spent on the prefetch. Otherwise the rows are prefetched
// into registers during the previous tile.
template <bool kBulk, bool kCustomWait, bool kCompact, bool kFold>
__global__ void __launch_bounds__(256, 1) k_mlp_bwd_tc(const float* __restrict__ X, int64_t ldx, int xvec, int64_t P,
                                                      MlpW w, const float* __restrict__ d_out,
                                                      const float* __restrict__ y_in,
                                                      float* __restrict__ d_hash, float* __restrict__ d_normal,
                                                      float* __restrict__ partials, TcGuard g, RowSrc src) {
  static_assert(!kFold || (kCompact && kBulk), "the folded MLP reads compact rows by bulk copy");
  constexpr uint32_t kRowB = (kCompact ? KC : KP) * 4;  // bytes per row in global and shared memory
  extern __shared__ __align__(1024) uint8_t smem[];
  const uint32_t wait_limit = kCustomWait ? g.limit : kWaitLimit;
  uint8_t* W2 = smem;
  uint8_t* WT2 = W2 + kWBytes;
  uint8_t* XT2 = WT2 + kWBytes;
  uint8_t* R1 = XT2 + kXtBytes;
  uint8_t* ROWS = R1 + kR1Bytes;  // kBulk only
  float* RED = reinterpret_cast<float*>(ROWS + (kBulk ? TM * kRowB : 0));  // [2][TM][4]
  float* W1s = RED + 2 * TM * 4;
  float* B0 = W1s + NO * NH;
  float* B1 = B0 + NH;
  uint64_t* bar = reinterpret_cast<uint64_t*>(B1 + 4);
  uint64_t* bar_rows = bar + 1;
  uint32_t* s_taddr = reinterpret_cast<uint32_t*>(bar + 2);
  // kFold: the SH columns of dW0, [16][128]: one column per TMEM lane of DZ^T (hidden unit hi
  // parts in lanes 0..63, lo parts in 64..127; lanes consecutive, so a warp's accesses are
  // conflict-free); the hidden bias of the last two tiles (read as float4: 16-byte aligned) and
  // their SH(d). The dynamic shared memory starts 1024-byte aligned, so aligning the address
  // aligns the offset.
  float* SHACC = reinterpret_cast<float*>((reinterpret_cast<uintptr_t>(bar) + 24 + 15) & ~uintptr_t(15));
  float* BETA = SHACC + TM * 16;  // [2][64]: tiles by parity
  float* SHT = BETA + 2 * NH;     // [2][16]
  const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31, q = wid & 3, hh = wid >> 2;
  const int m = 32 * q + lane;  // this thread's sample in the tile (its TMEM lane)
  // W0 [hi; lo] (hidden rows) for Z, W0^T [hi; lo] (feature rows) for dX, b0, W1, b1; X^T feature
  // rows 52..63 (hi and lo) zero
  for (int e = tid; e < NH * 64; e += blockDim.x) {
    const int n = e >> 6, k = e & 63;
    const int col = kFold ? fold_col(k) : (k < KIN ? k : -1);
    float h, l;
    tc::split_tf32(col >= 0 ? w.W0[n * KIN + col] : 0.0f, h, l);
    *reinterpret_cast<float*>(W2 + w_off(n, k)) = h;
    *reinterpret_cast<float*>(W2 + w_off(NH + n, k)) = l;
    *reinterpret_cast<float*>(WT2 + wt_off(k, n)) = h;
    *reinterpret_cast<float*>(WT2 + wt_off(64 + k, n)) = l;
  }
  constexpr int kXtZero = kFold ? 36 : 52;  // X^T feature rows never written by the tiles
  for (int e = tid; e < (64 - kXtZero) * TM; e += blockDim.x) {
    *reinterpret_cast<float*>(XT2 + xt_off(kXtZero + e / TM, e % TM)) = 0.0f;
    *reinterpret_cast<float*>(XT2 + xt_off(64 + kXtZero + e / TM, e % TM)) = 0.0f;
  }
  if (kFold && hh == 1) {
#pragma unroll
    for (int k = 0; k < 16; ++k) SHACC[k * TM + m] = 0.0f;
  }

  for (int i = tid; i < NH; i += blockDim.x) B0[i] = w.b0[i];
  for (int i = tid; i < NO * NH; i += blockDim.x) W1s[i] = w.W1[i];
  if (tid < NO) B1[tid] = w.b1[tid];
  if (tid == 0) {
    tc::mbar_init(bar, 1);
    tc::mbar_init(bar_rows, 1);
  }
  if (wid == 0) tc::tmem_alloc(s_taddr, 512);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = *s_taddr;
  const uint32_t lane_base = (uint32_t)(32 * q) << 16;
  const uint32_t w2 = tc::smem_u32(W2), wt2 = tc::smem_u32(WT2), xt2 = tc::smem_u32(XT2), r1 = tc::smem_u32(R1);
  float ones_prev = 0.0f;  // kFold: this lane's ones column of dW0 after the previous tile
  int it = 0;              // tiles this block has completed
  // kFold, warps 4..7 (lanes 0..127 = the rows of DZ^T): the SH columns of dW0 from a completed
  // tile: its column sum of dL/dz (its growth of the ones column, feature 35 of the X_hi product;
  // lane m is hidden unit m % 64, hi or lo part) times its SH(d)
  auto fold_sh_columns = [&](const float* sht) {
    float v[4];
    tc::tmem_ld4(tbase + lane_base + 128 + 32, v);
    tc::tmem_wait_ld();
    const float sum = v[3] - ones_prev;
    ones_prev = v[3];
#pragma unroll
    for (int k = 0; k < 16; ++k) SHACC[k * TM + m] = fmaf(sum, sht[k], SHACC[k * TM + m]);
  };
  // kFold, threads 0..63: the hidden bias and (thread 0) the SH(d) of tile `tile` into buffer
  // `buf`, a tile ahead (the global loads overlap the previous tile's dW0 MMAs)
  auto fold_prepare = [&](int64_t tile, int buf) {
    if (tid < NH) {
      float sh[16];
      ray_sh(src.rays_d, tile * TM / src.S, sh);
      BETA[NH * buf + tid] = fold_bias(w, tid, sh);
      if (tid == 0) {
#pragma unroll
        for (int k = 0; k < 16; ++k) SHT[16 * buf + k] = sh[k];
      }
    }
  };
  const int64_t ntiles = (P + TM - 1) / TM;
  // rows of tile t into ROWS (kBulk): one copy of the tile's valid rows, issued by thread 0
  auto fetch_rows = [&](int64_t t) {
    const int64_t m0 = t * TM;
    const uint32_t bytes = (uint32_t)(P - m0 < TM ? P - m0 : TM) * kRowB;
    tc::mbar_arrive_expect_tx(bar_rows, bytes);
    tc::bulk_g2s(ROWS, X + m0 * (kRowB / 4), bytes, bar_rows);
  };
  uint32_t rphase = 0;
  // thread 0's bookkeeping for a give-up: a rows copy in flight and the mbarrier parity it completes
  bool rows_pending = false;
  uint32_t rows_parity = 0;
  if (kBulk && tid == 0 && (int64_t)blockIdx.x < ntiles) {
    fetch_rows(blockIdx.x);
    rows_pending = true;
  }
  // dW1 accumulators of hidden units 32*hh+j, colour c, summed over this thread's samples: TMEM
  // columns 256 + 96*hh + 32*c + j of this thread's lane (registers are spent on the prefetch)
  const uint32_t g1addr = tbase + lane_base + 256 + 96 * hh;
  {
    float zero[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) zero[j] = 0.0f;
#pragma unroll
    for (int c = 0; c < NO; ++c) tc::tmem_st32(g1addr + 32 * c, zero);
    tc::tmem_wait_st();
  }
  float sb[NO] = {0.0f, 0.0f, 0.0f};
  bool first_w = true, failed = false;
  bool mma_pending = false;  // thread 0: its own wait on an MMA gave up
  uint32_t phase = 0;
  float4 pre[7];  // !kBulk: this tile's row chunks, loaded during the previous tile
  float dy[NO], yv[NO] = {0.0f, 0.0f, 0.0f};  // dL/dcolour and (y_in) the forward's colour of this sample
  if ((int64_t)blockIdx.x < ntiles) {
    const int64_t m0 = (int64_t)blockIdx.x * TM;
    if (kFold) fold_prepare(blockIdx.x, 0);
    if (!kBulk) load_row_chunks(X, ldx, xvec != 0, P, m0, m, hh, pre);
#pragma unroll
    for (int c = 0; c < NO; ++c) {
      dy[c] = m0 + m < P ? d_out[(m0 + m) * NO + c] : 0.0f;
      if (y_in) yv[c] = m0 + m < P ? y_in[(m0 + m) * NO + c] : 0.0f;
    }
  }
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t m0 = t * TM;
    const bool valid = m0 + m < P;
    if (kBulk) {
      const bool got = tc::mbar_wait(bar_rows, rphase, wait_limit);
      rphase ^= 1u;
      if (__syncthreads_or(!got)) {
        failed = true;
        break;
      }
      if (tid == 0) rows_pending = false;
    }
    // rows -> X_hi (TMEM, sample lanes), X_lo (sample rows, R1) and X^T (feature rows); column 51
    // (folded: 35) = 1 on real rows (db0)
    if constexpr (kFold) {
      const int c0 = hh ? 5 : 0;
      const float4* rrow = reinterpret_cast<const float4*>(ROWS + m * kRowB);
      float xh[20];  // features 4*c0 .. 4*c0 + 19: [hash 32 | normal 3 | one | 0 x 4]
#pragma unroll
      for (int jc = 0; jc < 5; ++jc) {
        const int c = c0 + jc;
        float4 u = (valid && c < 9) ? rrow[c] : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        if (c == 8) u.w = valid ? 1.0f : 0.0f;
        const float v[4] = {u.x, u.y, u.z, u.w};
        float lo[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          tc::split_tf32(v[i], xh[4 * jc + i], lo[i]);
          if (c < 9) {
            *reinterpret_cast<float*>(XT2 + xt_off(4 * c + i, m)) = xh[4 * jc + i];
            *reinterpret_cast<float*>(XT2 + xt_off(64 + 4 * c + i, m)) = lo[i];
          }
        }
        *reinterpret_cast<float4*>(R1 + kXBytes + x_off(c, m)) = make_float4(lo[0], lo[1], lo[2], lo[3]);
      }
      const uint32_t ta = tbase + lane_base + kAhiCol + 4 * c0;  // stores aligned to their widths
      if (hh == 0) {
        tc::tmem_st16(ta, xh);
        tc::tmem_st4(ta + 16, xh + 16);
      } else {
        tc::tmem_st4(ta, xh);
        tc::tmem_st8(ta + 4, xh + 4);
        tc::tmem_st8(ta + 12, xh + 12);
      }
      tc::tmem_wait_st();
    } else {
      const int c0 = hh ? 7 : 0;
      const float4* rrow = reinterpret_cast<const float4*>(ROWS + m * kRowB);
      const float3 dir = stage_dir<kCompact>(src, m0 + m, valid && hh);
      float xh[28];  // features 4*c0 .. 4*c0 + 27 (hh = 1: 28..55, with 52..55 the zero chunk 13)
#pragma unroll
      for (int jc = 0; jc < 7; ++jc) {
        const int c = c0 + jc;
        if (c < 13) {
          float4 u;
          if (kBulk)
            u = valid ? x_chunk<kCompact>(rrow, hh, jc, dir) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
          else
            u = pre[jc];
          float v[4] = {u.x, u.y, u.z, u.w};
          if (c == 12 && valid) v[3] = 1.0f;
          float lo[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            tc::split_tf32(v[i], xh[4 * jc + i], lo[i]);
            *reinterpret_cast<float*>(XT2 + xt_off(4 * c + i, m)) = xh[4 * jc + i];
            *reinterpret_cast<float*>(XT2 + xt_off(64 + 4 * c + i, m)) = lo[i];
          }
          *reinterpret_cast<float4*>(R1 + kXBytes + x_off(c, m)) = make_float4(lo[0], lo[1], lo[2], lo[3]);
        } else {  // feature chunk 13 (columns 52..55) is inside the Z contraction: zero
#pragma unroll
          for (int i = 0; i < 4; ++i) xh[4 * jc + i] = 0.0f;
          *reinterpret_cast<float4*>(R1 + kXBytes + x_off(13, m)) = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        }
      }
      // X_hi at TMEM column kAhiCol + feature, in stores aligned to their widths
      const uint32_t ta = tbase + lane_base + kAhiCol + 4 * c0;
      if (hh == 0) {
        tc::tmem_st16(ta, xh);
        tc::tmem_st8(ta + 16, xh + 16);
        tc::tmem_st4(ta + 24, xh + 24);
      } else {
        tc::tmem_st4(ta, xh);
        tc::tmem_st16(ta + 4, xh + 4);
        tc::tmem_st8(ta + 20, xh + 20);
      }
      tc::tmem_wait_st();
    }
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      issue_split_ts(tbase, tbase + kAhiCol, r1 + kXBytes, w2, kFold ? 5 : 7);
      tc::commit(bar);
      if (kBulk && t + gridDim.x < ntiles) {  // ROWS has been read: bring the next tile's rows
        fetch_rows(t + gridDim.x);
        rows_pending = true;
        rows_parity = rphase;
      }
    }
    // while the Z MMA runs: the previous tile's SH columns of dW0
    if (kFold && hh == 1 && it > 0) fold_sh_columns(SHT + 16 * ((it - 1) & 1));
    bool ok = tc::mbar_wait(bar, phase, wait_limit);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
      failed = true;
      mma_pending = !ok;
      break;
    }
    tc::fence_after_sync();
    float z[32];
    tmem_ld_sum32(tbase + lane_base + 32 * hh, z);
    float d[NO];
    if (y_in) {  // the forward's colours: the same bits as the recomputation below
#pragma unroll
      for (int c = 0; c < NO; ++c) d[c] = dy[c] * ((1.0f - yv[c]) * yv[c]);  // 0 on rows past P
    } else {     // block-uniform branch: every thread takes the same side of the barrier
      {
        float p0, p1, p2;
        colour_partial(z, hh, kFold ? BETA + NH * (it & 1) : B0, W1s, p0, p1, p2);
        float* r = RED + (hh * TM + m) * 4;
        r[0] = p0;
        r[1] = p1;
        r[2] = p2;
      }
      __syncthreads();
#pragma unroll
      for (int c = 0; c < NO; ++c) {
        const float o = (B1[c] + RED[m * 4 + c]) + RED[(TM + m) * 4 + c];
        const float y = sigmoidf_ref(o);
        d[c] = dy[c] * ((1.0f - y) * y);  // dL/d(pre-sigmoid); 0 on rows past P
      }
    }
    if (hh == 0) {
#pragma unroll
      for (int c = 0; c < NO; ++c) sb[c] += d[c];
    }
    // dW1 (TMEM accumulators), dL/dz (kept in z), then DZ: the Z MMA has read X
#pragma unroll
    for (int j4 = 0; j4 < 8; ++j4) {
      const float4 b = *reinterpret_cast<const float4*>((kFold ? BETA + NH * (it & 1) : B0) + 32 * hh + 4 * j4);
      z[4 * j4] += b.x;
      z[4 * j4 + 1] += b.y;
      z[4 * j4 + 2] += b.z;
      z[4 * j4 + 3] += b.w;
    }
#pragma unroll 1
    for (int c = 0; c < NO; ++c) {
      float acc[32];
      tc::tmem_ld32(g1addr + 32 * c, acc);
      tc::tmem_wait_ld();
      const float dc = c == 0 ? d[0] : (c == 1 ? d[1] : d[2]);
#pragma unroll
      for (int j = 0; j < 32; ++j) acc[j] = fmaf(dc, fmaxf(z[j], 0.0f), acc[j]);
      tc::tmem_st32(g1addr + 32 * c, acc);
    }
    tc::tmem_wait_st();
#pragma unroll
    for (int j4 = 0; j4 < 8; ++j4) {
      const int n = 32 * hh + 4 * j4;
      const float4 u0 = *reinterpret_cast<const float4*>(W1s + n);
      const float4 u1 = *reinterpret_cast<const float4*>(W1s + NH + n);
      const float4 u2 = *reinterpret_cast<const float4*>(W1s + 2 * NH + n);
      const float w0[4] = {u0.x, u0.y, u0.z, u0.w}, w1[4] = {u1.x, u1.y, u1.z, u1.w};
      const float w2[4] = {u2.x, u2.y, u2.z, u2.w};
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float dhid = d[0] * w0[i] + d[1] * w1[i] + d[2] * w2[i];
        z[4 * j4 + i] = z[4 * j4 + i] > 0.0f ? dhid : 0.0f;
      }
    }
    float zl[32];  // dL/dz split once: hi in z, lo in zl (stored as DZ now and as DZ^T below)
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const float v = z[j];
      tc::split_tf32(v, z[j], zl[j]);
    }
    // DZ_hi into TMEM (over X_hi: the Z MMA has completed), DZ_lo (sample rows) into R1
    tc::tmem_st32(tbase + lane_base + kAhiCol + 32 * hh, z);
#pragma unroll
    for (int j4 = 0; j4 < 8; ++j4)
      *reinterpret_cast<float4*>(R1 + kXBytes + x_off(8 * hh + j4, m)) =
          make_float4(zl[4 * j4], zl[4 * j4 + 1], zl[4 * j4 + 2], zl[4 * j4 + 3]);
    tc::tmem_wait_st();
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {  // dX = DZ W0 (B = W0^T [hi; lo], feature rows) into the columns Z used
      tc::fence_after_sync();
      issue_split_ts(tbase, tbase + kAhiCol, r1 + kXBytes, wt2, 8);
      tc::commit(bar);
    }
    ok = tc::mbar_wait(bar, phase, wait_limit);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
      failed = true;
      mma_pending = !ok;
      break;
    }
    tc::fence_after_sync();
    // DZ^T into R1 (the dX MMA has read DZ): rows 0..63 hi, 64..127 lo
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const int n = 32 * hh + j;
      *reinterpret_cast<float*>(R1 + dzt_off(n, m)) = z[j];
      *reinterpret_cast<float*>(R1 + dzt_off(NH + n, m)) = zl[j];
    }
    tc::fence_smem_to_async();
    tc::fence_before_sync();
    __syncthreads();
    // dW0 (+db0) += [DZ_hi | DZ_lo]^T X, K = the tile's samples; issued by a warp whose dX readout
    // is short (d_normal), so the d_hash readout warps are not held behind the issue
    if (tid == 128) {
      tc::fence_after_sync();
#pragma unroll 1
      for (int s = 0; s < 16; ++s) {
        const uint64_t ad = tc::sdesc(r1 + s * 2 * kDztSlab, kDztSlab, 128);
        const uint64_t b = tc::sdesc(xt2 + s * 2 * kXtSlab, kXtSlab, 128);
        tc::mma_tf32(tbase + 128, ad, b, kId128, !first_w);  // [128,192): x X_hi, [192,256): x X_lo
        first_w = false;
      }
      tc::commit(bar);
    }
    // next tile's rows fly during the dW0 MMAs and the dX readout
    if (t + gridDim.x < ntiles) {
      const int64_t mn = (t + gridDim.x) * TM;
      if (kFold) fold_prepare(t + gridDim.x, (it + 1) & 1);
      if (!kBulk) load_row_chunks(X, ldx, xvec != 0, P, mn, m, hh, pre);
#pragma unroll
      for (int c = 0; c < NO; ++c) {
        dy[c] = mn + m < P ? d_out[(mn + m) * NO + c] : 0.0f;
        if (y_in) yv[c] = mn + m < P ? y_in[(mn + m) * NO + c] : 0.0f;
      }
    }
    // dX readout while the dW0 MMAs run
    if (hh == 0) {
      float v[32];
      tmem_ld_sum32(tbase + lane_base, v);
      if (valid) {
        float4* o = reinterpret_cast<float4*>(d_hash + (m0 + m) * 32);
#pragma unroll
        for (int c = 0; c < 8; ++c) o[c] = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
      }
    } else {
      float v[4], u[4];
      constexpr int kNrmCol = kFold ? 32 : 48;  // the normal's feature columns
      tc::tmem_ld4(tbase + lane_base + kNrmCol, v);
      tc::tmem_ld4(tbase + lane_base + 64 + kNrmCol, u);
      tc::tmem_wait_ld();
      if (valid) {
        v[0] += u[0];
        v[1] += u[1];
        v[2] += u[2];
        d_normal[(m0 + m) * 3] = v[0];
        d_normal[(m0 + m) * 3 + 1] = v[1];
        d_normal[(m0 + m) * 3 + 2] = v[2];
      }
    }
    ok = tc::mbar_wait(bar, phase, wait_limit);  // R1 and X^T are rewritten by the next tile
    phase ^= 1u;
    tc::fence_before_sync();
    if (__syncthreads_or(!ok)) {
      failed = true;
      mma_pending = !ok;
      break;
    }
    tc::fence_after_sync();
    ++it;
  }
  if (kFold && hh == 1 && it > 0 && !failed) fold_sh_columns(SHT + 16 * ((it - 1) & 1));  // the last tile's
  if (failed && tid == 0) {
    // the MMAs and a rows copy may still run: let them finish (bounded) before tensor memory is
    // read and freed and the block leaves
    if (mma_pending) tc::mbar_wait(bar, phase ^ 1u, kDrainLimit);
    if (kBulk && rows_pending) tc::mbar_wait(bar_rows, rows_parity, kDrainLimit);
    report_timeout(g.status);
  }
  // weight-gradient partials of this block
  const bool have = blockIdx.x < ntiles && !failed;  // every block with a tile issued the dW0 MMAs
  float* pb = partials + (int64_t)blockIdx.x * WG;
  float* R2 = reinterpret_cast<float*>(R1);           // [64][64]: dW0 rows of DZ_lo x X_hi
  float* RW1 = R2 + 64 * 64;                          // [4 q][2 hh][3][32] dW1, then [4][3] db1
  __syncthreads();
  tc::fence_after_sync();  // thread 0's drain (after a give-up) before this block reads tensor memory
  if (q >= 2) {
    float v[32];
    tc::tmem_ld32(tbase + lane_base + 128 + 32 * hh, v);
    tc::tmem_wait_ld();
#pragma unroll
    for (int j = 0; j < 32; ++j) R2[(m - 64) * 64 + 32 * hh + j] = have ? v[j] : 0.0f;
  }
#pragma unroll 1
  for (int c = 0; c < NO; ++c) {
    float acc[32];
    tc::tmem_ld32(g1addr + 32 * c, acc);
    tc::tmem_wait_ld();
#pragma unroll
    for (int j = 0; j < 32; ++j) acc[j] = warp_sum(acc[j]);
    const float sbc = warp_sum(c == 0 ? sb[0] : (c == 1 ? sb[1] : sb[2]));
    if (lane == 0) {
#pragma unroll
      for (int j = 0; j < 32; ++j) RW1[((q * 2 + hh) * 3 + c) * 32 + j] = acc[j];
      if (hh == 0) RW1[4 * 2 * 3 * 32 + q * 3 + c] = sbc;
    }
  }
  __syncthreads();
  if (q < 2) {
    float v1[32], v2[32];
    tc::tmem_ld32(tbase + lane_base + 128 + 32 * hh, v1);
    tc::tmem_ld32(tbase + lane_base + 192 + 32 * hh, v2);
    tc::tmem_wait_ld();
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const int col = 32 * hh + j;
      const float val = have ? (v1[j] + v2[j]) + R2[m * 64 + col] : 0.0f;
      if (kFold) {  // folded feature col -> the column of W0 it came from; 35 is the ones column
        const int oc = fold_col(col);
        if (oc >= 0) pb[m * KP + oc] = val;
        if (col == 35) pb[NH * KP + NO * NH + m] = val;
      } else {
        if (col < KP) pb[m * KP + col] = val;
        if (col == KIN) pb[NH * KP + NO * NH + m] = val;  // ones column: db0
      }
    }
    if (kFold && hh == 0) {  // the SH columns 32..47 (hi + lo lanes) and the padding column
#pragma unroll
      for (int k = 0; k < 16; ++k) pb[m * KP + 32 + k] = have ? SHACC[k * TM + m] + SHACC[k * TM + 64 + m] : 0.0f;
      pb[m * KP + KIN] = 0.0f;
    }
  }
  if (tid < NO * NH) {
    const int c = tid / NH, n = tid % NH, h2 = n >> 5, j = n & 31;
    float s = 0.0f;
#pragma unroll
    for (int qq = 0; qq < 4; ++qq) s += RW1[((qq * 2 + h2) * 3 + c) * 32 + j];
    pb[NH * KP + c * NH + n] = have ? s : 0.0f;
  }
  if (tid < NO) {
    float s = 0.0f;
#pragma unroll
    for (int qq = 0; qq < 4; ++qq) s += RW1[4 * 2 * 3 * 32 + qq * 3 + tid];
    pb[NH * KP + NO * NH + NH + tid] = have ? s : 0.0f;
  }
  tc::fence_before_sync();
  __syncthreads();
  if (wid == 0) tc::tmem_dealloc(tbase, 512);
}

constexpr size_t kBwdSmemRegs = 2 * kWBytes + kXtBytes + kR1Bytes + sizeof(float) * (2 * TM * 4 + NO * NH + NH + 4) + 24;
constexpr size_t kBwdSmemBulk = kBwdSmemRegs + kRowsBytes;
constexpr size_t kBwdSmemCompact = kBwdSmemRegs + TM * KC * 4;
// SHACC, BETA, SHT after the compact layout, from the next 16-byte boundary (BETA is read as float4)
constexpr size_t kBwdSmemFold = (kBwdSmemCompact + 15) / 16 * 16 + sizeof(float) * (TM * 16 + 2 * NH + 32);
static_assert((TM * 16 * sizeof(float)) % 16 == 0, "BETA must stay 16-byte aligned after SHACC");
static_assert(kBwdSmemFold <= 227 * 1024, "the folded adjoint's shared memory exceeds a CTA's");


// Sum the per-block partials into dW0 (64,51), dW1 (3,64), db0 (64), db1 (3), in a fixed order
// (deterministic): a block of 32 x 8 threads takes 32 consecutive elements; thread (x, y) sums
// the partials of blocks y, y + 8, y + 16, ... in increasing order, and the 8 slice sums are then
// added in slice order. Loads are coalesced along the elements.
constexpr int kReduceSlices = 8;

__global__ void __launch_bounds__(256) k_mlp_wgrad_reduce(const float* __restrict__ partials, int nblocks,
                                                          float* __restrict__ dW0, float* __restrict__ db0,
                                                          float* __restrict__ dW1, float* __restrict__ db1) {
  __shared__ double part[kReduceSlices][32];
  const int e = blockIdx.x * 32 + threadIdx.x;
  double acc = 0.0;
  if (e < WG)
    for (int b = threadIdx.y; b < nblocks; b += kReduceSlices) acc += (double)__ldg(partials + (int64_t)b * WG + e);
  part[threadIdx.y][threadIdx.x] = acc;
  __syncthreads();
  if (threadIdx.y != 0 || e >= WG) return;
  double sum = 0.0;
#pragma unroll
  for (int y = 0; y < kReduceSlices; ++y) sum += part[y][threadIdx.x];
  const float v = (float)sum;
  if (e < NH * KP) {
    const int n = e / KP, k = e % KP;
    if (k < KIN) dW0[n * KIN + k] = v;
  } else if (e < NH * KP + NO * NH) {
    dW1[e - NH * KP] = v;
  } else if (e < NH * KP + NO * NH + NH) {
    db0[e - NH * KP - NO * NH] = v;
  } else {
    db1[e - NH * KP - NO * NH - NH] = v;
  }
}

// MLP input rows [hash 32 | SH 16 | normal 3 | 0] of the training forward. A block of 256 threads
// covers 64 consecutive samples: warp w gathers levels 4(w/2)..4(w/2)+3 for the samples
// 32(w%2)..32(w%2)+31, so each gather instruction reads one level for 32 consecutive samples of
// a ray, and neighbouring samples that share a coarse-level cell share its request. Warps of
// level group 0 also evaluate the SH of the view direction, group 1 copies the normal; the rows
// meet in shared memory and leave as one contiguous block (or row by row for a wider stride).
constexpr int kRowsPerBlock = 64;

template <bool kCompact>
__global__ void __launch_bounds__(256) k_hash_rows(HashArgs a) {
  constexpr int kChunks = kCompact ? KC / 4 : 13;  // float4 chunks per row
  __shared__ float4 srow[kRowsPerBlock * kChunks];
  const uint32_t mask = (1u << a.log2T) - 1u;
  const size_t T = (size_t)1 << a.log2T;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, g = w >> 1;
  const int ls = 32 * (w & 1) + lane;  // this thread's sample in the block
  for (int64_t base = (int64_t)blockIdx.x * kRowsPerBlock; base < a.P; base += (int64_t)gridDim.x * kRowsPerBlock) {
    const int64_t i = base + ls;
    if (i < a.P) {
      float x[3];
      sample_pos(a, i, x);
      float f[8];
#pragma unroll
      for (int qq = 0; qq < 4; ++qq) {
        const int l = 4 * g + qq;
        const float lw = a.lw[l];
        float f0 = 0.0f, f1 = 0.0f;
        if (lw != 0.0f) {
          LevelCell c;
          level_cell(x, a.res[l], mask, c);
          const float2* tab = reinterpret_cast<const float2*>(a.table) + (size_t)l * T;
          gather_level(tab, c, f0, f1);
          if (lw < 1.0f) {
            f0 *= lw;
            f1 *= lw;
          }
        }
        f[2 * qq] = f0;
        f[2 * qq + 1] = f1;
      }
      srow[ls * kChunks + 2 * g] = make_float4(f[0], f[1], f[2], f[3]);
      srow[ls * kChunks + 2 * g + 1] = make_float4(f[4], f[5], f[6], f[7]);
      if (g == 0 && !kCompact) {
        const int64_t r = i / a.S;
        float o[16];
        sh16(__ldg(a.rays_d + 3 * r), __ldg(a.rays_d + 3 * r + 1), __ldg(a.rays_d + 3 * r + 2), o);
#pragma unroll
        for (int c = 0; c < 4; ++c)
          srow[ls * kChunks + 8 + c] = make_float4(o[4 * c], o[4 * c + 1], o[4 * c + 2], o[4 * c + 3]);
      } else if (g == 1) {
        srow[ls * kChunks + kChunks - 1] = make_float4(a.normals[3 * i], a.normals[3 * i + 1], a.normals[3 * i + 2],
                                                       0.0f);
      }
    }
    __syncthreads();
    const int nrows = (int)(a.P - base < kRowsPerBlock ? a.P - base : kRowsPerBlock);
    if (a.ld == 4 * kChunks) {
      float4* out = reinterpret_cast<float4*>(a.out + base * (4 * kChunks));
      for (int k = tid; k < nrows * kChunks; k += 256) out[k] = srow[k];
    } else {
      for (int k = tid; k < nrows * kChunks; k += 256)
        reinterpret_cast<float4*>(a.out + (base + k / kChunks) * a.ld)[k % kChunks] = srow[k];
    }
    __syncthreads();
  }
}

// k_hash_rows over a.P samples, one wave of resident blocks; compact rows when a.ld == KC.
void launch_hash_rows(const HashArgs& a, cudaStream_t st) {
  static int rows_per_sm[2] = {0, 0};
  const bool compact = a.ld == KC;
  auto kern = compact ? k_hash_rows<true> : k_hash_rows<false>;
  if (rows_per_sm[compact] == 0) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, 256, 0) != cudaSuccess || nb < 1) nb = 4;
    rows_per_sm[compact] = nb;
  }
  kern<<<grid_for((a.P + kRowsPerBlock - 1) / kRowsPerBlock * 256, 256, rows_per_sm[compact]), 256, 0, st>>>(a);
}

template <bool kHashIn, bool kRowsOut>
int launch_fwd(const HashArgs& a, const float* X, int64_t ldx, int64_t P, const MlpW& w, float* colors,
               cudaStream_t st, RowSrc src = RowSrc{nullptr, 0}) {
  const int64_t tiles = (P + TM - 1) / TM;
  const bool compact = src.rays_d != nullptr;
  if (!kHashIn && (compact || ldx == KP) && (reinterpret_cast<uintptr_t>(X) & 15) == 0) {  // contiguous rows: two slots
    // compact rows whose tiles each lie inside one ray (samples per ray a multiple of the tile):
    // the folded MLP
    const bool fold = compact && src.S % TM == 0;
    const bool cw = custom_wait();
    auto kern2 = fold ? (cw ? k_mlp_fwd_rows2<true, true, true> : k_mlp_fwd_rows2<false, true, true>)
                 : compact ? (cw ? k_mlp_fwd_rows2<true, true, false> : k_mlp_fwd_rows2<false, true, false>)
                           : (cw ? k_mlp_fwd_rows2<true, false, false> : k_mlp_fwd_rows2<false, false, false>);
    cudaError_t e = cudaFuncSetAttribute(kern2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFwd2Smem);
    if (e != cudaSuccess) return set_error(VX_ERR_CUDA, "mlp forward: %s", cudaGetErrorString(e));
    const int64_t pairs = (tiles + 1) / 2;
    const unsigned blocks = (unsigned)(pairs < (int64_t)kSMs ? pairs : (int64_t)kSMs);
    kern2<<<blocks, 512, kFwd2Smem, st>>>(X, P, w, colors, t_guard, src);
    return VX_OK;
  }
  auto kern = custom_wait() ? k_mlp_fwd_tc<kHashIn, kRowsOut, true> : k_mlp_fwd_tc<kHashIn, kRowsOut, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFwdSmem);
  if (e != cudaSuccess) return set_error(VX_ERR_CUDA, "mlp forward: %s", cudaGetErrorString(e));
  const unsigned blocks = (unsigned)(tiles < (int64_t)kSMs * 2 ? tiles : (int64_t)kSMs * 2);
  const int xvec = X && (ldx % 4 == 0) && ((reinterpret_cast<uintptr_t>(X) & 15) == 0);
  kern<<<blocks, 256, kFwdSmem, st>>>(a, X, ldx, xvec, P, w, colors, t_guard);
  return VX_OK;
}

// The adjoint and its weight-gradient reduction. Full rows (src.rays_d == nullptr, any stride
// >= 51: 52-float contiguous rows take the bulk-copy kernel) or compact rows (bulk copy only).
int mlp_backward_launch(const float* x, int64_t ldx, int64_t n_points, const float* W0, const float* b0,
                        const float* W1, const float* b1, const float* d_colors, const float* colors, float* d_hash,
                        float* d_normal, float* dW0, float* db0, float* dW1, float* db1, float* partials,
                        int64_t n_partial_floats, cudaStream_t st, RowSrc src, const char* what) {
  VX_REQUIRE(x && W0 && b0 && W1 && b1 && d_colors && d_hash && d_normal && dW0 && db0 && dW1 && db1 && partials,
             "null pointer");
  VX_REQUIRE((reinterpret_cast<uintptr_t>(d_hash) & 15) == 0, "d_hash must be 16-byte aligned");
  const int nb = vx_mlp_blocks(n_points);
  VX_REQUIRE(n_partial_floats >= (int64_t)nb * WG, "partials buffer holds %lld floats, need %lld",
             (long long)n_partial_floats, (long long)nb * WG);
  MlpW w{W0, b0, W1, b1};
  const bool compact = src.rays_d != nullptr;
  if (n_points > 0) {
    const int xvec = (ldx % 4 == 0) && ((reinterpret_cast<uintptr_t>(x) & 15) == 0);
    const bool bulk = xvec && (compact || ldx == KP);
    // compact rows whose tiles each lie inside one ray: the folded MLP (as in the forward)
    const bool fold = compact && src.S % TM == 0;
    const size_t smem = fold ? kBwdSmemFold : compact ? kBwdSmemCompact : bulk ? kBwdSmemBulk : kBwdSmemRegs;
    const bool cw = custom_wait();
    auto kern = fold ? (cw ? k_mlp_bwd_tc<true, true, true, true> : k_mlp_bwd_tc<true, false, true, true>)
                : compact ? (cw ? k_mlp_bwd_tc<true, true, true, false> : k_mlp_bwd_tc<true, false, true, false>)
                : bulk ? (cw ? k_mlp_bwd_tc<true, true, false, false> : k_mlp_bwd_tc<true, false, false, false>)
                       : (cw ? k_mlp_bwd_tc<false, true, false, false> : k_mlp_bwd_tc<false, false, false, false>);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return set_error(VX_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    kern<<<nb, 256, smem, st>>>(x, ldx, xvec, n_points, w, d_colors, colors, d_hash, d_normal, partials, t_guard, src);
  } else {
    cudaMemsetAsync(partials, 0, sizeof(float) * WG, st);
  }
  k_mlp_wgrad_reduce<<<(WG + 31) / 32, dim3(32, kReduceSlices), 0, st>>>(partials, n_points > 0 ? nb : 1, dW0, db0,
                                                                        dW1, db1);
  count_launches(2);
  return check_launch(what);
}

}  // namespace vx

using namespace vx;

extern "C" {

int vx_appearance_mlp_forward(const float* table, int n_levels, int log2_size, int n_features,
                              const int32_t* level_res, const float* level_weights, const float* rays_o,
                              const float* rays_d, const float* mid, int n_samples, const float xyz_min[3],
                              const float xyz_max[3], int64_t n_points, const float* normals, const float* W0,
                              const float* b0, const float* W1, const float* b1, float* colors, float* rows,
                              int64_t ld_rows, void* stream) {
  HashArgs a{};
  if (int s = fill_hash(a, table, n_levels, log2_size, n_features, level_res, level_weights)) return s;
  VX_REQUIRE(n_levels == 16, "the fused appearance MLP takes 16 hash levels x 2 features (got %d)", n_levels);
  VX_REQUIRE(n_points >= 0 && n_samples >= 1, "bad sizes");
  if (n_points == 0) return VX_OK;
  VX_REQUIRE(table && rays_o && rays_d && mid && xyz_min && xyz_max && normals && W0 && b0 && W1 && b1 && colors,
             "null pointer");
  VX_REQUIRE(!rows || ((ld_rows == KC || ld_rows >= KP) && ld_rows % 4 == 0 && ((uintptr_t)rows & 15) == 0),
             "rows need a row stride of 36 floats (compact) or >= 52, a multiple of 4, and 16-byte alignment");
  VX_REQUIRE(!rows || ld_rows != KC || n_points < (int64_t(1) << 32), "compact rows take fewer than 2^32 samples");
  fill_positions(a, nullptr, rays_o, rays_d, mid, n_samples, xyz_min, xyz_max);
  a.P = n_points;
  a.out = rows;
  a.ld = ld_rows;
  a.normals = normals;
  MlpW w{W0, b0, W1, b1};
  cudaStream_t st = (cudaStream_t)stream;
  if (rows) {  // training: rows gathered at high occupancy, then the MLP on the rows
    launch_hash_rows(a, st);
    const RowSrc src{ld_rows == KC ? rays_d : nullptr, n_samples};
    if (int s = launch_fwd<false, false>(a, rows, ld_rows, n_points, w, colors, st, src)) return s;
    count_launches(2);
  } else {  // inference: features built in shared memory, nothing else written
    if (int s = launch_fwd<true, false>(a, nullptr, 0, n_points, w, colors, st)) return s;
    count_launches(1);
  }
  return check_launch("appearance_mlp_forward");
}

int vx_appearance_mlp_forward_chunked(const float* table, int n_levels, int log2_size, int n_features,
                                      const int32_t* level_res, const float* level_weights, const float* rays_o,
                                      const float* rays_d, const float* mid, int n_samples, const float xyz_min[3],
                                      const float xyz_max[3], int64_t n_points, const float* normals,
                                      const float* W0, const float* b0, const float* W1, const float* b1,
                                      float* colors, float* scratch_rows, int64_t scratch_count, void* stream) {
  HashArgs a{};
  if (int s = fill_hash(a, table, n_levels, log2_size, n_features, level_res, level_weights)) return s;
  VX_REQUIRE(n_levels == 16, "the fused appearance MLP takes 16 hash levels x 2 features (got %d)", n_levels);
  VX_REQUIRE(n_points >= 0 && n_samples >= 1, "bad sizes");
  VX_REQUIRE(n_points % n_samples == 0, "n_points must be whole rays (a multiple of n_samples)");
  if (n_points == 0) return VX_OK;
  VX_REQUIRE(table && rays_o && rays_d && mid && xyz_min && xyz_max && normals && W0 && b0 && W1 && b1 && colors &&
                 scratch_rows,
             "null pointer");
  VX_REQUIRE(((uintptr_t)scratch_rows & 15) == 0, "scratch rows must be 16-byte aligned");
  VX_REQUIRE(scratch_count >= n_samples, "scratch holds %lld rows, fewer than one ray's %d samples",
             (long long)scratch_count, n_samples);
  VX_REQUIRE(scratch_count < (int64_t(1) << 32), "the scratch takes fewer than 2^32 rows");
  fill_positions(a, nullptr, rays_o, rays_d, mid, n_samples, xyz_min, xyz_max);
  a.ld = KC;  // compact rows: SH(d) is recomputed from rays_d by the MLP kernel
  a.out = scratch_rows;
  MlpW w{W0, b0, W1, b1};
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t chunk = (scratch_count / n_samples) * n_samples;  // whole rays per pass
  int launches = 0;
  for (int64_t c0 = 0; c0 < n_points; c0 += chunk) {
    const int64_t len = n_points - c0 < chunk ? n_points - c0 : chunk;
    HashArgs ac = a;
    const int64_t r0 = c0 / n_samples;
    ac.rays_o = rays_o + 3 * r0;
    ac.rays_d = rays_d + 3 * r0;
    ac.mid = mid + c0;
    ac.normals = normals + 3 * c0;
    ac.P = len;
    launch_hash_rows(ac, st);
    if (int s = launch_fwd<false, false>(ac, scratch_rows, KC, len, w, colors + 3 * c0, st,
                                         RowSrc{ac.rays_d, n_samples}))
      return s;
    launches += 2;
  }
  count_launches(launches);
  return check_launch("appearance_mlp_forward_chunked");
}

int vx_mlp_blocks(int64_t n_points) {
  const int64_t tiles = (n_points + TM - 1) / TM;
  const int64_t cap = (int64_t)kSMs;
  return (int)(tiles < 1 ? 1 : (tiles < cap ? tiles : cap));
}

int vx_mlp_partial_floats(void) { return WG; }

int vx_tc_guard(int* status, int64_t wait_polls) {
  VX_REQUIRE(wait_polls <= (int64_t)UINT32_MAX, "wait_polls above 2^32 - 1");
  t_guard.status = status;
  t_guard.limit = wait_polls < 0 ? kWaitLimit : (uint32_t)wait_polls;
  return VX_OK;
}

int vx_tensor_core_timeouts(void) {
  int h = 0;
  const int zero = 0;
  if (cudaMemcpyFromSymbol(&h, g_tc_timeouts, sizeof(int)) != cudaSuccess) return -1;
  if (cudaMemcpyToSymbol(g_tc_timeouts, &zero, sizeof(int)) != cudaSuccess) return -1;
  return h;
}

int vx_radiance_mlp_forward(const float* x, int64_t ldx, int64_t n_points, int in_dim, int hidden, int out_dim,
                            const float* W0, const float* b0, const float* W1, const float* b1, float* colors,
                            void* stream) {
  VX_REQUIRE(in_dim == KIN && hidden == NH && out_dim == NO, "the fused MLP is %d -> %d -> %d (got %d -> %d -> %d)",
             KIN, NH, NO, in_dim, hidden, out_dim);
  VX_REQUIRE(n_points >= 0 && ldx >= KIN, "bad sizes");
  if (n_points == 0) return VX_OK;
  VX_REQUIRE(x && W0 && b0 && W1 && b1 && colors, "null pointer");
  MlpW w{W0, b0, W1, b1};
  HashArgs a{};
  if (int s = launch_fwd<false, false>(a, x, ldx, n_points, w, colors, (cudaStream_t)stream)) return s;
  count_launches(1);
  return check_launch("radiance_mlp_forward");
}

int vx_radiance_mlp_backward(const float* x, int64_t ldx, int64_t n_points, int in_dim, int hidden, int out_dim,
                             const float* W0, const float* b0, const float* W1, const float* b1, const float* d_colors,
                             const float* colors, float* d_hash, float* d_normal, float* dW0, float* db0, float* dW1,
                             float* db1, float* partials, int64_t n_partial_floats, void* stream) {
  VX_REQUIRE(in_dim == KIN && hidden == NH && out_dim == NO, "the fused MLP is %d -> %d -> %d", KIN, NH, NO);
  VX_REQUIRE(n_points >= 0 && ldx >= KIN, "bad sizes");
  return mlp_backward_launch(x, ldx, n_points, W0, b0, W1, b1, d_colors, colors, d_hash, d_normal, dW0, db0, dW1, db1,
                             partials, n_partial_floats, (cudaStream_t)stream, RowSrc{nullptr, 0},
                             "radiance_mlp_backward");
}

int vx_appearance_mlp_backward(const float* rows, const float* rays_d, int n_samples, int64_t n_points,
                               const float* W0, const float* b0, const float* W1, const float* b1,
                               const float* d_colors, const float* colors, float* d_hash, float* d_normal, float* dW0,
                               float* db0, float* dW1, float* db1, float* partials, int64_t n_partial_floats,
                               void* stream) {
  VX_REQUIRE(n_points >= 0 && n_samples >= 1, "bad sizes");
  VX_REQUIRE(rays_d && rows, "null pointer");
  VX_REQUIRE(((uintptr_t)rows & 15) == 0, "compact rows must be 16-byte aligned");
  VX_REQUIRE(n_points < (int64_t(1) << 32), "compact rows take fewer than 2^32 samples");
  return mlp_backward_launch(rows, KC, n_points, W0, b0, W1, b1, d_colors, colors, d_hash, d_normal, dW0, db0, dW1,
                             db1, partials, n_partial_floats, (cudaStream_t)stream, RowSrc{rays_d, n_samples},
                             "appearance_mlp_backward");
}

}  // extern "C"
