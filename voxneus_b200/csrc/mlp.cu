// Radiance MLP [hash 32 | SH 16 | normal 3] -> 64 ReLU -> 3 Sigmoid (models/radiance_mlp.py:42-53,
// 81-98) as two fused FP32 kernels: the forward writes only the colours; the adjoint recomputes
// the hidden layer, writes dL/d(hash features) and dL/d(normal), and reduces the weight gradients
// into per-block partials that a second kernel sums in a fixed order (deterministic).
//
// Both kernels stage a 128-sample tile of input rows in shared memory and run the 51 -> 64 layer
// as a register-tiled SIMT GEMM: thread (lane, warp) owns samples 4*lane..4*lane+3 and hidden
// units 8*warp..8*warp+7, reading the inputs as 16-byte shared loads and the weights as
// warp-broadcast loads. FP32 throughout (the parity bar of the colours is 1e-5 relative).
#include "hashgrid.cuh"

namespace vx {

constexpr int KIN = 51;   // input features
constexpr int KP = 52;    // padded
constexpr int NH = 64;    // hidden units
constexpr int NO = 3;     // colours
constexpr int TM = 128;   // samples per tile
constexpr int DZS = TM;   // row stride of the transposed dL/dz tile
constexpr int XRS = KP;   // row stride of the row-major input tile (16-byte rows)
constexpr int WG = NH * KP + NO * NH + NH + NO;  // per-block weight-gradient partial size

struct MlpW {
  const float* W0;  // (64, 51)
  const float* b0;  // (64)
  const float* W1;  // (3, 64)
  const float* b1;  // (3)
};

__device__ __forceinline__ void load_weights(const MlpW& w, float (*W0T)[NH], float* B0, float (*W1s)[NH], float* B1,
                                             int tid, int nthreads) {
  for (int i = tid; i < KP * NH; i += nthreads) {
    const int k = i / NH, n = i % NH;
    W0T[k][n] = (k < KIN) ? w.W0[n * KIN + k] : 0.0f;
  }
  for (int i = tid; i < NH; i += nthreads) B0[i] = w.b0[i];
  for (int i = tid; i < NO * NH; i += nthreads) W1s[i / NH][i % NH] = w.W1[i];
  if (tid < NO) B1[tid] = w.b1[tid];
}

// hidden pre-activations z[s][j] for samples 4*tm+s, units 8*tn+j
__device__ __forceinline__ void layer0(const float (*XT)[TM], const float (*W0T)[NH], const float* B0, int tm, int tn,
                                       float z[4][8]) {
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int j = 0; j < 8; ++j) z[s][j] = B0[8 * tn + j];
#pragma unroll 4
  for (int k = 0; k < KIN; ++k) {
    const float4 a = *reinterpret_cast<const float4*>(&XT[k][4 * tm]);
    const float4 w0 = *reinterpret_cast<const float4*>(&W0T[k][8 * tn]);
    const float4 w1 = *reinterpret_cast<const float4*>(&W0T[k][8 * tn + 4]);
    const float av[4] = {a.x, a.y, a.z, a.w};
    const float wv[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int j = 0; j < 8; ++j) z[s][j] = fmaf(av[s], wv[j], z[s][j]);
  }
}

// Stage rows m0..m0+127 (row stride ldx) as XT[k][m].
__device__ __forceinline__ void load_tile(const float* __restrict__ X, int64_t ldx, int64_t P, int64_t m0,
                                          float (*XT)[TM], int tid) {
  if (tid < TM) {
    const int64_t m = m0 + tid;
    const bool ok = m < P;
    const float* row = X + m * ldx;
#pragma unroll 4
    for (int k = 0; k < KP; ++k) XT[k][tid] = (ok && k < KIN) ? __ldg(row + k) : 0.0f;
  }
}

__global__ void __launch_bounds__(256) k_mlp_fwd(const float* __restrict__ X, int64_t ldx, int64_t P, MlpW w,
                                                 float* __restrict__ out) {
  __shared__ __align__(16) float XT[KP][TM];
  __shared__ __align__(16) float W0T[KP][NH];
  __shared__ float B0[NH], W1s[NO][NH], B1[NO];
  const int tid = threadIdx.x, tm = tid & 31, tn = tid >> 5;
  load_weights(w, W0T, B0, W1s, B1, tid, blockDim.x);
  const int64_t ntiles = (P + TM - 1) / TM;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t m0 = t * TM;
    __syncthreads();
    load_tile(X, ldx, P, m0, XT, tid);
    __syncthreads();
    float z[4][8];
    layer0(XT, W0T, B0, tm, tn, z);
    float part[4][NO];
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < NO; ++c) {
        float acc = 0.0f;
#pragma unroll
        for (int j = 0; j < 8; ++j) acc = fmaf(W1s[c][8 * tn + j], fmaxf(z[s][j], 0.0f), acc);
        part[s][c] = acc;
      }
    __syncthreads();  // XT reads done: reuse it for the layer-1 partial sums
    float* red = &XT[0][0];
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < NO; ++c) red[(tn * TM + 4 * tm + s) * NO + c] = part[s][c];
    __syncthreads();
    if (tid < TM && m0 + tid < P) {
#pragma unroll
      for (int c = 0; c < NO; ++c) {
        float o = B1[c];
#pragma unroll
        for (int g = 0; g < 8; ++g) o += red[(g * TM + tid) * NO + c];
        out[(m0 + tid) * NO + c] = sigmoidf_ref(o);
      }
    }
  }
}

// Appearance + MLP forward for (rays, midpoints): the 51 input features of a 128-sample tile
// are built straight into the shared tile — two threads per sample, each gathering 8 hash
// levels (float2 corner features); SH of the view direction and the normal complete the row
// — then the MLP runs on the tile. kRows also writes the rows (the adjoint's input), as
// 16-byte stores of each thread's columns.
template <bool kRows>
__global__ void __launch_bounds__(256) k_appearance_mlp_fwd(HashArgs a, MlpW w, float* __restrict__ colors) {
  __shared__ __align__(16) float XT[KP][TM];
  __shared__ __align__(16) float W0T[KP][NH];
  __shared__ float B0[NH], W1s[NO][NH], B1[NO];
  const int tid = threadIdx.x, tm = tid & 31, tn = tid >> 5;
  load_weights(w, W0T, B0, W1s, B1, tid, blockDim.x);
  const uint32_t mask = (1u << a.log2T) - 1u;
  const size_t T = (size_t)1 << a.log2T;
  const int64_t ntiles = (a.P + TM - 1) / TM;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t m0 = t * TM;
    __syncthreads();
    {
      const int m = tid & (TM - 1), half = tid >> 7;
      const int64_t i = m0 + m;
      float feat[16];
      float extra[16];
      if (i < a.P) {
        float x[3];
        sample_pos(a, i, x);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int l = 8 * half + q;
          const float lw = a.lw[l];
          float f0 = 0.0f, f1 = 0.0f;
          if (lw != 0.0f) {
            LevelCell c;
            level_cell(x, a.res[l], mask, c);
            const float2* tab = reinterpret_cast<const float2*>(a.table) + (size_t)l * T;
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
          }
          feat[2 * q] = f0;
          feat[2 * q + 1] = f1;
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
        for (int q = 0; q < 16; ++q) feat[q] = extra[q] = 0.0f;
      }
#pragma unroll
      for (int q = 0; q < 16; ++q) XT[16 * half + q][m] = feat[q];
      if (half == 0) {
#pragma unroll
        for (int q = 0; q < 16; ++q) XT[32 + q][m] = extra[q];
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) XT[48 + q][m] = extra[q];
      }
      if (kRows && i < a.P) {
        float4* row = reinterpret_cast<float4*>(a.out + i * a.ld);
#pragma unroll
        for (int q = 0; q < 4; ++q)
          row[4 * half + q] = make_float4(feat[4 * q], feat[4 * q + 1], feat[4 * q + 2], feat[4 * q + 3]);
        if (half == 0) {
#pragma unroll
          for (int q = 0; q < 4; ++q)
            row[8 + q] = make_float4(extra[4 * q], extra[4 * q + 1], extra[4 * q + 2], extra[4 * q + 3]);
        } else {
          row[12] = make_float4(extra[0], extra[1], extra[2], extra[3]);
        }
      }
    }
    __syncthreads();
    float z[4][8];
    layer0(XT, W0T, B0, tm, tn, z);
    float part[4][NO];
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < NO; ++c) {
        float acc = 0.0f;
#pragma unroll
        for (int j = 0; j < 8; ++j) acc = fmaf(W1s[c][8 * tn + j], fmaxf(z[s][j], 0.0f), acc);
        part[s][c] = acc;
      }
    __syncthreads();
    float* red = &XT[0][0];
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < NO; ++c) red[(tn * TM + 4 * tm + s) * NO + c] = part[s][c];
    __syncthreads();
    if (tid < TM && m0 + tid < a.P) {
#pragma unroll
      for (int c = 0; c < NO; ++c) {
        float o = B1[c];
#pragma unroll
        for (int g = 0; g < 8; ++g) o += red[(g * TM + tid) * NO + c];
        colors[(m0 + tid) * NO + c] = sigmoidf_ref(o);
      }
    }
  }
}

// Stage rows m0..m0+127 of X as XR[m][0..51] with column 51 = 1 on real rows and whole rows of
// zeros past P (the ones column turns the dW0 reduction's last column into db0; W0T's row 51 is
// zero, so the column adds nothing to the hidden layer).
__device__ __forceinline__ void load_rows(const float* __restrict__ X, int64_t ldx, int64_t P, int64_t m0,
                                          float (*XR)[XRS], int tid, int nthreads) {
  const int64_t nrows = P - m0 < TM ? P - m0 : TM;
  if ((ldx & 3) == 0 && (reinterpret_cast<uintptr_t>(X) & 15) == 0) {
    for (int e = tid; e < TM * (KP / 4); e += nthreads) {
      const int m = e / (KP / 4), c = e - (KP / 4) * m;
      float4 v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      if (m < nrows) {
        v = __ldg(reinterpret_cast<const float4*>(X + (m0 + m) * ldx) + c);
        if (c == KP / 4 - 1) v.w = 1.0f;
      }
      *reinterpret_cast<float4*>(&XR[m][4 * c]) = v;
    }
  } else {
    for (int e = tid; e < TM * KP; e += nthreads) {
      const int m = e / KP, k = e - KP * m;
      XR[m][k] = m < nrows ? (k < KIN ? __ldg(X + (m0 + m) * ldx + k) : 1.0f) : 0.0f;
    }
  }
}

// Adjoint. d_out (P,3) -> d_hash (P,32), d_normal (P,3), per-block weight-gradient partials.
// Thread (lane, warp) owns samples lane + 32 s (s = 0..3), so row-major 16-byte tile reads are
// bank-conflict free (rows 208 bytes apart); dL/dz is staged as DZT[n][4 lane + s]. The weight
// gradient runs on 4x4 micro-tiles (threads 0..207: units 4*(t/13).., columns 4*(t%13)..).
__global__ void __launch_bounds__(256, 2) k_mlp_bwd(const float* __restrict__ X, int64_t ldx, int64_t P, MlpW w,
                                                 const float* __restrict__ d_out, float* __restrict__ d_hash,
                                                 float* __restrict__ d_normal, float* __restrict__ partials) {
  extern __shared__ __align__(16) float smem[];
  float(*XR)[XRS] = reinterpret_cast<float(*)[XRS]>(smem);                   // TM x XRS
  float(*DZT)[DZS] = reinterpret_cast<float(*)[DZS]>(smem + TM * XRS);       // NH x DZS
  float(*W0T)[NH] = reinterpret_cast<float(*)[NH]>(smem + TM * XRS + NH * DZS);
  float* B0 = smem + TM * XRS + NH * DZS + KP * NH;
  float(*W1s)[NH] = reinterpret_cast<float(*)[NH]>(B0 + NH);
  float* B1 = B0 + NH + NO * NH;
  float(*DO)[NO] = reinterpret_cast<float(*)[NO]>(B1 + 4);
  const int tid = threadIdx.x, tm = tid & 31, tn = tid >> 5;
  load_weights(w, W0T, B0, W1s, B1, tid, blockDim.x);
  const bool wtile = tid < 16 * (KP / 4);
  const int n4 = tid / (KP / 4), k4 = tid - (KP / 4) * n4;
  float gW0[4][4];  // units 4*n4+j, columns 4*k4+i (column 51 accumulates db0)
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int i = 0; i < 4; ++i) gW0[j][i] = 0.0f;
  float gW1[NO][8], gB1[NO];
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int c = 0; c < NO; ++c) gW1[c][j] = 0.0f;
#pragma unroll
  for (int c = 0; c < NO; ++c) gB1[c] = 0.0f;
  const int64_t ntiles = (P + TM - 1) / TM;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int64_t m0 = t * TM;
    __syncthreads();
    load_rows(X, ldx, P, m0, XR, tid, blockDim.x);
    if (tid < TM) {
#pragma unroll
      for (int c = 0; c < NO; ++c) DO[tid][c] = (m0 + tid < P) ? d_out[(m0 + tid) * NO + c] : 0.0f;
    }
    __syncthreads();
    // hidden pre-activations, k in the same order as the forward kernels (bit-identical z)
    float z[4][8];
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int j = 0; j < 8; ++j) z[s][j] = B0[8 * tn + j];
#pragma unroll 1
    for (int k = 0; k < KP; k += 4) {
      float4 xa[4];
#pragma unroll
      for (int s = 0; s < 4; ++s) xa[s] = *reinterpret_cast<const float4*>(&XR[tm + 32 * s][k]);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const float4 w0 = *reinterpret_cast<const float4*>(&W0T[k + i][8 * tn]);
        const float4 w1 = *reinterpret_cast<const float4*>(&W0T[k + i][8 * tn + 4]);
        const float wv[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          const float xv = i == 0 ? xa[s].x : (i == 1 ? xa[s].y : (i == 2 ? xa[s].z : xa[s].w));
#pragma unroll
          for (int j = 0; j < 8; ++j) z[s][j] = fmaf(xv, wv[j], z[s][j]);
        }
      }
    }
    // recompute the colours for the sigmoid adjoint
    float* red = &DZT[0][0];
#pragma unroll
    for (int s = 0; s < 4; ++s)
#pragma unroll
      for (int c = 0; c < NO; ++c) {
        float acc = 0.0f;
#pragma unroll
        for (int j = 0; j < 8; ++j) acc = fmaf(W1s[c][8 * tn + j], fmaxf(z[s][j], 0.0f), acc);
        red[(tn * TM + tm + 32 * s) * NO + c] = acc;
      }
    __syncthreads();
    if (tid < TM) {
#pragma unroll
      for (int c = 0; c < NO; ++c) {
        float o = B1[c];
#pragma unroll
        for (int g = 0; g < 8; ++g) o += red[(g * TM + tid) * NO + c];
        const float y = sigmoidf_ref(o);
        DO[tid][c] = DO[tid][c] * ((1.0f - y) * y);  // dL/d(pre-sigmoid)
      }
    }
    __syncthreads();
    // dL/dh, ReLU adjoint and layer-1 weight gradients; dL/dz staged as DZT[n][4 lane + s]
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int m = tm + 32 * s;
      const float d0 = DO[m][0], d1 = DO[m][1], d2 = DO[m][2];
      if (tn == 0) {
        gB1[0] += d0;
        gB1[1] += d1;
        gB1[2] += d2;
      }
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int n = 8 * tn + j;
        const float h = fmaxf(z[s][j], 0.0f);
        gW1[0][j] = fmaf(d0, h, gW1[0][j]);
        gW1[1][j] = fmaf(d1, h, gW1[1][j]);
        gW1[2][j] = fmaf(d2, h, gW1[2][j]);
        const float dh = d0 * W1s[0][n] + d1 * W1s[1][n] + d2 * W1s[2][n];
        z[s][j] = (h > 0.0f) ? dh : 0.0f;
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
      *reinterpret_cast<float4*>(&DZT[8 * tn + j][4 * tm]) = make_float4(z[0][j], z[1][j], z[2][j], z[3][j]);
    __syncthreads();
    // dW0[n][k] += sum_m dz[m][n] x[m][k]; slot p of DZT holds sample (p >> 2) + 32 (p & 3)
    if (wtile) {
#pragma unroll 2
      for (int p = 0; p < TM; p += 4) {
        float4 d[4], x[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) d[j] = *reinterpret_cast<const float4*>(&DZT[4 * n4 + j][p]);
#pragma unroll
        for (int q = 0; q < 4; ++q) x[q] = *reinterpret_cast<const float4*>(&XR[(p >> 2) + 32 * q][4 * k4]);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float xv[4] = {x[q].x, x[q].y, x[q].z, x[q].w};
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const float dv = q == 0 ? d[j].x : (q == 1 ? d[j].y : (q == 2 ? d[j].z : d[j].w));
#pragma unroll
            for (int i = 0; i < 4; ++i) gW0[j][i] = fmaf(dv, xv[i], gW0[j][i]);
          }
        }
      }
    }
    // dX[m][k] = sum_n dz[m][n] W0[n][k]: hash columns 4*warp..+3, normal column 48+warp (warps 0..2)
    float dx[4][4], dn[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      dn[s] = 0.0f;
#pragma unroll
      for (int i = 0; i < 4; ++i) dx[s][i] = 0.0f;
    }
#pragma unroll 1
    for (int n = 0; n < NH; n += 4) {
      float4 wq[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) wq[i] = *reinterpret_cast<const float4*>(&W0T[4 * tn + i][n]);
      const float4 wn = tn < 3 ? *reinterpret_cast<const float4*>(&W0T[48 + tn][n]) : make_float4(0, 0, 0, 0);
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const float4 d = *reinterpret_cast<const float4*>(&DZT[n + jj][4 * tm]);
        const float dv[4] = {d.x, d.y, d.z, d.w};
        const float wnj = jj == 0 ? wn.x : (jj == 1 ? wn.y : (jj == 2 ? wn.z : wn.w));
#pragma unroll
        for (int s = 0; s < 4; ++s) {
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const float wv = jj == 0 ? wq[i].x : (jj == 1 ? wq[i].y : (jj == 2 ? wq[i].z : wq[i].w));
            dx[s][i] = fmaf(dv[s], wv, dx[s][i]);
          }
          dn[s] = fmaf(dv[s], wnj, dn[s]);
        }
      }
    }
    __syncthreads();  // XR reads (dW0) done: stage dX rows in XR
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      *reinterpret_cast<float4*>(&XR[tm + 32 * s][4 * tn]) = make_float4(dx[s][0], dx[s][1], dx[s][2], dx[s][3]);
      if (tn < 3) XR[tm + 32 * s][32 + tn] = dn[s];
    }
    __syncthreads();
    for (int e = tid; e < TM * 8; e += blockDim.x) {
      const int m = e >> 3, c = e & 7;
      if (m0 + m < P)
        reinterpret_cast<float4*>(d_hash + (m0 + m) * 32)[c] = *reinterpret_cast<const float4*>(&XR[m][4 * c]);
    }
    for (int e = tid; e < TM * 3; e += blockDim.x) {
      const int m = e / 3, c = e % 3;
      if (m0 + m < P) d_normal[(m0 + m) * 3 + c] = XR[m][32 + c];
    }
  }
  // per-block weight-gradient partials: [dW0 (64 x 52) | dW1 (3 x 64) | db0 (64) | db1 (3)]
  float* pb = partials + (int64_t)blockIdx.x * WG;
  if (wtile) {
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = 4 * n4 + j;
#pragma unroll
      for (int i = 0; i < 4; ++i) pb[n * KP + 4 * k4 + i] = gW0[j][i];
      if (k4 == KP / 4 - 1) pb[NH * KP + NO * NH + n] = gW0[j][3];
    }
  }
#pragma unroll
  for (int j = 0; j < 8; ++j)
#pragma unroll
    for (int c = 0; c < NO; ++c) gW1[c][j] = warp_sum(gW1[c][j]);
#pragma unroll
  for (int c = 0; c < NO; ++c) gB1[c] = warp_sum(gB1[c]);
  if (tm == 0) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int n = 8 * tn + j;
#pragma unroll
      for (int c = 0; c < NO; ++c) pb[NH * KP + c * NH + n] = gW1[c][j];
    }
    if (tn == 0) {
#pragma unroll
      for (int c = 0; c < NO; ++c) pb[NH * KP + NO * NH + NH + c] = gB1[c];
    }
  }
}

// Sum the per-block partials in block order into dW0 (64,51), dW1 (3,64), db0 (64), db1 (3).
__global__ void k_mlp_wgrad_reduce(const float* __restrict__ partials, int nblocks, float* __restrict__ dW0,
                                   float* __restrict__ db0, float* __restrict__ dW1, float* __restrict__ db1) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < WG; e += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int b = 0; b < nblocks; ++b) acc += (double)partials[(int64_t)b * WG + e];
    const float v = (float)acc;
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
}

constexpr size_t kBwdSmem =
    sizeof(float) * (TM * XRS + NH * DZS + KP * NH + NH + NO * NH + 4 + TM * NO);

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
  VX_REQUIRE(!rows || (ld_rows >= KP && ld_rows % 4 == 0 && ((uintptr_t)rows & 15) == 0),
             "rows need a row stride >= 52 floats, a multiple of 4, and 16-byte alignment");
  fill_positions(a, nullptr, rays_o, rays_d, mid, n_samples, xyz_min, xyz_max);
  a.P = n_points;
  a.out = rows;
  a.ld = ld_rows;
  a.normals = normals;
  MlpW w{W0, b0, W1, b1};
  const int64_t tiles = (n_points + TM - 1) / TM;
  const unsigned blocks = (unsigned)(tiles < (int64_t)kSMs * 4 ? tiles : (int64_t)kSMs * 4);
  if (rows)
    k_appearance_mlp_fwd<true><<<blocks, 256, 0, (cudaStream_t)stream>>>(a, w, colors);
  else
    k_appearance_mlp_fwd<false><<<blocks, 256, 0, (cudaStream_t)stream>>>(a, w, colors);
  count_launches(1);
  return check_launch("appearance_mlp_forward");
}

int vx_mlp_blocks(int64_t n_points) {
  const int64_t tiles = (n_points + TM - 1) / TM;
  const int64_t cap = (int64_t)kSMs * 2;
  return (int)(tiles < 1 ? 1 : (tiles < cap ? tiles : cap));
}

int vx_mlp_partial_floats(void) { return WG; }

int vx_radiance_mlp_forward(const float* x, int64_t ldx, int64_t n_points, int in_dim, int hidden, int out_dim,
                            const float* W0, const float* b0, const float* W1, const float* b1, float* colors,
                            void* stream) {
  VX_REQUIRE(in_dim == KIN && hidden == NH && out_dim == NO, "the fused MLP is %d -> %d -> %d (got %d -> %d -> %d)",
             KIN, NH, NO, in_dim, hidden, out_dim);
  VX_REQUIRE(n_points >= 0 && ldx >= KIN, "bad sizes");
  if (n_points == 0) return VX_OK;
  VX_REQUIRE(x && W0 && b0 && W1 && b1 && colors, "null pointer");
  MlpW w{W0, b0, W1, b1};
  const int64_t tiles = (n_points + TM - 1) / TM;
  const unsigned blocks = (unsigned)(tiles < (int64_t)kSMs * 4 ? tiles : (int64_t)kSMs * 4);
  k_mlp_fwd<<<blocks, 256, 0, (cudaStream_t)stream>>>(x, ldx, n_points, w, colors);
  count_launches(1);
  return check_launch("radiance_mlp_forward");
}

int vx_radiance_mlp_backward(const float* x, int64_t ldx, int64_t n_points, int in_dim, int hidden, int out_dim,
                             const float* W0, const float* b0, const float* W1, const float* b1, const float* d_colors,
                             float* d_hash, float* d_normal, float* dW0, float* db0, float* dW1, float* db1,
                             float* partials, int64_t n_partial_floats, void* stream) {
  VX_REQUIRE(in_dim == KIN && hidden == NH && out_dim == NO, "the fused MLP is %d -> %d -> %d", KIN, NH, NO);
  VX_REQUIRE(n_points >= 0 && ldx >= KIN, "bad sizes");
  VX_REQUIRE(x && W0 && b0 && W1 && b1 && d_colors && d_hash && d_normal && dW0 && db0 && dW1 && db1 && partials,
             "null pointer");
  VX_REQUIRE((reinterpret_cast<uintptr_t>(d_hash) & 15) == 0, "d_hash must be 16-byte aligned");
  const int nb = vx_mlp_blocks(n_points);
  VX_REQUIRE(n_partial_floats >= (int64_t)nb * WG, "partials buffer holds %lld floats, need %lld",
             (long long)n_partial_floats, (long long)nb * WG);
  MlpW w{W0, b0, W1, b1};
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaFuncSetAttribute(k_mlp_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBwdSmem);
  if (e != cudaSuccess) return set_error(VX_ERR_CUDA, "radiance_mlp_backward: %s", cudaGetErrorString(e));
  if (n_points > 0) {
    k_mlp_bwd<<<nb, 256, kBwdSmem, st>>>(x, ldx, n_points, w, d_colors, d_hash, d_normal, partials);
  } else {
    cudaMemsetAsync(partials, 0, sizeof(float) * WG, st);
  }
  k_mlp_wgrad_reduce<<<(WG + 255) / 256, 256, 0, st>>>(partials, n_points > 0 ? nb : 1, dW0, db0, dW1, db1);
  count_launches(2);
  return check_launch("radiance_mlp_backward");
}

}  // extern "C"
