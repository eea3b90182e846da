// Adam updates of the training step.
//
//   reference formula (adam_upd_kernel.cu:40-82 of the reference extension, the GPU path of
//   SparseGridAdam, training/optimizer.py:32-116):
//       step_size = lr * sqrt(1 - b2^t) / (1 - b1^t);  p -= step_size * m / (sqrt(v) + eps)
//     masked: elements whose gradient is exactly 0 keep p, m and v.
//   torch formula (torch.optim.Adam, the network optimizer of training/optimizer.py:119-154, and
//   SparseGridAdam's vectorised torch path, optimizer.py:86-113, when masked):
//       p -= (lr / (1 - b1^t)) * m / (sqrt(v) / sqrt(1 - b2^t) + eps)
//     (the division by sqrt(1 - b2^t) is a multiplication by its reciprocal, formed on the host)
//   both with m = b1 m + (1 - b1) g, v = b2 v + (1 - b2) g^2.
//
// HBM-bound streaming: 16 bytes read and 12 written per element (4 read for a masked element
// whose gradient is 0). Each thread keeps two float4 chunks of every operand in flight (the
// loads of both are issued before either update), so one wave of resident blocks covers the
// HBM latency; a scalar loop takes the tail and any segment whose pointers are not 16-byte
// aligned. One launch updates up to kMaxSegs tensors, each with its own step size.
#include "common.cuh"

namespace vx {
namespace {

constexpr int kMaxSegs = 8;

struct AdamSeg {
  float* p;
  const float* g;
  float* m;
  float* v;
  int64_t n;
  float step_size;
  float inv_bc2_sqrt;  // 1 / sqrt(1 - b2^t), torch formula only
  int vec;         // all four pointers 16-byte aligned
  const float* dev;  // nullable: {step size, 1/sqrt(1 - b2^t), step size when *flag} read on the device
  const int* flag;   // nullable: selects dev[2] instead of dev[0] when nonzero
};

struct AdamArgs {
  AdamSeg seg[kMaxSegs];
  int n_segs;
  float b1, b2, eps;
};

struct AdamScal {
  float step_size, inv_bc2_sqrt;
};

template <bool kMasked, bool kTorch>
__device__ __forceinline__ void adam1(float& p, float g, float& m, float& v, const AdamScal& s, const AdamArgs& a) {
  if (kMasked && g == 0.0f) return;
  m = a.b1 * m + (1.0f - a.b1) * g;
  v = a.b2 * v + (1.0f - a.b2) * g * g;
  if (kTorch)
    p -= s.step_size * m / (sqrtf(v) * s.inv_bc2_sqrt + a.eps);
  else
    p -= s.step_size * m / (sqrtf(v) + a.eps);
}

template <bool kMasked, bool kTorch>
__device__ __forceinline__ void adam4(float4& p, const float4& g, float4& m, float4& v, const AdamScal& s,
                                      const AdamArgs& a) {
  adam1<kMasked, kTorch>(p.x, g.x, m.x, v.x, s, a);
  adam1<kMasked, kTorch>(p.y, g.y, m.y, v.y, s, a);
  adam1<kMasked, kTorch>(p.z, g.z, m.z, v.z, s, a);
  adam1<kMasked, kTorch>(p.w, g.w, m.w, v.w, s, a);
}

__device__ __forceinline__ bool any_nonzero(const float4& g) {
  return g.x != 0.0f || g.y != 0.0f || g.z != 0.0f || g.w != 0.0f;
}

template <bool kMasked, bool kTorch>
__device__ __forceinline__ void adam_segment(const AdamSeg& s, const AdamArgs& a, int64_t tid, int64_t nt) {
  AdamScal sc{s.step_size, s.inv_bc2_sqrt};
  if (s.dev) {  // scalars of this step from device memory (a launch replayed from a CUDA graph)
    sc.step_size = (s.flag && *s.flag) ? s.dev[2] : s.dev[0];
    sc.inv_bc2_sqrt = s.dev[1];
  }
  int64_t done = 0;
  if (s.vec) {
    const int64_t n4 = s.n >> 2;
    float4* __restrict__ p4 = reinterpret_cast<float4*>(s.p);
    const float4* __restrict__ g4 = reinterpret_cast<const float4*>(s.g);
    float4* __restrict__ m4 = reinterpret_cast<float4*>(s.m);
    float4* __restrict__ v4 = reinterpret_cast<float4*>(s.v);
    for (int64_t i = tid; i < n4; i += 2 * nt) {
      const int64_t j = i + nt;
      const bool hj = j < n4;
      const float4 ga = __ldg(g4 + i);
      const float4 gb = hj ? __ldg(g4 + j) : make_float4(0.f, 0.f, 0.f, 0.f);
      const bool aa = !kMasked || any_nonzero(ga);
      const bool ab = hj && (!kMasked || any_nonzero(gb));
      float4 pa, ma, va, pb, mb, vb;
      if (aa) {
        pa = p4[i];
        ma = m4[i];
        va = v4[i];
      }
      if (ab) {
        pb = p4[j];
        mb = m4[j];
        vb = v4[j];
      }
      if (aa) {
        adam4<kMasked, kTorch>(pa, ga, ma, va, sc, a);
        p4[i] = pa;
        m4[i] = ma;
        v4[i] = va;
      }
      if (ab) {
        adam4<kMasked, kTorch>(pb, gb, mb, vb, sc, a);
        p4[j] = pb;
        m4[j] = mb;
        v4[j] = vb;
      }
    }
    done = n4 << 2;
  }
  for (int64_t i = done + tid; i < s.n; i += nt) {
    float p = s.p[i], m = s.m[i], v = s.v[i];
    const float g = __ldg(s.g + i);
    if (kMasked && g == 0.0f) continue;
    adam1<kMasked, kTorch>(p, g, m, v, sc, a);
    s.p[i] = p;
    s.m[i] = m;
    s.v[i] = v;
  }
}

template <bool kMasked, bool kTorch>
__global__ void __launch_bounds__(256) k_adam(const AdamArgs a) {
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nt = (int64_t)gridDim.x * blockDim.x;
#pragma unroll
  for (int si = 0; si < kMaxSegs; ++si)
    if (si < a.n_segs) adam_segment<kMasked, kTorch>(a.seg[si], a, tid, nt);
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

// One wave: as many blocks as stay resident on the 148 SMs (register-limited), queried once.
template <bool kMasked, bool kTorch>
unsigned adam_blocks(int64_t total) {
  static int per_sm = 0;
  if (per_sm == 0) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_adam<kMasked, kTorch>, 256, 0) != cudaSuccess || nb < 1)
      nb = 2;
    per_sm = nb;
  }
  return grid_for((total + 7) / 8, 256, per_sm);
}

int launch_adam(const AdamArgs& a, bool masked, bool torch_formula, int64_t total, cudaStream_t stream) {
  if (torch_formula && masked)
    k_adam<true, true><<<adam_blocks<true, true>(total), 256, 0, stream>>>(a);
  else if (torch_formula)
    k_adam<false, true><<<adam_blocks<false, true>(total), 256, 0, stream>>>(a);
  else if (masked)
    k_adam<true, false><<<adam_blocks<true, false>(total), 256, 0, stream>>>(a);
  else
    k_adam<false, false><<<adam_blocks<false, false>(total), 256, 0, stream>>>(a);
  count_launches(1);
  return check_launch(torch_formula ? (masked ? "masked_adam_torch" : "adam_torch")
                                    : (masked ? "masked_adam_upd" : "adam_upd"));
}

// The reference's step size, evaluated on the host in float (adam_upd_kernel.cu:50).
float reference_step_size(int step, float beta1, float beta2, float lr) {
  return lr * sqrtf(1.0f - powf(beta2, (float)step)) / (1.0f - powf(beta1, (float)step));
}

// torch.optim.Adam's per-step scalars, evaluated on the host in double.
void torch_step_scalars(int64_t step, float beta1, float beta2, float lr, float& step_size, float& inv_bc2_sqrt) {
  const double bc1 = 1.0 - pow((double)beta1, (double)step);
  const double bc2 = 1.0 - pow((double)beta2, (double)step);
  step_size = (float)((double)lr / bc1);
  inv_bc2_sqrt = (float)(1.0 / sqrt(bc2));
}

int adam_reference(bool masked, float* param, const float* grad, float* exp_avg, float* exp_avg_sq, int64_t n,
                   int step, float beta1, float beta2, float lr, float eps, void* stream,
                   const float* dev_step_size = nullptr) {
  VX_REQUIRE(n >= 0, "n < 0");
  VX_REQUIRE(dev_step_size || step >= 1, "step must be >= 1");
  if (n == 0) return VX_OK;
  VX_REQUIRE(param && grad && exp_avg && exp_avg_sq, "null pointer");
  AdamArgs a{};
  a.n_segs = 1;
  a.b1 = beta1;
  a.b2 = beta2;
  a.eps = eps;
  AdamSeg& s = a.seg[0];
  s.p = param;
  s.g = grad;
  s.m = exp_avg;
  s.v = exp_avg_sq;
  s.n = n;
  s.step_size = dev_step_size ? 0.0f : reference_step_size(step, beta1, beta2, lr);
  s.dev = dev_step_size;  // dev_step_size[1] is not read by the reference formula
  s.vec = aligned16(param) && aligned16(grad) && aligned16(exp_avg) && aligned16(exp_avg_sq);
  return launch_adam(a, masked, false, n, (cudaStream_t)stream);
}

}  // namespace
}  // namespace vx

using namespace vx;

extern "C" {

int vx_adam_upd(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, int64_t n, int step, float beta1,
                float beta2, float lr, float eps, void* stream) {
  return adam_reference(false, param, grad, exp_avg, exp_avg_sq, n, step, beta1, beta2, lr, eps, stream);
}

int vx_masked_adam_upd(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, int64_t n, int step,
                       float beta1, float beta2, float lr, float eps, void* stream) {
  return adam_reference(true, param, grad, exp_avg, exp_avg_sq, n, step, beta1, beta2, lr, eps, stream);
}

float vx_adam_reference_step_size(int step, float beta1, float beta2, float lr) {
  return reference_step_size(step, beta1, beta2, lr);
}

void vx_adam_torch_step_scalars(int64_t step, float beta1, float beta2, float lr, float out[2]) {
  torch_step_scalars(step, beta1, beta2, lr, out[0], out[1]);
}

int vx_masked_adam_upd_dev(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, int64_t n,
                           const float* step_size, float beta1, float beta2, float eps, void* stream) {
  VX_REQUIRE(step_size, "null step size");
  return adam_reference(true, param, grad, exp_avg, exp_avg_sq, n, 0, beta1, beta2, 0.0f, eps, stream, step_size);
}

}  // extern "C"

namespace vx {
namespace {

int adam_torch_segments(const vx_adam_segment* segs, int n_segs, float beta1, float beta2, float eps, bool masked,
                        void* stream) {
  VX_REQUIRE(n_segs >= 0, "n_segs < 0");
  if (n_segs == 0) return VX_OK;
  VX_REQUIRE(segs, "null pointer");
  for (int k = 0; k < n_segs; ++k) {  // validate everything before the first launch
    const vx_adam_segment& in = segs[k];
    VX_REQUIRE(in.n >= 0, "segment %d: n < 0", k);
    VX_REQUIRE(in.step_scalars || in.step >= 1, "segment %d: step must be >= 1", k);
    VX_REQUIRE(in.n == 0 || (in.param && in.grad && in.exp_avg && in.exp_avg_sq), "segment %d: null pointer", k);
  }
  for (int base = 0; base < n_segs; base += kMaxSegs) {
    AdamArgs a{};
    a.b1 = beta1;
    a.b2 = beta2;
    a.eps = eps;
    int64_t total = 0;
    for (int k = base; k < n_segs && k < base + kMaxSegs; ++k) {
      const vx_adam_segment& in = segs[k];
      if (in.n == 0) continue;
      AdamSeg& s = a.seg[a.n_segs++];
      s.p = in.param;
      s.g = in.grad;
      s.m = in.exp_avg;
      s.v = in.exp_avg_sq;
      s.n = in.n;
      if (in.step_scalars) {
        s.dev = in.step_scalars;
        s.flag = in.lr_flag;
      } else {
        torch_step_scalars(in.step, beta1, beta2, in.lr, s.step_size, s.inv_bc2_sqrt);
      }
      s.vec = aligned16(in.param) && aligned16(in.grad) && aligned16(in.exp_avg) && aligned16(in.exp_avg_sq);
      total += in.n;
    }
    if (a.n_segs == 0) continue;
    if (int st = launch_adam(a, masked, true, total, (cudaStream_t)stream)) return st;
  }
  return VX_OK;
}

}  // namespace
}  // namespace vx

extern "C" {

int vx_adam_torch(const vx_adam_segment* segs, int n_segs, float beta1, float beta2, float eps, void* stream) {
  return adam_torch_segments(segs, n_segs, beta1, beta2, eps, false, stream);
}

int vx_masked_adam_torch(const vx_adam_segment* segs, int n_segs, float beta1, float beta2, float eps, void* stream) {
  return adam_torch_segments(segs, n_segs, beta1, beta2, eps, true, stream);
}

}  // extern "C"
