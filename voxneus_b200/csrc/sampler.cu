// The NeuS multistep sampler (rendering/sampler.py:11-204) as one warp per ray.
//
// A warp owns a ray: its z values and SDF values live in shared memory (up to 256 per ray),
// every per-interval quantity is computed with lanes striding over the intervals, the
// transmittance product, the pdf normalisation and the CDF are warp-shuffle scans over
// 32-wide tiles, the inverse CDF is a binary search per new sample, and cat_z_vals'
// sort becomes a rank sort of the <= 32 new samples plus a merge of two sorted lists.
#include "common.cuh"

namespace vx {

// rendering/rays.py:102-128. Every product and sum rounded separately, in the order of the
// reference's float32 ops (torch.sum over the 3 components adds them left to right), so near
// and far are bit-identical to it (no fused multiply-adds).
__device__ __forceinline__ void near_far(float ox, float oy, float oz, float dx, float dy, float dz, float radius,
                                         float& nearv, float& farv) {
  const float a = __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
  const float b = __fmul_rn(2.0f, __fadd_rn(__fadd_rn(__fmul_rn(ox, dx), __fmul_rn(oy, dy)), __fmul_rn(oz, dz)));
  const float mid = __fdiv_rn(__fmul_rn(0.5f, -b), a);
  nearv = fmaxf(__fsub_rn(mid, radius), 0.05f);
  farv = fmaxf(__fadd_rn(mid, radius), __fadd_rn(nearv, 0.1f));
}

struct WarpArrays {
  float* z;    // current sorted z (n)
  float* f;    // SDF at z
  float* z2;   // merge target
  float* f2;
  float* cdf;  // per-interval scratch, then the CDF (n entries)
  float* w;    // interval weights
  float* nz;   // new samples (<= 32), sorted
  float* nf;
};

__device__ __forceinline__ bool inside_unit(float ox, float oy, float oz, float dx, float dy, float dz, float t) {
  const float x = ray_at(ox, dx, t), y = ray_at(oy, dy, t), z = ray_at(oz, dz, t);
  return sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z))) < 1.0f;
}

// sample_pdf (sampler.py:11-66) on the warp's bins A.z[0..n) with weights A.w[0..n-1).
// Lane j (< ns) ends holding its new sample in `out`; `u_ray` points at ns uniforms or is
// null (deterministic: u_det table). Returns the searchsorted index through idx_out.
__device__ void warp_sample_pdf(const WarpArrays& A, int n, int ns, const float* __restrict__ u_ray,
                                const float* __restrict__ u_det, float u_lane, int lane, float* out_vals,
                                int64_t* out_idx, float& my_new, int& my_idx) {
  const int nb = n - 1;  // number of weights
  // sums and scans accumulate in double and round once to float, like the reference's CPU
  // reductions (at::acc_type<float, false> is double)
  double part = 0.0;
  for (int i = lane; i < nb; i += 32) part += (double)(A.w[i] + 1e-5f);
  const float total = (float)warp_sum_d(part);
  // cdf[0] = 0, cdf[i+1] = sum_{j<=i} pdf_j
  double carry = 0.0;
  for (int base = 0; base < nb; base += 32) {
    const int i = base + lane;
    const float pdf = (i < nb) ? (A.w[i] + 1e-5f) / total : 0.0f;
    const double inc = warp_incl_sum_d((double)pdf, lane) + carry;
    if (i < nb) A.cdf[i + 1] = (float)inc;
    carry = __shfl_sync(0xffffffffu, inc, 31);
  }
  if (lane == 0) A.cdf[0] = 0.0f;
  __syncwarp();
  my_new = 0.0f;
  my_idx = 0;
  for (int j = lane; j < ns; j += 32) {
    const float u = j == lane ? u_lane : (u_ray ? u_ray[j] : u_det[j]);  // u_lane: this lane's, loaded early
    // searchsorted(cdf, u, right=True): number of entries <= u
    int lo = 0, hi = n;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (A.cdf[mid] <= u) lo = mid + 1; else hi = mid;
    }
    const int idx = lo;
    const int below = max(idx - 1, 0), above = min(idx, n - 1);
    const float c0 = A.cdf[below], c1 = A.cdf[above];
    const float b0 = A.z[below], b1 = A.z[above];
    float den = c1 - c0;
    if (den < 1e-5f) den = 1.0f;
    const float t = (u - c0) / den;
    const float v = __fadd_rn(b0, __fmul_rn(t, __fsub_rn(b1, b0)));
    if (out_vals) out_vals[j] = v;
    if (out_idx) out_idx[j] = idx;
    if (j == lane) {
      my_new = v;
      my_idx = idx;
    }
  }
}

// up_sample (sampler.py:243-292): interval weights into A.w, then the inverse CDF. Whole-warp
// chunks of 32 intervals: the inside-sphere test of z_{i+1} and the previous interval's cos come
// from the neighbouring lane (the same expressions on the same operands), and the occupancy
// factor 0.9 occ + 0.1 of each interval is looked up here, into A.z2, so that the serial scan
// below holds no global load.
__device__ void warp_upsample_weights(const WarpArrays& A, int n, float inv_s, float ox, float oy, float oz, float dx,
                                      float dy, float dz, const Occ& oc, int lane) {
  const int nb = n - 1;
  // alpha per interval (into A.w) and 1 - alpha + 1e-7 (into A.cdf)
  float cos_carry = 0.0f;  // cos of the interval before this chunk
  for (int base = 0; base < nb; base += 32) {
    const int i = base + lane;
    const bool valid = i < nb;
    const int ic = valid ? i : nb - 1;
    const float z0 = A.z[ic], z1 = A.z[ic + 1];
    const float f0 = A.f[ic], f1 = A.f[ic + 1];
    const bool in0 = inside_unit(ox, oy, oz, dx, dy, dz, z0);
    const bool in_next = __shfl_down_sync(0xffffffffu, in0, 1);
    const bool in1 = (lane == 31 || i >= nb - 1) ? inside_unit(ox, oy, oz, dx, dy, dz, z1) : in_next;
    const bool ins = in0 || in1;
    const float cosv = (f1 - f0) / (__fsub_rn(z1, z0) + 1e-5f);
    float prev = __shfl_up_sync(0xffffffffu, cosv, 1);
    if (lane == 0) prev = cos_carry;
    if (i == 0) prev = 0.0f;
    cos_carry = __shfl_sync(0xffffffffu, cosv, 31);
    float c = fminf(prev, cosv);
    c = fminf(fmaxf(c, -1e3f), 0.0f) * (ins ? 1.0f : 0.0f);
    const float fm = (f0 + f1) * 0.5f;
    const float dist = __fsub_rn(z1, z0);
    const float half = __fmul_rn(__fmul_rn(c, dist), 0.5f);
    const float e0 = __fsub_rn(fm, half), e1 = __fadd_rn(fm, half);
    const float c0 = sigmoidf_ref(e0 * inv_s), c1 = sigmoidf_ref(e1 * inv_s);
    const float alpha = __fadd_rn(__fsub_rn(c0, c1), 1e-5f) / __fadd_rn(c0, 1e-5f);
    if (valid) {
      A.w[i] = alpha;
      A.cdf[i] = __fadd_rn(__fsub_rn(1.0f, alpha), 1e-7f);
      if (oc.mask) {
        const float zm = (z0 + z1) * 0.5f;
        const float occ = occupied(oc, ray_at(ox, dx, zm), ray_at(oy, dy, zm), ray_at(oz, dz, zm)) ? 1.0f : 0.0f;
        A.z2[i] = __fadd_rn(__fmul_rn(occ, 0.90f), 0.10f);
      }
    }
  }
  __syncwarp();
  // exclusive product scan: T_i = prod_{j<i} (1 - alpha_j + 1e-7); w_i = alpha_i T_i
  double carry = 1.0;
  for (int base = 0; base < nb; base += 32) {
    const int i = base + lane;
    const double q = (i < nb) ? (double)A.cdf[i] : 1.0;
    const double inc = warp_incl_prod_d(q, lane);
    double exc = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0) exc = 1.0;
    exc *= carry;
    if (i < nb) {
      float w = A.w[i] * (float)exc;
      if (oc.mask) w = w * A.z2[i];
      A.w[i] = w;
    }
    carry *= __shfl_sync(0xffffffffu, inc, 31);
  }
  __syncwarp();
}

// Rank-sort the ns (<= 32) new samples held by lanes < ns into A.nz/A.nf (ascending).
__device__ __forceinline__ void warp_rank_sort_new(const WarpArrays& A, int ns, float v, float fv, int lane) {
  int rank = 0;
#pragma unroll 8
  for (int k = 0; k < ns; ++k) {
    const float o = __shfl_sync(0xffffffffu, v, k);
    if (lane < ns) rank += (o < v) || (o == v && k < lane);
  }
  if (lane < ns) {
    A.nz[rank] = v;
    A.nf[rank] = fv;
  }
  __syncwarp();
}

// Merge sorted A.z (n) with sorted A.nz (ns) into A.z2/A.f2 (ties: old first).
__device__ __forceinline__ void warp_merge(const WarpArrays& A, int n, int ns, int lane) {
  for (int i = lane; i < n; i += 32) {
    const float zi = A.z[i];
    int c = 0;
    for (int k = 0; k < ns; ++k) c += (A.nz[k] < zi);
    A.z2[i + c] = zi;
    A.f2[i + c] = A.f[i];
  }
  if (lane < ns) {
    const float v = A.nz[lane];
    int lo = 0, hi = n;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (A.z[mid] <= v) lo = mid + 1; else hi = mid;
    }
    A.z2[lane + lo] = v;
    A.f2[lane + lo] = A.nf[lane];
  }
  __syncwarp();
}

struct SamplerArgs {
  const float* rays_o;
  const float* rays_d;
  const float* near;  // nullable: computed from the unit sphere
  const float* far;
  int64_t n_rays;
  int n_samples, n_importance, steps, per_step, n_total;
  int perturb;
  const float* t_lin;   // linspace(0, 1, n_samples)
  const float* t_rand;  // (n_rays, n_samples) or null
  const float* u;       // (steps, n_rays, per_step) or null
  const float* u_det;   // linspace(0.5/per, 1-0.5/per, per)
  float radius;
  float* z_out;  // nullable
  float* dists;
  float* mid;
};

__global__ void __launch_bounds__(128, 9) k_sample_multistep(SamplerArgs a, const float* __restrict__ fgrid, Grid g, Occ oc) {
  extern __shared__ float smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int NT = a.n_total;
  float* base = smem + warp * (6 * NT + 64);
  WarpArrays A{base, base + NT, base + 2 * NT, base + 3 * NT, base + 4 * NT, base + 5 * NT, base + 6 * NT,
               base + 6 * NT + 32};
  const int64_t wpb = blockDim.x >> 5;
  for (int64_t r = blockIdx.x * wpb + warp; r < a.n_rays; r += (int64_t)gridDim.x * wpb) {
    const float ox = a.rays_o[3 * r], oy = a.rays_o[3 * r + 1], oz = a.rays_o[3 * r + 2];
    const float dx = a.rays_d[3 * r], dy = a.rays_d[3 * r + 1], dz = a.rays_d[3 * r + 2];
    float nearv, farv;
    if (a.near) {
      nearv = a.near[r];
      farv = a.far[r];
    } else {
      near_far(ox, oy, oz, dx, dy, dz, a.radius, nearv, farv);
    }
    int n = a.n_samples;
    // S0: stratified samples (sampler.py:85-125)
    for (int i = lane; i < n; i += 32) {
      const float t = a.t_lin[i];
      A.z2[i] = __fadd_rn(__fmul_rn(nearv, __fsub_rn(1.0f, t)), __fmul_rn(farv, t));
    }
    __syncwarp();
    for (int i = lane; i < n; i += 32) {
      float zi = A.z2[i];
      if (a.perturb) {
        const float zl = A.z2[max(i - 1, 0)], zh = A.z2[min(i + 1, n - 1)];
        const float upper = (i < n - 1) ? __fmul_rn(__fadd_rn(zh, zi), 0.5f) : zi;
        const float lower = (i > 0) ? __fmul_rn(__fadd_rn(zi, zl), 0.5f) : zi;
        zi = __fadd_rn(lower, __fmul_rn(__fsub_rn(upper, lower), a.t_rand[r * a.n_samples + i]));
      }
      A.z[i] = zi;
    }
    __syncwarp();
    if (a.n_importance > 0 && a.steps > 0) {
#pragma unroll 2
      for (int i = lane; i < n; i += 32) {
        const float t = A.z[i];
        A.f[i] = query_sdf(fgrid, g, ray_at(ox, dx, t), ray_at(oy, dy, t), ray_at(oz, dz, t));
      }
      __syncwarp();
      for (int s = 0; s < a.steps; ++s) {
        const float inv_s = 64.0f * (float)(1 << s);
        const float* u_ray = a.u ? a.u + ((int64_t)s * a.n_rays + r) * a.per_step : nullptr;
        // this lane's uniform, loaded before the weights so its latency is hidden
        const float u_lane = lane < a.per_step ? (u_ray ? u_ray[lane] : a.u_det[lane]) : 0.0f;
        warp_upsample_weights(A, n, inv_s, ox, oy, oz, dx, dy, dz, oc, lane);
        float v;
        int idx;
        warp_sample_pdf(A, n, a.per_step, u_ray, a.u_det, u_lane, lane, nullptr, nullptr, v, idx);
        const bool last = (s + 1 == a.steps);
        float fv = 0.0f;
        if (!last && lane < a.per_step) fv = query_sdf(fgrid, g, ray_at(ox, dx, v), ray_at(oy, dy, v), ray_at(oz, dz, v));
        if (lane >= a.per_step) v = __int_as_float(0x7f800000);
        warp_rank_sort_new(A, a.per_step, v, fv, lane);
        warp_merge(A, n, a.per_step, lane);
        n += a.per_step;
        float* t0 = A.z;
        A.z = A.z2;
        A.z2 = t0;
        t0 = A.f;
        A.f = A.f2;
        A.f2 = t0;
      }
    }
    // S7 (sampler.py:197-202): dists with the last repeated, mid = z + dists/2
    for (int i = lane; i < n; i += 32) {
      const float zi = A.z[i];
      float di;
      if (n == 1) di = __fdiv_rn(__fsub_rn(farv, nearv), 1.0f);
      else if (i < n - 1) di = __fsub_rn(A.z[i + 1], zi);
      else di = __fsub_rn(zi, A.z[i - 1]);
      const int64_t o = r * n + i;
      if (a.z_out) a.z_out[o] = zi;
      a.dists[o] = di;
      a.mid[o] = __fadd_rn(zi, __fmul_rn(di, 0.5f));
    }
    __syncwarp();
  }
}

// One up_sample step on caller-provided z / sdf (the up_sample module function).
__global__ void __launch_bounds__(128) k_up_sample(const float* __restrict__ rays_o, const float* __restrict__ rays_d,
                                                   const float* __restrict__ z_in, const float* __restrict__ sdf_in,
                                                   int64_t n_rays, int n, int ns, float inv_s,
                                                   const float* __restrict__ u, const float* __restrict__ u_det, Occ oc,
                                                   float* __restrict__ out) {
  extern __shared__ float smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  float* base = smem + warp * (5 * n + 2);
  // z, f, z2 (the intervals' occupancy factors), cdf, w
  WarpArrays A{base, base + n, base + 4 * n + 2, nullptr, base + 2 * n, base + 3 * n, nullptr, nullptr};
  const int64_t wpb = blockDim.x >> 5;
  for (int64_t r = blockIdx.x * wpb + warp; r < n_rays; r += (int64_t)gridDim.x * wpb) {
    const float ox = rays_o[3 * r], oy = rays_o[3 * r + 1], oz = rays_o[3 * r + 2];
    const float dx = rays_d[3 * r], dy = rays_d[3 * r + 1], dz = rays_d[3 * r + 2];
    for (int i = lane; i < n; i += 32) {
      A.z[i] = z_in[r * n + i];
      A.f[i] = sdf_in[r * n + i];
    }
    __syncwarp();
    warp_upsample_weights(A, n, inv_s, ox, oy, oz, dx, dy, dz, oc, lane);
    float v;
    int idx;
    const float u_lane = lane < ns ? (u ? u[r * ns + lane] : u_det[lane]) : 0.0f;
    warp_sample_pdf(A, n, ns, u ? u + r * ns : nullptr, u_det, u_lane, lane, out + r * ns, nullptr, v, idx);
    __syncwarp();
  }
}

// sample_pdf / inverse CDF as a module function. With cdf_in given, the CDF is not rebuilt
// (the caller feeds an identical CDF to compare searchsorted indices bit for bit).
__global__ void __launch_bounds__(128) k_sample_pdf(const float* __restrict__ bins, const float* __restrict__ weights,
                                                    const float* __restrict__ cdf_in, int64_t n_rays, int n, int ns,
                                                    const float* __restrict__ u, const float* __restrict__ u_det,
                                                    float* __restrict__ out, int64_t* __restrict__ idx_out) {
  extern __shared__ float smem[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  float* base = smem + warp * (3 * n + 2);
  WarpArrays A{base, nullptr, nullptr, nullptr, base + n, base + 2 * n, nullptr, nullptr};
  const int64_t wpb = blockDim.x >> 5;
  for (int64_t r = blockIdx.x * wpb + warp; r < n_rays; r += (int64_t)gridDim.x * wpb) {
    for (int i = lane; i < n; i += 32) {
      A.z[i] = bins[r * n + i];
      if (i < n - 1 && weights) A.w[i] = weights[r * (n - 1) + i];
    }
    __syncwarp();
    float v;
    int idx;
    if (cdf_in) {
      for (int i = lane; i < n; i += 32) A.cdf[i] = cdf_in[r * n + i];
      __syncwarp();
      for (int j = lane; j < ns; j += 32) {
        const float uu = u ? u[r * ns + j] : u_det[j];
        int lo = 0, hi = n;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (A.cdf[mid] <= uu) lo = mid + 1; else hi = mid;
        }
        const int below = max(lo - 1, 0), above = min(lo, n - 1);
        const float c0 = A.cdf[below], c1 = A.cdf[above];
        float den = c1 - c0;
        if (den < 1e-5f) den = 1.0f;
        const float t = (uu - c0) / den;
        out[r * ns + j] = __fadd_rn(A.z[below], __fmul_rn(t, __fsub_rn(A.z[above], A.z[below])));
        if (idx_out) idx_out[r * ns + j] = lo;
      }
    } else {
      const float u_lane = lane < ns ? (u ? u[r * ns + lane] : u_det[lane]) : 0.0f;
      warp_sample_pdf(A, n, ns, u ? u + r * ns : nullptr, u_det, u_lane, lane, out + r * ns,
                      idx_out ? idx_out + r * ns : nullptr,
                      v, idx);
    }
    __syncwarp();
  }
}

__global__ void k_near_far(const float* __restrict__ o, const float* __restrict__ d, int64_t n, float radius,
                           float* __restrict__ nearv, float* __restrict__ farv) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    float a, b;
    near_far(o[3 * i], o[3 * i + 1], o[3 * i + 2], d[3 * i], d[3 * i + 1], d[3 * i + 2], radius, a, b);
    nearv[i] = a;
    farv[i] = b;
  }
}

// Total order of torch.sort on floats: ascending, -0 equal to +0, NaN after everything.
__device__ __forceinline__ uint32_t sort_key(float v) {
  if (v != v) return 0xffffffffu;
  const uint32_t u = __float_as_uint(v == 0.0f ? 0.0f : v);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// cat_z_vals (rendering/sampler.py:295-320): the ray's old and new depths concatenated and put in
// ascending order, the SDF values carried along. One block per ray (grid-stride over rays): the
// keys are staged in shared memory and every element finds its place by counting the smaller
// keys, equal keys ranked by position in the concatenation (so a depth present in both lists keeps
// the old value first; equal depths carry equal SDF values). Unsorted new depths are fine.
__global__ void __launch_bounds__(128) k_cat_z_vals(const float* __restrict__ z_old, const float* __restrict__ z_new,
                                                    const float* __restrict__ sdf_old,
                                                    const float* __restrict__ sdf_new, int64_t n_rays, int n_old,
                                                    int n_new, float* __restrict__ z_out, float* __restrict__ sdf_out) {
  extern __shared__ uint32_t keys[];
  const int n = n_old + n_new;
  for (int64_t r = blockIdx.x; r < n_rays; r += gridDim.x) {
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      keys[i] = sort_key(i < n_old ? z_old[r * n_old + i] : z_new[r * n_new + (i - n_old)]);
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const uint32_t k = keys[i];
      int rank = 0;
      for (int j = 0; j < n; ++j) {
        const uint32_t kj = keys[j];
        rank += (kj < k) || (kj == k && j < i);
      }
      const bool old = i < n_old;
      z_out[r * n + rank] = old ? z_old[r * n_old + i] : z_new[r * n_new + (i - n_old)];
      if (sdf_out) sdf_out[r * n + rank] = old ? sdf_old[r * n_old + i] : sdf_new[r * n_new + (i - n_old)];
    }
    __syncthreads();
  }
}

}  // namespace vx

using namespace vx;

extern "C" {

int vx_near_far_from_sphere(const float* rays_o, const float* rays_d, int64_t n, float radius, float* near_out,
                            float* far_out, void* stream) {
  VX_REQUIRE(n >= 0, "n < 0");
  if (n == 0) return VX_OK;
  VX_REQUIRE(rays_o && rays_d && near_out && far_out, "null pointer");
  k_near_far<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(rays_o, rays_d, n, radius, near_out, far_out);
  count_launches(1);
  return check_launch("near_far_from_sphere");
}

int vx_sample_multistep(const float* grid, const int32_t res[3], const float xyz_min[3], const float xyz_max[3],
                        const float* rays_o, const float* rays_d, const float* near_in, const float* far_in,
                        int64_t n_rays, int n_samples, int n_importance, int up_sample_steps, int perturb,
                        const float* t_lin, const float* t_rand, const float* u, const float* u_det,
                        const uint8_t* occupancy, int occ_res, const float occ_min[3], const float occ_max[3],
                        float* z_out, float* dists_out, float* mid_out, void* stream) {
  VX_REQUIRE(res && res[0] >= 2 && res[1] >= 2 && res[2] >= 2, "grid resolution must be >= 2 per axis");
  VX_REQUIRE(n_rays >= 0, "n_rays < 0");
  VX_REQUIRE(n_samples >= 2, "n_samples must be >= 2");
  VX_REQUIRE(n_importance >= 0 && up_sample_steps >= 0, "negative importance count");
  const int per = (n_importance > 0 && up_sample_steps > 0) ? (n_importance / up_sample_steps > 1 ? n_importance / up_sample_steps : 1) : 0;
  VX_REQUIRE(per <= 32, "samples per upsampling step must be <= 32 (got %d)", per);
  const int total = n_samples + per * up_sample_steps;
  VX_REQUIRE(total <= 256, "total samples per ray must be <= 256 (got %d)", total);
  if (n_rays == 0) return VX_OK;
  VX_REQUIRE(grid && rays_o && rays_d && t_lin && dists_out && mid_out && xyz_min && xyz_max, "null pointer");
  VX_REQUIRE(!perturb || t_rand, "perturb requires t_rand");
  VX_REQUIRE(per == 0 || perturb || u_det, "deterministic upsampling requires u_det");
  VX_REQUIRE(per == 0 || !perturb || u, "perturbed upsampling requires u");
  VX_REQUIRE((near_in == nullptr) == (far_in == nullptr), "near and far must both be given or both null");
  VX_REQUIRE(!occupancy || (occ_res > 0 && occ_min && occ_max), "occupancy mask needs its resolution and bounds");
  SamplerArgs a{rays_o, rays_d, near_in, far_in, n_rays, n_samples, n_importance, up_sample_steps, per, total,
                perturb, t_lin, perturb ? t_rand : nullptr, perturb ? u : nullptr, u_det, 1.0f, z_out, dists_out,
                mid_out};
  Grid g = make_grid(res, xyz_min, xyz_max);
  Occ oc = make_occ(occupancy, occ_res, occ_min, occ_max);
  const int threads = 128;
  const size_t smem = (size_t)(threads / 32) * (6 * total + 64) * sizeof(float);
  // a warp per ray up to 64 blocks a SM (9 are resident): one wave of persistent warps left some
  // warps two rays and others one; the block scheduler balances single-ray warps better
  k_sample_multistep<<<grid_for(n_rays * 32, threads, 64), threads, smem, (cudaStream_t)stream>>>(a, grid, g, oc);
  count_launches(1);
  return check_launch("sample_multistep");
}

int vx_up_sample(const float* rays_o, const float* rays_d, const float* z, const float* sdf, int64_t n_rays, int n,
                 int n_importance, float inv_s, const float* u, const float* u_det, const uint8_t* occupancy,
                 int occ_res, const float occ_min[3], const float occ_max[3], float* out, void* stream) {
  VX_REQUIRE(n_rays >= 0 && n >= 2 && n <= 4096, "need 2 <= n <= 4096 samples per ray");
  VX_REQUIRE(n_importance >= 1 && n_importance <= 4096, "n_importance out of range");
  if (n_rays == 0) return VX_OK;
  VX_REQUIRE(rays_o && rays_d && z && sdf && out, "null pointer");
  VX_REQUIRE(u || u_det, "need u or u_det");
  VX_REQUIRE(!occupancy || (occ_res > 0 && occ_min && occ_max), "occupancy mask needs its resolution and bounds");
  Occ oc = make_occ(occupancy, occ_res, occ_min, occ_max);
  const int threads = 128;
  const size_t smem = (size_t)(threads / 32) * (5 * n + 2) * sizeof(float);
  VX_REQUIRE(smem <= 200 * 1024, "too many samples per ray for one block");
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_up_sample, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_up_sample<<<grid_for(n_rays * 32, threads, 8), threads, smem, (cudaStream_t)stream>>>(
      rays_o, rays_d, z, sdf, n_rays, n, n_importance, inv_s, u, u_det, oc, out);
  count_launches(1);
  return check_launch("up_sample");
}

int vx_sample_pdf(const float* bins, const float* weights, const float* cdf, int64_t n_rays, int n_bins,
                  int n_samples, const float* u, const float* u_det, float* out, int64_t* idx_out, void* stream) {
  VX_REQUIRE(n_rays >= 0 && n_bins >= 2 && n_bins <= 4096, "need 2 <= n_bins <= 4096");
  VX_REQUIRE(n_samples >= 1, "n_samples must be >= 1");
  if (n_rays == 0) return VX_OK;
  VX_REQUIRE(bins && out && (weights || cdf), "null pointer");
  VX_REQUIRE(u || u_det, "need u or u_det");
  const int threads = 128;
  const size_t smem = (size_t)(threads / 32) * (3 * n_bins + 2) * sizeof(float);
  VX_REQUIRE(smem <= 200 * 1024, "too many bins per ray for one block");
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_sample_pdf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_sample_pdf<<<grid_for(n_rays * 32, threads, 8), threads, smem, (cudaStream_t)stream>>>(
      bins, weights, cdf, n_rays, n_bins, n_samples, u, u_det, out, idx_out);
  count_launches(1);
  return check_launch("sample_pdf");
}

int vx_cat_z_vals(const float* z_old, const float* z_new, const float* sdf_old, const float* sdf_new, int64_t n_rays,
                  int n_old, int n_new, float* z_out, float* sdf_out, void* stream) {
  VX_REQUIRE(n_rays >= 0 && n_old >= 0 && n_new >= 0, "bad sizes");
  VX_REQUIRE((int64_t)n_old + n_new <= 8192, "at most 8192 depths per ray");
  if (n_rays == 0 || n_old + n_new == 0) return VX_OK;
  VX_REQUIRE((z_old || n_old == 0) && (z_new || n_new == 0) && z_out, "null pointer");
  VX_REQUIRE(!sdf_out || ((sdf_old || n_old == 0) && (sdf_new || n_new == 0)),
             "carrying SDF values needs both lists' values");
  const size_t smem = (size_t)(n_old + n_new) * sizeof(uint32_t);
  k_cat_z_vals<<<grid_for(n_rays * 128, 128, 8), 128, smem, (cudaStream_t)stream>>>(z_old, z_new, sdf_old, sdf_new,
                                                                                   n_rays, n_old, n_new, z_out,
                                                                                   sdf_out);
  count_launches(1);
  return check_launch("cat_z_vals");
}

}  // extern "C"
