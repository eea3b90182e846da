// Per-sample geometry (positions, SDF, Eq.7 normals, V_R corner marks) and per-ray NeuS
// compositing (Eq.2 alpha, inside-sphere mask, transmittance scan, weights, rgb/depth/
// normal/opacity), each with its hand-written adjoint.
//
// Geometry: one thread per sample, samples of a ray in consecutive threads so a warp walks
// 32 consecutive samples of one ray through the L2-resident grid. The adjoint recomputes
// positions, corners and normals instead of storing them.
//
// Compositing: one warp per ray over 32-sample tiles; the exclusive transmittance product
// is a warp-shuffle scan with a carry between tiles, the adjoint's suffix sum is the
// reverse scan. dL/ds is reduced per block into caller-provided partials and the last
// block to finish converts it to dL/dvariance (and applies the k-amplification rule).
#include "common.cuh"

namespace vx {

// ------------------------------- geometry -------------------------------------------------

__global__ void __launch_bounds__(256, 4) k_geometry_fwd(const float* __restrict__ f, Grid g,
                                                      const float* __restrict__ rays_o,
                                                      const float* __restrict__ rays_d,
                                                      const float* __restrict__ mid, int64_t n, int S,
                                                      float* __restrict__ sdf, float* __restrict__ normal,
                                                      float* __restrict__ grad, uint32_t* __restrict__ bitmap) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / S;
    const float t = mid[i];
    const float px = ray_at(__ldg(rays_o + 3 * r), __ldg(rays_d + 3 * r), t);
    const float py = ray_at(__ldg(rays_o + 3 * r + 1), __ldg(rays_d + 3 * r + 1), t);
    const float pz = ray_at(__ldg(rays_o + 3 * r + 2), __ldg(rays_d + 3 * r + 2), t);
    Eq7 e;
    eq7_setup(g, px, py, pz, e);
    float c[8];  // the cell's corner values, shared by the SDF and the gradient
    eq7_load_block(f, g, e, c);
    if (sdf) sdf[i] = query_sdf_block(f, g, px, py, pz, e, c);
    float w[8], gr[3], nn[3], len;
    eq7_weights(e, w);
    eq7_gradient_block(f, g, e, w, c, gr);
    normalize_eps(gr, nn, len);
    normal[3 * i] = nn[0];
    normal[3 * i + 1] = nn[1];
    normal[3 * i + 2] = nn[2];
    if (grad) {
      grad[3 * i] = gr[0];
      grad[3 * i + 1] = gr[1];
      grad[3 * i + 2] = gr[2];
    }
    if (bitmap) mark_corners(bitmap, g, e);
  }
}

// d_normal2 (row stride ld2) is a second dL/dnormal source (the appearance branch input).
__global__ void __launch_bounds__(256, 3) k_geometry_bwd(const float* __restrict__ f, Grid g,
                                                      const float* __restrict__ rays_o,
                                                      const float* __restrict__ rays_d,
                                                      const float* __restrict__ mid, int64_t n, int S,
                                                      const float* __restrict__ d_sdf,
                                                      const float* __restrict__ d_normal,
                                                      const float* __restrict__ d_normal2, int64_t ld2,
                                                      const float* __restrict__ d_grad,
                                                      const float* __restrict__ g_fwd, float* __restrict__ gg) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / S;
    const float t = mid[i];
    const float px = ray_at(__ldg(rays_o + 3 * r), __ldg(rays_d + 3 * r), t);
    const float py = ray_at(__ldg(rays_o + 3 * r + 1), __ldg(rays_d + 3 * r + 1), t);
    const float pz = ray_at(__ldg(rays_o + 3 * r + 2), __ldg(rays_d + 3 * r + 2), t);
    const float ds = d_sdf ? d_sdf[i] : 0.0f;
    float dn[3] = {0.0f, 0.0f, 0.0f};
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
    float dg[3] = {0.0f, 0.0f, 0.0f};
    if (d_grad) {
      dg[0] = d_grad[3 * i];
      dg[1] = d_grad[3 * i + 1];
      dg[2] = d_grad[3 * i + 2];
    }
    const bool any_n = dn[0] != 0.0f || dn[1] != 0.0f || dn[2] != 0.0f;
    const bool any_g = dg[0] != 0.0f || dg[1] != 0.0f || dg[2] != 0.0f;
    if (!any_n && !any_g) {
      if (ds != 0.0f) {
        Tri tr;
        gs_setup(g, px, py, pz, tr);
        gs_scatter(gg, g, tr, ds);
      }
      continue;
    }
    Eq7 e;
    eq7_setup(g, px, py, pz, e);
    float w[8];
    eq7_weights(e, w);
    // dL/dsdf on the grid_sample corners: summed with the Eq.7 terms of the same corners when the
    // cell is the same one (interior points), else scattered on its own
    float acc[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    if (ds != 0.0f) {
      Tri tr;
      gs_setup(g, px, py, pz, tr);
      if (tr.inb == 0xffu && tr.x0 == e.x0 && tr.y0 == e.y0 && tr.z0 == e.z0) {
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] = tr.w[k] * ds;
      } else {
        gs_scatter(gg, g, tr, ds);
      }
    }
    if (any_n) {
      float gr[3], nn[3], len, dgn[3];
      if (g_fwd) {  // the forward's Eq.7 gradient: the same bits, without the 32 stencil loads
        gr[0] = g_fwd[3 * i];
        gr[1] = g_fwd[3 * i + 1];
        gr[2] = g_fwd[3 * i + 2];
      } else {
        eq7_gradient(f, g, e, w, gr);
      }
      normalize_eps(gr, nn, len);
      normalize_eps_bwd(gr, len, dn, dgn);
      dg[0] += dgn[0];
      dg[1] += dgn[1];
      dg[2] += dgn[2];
    }
    eq7_scatter_acc(gg, g, e, w, dg, acc);
  }
}

// ------------------------------- compositing ----------------------------------------------

struct CompArgs {
  const float* colors;   // (N,S,3)
  const float* sdf;      // (N,S)
  const float* normals;  // (N,S,3)
  const float* dirs;     // ray directions: element (r,i) at dirs + r*dir_rs + i*dir_ss
  int64_t dir_rs, dir_ss;
  const float* zv;       // (N,S) depth values (midpoints)
  const float* dists;    // (N,S)
  const float* pts;      // (N,S,3) or null
  const float* rays_o;   // used with dirs to rebuild positions when pts is null
  const float* s_ptr;    // variance (is_var) or s itself
  int s_is_var;
  float s_max;
  float radius;          // <= 0: no inside-sphere mask
  const float* bg;       // background or null
  int bg_per_ray;
  int iter_cos;
  float cos_anneal;
  int64_t N;
  int S;
};

__device__ __forceinline__ float get_s(const CompArgs& a) {
  const float v = __ldg(a.s_ptr);
  if (!a.s_is_var) return v;
  return fminf(fmaxf(expf(v * 10.0f), 1e-4f), a.s_max);
}

struct SampleFwd {
  float cos_t;  // <n, d>
  float cosv;   // after optional iter_cos
  float f0, f1, p0, p1, diff, den, ratio, a, mask, am;
};

__device__ __forceinline__ void alpha_fwd(const CompArgs& a, float s, int64_t r, int i, float sdfv, const float n[3],
                                          SampleFwd& o) {
  const float* d = a.dirs + r * a.dir_rs + (int64_t)i * a.dir_ss;
  o.cos_t = n[0] * d[0] + n[1] * d[1] + n[2] * d[2];
  float c = o.cos_t;
  if (a.iter_cos) {
    c = -(fmaxf(-o.cos_t * 0.5f + 0.5f, 0.0f) * (1.0f - a.cos_anneal) + fmaxf(-o.cos_t, 0.0f) * a.cos_anneal);
  }
  o.cosv = c;
  const float off = (0.5f * a.dists[r * a.S + i]) * c;
  o.f0 = sdfv - off;
  o.f1 = sdfv + off;
  o.p0 = sigmoidf_ref(s * o.f0);
  o.p1 = sigmoidf_ref(s * o.f1);
  o.diff = o.p0 - o.p1;
  o.den = fmaxf(o.p0, 1e-5f);
  o.ratio = o.diff / o.den;
  o.a = fminf(fmaxf(o.ratio, 0.0f), 1.0f);
  o.mask = 1.0f;
  if (a.radius > 0.0f) {
    float x, y, z;
    const int64_t k = r * a.S + i;
    if (a.pts) {
      x = a.pts[3 * k];
      y = a.pts[3 * k + 1];
      z = a.pts[3 * k + 2];
    } else {
      const float t = a.zv[k];
      const float* dd = a.dirs + r * a.dir_rs + (int64_t)i * a.dir_ss;
      x = ray_at(a.rays_o[3 * r], dd[0], t);
      y = ray_at(a.rays_o[3 * r + 1], dd[1], t);
      z = ray_at(a.rays_o[3 * r + 2], dd[2], t);
    }
    const float rr = sqrtf(__fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z)));
    o.mask = (rr < a.radius) ? 1.0f : 0.0f;
  }
  o.am = o.a * o.mask;
}

__global__ void __launch_bounds__(128) k_composite_fwd(CompArgs a, float* __restrict__ rgb, float* __restrict__ depth,
                                                       float* __restrict__ nout, float* __restrict__ opacity,
                                                       float* __restrict__ wout, float* __restrict__ aout,
                                                       float* __restrict__ tout) {
  const int lane = threadIdx.x & 31;
  const int64_t wpb = blockDim.x >> 5;
  const float s = get_s(a);
  for (int64_t r = blockIdx.x * wpb + (threadIdx.x >> 5); r < a.N; r += (int64_t)gridDim.x * wpb) {
    double carry = 1.0;  // double accumulation, rounded once (the CPU cumprod does the same)
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};  // rgb, depth, nsum, opacity
    for (int base = 0; base < a.S; base += 32) {
      const int i = base + lane;
      const bool valid = i < a.S;
      float q = 1.0f, am = 0.0f;
      float nrm[3] = {0.f, 0.f, 0.f};
      if (valid) {
        const int64_t k = r * a.S + i;
        nrm[0] = a.normals[3 * k];
        nrm[1] = a.normals[3 * k + 1];
        nrm[2] = a.normals[3 * k + 2];
        SampleFwd o;
        alpha_fwd(a, s, r, i, a.sdf[k], nrm, o);
        am = o.am;
        q = fminf(fmaxf(__fadd_rn(__fsub_rn(1.0f, am), 1e-7f), 0.0f), 1.0f);
      }
      const double inc = warp_incl_prod_d((double)q, lane);
      double Td = __shfl_up_sync(0xffffffffu, inc, 1);
      if (lane == 0) Td = 1.0;
      const float T = (float)(Td * carry);
      carry *= __shfl_sync(0xffffffffu, inc, 31);
      if (valid) {
        const int64_t k = r * a.S + i;
        float w = am * T;
        if (T < 1e-4f) w = 0.0f;
        if (wout) wout[k] = w;
        if (aout) aout[k] = am;
        if (tout) tout[k] = T;
        acc[0] = fmaf(w, a.colors[3 * k], acc[0]);
        acc[1] = fmaf(w, a.colors[3 * k + 1], acc[1]);
        acc[2] = fmaf(w, a.colors[3 * k + 2], acc[2]);
        acc[3] = fmaf(w, a.zv[k], acc[3]);
        acc[4] = fmaf(w, nrm[0], acc[4]);
        acc[5] = fmaf(w, nrm[1], acc[5]);
        acc[6] = fmaf(w, nrm[2], acc[6]);
        acc[7] += w;
      }
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] = warp_sum(acc[c]);
    if (lane == 0) {
      float cr = acc[0], cg = acc[1], cb = acc[2];
      if (a.bg) {
        const float* b = a.bg_per_ray ? a.bg + 3 * r : a.bg;
        const float om = 1.0f - acc[7];
        cr += om * b[0];
        cg += om * b[1];
        cb += om * b[2];
      }
      if (rgb) {
        rgb[3 * r] = cr;
        rgb[3 * r + 1] = cg;
        rgb[3 * r + 2] = cb;
      }
      if (depth) depth[r] = acc[3];
      if (nout) {
        const float l = norm3(acc[4], acc[5], acc[6]) + 1e-8f;
        nout[3 * r] = acc[4] / l;
        nout[3 * r + 1] = acc[5] / l;
        nout[3 * r + 2] = acc[6] / l;
      }
      if (opacity) opacity[r] = acc[7];
    }
  }
}

struct CompGrads {
  const float* g_rgb;      // (N,3)
  const float* g_depth;    // (N)
  const float* g_normal;   // (N,3)
  const float* g_opacity;  // (N)
  const float* g_weights;  // (N,S)
  const float* g_alpha;    // (N,S)
  const float* g_trans;    // (N,S)
  float* d_colors;         // (N,S,3)
  float* d_sdf;            // (N,S)
  float* d_normals;        // (N,S,3)
  double* partials;        // one per block
  unsigned int* counter;   // zero before the first launch; the last block resets it
  float* d_s_out;          // dL/ds (or dL/dvariance) scalar, written by the last block
  float amp_k;             // > 0: multiply a negative dL/dvariance by amp_k
  int* amp_flag;           // nullable: set to 1 when amplified, else 0
};

// Composite adjoint. Per ray: pass 1 recomputes alpha (kept in shared memory), T and the
// composited normal sum; pass 2 forms dL/dw and dT_j T_j; a reverse warp scan turns those
// into the suffix sums G_i = sum_{j>i} dT_j T_j (cumprod's adjoint, divided by q_i below);
// pass 3 back-propagates through the clamps, Eq.2 and the normal inner product.
// kKeep: pass 1 keeps each sample's alpha terms and pass 2 its dL/dw in shared memory (13 floats
// per sample and warp), so pass 3 reads them instead of recomputing the alpha (two sigmoids, the
// divisions, the sphere mask) and reloading colours, depths and normals; the same values, so the
// same results. Without it (very long rays) pass 3 recomputes them.
constexpr int kCompKeepFields = 13;  // T, alpha, G | dw, mask, ratio, den, diff, p0, p1, f0, f1, cos_t

template <bool kKeep>
__global__ void __launch_bounds__(128, 8) k_composite_bwd(CompArgs a, CompGrads gr) {
  extern __shared__ float sm[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int64_t wpb = blockDim.x >> 5;
  float* T_s = sm + warp * (kKeep ? kCompKeepFields : 3) * a.S;  // transmittance
  float* A_s = T_s + a.S;            // masked alpha
  float* G_s = A_s + a.S;            // dT_j T_j, then the suffix sums
  float* D_s = G_s + a.S;            // kKeep: dL/dw, then the alpha terms below
  float* K_s = D_s + a.S;            // kKeep: [mask, ratio, den, diff, p0, p1, f0, f1, cos_t][S]
  __shared__ double ds_warp[32];
  __shared__ bool is_last;
  const float s = get_s(a);
  double ds_acc = 0.0;
  for (int64_t r = blockIdx.x * wpb + warp; r < a.N; r += (int64_t)gridDim.x * wpb) {
    // pass 1: alpha, transmittance and the normal sum
    double carry = 1.0;  // double accumulation, rounded once (the CPU cumprod does the same)
    float ns[3] = {0.f, 0.f, 0.f};
    for (int base = 0; base < a.S; base += 32) {
      const int i = base + lane;
      float q = 1.0f, am = 0.0f, nrm[3] = {0.f, 0.f, 0.f};
      if (i < a.S) {
        const int64_t k = r * a.S + i;
        nrm[0] = a.normals[3 * k];
        nrm[1] = a.normals[3 * k + 1];
        nrm[2] = a.normals[3 * k + 2];
        SampleFwd o;
        alpha_fwd(a, s, r, i, a.sdf[k], nrm, o);
        am = o.am;
        q = fminf(fmaxf(__fadd_rn(__fsub_rn(1.0f, am), 1e-7f), 0.0f), 1.0f);
        if (kKeep) {
          K_s[i] = o.mask;
          K_s[a.S + i] = o.ratio;
          K_s[2 * a.S + i] = o.den;
          K_s[3 * a.S + i] = o.diff;
          K_s[4 * a.S + i] = o.p0;
          K_s[5 * a.S + i] = o.p1;
          K_s[6 * a.S + i] = o.f0;
          K_s[7 * a.S + i] = o.f1;
          K_s[8 * a.S + i] = o.cos_t;
        }
      }
      const double inc = warp_incl_prod_d((double)q, lane);
      double Td = __shfl_up_sync(0xffffffffu, inc, 1);
      if (lane == 0) Td = 1.0;
      const float T = (float)(Td * carry);
      carry *= __shfl_sync(0xffffffffu, inc, 31);
      if (i < a.S) {
        T_s[i] = T;
        A_s[i] = am;
        const float w = (T < 1e-4f) ? 0.0f : am * T;
        ns[0] = fmaf(w, nrm[0], ns[0]);
        ns[1] = fmaf(w, nrm[1], ns[1]);
        ns[2] = fmaf(w, nrm[2], ns[2]);
      }
    }
    // dL/d(normal sum) through normal = nsum / (|nsum| + 1e-8)
    float gN[3] = {0.f, 0.f, 0.f};
    if (gr.g_normal) {
      ns[0] = warp_sum(ns[0]);
      ns[1] = warp_sum(ns[1]);
      ns[2] = warp_sum(ns[2]);
      const float l = norm3(ns[0], ns[1], ns[2]);
      const float gn[3] = {gr.g_normal[3 * r], gr.g_normal[3 * r + 1], gr.g_normal[3 * r + 2]};
      normalize_eps_bwd(ns, l, gn, gN);
    }
    float g_rgb[3] = {0.f, 0.f, 0.f};
    if (gr.g_rgb) {
      g_rgb[0] = gr.g_rgb[3 * r];
      g_rgb[1] = gr.g_rgb[3 * r + 1];
      g_rgb[2] = gr.g_rgb[3 * r + 2];
    }
    float g_op = gr.g_opacity ? gr.g_opacity[r] : 0.0f;
    if (a.bg && gr.g_rgb) {  // rgb += (1 - opacity) * bg
      const float* b = a.bg_per_ray ? a.bg + 3 * r : a.bg;
      g_op -= g_rgb[0] * b[0] + g_rgb[1] * b[1] + g_rgb[2] * b[2];
    }
    const float g_dep = gr.g_depth ? gr.g_depth[r] : 0.0f;
    __syncwarp();
    // pass 2: dL/dw (zero where T < 1e-4) and dT_i T_i
    for (int base = 0; base < a.S; base += 32) {
      const int i = base + lane;
      if (i < a.S) {
        const int64_t k = r * a.S + i;
        const float T = T_s[i];
        float dw = g_op + g_dep * a.zv[k];
        dw += g_rgb[0] * a.colors[3 * k] + g_rgb[1] * a.colors[3 * k + 1] + g_rgb[2] * a.colors[3 * k + 2];
        dw += gN[0] * a.normals[3 * k] + gN[1] * a.normals[3 * k + 1] + gN[2] * a.normals[3 * k + 2];
        if (gr.g_weights) dw += gr.g_weights[k];
        if (T < 1e-4f) dw = 0.0f;
        if (kKeep) D_s[i] = dw;
        float dT = dw * A_s[i];
        if (gr.g_trans) dT += gr.g_trans[k];
        G_s[i] = dT * T;
      }
    }
    __syncwarp();
    // reverse exclusive scan over tiles, last tile first: G_i = sum_{j > i} (dT_j T_j)
    double rcarry = 0.0;
    const int ntiles = (a.S + 31) / 32;
    for (int tI = ntiles - 1; tI >= 0; --tI) {
      const int i = tI * 32 + (31 - lane);  // lane 0 holds the tile's last element
      const double v = (i < a.S) ? (double)G_s[i] : 0.0;
      const double inc = warp_incl_sum_d(v, lane);
      double ex = __shfl_up_sync(0xffffffffu, inc, 1);
      if (lane == 0) ex = 0.0;
      ex += rcarry;
      rcarry += __shfl_sync(0xffffffffu, inc, 31);
      __syncwarp();
      if (i < a.S) G_s[i] = (float)ex;
      __syncwarp();
    }
    // pass 3: per-sample adjoint
    for (int base = 0; base < a.S; base += 32) {
      const int i = base + lane;
      if (i >= a.S) continue;
      const int64_t k = r * a.S + i;
      SampleFwd o;
      float dw;
      if (kKeep) {
        o.am = A_s[i];
        o.mask = K_s[i];
        o.ratio = K_s[a.S + i];
        o.den = K_s[2 * a.S + i];
        o.diff = K_s[3 * a.S + i];
        o.p0 = K_s[4 * a.S + i];
        o.p1 = K_s[5 * a.S + i];
        o.f0 = K_s[6 * a.S + i];
        o.f1 = K_s[7 * a.S + i];
        o.cos_t = K_s[8 * a.S + i];
        dw = D_s[i];
      } else {
        const float nrm[3] = {a.normals[3 * k], a.normals[3 * k + 1], a.normals[3 * k + 2]};
        alpha_fwd(a, s, r, i, a.sdf[k], nrm, o);
        dw = g_op + g_dep * a.zv[k];
        dw += g_rgb[0] * a.colors[3 * k] + g_rgb[1] * a.colors[3 * k + 1] + g_rgb[2] * a.colors[3 * k + 2];
        dw += gN[0] * nrm[0] + gN[1] * nrm[1] + gN[2] * nrm[2];
        if (gr.g_weights) dw += gr.g_weights[k];
        if (T_s[i] < 1e-4f) dw = 0.0f;
      }
      const float T = T_s[i];
      const float w = (T < 1e-4f) ? 0.0f : o.am * T;
      float dam = dw * T;
      if (gr.g_alpha) dam += gr.g_alpha[k];
      const float qraw = __fadd_rn(__fsub_rn(1.0f, o.am), 1e-7f);
      if (qraw >= 0.0f && qraw <= 1.0f) dam -= G_s[i] / qraw;
      const float da = dam * o.mask;
      const float dr = (o.ratio >= 0.0f && o.ratio <= 1.0f) ? da : 0.0f;
      const float ddiff = dr / o.den;
      const float dden = -dr * o.diff / (o.den * o.den);
      const float dp0 = ddiff + ((o.p0 >= 1e-5f) ? dden : 0.0f);
      const float dp1 = -ddiff;
      const float dz0 = dp0 * ((1.0f - o.p0) * o.p0);
      const float dz1 = dp1 * ((1.0f - o.p1) * o.p1);
      ds_acc += (double)(dz0 * o.f0) + (double)(dz1 * o.f1);
      const float df0 = dz0 * s, df1 = dz1 * s;
      if (gr.d_sdf) gr.d_sdf[k] = df0 + df1;
      const float dc = (df1 - df0) * (0.5f * a.dists[k]);
      float dt = dc;  // dL/d<n,d>
      if (a.iter_cos) {
        const float m1 = (-o.cos_t * 0.5f + 0.5f > 0.0f) ? -0.5f : 0.0f;
        const float m2 = (-o.cos_t > 0.0f) ? -1.0f : 0.0f;
        dt = -dc * (m1 * (1.0f - a.cos_anneal) + m2 * a.cos_anneal);
      }
      const float* d = a.dirs + r * a.dir_rs + (int64_t)i * a.dir_ss;
      if (gr.d_normals) {
        gr.d_normals[3 * k] = dt * d[0] + w * gN[0];
        gr.d_normals[3 * k + 1] = dt * d[1] + w * gN[1];
        gr.d_normals[3 * k + 2] = dt * d[2] + w * gN[2];
      }
      if (gr.d_colors) {
        gr.d_colors[3 * k] = w * g_rgb[0];
        gr.d_colors[3 * k + 1] = w * g_rgb[1];
        gr.d_colors[3 * k + 2] = w * g_rgb[2];
      }
    }
    __syncwarp();
  }
  // dL/ds: warp -> block -> per-block partial -> the last block to finish sums them in
  // block order (deterministic) and writes the scalar.
  ds_acc = warp_sum_d(ds_acc);
  if (lane == 0) ds_warp[warp] = ds_acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    for (int w = 0; w < (int)wpb; ++w) b += ds_warp[w];
    gr.partials[blockIdx.x] = b;
    __threadfence();
    const unsigned prev = atomicAdd(gr.counter, 1u);
    is_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  double part = 0.0;
  const volatile double* p = gr.partials;
  for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) part += p[b];
  part = warp_sum_d(part);
  __syncthreads();
  if (lane == 0) ds_warp[warp] = part;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    for (int w = 0; w < (int)wpb; ++w) tot += ds_warp[w];
    float out = (float)tot;
    if (a.s_is_var) {
      // s = clamp(exp(10 v), 1e-4, s_max): dv = ds * exp(10 v) * 10 inside the clamp range
      const float v = __ldg(a.s_ptr);
      const float e = expf(v * 10.0f);
      out = (e >= 1e-4f && e <= a.s_max) ? (out * e) * 10.0f : 0.0f;
      int amp = 0;
      if (gr.amp_k > 0.0f && out < 0.0f) {  // training/scheduler.py:29-31
        out *= gr.amp_k;
        amp = 1;
      }
      if (gr.amp_flag) *gr.amp_flag = amp;
    }
    *gr.d_s_out = out;
    *gr.counter = 0u;  // ready for the next launch
  }
}

// ---------------------------- standalone Eq.2 and composite_weights ----------------------

__global__ void k_neus_alpha(CompArgs a, int64_t n, float* __restrict__ alpha, const float* __restrict__ d_alpha,
                             float* __restrict__ d_sdf, float* __restrict__ d_normals, float* __restrict__ d_s) {
  const float s = get_s(a);
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = k / a.S;
    const int i = (int)(k % a.S);
    const float nrm[3] = {a.normals[3 * k], a.normals[3 * k + 1], a.normals[3 * k + 2]};
    SampleFwd o;
    alpha_fwd(a, s, r, i, a.sdf[k], nrm, o);
    if (alpha) alpha[k] = o.a;
    if (d_alpha) {
      const float da = d_alpha[k];
      const float dr = (o.ratio >= 0.0f && o.ratio <= 1.0f) ? da : 0.0f;
      const float ddiff = dr / o.den;
      const float dden = -dr * o.diff / (o.den * o.den);
      const float dp0 = ddiff + ((o.p0 >= 1e-5f) ? dden : 0.0f);
      const float dp1 = -ddiff;
      const float dz0 = dp0 * ((1.0f - o.p0) * o.p0);
      const float dz1 = dp1 * ((1.0f - o.p1) * o.p1);
      if (d_s) d_s[k] = dz0 * o.f0 + dz1 * o.f1;
      const float df0 = dz0 * s, df1 = dz1 * s;
      if (d_sdf) d_sdf[k] = df0 + df1;
      const float dc = (df1 - df0) * (0.5f * a.dists[k]);
      float dt = dc;
      if (a.iter_cos) {
        const float m1 = (-o.cos_t * 0.5f + 0.5f > 0.0f) ? -0.5f : 0.0f;
        const float m2 = (-o.cos_t > 0.0f) ? -1.0f : 0.0f;
        dt = -dc * (m1 * (1.0f - a.cos_anneal) + m2 * a.cos_anneal);
      }
      const float* d = a.dirs + r * a.dir_rs + (int64_t)i * a.dir_ss;
      if (d_normals) {
        d_normals[3 * k] = dt * d[0];
        d_normals[3 * k + 1] = dt * d[1];
        d_normals[3 * k + 2] = dt * d[2];
      }
    }
  }
}

// volume_render.py:12-40 forward (d_w == null) or adjoint (d_alpha != null).
__global__ void __launch_bounds__(128) k_composite_weights(const float* __restrict__ alpha, int64_t N, int S,
                                                           float* __restrict__ w_out, float* __restrict__ t_out,
                                                           const float* __restrict__ d_w, const float* __restrict__ d_t,
                                                           float* __restrict__ d_alpha) {
  extern __shared__ float sm[];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  const int64_t wpb = blockDim.x >> 5;
  float* T_s = sm + warp * 2 * S;
  float* G_s = T_s + S;
  for (int64_t r = blockIdx.x * wpb + warp; r < N; r += (int64_t)gridDim.x * wpb) {
    double carry = 1.0;  // double accumulation, rounded once (the CPU cumprod does the same)
    for (int base = 0; base < S; base += 32) {
      const int i = base + lane;
      const float am = (i < S) ? alpha[r * S + i] : 0.0f;
      const float q = (i < S) ? fminf(fmaxf(__fadd_rn(__fsub_rn(1.0f, am), 1e-7f), 0.0f), 1.0f) : 1.0f;
      const double inc = warp_incl_prod_d((double)q, lane);
      double Td = __shfl_up_sync(0xffffffffu, inc, 1);
      if (lane == 0) Td = 1.0;
      const float T = (float)(Td * carry);
      carry *= __shfl_sync(0xffffffffu, inc, 31);
      if (i < S) {
        T_s[i] = T;
        if (w_out) w_out[r * S + i] = (T < 1e-4f) ? 0.0f : am * T;
        if (t_out) t_out[r * S + i] = T;
        if (d_alpha) {
          float dw = d_w ? d_w[r * S + i] : 0.0f;
          if (T < 1e-4f) dw = 0.0f;
          float dT = dw * am;
          if (d_t) dT += d_t[r * S + i];
          G_s[i] = dT * T;
        }
      }
    }
    if (!d_alpha) continue;
    __syncwarp();
    double rcarry = 0.0;
    const int ntiles = (S + 31) / 32;
    for (int tI = ntiles - 1; tI >= 0; --tI) {
      const int i = tI * 32 + (31 - lane);
      const double v = (i < S) ? (double)G_s[i] : 0.0;
      const double inc = warp_incl_sum_d(v, lane);
      double ex = __shfl_up_sync(0xffffffffu, inc, 1);
      if (lane == 0) ex = 0.0;
      ex += rcarry;
      rcarry += __shfl_sync(0xffffffffu, inc, 31);
      __syncwarp();
      if (i < S) G_s[i] = (float)ex;
      __syncwarp();
    }
    for (int base = 0; base < S; base += 32) {
      const int i = base + lane;
      if (i >= S) continue;
      const float am = alpha[r * S + i];
      const float T = T_s[i];
      float dw = d_w ? d_w[r * S + i] : 0.0f;
      if (T < 1e-4f) dw = 0.0f;
      float da = dw * T;
      const float qraw = __fadd_rn(__fsub_rn(1.0f, am), 1e-7f);
      if (qraw >= 0.0f && qraw <= 1.0f) da -= G_s[i] / qraw;
      d_alpha[r * S + i] = da;
    }
    __syncwarp();
  }
}

}  // namespace vx

using namespace vx;

static int fill_comp(CompArgs& a, const float* colors, const float* sdf, const float* normals, const float* dirs,
                     int64_t dir_rs, int64_t dir_ss, const float* zv, const float* dists, const float* pts,
                     const float* rays_o, const float* s_ptr, int s_is_var, float s_max, float radius,
                     const float* bg, int bg_per_ray, int iter_cos, float cos_anneal, int64_t N, int S) {
  VX_REQUIRE(N >= 0 && S >= 1 && S <= 4096, "need N >= 0 and 1 <= S <= 4096");
  VX_REQUIRE(sdf && normals && dirs && dists && s_ptr, "null pointer");
  VX_REQUIRE(radius <= 0.0f || pts || rays_o, "inside-sphere mask needs pts or rays_o");
  a = CompArgs{colors, sdf, normals, dirs, dir_rs, dir_ss, zv, dists, pts, rays_o, s_ptr, s_is_var, s_max, radius,
               bg, bg_per_ray, iter_cos, cos_anneal, N, S};
  return VX_OK;
}

extern "C" {

int vx_render_geometry_forward(const float* grid, const int32_t res[3], const float xyz_min[3],
                               const float xyz_max[3], const float* rays_o, const float* rays_d, const float* mid,
                               int64_t n_rays, int n_samples, float* sdf, float* normal, float* grad,
                               uint32_t* vr_bitmap, void* stream) {
  VX_REQUIRE(res && res[0] >= 2 && res[1] >= 2 && res[2] >= 2, "grid resolution must be >= 2 per axis");
  VX_REQUIRE((int64_t)res[0] * res[1] * res[2] < (int64_t(1) << 31), "grid has 2^31 or more voxels");
  VX_REQUIRE(n_rays >= 0 && n_samples >= 1, "bad sizes");
  const int64_t n = n_rays * n_samples;
  if (n == 0) return VX_OK;
  VX_REQUIRE(grid && rays_o && rays_d && mid && normal && xyz_min && xyz_max, "null pointer");
  Grid g = make_grid(res, xyz_min, xyz_max);
  k_geometry_fwd<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(grid, g, rays_o, rays_d, mid, n, n_samples, sdf,
                                                                       normal, grad, vr_bitmap);
  count_launches(1);
  return check_launch("render_geometry_forward");
}

int vx_render_geometry_backward(const float* grid, const int32_t res[3], const float xyz_min[3],
                                const float xyz_max[3], const float* rays_o, const float* rays_d, const float* mid,
                                int64_t n_rays, int n_samples, const float* d_sdf, const float* d_normal,
                                const float* d_normal2, int64_t ld2, const float* d_grad, const float* grad_fwd,
                                float* grid_grad, void* stream) {
  VX_REQUIRE(res && res[0] >= 2 && res[1] >= 2 && res[2] >= 2, "grid resolution must be >= 2 per axis");
  VX_REQUIRE((int64_t)res[0] * res[1] * res[2] < (int64_t(1) << 31), "grid has 2^31 or more voxels");
  VX_REQUIRE(n_rays >= 0 && n_samples >= 1, "bad sizes");
  VX_REQUIRE(!d_normal2 || ld2 >= 3, "ld2 must be >= 3");
  const int64_t n = n_rays * n_samples;
  if (n == 0) return VX_OK;
  VX_REQUIRE(grid && rays_o && rays_d && mid && grid_grad && xyz_min && xyz_max, "null pointer");
  Grid g = make_grid(res, xyz_min, xyz_max);
  k_geometry_bwd<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(grid, g, rays_o, rays_d, mid, n, n_samples, d_sdf,
                                                                       d_normal, d_normal2, ld2, d_grad, grad_fwd,
                                                                       grid_grad);
  count_launches(1);
  return check_launch("render_geometry_backward");
}

int vx_composite_workspace_blocks(int64_t n_rays) { return (int)grid_for(n_rays * 32, 128, 8); }

int vx_composite_forward(const float* colors, const float* sdf, const float* normals, const float* dirs,
                         int64_t dir_ray_stride, int64_t dir_sample_stride, const float* z_vals, const float* dists,
                         const float* pts, const float* rays_o, const float* s_ptr, int s_is_variance, float s_max,
                         float sphere_radius, const float* background, int background_per_ray, int use_iter_cos,
                         float cos_anneal_ratio, int64_t n_rays, int n_samples, float* rgb, float* depth,
                         float* normal, float* opacity, float* weights, float* alpha, float* transmittance,
                         void* stream) {
  CompArgs a;
  if (int st = fill_comp(a, colors, sdf, normals, dirs, dir_ray_stride, dir_sample_stride, z_vals, dists, pts, rays_o,
                         s_ptr, s_is_variance, s_max, sphere_radius, background, background_per_ray, use_iter_cos,
                         cos_anneal_ratio, n_rays, n_samples))
    return st;
  if (n_rays == 0) return VX_OK;
  VX_REQUIRE(colors && z_vals, "null pointer");
  k_composite_fwd<<<grid_for(n_rays * 32, 128, 8), 128, 0, (cudaStream_t)stream>>>(a, rgb, depth, normal, opacity,
                                                                                     weights, alpha, transmittance);
  count_launches(1);
  return check_launch("composite_forward");
}

int vx_composite_backward(const float* colors, const float* sdf, const float* normals, const float* dirs,
                          int64_t dir_ray_stride, int64_t dir_sample_stride, const float* z_vals, const float* dists,
                          const float* pts, const float* rays_o, const float* s_ptr, int s_is_variance, float s_max,
                          float sphere_radius, const float* background, int background_per_ray, int use_iter_cos,
                          float cos_anneal_ratio, int64_t n_rays, int n_samples, const float* g_rgb,
                          const float* g_depth, const float* g_normal, const float* g_opacity, const float* g_weights,
                          const float* g_alpha, const float* g_transmittance, float* d_colors, float* d_sdf,
                          float* d_normals, double* partials, int n_partials, unsigned int* counter, float* d_s,
                          float amplify_k, int* amplified, void* stream) {
  CompArgs a;
  if (int st = fill_comp(a, colors, sdf, normals, dirs, dir_ray_stride, dir_sample_stride, z_vals, dists, pts, rays_o,
                         s_ptr, s_is_variance, s_max, sphere_radius, background, background_per_ray, use_iter_cos,
                         cos_anneal_ratio, n_rays, n_samples))
    return st;
  VX_REQUIRE(colors && z_vals && partials && counter && d_s, "null pointer");
  const int blocks = (int)grid_for(n_rays * 32, 128, 8);
  VX_REQUIRE(n_partials >= blocks, "partials buffer holds %d entries, need %d", n_partials, blocks);
  const size_t smem_keep = (size_t)4 * kCompKeepFields * n_samples * sizeof(float);
  const size_t smem = (size_t)4 * 3 * n_samples * sizeof(float);
  VX_REQUIRE(smem <= 200 * 1024, "too many samples per ray");
  CompGrads gr{g_rgb, g_depth, g_normal, g_opacity, g_weights, g_alpha, g_transmittance, d_colors, d_sdf, d_normals,
               partials, counter, d_s, amplify_k, amplified};
  if (smem_keep <= 32 * 1024) {  // up to 157 samples per ray: 8 blocks per SM still fit
    k_composite_bwd<true><<<blocks, 128, smem_keep, (cudaStream_t)stream>>>(a, gr);
  } else {
    if (smem > 48 * 1024)
      cudaFuncSetAttribute(k_composite_bwd<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_composite_bwd<false><<<blocks, 128, smem, (cudaStream_t)stream>>>(a, gr);
  }
  count_launches(1);
  return check_launch("composite_backward");
}

int vx_neus_alpha(const float* sdf, const float* normals, const float* dirs, int64_t dir_ray_stride,
                  int64_t dir_sample_stride, const float* dists, const float* s_ptr, int use_iter_cos,
                  float cos_anneal_ratio, int64_t n_rays, int n_samples, float* alpha, const float* d_alpha,
                  float* d_sdf, float* d_normals, float* d_s_elems, void* stream) {
  CompArgs a;
  if (int st = fill_comp(a, nullptr, sdf, normals, dirs, dir_ray_stride, dir_sample_stride, nullptr, dists, nullptr,
                         nullptr, s_ptr, 0, 0.0f, 0.0f, nullptr, 0, use_iter_cos, cos_anneal_ratio, n_rays,
                         n_samples))
    return st;
  const int64_t n = n_rays * n_samples;
  if (n == 0) return VX_OK;
  k_neus_alpha<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(a, n, alpha, d_alpha, d_sdf, d_normals, d_s_elems);
  count_launches(1);
  return check_launch("neus_alpha");
}

int vx_composite_weights(const float* alpha, int64_t n_rays, int n_samples, float* weights, float* transmittance,
                         const float* d_weights, const float* d_transmittance, float* d_alpha, void* stream) {
  VX_REQUIRE(n_rays >= 0 && n_samples >= 1 && n_samples <= 4096, "bad sizes");
  if (n_rays == 0) return VX_OK;
  VX_REQUIRE(alpha, "null pointer");
  const size_t smem = (size_t)4 * 2 * n_samples * sizeof(float);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_composite_weights, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_composite_weights<<<grid_for(n_rays * 32, 128, 8), 128, smem, (cudaStream_t)stream>>>(
      alpha, n_rays, n_samples, weights, transmittance, d_weights, d_transmittance, d_alpha);
  count_launches(1);
  return check_launch("composite_weights");
}

}  // extern "C"
