// nm_depth.cu -- soft expected-depth renderer over the device map, its adjoint, and the
// per-step kernel of scan-to-map pose refinement (sm_100a).  No reference counterpart.
//
// Per pixel ray (sensor pixel model, double): voxel DDA from the voxel holding the eye.  Every
// voxel after it, entered at t_in < t_max and left at t_out (clamped to t_max), carries the
// density sigma = softplus(scale L + bias) (L the map's log-odds, 0 for voxels of absent
// leaves), so that sigmoid(scale L + bias) is the probability of the ray ending within one
// voxel length of it; the start voxel holds the sensor and is empty.  The expected depth
// (remaining probability placed at t_max) is the integral of the transmittance:
//   D = res (t_1 + sum_k T_k (1 - exp(-sigma_k D_k)) / sigma_k),  T_{k+1} = T_k exp(-sigma_k D_k)
// with D_k = t_out - t_in, accumulated in FP32.  D is continuous in the pose.
// The adjoint replays the traversal twice instead of storing it: the first replay rebuilds D;
// the second walks front to back with the running prefix P of the transmittance integral, so
// the tail S = D/res - t_1 - P needs no per-ray storage:
//   dD/dsigma_k = res (T_k D_k^2 g(sigma_k D_k) - D_k S_k),  g(u) = (u e^-u - 1 + e^-u) / u^2
//   crossing c from voxel A into B: dD/dc = res (sigma_B - sigma_A) * (tail after c),
//     c = (b - e_a) / d_a  ->  dc/de_a = -1/d_a,  dc/dd_a = -c/d_a
// and for a left world-frame pose perturbation (rho, phi): dD/drho = dD_idx/de,
// dD/dphi = res (d x dD_idx/dd).  The DDA runs in double with explicit round-to-nearest
// operations (no contraction), so its voxel sequence equals the FP64 CPU definition's.
#include <math_constants.h>

#include <cstdint>

#include "nm_device.cuh"
#include "nm_internal.h"

namespace nm {

namespace {

// 8 x 8 pixels per CTA: many small CTAs balance the uneven ray lengths (forward 11 % faster
// than 16 x 16 on the headline frame)
constexpr int kDepthTile = 8;

struct LeafCache {
  unsigned long long key;
  int slot;
};

__device__ __forceinline__ void pixel_dir(const DepthParams& p, int w, int h, double d[3]) {
  double x, y, z;
  if (p.type == NM_SENSOR_FRUSTUM) {
    const double u = __dmul_rn((double)w, (double)p.su);
    const double v = __dmul_rn((double)h, (double)p.sv);
    x = __dadd_rn(__dmul_rn(u, (double)p.c0), -(double)p.hw);
    y = __dadd_rn(__dmul_rn(v, (double)p.c1), -(double)p.hh);
    z = 1.0;
  } else {
    x = __dmul_rn((double)__ldg(&p.sinu[w]), (double)__ldg(&p.cosv[h]));
    y = (double)__ldg(&p.sinv[h]);
    z = __dmul_rn((double)__ldg(&p.cosu[w]), (double)__ldg(&p.cosv[h]));
  }
  const double n = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
  x = __ddiv_rn(x, n);
  y = __ddiv_rn(y, n);
  z = __ddiv_rn(z, n);
#pragma unroll
  for (int i = 0; i < 3; ++i)
    d[i] = __dadd_rn(__dadd_rn(__dmul_rn(p.R[3 * i], x), __dmul_rn(p.R[3 * i + 1], y)),
                     __dmul_rn(p.R[3 * i + 2], z));
}

__device__ __forceinline__ float softplus(float x) {
  return x > 0.0f ? x + log1pf(expf(-x)) : log1pf(expf(x));
}

// g(u) = (u e^-u - 1 + e^-u) / u^2 given em1 = e^-u - 1; -1/2 at u = 0.
__device__ __forceinline__ float seg_g(float u, float em1) {
  if (u < 1e-2f) return -0.5f + u * (1.0f / 3.0f) - u * u * 0.125f;
  return (u * (1.0f + em1) + em1) / (u * u);
}

// Every walk of a ray (forward, adjoint replays, refinement) ends where its transmittance
// falls below this: what the rest of the ray could add to the expected depth is at most
// kStopTransmittance x its remaining length (< 1e-6 voxel lengths for rays up to 1000
// voxels), each such FP32 term being below half an ulp of the running integral once that
// exceeds 0.01 voxels, and the rest's gradients carry the factor T too (there, the FP32 tail
// A - P is rounding noise).  The three walks compute T with the same operations, so they
// stop at the same voxel.
constexpr float kStopTransmittance = 1e-9f;

// Density of a log-odds value, memoised on the last value seen: along a ray most voxels share
// a few values (the clamp of observed free space, 0 for unknown space), so the softplus and
// sigmoid are mostly reused and each visit costs one expm1.
struct DensityCache {
  bool has = false;
  float L = 0.0f;
  float sg = 0.0f, sig = 0.5f;
  __device__ __forceinline__ void at(const DepthParams& p, float l) {
    if (!has || l != L) {
      has = true;
      L = l;
      const float x = p.scale * l + p.bias;
      sg = softplus(x);
      sig = 1.0f / (1.0f + expf(-x));
    }
  }
};

// Visits the voxels of the ray after the start voxel: f(v, t_in, a_in, t_out, a_out), the
// voxel entered at t_in < t_max across axis a_in and left at t_out = min(next crossing,
// t_max) across a_out (-1 when clamped to t_max); f returns false to end the walk.  Crossings are (boundary - e) * (1 / d),
// the reciprocal taken once per ray; per-axis state is kept in scalars (no local memory).
template <class F>
__device__ __forceinline__ void walk(const double e[3], const double d[3], double t_max, F&& f) {
  int vx = (int)floor(e[0]), vy = (int)floor(e[1]), vz = (int)floor(e[2]);
  const int sx = d[0] > 0.0 ? 1 : (d[0] < 0.0 ? -1 : 0);
  const int sy = d[1] > 0.0 ? 1 : (d[1] < 0.0 ? -1 : 0);
  const int sz = d[2] > 0.0 ? 1 : (d[2] < 0.0 ? -1 : 0);
  const double rx = sx ? __drcp_rn(d[0]) : 0.0;
  const double ry = sy ? __drcp_rn(d[1]) : 0.0;
  const double rz = sz ? __drcp_rn(d[2]) : 0.0;
  auto cross = [](int v, int s, double e, double r) {
    return __dmul_rn(__dadd_rn((double)(v + (s > 0 ? 1 : 0)), -e), r);
  };
  double tx = sx ? cross(vx, sx, e[0], rx) : CUDART_INF;
  double ty = sy ? cross(vy, sy, e[1], ry) : CUDART_INF;
  double tz = sz ? cross(vz, sz, e[2], rz) : CUDART_INF;
  int a_in = 2;
  double t_in = tz;
  if (ty < t_in) {
    a_in = 1;
    t_in = ty;
  }
  if (tx < t_in) {
    a_in = 0;
    t_in = tx;
  }
  const long long cap = 3ll * (long long)t_max + 16;
  for (long long it = 0; it < cap && t_in < t_max; ++it) {
    if (a_in == 0) {
      vx += sx;
      tx = cross(vx, sx, e[0], rx);
    } else if (a_in == 1) {
      vy += sy;
      ty = cross(vy, sy, e[1], ry);
    } else {
      vz += sz;
      tz = cross(vz, sz, e[2], rz);
    }
    int a_out = 2;
    double t_out = tz;
    if (ty < t_out) {
      a_out = 1;
      t_out = ty;
    }
    if (tx < t_out) {
      a_out = 0;
      t_out = tx;
    }
    const int v[3] = {vx, vy, vz};
    if (!(t_out < t_max ? f(v, t_in, a_in, t_out, a_out) : f(v, t_in, a_in, t_max, -1))) break;
    a_in = a_out;
    t_in = t_out;
  }
}

__device__ __forceinline__ float voxel_logodds(const MapView& m, const float* vals, LeafCache& c,
                                               const int v[3], int* slot, int* l) {
  const unsigned long long key = leaf_key(v[0] >> 3, v[1] >> 3, v[2] >> 3);
  if (key != c.key) {
    c.key = key;
    c.slot = map_find(m, key);
  }
  *slot = c.slot;
  *l = local_index(v[0], v[1], v[2]);
  return c.slot >= 0 ? __ldg(&vals[(size_t)c.slot * kLeafVoxels + *l]) : 0.0f;
}

// Expected depth in index units (integral of the transmittance over [0, t_max]), FP32.  With
// `entry_step` given, also the mean, over where the ray ends, of the voxel step along the axis
// it entered the ending voxel across (1 / |d_a|, index units): the depth the ray covers from
// one face of that voxel to the opposite one.
__device__ __forceinline__ float expected_index_depth(const DepthParams& p, const MapView& m,
                                                      const float* vals, const double d[3],
                                                      float* t1_out, uint32_t* visits,
                                                      float* entry_step = nullptr) {
  LeafCache c{kEmptyKey, -1};
  DensityCache dc;
  float T = 1.0f, acc = 0.0f, W = 0.0f;
  double t1 = p.t_max;
  bool first = true;
  uint32_t n = 0;
  const float step[3] = {(float)(1.0 / fabs(d[0])), (float)(1.0 / fabs(d[1])),
                         (float)(1.0 / fabs(d[2]))};
  walk(p.eye, d, p.t_max, [&](const int v[3], double t_in, int a_in, double t_out, int) {
    ++n;
    int slot, l;
    dc.at(p, voxel_logodds(m, vals, c, v, &slot, &l));
    const float sg = dc.sg;
    const float Dk = (float)(t_out - t_in);
    if (first) {
      t1 = t_in;
      first = false;
    }
    const float em1 = expm1f(-sg * Dk);
    acc += T * (sg > 0.0f ? -em1 / sg : Dk);
    if (entry_step) W -= T * em1 * step[a_in];
    T *= 1.0f + em1;
    return T >= kStopTransmittance;
  });
  *t1_out = (float)t1;
  *visits += n;
  if (entry_step) *entry_step = T < 1.0f ? W / (1.0f - T) : 0.0f;
  return (float)t1 + acc;
}

// The time of the ray's first voxel crossing (the t_in of walk()'s first visit, the same
// operations), or t_max when the ray stays in its start voxel.
__device__ __forceinline__ double first_crossing(const double e[3], const double d[3],
                                                 double t_max) {
  double t = CUDART_INF;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int s = d[a] > 0.0 ? 1 : (d[a] < 0.0 ? -1 : 0);
    if (!s) continue;
    const int v = (int)floor(e[a]);
    const double c = __dmul_rn(__dadd_rn((double)(v + (s > 0 ? 1 : 0)), -e[a]), __drcp_rn(d[a]));
    t = c < t ? c : t;
  }
  return t < t_max ? t : t_max;
}

// Voxels nearer the eye than this (index units) take their log-odds gradient through
// scatter_gradient: there the rays of a warp share voxels and thousands of rays add into the
// same voxel.  Farther out lanes rarely share a voxel at the same step and a plain atomic is
// cheaper (headline frame, given depths: 1.59 ms plain, 1.44 ms aggregated everywhere,
// 1.09 ms aggregated within this span).
constexpr double kGatherSpan = 48.0;

// Adds x into grad_vals[slot * 512 + l] (nothing for slot < 0) with one atomic per voxel
// among the warp's lanes at this call: lanes holding the same voxel (rays near the eye and
// neighbouring rays walk the same voxels at the same step) are summed by a shuffle tree first,
// in rounds that each fold every second remaining lane of a group into the one before it.
__device__ __forceinline__ void scatter_gradient(float* grad_vals, int slot, int l, float x) {
  const unsigned act = __activemask();
  const int lane = (int)((threadIdx.y * blockDim.x + threadIdx.x) & 31u);
  const unsigned long long key =
      slot >= 0 ? (unsigned long long)slot * kLeafVoxels + (unsigned)l : ~0ull;
  const unsigned peers = __match_any_sync(act, key);
  int rank = __popc(peers & ((1u << lane) - 1u));  // position among the voxel's lanes
  unsigned above = lane == 31 ? 0u : peers & (~0u << (lane + 1));
  while (__any_sync(act, above != 0u)) {
    const int nxt = __ffs(above);
    const float y = __shfl_sync(act, x, nxt ? nxt - 1 : lane);
    if (nxt) x += y;
    above &= ~__ballot_sync(act, rank & 1);  // odd ranks have been folded into their left
    rank >>= 1;
  }
  if (slot >= 0 && lane == __ffs(peers) - 1) atomicAdd(&grad_vals[key], x);
}

// Gradient replay of one ray: adds gd-weighted log-odds gradients into grad_vals (when given)
// and returns the ray's pose gradient (6: rho, phi) times gd.
__device__ __forceinline__ void replay_gradients(const DepthParams& p, const MapView& m,
                                                 const float* vals, const double d[3], float D,
                                                 float t1, float gd, float* grad_vals,
                                                 float g6[6], uint32_t* visits) {
  LeafCache c{kEmptyKey, -1};
  DensityCache dc;
  uint32_t n = 0;
  float T = 1.0f, P = 0.0f, sg_prev = 0.0f;
  float ge[3] = {0.f, 0.f, 0.f}, gdir[3] = {0.f, 0.f, 0.f};
  const float inv_d[3] = {(float)(1.0 / d[0]), (float)(1.0 / d[1]), (float)(1.0 / d[2])};
  const float gv = gd * (float)p.res * p.scale;
  const float tail0 = D - t1;
  walk(p.eye, d, p.t_max, [&](const int v[3], double t_in, int a_in, double t_out, int) {
    int slot, l;
    dc.at(p, voxel_logodds(m, vals, c, v, &slot, &l));
    ++n;
    const float sg = dc.sg;
    const float Dk = (float)(t_out - t_in);
    // entry crossing: the density steps from sg_prev to sg
    const float gc = (sg - sg_prev) * (tail0 - P) * (a_in == 0 ? inv_d[0] : (a_in == 1 ? inv_d[1] : inv_d[2]));
    const float ti = (float)t_in;
    if (a_in == 0) {
      ge[0] -= gc;
      gdir[0] -= gc * ti;
    } else if (a_in == 1) {
      ge[1] -= gc;
      gdir[1] -= gc * ti;
    } else {
      ge[2] -= gc;
      gdir[2] -= gc * ti;
    }
    const float u = sg * Dk;
    const float em1 = expm1f(-u);
    const float Pn = P + T * (sg > 0.0f ? -em1 / sg : Dk);
    if (grad_vals) {
      const float dsig = T * Dk * Dk * seg_g(u, em1) - Dk * (tail0 - Pn);
      if (t_in < kGatherSpan)
        scatter_gradient(grad_vals, slot, l, gv * dc.sig * dsig);
      else if (slot >= 0)
        atomicAdd(&grad_vals[(size_t)slot * kLeafVoxels + l], gv * dc.sig * dsig);
    }
    P = Pn;
    T *= 1.0f + em1;
    sg_prev = sg;
    return T >= kStopTransmittance;
  });
  *visits += n;
  const float r = gd * (float)p.res;
  const float dx = (float)d[0], dy = (float)d[1], dz = (float)d[2];
  g6[0] = gd * ge[0];
  g6[1] = gd * ge[1];
  g6[2] = gd * ge[2];
  g6[3] = r * (dy * gdir[2] - dz * gdir[1]);
  g6[4] = r * (dz * gdir[0] - dx * gdir[2]);
  g6[5] = r * (dx * gdir[1] - dy * gdir[0]);
}

// Adds the active lanes' visit counts to the map's counter (one atomic per warp).
__device__ __forceinline__ void add_depth_visits(const MapView& m, uint32_t n) {
  const unsigned act = __activemask();
  const uint32_t sum = __reduce_add_sync(act, n);
  if (((threadIdx.y * blockDim.x + threadIdx.x) & 31) == (unsigned)(__ffs(act) - 1))
    atomicAdd(&m.ctr->depth_visits, (unsigned long long)sum);
}

// Sum of N doubles over the CTA (blockDim.x * blockDim.y threads, a multiple of 32); thread 0
// writes the CTA's partials to out[blockIdx * N ...].
template <int N>
__device__ __forceinline__ void block_partials(double (&x)[N], double* out) {
  __shared__ double s[32][N];
  const int tid = threadIdx.y * blockDim.x + threadIdx.x;
  const int nw = (blockDim.x * blockDim.y) >> 5;
#pragma unroll
  for (int i = 0; i < N; ++i)
    for (int o = 16; o > 0; o >>= 1) x[i] += __shfl_down_sync(0xffffffffu, x[i], o);
  if ((tid & 31) == 0)
#pragma unroll
    for (int i = 0; i < N; ++i) s[tid >> 5][i] = x[i];
  __syncthreads();
  if (tid == 0) {
    const size_t b = (size_t)blockIdx.y * gridDim.x + blockIdx.x;
    for (int i = 0; i < N; ++i) {
      double acc = 0.0;
      for (int w = 0; w < nw; ++w) acc += s[w][i];
      out[b * N + i] = acc;
    }
  }
}

__global__ void __launch_bounds__(kDepthTile * kDepthTile) k_depth_forward(DepthParams p, MapView m,
                                                                           const float* vals,
                                                                           float* depth) {
  const int w = blockIdx.x * kDepthTile + threadIdx.x;
  const int h = blockIdx.y * kDepthTile + threadIdx.y;
  if (w >= p.width || h >= p.height) return;
  double d[3];
  pixel_dir(p, w, h, d);
  float t1;
  uint32_t n = 0;
  depth[(size_t)h * p.width + w] = expected_index_depth(p, m, vals, d, &t1, &n) * (float)p.res;
  add_depth_visits(m, n);
}

// `depth` (may be null): the forward's output at this pose and these values; the ray's
// expected depth is then taken from it instead of a first replay.
__global__ void __launch_bounds__(kDepthTile * kDepthTile) k_depth_backward(
    DepthParams p, MapView m, const float* vals, const float* grad_depth, const float* depth,
    float* grad_vals, double* partials) {
  const int w = blockIdx.x * kDepthTile + threadIdx.x;
  const int h = blockIdx.y * kDepthTile + threadIdx.y;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  uint32_t n = 0;
  if (w < p.width && h < p.height) {
    const float gd = grad_depth[(size_t)h * p.width + w];
    if (gd != 0.0f) {
      double d[3];
      pixel_dir(p, w, h, d);
      float t1, D;
      if (depth) {
        D = depth[(size_t)h * p.width + w] / (float)p.res;
        t1 = (float)first_crossing(p.eye, d, p.t_max);
      } else {
        D = expected_index_depth(p, m, vals, d, &t1, &n);
      }
      float g6[6];
      replay_gradients(p, m, vals, d, D, t1, gd, grad_vals, g6, &n);
#pragma unroll
      for (int i = 0; i < 6; ++i) acc[i] = (double)g6[i];
    }
  }
  add_depth_visits(m, n);
  block_partials<6>(acc, partials);
}

// One walk giving the expected depth (as expected_index_depth, with the entry step) and the
// ray's pose gradient for a unit depth gradient, for the refinement step.  replay_gradients'
// crossing term is c (A - P) with c = (sigma_B - sigma_A) / d_a, P the transmittance integral
// before the crossing and A the whole integral (D / res - t_1), so per axis the sums of c,
// c P, c t and c t P (in double: A and P are close where c is large) give the gradient once
// A is known at the end of the walk.  Returns D (index units); g6 as replay_gradients' for
// gd = 1.
__device__ __forceinline__ float depth_and_pose_gradient(const DepthParams& p, const MapView& m,
                                                         const float* vals, const double d[3],
                                                         uint32_t* visits, float* entry_step,
                                                         float g6[6]) {
  LeafCache c{kEmptyKey, -1};
  DensityCache dc;
  float T = 1.0f, acc = 0.0f, W = 0.0f, sg_prev = 0.0f;
  double t1 = p.t_max;
  bool first = true;
  uint32_t n = 0;
  const float step[3] = {(float)(1.0 / fabs(d[0])), (float)(1.0 / fabs(d[1])),
                         (float)(1.0 / fabs(d[2]))};
  const float inv_d[3] = {(float)(1.0 / d[0]), (float)(1.0 / d[1]), (float)(1.0 / d[2])};
  double sc[3] = {0.0, 0.0, 0.0}, scp[3] = {0.0, 0.0, 0.0};
  double sct[3] = {0.0, 0.0, 0.0}, sctp[3] = {0.0, 0.0, 0.0};
  walk(p.eye, d, p.t_max, [&](const int v[3], double t_in, int a_in, double t_out, int) {
    ++n;
    int slot, l;
    dc.at(p, voxel_logodds(m, vals, c, v, &slot, &l));
    const float sg = dc.sg;
    const float Dk = (float)(t_out - t_in);
    if (first) {
      t1 = t_in;
      first = false;
    }
    if (sg != sg_prev) {
      const double cd = (double)((sg - sg_prev) * (a_in == 0 ? inv_d[0] : (a_in == 1 ? inv_d[1] : inv_d[2])));
      const double P = (double)acc, ti = (double)(float)t_in;
      if (a_in == 0) {
        sc[0] += cd;
        scp[0] += cd * P;
        sct[0] += cd * ti;
        sctp[0] += cd * ti * P;
      } else if (a_in == 1) {
        sc[1] += cd;
        scp[1] += cd * P;
        sct[1] += cd * ti;
        sctp[1] += cd * ti * P;
      } else {
        sc[2] += cd;
        scp[2] += cd * P;
        sct[2] += cd * ti;
        sctp[2] += cd * ti * P;
      }
    }
    const float em1 = expm1f(-sg * Dk);
    acc += T * (sg > 0.0f ? -em1 / sg : Dk);
    W -= T * em1 * step[a_in];
    T *= 1.0f + em1;
    sg_prev = sg;
    return T >= kStopTransmittance;
  });
  *visits += n;
  *entry_step = T < 1.0f ? W / (1.0f - T) : 0.0f;
  const double A = (double)acc;
  float ge[3], gdir[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    ge[a] = (float)(scp[a] - A * sc[a]);
    gdir[a] = (float)(sctp[a] - A * sct[a]);
  }
  const float r = (float)p.res;
  const float dx = (float)d[0], dy = (float)d[1], dz = (float)d[2];
  g6[0] = ge[0];
  g6[1] = ge[1];
  g6[2] = ge[2];
  g6[3] = r * (dy * gdir[2] - dz * gdir[1]);
  g6[4] = r * (dz * gdir[0] - dx * gdir[2]);
  g6[5] = r * (dx * gdir[1] - dy * gdir[0]);
  return (float)t1 + acc;
}

// Whether pixel (w, h) of the target lies on a silhouette: a 4-neighbour inside the image
// without a return, or with a range more than `edge` metres away.
__device__ __forceinline__ bool target_edge(const float* target, int W, int H, int w, int h,
                                            float r, float edge) {
  const int nx[4] = {w - 1, w + 1, w, w};
  const int ny[4] = {h, h, h - 1, h + 1};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (nx[k] < 0 || nx[k] >= W || ny[k] < 0 || ny[k] >= H) continue;
    const float q = target[(size_t)ny[k] * W + nx[k]];
    if (!(q > 0.0f && q < CUDART_INF_F) || fabsf(q - r) > edge) return true;
  }
  return false;
}

// One refinement step: L1 loss against `target` (metres; <= 0 or NaN = no return), truncated
// at max_residual when it is positive (residuals beyond it add max_residual and no gradient),
// its pose gradient, and the number of pixels that took part.  The prediction is the expected
// depth plus `surface_offset` times the entry step of the voxel where the ray ends (0: the
// surface at the face the ray enters; 0.5: at the middle of the voxel), the offset held fixed
// for the gradient.  Silhouette pixels of the target are left out when edge > 0.  Partials:
// loss, count, 6 gradients.
__global__ void __launch_bounds__(kDepthTile * kDepthTile) k_depth_refine(
    DepthParams p0, MapView m, const float* vals, const float* target, float max_residual,
    float surface_offset, float edge, const RefineState* st, double* partials) {
  // the pose of this step, from the device state (the eye as the host computes it)
  DepthParams p = p0;
#pragma unroll
  for (int a = 0; a < 3; ++a) p.eye[a] = __ddiv_rn(st->position[a], p.res);
#pragma unroll
  for (int i = 0; i < 9; ++i) p.R[i] = st->R[i];
  const int w = blockIdx.x * kDepthTile + threadIdx.x;
  const int h = blockIdx.y * kDepthTile + threadIdx.y;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  uint32_t n = 0;
  if (w < p.width && h < p.height) {
    const float r = target[(size_t)h * p.width + w];
    if (r > 0.0f && r < CUDART_INF_F &&
        !(edge > 0.0f && target_edge(target, p.width, p.height, w, h, r, edge))) {
      double d[3];
      pixel_dir(p, w, h, d);
      float step, g6[6];
      const float D = depth_and_pose_gradient(p, m, vals, d, &n, &step, g6);
      const float res = (D + surface_offset * step) * (float)p.res - r;
      const bool clipped = max_residual > 0.0f && fabsf(res) > max_residual;
      acc[0] = clipped ? (double)max_residual : fabs((double)res);
      acc[1] = 1.0;
      const float gd = clipped ? 0.0f : (res > 0.0f ? 1.0f : (res < 0.0f ? -1.0f : 0.0f));
      if (gd != 0.0f) {
#pragma unroll
        for (int i = 0; i < 6; ++i) acc[2 + i] = (double)(gd * g6[i]);
      }
    }
  }
  add_depth_visits(m, n);
  block_partials<8>(acc, partials);
}

// exp([phi]x) R (Rodrigues), row-major, in place.
__device__ void rotate_left(const double phi[3], double R[9]) {
  const double th = sqrt(phi[0] * phi[0] + phi[1] * phi[1] + phi[2] * phi[2]);
  const double K[9] = {0, -phi[2], phi[1], phi[2], 0, -phi[0], -phi[1], phi[0], 0};
  double E[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (th > 0.0) {
    const double a = sin(th) / th, b = (1.0 - cos(th)) / (th * th);
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c)
        E[3 * r + c] += a * K[3 * r + c] +
                        b * (K[3 * r] * K[c] + K[3 * r + 1] * K[3 + c] + K[3 * r + 2] * K[6 + c]);
  }
  double out[9];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      out[3 * r + c] = E[3 * r] * R[c] + E[3 * r + 1] * R[3 + c] + E[3 * r + 2] * R[6 + c];
  for (int i = 0; i < 9; ++i) R[i] = out[i];
}

// One block: the step's partials summed in a fixed order (loss, count, 6 gradients), then
// thread 0 records the mean loss and, before the last step, applies Adam on the left
// world-frame increment (rho, phi) with the learning rates cosine-decayed to zero.
__global__ void k_refine_update(const double* partials, int n, RefineState* st, float* losses,
                                int it) {
  __shared__ double s[256];
  __shared__ double h[8];
  for (int c = 0; c < 8; ++c) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partials[(size_t)i * 8 + c];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
      if ((int)threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
      __syncthreads();
    }
    if (threadIdx.x == 0) h[c] = s[0];
    __syncthreads();
  }
  if (threadIdx.x != 0 || st->error) return;
  if (h[1] < 1.0) {
    st->error |= kRefineNoPixels;
    return;
  }
  losses[it] = (float)(h[0] / h[1]);
  if (it >= st->steps) return;
  const double b1 = 0.9, b2 = 0.999, eps = 1e-8;
  const double t = (double)(it + 1);
  const double decay = 0.5 * (1.0 + cos(CUDART_PI * it / st->steps));
  double step[6];
  for (int i = 0; i < 6; ++i) {
    const double g = h[2 + i] / h[1];
    st->mom[i] = b1 * st->mom[i] + (1.0 - b1) * g;
    st->var[i] = b2 * st->var[i] + (1.0 - b2) * g * g;
    const double mh = st->mom[i] / (1.0 - pow(b1, t));
    const double vh = st->var[i] / (1.0 - pow(b2, t));
    step[i] = -decay * (i < 3 ? st->lr_position : st->lr_rotation) * mh / (sqrt(vh) + eps);
  }
  for (int a = 0; a < 3; ++a)
    if (fabs((st->position[a] + step[a]) / st->res) + st->t_max + 2.0 > (double)(1 << 23) - 16.0) {
      st->error |= kRefineOutOfRange;
      return;
    }
  for (int a = 0; a < 3; ++a) st->position[a] += step[a];
  rotate_left(step + 3, st->R);
}

// Column sums of an (n, N) array of partials in a fixed order (deterministic).
__global__ void k_sum_partials(const double* partials, int n, int N, double* out) {
  __shared__ double s[256];
  for (int c = 0; c < N; ++c) {
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partials[(size_t)i * N + c];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
      if ((int)threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[c] = s[0];
    __syncthreads();
  }
}

dim3 depth_grid(const DepthParams& p) {
  return dim3((p.width + kDepthTile - 1) / kDepthTile, (p.height + kDepthTile - 1) / kDepthTile);
}

}  // namespace

int depth_partial_blocks(const DepthParams& p) {
  const dim3 g = depth_grid(p);
  return (int)(g.x * g.y);
}

cudaError_t launch_depth_forward(const DepthParams& p, const MapView& m, const float* vals,
                                 float* depth, cudaStream_t s) {
  k_depth_forward<<<depth_grid(p), dim3(kDepthTile, kDepthTile), 0, s>>>(p, m, vals, depth);
  return cudaGetLastError();
}

cudaError_t launch_depth_backward(const DepthParams& p, const MapView& m, const float* vals,
                                  const float* grad_depth, const float* depth, float* grad_vals,
                                  double* partials, double* out6, cudaStream_t s) {
  const dim3 g = depth_grid(p);
  k_depth_backward<<<g, dim3(kDepthTile, kDepthTile), 0, s>>>(p, m, vals, grad_depth, depth,
                                                              grad_vals, partials);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_sum_partials<<<1, 256, 0, s>>>(partials, (int)(g.x * g.y), 6, out6);
  return cudaGetLastError();
}

cudaError_t launch_depth_refine(const DepthParams& p, const MapView& m, const float* vals,
                                const float* target, float max_residual, float surface_offset,
                                float edge, double* partials, RefineState* st, float* losses,
                                int it, cudaStream_t s) {
  const dim3 g = depth_grid(p);
  k_depth_refine<<<g, dim3(kDepthTile, kDepthTile), 0, s>>>(p, m, vals, target, max_residual,
                                                            surface_offset, edge, st, partials);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_refine_update<<<1, 256, 0, s>>>(partials, (int)(g.x * g.y), st, losses, it);
  return cudaGetLastError();
}

}  // namespace nm
