// nm_sim_device.cuh -- simulated-depth ray casting and range noise (device functions),
// shared by the render kernels (nm_sim.cu) and the traversal's fused render (nm_traverse.cu).
//
// Replaces getActiveCrossing / viewSimKernel (generateCloud.cu:20-82).  The ray cast is an
// exact hierarchical form of the closed-form voxel DDA the oracle runs: crossing times are
// always recomputed from the plane index, t(p) = (p - eye) / dir, so the walk has no
// accumulated state, and a skip over an empty leaf or brick lands on the same voxel the
// voxel-by-voxel walk reaches when it leaves that cube.  The landing voxel is found by
// ordering crossing events by (time, higher axis first): on each other axis the walk has
// crossed every plane whose time is below the exit time, or equal to it on a higher axis
// than the exit axis.
#pragma once

#include <cstdint>

#include "nm_sim.h"

namespace nm {
namespace {

// ---- ray casting -----------------------------------------------------------------------------

__device__ __forceinline__ float plane_time(int p, float e, float inv) {
  return __fmul_rn(__fadd_rn((float)p, -e), inv);
}

__device__ __forceinline__ float plane_time_f(float p, float e, float inv) {
  return __fmul_rn(__fadd_rn(p, -e), inv);
}

// Crossed-before-exit predicate for a plane on axis j (see the header comment).
__device__ __forceinline__ bool crossed(int p, float e, float inv, float T, bool higher) {
  const float t = plane_time(p, e, inv);
  return t < T || (t == T && higher);
}

// Voxel index on axis j after the walk has processed every event before the exit event
// (T, exit axis a), starting from voxel k inside [k .. far] (s = +1) or [far .. k] (s = -1).
__device__ __forceinline__ int advance_axis(int k, int far, int s, float e, float dir, float inv,
                                            float T, bool higher) {
  int est = (int)floorf(__fadd_rn(e, __fmul_rn(dir, T)));
  if (s > 0) {
    est = max(k, min(far, est));
    while (est < far && crossed(est + 1, e, inv, T, higher)) ++est;
    while (est > k && !crossed(est, e, inv, T, higher)) --est;
  } else {
    est = min(k, max(far, est));
    while (est > far && crossed(est, e, inv, T, higher)) --est;
    while (est < k && !crossed(est + 1, e, inv, T, higher)) ++est;
  }
  return est;
}

// 2 = empty brick (or outside the map), 1 = empty leaf (*leaf = d >= 1: every leaf within
// Chebyshev distance d - 1 of it is empty too), 0 = leaf with bits (*leaf = index).
__device__ __forceinline__ int sim_level(const SimMapView& v, int x, int y, int z, int* leaf) {
  const int bx = (x >> 6) - v.blo[0], by = (y >> 6) - v.blo[1], bz = (z >> 6) - v.blo[2];
  if ((unsigned)bx >= (unsigned)v.bdim[0] || (unsigned)by >= (unsigned)v.bdim[1] ||
      (unsigned)bz >= (unsigned)v.bdim[2])
    return 2;
  const long long bpos = ((long long)bx * v.bdim[1] + by) * v.bdim[2] + bz;
  const int32_t blk = __ldg(&v.brick_index[bpos]);
  if (blk < 0) return 2;
  const int e = (((x >> 3) & 7) << 6) | (((y >> 3) & 7) << 3) | ((z >> 3) & 7);
  const int32_t li = __ldg(&v.brick_leaves[(size_t)blk * 512 + e]);
  if (li < 0) {
    *leaf = -li;
    return 1;
  }
  *leaf = li;
  return 0;
}

// Distance (metres) to the first active voxel entered along the ray from `eye` (index space)
// in the unit direction `dir`, at a ray time within [tmin, tmax] (voxel units), or 0.  The
// voxel holding the eye is not tested.
__device__ __forceinline__ float sim_cast(const SimMapView& v, const float eye[3], float dir[3],
                                          float tmin, float tmax) {
  float result = 0.0f;
  float inv[3];
  int st[3];
  float t_in = 0.0f, t_out = INFINITY;
  bool miss = false;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (fabsf(dir[a]) < 1e-30f) dir[a] = 0.0f;
    if (dir[a] == 0.0f) {
      st[a] = 0;
      inv[a] = 0.0f;
      if (eye[a] < v.box_lo[a] || eye[a] > v.box_hi[a]) miss = true;
    } else {
      inv[a] = __frcp_rn(dir[a]);
      st[a] = dir[a] > 0.0f ? 1 : -1;
      float ta = plane_time_f(v.box_lo[a], eye[a], inv[a]);
      float tb = plane_time_f(v.box_hi[a], eye[a], inv[a]);
      if (ta > tb) {
        const float x = ta;
        ta = tb;
        tb = x;
      }
      if (ta > t_in) t_in = ta;
      if (tb < t_out) t_out = tb;
    }
  }
  if (!miss && !(t_in > t_out)) {
    int k[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) k[a] = (int)floorf(__fadd_rn(eye[a], __fmul_rn(dir[a], t_in)));
    float t = t_in;
    bool first = true;
    for (int iter = 0; iter < (1 << 22); ++iter) {
      int leaf = -1;
      const int lvl = sim_level(v, k[0], k[1], k[2], &leaf);
      if (lvl == 0) {
        // Voxel steps inside a leaf with active voxels: the leaf's words come from L1, and
        // only the stepped axis's next crossing changes (each crossing is the closed form of
        // its own plane, so the event sequence is the one the generic step takes).
        const uint32_t* lw = v.leaf_words + (size_t)leaf * 16;
        int k0 = k[0], k1 = k[1], k2 = k[2];
        const int b0 = k0 & ~7, b1 = k1 & ~7, b2 = k2 & ~7;
        float T0 = st[0] == 0 ? INFINITY : plane_time(st[0] > 0 ? k0 + 1 : k0, eye[0], inv[0]);
        float T1 = st[1] == 0 ? INFINITY : plane_time(st[1] > 0 ? k1 + 1 : k1, eye[1], inv[1]);
        float T2 = st[2] == 0 ? INFINITY : plane_time(st[2] > 0 ? k2 + 1 : k2, eye[2], inv[2]);
        bool hit = false, done = false;
        for (int it2 = 0; it2 < 24; ++it2) {
          if (!first) {
            const int l = ((k0 & 7) << 6) | ((k1 & 7) << 3) | (k2 & 7);
            if ((__ldg(&lw[l >> 5]) >> (l & 31)) & 1u) {
              hit = true;
              break;
            }
          }
          first = false;
          const int ax = (T0 < T1) ? ((T0 < T2) ? 0 : 2) : ((T1 < T2) ? 1 : 2);
          const float Tx = ax == 0 ? T0 : (ax == 1 ? T1 : T2);
          if (!(Tx <= t_out)) {
            done = true;
            break;
          }
          t = Tx;
          bool left;
          if (ax == 0) {
            k0 += st[0];
            left = (k0 & ~7) != b0;
            T0 = plane_time(st[0] > 0 ? k0 + 1 : k0, eye[0], inv[0]);
          } else if (ax == 1) {
            k1 += st[1];
            left = (k1 & ~7) != b1;
            T1 = plane_time(st[1] > 0 ? k1 + 1 : k1, eye[1], inv[1]);
          } else {
            k2 += st[2];
            left = (k2 & ~7) != b2;
            T2 = plane_time(st[2] > 0 ? k2 + 1 : k2, eye[2], inv[2]);
          }
          if (left) break;
        }
        k[0] = k0;
        k[1] = k1;
        k[2] = k2;
        if (hit) {
          if (t >= tmin && t <= tmax) result = __fmul_rn(t, v.res);
          break;
        }
        if (done) break;
        continue;  // left the leaf: the outer walk takes the next level
      }
      first = false;
      // the empty cube to leave: the brick (64^3 voxels), or the leaves within Chebyshev
      // distance d - 1 of this empty leaf (all empty; d = 1: the leaf itself)
      const int dc = lvl == 1 ? leaf : 0;
      int far[3];
      float T[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        if (st[a] == 0) {
          far[a] = k[a];
          T[a] = INFINITY;
        } else {
          const int L = k[a] >> 3;
          far[a] = lvl == 2 ? (st[a] > 0 ? (k[a] | 63) : (k[a] & ~63))
                            : (st[a] > 0 ? (L + dc) * 8 - 1 : (L - dc + 1) * 8);
          T[a] = plane_time(st[a] > 0 ? far[a] + 1 : far[a], eye[a], inv[a]);
        }
      }
      const int ax = (T[0] < T[1]) ? ((T[0] < T[2]) ? 0 : 2) : ((T[1] < T[2]) ? 1 : 2);
      const float Tx = T[ax];
      if (!(Tx <= t_out)) break;
#pragma unroll
      for (int a = 0; a < 3; ++a)
        if (a != ax && st[a] != 0)
          k[a] = advance_axis(k[a], far[a], st[a], eye[a], dir[a], inv[a], Tx, a > ax);
      k[ax] = far[ax] + st[ax];
      t = Tx;
    }
  }
  return result;
}

// Range of pixel (w, h): the first active voxel entered along the pixel ray, or 0.
__device__ __forceinline__ float sim_ray(const SimMapView& v, const SimRayParams& rp, int w, int h) {
  if (!v.any) return 0.0f;
  float d0, d1, d2;
  if (rp.type == NM_SENSOR_FRUSTUM) {
    const float u = __fmul_rn((float)w, rp.su);
    const float vv = __fmul_rn((float)h, rp.sv);
    d0 = __fadd_rn(__fmul_rn(u, rp.c0), -rp.hw);
    d1 = __fadd_rn(__fmul_rn(vv, rp.c1), -rp.hh);
    d2 = 1.0f;
  } else {
    const float cv = __ldg(&rp.cosv[h]);
    d0 = __fmul_rn(__ldg(&rp.sinu[w]), cv);
    d1 = __ldg(&rp.sinv[h]);
    d2 = __fmul_rn(__ldg(&rp.cosu[w]), cv);
  }
  const float* R = rp.R;
  const float m0 = __fadd_rn(__fadd_rn(__fmul_rn(R[0], d0), __fmul_rn(R[1], d1)), __fmul_rn(R[2], d2));
  const float m1 = __fadd_rn(__fadd_rn(__fmul_rn(R[3], d0), __fmul_rn(R[4], d1)), __fmul_rn(R[5], d2));
  const float m2 = __fadd_rn(__fadd_rn(__fmul_rn(R[6], d0), __fmul_rn(R[7], d1)), __fmul_rn(R[8], d2));
  const float norm = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(m0, m0), __fmul_rn(m1, m1)), __fmul_rn(m2, m2)));
  float dir[3] = {__fdiv_rn(m0, norm), __fdiv_rn(m1, norm), __fdiv_rn(m2, norm)};
  const float eye[3] = {rp.eye[0], rp.eye[1], rp.eye[2]};  // pos / res
  float tmin = rp.tmin, tmax = rp.tmax;                     // range limits / res
  if (rp.type == NM_SENSOR_FRUSTUM) {
    tmin = __fmul_rn(tmin, norm);
    tmax = __fmul_rn(tmax, norm);
  }
  return sim_cast(v, eye, dir, tmin, tmax);
}

// splitmix64 (Steele, Lea, Flood 2014) as a counter-based generator.
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

__device__ __forceinline__ float noisy(float x, uint64_t seed, long long i, float sigma_coef,
                                       float drop) {
  const uint64_t a = mix64(seed ^ mix64((uint64_t)i));
  const uint64_t b = mix64(a);
  const float u1 = ((float)(a >> 40) + 0.5f) * (1.0f / 16777216.0f);
  const float u2 = (float)((a >> 16) & 0xFFFFFFu) * (1.0f / 16777216.0f);
  const float u3 = (float)(b >> 40) * (1.0f / 16777216.0f);
  if (x > 0.0f) {
    const float g = sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
    x = x + g * sigma_coef * x * x;
    if (u3 < drop || !(x > 0.0f)) x = 0.0f;
  }
  return x;
}

}  // namespace
}  // namespace nm
