// nm_sim.cu -- simulation map build and simulated-depth ray casting on sm_100a.
//
// Replaces the NanoVDB sim grid upload (SimHandler.cpp:22-23) and generateCloud /
// viewSimKernel / getActiveCrossing (generateCloud.cu:20-94).
//
// Sim map layout: a dense grid of leaf indices over the map's leaf box (-1 = empty leaf),
// compact 8^3 bit leaves (16 words each), and one occupancy bit per 64^3-voxel brick for
// long empty-space skips.
//
// The ray cast is an exact hierarchical form of the closed-form voxel DDA the oracle runs:
// crossing times are always recomputed from the plane index, t(p) = (p - eye) / dir, so
// the walk has no accumulated state, and a skip over an empty leaf or brick lands on the
// same voxel the voxel-by-voxel walk reaches when it leaves that cube.  The landing voxel is
// found by ordering crossing events by (time, higher axis first): on each other axis the
// walk has crossed every plane whose time is below the exit time, or equal to it on a
// higher axis than the exit axis.
#include <cfloat>
#include <cmath>
#include <algorithm>
#include <cstdint>

#include "nm_sim.h"

namespace nm {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ void sim_build_set(const SimBuild& b, int i, int j, int k) {
  if (i < b.vmin[0] || i >= b.vmax[0] || j < b.vmin[1] || j >= b.vmax[1] || k < b.vmin[2] ||
      k >= b.vmax[2])
    return;
  const long long lx = (i >> 3) - b.llo[0], ly = (j >> 3) - b.llo[1], lz = (k >> 3) - b.llo[2];
  const long long pos = (lx * b.ldim[1] + ly) * b.ldim[2] + lz;
  const int l = ((i & 7) << 6) | ((j & 7) << 3) | (k & 7);
  atomicOr(&b.dense[pos * 16 + (l >> 5)], 1u << (l & 31));
}

__global__ void __launch_bounds__(256) k_voxelize_boxes(SimBuild b, const double* boxes, int nb) {
  const int bi = blockIdx.y;
  if (bi >= nb) return;
  const double* B = boxes + 6 * bi;
  const double r = (double)b.res;
  int lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = max(b.vmin[a], (int)floor(__ddiv_rn(B[a], r) - 0.5) - 1);
    hi[a] = min(b.vmax[a] - 1, (int)ceil(__ddiv_rn(B[3 + a], r) - 0.5) + 1);
    if (hi[a] < lo[a]) return;
  }
  const long long ni = hi[0] - lo[0] + 1, nj = hi[1] - lo[1] + 1, nk = hi[2] - lo[2] + 1;
  const long long total = ni * nj * nk;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int k = lo[2] + (int)(idx % nk);
    const int j = lo[1] + (int)((idx / nk) % nj);
    const int i = lo[0] + (int)(idx / (nk * nj));
    const double cx = __dmul_rn(__dadd_rn((double)i, 0.5), r);
    const double cy = __dmul_rn(__dadd_rn((double)j, 0.5), r);
    const double cz = __dmul_rn(__dadd_rn((double)k, 0.5), r);
    if (B[0] <= cx && cx <= B[3] && B[1] <= cy && cy <= B[4] && B[2] <= cz && cz <= B[5])
      sim_build_set(b, i, j, k);
  }
}

__global__ void __launch_bounds__(256) k_voxelize_cylinders(SimBuild b, const double* cyl, int nc) {
  const int ci = blockIdx.y;
  if (ci >= nc) return;
  const double* C = cyl + 5 * ci;
  const double r = (double)b.res;
  const double rr = __dmul_rn(C[2], C[2]);
  const double bl[3] = {__dadd_rn(C[0], -C[2]), __dadd_rn(C[1], -C[2]), C[3]};
  const double bh[3] = {__dadd_rn(C[0], C[2]), __dadd_rn(C[1], C[2]), C[4]};
  int lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = max(b.vmin[a], (int)floor(__ddiv_rn(bl[a], r) - 0.5) - 1);
    hi[a] = min(b.vmax[a] - 1, (int)ceil(__ddiv_rn(bh[a], r) - 0.5) + 1);
    if (hi[a] < lo[a]) return;
  }
  const long long ni = hi[0] - lo[0] + 1, nj = hi[1] - lo[1] + 1, nk = hi[2] - lo[2] + 1;
  const long long total = ni * nj * nk;
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int k = lo[2] + (int)(idx % nk);
    const int j = lo[1] + (int)((idx / nk) % nj);
    const int i = lo[0] + (int)(idx / (nk * nj));
    const double dx = __dadd_rn(__dmul_rn(__dadd_rn((double)i, 0.5), r), -C[0]);
    const double dy = __dadd_rn(__dmul_rn(__dadd_rn((double)j, 0.5), r), -C[1]);
    const double cz = __dmul_rn(__dadd_rn((double)k, 0.5), r);
    if (__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)) <= rr && C[3] <= cz && cz <= C[4])
      sim_build_set(b, i, j, k);
  }
}

__global__ void k_set_voxels(SimBuild b, const int32_t* ijk, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    sim_build_set(b, ijk[3 * i], ijk[3 * i + 1], ijk[3 * i + 2]);
}

// Voxel bounds of one 32-bit leaf word q (voxels x*64 + y*8 + z): x = q/2, the word's four
// bytes are y = 4*(q&1) + 0..3, each byte's bits are z.  mn/mx are leaf-local.
__device__ __forceinline__ void word_bounds(uint32_t w, int q, int mn[3], int mx[3]) {
  if (!w) return;
  const int x = q >> 1, y0 = (q & 1) << 2;
  const uint32_t zor = (w | (w >> 8) | (w >> 16) | (w >> 24)) & 0xffu;
  mn[0] = min(mn[0], x);
  mx[0] = max(mx[0], x);
  mn[1] = min(mn[1], y0 + ((__ffs(w) - 1) >> 3));
  mx[1] = max(mx[1], y0 + ((31 - __clz(w)) >> 3));
  mn[2] = min(mn[2], __ffs(zor) - 1);
  mx[2] = max(mx[2], 31 - __clz(zor));
}

// Pass 1: count non-empty leaves (one atomic per block).  Pass 2: give each a compact index
// (block-wide scan, one atomic per block and iteration), copy its words, set its brick bit
// (one atomic per distinct brick word in a warp) and fold its voxels into the active bounding
// box and voxel count (reduced per block, one set of atomics per block).  One thread per leaf.
__global__ void __launch_bounds__(256) k_compact(SimBuild b, SimMapView v, uint32_t* count,
                                                 int pass2, int32_t* bbox,
                                                 unsigned long long* nvox) {
  __shared__ uint32_t s_warp[8];
  __shared__ uint32_t s_base;
  __shared__ int s_red[8][6];
  __shared__ unsigned long long s_cnt[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long total = (long long)b.ldim[0] * b.ldim[1] * b.ldim[2];
  const long long stride = (long long)gridDim.x * blockDim.x;
  const uint4* src = reinterpret_cast<const uint4*>(b.dense);
  int mn[3] = {INT_MAX, INT_MAX, INT_MAX}, mx[3] = {INT_MIN, INT_MIN, INT_MIN};
  unsigned long long cnt = 0;
  uint32_t nonempty = 0;
  // every thread runs the same number of iterations so the block-wide scan stays uniform
  for (long long base = (long long)blockIdx.x * blockDim.x; base < total; base += stride) {
    const long long pos = base + threadIdx.x;
    uint4 w[4] = {};
    if (pos < total) {
#pragma unroll
      for (int i = 0; i < 4; ++i) w[i] = __ldg(&src[pos * 4 + i]);
    }
    const bool any = (w[0].x | w[0].y | w[0].z | w[0].w | w[1].x | w[1].y | w[1].z | w[1].w |
                      w[2].x | w[2].y | w[2].z | w[2].w | w[3].x | w[3].y | w[3].z | w[3].w) != 0u;
    if (!pass2) {
      nonempty += any ? 1u : 0u;
      continue;
    }
    const unsigned ball = __ballot_sync(kFull, any);
    if (lane == 0) s_warp[warp] = __popc(ball);
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t sum = 0;
      for (int i = 0; i < 8; ++i) {
        const uint32_t c = s_warp[i];
        s_warp[i] = sum;
        sum += c;
      }
      s_base = sum ? atomicAdd(count, sum) : 0u;
    }
    __syncthreads();
    const uint32_t idx = s_base + s_warp[warp] + __popc(ball & ((1u << lane) - 1u));
    __syncthreads();  // s_warp / s_base are rewritten by the next iteration
    uint32_t bword = 0xffffffffu, bbit = 0u;
    if (any) {
      uint4* dst = reinterpret_cast<uint4*>(v.leaf_words) + (size_t)idx * 4;
#pragma unroll
      for (int i = 0; i < 4; ++i) dst[i] = w[i];
      v.leaf_index[pos] = (int32_t)idx;
      const int lz = (int)(pos % b.ldim[2]);
      const int ly = (int)((pos / b.ldim[2]) % b.ldim[1]);
      const int lx = (int)(pos / ((long long)b.ldim[2] * b.ldim[1]));
      const int bx = lx + b.llo[0], by = ly + b.llo[1], bz = lz + b.llo[2];
      const long long bpos = ((long long)((bx >> 3) - v.blo[0]) * v.bdim[1] + ((by >> 3) - v.blo[1])) *
                                 v.bdim[2] + ((bz >> 3) - v.blo[2]);
      bword = (uint32_t)(bpos >> 5);
      bbit = 1u << (bpos & 31);
      int lmn[3] = {8, 8, 8}, lmx[3] = {-1, -1, -1};
      const uint32_t ww[16] = {w[0].x, w[0].y, w[0].z, w[0].w, w[1].x, w[1].y, w[1].z, w[1].w,
                               w[2].x, w[2].y, w[2].z, w[2].w, w[3].x, w[3].y, w[3].z, w[3].w};
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        cnt += (unsigned)__popc(ww[q]);
        word_bounds(ww[q], q, lmn, lmx);
      }
      const int o[3] = {bx * 8, by * 8, bz * 8};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        mn[a] = min(mn[a], o[a] + lmn[a]);
        mx[a] = max(mx[a], o[a] + lmx[a]);
      }
    }
    // brick bits: lanes of one warp that hit the same word OR their bits, the lowest sets them
    const unsigned peers = __match_any_sync(kFull, bword);
    const uint32_t bits = __reduce_or_sync(peers, bbit);
    if (any && lane == __ffs(peers) - 1) atomicOr(&v.brick_bits[bword], bits);
  }
  if (!pass2) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nonempty += __shfl_xor_sync(kFull, nonempty, o);
    if (lane == 0 && nonempty) atomicAdd(count, nonempty);
    return;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    cnt += __shfl_xor_sync(kFull, cnt, o);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      mn[a] = min(mn[a], __shfl_xor_sync(kFull, mn[a], o));
      mx[a] = max(mx[a], __shfl_xor_sync(kFull, mx[a], o));
    }
  }
  if (lane == 0) {
    s_cnt[warp] = cnt;
    for (int a = 0; a < 3; ++a) {
      s_red[warp][a] = mn[a];
      s_red[warp][3 + a] = mx[a];
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long c = 0;
    int bmn[3] = {INT_MAX, INT_MAX, INT_MAX}, bmx[3] = {INT_MIN, INT_MIN, INT_MIN};
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      c += s_cnt[i];
      for (int a = 0; a < 3; ++a) {
        bmn[a] = min(bmn[a], s_red[i][a]);
        bmx[a] = max(bmx[a], s_red[i][3 + a]);
      }
    }
    if (c) {
      atomicAdd(nvox, c);
      for (int a = 0; a < 3; ++a) {
        atomicMin(&bbox[a], bmn[a]);
        atomicMax(&bbox[3 + a], bmx[a]);
      }
    }
  }
}

__global__ void k_fill_i32(int32_t* p, long long n, int32_t v) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    p[i] = v;
}

// ---- ray casting -----------------------------------------------------------------------------

__device__ __forceinline__ float plane_time(int p, float e, float inv) {
  return __fmul_rn(__fadd_rn((float)p, -e), inv);
}

__device__ __forceinline__ float plane_time_f(float p, float e, float inv) {
  return __fmul_rn(__fadd_rn(p, -e), inv);
}

// Crossed-before-exit predicate for a plane on axis j (see the file comment).
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

// 2 = empty brick (or outside the map), 1 = empty leaf, 0 = leaf with bits (*leaf = index).
__device__ __forceinline__ int sim_level(const SimMapView& v, int x, int y, int z, int* leaf) {
  const int bx = (x >> 6) - v.blo[0], by = (y >> 6) - v.blo[1], bz = (z >> 6) - v.blo[2];
  if ((unsigned)bx >= (unsigned)v.bdim[0] || (unsigned)by >= (unsigned)v.bdim[1] ||
      (unsigned)bz >= (unsigned)v.bdim[2])
    return 2;
  const long long bpos = ((long long)bx * v.bdim[1] + by) * v.bdim[2] + bz;
  if (!((__ldg(&v.brick_bits[bpos >> 5]) >> (bpos & 31)) & 1u)) return 2;
  const int lx = (x >> 3) - v.llo[0], ly = (y >> 3) - v.llo[1], lz = (z >> 3) - v.llo[2];
  if ((unsigned)lx >= (unsigned)v.ldim[0] || (unsigned)ly >= (unsigned)v.ldim[1] ||
      (unsigned)lz >= (unsigned)v.ldim[2])
    return 1;
  const int32_t li = __ldg(&v.leaf_index[((long long)lx * v.ldim[1] + ly) * v.ldim[2] + lz]);
  if (li < 0) return 1;
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
      const int S = lvl == 2 ? 64 : 8;
      int far[3];
      float T[3];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        if (st[a] == 0) {
          far[a] = k[a];
          T[a] = INFINITY;
        } else {
          far[a] = st[a] > 0 ? (k[a] | (S - 1)) : (k[a] & ~(S - 1));
          T[a] = plane_time(st[a] > 0 ? far[a] + 1 : far[a], eye[a], inv[a]);
        }
      }
      const int ax = (T[0] < T[1]) ? ((T[0] < T[2]) ? 0 : 2) : ((T[1] < T[2]) ? 1 : 2);
      const float Tx = T[ax];
      if (!(Tx <= t_out)) break;
      if (S > 1) {
#pragma unroll
        for (int a = 0; a < 3; ++a)
          if (a != ax && st[a] != 0)
            k[a] = advance_axis(k[a], far[a], st[a], eye[a], dir[a], inv[a], Tx, a > ax);
      }
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
  const float eye[3] = {__fdiv_rn(rp.pos[0], v.res), __fdiv_rn(rp.pos[1], v.res),
                        __fdiv_rn(rp.pos[2], v.res)};
  float tmin, tmax;
  if (rp.type == NM_SENSOR_FRUSTUM) {
    tmin = __fmul_rn(__fdiv_rn(rp.min_range, v.res), norm);
    tmax = __fmul_rn(__fdiv_rn(rp.max_range, v.res), norm);
  } else {
    tmin = __fdiv_rn(rp.min_range, v.res);
    tmax = __fdiv_rn(rp.max_range, v.res);
  }
  return sim_cast(v, eye, dir, tmin, tmax);
}

__global__ void __launch_bounds__(256) k_sim_render(SimMapView v, SimRayParams rp, float* out) {
  const int w = blockIdx.x * 16 + (threadIdx.x & 15);
  const int h = blockIdx.y * 16 + (threadIdx.x >> 4);
  if (w >= rp.width || h >= rp.height) return;
  out[(size_t)h * rp.width + w] = sim_ray(v, rp, w, h);
}

// Arbitrary rays (agent observation / collision rays): origins in metres, directions of any
// length (normalised here), first active voxel within max_range metres, else 0.
__global__ void __launch_bounds__(256) k_sim_cast(SimMapView v, const float* origins,
                                                  const float* dirs, long long n, float max_range,
                                                  float* out) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    float r = 0.0f;
    if (v.any) {
      const float m0 = __ldg(&dirs[3 * i]), m1 = __ldg(&dirs[3 * i + 1]), m2 = __ldg(&dirs[3 * i + 2]);
      const float norm = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(m0, m0), __fmul_rn(m1, m1)), __fmul_rn(m2, m2)));
      if (norm > 0.0f && norm < INFINITY) {
        float dir[3] = {__fdiv_rn(m0, norm), __fdiv_rn(m1, norm), __fdiv_rn(m2, norm)};
        const float eye[3] = {__fdiv_rn(__ldg(&origins[3 * i]), v.res),
                              __fdiv_rn(__ldg(&origins[3 * i + 1]), v.res),
                              __fdiv_rn(__ldg(&origins[3 * i + 2]), v.res)};
        r = sim_cast(v, eye, dir, 0.0f, __fdiv_rn(max_range, v.res));
      }
    }
    out[i] = r;
  }
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

__global__ void k_noise(float* r, long long n, float sigma_coef, float drop, uint64_t seed) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    r[i] = noisy(r[i], seed, i, sigma_coef, drop);
}

// Render and range noise in one pass: the same ranges as k_sim_render followed by k_noise.
__global__ void __launch_bounds__(256) k_sim_render_noisy(SimMapView v, SimRayParams rp, float* out,
                                                          float sigma_coef, float drop,
                                                          uint64_t seed) {
  const int w = blockIdx.x * 16 + (threadIdx.x & 15);
  const int h = blockIdx.y * 16 + (threadIdx.x >> 4);
  if (w >= rp.width || h >= rp.height) return;
  const long long i = (long long)h * rp.width + w;
  out[i] = noisy(sim_ray(v, rp, w, h), seed, i, sigma_coef, drop);
}

// All slots of a tick plan in one launch: one CTA per 16x16 tile of some slot.
__global__ void __launch_bounds__(256) k_sim_render_batch(const RenderBatch* b, SimMapView v) {
  __shared__ SimRayParams s_rp;
  __shared__ int s_slot;
  const uint32_t tile = blockIdx.x;
  if (threadIdx.x == 0) {
    int sl = 0;
    while (sl + 1 < b->n && b->tile_start[sl + 1] <= tile) ++sl;
    s_slot = sl;
  }
  __syncthreads();
  const int sl = s_slot;
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&b->rp[sl]);
    uint32_t* dst = reinterpret_cast<uint32_t*>(&s_rp);
    for (int i = threadIdx.x; i < (int)(sizeof(SimRayParams) / 4); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const uint32_t lt = tile - b->tile_start[sl];
  const int tx = (int)(lt % (uint32_t)b->tiles_x[sl]), ty = (int)(lt / (uint32_t)b->tiles_x[sl]);
  const int w = tx * 16 + (threadIdx.x & 15), h = ty * 16 + (threadIdx.x >> 4);
  if (w >= s_rp.width || h >= s_rp.height) return;
  float x = sim_ray(v, s_rp, w, h);
  const long long i = (long long)h * s_rp.width + w;
  if (b->noise) x = noisy(x, b->noise_seed[sl], i, b->noise_coef, b->drop);
  b->out[sl][i] = x;
}

}  // namespace

cudaError_t launch_voxelize(const SimBuild& b, const double* d_boxes, int nb, const double* d_cyl,
                            int nc, cudaStream_t s) {
  if (nb > 0) k_voxelize_boxes<<<dim3(16, nb), 256, 0, s>>>(b, d_boxes, nb);
  if (nc > 0) k_voxelize_cylinders<<<dim3(16, nc), 256, 0, s>>>(b, d_cyl, nc);
  return cudaGetLastError();
}

cudaError_t launch_set_voxels(const SimBuild& b, const int32_t* d_ijk, long long n, cudaStream_t s) {
  if (n > 0) k_set_voxels<<<1184, 256, 0, s>>>(b, d_ijk, n);
  return cudaGetLastError();
}

cudaError_t launch_compact(const SimBuild& b, const SimMapView& v, uint32_t* d_count, int pass2,
                           int32_t* d_bbox, unsigned long long* d_nvox, cudaStream_t s) {
  k_compact<<<1184, 256, 0, s>>>(b, v, d_count, pass2, d_bbox, d_nvox);
  return cudaGetLastError();
}

cudaError_t launch_fill_i32(int32_t* p, long long n, int32_t val, cudaStream_t s) {
  k_fill_i32<<<1184, 256, 0, s>>>(p, n, val);
  return cudaGetLastError();
}

cudaError_t launch_sim_render_noisy(const SimMapView& v, const SimRayParams& rp, float* out,
                                    float sigma_coef, float drop, uint64_t seed, cudaStream_t s) {
  const dim3 grid((rp.width + 15) / 16, (rp.height + 15) / 16);
  k_sim_render_noisy<<<grid, 256, 0, s>>>(v, rp, out, sigma_coef, drop, seed);
  return cudaGetLastError();
}

cudaError_t launch_sim_render(const SimMapView& v, const SimRayParams& rp, float* out, cudaStream_t s) {
  const dim3 grid((rp.width + 15) / 16, (rp.height + 15) / 16);
  k_sim_render<<<grid, 256, 0, s>>>(v, rp, out);
  return cudaGetLastError();
}

cudaError_t launch_sim_cast(const SimMapView& v, const float* origins, const float* dirs,
                            long long n, float max_range, float* out, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  const long long blocks = std::min<long long>((n + 255) / 256, 148 * 16);
  k_sim_cast<<<(unsigned)blocks, 256, 0, s>>>(v, origins, dirs, n, max_range, out);
  return cudaGetLastError();
}

cudaError_t launch_render_batch(const RenderBatch* d_batch, uint32_t total_tiles,
                                const SimMapView& v, cudaStream_t s) {
  if (total_tiles > 0) k_sim_render_batch<<<total_tiles, 256, 0, s>>>(d_batch, v);
  return cudaGetLastError();
}

cudaError_t launch_noise(float* r, long long n, float sigma_coef, float drop, uint64_t seed,
                         cudaStream_t s) {
  k_noise<<<1184, 256, 0, s>>>(r, n, sigma_coef, drop, seed);
  return cudaGetLastError();
}

}  // namespace nm
