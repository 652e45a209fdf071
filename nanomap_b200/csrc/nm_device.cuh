// nm_device.cuh -- device helpers for the sm_100a kernels: rounding-policy arithmetic, the
// leaf hash table, and the voxel DDA of the host insertion path.
#pragma once

#include <cfloat>
#include <cstdint>

#include "nm_internal.h"

namespace nm {

// Programmatic dependent launch.  A kernel launched with programmatic stream serialisation
// may start while the kernel before it on the stream still runs; it calls wait_prior_grid()
// before its first access to memory that kernel writes, which returns once that kernel has
// finished and its writes are visible.  allow_dependent_launch() tells the hardware that this
// CTA no longer needs to hold the dependent back.  Both are no-ops when the launch carries no
// dependency.
__device__ __forceinline__ void wait_prior_grid() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void allow_dependent_launch() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Arithmetic with an explicit rounding mode.  Every product and sum is rounded on its own
// (the intrinsics are never contracted into fused multiply-adds), so the device reproduces
// the CPU oracle bit for bit under the same policy.
template <int RM>
struct Ar;

template <>
struct Ar<NM_ROUND_NEAREST> {
  static __device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
  static __device__ __forceinline__ double drcp(double a) { return __drcp_rn(a); }
  static __device__ __forceinline__ double dsqrt(double a) { return __dsqrt_rn(a); }
};

template <>
struct Ar<NM_ROUND_DOWN> {
  static __device__ __forceinline__ float fmul(float a, float b) { return __fmul_rd(a, b); }
  static __device__ __forceinline__ float fadd(float a, float b) { return __fadd_rd(a, b); }
  static __device__ __forceinline__ double dmul(double a, double b) { return __dmul_rd(a, b); }
  static __device__ __forceinline__ double dadd(double a, double b) { return __dadd_rd(a, b); }
  static __device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rd(a, b); }
  static __device__ __forceinline__ double drcp(double a) { return __drcp_rd(a); }
  static __device__ __forceinline__ double dsqrt(double a) { return __dsqrt_rd(a); }
};

constexpr int kKindMiss = 0;
constexpr int kKindHit = 1;

// ---- leaf hash table ----------------------------------------------------------------------

// Find the slot of `key`, inserting it when absent.  Returns -1 (and sets kErrProbe) when the
// probe limit is reached.  Linear probing; the insert is a single 64-bit CAS, and a slot's
// leaf storage is zero from allocation, so no other thread ever waits on an insert.
__device__ __forceinline__ int map_find_or_insert(const MapView& m, unsigned long long key) {
  uint32_t h = hash_key(key) & m.mask;
  const uint32_t limit = m.capacity < kMaxProbe ? m.capacity : kMaxProbe;
  for (uint32_t probe = 0; probe < limit; ++probe) {
    const unsigned long long k = __ldcg(&m.keys[h]);
    if (k == key) return (int)h;
    if (k == kEmptyKey) {
      const unsigned long long old = atomicCAS(&m.keys[h], kEmptyKey, key);
      if (old == kEmptyKey) {
        atomicAdd(&m.ctr->leaf_count, 1u);
        return (int)h;
      }
      if (old == key) return (int)h;
    }
    h = (h + 1) & m.mask;
  }
  atomicOr(&m.ctr->error_flags, kErrProbe);
  return -1;
}

__device__ __forceinline__ int map_find(const MapView& m, unsigned long long key) {
  uint32_t h = hash_key(key) & m.mask;
  const uint32_t limit = m.capacity < kMaxProbe ? m.capacity : kMaxProbe;
  for (uint32_t probe = 0; probe < limit; ++probe) {
    const unsigned long long k = __ldcg(&m.keys[h]);
    if (k == key) return (int)h;
    if (k == kEmptyKey) return -1;
    h = (h + 1) & m.mask;
  }
  return -1;
}

// Put `slot` on the touched list once per epoch; record the label plane for batched ticks.
__device__ __forceinline__ void mark_touched(const MapView& m, int slot, uint32_t epoch,
                                             int plane) {
  if (m.plane_mask) atomicOr(&m.plane_mask[slot], 1u << plane);
  if (__ldcg(&m.epoch[slot]) != epoch) {
    if (atomicExch(&m.epoch[slot], epoch) != epoch) {
      const uint32_t i = atomicAdd(&m.ctr->touched_count, 1u);
      m.touched[i] = (uint32_t)slot;
    }
  }
}

// Shared-memory leaf table of one CTA: `smask + 1` entries of (key, 32 label words).
__device__ __forceinline__ int smem_find_or_insert(unsigned long long* s_keys, uint32_t smask,
                                                   unsigned long long key) {
  uint32_t h = hash_key(key) & smask;
  const uint32_t limit = (smask + 1) < 32u ? (smask + 1) : 32u;
  for (uint32_t i = 0; i < limit; ++i) {
    const unsigned long long k = ((volatile unsigned long long*)s_keys)[h];
    if (k == key) return (int)h;
    if (k == kEmptyKey) {
      const unsigned long long old = atomicCAS(&s_keys[h], kEmptyKey, key);
      if (old == kEmptyKey || old == key) return (int)h;
    }
    h = (h + 1) & smask;
  }
  return -1;
}

__device__ __forceinline__ int local_index(int x, int y, int z) {
  return ((x & 7) << 6) | ((y & 7) << 3) | (z & 7);
}

// ---- sensor-frame point of one pixel --------------------------------------------------------

// Range image -> sensor-frame point, round to nearest (same operation order as the oracle's
// orc_ranges_to_points).  Returns false for pixels without a return.
__device__ __forceinline__ bool range_point_r(const FrameParams& f, int w, int h, float r,
                                              float p[3]) {
  if (!(r > 0.0f)) return false;
  if (f.type == NM_SENSOR_FRUSTUM) {
    const float u = __fmul_rn((float)w, f.su);
    const float v = __fmul_rn((float)h, f.sv);
    const float dx = __fadd_rn(__fmul_rn(u, f.c0), -f.hw);
    const float dy = __fadd_rn(__fmul_rn(v, f.c1), -f.hh);
    const float n = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), 1.0f));
    const float sc = __fdiv_rn(r, n);
    p[0] = __fmul_rn(dx, sc);
    p[1] = __fmul_rn(dy, sc);
    p[2] = sc;
  } else {
    const float su = __ldg(&f.sinu[w]), cu = __ldg(&f.cosu[w]);
    const float sv = __ldg(&f.sinv[h]), cv = __ldg(&f.cosv[h]);
    p[0] = __fmul_rn(__fmul_rn(su, cv), r);
    p[1] = __fmul_rn(sv, r);
    p[2] = __fmul_rn(__fmul_rn(cu, cv), r);
  }
  return true;
}

__device__ __forceinline__ bool range_point(const FrameParams& f, int w, int h, float p[3]) {
  return range_point_r(f, w, h, __ldg(&f.ranges[(size_t)h * f.width + w]), p);
}

__device__ __forceinline__ bool xyz_point(const FrameParams& f, int w, int h, float p[3]) {
  const unsigned char* rec = f.xyz + ((size_t)h * f.width + w) * (size_t)f.step;
  // records of 16 bytes or a multiple, 16-byte aligned: one 16-byte load (within the record,
  // so never past the input's end; one request where the input is read over the host link)
  if (((f.step & 15) | (int)(((uintptr_t)rec) & 15u)) == 0) {
    const float4 q = __ldg(reinterpret_cast<const float4*>(rec));
    p[0] = q.x;
    p[1] = q.y;
    p[2] = q.z;
  } else if ((((uintptr_t)rec) & 3u) == 0) {
    const float* q = reinterpret_cast<const float*>(rec);
    p[0] = __ldg(q);
    p[1] = __ldg(q + 1);
    p[2] = __ldg(q + 2);
  } else {
    uint32_t b[3];
    for (int c = 0; c < 3; ++c) {
      b[c] = (uint32_t)__ldg(rec + 4 * c) | ((uint32_t)__ldg(rec + 4 * c + 1) << 8) |
             ((uint32_t)__ldg(rec + 4 * c + 2) << 16) | ((uint32_t)__ldg(rec + 4 * c + 3) << 24);
      p[c] = __uint_as_float(b[c]);
    }
  }
  return true;
}

// ---- the insertion DDA (Handler.cpp:58-85) ---------------------------------------------------
//
// Rotate the sensor-frame point (float), take its length in double, drop it when
// |R p| / res >= max_time (NaN and Inf fall out here too), normalise, and walk the voxel DDA
// from the index-space eye over [0, ray_length].  Every voxel left by a step is reported as
// a miss; the voxel holding the end point is reported as a hit when the DDA time (the
// crossing that left it) is below max_time.  Step axis = smallest next crossing, ties to the
// higher axis; a zero direction component disables its axis.  Returns the number of label
// events, or -1 when the point was dropped.
template <int RM, class Emit>
__device__ __forceinline__ int trace_point(const FrameParams& f, float px, float py, float pz,
                                           Emit& emit) {
  using A = Ar<RM>;
  const float* R = f.R;
  const float dxf = A::fadd(A::fadd(A::fmul(R[0], px), A::fmul(R[1], py)), A::fmul(R[2], pz));
  const float dyf = A::fadd(A::fadd(A::fmul(R[3], px), A::fmul(R[4], py)), A::fmul(R[5], pz));
  const float dzf = A::fadd(A::fadd(A::fmul(R[6], px), A::fmul(R[7], py)), A::fmul(R[8], pz));
  const double dx = dxf, dy = dyf, dz = dzf;
  const double len = A::dsqrt(A::dadd(A::dadd(A::dmul(dx, dx), A::dmul(dy, dy)), A::dmul(dz, dz)));
  const double ray_len = A::ddiv(len, f.res_d);
  if (!(ray_len < (double)f.max_time)) return -1;
  if (!(len > 1.0e-7)) return -1;
  const double inv_len = A::drcp(len);
  const double n0 = A::dmul(dx, inv_len), n1 = A::dmul(dy, inv_len), n2 = A::dmul(dz, inv_len);

  int v0 = (int)floor(f.eye[0]), v1 = (int)floor(f.eye[1]), v2 = (int)floor(f.eye[2]);
  double t0n, t1n, t2n, d0, d1, d2;
  int s0, s1, s2;
#define NM_AXIS_INIT(nd, v, e, tn, d, s)                               \
  if (nd == 0.0) {                                                     \
    s = 0;                                                             \
    tn = DBL_MAX;                                                      \
    d = DBL_MAX;                                                       \
  } else {                                                             \
    const double inv = A::drcp(nd);                                    \
    if (inv > 0.0) {                                                   \
      s = 1;                                                           \
      tn = A::dmul(A::dadd((double)(v + 1), -(e)), inv);               \
      d = inv;                                                         \
    } else {                                                           \
      s = -1;                                                          \
      tn = A::dmul(A::dadd((double)(v), -(e)), inv);                   \
      d = -inv;                                                        \
    }                                                                  \
  }
  NM_AXIS_INIT(n0, v0, f.eye[0], t0n, d0, s0)
  NM_AXIS_INIT(n1, v1, f.eye[1], t1n, d1, s1)
  NM_AXIS_INIT(n2, v2, f.eye[2], t2n, d2, s2)
#undef NM_AXIS_INIT
  int c0 = v0, c1 = v1, c2 = v2;
  double t;
  int n = 0;
  for (;;) {
    const int a = (t0n < t1n) ? ((t0n < t2n) ? 0 : 2) : ((t1n < t2n) ? 1 : 2);
    if (a == 0) {
      t = t0n;
      t0n = A::dadd(t0n, d0);
      v0 += s0;
    } else if (a == 1) {
      t = t1n;
      t1n = A::dadd(t1n, d1);
      v1 += s1;
    } else {
      t = t2n;
      t2n = A::dadd(t2n, d2);
      v2 += s2;
    }
    if (!(t <= ray_len)) break;
    emit(c0, c1, c2, kKindMiss);
    ++n;
    c0 = v0;
    c1 = v1;
    c2 = v2;
  }
  if (t < (double)f.max_time) {
    emit(c0, c1, c2, kKindHit);
    ++n;
  }
  return n;
}

}  // namespace nm
