// nm_traverse.cu -- persistent traversal + per-frame labelling kernel (sm_100a).
//
// Replaces nodePassHDDA / voxelPassHDDA and the CUB compaction between them
// (frustumCastCloud.cu:44-246): one pass walks every ray voxel by voxel with the insertion
// DDA of Handler.cpp:58-85 and records one label per voxel (hit overrides miss), allocating
// map leaves on the fly.
//
// Work distribution: CTAs stay resident and take tiles of neighbouring pixels from a device
// counter, so the cost of a tile (set by its longest rays) no longer decides when an SM goes
// idle.  A tile holds one or more rays per thread.  Before the walk the tile's rays are
// ordered by range (a counting sort on 32 range buckets, longest first), so the 32 lanes of a
// warp walk rays of about the same length and finish together; with several rays per
// thread the rounds alternate direction, so every warp gets long and short rays.
//
// Per step the walk compares the three crossing times (non-negative doubles, one compare per
// pair, ties to the higher axis), advances the chosen axis with one rounded double add, and
// keeps the voxel as (leaf code, index inside the leaf).  The leaf code lx*2^20 + ly*2^10 + lz
// (mod 2^32) moves by one add per leaf crossing and is one-to-one over every leaf a frame can
// reach while max_range / res stays below kNarrowMaxTime voxels; it is both the tag and the
// hash source of a per-CTA shared-memory leaf table (32 label words per leaf).  A leaf that
// finds no room in the table goes straight to the device table.
//
// Labels collect per 32-voxel word in a register and go to shared memory with one shared atomic
// when the walk leaves the word (reading the word first to skip atomics that add no bits was
// measured slower: the read costs more than the atomics it saves).  After a
// tile, one lane per cached leaf ORs its words into the device label buffer and puts the leaf
// on the touched list (the device-table lookups of a warp's leaves overlap).
//
// Frames whose reach exceeds the code's range (max_range / res >= kNarrowMaxTime) take
// k_traverse_wide: one thread per ray with device-table lookups and label atomics.
//
// k_traverse_render renders each tile's ranges from the sim map into shared memory first
// (nm_sim_insert), so one launch does the simulated frame and its insertion.
#include <cfloat>
#include <climits>
#include <algorithm>
#include <cstdint>
#include <mutex>

#include "nm_device.cuh"
#include "nm_internal.h"
#include "nm_sim_device.cuh"

namespace nm {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kSortBuckets = 32;
// Word index of a leaf whose labels were lost (device table full): flushes skip it.
constexpr int kLostWord = INT_MIN;
// Word indices at or above kGlobFloor and below 0 name a device-table leaf g as
// -(g + 1) * 16 + w (w = miss word 0..15); capacities are at most 2^26 slots.
constexpr int kGlobFloor = -(1 << 30);

__device__ __forceinline__ uint32_t leaf_code(int lx, int ly, int lz) {
  return ((uint32_t)lx << 20) + ((uint32_t)ly << 10) + (uint32_t)lz;
}

// Table position of a leaf code: Fibonacci hashing, top bits (`sh` = 32 - log2 entries).
__device__ __forceinline__ uint32_t code_slot(uint32_t code, int sh) {
  return (code * 0x9E3779B1u) >> sh;
}

__device__ __forceinline__ int sext(uint32_t v, int bits) {
  return (int)(v << (32 - bits)) >> (32 - bits);
}

// Absolute leaf key of a code near the eye's leaf (every reachable leaf lies within 511 leaves
// of it on each axis, where the code is one-to-one).
__device__ __forceinline__ unsigned long long code_key(uint32_t code, uint32_t ecode, int elx,
                                                       int ely, int elz) {
  const uint32_t c = code - ecode;  // dx*2^20 + dy*2^10 + dz (mod 2^32)
  const int dz = sext(c & 0x3FFu, 10);
  const uint32_t c1 = (c - (uint32_t)dz) >> 10;
  const int dy = sext(c1 & 0x3FFu, 10);
  const int dx = sext(((c1 - (uint32_t)dy) >> 10) & 0xFFFu, 12);
  return leaf_key(elx + dx, ely + dy, elz + dz);
}

// Per-tile constants of the shared leaf table.
struct TileTable {
  unsigned long long* keys;  // absolute key per entry (valid where tags != sentinel)
  uint32_t* tags;            // leaf code per entry, `sentinel` = empty
  uint32_t* words;           // 32 label words per entry: 0..15 hit, 16..31 miss
  uint32_t smask;
  int sh;
  uint32_t sentinel;
  uint32_t ecode;
  int elx, ely, elz;
};

// Probe / insert of a code the inline probe missed.  Returns the miss-word base of the leaf:
// e * 32 + 16 for table entry e, -(g + 1) * 16 for device-table slot g, kLostWord when the
// device table is full.
__device__ __noinline__ int leaf_base_slow(const TileTable& tt, const MapView& m, uint32_t code,
                                           uint32_t epoch, int plane) {
  uint32_t h = code_slot(code, tt.sh);
  const uint32_t limit = (tt.smask + 1) < 16u ? (tt.smask + 1) : 16u;
  for (uint32_t i = 0; i < limit; ++i) {
    const uint32_t k = ((volatile uint32_t*)tt.tags)[h];
    if (k == code) return (int)(h * kLabelWords + 16);
    if (k == tt.sentinel) {
      const uint32_t old = atomicCAS(&tt.tags[h], tt.sentinel, code);
      if (old == tt.sentinel) {
        tt.keys[h] = code_key(code, tt.ecode, tt.elx, tt.ely, tt.elz);
        return (int)(h * kLabelWords + 16);
      }
      if (old == code) return (int)(h * kLabelWords + 16);
    }
    h = (h + 1) & tt.smask;
  }
  const int g = map_find_or_insert(m, code_key(code, tt.ecode, tt.elx, tt.ely, tt.elz));
  if (g < 0) return kLostWord;
  mark_touched(m, g, epoch, plane);
  return -(g + 1) * 16;
}

__device__ __forceinline__ int leaf_base(const TileTable& tt, const MapView& m, uint32_t code,
                                         uint32_t epoch, int plane) {
  const uint32_t e = code_slot(code, tt.sh);
  if (((volatile uint32_t*)tt.tags)[e] == code) return (int)(e * kLabelWords + 16);
  return leaf_base_slow(tt, m, code, epoch, plane);
}

// OR `bits` into label word `cw` (a table word, a device-table miss word, or lost).
__device__ __noinline__ void flush_device_word(const MapView& m, int cw, uint32_t bits, int plane) {
  if (cw < kGlobFloor) return;
  const uint32_t x = (uint32_t)(-cw - 1);
  const uint32_t g = x >> 4, w = 15u - (x & 15u);
  atomicOr(&m.labels[((size_t)plane * m.capacity + g) * kLabelWords + 16 + w], bits);
}

__device__ __forceinline__ void flush_word(uint32_t* s_words, const MapView& m, int cw,
                                           uint32_t bits, int plane) {
  if (cw >= 0)
    atomicOr(&s_words[cw], bits);
  else
    flush_device_word(m, cw, bits, plane);
}

// Hit label of voxel `l` of the leaf whose miss-word base is `wbase`.
__device__ __noinline__ void hit_device(const MapView& m, int wbase, int l, int plane) {
  if (wbase < kGlobFloor) return;
  const uint32_t g = (uint32_t)(-wbase / 16 - 1);
  atomicOr(&m.labels[((size_t)plane * m.capacity + g) * kLabelWords + (l >> 5)], 1u << (l & 31));
}

struct Ray {
  double t0, t1, t2;  // next crossing time per axis (never negative)
  double d0, d1, d2;  // crossing spacing per axis
  double len;         // ray length in voxels
  int ds0, ds1, ds2;  // step of the voxel index inside the leaf per axis: +-64, +-8, +-1 or 0
  int l;              // voxel index inside the leaf, x*64 + y*8 + z
  uint32_t hs0, hs1, hs2;  // leaf-code step per axis: +-2^20, +-2^10, +-1 or 0
  uint32_t code;           // leaf code of the current voxel
};

// Ray set-up of the insertion DDA (Handler.cpp:64-76 restated; see trace_point in
// nm_device.cuh for the same arithmetic in one piece).  Returns false when the point is
// dropped (beyond range, NaN/Inf, shorter than 1e-7).
template <int RM>
__device__ __forceinline__ bool setup_ray(const FrameParams& f, const float p[3], Ray& r) {
  using A = Ar<RM>;
  const float* R = f.R;
  const float dxf = A::fadd(A::fadd(A::fmul(R[0], p[0]), A::fmul(R[1], p[1])), A::fmul(R[2], p[2]));
  const float dyf = A::fadd(A::fadd(A::fmul(R[3], p[0]), A::fmul(R[4], p[1])), A::fmul(R[5], p[2]));
  const float dzf = A::fadd(A::fadd(A::fmul(R[6], p[0]), A::fmul(R[7], p[1])), A::fmul(R[8], p[2]));
  const double dx = dxf, dy = dyf, dz = dzf;
  const double len = A::dsqrt(A::dadd(A::dadd(A::dmul(dx, dx), A::dmul(dy, dy)), A::dmul(dz, dz)));
  const double ray_len = A::ddiv(len, f.res_d);
  if (!(ray_len < (double)f.max_time)) return false;
  if (!(len > 1.0e-7)) return false;
  r.len = ray_len;
  const double inv_len = A::drcp(len);
  const double nd[3] = {A::dmul(dx, inv_len), A::dmul(dy, inv_len), A::dmul(dz, inv_len)};
  double tn[3], dl[3];
  int st[3], v[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    v[a] = (int)floor(f.eye[a]);
    if (nd[a] == 0.0) {
      st[a] = 0;
      tn[a] = DBL_MAX;
      dl[a] = DBL_MAX;
    } else {
      const double inv = A::drcp(nd[a]);
      if (inv > 0.0) {
        st[a] = 1;
        tn[a] = A::dmul(A::dadd((double)(v[a] + 1), -f.eye[a]), inv);
        dl[a] = inv;
      } else {
        st[a] = -1;
        tn[a] = A::dmul(A::dadd((double)v[a], -f.eye[a]), inv);
        dl[a] = -inv;
      }
      if (tn[a] == 0.0) tn[a] = 0.0;  // canonical +0
    }
  }
  r.t0 = tn[0];
  r.t1 = tn[1];
  r.t2 = tn[2];
  r.d0 = dl[0];
  r.d1 = dl[1];
  r.d2 = dl[2];
  r.ds0 = st[0] * 64;
  r.ds1 = st[1] * 8;
  r.ds2 = st[2];
  r.hs0 = (uint32_t)st[0] << 20;
  r.hs1 = (uint32_t)st[1] << 10;
  r.hs2 = (uint32_t)st[2];
  r.l = ((v[0] & 7) << 6) | ((v[1] & 7) << 3) | (v[2] & 7);
  r.code = leaf_code(v[0] >> 3, v[1] >> 3, v[2] >> 3);
  return true;
}

__device__ __forceinline__ bool pixel_point(const FrameParams& f, int w, int h, float p[3]) {
  if (f.input_kind == 1) return range_point(f, w, h, p);
  if (f.input_kind == 2 && (uint32_t)(h * f.width + w) >= __ldg(f.n_valid)) return false;
  return xyz_point(f, w, h, p);
}

// Walk one ray from its set-up to its end, labelling every voxel it leaves as a miss and its
// end voxel as a hit (when the crossing that leaves it lies below max_time).  Returns the
// number of label events.
template <int RM>
__device__ __forceinline__ uint32_t walk_ray(const Ray& r, const TileTable& tt, const MapView& m,
                                             double max_time, uint32_t epoch, int plane) {
  using A = Ar<RM>;
  double t0 = r.t0, t1 = r.t1, t2 = r.t2;
  const double d0 = r.d0, d1 = r.d1, d2 = r.d2, len = r.len;
  int l = r.l;
  uint32_t code = r.code;
  int wbase = leaf_base(tt, m, code, epoch, plane);
  int cw = kLostWord;  // word the pending bits belong to
  uint32_t acc = 0u;   // pending miss bits of word cw
  uint32_t n = 0u;
  double t;
  for (;;) {
    const bool c01 = t0 < t1, c02 = t0 < t2, c12 = t1 < t2;
    const bool is0 = c01 && c02;
    const bool is1 = !c01 && c12;
    t = is0 ? t0 : (is1 ? t1 : t2);
    if (!(t <= len)) break;
    // miss label of the voxel being left
    const int wi = wbase + (l >> 5);
    if (wi != cw) {
      // acc holds at least the bit of the step that set cw (none only for the initial
      // kLostWord, which flush_device_word drops)
      if (cw >= 0)
        atomicOr(&tt.words[cw], acc);
      else
        flush_device_word(m, cw, acc, plane);
      cw = wi;
      acc = 0u;
    }
    acc |= 1u << (l & 31);
    ++n;
    // advance along the chosen axis: crossing time, index inside the leaf, leaf on wrap
    const double dstep = is0 ? d0 : (is1 ? d1 : d2);
    const double tn = A::dadd(t, dstep);
    if (is0) t0 = tn;
    if (is1) t1 = tn;
    if (!is0 && !is1) t2 = tn;
    const int msk = is0 ? 0x1C0 : (is1 ? 0x38 : 0x7);
    const int ds = is0 ? r.ds0 : (is1 ? r.ds1 : r.ds2);
    const int vv = (l & msk) + ds;
    l = (l & ~msk) | (vv & msk);
    if ((unsigned)vv > (unsigned)msk) {
      code += is0 ? r.hs0 : (is1 ? r.hs1 : r.hs2);
      wbase = leaf_base(tt, m, code, epoch, plane);
    }
  }
  if (acc) flush_word(tt.words, m, cw, acc, plane);
  if (t < max_time) {
    if (wbase >= 0)
      atomicOr(&tt.words[wbase - 16 + (l >> 5)], 1u << (l & 31));
    else
      hit_device(m, wbase, l, plane);
    ++n;
  }
  return n;
}

// Range bucket of a pixel for the tile's ray order: 0 = longest rays, kSortBuckets - 1 =
// shortest and rays without a return.
// `qs` = kSortBuckets / max_range (metres): the bucket is the range's fraction of max range.
__device__ __forceinline__ int range_bucket(float r_m, float qs) {
  if (!(r_m > 0.0f)) return kSortBuckets - 1;
  const float q = r_m * qs;
  const int k = q < (float)kSortBuckets ? (int)q : kSortBuckets - 1;
  return kSortBuckets - 1 - k;
}

template <int RM, int MaxF, bool Render = false>
__device__ __forceinline__ void traverse_body(const TickWork<MaxF>& work, const MapView& m,
                                              const SimRender* sr = nullptr) {
  extern __shared__ __align__(16) unsigned char smem[];
  const uint32_t smask = work.smask;
  const int nent = (int)smask + 1;
  const int nrays = work.tile_w * work.tile_h;
  unsigned long long* s_keys = reinterpret_cast<unsigned long long*>(smem);
  uint32_t* s_words = reinterpret_cast<uint32_t*>(s_keys + nent);
  uint32_t* s_tags = s_words + nent * kLabelWords;
  uint16_t* s_order = reinterpret_cast<uint16_t*>(s_tags + nent);
  uint8_t* s_bkt = reinterpret_cast<uint8_t*>(s_order + nrays);
  // the tile's sensor-frame points, computed once by the range sort; x = NaN for a pixel
  // without a point
  float* s_pts = reinterpret_cast<float*>(s_bkt + nrays);
  __shared__ FrameParams s_f;
  __shared__ uint32_t s_tile;
  __shared__ int s_frame;
  __shared__ uint32_t s_hist[kSortBuckets];
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int nthreads = blockDim.x;
  const int rounds = nrays / nthreads;
  uint32_t visits = 0, rays = 0;
  wait_prior_grid();
  // claim order: the first tiles of the queue are those of bucket 0 (longest walks), ...
  __shared__ uint32_t s_pre[kOrderBuckets + 1];
  if (work.order_counts) {
    if (tid < 32) {
      const uint32_t c0 = __ldcg(&work.order_counts[2 * lane]);
      const uint32_t c1 = __ldcg(&work.order_counts[2 * lane + 1]);
      uint32_t incl = c0 + c1;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += u;
      }
      s_pre[2 * lane] = incl - c0 - c1;
      s_pre[2 * lane + 1] = incl - c1;
      if (lane == 31) s_pre[kOrderBuckets] = incl;
    }
    __syncthreads();
  }

  for (;;) {
    if (tid == 0) {
      unsigned int* queue = &m.ctr->tile_queue;
      const uint32_t t = atomicAdd(queue, 1u);
      uint32_t tl = t;
      if (work.order_counts && t < s_pre[kOrderBuckets]) {
        int lo = 0, hi = kOrderBuckets - 1;  // the bucket b with s_pre[b] <= t < s_pre[b + 1]
        while (lo < hi) {
          const int mid = (lo + hi + 1) >> 1;
          if (s_pre[mid] <= t) lo = mid; else hi = mid - 1;
        }
        tl = __ldcg(&work.order_lists[(size_t)lo * work.order_cap + (t - s_pre[lo])]);
      }
      int fi = 0;
      while (fi + 1 < work.n_frames && work.tile_start[fi + 1] <= tl) ++fi;
      s_tile = tl;
      s_frame = fi;
      if (t == work.total_tiles + gridDim.x - 1) {  // last reader resets
        *queue = 0u;
        // every CTA read the counts before its first claim: clear them for the next pass
        if (work.order_counts)
          for (int b = 0; b < kOrderBuckets; ++b) work.order_counts[b] = 0u;
      }
    }
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= work.total_tiles) {
      allow_dependent_launch();  // the integration may start its CTAs on freed SMs
      break;
    }
    const int fi = s_frame;
    {
      const uint32_t* src = reinterpret_cast<const uint32_t*>(&work.fr[fi]);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&s_f);
      for (int i = tid; i < (int)(sizeof(FrameParams) / 4); i += nthreads) dst[i] = src[i];
    }
    if (tid < kSortBuckets) s_hist[tid] = 0u;
    __syncthreads();
    const FrameParams& f = s_f;
    const uint32_t lt = tile - work.tile_start[fi];
    const int tx = (int)(lt % (uint32_t)work.tiles_x[fi]);
    const int ty = (int)(lt / (uint32_t)work.tiles_x[fi]);
    const int x0 = tx * work.tile_w, y0 = ty * work.tile_h;
    // packed records (input kind 2) fill the first tiles only: later tiles have no work
    if (f.input_kind == 2 && (uint32_t)(y0 * f.width + x0) >= __ldg(f.n_valid)) {
      __syncthreads();
      continue;
    }
    TileTable tt;
    tt.keys = s_keys;
    tt.tags = s_tags;
    tt.words = s_words;
    tt.smask = smask;
    tt.sh = __clz((int)smask);
    tt.elx = (int)floor(f.eye[0]) >> 3;
    tt.ely = (int)floor(f.eye[1]) >> 3;
    tt.elz = (int)floor(f.eye[2]) >> 3;
    tt.ecode = leaf_code(tt.elx, tt.ely, tt.elz);
    tt.sentinel = tt.ecode + (1536u << 20);  // the code of no leaf within reach
    for (int i = tid; i < nent; i += nthreads) s_tags[i] = tt.sentinel;
    for (int i = tid; i < nent * kLabelWords; i += nthreads) s_words[i] = 0u;

    // the tile's ranges (Render: from the sim map, with the range noise), bucketed by length;
    // every thread runs the same number of iterations (nrays is a multiple of the block)
    const float qs = (float)kSortBuckets / (f.max_time * (float)f.res_d);
    const bool spread = f.type == NM_SENSOR_LASER;
    for (int k = tid; k < nrays; k += nthreads) {
      const int px = x0 + k % work.tile_w, py = y0 + k / work.tile_w;
      float rm = 0.0f;  // range in metres, 0 = no point
      float p[3] = {__int_as_float(0x7fffffff), 0.0f, 0.0f};
      if (px < f.width && py < f.height) {
        bool ok;
        if constexpr (Render) {
          float rr = sim_ray(sr->v, sr->rp, px, py);
          const long long i = (long long)py * f.width + px;
          if (sr->noise) rr = noisy(rr, sr->seed, i, sr->sigma_coef, sr->drop);
          if (sr->out) sr->out[i] = rr;
          rm = rr;
          ok = range_point_r(f, px, py, rr, p);
        } else if (f.input_kind == 1) {
          rm = __ldg(&f.ranges[(size_t)py * f.width + px]);
          ok = range_point_r(f, px, py, rm, p);
        } else {
          ok = pixel_point(f, px, py, p);
          if (ok) rm = sqrtf(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
        }
        if (!ok) p[0] = __int_as_float(0x7fffffff);
      }
      s_pts[3 * k] = p[0];
      s_pts[3 * k + 1] = p[1];
      s_pts[3 * k + 2] = p[2];
      const int b = range_bucket(rm, qs);
      s_bkt[k] = (uint8_t)b;
      const unsigned peers = __match_any_sync(kFull, b);
      if (lane == __ffs(peers) - 1) atomicAdd(&s_hist[b], (uint32_t)__popc(peers));
    }
    __syncthreads();
    if (tid < 32) {  // exclusive prefix over the buckets
      const uint32_t v = s_hist[lane];
      uint32_t incl = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t u = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += u;
      }
      s_hist[lane] = incl - v;
    }
    __syncthreads();
    for (int k = tid; k < nrays; k += nthreads) {
      const int b = s_bkt[k];
      const unsigned peers = __match_any_sync(kFull, b);
      const int leader = __ffs(peers) - 1;
      uint32_t base = 0;
      if (lane == leader) base = atomicAdd(&s_hist[b], (uint32_t)__popc(peers));
      base = __shfl_sync(peers, base, leader);
      const int q = base + __popc(peers & ((1u << lane) - 1u));  // rank, longest first
      // one ray per thread: thread t walks the ray at s_order[t], so warp w gets ranks
      // 32w..32w+31 (rays of about one length per warp: best for camera frames); for a laser
      // frame ranks w, w + W, w + 2W, ... (W warps: every warp gets rays of all lengths; a
      // spinning sensor's tile mixes ground hits with far walls and its few tiles leave SMs
      // idle, so spreading the long rays over the warps wins: 0.32 against 0.46 ms for a
      // 64x1024 frame at 20 m)
      const int nw = nthreads >> 5;
      s_order[(spread && rounds == 1) ? (q % nw) * 32 + q / nw : q] = (uint16_t)k;
    }
    __syncthreads();

    const int plane = f.plane;
    const uint32_t epoch = f.epoch;
    const double max_time = (double)f.max_time;
    for (int j = 0; j < rounds; ++j) {
      // alternate directions so every warp gets long and short rays
      const int pos = (j & 1) ? (j + 1) * nthreads - 1 - tid : j * nthreads + tid;
      const int k = s_order[pos];
      const float p[3] = {s_pts[3 * k], s_pts[3 * k + 1], s_pts[3 * k + 2]};
      Ray r;
      if (!isnan(p[0]) && setup_ray<RM>(f, p, r)) {
        rays += 1;
        visits += walk_ray<RM>(r, tt, m, max_time, epoch, plane);
      }
    }
    __syncthreads();

    // Flush the tile's leaf table: one lane per cached leaf, so the device-table lookups of
    // up to 32 leaves overlap; word reads are rotated by lane to avoid bank conflicts.
    for (int e = tid; e < nent; e += nthreads) {
      if (s_tags[e] == tt.sentinel) continue;
      const uint32_t* sw = s_words + e * kLabelWords;
      bool has = false;
#pragma unroll 4
      for (int w = 0; w < kLabelWords; ++w) has |= sw[(w + lane) & (kLabelWords - 1)] != 0u;
      if (!has) continue;
      const int g = map_find_or_insert(m, s_keys[e]);
      if (g < 0) continue;
      mark_touched(m, g, epoch, plane);
      uint32_t* dst = &m.labels[((size_t)plane * m.capacity + (size_t)g) * kLabelWords];
#pragma unroll 4
      for (int w = 0; w < kLabelWords; ++w) {
        const int wr = (w + lane) & (kLabelWords - 1);
        const uint32_t word = sw[wr];
        if (word) atomicOr(&dst[wr], word);
      }
    }
    __syncthreads();
  }

  unsigned long long vv = visits, rr = rays;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    vv += __shfl_xor_sync(kFull, vv, o);
    rr += __shfl_xor_sync(kFull, rr, o);
  }
  if (lane == 0 && (vv | rr)) {
    atomicAdd(&m.ctr->visits, vv);
    atomicAdd(&m.ctr->rays, rr);
  }
}

// ---- tile order (longest walks first) --------------------------------------------------------
//
// A frame's walk is bounded by its longest rays: a step costs a warp ~70 instructions issued
// at one per ~11 cycles while the SM's other warps run, so a 350-step ray takes most of a
// frame's traversal.  Claiming the tiles in decreasing order of their longest ray starts those
// rays first.  One CTA per tile takes the largest |R p|_1 / res over the tile's rays (the
// DDA's step count up to rounding) plus kSetupSteps, scales it to one of kOrderBuckets
// buckets, and appends the tile to that bucket's list (order inside a bucket is arbitrary).
constexpr float kSetupSteps = 8.0f;
constexpr int kOrderThreads = 128;

template <int MaxF>
__device__ __forceinline__ void tile_order_body(const TickWork<MaxF>& work, TileOrderBuffers b) {
  allow_dependent_launch();  // the walk's CTAs launch now and wait for this pass to finish
  // one CTA per tile, one thread per ray: every record load of the tile is in flight at once
  const uint32_t tile = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31;
  const int nrays = work.tile_w * work.tile_h;
  int fi = 0;
  while (fi + 1 < work.n_frames && work.tile_start[fi + 1] <= tile) ++fi;
  const FrameParams& f = work.fr[fi];
  const uint32_t lt = tile - work.tile_start[fi];
  const int x0 = (int)(lt % (uint32_t)work.tiles_x[fi]) * work.tile_w;
  const int y0 = (int)(lt / (uint32_t)work.tiles_x[fi]) * work.tile_h;
  const float inv_res = (float)(1.0 / f.res_d);
  float longest = 0.0f;
  for (int k = tid; k < nrays; k += kOrderThreads) {
    const int px = x0 + k % work.tile_w, py = y0 + k / work.tile_w;
    float p[3];
    if (px < f.width && py < f.height && pixel_point(f, px, py, p)) {
      const float* R = f.R;
      const float x = R[0] * p[0] + R[1] * p[1] + R[2] * p[2];
      const float y = R[3] * p[0] + R[4] * p[1] + R[5] * p[2];
      const float z = R[6] * p[0] + R[7] * p[1] + R[8] * p[2];
      const float len = sqrtf(x * x + y * y + z * z) * inv_res;
      if (len < f.max_time)
        longest = fmaxf(longest, (fabsf(x) + fabsf(y) + fabsf(z)) * inv_res + kSetupSteps);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) longest = fmaxf(longest, __shfl_xor_sync(kFull, longest, o));
  __shared__ float s_max[kOrderThreads / 32];
  if (lane == 0) s_max[tid >> 5] = longest;
  __syncthreads();
  if (tid == 0) {
#pragma unroll
    for (int w = 1; w < kOrderThreads / 32; ++w) longest = fmaxf(longest, s_max[w]);
    const float q = longest * work.order_scale;
    const int bkt = kOrderBuckets - 1 - (q < (float)(kOrderBuckets - 1) ? (int)q : kOrderBuckets - 1);
    const uint32_t r = atomicAdd(&b.counts[bkt], 1u);
    if (r < b.capacity) b.lists[(size_t)bkt * b.capacity + r] = tile;
  }
}

template <int MaxF>
__global__ void __launch_bounds__(kOrderThreads) k_tile_order(const __grid_constant__ TickWork<MaxF> work,
                                                              TileOrderBuffers b) {
  tile_order_body<MaxF>(work, b);
}

__global__ void __launch_bounds__(kOrderThreads) k_tile_order_dev(const TickWork<kMaxTickFrames>* work,
                                                                  TileOrderBuffers b) {
  tile_order_body<kMaxTickFrames>(*work, b);
}

int order_grid(uint32_t total_tiles) { return (int)total_tiles; }

// Label sink of the wide-frame kernel: device-table lookups on leaf changes, one atomic per
// new label bit.
struct WideEmit {
  const MapView* m;
  uint32_t epoch;
  int plane;
  unsigned long long ckey;
  int cslot;

  __device__ __forceinline__ void operator()(int x, int y, int z, int kind) {
    const unsigned long long key = leaf_key(x >> 3, y >> 3, z >> 3);
    if (key != ckey) {
      ckey = key;
      cslot = map_find_or_insert(*m, key);
      if (cslot >= 0) mark_touched(*m, cslot, epoch, plane);
    }
    if (cslot < 0) return;
    const int l = local_index(x, y, z);
    uint32_t* wp = &m->labels[((size_t)plane * m->capacity + (size_t)cslot) * kLabelWords +
                              (kind == kKindHit ? 0 : 16) + (l >> 5)];
    const uint32_t bit = 1u << (l & 31);
    if (!(__ldcg(wp) & bit)) atomicOr(wp, bit);
  }
};

// Frames whose reach is beyond the leaf code's range: one thread per ray over the work's
// tiles (grid-stride), the same DDA and labels without the shared leaf table.
template <int RM, int MaxF>
__device__ __forceinline__ void traverse_wide_body(const TickWork<MaxF>& work, const MapView& m) {
  const int nrays = work.tile_w * work.tile_h;
  uint32_t visits = 0, rays = 0;
  for (uint32_t tile = blockIdx.x; tile < work.total_tiles; tile += gridDim.x) {
    int fi = 0;
    while (fi + 1 < work.n_frames && work.tile_start[fi + 1] <= tile) ++fi;
    const FrameParams& f = work.fr[fi];
    const uint32_t lt = tile - work.tile_start[fi];
    const int x0 = (int)(lt % (uint32_t)work.tiles_x[fi]) * work.tile_w;
    const int y0 = (int)(lt / (uint32_t)work.tiles_x[fi]) * work.tile_h;
    for (int k = threadIdx.x; k < nrays; k += blockDim.x) {
      const int px = x0 + k % work.tile_w, py = y0 + k / work.tile_w;
      float p[3];
      if (px < f.width && py < f.height && pixel_point(f, px, py, p)) {
        WideEmit em{&m, f.epoch, f.plane, kEmptyKey, -1};
        const int n = trace_point<RM>(f, p[0], p[1], p[2], em);
        if (n >= 0) {
          visits += (uint32_t)n;
          rays += 1;
        }
      }
    }
  }
  unsigned long long vv = visits, rr = rays;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    vv += __shfl_xor_sync(kFull, vv, o);
    rr += __shfl_xor_sync(kFull, rr, o);
  }
  if ((threadIdx.x & 31) == 0 && (vv | rr)) {
    atomicAdd(&m.ctr->visits, vv);
    atomicAdd(&m.ctr->rays, rr);
  }
}

// Work list passed by value (single insert, one-shot tick).
template <int RM, int MaxF>
__global__ void __launch_bounds__(256) k_traverse(const __grid_constant__ TickWork<MaxF> work,
                                                  MapView m) {
  traverse_body<RM, MaxF>(work, m);
}

// One simulated frame rendered tile by tile inside the traversal (sim render + noise + insert).
template <int RM>
__global__ void __launch_bounds__(256) k_traverse_render(const __grid_constant__ TickWork<1> work,
                                                         MapView m,
                                                         const __grid_constant__ SimRender sr) {
  traverse_body<RM, 1, true>(work, m, &sr);
}

// Work list read from device memory (tick plans replayed as CUDA graphs).
template <int RM>
__global__ void __launch_bounds__(256) k_traverse_dev(const TickWork<kMaxTickFrames>* work,
                                                      MapView m) {
  traverse_body<RM, kMaxTickFrames>(*work, m);
}

template <int RM, int MaxF>
__global__ void __launch_bounds__(256) k_traverse_wide(const __grid_constant__ TickWork<MaxF> work,
                                                       MapView m) {
  traverse_wide_body<RM, MaxF>(work, m);
}

template <int RM>
__global__ void __launch_bounds__(256) k_traverse_wide_dev(const TickWork<kMaxTickFrames>* work,
                                                           MapView m) {
  traverse_wide_body<RM, kMaxTickFrames>(*work, m);
}

// Resident CTAs of a traversal kernel for a block size and dynamic shared memory, queried
// once per (kernel, shape) ahead of any stream capture.
struct GridCache {
  const void* fn = nullptr;
  size_t smem = 0;
  int block = 0;
  int blocks = 0;
};

int g_sm_count = 0;
constexpr int kGridCacheSize = 64;
GridCache g_grid_cache[kGridCacheSize];
int g_grid_next = 0;
std::mutex g_grid_mutex;

cudaError_t resident_grid(const void* fn, size_t smem, int block, int* grid) {
  std::lock_guard<std::mutex> lock(g_grid_mutex);
  for (GridCache& c : g_grid_cache)
    if (c.fn == fn && c.smem == smem && c.block == block) {
      *grid = g_sm_count * c.blocks;
      return cudaSuccess;
    }
  cudaError_t e = cudaSuccess;
  if (g_sm_count == 0) {
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
  }
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
  int blocks = 0;
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, block, smem);
  if (e != cudaSuccess) return e;
  if (blocks < 1) blocks = 1;
  GridCache& c = g_grid_cache[g_grid_next];
  g_grid_next = (g_grid_next + 1) % kGridCacheSize;
  c.fn = fn;
  c.smem = smem;
  c.block = block;
  c.blocks = blocks;
  *grid = g_sm_count * blocks;
  return cudaSuccess;
}

bool work_is_wide(const FrameParams* fr, int n) {
  for (int i = 0; i < n; ++i)
    if (!(fr[i].max_time < kNarrowMaxTime)) return true;
  return false;
}

}  // namespace

size_t traverse_smem_bytes(int tile_w, int tile_h, uint32_t smask, bool render) {
  const size_t nent = (size_t)smask + 1;
  const size_t nrays = (size_t)tile_w * tile_h;
  (void)render;
  return nent * (8 + kLabelWords * 4 + 4) + nrays * (2 + 1 + 12);
}

template <int MaxF>
cudaError_t launch_traverse_labels(const TickWork<MaxF>& w, const MapView& m, int rounding,
                                   cudaStream_t s, bool dependent) {
  const int block = min(256, w.tile_w * w.tile_h);
  const bool down = rounding == NM_ROUND_DOWN;
  int grid = 0;
  if (work_is_wide(w.fr, w.n_frames)) {
    const void* fn = down ? (const void*)k_traverse_wide<NM_ROUND_DOWN, MaxF>
                          : (const void*)k_traverse_wide<NM_ROUND_NEAREST, MaxF>;
    cudaError_t e = resident_grid(fn, 0, block, &grid);
    if (e != cudaSuccess) return e;
    grid = min(grid, (int)w.total_tiles);
    if (down)
      k_traverse_wide<NM_ROUND_DOWN, MaxF><<<grid, block, 0, s>>>(w, m);
    else
      k_traverse_wide<NM_ROUND_NEAREST, MaxF><<<grid, block, 0, s>>>(w, m);
    return cudaGetLastError();
  }
  const size_t smem = traverse_smem_bytes(w.tile_w, w.tile_h, w.smask, false);
  const void* fn = down ? (const void*)k_traverse<NM_ROUND_DOWN, MaxF>
                        : (const void*)k_traverse<NM_ROUND_NEAREST, MaxF>;
  cudaError_t e = resident_grid(fn, smem, block, &grid);
  if (e != cudaSuccess) return e;
  grid = min(grid, (int)w.total_tiles);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = dependent ? 1 : 0;
  if (down)
    e = cudaLaunchKernelEx(&cfg, k_traverse<NM_ROUND_DOWN, MaxF>, w, m);
  else
    e = cudaLaunchKernelEx(&cfg, k_traverse<NM_ROUND_NEAREST, MaxF>, w, m);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

bool traverse_render_fits(const FrameParams& f) { return f.max_time < kNarrowMaxTime; }

cudaError_t launch_traverse_render(const TickWork<1>& w, const MapView& m, const SimRender& sr,
                                   int rounding, cudaStream_t s) {
  if (!traverse_render_fits(w.fr[0])) return cudaErrorInvalidValue;
  const int block = min(256, w.tile_w * w.tile_h);
  const size_t smem = traverse_smem_bytes(w.tile_w, w.tile_h, w.smask, true);
  const bool down = rounding == NM_ROUND_DOWN;
  const void* fn = down ? (const void*)k_traverse_render<NM_ROUND_DOWN>
                        : (const void*)k_traverse_render<NM_ROUND_NEAREST>;
  int grid = 0;
  cudaError_t e = resident_grid(fn, smem, block, &grid);
  if (e != cudaSuccess) return e;
  grid = min(grid, (int)w.total_tiles);
  if (down)
    k_traverse_render<NM_ROUND_DOWN><<<grid, block, smem, s>>>(w, m, sr);
  else
    k_traverse_render<NM_ROUND_NEAREST><<<grid, block, smem, s>>>(w, m, sr);
  return cudaGetLastError();
}

namespace {
const void* dev_kernel(int rounding, bool wide) {
  if (wide)
    return rounding == NM_ROUND_DOWN ? (const void*)k_traverse_wide_dev<NM_ROUND_DOWN>
                                     : (const void*)k_traverse_wide_dev<NM_ROUND_NEAREST>;
  return rounding == NM_ROUND_DOWN ? (const void*)k_traverse_dev<NM_ROUND_DOWN>
                                   : (const void*)k_traverse_dev<NM_ROUND_NEAREST>;
}
}  // namespace

cudaError_t prepare_traverse_dev(int tile_w, int tile_h, uint32_t smask, int rounding, bool wide) {
  const int block = min(256, tile_w * tile_h);
  const size_t smem = wide ? 0 : traverse_smem_bytes(tile_w, tile_h, smask, false);
  int grid = 0;
  return resident_grid(dev_kernel(rounding, wide), smem, block, &grid);
}

cudaError_t launch_traverse_labels_dev(const TickWork<kMaxTickFrames>* d_work, uint32_t total_tiles,
                                       int tile_w, int tile_h, uint32_t smask, const MapView& m,
                                       int rounding, bool wide, cudaStream_t s) {
  const int block = min(256, tile_w * tile_h);
  const size_t smem = wide ? 0 : traverse_smem_bytes(tile_w, tile_h, smask, false);
  int grid = 0;
  const cudaError_t e = resident_grid(dev_kernel(rounding, wide), smem, block, &grid);
  if (e != cudaSuccess) return e;
  grid = min(grid, (int)total_tiles);
  const bool down = rounding == NM_ROUND_DOWN;
  if (wide) {
    if (down)
      k_traverse_wide_dev<NM_ROUND_DOWN><<<grid, block, 0, s>>>(d_work, m);
    else
      k_traverse_wide_dev<NM_ROUND_NEAREST><<<grid, block, 0, s>>>(d_work, m);
  } else {
    if (down)
      k_traverse_dev<NM_ROUND_DOWN><<<grid, block, smem, s>>>(d_work, m);
    else
      k_traverse_dev<NM_ROUND_NEAREST><<<grid, block, smem, s>>>(d_work, m);
  }
  return cudaGetLastError();
}

cudaError_t tile_order_reserve(TileOrderBuffers* b, uint32_t tiles, cudaStream_t s) {
  if (tiles <= b->capacity && b->counts) return cudaSuccess;
  // growth frees the old buffers (a device synchronisation): start at 16 K tiles (a 1280x720
  // frame has 7200 tiles of 16x8) and double
  const uint32_t cap = std::max<uint32_t>(tiles, std::max<uint32_t>(1u << 14, 2u * b->capacity));
  tile_order_release(b);
  cudaError_t e = cudaMalloc((void**)&b->counts, kOrderBuckets * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&b->lists, (size_t)kOrderBuckets * cap * 4);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->counts, 0, kOrderBuckets * 4, s);
  if (e != cudaSuccess) {
    tile_order_release(b);
    return e;
  }
  b->capacity = cap;
  b->pending = false;
  return cudaSuccess;
}

void tile_order_release(TileOrderBuffers* b) {
  cudaFree(b->counts);
  cudaFree(b->lists);
  *b = TileOrderBuffers{};
}

template <int MaxF>
float tile_order_scale(const TickWork<MaxF>& w) {
  float longest = 0.0f;
  for (int i = 0; i < w.n_frames; ++i) longest = std::max(longest, w.fr[i].max_time);
  return (float)kOrderBuckets / (longest * 1.7320508f + kSetupSteps);
}

namespace {
cudaError_t clear_pending_counts(TileOrderBuffers* b, cudaStream_t s) {
  if (!b->pending) return cudaSuccess;
  const cudaError_t e = cudaMemsetAsync(b->counts, 0, kOrderBuckets * 4, s);
  if (e == cudaSuccess) b->pending = false;
  return e;
}
}  // namespace

template <int MaxF>
cudaError_t launch_tile_order(const TickWork<MaxF>& w, TileOrderBuffers* b, cudaStream_t s) {
  if (w.total_tiles == 0) return cudaSuccess;
  if (w.total_tiles > b->capacity) return cudaErrorInvalidValue;
  cudaError_t e = clear_pending_counts(b, s);
  if (e != cudaSuccess) return e;
  k_tile_order<MaxF><<<order_grid(w.total_tiles), kOrderThreads, 0, s>>>(w, *b);
  e = cudaGetLastError();
  if (e == cudaSuccess) b->pending = true;
  return e;
}

cudaError_t launch_tile_order_dev(const TickWork<kMaxTickFrames>* d_work, uint32_t total_tiles,
                                  TileOrderBuffers* b, cudaStream_t s) {
  if (total_tiles == 0) return cudaSuccess;
  if (total_tiles > b->capacity) return cudaErrorInvalidValue;
  cudaError_t e = clear_pending_counts(b, s);
  if (e != cudaSuccess) return e;
  k_tile_order_dev<<<order_grid(total_tiles), kOrderThreads, 0, s>>>(d_work, *b);
  e = cudaGetLastError();
  if (e == cudaSuccess) b->pending = true;
  return e;
}

template float tile_order_scale<1>(const TickWork<1>&);
template float tile_order_scale<kMaxTickFrames>(const TickWork<kMaxTickFrames>&);
template cudaError_t launch_tile_order<1>(const TickWork<1>&, TileOrderBuffers*, cudaStream_t);
template cudaError_t launch_tile_order<kMaxTickFrames>(const TickWork<kMaxTickFrames>&,
                                                       TileOrderBuffers*, cudaStream_t);
template cudaError_t launch_traverse_labels<1>(const TickWork<1>&, const MapView&, int, cudaStream_t,
                                               bool);
template cudaError_t launch_traverse_labels<kMaxTickFrames>(const TickWork<kMaxTickFrames>&,
                                                            const MapView&, int, cudaStream_t, bool);

}  // namespace nm
