// nm_traverse.cu -- persistent traversal + per-frame labelling kernel (sm_100a).
//
// Replaces nodePassHDDA / voxelPassHDDA and the CUB compaction between them
// (frustumCastCloud.cu:44-246): one pass walks every ray voxel by voxel with the insertion
// DDA of Handler.cpp:58-85 and records one label per voxel (hit overrides miss), allocating
// map leaves on the fly.
//
// Work distribution: CTAs stay resident and take 16x16-pixel tiles from a device counter,
// so the cost of a tile (set by its longest rays) no longer decides when an SM goes idle.
// A tile holds several rays per thread; every lane walks one ray at a time and takes the
// tile's next ray as soon as its own ends, so lanes stay busy until the tile runs dry.
//
// Labels collect in a per-CTA shared-memory leaf table (hashed, 32 label words per leaf);
// a leaf that finds no room goes straight to the device table.  After a tile, one lane per
// cached leaf ORs its words into the device label buffer and puts the leaf on the touched
// list (the device-table lookups of a warp's leaves overlap).
//
// Host xyz records may arrive in chunks of tile rows: each chunk is then its own launch on
// its own stream and tile counter (TickWork::queue), started when its rows have arrived.
//
// Per step the walk compares the three crossing times (non-negative doubles, one compare per
// pair), keeps the voxel as (leaf, local) coordinates, and probes the leaf table only when the
// step leaves the current leaf.
//
// k_traverse_render renders each tile's ranges from the sim map into shared memory first
// (nm_sim_insert), so one launch does the simulated frame and its insertion.
#include <cfloat>
#include <cstdint>

#include "nm_device.cuh"
#include "nm_internal.h"
#include "nm_sim_device.cuh"

namespace nm {

namespace {

constexpr unsigned kFull = 0xffffffffu;

__device__ __noinline__ int smem_lookup_slow(unsigned long long* s_keys, uint32_t smask,
                                            unsigned long long key, uint32_t h) {
  h &= smask;
  const uint32_t limit = (smask + 1) < 16u ? (smask + 1) : 16u;
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

// Shared-table slot of a leaf: Fibonacci hashing of the packed key (high product bits), which
// spreads neighbouring leaves of a ray cone over the table.
__device__ __forceinline__ uint32_t leaf_hash(unsigned long long key) {
  return (uint32_t)((key * 0x9E3779B97F4A7C15ull) >> 40);
}

struct Ray {
  double t0, t1, t2;  // next crossing time per axis (never negative)
  double d0, d1, d2;  // crossing spacing per axis
  double len;         // ray length in voxels
  int ds0, ds1, ds2;  // step of the voxel index inside the leaf per axis: +-64, +-8, +-1 or 0
  int l;              // voxel index inside the leaf, x*64 + y*8 + z
  unsigned long long key;  // packed leaf coordinate
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
  r.l = ((v[0] & 7) << 6) | ((v[1] & 7) << 3) | (v[2] & 7);
  r.key = leaf_key(v[0] >> 3, v[1] >> 3, v[2] >> 3);
  return true;
}

__device__ __forceinline__ bool pixel_point(const FrameParams& f, int w, int h, float p[3]) {
  if (f.input_kind == 1) return range_point(f, w, h, p);
  if (f.input_kind == 2 && (uint32_t)(h * f.width + w) >= __ldg(f.n_valid)) return false;
  return xyz_point(f, w, h, p);
}

template <int RM, int MaxF, bool Render = false>
__device__ __forceinline__ void traverse_body(const TickWork<MaxF>& work, const MapView& m,
                                              const SimRender* sr = nullptr) {
  extern __shared__ __align__(16) unsigned char smem[];
  const uint32_t smask = work.smask;
  const int nent = (int)smask + 1;
  unsigned long long* s_keys = reinterpret_cast<unsigned long long*>(smem);
  uint32_t* s_words = reinterpret_cast<uint32_t*>(s_keys + nent);
  float* s_rng = reinterpret_cast<float*>(s_words + nent * kLabelWords);  // Render: tile ranges
  __shared__ FrameParams s_f;
  __shared__ uint32_t s_tile;
  __shared__ int s_frame;
  __shared__ uint32_t s_next;
  const int tid = threadIdx.x;
  const int lane = tid & 31, nwarps = blockDim.x >> 5;
  const int nrays = work.tile_w * work.tile_h;
  uint32_t visits = 0, rays = 0;

  for (;;) {
    if (tid == 0) {
      unsigned int* queue = work.queue ? &m.ctr->chunk_queue[work.queue - 1] : &m.ctr->tile_queue;
      const uint32_t t = atomicAdd(queue, 1u);
      int fi = 0;
      while (fi + 1 < work.n_frames && work.tile_start[fi + 1] <= t) ++fi;
      s_tile = t;
      s_frame = fi;
      s_next = 0u;
      if (t == work.total_tiles + gridDim.x - 1) *queue = 0u;  // last reader resets
    }
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= work.total_tiles) break;
    const int fi = s_frame;
    {
      const uint32_t* src = reinterpret_cast<const uint32_t*>(&work.fr[fi]);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&s_f);
      for (int i = tid; i < (int)(sizeof(FrameParams) / 4); i += blockDim.x) dst[i] = src[i];
    }
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
    for (int i = tid; i < nent; i += blockDim.x) s_keys[i] = kEmptyKey;
    for (int i = tid; i < nent * kLabelWords; i += blockDim.x) s_words[i] = 0u;
    if constexpr (Render) {
      // the tile's ranges: the sim map's first active voxel per pixel, then the range noise
      // (the same values nm_sim_render_noisy writes)
      for (int t = tid; t < nrays; t += blockDim.x) {
        const int px = x0 + t % work.tile_w, py = y0 + t / work.tile_w;
        float rr = 0.0f;
        if (px < f.width && py < f.height) {
          rr = sim_ray(sr->v, sr->rp, px, py);
          const long long i = (long long)py * f.width + px;
          if (sr->noise) rr = noisy(rr, sr->seed, i, sr->sigma_coef, sr->drop);
          if (sr->out) sr->out[i] = rr;
        }
        s_rng[t] = rr;
      }
    }
    __syncthreads();

    Ray r;
    bool active = false;
    bool glob = false;
    int slot = -1;
    int cw_idx = -1;
    uint32_t cw_bits = 0u;
    const int plane = f.plane;

    // Leaf lookup after a crossing (or at ray start): one inline probe finds leaves already
    // in the tile's table; a miss probes / inserts (or falls back to the device table).
    auto resolve = [&]() {
      const uint32_t hh = leaf_hash(r.key);
      const uint32_t h = hh & smask;
      if (((volatile unsigned long long*)s_keys)[h] == r.key) {
        glob = false;
        slot = (int)h;
        return;
      }
      const int sl = smem_lookup_slow(s_keys, smask, r.key, hh);
      if (sl >= 0) {
        glob = false;
        slot = sl;
      } else {
        glob = true;
        slot = map_find_or_insert(m, r.key);
        if (slot >= 0) mark_touched(m, slot, f.epoch, plane);
      }
    };
    auto label = [&](int kind) {
      const uint32_t bit = 1u << (r.l & 31);
      const int wi = (kind == kKindHit ? 0 : 16) + (r.l >> 5);
      if (!glob) {
        const int idx = slot * kLabelWords + wi;
        if (idx != cw_idx) {
          cw_idx = idx;
          cw_bits = ((volatile uint32_t*)s_words)[idx];
        }
        if (!(cw_bits & bit)) {
          atomicOr(&s_words[idx], bit);
          cw_bits |= bit;
        }
      } else if (slot >= 0) {
        uint32_t* wp = &m.labels[((size_t)plane * m.capacity + (size_t)slot) * kLabelWords + wi];
        if (!(__ldcg(wp) & bit)) atomicOr(wp, bit);
      }
    };

    for (;;) {
      if (!active) {
        const uint32_t k = atomicAdd(&s_next, 1u);
        if (k >= (uint32_t)nrays) break;
        const int px = x0 + (int)(k % (uint32_t)work.tile_w);
        const int py = y0 + (int)(k / (uint32_t)work.tile_w);
        float p[3];
        // pixels of a tile that overhangs the image are skipped before any input is read
        bool has_point = false;
        if (px < f.width && py < f.height)
          has_point = Render ? range_point_r(f, px, py, s_rng[k], p) : pixel_point(f, px, py, p);
        if (has_point && setup_ray<RM>(f, p, r)) {
          active = true;
          rays += 1;
          cw_idx = -1;
          resolve();
        }
        continue;
      }
      // crossing times are non-negative and never NaN (disabled axes hold DBL_MAX): one
      // double compare per pair; ties go to the higher axis
      const int a = (r.t0 < r.t1) ? ((r.t0 < r.t2) ? 0 : 2) : ((r.t1 < r.t2) ? 1 : 2);
      const double t = (a == 0) ? r.t0 : ((a == 1) ? r.t1 : r.t2);
      if (!(t <= r.len)) {
        if (t < (double)f.max_time) {
          label(kKindHit);
          visits += 1;
        }
        active = false;
        continue;
      }
      label(kKindMiss);
      visits += 1;
      // advance along axis a: crossing time, voxel index inside the leaf, leaf on wrap
      const double dstep = (a == 0) ? r.d0 : ((a == 1) ? r.d1 : r.d2);
      const double tnext = Ar<RM>::dadd(t, dstep);
      r.t0 = (a == 0) ? tnext : r.t0;
      r.t1 = (a == 1) ? tnext : r.t1;
      r.t2 = (a == 2) ? tnext : r.t2;
      const int msk = (a == 0) ? 0x1C0 : ((a == 1) ? 0x38 : 0x7);
      const int ds = (a == 0) ? r.ds0 : ((a == 1) ? r.ds1 : r.ds2);
      const int vv = (r.l & msk) + ds;
      const bool cross = (unsigned)vv > (unsigned)msk;
      r.l = (r.l & ~msk) | (vv & msk);
      if (cross) {
        const int sh = (a == 0) ? 42 : ((a == 1) ? 21 : 0);
        r.key += (unsigned long long)(long long)(ds > 0 ? 1 : -1) << sh;
        resolve();
      }
    }
    __syncthreads();

    // Flush the tile's leaf table: one lane per cached leaf, so the device-table lookups of
    // up to 32 leaves overlap; word reads are rotated by lane to avoid bank conflicts.
    for (int e = tid; e < nent; e += blockDim.x) {
      const unsigned long long key = s_keys[e];
      if (key == kEmptyKey) continue;
      const uint32_t* sw = s_words + e * kLabelWords;
      bool has = false;
#pragma unroll 4
      for (int w = 0; w < kLabelWords; ++w) has |= sw[(w + lane) & (kLabelWords - 1)] != 0u;
      if (!has) continue;
      const int g = map_find_or_insert(m, key);
      if (g < 0) continue;
      mark_touched(m, g, f.epoch, plane);
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
int persistent_grid(size_t smem_bytes, int block) {
  static int cached_blocks = 0;
  static size_t cached_smem = 0;
  static int cached_block = 0;
  static int sms = 0;
  if (cached_blocks == 0 || cached_smem != smem_bytes || cached_block != block) {
    cudaFuncSetAttribute(k_traverse<RM, MaxF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         160 * 1024);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int blocks = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_traverse<RM, MaxF>, block, smem_bytes);
    cached_blocks = blocks > 0 ? blocks : 1;
    cached_smem = smem_bytes;
    cached_block = block;
  }
  return sms * cached_blocks;
}

}  // namespace

template <int MaxF>
cudaError_t launch_traverse_labels(const TickWork<MaxF>& w, const MapView& m, int rounding,
                                   cudaStream_t s) {
  const size_t smem = (size_t)(w.smask + 1) * (8 + kLabelWords * 4);
  const int block = min(256, w.tile_w * w.tile_h);
  if (rounding == NM_ROUND_DOWN) {
    const int grid = min(persistent_grid<NM_ROUND_DOWN, MaxF>(smem, block), (int)w.total_tiles);
    k_traverse<NM_ROUND_DOWN, MaxF><<<grid, block, smem, s>>>(w, m);
  } else {
    const int grid = min(persistent_grid<NM_ROUND_NEAREST, MaxF>(smem, block), (int)w.total_tiles);
    k_traverse<NM_ROUND_NEAREST, MaxF><<<grid, block, smem, s>>>(w, m);
  }
  return cudaGetLastError();
}

cudaError_t launch_traverse_render(const TickWork<1>& w, const MapView& m, const SimRender& sr,
                                   int rounding, cudaStream_t s) {
  const int nrays = w.tile_w * w.tile_h;
  const size_t smem = (size_t)(w.smask + 1) * (8 + kLabelWords * 4) + (size_t)nrays * 4;
  const int block = min(256, nrays);
  static int cached[2] = {0, 0};
  static size_t cached_smem[2] = {0, 0};
  static int cached_block[2] = {0, 0};
  static int sms = 0;
  const int ri = rounding == NM_ROUND_DOWN ? 1 : 0;
  if (!cached[ri] || cached_smem[ri] != smem || cached_block[ri] != block) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int blocks = 0;
    if (ri) {
      cudaFuncSetAttribute(k_traverse_render<NM_ROUND_DOWN>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_traverse_render<NM_ROUND_DOWN>,
                                                    block, smem);
    } else {
      cudaFuncSetAttribute(k_traverse_render<NM_ROUND_NEAREST>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_traverse_render<NM_ROUND_NEAREST>,
                                                    block, smem);
    }
    cached[ri] = blocks > 0 ? blocks : 1;
    cached_smem[ri] = smem;
    cached_block[ri] = block;
  }
  const int grid = min(sms * cached[ri], (int)w.total_tiles);
  if (ri)
    k_traverse_render<NM_ROUND_DOWN><<<grid, block, smem, s>>>(w, m, sr);
  else
    k_traverse_render<NM_ROUND_NEAREST><<<grid, block, smem, s>>>(w, m, sr);
  return cudaGetLastError();
}

namespace {
struct DevGrid {
  int blocks = 0;
  size_t smem = 0;
  int block = 0;
  int sms = 0;
};
DevGrid g_dev_grid[2];
}  // namespace

cudaError_t prepare_traverse_dev(int tile_w, int tile_h, uint32_t smask, int rounding) {
  const size_t smem = (size_t)(smask + 1) * (8 + kLabelWords * 4);
  const int block = min(256, tile_w * tile_h);
  DevGrid& g = g_dev_grid[rounding == NM_ROUND_DOWN ? 1 : 0];
  if (g.blocks && g.smem == smem && g.block == block) return cudaSuccess;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&g.sms, cudaDevAttrMultiProcessorCount, dev);
  if (rounding == NM_ROUND_DOWN) {
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_traverse_dev<NM_ROUND_DOWN>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g.blocks, k_traverse_dev<NM_ROUND_DOWN>, block, smem);
  } else {
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_traverse_dev<NM_ROUND_NEAREST>, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    if (e == cudaSuccess)
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&g.blocks, k_traverse_dev<NM_ROUND_NEAREST>, block, smem);
  }
  if (g.blocks < 1) g.blocks = 1;
  g.smem = smem;
  g.block = block;
  return e;
}

cudaError_t launch_traverse_labels_dev(const TickWork<kMaxTickFrames>* d_work, uint32_t total_tiles,
                                       int tile_w, int tile_h, uint32_t smask, const MapView& m,
                                       int rounding, cudaStream_t s) {
  const cudaError_t e = prepare_traverse_dev(tile_w, tile_h, smask, rounding);
  if (e != cudaSuccess) return e;
  const DevGrid& g = g_dev_grid[rounding == NM_ROUND_DOWN ? 1 : 0];
  const int grid = min(g.sms * g.blocks, (int)total_tiles);
  if (rounding == NM_ROUND_DOWN)
    k_traverse_dev<NM_ROUND_DOWN><<<grid, g.block, g.smem, s>>>(d_work, m);
  else
    k_traverse_dev<NM_ROUND_NEAREST><<<grid, g.block, g.smem, s>>>(d_work, m);
  return cudaGetLastError();
}

template cudaError_t launch_traverse_labels<1>(const TickWork<1>&, const MapView&, int, cudaStream_t);
template cudaError_t launch_traverse_labels<kMaxTickFrames>(const TickWork<kMaxTickFrames>&,
                                                            const MapView&, int, cudaStream_t);

}  // namespace nm
