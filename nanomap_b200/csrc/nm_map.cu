// nm_map.cu -- sm_100a kernels of the mapping path: traversal + per-frame labels, label
// integration into the device leaf table, table growth and export.
//
// Replaces frustumCastCloud.cu:84-294 (leaf pass, CUB compaction, voxel pass with per-visit
// fp32 atomics, int8 quantisation) and the host map update of Handler.cpp:134-182.
#include <atomic>
#include <cfloat>
#include <cstddef>
#include <cstdint>

#include "nm_device.cuh"
#include "nm_internal.h"

namespace nm {

namespace {

constexpr unsigned kFull = 0xffffffffu;

// Count sink (accumulate mode): exact per-voxel hit and miss counts, one atomic per group of
// lanes that hit the same counter at the same time.
struct CountEmit {
  const MapView* m;
  uint32_t epoch;
  unsigned long long ckey;
  int cslot;

  __device__ __forceinline__ void operator()(int x, int y, int z, int kind) {
    const unsigned long long key = leaf_key(x >> 3, y >> 3, z >> 3);
    if (key != ckey) {
      ckey = key;
      cslot = map_find_or_insert(*m, key);
      if (cslot >= 0) mark_touched(*m, cslot, epoch, 0);
    }
    if (cslot < 0) return;
    const int l = local_index(x, y, z);
    const unsigned long long idx =
        (unsigned long long)cslot * 1024ull + (kind == kKindHit ? 0u : 512u) + (unsigned)l;
    const unsigned act = __activemask();
    const unsigned peers = __match_any_sync(act, idx);
    const int leader = __ffs(peers) - 1;
    if ((int)(threadIdx.x & 31) == leader) atomicAdd(&m->counts[idx], (unsigned)__popc(peers));
  }
};

__device__ __forceinline__ bool load_point(const FrameParams& f, int w, int h, float p[3]) {
  if (f.input_kind == 1) return range_point(f, w, h, p);
  if (f.input_kind == 2 && (uint32_t)(h * f.width + w) >= __ldg(f.n_valid)) return false;
  return xyz_point(f, w, h, p);
}

__device__ __forceinline__ void add_counts(MapCounters* ctr, uint32_t visits, uint32_t rays) {
  unsigned long long v = visits, r = rays;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v += __shfl_xor_sync(kFull, v, o);
    r += __shfl_xor_sync(kFull, r, o);
  }
  if ((threadIdx.x & 31) == 0 && (v | r)) {
    atomicAdd(&ctr->visits, v);
    atomicAdd(&ctr->rays, r);
  }
}

template <int RM>
__global__ void __launch_bounds__(256) k_traverse_count(FrameParams f, MapView m, int tiles_x,
                                                        int tile_w, int tile_h) {
  const int tid = threadIdx.x;
  const int tile = blockIdx.x;
  const int px = (tile % tiles_x) * tile_w + tid % tile_w;
  const int py = (tile / tiles_x) * tile_h + tid / tile_w;
  uint32_t visits = 0, rays = 0;
  if (px < f.width && py < f.height) {
    float p[3];
    if (load_point(f, px, py, p)) {
      CountEmit em{&m, f.epoch, kEmptyKey, -1};
      const int n = trace_point<RM>(f, p[0], p[1], p[2], em);
      if (n >= 0) {
        visits = (uint32_t)n;
        rays = 1;
      }
    }
  }
  add_counts(m.ctr, visits, rays);
}

// ---- integration (Handler.cpp:88-122 / SimHandler.cpp:88-122) ------------------------------

// Update of one voxel by `temp` (Handler.cpp:99-104 when Always: clamp, then set or clear
// the active bit by the thresholds; SimHandler.cpp:100-110 otherwise: clamp only on the side
// whose threshold was crossed).  `temp` == 0 leaves the voxel as it is.  Written with selects,
// so lanes with different outcomes take no divergent branches.
template <int RM, bool Always>
__device__ __forceinline__ float update_voxel(float v, uint32_t& abit, float temp,
                                              const IntegrateParams& p) {
  const float s = Ar<RM>::fadd(v, temp);
  float c;
  uint32_t a;
  if (Always) {
    c = s > p.clamp_max ? p.clamp_max : (s < p.clamp_min ? p.clamp_min : s);
    a = c > p.thres_hit ? 1u : (c < p.thres_miss ? 0u : abit);
  } else {
    const bool up = s > p.thres_hit;
    const bool down = !up && s < p.thres_miss;
    c = (up && s > p.clamp_max) ? p.clamp_max : ((down && s < p.clamp_min) ? p.clamp_min : s);
    a = up ? 1u : (down ? 0u : abit);
  }
  const bool apply = temp != 0.0f;
  abit = apply ? a : abit;
  return apply ? c : v;
}

// The frame's touched-leaf count and the probe error bit, read once per block: every warp
// reading the counter word itself queues thousands of requests on one L2 line.  Thread 0 reads
// the count and takes the block's ticket in one 64-bit atomic on (touched_count, done_blocks);
// the block with the last ticket knows that every block holds the count, so it resets the
// per-frame list for the next frame and folds it into the totals.
static_assert(offsetof(MapCounters, done_blocks) == offsetof(MapCounters, touched_count) + 4 &&
                  offsetof(MapCounters, touched_count) % 8 == 0,
              "touched_count and done_blocks form one 8-byte word");
__device__ __forceinline__ void read_integrate_counters(MapCounters* ctr, uint32_t* n,
                                                        bool* fatal) {
  __shared__ uint32_t s_n, s_err;
  wait_prior_grid();  // the walk that fills the counters may still run at launch
  if (threadIdx.x == 0) {
    unsigned long long* pair = reinterpret_cast<unsigned long long*>(&ctr->touched_count);
    const unsigned long long old = atomicAdd(pair, 1ull << 32);
    const uint32_t cnt = (uint32_t)old;
    s_err = *(const volatile unsigned int*)&ctr->error_flags;
    if ((uint32_t)(old >> 32) == gridDim.x - 1) {
      *pair = 0ull;  // touched_count = done_blocks = 0
      ctr->touched_total += cnt;
      ctr->frames += 1u;
    }
    s_n = cnt;
  }
  __syncthreads();
  *n = s_n;
  *fatal = (s_err & kErrProbe) != 0u;
}

// Warp of the integration grid that takes touched leaf i: leaf i goes to block i % grid, so
// the leaves of a small frame spread over all SMs instead of filling the first blocks.
__device__ __forceinline__ uint32_t integrate_warp() {
  return (threadIdx.x >> 5) * gridDim.x + blockIdx.x;
}

// Newly labelled voxels of the warp's leaves: one reduction per warp (called converged).
__device__ __forceinline__ void add_unique(MapCounters* ctr, unsigned long long uniq) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) uniq += __shfl_xor_sync(kFull, uniq, o);
  if ((threadIdx.x & 31) == 0 && uniq) atomicAdd(&ctr->unique_voxels, uniq);
}

// One warp per touched leaf.  Lane i owns float4 i, i+32, i+64, i+96 of the leaf's 512
// log-odds (voxels 4q..4q+3 of float4 q); label and active words are shared through
// shuffles.  Labels are cleared as they are consumed, so the next frame starts from zero.
template <int RM, bool Always>
__global__ void __launch_bounds__(256) k_integrate_label(MapView m, IntegrateParams p) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = integrate_warp();
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  uint32_t n;
  bool fatal;
  read_integrate_counters(m.ctr, &n, &fatal);
  unsigned long long uniq = 0;
  for (uint32_t i = gw; i < n; i += nw) {
    const uint32_t slot = m.touched[i];
    uint32_t planes = 1u;
    if (p.use_planes) {
      planes = m.plane_mask[slot];
      if (lane == 0) m.plane_mask[slot] = 0u;
    }
    float4* v4 = reinterpret_cast<float4*>(m.values + (size_t)slot * kLeafVoxels);
    uint32_t* act = m.active + (size_t)slot * kActiveWords;
    float4 v[4];
    uint32_t anib[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int q = lane + 32 * k;
      v[k] = v4[q];
      anib[k] = (act[q >> 3] >> ((q & 7) * 4)) & 0xFu;
    }
    uint32_t touched_any[4] = {0u, 0u, 0u, 0u};
    while (planes) {
      const int pl = __ffs(planes) - 1;
      planes &= planes - 1u;
      uint32_t* lab = m.labels + ((size_t)pl * m.capacity + slot) * kLabelWords;
      const uint32_t myw = lab[lane];
      if (myw) lab[lane] = 0u;
      if (fatal) continue;
      const float lh = p.lh[pl], lm = p.lm[pl];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int q = lane + 32 * k;
        const int w = q >> 3;
        const int sh = (q & 7) * 4;
        const uint32_t hn = (__shfl_sync(kFull, myw, w) >> sh) & 0xFu;
        const uint32_t mn = (__shfl_sync(kFull, myw, 16 + w) >> sh) & 0xFu;
        const uint32_t tn = hn | mn;
        touched_any[k] |= tn;
        uint32_t a0 = anib[k] & 1u, a1 = (anib[k] >> 1) & 1u, a2 = (anib[k] >> 2) & 1u,
                 a3 = (anib[k] >> 3) & 1u;
        v[k].x = update_voxel<RM, Always>(v[k].x, a0, (tn & 1u) ? ((hn & 1u) ? lh : lm) : 0.0f, p);
        v[k].y = update_voxel<RM, Always>(v[k].y, a1, (tn & 2u) ? ((hn & 2u) ? lh : lm) : 0.0f, p);
        v[k].z = update_voxel<RM, Always>(v[k].z, a2, (tn & 4u) ? ((hn & 4u) ? lh : lm) : 0.0f, p);
        v[k].w = update_voxel<RM, Always>(v[k].w, a3, (tn & 8u) ? ((hn & 8u) ? lh : lm) : 0.0f, p);
        anib[k] = a0 | (a1 << 1) | (a2 << 2) | (a3 << 3);
      }
    }
    if (fatal) continue;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int q = lane + 32 * k;
      if (touched_any[k]) {
        v4[q] = v[k];
        uniq += (unsigned)__popc(touched_any[k]);
      }
      // rebuild active word q>>3 from the 8 nibbles of lanes 8j..8j+7
      uint32_t word = anib[k] << ((q & 7) * 4);
      word |= __shfl_xor_sync(kFull, word, 1);
      word |= __shfl_xor_sync(kFull, word, 2);
      word |= __shfl_xor_sync(kFull, word, 4);
      uint32_t any = touched_any[k];
      any |= __shfl_xor_sync(kFull, any, 1);
      any |= __shfl_xor_sync(kFull, any, 2);
      any |= __shfl_xor_sync(kFull, any, 4);
      if ((lane & 7) == 0 && any) act[q >> 3] = word;
    }
  }
  add_unique(m.ctr, uniq);
}

template <int RM, bool Always>
__global__ void __launch_bounds__(256) k_integrate_count(MapView m, IntegrateParams p) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = integrate_warp();
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  uint32_t n;
  bool fatal;
  read_integrate_counters(m.ctr, &n, &fatal);
  unsigned long long uniq = 0;
  const float lh = p.lh[0], lm = p.lm[0];
  for (uint32_t i = gw; i < n; i += nw) {
    const uint32_t slot = m.touched[i];
    uint32_t* cnt = m.counts + (size_t)slot * 1024;
    float* val = m.values + (size_t)slot * kLeafVoxels;
    uint32_t* act = m.active + (size_t)slot * kActiveWords;
    for (int j = 0; j < 16; ++j) {
      const int l = j * 32 + lane;
      const uint32_t nh = cnt[l], nm_ = cnt[512 + l];
      uint32_t abit = (act[j] >> lane) & 1u;
      const bool t = (nh | nm_) != 0u;
      if (t) {
        cnt[l] = 0u;
        cnt[512 + l] = 0u;
        if (!fatal) {
          const float temp = Ar<RM>::fadd(Ar<RM>::fmul((float)nm_, lm), Ar<RM>::fmul((float)nh, lh));
          val[l] = update_voxel<RM, Always>(val[l], abit, temp, p);
          uniq += 1;
        }
      }
      const uint32_t word = __ballot_sync(kFull, abit != 0u);
      if (!fatal && __ballot_sync(kFull, t) != 0u && lane == 0) act[j] = word;
    }
  }
  add_unique(m.ctr, uniq);
}

// ---- growth, export --------------------------------------------------------------------------

__global__ void k_fill_keys(unsigned long long* keys, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    keys[i] = kEmptyKey;
}

// Move every leaf (values, active bits, pending labels and counts) to the larger table and
// rebuild the touched list of the current epoch.
__global__ void __launch_bounds__(256) k_rehash(MapView from, MapView to, uint32_t cur_epoch,
                                                int with_counts) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t s = gw; s < from.capacity; s += nw) {
    const unsigned long long key = from.keys[s];
    if (key == kEmptyKey) continue;
    int d = -1;
    if (lane == 0) d = map_find_or_insert(to, key);
    d = __shfl_sync(kFull, d, 0);
    if (d < 0) continue;
    const float4* sv = reinterpret_cast<const float4*>(from.values + (size_t)s * kLeafVoxels);
    float4* dv = reinterpret_cast<float4*>(to.values + (size_t)d * kLeafVoxels);
    for (int q = lane; q < 128; q += 32) dv[q] = sv[q];
    if (lane < kActiveWords)
      to.active[(size_t)d * kActiveWords + lane] = from.active[(size_t)s * kActiveWords + lane];
    for (int pl = 0; pl < from.planes; ++pl)
      to.labels[((size_t)pl * to.capacity + d) * kLabelWords + lane] =
          from.labels[((size_t)pl * from.capacity + s) * kLabelWords + lane];
    if (with_counts)
      for (int c = lane; c < 1024; c += 32)
        to.counts[(size_t)d * 1024 + c] = from.counts[(size_t)s * 1024 + c];
    if (lane == 0) {
      const uint32_t ep = from.epoch[s];
      to.epoch[d] = ep;
      if (from.plane_mask) to.plane_mask[d] = from.plane_mask[s];
      if (ep == cur_epoch) {
        const uint32_t i = atomicAdd(&to.ctr->touched_count, 1u);
        to.touched[i] = (uint32_t)d;
      }
    }
  }
}

__global__ void __launch_bounds__(256) k_export(MapView m, int32_t* origins, float* values,
                                                uint32_t* active, uint32_t* n_out,
                                                uint32_t max_out) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t s = gw; s < m.capacity; s += nw) {
    const unsigned long long key = m.keys[s];
    if (key == kEmptyKey) continue;
    uint32_t o = 0;
    if (lane == 0) o = atomicAdd(n_out, 1u);
    o = __shfl_sync(kFull, o, 0);
    if (o >= max_out) continue;
    if (origins && lane == 0) {
      int lx, ly, lz;
      key_leaf(key, &lx, &ly, &lz);
      origins[3 * (size_t)o] = lx * 8;
      origins[3 * (size_t)o + 1] = ly * 8;
      origins[3 * (size_t)o + 2] = lz * 8;
    }
    if (values)
      for (int q = lane; q < kLeafVoxels; q += 32)
        values[(size_t)o * kLeafVoxels + q] = m.values[(size_t)s * kLeafVoxels + q];
    if (active && lane < kActiveWords)
      active[(size_t)o * kActiveWords + lane] = m.active[(size_t)s * kActiveWords + lane];
  }
}

__global__ void __launch_bounds__(256) k_export_labels(MapView m, int plane, int32_t* origins,
                                                       uint32_t* words, uint32_t* n_out,
                                                       uint32_t max_out) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t s = gw; s < m.capacity; s += nw) {
    const unsigned long long key = m.keys[s];
    if (key == kEmptyKey) continue;
    const uint32_t w = m.labels[((size_t)plane * m.capacity + s) * kLabelWords + lane];
    if (__ballot_sync(kFull, w != 0u) == 0u) continue;
    uint32_t o = 0;
    if (lane == 0) o = atomicAdd(n_out, 1u);
    o = __shfl_sync(kFull, o, 0);
    if (o >= max_out) continue;
    if (lane == 0) {
      int lx, ly, lz;
      key_leaf(key, &lx, &ly, &lz);
      origins[3 * (size_t)o] = lx * 8;
      origins[3 * (size_t)o + 1] = ly * 8;
      origins[3 * (size_t)o + 2] = lz * 8;
    }
    words[(size_t)o * kLabelWords + lane] = w;
  }
}

}  // namespace

cudaError_t launch_traverse_counts(const FrameParams& f, const MapView& m, int rounding,
                                   cudaStream_t s) {
  const int tile_w = 16, tile_h = 16;
  const int tiles_x = (f.width + tile_w - 1) / tile_w;
  const int tiles_y = (f.height + tile_h - 1) / tile_h;
  const dim3 grid(tiles_x * tiles_y), block(tile_w * tile_h);
  if (rounding == NM_ROUND_DOWN) {
    k_traverse_count<NM_ROUND_DOWN><<<grid, block, 0, s>>>(f, m, tiles_x, tile_w, tile_h);
  } else {
    k_traverse_count<NM_ROUND_NEAREST><<<grid, block, 0, s>>>(f, m, tiles_x, tile_w, tile_h);
  }
  return cudaGetLastError();
}

namespace {

// Integration grids hold exactly the blocks that are resident at once (one wave): a second
// wave of blocks would only add block launches and counter traffic after the first finishes.
std::atomic<int> g_integrate_blocks_per_sm[8];

template <typename Kernel>
int integrate_blocks_per_sm(Kernel kernel, int variant) {
  int b = g_integrate_blocks_per_sm[variant].load(std::memory_order_relaxed);
  if (b == 0) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kernel, 256, 0) != cudaSuccess || b < 1) {
      cudaGetLastError();
      b = 1;
    }
    g_integrate_blocks_per_sm[variant].store(b, std::memory_order_relaxed);
  }
  return b;
}

template <typename Kernel>
cudaError_t launch_integrate_kernel(Kernel kernel, int variant, const MapView& m,
                                    const IntegrateParams& p, int sm_count, cudaStream_t s,
                                    bool dependent) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(sm_count * integrate_blocks_per_sm(kernel, variant));
  cfg.blockDim = dim3(256);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = dependent ? 1 : 0;
  const cudaError_t e = cudaLaunchKernelEx(&cfg, kernel, m, p);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

template <int RM, bool Always>
cudaError_t launch_integrate_t(const MapView& m, const IntegrateParams& p, bool label,
                               int sm_count, cudaStream_t s, bool dependent) {
  const int variant = (label ? 4 : 0) + (RM == NM_ROUND_DOWN ? 2 : 0) + (Always ? 1 : 0);
  if (label)
    return launch_integrate_kernel(k_integrate_label<RM, Always>, variant, m, p, sm_count, s,
                                   dependent);
  return launch_integrate_kernel(k_integrate_count<RM, Always>, variant, m, p, sm_count, s,
                                 dependent);
}

}  // namespace

cudaError_t launch_integrate(const MapView& m, const IntegrateParams& p, int update_mode,
                             int rounding, int sm_count, cudaStream_t s, bool dependent) {
  const bool label = update_mode == NM_UPDATE_LABEL;
  const bool always = p.clamp_mode == NM_CLAMP_ALWAYS;
  if (rounding == NM_ROUND_DOWN)
    return always ? launch_integrate_t<NM_ROUND_DOWN, true>(m, p, label, sm_count, s, dependent)
                  : launch_integrate_t<NM_ROUND_DOWN, false>(m, p, label, sm_count, s, dependent);
  return always ? launch_integrate_t<NM_ROUND_NEAREST, true>(m, p, label, sm_count, s, dependent)
                : launch_integrate_t<NM_ROUND_NEAREST, false>(m, p, label, sm_count, s, dependent);
}

void prepare_integrate() {
  integrate_blocks_per_sm(k_integrate_label<NM_ROUND_DOWN, true>, 7);
  integrate_blocks_per_sm(k_integrate_label<NM_ROUND_DOWN, false>, 6);
  integrate_blocks_per_sm(k_integrate_label<NM_ROUND_NEAREST, true>, 5);
  integrate_blocks_per_sm(k_integrate_label<NM_ROUND_NEAREST, false>, 4);
  integrate_blocks_per_sm(k_integrate_count<NM_ROUND_DOWN, true>, 3);
  integrate_blocks_per_sm(k_integrate_count<NM_ROUND_DOWN, false>, 2);
  integrate_blocks_per_sm(k_integrate_count<NM_ROUND_NEAREST, true>, 1);
  integrate_blocks_per_sm(k_integrate_count<NM_ROUND_NEAREST, false>, 0);
}

cudaError_t launch_rehash(const MapView& from, const MapView& to, uint32_t cur_epoch,
                          int update_mode, cudaStream_t s) {
  k_rehash<<<1184, 256, 0, s>>>(from, to, cur_epoch, update_mode == NM_UPDATE_ACCUMULATE ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_export(const MapView& m, int32_t* origins, float* values, uint32_t* active,
                          uint32_t* n_out, uint32_t max_out, cudaStream_t s) {
  k_export<<<1184, 256, 0, s>>>(m, origins, values, active, n_out, max_out);
  return cudaGetLastError();
}

cudaError_t launch_export_labels(const MapView& m, int plane, int32_t* origins, uint32_t* words,
                                 uint32_t* n_out, uint32_t max_out, cudaStream_t s) {
  k_export_labels<<<1184, 256, 0, s>>>(m, plane, origins, words, n_out, max_out);
  return cudaGetLastError();
}

cudaError_t launch_fill_keys(unsigned long long* keys, uint32_t n, cudaStream_t s) {
  k_fill_keys<<<1184, 256, 0, s>>>(keys, n);
  return cudaGetLastError();
}

}  // namespace nm
