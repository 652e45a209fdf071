// nm_filter.cu -- voxel filter on sm_100a (FilterType 1 of filterCloud.cu:84-434).
//
// Every point the insertion would trace is binned by the voxel holding its end point
// (q = eye + (R p) / res; key = that voxel relative to the eye voxel, `key_bits` per axis) in a
// device hash table, and adds its in-voxel position to the voxel's sums in 32-bit fixed point.
// Lanes of a warp that fall in the same voxel (neighbouring pixels mostly do) first add their
// values with shuffles, and one lane per voxel touches the table: integer sums, so the mean
// does not depend on the order of the atomics.  A voxel's first point appends its slot to a
// list; the second pass walks that list, emits one point per voxel at the mean (or the centre)
// of the voxel, as a world-frame offset from the eye, with its point count, and clears the
// slot for the next frame.  Each filtered point is also stored at the input index of its
// voxel's first point, tagged with the frame, and a block-scan compaction packs the tagged
// points densely in a 2-D-local order of their input pixels (64x64 super-tiles, then 16x16
// tiles, then rows): the traversal (input kind 2, identity rotation) then walks full tiles of
// rays from one small patch of the image.
//
// The reference clears and scans a dense box around the frustum (voxelBufferClear* /
// rayFromFilter*, filterCloud.cu:44-81, 279-434) and sums floats with atomics; this pipeline
// touches only the points and the occupied voxels, and its sums are exact.
#include <algorithm>
#include <cstdint>

#include "nm_device.cuh"
#include "nm_internal.h"

namespace nm {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr double kFix = 4294967296.0;  // 2^32: fractions in [0, 1) -> [0, 2^32)
constexpr int kFilterThreads = 256;
constexpr uint32_t kNone = 0xFFFFFFFFu;

__device__ __forceinline__ bool filter_point(const FrameParams& f, int w, int h, float p[3]) {
  if (f.input_kind == 1) return range_point(f, w, h, p);
  return xyz_point(f, w, h, p);
}

// Slot of `key` in the filter table, inserting it (and listing the slot) when absent.  The
// table holds at most half as many keys as slots, so a free slot is always found.
__device__ __forceinline__ uint32_t filter_slot(const FilterBuffers& b, unsigned long long key) {
  uint32_t h = hash_key(key) & b.table_mask;
  for (uint32_t probe = 0; probe <= b.table_mask; ++probe) {
    const unsigned long long k = __ldcg(&b.table_keys[h]);
    if (k == key) return h;
    if (k == kEmptyKey) {
      const unsigned long long old = atomicCAS(&b.table_keys[h], kEmptyKey, key);
      if (old == kEmptyKey) {
        b.used[atomicAdd(b.n_used, 1u)] = h;
        return h;
      }
      if (old == key) return h;
    }
    h = (h + 1) & b.table_mask;
  }
  return kNone;  // unreachable at load <= 1/2
}

// Bin every point.  The validity test and the rotation are those of the traversal (same
// rounding policy), so exactly the points the unfiltered insert would trace take part.
template <int RM>
__global__ void __launch_bounds__(kFilterThreads) k_filter_bin(FrameParams f, int key_bits,
                                                               FilterBuffers b) {
  using A = Ar<RM>;
  const int n = f.width * f.height;
  const double inv_res = __drcp_rn(f.res_d);
  const int bias = (1 << (key_bits - 1));
  const uint32_t fmask = (1u << key_bits) - 1u;
  const int ev[3] = {(int)floor(f.eye[0]), (int)floor(f.eye[1]), (int)floor(f.eye[2])};
  const int lane = threadIdx.x & 31;
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const int i = base + threadIdx.x;
    unsigned long long key = kEmptyKey;
    unsigned long long F[3] = {0ull, 0ull, 0ull};
    float p[3];
    if (i < n && filter_point(f, i % f.width, i / f.width, p)) {
      const float* R = f.R;
      const float d0 = A::fadd(A::fadd(A::fmul(R[0], p[0]), A::fmul(R[1], p[1])), A::fmul(R[2], p[2]));
      const float d1 = A::fadd(A::fadd(A::fmul(R[3], p[0]), A::fmul(R[4], p[1])), A::fmul(R[5], p[2]));
      const float d2 = A::fadd(A::fadd(A::fmul(R[6], p[0]), A::fmul(R[7], p[1])), A::fmul(R[8], p[2]));
      const double dx = d0, dy = d1, dz = d2;
      const double len = A::dsqrt(A::dadd(A::dadd(A::dmul(dx, dx), A::dmul(dy, dy)), A::dmul(dz, dz)));
      const double ray_len = A::ddiv(len, f.res_d);
      if (ray_len < (double)f.max_time && len > 1.0e-7) {
        const float d[3] = {d0, d1, d2};
        key = 0ull;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const double q = __dadd_rn(f.eye[a], __dmul_rn((double)d[a], inv_res));
          const double v = floor(q);
          F[a] = (unsigned long long)(long long)__dmul_rn(__dadd_rn(q, -v), kFix);
          key = (key << key_bits) | (unsigned long long)((uint32_t)((int)v - ev[a] + bias) & fmask);
        }
      }
    }
    const unsigned peers = __match_any_sync(kFull, key);
    if (key == kEmptyKey) continue;
    unsigned long long t0 = 0, t1 = 0, t2 = 0;
    for (unsigned m = peers; m; m &= m - 1u) {
      const int src = __ffs(m) - 1;
      t0 += __shfl_sync(peers, F[0], src);
      t1 += __shfl_sync(peers, F[1], src);
      t2 += __shfl_sync(peers, F[2], src);
    }
    if (lane == __ffs(peers) - 1) {  // the lowest lane holds the group's lowest input index
      const uint32_t s = filter_slot(b, key);
      if (s != kNone) {
        atomicAdd(&b.table_sums[3 * (size_t)s], t0);
        atomicAdd(&b.table_sums[3 * (size_t)s + 1], t1);
        atomicAdd(&b.table_sums[3 * (size_t)s + 2], t2);
        atomicAdd(&b.table_counts[s], (uint32_t)__popc(peers));
        atomicMin(&b.table_first[s], (uint32_t)i);
      }
    }
  }
}

// One output point per listed slot; the slot is cleared for the next frame.
__global__ void __launch_bounds__(kFilterThreads) k_filter_emit(FrameParams f, int key_bits,
                                                                int centre, FilterBuffers b) {
  const uint32_t ng = *b.n_used;
  const int bias = (1 << (key_bits - 1));
  const unsigned long long fmask = (1ull << key_bits) - 1ull;
  const int ev[3] = {(int)floor(f.eye[0]), (int)floor(f.eye[1]), (int)floor(f.eye[2])};
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
    const uint32_t s = b.used[g];
    const unsigned long long key = b.table_keys[s];
    const uint32_t cnt = b.table_counts[s];
    const uint32_t first = b.table_first[s];
    const double cn = (double)cnt;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int dv = (int)((key >> (key_bits * (2 - a))) & fmask) - bias;
      const double v = (double)(ev[a] + dv);
      const double S = (double)b.table_sums[3 * (size_t)s + a];
      const double mean = centre ? 0.5 : __dmul_rn(__ddiv_rn(S, cn), 1.0 / kFix);
      const float o =
          __double2float_rn(__dmul_rn(__dadd_rn(__dadd_rn(v, mean), -f.eye[a]), f.res_d));
      b.out_pts[3 * (size_t)g + a] = o;
      b.idx_pts[3 * (size_t)first + a] = o;
      b.table_sums[3 * (size_t)s + a] = 0ull;
    }
    b.idx_tags[first] = b.tag;
    b.out_keys[g] = key;
    b.out_counts[g] = cnt;
    b.table_counts[s] = 0u;
    b.table_first[s] = kNone;
    b.table_keys[s] = kEmptyKey;
  }
}

constexpr int kCompactItems = 1024;  // positions per compaction block (4 per thread)

// Compaction order: position j -> input index (or -1 outside the image).  Images at least
// 64 x 64 (and at most 2^28 pixels): super-tiles of 64x64 pixels row-major (stx per row), 4x4 tiles of 16x16 inside,
// rows of 16 inside a tile.  Other inputs (clouds without an image layout): input order.
struct CompactOrder {
  int width, height, stx, tiled;
  __device__ __forceinline__ int index(int j) const {
    if (!tiled) return j;
    const int st = j >> 12, r = j & 4095, t = r >> 8, k = r & 255;
    const int px = (st % stx) * 64 + (t & 3) * 16 + (k & 15);
    const int py = (st / stx) * 64 + (t >> 2) * 16 + (k >> 4);
    return (px < width && py < height) ? py * width + px : -1;
  }
};

// Tagged input indices per compaction block.
__global__ void __launch_bounds__(256) k_compact_count(const uint32_t* tags, uint32_t tag,
                                                       CompactOrder ord, int n,
                                                       uint32_t* block_counts) {
  __shared__ uint32_t s_cnt;
  if (threadIdx.x == 0) s_cnt = 0u;
  __syncthreads();
  const int base = blockIdx.x * kCompactItems;
  uint32_t c = 0;
  for (int r = 0; r < kCompactItems / 256; ++r) {
    const int j = base + r * 256 + threadIdx.x;
    const int i = j < n ? ord.index(j) : -1;
    c += (i >= 0 && tags[i] == tag) ? 1u : 0u;
  }
  c = __reduce_add_sync(kFull, c);
  if ((threadIdx.x & 31) == 0) atomicAdd(&s_cnt, c);
  __syncthreads();
  if (threadIdx.x == 0) block_counts[blockIdx.x] = s_cnt;
}

// Exclusive prefix of the block counts (one CTA, chunks of 256 with a carried total).
__global__ void __launch_bounds__(256) k_compact_scan(uint32_t* block_counts, int nb,
                                                      uint32_t* total) {
  __shared__ uint32_t s_warp[8];
  __shared__ uint32_t s_carry;
  if (threadIdx.x == 0) s_carry = 0u;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c0 = 0; c0 < nb; c0 += 256) {
    const int i = c0 + threadIdx.x;
    const uint32_t v = i < nb ? block_counts[i] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    uint32_t wofs = 0, chunk = 0;
    for (int w = 0; w < 8; ++w) {
      if (w < warp) wofs += s_warp[w];
      chunk += s_warp[w];
    }
    const uint32_t carry = s_carry;
    if (i < nb) block_counts[i] = carry + wofs + x - v;
    __syncthreads();
    if (threadIdx.x == 0) s_carry = carry + chunk;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = s_carry;
}

// Dense points in compaction order: each block writes its tagged points from its prefix on.
__global__ void __launch_bounds__(256) k_compact_write(const uint32_t* tags, uint32_t tag,
                                                       CompactOrder ord, int n,
                                                       const uint32_t* block_offsets,
                                                       const float* idx_pts, float* dense) {
  __shared__ uint32_t s_warp[8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int base = blockIdx.x * kCompactItems;
  uint32_t pos = block_offsets[blockIdx.x];
  for (int r = 0; r < kCompactItems / 256; ++r) {
    const int j = base + r * 256 + threadIdx.x;
    const int i = j < n ? ord.index(j) : -1;
    const bool v = i >= 0 && tags[i] == tag;
    const unsigned bal = __ballot_sync(kFull, v);
    if (lane == 0) s_warp[warp] = __popc(bal);
    __syncthreads();
    uint32_t wofs = 0, round = 0;
    for (int w = 0; w < 8; ++w) {
      if (w < warp) wofs += s_warp[w];
      round += s_warp[w];
    }
    if (v) {
      const uint32_t k = pos + wofs + __popc(bal & ((1u << lane) - 1u));
      dense[3 * (size_t)k] = idx_pts[3 * (size_t)i];
      dense[3 * (size_t)k + 1] = idx_pts[3 * (size_t)i + 1];
      dense[3 * (size_t)k + 2] = idx_pts[3 * (size_t)i + 2];
    }
    pos += round;
    __syncthreads();
  }
}

__global__ void k_filter_table_init(unsigned long long* keys, uint32_t* first, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    keys[i] = kEmptyKey;
    first[i] = kNone;
  }
}

bool compact_tiled(int64_t width, int64_t height) {
  return width >= 64 && height >= 64 && width * height <= (1ll << 28);
}

// Positions of the compaction order for a width x height input: both sides padded to 64 when
// tiled, else the input's own count.  For width * height <= c this stays below 3 c + 4096
// (tiled sides are at most c / 64 each, so the padding adds under 2 c + 4096).
int64_t compact_positions(int64_t width, int64_t height) {
  if (!compact_tiled(width, height)) return width * height;
  return ((width + 63) / 64) * ((height + 63) / 64) * 4096;
}

template <class T>
cudaError_t grow(T** p, size_t count) {
  cudaFree(*p);
  *p = nullptr;
  return cudaMalloc((void**)p, count * sizeof(T));
}

}  // namespace

// Bits per axis: the end voxel lies within max_time + 1 voxels of the eye voxel on every
// axis (|R p| / res < max_time), so fields dv + 2^(b-1) stay inside [1, 2^b - 2] and no key
// of a point equals the all-ones empty key.
int filter_key_bits(float max_time) {
  if (!(max_time >= 0.0f)) return 0;
  int b = 2;
  while (b <= 21 && (double)((1u << (b - 1)) - 1u) < (double)max_time + 4.0) ++b;
  return b <= 21 ? b : 0;
}

cudaError_t filter_reserve(FilterBuffers* b, int64_t n, cudaStream_t s) {
  if (n <= b->capacity) return cudaSuccess;
  const int64_t c = std::max<int64_t>(n, 1 << 16);
  uint64_t tc = 1;
  while (tc < 2 * (uint64_t)c) tc <<= 1;
  filter_release(b);
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = grow(&b->table_keys, tc);
  if (e == cudaSuccess) e = grow(&b->table_sums, 3 * tc);
  if (e == cudaSuccess) e = grow(&b->table_counts, tc);
  if (e == cudaSuccess) e = grow(&b->table_first, tc);
  if (e == cudaSuccess) e = grow(&b->used, c);
  if (e == cudaSuccess) e = grow(&b->n_used, 4);
  if (e == cudaSuccess) e = grow(&b->out_pts, 3 * c);
  if (e == cudaSuccess) e = grow(&b->out_keys, c);
  if (e == cudaSuccess) e = grow(&b->out_counts, c);
  if (e == cudaSuccess) e = grow(&b->idx_pts, 3 * c);
  if (e == cudaSuccess) e = grow(&b->idx_tags, c);
  if (e == cudaSuccess) e = grow(&b->dense_pts, 3 * c);
  if (e == cudaSuccess) e = grow(&b->block_counts, (3 * c + 4096 + kCompactItems - 1) / kCompactItems);
  if (e == cudaSuccess) e = grow(&b->n_dense, 4);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->table_sums, 0, 3 * tc * sizeof(unsigned long long), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->table_counts, 0, tc * sizeof(uint32_t), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b->idx_tags, 0, c * sizeof(uint32_t), s);
  if (e == cudaSuccess) {
    k_filter_table_init<<<1184, 256, 0, s>>>(b->table_keys, b->table_first, (uint32_t)tc);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    filter_release(b);
    return e;
  }
  b->capacity = c;
  b->table_mask = (uint32_t)(tc - 1);
  b->tag = 0u;
  return cudaSuccess;
}

void filter_release(FilterBuffers* b) {
  cudaFree(b->table_keys);
  cudaFree(b->table_sums);
  cudaFree(b->table_counts);
  cudaFree(b->table_first);
  cudaFree(b->used);
  cudaFree(b->n_used);
  cudaFree(b->out_pts);
  cudaFree(b->out_keys);
  cudaFree(b->out_counts);
  cudaFree(b->idx_pts);
  cudaFree(b->idx_tags);
  cudaFree(b->dense_pts);
  cudaFree(b->block_counts);
  cudaFree(b->n_dense);
  *b = FilterBuffers{};
}

cudaError_t run_voxel_filter(const FrameParams& f, int rounding, int centre, int key_bits,
                             const FilterBuffers& b, cudaStream_t s) {
  const int n = f.width * f.height;
  cudaError_t e = cudaMemsetAsync(b.n_used, 0, sizeof(uint32_t), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b.n_dense, 0, sizeof(uint32_t), s);
  if (e != cudaSuccess || n <= 0) return e;
  if (n > b.capacity || key_bits < 2 || key_bits > 21) return cudaErrorInvalidValue;
  const int grid = std::min<int>((n + kFilterThreads - 1) / kFilterThreads, 148 * 8);
  if (rounding == NM_ROUND_DOWN)
    k_filter_bin<NM_ROUND_DOWN><<<grid, kFilterThreads, 0, s>>>(f, key_bits, b);
  else
    k_filter_bin<NM_ROUND_NEAREST><<<grid, kFilterThreads, 0, s>>>(f, key_bits, b);
  e = cudaGetLastError();
  if (e == cudaSuccess) {
    k_filter_emit<<<grid, kFilterThreads, 0, s>>>(f, key_bits, centre, b);
    e = cudaGetLastError();
  }
  const CompactOrder ord{f.width, f.height, (f.width + 63) / 64,
                         compact_tiled(f.width, f.height) ? 1 : 0};
  const int nj = (int)compact_positions(f.width, f.height);
  const int nb = (nj + kCompactItems - 1) / kCompactItems;
  if (e == cudaSuccess) {
    k_compact_count<<<nb, 256, 0, s>>>(b.idx_tags, b.tag, ord, nj, b.block_counts);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    k_compact_scan<<<1, 256, 0, s>>>(b.block_counts, nb, b.n_dense);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    k_compact_write<<<nb, 256, 0, s>>>(b.idx_tags, b.tag, ord, nj, b.block_counts, b.idx_pts,
                                       b.dense_pts);
    e = cudaGetLastError();
  }
  return e;
}

}  // namespace nm
