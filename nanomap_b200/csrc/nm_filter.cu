// nm_filter.cu -- voxel filter on sm_100a (FilterType 1 of filterCloud.cu:84-434).
//
// Every point the insertion would trace is keyed by the voxel holding its end point
// (q = eye + (R p) / res; key = that voxel relative to the eye voxel, `key_bits` per axis).
// A radix sort of (key, point index) over the key's 3 * key_bits low bits groups the points of
// a voxel; head flags and a scan number the groups in key order; each point adds its in-voxel
// position to its group in 32-bit fixed point, summed per warp over lanes of the same group
// first (exact integer sums, so the mean does not depend on the order of the atomics); the
// finaliser emits one point per voxel, at the mean (or the centre) of the voxel, as a
// world-frame offset from the eye, with its point count.  The filtered points then go through
// the ordinary traversal as input kind 2 with an identity rotation.
//
// The reference clears and scans a dense box around the frustum (voxelBufferClear* /
// rayFromFilter*, filterCloud.cu:44-81, 279-434), sums floats with atomics and orders the
// output by an atomic counter; this pipeline touches only the points, and its output is
// deterministic.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <cstdint>

#include "nm_device.cuh"
#include "nm_internal.h"

namespace nm {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr double kFix = 4294967296.0;  // 2^32: fractions in [0, 1) -> [0, 2^32)
constexpr int kFilterThreads = 256;

__device__ __forceinline__ bool filter_point(const FrameParams& f, int w, int h, float p[3]) {
  if (f.input_kind == 1) return range_point(f, w, h, p);
  return xyz_point(f, w, h, p);
}

// Key and fixed-point fractions of every input point.  The validity test and the rotation
// are those of the traversal (same rounding policy), so exactly the points the unfiltered
// insert would trace take part.
template <int RM>
__global__ void __launch_bounds__(kFilterThreads) k_filter_keys(FrameParams f, int key_bits,
                                                                unsigned long long* keys,
                                                                uint32_t* idx, long long* frac) {
  using A = Ar<RM>;
  const int n = f.width * f.height;
  const double inv_res = __drcp_rn(f.res_d);
  const int bias = (1 << (key_bits - 1));
  const uint32_t fmask = (1u << key_bits) - 1u;
  const int ev[3] = {(int)floor(f.eye[0]), (int)floor(f.eye[1]), (int)floor(f.eye[2])};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    idx[i] = (uint32_t)i;
    unsigned long long key = kEmptyKey;
    float p[3];
    if (filter_point(f, i % f.width, i / f.width, p)) {
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
          frac[3 * (size_t)i + a] = (long long)__dmul_rn(__dadd_rn(q, -v), kFix);
          key = (key << key_bits) | (unsigned long long)((uint32_t)((int)v - ev[a] + bias) & fmask);
        }
      }
    }
    keys[i] = key;
  }
}

__global__ void k_filter_heads(const unsigned long long* keys, int n, uint32_t* heads) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const unsigned long long k = keys[i];
    heads[i] = (k != kEmptyKey && (i == 0 || keys[i - 1] != k)) ? 1u : 0u;
  }
}

// Group sums.  Keys are sorted, so the lanes of one group are contiguous: each lane adds the
// values of its group's lanes (shuffles within the group), and the group's first lane issues
// the atomics.  Invalid points (key ~0) sort last and add nothing.
__global__ void __launch_bounds__(kFilterThreads) k_filter_accumulate(
    const unsigned long long* keys, const uint32_t* idx, const uint32_t* seg,
    const long long* frac, int n, unsigned long long* group_key, long long* sums,
    uint32_t* counts) {
  const int lane = threadIdx.x & 31;
  for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    const int i = base + threadIdx.x;
    const unsigned long long key = i < n ? keys[i] : kEmptyKey;
    const bool valid = key != kEmptyKey;
    const uint32_t g = valid ? seg[i] - 1u : 0xFFFFFFFFu;
    long long s0 = 0, s1 = 0, s2 = 0;
    if (valid) {
      const uint32_t j = idx[i];
      s0 = frac[3 * (size_t)j];
      s1 = frac[3 * (size_t)j + 1];
      s2 = frac[3 * (size_t)j + 2];
      if (i == 0 || keys[i - 1] != key) group_key[g] = key;
    }
    const unsigned peers = __match_any_sync(kFull, g);
    long long t0 = 0, t1 = 0, t2 = 0;
    for (unsigned m = peers; m; m &= m - 1u) {
      const int src = __ffs(m) - 1;
      t0 += __shfl_sync(peers, s0, src);
      t1 += __shfl_sync(peers, s1, src);
      t2 += __shfl_sync(peers, s2, src);
    }
    if (valid && lane == __ffs(peers) - 1) {
      unsigned long long* su = reinterpret_cast<unsigned long long*>(sums + 3 * (size_t)g);
      atomicAdd(su, (unsigned long long)t0);
      atomicAdd(su + 1, (unsigned long long)t1);
      atomicAdd(su + 2, (unsigned long long)t2);
      atomicAdd(&counts[g], (uint32_t)__popc(peers));
    }
  }
}

__global__ void k_filter_finalize(FrameParams f, int key_bits, int centre, const uint32_t* seg,
                                  int n, const unsigned long long* group_key,
                                  const long long* sums, const uint32_t* counts, float* out_pts,
                                  uint32_t* n_out) {
  const uint32_t ng = seg[n - 1];
  if (blockIdx.x == 0 && threadIdx.x == 0) *n_out = ng;
  const int bias = (1 << (key_bits - 1));
  const unsigned long long fmask = (1ull << key_bits) - 1ull;
  const int ev[3] = {(int)floor(f.eye[0]), (int)floor(f.eye[1]), (int)floor(f.eye[2])};
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < ng; g += gridDim.x * blockDim.x) {
    const unsigned long long key = group_key[g];
    const double cn = (double)counts[g];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int dv = (int)((key >> (key_bits * (2 - a))) & fmask) - bias;
      const double v = (double)(ev[a] + dv);
      const double mean =
          centre ? 0.5 : __dmul_rn(__ddiv_rn((double)sums[3 * (size_t)g + a], cn), 1.0 / kFix);
      out_pts[3 * (size_t)g + a] =
          __double2float_rn(__dmul_rn(__dadd_rn(__dadd_rn(v, mean), -f.eye[a]), f.res_d));
    }
  }
}

template <class T>
cudaError_t grow(T** p, size_t count) {
  cudaFree(*p);
  *p = nullptr;
  return cudaMalloc((void**)p, count * sizeof(T));
}

}  // namespace

// Bits per axis: the end voxel lies within max_time + 1 voxels of the eye voxel on every
// axis (|R p| / res < max_time), so fields dv + 2^(b-1) stay inside [1, 2^b - 2] and the
// all-ones key (no point) sorts after every real one.
int filter_key_bits(float max_time) {
  if (!(max_time >= 0.0f)) return 0;
  const double need = 2.0 * ((double)max_time + 4.0);
  int b = 2;
  while (b <= 21 && (double)((1u << (b - 1)) - 1u) < need / 2.0) ++b;
  return b <= 21 ? b : 0;
}

cudaError_t filter_reserve(FilterBuffers* b, int64_t n) {
  if (n <= b->capacity) return cudaSuccess;
  const int64_t c = std::max<int64_t>(n, 1 << 16);
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = grow(&b->keys_in, c);
  if (e == cudaSuccess) e = grow(&b->keys_out, c);
  if (e == cudaSuccess) e = grow(&b->group_key, c);
  if (e == cudaSuccess) e = grow(&b->idx_in, c);
  if (e == cudaSuccess) e = grow(&b->idx_out, c);
  if (e == cudaSuccess) e = grow(&b->heads, c);
  if (e == cudaSuccess) e = grow(&b->seg, c);
  if (e == cudaSuccess) e = grow(&b->counts, c);
  if (e == cudaSuccess && !b->n_out) e = cudaMalloc((void**)&b->n_out, 16);
  if (e == cudaSuccess) e = grow(&b->frac, 3 * c);
  if (e == cudaSuccess) e = grow(&b->sums, 3 * c);
  if (e == cudaSuccess) e = grow(&b->out_pts, 3 * c);
  size_t a = 0, s = 0;
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortPairs(nullptr, a, b->keys_in, b->keys_out, b->idx_in, b->idx_out,
                                        (int)c, 0, 64);
  if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(nullptr, s, b->heads, b->seg, (int)c);
  if (e == cudaSuccess) {
    b->temp_bytes = std::max(a, s);
    e = grow(reinterpret_cast<unsigned char**>(&b->temp), b->temp_bytes);
  }
  if (e != cudaSuccess) {
    filter_release(b);
    return e;
  }
  b->capacity = c;
  return cudaSuccess;
}

void filter_release(FilterBuffers* b) {
  cudaFree(b->keys_in);
  cudaFree(b->keys_out);
  cudaFree(b->group_key);
  cudaFree(b->idx_in);
  cudaFree(b->idx_out);
  cudaFree(b->heads);
  cudaFree(b->seg);
  cudaFree(b->counts);
  cudaFree(b->n_out);
  cudaFree(b->frac);
  cudaFree(b->sums);
  cudaFree(b->out_pts);
  cudaFree(b->temp);
  *b = FilterBuffers{};
}

cudaError_t run_voxel_filter(const FrameParams& f, int rounding, int centre, int key_bits,
                             const FilterBuffers& b, cudaStream_t s) {
  const int n = f.width * f.height;
  if (n <= 0) return cudaMemsetAsync(b.n_out, 0, 4, s);
  if (n > b.capacity || key_bits < 2 || key_bits > 21) return cudaErrorInvalidValue;
  const int grid = std::min<int>((n + kFilterThreads - 1) / kFilterThreads, 148 * 8);
  if (rounding == NM_ROUND_DOWN)
    k_filter_keys<NM_ROUND_DOWN><<<grid, kFilterThreads, 0, s>>>(f, key_bits, b.keys_in, b.idx_in, b.frac);
  else
    k_filter_keys<NM_ROUND_NEAREST><<<grid, kFilterThreads, 0, s>>>(f, key_bits, b.keys_in, b.idx_in, b.frac);
  cudaError_t e = cudaGetLastError();
  size_t tb = b.temp_bytes;
  if (e == cudaSuccess)
    e = cub::DeviceRadixSort::SortPairs(b.temp, tb, b.keys_in, b.keys_out, b.idx_in, b.idx_out, n,
                                        0, 3 * key_bits, s);
  if (e == cudaSuccess) {
    k_filter_heads<<<grid, kFilterThreads, 0, s>>>(b.keys_out, n, b.heads);
    e = cudaGetLastError();
  }
  tb = b.temp_bytes;
  if (e == cudaSuccess) e = cub::DeviceScan::InclusiveSum(b.temp, tb, b.heads, b.seg, n, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b.sums, 0, (size_t)n * 3 * sizeof(long long), s);
  if (e == cudaSuccess) e = cudaMemsetAsync(b.counts, 0, (size_t)n * sizeof(uint32_t), s);
  if (e == cudaSuccess) {
    k_filter_accumulate<<<grid, kFilterThreads, 0, s>>>(b.keys_out, b.idx_out, b.seg, b.frac, n,
                                                        b.group_key, b.sums, b.counts);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    k_filter_finalize<<<grid, kFilterThreads, 0, s>>>(f, key_bits, centre, b.seg, n, b.group_key,
                                                      b.sums, b.counts, b.out_pts, b.n_out);
    e = cudaGetLastError();
  }
  return e;
}

}  // namespace nm
