// nm_sim.cu -- simulation map build and simulated-depth ray casting on sm_100a.
//
// Replaces the NanoVDB sim grid upload (SimHandler.cpp:22-23) and generateCloud /
// viewSimKernel / getActiveCrossing (generateCloud.cu:20-94).
//
// Sim map layout: a table over the brick box (64^3-voxel bricks) naming each non-empty brick's
// block of 512 leaf entries, each entry the index of a compact 8^3 bit leaf (16 words) or -1;
// empty bricks give the walk its long empty-space skips.
//
// The ray cast itself (sim_cast, sim_ray) and the range noise live in nm_sim_device.cuh,
// shared with the traversal kernel's fused render.
#include <cfloat>
#include <cmath>
#include <algorithm>
#include <cstdint>

#include "nm_sim.h"
#include "nm_sim_device.cuh"

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

// Pass 1: count non-empty leaves (one atomic per block) and flag their bricks in
// v.brick_index (set to 1; the host then numbers the flagged bricks).  Pass 2: give each leaf
// a compact index (block-wide scan, one atomic per block and iteration), copy its words, enter
// it in its brick's block, and fold its voxels into the active bounding box and voxel count
// (reduced per block, one set of atomics per block).  One thread per leaf of the build box.
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
    long long bpos = 0;
    int bx = 0, by = 0, bz = 0;
    if (any) {
      const int lz = (int)(pos % b.ldim[2]);
      const int ly = (int)((pos / b.ldim[2]) % b.ldim[1]);
      const int lx = (int)(pos / ((long long)b.ldim[2] * b.ldim[1]));
      bx = lx + b.llo[0];
      by = ly + b.llo[1];
      bz = lz + b.llo[2];
      bpos = ((long long)((bx >> 3) - v.blo[0]) * v.bdim[1] + ((by >> 3) - v.blo[1])) * v.bdim[2] +
             ((bz >> 3) - v.blo[2]);
    }
    if (!pass2) {
      nonempty += any ? 1u : 0u;
      if (any) v.brick_index[bpos] = 1;
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
    if (any) {
      uint4* dst = reinterpret_cast<uint4*>(v.leaf_words) + (size_t)idx * 4;
#pragma unroll
      for (int i = 0; i < 4; ++i) dst[i] = w[i];
      const int32_t blk = v.brick_index[bpos];
      const int e = ((bx & 7) << 6) | ((by & 7) << 3) | (bz & 7);
      v.brick_leaves[(size_t)blk * 512 + e] = (int32_t)idx;
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

// ---- empty-space distances (render acceleration) -----------------------------------------
//
// Every empty leaf of a non-empty brick gets its Chebyshev distance d, in leaves and capped at
// kSkipCap, to the nearest leaf with active voxels, stored as -d in its brick_leaves entry (-1:
// an empty leaf next to an occupied one, as before).  The render then skips the cube of
// (2d - 1)^3 leaves around it, all empty, in one exact step.  The distances come from a
// separable L-infinity distance transform over the build's leaf box: one pass per axis, each
// the minimum over offsets |o| < kSkipCap of max(|o|, the previous value at p + o); leaves
// outside the box count as empty.
constexpr int kSkipCap = 8;

__global__ void k_skip_init(SimBuild b, uint8_t* dist) {
  const long long total = (long long)b.ldim[0] * b.ldim[1] * b.ldim[2];
  const uint4* src = reinterpret_cast<const uint4*>(b.dense);
  for (long long pos = (long long)blockIdx.x * blockDim.x + threadIdx.x; pos < total;
       pos += (long long)gridDim.x * blockDim.x) {
    uint32_t any = 0u;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const uint4 w = __ldg(&src[pos * 4 + i]);
      any |= w.x | w.y | w.z | w.w;
    }
    dist[pos] = any ? 0 : (uint8_t)kSkipCap;
  }
}

__global__ void k_skip_pass(const uint8_t* src, uint8_t* dst, int nx, int ny, int nz, int axis) {
  const long long total = (long long)nx * ny * nz;
  const long long step = axis == 0 ? (long long)ny * nz : (axis == 1 ? (long long)nz : 1);
  const int n = axis == 0 ? nx : (axis == 1 ? ny : nz);
  for (long long pos = (long long)blockIdx.x * blockDim.x + threadIdx.x; pos < total;
       pos += (long long)gridDim.x * blockDim.x) {
    const int c = (int)((pos / step) % n);
    int best = src[pos];
    for (int o = 1; o < best; ++o) {  // an offset >= best cannot lower it
      if (c - o >= 0) best = min(best, max(o, (int)src[pos - o * step]));
      if (c + o < n) best = min(best, max(o, (int)src[pos + o * step]));
    }
    dst[pos] = (uint8_t)best;
  }
}

__global__ void k_skip_write(SimBuild b, SimMapView v, const uint8_t* dist) {
  const long long total = (long long)b.ldim[0] * b.ldim[1] * b.ldim[2];
  for (long long pos = (long long)blockIdx.x * blockDim.x + threadIdx.x; pos < total;
       pos += (long long)gridDim.x * blockDim.x) {
    const int d = dist[pos];
    if (d == 0) continue;  // an occupied leaf keeps its index
    const int lx = (int)(pos / ((long long)b.ldim[2] * b.ldim[1])) + b.llo[0];
    const int ly = (int)((pos / b.ldim[2]) % b.ldim[1]) + b.llo[1];
    const int lz = (int)(pos % b.ldim[2]) + b.llo[2];
    const long long bpos =
        ((long long)((lx >> 3) - v.blo[0]) * v.bdim[1] + ((ly >> 3) - v.blo[1])) * v.bdim[2] +
        ((lz >> 3) - v.blo[2]);
    const int32_t blk = v.brick_index[bpos];
    if (blk < 0) continue;
    const int e = ((lx & 7) << 6) | ((ly & 7) << 3) | (lz & 7);
    v.brick_leaves[(size_t)blk * 512 + e] = -d;
  }
}

__global__ void k_fill_i32(int32_t* p, long long n, int32_t v) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    p[i] = v;
}

// 8x8-pixel tiles of 64 threads: many small CTAs balance the uneven ray costs better than
// 16x16 tiles (5 % faster on the headline frame).
__global__ void __launch_bounds__(64) k_sim_render(SimMapView v, SimRayParams rp, float* out) {
  const int w = blockIdx.x * 8 + (threadIdx.x & 7);
  const int h = blockIdx.y * 8 + (threadIdx.x >> 3);
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

__global__ void k_noise(float* r, long long n, float sigma_coef, float drop, uint64_t seed) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    r[i] = noisy(r[i], seed, i, sigma_coef, drop);
}

// Render and range noise in one pass: the same ranges as k_sim_render followed by k_noise.
__global__ void __launch_bounds__(64) k_sim_render_noisy(SimMapView v, SimRayParams rp, float* out,
                                                         float sigma_coef, float drop,
                                                         uint64_t seed) {
  const int w = blockIdx.x * 8 + (threadIdx.x & 7);
  const int h = blockIdx.y * 8 + (threadIdx.x >> 3);
  if (w >= rp.width || h >= rp.height) return;
  const long long i = (long long)h * rp.width + w;
  out[i] = noisy(sim_ray(v, rp, w, h), seed, i, sigma_coef, drop);
}

// All slots of a tick plan in one launch: one CTA per kRenderTile^2-pixel tile of some slot.
__global__ void __launch_bounds__(kRenderTile * kRenderTile) k_sim_render_batch(const RenderBatch* b,
                                                                            SimMapView v) {
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
  const int w = tx * kRenderTile + (int)(threadIdx.x % kRenderTile);
  const int h = ty * kRenderTile + (int)(threadIdx.x / kRenderTile);
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

cudaError_t launch_skip_distances(const SimBuild& b, const SimMapView& v, uint8_t* d_a,
                                  uint8_t* d_b, cudaStream_t s) {
  k_skip_init<<<1184, 256, 0, s>>>(b, d_a);
  k_skip_pass<<<1184, 256, 0, s>>>(d_a, d_b, b.ldim[0], b.ldim[1], b.ldim[2], 0);
  k_skip_pass<<<1184, 256, 0, s>>>(d_b, d_a, b.ldim[0], b.ldim[1], b.ldim[2], 1);
  k_skip_pass<<<1184, 256, 0, s>>>(d_a, d_b, b.ldim[0], b.ldim[1], b.ldim[2], 2);
  k_skip_write<<<1184, 256, 0, s>>>(b, v, d_b);
  return cudaGetLastError();
}

cudaError_t launch_fill_i32(int32_t* p, long long n, int32_t val, cudaStream_t s) {
  k_fill_i32<<<1184, 256, 0, s>>>(p, n, val);
  return cudaGetLastError();
}

cudaError_t launch_sim_render_noisy(const SimMapView& v, const SimRayParams& rp, float* out,
                                    float sigma_coef, float drop, uint64_t seed, cudaStream_t s) {
  const dim3 grid((rp.width + 7) / 8, (rp.height + 7) / 8);
  k_sim_render_noisy<<<grid, 64, 0, s>>>(v, rp, out, sigma_coef, drop, seed);
  return cudaGetLastError();
}

cudaError_t launch_sim_render(const SimMapView& v, const SimRayParams& rp, float* out, cudaStream_t s) {
  const dim3 grid((rp.width + 7) / 8, (rp.height + 7) / 8);
  k_sim_render<<<grid, 64, 0, s>>>(v, rp, out);
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
  if (total_tiles > 0)
    k_sim_render_batch<<<total_tiles, kRenderTile * kRenderTile, 0, s>>>(d_batch, v);
  return cudaGetLastError();
}

cudaError_t launch_noise(float* r, long long n, float sigma_coef, float drop, uint64_t seed,
                         cudaStream_t s) {
  k_noise<<<1184, 256, 0, s>>>(r, n, sigma_coef, drop, seed);
  return cudaGetLastError();
}

}  // namespace nm
