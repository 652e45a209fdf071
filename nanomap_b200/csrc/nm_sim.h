// nm_sim.h -- simulation-map structures shared by the host code and the sm_100a kernels.
#pragma once

#include <climits>
#include <cstdint>
#include <cuda_runtime.h>

#include "nanomap_b200.h"
#include "nm_internal.h"

namespace nm {

// Build state: a dense leaf-major bit buffer over the leaf box (16 words per leaf).
struct SimBuild {
  float res;
  int32_t vmin[3], vmax[3];  // voxel region [vmin, vmax)
  int32_t llo[3], ldim[3];   // leaf box origin (leaf coordinates) and size
  uint32_t* dense;
  int32_t borrowed;          // dense belongs to the caller (not freed by the build)
};

// Two-level index, like the upper levels of a NanoVDB tree: a table over the brick box (64^3
// voxels per brick) names each non-empty brick's block of 512 leaf entries (its 8^3 leaves,
// x*64 + y*8 + z), and each entry names a compact 64-byte bit leaf.  Memory follows the
// occupied bricks and leaves, not the volume of the scene's box.
struct SimMapView {
  float res;
  int32_t any;
  int32_t llo[3], ldim[3];   // leaf box
  int32_t blo[3], bdim[3];   // brick box (64^3-voxel bricks)
  int32_t* brick_index;      // bdim product entries: block of the brick, -1 = empty brick
  int32_t* brick_leaves;     // 512 entries per block: compact leaf index; an empty leaf -d, d
                             // its Chebyshev distance in leaves (>= 1, capped) to an occupied one
  uint32_t* leaf_words;      // 16 words per non-empty leaf
  float box_lo[3], box_hi[3];  // active voxel box in index space, [amin, amax + 1]
};

struct SimRayParams {
  int32_t type, width, height, pad;
  float hw, hh, c0, c1, su, sv;
  const float* sinu;
  const float* cosu;
  const float* sinv;
  const float* cosv;
  float R[9];
  float pos[3];
  float min_range, max_range;
  // per-frame constants of every pixel's ray, divided on the host (IEEE round to nearest, the
  // same values as dividing on the device): the eye in voxel units and the range limits
  float eye[3];
  float tmin, tmax;  // min_range / res, max_range / res
  int32_t pad2;
};

// Fused simulated frame: the traversal renders each tile's ranges from the sim map (with the
// simulated sensors' range noise when `noise` is set) into shared memory and walks them; the
// ranges also go to `out` when it is set.  Passed by value to the kernel.
struct SimRender {
  SimMapView v;
  SimRayParams rp;
  float sigma_coef, drop;
  uint64_t seed;
  int32_t noise;
  int32_t pad;
  float* out;
};

cudaError_t launch_traverse_render(const TickWork<1>& w, const MapView& m, const SimRender& sr,
                                   int rounding, cudaStream_t s);

constexpr int kMaxRenderSlots = 32;
// Pixels per side of a batched render tile (one CTA of kRenderTile^2 threads per tile).
constexpr int kRenderTile = 8;

// Every slot of a tick plan rendered (and optionally noised) in one launch.
struct RenderBatch {
  int32_t n;
  int32_t noise;
  float noise_coef, drop;
  uint32_t tile_start[kMaxRenderSlots + 1];  // 16x16 tiles per slot, prefix sums
  int32_t tiles_x[kMaxRenderSlots];
  float* out[kMaxRenderSlots];
  uint64_t noise_seed[kMaxRenderSlots];
  SimRayParams rp[kMaxRenderSlots];
};

cudaError_t launch_render_batch(const RenderBatch* d_batch, uint32_t total_tiles,
                                const SimMapView& v, cudaStream_t s);
cudaError_t launch_voxelize(const SimBuild& b, const double* d_boxes, int nb, const double* d_cyl,
                            int nc, cudaStream_t s);
cudaError_t launch_set_voxels(const SimBuild& b, const int32_t* d_ijk, long long n, cudaStream_t s);
cudaError_t launch_compact(const SimBuild& b, const SimMapView& v, uint32_t* d_count, int pass2,
                           int32_t* d_bbox, unsigned long long* d_nvox, cudaStream_t s);
cudaError_t launch_fill_i32(int32_t* p, long long n, int32_t val, cudaStream_t s);
// After compaction, with the dense leaf buffer still there: the empty leaves' distances to the
// nearest occupied leaf into v.brick_leaves (-d); d_a and d_b hold one byte per leaf of the
// build's leaf box each.
cudaError_t launch_skip_distances(const SimBuild& b, const SimMapView& v, uint8_t* d_a,
                                  uint8_t* d_b, cudaStream_t s);
cudaError_t launch_sim_render_noisy(const SimMapView& v, const SimRayParams& rp, float* out,
                                    float sigma_coef, float drop, uint64_t seed, cudaStream_t s);
cudaError_t launch_sim_render(const SimMapView& v, const SimRayParams& rp, float* out,
                              cudaStream_t s);
cudaError_t launch_noise(float* r, long long n, float sigma_coef, float drop, uint64_t seed,
                         cudaStream_t s);
cudaError_t launch_sim_cast(const SimMapView& v, const float* origins, const float* dirs,
                            long long n, float max_range, float* out, cudaStream_t s);

}  // namespace nm
