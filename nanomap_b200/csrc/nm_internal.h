// nm_internal.h -- structures shared by the host code and the sm_100a kernels.
//
// Device map layout (one open-addressing hash table; the table position of a leaf is its
// storage slot, so inserting a leaf never has to publish an index):
//   keys      u64[C]          leaf key (packed leaf coordinate), ~0 = empty
//   values    f32[C][512]     log-odds, voxel index x*64 + y*8 + z inside the 8^3 leaf
//   active    u32[C][16]      active (occupied) bit per voxel
//   labels    u32[P][C][32]   per-frame labels per plane: words 0..15 hit, 16..31 miss
//   counts    u32[C][1024]    per-frame hit (0..511) and miss (512..1023) counts, accumulate mode
//   epoch     u32[C]          frame id that last put the slot on the touched list
//   plane_mask u32[C]         planes holding labels for the slot (batched ticks)
//   touched   u32[C]          slots labelled by the current frame / tick
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "nanomap_b200.h"

namespace nm {

constexpr uint64_t kEmptyKey = ~0ull;
constexpr int kLeafVoxels = 512;
constexpr int kLabelWords = 32;
constexpr int kActiveWords = 16;
constexpr int kMaxPlanes = 32;
constexpr uint32_t kMaxProbe = 4096;
// Largest leaf-table capacity (slots): at >2 KB per slot, 2^26 slots fill a 180 GB GPU.
constexpr uint64_t kMaxLeafCapacity = 1ull << 26;

// Device-side error bits (sticky until read by nm_map_stats).
constexpr uint32_t kErrProbe = 1u;     // leaf table probe limit reached: labels were lost
constexpr uint32_t kErrTimeout = 2u;   // a bounded wait gave up
constexpr uint32_t kErrPlane = 4u;     // plane index outside the allocated planes

struct MapCounters {
  unsigned long long rays;
  unsigned long long visits;
  unsigned long long unique_voxels;
  unsigned long long touched_total;
  unsigned int leaf_count;
  unsigned int error_flags;
  // one 8-byte word: the integration reads the frame's count and takes its block ticket with
  // one 64-bit atomic
  unsigned int touched_count;
  unsigned int done_blocks;
  unsigned int frames;
  unsigned int tile_queue;  // persistent traversal work counter (reset by its last reader)
  unsigned long long depth_visits;  // voxels visited by the expected-depth kernels
};

struct MapView {
  unsigned long long* keys;
  float* values;
  uint32_t* active;
  uint32_t* labels;
  uint32_t* counts;
  uint32_t* epoch;
  uint32_t* plane_mask;
  uint32_t* touched;
  MapCounters* ctr;
  uint32_t mask;       // capacity - 1 (capacity is a power of two)
  uint32_t capacity;
  int32_t planes;
  int32_t pad;
};

// Per-frame constants of one traversal launch.
struct FrameParams {
  int32_t type;        // NM_SENSOR_FRUSTUM / NM_SENSOR_LASER
  int32_t width, height;
  int32_t input_kind;  // 0 xyz records, 1 range image, 2 xyz records counted on the device
  float hw, hh, c0, c1, su, sv;  // frustum pixel model
  const float* sinu;   // laser tables (device)
  const float* cosu;
  const float* sinv;
  const float* cosv;
  const unsigned char* xyz;
  int64_t step;        // bytes between xyz records
  const float* ranges;
  const uint32_t* n_valid;  // input_kind 2: records [0, *n_valid) are valid
  float R[9];          // row-major, world-from-sensor
  double eye[3];       // index-space eye
  double res_d;
  float max_time;      // max_range / res
  uint32_t epoch;
  int32_t plane;
  int32_t pad;
};

constexpr int kMaxTickFrames = 32;

// Frames with max_range / res below this many voxels reach at most 501 leaves from the eye on
// every axis, inside the range where the traversal's 32-bit leaf code is one-to-one; farther
// reaching frames take the traversal without the shared leaf table.
constexpr float kNarrowMaxTime = 4000.0f;

// Work list of one traversal launch: frames and the prefix sum of their tile counts.
// Passed by value as a __grid_constant__ kernel parameter (no host-to-device copy, so a
// launch can be captured in a CUDA graph).
template <int MaxF>
struct TickWork {
  int32_t n_frames;
  int32_t tile_w, tile_h;
  uint32_t smask;         // shared-memory leaf table entries - 1 (power of two)
  uint32_t total_tiles;
  // claim order of the tiles (longest walks first; null = tile order): the number of tiles in
  // each of kOrderBuckets walk-length buckets, and bucket b's tiles at order_lists[b * order_cap];
  // the traversal zeroes the counts once every CTA has read them, for the next order pass
  uint32_t* order_counts;
  const uint32_t* order_lists;
  uint32_t order_cap;
  float order_scale;      // buckets per walk step: kOrderBuckets / (longest possible walk)
  uint32_t tile_start[MaxF + 1];
  int32_t tiles_x[MaxF];
  FrameParams fr[MaxF];
};

struct IntegrateParams {
  float lh[kMaxPlanes];
  float lm[kMaxPlanes];
  float thres_hit, thres_miss, clamp_min, clamp_max;
  int32_t clamp_mode;
  int32_t use_planes;  // 0: plane 0 only (plain path); 1: iterate plane_mask
  int32_t pad[2];
};

__host__ __device__ inline uint64_t leaf_key(int lx, int ly, int lz) {
  return ((uint64_t)((uint32_t)(lx + (1 << 20)) & 0x1FFFFFu) << 42) |
         ((uint64_t)((uint32_t)(ly + (1 << 20)) & 0x1FFFFFu) << 21) |
         (uint64_t)((uint32_t)(lz + (1 << 20)) & 0x1FFFFFu);
}

__host__ __device__ inline void key_leaf(uint64_t k, int* lx, int* ly, int* lz) {
  *lx = (int)((k >> 42) & 0x1FFFFFu) - (1 << 20);
  *ly = (int)((k >> 21) & 0x1FFFFFu) - (1 << 20);
  *lz = (int)(k & 0x1FFFFFu) - (1 << 20);
}

// MurmurHash3 fmix64 finaliser.
__host__ __device__ inline uint32_t hash_key(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return (uint32_t)k;
}

// Working buffers of the voxel filter, sized for `capacity` input points: a hash table of
// end-point voxels (at least 2 * capacity slots, kept empty between frames), the list of
// slots a frame used, and the filtered points: compact in first-use order (for export), at
// the input index of each voxel's first point, and packed densely in input order (for the
// traversal: full tiles of neighbouring rays).
struct FilterBuffers {
  unsigned long long* table_keys;  // voxel key per slot, ~0 = empty
  unsigned long long* table_sums;  // 3 fixed-point fraction sums per slot
  uint32_t* table_counts;          // points per slot
  uint32_t* table_first;           // lowest input index per slot, ~0 = none
  uint32_t* used;                  // slots used by the current frame, in first-use order
  uint32_t* n_used;                // device count of used slots = filtered points
  float* out_pts;                  // compact: 3 floats per filtered point, world offset (m)
  unsigned long long* out_keys;    // compact: voxel key per filtered point
  uint32_t* out_counts;            // compact: input points per filtered point
  float* idx_pts;                  // by input index: 3 floats at the voxel's first point
  uint32_t* idx_tags;              // by input index: tag of the frame that wrote idx_pts
  float* dense_pts;                // tagged idx_pts packed in input order
  uint32_t* block_counts;          // compaction: tagged indices per block, then their prefix
  uint32_t* n_dense;               // device count of dense points
  int64_t capacity;
  uint32_t table_mask;
  uint32_t tag;                    // tag of the current frame (never 0)
};

// Constants of one expected-depth launch (double ray geometry, FP32 accumulation).
struct DepthParams {
  int32_t type, width, height, pad;
  float hw, hh, c0, c1, su, sv;  // frustum pixel model
  const float* sinu;             // laser tables (device)
  const float* cosu;
  const float* sinv;
  const float* cosv;
  double R[9];    // world-from-sensor, row-major
  double eye[3];  // position / res
  double t_max;   // max_range / res
  double res;
  float scale, bias;  // occupancy = sigmoid(scale * log-odds + bias)
};

// ---- kernel launchers (defined in the .cu files) -----------------------------------------
// `dependent`: launched as a programmatic dependent of the preceding kernel on the stream (its
// CTAs start while that kernel finishes and wait for it before reading anything); not for
// stream capture.
template <int MaxF>
cudaError_t launch_traverse_labels(const TickWork<MaxF>& w, const MapView& m, int rounding,
                                   cudaStream_t s, bool dependent = false);
// Claim order of a traversal's tiles, longest walks first: kOrderBuckets buckets of the tiles'
// longest-ray walk estimates (bucket 0 = longest), each with its list of tiles.
constexpr int kOrderBuckets = 64;
struct TileOrderBuffers {
  uint32_t* counts;  // kOrderBuckets words, zero between passes (the traversal clears them)
  uint32_t* lists;   // kOrderBuckets * capacity words
  uint32_t capacity; // tiles per list
  bool pending;      // host side: a pass was launched and its traversal not (yet)
};
// Sizes (or grows) the buffers for `tiles` tiles.
cudaError_t tile_order_reserve(TileOrderBuffers* b, uint32_t tiles, cudaStream_t s);
void tile_order_release(TileOrderBuffers* b);
// kOrderBuckets / the longest walk any ray of these frames can take (steps + set-up).
template <int MaxF>
float tile_order_scale(const TickWork<MaxF>& w);
// Files every tile under the bucket of its longest ray's walk (|R p|_1 / res, the DDA's step
// count up to rounding, plus a set-up allowance).  The counts are zero on entry: the traversal
// that reads a pass's lists clears them; `b.pending` (a pass whose traversal was never launched)
// clears them first.
template <int MaxF>
cudaError_t launch_tile_order(const TickWork<MaxF>& w, TileOrderBuffers* b, cudaStream_t s);
cudaError_t launch_tile_order_dev(const TickWork<kMaxTickFrames>* d_work, uint32_t total_tiles,
                                  TileOrderBuffers* b, cudaStream_t s);

// Dynamic shared memory of one traversal CTA (leaf table, ray order, rendered ranges).
size_t traverse_smem_bytes(int tile_w, int tile_h, uint32_t smask, bool render);
// Whether a frame fits the fused render + traversal (reach within the leaf code's range).
bool traverse_render_fits(const FrameParams& f);
cudaError_t prepare_traverse_dev(int tile_w, int tile_h, uint32_t smask, int rounding, bool wide);
cudaError_t launch_traverse_labels_dev(const TickWork<kMaxTickFrames>* d_work, uint32_t total_tiles,
                                       int tile_w, int tile_h, uint32_t smask, const MapView& m,
                                       int rounding, bool wide, cudaStream_t s);
cudaError_t launch_traverse_counts(const FrameParams& f, const MapView& m, int rounding,
                                   cudaStream_t s);
cudaError_t launch_integrate(const MapView& m, const IntegrateParams& p, int update_mode,
                             int rounding, int sm_count, cudaStream_t s, bool dependent = false);
// Queries the integration kernels' resident blocks per SM ahead of any stream capture.
void prepare_integrate();
cudaError_t launch_rehash(const MapView& from, const MapView& to, uint32_t cur_epoch,
                          int update_mode, cudaStream_t s);
cudaError_t launch_export(const MapView& m, int32_t* origins, float* values, uint32_t* active,
                          uint32_t* n_out, uint32_t max_out, cudaStream_t s);
cudaError_t launch_export_labels(const MapView& m, int plane, int32_t* origins,
                                 uint32_t* words, uint32_t* n_out, uint32_t max_out,
                                 cudaStream_t s);
cudaError_t launch_fill_keys(unsigned long long* keys, uint32_t n, cudaStream_t s);
int depth_partial_blocks(const DepthParams& p);
cudaError_t launch_depth_forward(const DepthParams& p, const MapView& m, const float* vals,
                                 float* depth, cudaStream_t s);
cudaError_t launch_depth_backward(const DepthParams& p, const MapView& m, const float* vals,
                                  const float* grad_depth, const float* depth, float* grad_vals,
                                  double* partials, double* out6, cudaStream_t s);
// A refinement's pose and Adam state, kept on the device so that its steps queue without a
// host round trip: each step's kernel reads the pose from it and the update kernel writes it.
struct RefineState {
  double position[3];  // metres
  double R[9];         // world-from-sensor, row-major
  double mom[6], var[6];
  double res, t_max;   // to recompute the eye (index units) and check the addressable range
  float lr_position, lr_rotation;
  int32_t steps;
  uint32_t error;  // kRefineNoPixels / kRefineOutOfRange; once set, the pose stays
};
constexpr uint32_t kRefineNoPixels = 1u, kRefineOutOfRange = 2u;
// Step `it` of a refinement: the loss and pose gradient at st's pose (partials, then a fixed-
// order sum), losses[it] = mean loss, and for it < steps the Adam update of st.
cudaError_t launch_depth_refine(const DepthParams& p, const MapView& m, const float* vals,
                                const float* target, float max_residual, float surface_offset,
                                float edge, double* partials, RefineState* st, float* losses,
                                int it, cudaStream_t s);
cudaError_t filter_reserve(FilterBuffers* b, int64_t n, cudaStream_t s);
void filter_release(FilterBuffers* b);
int filter_key_bits(float max_time);  // bits per axis of a filter key; 0 if out of range
cudaError_t run_voxel_filter(const FrameParams& f, int rounding, int centre, int key_bits,
                             const FilterBuffers& b, cudaStream_t s);

}  // namespace nm
