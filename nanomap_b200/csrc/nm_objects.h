// nm_objects.h -- definitions of the opaque C ABI objects and the error helpers shared by the
// host translation units.
#pragma once

#include <atomic>
#include <cfenv>
#include <cstdarg>
#include <cstdio>
#include <string>

#include "nm_internal.h"
#include "nm_sim.h"

namespace nm {

// Record a failure message for nm_last_error() and return `code`.
int fail(int code, const char* fmt, ...);
const char* last_error();

struct RoundScope {
  int saved;
  explicit RoundScope(int rounding) : saved(std::fegetround()) {
    std::fesetround(rounding == NM_ROUND_DOWN ? FE_DOWNWARD : FE_TONEAREST);
  }
  ~RoundScope() { std::fesetround(saved); }
};

}  // namespace nm

#define NM_CUDA(call)                                                                    \
  do {                                                                                   \
    const cudaError_t e_ = (call);                                                       \
    if (e_ != cudaSuccess)                                                               \
      return nm::fail(NM_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                      __FILE__, __LINE__);                                               \
  } while (0)

// ---- object definitions ---------------------------------------------------------------------
//
// Objects are reference counted: a handle holds one reference, and every object that uses
// another holds one on it (sensors, maps and sim maps on their context; tick plans on their
// map, sim map and slot sensors).  nm_*_destroy drops the handle's reference, so handles may be
// destroyed in any order; the memory goes when the last user does.

struct nm_context_s {
  std::atomic<int> refs{1};
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  float* render_staging = nullptr;
  size_t render_staging_bytes = 0;
};

struct nm_sensor_s {
  std::atomic<int> refs{1};
  nm_context ctx = nullptr;
  nm_sensor_desc desc{};
  float fp[6] = {0, 0, 0, 0, 0, 0};
  float lh = 0.f, lm = 0.f;
  float* d_tables = nullptr;  // laser: sinu[W], cosu[W], sinv[H], cosv[H]
};

struct nm_map_s {
  std::atomic<int> refs{1};
  nm_context ctx = nullptr;
  nm_map_desc desc{};
  nm::MapView view{};
  nm::MapCounters* d_ctr = nullptr;
  uint32_t epoch = 1;
  uint64_t known_leaves = 0;
  uint64_t pending_bound = 0;
  uint32_t grow_count = 0;
  bool pending_labels = false;
  float pending_lh[nm::kMaxPlanes];
  float pending_lm[nm::kMaxPlanes];
  uint32_t pending_planes = 0;
  // host input staging: two device buffers used in turn, filled on the map's copy stream, so a
  // frame's copy runs while the frame before it is walked (created on first host input)
  unsigned char* staging[2] = {nullptr, nullptr};
  size_t staging_bytes[2] = {0, 0};
  int staging_next = 0;                            // buffer of the next host input
  int staging_held = -1;                           // buffer the current call filled
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_staged[2] = {nullptr, nullptr};   // buffer filled (copy stream)
  cudaEvent_t ev_free[2] = {nullptr, nullptr};     // work reading the buffer enqueued before it
  uint32_t* d_scratch_u32 = nullptr;  // export counters
  unsigned int* h_status = nullptr;   // page-locked copy of the map's status words
  // 16x16 tiles, 256-entry leaf table: fastest or within a few percent on every frame kind
  // measured (one ray per thread; tiles of two or more rays per thread lose SIMT sharing)
  int tile_w = 16, tile_h = 16, smem_entries = 256;
  nm::FilterBuffers filter{};  // voxel-filter buffers, grown on first filtered insert
  nm::TileOrderBuffers tile_order{};  // claim order of traversal tiles, grown on demand
  double* depth_scratch = nullptr;  // expected-depth partial sums (grown on demand)
  size_t depth_scratch_n = 0;
};

struct nm_simmap_s {
  std::atomic<int> refs{1};
  nm_context ctx = nullptr;
  nm::SimMapView view{};
  int32_t bbox[6] = {0, 0, 0, -1, -1, -1};
  uint64_t active_voxels = 0;
  uint64_t leaves = 0;
  uint64_t bricks = 0;  // non-empty 64^3-voxel bricks (blocks of 512 leaf entries)
  float* cast_staging = nullptr;  // host-side ray casts: origins, directions, distances
  size_t cast_staging_bytes = 0;
};


// Host helpers shared by the C ABI translation units (defined in nm_abi.cpp / nm_abi_sim.cpp).
namespace nm {
template <class T>
T retain(T obj) {
  if (obj) obj->refs.fetch_add(1, std::memory_order_relaxed);
  return obj;
}
// Drop one reference; the last one frees the object (and drops the references it holds).
void release(nm_context c);
void release(nm_sensor s);
void release(nm_map m);
void release(nm_simmap sm);
void release(nm_cave c);

// Sim map construction: begin_build allocates (or, given `buffer` of at least 64 bytes per
// leaf, borrows) the zeroed dense leaf buffer of the voxel region [vmin, vmax); finish_build
// compacts it into `sm` and frees it unless borrowed.
int begin_build(float res, const int32_t vmin[3], const int32_t vmax[3], SimBuild* b,
                cudaStream_t s, uint32_t* buffer = nullptr);
int finish_build(nm_context ctx, SimBuild& b, nm_simmap sm, cudaStream_t s);

cudaStream_t pick(nm_context ctx, void* stream);
int make_frame(nm_map m, nm_sensor s, const nm_pose* pose, FrameParams* f);
uint64_t frame_leaf_bound(nm_map m, nm_sensor s, const nm_pose& pose, const float R[9],
                          bool range_input, uint64_t n_rays);
void frame_box(nm_map m, nm_sensor s, const nm_pose& pose, const float R[9], bool range_input,
               double lo[3], double hi[3]);
double box_leaves(const double lo[3], const double hi[3]);
double ray_leaf_cap(nm_map m, nm_sensor s, uint64_t n_rays);
int ensure_capacity(nm_map m, uint64_t bound, cudaStream_t s);
int set_plane_constants(nm_map m, int plane, nm_sensor s);
IntegrateParams integrate_params(nm_map m);
// `dependent`: the last operation on `s` is a traversal kernel, so the integration may be
// launched as its programmatic dependent.
int do_integrate(nm_map m, cudaStream_t s, bool dependent = false);
int check_device_errors(nm_map m, cudaStream_t s);
int validate_pose(const nm_pose* pose);
// Ray parameters of a sensor at a pose over a sim map of voxel size `res`.
void make_ray_params(nm_sensor s, const nm_pose& pose, float res, SimRayParams* rp);
int check_launch_shape(int tile_w, int tile_h, int entries);
}  // namespace nm
