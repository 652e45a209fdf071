// nm_noalloc.cu -- per-frame labelling that allocates no device memory.
//
// nm_label_frame_static runs the traversal + labelling kernel of nm_traverse.cu on one range
// image and writes the frame's labelled leaves to caller buffers.  Its working memory (leaf
// hash table, label words, touched list, counters) is one file-scope static __device__ array
// of fixed size, so the call never calls cudaMalloc / cudaFree or an allocating library
// routine.  It exists for callers that cannot allocate device memory at the point where they
// label frames: real-time control loops that forbid allocation after start-up (an allocation
// can block on the device and fragment memory mid-mission), and hosts where another
// framework's pool already owns the device memory the library would otherwise take.
//
// Limits: a frame of at most kStaticMaxPixels pixels, at most kStaticLeafSlots / 2 distinct
// leaves labelled per call (checked on the device after the walk; more is NM_ERR_CAPACITY).
// The array (about 9 MiB) belongs to this file's device module.  CUDA loads modules lazily by
// default, so the driver places the array in a GPU's memory when the module is first used on
// that GPU: the first call on each device (which also looks up the array's device address)
// is the start-up warm-up, and should come before the caller's no-allocation phase and before
// any stream capture.  From then on the array stays resident until the process exits.  Every
// call shares it and it keeps the last call's contents, so each call first clears what must
// start at zero; calls that overlap on the GPU (different streams, or different host threads)
// race on it and must be serialised by the caller.
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "nm_host.h"
#include "nm_internal.h"
#include "nm_objects.h"

namespace nm {

namespace {

constexpr uint32_t kStaticLeafSlots = 1u << 16;
constexpr int64_t kStaticMaxPixels = 1ll << 23;
constexpr uint32_t kErrOutputFull = 8u;  // more labelled leaves than the caller's max_leaves
constexpr uint32_t kErrLeafLimit = 16u;  // more labelled leaves than kStaticLeafSlots / 2

struct StaticScratch {
  MapCounters ctr;
  unsigned long long keys[kStaticLeafSlots];
  alignas(16) uint32_t labels[(size_t)kStaticLeafSlots * kLabelWords];  // cleared as uint4
  uint32_t epoch[kStaticLeafSlots];
  uint32_t touched[kStaticLeafSlots];
};
static_assert(offsetof(StaticScratch, labels) % 16 == 0, "labels are cleared with 16-byte stores");

static __device__ __align__(256) StaticScratch g_static_scratch;

constexpr int kMaxDevices = 64;
StaticScratch* g_scratch_addr[kMaxDevices] = {nullptr};
std::mutex g_scratch_mutex;

// Everything the traversal expects to start at zero (or empty), in one pass.
__global__ void k_static_clear(StaticScratch* s) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (size_t i = t; i < kStaticLeafSlots; i += stride) {
    s->keys[i] = kEmptyKey;
    s->epoch[i] = 0u;
  }
  uint4* l4 = reinterpret_cast<uint4*>(s->labels);
  const size_t n4 = (size_t)kStaticLeafSlots * kLabelWords / 4;
  for (size_t i = t; i < n4; i += stride) l4[i] = make_uint4(0u, 0u, 0u, 0u);
  if (t < sizeof(MapCounters) / 4) reinterpret_cast<uint32_t*>(&s->ctr)[t] = 0u;
}

// Copy the touched leaves (origin + 32 label words) to the caller's buffers.
__global__ void __launch_bounds__(256) k_static_export(const StaticScratch* s, int32_t* origins,
                                                       uint32_t* words, uint32_t max_leaves,
                                                       uint32_t* status) {
  const int lane = threadIdx.x & 31;
  const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  const uint32_t n = s->ctr.touched_count;
  for (uint32_t i = gw; i < n && i < max_leaves; i += nw) {
    const uint32_t slot = s->touched[i];
    if (lane == 0) {
      int lx, ly, lz;
      key_leaf(s->keys[slot], &lx, &ly, &lz);
      origins[3 * (size_t)i] = lx * 8;
      origins[3 * (size_t)i + 1] = ly * 8;
      origins[3 * (size_t)i + 2] = lz * 8;
    }
    words[(size_t)i * kLabelWords + lane] = s->labels[(size_t)slot * kLabelWords + lane];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    status[0] = n;
    status[1] = s->ctr.error_flags | (n > max_leaves ? kErrOutputFull : 0u) |
                (n > kStaticLeafSlots / 2 ? kErrLeafLimit : 0u);
  }
}

// Device address of the static array on the current device (looked up once per device).
cudaError_t scratch_on_current_device(StaticScratch** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[dev] = static_cast<StaticScratch*>(p);
  }
  *out = g_scratch_addr[dev];
  return cudaSuccess;
}

}  // namespace

}  // namespace nm

extern "C" int nm_label_frame_static(nm_sensor s, const nm_pose* pose, const float* ranges,
                                     float res, int32_t rounding, int32_t* origins,
                                     uint32_t* words, uint32_t max_leaves, uint32_t* status,
                                     uint32_t flags, void* stream) {
  using namespace nm;
  if (!s || !ranges || !origins || !words || !status)
    return fail(NM_ERR_ARG, "null argument");
  int rc = validate_pose(pose);
  if (rc != NM_OK) return rc;
  if (!(std::isfinite(res) && res > 0.0f))
    return fail(NM_ERR_ARG, "resolution must be positive and finite");
  if (rounding != NM_ROUND_NEAREST && rounding != NM_ROUND_DOWN)
    return fail(NM_ERR_ARG, "unknown rounding %d", rounding);
  const int64_t pixels = (int64_t)s->desc.hres * s->desc.vres;
  if (pixels > kStaticMaxPixels)
    return fail(NM_ERR_ARG, "frame of %lld pixels exceeds the static-scratch limit of %lld pixels",
                (long long)pixels, (long long)kStaticMaxPixels);
  if (max_leaves == 0) return fail(NM_ERR_ARG, "max_leaves must be positive");
  NM_CUDA(cudaSetDevice(s->ctx->device));
  StaticScratch* sc = nullptr;
  NM_CUDA(scratch_on_current_device(&sc));

  // Per-frame constants (the same host derivation as every other insert).
  TickWork<1> w;
  std::memset(&w, 0, sizeof(w));
  FrameParams& f = w.fr[0];
  f.type = s->desc.type;
  f.width = s->desc.hres;
  f.height = s->desc.vres;
  f.hw = s->fp[0];
  f.hh = s->fp[1];
  f.c0 = s->fp[2];
  f.c1 = s->fp[3];
  f.su = s->fp[4];
  f.sv = s->fp[5];
  if (s->desc.type == NM_SENSOR_LASER) {
    f.sinu = s->d_tables;
    f.cosu = s->d_tables + s->desc.hres;
    f.sinv = s->d_tables + 2 * s->desc.hres;
    f.cosv = s->d_tables + 2 * s->desc.hres + s->desc.vres;
  }
  pose_rotation(*pose, s->desc.frame_transform, f.R);
  frame_constants(*pose, res, s->desc.max_range, rounding, f.eye, &f.max_time);
  f.res_d = (double)res;
  const double reach = (double)f.max_time + 2.0;
  for (int a = 0; a < 3; ++a)
    if (std::fabs(f.eye[a]) + reach > (double)(1 << 23) - 16.0)
      return fail(NM_ERR_ARG, "pose is outside the addressable range (+-%d voxels)", 1 << 23);
  f.input_kind = 1;
  f.ranges = ranges;
  f.epoch = 1u;
  f.plane = 0;
  w.n_frames = 1;
  w.tile_w = 16;
  w.tile_h = 16;
  w.smask = 127u;
  w.tiles_x[0] = (f.width + 15) / 16;
  w.tile_start[1] = (uint32_t)(w.tiles_x[0] * ((f.height + 15) / 16));
  w.total_tiles = w.tile_start[1];

  MapView v{};
  v.keys = sc->keys;
  v.labels = sc->labels;
  v.epoch = sc->epoch;
  v.touched = sc->touched;
  v.ctr = &sc->ctr;
  v.capacity = kStaticLeafSlots;
  v.mask = kStaticLeafSlots - 1u;
  v.planes = 1;

  cudaStream_t st = pick(s->ctx, stream);
  k_static_clear<<<s->ctx->sm_count * 4, 256, 0, st>>>(sc);
  NM_CUDA(cudaGetLastError());
  if (w.total_tiles > 0) NM_CUDA(launch_traverse_labels<1>(w, v, rounding, st));
  k_static_export<<<s->ctx->sm_count * 2, 256, 0, st>>>(sc, origins, words, max_leaves, status);
  NM_CUDA(cudaGetLastError());
  if (flags & NM_SYNC) {
    NM_CUDA(cudaStreamSynchronize(st));
    uint32_t hs[2] = {0u, 0u};
    NM_CUDA(cudaMemcpy(hs, status, sizeof(hs), cudaMemcpyDeviceToHost));
    if (hs[1] & kErrLeafLimit)
      return fail(NM_ERR_CAPACITY, "frame labels %u leaves, more than the static-scratch limit of %u",
                  hs[0], kStaticLeafSlots / 2);
    if (hs[1] & kErrProbe)
      return fail(NM_ERR_CAPACITY, "static-scratch leaf table of %u slots: probe limit reached, "
                  "frame labels more than %u leaves", kStaticLeafSlots, kStaticLeafSlots / 2);
    if (hs[1] & kErrOutputFull)
      return fail(NM_ERR_CAPACITY, "%u labelled leaves exceed max_leaves = %u", hs[0], max_leaves);
  }
  return NM_OK;
}
