// nm_abi.cpp -- host implementation of the C ABI declared in include/nanomap_b200.h.
//
// Owns device memory, derives the per-frame constants on the host (as Handler.cpp:32-41 and
// SensorAllocator.h:110-148 do), keeps the leaf table large enough, and launches the sm_100a
// kernels.  There is no CPU fallback: every compute entry point fails with NM_ERR_CUDA when no
// CUDA device is usable.  Built with -frounding-math so the rounding-mode sections below are
// evaluated at run time under the mode they select.
#include <algorithm>
#include <cstddef>
#include <cfenv>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "nm_internal.h"
#include "nm_sim.h"
#include "nm_host.h"
#include "nm_objects.h"

namespace nm {

namespace {
thread_local std::string g_error;
}  // namespace

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_error = buf;
  return code;
}

const char* last_error() { return g_error.c_str(); }

}  // namespace nm

using nm::fail;
using nm::RoundScope;

namespace {

uint32_t next_pow2(uint64_t v) {
  uint64_t p = 1;
  while (p < v) p <<= 1;
  return (uint32_t)std::min<uint64_t>(p, 1ull << 31);
}

}  // namespace

// ---- shared host math (declared in nm_host.h) ---------------------------------------------
namespace nm {

void pose_rotation(const nm_pose& pose, const float F[9], float R[9]) {
  RoundScope rs(NM_ROUND_NEAREST);
  double w = pose.orientation[0], x = pose.orientation[1], y = pose.orientation[2],
         z = pose.orientation[3];
  const double n = std::sqrt(w * w + x * x + y * y + z * z);
  w /= n;
  x /= n;
  y /= n;
  z /= n;
  const double M[9] = {1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y - w * z), 2.0 * (x * z + w * y),
                       2.0 * (x * y + w * z), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z - w * x),
                       2.0 * (x * z - w * y), 2.0 * (y * z + w * x), 1.0 - 2.0 * (x * x + y * y)};
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) {
      const double s = M[r * 3 + 0] * (double)F[c * 3 + 0] + M[r * 3 + 1] * (double)F[c * 3 + 1] +
                       M[r * 3 + 2] * (double)F[c * 3 + 2];
      R[r * 3 + c] = (float)s;
    }
}

void frame_constants(const nm_pose& pose, float res, float max_range, int rounding, double eye[3],
                     float* max_time) {
  double inv_res;
  {
    RoundScope rs(NM_ROUND_NEAREST);
    volatile double r = (double)res;
    inv_res = 1.0 / r;
  }
  RoundScope rs(rounding);
  for (int a = 0; a < 3; ++a) {
    volatile double p = (double)pose.position[a];
    eye[a] = p * inv_res;
  }
  volatile float mr = max_range, rf = res;
  *max_time = mr / rf;
}

void frustum_params(int W, int H, float hfov_deg, float vfov_deg, float out[6]) {
  RoundScope rs(NM_ROUND_NEAREST);
  const double kPi = 3.14159265358979323846;
  const float hh = (float)std::tan((double)vfov_deg * kPi / 360.0);
  float hw;
  if (hfov_deg > 0.0f) {
    hw = (float)std::tan((double)hfov_deg * kPi / 360.0);
  } else {
    volatile float fw = (float)W, fh = (float)H;
    const float aspect = fw / fh;
    hw = aspect * hh;
  }
  out[0] = hw;
  out[1] = hh;
  out[2] = 2.0f * hw;
  out[3] = 2.0f * hh;
  out[4] = (float)(1.0 / (double)W);
  out[5] = (float)(1.0 / (double)H);
}

void laser_tables(int W, int H, float hfov_deg, float vfov_deg, float* sinu, float* cosu,
                  float* sinv, float* cosv) {
  RoundScope rs(NM_ROUND_NEAREST);
  const double kPi = 3.14159265358979323846;
  volatile float fw = (float)W, fh = (float)H;
  const float su = hfov_deg / fw, sv = vfov_deg / fh;
  for (int w = 0; w < W; ++w) {
    const float u = -hfov_deg / 2.0f + (float)w * su;
    const double ur = (double)u * kPi / 180.0;
    sinu[w] = (float)std::sin(ur);
    cosu[w] = (float)std::cos(ur);
  }
  for (int h = 0; h < H; ++h) {
    const float v = -vfov_deg / 2.0f + (float)h * sv;
    const double vr = (double)v * kPi / 180.0;
    sinv[h] = (float)std::sin(vr);
    cosv[h] = (float)std::cos(vr);
  }
}

float logit(float p) {
  RoundScope rs(NM_ROUND_NEAREST);
  return (float)(std::log((double)p) - std::log(1.0 - (double)p));
}

}  // namespace nm

namespace nm {

int check_launch_shape(int tile_w, int tile_h, int entries) {
  const int64_t n = (int64_t)tile_w * tile_h;
  if (tile_w <= 0 || tile_h <= 0 || n % 64 != 0 || n > 4096 || (n < 256 && (n & (n - 1)) != 0))
    return fail(NM_ERR_ARG, "tile %dx%d: area must be 64, 128, or a multiple of 256 up to 4096",
                tile_w, tile_h);
  if (entries < 16 || entries > 512 || (entries & (entries - 1)) != 0)
    return fail(NM_ERR_ARG, "leaf table entries must be a power of two in 16..512");
  return NM_OK;
}

cudaStream_t pick(nm_context ctx, void* stream) {
  return stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
}

void free_view(nm::MapView& v) {
  cudaFree(v.keys);
  cudaFree(v.values);
  cudaFree(v.active);
  cudaFree(v.labels);
  cudaFree(v.counts);
  cudaFree(v.epoch);
  cudaFree(v.plane_mask);
  cudaFree(v.touched);
  v = nm::MapView{};
}

int alloc_view(nm_map m, uint32_t capacity, nm::MapView* out, cudaStream_t s) {
  nm::MapView v{};
  v.capacity = capacity;
  v.mask = capacity - 1;
  v.planes = m->desc.max_agents;
  v.ctr = m->d_ctr;
  const size_t C = capacity;
  cudaError_t e = cudaSuccess;
  auto A = [&](void** p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(p, bytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(*p, 0, bytes, s);
  };
  A((void**)&v.keys, C * 8);
  A((void**)&v.values, C * nm::kLeafVoxels * 4);
  A((void**)&v.active, C * nm::kActiveWords * 4);
  A((void**)&v.labels, (size_t)v.planes * C * nm::kLabelWords * 4);
  if (m->desc.update_mode == NM_UPDATE_ACCUMULATE) A((void**)&v.counts, C * 1024 * 4);
  A((void**)&v.epoch, C * 4);
  if (v.planes > 1) A((void**)&v.plane_mask, C * 4);
  A((void**)&v.touched, C * 4);
  if (e == cudaSuccess) e = nm::launch_fill_keys(v.keys, capacity, s);
  if (e != cudaSuccess) {
    free_view(v);
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? NM_ERR_CAPACITY : NM_ERR_CUDA,
                "leaf table of %u slots: %s", capacity, cudaGetErrorString(e));
  }
  *out = v;
  return NM_OK;
}

int grow_map(nm_map m, uint32_t new_capacity, cudaStream_t s) {
  nm::MapView nv{};
  int rc = alloc_view(m, new_capacity, &nv, s);
  if (rc != NM_OK) return rc;
  NM_CUDA(cudaMemsetAsync(&m->d_ctr->leaf_count, 0, 4, s));
  NM_CUDA(cudaMemsetAsync(&m->d_ctr->touched_count, 0, 4, s));
  NM_CUDA(nm::launch_rehash(m->view, nv, m->epoch, m->desc.update_mode, s));
  NM_CUDA(cudaStreamSynchronize(s));
  free_view(m->view);
  m->view = nv;
  m->grow_count += 1;
  unsigned int lc = 0;
  NM_CUDA(cudaMemcpy(&lc, &m->d_ctr->leaf_count, 4, cudaMemcpyDeviceToHost));
  m->known_leaves = lc;
  return NM_OK;
}

// Box (index-space voxels) holding every voxel one frame can touch: the eye and the far ends
// of the sensor's pixel directions at max range -- the frustum pyramid for frustum range
// images, a sampled azimuth/elevation band (padded) for laser range images, the range ball
// for xyz records (whose points may lie anywhere within range).
void frame_box(nm_map m, nm_sensor s, const nm_pose& pose, const float R[9], bool range_input,
               double lo[3], double hi[3]) {
  const double res = m->desc.res;
  const double rv = s->desc.max_range / res + 2.0;
  double e[3];
  for (int a = 0; a < 3; ++a) {
    e[a] = pose.position[a] / res;
    lo[a] = e[a] - rv;
    hi[a] = e[a] + rv;
  }
  if (!range_input) return;
  double flo[3] = {e[0], e[1], e[2]}, fhi[3] = {e[0], e[1], e[2]};
  auto add = [&](double dx, double dy, double dz, double len) {
    for (int a = 0; a < 3; ++a) {
      const double c = e[a] + (R[a * 3] * dx + R[a * 3 + 1] * dy + R[a * 3 + 2] * dz) * len;
      flo[a] = std::min(flo[a], c);
      fhi[a] = std::max(fhi[a], c);
    }
  };
  double pad = 2.0;
  if (s->desc.type == NM_SENSOR_FRUSTUM) {
    const double sx[2] = {-s->fp[0], s->fp[0]}, sy[2] = {-s->fp[1], s->fp[1]};
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) add(sx[i], sy[j], 1.0, rv + 1.0);
  } else {
    const double kPi = 3.14159265358979323846;
    const double hf = s->desc.hfov_deg * kPi / 180.0, vf = s->desc.vfov_deg * kPi / 180.0;
    const int nu = 96, nv = 9;
    for (int i = 0; i <= nu; ++i) {
      const double u = -hf / 2 + hf * i / nu;
      for (int j = 0; j <= nv; ++j) {
        const double v = -vf / 2 + vf * j / nv;
        add(std::sin(u) * std::cos(v), std::sin(v), std::cos(u) * std::cos(v), rv);
      }
    }
    pad = 2.0 + 0.01 * rv;  // sampling step (< 2 degrees) under-reaches by less than 1 %
  }
  for (int a = 0; a < 3; ++a) {
    lo[a] = std::max(lo[a], flo[a] - pad);
    hi[a] = std::min(hi[a], fhi[a] + pad);
  }
}

double box_leaves(const double lo[3], const double hi[3]) {
  double vol = 1.0;
  for (int a = 0; a < 3; ++a) vol *= std::floor(hi[a] / 8.0) - std::floor(lo[a] / 8.0) + 1.0;
  return vol;
}

double ray_leaf_cap(nm_map m, nm_sensor s, uint64_t n_rays) {
  const double rv = s->desc.max_range / m->desc.res + 2.0;
  return (double)n_rays * (3.0 * std::ceil(rv / 8.0) + 3.0);
}

// Upper bound on the leaves one frame can touch: the leaf count of frame_box, capped by
// rays x leaves-per-ray.
uint64_t frame_leaf_bound(nm_map m, nm_sensor s, const nm_pose& pose, const float R[9],
                          bool range_input, uint64_t n_rays) {
  double lo[3], hi[3];
  frame_box(m, s, pose, R, range_input, lo, hi);
  return (uint64_t)std::min(box_leaves(lo, hi), ray_leaf_cap(m, s, n_rays));
}

int ensure_capacity(nm_map m, uint64_t bound, cudaStream_t s) {
  const uint64_t limit = m->view.capacity / 2;
  if (m->known_leaves + m->pending_bound + bound <= limit) {
    m->pending_bound += bound;
    return NM_OK;
  }
  NM_CUDA(cudaStreamSynchronize(s));
  unsigned int lc = 0;
  NM_CUDA(cudaMemcpy(&lc, &m->d_ctr->leaf_count, 4, cudaMemcpyDeviceToHost));
  m->known_leaves = lc;
  m->pending_bound = 0;
  uint64_t cap = m->view.capacity;
  while (m->known_leaves + bound > cap / 2 && cap < nm::kMaxLeafCapacity) cap <<= 1;
  if (m->known_leaves + bound > cap / 2 && m->known_leaves >= cap / 2)
    return fail(NM_ERR_CAPACITY, "map holds %llu leaves; the leaf table stops at %llu slots",
                (unsigned long long)m->known_leaves, (unsigned long long)nm::kMaxLeafCapacity);
  if (cap != m->view.capacity) {
    const int rc = grow_map(m, (uint32_t)cap, s);
    if (rc != NM_OK) return rc;
  }
  m->pending_bound = bound;
  return NM_OK;
}

int validate_pose(const nm_pose* pose) {
  if (!pose) return fail(NM_ERR_ARG, "pose is null");
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(pose->position[a])) return fail(NM_ERR_ARG, "pose position is not finite");
  double n = 0;
  for (int a = 0; a < 4; ++a) {
    if (!std::isfinite(pose->orientation[a])) return fail(NM_ERR_ARG, "orientation is not finite");
    n += (double)pose->orientation[a] * pose->orientation[a];
  }
  if (!(n > 1e-20)) return fail(NM_ERR_ARG, "orientation quaternion is zero");
  return NM_OK;
}

int make_frame(nm_map m, nm_sensor s, const nm_pose* pose, nm::FrameParams* f) {
  int rc = validate_pose(pose);
  if (rc != NM_OK) return rc;
  if (!s) return fail(NM_ERR_ARG, "sensor is null");
  if (s->ctx != m->ctx) return fail(NM_ERR_ARG, "sensor and map belong to different contexts");
  std::memset(f, 0, sizeof(*f));
  f->type = s->desc.type;
  f->width = s->desc.hres;
  f->height = s->desc.vres;
  f->hw = s->fp[0];
  f->hh = s->fp[1];
  f->c0 = s->fp[2];
  f->c1 = s->fp[3];
  f->su = s->fp[4];
  f->sv = s->fp[5];
  if (s->desc.type == NM_SENSOR_LASER) {
    f->sinu = s->d_tables;
    f->cosu = s->d_tables + s->desc.hres;
    f->sinv = s->d_tables + 2 * s->desc.hres;
    f->cosv = s->d_tables + 2 * s->desc.hres + s->desc.vres;
  }
  nm::pose_rotation(*pose, s->desc.frame_transform, f->R);
  nm::frame_constants(*pose, m->desc.res, s->desc.max_range, m->desc.rounding, f->eye, &f->max_time);
  f->res_d = (double)m->desc.res;
  // keys hold 21-bit leaf coordinates: keep every voxel the frame can reach inside them
  const double reach = (double)f->max_time + 2.0;
  for (int a = 0; a < 3; ++a)
    if (std::fabs(f->eye[a]) + reach > (double)(1 << 23) - 16.0)
      return fail(NM_ERR_ARG, "pose is outside the map's addressable range (+-%d voxels)", 1 << 23);
  return NM_OK;
}

nm::IntegrateParams integrate_params(nm_map m) {
  nm::IntegrateParams p{};
  p.thres_hit = m->desc.thres_hit;
  p.thres_miss = m->desc.thres_miss;
  p.clamp_min = m->desc.clamp_min;
  p.clamp_max = m->desc.clamp_max;
  p.clamp_mode = m->desc.clamp_mode;
  p.use_planes = m->view.planes > 1 ? 1 : 0;
  for (int i = 0; i < nm::kMaxPlanes; ++i) {
    p.lh[i] = m->pending_lh[i];
    p.lm[i] = m->pending_lm[i];
  }
  return p;
}

int do_integrate(nm_map m, cudaStream_t s, bool dependent) {
  if (!m->pending_labels) return NM_OK;
  const nm::IntegrateParams p = integrate_params(m);
  NM_CUDA(nm::launch_integrate(m->view, p, m->desc.update_mode, m->desc.rounding,
                               m->ctx->sm_count, s, dependent));
  m->pending_labels = false;
  m->pending_planes = 0;
  m->epoch += 1;
  if (m->epoch == 0) m->epoch = 1;
  return NM_OK;
}

int check_device_errors(nm_map m, cudaStream_t s) {
  // leaf_count and error_flags are adjacent: one read
  static_assert(offsetof(nm::MapCounters, error_flags) ==
                    offsetof(nm::MapCounters, leaf_count) + 4, "counter layout");
  // one round trip: the status words are copied into page-locked memory on the map's
  // stream, then the stream is waited for
  unsigned int* w = m->h_status;
  NM_CUDA(cudaMemcpyAsync(w, &m->d_ctr->leaf_count, 2 * sizeof(unsigned int),
                          cudaMemcpyDeviceToHost, s));
  NM_CUDA(cudaStreamSynchronize(s));
  const unsigned int lc = w[0], flags = w[1];
  m->known_leaves = lc;
  m->pending_bound = 0;
  if (flags & nm::kErrProbe)
    return fail(NM_ERR_CAPACITY, "leaf table probe limit reached (%u leaves in %u slots)", lc,
                m->view.capacity);
  if (flags & nm::kErrTimeout) return fail(NM_ERR_TIMEOUT, "a device-side wait gave up");
  if (flags & nm::kErrPlane) return fail(NM_ERR_ARG, "label plane out of range");
  return NM_OK;
}

// Host input goes to the device through two staging buffers used in turn.  Buffer b is filled
// on the map's copy stream once the work that read it last has run (ev_free[b], recorded on
// that work's stream when the call that staged it had enqueued everything), and the call's
// stream waits for the copy (ev_staged[b]).  So with asynchronous calls frame k's copy runs
// while frame k - 1 is walked; a synchronous call (NM_SYNC) is copy then work, as before.
int stage_input(nm_map m, const void* src, size_t bytes, cudaStream_t s, const void** dev) {
  if (!m->copy_stream) {
    NM_CUDA(cudaStreamCreateWithFlags(&m->copy_stream, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i) {
      NM_CUDA(cudaEventCreateWithFlags(&m->ev_staged[i], cudaEventDisableTiming));
      NM_CUDA(cudaEventCreateWithFlags(&m->ev_free[i], cudaEventDisableTiming));
    }
  }
  const int b = m->staging_next;
  if (bytes > m->staging_bytes[b]) {
    // the old buffer may still be read by queued work: let that finish first
    NM_CUDA(cudaEventSynchronize(m->ev_free[b]));
    cudaFree(m->staging[b]);
    m->staging[b] = nullptr;
    m->staging_bytes[b] = 0;
    NM_CUDA(cudaMalloc((void**)&m->staging[b], bytes));
    m->staging_bytes[b] = bytes;
  }
  NM_CUDA(cudaStreamWaitEvent(m->copy_stream, m->ev_free[b], 0));
  NM_CUDA(cudaMemcpyAsync(m->staging[b], src, bytes, cudaMemcpyHostToDevice, m->copy_stream));
  NM_CUDA(cudaEventRecord(m->ev_staged[b], m->copy_stream));
  NM_CUDA(cudaStreamWaitEvent(s, m->ev_staged[b], 0));
  m->staging_next = b ^ 1;
  m->staging_held = b;
  *dev = m->staging[b];
  return NM_OK;
}

// Marks the end of the current call's use of its staging buffer: every kernel reading it is
// on `s` by now (on every return path of a call that staged input).
struct StagingRelease {
  nm_map m;
  cudaStream_t s;
  ~StagingRelease() {
    if (m && m->staging_held >= 0) {
      cudaEventRecord(m->ev_free[m->staging_held], s);
      m->staging_held = -1;
    }
  }
};

int set_plane_constants(nm_map m, int plane, nm_sensor s) {
  const uint32_t bit = 1u << plane;
  if (m->pending_planes & bit) {
    if (m->pending_lh[plane] != s->lh || m->pending_lm[plane] != s->lm)
      return fail(NM_ERR_ARG, "frames sharing label plane %d use different log-odds constants", plane);
  } else {
    m->pending_lh[plane] = s->lh;
    m->pending_lm[plane] = s->lm;
    m->pending_planes |= bit;
  }
  return NM_OK;
}

constexpr int kFilteredTile = 16;        // traversal tile edge of filtered frames
constexpr uint32_t kFilteredEntries = 512;  // leaf-table entries per tile of filtered frames

// Voxel filter of one frame: runs the filter on `f`'s input and rewrites `f` into the frame
// of the filtered points (input kind 2: one record per occupied voxel, already rotated into
// the world frame, packed in the input order of the voxels' first points, counted on the
// device).  A traversal tile covers consecutive records: neighbouring rays.
int apply_filter(nm_map m, nm::FrameParams& f, uint32_t flags, cudaStream_t s0) {
  const int64_t n = (int64_t)f.width * f.height;
  const int kb = nm::filter_key_bits(f.max_time);
  if (kb == 0) return fail(NM_ERR_UNSUPPORTED, "voxel filter: range of %g voxels is too long", (double)f.max_time);
  NM_CUDA(nm::filter_reserve(&m->filter, n, s0));
  m->filter.tag += 1u;
  if (m->filter.tag == 0u) {  // wrapped: no stale record may carry the new tag
    m->filter.tag = 1u;
    NM_CUDA(cudaMemsetAsync(m->filter.idx_tags, 0, (size_t)m->filter.capacity * 4, s0));
  }
  NM_CUDA(nm::run_voxel_filter(f, m->desc.rounding, (flags & NM_FILTER_CENTRE) ? 1 : 0, kb,
                               m->filter, s0));
  f.input_kind = 2;
  f.xyz = reinterpret_cast<const unsigned char*>(m->filter.dense_pts);
  f.step = 12;
  f.ranges = nullptr;
  f.n_valid = m->filter.n_dense;
  f.width = kFilteredTile;
  f.height = (int32_t)((n + f.width - 1) / f.width);
  for (int i = 0; i < 9; ++i) f.R[i] = (i % 4 == 0) ? 1.0f : 0.0f;
  return NM_OK;
}

int run_frame(nm_map m, nm_sensor s, nm::FrameParams& f, uint32_t flags, cudaStream_t s0,
              uint64_t bound, const nm::SimRender* sim) {
  int rc = ensure_capacity(m, bound, s0);
  if (rc != NM_OK) return rc;
  rc = set_plane_constants(m, 0, s);
  if (rc != NM_OK) return rc;
  f.epoch = m->epoch;
  f.plane = 0;
  bool dependent_integrate = false;  // the integration directly follows a traversal kernel
  if (m->desc.update_mode == NM_UPDATE_LABEL) {
    nm::TickWork<1> w;
    std::memset(&w, 0, sizeof(w));
    w.n_frames = 1;
    w.tile_w = m->tile_w;
    w.tile_h = m->tile_h;
    w.smask = (uint32_t)m->smem_entries - 1u;
    if (f.input_kind == 2) {
      // filtered rays: one per voxel, packed by image patch, so a tile's rays fan out over
      // more leaves than a tile of neighbouring pixels does: a larger leaf table
      w.tile_w = w.tile_h = kFilteredTile;
      w.smask = kFilteredEntries - 1u;
    }
    w.tiles_x[0] = (f.width + w.tile_w - 1) / w.tile_w;
    const int tiles_y = (f.height + w.tile_h - 1) / w.tile_h;
    w.tile_start[0] = 0;
    w.tile_start[1] = (uint32_t)(w.tiles_x[0] * tiles_y);
    w.total_tiles = w.tile_start[1];
    w.fr[0] = f;
    if (w.total_tiles > 0) {
      if (sim) {
        NM_CUDA(nm::launch_traverse_render(w, m->view, *sim, m->desc.rounding, s0));
        dependent_integrate = true;
      } else {
        // longest walks first (frames within the leaf code's reach; the others take the
        // table-free traversal, which claims no tiles)
        const bool ordered = f.max_time < nm::kNarrowMaxTime;
        if (ordered) {
          NM_CUDA(nm::tile_order_reserve(&m->tile_order, w.total_tiles, s0));
          w.order_scale = nm::tile_order_scale<1>(w);
          NM_CUDA(nm::launch_tile_order<1>(w, &m->tile_order, s0));
          w.order_counts = m->tile_order.counts;
          w.order_lists = m->tile_order.lists;
          w.order_cap = m->tile_order.capacity;
        }
        // the walk's CTAs start while the order pass finishes
        NM_CUDA(nm::launch_traverse_labels<1>(w, m->view, m->desc.rounding, s0, ordered));
        if (ordered) m->tile_order.pending = false;
        dependent_integrate = true;
      }
    }
  } else {
    NM_CUDA(nm::launch_traverse_counts(f, m->view, m->desc.rounding, s0));
    dependent_integrate = true;
  }
  m->pending_labels = true;
  if (!(flags & NM_DEFER_INTEGRATE)) {
    rc = do_integrate(m, s0, dependent_integrate);
    if (rc != NM_OK) return rc;
  }
  if (flags & NM_SYNC) return check_device_errors(m, s0);
  return NM_OK;
}

void release(nm_context c) {
  if (!c || c->refs.fetch_sub(1, std::memory_order_acq_rel) != 1) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  cudaFree(c->render_staging);
  delete c;
}

void release(nm_sensor s) {
  if (!s || s->refs.fetch_sub(1, std::memory_order_acq_rel) != 1) return;
  nm_context c = s->ctx;
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  cudaFree(s->d_tables);
  delete s;
  release(c);
}

void release(nm_map m) {
  if (!m || m->refs.fetch_sub(1, std::memory_order_acq_rel) != 1) return;
  nm_context c = m->ctx;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  cudaDeviceSynchronize();
  free_view(m->view);
  cudaFree(m->d_ctr);
  cudaFree(m->d_scratch_u32);
  cudaFreeHost(m->h_status);
  for (int i = 0; i < 2; ++i) {
    cudaFree(m->staging[i]);
    if (m->ev_staged[i]) cudaEventDestroy(m->ev_staged[i]);
    if (m->ev_free[i]) cudaEventDestroy(m->ev_free[i]);
  }
  if (m->copy_stream) cudaStreamDestroy(m->copy_stream);
  filter_release(&m->filter);
  nm::tile_order_release(&m->tile_order);
  cudaFree(m->depth_scratch);
  delete m;
  release(c);
}

}  // namespace nm

using namespace nm;

// ---- C ABI ----------------------------------------------------------------------------------
extern "C" {

int nm_abi_version(void) { return NM_ABI_VERSION; }

const char* nm_last_error(void) { return nm::last_error(); }

int nm_context_create(int32_t device, nm_context* out) {
  if (!out) return fail(NM_ERR_ARG, "out is null");
  *out = nullptr;
  int n = 0;
  NM_CUDA(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return fail(NM_ERR_ARG, "device %d not present (%d devices)", device, n);
  NM_CUDA(cudaSetDevice(device));
  cudaDeviceProp prop;
  NM_CUDA(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10)
    return fail(NM_ERR_UNSUPPORTED, "device %d is sm_%d%d; this library is built for sm_100a",
                device, prop.major, prop.minor);
  std::unique_ptr<nm_context_s> c(new nm_context_s());
  c->device = device;
  c->sm_count = prop.multiProcessorCount;
  c->stream = nullptr;  // the CUDA default stream, so NULL streams order with other libraries
  *out = c.release();
  return NM_OK;
}

int nm_context_destroy(nm_context ctx) {
  nm::release(ctx);
  return NM_OK;
}

int nm_context_sync(nm_context ctx) {
  if (!ctx) return fail(NM_ERR_ARG, "context is null");
  NM_CUDA(cudaStreamSynchronize(ctx->stream));
  return NM_OK;
}

int nm_alloc_device(nm_context ctx, size_t bytes, void** out) {
  if (!ctx || !out) return fail(NM_ERR_ARG, "null argument");
  *out = nullptr;
  NM_CUDA(cudaSetDevice(ctx->device));
  NM_CUDA(cudaMalloc(out, bytes ? bytes : 1));
  return NM_OK;
}

int nm_free_device(void* p) {
  NM_CUDA(cudaFree(p));
  return NM_OK;
}

int nm_sensor_create(nm_context ctx, const nm_sensor_desc* d, nm_sensor* out) {
  if (!ctx || !d || !out) return fail(NM_ERR_ARG, "null argument");
  *out = nullptr;
  if (d->type != NM_SENSOR_FRUSTUM && d->type != NM_SENSOR_LASER)
    return fail(NM_ERR_ARG, "unknown sensor type %d", d->type);
  if (d->hres <= 0 || d->vres <= 0 || d->hres > 65536 || d->vres > 65536)
    return fail(NM_ERR_ARG, "sensor resolution %dx%d out of range", d->hres, d->vres);
  if (!(d->max_range > 0.0f) || !(d->min_range >= 0.0f) || !(d->vfov_deg > 0.0f))
    return fail(NM_ERR_ARG, "sensor ranges / field of view invalid");
  if (d->type == NM_SENSOR_FRUSTUM && !(d->vfov_deg < 180.0f && d->hfov_deg < 180.0f))
    return fail(NM_ERR_ARG, "frustum field of view must be below 180 degrees");
  if (!d->explicit_log_odds && !(d->prob_hit > 0.f && d->prob_hit < 1.f && d->prob_miss > 0.f &&
                                 d->prob_miss < 1.f))
    return fail(NM_ERR_ARG, "ProbHit / ProbMiss must lie in (0, 1)");
  std::unique_ptr<nm_sensor_s> s(new nm_sensor_s());
  s->ctx = ctx;
  s->desc = *d;
  if (d->type == NM_SENSOR_FRUSTUM) {
    nm::frustum_params(d->hres, d->vres, d->hfov_deg, d->vfov_deg, s->fp);
  } else {
    std::vector<float> t(2 * (size_t)d->hres + 2 * (size_t)d->vres);
    nm::laser_tables(d->hres, d->vres, d->hfov_deg, d->vfov_deg, t.data(), t.data() + d->hres,
                     t.data() + 2 * d->hres, t.data() + 2 * d->hres + d->vres);
    NM_CUDA(cudaSetDevice(ctx->device));
    NM_CUDA(cudaMalloc((void**)&s->d_tables, t.size() * 4));
    NM_CUDA(cudaMemcpy(s->d_tables, t.data(), t.size() * 4, cudaMemcpyHostToDevice));
  }
  if (d->explicit_log_odds) {
    s->lh = d->log_odds_hit;
    s->lm = d->log_odds_miss;
  } else {
    s->lh = nm::logit(d->prob_hit);
    s->lm = nm::logit(d->prob_miss);
  }
  nm::retain(ctx);
  *out = s.release();
  return NM_OK;
}

int nm_sensor_destroy(nm_sensor s) {
  nm::release(s);
  return NM_OK;
}

int nm_sensor_params(nm_sensor s, float out[6]) {
  if (!s || !out) return fail(NM_ERR_ARG, "null argument");
  std::memcpy(out, s->fp, sizeof(s->fp));
  return NM_OK;
}

int nm_map_create(nm_context ctx, const nm_map_desc* d, nm_map* out) {
  if (!ctx || !d || !out) return fail(NM_ERR_ARG, "null argument");
  *out = nullptr;
  if (!(d->res > 0.0f)) return fail(NM_ERR_ARG, "map resolution must be positive");
  if (d->leaf_edge != 8) return fail(NM_ERR_UNSUPPORTED, "leaf edge %d (only 8 is supported)", d->leaf_edge);
  if (d->update_mode != NM_UPDATE_LABEL && d->update_mode != NM_UPDATE_ACCUMULATE)
    return fail(NM_ERR_ARG, "unknown update mode %d", d->update_mode);
  if (d->clamp_mode != NM_CLAMP_ALWAYS && d->clamp_mode != NM_CLAMP_ON_CROSSING)
    return fail(NM_ERR_ARG, "unknown clamp mode %d", d->clamp_mode);
  if (d->rounding != NM_ROUND_NEAREST && d->rounding != NM_ROUND_DOWN)
    return fail(NM_ERR_ARG, "unknown rounding %d", d->rounding);
  if (d->max_agents < 1 || d->max_agents > nm::kMaxPlanes)
    return fail(NM_ERR_ARG, "max_agents must be 1..%d", nm::kMaxPlanes);
  if (d->update_mode == NM_UPDATE_ACCUMULATE && d->max_agents != 1)
    return fail(NM_ERR_UNSUPPORTED, "accumulate mode keeps one label plane");
  if (d->initial_leaf_capacity > nm::kMaxLeafCapacity)
    return fail(NM_ERR_CAPACITY, "initial leaf capacity %u above %llu slots", d->initial_leaf_capacity,
                (unsigned long long)nm::kMaxLeafCapacity);
  NM_CUDA(cudaSetDevice(ctx->device));
  std::unique_ptr<nm_map_s> m(new nm_map_s());
  m->ctx = ctx;
  m->desc = *d;
  auto free_small = [&]() {
    cudaFree(m->d_ctr);
    cudaFree(m->d_scratch_u32);
    cudaFreeHost(m->h_status);
  };
  cudaError_t e = cudaMalloc((void**)&m->d_ctr, sizeof(nm::MapCounters));
  if (e == cudaSuccess) e = cudaMemsetAsync(m->d_ctr, 0, sizeof(nm::MapCounters), ctx->stream);
  if (e == cudaSuccess) e = cudaMalloc((void**)&m->d_scratch_u32, 64);
  if (e == cudaSuccess) e = cudaHostAlloc((void**)&m->h_status, 16, cudaHostAllocDefault);
  if (e != cudaSuccess) {
    free_small();
    cudaGetLastError();
    return fail(NM_ERR_CUDA, "map counters: %s", cudaGetErrorString(e));
  }
  const uint32_t cap = next_pow2(std::max<uint64_t>(d->initial_leaf_capacity ? d->initial_leaf_capacity : (1u << 18), 1024));
  const int rc = alloc_view(m.get(), cap, &m->view, ctx->stream);
  if (rc != NM_OK) {
    free_small();
    return rc;
  }
  e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    free_view(m->view);
    free_small();
    return fail(NM_ERR_CUDA, "map set-up: %s", cudaGetErrorString(e));
  }
  nm::prepare_integrate();
  for (int i = 0; i < nm::kMaxPlanes; ++i) m->pending_lh[i] = m->pending_lm[i] = 0.f;
  nm::retain(ctx);
  *out = m.release();
  return NM_OK;
}

int nm_map_destroy(nm_map m) {
  nm::release(m);
  return NM_OK;
}

int nm_map_reset(nm_map m) {
  if (!m) return fail(NM_ERR_ARG, "map is null");
  cudaStream_t s = m->ctx->stream;
  NM_CUDA(cudaDeviceSynchronize());
  const size_t C = m->view.capacity;
  NM_CUDA(nm::launch_fill_keys(m->view.keys, m->view.capacity, s));
  NM_CUDA(cudaMemsetAsync(m->view.values, 0, C * nm::kLeafVoxels * 4, s));
  NM_CUDA(cudaMemsetAsync(m->view.active, 0, C * nm::kActiveWords * 4, s));
  NM_CUDA(cudaMemsetAsync(m->view.labels, 0, (size_t)m->view.planes * C * nm::kLabelWords * 4, s));
  if (m->view.counts) NM_CUDA(cudaMemsetAsync(m->view.counts, 0, C * 1024 * 4, s));
  NM_CUDA(cudaMemsetAsync(m->view.epoch, 0, C * 4, s));
  if (m->view.plane_mask) NM_CUDA(cudaMemsetAsync(m->view.plane_mask, 0, C * 4, s));
  NM_CUDA(cudaMemsetAsync(m->d_ctr, 0, sizeof(nm::MapCounters), s));
  NM_CUDA(cudaStreamSynchronize(s));
  m->epoch = 1;
  m->known_leaves = 0;
  m->pending_bound = 0;
  m->pending_labels = false;
  m->pending_planes = 0;
  return NM_OK;
}

int nm_map_status_async(nm_map m, uint32_t* host_status, void* stream) {
  if (!m || !host_status) return fail(NM_ERR_ARG, "null argument");
  static_assert(offsetof(nm::MapCounters, error_flags) ==
                    offsetof(nm::MapCounters, leaf_count) + 4, "counter layout");
  NM_CUDA(cudaSetDevice(m->ctx->device));
  NM_CUDA(cudaMemcpyAsync(host_status, &m->d_ctr->leaf_count, 2 * sizeof(unsigned int),
                          cudaMemcpyDeviceToHost, pick(m->ctx, stream)));
  return NM_OK;
}

int nm_map_stats(nm_map m, nm_stats* out) {
  if (!m || !out) return fail(NM_ERR_ARG, "null argument");
  NM_CUDA(cudaDeviceSynchronize());
  nm::MapCounters c;
  NM_CUDA(cudaMemcpy(&c, m->d_ctr, sizeof(c), cudaMemcpyDeviceToHost));
  out->frames = c.frames;
  out->rays = c.rays;
  out->visits = c.visits;
  out->unique_voxels = c.unique_voxels;
  out->touched_leaves = c.touched_total;
  out->leaf_count = c.leaf_count;
  out->leaf_capacity = m->view.capacity;
  out->error_flags = c.error_flags;
  out->grow_count = m->grow_count;
  out->depth_visits = c.depth_visits;
  m->known_leaves = c.leaf_count;
  m->pending_bound = 0;
  if (c.error_flags) NM_CUDA(cudaMemset(&m->d_ctr->error_flags, 0, 4));
  return NM_OK;
}

int nm_map_insert_points(nm_map m, nm_sensor s, const nm_pose* pose, const void* cloud,
                         int32_t width, int32_t height, int32_t step, uint32_t flags,
                         void* stream) {
  if (!m || !s) return fail(NM_ERR_ARG, "null map or sensor");
  if (width < 0 || height < 0 || (int64_t)width * height > (1ll << 30))
    return fail(NM_ERR_ARG, "cloud size %dx%d out of range", width, height);
  if (step < 12) return fail(NM_ERR_ARG, "point step %d below 12 bytes", step);
  const int64_t n = (int64_t)width * height;
  if (n > 0 && !cloud) return fail(NM_ERR_ARG, "cloud is null");
  NM_CUDA(cudaSetDevice(m->ctx->device));
  cudaStream_t s0 = pick(m->ctx, stream);
  nm::FrameParams f;
  int rc = make_frame(m, s, pose, &f);
  if (rc != NM_OK) return rc;
  if (n == 0) return NM_OK;
  f.width = width;
  f.height = height;
  f.input_kind = 0;
  f.step = step;
  const uint64_t bound = frame_leaf_bound(m, s, *pose, f.R, false, (uint64_t)n);
  const void* dev = cloud;
  StagingRelease staged{m, s0};
  if (flags & NM_INPUT_HOST) {
    rc = stage_input(m, cloud, (size_t)n * step, s0, &dev);
    if (rc != NM_OK) return rc;
  }
  f.xyz = static_cast<const unsigned char*>(dev);
  if (flags & (NM_FILTER_MEAN | NM_FILTER_CENTRE)) {
    rc = apply_filter(m, f, flags, s0);
    if (rc != NM_OK) return rc;
  }
  return run_frame(m, s, f, flags, s0, bound, nullptr);
}

int nm_map_insert_ranges(nm_map m, nm_sensor s, const nm_pose* pose, const float* ranges,
                         uint32_t flags, void* stream) {
  if (!m || !s || !ranges) return fail(NM_ERR_ARG, "null argument");
  NM_CUDA(cudaSetDevice(m->ctx->device));
  cudaStream_t s0 = pick(m->ctx, stream);
  nm::FrameParams f;
  int rc = make_frame(m, s, pose, &f);
  if (rc != NM_OK) return rc;
  const int64_t n = (int64_t)s->desc.hres * s->desc.vres;
  f.input_kind = 1;
  const void* dev = ranges;
  StagingRelease staged{m, s0};
  if (flags & NM_INPUT_HOST) {
    rc = stage_input(m, ranges, (size_t)n * 4, s0, &dev);
    if (rc != NM_OK) return rc;
  }
  f.ranges = static_cast<const float*>(dev);
  const uint64_t bound = frame_leaf_bound(m, s, *pose, f.R, true, (uint64_t)n);
  if (flags & (NM_FILTER_MEAN | NM_FILTER_CENTRE)) {
    rc = apply_filter(m, f, flags, s0);
    if (rc != NM_OK) return rc;
  }
  return run_frame(m, s, f, flags, s0, bound, nullptr);
}

int nm_sim_insert(nm_simmap sm, nm_map m, nm_sensor s, const nm_pose* pose, float sigma_coef,
                  float drop_prob, uint64_t seed, float* ranges, uint32_t flags, void* stream) {
  if (!sm || !m || !s || !pose) return fail(NM_ERR_ARG, "null argument");
  if (sm->ctx != m->ctx || s->ctx != m->ctx)
    return fail(NM_ERR_ARG, "sim map, map and sensor belong to different contexts");
  if (!(std::isfinite(sigma_coef) && drop_prob >= 0.0f && drop_prob <= 1.0f))
    return fail(NM_ERR_ARG, "noise parameters invalid");
  if (flags & NM_INPUT_HOST) return fail(NM_ERR_ARG, "NM_INPUT_HOST does not apply (no input)");
  int rc = validate_pose(pose);
  if (rc != NM_OK) return rc;
  NM_CUDA(cudaSetDevice(m->ctx->device));
  cudaStream_t s0 = pick(m->ctx, stream);
  const int64_t n = (int64_t)s->desc.hres * s->desc.vres;
  const bool host_out = (flags & NM_OUTPUT_HOST) && ranges;
  float* out = host_out ? nullptr : ranges;
  nm::FrameParams f;
  rc = make_frame(m, s, pose, &f);
  if (rc != NM_OK) return rc;
  // the voxel filter and per-ray sums need the whole image first, and so do frames that reach
  // beyond the fused kernel's leaf code: render, then insert
  const bool two_pass = (flags & (NM_FILTER_MEAN | NM_FILTER_CENTRE)) ||
                        m->desc.update_mode != NM_UPDATE_LABEL || !nm::traverse_render_fits(f);
  if (host_out || (two_pass && !out)) {
    nm_context c = m->ctx;
    if ((size_t)n * 4 > c->render_staging_bytes) {
      cudaFree(c->render_staging);
      c->render_staging = nullptr;
      c->render_staging_bytes = 0;
      NM_CUDA(cudaMalloc((void**)&c->render_staging, (size_t)n * 4));
      c->render_staging_bytes = (size_t)n * 4;
    }
    out = c->render_staging;
  }
  const uint32_t pass = flags & ~(NM_OUTPUT_HOST | NM_SYNC);
  if (two_pass) {
    rc = nm_sim_render_noisy(sm, s, pose, out, sigma_coef, drop_prob, seed, 0, s0);
    if (rc == NM_OK) rc = nm_map_insert_ranges(m, s, pose, out, pass | (flags & NM_SYNC), s0);
  } else {
    f.input_kind = 1;
    f.ranges = nullptr;
    nm::SimRender sr;
    std::memset(&sr, 0, sizeof(sr));
    sr.v = sm->view;
    nm::make_ray_params(s, *pose, sm->view.res, &sr.rp);
    sr.sigma_coef = sigma_coef;
    sr.drop = drop_prob;
    sr.seed = seed;
    sr.noise = (sigma_coef != 0.0f || drop_prob != 0.0f) ? 1 : 0;
    sr.out = out;
    const uint64_t bound = frame_leaf_bound(m, s, *pose, f.R, true, (uint64_t)n);
    rc = run_frame(m, s, f, pass | (flags & NM_SYNC), s0, bound, &sr);
  }
  if (rc != NM_OK) return rc;
  if (host_out) {
    NM_CUDA(cudaMemcpyAsync(ranges, out, (size_t)n * 4, cudaMemcpyDeviceToHost, s0));
    NM_CUDA(cudaStreamSynchronize(s0));
  }
  return NM_OK;
}

int nm_map_filter_points(nm_map m, nm_sensor s, const nm_pose* pose, const void* input,
                         int32_t width, int32_t height, int32_t step, uint32_t flags,
                         float* points, uint32_t* counts, uint64_t max_points, uint64_t* n) {
  if (!m || !s || !n) return fail(NM_ERR_ARG, "null argument");
  *n = 0;
  if (step < 0 || (step > 0 && step < 12)) return fail(NM_ERR_ARG, "point step %d (0 = range image, else >= 12)", step);
  if (step > 0 && (width < 0 || height < 0 || (int64_t)width * height > (1ll << 30)))
    return fail(NM_ERR_ARG, "cloud size %dx%d out of range", width, height);
  NM_CUDA(cudaSetDevice(m->ctx->device));
  cudaStream_t s0 = m->ctx->stream;
  nm::FrameParams f;
  int rc = make_frame(m, s, pose, &f);
  if (rc != NM_OK) return rc;
  if (step > 0) {
    f.width = width;
    f.height = height;
    f.input_kind = 0;
    f.step = step;
  } else {
    f.input_kind = 1;
  }
  const int64_t np = (int64_t)f.width * f.height;
  if (np > 0 && !input) return fail(NM_ERR_ARG, "input is null");
  if (np == 0) return NM_OK;
  const void* dev = input;
  StagingRelease staged{m, s0};
  if (flags & NM_INPUT_HOST) {
    rc = stage_input(m, input, (size_t)np * (step > 0 ? (size_t)step : 4u), s0, &dev);
    if (rc != NM_OK) return rc;
  }
  if (step > 0)
    f.xyz = static_cast<const unsigned char*>(dev);
  else
    f.ranges = static_cast<const float*>(dev);
  rc = apply_filter(m, f, flags | NM_FILTER_MEAN, s0);
  if (rc != NM_OK) return rc;
  NM_CUDA(cudaStreamSynchronize(s0));
  uint32_t cnt = 0;
  NM_CUDA(cudaMemcpy(&cnt, m->filter.n_used, 4, cudaMemcpyDeviceToHost));
  *n = cnt;
  if (!cnt || (!points && !counts) || !max_points) return NM_OK;
  // the device emits voxels in first-use order; the caller gets them in voxel order
  std::vector<unsigned long long> keys(cnt);
  std::vector<float> pts(3 * (size_t)cnt);
  std::vector<uint32_t> cn(cnt);
  NM_CUDA(cudaMemcpy(keys.data(), m->filter.out_keys, (size_t)cnt * 8, cudaMemcpyDeviceToHost));
  NM_CUDA(cudaMemcpy(pts.data(), m->filter.out_pts, (size_t)cnt * 12, cudaMemcpyDeviceToHost));
  NM_CUDA(cudaMemcpy(cn.data(), m->filter.out_counts, (size_t)cnt * 4, cudaMemcpyDeviceToHost));
  std::vector<uint32_t> order(cnt);
  for (uint32_t i = 0; i < cnt; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return keys[a] < keys[b]; });
  const uint64_t k = std::min<uint64_t>(cnt, max_points);
  for (uint64_t i = 0; i < k; ++i) {
    if (points) std::memcpy(points + 3 * i, &pts[3 * (size_t)order[i]], 12);
    if (counts) counts[i] = cn[order[i]];
  }
  return NM_OK;
}

int nm_map_set_launch(nm_map m, int32_t tile_w, int32_t tile_h, int32_t leaf_table_entries) {
  if (!m) return fail(NM_ERR_ARG, "map is null");
  const int rc = nm::check_launch_shape(tile_w, tile_h, leaf_table_entries);
  if (rc != NM_OK) return rc;
  m->tile_w = tile_w;
  m->tile_h = tile_h;
  m->smem_entries = leaf_table_entries;
  return NM_OK;
}

int nm_map_integrate(nm_map m, void* stream) {
  if (!m) return fail(NM_ERR_ARG, "map is null");
  NM_CUDA(cudaSetDevice(m->ctx->device));
  return do_integrate(m, pick(m->ctx, stream));
}

int nm_map_export(nm_map m, int32_t* origins, float* values, uint32_t* active,
                  uint64_t max_leaves, uint64_t* n) {
  if (!m || !n) return fail(NM_ERR_ARG, "null argument");
  NM_CUDA(cudaSetDevice(m->ctx->device));
  cudaStream_t s = m->ctx->stream;
  NM_CUDA(cudaDeviceSynchronize());
  unsigned int lc = 0;
  NM_CUDA(cudaMemcpy(&lc, &m->d_ctr->leaf_count, 4, cudaMemcpyDeviceToHost));
  *n = lc;
  const uint64_t k = std::min<uint64_t>(lc, max_leaves);
  if (k == 0) return NM_OK;
  int32_t* d_o = nullptr;
  float* d_v = nullptr;
  uint32_t* d_a = nullptr;
  cudaError_t e = cudaSuccess;
  if (origins) e = cudaMalloc((void**)&d_o, k * 12);
  if (e == cudaSuccess && values) e = cudaMalloc((void**)&d_v, k * 2048);
  if (e == cudaSuccess && active) e = cudaMalloc((void**)&d_a, k * 64);
  if (e == cudaSuccess) e = cudaMemsetAsync(m->d_scratch_u32, 0, 4, s);
  if (e == cudaSuccess) e = nm::launch_export(m->view, d_o, d_v, d_a, m->d_scratch_u32, (uint32_t)k, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && origins) e = cudaMemcpy(origins, d_o, k * 12, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && values) e = cudaMemcpy(values, d_v, k * 2048, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && active) e = cudaMemcpy(active, d_a, k * 64, cudaMemcpyDeviceToHost);
  cudaFree(d_o);
  cudaFree(d_v);
  cudaFree(d_a);
  if (e != cudaSuccess) return fail(NM_ERR_CUDA, "export: %s", cudaGetErrorString(e));
  return NM_OK;
}

int nm_map_export_labels(nm_map m, int32_t agent, int32_t* origins, uint32_t* words,
                         uint64_t max_leaves, uint64_t* n) {
  if (!m || !n || !origins || !words) return fail(NM_ERR_ARG, "null argument");
  if (agent < 0 || agent >= m->view.planes) return fail(NM_ERR_ARG, "agent plane %d out of range", agent);
  if (m->desc.update_mode != NM_UPDATE_LABEL) return fail(NM_ERR_STATE, "map is not in label mode");
  NM_CUDA(cudaSetDevice(m->ctx->device));
  cudaStream_t s = m->ctx->stream;
  NM_CUDA(cudaDeviceSynchronize());
  unsigned int lc = 0;
  NM_CUDA(cudaMemcpy(&lc, &m->d_ctr->leaf_count, 4, cudaMemcpyDeviceToHost));
  const uint64_t cap = std::min<uint64_t>(lc, max_leaves);
  *n = 0;
  if (cap == 0) return NM_OK;
  int32_t* d_o = nullptr;
  uint32_t* d_w = nullptr;
  cudaError_t e = cudaMalloc((void**)&d_o, cap * 12);
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_w, cap * 128);
  if (e == cudaSuccess) e = cudaMemsetAsync(m->d_scratch_u32, 0, 4, s);
  if (e == cudaSuccess) e = nm::launch_export_labels(m->view, agent, d_o, d_w, m->d_scratch_u32, (uint32_t)cap, s);
  unsigned int cnt = 0;
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaMemcpy(&cnt, m->d_scratch_u32, 4, cudaMemcpyDeviceToHost);
  const uint64_t k = std::min<uint64_t>(cnt, cap);
  if (e == cudaSuccess && k) e = cudaMemcpy(origins, d_o, k * 12, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && k) e = cudaMemcpy(words, d_w, k * 128, cudaMemcpyDeviceToHost);
  cudaFree(d_o);
  cudaFree(d_w);
  if (e != cudaSuccess) return fail(NM_ERR_CUDA, "export labels: %s", cudaGetErrorString(e));
  *n = cnt;
  return NM_OK;
}

int nm_map_frame_params(nm_map m, nm_sensor s, const nm_pose* pose, float rotation[9],
                        double eye[3], float* max_time) {
  if (!m || !s || !rotation || !eye || !max_time) return fail(NM_ERR_ARG, "null argument");
  nm::FrameParams f;
  const int rc = make_frame(m, s, pose, &f);
  if (rc != NM_OK) return rc;
  std::memcpy(rotation, f.R, sizeof(f.R));
  std::memcpy(eye, f.eye, sizeof(f.eye));
  *max_time = f.max_time;
  return NM_OK;
}

int nm_frame_params(const nm_sensor_desc* desc, const nm_pose* pose, float res, int32_t rounding,
                    float rotation[9], double eye[3], float* max_time, float pixel_model[6]) {
  if (!desc || !rotation || !eye || !max_time || !pixel_model) return fail(NM_ERR_ARG, "null argument");
  const int rc = validate_pose(pose);
  if (rc != NM_OK) return rc;
  if (!(res > 0.0f)) return fail(NM_ERR_ARG, "resolution must be positive");
  if (rounding != NM_ROUND_NEAREST && rounding != NM_ROUND_DOWN) return fail(NM_ERR_ARG, "unknown rounding");
  nm::pose_rotation(*pose, desc->frame_transform, rotation);
  nm::frame_constants(*pose, res, desc->max_range, rounding, eye, max_time);
  if (desc->type == NM_SENSOR_FRUSTUM)
    nm::frustum_params(desc->hres, desc->vres, desc->hfov_deg, desc->vfov_deg, pixel_model);
  else
    for (int i = 0; i < 6; ++i) pixel_model[i] = 0.0f;
  return NM_OK;
}

int nm_map_tick(nm_map m, const nm_frame* frames, int32_t n_frames, uint32_t flags, void* stream) {
  if (!m || !frames) return fail(NM_ERR_ARG, "null argument");
  if (n_frames < 1 || n_frames > nm::kMaxTickFrames)
    return fail(NM_ERR_ARG, "a tick takes 1..%d frames (got %d)", nm::kMaxTickFrames, n_frames);
  if (m->desc.update_mode != NM_UPDATE_LABEL)
    return fail(NM_ERR_UNSUPPORTED, "batched ticks run in label mode");
  NM_CUDA(cudaSetDevice(m->ctx->device));
  cudaStream_t s0 = pick(m->ctx, stream);
  std::unique_ptr<nm::TickWork<nm::kMaxTickFrames>> w(new nm::TickWork<nm::kMaxTickFrames>());
  std::memset(w.get(), 0, sizeof(*w));
  w->n_frames = n_frames;
  w->tile_w = m->tile_w;
  w->tile_h = m->tile_h;
  w->smask = (uint32_t)m->smem_entries - 1u;
  uint64_t bound = 0;
  double ulo[3] = {0, 0, 0}, uhi[3] = {0, 0, 0}, cap = 0.0;
  for (int i = 0; i < n_frames; ++i) {
    const nm_frame& fr = frames[i];
    if (!fr.sensor || !fr.ranges) return fail(NM_ERR_ARG, "frame %d: null sensor or ranges", i);
    if (fr.agent < 0 || fr.agent >= m->view.planes)
      return fail(NM_ERR_ARG, "frame %d: agent plane %d outside 0..%d", i, fr.agent, m->view.planes - 1);
    int rc = make_frame(m, fr.sensor, &fr.pose, &w->fr[i]);
    if (rc != NM_OK) return rc;
    rc = set_plane_constants(m, fr.agent, fr.sensor);
    if (rc != NM_OK) return rc;
    nm::FrameParams& f = w->fr[i];
    f.input_kind = 1;
    f.ranges = fr.ranges;
    f.plane = fr.agent;
    w->tiles_x[i] = (f.width + w->tile_w - 1) / w->tile_w;
    const int ty = (f.height + w->tile_h - 1) / w->tile_h;
    w->tile_start[i + 1] = w->tile_start[i] + (uint32_t)(w->tiles_x[i] * ty);
    double lo[3], hi[3];
    frame_box(m, fr.sensor, fr.pose, f.R, true, lo, hi);
    for (int a = 0; a < 3; ++a) {
      ulo[a] = i == 0 ? lo[a] : std::min(ulo[a], lo[a]);
      uhi[a] = i == 0 ? hi[a] : std::max(uhi[a], hi[a]);
    }
    cap += ray_leaf_cap(m, fr.sensor, (uint64_t)fr.sensor->desc.hres * fr.sensor->desc.vres);
  }
  bound = (uint64_t)std::min(box_leaves(ulo, uhi), cap);
  w->total_tiles = w->tile_start[n_frames];
  int rc = ensure_capacity(m, bound, s0);
  if (rc != NM_OK) return rc;
  for (int i = 0; i < n_frames; ++i) w->fr[i].epoch = m->epoch;
  if (w->total_tiles > 0) {
    bool wide = false;
    for (int i = 0; i < n_frames; ++i) wide |= !(w->fr[i].max_time < nm::kNarrowMaxTime);
    if (!wide) {  // longest walks first
      NM_CUDA(nm::tile_order_reserve(&m->tile_order, w->total_tiles, s0));
      w->order_scale = nm::tile_order_scale<nm::kMaxTickFrames>(*w);
      NM_CUDA(nm::launch_tile_order<nm::kMaxTickFrames>(*w, &m->tile_order, s0));
      w->order_counts = m->tile_order.counts;
      w->order_lists = m->tile_order.lists;
      w->order_cap = m->tile_order.capacity;
    }
    NM_CUDA(nm::launch_traverse_labels<nm::kMaxTickFrames>(*w, m->view, m->desc.rounding, s0, !wide));
    if (!wide) m->tile_order.pending = false;
  }
  m->pending_labels = true;
  if (!(flags & NM_DEFER_INTEGRATE)) {
    rc = do_integrate(m, s0, w->total_tiles > 0);
    if (rc != NM_OK) return rc;
  }
  if (flags & NM_SYNC) return check_device_errors(m, s0);
  return NM_OK;
}

}  // extern "C"
