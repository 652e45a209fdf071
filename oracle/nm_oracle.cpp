/*
 * nm_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * A plain C++ CPU restatement of the NanoMap path the GPU library replaces.  Only
 * tests/, __graft_entry__.smoke() and bench.py (its cpu_baseline leg and its
 * `--impl reference` arm) load this library.  The product library never links it.
 *
 * What it restates (reference file:line):
 *   - pose -> rotation and index-space eye: Handler.cpp:32-41 (R = q.normalized() *
 *     FrameTransform, eye = worldToIndex(position), max_time = maxRange / res).
 *   - per-point insertion: Handler.cpp:58-85 / SimHandler.cpp:57-85 (rotate the point,
 *     ray_length = |R p| / res, skip when ray_length >= max_time, normalise, voxel DDA
 *     over [0, ray_length]: "miss" on every voxel left by a step, "hit" on the end voxel
 *     when the DDA time is below max_time).
 *   - integration: Handler.cpp:88-122 (clamp then threshold) and SimHandler.cpp:88-122
 *     (threshold then clamp), selected by clamp_mode.
 *   - simulated depth: generateCloud.cu:20-82 (first active voxel of the sim grid along
 *     the pixel ray, clipped to the grid's active bounding box; the voxel holding the ray
 *     start is not tested; range limits scale with the unnormalised pixel direction).
 *   - the pixel ray model: Sensor.h:213-250 (frustum pixel corners u = w/W, v = h/H;
 *     laser azimuth/elevation grid).
 *
 * Third-party arithmetic restated from published algorithms (none of it is vendored):
 *   - openvdb::math::DDA<Ray<double>,0> (OpenVDB, version unpinned by the reference):
 *     Amanatides & Woo, "A Fast Voxel Traversal Algorithm for Ray Tracing" (1987).  The
 *     step axis is the one with the smallest next crossing time; ties go to the higher
 *     axis index (z before y before x).  A zero direction component disables its axis.
 *   - Eigen 3.3.9 quaternion -> rotation matrix: the standard unit-quaternion formula,
 *     evaluated in double and rounded once to float.
 *
 * PARITY UNPINNED.  The reference ships no tests, fixtures or golden vectors, and it cannot
 * be built here (OpenVDB, NanoVDB, Eigen, TBB and Blosc are absent).  This oracle is pinned
 * only to hand-derived known-answer cases (tests/golden/dda_kat.json).
 *
 * Rounding policy.  The reference calls fesetround(FE_DOWNWARD) in SensorData::updatePose
 * (SensorData.h:42) and never restores it, so its CPU insertion runs rounded toward -inf.
 * Every entry point here takes `rounding` (0 = to nearest, 1 = toward -inf) and runs the
 * per-point arithmetic under that mode.  Build with -frounding-math -ffp-contract=off.
 */
#include <algorithm>
#include <array>
#include <cfenv>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "orc_types.h"

namespace {

constexpr int kHit = 1;
constexpr int kMiss = 0;
constexpr double kMinLen = 1.0e-7;  // directions this short are skipped (see trace_point)

struct RoundGuard {
  int saved;
  explicit RoundGuard(int rounding) : saved(std::fegetround()) {
    std::fesetround(rounding == 1 ? FE_DOWNWARD : FE_TONEAREST);
  }
  ~RoundGuard() { std::fesetround(saved); }
};

inline int argmin_hi(const double n[3]) {
  return (n[0] < n[1]) ? ((n[0] < n[2]) ? 0 : 2) : ((n[1] < n[2]) ? 1 : 2);
}
inline int argmin_hi_f(const float n[3]) {
  return (n[0] < n[1]) ? ((n[0] < n[2]) ? 0 : 2) : ((n[1] < n[2]) ? 1 : 2);
}

inline uint64_t leaf_key(int lx, int ly, int lz) {
  return ((uint64_t)(uint32_t)((lx + (1 << 20)) & 0x1FFFFF) << 42) |
         ((uint64_t)(uint32_t)((ly + (1 << 20)) & 0x1FFFFF) << 21) |
         (uint64_t)(uint32_t)((lz + (1 << 20)) & 0x1FFFFF);
}
inline void key_origin(uint64_t k, int32_t o[3]) {
  o[0] = ((int)((k >> 42) & 0x1FFFFF) - (1 << 20)) * 8;
  o[1] = ((int)((k >> 21) & 0x1FFFFF) - (1 << 20)) * 8;
  o[2] = ((int)(k & 0x1FFFFF) - (1 << 20)) * 8;
}
inline int local_index(int x, int y, int z) { return ((x & 7) << 6) | ((y & 7) << 3) | (z & 7); }

struct Frame {
  float R[9];  // row-major, world-from-sensor rotation
  double eye[3];
  double res_d;
  float max_time;
};

// Handler.cpp:58-85 restated.  Must run with the policy rounding mode active.
template <class Emit>
inline int64_t trace_point(const Frame& f, float px, float py, float pz, Emit&& emit) {
  const float* R = f.R;
  const float dxf = (R[0] * px + R[1] * py) + R[2] * pz;
  const float dyf = (R[3] * px + R[4] * py) + R[5] * pz;
  const float dzf = (R[6] * px + R[7] * py) + R[8] * pz;
  const double dx = dxf, dy = dyf, dz = dzf;
  const double len = std::sqrt((dx * dx + dy * dy) + dz * dz);
  const double ray_len = len / f.res_d;
  if (!(ray_len < (double)f.max_time)) return -1;  // beyond range, NaN or Inf
  // The reference's normalize() leaves a direction no longer than 1e-7 unnormalised;
  // its DDA then meets no voxel face before max range, so such points change nothing.
  if (!(len > kMinLen)) return -1;
  const double inv_len = 1.0 / len;
  const double nd[3] = {dx * inv_len, dy * inv_len, dz * inv_len};
  int vox[3];
  double next[3], delta[3];
  int step[3];
  for (int a = 0; a < 3; ++a) {
    vox[a] = (int)std::floor(f.eye[a]);
    if (nd[a] == 0.0) {
      step[a] = 0;
      next[a] = DBL_MAX;
      delta[a] = DBL_MAX;
    } else {
      const double inv = 1.0 / nd[a];
      if (inv > 0.0) {
        step[a] = 1;
        next[a] = ((double)(vox[a] + 1) - f.eye[a]) * inv;
        delta[a] = inv;
      } else {
        step[a] = -1;
        next[a] = ((double)vox[a] - f.eye[a]) * inv;
        delta[a] = -inv;
      }
    }
  }
  int cur[3] = {vox[0], vox[1], vox[2]};
  double t;
  int64_t n = 0;
  for (;;) {
    const int a = argmin_hi(next);
    t = next[a];
    next[a] += delta[a];
    vox[a] += step[a];
    if (!(t <= ray_len)) break;
    emit(cur, kMiss);
    ++n;
    cur[0] = vox[0];
    cur[1] = vox[1];
    cur[2] = vox[2];
  }
  if (t < (double)f.max_time) {
    emit(cur, kHit);
    ++n;
  }
  return n;
}

struct LeafLabels {
  uint32_t w[32];  // words 0..15 hit bits, 16..31 miss bits
};
struct LeafCounts {
  uint32_t hit[512];
  uint32_t miss[512];
};
struct LeafSeq {
  float v[512];
  uint8_t touched[512];
};
struct Leaf {
  float v[512];
  uint8_t a[512];
};

struct MapParams {
  float res;
  float thres_hit, thres_miss;
  float clamp_min, clamp_max;
  int32_t clamp_mode;   // 0: clamp then threshold (Handler.cpp:98-110); 1: SimHandler.cpp:98-110
  int32_t update_mode;  // 0 label, 1 accumulate from counts, 2 accumulate in ray order
  int32_t rounding;
};

struct OracleMap {
  MapParams p;
  std::unordered_map<uint64_t, Leaf> leaves;
  std::unordered_map<uint64_t, LeafLabels> last_labels;
  int64_t visits = 0, rays = 0, unique_voxels = 0;
};

inline void integrate_voxel(float& v, uint8_t& active, float temp, const MapParams& p) {
  if (temp != 0.0f) {
    v = v + temp;
    if (p.clamp_mode == 0) {
      if (v > p.clamp_max) {
        v = p.clamp_max;
      } else if (v < p.clamp_min) {
        v = p.clamp_min;
      }
      if (v > p.thres_hit) {
        active = 1;
      } else if (v < p.thres_miss) {
        active = 0;
      }
    } else {
      if (v > p.thres_hit) {
        active = 1;
        if (v > p.clamp_max) v = p.clamp_max;
      } else if (v < p.thres_miss) {
        active = 0;
        if (v < p.clamp_min) v = p.clamp_min;
      }
    }
  }
}

Leaf& get_leaf(OracleMap* m, uint64_t key) {
  auto it = m->leaves.find(key);
  if (it == m->leaves.end()) {
    Leaf L;
    std::memset(L.v, 0, sizeof(L.v));
    std::memset(L.a, 0, sizeof(L.a));
    it = m->leaves.emplace(key, L).first;
  }
  return it->second;
}

struct LabelSink {
  std::unordered_map<uint64_t, LeafLabels> map;
  uint64_t last_key = ~0ull;
  LeafLabels* last = nullptr;
  int64_t visits = 0, rays = 0;
  void operator()(const int v[3], int kind) {
    const uint64_t k = leaf_key(v[0] >> 3, v[1] >> 3, v[2] >> 3);
    if (k != last_key) {
      auto it = map.find(k);
      if (it == map.end()) {
        LeafLabels L;
        std::memset(&L, 0, sizeof(L));
        it = map.emplace(k, L).first;
      }
      last = &it->second;
      last_key = k;
    }
    const int l = local_index(v[0], v[1], v[2]);
    last->w[(kind == kHit ? 0 : 16) + (l >> 5)] |= 1u << (l & 31);
  }
};

struct CountSink {
  std::unordered_map<uint64_t, LeafCounts> map;
  uint64_t last_key = ~0ull;
  LeafCounts* last = nullptr;
  void operator()(const int v[3], int kind) {
    const uint64_t k = leaf_key(v[0] >> 3, v[1] >> 3, v[2] >> 3);
    if (k != last_key) {
      auto it = map.find(k);
      if (it == map.end()) {
        it = map.emplace(k, LeafCounts()).first;
        std::memset(&it->second, 0, sizeof(LeafCounts));
      }
      last = &it->second;
      last_key = k;
    }
    const int l = local_index(v[0], v[1], v[2]);
    if (kind == kHit)
      last->hit[l] += 1;
    else
      last->miss[l] += 1;
  }
};

struct SeqSink {
  std::unordered_map<uint64_t, LeafSeq> map;
  float lh, lm;
  void operator()(const int v[3], int kind) {
    const uint64_t k = leaf_key(v[0] >> 3, v[1] >> 3, v[2] >> 3);
    auto it = map.find(k);
    if (it == map.end()) {
      it = map.emplace(k, LeafSeq()).first;
      std::memset(&it->second, 0, sizeof(LeafSeq));
    }
    const int l = local_index(v[0], v[1], v[2]);
    it->second.v[l] += (kind == kHit) ? lh : lm;
    it->second.touched[l] = 1;
  }
};

// ---------------------------------------------------------------------------------------
// Sim map: sparse 8^3 bit leaves (restates the role of the NanoVDB sim grid).
struct SimMap {
  float res;
  bool any = false;
  int32_t amin[3] = {0, 0, 0}, amax[3] = {-1, -1, -1};
  std::unordered_map<uint64_t, std::array<uint32_t, 16>> leaves;
  void set(int i, int j, int k) {
    const uint64_t key = leaf_key(i >> 3, j >> 3, k >> 3);
    auto it = leaves.find(key);
    if (it == leaves.end()) {
      std::array<uint32_t, 16> z{};
      it = leaves.emplace(key, z).first;
    }
    const int l = local_index(i, j, k);
    it->second[l >> 5] |= 1u << (l & 31);
    const int c[3] = {i, j, k};
    for (int a = 0; a < 3; ++a) {
      if (!any || c[a] < amin[a]) amin[a] = c[a];
      if (!any || c[a] > amax[a]) amax[a] = c[a];
    }
    any = true;
  }
  bool active(const int v[3]) const {
    auto it = leaves.find(leaf_key(v[0] >> 3, v[1] >> 3, v[2] >> 3));
    if (it == leaves.end()) return false;
    const int l = local_index(v[0], v[1], v[2]);
    return (it->second[l >> 5] >> (l & 31)) & 1u;
  }
};

}  // namespace

extern "C" {

typedef struct {
  float res;
  float thres_hit, thres_miss;
  float clamp_min, clamp_max;
  int32_t clamp_mode, update_mode, rounding;
} orc_map_params;

int orc_version(void) { return 1; }

// Rotation (row-major, world-from-sensor) = rot(q / |q|) * F, with F given column-major
// (the FrameTransform order of the reference config files, Config.cpp:210-216).  The
// quaternion is (w, x, y, z).  Evaluated in double, rounded once to float, round-to-nearest.
void orc_rotation(const float q_in[4], const float F[9], float R[9]) {
  RoundGuard g(0);
  double w = q_in[0], x = q_in[1], y = q_in[2], z = q_in[3];
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

// Handler.cpp:33-39: eye = worldToIndex(position) (position times the map's inverse voxel
// size, the inverse taken once in round-to-nearest), max_time = maxRange / res in float.
void orc_frame_setup(const float pos[3], float res, float max_range, int rounding, double eye[3],
                     float* max_time) {
  double inv_res;
  {
    RoundGuard g(0);
    inv_res = 1.0 / (double)res;
  }
  RoundGuard g(rounding);
  for (int a = 0; a < 3; ++a) eye[a] = (double)pos[a] * inv_res;
  volatile float mr = max_range, rs = res;
  *max_time = mr / rs;
}

// Frustum pixel model (Sensor.h:156-171, 213-227).  halfHeight = tan(vfov/2); halfWidth =
// tan(hfov/2) when an explicit horizontal FOV is given, else aspect * halfHeight.
void orc_frustum_params(int W, int H, float hfov_deg, float vfov_deg, float out[6]) {
  RoundGuard g(0);
  const float hh = (float)std::tan((double)vfov_deg * 3.14159265358979323846 / 360.0);
  float hw;
  if (hfov_deg > 0.0f) {
    hw = (float)std::tan((double)hfov_deg * 3.14159265358979323846 / 360.0);
  } else {
    const float aspect = (float)W / (float)H;
    hw = aspect * hh;
  }
  out[0] = hw;
  out[1] = hh;
  out[2] = 2.0f * hw;
  out[3] = 2.0f * hh;
  out[4] = (float)(1.0 / (double)W);
  out[5] = (float)(1.0 / (double)H);
}

// Laser grid (Sensor.h:147-154, 228-249): u = -hfov/2 + w*hfov/W, v = -vfov/2 + h*vfov/H in
// degrees, direction (sin u cos v, sin v, cos u cos v).  Sines and cosines are taken in
// double and rounded to float once, so CPU and GPU share one table.
void orc_laser_tables(int W, int H, float hfov_deg, float vfov_deg, float* sinu, float* cosu,
                      float* sinv, float* cosv) {
  RoundGuard g(0);
  const float su = hfov_deg / (float)W, sv = vfov_deg / (float)H;
  for (int w = 0; w < W; ++w) {
    const float u = -hfov_deg / 2.0f + (float)w * su;
    const double ur = (double)u * 3.14159265358979323846 / 180.0;
    sinu[w] = (float)std::sin(ur);
    cosu[w] = (float)std::cos(ur);
  }
  for (int h = 0; h < H; ++h) {
    const float v = -vfov_deg / 2.0f + (float)h * sv;
    const double vr = (double)v * 3.14159265358979323846 / 180.0;
    sinv[h] = (float)std::sin(vr);
    cosv[h] = (float)std::cos(vr);
  }
}

static inline void sensor_dir(const orc_sensor* s, int w, int h, float d[3]) {
  if (s->type == 0) {
    const float u = (float)w * s->scale_u;
    const float v = (float)h * s->scale_v;
    d[0] = u * s->c0 - s->hw;
    d[1] = v * s->c1 - s->hh;
    d[2] = 1.0f;
  } else {
    d[0] = s->sinu[w] * s->cosv[h];
    d[1] = s->sinv[h];
    d[2] = s->cosu[w] * s->cosv[h];
  }
}

// Range image (radial metres; <= 0 or NaN = no return) -> sensor-frame xyz.  Invalid
// pixels become NaN points, which the insertion skips.  Round-to-nearest.
void orc_ranges_to_points(const orc_sensor* s, const float* ranges, float* xyz) {
  RoundGuard g(0);
  const int W = s->width, H = s->height;
  for (int h = 0; h < H; ++h)
    for (int w = 0; w < W; ++w) {
      const int i = h * W + w;
      const float r = ranges[i];
      float* p = xyz + 3 * (size_t)i;
      if (!(r > 0.0f)) {
        p[0] = p[1] = p[2] = NAN;
        continue;
      }
      float d[3];
      sensor_dir(s, w, h, d);
      if (s->type == 0) {
        const float n = std::sqrt((d[0] * d[0] + d[1] * d[1]) + 1.0f);
        const float sc = r / n;
        p[0] = d[0] * sc;
        p[1] = d[1] * sc;
        p[2] = sc;
      } else {
        p[0] = d[0] * r;
        p[1] = d[1] * r;
        p[2] = d[2] * r;
      }
    }
}

// Trace one point; writes (x, y, z, kind) per label event (kind 0 miss, 1 hit).
int64_t orc_trace(const float R[9], const double eye[3], double res_d, float max_time,
                  int rounding, float px, float py, float pz, int32_t* events,
                  int64_t max_events) {
  Frame f;
  std::memcpy(f.R, R, sizeof(f.R));
  std::memcpy(f.eye, eye, sizeof(f.eye));
  f.res_d = res_d;
  f.max_time = max_time;
  RoundGuard g(rounding);
  int64_t n = 0;
  trace_point(f, px, py, pz, [&](const int v[3], int kind) {
    if (n < max_events) {
      events[4 * n + 0] = v[0];
      events[4 * n + 1] = v[1];
      events[4 * n + 2] = v[2];
      events[4 * n + 3] = kind;
    }
    ++n;
  });
  return n;
}

void* orc_map_create(const orc_map_params* p) {
  OracleMap* m = new OracleMap();
  m->p.res = p->res;
  m->p.thres_hit = p->thres_hit;
  m->p.thres_miss = p->thres_miss;
  m->p.clamp_min = p->clamp_min;
  m->p.clamp_max = p->clamp_max;
  m->p.clamp_mode = p->clamp_mode;
  m->p.update_mode = p->update_mode;
  m->p.rounding = p->rounding;
  return m;
}

void orc_map_destroy(void* m) { delete static_cast<OracleMap*>(m); }

// One frame: label (or count) every voxel of every point, then integrate.  `stride` is in
// floats between consecutive points (3 for packed xyz).  `threads` > 1 splits the points
// over std::threads, each with its own label set, merged before integration.
int orc_map_insert(void* mp, const float R[9], const double eye[3], double res_d, float max_time,
                   float lh, float lm, const float* xyz, int64_t n, int64_t stride, int threads,
                   int keep_labels) {
  OracleMap* m = static_cast<OracleMap*>(mp);
  Frame f;
  std::memcpy(f.R, R, sizeof(f.R));
  std::memcpy(f.eye, eye, sizeof(f.eye));
  f.res_d = res_d;
  f.max_time = max_time;
  const int rounding = m->p.rounding;
  if (threads < 1) threads = 1;
  const MapParams& P = m->p;
  int64_t visits = 0, rays = 0;

  if (P.update_mode == 0) {
    std::vector<LabelSink> sinks(threads);
    std::vector<int64_t> tv(threads, 0), tr(threads, 0);
    auto work = [&](int t) {
      RoundGuard g(rounding);
      const int64_t b = n * t / threads, e = n * (t + 1) / threads;
      for (int64_t i = b; i < e; ++i) {
        const float* p = xyz + i * stride;
        const int64_t c = trace_point(f, p[0], p[1], p[2], sinks[t]);
        if (c >= 0) {
          tv[t] += c;
          tr[t] += 1;
        }
      }
    };
    if (threads == 1) {
      work(0);
    } else {
      std::vector<std::thread> th;
      for (int t = 0; t < threads; ++t) th.emplace_back(work, t);
      for (auto& x : th) x.join();
    }
    auto& merged = sinks[0].map;
    for (int t = 1; t < threads; ++t)
      for (auto& kv : sinks[t].map) {
        auto it = merged.find(kv.first);
        if (it == merged.end()) {
          merged.emplace(kv.first, kv.second);
        } else {
          for (int w = 0; w < 32; ++w) it->second.w[w] |= kv.second.w[w];
        }
      }
    for (int t = 0; t < threads; ++t) {
      visits += tv[t];
      rays += tr[t];
    }
    // integrate (Handler.cpp:113-120): hit overrides miss, one update per voxel.
    std::vector<std::pair<LeafLabels*, Leaf*>> work_items;
    work_items.reserve(merged.size());
    for (auto& kv : merged) work_items.emplace_back(&kv.second, &get_leaf(m, kv.first));
    int64_t uniq = 0;
    std::vector<int64_t> tu(threads, 0);
    auto integ = [&](int t) {
      RoundGuard g(rounding);
      const size_t b = work_items.size() * t / threads, e = work_items.size() * (t + 1) / threads;
      for (size_t i = b; i < e; ++i) {
        const LeafLabels& L = *work_items[i].first;
        Leaf& leaf = *work_items[i].second;
        for (int l = 0; l < 512; ++l) {
          const bool hit = (L.w[l >> 5] >> (l & 31)) & 1u;
          const bool miss = (L.w[16 + (l >> 5)] >> (l & 31)) & 1u;
          if (!hit && !miss) continue;
          tu[t] += 1;
          integrate_voxel(leaf.v[l], leaf.a[l], hit ? lh : lm, P);
        }
      }
    };
    if (threads == 1) {
      integ(0);
    } else {
      std::vector<std::thread> th;
      for (int t = 0; t < threads; ++t) th.emplace_back(integ, t);
      for (auto& x : th) x.join();
    }
    for (int t = 0; t < threads; ++t) uniq += tu[t];
    m->unique_voxels += uniq;
    if (keep_labels) m->last_labels = std::move(merged);
  } else if (P.update_mode == 1) {
    CountSink sink;
    {
      RoundGuard g(rounding);
      for (int64_t i = 0; i < n; ++i) {
        const float* p = xyz + i * stride;
        const int64_t c = trace_point(f, p[0], p[1], p[2], sink);
        if (c >= 0) {
          visits += c;
          rays += 1;
        }
      }
      for (auto& kv : sink.map) {
        Leaf& leaf = get_leaf(m, kv.first);
        for (int l = 0; l < 512; ++l) {
          const uint32_t nh = kv.second.hit[l], nm = kv.second.miss[l];
          if (nh == 0 && nm == 0) continue;
          m->unique_voxels += 1;
          const float temp = (float)nm * lm + (float)nh * lh;
          integrate_voxel(leaf.v[l], leaf.a[l], temp, P);
        }
      }
    }
  } else {
    SeqSink sink;
    sink.lh = lh;
    sink.lm = lm;
    RoundGuard g(rounding);
    for (int64_t i = 0; i < n; ++i) {
      const float* p = xyz + i * stride;
      const int64_t c = trace_point(f, p[0], p[1], p[2], sink);
      if (c >= 0) {
        visits += c;
        rays += 1;
      }
    }
    for (auto& kv : sink.map) {
      Leaf& leaf = get_leaf(m, kv.first);
      for (int l = 0; l < 512; ++l) {
        if (!kv.second.touched[l]) continue;
        m->unique_voxels += 1;
        integrate_voxel(leaf.v[l], leaf.a[l], kv.second.v[l], P);
      }
    }
  }
  m->visits += visits;
  m->rays += rays;
  return 0;
}

// Voxel filter (filterCloud.cu:84-133 and 279-318, FilterType 1) restated in the absolute
// index frame: every point that the insertion would trace is binned by the voxel holding its
// end point, q = eye + (R p) / res; each occupied voxel emits one point at the mean in-voxel
// position of its points (centre != 0: at the voxel centre, the integer-buffer variants
// rayFromFilterSimple / rayFromFilterSimpleQuad, filterCloud.cu:360-434).  The reference keys
// by q but accumulates fractions without the voxel-origin offset (filterCloud.cu:119 vs :126);
// here both use q.  Fractions are summed in 32-bit fixed point (exact and order-free; the sum
// of 2^30 fractions stays below 2^62).  Output: world-frame offsets from the eye (metres) and
// counts, sorted by voxel key (x, then y, then z relative to the eye voxel).
int64_t orc_voxel_filter(const float R[9], const double eye[3], double res_d, float max_time,
                         int rounding, int centre, const float* xyz, int64_t n, int64_t stride,
                         float* out_pts, uint32_t* out_counts, int64_t cap) {
  struct Acc {
    int64_t s[3];
    uint32_t n;
  };
  std::map<uint64_t, Acc> bins;
  const double kFix = 4294967296.0;  // 2^32
  double inv_res;
  {
    RoundGuard g(0);
    inv_res = 1.0 / res_d;
  }
  const int ev[3] = {(int)std::floor(eye[0]), (int)std::floor(eye[1]), (int)std::floor(eye[2])};
  for (int64_t i = 0; i < n; ++i) {
    const float* p = xyz + i * stride;
    float d[3];
    bool valid;
    {
      RoundGuard g(rounding);
      d[0] = (R[0] * p[0] + R[1] * p[1]) + R[2] * p[2];
      d[1] = (R[3] * p[0] + R[4] * p[1]) + R[5] * p[2];
      d[2] = (R[6] * p[0] + R[7] * p[1]) + R[8] * p[2];
      const double dx = d[0], dy = d[1], dz = d[2];
      const double len = std::sqrt((dx * dx + dy * dy) + dz * dz);
      const double ray_len = len / res_d;
      valid = (ray_len < (double)max_time) && (len > kMinLen);
    }
    if (!valid) continue;
    RoundGuard g(0);
    int64_t F[3];
    uint64_t key = 0;
    for (int a = 0; a < 3; ++a) {
      const double q = eye[a] + (double)d[a] * inv_res;
      const double v = std::floor(q);
      const double f = q - v;
      F[a] = (int64_t)(f * kFix);
      const int dv = (int)v - ev[a];
      key = (key << 21) | (uint64_t)((uint32_t)(dv + (1 << 20)) & 0x1FFFFFu);
    }
    Acc& A = bins[key];
    for (int a = 0; a < 3; ++a) A.s[a] += F[a];
    A.n += 1;
  }
  RoundGuard g(0);
  int64_t k = 0;
  for (auto& kv : bins) {
    if (k < cap && out_pts && out_counts) {
      for (int a = 0; a < 3; ++a) {
        const int dv = (int)((kv.first >> (42 - 21 * a)) & 0x1FFFFFu) - (1 << 20);
        const double v = (double)(ev[a] + dv);
        const double mean =
            centre ? 0.5 : ((double)kv.second.s[a] / (double)kv.second.n) * (1.0 / kFix);
        out_pts[3 * k + a] = (float)(((v + mean) - eye[a]) * res_d);
      }
      out_counts[k] = kv.second.n;
    }
    ++k;
  }
  return (int64_t)bins.size();
}

// Labels of the last frame inserted with keep_labels (label mode), sorted by leaf key.
int64_t orc_map_labels(void* mp, int32_t* origins, uint32_t* words, int64_t cap) {
  OracleMap* m = static_cast<OracleMap*>(mp);
  std::vector<uint64_t> keys;
  keys.reserve(m->last_labels.size());
  for (auto& kv : m->last_labels) keys.push_back(kv.first);
  std::sort(keys.begin(), keys.end());
  const int64_t n = (int64_t)keys.size();
  if (origins && words) {
    for (int64_t i = 0; i < n && i < cap; ++i) {
      key_origin(keys[i], origins + 3 * i);
      std::memcpy(words + 32 * i, m->last_labels[keys[i]].w, 32 * sizeof(uint32_t));
    }
  }
  return n;
}

// All leaves sorted by key: origins (3 ints), 512 values (x-major, z fastest), 512 active bytes.
int64_t orc_map_export(void* mp, int32_t* origins, float* values, uint8_t* active, int64_t cap) {
  OracleMap* m = static_cast<OracleMap*>(mp);
  std::vector<uint64_t> keys;
  keys.reserve(m->leaves.size());
  for (auto& kv : m->leaves) keys.push_back(kv.first);
  std::sort(keys.begin(), keys.end());
  const int64_t n = (int64_t)keys.size();
  if (origins && values && active) {
    for (int64_t i = 0; i < n && i < cap; ++i) {
      key_origin(keys[i], origins + 3 * i);
      const Leaf& L = m->leaves[keys[i]];
      std::memcpy(values + 512 * i, L.v, sizeof(L.v));
      std::memcpy(active + 512 * i, L.a, sizeof(L.a));
    }
  }
  return n;
}

void orc_map_stats(void* mp, int64_t out[4]) {
  OracleMap* m = static_cast<OracleMap*>(mp);
  out[0] = m->visits;
  out[1] = m->rays;
  out[2] = m->unique_voxels;
  out[3] = (int64_t)m->leaves.size();
}

// ---------------------------------------------------------------------------------------
// Sim map from primitives.  A voxel (i, j, k) is active when its centre ((i + 0.5) * res,
// ...) lies inside a box [min, max] (closed) or inside a vertical cylinder (cx, cy, r, z0,
// z1): (x - cx)^2 + (y - cy)^2 <= r^2 and z0 <= z <= z1.  Double arithmetic, nearest
// rounding, no fused multiply-add.  Voxels outside [vmin, vmax) are never set.
void* orc_simmap_create(float res, const int32_t vmin[3], const int32_t vmax[3],
                        const double* boxes, int nb, const double* cyl, int nc) {
  RoundGuard g(0);
  SimMap* s = new SimMap();
  s->res = res;
  const double r = (double)res;
  auto centre = [&](int i) { return ((double)i + 0.5) * r; };
  auto lo_idx = [&](double x, int a) {
    return std::max(vmin[a], (int)std::floor(x / r - 0.5) - 1);
  };
  auto hi_idx = [&](double x, int a) {
    return std::min(vmax[a] - 1, (int)std::ceil(x / r - 0.5) + 1);
  };
  for (int b = 0; b < nb; ++b) {
    const double* B = boxes + 6 * b;
    const int i0 = lo_idx(B[0], 0), i1 = hi_idx(B[3], 0);
    const int j0 = lo_idx(B[1], 1), j1 = hi_idx(B[4], 1);
    const int k0 = lo_idx(B[2], 2), k1 = hi_idx(B[5], 2);
    for (int i = i0; i <= i1; ++i) {
      const double cx = centre(i);
      if (!(B[0] <= cx && cx <= B[3])) continue;
      for (int j = j0; j <= j1; ++j) {
        const double cy = centre(j);
        if (!(B[1] <= cy && cy <= B[4])) continue;
        for (int k = k0; k <= k1; ++k) {
          const double cz = centre(k);
          if (B[2] <= cz && cz <= B[5]) s->set(i, j, k);
        }
      }
    }
  }
  for (int c = 0; c < nc; ++c) {
    const double* C = cyl + 5 * c;
    const double rr = C[2] * C[2];
    const int i0 = lo_idx(C[0] - C[2], 0), i1 = hi_idx(C[0] + C[2], 0);
    const int j0 = lo_idx(C[1] - C[2], 1), j1 = hi_idx(C[1] + C[2], 1);
    const int k0 = lo_idx(C[3], 2), k1 = hi_idx(C[4], 2);
    for (int i = i0; i <= i1; ++i) {
      const double dx = centre(i) - C[0];
      for (int j = j0; j <= j1; ++j) {
        const double dy = centre(j) - C[1];
        if (!(dx * dx + dy * dy <= rr)) continue;
        for (int k = k0; k <= k1; ++k) {
          const double cz = centre(k);
          if (C[3] <= cz && cz <= C[4]) s->set(i, j, k);
        }
      }
    }
  }
  return s;
}

void* orc_simmap_from_voxels(float res, const int32_t* ijk, int64_t n) {
  SimMap* s = new SimMap();
  s->res = res;
  for (int64_t i = 0; i < n; ++i) s->set(ijk[3 * i], ijk[3 * i + 1], ijk[3 * i + 2]);
  return s;
}

void orc_simmap_destroy(void* s) { delete static_cast<SimMap*>(s); }

void orc_simmap_bbox(void* sp, int32_t out[7]) {
  SimMap* s = static_cast<SimMap*>(sp);
  for (int a = 0; a < 3; ++a) {
    out[a] = s->amin[a];
    out[3 + a] = s->amax[a];
  }
  out[6] = s->any ? 1 : 0;
}

int64_t orc_simmap_export(void* sp, int32_t* origins, uint32_t* words, int64_t cap) {
  SimMap* s = static_cast<SimMap*>(sp);
  std::vector<uint64_t> keys;
  for (auto& kv : s->leaves) keys.push_back(kv.first);
  std::sort(keys.begin(), keys.end());
  const int64_t n = (int64_t)keys.size();
  if (origins && words)
    for (int64_t i = 0; i < n && i < cap; ++i) {
      key_origin(keys[i], origins + 3 * i);
      std::memcpy(words + 16 * i, s->leaves[keys[i]].data(), 64);
    }
  return n;
}

int64_t orc_simmap_count(void* sp) {
  SimMap* s = static_cast<SimMap*>(sp);
  int64_t c = 0;
  for (auto& kv : s->leaves)
    for (int w = 0; w < 16; ++w) c += __builtin_popcount(kv.second[w]);
  return c;
}

// Simulated range image (generateCloud.cu:20-82 restated with a closed-form voxel DDA).
// Ray: eye = position / res, direction = normalise(R d) where d is the sensor-frame pixel
// direction.  The ray is clipped to the active box [amin, amax + 1]; starting from the voxel
// holding the clipped start, each step enters the neighbour across the face with the
// smallest crossing time t = (plane - eye) / dir (ties to the higher axis).  The first
// entered voxel that is active ends the ray at its entry time t.  Output range = t * res
// when minRange/res * n <= t <= maxRange/res * n (n = |R d| for frustum pixels, 1 for
// laser beams), else 0.  Single precision, round to nearest.
static void sim_render_rows(const SimMap* s, const orc_sensor* sen, const float pos[3],
                            const float R[9], float* out, int h0, int h1);

void orc_sim_render(void* sp, const orc_sensor* sen, const float pos[3], const float R[9],
                    float* out, int threads) {
  const SimMap* s = static_cast<SimMap*>(sp);
  const int H = sen->height;
  if (threads <= 1) {
    sim_render_rows(s, sen, pos, R, out, 0, H);
    return;
  }
  std::vector<std::thread> th;
  for (int t = 0; t < threads; ++t)
    th.emplace_back(sim_render_rows, s, sen, pos, R, out, H * t / threads, H * (t + 1) / threads);
  for (auto& x : th) x.join();
}

// First active voxel entered along the ray from `eye` (index space) in the unit direction
// `dir`, at a ray time within [tmin, tmax]: its distance in metres, or 0.  The voxel holding
// the eye is not tested (generateCloud.cu:28-39).  Round-to-nearest float.
static float sim_cast(const SimMap* s, const float eye[3], float dir[3], float tmin, float tmax) {
  const float res = s->res;
  const float lo[3] = {(float)s->amin[0], (float)s->amin[1], (float)s->amin[2]};
  const float hi[3] = {(float)(s->amax[0] + 1), (float)(s->amax[1] + 1), (float)(s->amax[2] + 1)};
  float inv[3];
  int stp[3];
  float t_in = 0.0f, t_out = INFINITY;
  bool miss = false;
  for (int a = 0; a < 3; ++a) {
    if (std::fabs(dir[a]) < 1e-30f) dir[a] = 0.0f;
    if (dir[a] == 0.0f) {
      stp[a] = 0;
      inv[a] = 0.0f;
      if (eye[a] < lo[a] || eye[a] > hi[a]) miss = true;
    } else {
      inv[a] = 1.0f / dir[a];
      stp[a] = dir[a] > 0.0f ? 1 : -1;
      float ta = (lo[a] - eye[a]) * inv[a];
      float tb = (hi[a] - eye[a]) * inv[a];
      if (ta > tb) std::swap(ta, tb);
      if (ta > t_in) t_in = ta;
      if (tb < t_out) t_out = tb;
    }
  }
  if (miss || t_in > t_out) return 0.0f;
  int k[3];
  for (int a = 0; a < 3; ++a) k[a] = (int)std::floor(eye[a] + dir[a] * t_in);
  for (;;) {
    float tn[3];
    for (int a = 0; a < 3; ++a)
      tn[a] = (stp[a] == 0) ? INFINITY
                            : ((float)(k[a] + (stp[a] > 0 ? 1 : 0)) - eye[a]) * inv[a];
    const int a = argmin_hi_f(tn);
    const float t = tn[a];
    if (!(t <= t_out)) break;
    k[a] += stp[a];
    if (s->active(k)) return (t >= tmin && t <= tmax) ? t * res : 0.0f;
  }
  return 0.0f;
}

static void sim_render_rows(const SimMap* s, const orc_sensor* sen, const float pos[3],
                            const float R[9], float* out, int h0, int h1) {
  RoundGuard g(0);
  const int W = sen->width;
  const float res = s->res;
  const float eye[3] = {pos[0] / res, pos[1] / res, pos[2] / res};
  for (int h = h0; h < h1; ++h)
    for (int w = 0; w < W; ++w) {
      float* o = out + (size_t)h * W + w;
      *o = 0.0f;
      if (!s->any) continue;
      float d[3];
      sensor_dir(sen, w, h, d);
      const float m0 = (R[0] * d[0] + R[1] * d[1]) + R[2] * d[2];
      const float m1 = (R[3] * d[0] + R[4] * d[1]) + R[5] * d[2];
      const float m2 = (R[6] * d[0] + R[7] * d[1]) + R[8] * d[2];
      const float norm = std::sqrt((m0 * m0 + m1 * m1) + m2 * m2);
      float dir[3] = {m0 / norm, m1 / norm, m2 / norm};
      float tmin, tmax;
      if (sen->type == 0) {
        tmin = (sen->min_range / res) * norm;
        tmax = (sen->max_range / res) * norm;
      } else {
        tmin = sen->min_range / res;
        tmax = sen->max_range / res;
      }
      *o = sim_cast(s, eye, dir, tmin, tmax);
    }
}

// Arbitrary rays (agent observation / collision rays): origins in metres, directions of any
// length, distances to the first active voxel within max_range metres, else 0.
void orc_sim_cast(void* sp, const float* origins, const float* dirs, int64_t n, float max_range,
                  float* out) {
  const SimMap* s = static_cast<const SimMap*>(sp);
  RoundGuard g(0);
  const float res = s->res;
  for (int64_t i = 0; i < n; ++i) {
    out[i] = 0.0f;
    if (!s->any) continue;
    const float m0 = dirs[3 * i], m1 = dirs[3 * i + 1], m2 = dirs[3 * i + 2];
    const float norm = std::sqrt((m0 * m0 + m1 * m1) + m2 * m2);
    if (!(norm > 0.0f && norm < INFINITY)) continue;
    float dir[3] = {m0 / norm, m1 / norm, m2 / norm};
    const float eye[3] = {origins[3 * i] / res, origins[3 * i + 1] / res, origins[3 * i + 2] / res};
    out[i] = sim_cast(s, eye, dir, 0.0f, max_range / res);
  }
}

// Analytic range image of axis-aligned boxes (world metres), FP64 slab intersections, rounded
// to float.  Used to make the synthetic depth of the small plain-mapping scene.  The ray is
// the pixel direction R d (R given in double, row-major); range = distance to the nearest
// box entry, 0 when none lies within max_range.
void orc_render_boxes(const orc_sensor* sen, const double pos[3], const double Rd[9],
                      const double* boxes, int nb, float* out) {
  RoundGuard g(0);
  const int W = sen->width, H = sen->height;
  for (int h = 0; h < H; ++h)
    for (int w = 0; w < W; ++w) {
      double d[3];
      if (sen->type == 0) {
        const double u = (double)w / W, v = (double)h / H;
        d[0] = (2.0 * u - 1.0) * sen->hw;
        d[1] = (2.0 * v - 1.0) * sen->hh;
        d[2] = 1.0;
      } else {
        d[0] = (double)sen->sinu[w] * sen->cosv[h];
        d[1] = (double)sen->sinv[h];
        d[2] = (double)sen->cosu[w] * sen->cosv[h];
      }
      double m[3];
      for (int r = 0; r < 3; ++r) m[r] = Rd[r * 3] * d[0] + Rd[r * 3 + 1] * d[1] + Rd[r * 3 + 2] * d[2];
      const double n = std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
      for (int r = 0; r < 3; ++r) m[r] /= n;
      double best = INFINITY;
      for (int b = 0; b < nb; ++b) {
        const double* B = boxes + 6 * b;
        double t0 = 0.0, t1 = INFINITY;
        bool ok = true;
        for (int a = 0; a < 3 && ok; ++a) {
          if (m[a] == 0.0) {
            if (pos[a] < B[a] || pos[a] > B[3 + a]) ok = false;
          } else {
            double ta = (B[a] - pos[a]) / m[a], tb = (B[3 + a] - pos[a]) / m[a];
            if (ta > tb) std::swap(ta, tb);
            t0 = std::max(t0, ta);
            t1 = std::min(t1, tb);
            if (t0 > t1) ok = false;
          }
        }
        if (ok && t0 < best) best = t0;
      }
      out[(size_t)h * W + w] = (best <= (double)sen->max_range && best > 0.0) ? (float)best : 0.0f;
    }
}

}  // extern "C"
