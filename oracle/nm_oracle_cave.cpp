// nm_oracle_cave.cpp -- CPU restatement of the reference's procedural cave generator.
// TEST INFRASTRUCTURE ONLY: the checker of the device cave generator, never the product.
//
// Follows nanomap/mapgen/procedural/CaveGen.cpp stage by stage on a sparse set of voxel
// coordinates (the reference keeps the cells in an OpenVDB FloatGrid):
//   populate       CaveGen::populateMap (CaveGen.cpp:13-47), populateMap2D (:49-84)
//   smooth         CaveGen::smoothMap (:95-129) + getActiveNeighbourCount (:258-273),
//                  smoothMapXY (:130-176) + get2DNeighbourCount (:275-292)
//   floor_ceil     CaveGen::setFloorAndCeil (:86-94)
//   regions        CaveGen::getRegions (:178-240): flood fill from each on cell in the grid's
//                  value order; the first of the largest regions wins (:232-239)
//   keep_largest   CaveGen::keepLargestRegion (:242-252)
//   voxels         addTile(1, c) + voxelizeActiveTiles (:300-313, 329-333), and for the shell
//                  the active topology of tools::topologyToLevelSet(grid) with its defaults
//                  (half width 3, closing 1): band = dilate^3(M) \ erode^3(M) with
//                  M = erode(dilate(T)), face-neighbour morphology.
// The fill draws from the C library's srand/rand exactly as the reference does; the
// alternative counter-based fill is splitmix64 of the seed and the cell's lattice position.
//
// PARITY UNPINNED against the reference: the reference ships no cave tests or fixtures and
// OpenVDB (the value order and topologyToLevelSet) is not available here; the order is
// restated from OpenVDB's published tree layout (root table ordered by coordinate, 32^3 /
// 16^3 / 8^3 child tables indexed x-major) and the band from the published morphology.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <set>
#include <unordered_set>
#include <vector>

namespace {

using Coord = std::array<int, 3>;

struct CoordHash {
  size_t operator()(const Coord& c) const {
    return ((size_t)(uint32_t)c[0] * 73856093u) ^ ((size_t)(uint32_t)c[1] * 19349663u) ^
           ((size_t)(uint32_t)c[2] * 83492791u);
  }
};

// OpenVDB's value order of a 5-4-3 tree, as a lexicographic comparison of the path from the
// root: root table key (coordinate with the low 12 bits cleared, compared x, y, z), then the
// child index at the 32^3, 16^3 and 8^3 levels (x-major).
std::array<int, 12> order_path(const Coord& c) {
  std::array<int, 12> p;
  for (int a = 0; a < 3; ++a) p[a] = c[a] >> 12;
  for (int a = 0; a < 3; ++a) p[3 + a] = (c[a] >> 7) & 31;
  for (int a = 0; a < 3; ++a) p[6 + a] = (c[a] >> 3) & 15;
  for (int a = 0; a < 3; ++a) p[9 + a] = c[a] & 7;
  return p;
}
bool order_less(const Coord& a, const Coord& b) { return order_path(a) < order_path(b); }

uint64_t splitmix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

struct Cave {
  double size[3];
  double res;
  int fill, smoothing, amax, amin;
  uint32_t seed;
  int D[3];
  std::unordered_set<Coord, CoordHash> on;
  bool is_on(int x, int y, int z) const { return on.count(Coord{x, y, z}) != 0; }
};

}  // namespace

extern "C" {

void* orc_cave_new(const double size[3], double res, int fill, int smoothing, int amax, int amin,
                   uint32_t seed) {
  Cave* c = new Cave();
  for (int a = 0; a < 3; ++a) c->size[a] = size[a];
  c->res = res;
  c->fill = fill;
  c->smoothing = smoothing;
  c->amax = amax;
  c->amin = amin;
  c->seed = seed;
  for (int a = 0; a < 3; ++a) {
    const int n = (int)std::ceil(size[a] / res);
    c->D[a] = (n % 2 != 0) ? (n + 1) / 2 : n / 2;
  }
  return c;
}

void orc_cave_free(void* h) { delete static_cast<Cave*>(h); }

void orc_cave_dims(void* h, int32_t D[3]) {
  const Cave* c = static_cast<Cave*>(h);
  for (int a = 0; a < 3; ++a) D[a] = c->D[a];
}

// CaveGen::populateMap / populateMap2D.  counter = 1: splitmix64 fill keyed by the lattice
// position (i, j, k) = ((x + Dx - 8) / 8, (y + Dy - 8) / 8, (z + Dz) / 8).
void orc_cave_populate(void* h, int mode_2d, int counter) {
  Cave* c = static_cast<Cave*>(h);
  c->on.clear();
  const int Dx = c->D[0], Dy = c->D[1], Dz = c->D[2];
  if (!counter) srand(c->seed);
  auto draw = [&](int x, int y, int z) {
    if (!counter) return rand() % 100;
    const uint64_t i = (uint64_t)((x + Dx - 8) / 8), j = (uint64_t)((y + Dy - 8) / 8);
    const uint64_t k = mode_2d ? 0 : (uint64_t)((z + Dz) / 8);
    const uint64_t hh = splitmix64(((uint64_t)c->seed << 32) ^ ((i << 42) | (j << 21) | k));
    return (int)((uint32_t)(hh >> 32) % 100u);
  };
  for (int x = -Dx + 8; x < Dx - 8; x += 8)
    for (int y = -Dy + 8; y < Dy - 8; y += 8) {
      if (mode_2d) {
        if (draw(x, y, 0) < c->fill)
          for (int z = -Dz; z < Dz; z += 8) c->on.insert(Coord{x, y, z});
      } else {
        for (int z = -Dz + 8; z < Dz - 8; z += 8)
          if (draw(x, y, z) < c->fill) c->on.insert(Coord{x, y, z});
      }
    }
}

// smoothing_count steps of CaveGen::smoothMap (3-D) or smoothMapXY (2-D).  Each step writes a
// fresh grid, so cells outside the swept range (the ceiling plane) do not survive it.
void orc_cave_smooth(void* h, int mode_2d) {
  Cave* c = static_cast<Cave*>(h);
  const int Dx = c->D[0], Dy = c->D[1], Dz = c->D[2];
  for (int it = 0; it < c->smoothing; ++it) {
    std::unordered_set<Coord, CoordHash> next;
    for (int x = -Dx + 8; x < Dx - 8; x += 8)
      for (int y = -Dy + 8; y < Dy - 8; y += 8) {
        if (mode_2d) {
          int cnt = 0;
          for (int dx = -8; dx <= 8; dx += 8)
            for (int dy = -8; dy <= 8; dy += 8)
              if (!(dx == 0 && dy == 0) && c->is_on(x + dx, y + dy, -Dz)) ++cnt;
          const bool v = cnt > c->amax ? true : (cnt < c->amin ? false : c->is_on(x, y, -Dz));
          if (v)
            for (int z = -Dz; z < Dz; z += 8) next.insert(Coord{x, y, z});
        } else {
          for (int z = -Dz; z < Dz; z += 8) {
            int cnt = 0;
            for (int dx = -8; dx <= 8; dx += 8)
              for (int dy = -8; dy <= 8; dy += 8)
                for (int dz = -8; dz <= 8; dz += 8)
                  if (!(dx == 0 && dy == 0 && dz == 0) && c->is_on(x + dx, y + dy, z + dz)) ++cnt;
            const bool v = cnt > c->amax ? true : (cnt < c->amin ? false : c->is_on(x, y, z));
            if (v) next.insert(Coord{x, y, z});
          }
        }
      }
    c->on.swap(next);
  }
}

// Test hook: replace the on cells by the given voxel coordinates.
void orc_cave_set_cells(void* h, const int32_t* xyz, int64_t n) {
  Cave* c = static_cast<Cave*>(h);
  c->on.clear();
  for (int64_t q = 0; q < n; ++q) c->on.insert(Coord{xyz[3 * q], xyz[3 * q + 1], xyz[3 * q + 2]});
}

void orc_cave_floor_ceil(void* h) {
  Cave* c = static_cast<Cave*>(h);
  const int Dx = c->D[0], Dy = c->D[1], Dz = c->D[2];
  for (int x = -Dx + 8; x < Dx - 8; x += 8)
    for (int y = -Dy + 8; y < Dy - 8; y += 8) {
      c->on.insert(Coord{x, y, -Dz});
      c->on.insert(Coord{x, y, Dz});
    }
}

namespace {
std::vector<Coord> sorted_cells(const Cave* c) {
  std::vector<Coord> v(c->on.begin(), c->on.end());
  std::sort(v.begin(), v.end(), order_less);
  return v;
}

// Regions in discovery order (flood fill by face steps of 8 from each unvisited on cell, in
// value order); returns the index of the first largest.
std::vector<std::vector<Coord>> find_regions(const Cave* c, size_t* best) {
  std::vector<std::vector<Coord>> regions;
  std::unordered_set<Coord, CoordHash> seen;
  for (const Coord& start : sorted_cells(c)) {
    if (seen.count(start)) continue;
    std::vector<Coord> region{start};
    std::vector<Coord> stack{start};
    seen.insert(start);
    while (!stack.empty()) {
      const Coord cur = stack.back();
      stack.pop_back();
      for (int a = 0; a < 3; ++a)
        for (int d = -8; d <= 8; d += 16) {
          Coord n = cur;
          n[a] += d;
          if (c->on.count(n) && !seen.count(n)) {
            seen.insert(n);
            stack.push_back(n);
            region.push_back(n);
          }
        }
    }
    regions.push_back(std::move(region));
  }
  *best = 0;
  for (size_t r = 0; r < regions.size(); ++r)
    if (regions[r].size() > regions[*best].size()) *best = r;
  return regions;
}
}  // namespace

void orc_cave_regions(void* h, int64_t* n_regions, int64_t* largest) {
  size_t best = 0;
  const auto regions = find_regions(static_cast<Cave*>(h), &best);
  *n_regions = (int64_t)regions.size();
  *largest = regions.empty() ? 0 : (int64_t)regions[best].size();
}

void orc_cave_keep_largest(void* h) {
  Cave* c = static_cast<Cave*>(h);
  size_t best = 0;
  auto regions = find_regions(c, &best);
  c->on.clear();
  if (!regions.empty())
    for (const Coord& q : regions[best]) c->on.insert(q);
}

// On cells in value order; returns their number (writes at most max_cells).
int64_t orc_cave_cells(void* h, int32_t* xyz, int64_t max_cells) {
  const auto v = sorted_cells(static_cast<Cave*>(h));
  for (size_t q = 0; q < v.size() && (int64_t)q < max_cells; ++q)
    for (int a = 0; a < 3; ++a) xyz[3 * q + a] = v[q][a];
  return (int64_t)v.size();
}

// Active voxels of the saved grid, sorted by (x, y, z): the on cells' leaves, or (shell = 1)
// the level-set band around them.  Returns their number (writes at most max_voxels).
int64_t orc_cave_voxels(void* h, int shell, int half_width, int closing, int32_t* xyz,
                        int64_t max_voxels) {
  const Cave* c = static_cast<Cave*>(h);
  if (c->on.empty()) return 0;
  int lo[3] = {INT32_MAX, INT32_MAX, INT32_MAX}, hi[3] = {INT32_MIN, INT32_MIN, INT32_MIN};
  for (const Coord& q : c->on)
    for (int a = 0; a < 3; ++a) {
      lo[a] = std::min(lo[a], (q[a] >> 3) * 8);
      hi[a] = std::max(hi[a], (q[a] >> 3) * 8 + 7);
    }
  const int pad = shell ? closing + half_width + 1 : 0;
  int o[3], n[3];
  for (int a = 0; a < 3; ++a) {
    o[a] = lo[a] - pad;
    n[a] = hi[a] - lo[a] + 1 + 2 * pad;
  }
  const size_t total = (size_t)n[0] * n[1] * n[2];
  auto at = [&](int x, int y, int z) { return ((size_t)x * n[1] + y) * n[2] + z; };
  std::vector<uint8_t> T(total, 0);
  for (const Coord& q : c->on) {
    const int bx = (q[0] >> 3) * 8 - o[0], by = (q[1] >> 3) * 8 - o[1], bz = (q[2] >> 3) * 8 - o[2];
    for (int x = 0; x < 8; ++x)
      for (int y = 0; y < 8; ++y)
        for (int z = 0; z < 8; ++z) T[at(bx + x, by + y, bz + z)] = 1;
  }
  // one face-neighbour step: dilation keeps a voxel on when it or any face neighbour is on,
  // erosion when it and all six are (outside the volume counts as off)
  auto step = [&](const std::vector<uint8_t>& in, bool erode) {
    std::vector<uint8_t> out(total, 0);
    for (int x = 0; x < n[0]; ++x)
      for (int y = 0; y < n[1]; ++y)
        for (int z = 0; z < n[2]; ++z) {
          const int nb[6][3] = {{x - 1, y, z}, {x + 1, y, z}, {x, y - 1, z},
                                {x, y + 1, z}, {x, y, z - 1}, {x, y, z + 1}};
          bool any = false, all = true;
          for (const auto& p : nb) {
            const bool inside = p[0] >= 0 && p[0] < n[0] && p[1] >= 0 && p[1] < n[1] &&
                                p[2] >= 0 && p[2] < n[2];
            const bool v = inside && in[at(p[0], p[1], p[2])];
            any = any || v;
            all = all && v;
          }
          const bool self = in[at(x, y, z)] != 0;
          out[at(x, y, z)] = erode ? (self && all) : (self || any);
        }
    return out;
  };
  std::vector<uint8_t> R = T;
  if (shell) {
    std::vector<uint8_t> M = T;
    for (int i = 0; i < closing; ++i) M = step(M, false);
    for (int i = 0; i < closing; ++i) M = step(M, true);
    std::vector<uint8_t> Dl = M, E = M;
    for (int i = 0; i < half_width; ++i) Dl = step(Dl, false);
    for (int i = 0; i < half_width; ++i) E = step(E, true);
    for (size_t q = 0; q < total; ++q) R[q] = Dl[q] && !E[q];
  }
  int64_t cnt = 0;
  for (int x = 0; x < n[0]; ++x)
    for (int y = 0; y < n[1]; ++y)
      for (int z = 0; z < n[2]; ++z)
        if (R[at(x, y, z)]) {
          if (cnt < max_voxels) {
            xyz[3 * cnt] = x + o[0];
            xyz[3 * cnt + 1] = y + o[1];
            xyz[3 * cnt + 2] = z + o[2];
          }
          ++cnt;
        }
  return cnt;
}

}  // extern "C"
