// nm_cave.cu -- procedural cave generation on the device (replaces CaveGen.cpp).
//
// Every stage of the reference's generator is one or a few grid-stride kernels over the cell
// lattice (a few thousand to a few million one-byte cells), and the level-set shell is
// face-neighbour morphology on 8^3 leaf bit masks in the sim map's build layout, so the
// result goes into a device sim map without a host round trip:
//   k_cave_fill        counter-based fill (the C library sequence is drawn on the host)
//   k_cave_smooth3d/2d one cellular-automaton step (CaveGen::smoothMap / smoothMapXY)
//   k_cc_*             6-connected regions by lock-free union-find (CaveGen::getRegions)
//   k_cave_tiles       cells -> whole leaves (addTile(1, ...) + voxelizeActiveTiles)
//   k_leaf_morph       one dilation or erosion step on 64-bit x-slices, walking runs of
//                      leaves along x
//   k_compact (nm_sim.cu) compacts the band into the sim map
#include <climits>
#include <cstdint>

#include "nm_cave.h"

namespace nm {

namespace {

constexpr int kGrid = 1184;  // 148 SMs x 8 resident blocks of 256 threads
constexpr int kUnionIters = 1 << 20;

__host__ __device__ inline unsigned long long splitmix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ void cell_ijk(const CaveLattice& L, long long c, int* i, int* j,
                                         int* k) {
  const int nzp = L.nz + 1;
  *k = (int)(c % nzp);
  const long long r = c / nzp;
  *j = (int)(r % L.ny);
  *i = (int)(r / L.ny);
}

// Counter-based fill: one draw per cell (3-D) or per column (2-D), splitmix64 of the seed and
// the cell's lattice position.
__global__ void k_cave_fill(CaveLattice L, uint32_t seed, int pct, int mode_2d) {
  const long long n = cave_cell_count(L);
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    cell_ijk(L, c, &i, &j, &k);
    bool on = false;
    if (mode_2d ? (k < L.nz) : (k >= 1 && k < L.kf)) {
      const unsigned long long pos = ((unsigned long long)i << 42) |
                                     ((unsigned long long)j << 21) |
                                     (unsigned long long)(mode_2d ? 0 : k);
      const unsigned long long h = splitmix64(((unsigned long long)seed << 32) ^ pos);
      on = (int)((uint32_t)(h >> 32) % 100u) < pct;
    }
    L.cells[c] = on ? 1 : 0;
  }
}

// Draw d of the reference's fill loops: 3-D, d = ((i * ny) + j) * (kf - 1) + (k - 1) over the
// fill planes k in [1, kf); 2-D, d = i * ny + j for the whole column below the ceiling.  The
// cells start cleared.
__global__ void k_cave_fill_libc(CaveLattice L, const uint32_t* __restrict__ mats, int nmats,
                                 const uint32_t* __restrict__ state0, long long n_draws, int pct,
                                 int mode_2d) {
  const long long nchunks = (n_draws + kLibcChunk - 1) / kLibcChunk;
  const int nzp = L.nz + 1;
  const int nfill = L.kf - 1;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nchunks;
       t += (long long)gridDim.x * blockDim.x) {
    uint32_t r[31];
#pragma unroll
    for (int q = 0; q < 31; ++q) r[q] = __ldg(&state0[q]);
    for (int j = 0; j < nmats; ++j) {
      if (!((t >> j) & 1)) continue;
      const uint32_t* M = mats + (size_t)j * 961;
      uint32_t y[31];
#pragma unroll
      for (int a = 0; a < 31; ++a) {
        uint32_t acc = 0u;
#pragma unroll
        for (int b = 0; b < 31; ++b) acc += __ldg(&M[a * 31 + b]) * r[b];
        y[a] = acc;
      }
#pragma unroll
      for (int q = 0; q < 31; ++q) r[q] = y[q];
    }
    // r[q] holds the word 31 - q draws back; the oldest word sits at slot p and is replaced by
    // the new one, with slot (p + 28) mod 31 holding the word 3 back
    long long d = t * kLibcChunk;
    for (int g = 0; g < kLibcChunk / 31; ++g) {
#pragma unroll
      for (int p = 0; p < 31; ++p) {
        const uint32_t v = r[p] + r[(p + 28) % 31];
        r[p] = v;
        const long long dd = d + p;
        if (dd < n_draws) {
          const uint8_t on = ((int)((v >> 1) % 100u) < pct) ? 1 : 0;
          if (mode_2d) {
            uint8_t* col = L.cells + dd * nzp;
            for (int k = 0; k < L.nz; ++k) col[k] = on;
          } else {
            const long long c = (dd / nfill) * nzp + 1 + (dd % nfill);
            L.cells[c] = on;
          }
        }
      }
      d += 31;
    }
  }
}

// One step of CaveGen::smoothMap: 26-neighbour count on the lattice (planes below the ceiling,
// and the ceiling plane where it is a face neighbour); more than amax -> on, fewer than amin
// -> off, else unchanged.  The ceiling plane is not part of the step's output (off after).
__global__ void k_cave_smooth3d(CaveLattice L, const uint8_t* __restrict__ cur,
                                uint8_t* __restrict__ next, int amax, int amin) {
  const long long n = cave_cell_count(L);
  const int ktop = L.ceil_adjacent ? L.nz : L.nz - 1;  // highest plane a neighbour can be in
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    cell_ijk(L, c, &i, &j, &k);
    if (k >= L.nz) {
      next[c] = 0;
      continue;
    }
    int cnt = 0;
    for (int dx = -1; dx <= 1; ++dx) {
      const int ii = i + dx;
      if (ii < 0 || ii >= L.nx) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int jj = j + dy;
        if (jj < 0 || jj >= L.ny) continue;
        const long long base = ((long long)ii * L.ny + jj) * (L.nz + 1);
        for (int dz = -1; dz <= 1; ++dz) {
          const int kk = k + dz;
          if (kk < 0 || kk > ktop || (dx == 0 && dy == 0 && dz == 0)) continue;
          cnt += cur[base + kk];
        }
      }
    }
    next[c] = cnt > amax ? 1 : (cnt < amin ? 0 : cur[c]);
  }
}

// The 26-neighbour count of k_cave_smooth3d in two passes: the 3 x 3 in-plane sums of every
// cell (all planes, the ceiling included), then per cell the sums of its plane and the planes
// below and above it (where they are neighbours) minus the cell itself.
__global__ void k_cave_plane_sums(CaveLattice L, const uint8_t* __restrict__ cur,
                                  uint8_t* __restrict__ sums) {
  const long long n = cave_cell_count(L);
  const int nzp = L.nz + 1;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    int i, j, k;
    cell_ijk(L, c, &i, &j, &k);
    int sum = 0;
    for (int dx = -1; dx <= 1; ++dx) {
      const int ii = i + dx;
      if (ii < 0 || ii >= L.nx) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int jj = j + dy;
        if (jj < 0 || jj >= L.ny) continue;
        sum += cur[((long long)ii * L.ny + jj) * nzp + k];
      }
    }
    sums[c] = (uint8_t)sum;
  }
}

__global__ void k_cave_smooth3d_sums(CaveLattice L, const uint8_t* __restrict__ cur,
                                     const uint8_t* __restrict__ sums, uint8_t* __restrict__ next,
                                     int amax, int amin) {
  const long long n = cave_cell_count(L);
  const int nzp = L.nz + 1;
  const int ktop = L.ceil_adjacent ? L.nz : L.nz - 1;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(c % nzp);
    if (k >= L.nz) {
      next[c] = 0;
      continue;
    }
    int cnt = sums[c] - cur[c];
    if (k > 0) cnt += sums[c - 1];
    if (k + 1 <= ktop) cnt += sums[c + 1];
    next[c] = cnt > amax ? 1 : (cnt < amin ? 0 : cur[c]);
  }
}

// One step of CaveGen::smoothMapXY: 8-neighbour count in the floor plane (k = 0), the result
// written to the whole column below the ceiling.
__global__ void k_cave_smooth2d(CaveLattice L, const uint8_t* __restrict__ cur,
                                uint8_t* __restrict__ next, int amax, int amin) {
  const long long ncol = (long long)L.nx * L.ny;
  const int nzp = L.nz + 1;
  for (long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x; col < ncol;
       col += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(col / L.ny), j = (int)(col % L.ny);
    int cnt = 0;
    for (int dx = -1; dx <= 1; ++dx) {
      const int ii = i + dx;
      if (ii < 0 || ii >= L.nx) continue;
      for (int dy = -1; dy <= 1; ++dy) {
        const int jj = j + dy;
        if (jj < 0 || jj >= L.ny || (dx == 0 && dy == 0)) continue;
        cnt += cur[((long long)ii * L.ny + jj) * nzp];
      }
    }
    const uint8_t v = cnt > amax ? 1 : (cnt < amin ? 0 : cur[col * nzp]);
    for (int k = 0; k < L.nz; ++k) next[col * nzp + k] = v;
    next[col * nzp + L.nz] = 0;
  }
}

__global__ void k_cave_floor_ceil(CaveLattice L) {
  const long long ncol = (long long)L.nx * L.ny;
  const int nzp = L.nz + 1;
  for (long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x; col < ncol;
       col += (long long)gridDim.x * blockDim.x) {
    L.cells[col * nzp] = 1;
    L.cells[col * nzp + L.nz] = 1;
  }
}

// ---- regions: union-find with roots linked toward the smaller cell index ----------------
// parent[x] <= x always holds, so every find ends; a union retries only when another thread
// linked one of its roots meanwhile, and gives up (error flag) after kUnionIters tries.

__device__ __forceinline__ int cc_find(int32_t* parent, int x) {
  for (;;) {
    const int p = __ldcg(&parent[x]);
    if (p == x) return x;
    const int g = __ldcg(&parent[p]);
    if (g != p) parent[x] = g;  // path halving; any ancestor is a valid parent
    x = g;
  }
}

__device__ void cc_union(int32_t* parent, int a, int b, unsigned int* err) {
  for (int it = 0; it < kUnionIters; ++it) {
    a = cc_find(parent, a);
    b = cc_find(parent, b);
    if (a == b) return;
    if (a < b) {
      const int t = a;
      a = b;
      b = t;
    }
    if (atomicCAS(&parent[a], a, b) == a) return;
  }
  atomicOr(err, 1u);
}

__global__ void k_cc_init(CaveLattice L, int32_t* parent, uint32_t* size,
                          unsigned long long* min_key, CaveStats* stats) {
  const long long n = cave_cell_count(L);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    stats->n_regions = 0;
    stats->largest = 0;
    stats->best_key = ~0ull;
    stats->error = 0;
  }
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    size[c] = 0;
    min_key[c] = ~0ull;
  }
}

// One thread per column: every on cell is linked to the lowest cell of its vertical run (the
// ceiling joins the run below it only where it is a face neighbour), so runs are depth-1
// trees and the unions below are needed along x and y only.
__global__ void k_cc_columns(CaveLattice L, int32_t* parent) {
  const long long ncol = (long long)L.nx * L.ny;
  const int nzp = L.nz + 1;
  for (long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x; col < ncol;
       col += (long long)gridDim.x * blockDim.x) {
    const long long c0 = col * nzp;
    int bottom = -1;
    for (int k = 0; k < nzp; ++k) {
      const long long c = c0 + k;
      const bool joins = k > 0 && (k < L.nz || L.ceil_adjacent);
      if (!L.cells[c]) {
        parent[c] = -1;
        bottom = -1;
        continue;
      }
      if (bottom < 0 || !joins) bottom = (int)c;
      parent[c] = bottom;
    }
  }
}

__global__ void k_cc_union(CaveLattice L, int32_t* parent, CaveStats* stats) {
  const long long n = cave_cell_count(L);
  const int nzp = L.nz + 1;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    if (!L.cells[c]) continue;
    int i, j, k;
    cell_ijk(L, c, &i, &j, &k);
    // a cell whose run continues below joins a neighbour's run only where that run does not
    // continue below too: otherwise the pair below has joined the same two runs already
    const bool below = k > 0 && (k < L.nz || L.ceil_adjacent) && L.cells[c - 1];
    const long long cx = c + (long long)L.ny * nzp, cy = c + nzp;
    if (i + 1 < L.nx && L.cells[cx] && !(below && L.cells[cx - 1]))
      cc_union(parent, (int)c, (int)cx, &stats->error);
    if (j + 1 < L.ny && L.cells[cy] && !(below && L.cells[cy - 1]))
      cc_union(parent, (int)c, (int)cy, &stats->error);
  }
}

// Region sizes and smallest order keys.  Neighbouring cells mostly share a root, so the lanes
// of a warp with the same root combine their count and key before one lane updates the root.
__global__ void k_cc_flatten(CaveLattice L, int32_t* parent, uint32_t* size,
                             unsigned long long* min_key) {
  const long long n = cave_cell_count(L);
  const long long stride = (long long)gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  for (long long base = (long long)blockIdx.x * blockDim.x; base < n; base += stride) {
    const long long c = base + threadIdx.x;
    const bool on = c < n && L.cells[c];
    int r = -1;
    uint32_t hi = 0xffffffffu, lo = 0xffffffffu;
    if (on) {
      r = cc_find(parent, (int)c);
      int i, j, k, x, y, z;
      cell_ijk(L, c, &i, &j, &k);
      cave_cell_xyz(L, i, j, k, &x, &y, &z);
      const unsigned long long key = vdb_order_key(x, y, z);
      hi = (uint32_t)(key >> 32);
      lo = (uint32_t)key;
    }
    const unsigned peers = __match_any_sync(0xffffffffu, r);
    const uint32_t mhi = __reduce_min_sync(peers, hi);
    const uint32_t mlo = __reduce_min_sync(peers, hi == mhi ? lo : 0xffffffffu);
    if (on && lane == __ffs(peers) - 1) {
      atomicAdd(&size[r], (uint32_t)__popc(peers));
      atomicMin(&min_key[r], ((unsigned long long)mhi << 32) | mlo);
    }
  }
}

// After k_cc_flatten every on cell's parent chain ends at its root; store the root itself.
__global__ void k_cc_roots(CaveLattice L, int32_t* parent, const uint32_t* size,
                           CaveStats* stats) {
  const long long n = cave_cell_count(L);
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    if (!L.cells[c]) continue;
    if (parent[c] == (int)c) {
      atomicAdd(&stats->n_regions, 1u);
      atomicMax(&stats->largest, size[c]);
    } else {
      parent[c] = cc_find(parent, (int)c);
    }
  }
}

__global__ void k_cc_best(CaveLattice L, const int32_t* parent, const uint32_t* size,
                          const unsigned long long* min_key, CaveStats* stats) {
  const long long n = cave_cell_count(L);
  const uint32_t largest = stats->largest;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x)
    if (L.cells[c] && parent[c] == (int)c && size[c] == largest)
      atomicMin(&stats->best_key, min_key[c]);
}

__global__ void k_cave_keep(CaveLattice L, const int32_t* parent,
                            const unsigned long long* min_key, const CaveStats* stats) {
  const long long n = cave_cell_count(L);
  const unsigned long long best = stats->best_key;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x)
    if (L.cells[c]) L.cells[c] = (min_key[parent[c]] == best) ? 1 : 0;
}

// ---- leaves ------------------------------------------------------------------------------

__global__ void k_cave_tiles(CaveLattice L, uint32_t* dense, int3 llo, int3 ldim) {
  const long long n = cave_cell_count(L);
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x) {
    if (!L.cells[c]) continue;
    int i, j, k, x, y, z;
    cell_ijk(L, c, &i, &j, &k);
    cave_cell_xyz(L, i, j, k, &x, &y, &z);
    const long long lx = (x >> 3) - llo.x, ly = (y >> 3) - llo.y, lz = (z >> 3) - llo.z;
    if (lx < 0 || lx >= ldim.x || ly < 0 || ly >= ldim.y || lz < 0 || lz >= ldim.z) continue;
    uint4* w = reinterpret_cast<uint4*>(dense + ((lx * ldim.y + ly) * ldim.z + lz) * 16);
    const uint4 ones = make_uint4(~0u, ~0u, ~0u, ~0u);
    w[0] = ones;
    w[1] = ones;
    w[2] = ones;
    w[3] = ones;
  }
}

// Leaf bits: voxel (x, y, z) of a leaf is bit x*64 + y*8 + z, so x-slice x is the 64-bit word
// x of the leaf with bit y*8 + z.  For each direction, the mask of voxels whose face
// neighbour in that direction is on; dilation ORs them into the slice, erosion ANDs them.
// Two adjacent lanes per leaf, each with four x-slices (h = 0: x 0..3, h = 1: x 4..7): a lane
// loads its half of the leaf and of the four face-neighbour leaves along y and z as 16-byte
// vectors, swaps the middle slices with its partner, and reads the x neighbour's edge slice.
__device__ __forceinline__ void load_half(const ulonglong2* src, long long pos, int h, bool ok,
                                          unsigned long long s[4]) {
  if (ok) {
    const ulonglong2 a = __ldg(&src[pos * 4 + 2 * h]);
    const ulonglong2 b = __ldg(&src[pos * 4 + 2 * h + 1]);
    s[0] = a.x;
    s[1] = a.y;
    s[2] = b.x;
    s[3] = b.y;
  } else {
    s[0] = s[1] = s[2] = s[3] = 0ull;
  }
}

// A pair of lanes walks a run of kMorphRun leaves along x at one (y, z) leaf position: the next
// leaf's half is loaded one step ahead (it is the x+ edge now and this lane's leaf next), and
// the previous leaf's last slice is kept, so only the run's first leaf reads an x neighbour
// from memory.  Leaves next to each other along z and y are walked by neighbouring lanes and
// warps at about the same time, so those loads are served by L1 / L2.
constexpr int kMorphRun = 16;

__global__ void __launch_bounds__(256) k_leaf_morph(const unsigned long long* __restrict__ src,
                                                    unsigned long long* __restrict__ dst,
                                                    int3 ldim, int erode) {
  constexpr unsigned long long kZ0 = 0x0101010101010101ull, kZ7 = 0x8080808080808080ull;
  const long long syz = (long long)ldim.y * ldim.z, sy = ldim.z;
  const long long nseg = (ldim.x + kMorphRun - 1) / kMorphRun;
  const long long n = nseg * syz * 2;
  const ulonglong2* v2 = reinterpret_cast<const ulonglong2*>(src);
  ulonglong2* d2 = reinterpret_cast<ulonglong2*>(dst);
  const long long stride = (long long)gridDim.x * blockDim.x;
  // a warp-uniform loop (and a fixed number of steps per run): the partner exchanges need
  // both lanes of every pair
  for (long long base = (long long)blockIdx.x * blockDim.x; base < n; base += stride) {
    const long long t = base + threadIdx.x;
    const bool live0 = t < n;
    const long long pr = live0 ? (t >> 1) : 0;
    const int h = (int)(t & 1);
    const long long yz = pr % syz;
    const int x0 = (int)(pr / syz) * kMorphRun;
    const int lz = (int)(yz % ldim.z);
    const int ly = (int)(yz / ldim.z);
    unsigned long long s[4];
    load_half(v2, (long long)x0 * syz + yz, h, live0, s);
    // x- edge of the run's first leaf (slice 7 of leaf x0 - 1), needed by h = 0
    unsigned long long prev7 =
        (live0 && h == 0 && x0 > 0) ? __ldg(&src[((long long)(x0 - 1) * syz + yz) * 8 + 7]) : 0ull;
    for (int it = 0; it < kMorphRun; ++it) {
      const int lx = x0 + it;
      const bool live = live0 && lx < ldim.x;
      const long long pos = (long long)lx * syz + yz;
      unsigned long long nx[4], zp[4], zm[4], yp[4], ym[4];
      load_half(v2, pos + syz, h, live && lx + 1 < ldim.x, nx);
      load_half(v2, pos + 1, h, live && lz + 1 < ldim.z, zp);
      load_half(v2, pos - 1, h, live && lz > 0, zm);
      load_half(v2, pos + sy, h, live && ly + 1 < ldim.y, yp);
      load_half(v2, pos - sy, h, live && ly > 0, ym);
      // inner edges: h = 0 needs slice 4 (partner's s[0]), h = 1 slice 3 (partner's s[3])
      const unsigned long long other = __shfl_xor_sync(0xffffffffu, h == 0 ? s[3] : s[0], 1);
      // x+ edge for h = 1: slice 0 of the next leaf, which the h = 0 partner loaded
      const unsigned long long next0 = __shfl_xor_sync(0xffffffffu, nx[0], 1);
      const unsigned long long edge = h == 0 ? prev7 : next0;
      unsigned long long out[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const unsigned long long c = s[i];
        const unsigned long long nzp = ((c >> 1) & ~kZ7) | ((zp[i] << 7) & kZ7);
        const unsigned long long nzm = ((c << 1) & ~kZ0) | ((zm[i] >> 7) & kZ0);
        const unsigned long long nyp = (c >> 8) | (yp[i] << 56);
        const unsigned long long nym = (c << 8) | (ym[i] >> 56);
        const unsigned long long nxp = i < 3 ? s[i + 1] : (h == 0 ? other : edge);
        const unsigned long long nxm = i > 0 ? s[i - 1] : (h == 0 ? edge : other);
        out[i] = erode ? (c & nzp & nzm & nyp & nym & nxp & nxm)
                       : (c | nzp | nzm | nyp | nym | nxp | nxm);
      }
      if (live) {
        d2[pos * 4 + 2 * h] = make_ulonglong2(out[0], out[1]);
        d2[pos * 4 + 2 * h + 1] = make_ulonglong2(out[2], out[3]);
      }
      // the next leaf's x- edge for h = 0 is this leaf's slice 7, held by the h = 1 partner
      prev7 = __shfl_xor_sync(0xffffffffu, s[3], 1);
#pragma unroll
      for (int i = 0; i < 4; ++i) s[i] = nx[i];
    }
  }
}

__global__ void k_leaf_andnot(const unsigned long long* a, const unsigned long long* b,
                              unsigned long long* dst, long long n) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n;
       t += (long long)gridDim.x * blockDim.x)
    dst[t] = a[t] & ~b[t];
}

int grid_for(long long n) {
  const long long g = (n + 255) / 256;
  return (int)(g < 1 ? 1 : (g > kGrid ? kGrid : g));
}

}  // namespace

cudaError_t launch_cave_fill(const CaveLattice& L, uint32_t seed, int pct, int mode_2d,
                             cudaStream_t s) {
  k_cave_fill<<<grid_for(cave_cell_count(L)), 256, 0, s>>>(L, seed, pct, mode_2d);
  return cudaGetLastError();
}

cudaError_t launch_cave_fill_libc(const CaveLattice& L, const uint32_t* mats, int nmats,
                                  const uint32_t* state0, long long n_draws, int pct, int mode_2d,
                                  cudaStream_t s) {
  const long long nchunks = (n_draws + kLibcChunk - 1) / kLibcChunk;
  if (nchunks > 0)
    k_cave_fill_libc<<<grid_for(nchunks), 256, 0, s>>>(L, mats, nmats, state0, n_draws, pct,
                                                       mode_2d);
  return cudaGetLastError();
}

cudaError_t launch_cave_smooth(const CaveLattice& L, const uint8_t* cur, uint8_t* next, int amax,
                               int amin, int mode_2d, uint8_t* scratch, cudaStream_t s) {
  if (mode_2d) {
    k_cave_smooth2d<<<grid_for((long long)L.nx * L.ny), 256, 0, s>>>(L, cur, next, amax, amin);
  } else if (scratch) {
    const int g = grid_for(cave_cell_count(L));
    k_cave_plane_sums<<<g, 256, 0, s>>>(L, cur, scratch);
    k_cave_smooth3d_sums<<<g, 256, 0, s>>>(L, cur, scratch, next, amax, amin);
  } else {
    k_cave_smooth3d<<<grid_for(cave_cell_count(L)), 256, 0, s>>>(L, cur, next, amax, amin);
  }
  return cudaGetLastError();
}

cudaError_t launch_cave_floor_ceil(const CaveLattice& L, cudaStream_t s) {
  k_cave_floor_ceil<<<grid_for((long long)L.nx * L.ny), 256, 0, s>>>(L);
  return cudaGetLastError();
}

cudaError_t launch_cave_regions(const CaveLattice& L, int32_t* parent, uint32_t* size,
                                unsigned long long* min_key, CaveStats* stats, cudaStream_t s) {
  const int g = grid_for(cave_cell_count(L));
  k_cc_init<<<g, 256, 0, s>>>(L, parent, size, min_key, stats);
  k_cc_columns<<<grid_for((long long)L.nx * L.ny), 256, 0, s>>>(L, parent);
  k_cc_union<<<g, 256, 0, s>>>(L, parent, stats);
  k_cc_flatten<<<g, 256, 0, s>>>(L, parent, size, min_key);
  k_cc_roots<<<g, 256, 0, s>>>(L, parent, size, stats);
  k_cc_best<<<g, 256, 0, s>>>(L, parent, size, min_key, stats);
  return cudaGetLastError();
}

cudaError_t launch_cave_keep(const CaveLattice& L, const int32_t* parent,
                             const unsigned long long* min_key, const CaveStats* stats,
                             cudaStream_t s) {
  k_cave_keep<<<grid_for(cave_cell_count(L)), 256, 0, s>>>(L, parent, min_key, stats);
  return cudaGetLastError();
}

cudaError_t launch_cave_tiles(const CaveLattice& L, uint32_t* dense, const int32_t llo[3],
                              const int32_t ldim[3], cudaStream_t s) {
  k_cave_tiles<<<grid_for(cave_cell_count(L)), 256, 0, s>>>(
      L, dense, make_int3(llo[0], llo[1], llo[2]), make_int3(ldim[0], ldim[1], ldim[2]));
  return cudaGetLastError();
}

cudaError_t launch_leaf_morph(const uint32_t* src, uint32_t* dst, const int32_t ldim[3],
                              int erode, cudaStream_t s) {
  const long long n = (long long)((ldim[0] + kMorphRun - 1) / kMorphRun) * ldim[1] * ldim[2] * 2;
  k_leaf_morph<<<grid_for(n), 256, 0, s>>>(reinterpret_cast<const unsigned long long*>(src),
                                           reinterpret_cast<unsigned long long*>(dst),
                                           make_int3(ldim[0], ldim[1], ldim[2]), erode);
  return cudaGetLastError();
}

cudaError_t launch_leaf_andnot(const uint32_t* a, const uint32_t* b, uint32_t* dst, long long n,
                               cudaStream_t s) {
  k_leaf_andnot<<<grid_for(n * 8), 256, 0, s>>>(reinterpret_cast<const unsigned long long*>(a),
                                                reinterpret_cast<const unsigned long long*>(b),
                                                reinterpret_cast<unsigned long long*>(dst), n * 8);
  return cudaGetLastError();
}

}  // namespace nm
