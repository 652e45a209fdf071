// nm_cave.h -- procedural cave lattice shared by the host code and the sm_100a kernels.
//
// The cave generator of the reference (CaveGen.cpp) works on cells 8 voxels apart: with
// D = half sizes in voxels, cell (i, j, k) is voxel (-Dx + 8 + 8i, -Dy + 8 + 8j, -Dz + 8k)
// for k < nz, and plane k = nz is the ceiling z = +Dz of setFloorAndCeil (8 voxels above
// plane nz - 1 only when 2·Dz is a multiple of 8).  Cells are one byte, z fastest.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace nm {

struct CaveLattice {
  int32_t half[3];        // Dx, Dy, Dz
  int32_t nx, ny, nz;     // cells along x, y; planes below the ceiling
  int32_t kf;             // 3-D fill planes: k in [1, kf)
  int32_t ceil_adjacent;  // the ceiling plane is a face neighbour of plane nz - 1
  uint8_t* cells;         // nx * ny * (nz + 1)
};

__host__ __device__ inline long long cave_cell_count(const CaveLattice& L) {
  return (long long)L.nx * L.ny * (L.nz + 1);
}

__host__ __device__ inline void cave_cell_xyz(const CaveLattice& L, int i, int j, int k, int* x,
                                              int* y, int* z) {
  *x = -L.half[0] + 8 + 8 * i;
  *y = -L.half[1] + 8 + 8 * j;
  *z = k < L.nz ? -L.half[2] + 8 * k : L.half[2];
}

// Position of a voxel in OpenVDB's value order for a 5-4-3 tree (root table ordered by
// coordinate, then child index, x-major, at each level): root key fields (c >> 12) with an
// offset of 256 (coordinates inside +-2^20), then the 32^3, 16^3 and 8^3 child indices.
__host__ __device__ inline unsigned long long vdb_order_key(int x, int y, int z) {
  unsigned long long k = (unsigned long long)((x >> 12) + 256);
  k = (k << 9) | (unsigned long long)((y >> 12) + 256);
  k = (k << 9) | (unsigned long long)((z >> 12) + 256);
  k = (k << 5) | (unsigned long long)((x >> 7) & 31);
  k = (k << 5) | (unsigned long long)((y >> 7) & 31);
  k = (k << 5) | (unsigned long long)((z >> 7) & 31);
  k = (k << 4) | (unsigned long long)((x >> 3) & 15);
  k = (k << 4) | (unsigned long long)((y >> 3) & 15);
  k = (k << 4) | (unsigned long long)((z >> 3) & 15);
  k = (k << 3) | (unsigned long long)(x & 7);
  k = (k << 3) | (unsigned long long)(y & 7);
  k = (k << 3) | (unsigned long long)(z & 7);
  return k;
}

// Region statistics of the union-find pass.
struct CaveStats {
  unsigned int n_regions;
  unsigned int largest;
  unsigned long long best_key;  // smallest order key among the largest regions
  unsigned int error;           // a union gave up after its iteration limit
  unsigned int pad;
};

cudaError_t launch_cave_fill(const CaveLattice& L, uint32_t seed, int pct, int mode_2d,
                             cudaStream_t s);
// The C library's rand() sequence as the reference's fill draws it, generated on the device:
// an additive feedback generator r[i] = r[i-31] + r[i-3] (mod 2^32), output r[i] >> 1.
// Thread t starts from state0 (the 31 words before the first draw) advanced by
// kLibcChunk * t draws with the jump matrices mats[j] = A^(kLibcChunk * 2^j) (31 x 31, row
// major) for the set bits j of t, and makes draws [t * kLibcChunk, (t + 1) * kLibcChunk).
constexpr int kLibcChunk = 31 * 32;
cudaError_t launch_cave_fill_libc(const CaveLattice& L, const uint32_t* mats, int nmats,
                                  const uint32_t* state0, long long n_draws, int pct, int mode_2d,
                                  cudaStream_t s);
// One smoothing step; `scratch` (one byte per cell, may be null) holds the in-plane sums of
// the two-pass 3-D form.
cudaError_t launch_cave_smooth(const CaveLattice& L, const uint8_t* cur, uint8_t* next, int amax,
                               int amin, int mode_2d, uint8_t* scratch, cudaStream_t s);
cudaError_t launch_cave_floor_ceil(const CaveLattice& L, cudaStream_t s);
// Regions: labels (one int per cell), sizes and minimum order keys per root, statistics.
cudaError_t launch_cave_regions(const CaveLattice& L, int32_t* parent, uint32_t* size,
                                unsigned long long* min_key, CaveStats* stats, cudaStream_t s);
cudaError_t launch_cave_keep(const CaveLattice& L, const int32_t* parent,
                             const unsigned long long* min_key, const CaveStats* stats,
                             cudaStream_t s);
// Leaves of the on cells into a dense leaf-box bit buffer (16 words per leaf, x*64+y*8+z).
cudaError_t launch_cave_tiles(const CaveLattice& L, uint32_t* dense, const int32_t llo[3],
                              const int32_t ldim[3], cudaStream_t s);
// One face-neighbour dilation (erode = 0) or erosion (erode = 1) of a leaf-box bit buffer;
// voxels outside the box are off.
cudaError_t launch_leaf_morph(const uint32_t* src, uint32_t* dst, const int32_t ldim[3],
                              int erode, cudaStream_t s);
// dst = a & ~b over n leaves (dst may alias a).
cudaError_t launch_leaf_andnot(const uint32_t* a, const uint32_t* b, uint32_t* dst, long long n,
                               cudaStream_t s);

}  // namespace nm
