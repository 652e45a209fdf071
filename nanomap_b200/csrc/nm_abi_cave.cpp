// nm_abi_cave.cpp -- C ABI of the procedural cave generator (replaces
// nanomap::mapgen::CaveGen, CaveGen.h:32-68 / CaveGen.cpp).
//
// The cell lattice stays on the device between stages.  The reference's fill draws
// rand() % 100 per cell after srand(seed) in x, y, z loop order (CaveGen.cpp:31-42, 66-79).
// The C library's generator (glibc's default, a 128-byte state) is the additive feedback
// generator r[i] = r[i-31] + r[i-3] mod 2^32 with output r[i] >> 1, seeded by
// r[0] = seed (1 for 0), r[i] = 16807 r[i-1] mod (2^31 - 1) for i < 31, r[i] = r[i-31] for
// i < 34, and 310 discarded draws.  It is linear, so the device draws it in parallel: the host
// seeds it, checks its first draws against the C library's own reentrant generator
// (initstate_r / random_r, which leaves the caller's rand() state alone) and builds jump
// matrices; each device thread jumps to its chunk.  NM_CAVE_COUNTER_RNG fills from a
// counter-based generator instead.  Every later stage runs on the device; the result is a
// device sim map.
#include <algorithm>
#include <array>
#include <cfenv>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "nm_cave.h"
#include "nm_objects.h"

using nm::fail;

struct nm_cave_s {
  std::atomic<int> refs{1};
  nm_context ctx = nullptr;
  nm_cave_desc desc{};
  nm::CaveLattice L{};
  uint8_t* d_cells[2] = {nullptr, nullptr};
  int cur = 0;
  int32_t* d_parent = nullptr;
  uint32_t* d_size = nullptr;
  unsigned long long* d_min_key = nullptr;
  nm::CaveStats* d_stats = nullptr;
  bool regions_valid = false;  // the region labels describe the current cells
  nm::CaveStats stats{};
  // scratch kept between calls: the shell's three leaf-box buffers and the fill's jump
  // matrices (grown on demand, freed with the cave)
  uint32_t* shell_buf[3] = {nullptr, nullptr, nullptr};
  size_t shell_bytes[3] = {0, 0, 0};
  uint32_t* fill_buf = nullptr;
  size_t fill_bytes = 0;
};

namespace nm {
void release(nm_cave c) {
  if (!c || c->refs.fetch_sub(1, std::memory_order_acq_rel) != 1) return;
  nm_context ctx = c->ctx;
  cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  cudaFree(c->d_cells[0]);
  cudaFree(c->d_cells[1]);
  cudaFree(c->d_parent);
  cudaFree(c->d_size);
  cudaFree(c->d_min_key);
  cudaFree(c->d_stats);
  for (int i = 0; i < 3; ++i) cudaFree(c->shell_buf[i]);
  cudaFree(c->fill_buf);
  delete c;
  release(ctx);
}
}  // namespace nm

namespace {

int floor_div8(int v) { return v >> 3; }  // arithmetic shift: floor for negatives

// CaveGen::populateMap's dimensions (CaveGen.cpp:17-30): ceil(size / res) voxels, halved
// rounding up, evaluated in double under round-to-nearest.
int lattice_from_desc(const nm_cave_desc& d, nm::CaveLattice* L) {
  const int saved = std::fegetround();
  std::fesetround(FE_TONEAREST);
  double full[3];
  for (int a = 0; a < 3; ++a) full[a] = std::ceil(d.map_size[a] / d.grid_res);
  std::fesetround(saved);
  for (int a = 0; a < 3; ++a) {
    if (!(full[a] >= 1.0) || full[a] > (double)(1 << 21))
      return fail(NM_ERR_ARG, "map_size / grid_res on axis %d gives %g voxels (1 .. 2^21)", a,
                  full[a]);
    const int n = (int)full[a];
    L->half[a] = (n % 2 != 0) ? (n + 1) / 2 : n / 2;
  }
  const int Dx = L->half[0], Dy = L->half[1], Dz = L->half[2];
  L->nx = (2 * Dx - 16 > 0) ? (2 * Dx - 16 + 7) / 8 : 0;
  L->ny = (2 * Dy - 16 > 0) ? (2 * Dy - 16 + 7) / 8 : 0;
  L->nz = (2 * Dz + 7) / 8;
  L->kf = (2 * Dz - 8 > 0) ? (2 * Dz - 8 + 7) / 8 : 0;
  L->ceil_adjacent = ((2 * Dz) % 8 == 0) ? 1 : 0;
  const long long n = nm::cave_cell_count(*L);
  if (n >= (1ll << 31)) return fail(NM_ERR_CAPACITY, "cave lattice has %lld cells", n);
  return NM_OK;
}

nm::CaveLattice current(nm_cave c) {
  nm::CaveLattice L = c->L;
  L.cells = c->d_cells[c->cur];
  return L;
}

// Leaf box of the cells' leaves, widened by `margin` leaves on every side.
void cave_leaf_box(const nm::CaveLattice& L, int margin, int32_t llo[3], int32_t ldim[3]) {
  int lo[3], hi[3];
  nm::cave_cell_xyz(L, 0, 0, 0, &lo[0], &lo[1], &lo[2]);
  nm::cave_cell_xyz(L, std::max(L.nx - 1, 0), std::max(L.ny - 1, 0), L.nz, &hi[0], &hi[1],
                    &hi[2]);
  for (int a = 0; a < 3; ++a) {
    llo[a] = floor_div8(lo[a]) - margin;
    ldim[a] = floor_div8(hi[a]) + margin - llo[a] + 1;
  }
}

// Grow a scratch buffer to at least `bytes` (contents not kept).
cudaError_t grow(uint32_t** buf, size_t* have, size_t bytes) {
  if (*buf && *have >= bytes) return cudaSuccess;
  cudaFree(*buf);
  *buf = nullptr;
  *have = 0;
  const cudaError_t e = cudaMalloc((void**)buf, bytes);
  if (e == cudaSuccess) *have = bytes;
  return e;
}

int build_cave_simmap(nm_cave c, int shell, int half_width, int closing, nm_simmap* out) {
  if (!c || !out) return fail(NM_ERR_ARG, "null argument");
  *out = nullptr;
  if (shell && (half_width < 1 || half_width > 64 || closing < 0 || closing > 64))
    return fail(NM_ERR_ARG, "half_width must be in [1, 64] and closing in [0, 64]");
  nm_context ctx = c->ctx;
  NM_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const int reach = shell ? closing + half_width : 0;
  int32_t llo[3], ldim[3], vmin[3], vmax[3];
  cave_leaf_box(c->L, reach / 8 + 1, llo, ldim);
  long long nleaf = 1;
  for (int a = 0; a < 3; ++a) {
    vmin[a] = llo[a] * 8;
    vmax[a] = (llo[a] + ldim[a]) * 8;
    nleaf *= ldim[a];
  }
  if (nleaf > (1ll << 32)) return fail(NM_ERR_CAPACITY, "cave leaf box has %lld leaves", nleaf);
  // the tiles need one leaf-box buffer, the shell three
  const size_t bytes = (size_t)nleaf * 64;
  for (int i = 0; i < (shell ? 3 : 1); ++i) {
    const cudaError_t e = grow(&c->shell_buf[i], &c->shell_bytes[i], bytes);
    if (e != cudaSuccess)
      return fail(NM_ERR_CUDA, "cave shell buffers (%lld leaves): %s", nleaf,
                  cudaGetErrorString(e));
  }
  uint32_t* buf[3] = {c->shell_buf[0], c->shell_buf[1], c->shell_buf[2]};
  std::unique_ptr<nm_simmap_s> sm(new nm_simmap_s());
  sm->ctx = ctx;
  nm::SimBuild b{};
  int rc = nm::begin_build((float)c->desc.grid_res, vmin, vmax, &b, s, buf[0]);
  if (rc != NM_OK) return rc;
  NM_CUDA(nm::launch_cave_tiles(current(c), b.dense, b.llo, b.ldim, s));
  if (shell) {
    // closing: M = erode^c(dilate^c(T)), ping-pong between buf[0] and buf[1]; 2c steps end
    // in buf[0]
    int m = 0;
    for (int i = 0; i < 2 * closing; ++i) {
      NM_CUDA(nm::launch_leaf_morph(buf[m], buf[1 - m], b.ldim, i >= closing, s));
      m = 1 - m;
    }
    // E = erode^h(M) into buf[1] / buf[2]; D = dilate^h(M) through the buffer E left free
    // and buf[0] (M is not needed after D's first step); band = D & ~E
    int e_buf = 1;
    for (int i = 0; i < half_width; ++i) {
      const int src = (i == 0) ? 0 : e_buf;
      const int dst = (i == 0) ? 1 : 3 - e_buf;
      NM_CUDA(nm::launch_leaf_morph(buf[src], buf[dst], b.ldim, 1, s));
      e_buf = dst;
    }
    const int free_buf = 3 - e_buf;
    int d_buf = 0;
    for (int i = 0; i < half_width; ++i) {
      const int dst = (d_buf == 0) ? free_buf : 0;
      NM_CUDA(nm::launch_leaf_morph(buf[d_buf], buf[dst], b.ldim, 0, s));
      d_buf = dst;
    }
    NM_CUDA(nm::launch_leaf_andnot(buf[d_buf], buf[e_buf], buf[d_buf], nleaf, s));
    b.dense = buf[d_buf];  // still borrowed: the build compacts it and leaves it to the cave
  }
  rc = nm::finish_build(ctx, b, sm.get(), s);
  if (rc != NM_OK) return rc;
  nm::retain(ctx);
  *out = sm.release();
  return NM_OK;
}

// Seeded state of the C library generator: the 31 words before the first draw.
void libc_state(uint32_t seed, uint32_t state[31]) {
  int32_t r[344];
  r[0] = (int32_t)(seed == 0 ? 1u : seed);
  for (int i = 1; i < 31; ++i) {
    long long v = (16807LL * r[i - 1]) % 2147483647LL;
    if (v < 0) v += 2147483647LL;
    r[i] = (int32_t)v;
  }
  for (int i = 31; i < 34; ++i) r[i] = r[i - 31];
  for (int i = 34; i < 344; ++i) r[i] = (int32_t)((uint32_t)r[i - 31] + (uint32_t)r[i - 3]);
  for (int q = 0; q < 31; ++q) state[q] = (uint32_t)r[313 + q];
}

// The first draws from `state` must equal the C library's for this seed.
bool libc_state_matches(uint32_t seed, const uint32_t state[31]) {
  struct random_data rd;
  std::memset(&rd, 0, sizeof(rd));
  alignas(8) char buf[128];
  std::memset(buf, 0, sizeof(buf));
  if (initstate_r(seed, buf, sizeof(buf), &rd) != 0) return false;
  std::vector<uint32_t> r(state, state + 31);
  for (int k = 0; k < 200; ++k) {
    const uint32_t v = r[r.size() - 31] + r[r.size() - 3];
    r.push_back(v);
    int32_t want = 0;
    random_r(&rd, &want);
    if ((int32_t)(v >> 1) != want) return false;
  }
  return true;
}

using Mat31 = std::array<uint32_t, 961>;

Mat31 mat_mul(const Mat31& X, const Mat31& Y) {
  Mat31 Z{};
  for (int a = 0; a < 31; ++a)
    for (int c = 0; c < 31; ++c) {
      const uint32_t x = X[a * 31 + c];
      if (!x) continue;
      for (int b = 0; b < 31; ++b) Z[a * 31 + b] += x * Y[c * 31 + b];
    }
  return Z;
}

// A^(kLibcChunk * 2^j) for j < n, A the one-draw step of the state (r[i-31] .. r[i-1]).
std::vector<uint32_t> libc_jump_mats(int n) {
  Mat31 A{};
  for (int m = 0; m < 30; ++m) A[m * 31 + m + 1] = 1u;
  A[30 * 31 + 0] = 1u;
  A[30 * 31 + 28] = 1u;
  Mat31 P{}, B = A;
  for (int q = 0; q < 31; ++q) P[q * 31 + q] = 1u;
  for (int e = nm::kLibcChunk; e > 0; e >>= 1) {
    if (e & 1) P = mat_mul(P, B);
    B = mat_mul(B, B);
  }
  std::vector<uint32_t> out((size_t)n * 961);
  for (int j = 0; j < n; ++j) {
    std::copy(P.begin(), P.end(), out.begin() + (size_t)j * 961);
    P = mat_mul(P, P);
  }
  return out;
}

int check_cave(nm_cave c) {
  if (!c) return fail(NM_ERR_ARG, "cave is null");
  NM_CUDA(cudaSetDevice(c->ctx->device));
  return NM_OK;
}

int run_regions(nm_cave c, nm::CaveStats* st) {
  if (c->regions_valid) {
    *st = c->stats;
    return NM_OK;
  }
  cudaStream_t s = c->ctx->stream;
  NM_CUDA(nm::launch_cave_regions(current(c), c->d_parent, c->d_size, c->d_min_key, c->d_stats,
                                  s));
  NM_CUDA(cudaMemcpyAsync(st, c->d_stats, sizeof(*st), cudaMemcpyDeviceToHost, s));
  NM_CUDA(cudaStreamSynchronize(s));
  if (st->error) return fail(NM_ERR_TIMEOUT, "cave regions: a union gave up after its limit");
  c->stats = *st;
  c->regions_valid = true;
  return NM_OK;
}

}  // namespace

extern "C" {

int nm_cave_create(nm_context ctx, const nm_cave_desc* desc, nm_cave* out) {
  if (!ctx || !desc || !out) return fail(NM_ERR_ARG, "null argument");
  *out = nullptr;
  if (!(desc->grid_res > 0.0) || !std::isfinite(desc->grid_res))
    return fail(NM_ERR_ARG, "grid_res must be positive");
  for (int a = 0; a < 3; ++a)
    if (!(desc->map_size[a] > 0.0) || !std::isfinite(desc->map_size[a]))
      return fail(NM_ERR_ARG, "map_size must be positive");
  if (desc->smoothing_count < 0 || desc->smoothing_count > 1000000)
    return fail(NM_ERR_ARG, "smoothing_count out of range");
  nm::CaveLattice L{};
  int rc = lattice_from_desc(*desc, &L);
  if (rc != NM_OK) return rc;
  NM_CUDA(cudaSetDevice(ctx->device));
  nm_cave c = new nm_cave_s();
  c->ctx = nm::retain(ctx);
  c->desc = *desc;
  c->desc.file_out[sizeof(c->desc.file_out) - 1] = '\0';
  c->L = L;
  const long long n = std::max<long long>(nm::cave_cell_count(L), 1);
  cudaError_t e = cudaMalloc((void**)&c->d_cells[0], (size_t)n);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_cells[1], (size_t)n);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_parent, (size_t)n * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_size, (size_t)n * 4);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_min_key, (size_t)n * 8);
  if (e == cudaSuccess) e = cudaMalloc((void**)&c->d_stats, sizeof(nm::CaveStats));
  if (e == cudaSuccess) e = cudaMemsetAsync(c->d_cells[0], 0, (size_t)n, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    nm::release(c);  // frees what was allocated and the context reference
    return fail(NM_ERR_CUDA, "cave buffers (%lld cells): %s", n, cudaGetErrorString(e));
  }
  *out = c;
  return NM_OK;
}

int nm_cave_destroy(nm_cave c) {
  nm::release(c);
  return NM_OK;
}

int nm_cave_dims(nm_cave c, int32_t half[3], int32_t cells[3]) {
  if (!c) return fail(NM_ERR_ARG, "cave is null");
  if (half)
    for (int a = 0; a < 3; ++a) half[a] = c->L.half[a];
  if (cells) {
    cells[0] = c->L.nx;
    cells[1] = c->L.ny;
    cells[2] = c->L.nz;
  }
  return NM_OK;
}

int nm_cave_populate(nm_cave c, uint32_t flags) {
  int rc = check_cave(c);
  if (rc != NM_OK) return rc;
  c->regions_valid = false;
  cudaStream_t s = c->ctx->stream;
  const int mode_2d = (flags & NM_CAVE_2D) ? 1 : 0;
  c->cur = 0;
  const nm::CaveLattice L = current(c);
  if (flags & NM_CAVE_COUNTER_RNG) {
    NM_CUDA(nm::launch_cave_fill(L, c->desc.seed, c->desc.fill_percentage, mode_2d, s));
    NM_CUDA(cudaStreamSynchronize(s));
    return NM_OK;
  }
  const long long n = nm::cave_cell_count(L);
  const long long n_draws = mode_2d ? (long long)L.nx * L.ny
                                    : (L.kf > 1 ? (long long)L.nx * L.ny * (L.kf - 1) : 0);
  uint32_t state[31];
  libc_state(c->desc.seed, state);
  if (!libc_state_matches(c->desc.seed, state))
    return fail(NM_ERR_UNSUPPORTED,
                "the C library's rand() sequence is not the additive feedback generator this "
                "fill reproduces; use NM_CAVE_COUNTER_RNG");
  NM_CUDA(cudaMemsetAsync(L.cells, 0, (size_t)std::max<long long>(n, 1), s));
  if (n_draws > 0) {
    const long long nchunks = (n_draws + nm::kLibcChunk - 1) / nm::kLibcChunk;
    int nmats = 1;
    while ((1ll << nmats) < nchunks) ++nmats;
    const std::vector<uint32_t> mats = libc_jump_mats(nmats);
    cudaError_t e = grow(&c->fill_buf, &c->fill_bytes, (mats.size() + 31) * 4);
    uint32_t* d_buf = c->fill_buf;
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_buf, mats.data(), mats.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_buf + mats.size(), state, 31 * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = nm::launch_cave_fill_libc(L, d_buf, nmats, d_buf + mats.size(), n_draws,
                                    c->desc.fill_percentage, mode_2d, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return fail(NM_ERR_CUDA, "cave fill: %s", cudaGetErrorString(e));
  }
  NM_CUDA(cudaStreamSynchronize(s));
  return NM_OK;
}

int nm_cave_smooth(nm_cave c, uint32_t flags) {
  int rc = check_cave(c);
  if (rc != NM_OK) return rc;
  c->regions_valid = false;
  cudaStream_t s = c->ctx->stream;
  const int mode_2d = (flags & NM_CAVE_2D) ? 1 : 0;
  for (int it = 0; it < c->desc.smoothing_count; ++it) {
    const nm::CaveLattice L = current(c);
    // the region labels' buffer (4 bytes per cell) is free while the cells change
    NM_CUDA(nm::launch_cave_smooth(L, L.cells, c->d_cells[1 - c->cur], c->desc.active_max,
                                   c->desc.active_min, mode_2d,
                                   reinterpret_cast<uint8_t*>(c->d_parent), s));
    c->cur = 1 - c->cur;
  }
  NM_CUDA(cudaStreamSynchronize(s));
  return NM_OK;
}

int nm_cave_floor_ceil(nm_cave c) {
  int rc = check_cave(c);
  if (rc != NM_OK) return rc;
  c->regions_valid = false;
  NM_CUDA(nm::launch_cave_floor_ceil(current(c), c->ctx->stream));
  NM_CUDA(cudaStreamSynchronize(c->ctx->stream));
  return NM_OK;
}

int nm_cave_regions(nm_cave c, int64_t* n_regions, int64_t* largest) {
  int rc = check_cave(c);
  if (rc != NM_OK) return rc;
  nm::CaveStats st{};
  rc = run_regions(c, &st);
  if (rc != NM_OK) return rc;
  if (n_regions) *n_regions = st.n_regions;
  if (largest) *largest = st.largest;
  return NM_OK;
}

int nm_cave_keep_largest(nm_cave c) {
  int rc = check_cave(c);
  if (rc != NM_OK) return rc;
  nm::CaveStats st{};
  rc = run_regions(c, &st);
  if (rc != NM_OK) return rc;
  c->regions_valid = false;
  NM_CUDA(nm::launch_cave_keep(current(c), c->d_parent, c->d_min_key, c->d_stats,
                               c->ctx->stream));
  NM_CUDA(cudaStreamSynchronize(c->ctx->stream));
  return NM_OK;
}

int nm_cave_cells(nm_cave c, int32_t* xyz, int64_t max_cells, int64_t* n) {
  int rc = check_cave(c);
  if (rc != NM_OK) return rc;
  if (!n || (max_cells > 0 && !xyz)) return fail(NM_ERR_ARG, "null argument");
  const nm::CaveLattice L = current(c);
  const long long total = nm::cave_cell_count(L);
  std::vector<uint8_t> cells((size_t)std::max<long long>(total, 1));
  if (total > 0) NM_CUDA(cudaMemcpy(cells.data(), L.cells, (size_t)total, cudaMemcpyDeviceToHost));
  std::vector<std::pair<unsigned long long, std::array<int32_t, 3>>> on;
  const int nzp = L.nz + 1;
  for (long long idx = 0; idx < total; ++idx) {
    if (!cells[(size_t)idx]) continue;
    const int k = (int)(idx % nzp), j = (int)((idx / nzp) % L.ny), i = (int)(idx / nzp / L.ny);
    int x, y, z;
    nm::cave_cell_xyz(L, i, j, k, &x, &y, &z);
    on.push_back({nm::vdb_order_key(x, y, z), {x, y, z}});
  }
  std::sort(on.begin(), on.end(),
            [](const auto& a, const auto& b) { return a.first < b.first; });
  *n = (int64_t)on.size();
  const size_t m = std::min<size_t>(on.size(), (size_t)std::max<int64_t>(max_cells, 0));
  for (size_t q = 0; q < m; ++q)
    for (int a = 0; a < 3; ++a) xyz[3 * q + a] = on[q].second[a];
  return NM_OK;
}

int nm_cave_simmap(nm_cave c, int32_t shell, int32_t half_width, int32_t closing,
                   nm_simmap* out) {
  return build_cave_simmap(c, shell, half_width, closing, out);
}

int nm_cave_save(nm_cave c, int32_t shell, int32_t half_width, int32_t closing,
                 const char* path, char* written_path) {
  if (!c || !path) return fail(NM_ERR_ARG, "null argument");
  const std::string name(path);
  if (name.size() >= 512) return fail(NM_ERR_ARG, "output path too long");
  const bool vdb = name.size() >= 4 && name.compare(name.size() - 4, 4, ".vdb") == 0;
  nm_simmap sm = nullptr;
  int rc = build_cave_simmap(c, shell, half_width, closing, &sm);
  if (rc != NM_OK) return rc;
  uint64_t nleaves = 0;
  nm_simmap_info(sm, nullptr, nullptr, &nleaves);
  std::vector<int32_t> origins((size_t)nleaves * 3 + 3);
  std::vector<uint32_t> words((size_t)nleaves * 16 + 16);
  uint64_t got = 0;
  rc = nm_simmap_export(sm, origins.data(), words.data(), nleaves, &got);
  nm::release(sm);
  if (rc != NM_OK) return rc;
  std::vector<int32_t> ijk;
  for (uint64_t q = 0; q < got; ++q)
    for (int l = 0; l < 512; ++l)
      if (words[q * 16 + (l >> 5)] >> (l & 31) & 1u) {
        ijk.push_back(origins[3 * q] + (l >> 6));
        ijk.push_back(origins[3 * q + 1] + ((l >> 3) & 7));
        ijk.push_back(origins[3 * q + 2] + (l & 7));
      }
  if (vdb) {
    rc = nm_vdb_write_active_voxels(name.c_str(), "grid", c->desc.grid_res, ijk.data(),
                                    (int64_t)(ijk.size() / 3));
    if (rc != NM_OK) return rc;
    if (written_path) std::snprintf(written_path, 512, "%s", name.c_str());
    return NM_OK;
  }
  FILE* f = std::fopen(name.c_str(), "wb");
  if (!f) return fail(NM_ERR_IO, "cannot write '%s'", name.c_str());
  const char magic[8] = {'N', 'M', 'S', 'I', 'M', 'v', '1', '\0'};
  const float res = (float)c->desc.grid_res;
  const int64_t count = (int64_t)(ijk.size() / 3);
  bool ok = std::fwrite(magic, 1, 8, f) == 8 && std::fwrite(&res, 4, 1, f) == 1 &&
            std::fwrite(&count, 8, 1, f) == 1 &&
            (count == 0 || std::fwrite(ijk.data(), 12, (size_t)count, f) == (size_t)count);
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return fail(NM_ERR_IO, "short write to '%s'", name.c_str());
  if (written_path) std::snprintf(written_path, 512, "%s", name.c_str());
  return NM_OK;
}

}  // extern "C"
