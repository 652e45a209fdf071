// nm_abi_sim.cpp -- C ABI of the simulation map: build, info, export, render, sensor noise.
//
// Replaces SimHandler's sim-grid upload (SimHandler.cpp:22-23: openToNanoVDB + deviceUpload)
// and the generateCloud launcher (generateCloud.cu:84-94).
#include <algorithm>
#include <climits>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "nm_host.h"
#include "nm_objects.h"

using nm::begin_build;
using nm::fail;
using nm::finish_build;

namespace {

int floor_div(int v, int d) { return (v >= 0) ? v / d : -((-v + d - 1) / d); }

}  // namespace

namespace nm {

// Shared tail of the builders: compact the dense leaf buffer into the sparse view.
int finish_build(nm_context ctx, nm::SimBuild& b, nm_simmap sm, cudaStream_t s) {
  nm::SimMapView& v = sm->view;
  v.res = b.res;
  for (int a = 0; a < 3; ++a) {
    v.llo[a] = b.llo[a];
    v.ldim[a] = b.ldim[a];
    v.blo[a] = floor_div(b.llo[a], 8);
    v.bdim[a] = floor_div(b.llo[a] + b.ldim[a] - 1, 8) - v.blo[a] + 1;
  }
  uint32_t* d_count = nullptr;
  int32_t* d_bbox = nullptr;
  unsigned long long* d_nvox = nullptr;
  const long long bprod = (long long)v.bdim[0] * v.bdim[1] * v.bdim[2];
  NM_CUDA(cudaMalloc((void**)&d_count, 4));
  NM_CUDA(cudaMalloc((void**)&d_bbox, 24));
  NM_CUDA(cudaMalloc((void**)&d_nvox, 8));
  NM_CUDA(cudaMalloc((void**)&v.brick_index, (size_t)bprod * 4));
  NM_CUDA(cudaMemsetAsync(v.brick_index, 0, (size_t)bprod * 4, s));
  NM_CUDA(cudaMemsetAsync(d_count, 0, 4, s));
  NM_CUDA(nm::launch_compact(b, v, d_count, 0, d_bbox, d_nvox, s));
  uint32_t nleaves = 0;
  std::vector<int32_t> bricks((size_t)bprod);
  NM_CUDA(cudaMemcpyAsync(&nleaves, d_count, 4, cudaMemcpyDeviceToHost, s));
  NM_CUDA(cudaMemcpyAsync(bricks.data(), v.brick_index, (size_t)bprod * 4, cudaMemcpyDeviceToHost, s));
  NM_CUDA(cudaStreamSynchronize(s));
  // number the flagged bricks in brick-box order; the others are empty (-1)
  int32_t nblocks = 0;
  for (int32_t& x : bricks) x = x ? nblocks++ : -1;
  NM_CUDA(cudaMemcpyAsync(v.brick_index, bricks.data(), (size_t)bprod * 4, cudaMemcpyHostToDevice, s));
  NM_CUDA(cudaMalloc((void**)&v.brick_leaves, (size_t)std::max(nblocks, 1) * 512 * 4));
  NM_CUDA(nm::launch_fill_i32(v.brick_leaves, (long long)std::max(nblocks, 1) * 512, -1, s));
  NM_CUDA(cudaMalloc((void**)&v.leaf_words, (size_t)std::max<uint32_t>(nleaves, 1) * 64));
  sm->bricks = (uint64_t)nblocks;
  const int32_t init[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MIN, INT_MIN, INT_MIN};
  NM_CUDA(cudaMemcpyAsync(d_bbox, init, 24, cudaMemcpyHostToDevice, s));
  NM_CUDA(cudaMemsetAsync(d_nvox, 0, 8, s));
  NM_CUDA(cudaMemsetAsync(d_count, 0, 4, s));
  NM_CUDA(nm::launch_compact(b, v, d_count, 1, d_bbox, d_nvox, s));
  // empty-space distances for the render (one byte per leaf of the leaf box, twice)
  const size_t lprod = (size_t)b.ldim[0] * b.ldim[1] * b.ldim[2];
  uint8_t* d_dist = nullptr;
  NM_CUDA(cudaMalloc((void**)&d_dist, 2 * lprod));
  const cudaError_t de = nm::launch_skip_distances(b, v, d_dist, d_dist + lprod, s);
  if (de != cudaSuccess) {
    cudaFree(d_dist);
    return fail(NM_ERR_CUDA, "sim map distances: %s", cudaGetErrorString(de));
  }
  unsigned long long nvox = 0;
  NM_CUDA(cudaMemcpyAsync(sm->bbox, d_bbox, 24, cudaMemcpyDeviceToHost, s));
  NM_CUDA(cudaMemcpyAsync(&nvox, d_nvox, 8, cudaMemcpyDeviceToHost, s));
  NM_CUDA(cudaStreamSynchronize(s));
  cudaFree(d_count);
  cudaFree(d_bbox);
  cudaFree(d_nvox);
  cudaFree(d_dist);
  if (!b.borrowed) cudaFree(b.dense);
  b.dense = nullptr;
  sm->leaves = nleaves;
  sm->active_voxels = nvox;
  v.any = nvox > 0 ? 1 : 0;
  if (!v.any)
    for (int a = 0; a < 3; ++a) {
      sm->bbox[a] = 0;
      sm->bbox[3 + a] = -1;
    }
  for (int a = 0; a < 3; ++a) {
    v.box_lo[a] = (float)sm->bbox[a];
    v.box_hi[a] = (float)(sm->bbox[3 + a] + 1);
  }
  (void)ctx;
  return NM_OK;
}

int begin_build(float res, const int32_t vmin[3], const int32_t vmax[3], nm::SimBuild* b,
                cudaStream_t s, uint32_t* buffer) {
  b->res = res;
  long long prod = 1;
  for (int a = 0; a < 3; ++a) {
    if (vmax[a] <= vmin[a]) return fail(NM_ERR_ARG, "empty voxel region on axis %d", a);
    if (vmin[a] < -(1 << 23) || vmax[a] > (1 << 23))
      return fail(NM_ERR_ARG, "voxel region exceeds +-%d voxels", 1 << 23);
    b->vmin[a] = vmin[a];
    b->vmax[a] = vmax[a];
    b->llo[a] = floor_div(vmin[a], 8);
    b->ldim[a] = floor_div(vmax[a] - 1, 8) - b->llo[a] + 1;
    prod *= b->ldim[a];
  }
  if (prod > (1ll << 32)) return fail(NM_ERR_CAPACITY, "voxel region has %lld leaves", prod);
  b->dense = buffer;
  b->borrowed = buffer ? 1 : 0;
  if (!buffer) NM_CUDA(cudaMalloc((void**)&b->dense, (size_t)prod * 64));
  NM_CUDA(cudaMemsetAsync(b->dense, 0, (size_t)prod * 64, s));
  return NM_OK;
}

}  // namespace nm

namespace {

cudaStream_t pick(nm_context ctx, void* stream) {
  return stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
}

}  // namespace

namespace nm {

void make_ray_params(nm_sensor s, const nm_pose& pose, float res, SimRayParams* rp) {
  std::memset(rp, 0, sizeof(*rp));
  rp->type = s->desc.type;
  rp->width = s->desc.hres;
  rp->height = s->desc.vres;
  rp->hw = s->fp[0];
  rp->hh = s->fp[1];
  rp->c0 = s->fp[2];
  rp->c1 = s->fp[3];
  rp->su = s->fp[4];
  rp->sv = s->fp[5];
  if (s->desc.type == NM_SENSOR_LASER) {
    rp->sinu = s->d_tables;
    rp->cosu = s->d_tables + s->desc.hres;
    rp->sinv = s->d_tables + 2 * s->desc.hres;
    rp->cosv = s->d_tables + 2 * s->desc.hres + s->desc.vres;
  }
  pose_rotation(pose, s->desc.frame_transform, rp->R);
  for (int a = 0; a < 3; ++a) rp->pos[a] = pose.position[a];
  rp->min_range = s->desc.min_range;
  rp->max_range = s->desc.max_range;
  {
    RoundScope rn(NM_ROUND_NEAREST);
    for (int a = 0; a < 3; ++a) rp->eye[a] = rp->pos[a] / res;
    rp->tmin = rp->min_range / res;
    rp->tmax = rp->max_range / res;
  }
}

}  // namespace nm

namespace nm {
void release(nm_simmap sm) {
  if (!sm || sm->refs.fetch_sub(1, std::memory_order_acq_rel) != 1) return;
  nm_context c = sm->ctx;
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  cudaFree(sm->view.brick_index);
  cudaFree(sm->view.brick_leaves);
  cudaFree(sm->view.leaf_words);
  cudaFree(sm->cast_staging);
  delete sm;
  release(c);
}
}  // namespace nm

namespace {
// Shared body of the two render entry points; noise (sigma coefficient, drop probability,
// seed) is applied in the render kernel when `noise` is given.
int render_impl(nm_simmap sm, nm_sensor s, const nm_pose* pose, float* ranges, uint32_t flags,
                void* stream, const float* noise, uint64_t seed) {
  if (!sm || !s || !pose || !ranges) return fail(NM_ERR_ARG, "null argument");
  if (s->ctx != sm->ctx) return fail(NM_ERR_ARG, "sensor and sim map belong to different contexts");
  for (int a = 0; a < 3; ++a)
    if (!std::isfinite(pose->position[a])) return fail(NM_ERR_ARG, "pose position is not finite");
  double qn = 0;
  for (int a = 0; a < 4; ++a) qn += (double)pose->orientation[a] * pose->orientation[a];
  if (!(qn > 1e-20) || !std::isfinite(qn)) return fail(NM_ERR_ARG, "orientation quaternion invalid");
  if (noise && !(std::isfinite(noise[0]) && noise[1] >= 0.0f && noise[1] <= 1.0f))
    return fail(NM_ERR_ARG, "noise parameters invalid");
  nm_context ctx = sm->ctx;
  NM_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = nm::pick(ctx, stream);
  nm::SimRayParams rp;
  nm::make_ray_params(s, *pose, sm->view.res, &rp);
  const size_t bytes = (size_t)rp.width * rp.height * 4;
  float* dst = ranges;
  if (flags & NM_OUTPUT_HOST) {
    if (bytes > ctx->render_staging_bytes) {
      cudaFree(ctx->render_staging);
      ctx->render_staging = nullptr;
      ctx->render_staging_bytes = 0;
      NM_CUDA(cudaMalloc((void**)&ctx->render_staging, bytes));
      ctx->render_staging_bytes = bytes;
    }
    dst = ctx->render_staging;
  }
  if (noise)
    NM_CUDA(nm::launch_sim_render_noisy(sm->view, rp, dst, noise[0], noise[1], seed, st));
  else
    NM_CUDA(nm::launch_sim_render(sm->view, rp, dst, st));
  if (flags & NM_OUTPUT_HOST) {
    NM_CUDA(cudaMemcpyAsync(ranges, dst, bytes, cudaMemcpyDeviceToHost, st));
    NM_CUDA(cudaStreamSynchronize(st));
  } else if (flags & NM_SYNC) {
    NM_CUDA(cudaStreamSynchronize(st));
  }
  return NM_OK;
}
}  // namespace

extern "C" {

int nm_simmap_create_primitives(nm_context ctx, float res, const int32_t vox_min[3],
                                const int32_t vox_max[3], const double* boxes, int32_t n_boxes,
                                const double* cylinders, int32_t n_cylinders, nm_simmap* out) {
  if (!ctx || !vox_min || !vox_max || !out) return fail(NM_ERR_ARG, "null argument");
  *out = nullptr;
  if (!(res > 0.0f)) return fail(NM_ERR_ARG, "resolution must be positive");
  if (n_boxes < 0 || n_cylinders < 0 || (n_boxes > 0 && !boxes) || (n_cylinders > 0 && !cylinders))
    return fail(NM_ERR_ARG, "primitive arrays invalid");
  if (n_boxes > 65535 || n_cylinders > 65535)
    return fail(NM_ERR_ARG, "at most 65535 boxes and 65535 cylinders per call");
  NM_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  std::unique_ptr<nm_simmap_s> sm(new nm_simmap_s());
  sm->ctx = ctx;
  nm::SimBuild b{};
  int rc = begin_build(res, vox_min, vox_max, &b, s);
  if (rc != NM_OK) return rc;
  double* d_boxes = nullptr;
  double* d_cyl = nullptr;
  if (n_boxes) {
    NM_CUDA(cudaMalloc((void**)&d_boxes, (size_t)n_boxes * 48));
    NM_CUDA(cudaMemcpyAsync(d_boxes, boxes, (size_t)n_boxes * 48, cudaMemcpyHostToDevice, s));
  }
  if (n_cylinders) {
    NM_CUDA(cudaMalloc((void**)&d_cyl, (size_t)n_cylinders * 40));
    NM_CUDA(cudaMemcpyAsync(d_cyl, cylinders, (size_t)n_cylinders * 40, cudaMemcpyHostToDevice, s));
  }
  NM_CUDA(nm::launch_voxelize(b, d_boxes, n_boxes, d_cyl, n_cylinders, s));
  rc = finish_build(ctx, b, sm.get(), s);
  cudaFree(d_boxes);
  cudaFree(d_cyl);
  if (rc != NM_OK) return rc;
  nm::retain(ctx);
  *out = sm.release();
  return NM_OK;
}

int nm_simmap_create_voxels(nm_context ctx, float res, const int32_t* ijk, int64_t n,
                            nm_simmap* out) {
  if (!ctx || !out || (n > 0 && !ijk) || n < 0) return fail(NM_ERR_ARG, "invalid argument");
  *out = nullptr;
  if (!(res > 0.0f)) return fail(NM_ERR_ARG, "resolution must be positive");
  NM_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  int32_t vmin[3] = {0, 0, 0}, vmax[3] = {1, 1, 1};
  if (n > 0) {
    for (int a = 0; a < 3; ++a) {
      vmin[a] = INT_MAX;
      vmax[a] = INT_MIN;
    }
    for (int64_t i = 0; i < n; ++i)
      for (int a = 0; a < 3; ++a) {
        vmin[a] = std::min(vmin[a], ijk[3 * i + a]);
        vmax[a] = std::max(vmax[a], ijk[3 * i + a] + 1);
      }
  }
  std::unique_ptr<nm_simmap_s> sm(new nm_simmap_s());
  sm->ctx = ctx;
  nm::SimBuild b{};
  int rc = begin_build(res, vmin, vmax, &b, s);
  if (rc != NM_OK) return rc;
  int32_t* d_ijk = nullptr;
  if (n > 0) {
    NM_CUDA(cudaMalloc((void**)&d_ijk, (size_t)n * 12));
    NM_CUDA(cudaMemcpyAsync(d_ijk, ijk, (size_t)n * 12, cudaMemcpyHostToDevice, s));
    NM_CUDA(nm::launch_set_voxels(b, d_ijk, n, s));
  }
  rc = finish_build(ctx, b, sm.get(), s);
  cudaFree(d_ijk);
  if (rc != NM_OK) return rc;
  nm::retain(ctx);
  *out = sm.release();
  return NM_OK;
}

int nm_simmap_load(nm_context ctx, const char* path, nm_simmap* out) {
  if (!ctx || !path || !out) return fail(NM_ERR_ARG, "null argument");
  *out = nullptr;
  const size_t len = std::strlen(path);
  if (len >= 4 && std::strcmp(path + len - 4, ".vdb") == 0) {
    // the grid named "grid" (else the file's first grid), as SimManager::loadGridFromFile
    // (SimManager.h:196-213) reads it: its active voxels, on a uniform voxel size, translated by
    // whole voxels (world = (index + shift) * res)
    double vs[3], tr[3];
    int64_t n = 0;
    int rc = nm_vdb_active_voxels(path, nullptr, vs, tr, nullptr, 0, &n);
    if (rc != NM_OK) return rc;
    if (!(vs[0] > 0.0) || std::fabs(vs[1] - vs[0]) > 1e-9 * vs[0] ||
        std::fabs(vs[2] - vs[0]) > 1e-9 * vs[0])
      return fail(NM_ERR_UNSUPPORTED, "%s: voxel size (%g, %g, %g) is not uniform", path, vs[0],
                  vs[1], vs[2]);
    int32_t shift[3];
    for (int a = 0; a < 3; ++a) {
      const double q = tr[a] / vs[0];
      shift[a] = (int32_t)std::lround(q);
      if (std::fabs(q - shift[a]) > 1e-6 || std::fabs(q) > 1e9)
        return fail(NM_ERR_UNSUPPORTED, "%s: translation (%g, %g, %g) is not a whole number of voxels",
                    path, tr[0], tr[1], tr[2]);
    }
    std::vector<int32_t> ijk((size_t)n * 3);
    rc = nm_vdb_active_voxels(path, nullptr, vs, tr, ijk.data(), n, &n);
    if (rc != NM_OK) return rc;
    for (int64_t i = 0; i < n; ++i)
      for (int a = 0; a < 3; ++a) ijk[3 * i + a] += shift[a];
    return nm_simmap_create_voxels(ctx, (float)vs[0], ijk.data(), n, out);
  }
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(NM_ERR_IO, "cannot open sim grid '%s'", path);
  char magic[8];
  float res = 0.f;
  int64_t n = 0;
  bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "NMSIMv1", 8) == 0 &&
            std::fread(&res, 4, 1, f) == 1 && std::fread(&n, 8, 1, f) == 1 && n >= 0 &&
            n < (1ll << 34);
  std::vector<int32_t> ijk;
  if (ok) {
    ijk.resize((size_t)n * 3);
    ok = n == 0 || std::fread(ijk.data(), 12, (size_t)n, f) == (size_t)n;
  }
  std::fclose(f);
  if (!ok) return fail(NM_ERR_IO, "%s: not an NMSIMv1 voxel list", path);
  return nm_simmap_create_voxels(ctx, res, ijk.data(), n, out);
}


int nm_simmap_destroy(nm_simmap sm) {
  nm::release(sm);
  return NM_OK;
}

int nm_simmap_info(nm_simmap sm, int32_t bbox[6], uint64_t* active_voxels, uint64_t* leaves) {
  if (!sm) return fail(NM_ERR_ARG, "sim map is null");
  if (bbox) std::memcpy(bbox, sm->bbox, 24);
  if (active_voxels) *active_voxels = sm->active_voxels;
  if (leaves) *leaves = sm->leaves;
  return NM_OK;
}

int nm_simmap_export(nm_simmap sm, int32_t* origins, uint32_t* words, uint64_t max_leaves,
                     uint64_t* n) {
  if (!sm || !n) return fail(NM_ERR_ARG, "null argument");
  NM_CUDA(cudaSetDevice(sm->ctx->device));
  *n = sm->leaves;
  const nm::SimMapView& v = sm->view;
  const long long bprod = (long long)v.bdim[0] * v.bdim[1] * v.bdim[2];
  std::vector<int32_t> bricks((size_t)bprod);
  std::vector<int32_t> blocks((size_t)std::max<uint64_t>(sm->bricks, 1) * 512);
  NM_CUDA(cudaMemcpy(bricks.data(), v.brick_index, (size_t)bprod * 4, cudaMemcpyDeviceToHost));
  NM_CUDA(cudaMemcpy(blocks.data(), v.brick_leaves, blocks.size() * 4, cudaMemcpyDeviceToHost));
  std::vector<uint32_t> all((size_t)sm->leaves * 16);
  if (sm->leaves)
    NM_CUDA(cudaMemcpy(all.data(), v.leaf_words, all.size() * 4, cudaMemcpyDeviceToHost));
  uint64_t o = 0;
  for (long long bpos = 0; bpos < bprod && o < max_leaves; ++bpos) {
    const int32_t blk = bricks[(size_t)bpos];
    if (blk < 0) continue;
    const int bz = (int)(bpos % v.bdim[2]) + v.blo[2];
    const int by = (int)((bpos / v.bdim[2]) % v.bdim[1]) + v.blo[1];
    const int bx = (int)(bpos / ((long long)v.bdim[2] * v.bdim[1])) + v.blo[0];
    for (int e = 0; e < 512 && o < max_leaves; ++e) {
      const int32_t li = blocks[(size_t)blk * 512 + e];
      if (li < 0) continue;
      if (origins) {
        origins[3 * o] = (bx * 8 + (e >> 6)) * 8;
        origins[3 * o + 1] = (by * 8 + ((e >> 3) & 7)) * 8;
        origins[3 * o + 2] = (bz * 8 + (e & 7)) * 8;
      }
      if (words) std::memcpy(words + 16 * o, all.data() + (size_t)li * 16, 64);
      ++o;
    }
  }
  return NM_OK;
}


int nm_sim_render(nm_simmap sm, nm_sensor s, const nm_pose* pose, float* ranges, uint32_t flags,
                  void* stream) {
  return render_impl(sm, s, pose, ranges, flags, stream, nullptr, 0);
}

int nm_sim_render_noisy(nm_simmap sm, nm_sensor s, const nm_pose* pose, float* ranges,
                        float sigma_coef, float drop_prob, uint64_t seed, uint32_t flags,
                        void* stream) {
  const float noise[2] = {sigma_coef, drop_prob};
  return render_impl(sm, s, pose, ranges, flags, stream, noise, seed);
}

int nm_sim_cast_rays(nm_simmap sm, const float* origins, const float* directions, int64_t n,
                     float max_range, float* distances, uint32_t flags, void* stream) {
  if (!sm || n < 0 || (n > 0 && (!origins || !directions || !distances)))
    return fail(NM_ERR_ARG, "invalid argument");
  if (!(max_range >= 0.0f) || !std::isfinite(max_range)) return fail(NM_ERR_ARG, "max_range invalid");
  if (n == 0) return NM_OK;
  nm_context ctx = sm->ctx;
  NM_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t st = pick(ctx, stream);
  const float* d_o = origins;
  const float* d_d = directions;
  float* d_out = distances;
  const bool host_in = (flags & NM_INPUT_HOST) != 0, host_out = (flags & NM_OUTPUT_HOST) != 0;
  if (host_in || host_out) {
    const size_t bytes = (size_t)n * 7 * sizeof(float);
    if (bytes > sm->cast_staging_bytes) {
      cudaFree(sm->cast_staging);
      sm->cast_staging = nullptr;
      sm->cast_staging_bytes = 0;
      NM_CUDA(cudaMalloc((void**)&sm->cast_staging, bytes));
      sm->cast_staging_bytes = bytes;
    }
    if (host_in) {
      NM_CUDA(cudaMemcpyAsync(sm->cast_staging, origins, (size_t)n * 12, cudaMemcpyHostToDevice, st));
      NM_CUDA(cudaMemcpyAsync(sm->cast_staging + 3 * n, directions, (size_t)n * 12,
                              cudaMemcpyHostToDevice, st));
      d_o = sm->cast_staging;
      d_d = sm->cast_staging + 3 * n;
    }
    if (host_out) d_out = sm->cast_staging + 6 * n;
  }
  NM_CUDA(nm::launch_sim_cast(sm->view, d_o, d_d, n, max_range, d_out, st));
  if (host_out) {
    NM_CUDA(cudaMemcpyAsync(distances, d_out, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
    NM_CUDA(cudaStreamSynchronize(st));
  } else if (flags & NM_SYNC) {
    NM_CUDA(cudaStreamSynchronize(st));
  }
  return NM_OK;
}

int nm_observation_sphere(int32_t n, float* directions) {
  if (n < 2 || !directions) return fail(NM_ERR_ARG, "an observation sphere needs n >= 2 rays");
  nm::RoundScope rs(NM_ROUND_NEAREST);
  // Spiral over the sphere (Agent.h:147-179): n points with latitude parameter s running
  // over (-1, 1), longitude s * (0.1 + 1.2 n), evaluated in float like the reference.
  const float x = (float)(0.1 + 1.2 * n);
  const float start = (float)(-1.0 + 1.0 / (n - 1.0));
  const float inc = (float)((2.0 - 2.0 / (n - 1.0)) / (n - 1.0));
  for (int i = 0; i < n; ++i) {
    const float sv = start + (float)i * inc;
    const float lon = sv * x;
    const float lat = (float)((3.14159265358979323846 / 2.0) * std::copysign(1.0, (double)sv) *
                              (1.0 - std::sqrt(1.0 - std::fabs((double)sv))));
    float p[3] = {std::cos(lon) * std::cos(lat), std::sin(lon) * std::cos(lat), std::sin(lat)};
    const float nn = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
    for (int a = 0; a < 3; ++a) directions[3 * i + a] = p[a] / nn;
  }
  return NM_OK;
}

int nm_ranges_add_noise(nm_context ctx, float* ranges, int64_t n, float sigma_coef,
                        float drop_prob, uint64_t seed, void* stream) {
  if (!ctx || (!ranges && n > 0) || n < 0) return fail(NM_ERR_ARG, "invalid argument");
  NM_CUDA(cudaSetDevice(ctx->device));
  NM_CUDA(nm::launch_noise(ranges, n, sigma_coef, drop_prob, seed, pick(ctx, stream)));
  return NM_OK;
}

}  // extern "C"
