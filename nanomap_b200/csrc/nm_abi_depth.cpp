// nm_abi_depth.cpp -- C ABI of the soft expected-depth renderer, its adjoint, and scan-to-map
// pose refinement.  No reference counterpart: these run beside the unchanged mapping path and
// read the device map in place.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "nm_host.h"
#include "nm_objects.h"

using nm::fail;

namespace {

bool finite_all(const double* v, int n) {
  for (int i = 0; i < n; ++i)
    if (!std::isfinite(v[i])) return false;
  return true;
}

int make_depth_params(nm_map m, nm_sensor s, const nm_ray_pose* rp, float scale, float bias,
                      nm::DepthParams* p) {
  if (!m || !s || !rp) return fail(NM_ERR_ARG, "null argument");
  if (s->ctx != m->ctx) return fail(NM_ERR_ARG, "sensor and map belong to different contexts");
  if (!finite_all(rp->position, 3) || !finite_all(rp->rotation, 9))
    return fail(NM_ERR_ARG, "ray pose is not finite");
  if (!std::isfinite(scale) || !std::isfinite(bias)) return fail(NM_ERR_ARG, "scale/bias not finite");
  std::memset(p, 0, sizeof(*p));
  p->type = s->desc.type;
  p->width = s->desc.hres;
  p->height = s->desc.vres;
  p->hw = s->fp[0];
  p->hh = s->fp[1];
  p->c0 = s->fp[2];
  p->c1 = s->fp[3];
  p->su = s->fp[4];
  p->sv = s->fp[5];
  if (s->desc.type == NM_SENSOR_LASER) {
    p->sinu = s->d_tables;
    p->cosu = s->d_tables + s->desc.hres;
    p->sinv = s->d_tables + 2 * s->desc.hres;
    p->cosv = s->d_tables + 2 * s->desc.hres + s->desc.vres;
  }
  nm::RoundScope rs(NM_ROUND_NEAREST);
  p->res = (double)m->desc.res;
  for (int i = 0; i < 9; ++i) p->R[i] = rp->rotation[i];
  for (int a = 0; a < 3; ++a) p->eye[a] = rp->position[a] / p->res;
  p->t_max = (double)s->desc.max_range / p->res;
  p->scale = scale;
  p->bias = bias;
  for (int a = 0; a < 3; ++a)
    if (std::fabs(p->eye[a]) + p->t_max + 2.0 > (double)(1 << 23) - 16.0)
      return fail(NM_ERR_ARG, "pose is outside the map's addressable range (+-%d voxels)", 1 << 23);
  return NM_OK;
}

// Caller arrays in slot layout must cover every slot the kernels can address.
int check_values_len(nm_map m, const float* values, const float* grad_values, uint64_t n) {
  if (!values && !grad_values) return NM_OK;
  const uint64_t need = (uint64_t)m->view.capacity * nm::kLeafVoxels;
  if (n < need)
    return fail(NM_ERR_ARG, "log-odds arrays hold %llu floats, the map's %u slots need %llu",
                (unsigned long long)n, m->view.capacity, (unsigned long long)need);
  return NM_OK;
}

int reserve_scratch(nm_map m, size_t n) {
  if (n <= m->depth_scratch_n) return NM_OK;
  cudaFree(m->depth_scratch);
  m->depth_scratch = nullptr;
  m->depth_scratch_n = 0;
  NM_CUDA(cudaMalloc((void**)&m->depth_scratch, n * sizeof(double)));
  m->depth_scratch_n = n;
  return NM_OK;
}

}  // namespace

extern "C" {

int nm_ray_pose_from_pose(nm_sensor s, const nm_pose* pose, nm_ray_pose* out) {
  if (!s || !out) return fail(NM_ERR_ARG, "null argument");
  const int rc = nm::validate_pose(pose);
  if (rc != NM_OK) return rc;
  nm::RoundScope rs(NM_ROUND_NEAREST);
  double w = pose->orientation[0], x = pose->orientation[1], y = pose->orientation[2],
         z = pose->orientation[3];
  const double n = std::sqrt(w * w + x * x + y * y + z * z);
  w /= n;
  x /= n;
  y /= n;
  z /= n;
  const double M[9] = {1.0 - 2.0 * (y * y + z * z), 2.0 * (x * y - w * z), 2.0 * (x * z + w * y),
                       2.0 * (x * y + w * z), 1.0 - 2.0 * (x * x + z * z), 2.0 * (y * z - w * x),
                       2.0 * (x * z - w * y), 2.0 * (y * z + w * x), 1.0 - 2.0 * (x * x + y * y)};
  const float* F = s->desc.frame_transform;  // column-major
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      out->rotation[3 * r + c] = M[3 * r] * (double)F[3 * c] + M[3 * r + 1] * (double)F[3 * c + 1] +
                                 M[3 * r + 2] * (double)F[3 * c + 2];
  for (int a = 0; a < 3; ++a) out->position[a] = (double)pose->position[a];
  return NM_OK;
}

int nm_map_values_copy(nm_map m, float* dst, uint64_t max_floats, uint64_t* n_floats,
                       void* stream) {
  if (!m || !n_floats) return fail(NM_ERR_ARG, "null argument");
  const uint64_t n = (uint64_t)m->view.capacity * nm::kLeafVoxels;
  *n_floats = n;
  if (!dst) return NM_OK;
  if (max_floats < n) return fail(NM_ERR_ARG, "destination holds %llu floats, map needs %llu",
                                  (unsigned long long)max_floats, (unsigned long long)n);
  NM_CUDA(cudaSetDevice(m->ctx->device));
  NM_CUDA(cudaMemcpyAsync(dst, m->view.values, n * sizeof(float), cudaMemcpyDeviceToDevice,
                          nm::pick(m->ctx, stream)));
  return NM_OK;
}

int nm_map_slot_origins(nm_map m, int32_t* origins, uint64_t max_slots, uint64_t* n_slots) {
  if (!m || !n_slots) return fail(NM_ERR_ARG, "null argument");
  const uint32_t C = m->view.capacity;
  *n_slots = C;
  if (!origins) return NM_OK;
  NM_CUDA(cudaSetDevice(m->ctx->device));
  NM_CUDA(cudaDeviceSynchronize());
  std::vector<unsigned long long> keys(C);
  NM_CUDA(cudaMemcpy(keys.data(), m->view.keys, (size_t)C * 8, cudaMemcpyDeviceToHost));
  const uint64_t k = std::min<uint64_t>(C, max_slots);
  for (uint64_t i = 0; i < k; ++i) {
    if (keys[i] == nm::kEmptyKey) {
      origins[3 * i] = origins[3 * i + 1] = origins[3 * i + 2] = INT32_MIN;
    } else {
      int lx, ly, lz;
      nm::key_leaf(keys[i], &lx, &ly, &lz);
      origins[3 * i] = lx * 8;
      origins[3 * i + 1] = ly * 8;
      origins[3 * i + 2] = lz * 8;
    }
  }
  return NM_OK;
}

int nm_depth_render(nm_map m, nm_sensor s, const nm_ray_pose* pose, const float* values,
                    uint64_t n_floats, float scale, float bias, float* depth, void* stream) {
  nm::DepthParams p;
  int rc = make_depth_params(m, s, pose, scale, bias, &p);
  if (rc != NM_OK) return rc;
  if (!depth) return fail(NM_ERR_ARG, "depth is null");
  rc = check_values_len(m, values, nullptr, n_floats);
  if (rc != NM_OK) return rc;
  NM_CUDA(cudaSetDevice(m->ctx->device));
  NM_CUDA(nm::launch_depth_forward(p, m->view, values ? values : m->view.values, depth,
                                   nm::pick(m->ctx, stream)));
  return NM_OK;
}

int nm_depth_backward(nm_map m, nm_sensor s, const nm_ray_pose* pose, const float* values,
                      uint64_t n_floats, float scale, float bias, const float* grad_depth,
                      const float* depth, float* grad_values, double grad_pose[6],
                      void* stream) {
  nm::DepthParams p;
  int rc = make_depth_params(m, s, pose, scale, bias, &p);
  if (rc != NM_OK) return rc;
  if (!grad_depth) return fail(NM_ERR_ARG, "grad_depth is null");
  rc = check_values_len(m, values, grad_values, n_floats);
  if (rc != NM_OK) return rc;
  NM_CUDA(cudaSetDevice(m->ctx->device));
  const int nb = nm::depth_partial_blocks(p);
  rc = reserve_scratch(m, (size_t)nb * 6 + 8);
  if (rc != NM_OK) return rc;
  cudaStream_t s0 = nm::pick(m->ctx, stream);
  double* out6 = m->depth_scratch + (size_t)nb * 6;
  NM_CUDA(nm::launch_depth_backward(p, m->view, values ? values : m->view.values, grad_depth,
                                    depth, grad_values, m->depth_scratch, out6, s0));
  if (grad_pose) {
    NM_CUDA(cudaMemcpyAsync(grad_pose, out6, 6 * sizeof(double), cudaMemcpyDeviceToHost, s0));
    NM_CUDA(cudaStreamSynchronize(s0));
  }
  return NM_OK;
}

int nm_pose_refine(nm_map m, nm_sensor s, nm_ray_pose* pose, const float* target, float scale,
                   float bias, float max_residual, int32_t steps, float lr_position,
                   float lr_rotation, float* losses) {
  nm_refine_desc d;
  d.scale = scale;
  d.bias = bias;
  d.max_residual = max_residual;
  d.steps = steps;
  d.lr_position = lr_position;
  d.lr_rotation = lr_rotation;
  d.surface_offset = 0.0f;
  d.edge_threshold = 0.0f;
  return nm_pose_refine_desc(m, s, pose, target, &d, losses);
}

int nm_pose_refine_desc(nm_map m, nm_sensor s, nm_ray_pose* pose, const float* target,
                        const nm_refine_desc* desc, float* losses) {
  if (!pose || !target || !desc) return fail(NM_ERR_ARG, "null argument");
  const float scale = desc->scale, bias = desc->bias, max_residual = desc->max_residual;
  const int32_t steps = desc->steps;
  const float lr_position = desc->lr_position, lr_rotation = desc->lr_rotation;
  if (!(max_residual >= 0.0f)) return fail(NM_ERR_ARG, "max_residual must be >= 0");
  if (steps < 0) return fail(NM_ERR_ARG, "steps must be >= 0");
  if (!(lr_position >= 0.0f) || !(lr_rotation >= 0.0f)) return fail(NM_ERR_ARG, "bad learning rate");
  if (!(desc->surface_offset >= 0.0f && desc->surface_offset <= 1.0f))
    return fail(NM_ERR_ARG, "surface_offset must lie in [0, 1]");
  if (!(desc->edge_threshold >= 0.0f)) return fail(NM_ERR_ARG, "edge_threshold must be >= 0");
  nm::DepthParams p;
  int rc = make_depth_params(m, s, pose, scale, bias, &p);
  if (rc != NM_OK) return rc;
  NM_CUDA(cudaSetDevice(m->ctx->device));
  const int nb = nm::depth_partial_blocks(p);
  // partials, then the device state, then the losses
  const size_t state_doubles = (sizeof(nm::RefineState) + 7) / 8;
  rc = reserve_scratch(m, (size_t)nb * 8 + state_doubles + ((size_t)steps + 2) / 2);
  if (rc != NM_OK) return rc;
  cudaStream_t s0 = m->ctx->stream;
  nm::RefineState* d_st = reinterpret_cast<nm::RefineState*>(m->depth_scratch + (size_t)nb * 8);
  float* d_losses = reinterpret_cast<float*>(m->depth_scratch + (size_t)nb * 8 + state_doubles);
  nm::RefineState st{};
  std::memcpy(st.position, pose->position, sizeof(st.position));
  std::memcpy(st.R, pose->rotation, sizeof(st.R));
  st.res = p.res;
  st.t_max = p.t_max;
  st.lr_position = lr_position;
  st.lr_rotation = lr_rotation;
  st.steps = steps;
  NM_CUDA(cudaMemcpyAsync(d_st, &st, sizeof(st), cudaMemcpyHostToDevice, s0));
  // every step queued at once: the kernels read the pose from d_st, the update kernel writes it
  for (int it = 0; it <= steps; ++it)
    NM_CUDA(nm::launch_depth_refine(p, m->view, m->view.values, target, max_residual,
                                    desc->surface_offset, desc->edge_threshold,
                                    m->depth_scratch, d_st, d_losses, it, s0));
  NM_CUDA(cudaMemcpyAsync(&st, d_st, sizeof(st), cudaMemcpyDeviceToHost, s0));
  NM_CUDA(cudaStreamSynchronize(s0));
  if (st.error & nm::kRefineNoPixels) return fail(NM_ERR_ARG, "target has no valid pixels");
  if (st.error & nm::kRefineOutOfRange)
    return fail(NM_ERR_ARG, "pose left the map's addressable range (+-%d voxels)", 1 << 23);
  if (losses)
    NM_CUDA(cudaMemcpy(losses, d_losses, ((size_t)steps + 1) * sizeof(float), cudaMemcpyDeviceToHost));
  nm_ray_pose cur = *pose;
  std::memcpy(cur.position, st.position, sizeof(cur.position));
  std::memcpy(cur.rotation, st.R, sizeof(cur.rotation));
  *pose = cur;
  return NM_OK;
}

}  // extern "C"
