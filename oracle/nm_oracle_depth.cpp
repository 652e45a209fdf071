/*
 * nm_oracle_depth.cpp -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * FP64 CPU restatement of the soft expected-depth renderer and its gradient.  The reference
 * has no counterpart (it is an addition of this library); the definition below is the
 * specification the GPU kernels are checked against.
 *
 * Ray of pixel (w, h): sensor-frame direction from the pixel model of Sensor.h:213-250
 * (frustum pixel corners u = w/W, v = h/H; laser azimuth/elevation tables), evaluated in
 * double and normalised; world direction d = R ds (R world-from-sensor, row-major); index-
 * space eye e = position / res; t_max = max_range / res.
 *
 * Traversal: voxel DDA (Amanatides & Woo, 1987) from the voxel holding e; next crossing per
 * axis tn_a = (boundary_a - e_a) * r_a with r_a = 1 / d_a (once per ray), recomputed from the
 * boundary after every step; the
 * axis with the smallest tn steps, ties to the higher axis.  Voxel k is entered at t_in (axis
 * a_in) when t_in < t_max and left at t_out = min(next crossing, t_max) (axis a_out, none when
 * clamped).  The start voxel holds the sensor and takes no part.
 *
 * Expected depth: occupancy o_k = sigmoid(x_k), x_k = scale * L_k + bias (L_k the voxel's
 * log-odds, 0 for voxels of absent leaves), is the probability that the ray ends inside one
 * voxel length of voxel k: the density along the ray is sigma_k = -ln(1 - o_k) = softplus(x_k),
 * a segment of length D_k = t_out - t_in ends the ray with probability 1 - exp(-sigma_k D_k),
 * and the start voxel (holding the sensor) is empty.  With transmittance
 * T(t) = exp(-int_0^t sigma), the expected depth (the remaining probability placed at t_max) is
 *   D = res * int_0^t_max T(t) dt = res * (t_1 + sum_k T_k (1 - exp(-sigma_k D_k)) / sigma_k),
 * t_1 the first crossing, T_k the transmittance at the entry of voxel k.  D is continuous in
 * the pose: a ray that clips a voxel's corner spends a short segment in it.
 *
 * Gradients:
 *   dD/dsigma_k = res * (T_k D_k^2 g(sigma_k D_k) - D_k S_k),  g(u) = (u e^-u - 1 + e^-u) / u^2,
 *     S_k = int_{t_out,k}^{t_max} T dt;  dsigma/dL = scale * sigmoid(x)
 *   crossing c from voxel A into voxel B:  dD/dc = res * (sigma_B - sigma_A) * int_c^t_max T dt,
 *     and c = (b - e_a) / d_a:  dc/de_a = -1/d_a,  dc/dd_a = -c/d_a.
 * Pose perturbation (left, world frame): position p + rho, rotation exp([phi]x) R, so that
 * d' = d + phi x d:  dD/drho = (1/res) dD/de,  dD/dphi = d x dD/dd.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>

#include "orc_types.h"

namespace {

struct LeafValues {
  std::unordered_map<uint64_t, const float*> leaves;
  static uint64_t key(int lx, int ly, int lz) {
    return ((uint64_t)((uint32_t)(lx + (1 << 20)) & 0x1FFFFFu) << 42) |
           ((uint64_t)((uint32_t)(ly + (1 << 20)) & 0x1FFFFFu) << 21) |
           (uint64_t)((uint32_t)(lz + (1 << 20)) & 0x1FFFFFu);
  }
  // Value pointer of voxel v inside its leaf (nullptr when the leaf is absent) and the
  // voxel's index inside the leaf.
  const float* leaf(const int v[3], int* l, int64_t* leaf_index, const float* base) const {
    auto it = leaves.find(key(v[0] >> 3, v[1] >> 3, v[2] >> 3));
    *l = ((v[0] & 7) << 6) | ((v[1] & 7) << 3) | (v[2] & 7);
    if (it == leaves.end()) return nullptr;
    *leaf_index = (it->second - base) / 512;
    return it->second;
  }
};

void ray_of_pixel(const orc_sensor* s, int w, int h, const double R[9], double d[3]) {
  double x, y, z;
  if (s->type == 0) {
    const double u = (double)w * (double)s->scale_u;
    const double v = (double)h * (double)s->scale_v;
    x = u * (double)s->c0 - (double)s->hw;
    y = v * (double)s->c1 - (double)s->hh;
    z = 1.0;
  } else {
    x = (double)s->sinu[w] * (double)s->cosv[h];
    y = (double)s->sinv[h];
    z = (double)s->cosu[w] * (double)s->cosv[h];
  }
  const double n = std::sqrt((x * x + y * y) + z * z);
  x /= n;
  y /= n;
  z /= n;
  for (int i = 0; i < 3; ++i) d[i] = (R[3 * i] * x + R[3 * i + 1] * y) + R[3 * i + 2] * z;
}

double sigmoid(double x) { return 1.0 / (1.0 + std::exp(-x)); }
double softplus(double x) { return x > 0.0 ? x + std::log1p(std::exp(-x)) : std::log1p(std::exp(x)); }
// (1 - exp(-sigma D)) / sigma, the segment's integral of the transmittance (per unit T_k)
double seg_integral(double sigma, double D) { return sigma > 0.0 ? -std::expm1(-sigma * D) / sigma : D; }
// g(u) = (u e^-u - 1 + e^-u) / u^2 (-> -1/2 as u -> 0)
double seg_g(double u) {
  if (u < 1e-3) return -0.5 + u / 3.0 - u * u / 8.0;
  return (u * std::exp(-u) + std::expm1(-u)) / (u * u);
}

// Visits every voxel of the ray after the start voxel: f(v, t_in, a_in, t_out, a_out), with
// a_out = -1 when the exit is clamped to t_max.
template <class F>
void walk(const double e[3], const double d[3], double t_max, F&& f) {
  int v[3], s[3];
  double tn[3], r[3];
  for (int a = 0; a < 3; ++a) {
    v[a] = (int)std::floor(e[a]);
    s[a] = d[a] > 0.0 ? 1 : (d[a] < 0.0 ? -1 : 0);
    r[a] = s[a] ? 1.0 / d[a] : 0.0;
    tn[a] = s[a] ? ((double)(v[a] + (s[a] > 0 ? 1 : 0)) - e[a]) * r[a] : INFINITY;
  }
  auto next_axis = [&]() {
    int a = 2;
    if (tn[1] < tn[a]) a = 1;
    if (tn[0] < tn[a]) a = 0;
    return a;
  };
  int a_in = next_axis();
  double t_in = tn[a_in];
  const long cap = 3L * (long)t_max + 16;
  for (long it = 0; it < cap && t_in < t_max; ++it) {
    v[a_in] += s[a_in];
    tn[a_in] = ((double)(v[a_in] + (s[a_in] > 0 ? 1 : 0)) - e[a_in]) * r[a_in];
    const int a_out = next_axis();
    const double t_out = tn[a_out];
    if (t_out < t_max) {
      f(v, t_in, a_in, t_out, a_out);
    } else {
      f(v, t_in, a_in, t_max, -1);
    }
    a_in = a_out;
    t_in = t_out;
  }
}

// Transmittance below which a ray's remaining voxels are left out (0: never).  The definition
// walks every ray to t_max; a threshold lets a test measure what ending the walks early, as
// the GPU kernels do below 1e-9, changes.
double g_stop_transmittance = 0.0;

}  // namespace

extern "C" {

void orc_depth_set_stop(double t) { g_stop_transmittance = t; }

// For each listed pixel: expected depth (metres), its pose gradient (6: d/drho, d/dphi) and a
// hash of its voxel sequence; when grad_depth is given, grad_values (n_leaves * 512, same
// order as `values`) receives sum_pixels grad_depth * dD/dL.
void orc_depth(const orc_sensor* s, const double pos[3], const double R[9], double res,
               const int32_t* origins, const float* values, int64_t n_leaves, double scale,
               double bias, const int32_t* pixels, int64_t n_pix, double* depth,
               double* dpose, uint64_t* seq_hash, const double* grad_depth,
               double* grad_values) {
  LeafValues lv;
  lv.leaves.reserve((size_t)n_leaves * 2);
  for (int64_t i = 0; i < n_leaves; ++i)
    lv.leaves[LeafValues::key(origins[3 * i] >> 3, origins[3 * i + 1] >> 3, origins[3 * i + 2] >> 3)] =
        values + 512 * i;
  const double e[3] = {pos[0] / res, pos[1] / res, pos[2] / res};
  const double t_max = (double)s->max_range / res;
  for (int64_t p = 0; p < n_pix; ++p) {
    const int w = pixels[p] % s->width, h = pixels[p] / s->width;
    double d[3];
    ray_of_pixel(s, w, h, R, d);
    // pass 1: expected depth
    double T = 1.0, acc = 0.0, t1 = t_max;
    bool first = true;
    uint64_t hash = 1469598103934665603ull;
    walk(e, d, t_max, [&](const int v[3], double t_in, int a, double t_out, int) {
      if (T < g_stop_transmittance) return;
      int l;
      int64_t li;
      const float* leaf = lv.leaf(v, &l, &li, values);
      const double L = leaf ? (double)leaf[l] : 0.0;
      const double sg = softplus(scale * L + bias);
      if (first) {
        t1 = t_in;
        first = false;
      }
      // the hash covers the voxels that still carry weight: a change of the sequence beyond
      // them cannot move D by more than ~1e-12 of its range
      if (T > 1e-12) {
        for (int c = 0; c < 3; ++c) hash = (hash ^ (uint64_t)(uint32_t)v[c]) * 1099511628211ull;
        hash = (hash ^ (uint64_t)a) * 1099511628211ull;
      }
      acc += T * seg_integral(sg, t_out - t_in);
      T *= std::exp(-sg * (t_out - t_in));
    });
    const double D = t1 + acc;
    depth[p] = D * res;
    if (seq_hash) seq_hash[p] = hash;
    if (!dpose && !grad_values) continue;
    // pass 2: gradients
    const double gd = grad_depth ? grad_depth[p] : 0.0;
    double ge[3] = {0, 0, 0}, gdir[3] = {0, 0, 0};
    double T2 = 1.0, P = 0.0, sg_prev = 0.0;
    walk(e, d, t_max, [&](const int v[3], double t_in, int a_in, double t_out, int) {
      if (T2 < g_stop_transmittance) return;
      int l;
      int64_t li = -1;
      const float* leaf = lv.leaf(v, &l, &li, values);
      const double L = leaf ? (double)leaf[l] : 0.0;
      const double x = scale * L + bias;
      const double sg = softplus(x);
      const double Dk = t_out - t_in;
      // entry crossing: density steps from sg_prev to sg
      const double gc = (sg - sg_prev) * (D - t1 - P);
      ge[a_in] -= gc / d[a_in];
      gdir[a_in] -= gc * t_in / d[a_in];
      const double Pn = P + T2 * seg_integral(sg, Dk);
      if (leaf && grad_values) {
        const double dsig = T2 * Dk * Dk * seg_g(sg * Dk) - Dk * (D - t1 - Pn);
        grad_values[512 * li + l] += gd * res * scale * sigmoid(x) * dsig;
      }
      P = Pn;
      T2 *= std::exp(-sg * Dk);
      sg_prev = sg;
    });
    if (dpose) {
      // dD/drho = res * dD_idx/de * (1/res);  dD/dphi = res * (d x dD_idx/dd)
      for (int a = 0; a < 3; ++a) dpose[6 * p + a] = ge[a];
      dpose[6 * p + 3] = res * (d[1] * gdir[2] - d[2] * gdir[1]);
      dpose[6 * p + 4] = res * (d[2] * gdir[0] - d[0] * gdir[2]);
      dpose[6 * p + 5] = res * (d[0] * gdir[1] - d[1] * gdir[0]);
    }
  }
}

}  // extern "C"
