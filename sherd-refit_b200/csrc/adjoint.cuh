// adjoint.cuh — values and exact pose gradients of two alignment objectives of
// an assembled group's edges (a fragment pair A, B with B's frame mapped into
// A's by T), for joint pose refinement.
//
// Per (group pose, edge) three work units, one CTA each:
//
//   plane   E   = 1/2 sum_i r_i^2, r_i = (T x_i - q_j) . n_j over B's fracture
//                 samples x_i whose nearest A fracture sample q_j (normal n_j)
//                 is strictly within the correspondence radius: the point-to-
//                 plane residual of the ICP (matching/icp.rs:361-392, 599-640).
//   side B  T_B = sum_i s((tight - d_i) / w), F_B = sum_i s((facing - d_i) / w)
//                 over B's fracture samples moved by T, d_i the distance to A's
//                 fracture faces, s the logistic sigmoid: the smoothed counts
//                 of R 6's tight fraction tight = #(d < tight) / #(d < facing)
//                 (verify.rs:338-349); T_B / F_B is its smoothed form.
//   side A  T_A, F_A the same for A's fracture samples moved by T^-1 against
//                 B's fracture faces (verify.rs:326-327's d2).
//
// Each unit also writes the gradient of its values with respect to the left
// twist xi = (w, v) of the pose it moves points by, T -> exp(xi^) T (for side
// A, T^-1 -> exp(xi^) T^-1), the twist expressed in the fixed fragment's
// frame: with g_i = dvalue/dp_i at the moved point p_i, dvalue/dxi =
// sum_i (p_i x g_i, g_i). The assignment is held fixed, so g_i is exact:
//   * plane: g_i = r_i n_j (the match j is piecewise constant in T), and the
//     gradient is the ICP's own J^T r with rows (p x n, n) (icp.rs:616-624);
//   * sides: the nearest face is held, and the distance to one triangle is
//     differentiable with g = (p - c) / |p - c| in every region of the
//     triangle (face, edge or vertex Voronoi region), c being the closest
//     point on it. The sigmoids read the softened distance
//     d = sqrt(|p - c|^2 + (w/10)^2), which removes the kink of |p - c| where
//     a sample crosses the other fracture surface (at contact, where most
//     samples are, that kink would make the objective non-smooth), so
//     d s(z)/dp = s(z) (1 - s(z)) (-1/w) (p - c) / d.
// The matches and faces are found with the library's own f32 searches (the
// bit-exact bounded NN and the lowest-id closest face); the distance to the
// assigned face is then recomputed in f64 from its f32 vertices, so values
// and gradients are smooth f64 functions of T that central differences can
// check. Points beyond facing + window_k * w contribute nothing (their sigmoid
// terms are below 1e-13 at window_k = 30).
//
// No correspondence is stored: a unit finds, scores and differentiates each
// point in one pass and keeps only its 14 running sums.
#pragma once

#include "verify.cuh"

namespace sherd {

constexpr int ADJ_BLOCK = 256;
constexpr int ADJ_SUMS = 14;    // side: T, F, dT/dxi (6), dF/dxi (6); plane: E, dE/dxi (6)
constexpr int ADJ_VALUES = 5;   // per (pose, edge): E, T_B, F_B, T_A, F_A

struct AdjointConsts {
  double radius_k;  // correspondence radius = radius_k * t * sc.icp
  double width_k;   // sigmoid width w = width_k * t
  double window_k;  // distances beyond facing + window_k * w are left out
};

// The closest point on triangle abc to p in f64: Ericson, Real-Time Collision
// Detection, sec. 5.1.5 (the same regions tri_distance tests in f32).
__device__ __forceinline__ void closest_on_triangle(const double *p, const double *a, const double *b,
                                                    const double *c, double *q) {
  double ab[3], ac[3], ap[3];
  for (int k = 0; k < 3; ++k) {
    ab[k] = b[k] - a[k];
    ac[k] = c[k] - a[k];
    ap[k] = p[k] - a[k];
  }
  auto dot3 = [](const double *u, const double *v) { return (u[0] * v[0] + u[1] * v[1]) + u[2] * v[2]; };
  auto set = [&](const double *o, const double *e1, double s1, const double *e2, double s2) {
    for (int k = 0; k < 3; ++k) q[k] = (o[k] + e1[k] * s1) + e2[k] * s2;
  };
  const double zero[3] = {0.0, 0.0, 0.0};
  double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  if (d1 <= 0.0 && d2 <= 0.0) return set(a, zero, 0.0, zero, 0.0);
  double bp[3] = {p[0] - b[0], p[1] - b[1], p[2] - b[2]};
  double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
  if (d3 >= 0.0 && d4 <= d3) return set(b, zero, 0.0, zero, 0.0);
  double vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) return set(a, ab, d1 / (d1 - d3), zero, 0.0);
  double cp[3] = {p[0] - c[0], p[1] - c[1], p[2] - c[2]};
  double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
  if (d6 >= 0.0 && d5 <= d6) return set(c, zero, 0.0, zero, 0.0);
  double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return set(a, ac, d2 / (d2 - d6), zero, 0.0);
  double va = d3 * d6 - d5 * d4;
  double e43 = d4 - d3, e56 = d5 - d6;
  if (va <= 0.0 && e43 >= 0.0 && e56 >= 0.0) {
    double bc[3] = {c[0] - b[0], c[1] - b[1], c[2] - b[2]};
    return set(b, bc, e43 / (e43 + e56), zero, 0.0);
  }
  double den = (va + vb) + vc;
  set(a, ab, vb / den, ac, vc / den);
}

__device__ __forceinline__ double logistic(double z) { return 1.0 / (1.0 + exp(-z)); }

// acc[o .. o+6) += (p x g, g), a point's share of d value / d xi.
__device__ __forceinline__ void add_twist(double *acc, int o, const double *p, const double *g) {
  acc[o + 0] += p[1] * g[2] - p[2] * g[1];
  acc[o + 1] += p[2] * g[0] - p[0] * g[2];
  acc[o + 2] += p[0] * g[1] - p[1] * g[0];
  acc[o + 3] += g[0];
  acc[o + 4] += g[1];
  acc[o + 5] += g[2];
}

// Unit u = (pose * n_edges + edge) * 3 + kind; kind 0 plane, 1 side B, 2 side A.
// values: n_poses * n_edges * ADJ_VALUES; grads: the same * 6.
__global__ void __launch_bounds__(ADJ_BLOCK) k_adjoint(const PairView *edges, uint32_t n_edges,
                                                       const double *poses, const double *inverses,
                                                       AdjointConsts kc, double *values,
                                                       double *grads, uint32_t *status) {
  __shared__ double s_m[12];
  __shared__ double s_red[ADJ_BLOCK / 32][ADJ_SUMS];
  uint32_t unit = blockIdx.x;
  uint32_t kind = unit % 3u, pe = unit / 3u, e = pe % n_edges;
  const PairView &pr = edges[e];
  if (threadIdx.x < 12) s_m[threadIdx.x] = (kind == 2 ? inverses : poses)[16 * size_t(pe) + threadIdx.x];
  __syncthreads();
  double m[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) m[k] = s_m[k];
  double acc[ADJ_SUMS];
#pragma unroll
  for (int k = 0; k < ADJ_SUMS; ++k) acc[k] = 0.0;
  uint32_t st = 0;
  const double t = pr.sc.t;
  if (kind == 0) {
    const double r = kc.radius_k * t * pr.sc.icp;
    const double r2 = r * r;
    const CloudView &tgt = pr.frac_tgt;
    for (uint32_t i = threadIdx.x; i < pr.n_frac; i += ADJ_BLOCK) {
      double4 x = ldg4(pr.frac_src + i);
      double p[3];
      apply_pose(m, x.x, x.y, x.z, p[0], p[1], p[2]);
      double d2;
      int j = nearest_within_sq(tgt, p[0], p[1], p[2], r2, d2, st);
      if (j < 0 || !(d2 < r2)) continue;
      double4 q = ldg4(tgt.pts + j), n = ldg4(tgt.nrm + j);
      double res = ((p[0] - q.x) * n.x + (p[1] - q.y) * n.y) + (p[2] - q.z) * n.z;
      acc[0] += 0.5 * res * res;
      double g[3] = {res * n.x, res * n.y, res * n.z};
      add_twist(acc, 1, p, g);
    }
  } else {
    const SurfView &moving = kind == 1 ? pr.b : pr.a;
    const MeshView &scene = kind == 1 ? pr.a.frac : pr.b.frac;
    const double w = kc.width_k * t;
    const double soft2 = 0.01 * w * w;  // (w / 10)^2
    const float window = float(pr.sc.facing + kc.window_k * w);
    for (uint32_t i = threadIdx.x; i < moving.n_pf; i += ADJ_BLOCK) {
      double4 x = ldg4(moving.pf + i);
      double p[3];
      apply_pose(m, x.x, x.y, x.z, p[0], p[1], p[2]);
      uint32_t slot;
      mesh_nearest_face(scene, F3{float(p[0]), float(p[1]), float(p[2])}, window, slot, st);
      if (slot == MISS) continue;
      F3 fa, fb, fc;
      uint32_t id;
      tri_at(scene, slot, fa, fb, fc, id);
      double a[3] = {fa.x, fa.y, fa.z}, b[3] = {fb.x, fb.y, fb.z}, c[3] = {fc.x, fc.y, fc.z}, q[3];
      closest_on_triangle(p, a, b, c, q);
      double dv[3] = {p[0] - q[0], p[1] - q[1], p[2] - q[2]};
      double d = sqrt(((dv[0] * dv[0] + dv[1] * dv[1]) + dv[2] * dv[2]) + soft2);
      double st_ = logistic((pr.sc.tight - d) / w), sf = logistic((pr.sc.facing - d) / w);
      acc[0] += st_;
      acc[1] += sf;
      double kt = -st_ * (1.0 - st_) / (w * d), kf = -sf * (1.0 - sf) / (w * d);
      double gt[3] = {kt * dv[0], kt * dv[1], kt * dv[2]};
      double gf[3] = {kf * dv[0], kf * dv[1], kf * dv[2]};
      add_twist(acc, 2, p, gt);
      add_twist(acc, 8, p, gf);
    }
  }
  // Fixed-order reduction: lanes by shuffle, then the warps in index order.
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < ADJ_SUMS; ++k) {
    double v = acc[k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, off);
    if (lane == 0) s_red[warp][k] = v;
  }
  if (st) atomicOr(status, st);
  __syncthreads();
  if (threadIdx.x < ADJ_SUMS) {
    double v = 0.0;
    for (int k = 0; k < ADJ_BLOCK / 32; ++k) v += s_red[k][threadIdx.x];
    const int k = threadIdx.x;
    double *val = values + size_t(pe) * ADJ_VALUES;
    double *grad = grads + size_t(pe) * ADJ_VALUES * 6;
    if (kind == 0) {
      if (k == 0) val[0] = v;
      else if (k <= 6) grad[k - 1] = v;
    } else {
      const int base = kind == 1 ? 1 : 3;  // T then F of this side
      if (k < 2) val[base + k] = v;
      else if (k < 8) grad[6 * base + (k - 2)] = v;
      else grad[6 * (base + 1) + (k - 8)] = v;
    }
  }
}

}  // namespace sherd
