// icp.cuh — one point-to-plane registration_icp rung as a CTA-cooperative
// routine (matching/icp.rs:308-440, 599-778).
//
// Every pass over the moving cloud is one fused loop: transform the point by
// the current pose (f64, R p + tau), find the nearest target inside the strict
// radius (exact, lowest index on ties), and accumulate the correspondence
// count, the squared error and the 27 normal-equation terms (21 of the lower
// triangle of J^T J, 6 of J^T r) in f64 registers. A pass ends with a warp
// shuffle tree and a fixed-order sum over the warps, both compensated (TwoSum,
// the rounding errors carried and added once), so a rung is bit-for-bit
// reproducible run to run. One thread then runs Open3D's convergence test,
// Eigen's pivoted LDLT (f64) and the Rz Ry Rx update, and publishes the pose.
//
// The points are the reference numerics (Numerics::REFERENCE, f64 point loops,
// World assembly); the difference from the CPU oracle is the summation order
// of the per-pass sums and the pose being re-applied to the source each pass
// (T S) where the reference moves the previous pass's points (U P).
#pragma once

#include "traverse.cuh"

namespace sherd {

constexpr int ICP_BLOCK = 128;
constexpr int ICP_SUMS = 29;  // count, err2, jtj[21], jtr[6]

struct IcpShared {
  double red[ICP_BLOCK / 32][ICP_SUMS];
  double carry[ICP_BLOCK / 32][ICP_SUMS];  // the rounding errors of red's warp sums
  double sums[ICP_SUMS];
  double t[16];
  int stop;
};

// icp::eigen_pivots (icp.rs:661-674).
__device__ void eigen_pivots(const double a[6][6], int perm[6]) {
  for (int k = 0; k < 6; ++k) perm[k] = k;
  for (int k = 0; k < 6; ++k) {
    int best = k;
    for (int i = k + 1; i < 6; ++i)
      if (fabs(a[perm[i]][perm[i]]) > fabs(a[perm[best]][perm[best]])) best = i;
    int tmp = perm[k];
    perm[k] = perm[best];
    perm[best] = tmp;
  }
}

// icp::solve_ldlt (icp.rs:692-753).
__device__ bool solve_ldlt(const double a[6][6], const double b[6], double x[6]) {
  int perm[6];
  eigen_pivots(a, perm);
  double m[6][6];
  for (int k = 0; k < 6; ++k)
    for (int l = 0; l < 6; ++l) m[k][l] = a[perm[k]][perm[l]];
#pragma unroll 1
  for (int k = 0; k < 6; ++k) {
    if (k > 0) {
      double temp[6];
      for (int j = 0; j < k; ++j) temp[j] = m[j][j] * m[k][j];
      double diagonal = m[k][k];
      for (int j = 0; j < k; ++j) diagonal -= m[k][j] * temp[j];
      m[k][k] = diagonal;
      for (int r = k + 1; r < 6; ++r) {
        double below = m[r][k];
        for (int j = 0; j < k; ++j) below -= m[r][j] * temp[j];
        m[r][k] = below;
      }
    }
    double pivot = m[k][k];
    if (pivot != 0.0)
      for (int r = k + 1; r < 6; ++r) m[r][k] /= pivot;
  }
  double y[6];
  for (int k = 0; k < 6; ++k) y[k] = b[perm[k]];
  for (int i = 0; i < 6; ++i) {
    double value = y[i];
    for (int j = 0; j < i; ++j) value -= m[i][j] * y[j];
    y[i] = value;
  }
  for (int i = 0; i < 6; ++i) {
    double pivot = m[i][i];
    y[i] = fabs(pivot) > 2.2250738585072014e-308 ? y[i] / pivot : 0.0;
  }
  for (int i = 5; i >= 0; --i) {
    double value = y[i];
    for (int j = i + 1; j < 6; ++j) value -= m[j][i] * y[j];
    y[i] = value;
  }
  for (int k = 0; k < 6; ++k) x[perm[k]] = y[k];
  for (int k = 0; k < 6; ++k)
    if (!isfinite(x[k])) return false;
  return true;
}

__device__ void mat3mul(const double a[3][3], const double b[3][3], double o[3][3]) {
  double r[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r[i][j] = (a[i][0] * b[0][j] + a[i][1] * b[1][j]) + a[i][2] * b[2][j];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) o[i][j] = r[i][j];
}

// icp::euler_zyx (icp.rs:770-778).
__device__ void euler_zyx(double al, double be, double ga, double r[3][3]) {
  double sa, ca, sb, cb, sg, cg;
  sincos(al, &sa, &ca);
  sincos(be, &sb, &cb);
  sincos(ga, &sg, &cg);
  double rx[3][3] = {{1, 0, 0}, {0, ca, -sa}, {0, sa, ca}};
  double ry[3][3] = {{cb, 0, sb}, {0, 1, 0}, {-sb, 0, cb}};
  double rz[3][3] = {{cg, -sg, 0}, {sg, cg, 0}, {0, 0, 1}};
  double t[3][3];
  mat3mul(rz, ry, t);
  mat3mul(t, rx, r);
}

__device__ void matmul4(const double *a, const double *b, double *o) {
  double r[16];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double s = a[4 * i] * b[j];
      for (int k = 1; k < 4; ++k) s += a[4 * i + k] * b[4 * k + j];
      r[4 * i + j] = s;
    }
  for (int i = 0; i < 16; ++i) o[i] = r[i];
}

// The point-to-plane update from the pass sums (icp.rs:408-440): identity when
// there is no correspondence, no normal or no finite solution. Run by one
// thread per pass and kept out of line, so that its 6x6 working arrays do not
// count against the registers of the point loops.
__device__ __noinline__ void plane_update(const double *s, bool has_normals, double u[16]) {
  for (int i = 0; i < 16; ++i) u[i] = (i % 5 == 0) ? 1.0 : 0.0;
  if (s[0] == 0.0 || !has_normals) return;
  double a[6][6], rhs[6], x[6];
  int q = 2;
  for (int k = 0; k < 6; ++k)
    for (int l = 0; l <= k; ++l) {
      a[k][l] = s[q];
      a[l][k] = s[q];
      ++q;
    }
  for (int k = 0; k < 6; ++k) rhs[k] = -s[23 + k];
  if (!solve_ldlt(a, rhs, x)) return;
  double r[3][3];
  euler_zyx(x[0], x[1], x[2], r);
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) u[4 * i + j] = r[i][j];
    u[4 * i + 3] = x[3 + i];
  }
}

// T <- U T for the update of the pass sums in sh (thread 0 only).
__device__ __noinline__ void plane_step(IcpShared &sh, bool has_normals) {
  double u[16];
  plane_update(sh.sums, has_normals, u);
  matmul4(u, sh.t, sh.t);
}

// The rotation of the SVD of m with a reflection on the smallest singular
// value undone, R = U diag(1, 1, det(U) det(V)) V^T: the rotation part of
// Eigen's umeyama (icp.rs:585-590). One-sided Jacobi (Hestenes): plane
// rotations of the columns of a = m V until every two are orthogonal; then
// a_j = sigma_j u_j, with u2 taken as u0 x u1. R is unique whenever the
// second singular value is not zero.
__device__ __noinline__ void svd_rotation(const double m[3][3], double r[3][3]) {
  double a[3][3], v[3][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0}};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) a[i][j] = m[i][j];
  for (int sweep = 0; sweep < 30; ++sweep) {
    bool turned = false;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        double al = (a[0][p] * a[0][p] + a[1][p] * a[1][p]) + a[2][p] * a[2][p];
        double be = (a[0][q] * a[0][q] + a[1][q] * a[1][q]) + a[2][q] * a[2][q];
        double ga = (a[0][p] * a[0][q] + a[1][p] * a[1][q]) + a[2][p] * a[2][q];
        if (!(fabs(ga) > 1e-15 * sqrt(al * be))) continue;
        turned = true;
        double ze = (be - al) / (2.0 * ga);
        double tt = (ze >= 0.0 ? 1.0 : -1.0) / (fabs(ze) + sqrt(1.0 + ze * ze));
        double c = 1.0 / sqrt(1.0 + tt * tt), sn = c * tt;
        for (int i = 0; i < 3; ++i) {
          double x = a[i][p], y = a[i][q];
          a[i][p] = c * x - sn * y;
          a[i][q] = sn * x + c * y;
          x = v[i][p];
          y = v[i][q];
          v[i][p] = c * x - sn * y;
          v[i][q] = sn * x + c * y;
        }
      }
    if (!turned) break;
  }
  double sv[3];
  int ord[3] = {0, 1, 2};
  for (int j = 0; j < 3; ++j) sv[j] = sqrt((a[0][j] * a[0][j] + a[1][j] * a[1][j]) + a[2][j] * a[2][j]);
  for (int x = 0; x < 2; ++x)
    for (int y = 0; y < 2 - x; ++y)
      if (sv[ord[y]] < sv[ord[y + 1]]) {
        int t = ord[y];
        ord[y] = ord[y + 1];
        ord[y + 1] = t;
      }
  const double smax = sv[ord[0]];
  double u[3][3], w[3][3];
  bool have[3];
  for (int k = 0; k < 3; ++k) {
    int j = ord[k];
    for (int i = 0; i < 3; ++i) w[i][k] = v[i][j];
    have[k] = smax > 0.0 && sv[j] > 1e-12 * smax;
    for (int i = 0; i < 3; ++i) u[i][k] = have[k] ? a[i][j] / sv[j] : 0.0;
  }
  if (!have[0]) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) r[i][j] = i == j ? 1.0 : 0.0;
    return;
  }
  if (!have[1]) {  // any unit vector orthogonal to u0
    int e = fabs(u[0][0]) <= fabs(u[1][0]) ? (fabs(u[0][0]) <= fabs(u[2][0]) ? 0 : 2)
                                          : (fabs(u[1][0]) <= fabs(u[2][0]) ? 1 : 2);
    double ev[3] = {0.0, 0.0, 0.0};
    ev[e] = 1.0;
    double c[3] = {u[1][0] * ev[2] - u[2][0] * ev[1], u[2][0] * ev[0] - u[0][0] * ev[2],
                   u[0][0] * ev[1] - u[1][0] * ev[0]};
    double nc = sqrt((c[0] * c[0] + c[1] * c[1]) + c[2] * c[2]);
    for (int i = 0; i < 3; ++i) u[i][1] = c[i] / nc;
  }
  // u2 = u0 x u1 always: for rank 3 the SVD's own u2 is +-(u0 x u1) and the
  // det(U) det(V) factor below absorbs the sign; for rank 2, a2 / sigma2 is
  // round-off.
  u[0][2] = u[1][0] * u[2][1] - u[2][0] * u[1][1];
  u[1][2] = u[2][0] * u[0][1] - u[0][0] * u[2][1];
  u[2][2] = u[0][0] * u[1][1] - u[1][0] * u[0][1];
  auto det3 = [](const double x[3][3]) {
    return x[0][0] * (x[1][1] * x[2][2] - x[1][2] * x[2][1]) -
           x[0][1] * (x[1][0] * x[2][2] - x[1][2] * x[2][0]) +
           x[0][2] * (x[1][0] * x[2][1] - x[1][1] * x[2][0]);
  };
  const double d = det3(u) * det3(w) < 0.0 ? -1.0 : 1.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      r[i][j] = (u[i][0] * w[j][0] + u[i][1] * w[j][1]) + d * u[i][2] * w[j][2];
}

// icp::umeyama without scaling (icp.rs:527-592) from a point-to-point pass's
// sums: s[0] count, s[2..5) and s[5..8) the sums of the moved source and of
// the target points, s[8..17) the covariance already scaled by 1/n. T <- U T
// (thread 0 only); identity when there is no correspondence.
__device__ __noinline__ void point_step(IcpShared &sh) {
  const double *s = sh.sums;
  double u[16];
  for (int i = 0; i < 16; ++i) u[i] = (i % 5 == 0) ? 1.0 : 0.0;
  if (s[0] != 0.0) {
    const double one_over_n = 1.0 / s[0];
    double mp[3], mq[3], sigma[3][3], r[3][3];
    for (int k = 0; k < 3; ++k) {
      mp[k] = s[2 + k] * one_over_n;
      mq[k] = s[5 + k] * one_over_n;
    }
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) sigma[i][j] = s[8 + 3 * i + j];
    svd_rotation(sigma, r);
    for (int i = 0; i < 3; ++i) {
      for (int j = 0; j < 3; ++j) u[4 * i + j] = r[i][j];
      u[4 * i + 3] = mq[i] - ((r[i][0] * mp[0] + r[i][1] * mp[1]) + r[i][2] * mp[2]);
    }
  }
  matmul4(u, sh.t, sh.t);
}

// Knuth's TwoSum: s = fl(a + b) and the exact rounding error e, a + b = s + e
// (no multiply-add is contracted in this build, so the identity holds).
__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e) {
  s = a + b;
  double bp = s - a;
  e = (a - (s - bp)) + (b - bp);
}

// The sum of x over the warp for lane 0, compensated: the shuffle tree adds
// the 32 partials pairwise and carries every addition's rounding error
// (TwoSum) beside it; returns the sum and the carried error separately.
__device__ __forceinline__ void warp_sum_compensated(double x, double &sum, double &carry) {
  double c = 0.0;
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    double y = __shfl_down_sync(0xffffffffu, x, o), cy = __shfl_down_sync(0xffffffffu, c, o);
    double s, e;
    two_sum(x, y, s, e);
    x = s;
    c = (c + cy) + e;
  }
  sum = x;
  carry = c;
}

// A source point's match (a target slot, or -1) as the pass keeps it: an int,
// or 16 bits (0xFFFF for none) when every target of the batch has fewer than
// 65535 points, which halves the bytes the ladder writes and re-reads.
__device__ __forceinline__ int hint_get(const int *h, uint32_t i) { return h[i]; }
__device__ __forceinline__ int hint_get(const uint16_t *h, uint32_t i) {
  uint16_t v = h[i];
  return v == 0xFFFFu ? -1 : int(v);
}
__device__ __forceinline__ void hint_set(int *h, uint32_t i, int s) { h[i] = s; }
__device__ __forceinline__ void hint_set(uint16_t *h, uint32_t i, int s) {
  h[i] = s < 0 ? uint16_t(0xFFFFu) : uint16_t(s);
}

// Sums B..E-1 of one pass (count, err2, the 21 lower-triangle terms of J^T J
// and the 6 of J^T r, in that order) over the correspondences found in hint[],
// reduced over the warp into sh.red[warp][B..E). The squared distance is
// re-formed exactly as the search formed it.
template <int B, int E, class H>
__device__ __forceinline__ void icp_accumulate(const double4 *src, uint32_t ns, const CloudView &tgt,
                                               const double *t, double r2, bool valid,
                                               const H *hint, IcpShared &sh) {
  double acc[E - B];
#pragma unroll
  for (int k = 0; k < E - B; ++k) acc[k] = 0.0;
  if (valid) {
    for (uint32_t i = threadIdx.x; i < ns; i += ICP_BLOCK) {
      int s = hint_get(hint, i);
      if (s < 0) continue;
      double4 p = src[i];
      double x, y, z;
      apply_pose(t, p.x, p.y, p.z, x, y, z);
      double4 q = tgt.pts[s];
      double dx = x - q.x, dy = y - q.y, dz = z - q.z;
      double d2 = (dx * dx + dy * dy) + dz * dz;
      if (!(d2 < r2)) continue;
      double v[ICP_SUMS];
      v[0] = 1.0;
      v[1] = d2;
#pragma unroll
      for (int m = 2; m < ICP_SUMS; ++m) v[m] = 0.0;
      if (tgt.nrm) {
        double4 n = tgt.nrm[s];
        double row[6] = {y * n.z - z * n.y, z * n.x - x * n.z, x * n.y - y * n.x, n.x, n.y, n.z};
        double r = (x - q.x) * n.x + (y - q.y) * n.y + (z - q.z) * n.z;
        int m = 2;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
#pragma unroll
          for (int l = 0; l <= k; ++l) v[m++] = row[k] * row[l];
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) v[23 + k] = row[k] * r;
      }
#pragma unroll
      for (int k = 0; k < E - B; ++k) acc[k] += v[B + k];
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < E - B; ++k) {
    double x, c;
    warp_sum_compensated(acc[k], x, c);
    if (lane == 0) {
      sh.red[warp][B + k] = x;
      sh.carry[warp][B + k] = c;
    }
  }
}

// The sums of a point-to-point pass over the correspondences in hint[]:
// MOMENTS gives count, err2 and the sums of the moved source and matched target
// points (s[0..8)); otherwise the 9 covariance terms ((q - mean_q) / n)(p -
// mean_p)^T (s[8..17)), centred as umeyama centres them (icp.rs:548-570).
template <bool MOMENTS, class H>
__device__ __forceinline__ void p2p_accumulate(const double4 *src, uint32_t ns,
                                               const CloudView &tgt, const double *t, double r2,
                                               bool valid, const H *hint, const double *mean,
                                               double one_over_n, IcpShared &sh) {
  constexpr int N = MOMENTS ? 8 : 9, B = MOMENTS ? 0 : 8;
  double acc[N];
#pragma unroll
  for (int k = 0; k < N; ++k) acc[k] = 0.0;
  if (valid) {
    for (uint32_t i = threadIdx.x; i < ns; i += ICP_BLOCK) {
      int s = hint_get(hint, i);
      if (s < 0) continue;
      double4 p = src[i];
      double x, y, z;
      apply_pose(t, p.x, p.y, p.z, x, y, z);
      double4 q = tgt.pts[s];
      double dx = x - q.x, dy = y - q.y, dz = z - q.z;
      double d2 = (dx * dx + dy * dy) + dz * dz;
      if (!(d2 < r2)) continue;
      if (MOMENTS) {
        acc[0] += 1.0;
        acc[1] += d2;
        acc[2] += x;
        acc[3] += y;
        acc[4] += z;
        acc[5] += q.x;
        acc[6] += q.y;
        acc[7] += q.z;
      } else {
        double a[3] = {x - mean[0], y - mean[1], z - mean[2]};
        double b[3] = {(q.x - mean[3]) * one_over_n, (q.y - mean[4]) * one_over_n,
                       (q.z - mean[5]) * one_over_n};
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
          for (int c = 0; c < 3; ++c) acc[3 * r + c] += b[r] * a[c];
      }
    }
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double x, c;
    warp_sum_compensated(acc[k], x, c);
    if (lane == 0) {
      sh.red[warp][B + k] = x;
      sh.carry[warp][B + k] = c;
    }
  }
}

// sh.sums[lo..hi) from the warps' partial sums, in warp order: the final sum
// of the partials is compensated (TwoSum over the warps' sums, their carried
// errors added once at the end), so the block total is the partials' exact
// sum up to a last rounding whatever their magnitudes.
__device__ __forceinline__ void reduce_sums(IcpShared &sh, int lo, int hi) {
  __syncthreads();
  if (int(threadIdx.x) >= lo && int(threadIdx.x) < hi) {
    double v = sh.red[0][threadIdx.x], c = sh.carry[0][threadIdx.x];
    for (int w = 1; w < ICP_BLOCK / 32; ++w) {
      double s, e;
      two_sum(v, sh.red[w][threadIdx.x], s, e);
      v = s;
      c = (c + sh.carry[w][threadIdx.x]) + e;
    }
    sh.sums[threadIdx.x] = v + c;
  }
  __syncthreads();
}

// One correspondence pass (icp::correspondences + icp::normal_equations) over
// `src` under the pose sh.t; leaves the block totals in sh.sums. `hint[i]`
// carries each source point's last match (a target slot, or -1) from pass to
// pass as the warm start of its search.
template <class H>
__device__ void icp_pass(const double4 *src, uint32_t ns, const CloudView &tgt, double r2,
                         bool valid, IcpShared &sh, H *hint, uint32_t &status,
                         bool point_to_point = false) {
  // The pose is read from shared memory where it is used (a broadcast load):
  // twelve doubles held in registers across the search and the accumulation
  // would cost 24 registers that the ladder's occupancy cannot spare.
  const double *t = sh.t;
  // Two kinds of loops over the moving points, so that the 29 accumulators are
  // never live across the nearest-neighbour search: the first finds every
  // point's match (kept in hint[i], which also warm-starts the next pass), the
  // others re-form the moved point and add each correspondence into half of
  // the sums; every thread adds its points into each sum in the same order.
  if (valid) {
    for (uint32_t i = threadIdx.x; i < ns; i += ICP_BLOCK) {
      double4 p = src[i];
      double x, y, z;
      apply_pose(t, p.x, p.y, p.z, x, y, z);
      double d2;
      hint_set(hint, i, nearest_within_sq(tgt, x, y, z, r2, d2, status, hint_get(hint, i)));
    }
  }
  if (point_to_point) {
    p2p_accumulate<true>(src, ns, tgt, t, r2, valid, hint, nullptr, 0.0, sh);
    reduce_sums(sh, 0, 8);
    double one_over_n = sh.sums[0] != 0.0 ? 1.0 / sh.sums[0] : 0.0;
    double mean[6];
    for (int k = 0; k < 6; ++k) mean[k] = sh.sums[2 + k] * one_over_n;
    p2p_accumulate<false>(src, ns, tgt, t, r2, valid, hint, mean, one_over_n, sh);
    reduce_sums(sh, 8, 17);
    return;
  }
  icp_accumulate<0, 15>(src, ns, tgt, t, r2, valid, hint, sh);
  icp_accumulate<15, ICP_SUMS>(src, ns, tgt, t, r2, valid, hint, sh);
  reduce_sums(sh, 0, ICP_SUMS);
}

// Open3D's (fitness, inlier_rmse) from the pass sums (icp.rs:385-391).
__device__ __forceinline__ void fit_rmse(const double *s, uint32_t ns, double &fit, double &rmse) {
  if (s[0] == 0.0) {
    fit = 0.0;
    rmse = 0.0;
    return;
  }
  fit = s[0] / double(ns);
  rmse = sqrt(s[1] / s[0]);
}

// icp::register (icp.rs:308-356) for the pose in sh.t; every thread of the
// block calls it. On return sh.t holds the refined pose and thread 0 has
// written *out.
template <class H>
__device__ void icp_rung_block(const double4 *src, uint32_t ns, const CloudView &tgt,
                               double distance, int max_iter, IcpShared &sh, H *hint,
                               sherd_registration *out, uint32_t &status,
                               bool point_to_point = false, bool keep_hints = false) {
  if (ns == 0 || tgt.n == 0) {
    if (threadIdx.x == 0) {
      for (int k = 0; k < 16; ++k) out->transform[k] = sh.t[k];
      out->fitness = 0.0;
      out->inlier_rmse = 0.0;
      out->correspondences = 0;
      out->iterations = 0;
      out->converged = 0;
    }
    __syncthreads();
    return;
  }
  bool valid = distance > 0.0;  // a NaN radius is not valid either
  double r2 = distance * distance;
  // keep_hints: the previous rung ran over the same source and target, so its
  // last matches seed this rung's first searches (the answers do not depend on
  // the seed, only the work does).
  if (!keep_hints)
    for (uint32_t i = threadIdx.x; i < ns; i += ICP_BLOCK) hint_set(hint, i, -1);
  icp_pass(src, ns, tgt, r2, valid, sh, hint, status, point_to_point);
  double fit, rmse;
  fit_rmse(sh.sums, ns, fit, rmse);
  uint32_t iterations = 0;
  bool converged = false;
  for (int it = 0; it < max_iter; ++it) {
    if (threadIdx.x == 0) {
      if (point_to_point)
        point_step(sh);
      else
        plane_step(sh, tgt.nrm != nullptr);
    }
    __syncthreads();
    icp_pass(src, ns, tgt, r2, valid, sh, hint, status, point_to_point);
    ++iterations;
    double nfit, nrmse;
    fit_rmse(sh.sums, ns, nfit, nrmse);
    converged = fabs(nfit - fit) < 1e-6 && fabs(nrmse - rmse) < 1e-6;
    fit = nfit;
    rmse = nrmse;
    if (converged) break;
  }
  if (threadIdx.x == 0) {
    for (int k = 0; k < 16; ++k) out->transform[k] = sh.t[k];
    out->fitness = fit;
    out->inlier_rmse = rmse;
    out->correspondences = (unsigned long long)sh.sums[0];
    out->iterations = iterations;
    out->converged = converged ? 1u : 0u;
  }
  __syncthreads();
}

}  // namespace sherd
