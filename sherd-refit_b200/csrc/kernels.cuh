// kernels.cuh — the __global__ entry points of the backend.
#pragma once

#include "verify.cuh"

namespace sherd {

struct Pose16 {
  double m[16];
};

// ---- Executor-shaped batch kernels (one thread per query) -------------------

__global__ void k_first_hit(MeshView m, const float *org, const float *dir, uint32_t n, float *t,
                            uint32_t *prim, uint32_t *status) {
  uint32_t st = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    F3 o = {org[3 * i], org[3 * i + 1], org[3 * i + 2]};
    F3 d = {dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]};
    first_hit(m, o, d, t[i], prim[i], st);
  }
  if (st) atomicOr(status, st);
}

__global__ void k_bounded_all(MeshView m, const double *pts, uint32_t n, Pose16 pose, float window,
                              double *out, uint32_t *status) {
  uint32_t st = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double x, y, z;
    apply_pose(pose.m, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], x, y, z);
    float d = mesh_distance(m, {float(x), float(y), float(z)}, window, st);
    out[i] = d == f_inf() ? d_inf() : double(d);
  }
  if (st) atomicOr(status, st);
}

// DistReduce::Min: every query searches with the best distance so far as its
// window; the minimum is order-independent, so this is the CPU's scan.
__global__ void k_bounded_min(MeshView m, const double *pts, uint32_t n, Pose16 pose,
                              unsigned *best_key, uint32_t *status) {
  uint32_t st = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double x, y, z;
    apply_pose(pose.m, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], x, y, z);
    float window = key2f(*((volatile unsigned *)best_key));
    float d = mesh_distance(m, {float(x), float(y), float(z)}, window, st);
    if (d != f_inf()) atomicMin(best_key, f2key(d));
  }
  if (st) atomicOr(status, st);
}

__global__ void k_inside(MeshView m, const double *pts, uint32_t n, Pose16 pose,
                         sherd_inside_outcome *out, uint32_t *status) {
  uint32_t st = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double x, y, z;
    apply_pose(pose.m, pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], x, y, z);
    F3 p = {float(x), float(y), float(z)};
    sherd_inside_outcome o = {0.0f, 0u};
    bool in_box = !(p.x < m.lo[0] || p.x > m.hi[0] || p.y < m.lo[1] || p.y > m.hi[1] ||
                    p.z < m.lo[2] || p.z > m.hi[2]);
    if (in_box && inside_mesh(m, p, st)) o = {mesh_distance(m, p, f_inf(), st), 1u};
    out[i] = o;
  }
  if (st) atomicOr(status, st);
}

__global__ void k_nn_within(CloudView c, const double *q, uint32_t n, double r2, uint32_t *idx,
                            double *d2, uint32_t *status) {
  uint32_t st = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double best;
    int s = nearest_within_sq(c, q[3 * i], q[3 * i + 1], q[3 * i + 2], r2, best, st);
    idx[i] = s < 0 ? MISS : uint32_t(c.pts[s].w);
    d2[i] = s < 0 ? d_inf() : best;
  }
  if (st) atomicOr(status, st);
}

__global__ void k_nn_below(CloudView c, const double *q, uint32_t n, double bound, uint32_t *idx,
                           double *dist, uint32_t *status) {
  uint32_t st = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d = 0.0;
    int s = nearest_below(c, q[3 * i], q[3 * i + 1], q[3 * i + 2], bound, d, st);
    idx[i] = s < 0 ? MISS : uint32_t(c.pts[s].w);
    dist[i] = s < 0 ? d_inf() : d;
  }
  if (st) atomicOr(status, st);
}

// ---- preprocessing rays -------------------------------------------------------

// mesh::geometry::face_geometry (mesh/geometry.rs:70-96).
__global__ void k_face_geometry(const double *v, const uint32_t *f, uint32_t nf, double *normals,
                                double *areas, double *centroids) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nf) return;
  const double *a = v + 3 * size_t(f[3 * i]), *b = v + 3 * size_t(f[3 * i + 1]),
               *c = v + 3 * size_t(f[3 * i + 2]);
  double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  double e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                 e1[0] * e2[1] - e1[1] * e2[0]};
  double len = sqrt((n[0] * n[0] + n[1] * n[1]) + n[2] * n[2]);
  double den = len > 1e-12 ? len : 1e-12;
  if (normals)
    for (int k = 0; k < 3; ++k) normals[3 * i + k] = n[k] / den;
  if (areas) areas[i] = 0.5 * len;
  if (centroids)
    for (int k = 0; k < 3; ++k) centroids[3 * i + k] = (a[k] + b[k] + c[k]) / 3.0;
}

// thickness::cast_inward_rays (thickness.rs:115-132) fused with the filter of
// thickness_from_hits (thickness.rs:139-162, looking_back 185-204): valid hit
// distances are appended to ok[], the ones whose face looks back to far[].
__global__ void k_thickness_rays(MeshView m, const double *centroids, const double *normals,
                                 uint32_t nf, uint32_t stride, uint32_t n, float *t_out,
                                 uint32_t *prim_out, float *ok, float *far, unsigned *counts,
                                 uint32_t *status) {
  uint32_t st = 0;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    uint32_t face = k * stride;
    const double *c = centroids + 3 * size_t(face), *nn = normals + 3 * size_t(face);
    double d[3] = {-nn[0], -nn[1], -nn[2]};
    F3 o = {float(c[0] + d[0] * 1e-3), float(c[1] + d[1] * 1e-3), float(c[2] + d[2] * 1e-3)};
    F3 dir = {float(d[0]), float(d[1]), float(d[2])};
    float t;
    uint32_t prim;
    first_hit(m, o, dir, t, prim, st);
    if (t_out) t_out[k] = t;
    if (prim_out) prim_out[k] = prim;
    if (!(isfinite(t) && prim < nf)) continue;
    ok[atomicAdd(&counts[0], 1u)] = t;
    const double *hit = normals + 3 * size_t(prim);
    double dd = -((hit[0] * nn[0] + hit[1] * nn[1]) + hit[2] * nn[2]);
    if (dd > 0.7) far[atomicAdd(&counts[1], 1u)] = t;
  }
  if (st) atomicOr(status, st);
}

// The same filter over given hits (the injected mode).
__global__ void k_thickness_filter(const double *normals, uint32_t nf, const uint32_t *idx,
                                   const float *t_hit, const uint32_t *prim, uint32_t n, float *ok,
                                   float *far, unsigned *counts) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    float t = t_hit[k];
    uint32_t p = prim[k];
    if (!(isfinite(t) && p < nf)) continue;
    ok[atomicAdd(&counts[0], 1u)] = t;
    const double *hit = normals + 3 * size_t(p), *from = normals + 3 * size_t(idx[k]);
    double dd = -((hit[0] * from[0] + hit[1] * from[1]) + hit[2] * from[2]);
    if (dd > 0.7) far[atomicAdd(&counts[1], 1u)] = t;
  }
}

// thickness::hist_mode (thickness.rs:212-262) over an ascending array, in one
// block: numpy's percentile(90) interpolation in the array's dtype, 60 equal
// bins over [0, p90] with numpy's edge corrections, the first fullest bin.
__global__ void k_hist_mode(const float *sorted, uint32_t n, float *out) {
  __shared__ unsigned counts[60];
  __shared__ float edges[61];
  __shared__ float range[2];
  if (threadIdx.x < 60) counts[threadIdx.x] = 0;
  if (threadIdx.x == 0) {
    float p90;
    if (n == 1) {
      p90 = sorted[0];
    } else {
      double vi = double(n - 1) * (90.0 / 100.0);
      double prev = floor(vi);
      uint32_t i = uint32_t(prev);
      double gamma = vi - prev;
      float a = sorted[i], b = sorted[i + 1 < n ? i + 1 : n - 1];
      float diff = b - a;
      p90 = gamma >= 0.5 ? b - diff * float(1.0 - gamma) : a + diff * float(gamma);
    }
    float first = 0.0f, last = p90;
    if (p90 == 0.0f) {
      first = -0.5f;
      last = 0.5f;
    }
    float step = (last - first) / 60.0f;
    for (int k = 0; k <= 60; ++k) edges[k] = float(k) * step + first;
    edges[60] = last;
    range[0] = first;
    range[1] = last;
  }
  __syncthreads();
  float first = range[0], last = range[1], denom = last - first;
  for (uint32_t j = threadIdx.x; j < n; j += blockDim.x) {
    float v = sorted[j];
    if (!(v >= first && v <= last)) continue;
    unsigned i = unsigned(((v - first) / denom) * 60.0f);
    if (i == 60u) i -= 1;
    if (v < edges[i]) i -= 1;
    if (i != 59u && v >= edges[i + 1]) i += 1;
    atomicAdd(&counts[i], 1u);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int k = 0;
    for (int i = 1; i < 60; ++i)
      if (counts[i] > counts[k]) k = i;
    *out = 0.5f * (edges[k] + edges[k + 1]);
  }
}

struct ConeConsts {
  double cos_a, sin_a;
  double cp[6], sp[6];
};

// segment::classify_faces (segment.rs:318-376): seven rays per face.
__global__ void k_cone_votes(MeshView m, const double *centroids, const double *normals,
                             const double *ns, const double *hit_normals, uint32_t nf, double thick,
                             ConeConsts cc, uint8_t *good, uint32_t *status) {
  uint32_t st = 0;
  float min_hit = float(0.1 * thick);
  float thick_f = float(thick);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nf; i += gridDim.x * blockDim.x) {
    const double *n = ns + 3 * size_t(i), *fnv = normals + 3 * size_t(i),
                 *c = centroids + 3 * size_t(i);
    uint8_t g = 0;
    bool finite = isfinite(n[0]) && isfinite(n[1]) && isfinite(n[2]);
    double a[3] = {1.0, 0.0, 0.0};
    if (!(fabs(n[0]) < 0.9)) {
      a[0] = 0.0;
      a[1] = 1.0;
    }
    double cr[3] = {n[1] * a[2] - n[2] * a[1], n[2] * a[0] - n[0] * a[2],
                    n[0] * a[1] - n[1] * a[0]};
    double len = sqrt((cr[0] * cr[0] + cr[1] * cr[1]) + cr[2] * cr[2]);
    if (finite && len > 0.0) {
      double e1[3] = {cr[0] / len, cr[1] / len, cr[2] / len};
      double e2[3] = {n[1] * e1[2] - n[2] * e1[1], n[2] * e1[0] - n[0] * e1[2],
                      n[0] * e1[1] - n[1] * e1[0]};
      F3 o = {float(c[0] - fnv[0] * 1e-3), float(c[1] - fnv[1] * 1e-3),
              float(c[2] - fnv[2] * 1e-3)};
      for (int k = 0; k < 7; ++k) {
        double d[3];
        if (k == 0) {
          d[0] = -n[0];
          d[1] = -n[1];
          d[2] = -n[2];
        } else {
          double cp = cc.cp[k - 1], sp = cc.sp[k - 1];
          for (int q = 0; q < 3; ++q) d[q] = -(cc.cos_a * n[q]) + cc.sin_a * (cp * e1[q] + sp * e2[q]);
        }
        F3 dir = {float(d[0]), float(d[1]), float(d[2])};
        float dh;
        uint32_t prim;
        first_hit(m, o, dir, dh, prim, st);
        if (prim == MISS) continue;
        if (!isfinite(dh) || prim >= nf || dh <= min_hit) continue;
        float ratio = dh / thick_f;
        if (ratio <= 0.5f || ratio >= 1.8f) continue;
        const double *h = hit_normals + 3 * size_t(prim);
        double al = (h[0] * d[0] + h[1] * d[1]) + h[2] * d[2];
        if (al > 0.7) ++g;
      }
    }
    good[i] = g;
  }
  if (st) atomicOr(status, st);
}

// ---- ICP -----------------------------------------------------------------------

// Executor::icp_rung: one block per candidate.
__global__ void __launch_bounds__(ICP_BLOCK, 4) k_icp_rung(const double4 *src, uint32_t ns,
                                                        CloudView tgt, const double *inits,
                                                        sherd_icp_options opt, int *hints,
                                                        sherd_registration *out, uint32_t *status) {
  __shared__ IcpShared sh;
  uint32_t st = 0;
  if (threadIdx.x < 16) {
    double v = inits[16 * blockIdx.x + threadIdx.x];
    sh.t[threadIdx.x] = v;
    // A non-finite start (which only a caller passing device-resident poses can hand over,
    // the host-buffer entry refusing it first) is reported; the rung itself stays in bounds
    // (no distance compares below a NaN radius, so it finds no correspondence).
    if (!isfinite(v)) st |= ST_RANGE;
  }
  __syncthreads();
  icp_rung_block(src, ns, tgt, opt.max_correspondence_distance, opt.max_iteration, sh,
                 hints + size_t(ns) * blockIdx.x, out + blockIdx.x, st,
                 opt.estimation == SHERD_POINT_TO_POINT);
  if (st) atomicOr(status, st);
}

// Executor::coarse_scores (cpu.rs:46-68, 136-169): one warp per pose, its
// lanes over the points, the agreeing points counted by ballot.
__global__ void k_coarse_scores(CloudView tgt, const double *pts, const double *nrm, uint32_t n,
                                const double *poses, uint32_t k, double radius,
                                double normal_agree, double *out, uint32_t *status) {
  uint32_t st = 0;
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t h = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; h < k; h += warps) {
    const double *t = poses + 16 * size_t(h);
    uint32_t agree = 0;
    for (uint32_t base = 0; base < n; base += 32) {
      uint32_t i = base + lane;
      bool ok = false;
      if (i < n) {
        double x, y, z;
        apply_pose(t, pts[3 * size_t(i)], pts[3 * size_t(i) + 1], pts[3 * size_t(i) + 2], x, y, z);
        double d;
        int s = nearest_below(tgt, x, y, z, radius, d, st);
        if (s >= 0) {
          double u, v, w;
          rotate_pose(t, nrm[3 * size_t(i)], nrm[3 * size_t(i) + 1], nrm[3 * size_t(i) + 2], u, v, w);
          double4 m = ldg4(tgt.nrm + s);
          ok = (m.x * u + m.y * v) + m.z * w > normal_agree;
        }
      }
      agree += __popc(__ballot_sync(0xFFFFFFFFu, ok));
    }
    if (lane == 0) out[h] = n ? double(agree) / double(n) : 0.0;
  }
  if (st) atomicOr(status, st);
}

// verify::penetration_share (verify.rs:509-527): points inside the mesh and
// deeper than `pen`, counted per warp by ballot.
__global__ void k_penetration_share(MeshView m, const double *pts, uint32_t n, Pose16 pose,
                                    double pen, unsigned long long *count, uint32_t *status) {
  uint32_t st = 0;
  unsigned long long mine = 0;
  for (uint32_t base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
    uint32_t i = base + threadIdx.x;
    bool deeper = false;
    if (i < n) {
      double x, y, z;
      apply_pose(pose.m, pts[3 * size_t(i)], pts[3 * size_t(i) + 1], pts[3 * size_t(i) + 2], x, y, z);
      F3 p = {float(x), float(y), float(z)};
      bool in_box = !(p.x < m.lo[0] || p.x > m.hi[0] || p.y < m.lo[1] || p.y > m.hi[1] ||
                      p.z < m.lo[2] || p.z > m.hi[2]);
      if (in_box && inside_mesh(m, p, st))
        deeper = double(mesh_distance(m, p, f_inf(), st)) > pen;
    }
    unsigned ballot = __ballot_sync(0xFFFFFFFFu, deeper);
    if ((threadIdx.x & 31) == 0) mine += __popc(ballot);
  }
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(count, mine);
  if (st) atomicOr(status, st);
}

// ---- the batched stage-2 path ----------------------------------------------------

// Resident ladder CTAs per SM a k_ladder variant's register budget is cut for
// (65536 / (ICP_BLOCK * MINB) registers a thread at most). The batch picks a
// variant per point-count bucket (the autotuner in sherd.cu); the last is the
// default.
constexpr int LADDER_VARIANTS = 3;
constexpr int LADDER_MINB[LADDER_VARIANTS] = {6, 8, 10};
// The variant a bucket runs until the autotuner has timed it (and when it has
// too few items to time): 8 CTAs per SM, which the 4-wide nearest-point walk
// made 15-20 % faster than 10 on the collection.
constexpr int LADDER_DEFAULT = 1;

struct QueueCtl {
  unsigned *head;             // next queue position to take
  const uint32_t *order;      // item indices, most expensive first
  uint32_t n;                 // queue length
  const uint32_t *abort_flag; // host-mapped; non-zero asks the kernel to stop
  unsigned long long budget_ns;
};

// Takes the next queue entry for the whole block, or returns false when the
// queue is empty, the host asked to stop or the time budget is spent.
__device__ __forceinline__ bool take(const QueueCtl &q, unsigned long long start, unsigned &slot,
                                     uint32_t &st) {
  __shared__ unsigned s_item;
  if (threadIdx.x == 0) {
    unsigned item = 0xFFFFFFFFu;
    if (q.abort_flag && *((volatile const uint32_t *)q.abort_flag)) {
      st |= ST_ABORTED;
    } else if (q.budget_ns && global_ns() - start > q.budget_ns) {
      st |= ST_TIMEOUT;
    } else {
      unsigned pos = atomicAdd(q.head, 1u);
      if (pos < q.n) item = q.order[pos];
    }
    s_item = item;
  }
  __syncthreads();
  slot = s_item;
  __syncthreads();
  return slot != 0xFFFFFFFFu;
}

// R 5.6's point-to-plane rungs r_lo..r_hi-1 of the four per (pair, start)
// (ladder.rs:142-161): from the item's start pose when r_lo is 0, else from
// its rung r_lo - 1. With skip_partial, items an early rejection left partial
// are passed over.
template <class H, int MINB>
__global__ void __launch_bounds__(ICP_BLOCK, MINB) k_ladder(const PairView *pairs,
                                                      const sherd_work_item *items, QueueCtl q,
                                                      H *hints, size_t hint_stride,
                                                      sherd_candidate *out, int r_lo, int r_hi,
                                                      int skip_partial, uint32_t *status) {
  __shared__ IcpShared sh;
  uint32_t st = 0;
  H *hint = hints + hint_stride * blockIdx.x;
  unsigned long long start = global_ns();
  unsigned it;
  while (take(q, start, it, st)) {
    const sherd_work_item &w = items[it];
    const PairView &pr = pairs[w.pair];
    sherd_candidate *c = out + it;
    if (skip_partial && c->scores.partial) continue;  // the same for the whole block
    if (threadIdx.x < 16)
      sh.t[threadIdx.x] = r_lo == 0 ? w.init[threadIdx.x] : c->rungs[r_lo - 1].transform[threadIdx.x];
    if (threadIdx.x == 0 && r_lo == 0) {
      c->pair = w.pair;
      c->start = w.start;
    }
    __syncthreads();
    const double k[4] = {0.2, 0.08, 0.08, 0.04};
    for (int r = r_lo; r < r_hi; ++r) {
      double distance = k[r] * pr.sc.t * pr.sc.icp;
      // Rungs 1 and 3 follow a rung over the same clouds (0 and 2): when that
      // rung ran in this launch, its matches are this block's hints.
      const bool keep = (r & 1) && r > r_lo;
      if (r < 2)
        icp_rung_block(pr.reg_src, pr.n_reg, pr.reg_tgt, distance, 30, sh, hint, &c->rungs[r], st,
                       false, keep);
      else
        icp_rung_block(pr.frac_src, pr.n_frac, pr.frac_tgt, distance, 30, sh, hint, &c->rungs[r],
                       st, false, keep);
    }
  }
  if (st) atomicOr(status, st);
}

// R 6 + R 6.5 at each item's rung `pose_rung` pose (verify.rs:590-638): the
// last rung, or rung 1 for R 5.6's early-rejection check (full = 0). With
// `inv` set, the penetration half is left to the wavefront kernels below and
// the inverse pose of every item is written for them. With skip_partial,
// items an early rejection left partial are passed over.
__global__ void __launch_bounds__(VER_BLOCK, 3) k_verify_items(const PairView *pairs,
                                                            const sherd_work_item *items,
                                                            QueueCtl q, sherd_params p,
                                                            unsigned *scratch, size_t stride,
                                                            sherd_candidate *out, int full,
                                                            double *inv, int pose_rung,
                                                            int skip_partial, uint32_t *status) {
  __shared__ VerShared sh;
  uint32_t st = 0;
  unsigned long long start = global_ns();
  unsigned *mine = scratch + stride * blockIdx.x;
  unsigned it;
  while (take(q, start, it, st)) {
    const PairView &pr = pairs[items[it].pair];
    sherd_candidate *c = out + it;
    if (skip_partial && c->scores.partial) continue;  // the same for the whole block
    if (threadIdx.x < 16) sh.t[threadIdx.x] = c->rungs[pose_rung].transform[threadIdx.x];
    __syncthreads();
    if (pr.scratch_floats > stride) {
      if (threadIdx.x == 0) {
        st |= ST_SCRATCH;
        c->status = uint32_t(-SHERD_E_INVALID);
      }
      __syncthreads();
      continue;
    }
    verify_block(pr, full != 0, p, mine, sh, &c->scores, &c->accepted, st, inv == nullptr,
                 inv ? inv + 16 * size_t(it) : nullptr);
  }
  if (st) atomicOr(status, st);
}

// R 5.6's early rejection (pair.rs:315-340) after the fracture and seam
// scores at rung 1: an item below the tight limit keeps those partial scores,
// is rejected, and its pc_frac rungs stay unrun (the rung-1 pose, zero
// counts); the others are cleared to go on.
__global__ void k_early_mark(sherd_candidate *cands, const uint32_t *order, uint32_t n,
                             double limit) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  sherd_candidate &c = cands[order[k]];
  if (c.status) return;
  if (c.scores.tight < limit) {
    for (int r = 2; r < 4; ++r) {
      sherd_registration &g = c.rungs[r];
      for (int k = 0; k < 16; ++k) g.transform[k] = c.rungs[1].transform[k];
      g.fitness = 0.0;
      g.inlier_rmse = 0.0;
      g.correspondences = 0;
      g.iterations = 0;
      g.converged = 0;
    }
    c.accepted = 0;
  } else {
    c.scores.partial = 0;
  }
}

// ---- the penetration wavefront of the batched path ------------------------------
//
// R 6.4 for every (item, side) of a batch at once: side 0 is B's surface
// samples moved by T against A's mesh, side 1 A's moved by T^-1 against B's.
// The samples of all units are one flat list of 32-point chunks that warps
// take from a global counter, so no block ever waits at a barrier for its
// slowest lane. Each warp keeps two shared queues: the points of its chunks
// that fall in the mesh's box, and the ones the parity test calls inside; a
// queue is drained 32 entries at a time, so the parity and depth queries run
// with every lane of the warp busy. A unit's count, deepest depth and minimum
// distance are combined with global atomics, which makes them independent of
// the order the points are taken in, as R 6.4's statistics are.

struct PenState {
  unsigned *deeper;    // per unit: points deeper than sc.pen
  unsigned *deep;      // per unit: f2key(deepest depth) + 1, 0 when nothing is inside
  unsigned *best;      // per unit: f2key(smallest distance) for the nothing-inside case
  const uint32_t *chunk0;  // per unit: its first chunk in the flat list (n_units + 1)
  const uint32_t *coarse;  // the unit of every 256th chunk (chunk k << 8)
  uint32_t n_units, n_chunks;
};

struct PenUnit {
  const double4 *pts;
  uint32_t n;
  const MeshView *mesh;
  const double *pose;
  double pen;
  bool avail;
};

__device__ __forceinline__ PenUnit pen_unit(const PairView *pairs, const sherd_work_item *items,
                                            const sherd_candidate *cands, const double *inv,
                                            uint32_t u) {
  uint32_t item = u >> 1, side = u & 1u;
  const PairView &pr = pairs[items[item].pair];
  PenUnit x;
  x.avail = pr.a.has_mesh && pr.b.has_mesh && pr.a.watertight && pr.b.watertight &&
            !cands[item].scores.partial;
  x.pts = side ? pr.a.s : pr.b.s;
  x.n = side ? pr.a.n_s : pr.b.n_s;
  x.mesh = side ? &pr.b.mesh : &pr.a.mesh;
  x.pose = side ? inv + 16 * size_t(item) : cands[item].rungs[3].transform;
  x.pen = pr.sc.pen;
  return x;
}

// The unit a chunk belongs to: the unit of the last 256-chunk mark before it,
// then forward over the units that start at or before it (units without
// chunks included).
__device__ __forceinline__ uint32_t unit_of_chunk(const PenState &ps, uint32_t chunk) {
  uint32_t u = __ldg(ps.coarse + (chunk >> 8));
  while (__ldg(ps.chunk0 + u + 1) <= chunk) ++u;
  return u;
}

struct WarpQueue {
  unsigned long long box[64];
  unsigned long long in[64];
  int n_box, n_in;
};

__device__ __forceinline__ void wq_push(unsigned long long *q, int *count, bool pred,
                                        unsigned long long v) {
  unsigned mask = __ballot_sync(0xffffffffu, pred);
  int lane = threadIdx.x & 31;
  int base = *count;
  if (pred) q[base + __popc(mask & ((1u << lane) - 1u))] = v;
  __syncwarp();
  if (lane == 0) *count = base + __popc(mask);
  __syncwarp();
}

// Pops up to 32 entries; returns whether this lane got one.
__device__ __forceinline__ bool wq_pop(unsigned long long *q, int *count, unsigned long long &v) {
  int lane = threadIdx.x & 31;
  int n = *count;
  int take = n < 32 ? n : 32;
  bool got = lane < take;
  if (got) v = q[n - take + lane];
  __syncwarp();
  if (lane == 0) *count = n - take;
  __syncwarp();
  return got;
}

// Takes the next chunk for the warp. The abort flag lives in host-mapped
// memory, a round trip over the bus, so a warp polls it (and the time budget)
// only every 128 chunks it takes.
__device__ __forceinline__ bool take_chunk(unsigned *head, uint32_t n_chunks,
                                           const uint32_t *abort_flag, unsigned long long budget,
                                           unsigned long long start, uint32_t &taken,
                                           uint32_t &chunk, uint32_t &st) {
  uint32_t c = 0xFFFFFFFFu;
  if ((threadIdx.x & 31) == 0) {
    bool stop = false;
    if ((taken++ & 127u) == 0u) {
      if (abort_flag && *((volatile const uint32_t *)abort_flag)) {
        st |= ST_ABORTED;
        stop = true;
      } else if (budget && global_ns() - start > budget) {
        st |= ST_TIMEOUT;
        stop = true;
      }
    }
    if (!stop) c = atomicAdd(head, 1u);
  }
  chunk = __shfl_sync(0xffffffffu, c, 0);
  return chunk < n_chunks;
}

// k_pen_inside takes its chunks in runs: CHUNK_RUN consecutive chunks (of
// one unit, mostly) per atomic, the unit of each following from the previous
// one. A unit is then shared by a few dozen warps rather than hundreds, so the
// running deepest depth its points are checked against is known early, and
// few points need their depth searched exactly.
#ifndef PEN_CHUNK_RUN
#define PEN_CHUNK_RUN 64
#endif
constexpr uint32_t CHUNK_RUN = PEN_CHUNK_RUN;

struct ChunkRun {
  uint32_t next = 0, end = 0;       // chunks [next, end) still to do
  uint32_t unit = 0, unit_end = 0;  // the unit of `next` and the first chunk after it
  uint32_t taken = 0;               // runs taken (the abort flag is polled every 8)
};

__device__ __forceinline__ bool next_chunk(ChunkRun &r, const PenState &ps, unsigned *head,
                                           const uint32_t *abort_flag, unsigned long long budget,
                                           unsigned long long start, uint32_t &chunk, uint32_t &u,
                                           uint32_t &st) {
  if (r.next >= r.end) {
    uint32_t c = 0xFFFFFFFFu;
    if ((threadIdx.x & 31) == 0) {
      bool stop = false;
      if ((r.taken++ & 7u) == 0u) {
        if (abort_flag && *((volatile const uint32_t *)abort_flag)) {
          st |= ST_ABORTED;
          stop = true;
        } else if (budget && global_ns() - start > budget) {
          st |= ST_TIMEOUT;
          stop = true;
        }
      }
      if (!stop) c = atomicAdd(head, CHUNK_RUN);
    }
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= ps.n_chunks) return false;
    r.next = c;
    r.end = min(c + CHUNK_RUN, ps.n_chunks);
    r.unit = unit_of_chunk(ps, c);
    r.unit_end = __ldg(ps.chunk0 + r.unit + 1);
  }
  chunk = r.next++;
  while (chunk >= r.unit_end) {
    ++r.unit;
    r.unit_end = __ldg(ps.chunk0 + r.unit + 1);
  }
  u = r.unit;
  return true;
}

__device__ __forceinline__ F3 unit_point(const PenUnit &x, uint32_t i) {
  double4 q = ldg4(x.pts + i);
  double a, b, c;
  apply_pose(x.pose, q.x, q.y, q.z, a, b, c);
  return {float(a), float(b), float(c)};
}

// The +axis ray parity of every active lane's point (RayScene::crossings,
// spatial/bvh.rs:160-175, under crossings_axis's rule), the 32 lanes sharing
// the work: each lane's grid cell is a run of entries, the runs of the warp are
// laid end to end (a prefix sum of their lengths), and every round each lane
// tests the next entry of that flattened list for its owner (the last lane
// whose run starts at or before it). Rounds therefore keep every lane busy
// however unevenly the cells are filled, and the lanes of one owner read its
// run's rectangles as consecutive, coalesced loads. A crossing toggles the
// owner's bit in the warp's parity word; `axis` is the same for the warp.
__device__ __forceinline__ uint32_t warp_crossings(const MeshView *m, F3 p, int axis, bool active,
                                                   unsigned *par_word) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  uint32_t b = 0, len = 0;
  unsigned long long rect = 0, tri = 0;
  if (active && m->nf) {
    const AxisGrid &g = m->grid[axis];
    float pc[3] = {p.x, p.y, p.z};
    float pu = pc[(axis + 1) % 3], pv = pc[(axis + 2) % 3];
    float fu = floorf((pu - g.lo_u) * g.inv_cell), fv = floorf((pv - g.lo_v) * g.inv_cell);
    if (fu >= 0.0f && fv >= 0.0f && fu < float(g.nu) && fv < float(g.nv)) {
      size_t cell = size_t(fu) * g.nv + size_t(fv);
      b = __ldg(g.start + cell);
      len = __ldg(g.start + cell + 1) - b;
      rect = reinterpret_cast<unsigned long long>(g.rect);
      tri = reinterpret_cast<unsigned long long>(g.tri);
    }
  }
  uint32_t incl = len;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(FULL, incl, o);
    if (lane >= o) incl += y;
  }
  const uint32_t off = incl - len, total = __shfl_sync(FULL, incl, 31);
  if (lane == 0) *par_word = 0u;
  __syncwarp();
  const F3 d = {axis == 0 ? 1.0f : 0.0f, axis == 1 ? 1.0f : 0.0f, axis == 2 ? 1.0f : 0.0f};
  for (uint32_t base = 0; base < total; base += 32) {
    const uint32_t w = base + lane;
    int j = 0;  // the last lane whose run starts at or before w (off[0] = 0 <= w)
#pragma unroll
    for (int step = 16; step; step >>= 1)
      if (__shfl_sync(FULL, off, j + step) <= w) j += step;
    const float qx = __shfl_sync(FULL, p.x, j), qy = __shfl_sync(FULL, p.y, j),
                qz = __shfl_sync(FULL, p.z, j);
    const uint32_t bj = __shfl_sync(FULL, b, j), oj = __shfl_sync(FULL, off, j);
    const float4 *rj = reinterpret_cast<const float4 *>(__shfl_sync(FULL, rect, j));
    const float4 *tj = reinterpret_cast<const float4 *>(__shfl_sync(FULL, tri, j));
    if (w < total) {
      const size_t k = size_t(bj) + (w - oj);
      const float qc[3] = {qx, qy, qz};
      const float qu = qc[(axis + 1) % 3], qv = qc[(axis + 2) % 3];
      const float4 r = __ldg(rj + k);
      if (!(qu < r.x || qu > r.y || qv < r.z || qv > r.w)) {
        const float4 t0 = __ldg(tj + 3 * k), t1 = __ldg(tj + 3 * k + 1), t2 = __ldg(tj + 3 * k + 2);
        if (moller_trumbore_edges({qx, qy, qz}, d, {t0.x, t0.y, t0.z}, {t1.x, t1.y, t1.z},
                                  {t2.x, t2.y, t2.z}) >= 0.0f)
          atomicXor(par_word, 1u << j);
      }
    }
  }
  __syncwarp();
  const uint32_t bits = *par_word;
  __syncwarp();
  return (bits >> lane) & 1u;
}

// RayScene::inside (spatial/bvh.rs:146-157) for every lane's point at once, by
// warp_crossings: the majority of the three parities, the third ray cast only
// for the lanes whose first two disagree.
__device__ __forceinline__ bool warp_inside(const MeshView *m, F3 p, bool active,
                                            unsigned *par_word) {
  const uint32_t a = warp_crossings(m, p, 0, active, par_word);
  const uint32_t b = warp_crossings(m, p, 1, active, par_word);
  const bool third = active && a != b;
  uint32_t c = 0;
  if (__any_sync(0xffffffffu, third)) c = warp_crossings(m, p, 2, third, par_word);
  return active && (a == b ? a != 0u : c != 0u);
}

__global__ void k_pen_init(PenState ps) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < ps.n_units; u += gridDim.x * blockDim.x) {
    ps.deeper[u] = 0;
    ps.deep[u] = 0;
    ps.best[u] = f2key(3.4028234663852886e38f);
  }
}

// Box test, parity, depth: the first pass of one_penetration (verify.rs:541-568).
__global__ void __launch_bounds__(256, PEN_INSIDE_MINB) k_pen_inside(const PairView *pairs, const sherd_work_item *items,
                                                    const sherd_candidate *cands, const double *inv,
                                                    PenState ps, unsigned *head,
                                                    const uint32_t *abort_flag,
                                                    unsigned long long budget, uint32_t *status) {
  __shared__ WarpQueue wqs[8];
  __shared__ unsigned parity[8];
  WarpQueue &q = wqs[threadIdx.x >> 5];
  unsigned *par_word = parity + (threadIdx.x >> 5);
  int lane = threadIdx.x & 31;
  if (lane == 0) q.n_box = q.n_in = 0;
  __syncwarp();
  uint32_t st = 0;
  unsigned long long start = global_ns();
  // An inside point's depth D (its distance to the mesh) enters the unit's
  // statistics twice: whether D > pen, and the unit's deepest D. Both are
  // exact without the full nearest-face search of every point. With w the
  // largest f32 <= pen (so D > pen exactly when D > w): the bound grid or a
  // walk that stops at the first face within w decides "deeper"; then the
  // point can only raise the running maximum M if no face lies within M, and
  // only then is D itself searched (within w when not deeper, unbounded
  // otherwise; the same value mesh_distance gives). M only ever holds depths
  // of inside points, so the last point to raise it holds the true maximum.
  auto depth_stage = [&](bool drain) {
    while (q.n_in >= 32 || (drain && q.n_in > 0)) {
      unsigned long long e;
      if (wq_pop(q.in, &q.n_in, e)) {
        uint32_t u = uint32_t(e >> 32), i = uint32_t(e);
        PenUnit x = pen_unit(pairs, items, cands, inv, u);
        const MeshView &m = *x.mesh;
        F3 p = unit_point(x, i);
        const float w = __double2float_rd(x.pen);
        const bool deeper = !(mesh_may_reach(m, p, w) && mesh_any_within(m, p, w, st));
        if (deeper) atomicAdd(&ps.deeper[u], 1u);
        const unsigned key = *((volatile unsigned *)&ps.deep[u]);
        bool raise = true;
        if (key != 0u) {
          const float top = key2f(key - 1u);
          if (!deeper && top >= w)
            raise = false;  // D <= w <= M
          else if (mesh_may_reach(m, p, top) && mesh_any_within(m, p, top, st))
            raise = false;  // D <= M
        }
        if (raise) {
          float depth = mesh_distance(m, p, deeper ? f_inf() : w, st);
          atomicMax(&ps.deep[u], f2key(depth) + 1u);
        }
      }
    }
  };
  auto parity_stage = [&](bool drain) {
    while (q.n_box >= 32 || (drain && q.n_box > 0)) {
      unsigned long long e = 0;
      bool got = wq_pop(q.box, &q.n_box, e);
      F3 p = {0.0f, 0.0f, 0.0f};
      const MeshView *m = nullptr;
      if (got) {
        uint32_t u = uint32_t(e >> 32), i = uint32_t(e);
        PenUnit x = pen_unit(pairs, items, cands, inv, u);
        p = unit_point(x, i);
        m = x.mesh;
      }
      bool inside = warp_inside(m, p, got, par_word);
      wq_push(q.in, &q.n_in, inside, e);
      depth_stage(false);
    }
  };
  ChunkRun run;
  uint32_t chunk, u;
  while (next_chunk(run, ps, head, abort_flag, budget, start, chunk, u, st)) {
    PenUnit x = pen_unit(pairs, items, cands, inv, u);
    uint32_t i = (chunk - ps.chunk0[u]) * 32u + lane;
    bool in_box = false;
    if (x.avail && i < x.n) {
      F3 p = unit_point(x, i);
      const MeshView &m = *x.mesh;
      in_box = !(p.x < m.lo[0] || p.x > m.hi[0] || p.y < m.lo[1] || p.y > m.hi[1] ||
                 p.z < m.lo[2] || p.z > m.hi[2]);
    }
    wq_push(q.box, &q.n_box, in_box, (unsigned long long)u << 32 | i);
    parity_stage(false);
  }
  parity_stage(true);
  depth_stage(true);
  if (st) atomicOr(status, st);
}

// The nothing-inside case (verify.rs:569-579): 32 points spread over each such
// unit seed its shrinking window with unbounded queries.
__global__ void k_pen_seed(const PairView *pairs, const sherd_work_item *items,
                           const sherd_candidate *cands, const double *inv, PenState ps,
                           uint32_t *status) {
  uint32_t st = 0;
  uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t u = warp; u < ps.n_units; u += warps) {
    PenUnit x = pen_unit(pairs, items, cands, inv, u);
    if (!x.avail || x.n == 0 || ps.deep[u] != 0) continue;
    if (lane < x.n) {
      uint32_t i = uint32_t((unsigned long long)lane * x.n / 32u);
      float window = key2f(*((volatile unsigned *)&ps.best[u]));
      float d = mesh_distance(*x.mesh, unit_point(x, i), window, st);
      if (d != f_inf()) atomicMin(&ps.best[u], f2key(d));
    }
  }
  if (st) atomicOr(status, st);
}

// The shrinking-window scan over every point of the nothing-inside units; a
// point farther from the mesh's box than the window cannot beat it.
__global__ void __launch_bounds__(256) k_pen_min(const PairView *pairs, const sherd_work_item *items,
                                                 const sherd_candidate *cands, const double *inv,
                                                 PenState ps, unsigned *head,
                                                 const uint32_t *abort_flag,
                                                 unsigned long long budget, uint32_t *status) {
  __shared__ WarpQueue wqs[8];
  WarpQueue &q = wqs[threadIdx.x >> 5];
  int lane = threadIdx.x & 31;
  if (lane == 0) q.n_box = q.n_in = 0;
  __syncwarp();
  uint32_t st = 0;
  unsigned long long start = global_ns();
  auto query_stage = [&](bool drain) {
    while (q.n_box >= 32 || (drain && q.n_box > 0)) {
      unsigned long long e;
      if (wq_pop(q.box, &q.n_box, e)) {
        uint32_t u = uint32_t(e >> 32), i = uint32_t(e);
        PenUnit x = pen_unit(pairs, items, cands, inv, u);
        float window = key2f(*((volatile unsigned *)&ps.best[u]));
        float d = mesh_distance(*x.mesh, unit_point(x, i), window, st);
        if (d != f_inf()) atomicMin(&ps.best[u], f2key(d));
      }
    }
  };
  uint32_t chunk, taken = 0;
  while (take_chunk(head, ps.n_chunks, abort_flag, budget, start, taken, chunk, st)) {
    uint32_t u = unit_of_chunk(ps, chunk);
    PenUnit x = pen_unit(pairs, items, cands, inv, u);
    uint32_t i = (chunk - ps.chunk0[u]) * 32u + lane;
    bool want = false;
    if (x.avail && i < x.n && ps.deep[u] == 0) {
      F3 p = unit_point(x, i);
      float pc[3] = {p.x, p.y, p.z};
      float window = key2f(*((volatile unsigned *)&ps.best[u]));
      float gap = sqrtf(box_dist2(x.mesh->lo, x.mesh->hi, pc));
      // The window only shrinks, so a point the bound grid puts out of reach
      // now stays out of reach when its query would run.
      want = !(gap > window + 1e-5f * window + x.mesh->pad) && mesh_may_reach(*x.mesh, p, window);
    }
    wq_push(q.box, &q.n_box, want, (unsigned long long)u << 32 | i);
    query_stage(false);
  }
  query_stage(true);
  if (st) atomicOr(status, st);
}

// penetration_scores (verify.rs:483-498) from the two units of each item, and
// the verdict (verify.rs:632-638).
__global__ void k_pen_finalize(const PairView *pairs, const sherd_work_item *items,
                               sherd_candidate *cands, PenState ps, sherd_params p, uint32_t n_items) {
  uint32_t it = blockIdx.x * blockDim.x + threadIdx.x;
  if (it >= n_items) return;
  const PairView &pr = pairs[items[it].pair];
  sherd_candidate &c = cands[it];
  if (c.status || c.scores.partial) return;  // an early rejection's scores are final
  sherd_scores &s = c.scores;
  bool avail = pr.a.has_mesh && pr.b.has_mesh && pr.a.watertight && pr.b.watertight;
  if (avail) {
    double frac[2], mins[2];
    for (int side = 0; side < 2; ++side) {
      uint32_t u = 2 * it + side;
      uint32_t n = side ? pr.a.n_s : pr.b.n_s;
      if (n == 0) {
        frac[side] = 0.0;
        mins[side] = 0.0;
        continue;
      }
      frac[side] = double(ps.deeper[u]) / double(n);
      mins[side] = ps.deep[u] ? -double(key2f(ps.deep[u] - 1u)) : double(key2f(ps.best[u]));
    }
    // side 0 is pen_b / min_b, side 1 pen_a / min_a
    s.pen = fmax(frac[1], frac[0]);
    s.pen_depth = fmax(-mins[1], -mins[0]) / pr.sc.t;
  }
  const sherd_scales &sc = pr.sc;
  c.accepted = (s.tight >= p.min_tight && s.gap * sc.t <= sc.gap && s.pen <= p.max_pen &&
                s.seam >= p.min_seam && s.cont_n >= p.min_cont_n)
                   ? 1u
                   : 0u;
}

}  // namespace sherd
