// verify.cuh — R 6's verification of one candidate pose as a CTA-cooperative
// routine (matching/verify.rs:318-638).
//
// Every score is computed on the device from the fragments' resident BVHs:
//   tight/gap/contact  bounded point-to-fracture distances of both sample sets
//                      (the window is sc.facing), integer counts, and the
//                      median of the facing distances by a block radix select
//                      on the f32 bit patterns (numpy's even-n midpoint in f64);
//   seam               for each of A's breakline points the nearest point of B's
//                      breakline moved by the pose, found through a tree over
//                      B's breakline in B's own frame and re-measured exactly in
//                      A's frame, then a bitmap of A's t/3 voxels;
//   cont/cont_n        nearest A margin point of each moved B margin point and
//                      two radix-select medians over f64 keys;
//   pen/pen_depth      AABB reject, three axis parities, the depth of inside
//                      points, and the shrinking-window minimum distance when
//                      nothing is inside (a block atomicMin on the f32 bits).
#pragma once

#include "icp.cuh"

namespace sherd {

constexpr int VER_BLOCK = 256;

// Query arrays (pf, s, and the trees' own sorted points when a breakline or a
// margin is the querying side) are in Morton order, so the 32 queries of a warp
// are neighbours and traverse the same nodes. Every statistic R 6 takes over
// them (counts, extrema, medians, a voxel set) is independent of their order.
// Arrays a tree answers with (brk_p/brk_ns, margin_p/margin_n) stay in the
// caller's order, because the lowest-index tie rule is stated on that order.
struct SurfView {
  MeshView frac;
  MeshView mesh;
  uint32_t has_mesh, watertight;
  double frac_area;
  const double4 *pf;  // Morton order, w = original index
  uint32_t n_pf;
  const double4 *s;   // Morton order, w = original index
  uint32_t n_s;
  const double *brk_p;
  const double *brk_ns;
  uint32_t n_brk;
  CloudView brk_tree;  // over brk_p in this fragment's own frame
  const double *margin_p;
  const double *margin_n;
  uint32_t n_margin;
  CloudView margin_tree;
};

struct PairView {
  SurfView a, b;
  CloudView reg_tgt, frac_tgt;
  const double4 *reg_src;
  uint32_t n_reg;
  const double4 *frac_src;
  uint32_t n_frac;
  sherd_scales sc;
  const uint32_t *a_cell;  // dense id of floor(A.brk_p / (t/3)) per A breakline point
  uint32_t n_cells;
  uint32_t scratch_floats;  // per-item scratch this pair needs, in 4-byte words
};

constexpr int MAX_CELL_WORDS = 2048;  // bitmap of up to 65 536 seam voxels
constexpr int PEN_CHUNK = 1024;       // sample points per compaction round

struct VerShared {
  unsigned q_box[PEN_CHUNK];  // points of a round inside the mesh's box
  unsigned q_in[PEN_CHUNK];   // ... and inside the mesh
  unsigned n_box, n_in;
  double inv[16];
  double t[16];
  unsigned hist[256];
  unsigned long long prefix;
  unsigned kk;
  unsigned cnt[8];
  unsigned best_key;
  unsigned deep_key;
  unsigned cells[MAX_CELL_WORDS];
};

// icp.rs's pose_inverse twin: verify::pose_inverse (verify.rs:739-798).
__device__ void pose_inverse(const double *t, double *out) {
  double m[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) m[i][j] = t[4 * i + j];
  int piv[4] = {0, 1, 2, 3};
  for (int k = 0; k < 4; ++k) {
    int best = k;
    for (int i = k + 1; i < 4; ++i)
      if (fabs(m[i][k]) > fabs(m[best][k])) best = i;
    if (best != k) {
      for (int c = 0; c < 4; ++c) {
        double x = m[k][c];
        m[k][c] = m[best][c];
        m[best][c] = x;
      }
      int x = piv[k];
      piv[k] = piv[best];
      piv[best] = x;
    }
    double pivot = m[k][k];
    if (pivot == 0.0) continue;
    for (int r = k + 1; r < 4; ++r) {
      m[r][k] /= pivot;
      double factor = m[r][k];
      for (int c = k + 1; c < 4; ++c) m[r][c] -= factor * m[k][c];
    }
  }
  for (int col = 0; col < 4; ++col) {
    double y[4], x[4];
    for (int i = 0; i < 4; ++i) {
      double acc = 0.0;
      for (int j = 0; j < i; ++j) acc += m[i][j] * y[j];
      y[i] = (piv[i] == col ? 1.0 : 0.0) - acc;
    }
    for (int i = 3; i >= 0; --i) {
      double acc = 0.0;
      for (int j = i + 1; j < 4; ++j) acc += m[i][j] * x[j];
      x[i] = (y[i] - acc) / m[i][i];
    }
    for (int r = 0; r < 4; ++r) out[4 * r + col] = x[r];
  }
}

__device__ __forceinline__ F3 narrow3(double x, double y, double z) {
  return {float(x), float(y), float(z)};
}

// The k-th smallest of n keys (k < n), by 8-bit radix digits over the block.
template <typename K, int BITS>
__device__ K block_select(const K *keys, uint32_t n, uint32_t k, VerShared &sh) {
  if (threadIdx.x == 0) {
    sh.prefix = 0;
    sh.kk = k;
  }
  __syncthreads();
  unsigned long long mask = 0;
  for (int shift = BITS - 8; shift >= 0; shift -= 8) {
    for (int b = threadIdx.x; b < 256; b += blockDim.x) sh.hist[b] = 0;
    __syncthreads();
    unsigned long long prefix = sh.prefix;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
      unsigned long long key = (unsigned long long)keys[i];
      if ((key & mask) == prefix) atomicAdd(&sh.hist[(key >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      unsigned kk = sh.kk, cum = 0;
      int b = 0;
      for (; b < 255; ++b) {
        if (cum + sh.hist[b] > kk) break;
        cum += sh.hist[b];
      }
      sh.kk = kk - cum;
      sh.prefix = prefix | ((unsigned long long)b << shift);
    }
    mask |= 255ULL << shift;
    __syncthreads();
  }
  return K(sh.prefix);
}

// numpy's median of n f32 values held as their bit patterns (all >= 0).
__device__ double median_f32(const unsigned *keys, uint32_t n, VerShared &sh) {
  if (n % 2 == 1) return double(key2f(block_select<unsigned, 32>(keys, n, n / 2, sh)));
  double lo = double(key2f(block_select<unsigned, 32>(keys, n, n / 2 - 1, sh)));
  double hi = double(key2f(block_select<unsigned, 32>(keys, n, n / 2, sh)));
  return (lo + hi) / 2.0;
}

// numpy's median of n f64 values held as order-preserving keys.
__device__ double median_f64(const unsigned long long *keys, uint32_t n, VerShared &sh) {
  if (n % 2 == 1) return key2d(block_select<unsigned long long, 64>(keys, n, n / 2, sh));
  double lo = key2d(block_select<unsigned long long, 64>(keys, n, n / 2 - 1, sh));
  double hi = key2d(block_select<unsigned long long, 64>(keys, n, n / 2, sh));
  return (lo + hi) / 2.0;
}

// verify::one_side (verify.rs:338-349) for `pts` moved by `pose` against the
// other fragment's fracture scene.
__device__ __noinline__ void one_side(const double4 *pts, uint32_t n, const double *pose, const MeshView &scene,
                         double area, const sherd_scales &sc, unsigned *scratch, VerShared &sh,
                         double &tight, double &gap, double &contact, uint32_t &status) {
  if (threadIdx.x < 3) sh.cnt[threadIdx.x] = 0;
  __syncthreads();
  float window = float(sc.facing);
  unsigned facing = 0, tight_n = 0, touching = 0;
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
    double4 q = ldg4(pts + i);
    double x, y, z;
    apply_pose(pose, q.x, q.y, q.z, x, y, z);
    float d = mesh_distance(scene, narrow3(x, y, z), window, status);
    double dd = d == f_inf() ? d_inf() : double(d);
    if (dd < 2.0 * sc.tight) ++touching;
    if (dd < sc.facing) {
      ++facing;
      if (dd < sc.tight) ++tight_n;
      unsigned slot = atomicAdd(&sh.cnt[0], 1u);
      scratch[slot] = f2key(d);
    }
  }
  atomicAdd(&sh.cnt[1], tight_n);
  atomicAdd(&sh.cnt[2], touching);
  __syncthreads();
  unsigned nf = sh.cnt[0], nt = sh.cnt[1], nto = sh.cnt[2];
  (void)facing;
  __syncthreads();
  if (nf < 20) {
    tight = 0.0;
    gap = 1.0;
    contact = 0.0;
    return;
  }
  tight = double(nt) / double(nf);
  gap = median_f32(scratch, nf, sh) / sc.t;
  double share = double(nto) / double(n);
  contact = share * area / (sc.t * sc.t);
}

// The nearest of B's breakline points, moved by `t`, to A's point `a` under
// PointTree::nearest_below (kdtree.rs:182-190); the tree is over B in B's own
// frame and is searched around q = t^-1 a with a slack that covers the
// rounding of both transforms, every candidate re-measured exactly in A's
// frame. Returns B's original index or MISS.
__device__ __noinline__ uint32_t seam_nearest(const SurfView &b, const double *t, const double *a_pt, double qx,
                                 double qy, double qz, double bound, uint32_t &status) {
  if (!(bound > 0.0) || b.n_brk == 0) return MISS;
  const CloudView &c = b.brk_tree;
  double widened = (bound * bound) * (1.0 + 4.0 * 2.220446049250313e-16);
  double mag = fabs(t[3]) + fabs(t[7]) + fabs(t[11]) + fabs(qx) + fabs(qy) + fabs(qz) + 1.0;
  double slack = 1e-9 * mag;
  float qc[3] = {float(qx), float(qy), float(qz)};
  double best = widened;
  int best_s = -1;
  uint32_t best_i = MISS;
  auto bound2 = [&]() {
    double r = sqrt(best) * (1.0 + 1e-6) + slack;
    float b2 = __double2float_ru(r * r);
    return b2 + 1e-5f * b2 + 1e-30f;
  };
  auto leaf = [&](int first, int count) {
    for (int s = first; s < first + count; ++s) {
      double4 p = ldg4(c.pts + s);
      double mx, my, mz;
      apply_pose(t, p.x, p.y, p.z, mx, my, mz);
      double dx = a_pt[0] - mx, dy = a_pt[1] - my, dz = a_pt[2] - mz;
      double d2 = (dx * dx + dy * dy) + dz * dz;
      if (d2 > widened) continue;
      uint32_t id = uint32_t(p.w);
      if (best_s < 0 || d2 < best || (d2 == best && id < best_i)) {
        best = d2;
        best_s = s;
        best_i = id;
      }
    }
  };
  if (c.root_leaf) {
    leaf(0, c.root_leaf);
  } else {
    int stack_n[STACK];
    float stack_k[STACK];
    int sp = 0, node = 0;
    uint32_t visits = 0;
    for (;;) {
      if (++visits > 2u * c.n + 64u) {
        status |= ST_STACK;
        break;
      }
      Child2 n = load_node(c.nodes, node);
      float k[2] = {box_dist2(n.lo0, n.hi0, qc), box_dist2(n.lo1, n.hi1, qc)};
      int near_c = k[1] < k[0] ? 1 : 0;
      int next = -1;
      for (int q = 0; q < 2; ++q) {
        int ch = q == 0 ? near_c : 1 - near_c;
        if (!(k[ch] <= bound2())) continue;
        if (n.cnt[ch]) {
          leaf(n.ref[ch], n.cnt[ch]);
        } else if (next < 0) {
          next = n.ref[ch];
        } else if (sp < STACK) {
          stack_n[sp] = n.ref[ch];
          stack_k[sp++] = k[ch];
        } else {
          status |= ST_STACK;
        }
      }
      if (next >= 0) {
        node = next;
        continue;
      }
      bool more = false;
      while (sp > 0) {
        --sp;
        if (stack_k[sp] <= bound2()) {
          node = stack_n[sp];
          more = true;
          break;
        }
      }
      if (!more) break;
    }
  }
  if (best_s < 0) return MISS;
  if (!(sqrt(best) < bound)) return MISS;
  return best_i;
}

// verify::seam_score (verify.rs:378-442).
__device__ __noinline__ double seam_score(const PairView &pr, VerShared &sh, uint32_t &status) {
  const SurfView &a = pr.a, &b = pr.b;
  uint32_t words = (pr.n_cells + 31) / 32;
  for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) sh.cells[w] = 0;
  __syncthreads();
  if (b.n_brk > 0) {
    for (uint32_t k = threadIdx.x; k < a.n_brk; k += blockDim.x) {
      double4 aq = ldg4(a.brk_tree.pts + k);
      uint32_t i = uint32_t(aq.w);
      const double ap[3] = {aq.x, aq.y, aq.z};
      double qx, qy, qz;
      apply_pose(sh.inv, ap[0], ap[1], ap[2], qx, qy, qz);
      uint32_t j = seam_nearest(b, sh.t, ap, qx, qy, qz, pr.sc.seam, status);
      if (j == MISS) continue;
      double nx, ny, nz;
      rotate_pose(sh.t, b.brk_ns[3 * j], b.brk_ns[3 * j + 1], b.brk_ns[3 * j + 2], nx, ny, nz);
      const double *an = a.brk_ns + 3 * i;
      if (an[0] * nx + an[1] * ny + an[2] * nz > 0.7) {
        uint32_t cid = pr.a_cell[i];
        atomicOr(&sh.cells[cid >> 5], 1u << (cid & 31));
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) sh.cnt[3] = 0;
  __syncthreads();
  unsigned local = 0;
  for (uint32_t w = threadIdx.x; w < words; w += blockDim.x) local += __popc(sh.cells[w]);
  atomicAdd(&sh.cnt[3], local);
  __syncthreads();
  unsigned count = sh.cnt[3];
  __syncthreads();
  return count == 0 ? 0.0 : double(count) / 3.0;
}

// verify::continuity_scores (verify.rs:450-474).
__device__ __noinline__ void continuity(const PairView &pr, unsigned long long *steps,
                           unsigned long long *agree, VerShared &sh, double &cont, double &cont_n,
                           uint32_t &status) {
  const SurfView &a = pr.a, &b = pr.b;
  cont = 1.0;
  cont_n = -1.0;
  if (a.n_margin == 0 || b.n_margin == 0) return;
  if (threadIdx.x == 0) sh.cnt[4] = 0;
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < b.n_margin; k += blockDim.x) {
    double4 mq = ldg4(b.margin_tree.pts + k);
    uint32_t m = uint32_t(mq.w);
    double x, y, z;
    apply_pose(sh.t, mq.x, mq.y, mq.z, x, y, z);
    double dist;
    int s = nearest_below(a.margin_tree, x, y, z, pr.sc.near, dist, status);
    if (s < 0) continue;
    uint32_t j = uint32_t(a.margin_tree.pts[s].w);
    const double *np = a.margin_p + 3 * j, *nn = a.margin_n + 3 * j;
    double dx = x - np[0], dy = y - np[1], dz = z - np[2];
    double step = fabs(dx * nn[0] + dy * nn[1] + dz * nn[2]);
    double rx, ry, rz;
    rotate_pose(sh.t, b.margin_n[3 * m], b.margin_n[3 * m + 1], b.margin_n[3 * m + 2], rx, ry, rz);
    double ag = rx * nn[0] + ry * nn[1] + rz * nn[2];
    unsigned slot = atomicAdd(&sh.cnt[4], 1u);
    steps[slot] = d2key(step);
    agree[slot] = d2key(ag);
  }
  __syncthreads();
  unsigned n = sh.cnt[4];
  __syncthreads();
  if (n <= 20) return;
  cont = median_f64(steps, n, sh) / pr.sc.t;
  cont_n = median_f64(agree, n, sh);
}

// Appends `slot` to a shared queue for every lane whose `pred` holds, with one
// shared atomic per warp.
__device__ __forceinline__ void warp_append(bool pred, unsigned slot, unsigned *queue,
                                            unsigned *count) {
  unsigned act = __activemask();
  unsigned mask = __ballot_sync(act, pred);
  if (!mask) return;
  int lane = threadIdx.x & 31;
  int leader = __ffs(mask) - 1;
  unsigned base = 0;
  if (lane == leader) base = atomicAdd(count, unsigned(__popc(mask)));
  base = __shfl_sync(act, base, leader);
  if (pred) queue[base + __popc(mask & ((1u << lane) - 1u))] = slot;
}

__device__ __forceinline__ F3 moved_point(const double4 *pts, uint32_t i, const double *pose) {
  double4 q = ldg4(pts + i);
  double x, y, z;
  apply_pose(pose, q.x, q.y, q.z, x, y, z);
  return narrow3(x, y, z);
}

// verify::one_penetration (verify.rs:541-580): (fraction deeper than pen,
// smallest signed distance). The points go through in rounds of PEN_CHUNK: the
// box test compacts the ones inside the mesh's box into a shared queue, the
// parity test runs densely over that queue and compacts the inside points into
// a second one, and the depth queries run densely over those, so a warp's
// lanes all do the same stage of the test. When nothing is inside, the
// shrinking-window minimum of cpu.rs:98-111 is seeded from 32 points spread over
// the set before the whole block scans it; a point whose distance to the mesh's
// box already exceeds the window is skipped (it cannot beat it). Counts, the
// maximum and the minimum do not depend on the order points are taken in.
__device__ __noinline__ void one_penetration(const double4 *pts, uint32_t n, const double *pose,
                                const MeshView &scene, double pen, VerShared &sh,
                                double &fraction, double &mins, uint32_t &status) {
  fraction = 0.0;
  mins = 0.0;
  if (n == 0) return;
  if (threadIdx.x == 0) {
    sh.cnt[5] = 0;
    sh.deep_key = 0;  // 0: no inside point yet; else f2key(depth) + 1
    sh.best_key = f2key(3.4028234663852886e38f);
  }
  __syncthreads();
  unsigned deeper = 0;
  for (uint32_t base = 0; base < n; base += PEN_CHUNK) {
    uint32_t end = min(n, base + uint32_t(PEN_CHUNK));
    if (threadIdx.x == 0) {
      sh.n_box = 0;
      sh.n_in = 0;
    }
    __syncthreads();
    for (uint32_t i = base + threadIdx.x; i < base + PEN_CHUNK; i += blockDim.x) {
      bool in_box = false;
      if (i < end) {
        F3 p = moved_point(pts, i, pose);
        in_box = !(p.x < scene.lo[0] || p.x > scene.hi[0] || p.y < scene.lo[1] ||
                   p.y > scene.hi[1] || p.z < scene.lo[2] || p.z > scene.hi[2]);
      }
      warp_append(in_box, i, sh.q_box, &sh.n_box);
    }
    __syncthreads();
    unsigned nb = sh.n_box;
    for (uint32_t k = threadIdx.x; k < nb; k += blockDim.x) {
      uint32_t i = sh.q_box[k];
      warp_append(inside_mesh(scene, moved_point(pts, i, pose), status), i, sh.q_in, &sh.n_in);
    }
    __syncthreads();
    unsigned ni = sh.n_in;
    for (uint32_t k = threadIdx.x; k < ni; k += blockDim.x) {
      float depth = mesh_distance(scene, moved_point(pts, sh.q_in[k], pose), f_inf(), status);
      atomicMax(&sh.deep_key, f2key(depth) + 1u);
      if (double(depth) > pen) ++deeper;
    }
    __syncthreads();
  }
  atomicAdd(&sh.cnt[5], deeper);
  __syncthreads();
  fraction = double(sh.cnt[5]) / double(n);
  unsigned dk = sh.deep_key;
  __syncthreads();
  if (dk != 0) {
    mins = -double(key2f(dk - 1u));
    return;
  }
  auto scan = [&](uint32_t i) {
    F3 p = moved_point(pts, i, pose);
    float window = key2f(*((volatile unsigned *)&sh.best_key));
    float pc[3] = {p.x, p.y, p.z};
    // Every face is at least the box's distance away; the slack keeps a face
    // whose rounded distance ties the window within a few ulps.
    float gap = sqrtf(box_dist2(scene.lo, scene.hi, pc));
    if (gap > window + 1e-5f * window + scene.pad) return;
    float d = mesh_distance(scene, p, window, status);
    if (d != f_inf()) atomicMin(&sh.best_key, f2key(d));
  };
  if (threadIdx.x < 32) scan(uint32_t((unsigned long long)threadIdx.x * n / 32u));
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) scan(i);
  __syncthreads();
  mins = double(key2f(sh.best_key));
  __syncthreads();
}

// verify::verify (verify.rs:590-626) + accept (verify.rs:632-638) at the pose
// in sh.t. Every thread calls it; thread 0 writes *out.
// `pen_here` false leaves the penetration scores to the batched path's
// wavefront kernels (which read the inverse pose from `inv_out`) and the
// verdict to its finalising kernel.
__device__ void verify_block(const PairView &pr, bool full, const sherd_params &p,
                             unsigned *scratch, VerShared &sh, sherd_scores *out,
                             uint32_t *accepted, uint32_t &status, bool pen_here = true,
                             double *inv_out = nullptr) {
  if (threadIdx.x == 0) pose_inverse(sh.t, sh.inv);
  __syncthreads();
  if (inv_out && threadIdx.x < 16) inv_out[threadIdx.x] = sh.inv[threadIdx.x];
  const sherd_scales &sc = pr.sc;
  double ta, ga, ca, tb, gb, cb;
  one_side(pr.b.pf, pr.b.n_pf, sh.t, pr.a.frac, pr.b.frac_area, sc, scratch, sh, tb, gb, cb,
           status);
  one_side(pr.a.pf, pr.a.n_pf, sh.inv, pr.b.frac, pr.a.frac_area, sc, scratch, sh, ta, ga, ca,
           status);
  double seam = seam_score(pr, sh, status);
  double cont = 1.0, cont_n = -1.0, pen = 0.0, pen_depth = 0.0;
  uint32_t unavailable = 0;
  if (full) {
    unsigned long long *steps = reinterpret_cast<unsigned long long *>(scratch);
    continuity(pr, steps, steps + pr.b.n_margin, sh, cont, cont_n, status);
    if (!pr.a.has_mesh || !pr.b.has_mesh || !(pr.a.watertight && pr.b.watertight)) {
      unavailable = 1;
    } else if (pen_here) {
      double pen_b, min_b, pen_a, min_a;
      one_penetration(pr.b.s, pr.b.n_s, sh.t, pr.a.mesh, sc.pen, sh, pen_b, min_b, status);
      one_penetration(pr.a.s, pr.a.n_s, sh.inv, pr.b.mesh, sc.pen, sh, pen_a, min_a, status);
      pen = fmax(pen_a, pen_b);
      pen_depth = fmax(-min_a, -min_b) / sc.t;
    }
  }
  if (threadIdx.x == 0) {
    sherd_scores s;
    s.tight_a = ta;
    s.tight_b = tb;
    s.tight = fmin(ta, tb);
    s.gap_a = ga;
    s.gap_b = gb;
    s.gap = fmax(ga, gb);
    s.contact_a = ca;
    s.contact_b = cb;
    s.contact = fmin(ca, cb);
    s.seam = seam;
    s.gap_limit = sc.gap / sc.t;
    s.tight_delta = sc.tight / sc.t;
    s.cont = cont;
    s.cont_n = cont_n;
    s.pen = pen;
    s.pen_depth = pen_depth;
    s.pen_unavailable = unavailable;
    s.partial = full ? 0u : 1u;
    s.brk = 0.0;
    s.brk_best = 0.0;
    *out = s;
    if (accepted && pen_here)
      *accepted = (s.tight >= p.min_tight && s.gap * sc.t <= sc.gap && s.pen <= p.max_pen &&
                   s.seam >= p.min_seam && s.cont_n >= p.min_cont_n)
                      ? 1u
                      : 0u;
  }
  __syncthreads();
}

}  // namespace sherd
