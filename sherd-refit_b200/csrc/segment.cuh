// segment.cuh — R 3.4's shell/fracture segmentation (fragment/segment.rs:189-631)
// on the device.
//
// The steps and the arrays between them:
//   voxel keys of the face centroids -> (radix sort) -> representatives, the
//   lowest face of every t/8 voxel, ascending -> each face's nearest
//   representative (point LBVH, lowest index on a tie) -> radius balls around
//   the representatives over the centroid LBVH (smoothed normals, majority
//   filter, shell reference normals) -> cone votes -> islands (lock-free
//   union-find over the face adjacency, component areas summed in face order)
//   -> boundary growth passes.
//
// Bit-exactness to a sequential restatement: a radius ball is collected in
// shared memory (sized per call by a counting pass to the largest ball),
// sorted by face index and summed by one thread in that order
// (PointTree::within returns its members ascending, kdtree.rs:219-245); a
// component's area is summed by one thread in face order (components.rs:
// 180-185). Everything else is a per-face decision or an exact reduction.
#pragma once

#include "kernels.cuh"

namespace sherd {

constexpr int BALL_BLOCK = 128;
constexpr uint32_t VOXEL_LIMIT = 1u << 21;

enum BallMode { BALL_NORMALS = 0, BALL_MAJORITY = 1, BALL_SHELL_NORMALS = 2 };

// The exact per-axis minimum of the centroids, as order-preserving keys.
__global__ void k_min_bound(const double *c, uint32_t n, unsigned long long *mb) {
  unsigned long long m[3] = {~0ull, ~0ull, ~0ull};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int k = 0; k < 3; ++k) m[k] = min(m[k], d2key(c[3 * size_t(i) + k]));
  for (int k = 0; k < 3; ++k) atomicMin(mb + k, m[k]);
}

// voxel_representatives (segment.rs:217-259): floor((c - (min - 1)) / spacing)
// per axis, packed 21 bits an axis so that the key order is the tuple order.
__global__ void k_voxel_keys(const double *c, uint32_t n, const unsigned long long *mb,
                             double spacing, unsigned long long *key, uint32_t *idx,
                             uint32_t *status) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long k = 0;
  for (int a = 0; a < 3; ++a) {
    double lo = key2d(mb[a]) - 1.0;
    double v = floor((c[3 * size_t(i) + a] - lo) / spacing);
    if (!(v >= 0.0 && v < double(VOXEL_LIMIT))) {
      atomicOr(status, ST_RANGE);
      v = 0.0;
    }
    k = (k << 21) | (unsigned long long)v;
  }
  key[i] = k;
  idx[i] = i;
}

__global__ void k_run_heads(const unsigned long long *key, uint32_t n, uint8_t *head) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) head[i] = i == 0 || key[i] != key[i - 1];
}

__global__ void k_gather_points(const double *src, const uint32_t *idx, uint32_t n, double *dst) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int k = 0; k < 3; ++k) dst[3 * size_t(i) + k] = src[3 * size_t(idx[i]) + k];
}

// coarse_grid's near (segment.rs:189-200): the representative nearest each
// centroid, an index into the ascending representative list.
__global__ void k_nearest_rep(CloudView reps, const double *c, uint32_t n, uint32_t *near,
                              uint32_t *status) {
  uint32_t st = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d2;
    int s = nearest_within_sq(reps, c[3 * size_t(i)], c[3 * size_t(i) + 1], c[3 * size_t(i) + 2],
                              d_inf(), d2, st);
    near[i] = s < 0 ? 0u : uint32_t(reps.pts[s].w);
  }
  if (st) atomicOr(status, st);
}

// Every leaf range of a point LBVH whose box comes within `bound` of q.
template <class Leaf>
__device__ void cloud_walk_within(const CloudView &c, const float *q, float bound, Leaf &&leaf,
                                  uint32_t &status) {
  if (c.root_leaf) {
    leaf(0, int(c.root_leaf));
    return;
  }
  const float b2 = bound * bound;
  int stack[STACK];
  int sp = 0, node = 0;
  uint32_t visits = 0;
  for (;;) {
    if (++visits > 2u * c.n + 64u) {
      status |= ST_STACK;
      return;
    }
    Child2 n = load_node(c.nodes, node);
    int next = -1;
    for (int ch = 0; ch < 2; ++ch) {
      float k = box_dist2(ch ? n.lo1 : n.lo0, ch ? n.hi1 : n.hi0, q);
      if (!(k <= b2)) continue;
      if (n.cnt[ch]) {
        leaf(n.ref[ch], n.cnt[ch]);
      } else if (next < 0) {
        next = n.ref[ch];
      } else if (sp < STACK) {
        stack[sp++] = n.ref[ch];
      } else {
        status |= ST_STACK;
      }
    }
    if (next >= 0) {
      node = next;
    } else if (sp > 0) {
      node = stack[--sp];
    } else {
      return;
    }
  }
}

__device__ __forceinline__ float ball_bound(const CloudView &c, double radius) {
  return float(radius) * (1.0f + 1e-6f) + c.pad;
}

__device__ __forceinline__ bool in_ball(const double *q, double4 p, double r2) {
  double ex = q[0] - p.x, ey = q[1] - p.y, ez = q[2] - p.z;
  return (ex * ex + ey * ey) + ez * ez <= r2;
}

// One thread per representative: the largest ball and the most leaf ranges
// any representative needs, which size k_ball's shared memory.
__global__ void k_ball_size(CloudView all, const double *cent, const uint32_t *rep,
                            uint32_t n_rep, double radius, int mode, const uint8_t *frac,
                            uint32_t *max_members, uint32_t *max_ranges, uint32_t *status) {
  uint32_t st = 0, mm = 0, mr = 0;
  const double r2 = radius * radius;
  const float bound = ball_bound(all, radius);
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n_rep; r += gridDim.x * blockDim.x) {
    const double *q = cent + 3 * size_t(rep[r]);
    float qf[3] = {float(q[0]), float(q[1]), float(q[2])};
    uint32_t members = 0, ranges = 0;
    cloud_walk_within(
        all, qf, bound,
        [&](int first, int count) {
          ++ranges;
          for (int s = first; s < first + count; ++s) {
            double4 p = ldg4(all.pts + s);
            if (in_ball(q, p, r2) && !(mode == BALL_SHELL_NORMALS && frac[uint32_t(p.w)])) ++members;
          }
        },
        st);
    mm = max(mm, members);
    mr = max(mr, ranges);
  }
  atomicMax(max_members, mm);
  atomicMax(max_ranges, mr);
  if (st) atomicOr(status, st);
}

// One CTA per representative: the ball of every centroid with d2 <= r2
// (inclusive, d2 = ((dx dx + dy dy) + dz dz)), sorted by face index, summed
// by one thread in that order.
//   BALL_NORMALS / BALL_SHELL_NORMALS: ball_normals (segment.rs:267-296),
//     m = sum A FN / max(sum A, 1e-12), m / max(|m|, 1e-12), and whether the
//     ball is non-empty; the shell form keeps only faces with frac == 0.
//   BALL_MAJORITY: majority_filter (segment.rs:402-427), wet > 0.5 total.
__global__ void __launch_bounds__(BALL_BLOCK) k_ball(CloudView all, const double *cent,
                                                     const uint32_t *rep, uint32_t n_rep,
                                                     double radius, int mode,
                                                     const double *normals, const double *areas,
                                                     const uint8_t *frac, double *out3,
                                                     uint8_t *flag, uint32_t cap, uint32_t rcap,
                                                     uint32_t *status) {
  extern __shared__ uint32_t s_dyn[];
  uint32_t *s_idx = s_dyn;                              // cap member slots (a power of two)
  int *s_first = reinterpret_cast<int *>(s_dyn + cap);  // rcap leaf ranges
  int *s_count = s_first + rcap;
  __shared__ uint32_t s_n, s_nr, s_st;
  const double r2 = radius * radius;
  const float bound = ball_bound(all, radius);
  if (threadIdx.x == 0) s_st = 0;
  for (uint32_t r = blockIdx.x; r < n_rep; r += gridDim.x) {
    const double *q = cent + 3 * size_t(rep[r]);
    if (threadIdx.x == 0) {
      float qf[3] = {float(q[0]), float(q[1]), float(q[2])};
      uint32_t nr = 0, st = 0;
      cloud_walk_within(
          all, qf, bound,
          [&](int first, int count) {
            if (nr < rcap) {
              s_first[nr] = first;
              s_count[nr] = count;
              ++nr;
            } else {
              st |= ST_SCRATCH;
            }
          },
          st);
      s_nr = nr;
      s_n = 0;
      s_st |= st;
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < s_nr; k += BALL_BLOCK) {
      for (int s = s_first[k]; s < s_first[k] + s_count[k]; ++s) {
        double4 p = ldg4(all.pts + s);
        if (!in_ball(q, p, r2)) continue;
        uint32_t j = uint32_t(p.w);
        if (mode == BALL_SHELL_NORMALS && frac[j]) continue;
        uint32_t at = atomicAdd(&s_n, 1u);
        if (at < cap) s_idx[at] = j;
      }
    }
    __syncthreads();
    uint32_t n = s_n;
    if (n > cap) {
      if (threadIdx.x == 0) s_st |= ST_SCRATCH;
      n = cap;
    }
    uint32_t pw = 1;
    while (pw < n) pw <<= 1;
    for (uint32_t i = n + threadIdx.x; i < pw; i += BALL_BLOCK) s_idx[i] = 0xFFFFFFFFu;
    __syncthreads();
    for (uint32_t size = 2; size <= pw; size <<= 1) {
      for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
        for (uint32_t i = threadIdx.x; i < pw; i += BALL_BLOCK) {
          uint32_t j = i ^ stride;
          if (j > i) {
            uint32_t a = s_idx[i], b = s_idx[j];
            if ((a > b) == ((i & size) == 0)) {
              s_idx[i] = b;
              s_idx[j] = a;
            }
          }
        }
        __syncthreads();
      }
    }
    if (threadIdx.x == 0) {
      if (mode == BALL_MAJORITY) {
        double wet = 0.0, total = 0.0;
        for (uint32_t k = 0; k < n; ++k) {
          uint32_t j = s_idx[k];
          double a = areas[j];
          total += a;
          if (frac[j]) wet += a;
        }
        flag[r] = wet > 0.5 * total;
      } else {
        double m[3] = {0.0, 0.0, 0.0}, wsum = 0.0;
        for (uint32_t k = 0; k < n; ++k) {
          uint32_t j = s_idx[k];
          const double *nn = normals + 3 * size_t(j);
          double a = areas[j];
          m[0] += nn[0] * a;
          m[1] += nn[1] * a;
          m[2] += nn[2] * a;
          wsum += a;
        }
        double den = fmax(wsum, 1e-12);
        for (int c = 0; c < 3; ++c) m[c] /= den;
        double norm = fmax(sqrt((m[0] * m[0] + m[1] * m[1]) + m[2] * m[2]), 1e-12);
        for (int c = 0; c < 3; ++c) out3[3 * size_t(r) + c] = m[c] / norm;
        flag[r] = n > 0;
      }
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && s_st) atomicOr(status, s_st);
}

// A representative's answer to every face it represents.
__global__ void k_spread(const uint32_t *near, uint32_t n, const double *g3, const uint8_t *gflag,
                         double *face3, uint8_t *faceflag) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t r = near[i];
  if (face3)
    for (int k = 0; k < 3; ++k) face3[3 * size_t(i) + k] = g3[3 * size_t(r) + k];
  if (faceflag) faceflag[i] = gflag[r];
}

__global__ void k_votes_to_frac(const uint8_t *good, uint32_t n, uint32_t votes, uint8_t *frac) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) frac[i] = uint32_t(good[i]) < votes;
}

// face_adjacency (adjacency.rs:43-51, 138-160): the 3 nf edge keys in
// slot-major order, (lo << 32) | hi, with their positions.
__global__ void k_edge_keys(const uint32_t *f, uint32_t nf, unsigned long long *key,
                            uint32_t *pos) {
  uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nf) return;
  const int slot[3][2] = {{0, 1}, {1, 2}, {2, 0}};
  for (int s = 0; s < 3; ++s) {
    uint32_t a = f[3 * size_t(t) + slot[s][0]], b = f[3 * size_t(t) + slot[s][1]];
    uint32_t lo = min(a, b), hi = max(a, b);
    size_t at = size_t(s) * nf + t;
    key[at] = (unsigned long long)lo << 32 | hi;
    pos[at] = uint32_t(at);
  }
}

// Every two consecutive equal keys of the stably sorted list are one face
// pair; entry w is (MISS, MISS) when keys w and w + 1 differ.
__global__ void k_face_pairs(const unsigned long long *key, const uint32_t *pos, uint32_t m,
                             uint32_t nf, uint32_t *fa, uint32_t *fb) {
  uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w + 1 >= m) return;
  bool pair = key[w] == key[w + 1];
  fa[w] = pair ? pos[w] % nf : MISS;
  fb[w] = pair ? pos[w + 1] % nf : MISS;
}

__device__ __forceinline__ uint32_t uf_find(uint32_t *parent, uint32_t x) {
  volatile uint32_t *p = parent;
  for (;;) {
    uint32_t up = p[x];
    if (up == x) return x;
    uint32_t upup = p[up];
    if (upup != up) p[x] = upup;  // path halving; only ever points to an ancestor
    x = upup;
  }
}

__global__ void k_uf_init(uint32_t *parent, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) parent[i] = i;
}

// mask_components (components.rs:120-159): union of every pair whose two
// faces have mask == target, the larger root hooked under the smaller by
// compare-and-swap on a root, so no union is lost and each component's root is
// its lowest face.
__global__ void k_uf_union(const uint32_t *fa, const uint32_t *fb, uint32_t m, const uint8_t *mask,
                           uint8_t target, uint32_t *parent, uint32_t *status) {
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < m; w += gridDim.x * blockDim.x) {
    uint32_t a = fa[w], b = fb[w];
    if (a == MISS || mask[a] != target || mask[b] != target) continue;
    for (int tries = 0;; ++tries) {
      if (tries == (1 << 20)) {
        atomicOr(status, ST_STACK);
        break;
      }
      uint32_t ra = uf_find(parent, a), rb = uf_find(parent, b);
      if (ra == rb) break;
      if (ra < rb) {
        uint32_t t = ra;
        ra = rb;
        rb = t;
      }
      if (atomicCAS(parent + ra, ra, rb) == ra) break;
    }
  }
}

// Each face of the set gets its root as a sort key (MISS outside the set).
__global__ void k_uf_roots(uint32_t *parent, const uint8_t *mask, uint8_t target, uint32_t n,
                           uint32_t *root, uint32_t *face) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  root[i] = mask[i] == target ? uf_find(parent, i) : MISS;
  face[i] = i;
}

// One thread per component: its area, summed in face order (the roots were
// sorted stably, so each run lists its faces ascending).
__global__ void k_component_areas(const uint32_t *root, const uint32_t *face, uint32_t n,
                                  const double *areas, double *size) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || root[i] == MISS || (i > 0 && root[i - 1] == root[i])) return;
  double s = 0.0;
  uint32_t j = i;
  for (; j < n && root[j] == root[i]; ++j) s += areas[face[j]];
  size[root[i]] = s;
}

// drop_small_components (components.rs:186-190).
__global__ void k_drop_small(uint8_t *mask, uint8_t target, uint32_t n, uint32_t *parent,
                             const double *size, double min_area) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || mask[i] != target) return;
  if (size[uf_find(parent, i)] < min_area) mask[i] = !target;
}

// refine_boundary (segment.rs:438-474), one pass in two launches: the
// fracture faces touching the shell at the start of the pass, then the flips.
__global__ void k_grow_candidates(const uint32_t *fa, const uint32_t *fb, uint32_t m,
                                  const uint8_t *frac, uint8_t *cand) {
  uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= m || fa[w] == MISS) return;
  uint32_t a = fa[w], b = fb[w];
  if (frac[a] != frac[b]) cand[frac[a] ? a : b] = 1;
}

__global__ void k_grow_flip(uint8_t *cand, uint8_t *frac, uint32_t n, const double *normals,
                            const double *ref, const uint8_t *has_ref, double cos_grow,
                            uint32_t *flipped) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !cand[i]) return;
  cand[i] = 0;
  const double *nn = normals + 3 * size_t(i), *r = ref + 3 * size_t(i);
  if (has_ref[i] && (nn[0] * r[0] + nn[1] * r[1]) + nn[2] * r[2] > cos_grow) {
    frac[i] = 0;
    *flipped = 1;
  }
}

// The shell's normal noise for the automatic growth angle: the clamped dot of
// each shell face's normal with its smoothed normal (the angle is taken on
// the host, with the same acos as the reference's).
__global__ void k_shell_dots(const uint8_t *frac, uint32_t n, const double *normals,
                             const double *ns, double *dots) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double *a = normals + 3 * size_t(i), *b = ns + 3 * size_t(i);
  double c = (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
  dots[i] = frac[i] ? 2.0 : fmin(1.0, fmax(-1.0, c));
}

}  // namespace sherd
