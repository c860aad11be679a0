// traverse.cuh — per-thread short-stack BVH traversal for the four queries of
// the hot path. Every query is exact under one tie rule:
//   first hit      smallest t, then lowest original face index
//   crossings      every face the ray crosses (no pruning by distance)
//   distance       smallest f32 point-to-triangle distance (a value, no id)
//   nearest point  smallest f64 squared distance, then lowest original index
// Pruning only ever drops a node whose padded box is provably beyond the best
// answer so far (relative slack 4e-6 on top of the box padding), so the result
// is the brute-force result the CPU oracle computes.
#pragma once

#include "lbvh.cuh"

namespace sherd {

struct Child2 {
  float lo0[3], hi0[3], lo1[3], hi1[3];
  int ref[2], cnt[2];
};

__device__ __forceinline__ Child2 load_node(const BNode *nodes, int i) {
  const float4 *p = reinterpret_cast<const float4 *>(nodes + i);
  float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2);
  int4 d = __ldg(reinterpret_cast<const int4 *>(p + 3));
  Child2 n;
  n.lo0[0] = a.x; n.lo0[1] = a.y; n.lo0[2] = a.z; n.hi0[0] = a.w;
  n.hi0[1] = b.x; n.hi0[2] = b.y; n.lo1[0] = b.z; n.lo1[1] = b.w;
  n.lo1[2] = c.x; n.hi1[0] = c.y; n.hi1[1] = c.z; n.hi1[2] = c.w;
  n.ref[0] = d.x; n.ref[1] = d.y; n.cnt[0] = d.z; n.cnt[1] = d.w;
  return n;
}

struct Ray {
  float o[3], d[3], inv[3];
  bool zero[3];
};

__device__ __forceinline__ Ray make_ray(F3 o, F3 d) {
  Ray r;
  r.o[0] = o.x; r.o[1] = o.y; r.o[2] = o.z;
  r.d[0] = d.x; r.d[1] = d.y; r.d[2] = d.z;
  for (int a = 0; a < 3; ++a) {
    r.zero[a] = r.d[a] == 0.0f;
    r.inv[a] = r.zero[a] ? 0.0f : 1.0f / r.d[a];
  }
  return r;
}

// Entry parameter of the ray into a padded box over [0, inf), or +inf.
__device__ __forceinline__ float slab_enter(const Ray &r, const float *lo, const float *hi) {
  float tmin = 0.0f, tmax = f_inf();
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (r.zero[a]) {
      if (r.o[a] < lo[a] || r.o[a] > hi[a]) return f_inf();
    } else {
      float t0 = (lo[a] - r.o[a]) * r.inv[a], t1 = (hi[a] - r.o[a]) * r.inv[a];
      tmin = fmaxf(tmin, fminf(t0, t1));
      tmax = fminf(tmax, fmaxf(t0, t1));
    }
  }
  return tmin <= tmax + 4e-6f * fabsf(tmax) ? tmin : f_inf();
}

__device__ __forceinline__ void tri_at(const MeshView &m, uint32_t s, F3 &a, F3 &b, F3 &c,
                                       uint32_t &id) {
  float4 x = __ldg(m.tri + 3 * s), y = __ldg(m.tri + 3 * s + 1), z = __ldg(m.tri + 3 * s + 2);
  a = {x.x, x.y, x.z};
  b = {y.x, y.y, y.z};
  c = {z.x, z.y, z.z};
  id = __float_as_uint(x.w);
}

// RayScene::first_hit (spatial/bvh.rs:84-90).
__device__ __noinline__ void first_hit(const MeshView &m, F3 o, F3 d, float &best, uint32_t &best_id,
                          uint32_t &status) {
  best = f_inf();
  best_id = MISS;
  if (m.nf == 0) return;
  Ray r = make_ray(o, d);
  float dn = sqrtf(dot(d, d));
  float pad_t = dn > 0.0f ? 4.0f * m.pad / dn : f_inf();
  auto bound = [&]() { return best == f_inf() ? f_inf() : best + 4e-6f * best + pad_t; };
  auto leaf = [&](int first, int count) {
    for (int s = first; s < first + count; ++s) {
      F3 a, b, c;
      uint32_t id;
      tri_at(m, s, a, b, c, id);
      float t = moller_trumbore(o, d, a, b, c);
      if (t < 0.0f) continue;
      if (t < best || (t == best && id < best_id)) {
        best = t;
        best_id = id;
      }
    }
  };
  if (m.root_leaf) {
    leaf(0, m.root_leaf);
    return;
  }
  int stack_n[STACK];
  float stack_t[STACK];
  int sp = 0, node = 0;
  uint32_t visits = 0;
  for (;;) {
    if (++visits > 2u * m.nf + 64u) {
      status |= ST_STACK;
      break;
    }
    Child2 n = load_node(m.nodes, node);
    float te[2] = {slab_enter(r, n.lo0, n.hi0), slab_enter(r, n.lo1, n.hi1)};
    int near_c = te[1] < te[0] ? 1 : 0;
    int next = -1;
    for (int q = 0; q < 2; ++q) {
      int c = q == 0 ? near_c : 1 - near_c;
      // A box the ray misses enters at +inf, which the bound (+inf until the
      // first hit) would otherwise let through.
      if (te[c] == f_inf() || !(te[c] <= bound())) continue;
      if (n.cnt[c]) {
        leaf(n.ref[c], n.cnt[c]);
      } else if (next < 0) {
        next = n.ref[c];
      } else if (sp < STACK) {
        stack_n[sp] = n.ref[c];
        stack_t[sp++] = te[c];
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
      if (stack_t[sp] <= bound()) {
        node = stack_n[sp];
        more = true;
        break;
      }
    }
    if (!more) break;
  }
}

// RayScene::crossings (spatial/bvh.rs:160-175) along +x, +y or +z: the faces
// the axis ray from p crosses. A face counts when p's projection lies inside
// the face's projected rectangle padded outward by the mesh padding (f32,
// directed rounding) and Moller-Trumbore reports a crossing; the padding is
// far above the test's rounding, so this is the reference's count except for
// a ray grazing a face edge-on, where it states one rule for both sides. Every
// such face was binned into p's cell of the axis grid (rectangle containment
// implies cell containment, the cell index being monotone in the coordinate),
// so scanning that one cell is the whole traversal.
__device__ __noinline__ uint32_t crossings_axis(const MeshView &m, F3 p, int axis, uint32_t &status) {
  if (m.nf == 0) return 0;
  const AxisGrid &g = m.grid[axis];
  float pc[3] = {p.x, p.y, p.z};
  float pu = pc[(axis + 1) % 3], pv = pc[(axis + 2) % 3];
  float fu = floorf((pu - g.lo_u) * g.inv_cell), fv = floorf((pv - g.lo_v) * g.inv_cell);
  if (!(fu >= 0.0f && fv >= 0.0f && fu < float(g.nu) && fv < float(g.nv))) return 0;
  size_t cell = size_t(fu) * g.nv + size_t(fv);
  uint32_t b = __ldg(g.start + cell), e = __ldg(g.start + cell + 1);
  F3 d = {axis == 0 ? 1.0f : 0.0f, axis == 1 ? 1.0f : 0.0f, axis == 2 ? 1.0f : 0.0f};
  uint32_t hits = 0;
  for (uint32_t k = b; k < e; ++k) {
    float4 r = __ldg(g.rect + k);
    if (pu < r.x || pu > r.y || pv < r.z || pv > r.w) continue;
    float4 t0 = __ldg(g.tri + 3 * size_t(k)), t1 = __ldg(g.tri + 3 * size_t(k) + 1),
           t2 = __ldg(g.tri + 3 * size_t(k) + 2);
    if (moller_trumbore_edges(p, d, {t0.x, t0.y, t0.z}, {t1.x, t1.y, t1.z}, {t2.x, t2.y, t2.z}) >=
        0.0f)
      ++hits;
  }
  (void)status;
  return hits;
}

// RayScene::inside (spatial/bvh.rs:146-157): the majority of three parities.
// When the first two agree the third cannot change the majority, so it is
// cast only when they differ.
__device__ __forceinline__ bool inside_mesh(const MeshView &m, F3 p, uint32_t &status) {
  uint32_t a = crossings_axis(m, p, 0, status) & 1u;
  uint32_t b = crossings_axis(m, p, 1, status) & 1u;
  if (a == b) return a != 0;
  return (crossings_axis(m, p, 2, status) & 1u) != 0;
}

__device__ __forceinline__ float box_dist2(const float *lo, const float *hi, const float *p) {
  float s = 0.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float g = fmaxf(fmaxf(lo[a] - p[a], p[a] - hi[a]), 0.0f);
    s += g * g;
  }
  return s;
}

// A walk over a 4-wide tree (WNode) with the binary tree's own boxes: at each
// node the children in ascending box distance, leaves scored first (nearest
// first, each against the bound as it stands), then the nearest node taken
// and the others stacked with the nearest on top. Every leaf whose box lies
// within the bound is scored, whatever the order, so a search's answer is the
// binary walk's. `bound2()` is the squared bound on box distances; `leaf`
// returns true to end the walk. (Point clouds only: on the mesh trees the
// closest-face walks measured 4 % faster in the minimum pass but the inside
// pass, whose kernel the wider walk costs registers, 50 % slower.)
template <class Leaf, class Bound2>
__device__ __forceinline__ void wide_walk(const WNode *wide, const float *pc, uint32_t limit,
                                          Leaf &&leaf, Bound2 &&bound2, uint32_t &status) {
  int stack_n[STACK];
  float stack_k[STACK];
  int sp = 0, node = 0;
  uint32_t visits = 0;
  auto push = [&](int r, float k) {
    if (sp < STACK) {
      stack_n[sp] = r;
      stack_k[sp++] = k;
    } else {
      status |= ST_STACK;
    }
  };
  auto bd = [&](float x0, float y0, float z0, float x1, float y1, float z1) {
    const float lo[3] = {x0, y0, z0}, hi[3] = {x1, y1, z1};
    return box_dist2(lo, hi, pc);
  };
  auto order = [](float &ka, int &ra, int &na, float &kb, int &rb, int &nb) {
    if (kb < ka) {
      float tk = ka; ka = kb; kb = tk;
      int tr = ra; ra = rb; rb = tr;
      int tn = na; na = nb; nb = tn;
    }
  };
  for (;;) {
    if (++visits > limit) {
      status |= ST_STACK;
      return;
    }
    const float4 *w = reinterpret_cast<const float4 *>(wide + node);
    const float4 lx = __ldg(w), ly = __ldg(w + 1), lz = __ldg(w + 2);
    const float4 hx = __ldg(w + 3), hy = __ldg(w + 4), hz = __ldg(w + 5);
    const int4 rf = __ldg(reinterpret_cast<const int4 *>(w + 6));
    const int4 ct = __ldg(reinterpret_cast<const int4 *>(w + 7));
    float k0 = bd(lx.x, ly.x, lz.x, hx.x, hy.x, hz.x), k1 = bd(lx.y, ly.y, lz.y, hx.y, hy.y, hz.y);
    float k2 = bd(lx.z, ly.z, lz.z, hx.z, hy.z, hz.z), k3 = bd(lx.w, ly.w, lz.w, hx.w, hy.w, hz.w);
    int r0 = rf.x, r1 = rf.y, r2 = rf.z, r3 = rf.w;
    int n0 = ct.x, n1 = ct.y, n2 = ct.z, n3 = ct.w;
    order(k0, r0, n0, k1, r1, n1);
    order(k2, r2, n2, k3, r3, n3);
    order(k0, r0, n0, k2, r2, n2);
    order(k1, r1, n1, k3, r3, n3);
    order(k1, r1, n1, k2, r2, n2);
    if (n0 > 0 && k0 <= bound2() && leaf(r0, n0)) return;
    if (n1 > 0 && k1 <= bound2() && leaf(r1, n1)) return;
    if (n2 > 0 && k2 <= bound2() && leaf(r2, n2)) return;
    if (n3 > 0 && k3 <= bound2() && leaf(r3, n3)) return;
    const float b = bound2();
    const bool i0 = n0 == 0 && k0 <= b, i1 = n1 == 0 && k1 <= b, i2 = n2 == 0 && k2 <= b,
               i3 = n3 == 0 && k3 <= b;
    const int first = i0 ? 0 : i1 ? 1 : i2 ? 2 : i3 ? 3 : 4;
    if (i3 && first != 3) push(r3, k3);
    if (i2 && first != 2) push(r2, k2);
    if (i1 && first != 1) push(r1, k1);
    if (first < 4) {
      node = first == 0 ? r0 : first == 1 ? r1 : first == 2 ? r2 : r3;
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
    if (!more) return;
  }
}

// The closest-face walk shared by mesh_distance and mesh_nearest_face: nodes
// nearer than the current bound (padded, so that a tie is still visited) are
// opened nearest child first, and `leaf(first, count)` scores each leaf range.
// `bound()` is the current search radius (+inf before anything is found).
template <class Leaf, class Bound>
__device__ __forceinline__ void mesh_walk(const MeshView &m, const float *pc, Leaf &&leaf,
                                          Bound &&bound, uint32_t &status) {
  auto bound2 = [&]() {
    float b = bound();
    if (b == f_inf()) return f_inf();
    float s = b + 4e-6f * b + m.pad;
    return s * s;
  };
  if (m.root_leaf) {
    leaf(0, int(m.root_leaf));
    return;
  }
  int stack_n[STACK];
  float stack_k[STACK];
  int sp = 0, node = 0;
  uint32_t visits = 0;
  for (;;) {
    if (++visits > 2u * m.nf + 64u) {
      status |= ST_STACK;
      break;
    }
    Child2 n = load_node(m.nodes, node);
    float k[2] = {box_dist2(n.lo0, n.hi0, pc), box_dist2(n.lo1, n.hi1, pc)};
    int near_c = k[1] < k[0] ? 1 : 0;
    int next = -1;
    for (int q = 0; q < 2; ++q) {
      int c = q == 0 ? near_c : 1 - near_c;
      if (!(k[c] <= bound2())) continue;
      if (n.cnt[c]) {
        leaf(n.ref[c], n.cnt[c]);
      } else if (next < 0) {
        next = n.ref[c];
      } else if (sp < STACK) {
        stack_n[sp] = n.ref[c];
        stack_k[sp++] = k[c];
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

// RayScene::bounded_distance (spatial/bvh.rs:123-131): the distance to the
// nearest face when it is <= window (inclusive), else +inf. window = +inf is
// RayScene::distance (bvh.rs:110-113).
__device__ __noinline__ float mesh_distance(const MeshView &m, F3 p, float window, uint32_t &status) {
  float best = f_inf();
  if (m.nf == 0 || !(window > 0.0f)) return best;
  float pc[3] = {p.x, p.y, p.z};
  mesh_walk(
      m, pc,
      [&](int first, int count) {
        for (int s = first; s < first + count; ++s) {
          F3 a, b, c;
          uint32_t id;
          tri_at(m, s, a, b, c, id);
          float dd = tri_distance(p, a, b, c);
          if (dd <= window && dd < best) best = dd;
        }
      },
      [&]() { return fminf(best, window); }, status);
  return best;
}

// Whether some face lies within `window` of p (inclusive): the same walk as
// mesh_distance with its bound held at the window, stopping at the first face
// found. True exactly when mesh_distance(m, p, window) would be finite, so a
// caller that only needs "within the window or not" is spared the rest of the
// nearest-face search.
__device__ __noinline__ bool mesh_any_within(const MeshView &m, F3 p, float window,
                                             uint32_t &status) {
  if (m.nf == 0 || !(window >= 0.0f)) return false;
  const float pc[3] = {p.x, p.y, p.z};
  auto test = [&](int first, int count) {
    for (int s = first; s < first + count; ++s) {
      F3 a, b, c;
      uint32_t id;
      tri_at(m, s, a, b, c, id);
      if (tri_distance(p, a, b, c) <= window) return true;
    }
    return false;
  };
  if (m.root_leaf) return test(0, int(m.root_leaf));
  const float s = window + 4e-6f * window + m.pad;
  const float bound2 = s * s;

  int stack_n[STACK];
  int sp = 0, node = 0;
  uint32_t visits = 0;
  for (;;) {
    if (++visits > 2u * m.nf + 64u) {
      status |= ST_STACK;
      return false;
    }
    Child2 n = load_node(m.nodes, node);
    float k[2] = {box_dist2(n.lo0, n.hi0, pc), box_dist2(n.lo1, n.hi1, pc)};
    int near_c = k[1] < k[0] ? 1 : 0;
    int next = -1;
    for (int q = 0; q < 2; ++q) {
      int c = q == 0 ? near_c : 1 - near_c;
      if (!(k[c] <= bound2)) continue;
      if (n.cnt[c]) {
        if (test(n.ref[c], n.cnt[c])) return true;
      } else if (next < 0) {
        next = n.ref[c];
      } else if (sp < STACK) {
        stack_n[sp++] = n.ref[c];
      } else {
        status |= ST_STACK;
      }
    }
    if (next >= 0) {
      node = next;
      continue;
    }
    if (sp == 0) return false;
    node = stack_n[--sp];
  }
}

// A lower bound on the distance from p to every face of the mesh, read from
// the mesh's bound grid (0 where p is off the grid or the mesh has none): the
// smallest distance from p's grid cell, widened by a thousandth of a cell, to
// any leaf box of the tree, rounded down. A walk whose bound stays below it
// scores no leaf.
__device__ __forceinline__ float mesh_lower_bound(const MeshView &m, F3 p) {
  const LbGrid &g = m.lbg;
  if (!g.lb) return 0.0f;
  float fx = floorf((p.x - g.lo[0]) * g.inv_cell), fy = floorf((p.y - g.lo[1]) * g.inv_cell),
        fz = floorf((p.z - g.lo[2]) * g.inv_cell);
  if (!(fx >= 0.0f && fy >= 0.0f && fz >= 0.0f && fx < float(g.n[0]) && fy < float(g.n[1]) &&
        fz < float(g.n[2])))
    return 0.0f;
  return __ldg(g.lb + (size_t(fx) * g.n[1] + size_t(fy)) * g.n[2] + size_t(fz));
}

// Whether a walk bounded at `window` (mesh_distance, mesh_any_within) from p
// can score a face at all: false when the mesh's bound grid puts every leaf
// box beyond the walk's padded bound, with a relative margin of 1e-4 over the
// rounding of the walk's own box distances.
__device__ __forceinline__ bool mesh_may_reach(const MeshView &m, F3 p, float window) {
  return !(mesh_lower_bound(m, p) > (window + 4e-6f * window + m.pad) * 1.0001f);
}

// mesh_distance that also names the face: the sorted slot of the nearest face
// within the window, an exact f32 tie going to the lowest original face id
// (the rule first_hit uses); slot = MISS when nothing is within the window.
__device__ __noinline__ float mesh_nearest_face(const MeshView &m, F3 p, float window, uint32_t &slot,
                                                uint32_t &status) {
  float best = f_inf();
  uint32_t best_id = MISS;
  slot = MISS;
  if (m.nf == 0 || !(window > 0.0f)) return best;
  float pc[3] = {p.x, p.y, p.z};
  mesh_walk(
      m, pc,
      [&](int first, int count) {
        for (int s = first; s < first + count; ++s) {
          F3 a, b, c;
          uint32_t id;
          tri_at(m, s, a, b, c, id);
          float dd = tri_distance(p, a, b, c);
          if (dd <= window && (dd < best || (dd == best && id < best_id))) {
            best = dd;
            best_id = id;
            slot = uint32_t(s);
          }
        }
      },
      [&]() { return fminf(best, window); }, status);
  return best;
}

// PointTree::nearest_within_squared (spatial/kdtree.rs:202-217): the nearest
// point with d2 <= r2, lowest original index on an exact tie. Returns the
// sorted slot (or -1) and its squared distance; d2 = ((dx dx + dy dy) + dz dz).
//
// `hint` (a sorted slot, or -1) seeds the search with a point that is already
// a candidate, typically the previous ICP pass's match: its exact distance is
// the initial bound, so the traversal prunes from the first node. The answer
// is the same with or without it: the hint is a valid candidate, anything
// nearer replaces it, and an exact tie still goes to the lower index.
__device__ __noinline__ int nearest_within_sq(const CloudView &c, double qx, double qy, double qz, double r2,
                                 double &best, uint32_t &status, int hint = -1) {
  best = r2;
  int best_s = -1;
  uint32_t best_i = MISS;
  if (c.n == 0 || !(r2 >= 0.0)) return -1;
  if (hint >= 0) {
    double4 p = ldg4(c.pts + hint);
    double dx = qx - p.x, dy = qy - p.y, dz = qz - p.z;
    double d2 = (dx * dx + dy * dy) + dz * dz;
    if (d2 <= r2) {
      best = d2;
      best_s = hint;
      best_i = uint32_t(p.w);
    }
  }
  float qc[3] = {float(qx), float(qy), float(qz)};
  auto bound2 = [&]() {
    float b = __double2float_ru(best);
    return b + 1e-5f * b + 1e-30f;
  };
  auto leaf = [&](int first, int count) {
    for (int s = first; s < first + count; ++s) {
      double4 p = ldg4(c.pts + s);
      double dx = qx - p.x, dy = qy - p.y, dz = qz - p.z;
      double d2 = (dx * dx + dy * dy) + dz * dz;
      if (d2 > r2) continue;
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
    return best_s;
  }
  // Box distances are taken from the f32-rounded query; the padding of the
  // boxes (>= the rounding of the query) keeps them lower bounds.
  int stack_n[STACK];
  float stack_k[STACK];
  int sp = 0, node = 0;
  uint32_t visits = 0;
  if (c.wide) {
    wide_walk(
        c.wide, qc, 2u * c.n + 64u,
        [&](int first, int count) {
          leaf(first, count);
          return false;
        },
        bound2, status);
    return best_s;
  }
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
  return best_s;
}

// PointTree::nearest_below (spatial/kdtree.rs:182-190): the unbounded nearest
// point when sqrt(d2) < bound. Returns the sorted slot or -1.
__device__ __forceinline__ int nearest_below(const CloudView &c, double qx, double qy, double qz,
                                             double bound, double &dist, uint32_t &status) {
  if (!(bound > 0.0)) return -1;
  double widened = (bound * bound) * (1.0 + 4.0 * 2.220446049250313e-16);
  double d2;
  int s = nearest_within_sq(c, qx, qy, qz, widened, d2, status);
  if (s < 0) return -1;
  double d = sqrt(d2);
  if (!(d < bound)) return -1;
  dist = d;
  return s;
}

}  // namespace sherd
