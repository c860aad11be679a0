// oracle.cpp — CPU restatement of sherd-refit's geometry hot path.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker the CUDA backend is
// compared against; it is built into oracle/_build/liboracle.so and loaded by
// the tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg,
// never by the product library.
//
// Every function restates the reference (Rust crate `sherd-core`) and cites
// the file:line it follows. The reference's third-party geometry (parry3d
// 0.30.2 ray casts and point projection, kiddo 6.2.0 nearest neighbours) is
// not vendored; its published algorithms are restated here with one tie rule
// shared with the CUDA backend:
//   * first hit: Moller-Trumbore in f32 (the inside test's own kernel,
//     spatial/bvh.rs:199-220), smallest t, then lowest face index;
//   * point-to-triangle distance: the Voronoi-region closest point of
//     Ericson, "Real-Time Collision Detection", sec. 5.1.5, in f32;
//   * nearest neighbour: smallest squared distance ((dx^2 + dy^2) + dz^2 in
//     f64), then lowest point index (kiddo's observed rule, kdtree.rs:104-109).
// Spatial pruning (BVH boxes, KD planes) is conservative, so every answer is
// the brute-force answer under that rule.
//
// Built with -ffp-contract=off: the reference's arithmetic has no fused
// multiply-adds (Rust does not contract), and neither may this.

#include "../include/sherd_cuda.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

namespace {

constexpr float F_INF = std::numeric_limits<float>::infinity();
constexpr double D_INF = std::numeric_limits<double>::infinity();
constexpr uint32_t MISS = 0xFFFFFFFFu;

// Runs fn(0..n-1) on `threads` threads (in order on one).
template <class F>
void parallel_for(uint32_t n, int threads, F &&fn) {
  if (threads <= 1 || n < 2) {
    for (uint32_t i = 0; i < n; ++i) fn(i);
    return;
  }
  std::atomic<uint32_t> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; ++t)
    pool.emplace_back([&] {
      for (;;) {
        uint32_t i = next.fetch_add(1);
        if (i >= n) break;
        fn(i);
      }
    });
  for (auto &th : pool) th.join();
}

int default_threads() {
  unsigned h = std::thread::hardware_concurrency();
  return h ? int(h) : 1;
}

struct V3f {
  float x, y, z;
};
inline V3f sub(V3f a, V3f b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3f cross(V3f a, V3f b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline float dot(V3f a, V3f b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

// ---------------------------------------------------------------------------
// Poses (row-major 4x4 doubles)
// ---------------------------------------------------------------------------

// types::apply_transform (types.rs:175-181): R p + tau, left to right.
inline void apply(const double *t, const double *p, double *o) {
  for (int i = 0; i < 3; ++i)
    o[i] = t[4 * i] * p[0] + t[4 * i + 1] * p[1] + t[4 * i + 2] * p[2] + t[4 * i + 3];
}
// verify::rotate (verify.rs:711-717): R n, not renormalised.
inline void rotate(const double *t, const double *n, double *o) {
  for (int i = 0; i < 3; ++i) o[i] = t[4 * i] * n[0] + t[4 * i + 1] * n[1] + t[4 * i + 2] * n[2];
}
inline double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

void matmul4(const double *a, const double *b, double *o) {
  double r[16];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      double s = a[4 * i] * b[j];
      for (int k = 1; k < 4; ++k) s += a[4 * i + k] * b[4 * k + j];
      r[4 * i + j] = s;
    }
  std::memcpy(o, r, sizeof r);
}

// verify::pose_inverse (verify.rs:739-798): dgetf2 partial pivoting then one
// forward/back substitution per column of P*I.
void pose_inverse(const double *t, double *out) {
  double m[4][4];
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) m[i][j] = t[4 * i + j];
  int piv[4] = {0, 1, 2, 3};
  for (int k = 0; k < 4; ++k) {
    int best = k;
    for (int i = k + 1; i < 4; ++i)
      if (std::fabs(m[i][k]) > std::fabs(m[best][k])) best = i;
    if (best != k) {
      for (int c = 0; c < 4; ++c) std::swap(m[k][c], m[best][c]);
      std::swap(piv[k], piv[best]);
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

// ---------------------------------------------------------------------------
// Triangle BVH (RayScene, spatial/bvh.rs:36-192), f32 geometry
// ---------------------------------------------------------------------------

// Moller-Trumbore as spatial/bvh.rs:199-220 writes it. Returns the ray
// parameter of a crossing, or a negative value when there is none.
inline float moller_trumbore(V3f o, V3f d, V3f v0, V3f v1, V3f v2) {
  const float EPS = 1e-9f;
  V3f e1 = sub(v1, v0), e2 = sub(v2, v0);
  V3f pvec = cross(d, e2);
  float det = dot(e1, pvec);
  if (std::fabs(det) < EPS) return -1.0f;
  float inv = 1.0f / det;
  V3f tvec = sub(o, v0);
  float u = inv * dot(tvec, pvec);
  if (!(u >= 0.0f && u <= 1.0f)) return -1.0f;
  V3f qvec = cross(tvec, e1);
  float v = inv * dot(d, qvec);
  if (v < 0.0f || u + v > 1.0f) return -1.0f;
  float t = inv * dot(e2, qvec);
  return t > EPS ? t : -1.0f;
}

// Closest point on a triangle (Ericson 5.1.5, Voronoi regions), f32; returns
// the Euclidean distance sqrt((dx^2 + dy^2) + dz^2).
inline float tri_distance(V3f p, V3f a, V3f b, V3f c) {
  V3f ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
  float d1 = dot(ab, ap), d2 = dot(ac, ap);
  V3f q;
  if (d1 <= 0.0f && d2 <= 0.0f) {
    q = a;
  } else {
    V3f bp = sub(p, b);
    float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) {
      q = b;
    } else {
      float vc = d1 * d4 - d3 * d2;
      if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        float s = d1 / (d1 - d3);
        q = {a.x + s * ab.x, a.y + s * ab.y, a.z + s * ab.z};
      } else {
        V3f cp = sub(p, c);
        float d5 = dot(ab, cp), d6 = dot(ac, cp);
        if (d6 >= 0.0f && d5 <= d6) {
          q = c;
        } else {
          float vb = d5 * d2 - d1 * d6;
          if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
            float s = d2 / (d2 - d6);
            q = {a.x + s * ac.x, a.y + s * ac.y, a.z + s * ac.z};
          } else {
            float va = d3 * d6 - d5 * d4;
            float e43 = d4 - d3, e56 = d5 - d6;
            if (va <= 0.0f && e43 >= 0.0f && e56 >= 0.0f) {
              float s = e43 / (e43 + e56);
              V3f bc = sub(c, b);
              q = {b.x + s * bc.x, b.y + s * bc.y, b.z + s * bc.z};
            } else {
              float den = (va + vb) + vc;
              float v = vb / den, w = vc / den;
              q = {(a.x + ab.x * v) + ac.x * w, (a.y + ab.y * v) + ac.y * w,
                   (a.z + ab.z * v) + ac.z * w};
            }
          }
        }
      }
    }
  }
  V3f dq = sub(q, p);
  return std::sqrt(dot(dq, dq));
}

struct TriNode {
  float lo[3], hi[3];
  int32_t left, right;  // children, -1 for a leaf
  uint32_t first, count;
};

struct Mesh {
  std::vector<V3f> v;
  std::vector<uint32_t> f;  // 3 per face, face ids are positions in this mesh
  std::vector<TriNode> nodes;
  std::vector<uint32_t> order;
  float lo[3], hi[3];
  double pad;  // conservative box padding for every pruning test

  V3f vert(uint32_t face, int k) const { return v[f[3 * face + k]]; }
  uint32_t n_faces() const { return uint32_t(f.size() / 3); }

  void build() {
    uint32_t nf = n_faces();
    lo[0] = lo[1] = lo[2] = F_INF;
    hi[0] = hi[1] = hi[2] = -F_INF;
    double mag = 1.0;
    for (uint32_t i = 0; i < nf; ++i)
      for (int k = 0; k < 3; ++k) {
        V3f p = vert(i, k);
        float c[3] = {p.x, p.y, p.z};
        for (int a = 0; a < 3; ++a) {
          lo[a] = std::min(lo[a], c[a]);
          hi[a] = std::max(hi[a], c[a]);
          mag = std::max(mag, std::fabs(double(c[a])));
        }
      }
    pad = 1e-5 * mag;
    order.resize(nf);
    for (uint32_t i = 0; i < nf; ++i) order[i] = i;
    nodes.clear();
    nodes.reserve(2 * nf / 2 + 8);
    if (nf) build_node(0, nf);
  }

  int build_node(uint32_t b, uint32_t e) {
    int id = int(nodes.size());
    nodes.push_back({});
    TriNode nd;
    for (int a = 0; a < 3; ++a) {
      nd.lo[a] = F_INF;
      nd.hi[a] = -F_INF;
    }
    float clo[3] = {F_INF, F_INF, F_INF}, chi[3] = {-F_INF, -F_INF, -F_INF};
    for (uint32_t i = b; i < e; ++i) {
      double cen[3] = {0, 0, 0};
      for (int k = 0; k < 3; ++k) {
        V3f p = vert(order[i], k);
        float c[3] = {p.x, p.y, p.z};
        for (int a = 0; a < 3; ++a) {
          nd.lo[a] = std::min(nd.lo[a], c[a]);
          nd.hi[a] = std::max(nd.hi[a], c[a]);
          cen[a] += c[a];
        }
      }
      for (int a = 0; a < 3; ++a) {
        clo[a] = std::min(clo[a], float(cen[a] / 3));
        chi[a] = std::max(chi[a], float(cen[a] / 3));
      }
    }
    if (e - b <= 4) {
      nd.left = nd.right = -1;
      nd.first = b;
      nd.count = e - b;
      nodes[id] = nd;
      return id;
    }
    int axis = 0;
    for (int a = 1; a < 3; ++a)
      if (chi[a] - clo[a] > chi[axis] - clo[axis]) axis = a;
    uint32_t mid = (b + e) / 2;
    auto key = [&](uint32_t face) {
      float s = 0;
      for (int k = 0; k < 3; ++k) {
        V3f p = vert(face, k);
        s += (axis == 0 ? p.x : axis == 1 ? p.y : p.z);
      }
      return s;
    };
    std::nth_element(order.begin() + b, order.begin() + mid, order.begin() + e,
                     [&](uint32_t x, uint32_t y) {
                       float kx = key(x), ky = key(y);
                       return kx < ky || (kx == ky && x < y);
                     });
    nd.count = 0;
    nd.first = 0;
    nd.left = build_node(b, mid);
    nd.right = build_node(mid, e);
    nodes[id] = nd;
    return id;
  }

  // Entry parameter of the ray into the padded box (twice the padding, so it
  // also holds every face rectangle of crossings()), or +inf when it misses.
  double ray_box(const TriNode &n, const double *o, const double *invd) const {
    double t0 = 0.0, t1 = D_INF;
    for (int a = 0; a < 3; ++a) {
      double l = double(n.lo[a]) - 2.0 * pad, h = double(n.hi[a]) + 2.0 * pad;
      if (std::isinf(invd[a])) {
        if (o[a] < l || o[a] > h) return D_INF;
        continue;
      }
      double ta = (l - o[a]) * invd[a], tb = (h - o[a]) * invd[a];
      if (ta > tb) std::swap(ta, tb);
      t0 = std::max(t0, ta);
      t1 = std::min(t1, tb);
    }
    return t0 <= t1 ? t0 : D_INF;
  }

  double box_dist(const TriNode &n, const float *p) const {
    double s = 0.0;
    for (int a = 0; a < 3; ++a) {
      double l = double(n.lo[a]) - pad, h = double(n.hi[a]) + pad, q = p[a];
      double g = q < l ? l - q : (q > h ? q - h : 0.0);
      s += g * g;
    }
    return std::sqrt(s);
  }

  // RayScene::first_hit (bvh.rs:84-90) under the tie rule of this file.
  void first_hit(V3f o, V3f d, float *t_out, uint32_t *prim_out) const {
    float best = F_INF;
    uint32_t bi = MISS;
    if (nodes.empty()) {
      *t_out = best;
      *prim_out = bi;
      return;
    }
    double od[3] = {o.x, o.y, o.z}, dd[3] = {d.x, d.y, d.z}, invd[3];
    double dn = std::sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
    for (int a = 0; a < 3; ++a) invd[a] = 1.0 / dd[a];
    double slack = dn > 0 ? 4.0 * pad / dn : D_INF;
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
      const TriNode &n = nodes[stack[--sp]];
      double te = ray_box(n, od, invd);
      if (te == D_INF || te > double(best) + slack) continue;
      if (n.left < 0) {
        for (uint32_t i = n.first; i < n.first + n.count; ++i) {
          uint32_t face = order[i];
          float t = moller_trumbore(o, d, vert(face, 0), vert(face, 1), vert(face, 2));
          if (t < 0.0f) continue;
          if (t < best || (t == best && face < bi)) {
            best = t;
            bi = face;
          }
        }
      } else {
        stack[sp++] = n.left;
        stack[sp++] = n.right;
      }
    }
    *t_out = best;
    *prim_out = bi;
  }

  // RayScene::crossings (bvh.rs:160-175) along a coordinate axis: the faces
  // whose projected rectangle, padded outward by the mesh padding in f32 with
  // directed rounding, holds the origin's projection and that Moller-Trumbore
  // reports crossed (the rule the CUDA backend's axis grids implement).
  uint32_t crossings(V3f o, V3f d) const {
    if (nodes.empty()) return 0;
    int axis = d.x != 0.0f ? 0 : (d.y != 0.0f ? 1 : 2);
    int au = (axis + 1) % 3, av = (axis + 2) % 3;
    float oc[3] = {o.x, o.y, o.z};
    float padf = float(pad);
    auto rd = [](float a, float b) {  // a - b rounded toward -inf
      float r = a - b;
      if (double(r) > double(a) - double(b)) r = std::nextafter(r, -F_INF);
      return r;
    };
    auto ru = [](float a, float b) {  // a + b rounded toward +inf
      float r = a + b;
      if (double(r) < double(a) + double(b)) r = std::nextafter(r, F_INF);
      return r;
    };
    auto in_rect = [&](uint32_t face) {
      float lo_u = F_INF, hi_u = -F_INF, lo_v = F_INF, hi_v = -F_INF;
      for (int k = 0; k < 3; ++k) {
        V3f p = vert(face, k);
        float c[3] = {p.x, p.y, p.z};
        lo_u = std::min(lo_u, c[au]);
        hi_u = std::max(hi_u, c[au]);
        lo_v = std::min(lo_v, c[av]);
        hi_v = std::max(hi_v, c[av]);
      }
      return !(oc[au] < rd(lo_u, padf) || oc[au] > ru(hi_u, padf) || oc[av] < rd(lo_v, padf) ||
               oc[av] > ru(hi_v, padf));
    };
    double od[3] = {o.x, o.y, o.z}, invd[3] = {1.0 / d.x, 1.0 / d.y, 1.0 / d.z};
    uint32_t hits = 0;
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
      const TriNode &n = nodes[stack[--sp]];
      if (ray_box(n, od, invd) == D_INF) continue;
      if (n.left < 0) {
        for (uint32_t i = n.first; i < n.first + n.count; ++i) {
          uint32_t face = order[i];
          if (!in_rect(face)) continue;
          if (moller_trumbore(o, d, vert(face, 0), vert(face, 1), vert(face, 2)) >= 0.0f) ++hits;
        }
      } else {
        stack[sp++] = n.left;
        stack[sp++] = n.right;
      }
    }
    return hits;
  }

  // RayScene::inside (bvh.rs:146-157): majority of the +x, +y, +z parities.
  bool inside(V3f p) const {
    int votes = 0;
    const V3f dirs[3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    for (int a = 0; a < 3; ++a)
      if (crossings(p, dirs[a]) % 2 == 1) ++votes;
    return votes >= 2;
  }

  // Distance to the nearest face when it is <= window (inclusive), else +inf.
  // RayScene::bounded_distance (bvh.rs:123-131) with window = +inf is
  // RayScene::distance (bvh.rs:110-113).
  float distance(V3f p, float window) const {
    if (nodes.empty() || !(window > 0.0f)) return F_INF;
    float best = F_INF;
    float pf[3] = {p.x, p.y, p.z};
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
      const TriNode &n = nodes[stack[--sp]];
      double bound = std::min(double(best), double(window));
      if (box_dist(n, pf) > bound + pad) continue;
      if (n.left < 0) {
        for (uint32_t i = n.first; i < n.first + n.count; ++i) {
          uint32_t face = order[i];
          float dd = tri_distance(p, vert(face, 0), vert(face, 1), vert(face, 2));
          if (dd <= window && dd < best) best = dd;
        }
      } else {
        stack[sp++] = n.left;
        stack[sp++] = n.right;
      }
    }
    return best;
  }

  // distance() that also names the face: the nearest face within the window,
  // an exact f32 tie going to the lowest face id; MISS-like 0xFFFFFFFF when
  // nothing is within the window.
  float nearest_face(V3f p, float window, uint32_t *face_out) const {
    *face_out = 0xFFFFFFFFu;
    if (nodes.empty() || !(window > 0.0f)) return F_INF;
    float best = F_INF;
    float pf[3] = {p.x, p.y, p.z};
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
      const TriNode &n = nodes[stack[--sp]];
      double bound = std::min(double(best), double(window));
      if (box_dist(n, pf) > bound + pad) continue;
      if (n.left < 0) {
        for (uint32_t i = n.first; i < n.first + n.count; ++i) {
          uint32_t face = order[i];
          float dd = tri_distance(p, vert(face, 0), vert(face, 1), vert(face, 2));
          if (dd <= window && (dd < best || (dd == best && face < *face_out))) {
            best = dd;
            *face_out = face;
          }
        }
      } else {
        stack[sp++] = n.left;
        stack[sp++] = n.right;
      }
    }
    return best;
  }
};

// ---------------------------------------------------------------------------
// KD tree over f64 points (PointTree, spatial/kdtree.rs:31-258)
// ---------------------------------------------------------------------------

struct KdNode {
  int32_t axis;  // -1 for a leaf
  double split;
  int32_t left, right;
  uint32_t first, count;
};

struct Cloud {
  std::vector<double> p;  // 3 per point
  std::vector<double> n;  // 3 per point, or empty
  std::vector<uint32_t> order;
  std::vector<KdNode> nodes;

  uint32_t size() const { return uint32_t(p.size() / 3); }

  void build() {
    uint32_t np = size();
    order.resize(np);
    for (uint32_t i = 0; i < np; ++i) order[i] = i;
    nodes.clear();
    if (np) build_node(0, np);
  }

  int build_node(uint32_t b, uint32_t e) {
    int id = int(nodes.size());
    nodes.push_back({});
    KdNode nd{};
    if (e - b <= 8) {
      nd.axis = -1;
      nd.first = b;
      nd.count = e - b;
      nodes[id] = nd;
      return id;
    }
    double lo[3] = {D_INF, D_INF, D_INF}, hi[3] = {-D_INF, -D_INF, -D_INF};
    for (uint32_t i = b; i < e; ++i)
      for (int a = 0; a < 3; ++a) {
        lo[a] = std::min(lo[a], p[3 * order[i] + a]);
        hi[a] = std::max(hi[a], p[3 * order[i] + a]);
      }
    int axis = 0;
    for (int a = 1; a < 3; ++a)
      if (hi[a] - lo[a] > hi[axis] - lo[axis]) axis = a;
    uint32_t mid = (b + e) / 2;
    std::nth_element(order.begin() + b, order.begin() + mid, order.begin() + e,
                     [&](uint32_t x, uint32_t y) {
                       double kx = p[3 * x + axis], ky = p[3 * y + axis];
                       return kx < ky || (kx == ky && x < y);
                     });
    nd.axis = axis;
    nd.split = p[3 * order[mid] + axis];
    nd.left = build_node(b, mid);
    nd.right = build_node(mid, e);
    nodes[id] = nd;
    return id;
  }

  // PointTree::nearest_within_squared (kdtree.rs:202-217): the nearest point
  // with d2 <= r2, lowest index on an exact tie.
  bool nearest_within_sq(const double *q, double r2, uint32_t *bi, double *bd) const {
    if (!(r2 >= 0.0) || nodes.empty()) return false;
    bool found = false;
    double best = r2;
    uint32_t besti = MISS;
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
      const KdNode &nd = nodes[stack[--sp]];
      if (nd.axis < 0) {
        for (uint32_t k = nd.first; k < nd.first + nd.count; ++k) {
          uint32_t i = order[k];
          double dx = q[0] - p[3 * i], dy = q[1] - p[3 * i + 1], dz = q[2] - p[3 * i + 2];
          double d2 = (dx * dx + dy * dy) + dz * dz;
          if (d2 > r2) continue;
          if (!found || d2 < best || (d2 == best && i < besti)) {
            found = true;
            best = d2;
            besti = i;
          }
        }
        continue;
      }
      double diff = q[nd.axis] - nd.split;
      double lb = diff * diff;
      int near_c = diff < 0 ? nd.left : nd.right, far_c = diff < 0 ? nd.right : nd.left;
      // Both sides of the plane can hold points equal to the split value, so
      // the far side is kept whenever its bound does not exceed the best.
      if (lb <= best) stack[sp++] = far_c;
      stack[sp++] = near_c;
    }
    if (found) {
      *bi = besti;
      *bd = best;
    }
    return found;
  }

  // PointTree::nearest_below (kdtree.rs:182-190).
  bool nearest_below(const double *q, double bound, uint32_t *bi, double *dist) const {
    if (!(bound > 0.0)) return false;
    double widened = (bound * bound) * (1.0 + 4.0 * std::numeric_limits<double>::epsilon());
    uint32_t i;
    double d2;
    if (!nearest_within_sq(q, widened, &i, &d2)) return false;
    double d = std::sqrt(d2);
    if (!(d < bound)) return false;
    *bi = i;
    *dist = d;
    return true;
  }
};

// ---------------------------------------------------------------------------
// ICP (matching/icp.rs:308-890), reference numerics (f64 point loops, World)
// ---------------------------------------------------------------------------

// icp::eigen_pivots (icp.rs:661-674).
void eigen_pivots(const double a[6][6], int perm[6]) {
  for (int k = 0; k < 6; ++k) perm[k] = k;
  for (int k = 0; k < 6; ++k) {
    int best = k;
    for (int i = k + 1; i < 6; ++i)
      if (std::fabs(a[perm[i]][perm[i]]) > std::fabs(a[perm[best]][perm[best]])) best = i;
    std::swap(perm[k], perm[best]);
  }
}

// icp::solve_ldlt (icp.rs:692-753).
bool solve_ldlt(const double a[6][6], const double b[6], double x[6]) {
  int perm[6];
  eigen_pivots(a, perm);
  double m[6][6];
  for (int k = 0; k < 6; ++k)
    for (int l = 0; l < 6; ++l) m[k][l] = a[perm[k]][perm[l]];
  for (int k = 0; k < 6; ++k) {
    if (k > 0) {
      double temp[6] = {0, 0, 0, 0, 0, 0};
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
    y[i] = std::fabs(pivot) > std::numeric_limits<double>::min() ? y[i] / pivot : 0.0;
  }
  for (int i = 5; i >= 0; --i) {
    double value = y[i];
    for (int j = i + 1; j < 6; ++j) value -= m[j][i] * y[j];
    y[i] = value;
  }
  for (int k = 0; k < 6; ++k) x[perm[k]] = y[k];
  for (int k = 0; k < 6; ++k)
    if (!std::isfinite(x[k])) return false;
  return true;
}

void mat3mul(const double a[3][3], const double b[3][3], double o[3][3]) {
  double r[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) r[i][j] = (a[i][0] * b[0][j] + a[i][1] * b[1][j]) + a[i][2] * b[2][j];
  std::memcpy(o, r, sizeof r);
}

// icp::euler_zyx (icp.rs:770-778): Rz(g) Ry(b) Rx(a).
void euler_zyx(double al, double be, double ga, double r[3][3]) {
  double sa = std::sin(al), ca = std::cos(al), sb = std::sin(be), cb = std::cos(be);
  double sg = std::sin(ga), cg = std::cos(ga);
  double rx[3][3] = {{1, 0, 0}, {0, ca, -sa}, {0, sa, ca}};
  double ry[3][3] = {{cb, 0, sb}, {0, 1, 0}, {-sb, 0, cb}};
  double rz[3][3] = {{cg, -sg, 0}, {sg, cg, 0}, {0, 0, 1}};
  double t[3][3];
  mat3mul(rz, ry, t);
  mat3mul(t, rx, r);
}

struct Corr {
  uint32_t i, j;
};

// icp::correspondences (icp.rs:361-392).
void correspondences(const std::vector<double> &moved, const Cloud &tgt, double distance,
                     std::vector<Corr> &out, double *fit, double *rmse, int threads = 1) {
  out.clear();
  *fit = 0.0;
  *rmse = 0.0;
  if (tgt.nodes.empty()) return;
  if (!(distance > 0.0)) return;
  double r2 = distance * distance;
  double err = 0.0;
  size_t n = moved.size() / 3;
  if (threads > 1 && n >= 4096) {
    // The searches on `threads` threads, the sum afterwards in point order: the same
    // correspondences and the same rounding as the loop below.
    std::vector<uint32_t> js(n);
    std::vector<double> d2s(n);
    std::vector<uint8_t> ok(n);
    parallel_for(uint32_t(n), threads, [&](uint32_t i) {
      ok[i] = tgt.nearest_within_sq(&moved[3 * size_t(i)], r2, &js[i], &d2s[i]) && d2s[i] < r2;
    });
    for (size_t i = 0; i < n; ++i) {
      if (!ok[i]) continue;
      err += d2s[i];
      out.push_back({uint32_t(i), js[i]});
    }
  } else {
    for (size_t i = 0; i < n; ++i) {
      uint32_t j;
      double d2;
      if (!tgt.nearest_within_sq(&moved[3 * i], r2, &j, &d2)) continue;
      if (d2 >= r2) continue;
      err += d2;
      out.push_back({uint32_t(i), j});
    }
  }
  if (out.empty()) return;
  double nc = double(out.size()), ns = double(n);
  *fit = nc / ns;
  *rmse = std::sqrt(err / nc);
}

// icp::point_to_plane (icp.rs:408-440) with normal_equations (icp.rs:599-640)
// under Assembly::World and Precision::F64.
// icp::normal_equations (icp.rs:599-640) under Assembly::World and
// Precision::F64: J^T J (lower triangle) and J^T r, rows (p x n, n), in
// correspondence order.
void normal_equations(const std::vector<double> &moved, const Cloud &tgt,
                      const std::vector<Corr> &corr, double jtj[6][6], double jtr[6]) {
  for (int k = 0; k < 6; ++k) {
    jtr[k] = 0.0;
    for (int l = 0; l < 6; ++l) jtj[k][l] = 0.0;
  }
  for (const Corr &c : corr) {
    const double *p = &moved[3 * c.i], *q = &tgt.p[3 * c.j], *n = &tgt.n[3 * c.j];
    double pc[3] = {p[0] - 0.0, p[1] - 0.0, p[2] - 0.0};
    double row[6] = {pc[1] * n[2] - pc[2] * n[1], pc[2] * n[0] - pc[0] * n[2],
                     pc[0] * n[1] - pc[1] * n[0], n[0], n[1], n[2]};
    double r = (p[0] - q[0]) * n[0] + (p[1] - q[1]) * n[1] + (p[2] - q[2]) * n[2];
    for (int k = 0; k < 6; ++k) {
      for (int l = 0; l <= k; ++l) jtj[k][l] = jtj[k][l] + row[k] * row[l];
      jtr[k] = jtr[k] + row[k] * r;
    }
  }
}

void point_to_plane(const std::vector<double> &moved, const Cloud &tgt,
                    const std::vector<Corr> &corr, double u[16]) {
  for (int i = 0; i < 16; ++i) u[i] = (i % 5 == 0) ? 1.0 : 0.0;
  if (corr.empty() || tgt.n.size() != tgt.p.size()) return;
  double jtj[6][6], jtr[6];
  normal_equations(moved, tgt, corr, jtj, jtr);
  double a[6][6];
  for (int k = 0; k < 6; ++k)
    for (int l = 0; l <= k; ++l) {
      a[k][l] = jtj[k][l];
      a[l][k] = jtj[k][l];
    }
  double rhs[6], x[6];
  for (int k = 0; k < 6; ++k) rhs[k] = -jtr[k];
  if (!solve_ldlt(a, rhs, x)) return;
  double r[3][3];
  euler_zyx(x[0], x[1], x[2], r);
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) u[4 * i + j] = r[i][j];
    u[4 * i + 3] = x[3 + i];
  }
}

// The rotation of a 3x3 SVD with the reflection on the smallest singular
// value undone, R = U diag(1, 1, det(U) det(V)) V^T, as Eigen's umeyama takes
// it from nalgebra 0.34.2's SVD (icp.rs:585-590; the SVD itself is
// third-party and not in the reference tree). Restated with the eigen-
// decomposition of m^T m by cyclic Jacobi: V its eigenvectors, singular values
// the roots of its eigenvalues (descending), u0 and u1 from m V / sigma and
// u2 = u0 x u1. R is unique whenever the second singular value is not zero,
// so any exact SVD gives it up to rounding.
void svd_rotation(const double m[3][3], double r[3][3]) {
  double s[3][3], v[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      double acc = 0.0;
      for (int k = 0; k < 3; ++k) acc += m[k][i] * m[k][j];
      s[i][j] = acc;
    }
  for (int sweep = 0; sweep < 50; ++sweep) {
    double off = std::fabs(s[0][1]) + std::fabs(s[0][2]) + std::fabs(s[1][2]);
    double scale = std::fabs(s[0][0]) + std::fabs(s[1][1]) + std::fabs(s[2][2]);
    if (!(off > 1e-30 * scale)) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (s[p][q] == 0.0) continue;
        double theta = (s[q][q] - s[p][p]) / (2.0 * s[p][q]);
        double t = (theta >= 0.0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), sn = t * c;
        for (int k = 0; k < 3; ++k) {  // s <- J^T s J, v <- v J
          double x = s[k][p], y = s[k][q];
          s[k][p] = c * x - sn * y;
          s[k][q] = sn * x + c * y;
        }
        for (int k = 0; k < 3; ++k) {
          double x = s[p][k], y = s[q][k];
          s[p][k] = c * x - sn * y;
          s[q][k] = sn * x + c * y;
        }
        for (int k = 0; k < 3; ++k) {
          double x = v[k][p], y = v[k][q];
          v[k][p] = c * x - sn * y;
          v[k][q] = sn * x + c * y;
        }
      }
  }
  int ord[3] = {0, 1, 2};
  std::sort(ord, ord + 3, [&](int a, int b) { return s[a][a] > s[b][b]; });
  double sv[3], u[3][3], w[3][3];
  bool have[3];
  double smax = std::sqrt(std::max(s[ord[0]][ord[0]], 0.0));
  for (int k = 0; k < 3; ++k) {
    int j = ord[k];
    sv[k] = std::sqrt(std::max(s[j][j], 0.0));
    for (int i = 0; i < 3; ++i) w[i][k] = v[i][j];
    have[k] = smax > 0.0 && sv[k] > 1e-12 * smax;
    for (int i = 0; i < 3; ++i) {
      double mv = m[i][0] * w[0][k] + m[i][1] * w[1][k] + m[i][2] * w[2][k];
      u[i][k] = have[k] ? mv / sv[k] : 0.0;
    }
  }
  if (!have[0]) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) r[i][j] = i == j ? 1.0 : 0.0;
    return;
  }
  auto cross = [](const double *a, const double *b, double *o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
  };
  double c0[3] = {u[0][0], u[1][0], u[2][0]}, c1[3], c2[3];
  if (have[1]) {  // m w1 / sigma1, made orthogonal to u0 again
    double dp = c0[0] * u[0][1] + c0[1] * u[1][1] + c0[2] * u[2][1];
    for (int i = 0; i < 3; ++i) c1[i] = u[i][1] - dp * c0[i];
    double n1 = std::sqrt(c1[0] * c1[0] + c1[1] * c1[1] + c1[2] * c1[2]);
    for (double &x : c1) x /= n1;
  } else {
    int e = 0;
    for (int i = 1; i < 3; ++i)
      if (std::fabs(c0[i]) < std::fabs(c0[e])) e = i;
    double ev[3] = {0, 0, 0};
    ev[e] = 1.0;
    cross(c0, ev, c1);
    double n1 = std::sqrt(c1[0] * c1[0] + c1[1] * c1[1] + c1[2] * c1[2]);
    for (double &x : c1) x /= n1;
  }
  // u2 = u0 x u1 always: for rank 3 the SVD's own u2 is +-(u0 x u1) and the
  // det(U) det(V) factor below absorbs the sign; for rank 2 it is the only
  // stable choice (m w2 / sigma2 is round-off there).
  cross(c0, c1, c2);
  for (int i = 0; i < 3; ++i) {
    u[i][0] = c0[i];
    u[i][1] = c1[i];
    u[i][2] = c2[i];
  }
  auto det3 = [](const double x[3][3]) {
    return x[0][0] * (x[1][1] * x[2][2] - x[1][2] * x[2][1]) -
           x[0][1] * (x[1][0] * x[2][2] - x[1][2] * x[2][0]) +
           x[0][2] * (x[1][0] * x[2][1] - x[1][1] * x[2][0]);
  };
  double d = det3(u) * det3(w) < 0.0 ? -1.0 : 1.0;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      r[i][j] = u[i][0] * w[j][0] + u[i][1] * w[j][1] + d * u[i][2] * w[j][2];
}

// icp::umeyama without scaling (icp.rs:527-592) over the correspondences in
// their order: means as sum * (1/n), the covariance with 1/n folded into each
// term, R from the SVD, tau = mean_q - R mean_p.
void point_to_point(const std::vector<double> &moved, const Cloud &tgt,
                    const std::vector<Corr> &corr, double u[16]) {
  for (int i = 0; i < 16; ++i) u[i] = (i % 5 == 0) ? 1.0 : 0.0;
  if (corr.empty()) return;
  double one_over_n = 1.0 / double(corr.size());
  double sp[3] = {0, 0, 0}, sq[3] = {0, 0, 0};
  for (const Corr &c : corr)
    for (int k = 0; k < 3; ++k) {
      sp[k] = sp[k] + moved[3 * c.i + k];
      sq[k] = sq[k] + tgt.p[3 * c.j + k];
    }
  double mp[3], mq[3];
  for (int k = 0; k < 3; ++k) {
    mp[k] = sp[k] * one_over_n;
    mq[k] = sq[k] * one_over_n;
  }
  double sigma[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  for (const Corr &c : corr) {
    double a[3], b[3];
    for (int k = 0; k < 3; ++k) {
      a[k] = moved[3 * c.i + k] - mp[k];
      b[k] = (tgt.p[3 * c.j + k] - mq[k]) * one_over_n;
    }
    for (int r = 0; r < 3; ++r)
      for (int cc = 0; cc < 3; ++cc) sigma[r][cc] = sigma[r][cc] + b[r] * a[cc];
  }
  double rot[3][3];
  svd_rotation(sigma, rot);
  for (int i = 0; i < 3; ++i) {
    for (int j = 0; j < 3; ++j) u[4 * i + j] = rot[i][j];
    u[4 * i + 3] = mq[i] - (rot[i][0] * mp[0] + rot[i][1] * mp[1] + rot[i][2] * mp[2]);
  }
}

void transform_points(std::vector<double> &pts, const double *m) {
  size_t n = pts.size() / 3;
  for (size_t i = 0; i < n; ++i) {
    double p[3] = {pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]}, o[3];
    apply(m, p, o);
    pts[3 * i] = o[0];
    pts[3 * i + 1] = o[1];
    pts[3 * i + 2] = o[2];
  }
}

// icp::register (icp.rs:308-356), point-to-plane.
sherd_registration icp_register(const double *src, uint32_t ns, const Cloud &tgt,
                                const double *init, const sherd_icp_options &opt,
                                int threads = 1) {
  sherd_registration out{};
  std::memcpy(out.transform, init, sizeof out.transform);
  if (ns == 0 || tgt.size() == 0) return out;
  double t[16];
  std::memcpy(t, init, sizeof t);
  std::vector<double> moved(src, src + 3 * size_t(ns));
  transform_points(moved, init);
  std::vector<Corr> corr;
  double fit, rmse;
  correspondences(moved, tgt, opt.max_correspondence_distance, corr, &fit, &rmse, threads);
  uint32_t iterations = 0;
  bool converged = false;
  for (int it = 0; it < opt.max_iteration; ++it) {
    double u[16];
    if (opt.estimation == SHERD_POINT_TO_POINT)
      point_to_point(moved, tgt, corr, u);
    else
      point_to_plane(moved, tgt, corr, u);
    matmul4(u, t, t);
    transform_points(moved, u);
    ++iterations;
    double nfit, nrmse;
    correspondences(moved, tgt, opt.max_correspondence_distance, corr, &nfit, &nrmse, threads);
    converged = std::fabs(nfit - fit) < 1e-6 && std::fabs(nrmse - rmse) < 1e-6;
    fit = nfit;
    rmse = nrmse;
    if (converged) break;
  }
  std::memcpy(out.transform, t, sizeof t);
  out.fitness = fit;
  out.inlier_rmse = rmse;
  out.correspondences = corr.size();
  out.iterations = iterations;
  out.converged = converged ? 1u : 0u;
  return out;
}

// ---------------------------------------------------------------------------
// Verification (matching/verify.rs:318-638)
// ---------------------------------------------------------------------------

struct Surfaces {
  const Mesh *fracture = nullptr;
  const Mesh *mesh = nullptr;
  bool watertight = false;
  double frac_area = 0.0;
  std::vector<double> pf, s, brk_p, brk_ns, margin_p, margin_n;
  Cloud margin_tree;
};

// verify::median (verify.rs:693-700): numpy's median, sorted in place.
double median(std::vector<double> &v) {
  std::sort(v.begin(), v.end());
  size_t n = v.size();
  if (n == 0) return std::nan("");
  if (n % 2 == 1) return v[n / 2];
  return (v[n / 2 - 1] + v[n / 2]) / 2.0;
}

V3f narrow(const double *p) { return {float(p[0]), float(p[1]), float(p[2])}; }

// CpuExecutor::bounded_distance (executor/cpu.rs:84-113).
void bounded_distance(const Mesh &m, const double *pts, uint32_t n, const double *pose,
                      double max_dist, int reduce, double *out) {
  float window = float(max_dist);
  if (reduce == SHERD_REDUCE_ALL) {
    for (uint32_t i = 0; i < n; ++i) {
      double q[3];
      apply(pose, pts + 3 * i, q);
      float d = m.distance(narrow(q), window);
      out[i] = d == F_INF ? D_INF : double(d);
    }
  } else {
    float best = window;
    for (uint32_t i = 0; i < n; ++i) {
      double q[3];
      apply(pose, pts + 3 * i, q);
      float d = m.distance(narrow(q), best);
      if (d != F_INF) best = std::min(best, d);
    }
    out[0] = double(best);
  }
}

// CpuExecutor::inside (executor/cpu.rs:115-128) and depth_inside (cpu.rs:182-188).
void inside_batch(const Mesh &m, const double *pts, uint32_t n, const double *pose,
                  sherd_inside_outcome *out) {
  for (uint32_t i = 0; i < n; ++i) {
    double q[3];
    apply(pose, pts + 3 * i, q);
    V3f p = narrow(q);
    float c[3] = {p.x, p.y, p.z};
    bool outside_box = false;
    for (int k = 0; k < 3; ++k)
      if (c[k] < m.lo[k] || c[k] > m.hi[k]) outside_box = true;
    if (outside_box || !m.inside(p)) {
      out[i] = {0.0f, 0u};
      continue;
    }
    out[i] = {float(double(m.distance(p, F_INF))), 1u};
  }
}

// verify::one_side (verify.rs:338-349).
void one_side(const std::vector<double> &d, double area, const sherd_scales &sc, double *tight,
              double *gap, double *contact) {
  std::vector<double> facing;
  for (double x : d)
    if (x < sc.facing) facing.push_back(x);
  if (facing.size() < 20) {
    *tight = 0.0;
    *gap = 1.0;
    *contact = 0.0;
    return;
  }
  size_t nt = 0;
  for (double x : facing)
    if (x < sc.tight) ++nt;
  *tight = double(nt) / double(facing.size());
  *gap = median(facing) / sc.t;
  size_t touching = 0;
  for (double x : d)
    if (x < 2.0 * sc.tight) ++touching;
  double share = double(touching) / double(d.size());
  *contact = share * area / (sc.t * sc.t);
}

// verify::seam_points + seam_cells + seam_score (verify.rs:378-442, 809-811).
double seam_score(const Surfaces &a, const Surfaces &b, const double *t, const sherd_scales &sc) {
  size_t nb = b.brk_p.size() / 3, na = a.brk_p.size() / 3;
  Cloud moved;
  moved.p.resize(3 * nb);
  std::vector<double> normals(3 * nb);
  for (size_t j = 0; j < nb; ++j) {
    apply(t, &b.brk_p[3 * j], &moved.p[3 * j]);
    rotate(t, &b.brk_ns[3 * j], &normals[3 * j]);
  }
  if (nb == 0) return 0.0;
  moved.build();
  double voxel = sc.t / 3.0;
  std::vector<std::array<int64_t, 3>> cells;
  for (size_t i = 0; i < na; ++i) {
    uint32_t j;
    double dist;
    if (!moved.nearest_below(&a.brk_p[3 * i], sc.seam, &j, &dist)) continue;
    if (dot3(&a.brk_ns[3 * i], &normals[3 * j]) > 0.7) {
      const double *p = &a.brk_p[3 * i];
      cells.push_back({int64_t(std::floor(p[0] / voxel)), int64_t(std::floor(p[1] / voxel)),
                       int64_t(std::floor(p[2] / voxel))});
    }
  }
  if (cells.empty()) return 0.0;
  std::sort(cells.begin(), cells.end());
  cells.erase(std::unique(cells.begin(), cells.end()), cells.end());
  return double(cells.size()) / 3.0;
}

// verify::continuity_scores (verify.rs:450-474).
void continuity_scores(const Surfaces &a, const Surfaces &b, const double *t,
                       const sherd_scales &sc, double *cont, double *cont_n) {
  *cont = 1.0;
  *cont_n = -1.0;
  if (a.margin_tree.nodes.empty() || b.margin_p.empty()) return;
  std::vector<double> steps, agreements;
  size_t nb = b.margin_p.size() / 3;
  for (size_t k = 0; k < nb; ++k) {
    double moved[3];
    apply(t, &b.margin_p[3 * k], moved);
    uint32_t j;
    double dist;
    if (!a.margin_tree.nearest_below(moved, sc.near, &j, &dist)) continue;
    const double *np = &a.margin_p[3 * j], *nn = &a.margin_n[3 * j];
    double delta[3] = {moved[0] - np[0], moved[1] - np[1], moved[2] - np[2]};
    steps.push_back(std::fabs(dot3(delta, nn)));
    double rn[3];
    rotate(t, &b.margin_n[3 * k], rn);
    agreements.push_back(dot3(rn, nn));
  }
  if (steps.size() <= 20) return;
  *cont = median(steps) / sc.t;
  *cont_n = median(agreements);
}

// verify::one_penetration (verify.rs:541-580).
void one_penetration(const std::vector<double> &pts, const double *t, const Mesh &scene,
                     double pen, double *fraction, double *mins) {
  *fraction = 0.0;
  *mins = 0.0;
  uint32_t n = uint32_t(pts.size() / 3);
  if (n == 0) return;
  std::vector<sherd_inside_outcome> outc(n);
  inside_batch(scene, pts.data(), n, t, outc.data());
  double deepest = -D_INF;
  size_t deeper = 0;
  for (auto &o : outc) {
    if (!o.inside) continue;
    double dd = double(o.depth);
    deepest = std::max(deepest, dd);
    if (dd > pen) ++deeper;
  }
  *fraction = double(deeper) / double(n);
  if (deepest > -D_INF) {
    *mins = -deepest;
    return;
  }
  double best;
  bounded_distance(scene, pts.data(), n, t, double(std::numeric_limits<float>::max()),
                   SHERD_REDUCE_MIN, &best);
  *mins = best;
}

// verify::verify (verify.rs:590-626).
sherd_scores verify(const Surfaces &a, const Surfaces &b, const double *t, const sherd_scales &sc,
                    bool full) {
  sherd_scores s{};
  double inv[16];
  pose_inverse(t, inv);
  std::vector<double> d1(b.pf.size() / 3), d2(a.pf.size() / 3);
  bounded_distance(*a.fracture, b.pf.data(), uint32_t(d1.size()), t, sc.facing,
                   SHERD_REDUCE_ALL, d1.data());
  bounded_distance(*b.fracture, a.pf.data(), uint32_t(d2.size()), inv, sc.facing,
                   SHERD_REDUCE_ALL, d2.data());
  one_side(d2, a.frac_area, sc, &s.tight_a, &s.gap_a, &s.contact_a);
  one_side(d1, b.frac_area, sc, &s.tight_b, &s.gap_b, &s.contact_b);
  s.tight = std::min(s.tight_a, s.tight_b);
  s.gap = std::max(s.gap_a, s.gap_b);
  s.contact = std::min(s.contact_a, s.contact_b);
  s.seam = seam_score(a, b, t, sc);
  s.gap_limit = sc.gap / sc.t;
  s.tight_delta = sc.tight / sc.t;
  s.cont = 1.0;
  s.cont_n = -1.0;
  s.pen = 0.0;
  s.pen_depth = 0.0;
  if (!full) {
    s.partial = 1;
    return s;
  }
  continuity_scores(a, b, t, sc, &s.cont, &s.cont_n);
  if (!a.mesh || !b.mesh || !(a.watertight && b.watertight)) {
    s.pen_unavailable = 1;
    return s;
  }
  double pen_b, min_b, pen_a, min_a;
  one_penetration(b.s, t, *a.mesh, sc.pen, &pen_b, &min_b);
  one_penetration(a.s, inv, *b.mesh, sc.pen, &pen_a, &min_a);
  s.pen = std::max(pen_a, pen_b);
  s.pen_depth = std::max(-min_a, -min_b) / sc.t;
  return s;
}

uint32_t accept(const sherd_scores &s, const sherd_params &p, const sherd_scales &sc) {
  return (s.tight >= p.min_tight && s.gap * sc.t <= sc.gap && s.pen <= p.max_pen &&
          s.seam >= p.min_seam && s.cont_n >= p.min_cont_n)
             ? 1u
             : 0u;
}

// ---------------------------------------------------------------------------
// The adjoint of the group-alignment objectives (no reference function: the
// values are R 6's tight fraction, smoothed, and the ICP's point-to-plane
// residual; the gradients are taken with the assignment held fixed)
// ---------------------------------------------------------------------------

// Ericson, Real-Time Collision Detection, sec. 5.1.5, in f64.
void closest_on_triangle(const double *p, const double *a, const double *b, const double *c,
                         double *q) {
  auto dot3 = [](const double *u, const double *v) { return (u[0] * v[0] + u[1] * v[1]) + u[2] * v[2]; };
  auto put = [&](const double *o, const double *e1, double s1, const double *e2, double s2) {
    for (int k = 0; k < 3; ++k) q[k] = (o[k] + e1[k] * s1) + e2[k] * s2;
  };
  const double z[3] = {0.0, 0.0, 0.0};
  double ab[3], ac[3], ap[3], bp[3], cp[3];
  for (int k = 0; k < 3; ++k) {
    ab[k] = b[k] - a[k];
    ac[k] = c[k] - a[k];
    ap[k] = p[k] - a[k];
    bp[k] = p[k] - b[k];
    cp[k] = p[k] - c[k];
  }
  double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
  if (d1 <= 0.0 && d2 <= 0.0) return put(a, z, 0.0, z, 0.0);
  double d3 = dot3(ab, bp), d4 = dot3(ac, bp);
  if (d3 >= 0.0 && d4 <= d3) return put(b, z, 0.0, z, 0.0);
  double vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3 <= 0.0) return put(a, ab, d1 / (d1 - d3), z, 0.0);
  double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
  if (d6 >= 0.0 && d5 <= d6) return put(c, z, 0.0, z, 0.0);
  double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return put(a, ac, d2 / (d2 - d6), z, 0.0);
  double va = d3 * d6 - d5 * d4;
  double e43 = d4 - d3, e56 = d5 - d6;
  if (va <= 0.0 && e43 >= 0.0 && e56 >= 0.0) {
    double bc[3] = {c[0] - b[0], c[1] - b[1], c[2] - b[2]};
    return put(b, bc, e43 / (e43 + e56), z, 0.0);
  }
  double den = (va + vb) + vc;
  put(a, ab, vb / den, ac, vc / den);
}

void add_twist(double *acc, const double *p, const double *g) {
  acc[0] += p[1] * g[2] - p[2] * g[1];
  acc[1] += p[2] * g[0] - p[0] * g[2];
  acc[2] += p[0] * g[1] - p[1] * g[0];
  acc[3] += g[0];
  acc[4] += g[1];
  acc[5] += g[2];
}

struct AdjointSide {
  const std::vector<double> *pts;  // the moving fragment's fracture samples (its own frame)
  const Mesh *scene;               // the fixed fragment's fracture faces
};

// The two smoothed counts of one side and their twist gradients; `assign`
// (per point, a face id or -1) is filled, or read when `frozen`.
void adjoint_side(const AdjointSide &side, const double *m, const sherd_scales &sc, double w,
                  double window_k, bool frozen, int32_t *assign, double *val2, double *grad12) {
  float window = float(sc.facing + window_k * w);
  size_t n = side.pts->size() / 3;
  for (size_t i = 0; i < n; ++i) {
    double p[3];
    apply(m, &(*side.pts)[3 * i], p);
    uint32_t face;
    if (frozen) {
      if (assign[i] < 0) continue;
      face = uint32_t(assign[i]);
    } else {
      side.scene->nearest_face(narrow(p), window, &face);
      assign[i] = face == 0xFFFFFFFFu ? -1 : int32_t(face);
      if (face == 0xFFFFFFFFu) continue;
    }
    double v[3][3];
    for (int k = 0; k < 3; ++k) {
      V3f x = side.scene->vert(face, k);
      v[k][0] = x.x;
      v[k][1] = x.y;
      v[k][2] = x.z;
    }
    double q[3];
    closest_on_triangle(p, v[0], v[1], v[2], q);
    double dv[3] = {p[0] - q[0], p[1] - q[1], p[2] - q[2]};
    // The softened distance sqrt(|p - c|^2 + (w/10)^2): smooth where a sample crosses.
    double d = std::sqrt(((dv[0] * dv[0] + dv[1] * dv[1]) + dv[2] * dv[2]) + 0.01 * w * w);
    double st = 1.0 / (1.0 + std::exp(-((sc.tight - d) / w)));
    double sf = 1.0 / (1.0 + std::exp(-((sc.facing - d) / w)));
    val2[0] += st;
    val2[1] += sf;
    double kt = -st * (1.0 - st) / (w * d), kf = -sf * (1.0 - sf) / (w * d);
    double gt[3] = {kt * dv[0], kt * dv[1], kt * dv[2]};
    double gf[3] = {kf * dv[0], kf * dv[1], kf * dv[2]};
    add_twist(grad12, p, gt);
    add_twist(grad12 + 6, p, gf);
  }
}

// ---------------------------------------------------------------------------
// The stage-2 ladder of one candidate (ladder.rs:105-161, pair.rs:298-372)
// ---------------------------------------------------------------------------

struct Pair {
  const Surfaces *a, *b;
  const Cloud *reg_target, *frac_target;
  std::vector<double> reg_source, frac_source;
  sherd_scales sc;
};

sherd_candidate ladder_verify(const Pair &pr, const sherd_work_item &item,
                              const sherd_params &p, uint32_t pair_index) {
  sherd_candidate c{};
  c.pair = pair_index;
  c.start = item.start;
  static const double K[4] = {0.2, 0.08, 0.08, 0.04};
  double pose[16];
  std::memcpy(pose, item.init, sizeof pose);
  for (int r = 0; r < 4; ++r) {
    if (r == 2 && p.early_reject_tight > 0.0) {
      // R 5.6's early rejection (pair.rs:315-340): the fracture scores at the
      // pc_reg pose, and below the limit the partial scores of verify.rs:584-
      // 617 with the pc_frac rungs not run.
      sherd_scores s = verify(*pr.a, *pr.b, pose, pr.sc, false);
      if (s.tight < p.early_reject_tight) {
        for (int q = 2; q < 4; ++q) {
          c.rungs[q] = sherd_registration{};
          std::memcpy(c.rungs[q].transform, pose, sizeof pose);
        }
        c.scores = s;
        c.accepted = 0;
        return c;
      }
    }
    sherd_icp_options o{SHERD_POINT_TO_PLANE, 30, K[r] * pr.sc.t * pr.sc.icp};
    const std::vector<double> &src = r < 2 ? pr.reg_source : pr.frac_source;
    const Cloud &tgt = r < 2 ? *pr.reg_target : *pr.frac_target;
    c.rungs[r] = icp_register(src.data(), uint32_t(src.size() / 3), tgt, pose, o);
    std::memcpy(pose, c.rungs[r].transform, sizeof pose);
  }
  c.scores = verify(*pr.a, *pr.b, pose, pr.sc, true);
  c.accepted = accept(c.scores, p, pr.sc);
  return c;
}

// ---------------------------------------------------------------------------
// Thickness (fragment/thickness.rs:99-390)
// ---------------------------------------------------------------------------

// thickness::percentile90 (thickness.rs:272-290).
float percentile90(std::vector<float> v) {
  std::sort(v.begin(), v.end());
  size_t n = v.size();
  if (n == 1) return v[0];
  double vi = double(n - 1) * (90.0 / 100.0);
  double prev = std::floor(vi);
  size_t i = size_t(prev);
  double gamma = vi - prev;
  float a = v[i], b = v[std::min(i + 1, n - 1)];
  float diff = b - a;
  if (gamma >= 0.5) return b - diff * float(1.0 - gamma);
  return a + diff * float(gamma);
}

// thickness::hist_mode and bin_edges (thickness.rs:212-262).
float hist_mode(const std::vector<float> &x) {
  const int BINS = 60;
  float p90 = percentile90(x);
  float first = 0.0f, last = p90;
  if (p90 == 0.0f) {
    first = -0.5f;
    last = 0.5f;
  }
  float step = (last - first) / float(BINS);
  float edges[BINS + 1];
  for (int k = 0; k <= BINS; ++k) edges[k] = float(k) * step + first;
  edges[BINS] = last;
  float denom = last - first;
  uint64_t counts[BINS] = {};
  for (float v : x) {
    if (!(v >= first && v <= last)) continue;
    size_t i = size_t(((v - first) / denom) * float(BINS));
    if (i == size_t(BINS)) i -= 1;
    if (v < edges[i]) i -= 1;
    if (i != size_t(BINS - 1) && v >= edges[i + 1]) i += 1;
    counts[i] += 1;
  }
  int k = 0;
  for (int i = 1; i < BINS; ++i)
    if (counts[i] > counts[k]) k = i;
  return 0.5f * (edges[k] + edges[k + 1]);
}

// thickness::thickness_from_hits (thickness.rs:139-162) with looking_back
// (thickness.rs:185-204).
bool thickness_from_hits(const double *normals, uint32_t nf, const uint32_t *idx,
                         const float *t_hit, const uint32_t *prim, uint32_t n, float *t,
                         float *mode) {
  std::vector<float> ok_d, far;
  for (uint32_t k = 0; k < n; ++k) {
    float d = t_hit[k];
    uint32_t p = prim[k];
    if (!(std::isfinite(d) && p < nf)) continue;
    ok_d.push_back(d);
    const double *hit = normals + 3 * size_t(p), *from = normals + 3 * size_t(idx[k]);
    double dd = -((hit[0] * from[0] + hit[1] * from[1]) + hit[2] * from[2]);
    if (dd > 0.7) far.push_back(d);
  }
  if (ok_d.size() < 100) return false;
  float raw = hist_mode(ok_d);
  *mode = raw;
  *t = far.size() >= 100 ? hist_mode(far) : raw;
  return true;
}

// mesh::geometry::face_geometry (mesh/geometry.rs:70-96).
void face_geometry(const double *v, const uint32_t *f, uint32_t nf, double *normals,
                   double *areas, double *centroids) {
  for (uint32_t i = 0; i < nf; ++i) {
    const double *a = v + 3 * size_t(f[3 * i]), *b = v + 3 * size_t(f[3 * i + 1]),
                 *c = v + 3 * size_t(f[3 * i + 2]);
    double e1[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    double e2[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
    double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                   e1[0] * e2[1] - e1[1] * e2[0]};
    double len = std::sqrt((n[0] * n[0] + n[1] * n[1]) + n[2] * n[2]);
    double den = std::max(len, 1e-12);
    if (normals)
      for (int k = 0; k < 3; ++k) normals[3 * i + k] = n[k] / den;
    if (areas) areas[i] = 0.5 * len;
    if (centroids)
      for (int k = 0; k < 3; ++k) centroids[3 * i + k] = (a[k] + b[k] + c[k]) / 3.0;
  }
}

// segment::cone_basis (segment.rs:383-395).
bool cone_basis(const double *n, double e1[3], double e2[3]) {
  for (int k = 0; k < 3; ++k)
    if (!std::isfinite(n[k])) return false;
  double a[3] = {1, 0, 0};
  if (!(std::fabs(n[0]) < 0.9)) {
    a[0] = 0;
    a[1] = 1;
  }
  double c[3] = {n[1] * a[2] - n[2] * a[1], n[2] * a[0] - n[0] * a[2], n[0] * a[1] - n[1] * a[0]};
  double len = std::sqrt((c[0] * c[0] + c[1] * c[1]) + c[2] * c[2]);
  if (len <= 0.0) return false;
  for (int k = 0; k < 3; ++k) e1[k] = c[k] / len;
  e2[0] = n[1] * e1[2] - n[2] * e1[1];
  e2[1] = n[2] * e1[0] - n[0] * e1[2];
  e2[2] = n[0] * e1[1] - n[1] * e1[0];
  return true;
}

// segment::classify_faces (segment.rs:318-376).
uint8_t cone_vote(const Mesh &m, const double *c, const double *fnv, const double *n,
                  const double *hit_normals, uint32_t nf, double thick) {
  double e1[3], e2[3];
  if (!cone_basis(n, e1, e2)) return 0;
  const double PI = 3.14159265358979323846;
  double angle = 15.0 * (PI / 180.0);
  double cos_a = std::cos(angle), sin_a = std::sin(angle);
  float min_hit = float(0.1 * thick);
  float thick_f = float(thick);
  V3f origin = {float(c[0] - fnv[0] * 1e-3), float(c[1] - fnv[1] * 1e-3),
                float(c[2] - fnv[2] * 1e-3)};
  uint8_t good = 0;
  for (int k = 0; k < 7; ++k) {
    double d[3];
    if (k == 0) {
      d[0] = -n[0];
      d[1] = -n[1];
      d[2] = -n[2];
    } else {
      double phi = 2.0 * PI * double(k - 1) / 6.0;
      double cp = std::cos(phi), sp = std::sin(phi);
      for (int q = 0; q < 3; ++q) d[q] = -(cos_a * n[q]) + sin_a * (cp * e1[q] + sp * e2[q]);
    }
    V3f dir = {float(d[0]), float(d[1]), float(d[2])};
    float dh;
    uint32_t prim;
    m.first_hit(origin, dir, &dh, &prim);
    if (prim == MISS) continue;
    if (!std::isfinite(dh) || prim >= nf || dh <= min_hit) continue;
    float ratio = dh / thick_f;
    if (ratio <= 0.5f || ratio >= 1.8f) continue;
    const double *h = hit_normals + 3 * size_t(prim);
    double al = (h[0] * d[0] + h[1] * d[1]) + h[2] * d[2];
    if (al > 0.7) ++good;
  }
  return good;
}


}  // namespace

// ===========================================================================
// C ABI (loaded by the tests through ctypes)
// ===========================================================================
// ---------------------------------------------------------------------------
// Segmentation, R 3.4 (fragment/segment.rs:189-631, mesh/adjacency.rs:43-175,
// mesh/components.rs:120-191)
// ---------------------------------------------------------------------------

// Points bucketed in cubes of side `cell`: every point within r <= cell of a
// query lies in the 27 cubes around the query's own.
struct BallGrid {
  const double *p = nullptr;
  size_t n = 0;
  double cell = 1.0, lo[3] = {0, 0, 0};
  std::map<std::array<int64_t, 3>, std::vector<uint32_t>> cells;

  BallGrid(const double *pts, size_t count, double side) : p(pts), n(count), cell(side) {
    for (int k = 0; k < 3; ++k) lo[k] = D_INF;
    for (size_t i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) lo[k] = std::min(lo[k], p[3 * i + k]);
    for (size_t i = 0; i < n; ++i) cells[key(p + 3 * i)].push_back(uint32_t(i));
  }
  std::array<int64_t, 3> key(const double *q) const {
    return {int64_t(std::floor((q[0] - lo[0]) / cell)), int64_t(std::floor((q[1] - lo[1]) / cell)),
            int64_t(std::floor((q[2] - lo[2]) / cell))};
  }
  // PointTree::within (kdtree.rs:219-245): every point with d2 <= r2, d2 =
  // ((dx dx + dy dy) + dz dz), ascending by index.
  void within(const double *q, double r, std::vector<uint32_t> &out) const {
    out.clear();
    if (r < 0.0 || n == 0) return;
    double r2 = r * r;
    std::array<int64_t, 3> c = key(q);
    for (int64_t dx = -1; dx <= 1; ++dx)
      for (int64_t dy = -1; dy <= 1; ++dy)
        for (int64_t dz = -1; dz <= 1; ++dz) {
          auto it = cells.find({c[0] + dx, c[1] + dy, c[2] + dz});
          if (it == cells.end()) continue;
          for (uint32_t j : it->second) {
            const double *x = p + 3 * size_t(j);
            double ex = q[0] - x[0], ey = q[1] - x[1], ez = q[2] - x[2];
            if ((ex * ex + ey * ey) + ez * ez <= r2) out.push_back(j);
          }
        }
    std::sort(out.begin(), out.end());
  }
};

// voxel_representatives (segment.rs:217-259): the lowest index of every
// occupied voxel floor((c - (min - 1)) / spacing), ascending.
std::vector<uint32_t> voxel_representatives(const double *c, size_t n, double spacing) {
  std::vector<uint32_t> rep;
  if (n == 0 || !std::isfinite(spacing) || spacing <= 0.0) return rep;
  double mb[3] = {D_INF, D_INF, D_INF};
  for (size_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) mb[k] = std::min(mb[k], c[3 * i + k]);
  for (double &m : mb) m -= 1.0;
  std::vector<std::pair<std::array<int64_t, 3>, uint32_t>> cells(n);
  for (size_t i = 0; i < n; ++i) {
    for (int k = 0; k < 3; ++k)
      cells[i].first[k] = int64_t(std::floor((c[3 * i + k] - mb[k]) / spacing));
    cells[i].second = uint32_t(i);
  }
  std::sort(cells.begin(), cells.end());
  for (size_t i = 0; i < n; ++i)
    if (i == 0 || cells[i - 1].first != cells[i].first) rep.push_back(cells[i].second);
  std::sort(rep.begin(), rep.end());
  return rep;
}

// ball_normals (segment.rs:267-296) over the points `idx` of a BallGrid:
// m = sum A FN / max(sum A, 1e-12), then m / max(|m|, 1e-12), summed in
// ascending index order; `has` is false for an empty ball.
void ball_normals(const BallGrid &grid, const std::vector<std::array<double, 3>> &queries,
                  const double *normals, const double *areas, double radius,
                  std::vector<std::array<double, 3>> &out, std::vector<uint8_t> &has) {
  out.assign(queries.size(), {0.0, 0.0, 0.0});
  has.assign(queries.size(), 0);
  parallel_for(uint32_t(queries.size()), default_threads(), [&](uint32_t r) {
    std::vector<uint32_t> ball;
    grid.within(queries[r].data(), radius, ball);
    double m[3] = {0.0, 0.0, 0.0}, wsum = 0.0;
    for (uint32_t j : ball) {
      const double *n = normals + 3 * size_t(j);
      double a = areas[j];
      for (int k = 0; k < 3; ++k) m[k] += n[k] * a;
      wsum += a;
    }
    double den = std::max(wsum, 1e-12);
    for (double &x : m) x /= den;
    double norm = std::max(std::sqrt((m[0] * m[0] + m[1] * m[1]) + m[2] * m[2]), 1e-12);
    out[r] = {m[0] / norm, m[1] / norm, m[2] / norm};
    has[r] = !ball.empty();
  });
}

// face_adjacency (adjacency.rs:138-160): edge keys in slot-major order,
// sorted stably, every two consecutive equal keys one face pair.
void face_adjacency(const uint32_t *f, uint32_t nf, std::vector<uint32_t> &fa,
                    std::vector<uint32_t> &fb) {
  size_t m = size_t(3) * nf;
  std::vector<uint64_t> keys(m);
  const int slot[3][2] = {{0, 1}, {1, 2}, {2, 0}};
  for (int s = 0; s < 3; ++s)
    for (uint32_t t = 0; t < nf; ++t) {
      uint32_t a = f[3 * t + slot[s][0]], b = f[3 * t + slot[s][1]];
      uint32_t lo = std::min(a, b), hi = std::max(a, b);
      keys[size_t(s) * nf + t] = (uint64_t(lo) << 32) | hi;
    }
  std::vector<uint32_t> order(m);
  for (size_t i = 0; i < m; ++i) order[i] = uint32_t(i);
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t x, uint32_t y) { return keys[x] < keys[y]; });
  fa.clear();
  fb.clear();
  for (size_t w = 0; w + 1 < m; ++w) {
    uint32_t i = order[w], j = order[w + 1];
    if (keys[i] == keys[j]) {
      fa.push_back(i % nf);
      fb.push_back(j % nf);
    }
  }
}

// drop_small_components (components.rs:170-191) over mask_components
// (components.rs:120-159): components of mask == target over the pairs whose
// both faces are in the set, areas summed in face order, those below
// min_area flipped.
void drop_small_components(std::vector<uint8_t> &mask, bool target, double min_area,
                           const std::vector<uint32_t> &fa, const std::vector<uint32_t> &fb,
                           const double *areas) {
  size_t n = mask.size();
  std::vector<uint32_t> parent(n);
  for (size_t i = 0; i < n; ++i) parent[i] = uint32_t(i);
  auto find = [&](uint32_t x) {
    while (parent[x] != x) {
      parent[x] = parent[parent[x]];
      x = parent[x];
    }
    return x;
  };
  for (size_t i = 0; i < fa.size(); ++i) {
    uint32_t a = fa[i], b = fb[i];
    if (bool(mask[a]) == target && bool(mask[b]) == target) {
      uint32_t ra = find(a), rb = find(b);
      if (ra != rb) parent[std::max(ra, rb)] = std::min(ra, rb);
    }
  }
  std::vector<double> size(n, 0.0);
  for (size_t i = 0; i < n; ++i)
    if (bool(mask[i]) == target) size[find(uint32_t(i))] += areas[i];
  for (size_t i = 0; i < n; ++i)
    if (bool(mask[i]) == target && size[find(uint32_t(i))] < min_area) mask[i] = !target;
}

// refine_boundary (segment.rs:438-474): at most 60 passes; each flips, all
// at once, the fracture faces touching the shell whose normal is within the
// angle of their fixed shell reference normal.
void refine_boundary(std::vector<uint8_t> &frac, const std::vector<uint32_t> &fa,
                     const std::vector<uint32_t> &fb, const double *normals,
                     const std::vector<std::array<double, 3>> &ref,
                     const std::vector<uint8_t> &has_ref, double angle_deg) {
  double cos_grow = std::cos(angle_deg * (3.14159265358979323846 / 180.0));
  std::vector<uint8_t> cand(frac.size(), 0);
  for (int pass = 0; pass < 60; ++pass) {
    std::vector<uint32_t> list;
    for (size_t i = 0; i < fa.size(); ++i) {
      uint32_t a = fa[i], b = fb[i];
      if (frac[a] != frac[b]) {
        uint32_t face = frac[a] ? a : b;
        if (!cand[face]) {
          cand[face] = 1;
          list.push_back(face);
        }
      }
    }
    if (list.empty()) break;
    bool flipped = false;
    for (uint32_t face : list) {
      cand[face] = 0;
      const double *n = normals + 3 * size_t(face);
      const double *r = ref[face].data();
      if (has_ref[face] && (n[0] * r[0] + n[1] * r[1]) + n[2] * r[2] > cos_grow) {
        frac[face] = 0;
        flipped = true;
      }
    }
    if (!flipped) break;
  }
}

// segment::run (segment.rs:511-631).
void segment(const Mesh &scene, const double *v, const uint32_t *f, uint32_t nf, double thick,
             double res, const sherd_seg_params &sp, const uint8_t *good_in, uint8_t *labels,
             sherd_seg_info *info, const sherd_seg_trace *trace) {
  info->votes = res > sp.coarse_at * thick ? sp.votes_coarse : sp.votes;
  info->smooth_radius = std::max(thick / 3.0, sp.smooth_res * res);
  info->boundary_angle = sp.boundary_angle;
  info->n_rep = 0;
  if (nf == 0 || !std::isfinite(thick) || thick <= 0.0) {
    std::fill(labels, labels + nf, 0);
    return;
  }
  std::vector<double> normals(size_t(3) * nf), areas(nf), cent(size_t(3) * nf);
  face_geometry(v, f, nf, normals.data(), areas.data(), cent.data());
  // 3.4.1 the grid
  std::vector<uint32_t> rep = voxel_representatives(cent.data(), nf, thick * (1.0 / 8.0));
  info->n_rep = uint32_t(rep.size());
  std::vector<double> rep_xyz(3 * rep.size());
  std::vector<std::array<double, 3>> rep_pts(rep.size());
  for (size_t r = 0; r < rep.size(); ++r)
    for (int k = 0; k < 3; ++k) rep_pts[r][k] = rep_xyz[3 * r + k] = cent[3 * size_t(rep[r]) + k];
  Cloud rep_cloud;
  rep_cloud.p = rep_xyz;
  rep_cloud.build();
  std::vector<uint32_t> near(nf);
  parallel_for(nf, default_threads(), [&](uint32_t i) {
    uint32_t j;
    double d2;
    rep_cloud.nearest_within_sq(&cent[3 * size_t(i)], D_INF, &j, &d2);
    near[i] = j;
  });
  BallGrid all(cent.data(), nf, std::max(info->smooth_radius, thick * 0.5));
  // 3.4.2 the smoothed normals
  std::vector<std::array<double, 3>> ns_g, ref_g;
  std::vector<uint8_t> has_g;
  ball_normals(all, rep_pts, normals.data(), areas.data(), info->smooth_radius, ns_g, has_g);
  std::vector<double> ns(size_t(3) * nf);
  for (uint32_t i = 0; i < nf; ++i)
    for (int k = 0; k < 3; ++k) ns[3 * size_t(i) + k] = ns_g[near[i]][k];
  // 3.4.3 the cone vote
  std::vector<uint8_t> good(nf);
  if (good_in) {
    std::copy(good_in, good_in + nf, good.begin());
  } else {
    const double *hit = sp.smoothed_hit_normal ? ns.data() : normals.data();
    parallel_for(nf, default_threads(), [&](uint32_t i) {
      good[i] = cone_vote(scene, &cent[3 * size_t(i)], &normals[3 * size_t(i)], &ns[3 * size_t(i)],
                          hit, nf, thick);
    });
  }
  std::vector<uint8_t> frac(nf);
  for (uint32_t i = 0; i < nf; ++i) frac[i] = uint32_t(good[i]) < info->votes;
  if (trace) {
    if (trace->rep) std::copy(rep.begin(), rep.end(), trace->rep);
    if (trace->near) std::copy(near.begin(), near.end(), trace->near);
    if (trace->ns) std::copy(ns.begin(), ns.end(), trace->ns);
    if (trace->good) std::copy(good.begin(), good.end(), trace->good);
    if (trace->frac_raw) std::copy(frac.begin(), frac.end(), trace->frac_raw);
  }
  // 3.4.4 the majority filter
  std::vector<uint8_t> per_rep(rep.size());
  parallel_for(uint32_t(rep.size()), default_threads(), [&](uint32_t r) {
    std::vector<uint32_t> ball;
    all.within(rep_pts[r].data(), thick * 0.25, ball);
    double wet = 0.0, total = 0.0;
    for (uint32_t j : ball) {
      total += areas[j];
      if (frac[j]) wet += areas[j];
    }
    per_rep[r] = wet > 0.5 * total;
  });
  for (uint32_t i = 0; i < nf; ++i) frac[i] = per_rep[near[i]];
  if (trace && trace->frac_majority) std::copy(frac.begin(), frac.end(), trace->frac_majority);
  // 3.4.5-3.4.6 islands
  std::vector<uint32_t> fa, fb;
  face_adjacency(f, nf, fa, fb);
  drop_small_components(frac, true, 0.5 * thick * thick, fa, fb, areas.data());
  drop_small_components(frac, false, 2.0 * thick * thick, fa, fb, areas.data());
  if (trace && trace->frac_islands) std::copy(frac.begin(), frac.end(), trace->frac_islands);
  // 3.4.7 the boundary growth
  std::vector<uint32_t> shell;
  for (uint32_t i = 0; i < nf; ++i)
    if (!frac[i]) shell.push_back(i);
  double angle = sp.boundary_angle;
  if (sp.boundary_angle_auto && !shell.empty()) {
    std::vector<double> noise;
    for (uint32_t i : shell) {
      const double *a = &normals[3 * size_t(i)], *b = &ns[3 * size_t(i)];
      double c = std::min(1.0, std::max(-1.0, (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2]));
      noise.push_back(std::acos(c) * (180.0 / 3.14159265358979323846));
    }
    angle = std::max(angle, median(noise) + 15.0);
  }
  info->boundary_angle = angle;
  std::vector<std::array<double, 3>> reference(nf, {0.0, 0.0, 0.0});
  std::vector<uint8_t> has_ref(nf, 0);
  if (!shell.empty()) {
    std::vector<double> sp_xyz(3 * shell.size()), sn(3 * shell.size()), sa(shell.size());
    for (size_t k = 0; k < shell.size(); ++k) {
      for (int q = 0; q < 3; ++q) {
        sp_xyz[3 * k + q] = cent[3 * size_t(shell[k]) + q];
        sn[3 * k + q] = normals[3 * size_t(shell[k]) + q];
      }
      sa[k] = areas[shell[k]];
    }
    BallGrid shell_grid(sp_xyz.data(), shell.size(), thick * 0.5);
    ball_normals(shell_grid, rep_pts, sn.data(), sa.data(), thick * 0.5, ref_g, has_g);
    for (uint32_t i = 0; i < nf; ++i) {
      reference[i] = ref_g[near[i]];
      has_ref[i] = has_g[near[i]];
    }
  }
  if (trace && trace->has_ref) std::copy(has_ref.begin(), has_ref.end(), trace->has_ref);
  refine_boundary(frac, fa, fb, normals.data(), reference, has_ref, angle);
  // 3.4.8 one more island pass
  drop_small_components(frac, true, 0.5 * thick * thick, fa, fb, areas.data());
  std::copy(frac.begin(), frac.end(), labels);
}

extern "C" {

void *or_mesh_new(const float *v, uint32_t nv, const uint32_t *f, uint32_t nf) {
  if (nf == 0) return nullptr;
  Mesh *m = new Mesh;
  m->v.resize(nv);
  for (uint32_t i = 0; i < nv; ++i) m->v[i] = {v[3 * i], v[3 * i + 1], v[3 * i + 2]};
  m->f.assign(f, f + 3 * size_t(nf));
  m->build();
  return m;
}

// RayScene::of_subset (bvh.rs:71-78): the kept faces, or face 0.
void *or_mesh_subset(const void *mesh, const uint8_t *keep) {
  const Mesh *m = static_cast<const Mesh *>(mesh);
  Mesh *s = new Mesh;
  s->v = m->v;
  uint32_t nf = m->n_faces();
  for (uint32_t i = 0; i < nf; ++i)
    if (keep[i])
      for (int k = 0; k < 3; ++k) s->f.push_back(m->f[3 * i + k]);
  if (s->f.empty())
    for (int k = 0; k < 3; ++k) s->f.push_back(m->f[k]);
  s->build();
  return s;
}

void or_mesh_free(void *m) { delete static_cast<Mesh *>(m); }

void or_mesh_aabb(const void *mesh, float *lo, float *hi) {
  const Mesh *m = static_cast<const Mesh *>(mesh);
  for (int k = 0; k < 3; ++k) {
    lo[k] = m->lo[k];
    hi[k] = m->hi[k];
  }
}

void or_first_hit(const void *mesh, const float *org, const float *dir, uint32_t n, float *t,
                  uint32_t *prim, int threads) {
  const Mesh *m = static_cast<const Mesh *>(mesh);
  parallel_for(n, threads, [&](uint32_t i) {
    m->first_hit({org[3 * i], org[3 * i + 1], org[3 * i + 2]},
                 {dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]}, &t[i], &prim[i]);
  });
}

void or_bounded_distance(const void *mesh, const double *pts, uint32_t n, const double *pose,
                         double max_dist, int reduce, double *out) {
  bounded_distance(*static_cast<const Mesh *>(mesh), pts, n, pose, max_dist, reduce, out);
}

void or_inside(const void *mesh, const double *pts, uint32_t n, const double *pose,
               sherd_inside_outcome *out, int threads) {
  const Mesh *m = static_cast<const Mesh *>(mesh);
  parallel_for(n, threads, [&](uint32_t i) { inside_batch(*m, pts + 3 * size_t(i), 1, pose, out + i); });
}

uint32_t or_crossings(const void *mesh, const float *org, const float *dir) {
  return static_cast<const Mesh *>(mesh)->crossings({org[0], org[1], org[2]},
                                                     {dir[0], dir[1], dir[2]});
}

void *or_cloud_new(const double *p, const double *nrm, uint32_t np) {
  if (np == 0) return nullptr;
  Cloud *c = new Cloud;
  c->p.assign(p, p + 3 * size_t(np));
  if (nrm) c->n.assign(nrm, nrm + 3 * size_t(np));
  c->build();
  return c;
}

void or_cloud_free(void *c) { delete static_cast<Cloud *>(c); }

void or_nearest_within_sq(const void *cloud, const double *q, uint32_t n, double r2,
                          uint32_t *idx, double *d2, int threads) {
  const Cloud *c = static_cast<const Cloud *>(cloud);
  parallel_for(n, threads, [&](uint32_t i) {
    if (!c->nearest_within_sq(q + 3 * size_t(i), r2, &idx[i], &d2[i])) {
      idx[i] = MISS;
      d2[i] = D_INF;
    }
  });
}

void or_nearest_below(const void *cloud, const double *q, uint32_t n, double bound,
                      uint32_t *idx, double *dist, int threads) {
  const Cloud *c = static_cast<const Cloud *>(cloud);
  parallel_for(n, threads, [&](uint32_t i) {
    if (!c->nearest_below(q + 3 * size_t(i), bound, &idx[i], &dist[i])) {
      idx[i] = MISS;
      dist[i] = D_INF;
    }
  });
}

void or_icp_rung(const double *src, uint32_t ns, const void *target, const double *inits,
                 uint32_t k, sherd_icp_options opt, sherd_registration *out, int threads) {
  const Cloud *c = static_cast<const Cloud *>(target);
  if (k < uint32_t(std::max(threads, 1))) {  // few poses: the threads share each pass instead
    for (uint32_t i = 0; i < k; ++i) out[i] = icp_register(src, ns, *c, inits + 16 * size_t(i), opt, threads);
    return;
  }
  parallel_for(k, threads, [&](uint32_t i) {
    out[i] = icp_register(src, ns, *c, inits + 16 * size_t(i), opt);
  });
}

void *or_surfaces_new(const void *fracture, const void *mesh, uint32_t watertight,
                      double frac_area, const double *pf, uint32_t n_pf, const double *s,
                      uint32_t n_s, const double *brk_p, const double *brk_ns, uint32_t n_brk,
                      const double *margin_p, const double *margin_n, uint32_t n_margin) {
  Surfaces *x = new Surfaces;
  x->fracture = static_cast<const Mesh *>(fracture);
  x->mesh = static_cast<const Mesh *>(mesh);
  x->watertight = watertight != 0;
  x->frac_area = frac_area;
  x->pf.assign(pf, pf + 3 * size_t(n_pf));
  x->s.assign(s, s + 3 * size_t(n_s));
  x->brk_p.assign(brk_p, brk_p + 3 * size_t(n_brk));
  x->brk_ns.assign(brk_ns, brk_ns + 3 * size_t(n_brk));
  x->margin_p.assign(margin_p, margin_p + 3 * size_t(n_margin));
  x->margin_n.assign(margin_n, margin_n + 3 * size_t(n_margin));
  x->margin_tree.p = x->margin_p;
  x->margin_tree.build();
  return x;
}

void or_surfaces_free(void *s) { delete static_cast<Surfaces *>(s); }

void or_verify(const void *a, const void *b, const double *pose, const sherd_scales *sc,
               int full, sherd_scores *out) {
  *out = verify(*static_cast<const Surfaces *>(a), *static_cast<const Surfaces *>(b), pose, *sc,
                full != 0);
}

uint32_t or_accept(const sherd_scores *s, const sherd_params *p, const sherd_scales *sc) {
  return accept(*s, *p, *sc);
}

void *or_pair_new(const void *a, const void *b, const void *reg_target, const void *frac_target,
                  const double *reg_source, uint32_t n_reg, const double *frac_source,
                  uint32_t n_frac, const sherd_scales *sc) {
  Pair *p = new Pair;
  p->a = static_cast<const Surfaces *>(a);
  p->b = static_cast<const Surfaces *>(b);
  p->reg_target = static_cast<const Cloud *>(reg_target);
  p->frac_target = static_cast<const Cloud *>(frac_target);
  p->reg_source.assign(reg_source, reg_source + 3 * size_t(n_reg));
  p->frac_source.assign(frac_source, frac_source + 3 * size_t(n_frac));
  p->sc = *sc;
  return p;
}

void or_pair_free(void *p) { delete static_cast<Pair *>(p); }

// The CPU baseline of the batched path: every item on `threads` host threads
// (0 = all cores). Returns the thread count used.
int or_ladder_verify_batch(void *const *pairs, uint32_t n_pairs, const sherd_work_item *items,
                           uint32_t n_items, const sherd_params *p, int threads,
                           sherd_candidate *out) {
  if (threads <= 0) threads = default_threads();
  parallel_for(n_items, threads, [&](uint32_t i) {
    uint32_t pi = items[i].pair;
    if (pi >= n_pairs) {
      out[i] = sherd_candidate{};
      out[i].status = uint32_t(-SHERD_E_INVALID);
      return;
    }
    out[i] = ladder_verify(*static_cast<const Pair *>(pairs[pi]), items[i], *p, pi);
  });
  return threads;
}

void or_face_geometry(const double *v, const uint32_t *f, uint32_t nf, double *normals,
                      double *areas, double *centroids) {
  face_geometry(v, f, nf, normals, areas, centroids);
}

// thickness::face_indices (thickness.rs:387-390).
uint32_t or_face_indices(uint32_t n_faces, uint32_t n, uint32_t *out) {
  uint32_t nn = n ? n : 1;
  uint32_t stride = (n_faces + nn - 1) / nn;
  if (stride < 1) stride = 1;
  uint32_t k = 0;
  for (uint32_t i = 0; i < n_faces; i += stride) {
    if (out) out[k] = i;
    ++k;
  }
  return k;
}

// thickness::cast_inward_rays (thickness.rs:115-132).
void or_cast_inward_rays(const void *mesh, const double *centroids, const double *normals,
                         const uint32_t *idx, uint32_t n, float *t_hit, uint32_t *prim,
                         int threads) {
  const Mesh *m = static_cast<const Mesh *>(mesh);
  parallel_for(n, threads, [&](uint32_t k) {
    const double *c = centroids + 3 * size_t(idx[k]), *nn = normals + 3 * size_t(idx[k]);
    double d[3] = {-nn[0], -nn[1], -nn[2]};
    V3f o = {float(c[0] + d[0] * 1e-3), float(c[1] + d[1] * 1e-3), float(c[2] + d[2] * 1e-3)};
    V3f dir = {float(d[0]), float(d[1]), float(d[2])};
    m->first_hit(o, dir, &t_hit[k], &prim[k]);
  });
}

int or_thickness_from_hits(const double *normals, uint32_t nf, const uint32_t *idx,
                           const float *t_hit, const uint32_t *prim, uint32_t n, float *t,
                           float *mode) {
  return thickness_from_hits(normals, nf, idx, t_hit, prim, n, t, mode) ? 1 : 0;
}

float or_percentile90(const float *x, uint32_t n) {
  return percentile90(std::vector<float>(x, x + n));
}

float or_hist_mode(const float *x, uint32_t n) { return hist_mode(std::vector<float>(x, x + n)); }

void or_cone_votes(const void *mesh, const double *centroids, const double *normals,
                   const double *ns, const double *hit_normals, uint32_t nf, double thick,
                   uint8_t *good, int threads) {
  const Mesh *m = static_cast<const Mesh *>(mesh);
  parallel_for(nf, threads, [&](uint32_t i) {
    good[i] = cone_vote(*m, centroids + 3 * size_t(i), normals + 3 * size_t(i),
                        ns + 3 * size_t(i), hit_normals, nf, thick);
  });
}

void or_eigen_pivots(const double *a36, int *perm) {
  double a[6][6];
  std::memcpy(a, a36, sizeof a);
  eigen_pivots(a, perm);
}

int or_solve_ldlt(const double *a36, const double *b, double *x) {
  double a[6][6];
  std::memcpy(a, a36, sizeof a);
  return solve_ldlt(a, b, x) ? 1 : 0;
}

void or_pose_inverse(const double *t, double *out) { pose_inverse(t, out); }

void or_euler_zyx(double a, double b, double g, double *r9) {
  double r[3][3];
  euler_zyx(a, b, g, r);
  std::memcpy(r9, r, sizeof r);
}

float or_tri_distance(const float *p, const float *a, const float *b, const float *c) {
  return tri_distance({p[0], p[1], p[2]}, {a[0], a[1], a[2]}, {b[0], b[1], b[2]},
                      {c[0], c[1], c[2]});
}

float or_moller_trumbore(const float *o, const float *d, const float *a, const float *b,
                         const float *c) {
  return moller_trumbore({o[0], o[1], o[2]}, {d[0], d[1], d[2]}, {a[0], a[1], a[2]},
                         {b[0], b[1], b[2]}, {c[0], c[1], c[2]});
}

int or_default_threads(void) { return default_threads(); }

// The adjoint of the group-alignment objectives for one pair at pose t (B's
// frame into A's) and t_inv: values[5] = E, T_B, F_B, T_A, F_A and grads[30],
// six twist components per value (the CUDA backend's sherd_adjoint). The
// assignment (per B fracture source point its target index, per B and A
// fracture sample its face id, -1 for none) is written, or read when frozen.
void or_adjoint(const void *pair, const double *t, const double *t_inv,
                const sherd_adjoint_options *o, int frozen, int32_t *assign, double *values,
                double *grads) {
  const Pair &pr = *static_cast<const Pair *>(pair);
  std::fill(values, values + 5, 0.0);
  std::fill(grads, grads + 30, 0.0);
  const sherd_scales &sc = pr.sc;
  size_t nf = pr.frac_source.size() / 3, nb = pr.b->pf.size() / 3;
  double r = o->radius_k * sc.t * sc.icp, r2 = r * r;
  const Cloud &tgt = *pr.frac_target;
  for (size_t i = 0; i < nf; ++i) {
    double p[3];
    apply(t, &pr.frac_source[3 * i], p);
    uint32_t j;
    if (frozen) {
      if (assign[i] < 0) continue;
      j = uint32_t(assign[i]);
    } else {
      double d2;
      if (!tgt.nearest_within_sq(p, r2, &j, &d2) || !(d2 < r2)) {
        assign[i] = -1;
        continue;
      }
      assign[i] = int32_t(j);
    }
    const double *q = &tgt.p[3 * j], *n = &tgt.n[3 * j];
    double res = ((p[0] - q[0]) * n[0] + (p[1] - q[1]) * n[1]) + (p[2] - q[2]) * n[2];
    values[0] += 0.5 * res * res;
    double g[3] = {res * n[0], res * n[1], res * n[2]};
    add_twist(grads, p, g);
  }
  double w = o->width_k * sc.t;
  adjoint_side({&pr.b->pf, pr.a->fracture}, t, sc, w, o->window_k,
               frozen != 0, assign + nf, values + 1, grads + 6);
  adjoint_side({&pr.a->pf, pr.b->fracture}, t_inv, sc, w, o->window_k, frozen != 0,
               assign + nf + nb, values + 3, grads + 18);
}

// icp::correspondences + icp::normal_equations at `pose` (icp.rs:361-392,
// 599-640): J^T J (36, symmetric) and J^T r of the point-to-plane system.
void or_normal_equations(const double *src, uint32_t ns, const void *target, const double *pose,
                         double distance, double *jtj36, double *jtr6) {
  const Cloud &tgt = *static_cast<const Cloud *>(target);
  std::vector<double> moved(src, src + size_t(3) * ns);
  transform_points(moved, pose);
  std::vector<Corr> corr;
  double fit, rmse;
  correspondences(moved, tgt, distance, corr, &fit, &rmse);
  double jtj[6][6], jtr[6];
  normal_equations(moved, tgt, corr, jtj, jtr);
  for (int k = 0; k < 6; ++k) {
    jtr6[k] = jtr[k];
    for (int l = 0; l <= k; ++l) jtj36[6 * k + l] = jtj36[6 * l + k] = jtj[k][l];
  }
}

// segment::segment_faces (segment.rs:476-631); `good_in` (nullable) replaces
// the cone vote, to run the later steps on given votes.
void or_segment(const void *mesh, const double *v, const uint32_t *f, uint32_t nf, double thick,
                double res, const sherd_seg_params *sp, const uint8_t *good_in, uint8_t *labels,
                sherd_seg_info *info, const sherd_seg_trace *trace) {
  segment(*static_cast<const Mesh *>(mesh), v, f, nf, thick, res, *sp, good_in, labels, info,
          trace);
}

// CpuExecutor::coarse_scores (executor/cpu.rs:46-68) with agreeing
// (cpu.rs:136-169), for k row-major 4x4 poses.
void or_coarse_scores(const void *target, const double *points, const double *normals, uint32_t n,
                      const double *poses, uint32_t k, double radius, double normal_agree,
                      double *out) {
  const Cloud &tgt = *static_cast<const Cloud *>(target);
  for (uint32_t h = 0; h < k; ++h) {
    const double *t = poses + 16 * size_t(h);
    if (n == 0) {
      out[h] = 0.0;
      continue;
    }
    uint32_t agree = 0;
    for (uint32_t i = 0; i < n; ++i) {
      double moved[3], turned[3];
      apply(t, points + 3 * size_t(i), moved);
      uint32_t j;
      double d;
      if (!tgt.nearest_below(moved, radius, &j, &d)) continue;
      rotate(t, normals + 3 * size_t(i), turned);
      const double *m = &tgt.n[3 * size_t(j)];
      if ((m[0] * turned[0] + m[1] * turned[1]) + m[2] * turned[2] > normal_agree) ++agree;
    }
    out[h] = double(agree) / double(n);
  }
}

// The rotation svd_rotation takes from a row-major 3x3 (for its own test).
void or_svd_rotation(const double *m9, double *r9) {
  double m[3][3], r[3][3];
  for (int i = 0; i < 9; ++i) m[i / 3][i % 3] = m9[i];
  svd_rotation(m, r);
  for (int i = 0; i < 9; ++i) r9[i] = r[i / 3][i % 3];
}

// verify::penetration_share (verify.rs:509-527).
double or_penetration_share(const void *mesh, const double *points, uint32_t n, const double *pose,
                            double pen) {
  if (n == 0) return 0.0;
  std::vector<sherd_inside_outcome> out(n);
  inside_batch(*static_cast<const Mesh *>(mesh), points, n, pose, out.data());
  size_t deeper = 0;
  for (const auto &o : out)
    if (o.inside && double(o.depth) > pen) ++deeper;
  return double(deeper) / double(n);
}

// refine::vertex_normals (refine.rs:121-151), Open3D's ComputeVertexNormals:
// each face's unnormalised normal (v1 - v0) x (v2 - v0) added to its three
// vertices in face order, then one normalisation; a zero (or NaN) sum becomes
// (0, 0, 1).
void or_vertex_normals(const double *v, uint32_t nv, const uint32_t *f, uint32_t nf,
                       double *out) {
  std::fill(out, out + 3 * size_t(nv), 0.0);
  for (uint32_t i = 0; i < nf; ++i) {
    const uint32_t *tri = f + 3 * size_t(i);
    const double *o = v + 3 * size_t(tri[0]), *b = v + 3 * size_t(tri[1]),
                 *c = v + 3 * size_t(tri[2]);
    double e1[3] = {b[0] - o[0], b[1] - o[1], b[2] - o[2]};
    double e2[3] = {c[0] - o[0], c[1] - o[1], c[2] - o[2]};
    double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                   e1[0] * e2[1] - e1[1] * e2[0]};
    for (int k = 0; k < 3; ++k) {
      double *s = out + 3 * size_t(tri[k]);
      for (int a = 0; a < 3; ++a) s[a] += n[a];
    }
  }
  for (uint32_t j = 0; j < nv; ++j) {
    double *n = out + 3 * size_t(j);
    double len = std::sqrt((n[0] * n[0] + n[1] * n[1]) + n[2] * n[2]);
    if (len > 0.0) {
      for (int a = 0; a < 3; ++a) n[a] /= len;
    } else {
      n[0] = 0.0;
      n[1] = 0.0;
      n[2] = 1.0;
    }
  }
}

// types::apply_transform_fused / rotate_fused (types.rs:202-214): row i of the
// row-major pose is fma(t_i2, p2, fma(t_i1, p1, t_i0 p0)), plus t_i3 for a
// point (rotate_only = 0); a normal takes the rotation block alone.
void or_place_fused(const double *pts, uint32_t n, const double *t, int rotate_only, double *out) {
  for (uint32_t i = 0; i < n; ++i) {
    const double *p = pts + 3 * size_t(i);
    for (int r = 0; r < 3; ++r) {
      double s = std::fma(t[4 * r + 2], p[2], std::fma(t[4 * r + 1], p[1], t[4 * r] * p[0]));
      out[3 * size_t(i) + r] = rotate_only ? s : s + t[4 * r + 3];
    }
  }
}

// ball_normals (segment.rs:267-296) of arbitrary query points over the n
// points `p` (with their unit normals and areas): the balls of radius r, each
// summed in ascending point order; has[q] = 0 for an empty ball.
void or_ball_normals(const double *p, uint32_t n, const double *normals, const double *areas,
                     const double *queries, uint32_t nq, double radius, double *out3,
                     uint8_t *has) {
  BallGrid grid(p, n, std::max(radius, 1e-300));
  std::vector<std::array<double, 3>> q(nq), out;
  for (uint32_t i = 0; i < nq; ++i)
    for (int k = 0; k < 3; ++k) q[i][k] = queries[3 * size_t(i) + k];
  std::vector<uint8_t> h;
  ball_normals(grid, q, normals, areas, radius, out, h);
  for (uint32_t i = 0; i < nq; ++i) {
    for (int k = 0; k < 3; ++k) out3[3 * size_t(i) + k] = out[i][k];
    has[i] = h[i];
  }
}

// voxel_representatives (segment.rs:217-259): writes the ascending
// representatives (room for n) and returns their count.
uint32_t or_voxel_representatives(const double *p, uint32_t n, double spacing, uint32_t *out) {
  std::vector<uint32_t> rep = voxel_representatives(p, n, spacing);
  std::copy(rep.begin(), rep.end(), out);
  return uint32_t(rep.size());
}

// nms::nms (nms.rs:61-99) over row-major 4x4 poses: walk `order`, stop at the
// first score below `floor`, keep a pose unless a kept one is nearer than
// trans_tol in translation ((dx dx + dy dy) + dz dz under the root) and
// trace(A^T B) > 2.9 (summed per column as (a0 b0 + a1 b1) + a2 b2), stop once
// topk are kept (tested after keeping). Returns the count written to kept.
uint32_t or_nms(const uint32_t *order, uint32_t n_order, const double *poses, const double *score,
                double trans_tol, uint32_t topk, double floor, uint32_t *kept) {
  uint32_t m = 0;
  for (uint32_t o = 0; o < n_order; ++o) {
    const uint32_t h = order[o];
    if (score[h] < floor) break;
    const double *t = poses + 16 * size_t(h);
    bool duplicate = false;
    for (uint32_t k = 0; k < m && !duplicate; ++k) {
      const double *u = poses + 16 * size_t(kept[k]);
      const double dx = t[3] - u[3], dy = t[7] - u[7], dz = t[11] - u[11];
      if (!(std::sqrt((dx * dx + dy * dy) + dz * dz) < trans_tol)) continue;
      double trace = 0.0;
      for (int c = 0; c < 3; ++c) trace += (t[c] * u[c] + t[4 + c] * u[4 + c]) + t[8 + c] * u[8 + c];
      duplicate = trace > 2.9;
    }
    if (!duplicate) kept[m++] = h;
    if (m >= topk) break;
  }
  return m;
}

}  // extern "C"
