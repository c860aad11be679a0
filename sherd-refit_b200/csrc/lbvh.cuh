// lbvh.cuh — device-built linear BVH (Karras 2012) over triangles or points.
//
// Build: 63-bit Morton codes of the primitive centres over the scene box, a
// CUB radix sort of (code, primitive) pairs, the Karras hierarchy over the
// sorted codes (equal codes split by index), a bottom-up box refit with one
// atomic arrival counter per node, and a final pass that writes the compact
// traversal layout:
//
//   BNode (64 B, four 16-byte loads): both children's boxes, already padded
//   outward, and for each child either an internal node index or a leaf range
//   (first, count) of consecutive sorted primitives. A Karras subtree holding
//   at most TRI_LEAF / POINT_LEAF primitives is a leaf range, so leaves hold
//   several primitives without a separate collapse pass.
//
// Primitives are stored in sorted (leaf) order next to their original index,
// so a leaf is one contiguous, coalesced run of memory.
#pragma once

#include "common.cuh"

namespace sherd {

struct __align__(16) BNode {
  float4 a;  // lo0.x lo0.y lo0.z hi0.x
  float4 b;  // hi0.y hi0.z lo1.x lo1.y
  float4 c;  // lo1.z hi1.x hi1.y hi1.z
  int4 d;    // ref0 ref1 cnt0 cnt1  (cnt > 0: leaf range at ref; cnt == 0: node ref)
};

// The 4-wide form of a point tree for the nearest-point search: the node at a
// binary node's index holds that node's grandchildren (or a child itself where
// the child is a leaf range), so a descent takes half as many dependent loads.
// The boxes are the binary tree's own padded boxes. 128 B, eight 16-byte loads:
// the four children's boxes by coordinate, then per child the internal node
// index or the leaf's first slot, and the leaf's count (0 for a node, -1 for no
// child; an absent child's box is empty, so every box distance to it is +inf).
struct __align__(16) WNode {
  float4 lox, loy, loz, hix, hiy, hiz;
  int4 ref, cnt;
};

// The crossing grid of one axis: the mesh projected onto the plane of the other
// two axes (u, v) = ((a+1)%3, (a+2)%3), cut into square cells; each cell lists
// (CSR) the sorted slots of every face whose padded projected rectangle
// touches it. An axis ray from p can only cross faces in p's own cell.
struct AxisGrid {
  const uint32_t *start;  // nu * nv + 1 offsets into the entry arrays
  const float4 *rect;     // per entry: the face's padded projected rectangle (u0, u1, v0, v1)
  const float4 *tri;      // per entry, 3 float4: v0, e1 = v1 - v0, e2 = v2 - v0 (f32)
  float lo_u, lo_v, inv_cell;
  uint32_t nu, nv;
};

// The mesh's bound grid: a cube-celled grid over the mesh's box widened by a
// quarter of its largest extent on every side, holding per cell a lower bound
// (rounded down) on the distance from any point of the cell to any leaf box of
// the tree, and so to any face. Null `lb` when the mesh is a single leaf.
struct LbGrid {
  const float *lb;
  float lo[3];
  float cell, inv_cell;
  uint32_t n[3];
};

// What the traversal kernels take by value.
struct MeshView {
  const BNode *nodes;
  const float4 *tri;  // 3 per sorted slot: (v0, original face id bits), (v1, 0), (v2, 0)
  uint32_t nf;
  uint32_t root_leaf;  // nf when the whole mesh is one leaf, else 0
  float pad;           // outward padding of every node box
  float lo[3], hi[3];  // exact vertex box (RayScene::aabb)
  AxisGrid grid[3];    // crossing grids for the +x, +y, +z parity rays
  LbGrid lbg;          // lower bounds of the distance to the mesh, per cell
};

struct CloudView {
  const BNode *nodes;
  const double4 *pts;  // sorted: (x, y, z, original index)
  const double4 *nrm;  // sorted unit normals (x, y, z, 0), or null
  uint32_t n;
  uint32_t root_leaf;
  float pad;
  const WNode *wide;   // the 4-wide form of `nodes`, or null
};

// ---- Morton codes -----------------------------------------------------------

__device__ __forceinline__ unsigned long long expand21(unsigned v) {
  unsigned long long x = v & 0x1fffffu;
  x = (x | x << 32) & 0x1f00000000ffffULL;
  x = (x | x << 16) & 0x1f0000ff0000ffULL;
  x = (x | x << 8) & 0x100f00f00f00f00fULL;
  x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
  x = (x | x << 2) & 0x1249249249249249ULL;
  return x;
}

__device__ __forceinline__ unsigned quant21(double c, double lo, double inv_ext) {
  double u = (c - lo) * inv_ext;
  u = u < 0.0 ? 0.0 : (u > 1.0 ? 1.0 : u);
  unsigned q = unsigned(u * 2097151.0);
  return q > 2097151u ? 2097151u : q;
}

__device__ __forceinline__ unsigned long long morton3(double x, double y, double z,
                                                      const double *lo, const double *inv) {
  return (expand21(quant21(x, lo[0], inv[0])) << 2) | (expand21(quant21(y, lo[1], inv[1])) << 1) |
         expand21(quant21(z, lo[2], inv[2]));
}

// Order-preserving float -> uint, for atomic min/max of signed floats.
__device__ __forceinline__ unsigned ford(float x) {
  unsigned b = __float_as_uint(x);
  return (b >> 31) ? ~b : (b | 0x80000000u);
}
__host__ __device__ inline float fordinv(unsigned k) {
  unsigned b = (k >> 31) ? (k & 0x7fffffffu) : ~k;
  float f;
  memcpy(&f, &b, 4);
  return f;
}

// Scene box of f32 vertices: bounds[0..2] = ford(min), bounds[3..5] = ford(max).
__global__ void k_bounds_f32(const float *v, uint32_t nv, unsigned *bounds) {
  float lo[3] = {f_inf(), f_inf(), f_inf()}, hi[3] = {-f_inf(), -f_inf(), -f_inf()};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += gridDim.x * blockDim.x)
    for (int k = 0; k < 3; ++k) {
      float x = v[3 * i + k];
      lo[k] = fminf(lo[k], x);
      hi[k] = fmaxf(hi[k], x);
    }
  for (int k = 0; k < 3; ++k) {
    for (int o = 16; o; o >>= 1) {
      lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
      hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&bounds[k], ford(lo[k]));
      atomicMax(&bounds[3 + k], ford(hi[k]));
    }
  }
}

// Scene box of f64 points, rounded outward to f32.
__global__ void k_bounds_f64(const double *p, uint32_t n, unsigned *bounds) {
  float lo[3] = {f_inf(), f_inf(), f_inf()}, hi[3] = {-f_inf(), -f_inf(), -f_inf()};
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    for (int k = 0; k < 3; ++k) {
      double x = p[3 * i + k];
      lo[k] = fminf(lo[k], __double2float_rd(x));
      hi[k] = fmaxf(hi[k], __double2float_ru(x));
    }
  for (int k = 0; k < 3; ++k) {
    for (int o = 16; o; o >>= 1) {
      lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
      hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&bounds[k], ford(lo[k]));
      atomicMax(&bounds[3 + k], ford(hi[k]));
    }
  }
}

struct BuildBox {
  double lo[3], inv[3];
};

__global__ void k_morton_tri(const float *v, const uint32_t *f, uint32_t nf, BuildBox box,
                             unsigned long long *keys, uint32_t *vals) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nf) return;
  double c[3];
  for (int k = 0; k < 3; ++k)
    c[k] = (double(v[3 * f[3 * i] + k]) + double(v[3 * f[3 * i + 1] + k]) +
            double(v[3 * f[3 * i + 2] + k])) / 3.0;
  keys[i] = morton3(c[0], c[1], c[2], box.lo, box.inv);
  vals[i] = i;
}

__global__ void k_morton_pts(const double *p, uint32_t n, BuildBox box, unsigned long long *keys,
                             uint32_t *vals) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keys[i] = morton3(p[3 * i], p[3 * i + 1], p[3 * i + 2], box.lo, box.inv);
  vals[i] = i;
}

// ---- Karras hierarchy -------------------------------------------------------

__device__ __forceinline__ int kdelta(const unsigned long long *keys, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  unsigned long long a = keys[i], b = keys[j];
  if (a == b) return 64 + __clz(unsigned(i) ^ unsigned(j));
  return __clzll(a ^ b);
}

// Internal node i of n-1: children (leaf primitive k encoded as k | 0x80000000),
// the primitive range it covers and the parent links.
__global__ void k_karras(const unsigned long long *keys, int n, int *left, int *right, int *first,
                         int *last, int *parent_int, int *parent_leaf) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  int d = (kdelta(keys, n, i, i + 1) - kdelta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
  int dmin = kdelta(keys, n, i, i - d);
  int lmax = 2;
  while (kdelta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (kdelta(keys, n, i, i + (l + t) * d) > dmin) l += t;
  int j = i + l * d;
  int dnode = kdelta(keys, n, i, j);
  int s = 0;
  for (int div = 2;; div <<= 1) {
    int t = (l + div - 1) / div;
    if (kdelta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    if (t <= 1) break;
  }
  int gamma = i + s * d + (d < 0 ? -1 : 0);
  int lo = i < j ? i : j, hi = i < j ? j : i;
  first[i] = lo;
  last[i] = hi;
  if (lo == gamma) {
    left[i] = gamma | int(0x80000000);
    parent_leaf[gamma] = i;
  } else {
    left[i] = gamma;
    parent_int[gamma] = i;
  }
  if (hi == gamma + 1) {
    right[i] = (gamma + 1) | int(0x80000000);
    parent_leaf[gamma + 1] = i;
  } else {
    right[i] = gamma + 1;
    parent_int[gamma + 1] = i;
  }
}

struct Box {
  float lo[3], hi[3];
};

__device__ __forceinline__ Box tri_box(const float *v, const uint32_t *f, uint32_t face) {
  Box b;
  for (int k = 0; k < 3; ++k) {
    float a0 = v[3 * f[3 * face] + k], a1 = v[3 * f[3 * face + 1] + k], a2 = v[3 * f[3 * face + 2] + k];
    b.lo[k] = fminf(a0, fminf(a1, a2));
    b.hi[k] = fmaxf(a0, fmaxf(a1, a2));
  }
  return b;
}

__device__ __forceinline__ Box pt_box(const double *p, uint32_t i) {
  Box b;
  for (int k = 0; k < 3; ++k) {
    b.lo[k] = __double2float_rd(p[3 * i + k]);
    b.hi[k] = __double2float_ru(p[3 * i + k]);
  }
  return b;
}

template <bool TRI>
__device__ __forceinline__ Box prim_box(const float *v, const uint32_t *f, const double *p,
                                        const uint32_t *sorted, int k) {
  return TRI ? tri_box(v, f, sorted[k]) : pt_box(p, sorted[k]);
}

__device__ __forceinline__ Box load_box(const float *ib, int node) {
  Box b;
  for (int k = 0; k < 3; ++k) {
    b.lo[k] = __ldcg(ib + 6 * node + k);
    b.hi[k] = __ldcg(ib + 6 * node + 3 + k);
  }
  return b;
}

// Bottom-up refit: one thread per primitive walks to the root; the second
// thread to reach a node computes its box.
template <bool TRI>
__global__ void k_refit(const float *v, const uint32_t *f, const double *p, const uint32_t *sorted,
                        int n, const int *left, const int *right, const int *parent_int,
                        const int *parent_leaf, unsigned *flags, float *ibox) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int node = parent_leaf[k];
  for (int steps = 0; node >= 0 && steps < 256; ++steps) {
    __threadfence();
    if (atomicAdd(&flags[node], 1u) == 0u) return;
    __threadfence();
    Box out;
    for (int c = 0; c < 2; ++c) {
      int ref = c == 0 ? left[node] : right[node];
      Box b = ref < 0 ? prim_box<TRI>(v, f, p, sorted, ref & 0x7fffffff) : load_box(ibox, ref);
      for (int a = 0; a < 3; ++a) {
        out.lo[a] = c == 0 ? b.lo[a] : fminf(out.lo[a], b.lo[a]);
        out.hi[a] = c == 0 ? b.hi[a] : fmaxf(out.hi[a], b.hi[a]);
      }
    }
    for (int a = 0; a < 3; ++a) {
      __stcg(ibox + 6 * node + a, out.lo[a]);
      __stcg(ibox + 6 * node + 3 + a, out.hi[a]);
    }
    node = parent_int[node];
  }
}

// The traversal layout, one BNode per internal node, boxes padded outward.
template <bool TRI>
__global__ void k_emit(const float *v, const uint32_t *f, const double *p, const uint32_t *sorted,
                       int n, const int *left, const int *right, const int *first, const int *last,
                       const float *ibox, float pad, int leaf_max, BNode *nodes) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  Box bx[2];
  int ref[2], cnt[2];
  for (int c = 0; c < 2; ++c) {
    int r = c == 0 ? left[i] : right[i];
    if (r < 0) {
      int k = r & 0x7fffffff;
      bx[c] = prim_box<TRI>(v, f, p, sorted, k);
      ref[c] = k;
      cnt[c] = 1;
    } else {
      bx[c] = load_box(ibox, r);
      int size = last[r] - first[r] + 1;
      if (size <= leaf_max) {
        ref[c] = first[r];
        cnt[c] = size;
      } else {
        ref[c] = r;
        cnt[c] = 0;
      }
    }
    for (int a = 0; a < 3; ++a) {
      bx[c].lo[a] = __fsub_rd(bx[c].lo[a], pad);
      bx[c].hi[a] = __fadd_ru(bx[c].hi[a], pad);
    }
  }
  BNode nd;
  nd.a = make_float4(bx[0].lo[0], bx[0].lo[1], bx[0].lo[2], bx[0].hi[0]);
  nd.b = make_float4(bx[0].hi[1], bx[0].hi[2], bx[1].lo[0], bx[1].lo[1]);
  nd.c = make_float4(bx[1].lo[2], bx[1].hi[0], bx[1].hi[1], bx[1].hi[2]);
  nd.d = make_int4(ref[0], ref[1], cnt[0], cnt[1]);
  nodes[i] = nd;
}

// One WNode per binary node i: i's children, a child that is an internal node
// replaced by that node's two children.
__global__ void k_widen(const BNode *nodes, int ni, WNode *wide) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ni) return;
  float lo[4][3], hi[4][3];
  int ref[4], cnt[4], m = 0;
  auto put = [&](const BNode &b, int c) {
    const float4 a = b.a, bb = b.b, cc = b.c;
    if (c == 0) {
      lo[m][0] = a.x; lo[m][1] = a.y; lo[m][2] = a.z;
      hi[m][0] = a.w; hi[m][1] = bb.x; hi[m][2] = bb.y;
      ref[m] = b.d.x;
      cnt[m] = b.d.z;
    } else {
      lo[m][0] = bb.z; lo[m][1] = bb.w; lo[m][2] = cc.x;
      hi[m][0] = cc.y; hi[m][1] = cc.z; hi[m][2] = cc.w;
      ref[m] = b.d.y;
      cnt[m] = b.d.w;
    }
    ++m;
  };
  const BNode b = nodes[i];
  for (int c = 0; c < 2; ++c) {
    const int r = c == 0 ? b.d.x : b.d.y, n = c == 0 ? b.d.z : b.d.w;
    if (n > 0) {
      put(b, c);
    } else {
      const BNode g = nodes[r];
      put(g, 0);
      put(g, 1);
    }
  }
  for (; m < 4; ++m) {
    for (int a = 0; a < 3; ++a) {
      lo[m][a] = f_inf();
      hi[m][a] = -f_inf();
    }
    ref[m] = -1;
    cnt[m] = -1;
  }
  WNode w;
  w.lox = make_float4(lo[0][0], lo[1][0], lo[2][0], lo[3][0]);
  w.loy = make_float4(lo[0][1], lo[1][1], lo[2][1], lo[3][1]);
  w.loz = make_float4(lo[0][2], lo[1][2], lo[2][2], lo[3][2]);
  w.hix = make_float4(hi[0][0], hi[1][0], hi[2][0], hi[3][0]);
  w.hiy = make_float4(hi[0][1], hi[1][1], hi[2][1], hi[3][1]);
  w.hiz = make_float4(hi[0][2], hi[1][2], hi[2][2], hi[3][2]);
  w.ref = make_int4(ref[0], ref[1], ref[2], ref[3]);
  w.cnt = make_int4(cnt[0], cnt[1], cnt[2], cnt[3]);
  wide[i] = w;
}

// ---- crossing grids ---------------------------------------------------------

__device__ __forceinline__ void grid_rect(const float4 *tri, uint32_t s, int axis, const AxisGrid &g,
                                          float pad, int &u0, int &u1, int &v0, int &v1) {
  int au = (axis + 1) % 3, av = (axis + 2) % 3;
  float umin = f_inf(), umax = -f_inf(), vmin = f_inf(), vmax = -f_inf();
  for (int k = 0; k < 3; ++k) {
    float4 p = tri[3 * s + k];
    float c[3] = {p.x, p.y, p.z};
    umin = fminf(umin, c[au]);
    umax = fmaxf(umax, c[au]);
    vmin = fminf(vmin, c[av]);
    vmax = fmaxf(vmax, c[av]);
  }
  u0 = int(floorf((__fsub_rd(umin, pad) - g.lo_u) * g.inv_cell));
  u1 = int(floorf((__fadd_ru(umax, pad) - g.lo_u) * g.inv_cell));
  v0 = int(floorf((__fsub_rd(vmin, pad) - g.lo_v) * g.inv_cell));
  v1 = int(floorf((__fadd_ru(vmax, pad) - g.lo_v) * g.inv_cell));
  u0 = max(u0, 0);
  v0 = max(v0, 0);
  u1 = min(u1, int(g.nu) - 1);
  v1 = min(v1, int(g.nv) - 1);
}

__global__ void k_grid_count(const float4 *tri, uint32_t nf, int axis, AxisGrid g, float pad,
                             unsigned *count) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nf) return;
  int u0, u1, v0, v1;
  grid_rect(tri, s, axis, g, pad, u0, u1, v0, v1);
  for (int u = u0; u <= u1; ++u)
    for (int v = v0; v <= v1; ++v) atomicAdd(&count[size_t(u) * g.nv + v], 1u);
}

// Writes every face's entries: its padded projected rectangle and its vertex
// and edges, so the parity test reads one contiguous run per cell.
__global__ void k_grid_fill(const float4 *tri, uint32_t nf, int axis, AxisGrid g, float pad,
                            unsigned *cursor, float4 *rect, float4 *edge) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nf) return;
  int u0, u1, v0, v1;
  grid_rect(tri, s, axis, g, pad, u0, u1, v0, v1);
  int au = (axis + 1) % 3, av = (axis + 2) % 3;
  float4 a = tri[3 * s], b = tri[3 * s + 1], c = tri[3 * s + 2];
  float ac[3] = {a.x, a.y, a.z}, bc[3] = {b.x, b.y, b.z}, cc[3] = {c.x, c.y, c.z};
  float4 r = make_float4(__fsub_rd(fminf(ac[au], fminf(bc[au], cc[au])), pad),
                         __fadd_ru(fmaxf(ac[au], fmaxf(bc[au], cc[au])), pad),
                         __fsub_rd(fminf(ac[av], fminf(bc[av], cc[av])), pad),
                         __fadd_ru(fmaxf(ac[av], fmaxf(bc[av], cc[av])), pad));
  float4 t0 = make_float4(a.x, a.y, a.z, 0.0f);
  float4 t1 = make_float4(b.x - a.x, b.y - a.y, b.z - a.z, 0.0f);
  float4 t2 = make_float4(c.x - a.x, c.y - a.y, c.z - a.z, 0.0f);
  for (int u = u0; u <= u1; ++u)
    for (int v = v0; v <= v1; ++v) {
      unsigned k = atomicAdd(&cursor[size_t(u) * g.nv + v], 1u);
      rect[k] = r;
      edge[3 * size_t(k)] = t0;
      edge[3 * size_t(k) + 1] = t1;
      edge[3 * size_t(k) + 2] = t2;
    }
}

// One thread per cell of the bound grid: the smallest box-to-box distance
// from the cell (widened by 1e-3 cell on every side) to a leaf box of the
// tree, every step rounded down, by a nearest-first walk that skips subtrees
// whose box is no nearer than the best so far.
__global__ void k_lb_grid(const BNode *nodes, LbGrid g, float *lb) {
  size_t c = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  size_t total = size_t(g.n[0]) * g.n[1] * g.n[2];
  if (c >= total) return;
  uint32_t iz = uint32_t(c % g.n[2]), iy = uint32_t((c / g.n[2]) % g.n[1]),
           ix = uint32_t(c / (size_t(g.n[2]) * g.n[1]));
  const uint32_t idx[3] = {ix, iy, iz};
  float clo[3], chi[3];
  for (int a = 0; a < 3; ++a) {
    clo[a] = __fsub_rd(__fadd_rd(g.lo[a], __fmul_rd(float(idx[a]), g.cell)), 1e-3f * g.cell);
    chi[a] = __fadd_ru(__fadd_ru(g.lo[a], __fmul_ru(float(idx[a] + 1), g.cell)), 1e-3f * g.cell);
  }
  auto gap2 = [&](const float4 &a, const float4 &b, const float4 &cc, int child) {
    float blo[3], bhi[3];
    if (child == 0) {
      blo[0] = a.x; blo[1] = a.y; blo[2] = a.z; bhi[0] = a.w; bhi[1] = b.x; bhi[2] = b.y;
    } else {
      blo[0] = b.z; blo[1] = b.w; blo[2] = cc.x; bhi[0] = cc.y; bhi[1] = cc.z; bhi[2] = cc.w;
    }
    float s = 0.0f;
    for (int k = 0; k < 3; ++k) {
      float d = fmaxf(fmaxf(__fsub_rd(blo[k], chi[k]), __fsub_rd(clo[k], bhi[k])), 0.0f);
      s = __fadd_rd(s, __fmul_rd(d, d));
    }
    return s;
  };
  float best = f_inf();
  int stack_n[STACK];
  float stack_k[STACK];
  int sp = 0, node = 0;
  for (int visits = 0; visits < (1 << 22); ++visits) {
    const float4 *q = reinterpret_cast<const float4 *>(nodes + node);
    float4 a = q[0], b = q[1], cc = q[2];
    int4 d = reinterpret_cast<const int4 *>(q)[3];
    const int ref[2] = {d.x, d.y}, cnt[2] = {d.z, d.w};
    float k[2] = {gap2(a, b, cc, 0), gap2(a, b, cc, 1)};
    int near_c = k[1] < k[0] ? 1 : 0;
    int next = -1;
    for (int qq = 0; qq < 2; ++qq) {
      int ch = qq == 0 ? near_c : 1 - near_c;
      if (!(k[ch] < best)) continue;
      if (cnt[ch]) {
        best = k[ch];
      } else if (next < 0) {
        next = ref[ch];
      } else if (sp < STACK) {
        stack_n[sp] = ref[ch];
        stack_k[sp++] = k[ch];
      } else {
        best = 0.0f;  // out of stack: the bound falls back to 0 (no pruning)
        sp = 0;
        next = -1;
        break;
      }
    }
    if (next >= 0) {
      node = next;
      continue;
    }
    bool more = false;
    while (sp > 0) {
      --sp;
      if (stack_k[sp] < best) {
        node = stack_n[sp];
        more = true;
        break;
      }
    }
    if (!more) {
      lb[c] = best == f_inf() ? 0.0f : __fsqrt_rd(best);
      return;
    }
  }
  lb[c] = 0.0f;  // walk cap reached: no bound
}

__global__ void k_store_tris(const float *v, const uint32_t *f, const uint32_t *sorted, uint32_t nf,
                             float4 *tri) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nf) return;
  uint32_t face = sorted[s];
  const float *a = v + 3 * f[3 * face], *b = v + 3 * f[3 * face + 1], *c = v + 3 * f[3 * face + 2];
  tri[3 * s] = make_float4(a[0], a[1], a[2], __uint_as_float(face));
  tri[3 * s + 1] = make_float4(b[0], b[1], b[2], 0.0f);
  tri[3 * s + 2] = make_float4(c[0], c[1], c[2], 0.0f);
}

__global__ void k_store_pts(const double *p, const double *nrm, const uint32_t *sorted, uint32_t n,
                            double4 *pts, double4 *nout) {
  uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  uint32_t i = sorted[s];
  pts[s] = make_double4(p[3 * i], p[3 * i + 1], p[3 * i + 2], double(i));
  if (nrm) nout[s] = make_double4(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2], 0.0);
}

}  // namespace sherd
