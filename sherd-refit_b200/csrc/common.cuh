// common.cuh — shared definitions of the sm_100a geometry backend.
//
// The whole library is compiled with -fmad=false: the reference's arithmetic
// (Rust, no contraction) never fuses a multiply into an add, and bit-exact
// agreement of hit distances, point-to-triangle distances and decisions with
// the CPU oracle depends on every operation here being the same IEEE operation
// in the same order.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/sherd_cuda.h"

namespace sherd {

constexpr uint32_t MISS = 0xFFFFFFFFu;
#ifndef TRI_LEAF_MAX
#define TRI_LEAF_MAX 6
#endif
constexpr int TRI_LEAF = TRI_LEAF_MAX;  // faces per BVH leaf, at most
#ifndef POINT_LEAF_MAX
#define POINT_LEAF_MAX 2
#endif
constexpr int POINT_LEAF = POINT_LEAF_MAX;  // points per BVH leaf, at most
// Resident 256-thread CTAs per SM k_pen_inside is compiled for (48 registers a
// thread): 5 measured 916 ms on the collection against 990 with the compiler's
// own 64 registers (3-4 CTAs) and 1003 at 4; k_pen_min gained nothing at 4-6.
#ifndef PEN_INSIDE_MINB
#define PEN_INSIDE_MINB 5
#endif
// Whether point clouds carry the 4-wide tree that nearest_within_sq walks.
#ifndef WIDE_NN
#define WIDE_NN 1
#endif
constexpr int STACK = 64;      // traversal stack entries (Karras depth <= 63 + log2 n)

__host__ __device__ inline float f_inf() { return __builtin_huge_valf(); }
__host__ __device__ inline double d_inf() { return __builtin_huge_val(); }

// A read-only 32-byte load as two 16-byte loads through the texture path.
__device__ __forceinline__ double4 ldg4(const double4 *p) {
  const double2 *q = reinterpret_cast<const double2 *>(p);
  double2 a = __ldg(q), b = __ldg(q + 1);
  return make_double4(a.x, a.y, b.x, b.y);
}

// Status bits a kernel can raise for its call (read back by the host).
enum : uint32_t {
  ST_STACK = 1u,    // a traversal stack overflowed (answer not trusted)
  ST_TIMEOUT = 2u,  // the persistent kernel ran past its time budget
  ST_ABORTED = 4u,  // the host asked the persistent kernel to stop
  ST_SCRATCH = 8u,  // a per-item scratch buffer was too small
  ST_RANGE = 16u,   // a value outside the range a kernel's encoding supports
};

struct F3 {
  float x, y, z;
};
__device__ __forceinline__ F3 sub(F3 a, F3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ F3 cross(F3 a, F3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ float dot(F3 a, F3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

// types::apply_transform (types.rs:175-181): R p + tau, f64, left to right.
__device__ __forceinline__ void apply_pose(const double *t, double px, double py, double pz,
                                           double &ox, double &oy, double &oz) {
  ox = t[0] * px + t[1] * py + t[2] * pz + t[3];
  oy = t[4] * px + t[5] * py + t[6] * pz + t[7];
  oz = t[8] * px + t[9] * py + t[10] * pz + t[11];
}
// verify::rotate (verify.rs:711-717): R n, f64.
__device__ __forceinline__ void rotate_pose(const double *t, double px, double py, double pz,
                                            double &ox, double &oy, double &oz) {
  ox = t[0] * px + t[1] * py + t[2] * pz;
  oy = t[4] * px + t[5] * py + t[6] * pz;
  oz = t[8] * px + t[9] * py + t[10] * pz;
}

// Moller-Trumbore exactly as spatial/bvh.rs:199-220 writes it: the ray
// parameter of a crossing, or -1 when there is none.
__device__ __forceinline__ float moller_trumbore(F3 o, F3 d, F3 v0, F3 v1, F3 v2) {
  const float EPS = 1e-9f;
  F3 e1 = sub(v1, v0), e2 = sub(v2, v0);
  F3 pvec = cross(d, e2);
  float det = dot(e1, pvec);
  if (fabsf(det) < EPS) return -1.0f;
  float inv = 1.0f / det;
  F3 tvec = sub(o, v0);
  float u = inv * dot(tvec, pvec);
  if (!(u >= 0.0f && u <= 1.0f)) return -1.0f;
  F3 qvec = cross(tvec, e1);
  float v = inv * dot(d, qvec);
  if (v < 0.0f || u + v > 1.0f) return -1.0f;
  float t = inv * dot(e2, qvec);
  return t > EPS ? t : -1.0f;
}

// moller_trumbore with the two edges already formed (e1 = v1 - v0 and
// e2 = v2 - v0 in f32, the same values the test computes itself).
__device__ __forceinline__ float moller_trumbore_edges(F3 o, F3 d, F3 v0, F3 e1, F3 e2) {
  const float EPS = 1e-9f;
  F3 pvec = cross(d, e2);
  float det = dot(e1, pvec);
  if (fabsf(det) < EPS) return -1.0f;
  float inv = 1.0f / det;
  F3 tvec = sub(o, v0);
  float u = inv * dot(tvec, pvec);
  if (!(u >= 0.0f && u <= 1.0f)) return -1.0f;
  F3 qvec = cross(tvec, e1);
  float v = inv * dot(d, qvec);
  if (v < 0.0f || u + v > 1.0f) return -1.0f;
  float t = inv * dot(e2, qvec);
  return t > EPS ? t : -1.0f;
}

// Point-to-triangle distance: the Voronoi-region closest point of Ericson,
// "Real-Time Collision Detection" 5.1.5, in f32 (the reference's scene is f32).
__device__ __forceinline__ float tri_distance(F3 p, F3 a, F3 b, F3 c) {
  F3 ab = sub(b, a), ac = sub(c, a), ap = sub(p, a);
  float d1 = dot(ab, ap), d2 = dot(ac, ap);
  F3 q;
  if (d1 <= 0.0f && d2 <= 0.0f) {
    q = a;
  } else {
    F3 bp = sub(p, b);
    float d3 = dot(ab, bp), d4 = dot(ac, bp);
    if (d3 >= 0.0f && d4 <= d3) {
      q = b;
    } else {
      float vc = d1 * d4 - d3 * d2;
      if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
        float s = d1 / (d1 - d3);
        q = {a.x + s * ab.x, a.y + s * ab.y, a.z + s * ab.z};
      } else {
        F3 cp = sub(p, c);
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
              F3 bc = sub(c, b);
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
  F3 dq = sub(q, p);
  return sqrtf(dot(dq, dq));
}

// Orders non-negative floats (and +inf) as unsigned integers, for atomicMin.
__device__ __forceinline__ unsigned f2key(float x) { return __float_as_uint(x); }
__device__ __forceinline__ float key2f(unsigned k) { return __uint_as_float(k); }

// An order-preserving map of f64 bit patterns onto u64 (negative values too).
__device__ __forceinline__ unsigned long long d2key(double x) {
  unsigned long long b = __double_as_longlong(x);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}
__device__ __forceinline__ double key2d(unsigned long long k) {
  unsigned long long b = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFULL) : ~k;
  return __longlong_as_double(b);
}

// What the input checks found in an uploaded array: the largest |x| of its
// finite coordinates (the f64 bits of a non-negative value, which order as
// u64), whether any coordinate was not finite, and whether any index reached
// its limit.
struct InputCheck {
  unsigned long long max_abs;
  unsigned non_finite;
  unsigned bad_index;
};

__device__ __forceinline__ void input_check_commit(InputCheck *out, unsigned long long m, unsigned nonf,
                                                   unsigned bad) {
  for (int o = 16; o; o >>= 1) {
    unsigned long long other = __shfl_xor_sync(0xffffffffu, m, o);
    m = other > m ? other : m;
    nonf |= __shfl_xor_sync(0xffffffffu, nonf, o);
    bad |= __shfl_xor_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (m) atomicMax(&out->max_abs, m);
    if (nonf) atomicOr(&out->non_finite, 1u);
    if (bad) atomicOr(&out->bad_index, 1u);
  }
}

// Coordinates: every value finite, and the largest magnitude.
__global__ void k_check_coords(const double *p, size_t n, InputCheck *out) {
  unsigned long long m = 0;
  unsigned nonf = 0;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
    double x = p[i];
    if (isfinite(x)) {
      unsigned long long b = (unsigned long long)__double_as_longlong(fabs(x));
      m = b > m ? b : m;
    } else {
      nonf = 1;
    }
  }
  input_check_commit(out, m, nonf, 0);
}

// Indices: every one below `limit`.
__global__ void k_check_indices(const uint32_t *f, size_t n, uint32_t limit, InputCheck *out) {
  unsigned bad = 0;
  for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
    bad |= f[i] >= limit ? 1u : 0u;
  input_check_commit(out, 0, 0, bad);
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

}  // namespace sherd
