// preprocess.cuh — R 3.5.3-3.5.5 on the device (fragment/breakline.rs): the
// breakline points, their shell and fracture macro normals, frames, validity
// and dihedrals. The adjacency, the nearest-point searches, the radius balls
// and the voxel grid are segmentation's kernels (segment.cuh); the kernels
// here are the per-element steps between them.
#pragma once

#include "segment.cuh"

namespace sherd {

__global__ void k_iota(uint32_t *a, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}

// Entry w of the sorted edge list is a breakline edge when it pairs two faces
// (k_face_pairs) whose fracture labels differ (breakline.rs:227-235).
__global__ void k_brk_flags(const uint32_t *fa, const uint32_t *fb, uint32_t m, const uint8_t *frac,
                            uint8_t *flag) {
  uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= m) return;
  uint32_t a = fa[w], b = fb[w];
  flag[w] = a != MISS && ((frac[a] != 0) != (frac[b] != 0));
}

// The midpoint 0.5 (a + b) of each breakline edge, its vertices read from the
// sorted edge key (lo << 32 | hi).
__global__ void k_brk_points(const unsigned long long *key, const uint32_t *sel, uint32_t n,
                             const double *v, double *p) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned long long k = key[sel[i]];
  const double *a = v + 3 * size_t(uint32_t(k >> 32)), *b = v + 3 * size_t(uint32_t(k));
  for (int c = 0; c < 3; ++c) p[3 * size_t(i) + c] = 0.5 * (a[c] + b[c]);
}

// The two face selections of one macro normal (breakline.rs:318-324): every
// face of the mask, and those at distance >= inner from the breakline.
__global__ void k_macro_masks(const uint8_t *frac, uint8_t fracture, const double *dist,
                              double inner, uint32_t nf, uint8_t *every, uint8_t *far) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nf) return;
  bool in = (frac[j] != 0) == (fracture != 0);
  every[j] = in;
  far[j] = in && dist[j] >= inner;
}

__global__ void k_gather1(const double *src, const uint32_t *idx, uint32_t n, double *dst) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[idx[i]];
}

__device__ __forceinline__ double norm3(const double *a) {
  return sqrt((a[0] * a[0] + a[1] * a[1]) + a[2] * a[2]);
}

// The points whose macro normal is shorter than VALID_MIN (0.5) take the
// fallback over the whole mask (breakline.rs:326-336).
__global__ void k_short_normals(const double *n3, uint32_t n, uint8_t *flag) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[i] = norm3(n3 + 3 * size_t(i)) < 0.5;
}

__global__ void k_scatter3(const double *src, const uint32_t *idx, uint32_t n, double *dst) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int c = 0; c < 3; ++c) dst[3 * size_t(idx[i]) + c] = src[3 * size_t(i) + c];
}

// f = nf - (nf . ns) ns over max(|.|, 1e-9); valid = |ns|, |nf|, |ns x f| all
// above 0.5 (breakline.rs:240-258); the dihedral acos(clamp(ns . nf)) in
// degrees (breakline.rs:189-195).
__global__ void k_brk_frames(const double *ns, const double *nf, uint32_t n, double *f,
                             uint8_t *valid, double *dih) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double *s = ns + 3 * size_t(i), *r = nf + 3 * size_t(i);
  double d = (r[0] * s[0] + r[1] * s[1]) + r[2] * s[2];
  double g[3] = {r[0] - d * s[0], r[1] - d * s[1], r[2] - d * s[2]};
  double den = fmax(norm3(g), 1e-9);
  for (int c = 0; c < 3; ++c) g[c] /= den;
  for (int c = 0; c < 3; ++c) f[3 * size_t(i) + c] = g[c];
  double t[3] = {s[1] * g[2] - s[2] * g[1], s[2] * g[0] - s[0] * g[2], s[0] * g[1] - s[1] * g[0]};
  valid[i] = norm3(s) > 0.5 && norm3(r) > 0.5 && norm3(t) > 0.5;
  double dd = (s[0] * r[0] + s[1] * r[1]) + s[2] * r[2];
  dih[i] = acos(fmin(fmax(dd, -1.0), 1.0)) * (180.0 / 3.141592653589793);
}

// The representatives that carry a valid frame (breakline.rs:261-265).
__global__ void k_valid_reps(const uint32_t *rep, uint32_t n, const uint8_t *valid, uint8_t *flag) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[i] = valid[rep[i]];
}

}  // namespace sherd
