// refine.cuh — R 9, full-resolution join refinement (refine.rs): the vertex
// normals of an original mesh, the fused placement of a fracture cloud, and a
// point-to-plane rung spread over the whole device for one pose.
//
// A join's rung registers a single pose on up to 150 000 source points
// (refine.rs:56). k_icp_rung gives each pose one block, which here would leave
// every SM but one idle, so each pass of a wide rung is one launch over the
// whole device (k_wide_pass): every block takes its own contiguous slice of
// the source and runs the block rung's correspondence pass over it (icp_pass:
// moved point, nearest target inside the strict radius, the 29 normal-equation
// sums); the last block to finish adds the slices' sums in a fixed order (a
// rung is reproducible run to run), runs Open3D's convergence test and the
// point-to-plane update, and publishes the pose of the next pass. A finished
// rung (converged, or out of iterations) sets `done`, after which the kernel
// returns at once, so the host launches the whole iteration budget without
// reading anything back.
#pragma once

#include "kernels.cuh"

namespace sherd {

// ---- vertex normals (refine.rs:121-151) --------------------------------------

// The (vertex, face) incidence in face-major order: one entry per corner.
__global__ void k_incidence(const uint32_t *f, uint32_t n_corners, uint32_t *vertex,
                            uint32_t *face) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_corners) return;
  vertex[i] = f[i];
  face[i] = i / 3u;
}

// One thread per vertex over the incidence sorted (stably) by vertex, so its
// faces come in ascending order, as the reference's face loop adds them; a
// face that names the vertex twice adds its normal twice, as there.
__global__ void k_vertex_normals(const double *v, const uint32_t *f, const uint32_t *vertex,
                                 const uint32_t *face, uint32_t n_corners, uint32_t nv,
                                 double *out) {
  uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nv) return;
  uint32_t lo = 0, hi = n_corners;
  while (lo < hi) {
    uint32_t mid = lo + (hi - lo) / 2u;
    if (vertex[mid] < j)
      lo = mid + 1u;
    else
      hi = mid;
  }
  double s[3] = {0.0, 0.0, 0.0};
  for (uint32_t k = lo; k < n_corners && vertex[k] == j; ++k) {
    const uint32_t *tri = f + 3 * size_t(face[k]);
    const double *o = v + 3 * size_t(tri[0]), *b = v + 3 * size_t(tri[1]),
                 *c = v + 3 * size_t(tri[2]);
    double e1[3] = {b[0] - o[0], b[1] - o[1], b[2] - o[2]};
    double e2[3] = {c[0] - o[0], c[1] - o[1], c[2] - o[2]};
    s[0] += e1[1] * e2[2] - e1[2] * e2[1];
    s[1] += e1[2] * e2[0] - e1[0] * e2[2];
    s[2] += e1[0] * e2[1] - e1[1] * e2[0];
  }
  double len = sqrt((s[0] * s[0] + s[1] * s[1]) + s[2] * s[2]);
  double *n = out + 3 * size_t(j);
  if (len > 0.0) {
    n[0] = s[0] / len;
    n[1] = s[1] / len;
    n[2] = s[2] / len;
  } else {
    n[0] = 0.0;
    n[1] = 0.0;
    n[2] = 1.0;
  }
}

// refine::select_candidates' predicate (refine.rs:161-178) per vertex: its
// nearest centroid within the radius (near, MISS when none) is a fracture
// face. Writes the flag and the vertex's own index (the select's input).
__global__ void k_fracture_flags(const uint32_t *near, const uint8_t *fracture, uint32_t nv,
                                 uint8_t *flags, uint32_t *lin) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  uint32_t j = near[i];
  flags[i] = (j != MISS && fracture[j]) ? 1 : 0;
  lin[i] = i;
}

// refine::cloud_from_indices (refine.rs:208-214): the selected vertices'
// points and normals, in selection order.
__global__ void k_gather_cloud(const double *v, const double *normals, const uint32_t *sel,
                               uint32_t m, double *points_out, double *normals_out) {
  uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  size_t i = sel[k];
  for (int a = 0; a < 3; ++a) {
    points_out[3 * size_t(k) + a] = v[3 * i + a];
    normals_out[3 * size_t(k) + a] = normals[3 * i + a];
  }
}

// ---- placement (types.rs:202-214) ---------------------------------------------

// Row r of the row-major pose: fma(t_r2, p2, fma(t_r1, p1, t_r0 p0)), plus
// t_r3 for a point; a normal (rotate_only) takes the rotation block alone.
__global__ void k_place_fused(const double *p, uint32_t n, Pose16 t, int rotate_only,
                              double *out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double *q = p + 3 * size_t(i);
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    double s = fma(t.m[4 * r + 2], q[2], fma(t.m[4 * r + 1], q[1], t.m[4 * r] * q[0]));
    out[3 * size_t(i) + r] = rotate_only ? s : s + t.m[4 * r + 3];
  }
}

// ---- the wide rung ------------------------------------------------------------------

struct WideState {
  double t[16];     // the pose of the next pass
  double fit, rmse; // the last pass's
  uint32_t pass;    // passes run so far in this rung
  uint32_t done;
  uint32_t ticket;  // blocks of the current pass that have written their sums
};

// Starts a rung at `init` (16 doubles on the device).
__global__ void k_wide_reset(WideState *s, const double *init) {
  if (threadIdx.x < 16) s->t[threadIdx.x] = init[threadIdx.x];
  if (threadIdx.x == 0) {
    s->fit = 0.0;
    s->rmse = 0.0;
    s->pass = 0;
    s->done = 0;
    s->ticket = 0;
  }
}

// icp::register's control after a pass (icp.rs:308-356), thread 0 of the last
// block, with the pass's sums in sh.sums: after the first pass only the
// initial fitness and rmse are kept; after pass p >= 1 the rung ends when both
// moved by less than 1e-6 or p reaches max_iter; otherwise the point-to-plane
// update of these sums moves the pose.
__device__ __noinline__ void wide_control(const double *sums, uint32_t ns, int max_iter,
                                          WideState *state, sherd_registration *out) {
  double fit, rmse;
  fit_rmse(sums, ns, fit, rmse);
  uint32_t pass = state->pass;
  bool converged = false, finish;
  if (pass == 0) {
    finish = max_iter <= 0;
  } else {
    converged = fabs(fit - state->fit) < 1e-6 && fabs(rmse - state->rmse) < 1e-6;
    finish = converged || int(pass) >= max_iter;
  }
  state->fit = fit;
  state->rmse = rmse;
  state->pass = pass + 1;
  if (finish) {
    for (int k = 0; k < 16; ++k) out->transform[k] = state->t[k];
    out->fitness = fit;
    out->inlier_rmse = rmse;
    out->correspondences = (unsigned long long)sums[0];
    out->iterations = pass;
    out->converged = converged ? 1u : 0u;
    state->done = 1;
    return;
  }
  double u[16];
  plane_update(sums, true, u);
  matmul4(u, state->t, state->t);
}

// One pass: block b over its slice [b chunk, (b + 1) chunk) of the source,
// its 29 sums written to partials[b]. The block that finishes last (a ticket
// taken after a fence) adds the slices' sums, each sum by one warp over the
// blocks in a fixed lane order and a fixed shuffle tree, so the total does not
// depend on which block came last, and runs the rung's control. Every block
// reads the state before it takes its ticket and only the last one writes it,
// so the state is the same for the whole pass. No block waits for another.
__global__ void __launch_bounds__(ICP_BLOCK, 4)
    k_wide_pass(const double4 *src, uint32_t ns, CloudView tgt, double distance, int max_iter,
                WideState *state, int *hints, uint32_t chunk, double *partials,
                sherd_registration *out, uint32_t *status) {
  __shared__ IcpShared sh;
  __shared__ uint32_t last;
  if (state->done) return;  // the same value for every block of the pass
  uint32_t st = 0;
  if (threadIdx.x < 16) sh.t[threadIdx.x] = state->t[threadIdx.x];
  __syncthreads();
  uint32_t lo = min(ns, blockIdx.x * chunk);
  uint32_t hi = min(ns, lo + chunk);
  icp_pass(src + lo, hi - lo, tgt, distance * distance, distance > 0.0, sh, hints + lo, st);
  if (st) atomicOr(status, st);
  if (threadIdx.x < ICP_SUMS) partials[size_t(blockIdx.x) * ICP_SUMS + threadIdx.x] = sh.sums[threadIdx.x];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&state->ticket, 1u) == gridDim.x - 1u;
  __syncthreads();
  if (!last) return;
  __threadfence();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = warp; k < ICP_SUMS; k += ICP_BLOCK / 32) {
    double v = 0.0;
    for (uint32_t b = lane; b < gridDim.x; b += 32u) v += __ldcg(partials + size_t(b) * ICP_SUMS + k);
    for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sh.sums[k] = v;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    state->ticket = 0;
    wide_control(sh.sums, ns, max_iter, state, out);
  }
}

}  // namespace sherd
