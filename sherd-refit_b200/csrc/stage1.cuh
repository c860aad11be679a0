// stage1.cuh — R 5.1's hypotheses on the device (matching/hypotheses.rs), in
// front of R 5.2's coarse score (k_coarse_scores).
//
// Every pair (i, j) of the two breakline subsets whose dihedrals are
// complementary, |dih_A + dih_B - 180| < tol, is a pose: B's frame laid onto
// A's, R = RA RB^T and tau = P_A - R P_B (hypotheses.rs:139-211). The pairs are
// tested one thread each over the row-major (i, j) grid and compacted in that
// order (np.where's order, which is what the fixture's hyp.pa / hyp.pb carry),
// then each kept pair's pose is written as a row-major 4x4 straight into the
// buffer the coarse score reads, so tens of thousands of poses never leave
// HBM between the two stages.
#pragma once

#include "kernels.cuh"

namespace sherd {

struct FramesView {
  const double *p, *ns, *f, *dih;
  uint32_t n;
};

// flags[e] for e = i n_ib + j: the dihedral test of hypotheses.rs:158-162,
// (dih_A + dih_B - 180).abs() < tol in the reference's order; lin[e] = e.
__global__ void k_hyp_flags(const double *dih_a, const uint32_t *ia, uint32_t n_ia,
                            const double *dih_b, const uint32_t *ib, uint32_t n_ib, double tol,
                            uint8_t *flags, uint32_t *lin) {
  uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_ia * n_ib) return;  // the host keeps n_ia n_ib below 2^31
  uint32_t i = e / n_ib, j = e - (e / n_ib) * n_ib;
  flags[e] = fabs(dih_a[ia[i]] + dih_b[ib[j]] - 180.0) < tol ? 1 : 0;
  lin[e] = e;
}

// The pose of each kept pair (hypotheses.rs:188-211): the tangent is ns x f in
// f64 (breakline.rs:180-182, 361-363); row i of R is
// ta_i (-tb) + nsa_i nsb + fa_i (-fb), each term in the reference's j = 0, 1, 2
// order, and tau_i = P_A,i - ((R_i0 P_B,0 + R_i1 P_B,1) + R_i2 P_B,2).
__global__ void k_hyp_poses(FramesView a, FramesView b, const uint32_t *ia, const uint32_t *ib,
                            uint32_t n_ib, const uint32_t *sel, uint32_t n, uint32_t *pa,
                            uint32_t *pb, double *poses) {
  uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= n) return;
  uint32_t e = sel[h];
  uint32_t i = e / n_ib, j = e - (e / n_ib) * n_ib;
  pa[h] = i;
  pb[h] = j;
  const size_t ka = 3 * size_t(ia[i]), kb = 3 * size_t(ib[j]);
  const double *nsa = a.ns + ka, *fa = a.f + ka, *nsb = b.ns + kb, *fb = b.f + kb;
  const double ta[3] = {nsa[1] * fa[2] - nsa[2] * fa[1], nsa[2] * fa[0] - nsa[0] * fa[2],
                        nsa[0] * fa[1] - nsa[1] * fa[0]};
  const double tb[3] = {nsb[1] * fb[2] - nsb[2] * fb[1], nsb[2] * fb[0] - nsb[0] * fb[2],
                        nsb[0] * fb[1] - nsb[1] * fb[0]};
  double r[3][3];
#pragma unroll
  for (int x = 0; x < 3; ++x)
#pragma unroll
    for (int k = 0; k < 3; ++k)
      r[x][k] = (ta[x] * -tb[k] + nsa[x] * nsb[k]) + fa[x] * -fb[k];
  const double *pa3 = a.p + ka, *pb3 = b.p + kb;
  double *t = poses + 16 * size_t(h);
#pragma unroll
  for (int x = 0; x < 3; ++x) {
    t[4 * x] = r[x][0];
    t[4 * x + 1] = r[x][1];
    t[4 * x + 2] = r[x][2];
    t[4 * x + 3] = pa3[x] - ((r[x][0] * pb3[0] + r[x][1] * pb3[1]) + r[x][2] * pb3[2]);
  }
  t[12] = 0.0;
  t[13] = 0.0;
  t[14] = 0.0;
  t[15] = 1.0;
}

}  // namespace sherd
