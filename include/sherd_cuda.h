/*
 * sherd_cuda.h — C ABI of the B200 geometry backend for sherd-refit.
 *
 * This is the drop-in boundary. It mirrors the reference's `Executor` trait
 * (crates/sherd-core/src/executor/mod.rs:105-137) method for method, adds the
 * `cone_cast` extension the trait's own documentation reserves for the
 * preprocessing rays (executor/mod.rs:9-10), and adds the batched
 * ladder + verification entry point that replaces the per-rung, per-candidate
 * call pattern of `Pair::stage2_batch` (matching/pair.rs:298-372).
 *
 * Conventions
 *  - Every entry point returns an int status: SHERD_OK (0) or a negative
 *    SHERD_E_* code. `sherd_last_error(ctx)` holds a message for the calling
 *    thread's last failure. There is no CPU fallback: a failure is reported,
 *    never answered on the host.
 *  - Host arrays are caller-owned and copied in (or written out) during the
 *    call. Device objects are opaque handles with explicit *_free calls.
 *  - 4x4 poses are 16 doubles, row-major, mapping the moving fragment's frame
 *    into the fixed one (the reference's `Matrix4<f64>`, written row by row).
 *  - Points are f64 triples (the reference's `[[f64; 3]]` batches); triangle
 *    meshes are f32 vertices (the reference's `RayScene` is f32,
 *    spatial/bvh.rs:43-50) and u32 faces.
 *  - A context is thread-safe: calls from several host threads serialise on
 *    an internal lock and run on the context's stream.
 */
#ifndef SHERD_CUDA_H
#define SHERD_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define SHERD_OK 0
#define SHERD_E_INVALID (-1)  /* bad argument (null, size, NaN pose, ...)  */
#define SHERD_E_OOM (-2)      /* device allocation failed                    */
#define SHERD_E_TIMEOUT (-3)  /* a kernel ran past the context's time budget */
#define SHERD_E_ABORTED (-4)  /* sherd_abort() was called during the call    */
#define SHERD_E_DEVICE (-5)   /* CUDA runtime error                          */
#define SHERD_E_EMPTY (-6)    /* a result needs data the input does not have */

/* ---- POD types shared with the host side ------------------------------- */

/* InsideOutcome (executor/batch.rs:339-368): 8 bytes, depth when inside. */
typedef struct sherd_inside_outcome {
    float depth;
    uint32_t inside;
} sherd_inside_outcome;

/* DistReduce (executor/batch.rs:270-281). */
enum { SHERD_REDUCE_ALL = 0, SHERD_REDUCE_MIN = 1 };

/* Estimation (matching/icp.rs:77-84). */
enum { SHERD_POINT_TO_POINT = 0, SHERD_POINT_TO_PLANE = 1 };

/* Options (matching/icp.rs:139-152), under the reference numerics. */
typedef struct sherd_icp_options {
    int32_t estimation;
    int32_t max_iteration;
    double max_correspondence_distance;
} sherd_icp_options;

/* Registration (matching/icp.rs:181-195). */
typedef struct sherd_registration {
    double transform[16];
    double fitness;
    double inlier_rmse;
    uint64_t correspondences;
    uint32_t iterations;
    uint32_t converged;
} sherd_registration;

/* Scales (matching/scales.rs:28-56), field for field. */
typedef struct sherd_scales {
    double t, res, coarse, stage1, tight, facing, gap, seam, near, pen, nms, icp;
} sherd_scales;

/* The five limits of R 6.5's accept rule (matching/verify.rs:632-638) and the
 * thresholds of Params (params.rs:141-190) that Scales::for_pair reads. */
typedef struct sherd_params {
    double min_tight, max_gap, max_pen, min_seam, min_cont_n;
    double coarse_delta, stage1_delta, tight_delta, facing_delta, seam_delta,
        near_delta, pen_delta, nms_delta, icp_delta;
    double coarse_res, stage1_res, tight_res, facing_res, gap_res, seam_res,
        near_res, pen_res, icp_res;
    /* R 5.6's early rejection (params.rs:78-80, pair.rs:315-340), 0 = off:
     * after the two pc_reg rungs an item whose fracture tight fraction is
     * below this keeps those scores (partial), skips the pc_frac rungs and
     * the rest of R 6, and is rejected. Its rungs[2] and rungs[3] are not
     * run: they hold the pose after rungs[1] with zero counts. */
    double early_reject_tight;
} sherd_params;

/* Scores (matching/verify.rs:72-135): the twenty numbers of R 6. */
typedef struct sherd_scores {
    double tight_a, tight_b, tight;
    double gap_a, gap_b, gap;
    double contact_a, contact_b, contact;
    double seam, gap_limit, tight_delta;
    double cont, cont_n;
    double pen, pen_depth;
    uint32_t pen_unavailable, partial;
    double brk, brk_best;
} sherd_scores;

/* One (pair, start) of the batched stage-2 path. */
typedef struct sherd_work_item {
    uint32_t pair;   /* index into the pairs array of the batch call   */
    uint32_t start;  /* caller's own id for the start, copied through  */
    double init[16]; /* stage-1 pose the 4-rung ladder starts from     */
} sherd_work_item;

/* What one work item produces: every rung's registration (the fixture
 * carries all four, s2.T_reg1..s2.T_frac2), the R 6 scores at the last
 * pose and the R 6.5 verdict. */
typedef struct sherd_candidate {
    uint32_t pair;
    uint32_t start;
    uint32_t accepted;
    uint32_t status; /* 0 ok; otherwise a SHERD_E_* code for this item   */
    sherd_registration rungs[4];
    sherd_scores scores;
} sherd_candidate;

/* Scheduling of sherd_ladder_verify_batch. */
enum {
    SHERD_SCHED_BATCHED = 0, /* every item in persistent kernels, one graph */
    SHERD_SCHED_PLAIN = 1    /* one launch sequence per pair, synchronised  */
};

/* ---- opaque handles ---------------------------------------------------- */
typedef struct sherd_ctx sherd_ctx;
typedef struct sherd_mesh sherd_mesh;         /* triangle LBVH, f32       */
typedef struct sherd_cloud sherd_cloud;       /* point LBVH, f64 + normals */
typedef struct sherd_surfaces sherd_surfaces; /* one fragment as R 6 reads it */
typedef struct sherd_pair sherd_pair;         /* two fragments + ladder clouds */
typedef struct sherd_batch sherd_batch;       /* a device-resident stage-2 batch */

/* ---- context ----------------------------------------------------------- */

/* Opens device `device` (cudaSetDevice) and creates a context with its own
 * stream. Replaces the reference's backend resolution of a GPU executor
 * (crates/sherd-backend/src/lib.rs:203-318): it fails instead of falling back,
 * as `--backend gpu` does (lib.rs:233-237). */
int sherd_open(int device, sherd_ctx **out);
int sherd_close(sherd_ctx *ctx);
/* Message of the calling thread's last failure on this context ("" if none). */
const char *sherd_last_error(const sherd_ctx *ctx);
/* Kernel time budget in milliseconds for the persistent kernels (0 = none).
 * A kernel past its budget stops taking work and the call returns
 * SHERD_E_TIMEOUT; no device wait is unbounded. */
int sherd_set_timeout_ms(sherd_ctx *ctx, uint32_t ms);
/* Sets the host-mapped abort flag the persistent kernels poll; the running
 * call returns SHERD_E_ABORTED. Cleared at the start of every batch call.
 * Mirrors the reference's cancellation flag (progress.rs:38-106). */
int sherd_abort(sherd_ctx *ctx);
/* A JSON object of per-method call counts, items and device milliseconds.
 * Mirrors the wgpu executor's Stats (sherd-gpu/src/executor.rs:50-216). */
int sherd_stats_json(sherd_ctx *ctx, char *buf, size_t len);
/* Executor::name (executor/mod.rs:107): "cuda". */
const char *sherd_name(void);
/* Executor::device_slack (executor/mod.rs:134-136). */
uint32_t sherd_device_slack(const sherd_ctx *ctx);

/* ---- meshes (RayScene, spatial/bvh.rs:36-192) -------------------------- */

/* Uploads a triangle mesh and builds its LBVH on the device.
 * RayScene::of_mesh (spatial/bvh.rs:56-62). nf == 0 is SHERD_E_EMPTY, as
 * RayScene refuses an empty mesh. */
int sherd_mesh_upload(sherd_ctx *ctx, const float *v, uint32_t nv,
                      const uint32_t *f, uint32_t nf, sherd_mesh **out);
/* The faces `keep[i] != 0` selects, on the same vertices, falling back to the
 * first face when nothing is selected. RayScene::of_subset (bvh.rs:71-78). */
int sherd_mesh_subset(sherd_ctx *ctx, const sherd_mesh *mesh,
                      const uint8_t *keep, sherd_mesh **out);
int sherd_mesh_free(sherd_mesh *mesh);
/* RayScene::aabb (bvh.rs:182-185) and RayScene::n_faces (bvh.rs:189-191). */
int sherd_mesh_aabb(const sherd_mesh *mesh, float lo[3], float hi[3]);
uint32_t sherd_mesh_faces(const sherd_mesh *mesh);

/* RayScene::first_hit (bvh.rs:84-90) for n rays: t in units of |dir|,
 * +inf and 0xFFFFFFFF on a miss. Tie rule: smallest t, then lowest face
 * index (face indices are those of the uploaded mesh, or of the subset). */
int sherd_first_hit(sherd_ctx *ctx, const sherd_mesh *mesh, const float *origins,
                    const float *dirs, uint32_t n, float *t_out, uint32_t *prim_out);

/* Executor::bounded_distance (executor/mod.rs:118, cpu.rs:84-113): points
 * moved by `pose` in f64, narrowed to f32, distance to the nearest triangle
 * when it is <= (float)max_dist, else +inf. REDUCE_MIN writes one value, the
 * minimum (the shrinking-window scan of cpu.rs:98-111). */
int sherd_bounded_distance(sherd_ctx *ctx, const sherd_mesh *mesh,
                           const double *points, uint32_t n, const double pose[16],
                           double max_dist, int reduce, double *out);

/* Executor::inside (executor/mod.rs:121, cpu.rs:115-128, bvh.rs:146-175):
 * AABB reject, then the majority of three axis-ray parities; depth is the
 * unbounded point-to-surface distance of an inside point. */
int sherd_inside(sherd_ctx *ctx, const sherd_mesh *mesh, const double *points,
                 uint32_t n, const double pose[16], sherd_inside_outcome *out);

/* verify::penetration_share (verify.rs:509-527), R 8's assembly question:
 * the share of the n points, moved by `pose`, that the parity test calls
 * inside `mesh` with a depth above `pen` (0 for n == 0). */
int sherd_penetration_share(sherd_ctx *ctx, const sherd_mesh *mesh, const double *points,
                            uint32_t n, const double pose[16], double pen, double *share);

/* ---- preprocessing rays: the cone_cast extension ----------------------- */

/* mesh::geometry::face_geometry (mesh/geometry.rs:70-96) in f64 on the
 * device: unit normals (floor 1e-12), areas and centroids. Outputs nf*3,
 * nf and nf*3 doubles; any output may be NULL. */
int sherd_face_geometry(sherd_ctx *ctx, const double *v, uint32_t nv,
                        const uint32_t *f, uint32_t nf, double *normals,
                        double *areas, double *centroids);

/* R 3.2 wall thickness (fragment/thickness.rs:99-162): one inward ray per
 * sampled face (stride ceil(nf / max_rays)), the 60-bin histogram mode over
 * [0, p90] and the looks-back filter. `found` is 0 when fewer than 100 rays
 * hit (the reference's signal for its OBB fallback). t_hit/prim (nullable,
 * ceil(nf/stride) entries) receive the raw hits. */
int sherd_thickness(sherd_ctx *ctx, const sherd_mesh *mesh, const double *centroids,
                    const double *normals, uint32_t nf, uint32_t max_rays,
                    float *t, float *thick_mode, uint32_t *found, float *t_hit,
                    uint32_t *prim);

/* R 3.2 from given hits (thickness.rs:139-162): the reference's injected
 * mode, fed a fixture's thick.idx / t_hit / prim. Runs on the device. */
int sherd_thickness_from_hits(sherd_ctx *ctx, const double *normals, uint32_t nf,
                              const uint32_t *idx, const float *t_hit,
                              const uint32_t *prim, uint32_t n, float *t,
                              float *thick_mode, uint32_t *found);

/* R 3.4.3 cone vote (fragment/segment.rs:318-376): seven rays per face round
 * -NS within 15 degrees; `good[i]` counts the rays that reach the far wall.
 * centroids/normals are the f64 face geometry, ns the smoothed normals,
 * hit_normals the normals the hit face is judged by. */
int sherd_cone_votes(sherd_ctx *ctx, const sherd_mesh *mesh, const double *centroids,
                     const double *normals, const double *ns,
                     const double *hit_normals, uint32_t nf, double thick,
                     uint8_t *good);

/* ---- point clouds (PointTree, spatial/kdtree.rs:31-258) ---------------- */

/* Uploads a point cloud (and optional unit normals) and builds its point
 * LBVH. np == 0 is SHERD_E_EMPTY, as PointTree::build refuses it. */
int sherd_cloud_upload(sherd_ctx *ctx, const double *points, const double *normals,
                       uint32_t np, sherd_cloud **out);
int sherd_cloud_free(sherd_cloud *cloud);
uint32_t sherd_cloud_points(const sherd_cloud *cloud);

/* PointTree::nearest_within_squared (kdtree.rs:202-217): nearest point with
 * d2 <= r2 (inclusive), lowest index on exact ties; miss = 0xFFFFFFFF, +inf. */
int sherd_nearest_within_sq(sherd_ctx *ctx, const sherd_cloud *cloud,
                            const double *queries, uint32_t n, double r2,
                            uint32_t *idx, double *d2);
/* PointTree::nearest_below (kdtree.rs:182-190): the unbounded nearest when
 * sqrt(d2) < bound, else a miss. The NN queries/s unit. */
int sherd_nearest_below(sherd_ctx *ctx, const sherd_cloud *cloud,
                        const double *queries, uint32_t n, double bound,
                        uint32_t *idx, double *dist);

/* Executor::coarse_scores (executor/mod.rs:110, cpu.rs:46-68,136-169): for
 * each of the k row-major 4x4 `poses` (Poses::Homogeneous; a Split batch
 * passes its rotations and translations as 4x4), the fraction of the n
 * `points` whose moved position has its nearest `target` point strictly
 * within `radius` (PointTree::nearest_below, ties to the lowest index) and
 * whose turned normal agrees with that point's normal (dot > normal_agree):
 * count / n, a division. `target` is A's breakline with its shell normals;
 * the reference's NearMask is a prefilter that moves no score and has no
 * counterpart here. n == 0 gives zeros. */
int sherd_coarse_scores(sherd_ctx *ctx, const sherd_cloud *target, const double *points,
                        const double *normals, uint32_t n, const double *poses, uint32_t k,
                        double radius, double normal_agree, double *out);

/* ---- ICP (matching/icp.rs:308-440) ------------------------------------- */

/* Executor::icp_rung (executor/mod.rs:114, cpu.rs:70-82): one
 * registration_icp per init, every candidate an independent rung, for both
 * estimations: point-to-plane (the target must carry normals; a target
 * without them leaves the pose unchanged, as icp.rs:414-416 does) and the
 * stage-1 point-to-point rung (Eigen's umeyama without scaling, icp.rs:
 * 527-592). */
int sherd_icp_rung(sherd_ctx *ctx, const double *source, uint32_t n_source,
                   const sherd_cloud *target, const double *inits, uint32_t k,
                   sherd_icp_options options, sherd_registration *out);

/* For callers that cannot allocate device memory during a run: a worker held
 * to a fixed device-memory budget set up front, or code that must not call
 * cudaMalloc/cudaFree while other streams are in flight (both can block or
 * synchronise the whole device). No counterpart in the reference.
 *
 * The same rung as sherd_icp_rung (point-to-plane or point-to-point), with
 * every buffer already on the device: `source` holds n_source points as 4
 * doubles each (x, y, z, unused; 16-byte aligned), `inits` k row-major 4x4
 * poses, `out` room for k registrations (both 8-byte aligned). Each buffer
 * must be device memory of the context's GPU (or managed memory): a host
 * pointer or a misaligned one is refused with SHERD_E_INVALID before anything
 * is launched. The poses are read on the device only, so a non-finite one is
 * not refused up front: its rung finds no correspondence and the call returns
 * SHERD_E_INVALID after it ran; pass finite poses.
 * The per-point working memory (each source point's last match) lives in one
 * array inside this library, sized at SHERD_NOALLOC_CAPACITY entries and held
 * by every GPU that loads the library until the process exits; a call with
 * k * n_source above it is refused with SHERD_E_INVALID. The call allocates
 * nothing, waits for its own work, and leaves the array holding the last
 * call's contents (each rung resets the part it uses before reading it). All
 * calls share the one array, so two calls that overlap on the GPU (from two
 * contexts, or two host threads on different contexts of one device) race.
 * The first call on each device looks the array's device address up
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture on the device. */
#define SHERD_NOALLOC_CAPACITY (1u << 20)
int sherd_icp_rung_noalloc(sherd_ctx *ctx, const double *source, uint32_t n_source,
                           const sherd_cloud *target, const double *inits, uint32_t k,
                           sherd_icp_options options, sherd_registration *out);

/* ---- verification (matching/verify.rs) ---------------------------------- */

/* Surfaces (verify.rs:223-299): one fragment as R 6 reads it. `fracture` is
 * the fracture-face scene, `mesh` the whole working mesh (NULL leaves the
 * penetration test unavailable). Points are copied to the device. */
int sherd_surfaces_create(sherd_ctx *ctx, const sherd_mesh *fracture,
                          const sherd_mesh *mesh, uint32_t watertight,
                          double frac_area, const double *pf, uint32_t n_pf,
                          const double *s, uint32_t n_s, const double *brk_p,
                          const double *brk_ns, uint32_t n_brk,
                          const double *margin_p, const double *margin_n,
                          uint32_t n_margin, sherd_surfaces **out);
int sherd_surfaces_free(sherd_surfaces *s);

/* verify::verify (verify.rs:590-626) for one pose, every score on the device.
 * full = 0 computes only the fracture scores and the seam (partial = 1). */
int sherd_verify(sherd_ctx *ctx, const sherd_surfaces *a, const sherd_surfaces *b,
                 const double pose[16], const sherd_scales *sc, int full,
                 sherd_scores *out);

/* Scales::for_pair (scales.rs:72-88). Pure host arithmetic. */
int sherd_scales_for_pair(const sherd_params *p, double t, double res,
                          sherd_scales *out);
/* Params::default (params.rs:141-190), the thresholds this ABI reads. */
void sherd_params_default(sherd_params *out);
/* verify::accept (verify.rs:632-638). */
uint32_t sherd_accept(const sherd_scores *s, const sherd_params *p,
                      const sherd_scales *sc);

/* ---- the batched stage-2 path ------------------------------------------ */

/* A pair as Pair::stage2_batch reads it (pair.rs:298-372, 592-630): A's two
 * ICP targets (pc_reg, pc_frac, with normals), B's two moving clouds, both
 * fragments' Surfaces and the pair's Scales. */
int sherd_pair_create(sherd_ctx *ctx, const sherd_surfaces *a, const sherd_surfaces *b,
                      const sherd_cloud *reg_target, const sherd_cloud *frac_target,
                      const double *reg_source, uint32_t n_reg,
                      const double *frac_source, uint32_t n_frac,
                      const sherd_scales *sc, sherd_pair **out);
int sherd_pair_free(sherd_pair *pair);

/* R 5.6 + R 6 + R 6.5 for every (pair, start): the four point-to-plane rungs
 * (0.2 t, 0.08 t on pc_reg; 0.08 t, 0.04 t on pc_frac; 30 iterations each,
 * ladder.rs:51-61, 142-161), the full verification at the last pose and the
 * verdict. SHERD_SCHED_BATCHED runs every item in persistent kernels fed by
 * device work queues, one captured CUDA graph per stage (ladder, fracture/seam/
 * continuity scores, penetration inside tests, penetration minimum distances,
 * verdicts); SHERD_SCHED_PLAIN launches the ladder and verification kernels
 * once per pair and synchronises between pairs. */
int sherd_ladder_verify_batch(sherd_ctx *ctx, sherd_pair *const *pairs,
                              uint32_t n_pairs, const sherd_work_item *items,
                              uint32_t n_items, const sherd_params *p, int sched,
                              sherd_candidate *out);

/* A stage-2 batch made resident on the device: the pair views, work items,
 * queue order, candidate records and per-CTA scratch are uploaded and sized
 * once, and SHERD_SCHED_BATCHED captures each stage (queue resets and its
 * persistent kernels) as a CUDA graph, five in all. Running it
 * again recomputes every candidate from the same resident inputs. This is the
 * device-side form of sherd_ladder_verify_batch, for callers that keep their
 * inputs on the GPU between calls. */
int sherd_batch_create(sherd_ctx *ctx, sherd_pair *const *pairs, uint32_t n_pairs,
                       const sherd_work_item *items, uint32_t n_items,
                       const sherd_params *p, int sched, sherd_batch **out);
/* Launches the batch and waits for it. `ms` (nullable) receives the device
 * milliseconds of each stage, CUDA events on the context's stream:
 * [0] ladder, [1] fracture/seam/continuity verification, [2] penetration
 * box/parity/depth pass, [3] penetration minimum pass, [4] finalising pass,
 * [5] the whole run. Under SHERD_SCHED_PLAIN only [5] is measured (the
 * others are -1). */
#define SHERD_BATCH_TIMES 6
int sherd_batch_run(sherd_batch *batch, float ms[SHERD_BATCH_TIMES]);
/* Copies the candidates of the last run to the host (n_items records). */
int sherd_batch_results(sherd_batch *batch, sherd_candidate *out);
int sherd_batch_free(sherd_batch *batch);

/* ---- segmentation: R 3.4 end to end (fragment/segment.rs:511-631) ------- */

/* SegParams (segment.rs:86-118); sherd_seg_params_default gives the shipped values. */
typedef struct sherd_seg_params {
    double smooth_res;             /* smoothing radius max(t/3, smooth_res * res)       */
    double coarse_at;              /* coarse mesh: res > coarse_at * t                   */
    double boundary_angle;         /* shell growth limit, degrees                        */
    uint32_t votes;                /* cone rays of seven that must reach the far wall   */
    uint32_t votes_coarse;         /* ... on a coarse mesh                               */
    uint32_t smoothed_hit_normal;  /* judge the hit face by its smoothed normal          */
    uint32_t boundary_angle_auto;  /* max(angle, median shell normal noise + 15 deg)     */
} sherd_seg_params;

/* What Segmentation reports besides the labels (segment.rs:121-141); the
 * area fractions are the caller's, a pairwise sum of the areas under the
 * labels (segment.rs:645-648). */
typedef struct sherd_seg_info {
    uint32_t votes;         /* the vote count this mesh's resolution asked for */
    uint32_t n_rep;         /* voxel representatives                           */
    double smooth_radius;   /* max(t/3, smooth_res * res)                      */
    double boundary_angle;  /* the growth angle used, degrees                  */
} sherd_seg_info;

/* SegTrace (segment.rs:143-166): every intermediate array, each nullable.
 * rep holds n_rep entries (at most nf), ns 3 doubles per face, the rest one
 * entry per face. */
typedef struct sherd_seg_trace {
    uint32_t *rep, *near;
    double *ns;
    uint8_t *good, *frac_raw, *frac_majority, *frac_islands, *has_ref;
} sherd_seg_trace;

void sherd_seg_params_default(sherd_seg_params *out);

/* segment::segment_faces (segment.rs:476-631): shell/fracture labels
 * (1 = fracture) of the working mesh `v` (f64, nv) / `f` (nf), whose ray
 * scene `mesh` was uploaded from the same faces; `thick` is R 3.2's wall and
 * `res` the median edge. Every step runs on the device: voxel representatives
 * (lowest face per t/8 voxel, ascending), each face's nearest representative,
 * the smoothed normals, the seven-ray cone vote, the majority filter, the
 * island removals over the face adjacency, the shell reference normals and the
 * boundary growth. Radius balls are inclusive and summed in ascending face
 * order, component areas in face order, as the reference does, so the labels
 * are bit-exact to a sequential restatement. */
int sherd_segment(sherd_ctx *ctx, const sherd_mesh *mesh, const double *v, uint32_t nv,
                  const uint32_t *f, uint32_t nf, double thick, double res,
                  const sherd_seg_params *sp, uint8_t *labels, sherd_seg_info *info,
                  const sherd_seg_trace *trace);

/* ---- differentiation: the adjoint of two group-alignment objectives ----- */

/* Options of sherd_adjoint. No counterpart in the reference: the objectives
 * are built from R 6's tight fraction (verify.rs:338-349) and the ICP's
 * point-to-plane residual (icp.rs:361-392, 599-640). */
typedef struct sherd_adjoint_options {
    double radius_k; /* correspondence radius in units of t * Scales::icp (0.04: the last rung) */
    double width_k;  /* sigmoid width w in units of t (0.01)                               */
    double window_k; /* distances beyond facing + window_k * w are left out (30)           */
} sherd_adjoint_options;
#define SHERD_ADJOINT_VALUES 5

/* For every group pose g and edge e (a pair: A fixed, B moving, its Scales):
 * values[(g * n_edges + e) * 5 + k], k =
 *   0  E   = 1/2 sum r^2, r = (T x - q) . n over B's fracture samples x whose
 *          nearest A fracture sample q is strictly within the radius;
 *   1  T_B = sum sigmoid((tight - d) / w), 2 F_B = sum sigmoid((facing - d) / w)
 *          over B's fracture samples moved by T, d = sqrt(dist^2 + (w/10)^2)
 *          their softened distance to A's fracture faces; T_B / F_B is R 6's
 *          tight fraction, smoothed;
 *   3  T_A, 4 F_A the same for A's samples moved by T^-1 against B's faces;
 * and grads[((g * n_edges + e) * 5 + k) * 6 + j] = d values[k] / d xi_j, xi =
 * (w, v) the left twist of the pose that moves the points, expressed in the
 * fixed fragment's frame: T -> exp(xi^) T for k = 0, 1, 2 (A's frame) and
 * T^-1 -> exp(xi^) T^-1 for k = 3, 4 (B's frame). For k = 0 it is the ICP's
 * J^T r (icp.rs:616-624). Matches and nearest faces are held fixed (exact
 * gradients of a piecewise-smooth objective); the distance to the assigned
 * face is f64. `poses` and `inverses` are n_poses * n_edges row-major 4x4 T
 * and T^-1. Nothing is stored between calls. */
int sherd_adjoint(sherd_ctx *ctx, sherd_pair *const *edges, uint32_t n_edges,
                  const double *poses, const double *inverses, uint32_t n_poses,
                  const sherd_adjoint_options *opt, double *values, double *grads);

/* ---- io::load_mesh (io/mod.rs:114-137, io/ply.rs, mesh/clean.rs) -------- */

/* A mesh read from a file, in host memory. */
typedef struct sherd_host_mesh sherd_host_mesh;

/* Reads a PLY file (ASCII, binary little- or big-endian; any numeric property
 * types; x, y, z widened to f64; the vertex_indices or vertex_index list,
 * polygons as the fan (i0, i_{k-1}, i_k), faces under three corners dropped;
 * other elements and properties read past) and cleans it as mesh/clean.rs:
 * 138-142: duplicate vertices merged onto their first occurrence (+0 = -0, NaN
 * never equal), faces with a repeated corner dropped, unreferenced vertices
 * removed. *nv, *nf receive the sizes; SHERD_E_EMPTY when no triangle is
 * left, SHERD_E_INVALID on a malformed file (message in
 * sherd_last_error(NULL)). Host code, no device. */
int sherd_mesh_read(const char *path, sherd_host_mesh **out, uint32_t *nv, uint32_t *nf);
/* Copies the mesh out: v receives 3 nv doubles, f 3 nf indices. */
int sherd_host_mesh_copy(const sherd_host_mesh *m, double *v, uint32_t *f);
int sherd_host_mesh_free(sherd_host_mesh *m);

/* ---- R 3.5.3-3.5.5: breaklines and their frames (fragment/breakline.rs) --- */

/* breakline::build (breakline.rs:207-300) in f64 on one labelled working mesh
 * (v: nv xyz f64; f: nf faces; frac: 1 for a fracture face): the midpoints of
 * the edges whose two faces differ in label, in the face adjacency's
 * ascending edge-key order; the shell (ns) and fracture (nf) macro normals,
 * area-weighted ball normals over the mask's faces between macro_inner t and
 * macro_outer t of the point (the whole macro_outer ball where that is empty
 * or gives a normal shorter than 0.5; zero where the mask has no face); the
 * frame f = nf - (nf . ns) ns normalised; valid = |ns|, |nf|, |ns x f| > 0.5;
 * the dihedral acos(ns . nf) in degrees; and the hypothesis subset `sub`, the
 * valid lowest-index representatives of the brk_voxel t voxels, ascending.
 * Outputs: *count points, and when capacity >= *count: p, ns, nf, f (xyz
 * each), dih, valid, sub (room for *count; *n_sub written). capacity = 0
 * asks for the count alone; a non-zero capacity below it is refused. Points,
 * normals, frames, validity and subset are bit-identical to the sequential
 * restatement (ball sums in ascending face order); dih to the device acos. */
int sherd_breaklines(sherd_ctx *ctx, const double *v, uint32_t nv, const uint32_t *f, uint32_t nf,
                     const uint8_t *frac, double t, double macro_inner, double macro_outer,
                     double brk_voxel, uint32_t capacity, double *p, double *ns, double *nfr,
                     double *fr, double *dih, uint8_t *valid, uint32_t *sub, uint32_t *n_sub,
                     uint32_t *count);

/* ---- stage 1: hypotheses, coarse score, suppression (R 5.1-5.5) --------- */

/* One fragment's breakline as R 5 reads it (hypotheses.rs:53-82): n points
 * p, shell macro-normals ns and in-plane axes f (xyz f64 each; the tangent is
 * ns x f, formed here in f64), and the dihedral of each point in degrees. */
typedef struct sherd_frames {
    const double *p;
    const double *ns;
    const double *f;
    const double *dih;
    uint32_t n;
} sherd_frames;

/* R 5.1 and R 5.2 in one call (hypotheses.rs:149-211, coarse.rs:113-133):
 * every (i, j) of the subsets ia (positions into a's points) and ib with
 * |dih_a[ia[i]] + dih_b[ib[j]] - 180| < dihedral_tol, in row-major (i, j)
 * order; its pose R = RA RB^T, tau = P_A - R P_B (RA = [t | ns | f] at ia[i],
 * RB = [-t | ns | -f] at ib[j]); and its coarse score against `target` (A's
 * whole breakline with its shell normals): the fraction of the probe (q, qn:
 * n_probe points of B and their shell normals) within `delta` of the target
 * after the pose, with the matched normal . R qn > normal_agree. The poses stay
 * on the device between the two stages. Outputs: *count, and when capacity >=
 * *count, pa[h], pb[h] (positions into ia and ib), poses[16 h..] (row-major
 * 4x4) and scores[h]. capacity = 0 asks for the count alone; a non-zero
 * capacity below the count is refused (SHERD_E_INVALID, *count set). n_ia n_ib
 * must stay below 2^31. Poses and scores are bit-identical to the reference's
 * sequential restatement. */
int sherd_hypotheses_coarse(sherd_ctx *ctx, const sherd_frames *a, const sherd_frames *b,
                            const uint32_t *ia, uint32_t n_ia, const uint32_t *ib, uint32_t n_ib,
                            double dihedral_tol, const sherd_cloud *target, const double *q,
                            const double *qn, uint32_t n_probe, double delta,
                            double normal_agree, uint32_t capacity, uint32_t *pa, uint32_t *pb,
                            double *poses, double *scores, uint32_t *count);

/* nms::order_by_score (nms.rs:46-59): the indices 0..n-1 by descending score
 * (f64 total order), ties by ascending index, the first `limit` of them.
 * `order` has room for min(n, limit); *n_order receives that count. Host code,
 * no device. */
int sherd_order_by_score(const double *score, uint32_t n, uint32_t limit, uint32_t *order,
                         uint32_t *n_order);

/* nms::nms (nms.rs:61-86), R 5.3 and R 5.5's greedy suppression: walk
 * `order`; stop at the first score below `floor`; keep a pose unless a kept one
 * is nearer than trans_tol in translation and trace(R^T R') > 2.9; stop once
 * `topk` are kept (tested after keeping, so topk = 0 keeps one). `poses` holds
 * n_poses row-major 4x4 poses that order indexes. `kept` has room for
 * min(n_order, max(topk, 1)); *n_kept receives the count. Host code. */
int sherd_nms(const uint32_t *order, uint32_t n_order, const double *poses, const double *score,
              uint32_t n_poses, double trans_tol, uint32_t topk, double floor, uint32_t *kept,
              uint32_t *n_kept);

/* ---- R 9: full-resolution join refinement (refine.rs) ------------------- */

/* refine::vertex_normals (refine.rs:121-151), Open3D's ComputeVertexNormals:
 * every face's unnormalised normal (v1 - v0) x (v2 - v0) added to its three
 * vertices, each vertex's sum taken in ascending face order, then one
 * normalisation; a vertex whose sum is zero (or not a number) gets (0, 0, 1).
 * Bit-identical to the reference's sequential loop. `normals` receives nv
 * f64 triples. 3 * nf must stay below 2^31. */
int sherd_vertex_normals(sherd_ctx *ctx, const double *v, uint32_t nv, const uint32_t *f,
                         uint32_t nf, double *normals);

/* refine::fracture_cloud (refine.rs:217-227) up to the cap, in one call, so
 * the mesh crosses to the device once and only the chosen vertices come back:
 * the vertices of the original mesh (v, f) whose nearest working-mesh face
 * centroid (refine::select_candidates, refine.rs:161-178: PointTree::
 * nearest_below, strictly within `radius` = max(0.15 t, 1.5 res)) is a
 * fracture face (`fracture`, one flag per centroid), in ascending order, with
 * their points and their refine::vertex_normals. Writes min(count, cap)
 * indices, points and normals (f64 triples); *n_out = count, the number
 * selected (above `cap`, call again with a larger cap). The same values as
 * sherd_nearest_below over a cloud of the centroids and
 * sherd_vertex_normals. refine::cap_selection's draw stays with the caller. */
int sherd_fracture_cloud(sherd_ctx *ctx, const double *v, uint32_t nv, const uint32_t *f,
                         uint32_t nf, const double *centroids, const uint8_t *fracture,
                         uint32_t n_cent, double radius, uint32_t cap, uint32_t *idx_out,
                         double *points_out, double *normals_out, uint32_t *n_out);

/* refine::refine_one (refine.rs:334-386) for one join: the moving fragment's
 * cloud `source` (n_source points) placed by pose_moving, the fixed one's
 * `target` and `target_normals` (n_target) placed by pose_fixed, both as
 * types::apply_transform_fused / rotate_fused place them (types.rs:202-214,
 * bit-identical); then two point-to-plane registration_icp rungs from the
 * identity, at distances dist[0] and dist[1], max_iteration each, the second
 * starting from the first's pose. out[0], out[1] receive the two rungs
 * (transform = the correction in the fixed fragment's world frame; the caller
 * applies out[1].transform to pose_moving). Each pass is spread over the
 * whole device, a slice of the source per block, its sums added in block
 * order (reproducible run to run). An empty cloud on either side leaves both
 * rungs at the identity with no correspondence. */
int sherd_refine_join(sherd_ctx *ctx, const double *source, uint32_t n_source,
                      const double *target, const double *target_normals, uint32_t n_target,
                      const double pose_fixed[16], const double pose_moving[16],
                      const double dist[2], int32_t max_iteration, sherd_registration out[2]);

#ifdef __cplusplus
}
#endif
#endif /* SHERD_CUDA_H */
