// sherd.cu — the C ABI of the B200 geometry backend (include/sherd_cuda.h).
//
// One translation unit: the device code lives in the headers it includes.
// Host responsibilities: the context (device, stream, lock, status word,
// host-mapped abort flag, statistics), device handles for meshes, clouds,
// surfaces and pairs (each built on the device: LBVHs, sorted primitives),
// argument checking, and the launch sequences. No entry point computes a
// result on the host; a CUDA failure is an error status, never a fallback.

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "kernels.cuh"
#include "adjoint.cuh"
#include "segment.cuh"
#include "refine.cuh"
#include "stage1.cuh"
#include "preprocess.cuh"
#include "meshio.h"

using namespace sherd;

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------

struct MethodStats {
  uint64_t calls = 0, items = 0;
  double ms = 0.0;
};

struct sherd_ctx {
  int device = 0;
  int sm_count = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::mutex mu;
  uint32_t timeout_ms = 0;
  uint32_t *abort_host = nullptr;  // pinned, mapped
  uint32_t *abort_dev = nullptr;
  uint32_t *d_status = nullptr;
  std::map<std::string, MethodStats> stats;
  // Two more streams and their events, to run the ladder's point-count buckets
  // side by side inside the captured ladder graph.
  cudaStream_t side[2] = {nullptr, nullptr};
  cudaEvent_t fork_ev = nullptr, join_ev[2] = {nullptr, nullptr};
  // The ladder autotuner's choices on this context's device: per point-count
  // bucket the k_ladder variant (-1 until tuned), the timings it was chosen
  // from and the sample they were taken on.
  int ladder_tuned[3] = {-1, -1, -1};
  float ladder_tune_ms[3][3] = {};
  uint32_t ladder_tune_items[3] = {};
  // Device buffers the entry points allocate (stream-ordered, on `stream`).
  cudaMemPool_t pool = nullptr;
};

// The context an entry point allocates its device buffers from (its pool, on
// its stream), for as long as the entry point holds it (CtxLock); null
// otherwise, and while a stage graph is being captured.
thread_local sherd_ctx *t_alloc_ctx = nullptr;
constexpr uint64_t POOL_KEEP_BYTES = uint64_t(4) << 30;

// An entry point's hold on its context: the context's lock, and its stream as
// the stream device buffers are allocated and freed on (stream-ordered).
struct CtxLock {
  std::lock_guard<std::mutex> guard;
  sherd_ctx *prev;
  explicit CtxLock(sherd_ctx *c) : guard(c->mu), prev(t_alloc_ctx) { t_alloc_ctx = c; }
  ~CtxLock() { t_alloc_ctx = prev; }
};

// Working memory of sherd_icp_rung_noalloc: each source point's last match, for
// every candidate of one call. A file-scope device array, so that entry point
// never allocates; every GPU that loads the library holds it until exit.
static __device__ __align__(256) int g_noalloc_hints[SHERD_NOALLOC_CAPACITY];

namespace {

thread_local std::map<const sherd_ctx *, std::string> t_errors;

// The device address of g_noalloc_hints, looked up once per device with that
// device current (host code cannot use the symbol itself as an address).
std::mutex g_symbol_mu;
std::map<int, int *> g_noalloc_address;

cudaError_t noalloc_address(int device, int **out) {
  std::lock_guard<std::mutex> lock(g_symbol_mu);
  auto it = g_noalloc_address.find(device);
  if (it != g_noalloc_address.end()) {
    *out = it->second;
    return cudaSuccess;
  }
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_hints);
  if (e != cudaSuccess) return e;
  g_noalloc_address[device] = static_cast<int *>(p);
  *out = static_cast<int *>(p);
  return cudaSuccess;
}

// An NVTX range over one host-side scope (the enqueue of a stage or an entry
// point), for nsys / ncu --nvtx; a no-op unless a tool is attached.
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

int fail(const sherd_ctx *ctx, int code, const std::string &msg) {
  t_errors[ctx] = msg;
  return code;
}

int cuda_fail(const sherd_ctx *ctx, cudaError_t e, const char *what) {
  int code = e == cudaErrorMemoryAllocation ? SHERD_E_OOM : SHERD_E_DEVICE;
  cudaGetLastError();
  return fail(ctx, code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                          \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
  } while (0)

template <typename T>
struct DBuf {  // owning device buffer
  T *p = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;  // the stream it came from the context's pool on
  DBuf() = default;
  DBuf(const DBuf &) = delete;
  DBuf &operator=(const DBuf &) = delete;
  ~DBuf() { reset(); }
  // Allocated inside an entry point, a buffer comes from the context's pool on
  // the context's stream and goes back on that stream: the free is ordered
  // after the work queued before it, and neither call waits for the device.
  // Allocated anywhere else, the plain synchronous calls.
  void reset() {
    if (p) {
      if (s)
        cudaFreeAsync(p, s);
      else
        cudaFree(p);
    }
    p = nullptr;
    n = 0;
    s = nullptr;
  }
  cudaError_t alloc(size_t count) {
    reset();
    n = count;
    if (!count) return cudaSuccess;
    if (sherd_ctx *c = t_alloc_ctx) {
      cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&p), count * sizeof(T), c->pool,
                                              c->stream);
      if (e == cudaSuccess) s = c->stream;
      return e;
    }
    return cudaMalloc(&p, count * sizeof(T));
  }
};

unsigned blocks_for(size_t n, int threads = 256) {
  size_t b = (n + threads - 1) / threads;
  return unsigned(std::max<size_t>(1, std::min<size_t>(b, 1u << 30)));
}

bool finite_pose(const double *t) {
  if (!t) return false;
  for (int i = 0; i < 16; ++i)
    if (!std::isfinite(t[i])) return false;
  return true;
}

Pose16 pose_of(const double *t) {
  Pose16 p;
  std::memcpy(p.m, t, sizeof p.m);
  return p;
}

// Runs the status check after a launch sequence: synchronises the stream and
// turns the kernels' status bits into an error code.
int finish(sherd_ctx *ctx, const char *method, size_t items, bool timed) {
  CK(cudaEventRecord(ctx->ev1, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  CK(cudaGetLastError());
  uint32_t st = 0;
  CK(cudaMemcpy(&st, ctx->d_status, 4, cudaMemcpyDeviceToHost));
  MethodStats &m = ctx->stats[method];
  m.calls += 1;
  m.items += items;
  if (timed) {
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) == cudaSuccess) m.ms += ms;
  }
  if (st & ST_ABORTED) return fail(ctx, SHERD_E_ABORTED, std::string(method) + ": aborted");
  if (st & ST_TIMEOUT) return fail(ctx, SHERD_E_TIMEOUT, std::string(method) + ": time budget spent");
  if (st & ST_RANGE)
    return fail(ctx, SHERD_E_INVALID, std::string(method) + ": input outside the supported range");
  if (st & ST_STACK) return fail(ctx, SHERD_E_DEVICE, std::string(method) + ": traversal stack overflow");
  if (st & ST_SCRATCH) return fail(ctx, SHERD_E_INVALID, std::string(method) + ": scratch too small");
  return SHERD_OK;
}

int begin(sherd_ctx *ctx) {
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemsetAsync(ctx->d_status, 0, 4, ctx->stream));
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  return SHERD_OK;
}

template <typename T>
int upload(sherd_ctx *ctx, DBuf<T> &buf, const T *host, size_t n) {
  CK(buf.alloc(n));
  if (n) CK(cudaMemcpyAsync(buf.p, host, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  return SHERD_OK;
}

// Checks of inputs already on the device, in place of host loops over them:
// each call of coords/indices adds one launch into `slot`, read() waits for
// them and hands back what they found.
struct DevInputCheck {
  DBuf<InputCheck> d;
  int open(sherd_ctx *ctx, int slots) {
    CK(d.alloc(slots));
    CK(cudaMemsetAsync(d.p, 0, sizeof(InputCheck) * slots, ctx->stream));
    return SHERD_OK;
  }
  int coords(sherd_ctx *ctx, int slot, const double *p, size_t n) {
    if (!n) return SHERD_OK;
    k_check_coords<<<std::min(blocks_for(n), unsigned(ctx->sm_count) * 8u), 256, 0, ctx->stream>>>(
        p, n, d.p + slot);
    CK(cudaGetLastError());
    return SHERD_OK;
  }
  int indices(sherd_ctx *ctx, int slot, const uint32_t *f, size_t n, uint32_t limit) {
    if (!n) return SHERD_OK;
    k_check_indices<<<std::min(blocks_for(n), unsigned(ctx->sm_count) * 8u), 256, 0, ctx->stream>>>(
        f, n, limit, d.p + slot);
    CK(cudaGetLastError());
    return SHERD_OK;
  }
  int read(sherd_ctx *ctx, InputCheck *h) {
    CK(cudaMemcpyAsync(h, d.p, sizeof(InputCheck) * d.n, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    return SHERD_OK;
  }
};

// The largest finite magnitude a coordinate check saw, at least 1.
double checked_mag(const InputCheck &c) {
  double m;
  std::memcpy(&m, &c.max_abs, 8);
  return std::max(1.0, m);
}

}  // namespace

// ---------------------------------------------------------------------------
// handles
// ---------------------------------------------------------------------------

struct sherd_mesh {
  sherd_ctx *ctx = nullptr;
  std::vector<float> hv;     // host copy of the vertices (subsets reuse them)
  std::vector<uint32_t> hf;  // host copy of the faces
  DBuf<BNode> nodes;
  DBuf<float4> tri;
  DBuf<uint32_t> gstart[3];
  DBuf<float4> grect[3], gtri[3];
  DBuf<float> lb;            // the bound grid's cells
  MeshView view{};
};

struct sherd_cloud {
  sherd_ctx *ctx = nullptr;
  DBuf<BNode> nodes;
  DBuf<WNode> wide;  // the 4-wide form of nodes, for the nearest-point search
  DBuf<double4> pts, nrm;
  CloudView view{};
};

struct sherd_surfaces {
  sherd_ctx *ctx = nullptr;
  const sherd_mesh *fracture = nullptr, *mesh = nullptr;
  std::vector<double> brk_p_host;
  DBuf<double> brk_p, brk_ns, margin_p, margin_n;
  sherd_cloud pf_sorted, s_sorted, brk_tree, margin_tree;
  bool has_brk_tree = false, has_margin_tree = false;
  SurfView view{};
};

struct sherd_pair {
  sherd_ctx *ctx = nullptr;
  const sherd_surfaces *a = nullptr, *b = nullptr;
  sherd_cloud reg_src, frac_src;
  DBuf<uint32_t> a_cell;
  PairView view{};
};

namespace {

// Builds the LBVH over f32 triangles (TRI) or f64 points (!TRI) already on the
// device; fills nodes, the sorted slot order and the root description.
template <bool TRI>
int build_lbvh(sherd_ctx *ctx, const float *d_v, uint32_t nv, const uint32_t *d_f, const double *d_p,
               uint32_t n, float pad, int leaf_max, DBuf<BNode> &nodes, DBuf<uint32_t> &sorted,
               float lo[3], float hi[3]) {
  cudaStream_t s = ctx->stream;
  DBuf<unsigned> bounds;
  CK(bounds.alloc(6));
  unsigned init[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
  CK(cudaMemcpyAsync(bounds.p, init, sizeof init, cudaMemcpyHostToDevice, s));
  if (TRI)
    k_bounds_f32<<<std::min(blocks_for(nv), 1024u), 256, 0, s>>>(d_v, nv, bounds.p);
  else
    k_bounds_f64<<<std::min(blocks_for(n), 1024u), 256, 0, s>>>(d_p, n, bounds.p);
  CK(cudaGetLastError());
  unsigned hb[6];
  CK(cudaMemcpyAsync(hb, bounds.p, sizeof hb, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  BuildBox box;
  for (int k = 0; k < 3; ++k) {
    lo[k] = fordinv(hb[k]);
    hi[k] = fordinv(hb[3 + k]);
    box.lo[k] = lo[k];
    double ext = double(hi[k]) - double(lo[k]);
    box.inv[k] = ext > 0.0 ? 1.0 / ext : 0.0;
  }
  DBuf<unsigned long long> keys, keys2;
  DBuf<uint32_t> vals;
  CK(keys.alloc(n));
  CK(keys2.alloc(n));
  CK(vals.alloc(n));
  CK(sorted.alloc(n));
  if (TRI)
    k_morton_tri<<<blocks_for(n), 256, 0, s>>>(d_v, d_f, n, box, keys.p, vals.p);
  else
    k_morton_pts<<<blocks_for(n), 256, 0, s>>>(d_p, n, box, keys.p, vals.p);
  CK(cudaGetLastError());
  size_t temp_bytes = 0;
  CK(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, keys.p, keys2.p, vals.p, sorted.p,
                                     int(n), 0, 63, s));
  DBuf<unsigned char> temp;
  CK(temp.alloc(temp_bytes));
  CK(cub::DeviceRadixSort::SortPairs(temp.p, temp_bytes, keys.p, keys2.p, vals.p, sorted.p, int(n),
                                     0, 63, s));
  if (int(n) <= leaf_max) {
    nodes.reset();
    CK(cudaStreamSynchronize(s));
    return SHERD_OK;
  }
  int ni = int(n) - 1;
  DBuf<int> left, right, first, last, pint, pleaf;
  DBuf<unsigned> flags;
  DBuf<float> ibox;
  CK(left.alloc(ni));
  CK(right.alloc(ni));
  CK(first.alloc(ni));
  CK(last.alloc(ni));
  CK(pint.alloc(ni));
  CK(pleaf.alloc(n));
  CK(flags.alloc(ni));
  CK(ibox.alloc(size_t(6) * ni));
  CK(nodes.alloc(ni));
  CK(cudaMemsetAsync(flags.p, 0, sizeof(unsigned) * ni, s));
  CK(cudaMemsetAsync(pint.p, 0xFF, sizeof(int) * ni, s));  // root's parent is -1
  k_karras<<<blocks_for(ni), 256, 0, s>>>(keys2.p, int(n), left.p, right.p, first.p, last.p, pint.p,
                                          pleaf.p);
  CK(cudaGetLastError());
  k_refit<TRI><<<blocks_for(n), 256, 0, s>>>(d_v, d_f, d_p, sorted.p, int(n), left.p, right.p,
                                             pint.p, pleaf.p, flags.p, ibox.p);
  CK(cudaGetLastError());
  k_emit<TRI><<<blocks_for(ni), 256, 0, s>>>(d_v, d_f, d_p, sorted.p, int(n), left.p, right.p,
                                             first.p, last.p, ibox.p, pad, leaf_max, nodes.p);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s));
  return SHERD_OK;
}

int mesh_build(sherd_ctx *ctx, sherd_mesh *m) {
  uint32_t nv = uint32_t(m->hv.size() / 3), nf = uint32_t(m->hf.size() / 3);
  DBuf<float> dv;
  DBuf<uint32_t> df, sorted;
  int rc = upload(ctx, dv, m->hv.data(), m->hv.size());
  if (rc) return rc;
  rc = upload(ctx, df, m->hf.data(), m->hf.size());
  if (rc) return rc;
  double mag = 1.0;
  for (float x : m->hv) mag = std::max(mag, double(std::fabs(x)));
  float pad = float(1e-5 * mag);
  float lo[3], hi[3];
  rc = build_lbvh<true>(ctx, dv.p, nv, df.p, nullptr, nf, pad, TRI_LEAF, m->nodes, sorted, lo, hi);
  if (rc) return rc;
  CK(m->tri.alloc(size_t(3) * nf));
  k_store_tris<<<blocks_for(nf), 256, 0, ctx->stream>>>(dv.p, df.p, sorted.p, nf, m->tri.p);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(ctx->stream));
  // The exact vertex box of RayScene::aabb (bvh.rs:182-185).
  float vlo[3] = {f_inf(), f_inf(), f_inf()}, vhi[3] = {-f_inf(), -f_inf(), -f_inf()};
  for (uint32_t i = 0; i < nv; ++i)
    for (int k = 0; k < 3; ++k) {
      vlo[k] = std::min(vlo[k], m->hv[3 * i + k]);
      vhi[k] = std::max(vhi[k], m->hv[3 * i + k]);
    }
  // The three crossing grids: cells about one mean edge across, at most 16 M
  // cells per axis, every face binned with the box padding.
  double edge = 0.0;
  for (uint32_t i = 0; i < nf; ++i) {
    const float *a = &m->hv[3 * m->hf[3 * i]], *b = &m->hv[3 * m->hf[3 * i + 1]];
    edge += std::sqrt(double(a[0] - b[0]) * (a[0] - b[0]) + double(a[1] - b[1]) * (a[1] - b[1]) +
                      double(a[2] - b[2]) * (a[2] - b[2]));
  }
  edge = std::max(edge / std::max<uint32_t>(nf, 1), 1e-6);
  for (int axis = 0; axis < 3; ++axis) {
    int au = (axis + 1) % 3, av = (axis + 2) % 3;
    AxisGrid g{};
    double lo_u = double(vlo[au]) - 2.0 * pad, lo_v = double(vlo[av]) - 2.0 * pad;
    double ext_u = double(vhi[au]) - lo_u + 2.0 * pad, ext_v = double(vhi[av]) - lo_v + 2.0 * pad;
    double cell = edge;
    while ((ext_u / cell + 1.0) * (ext_v / cell + 1.0) > 16.0e6) cell *= 1.5;
    g.lo_u = float(lo_u);
    g.lo_v = float(lo_v);
    g.inv_cell = float(1.0 / cell);
    g.nu = uint32_t(ext_u / cell) + 2;
    g.nv = uint32_t(ext_v / cell) + 2;
    size_t cells = size_t(g.nu) * g.nv;
    DBuf<unsigned> count;
    CK(count.alloc(cells + 1));
    CK(cudaMemsetAsync(count.p, 0, sizeof(unsigned) * (cells + 1), ctx->stream));
    k_grid_count<<<blocks_for(nf), 256, 0, ctx->stream>>>(m->tri.p, nf, axis, g, pad, count.p);
    CK(cudaGetLastError());
    CK(m->gstart[axis].alloc(cells + 1));
    size_t temp_bytes = 0;
    CK(cub::DeviceScan::ExclusiveSum(nullptr, temp_bytes, count.p, m->gstart[axis].p, int(cells + 1),
                                     ctx->stream));
    DBuf<unsigned char> temp;
    CK(temp.alloc(temp_bytes));
    CK(cub::DeviceScan::ExclusiveSum(temp.p, temp_bytes, count.p, m->gstart[axis].p, int(cells + 1),
                                     ctx->stream));
    uint32_t total = 0;
    CK(cudaMemcpyAsync(&total, m->gstart[axis].p + cells, 4, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    CK(m->grect[axis].alloc(std::max<uint32_t>(total, 1)));
    CK(m->gtri[axis].alloc(3 * size_t(std::max<uint32_t>(total, 1))));
    CK(cudaMemcpyAsync(count.p, m->gstart[axis].p, sizeof(unsigned) * cells, cudaMemcpyDeviceToDevice,
                       ctx->stream));
    k_grid_fill<<<blocks_for(nf), 256, 0, ctx->stream>>>(m->tri.p, nf, axis, g, pad, count.p,
                                                        m->grect[axis].p, m->gtri[axis].p);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->stream));
    g.start = m->gstart[axis].p;
    g.rect = m->grect[axis].p;
    g.tri = m->gtri[axis].p;
    m->view.grid[axis] = g;
  }
  MeshView &v = m->view;
  v.nodes = m->nodes.p;
  v.tri = m->tri.p;
  v.nf = nf;
  v.root_leaf = nf <= uint32_t(TRI_LEAF) ? nf : 0;
  v.pad = pad;
  for (int k = 0; k < 3; ++k) {
    v.lo[k] = vlo[k];
    v.hi[k] = vhi[k];
  }
  // The bound grid (LbGrid): cube cells, 64 across the largest extent of the
  // vertex box widened by a quarter of that extent on every side.
  v.lbg = LbGrid{};
  if (!v.root_leaf && nf > 0) {
    double mx = 0.0;
    for (int k = 0; k < 3; ++k) mx = std::max(mx, double(vhi[k]) - double(vlo[k]));
    const double margin = 0.25 * mx + 2.0 * double(pad);
    const double cell = (mx + 2.0 * margin) / 64.0;
    if (cell > 0.0 && std::isfinite(cell)) {
      LbGrid g{};
      size_t total = 1;
      for (int k = 0; k < 3; ++k) {
        g.lo[k] = std::nextafter(float(double(vlo[k]) - margin), -f_inf());
        g.n[k] = uint32_t(std::ceil((double(vhi[k]) - double(vlo[k]) + 2.0 * margin) / cell)) + 1;
        total *= g.n[k];
      }
      g.cell = float(cell);
      g.inv_cell = float(1.0 / double(g.cell));
      CK(m->lb.alloc(total));
      k_lb_grid<<<unsigned((total + 255) / 256), 256, 0, ctx->stream>>>(m->nodes.p, g, m->lb.p);
      CK(cudaGetLastError());
      g.lb = m->lb.p;
      v.lbg = g;
    }
  }
  return SHERD_OK;
}

// Builds the point LBVH over np points already on the device (normals
// optional); `pad` is the outward padding of its boxes.
int cloud_build_dev(sherd_ctx *ctx, const double *dp, const double *dn, uint32_t np, float pad,
                    sherd_cloud *c) {
  DBuf<uint32_t> sorted;
  float lo[3], hi[3];
  int rc = build_lbvh<false>(ctx, nullptr, 0, nullptr, dp, np, pad, POINT_LEAF, c->nodes, sorted,
                             lo, hi);
  if (rc) return rc;
  CK(c->pts.alloc(np));
  if (dn) CK(c->nrm.alloc(np));
  k_store_pts<<<blocks_for(np), 256, 0, ctx->stream>>>(dp, dn, sorted.p, np, c->pts.p,
                                                       dn ? c->nrm.p : nullptr);
  CK(cudaGetLastError());
  const bool tree = np > uint32_t(POINT_LEAF);
  if (tree && WIDE_NN) {
    CK(c->wide.alloc(np - 1));
    k_widen<<<blocks_for(np - 1), 256, 0, ctx->stream>>>(c->nodes.p, int(np - 1), c->wide.p);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(ctx->stream));
  c->ctx = ctx;
  CloudView &v = c->view;
  v.nodes = c->nodes.p;
  v.pts = c->pts.p;
  v.nrm = dn ? c->nrm.p : nullptr;
  v.n = np;
  v.root_leaf = np <= uint32_t(POINT_LEAF) ? np : 0;
  v.pad = pad;
  v.wide = tree && WIDE_NN ? c->wide.p : nullptr;
  return SHERD_OK;
}

int cloud_build(sherd_ctx *ctx, const double *p, const double *nrm, uint32_t np, sherd_cloud *c) {
  DBuf<double> dp, dn;
  int rc = upload(ctx, dp, p, size_t(3) * np);
  if (rc) return rc;
  if (nrm) {
    rc = upload(ctx, dn, nrm, size_t(3) * np);
    if (rc) return rc;
  }
  double mag = 1.0;
  for (size_t i = 0; i < size_t(3) * np; ++i) mag = std::max(mag, std::fabs(p[i]));
  return cloud_build_dev(ctx, dp.p, nrm ? dn.p : nullptr, np, float(1e-6 * mag), c);
}

// The cone's constants in f64 on the host, as segment.rs:330-355 computes
// them: 15 degrees through to_radians and the six azimuths 2 pi (k-1) / 6.
ConeConsts cone_consts() {
  const double PI = 3.14159265358979323846;
  ConeConsts cc;
  double angle = 15.0 * (PI / 180.0);
  cc.cos_a = std::cos(angle);
  cc.sin_a = std::sin(angle);
  for (int k = 1; k < 7; ++k) {
    double phi = 2.0 * PI * double(k - 1) / 6.0;
    cc.cp[k - 1] = std::cos(phi);
    cc.sp[k - 1] = std::sin(phi);
  }
  return cc;
}

template <typename K, typename V>
int radix_sort_pairs(sherd_ctx *ctx, const K *kin, K *kout, const V *vin, V *vout, uint32_t n,
                     int end_bit) {
  size_t bytes = 0;
  CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, kin, kout, vin, vout, int(n), 0, end_bit,
                                     ctx->stream));
  DBuf<unsigned char> tmp;
  CK(tmp.alloc(bytes));
  CK(cub::DeviceRadixSort::SortPairs(tmp.p, bytes, kin, kout, vin, vout, int(n), 0, end_bit,
                                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return SHERD_OK;
}

bool has_nan(const double *p, size_t n) {
  for (size_t i = 0; i < n; ++i)
    if (std::isnan(p[i])) return true;
  return false;
}

// The dense ids of R 6.2's voxels floor(A.brk_p / (t/3)) (verify.rs:400-414,
// 809-811): equal voxels share an id, so the device counts distinct ids.
int seam_cells(sherd_ctx *ctx, const std::vector<double> &brk, double t, DBuf<uint32_t> &out,
               uint32_t &n_cells) {
  size_t n = brk.size() / 3;
  double voxel = t / 3.0;
  std::vector<std::array<int64_t, 3>> cells(n);
  for (size_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) cells[i][k] = int64_t(std::floor(brk[3 * i + k] / voxel));
  std::vector<std::array<int64_t, 3>> uniq = cells;
  std::sort(uniq.begin(), uniq.end());
  uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
  std::vector<uint32_t> ids(n);
  for (size_t i = 0; i < n; ++i)
    ids[i] = uint32_t(std::lower_bound(uniq.begin(), uniq.end(), cells[i]) - uniq.begin());
  n_cells = uint32_t(uniq.size());
  if (n_cells > uint32_t(MAX_CELL_WORDS) * 32u)
    return fail(ctx, SHERD_E_INVALID, "breakline spans more than 65536 seam voxels");
  return upload(ctx, out, ids.data(), n);
}

// Per-item scratch in 4-byte words, a multiple of 64 so that every CTA's slot
// (and the 8-byte keys of the continuity medians) stays 256-byte aligned.
uint32_t scratch_words(const PairView &v) {
  uint32_t w = std::max<uint32_t>({v.a.n_pf, v.b.n_pf, 4u * v.b.n_margin, 1u});
  return (w + 63u) / 64u * 64u;
}

}  // namespace

extern "C" {

const char *sherd_name(void) { return "cuda"; }

int sherd_open(int device, sherd_ctx **out) {
  if (!out) return SHERD_E_INVALID;
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || device < 0 || device >= count) {
    cudaGetLastError();
    t_errors[nullptr] = "no such CUDA device";
    return SHERD_E_DEVICE;
  }
  sherd_ctx *ctx = new sherd_ctx;
  ctx->device = device;
  auto bad = [&](cudaError_t err) {
    t_errors[nullptr] = cudaGetErrorString(err);
    delete ctx;
    return SHERD_E_DEVICE;
  };
  if ((e = cudaSetDevice(device)) != cudaSuccess) return bad(e);
  if ((e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device)) !=
      cudaSuccess)
    return bad(e);
  if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) return bad(e);
  if ((e = cudaEventCreate(&ctx->ev0)) != cudaSuccess) return bad(e);
  if ((e = cudaEventCreate(&ctx->ev1)) != cudaSuccess) return bad(e);
  for (int k = 0; k < 2; ++k) {
    if ((e = cudaStreamCreateWithFlags(&ctx->side[k], cudaStreamNonBlocking)) != cudaSuccess) return bad(e);
    if ((e = cudaEventCreateWithFlags(&ctx->join_ev[k], cudaEventDisableTiming)) != cudaSuccess) return bad(e);
  }
  if ((e = cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming)) != cudaSuccess) return bad(e);
  // The context's own stream-ordered pool: it keeps up to POOL_KEEP_BYTES of
  // what the entry points free for their next buffers instead of handing it
  // back to the device at every synchronisation.
  {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if ((e = cudaMemPoolCreate(&ctx->pool, &props)) != cudaSuccess) return bad(e);
    uint64_t keep = POOL_KEEP_BYTES;
    if ((e = cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess)
      return bad(e);
  }
  if ((e = cudaHostAlloc(&ctx->abort_host, 4, cudaHostAllocMapped)) != cudaSuccess) return bad(e);
  *ctx->abort_host = 0;
  if ((e = cudaHostGetDevicePointer(&ctx->abort_dev, ctx->abort_host, 0)) != cudaSuccess) return bad(e);
  if ((e = cudaMalloc(&ctx->d_status, 4)) != cudaSuccess) return bad(e);
  *out = ctx;
  return SHERD_OK;
}

int sherd_close(sherd_ctx *ctx) {
  if (!ctx) return SHERD_E_INVALID;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->d_status) cudaFree(ctx->d_status);
  if (ctx->abort_host) cudaFreeHost(ctx->abort_host);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  for (int k = 0; k < 2; ++k) {
    if (ctx->side[k]) cudaStreamDestroy(ctx->side[k]);
    if (ctx->join_ev[k]) cudaEventDestroy(ctx->join_ev[k]);
  }
  if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
  if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  t_errors.erase(ctx);
  delete ctx;
  return SHERD_OK;
}

const char *sherd_last_error(const sherd_ctx *ctx) {
  auto it = t_errors.find(ctx);
  return it == t_errors.end() ? "" : it->second.c_str();
}

int sherd_set_timeout_ms(sherd_ctx *ctx, uint32_t ms) {
  if (!ctx) return SHERD_E_INVALID;
  CtxLock lock(ctx);
  ctx->timeout_ms = ms;
  return SHERD_OK;
}

int sherd_abort(sherd_ctx *ctx) {
  if (!ctx) return SHERD_E_INVALID;
  // Deliberately not under the lock: it is meant to reach a running call.
  __atomic_store_n(ctx->abort_host, 1u, __ATOMIC_SEQ_CST);
  return SHERD_OK;
}

int sherd_stats_json(sherd_ctx *ctx, char *buf, size_t len) {
  if (!ctx || !buf || !len) return SHERD_E_INVALID;
  CtxLock lock(ctx);
  std::string s = "{\"backend\": \"cuda\", \"device\": " + std::to_string(ctx->device) +
                  ", \"sm_count\": " + std::to_string(ctx->sm_count) + ", \"methods\": {";
  bool firstm = true;
  for (auto &kv : ctx->stats) {
    char tmp[256];
    std::snprintf(tmp, sizeof tmp, "%s\"%s\": {\"calls\": %llu, \"items\": %llu, \"ms\": %.3f}",
                  firstm ? "" : ", ", kv.first.c_str(), (unsigned long long)kv.second.calls,
                  (unsigned long long)kv.second.items, kv.second.ms);
    s += tmp;
    firstm = false;
  }
  s += "}, \"ladder_autotune\": {";
  for (int b = 0; b < 3; ++b) {
    char tmp[256];
    int v = ctx->ladder_tuned[b];
    std::snprintf(tmp, sizeof tmp,
                  "%s\"bucket%d\": {\"ctas_per_sm\": %d, \"sample_items\": %u, \"ms\": [%.3f, %.3f, %.3f]}",
                  b ? ", " : "", b, v >= 0 ? LADDER_MINB[v] : -1, ctx->ladder_tune_items[b],
                  ctx->ladder_tune_ms[b][0], ctx->ladder_tune_ms[b][1], ctx->ladder_tune_ms[b][2]);
    s += tmp;
  }
  s += "}}";
  if (s.size() + 1 > len) return fail(ctx, SHERD_E_INVALID, "stats buffer too small");
  std::memcpy(buf, s.c_str(), s.size() + 1);
  return SHERD_OK;
}

uint32_t sherd_device_slack(const sherd_ctx *ctx) {
  // A caller parked on the device is a worker not preparing the next batch
  // (executor/mod.rs:123-136): one extra worker per 37 SMs.
  return ctx ? uint32_t(std::max(1, ctx->sm_count / 37)) : 0u;
}

// ---- meshes -------------------------------------------------------------

int sherd_mesh_upload(sherd_ctx *ctx, const float *v, uint32_t nv, const uint32_t *f, uint32_t nf,
                      sherd_mesh **out) {
  if (!ctx || !out || (!v && nv) || (!f && nf)) return fail(ctx, SHERD_E_INVALID, "null argument");
  *out = nullptr;
  if (nf == 0) return fail(ctx, SHERD_E_EMPTY, "a mesh needs at least one face");
  for (size_t i = 0; i < size_t(3) * nf; ++i)
    if (f[i] >= nv) return fail(ctx, SHERD_E_INVALID, "face index beyond the vertex array");
  for (size_t i = 0; i < size_t(3) * nv; ++i)
    if (!std::isfinite(v[i])) return fail(ctx, SHERD_E_INVALID, "non-finite vertex");
  CtxLock lock(ctx);
  CK(cudaSetDevice(ctx->device));
  sherd_mesh *m = new sherd_mesh;
  m->ctx = ctx;
  m->hv.assign(v, v + size_t(3) * nv);
  m->hf.assign(f, f + size_t(3) * nf);
  int rc = mesh_build(ctx, m);
  if (rc) {
    delete m;
    return rc;
  }
  *out = m;
  return SHERD_OK;
}

int sherd_mesh_subset(sherd_ctx *ctx, const sherd_mesh *mesh, const uint8_t *keep, sherd_mesh **out) {
  if (!ctx || !mesh || !keep || !out) return fail(ctx, SHERD_E_INVALID, "null argument");
  *out = nullptr;
  CtxLock lock(ctx);
  CK(cudaSetDevice(ctx->device));
  sherd_mesh *m = new sherd_mesh;
  m->ctx = ctx;
  m->hv = mesh->hv;
  size_t nf = mesh->hf.size() / 3;
  for (size_t i = 0; i < nf; ++i)
    if (keep[i]) m->hf.insert(m->hf.end(), mesh->hf.begin() + 3 * i, mesh->hf.begin() + 3 * i + 3);
  if (m->hf.empty()) m->hf.assign(mesh->hf.begin(), mesh->hf.begin() + 3);
  int rc = mesh_build(ctx, m);
  if (rc) {
    delete m;
    return rc;
  }
  *out = m;
  return SHERD_OK;
}

int sherd_mesh_free(sherd_mesh *mesh) {
  if (!mesh) return SHERD_E_INVALID;
  cudaSetDevice(mesh->ctx->device);
  CtxLock lock(mesh->ctx);
  delete mesh;
  return SHERD_OK;
}

int sherd_mesh_aabb(const sherd_mesh *mesh, float lo[3], float hi[3]) {
  if (!mesh || !lo || !hi) return SHERD_E_INVALID;
  for (int k = 0; k < 3; ++k) {
    lo[k] = mesh->view.lo[k];
    hi[k] = mesh->view.hi[k];
  }
  return SHERD_OK;
}

uint32_t sherd_mesh_faces(const sherd_mesh *mesh) { return mesh ? mesh->view.nf : 0; }

int sherd_first_hit(sherd_ctx *ctx, const sherd_mesh *mesh, const float *origins, const float *dirs,
                    uint32_t n, float *t_out, uint32_t *prim_out) {
  if (!ctx || !mesh || ((!origins || !dirs || !t_out || !prim_out) && n))
    return fail(ctx, SHERD_E_INVALID, "null argument");
  if (n == 0) return SHERD_OK;
  CtxLock lock(ctx);
  int rc = begin(ctx);
  if (rc) return rc;
  DBuf<float> o, d, t;
  DBuf<uint32_t> p;
  if ((rc = upload(ctx, o, origins, size_t(3) * n)) || (rc = upload(ctx, d, dirs, size_t(3) * n)))
    return rc;
  CK(t.alloc(n));
  CK(p.alloc(n));
  k_first_hit<<<blocks_for(n), 128, 0, ctx->stream>>>(mesh->view, o.p, d.p, n, t.p, p.p,
                                                     ctx->d_status);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(t_out, t.p, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(prim_out, p.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
  return finish(ctx, "first_hit", n, true);
}

int sherd_bounded_distance(sherd_ctx *ctx, const sherd_mesh *mesh, const double *points, uint32_t n,
                           const double pose[16], double max_dist, int reduce, double *out) {
  if (!ctx || !mesh || !out || (!points && n)) return fail(ctx, SHERD_E_INVALID, "null argument");
  if (!finite_pose(pose)) return fail(ctx, SHERD_E_INVALID, "pose is not finite");
  if (reduce != SHERD_REDUCE_ALL && reduce != SHERD_REDUCE_MIN)
    return fail(ctx, SHERD_E_INVALID, "unknown reduction");
  float window = float(max_dist);
  if (reduce == SHERD_REDUCE_MIN && n == 0) {
    *out = double(window);
    return SHERD_OK;
  }
  if (n == 0) return SHERD_OK;
  CtxLock lock(ctx);
  int rc = begin(ctx);
  if (rc) return rc;
  DBuf<double> p, o;
  if ((rc = upload(ctx, p, points, size_t(3) * n))) return rc;
  if (reduce == SHERD_REDUCE_ALL) {
    CK(o.alloc(n));
    k_bounded_all<<<blocks_for(n, 128), 128, 0, ctx->stream>>>(mesh->view, p.p, n, pose_of(pose),
                                                              window, o.p, ctx->d_status);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, o.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    return finish(ctx, "bounded_distance", n, true);
  }
  // The scan of cpu.rs:98-111 starts from the window and keeps the smaller
  // of it and every distance found within the shrinking window.
  DBuf<unsigned> best;
  CK(best.alloc(1));
  unsigned key0;
  float w = window;
  std::memcpy(&key0, &w, 4);
  if (!(window > 0.0f)) key0 = 0u;  // a non-positive window finds nothing
  CK(cudaMemcpyAsync(best.p, &key0, 4, cudaMemcpyHostToDevice, ctx->stream));
  if (window > 0.0f) {
    k_bounded_min<<<blocks_for(n, 128), 128, 0, ctx->stream>>>(mesh->view, p.p, n, pose_of(pose),
                                                              best.p, ctx->d_status);
    CK(cudaGetLastError());
  }
  unsigned key = 0;
  CK(cudaMemcpyAsync(&key, best.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
  rc = finish(ctx, "bounded_distance_min", n, true);
  if (rc) return rc;
  float f;
  std::memcpy(&f, &key, 4);
  *out = window > 0.0f ? double(f) : double(window);
  return SHERD_OK;
}

int sherd_inside(sherd_ctx *ctx, const sherd_mesh *mesh, const double *points, uint32_t n,
                 const double pose[16], sherd_inside_outcome *out) {
  if (!ctx || !mesh || ((!points || !out) && n)) return fail(ctx, SHERD_E_INVALID, "null argument");
  if (!finite_pose(pose)) return fail(ctx, SHERD_E_INVALID, "pose is not finite");
  if (n == 0) return SHERD_OK;
  CtxLock lock(ctx);
  int rc = begin(ctx);
  if (rc) return rc;
  DBuf<double> p;
  DBuf<sherd_inside_outcome> o;
  if ((rc = upload(ctx, p, points, size_t(3) * n))) return rc;
  CK(o.alloc(n));
  k_inside<<<blocks_for(n, 128), 128, 0, ctx->stream>>>(mesh->view, p.p, n, pose_of(pose), o.p,
                                                       ctx->d_status);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, o.p, sizeof(sherd_inside_outcome) * n, cudaMemcpyDeviceToHost,
                     ctx->stream));
  return finish(ctx, "inside", n, true);
}

int sherd_penetration_share(sherd_ctx *ctx, const sherd_mesh *mesh, const double *points,
                            uint32_t n, const double pose[16], double pen, double *share) {
  if (!ctx || !mesh || !share || (!points && n)) return fail(ctx, SHERD_E_INVALID, "null argument");
  if (!finite_pose(pose)) return fail(ctx, SHERD_E_INVALID, "pose is not finite");
  *share = 0.0;
  if (n == 0) return SHERD_OK;
  CtxLock lock(ctx);
  int rc = begin(ctx);
  if (rc) return rc;
  DBuf<double> p;
  DBuf<unsigned long long> cnt;
  if ((rc = upload(ctx, p, points, size_t(3) * n))) return rc;
  CK(cnt.alloc(1));
  CK(cudaMemsetAsync(cnt.p, 0, sizeof(unsigned long long), ctx->stream));
  unsigned grid = std::min(blocks_for(n, 128), unsigned(ctx->sm_count) * 16u);
  // Whole warps: the kernel's ballot needs every lane of a warp in the loop.
  k_penetration_share<<<grid, 128, 0, ctx->stream>>>(mesh->view, p.p, n, pose_of(pose), pen, cnt.p,
                                                     ctx->d_status);
  CK(cudaGetLastError());
  unsigned long long deeper = 0;
  CK(cudaMemcpyAsync(&deeper, cnt.p, sizeof deeper, cudaMemcpyDeviceToHost, ctx->stream));
  rc = finish(ctx, "penetration_share", n, true);
  if (rc) return rc;
  *share = double(deeper) / double(n);
  return SHERD_OK;
}

// ---- preprocessing rays ------------------------------------------------------

int sherd_face_geometry(sherd_ctx *ctx, const double *v, uint32_t nv, const uint32_t *f, uint32_t nf,
                        double *normals, double *areas, double *centroids) {
  if (!ctx || ((!v && nv) || (!f && nf))) return fail(ctx, SHERD_E_INVALID, "null argument");
  if (nf == 0) return SHERD_OK;
  CtxLock lock(ctx);
  int rc = begin(ctx);
  if (rc) return rc;
  DBuf<double> dv, dn, da, dc;
  DBuf<uint32_t> df;
  if ((rc = upload(ctx, dv, v, size_t(3) * nv)) || (rc = upload(ctx, df, f, size_t(3) * nf))) return rc;
  DevInputCheck chk;
  InputCheck got;
  if ((rc = chk.open(ctx, 1)) || (rc = chk.indices(ctx, 0, df.p, size_t(3) * nf, nv)) ||
      (rc = chk.read(ctx, &got)))
    return rc;
  if (got.bad_index) return fail(ctx, SHERD_E_INVALID, "face index beyond the vertex array");
  if (normals) CK(dn.alloc(size_t(3) * nf));
  if (areas) CK(da.alloc(nf));
  if (centroids) CK(dc.alloc(size_t(3) * nf));
  k_face_geometry<<<blocks_for(nf), 256, 0, ctx->stream>>>(dv.p, df.p, nf, dn.p, da.p, dc.p);
  CK(cudaGetLastError());
  if (normals) CK(cudaMemcpyAsync(normals, dn.p, 24 * size_t(nf), cudaMemcpyDeviceToHost, ctx->stream));
  if (areas) CK(cudaMemcpyAsync(areas, da.p, 8 * size_t(nf), cudaMemcpyDeviceToHost, ctx->stream));
  if (centroids)
    CK(cudaMemcpyAsync(centroids, dc.p, 24 * size_t(nf), cudaMemcpyDeviceToHost, ctx->stream));
  return finish(ctx, "face_geometry", nf, true);
}

namespace {

// Sorts the valid and the looking-back distances and takes both histogram
// modes on the device (thickness.rs:139-162).
int thickness_modes(sherd_ctx *ctx, DBuf<float> &ok, DBuf<float> &far, DBuf<unsigned> &counts,
                    float *t, float *mode, uint32_t *found) {
  unsigned hc[2];
  CK(cudaMemcpyAsync(hc, counts.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (hc[0] < 100) {
    *found = 0;
    return SHERD_OK;
  }
  DBuf<float> sorted;
  DBuf<float> modes;
  CK(sorted.alloc(std::max(hc[0], 1u)));
  CK(modes.alloc(2));
  size_t temp_bytes = 0;
  CK(cub::DeviceRadixSort::SortKeys(nullptr, temp_bytes, ok.p, sorted.p, int(hc[0]), 0, 32,
                                    ctx->stream));
  DBuf<unsigned char> temp;
  CK(temp.alloc(temp_bytes));
  CK(cub::DeviceRadixSort::SortKeys(temp.p, temp_bytes, ok.p, sorted.p, int(hc[0]), 0, 32,
                                    ctx->stream));
  k_hist_mode<<<1, 1024, 0, ctx->stream>>>(sorted.p, hc[0], modes.p);
  CK(cudaGetLastError());
  if (hc[1] >= 100) {
    CK(cub::DeviceRadixSort::SortKeys(temp.p, temp_bytes, far.p, sorted.p, int(hc[1]), 0, 32,
                                      ctx->stream));
    k_hist_mode<<<1, 1024, 0, ctx->stream>>>(sorted.p, hc[1], modes.p + 1);
    CK(cudaGetLastError());
  }
  float hm[2];
  CK(cudaMemcpyAsync(hm, modes.p, 8, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  *mode = hm[0];
  *t = hc[1] >= 100 ? hm[1] : hm[0];
  *found = 1;
  return SHERD_OK;
}

}  // namespace

int sherd_thickness(sherd_ctx *ctx, const sherd_mesh *mesh, const double *centroids,
                    const double *normals, uint32_t nf, uint32_t max_rays, float *t,
                    float *thick_mode, uint32_t *found, float *t_hit, uint32_t *prim) {
  if (!ctx || !mesh || !centroids || !normals || !t || !thick_mode || !found)
    return fail(ctx, SHERD_E_INVALID, "null argument");
  if (nf != mesh->view.nf) return fail(ctx, SHERD_E_INVALID, "face count differs from the mesh");
  *found = 0;
  if (nf == 0) return SHERD_OK;
  uint32_t n_req = max_rays ? max_rays : 1;
  uint32_t stride = std::max<uint32_t>(1, (nf + n_req - 1) / n_req);
  uint32_t n = (nf + stride - 1) / stride;
  CtxLock lock(ctx);
  int rc = begin(ctx);
  if (rc) return rc;
  DBuf<double> dc, dn;
  DBuf<float> th, ok, far;
  DBuf<uint32_t> pr;
  DBuf<unsigned> counts;
  if ((rc = upload(ctx, dc, centroids, size_t(3) * nf)) || (rc = upload(ctx, dn, normals, size_t(3) * nf)))
    return rc;
  CK(th.alloc(n));
  CK(pr.alloc(n));
  CK(ok.alloc(n));
  CK(far.alloc(n));
  CK(counts.alloc(2));
  CK(cudaMemsetAsync(counts.p, 0, 8, ctx->stream));
  k_thickness_rays<<<blocks_for(n, 128), 128, 0, ctx->stream>>>(
      mesh->view, dc.p, dn.p, nf, stride, n, th.p, pr.p, ok.p, far.p, counts.p, ctx->d_status);
  CK(cudaGetLastError());
  rc = thickness_modes(ctx, ok, far, counts, t, thick_mode, found);
  if (rc) return rc;
  if (t_hit) CK(cudaMemcpyAsync(t_hit, th.p, 4 * size_t(n), cudaMemcpyDeviceToHost, ctx->stream));
  if (prim) CK(cudaMemcpyAsync(prim, pr.p, 4 * size_t(n), cudaMemcpyDeviceToHost, ctx->stream));
  return finish(ctx, "thickness", n, true);
}

int sherd_thickness_from_hits(sherd_ctx *ctx, const double *normals, uint32_t nf, const uint32_t *idx,
                              const float *t_hit, const uint32_t *prim, uint32_t n, float *t,
                              float *thick_mode, uint32_t *found) {
  if (!ctx || !normals || !t || !thick_mode || !found || ((!idx || !t_hit || !prim) && n))
    return fail(ctx, SHERD_E_INVALID, "null argument");
  for (uint32_t k = 0; k < n; ++k)
    if (idx[k] >= nf) return fail(ctx, SHERD_E_INVALID, "ray face id beyond the mesh");
  *found = 0;
  if (n == 0) return SHERD_OK;
  CtxLock lock(ctx);
  int rc = begin(ctx);
  if (rc) return rc;
  DBuf<double> dn;
  DBuf<uint32_t> di, dp;
  DBuf<float> dt, ok, far;
  DBuf<unsigned> counts;
  if ((rc = upload(ctx, dn, normals, size_t(3) * nf)) || (rc = upload(ctx, di, idx, n)) ||
      (rc = upload(ctx, dt, t_hit, n)) || (rc = upload(ctx, dp, prim, n)))
    return rc;
  CK(ok.alloc(n));
  CK(far.alloc(n));
  CK(counts.alloc(2));
  CK(cudaMemsetAsync(counts.p, 0, 8, ctx->stream));
  k_thickness_filter<<<blocks_for(n), 256, 0, ctx->stream>>>(dn.p, nf, di.p, dt.p, dp.p, n, ok.p,
                                                            far.p, counts.p);
  CK(cudaGetLastError());
  rc = thickness_modes(ctx, ok, far, counts, t, thick_mode, found);
  if (rc) return rc;
  return finish(ctx, "thickness_from_hits", n, true);
}

int sherd_cone_votes(sherd_ctx *ctx, const sherd_mesh *mesh, const double *centroids,
                     const double *normals, const double *ns, const double *hit_normals,
                     uint32_t nf, double thick, uint8_t *good) {
  if (!ctx || !mesh || ((!centroids || !normals || !ns || !hit_normals || !good) && nf))
    return fail(ctx, SHERD_E_INVALID, "null argument");
  if (nf != mesh->view.nf) return fail(ctx, SHERD_E_INVALID, "face count differs from the mesh");
  if (nf == 0) return SHERD_OK;
  ConeConsts cc = cone_consts();
  CtxLock lock(ctx);
  int rc = begin(ctx);
  if (rc) return rc;
  DBuf<double> dc, dn, dns, dh;
  DBuf<uint8_t> dg;
  if ((rc = upload(ctx, dc, centroids, size_t(3) * nf)) || (rc = upload(ctx, dn, normals, size_t(3) * nf)) ||
      (rc = upload(ctx, dns, ns, size_t(3) * nf)) || (rc = upload(ctx, dh, hit_normals, size_t(3) * nf)))
    return rc;
  CK(dg.alloc(nf));
  k_cone_votes<<<blocks_for(nf, 128), 128, 0, ctx->stream>>>(mesh->view, dc.p, dn.p, dns.p, dh.p, nf,
                                                            thick, cc, dg.p, ctx->d_status);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(good, dg.p, nf, cudaMemcpyDeviceToHost, ctx->stream));
  return finish(ctx, "cone_votes", size_t(nf) * 7, true);
}

// ---- clouds ----------------------------------------------------------------

int sherd_cloud_upload(sherd_ctx *ctx, const double *points, const double *normals, uint32_t np,
                       sherd_cloud **out) {
  if (!ctx || !out || (!points && np)) return fail(ctx, SHERD_E_INVALID, "null argument");
  *out = nullptr;
  if (np == 0) return fail(ctx, SHERD_E_EMPTY, "a cloud needs at least one point");
  for (size_t i = 0; i < size_t(3) * np; ++i)
    if (!std::isfinite(points[i])) return fail(ctx, SHERD_E_INVALID, "non-finite point");
  CtxLock lock(ctx);
  CK(cudaSetDevice(ctx->device));
  sherd_cloud *c = new sherd_cloud;
  int rc = cloud_build(ctx, points, normals, np, c);
  if (rc) {
    delete c;
    return rc;
  }
  *out = c;
  return SHERD_OK;
}

int sherd_cloud_free(sherd_cloud *cloud) {
  if (!cloud) return SHERD_E_INVALID;
  cudaSetDevice(cloud->ctx->device);
  CtxLock lock(cloud->ctx);
  delete cloud;
  return SHERD_OK;
}

uint32_t sherd_cloud_points(const sherd_cloud *cloud) { return cloud ? cloud->view.n : 0; }

int sherd_nearest_within_sq(sherd_ctx *ctx, const sherd_cloud *cloud, const double *queries, uint32_t n,
                            double r2, uint32_t *idx, double *d2) {
  if (!ctx || !cloud || ((!queries || !idx || !d2) && n)) return fail(ctx, SHERD_E_INVALID, "null argument");
  if (n == 0) return SHERD_OK;
  CtxLock lock(ctx);
  int rc = begin(ctx);
  if (rc) return rc;
  DBuf<double> q, o;
  DBuf<uint32_t> i;
  if ((rc = upload(ctx, q, queries, size_t(3) * n))) return rc;
  CK(o.alloc(n));
  CK(i.alloc(n));
  k_nn_within<<<blocks_for(n, 128), 128, 0, ctx->stream>>>(cloud->view, q.p, n, r2, i.p, o.p,
                                                          ctx->d_status);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(idx, i.p, 4 * size_t(n), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(d2, o.p, 8 * size_t(n), cudaMemcpyDeviceToHost, ctx->stream));
  return finish(ctx, "nearest_within_sq", n, true);
}

int sherd_nearest_below(sherd_ctx *ctx, const sherd_cloud *cloud, const double *queries, uint32_t n,
                        double bound, uint32_t *idx, double *dist) {
  if (!ctx || !cloud || ((!queries || !idx || !dist) && n)) return fail(ctx, SHERD_E_INVALID, "null argument");
  if (n == 0) return SHERD_OK;
  CtxLock lock(ctx);
  int rc = begin(ctx);
  if (rc) return rc;
  DBuf<double> q, o;
  DBuf<uint32_t> i;
  if ((rc = upload(ctx, q, queries, size_t(3) * n))) return rc;
  CK(o.alloc(n));
  CK(i.alloc(n));
  k_nn_below<<<blocks_for(n, 128), 128, 0, ctx->stream>>>(cloud->view, q.p, n, bound, i.p, o.p,
                                                         ctx->d_status);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(idx, i.p, 4 * size_t(n), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaMemcpyAsync(dist, o.p, 8 * size_t(n), cudaMemcpyDeviceToHost, ctx->stream));
  return finish(ctx, "nearest_below", n, true);
}

int sherd_coarse_scores(sherd_ctx *ctx, const sherd_cloud *target, const double *points,
                        const double *normals, uint32_t n, const double *poses, uint32_t k,
                        double radius, double normal_agree, double *out) {
  if (!ctx || !target || ((!points || !normals) && n) || ((!poses || !out) && k))
    return fail(ctx, SHERD_E_INVALID, "null argument");
  if (!target->view.nrm) return fail(ctx, SHERD_E_INVALID, "the target carries no normals");
  if (k == 0) return SHERD_OK;
  for (uint32_t h = 0; h < k; ++h)
    if (!finite_pose(poses + 16 * size_t(h))) return fail(ctx, SHERD_E_INVALID, "pose is not finite");
  if (n == 0) {
    std::fill(out, out + k, 0.0);
    return SHERD_OK;
  }
  CtxLock lock(ctx);
  int rc = begin(ctx);
  if (rc) return rc;
  DBuf<double> dp, dn, dt, dout;
  if ((rc = upload(ctx, dp, points, size_t(3) * n)) || (rc = upload(ctx, dn, normals, size_t(3) * n)) ||
      (rc = upload(ctx, dt, poses, size_t(16) * k)))
    return rc;
  CK(dout.alloc(k));
  unsigned grid = std::min(blocks_for(size_t(k) * 32, 128), unsigned(ctx->sm_count) * 16u);
  k_coarse_scores<<<grid, 128, 0, ctx->stream>>>(target->view, dp.p, dn.p, n, dt.p, k, radius,
                                                 normal_agree, dout.p, ctx->d_status);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, dout.p, sizeof(double) * k, cudaMemcpyDeviceToHost, ctx->stream));
  return finish(ctx, "coarse_scores", size_t(n) * k, true);
}

// ---- ICP -----------------------------------------------------------------------

int sherd_icp_rung(sherd_ctx *ctx, const double *source, uint32_t n_source, const sherd_cloud *target,
                   const double *inits, uint32_t k, sherd_icp_options options,
                   sherd_registration *out) {
  if (!ctx || !target || ((!inits || !out) && k) || (!source && n_source))
    return fail(ctx, SHERD_E_INVALID, "null argument");
  if (options.estimation != SHERD_POINT_TO_PLANE && options.estimation != SHERD_POINT_TO_POINT)
    return fail(ctx, SHERD_E_INVALID, "unknown estimation");
  if (options.max_iteration < 0) return fail(ctx, SHERD_E_INVALID, "negative iteration cap");
  for (uint32_t c = 0; c < k; ++c)
    if (!finite_pose(inits + 16 * size_t(c))) return fail(ctx, SHERD_E_INVALID, "init pose is not finite");
  if (k == 0) return SHERD_OK;
  CtxLock lock(ctx);
  int rc = begin(ctx);
  if (rc) return rc;
  sherd_cloud src;
  DBuf<double> di;
  DBuf<sherd_registration> dout;
  DBuf<int> hints;
  CK(hints.alloc(std::max<size_t>(1, size_t(n_source) * k)));
  if (n_source) {
    if (has_nan(source, size_t(3) * n_source)) return fail(ctx, SHERD_E_INVALID, "non-finite source point");
    rc = cloud_build(ctx, source, nullptr, n_source, &src);
    if (rc) return rc;
  }
  if ((rc = upload(ctx, di, inits, size_t(16) * k))) return rc;
  CK(dout.alloc(k));
  CK(cudaMemsetAsync(ctx->d_status, 0, 4, ctx->stream));
  CK(cudaEventRecord(ctx->ev0, ctx->stream));
  k_icp_rung<<<k, ICP_BLOCK, 0, ctx->stream>>>(n_source ? src.pts.p : nullptr, n_source, target->view,
                                               di.p, options, hints.p, dout.p, ctx->d_status);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, dout.p, sizeof(sherd_registration) * k, cudaMemcpyDeviceToHost, ctx->stream));
  return finish(ctx, "icp_rung", k, true);
}

int sherd_icp_rung_noalloc(sherd_ctx *ctx, const double *source, uint32_t n_source,
                           const sherd_cloud *target, const double *inits, uint32_t k,
                           sherd_icp_options options, sherd_registration *out) {
  if (!ctx || !target || ((!inits || !out) && k) || (!source && n_source))
    return fail(ctx, SHERD_E_INVALID, "null argument");
  if (options.estimation != SHERD_POINT_TO_PLANE && options.estimation != SHERD_POINT_TO_POINT)
    return fail(ctx, SHERD_E_INVALID, "unknown estimation");
  if (options.max_iteration < 0) return fail(ctx, SHERD_E_INVALID, "negative iteration cap");
  if (uint64_t(k) * n_source > SHERD_NOALLOC_CAPACITY)
    return fail(ctx, SHERD_E_INVALID,
                "k * n_source exceeds SHERD_NOALLOC_CAPACITY (1048576): split the candidates "
                "over several calls or use sherd_icp_rung");
  if ((reinterpret_cast<uintptr_t>(source) & 15u) != 0)
    return fail(ctx, SHERD_E_INVALID, "source must be 16-byte aligned (4 doubles per point)");
  if ((reinterpret_cast<uintptr_t>(inits) & 7u) != 0 || (reinterpret_cast<uintptr_t>(out) & 7u) != 0)
    return fail(ctx, SHERD_E_INVALID, "inits and out must be 8-byte aligned");
  if (k == 0) return SHERD_OK;
  // Every buffer must be memory this context's GPU can address as device memory: a host
  // pointer would fault inside the kernel, so it is refused here, before any launch. The
  // query allocates nothing.
  const void *bufs[3] = {inits, out, n_source ? source : nullptr};
  for (const void *b : bufs) {
    if (!b) continue;
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, b) != cudaSuccess) {
      cudaGetLastError();
      return fail(ctx, SHERD_E_INVALID, "source, inits and out must be device memory");
    }
    bool ok = at.type == cudaMemoryTypeManaged ||
              (at.type == cudaMemoryTypeDevice && at.device == ctx->device);
    if (!ok)
      return fail(ctx, SHERD_E_INVALID,
                  "source, inits and out must be device (or managed) memory of the context's GPU");
  }
  CtxLock lock(ctx);
  int rc = begin(ctx);  // makes the context's device current
  if (rc) return rc;
  // The first call on a device looks the array's address up; that call should
  // come before any stream capture on the device.
  int *hints = nullptr;
  CK(noalloc_address(ctx->device, &hints));
  k_icp_rung<<<k, ICP_BLOCK, 0, ctx->stream>>>(reinterpret_cast<const double4 *>(source), n_source,
                                               target->view, inits, options, hints, out,
                                               ctx->d_status);
  CK(cudaGetLastError());
  return finish(ctx, "icp_rung_noalloc", k, true);
}

// ---- verification ------------------------------------------------------------

int sherd_surfaces_create(sherd_ctx *ctx, const sherd_mesh *fracture, const sherd_mesh *mesh,
                          uint32_t watertight, double frac_area, const double *pf, uint32_t n_pf,
                          const double *s, uint32_t n_s, const double *brk_p, const double *brk_ns,
                          uint32_t n_brk, const double *margin_p, const double *margin_n,
                          uint32_t n_margin, sherd_surfaces **out) {
  if (!ctx || !fracture || !out || (!pf && n_pf) || (!s && n_s) || ((!brk_p || !brk_ns) && n_brk) ||
      ((!margin_p || !margin_n) && n_margin))
    return fail(ctx, SHERD_E_INVALID, "null argument");
  *out = nullptr;
  CtxLock lock(ctx);
  CK(cudaSetDevice(ctx->device));
  sherd_surfaces *x = new sherd_surfaces;
  x->ctx = ctx;
  x->fracture = fracture;
  x->mesh = mesh;
  auto up = [&](DBuf<double> &b, const double *h, uint32_t n) { return upload(ctx, b, h, size_t(3) * n); };
  int rc = 0;
  if ((rc = up(x->brk_p, brk_p, n_brk)) || (rc = up(x->brk_ns, brk_ns, n_brk)) ||
      (rc = up(x->margin_p, margin_p, n_margin)) || (rc = up(x->margin_n, margin_n, n_margin))) {
    delete x;
    return rc;
  }
  // The two query-only sample sets, in Morton order (the LBVH builder's sort).
  if ((n_pf && (rc = cloud_build(ctx, pf, nullptr, n_pf, &x->pf_sorted))) ||
      (n_s && (rc = cloud_build(ctx, s, nullptr, n_s, &x->s_sorted)))) {
    delete x;
    return rc;
  }
  if (n_brk) {
    if ((rc = cloud_build(ctx, brk_p, nullptr, n_brk, &x->brk_tree))) {
      delete x;
      return rc;
    }
    x->has_brk_tree = true;
    x->brk_p_host.assign(brk_p, brk_p + size_t(3) * n_brk);
  }
  if (n_margin) {
    if ((rc = cloud_build(ctx, margin_p, nullptr, n_margin, &x->margin_tree))) {
      delete x;
      return rc;
    }
    x->has_margin_tree = true;
  }
  CK(cudaStreamSynchronize(ctx->stream));
  SurfView &v = x->view;
  v.frac = fracture->view;
  if (mesh) v.mesh = mesh->view;
  v.has_mesh = mesh ? 1u : 0u;
  v.watertight = watertight ? 1u : 0u;
  v.frac_area = frac_area;
  v.pf = n_pf ? x->pf_sorted.pts.p : nullptr;
  v.n_pf = n_pf;
  v.s = n_s ? x->s_sorted.pts.p : nullptr;
  v.n_s = n_s;
  v.brk_p = x->brk_p.p;
  v.brk_ns = x->brk_ns.p;
  v.n_brk = n_brk;
  v.brk_tree = x->brk_tree.view;
  v.margin_p = x->margin_p.p;
  v.margin_n = x->margin_n.p;
  v.n_margin = n_margin;
  v.margin_tree = x->margin_tree.view;
  *out = x;
  return SHERD_OK;
}

int sherd_surfaces_free(sherd_surfaces *s) {
  if (!s) return SHERD_E_INVALID;
  cudaSetDevice(s->ctx->device);
  CtxLock lock(s->ctx);
  delete s;
  return SHERD_OK;
}

void sherd_params_default(sherd_params *p) {
  if (!p) return;
  *p = sherd_params{0.25, 0.03, 0.005, 3.0, 0.8,
                    0.15, 0.06, 0.01, 0.3, 0.12, 0.5, 0.06, 0.5, 0.04,
                    2.3, 0.9, 0.15, 1.0, 0.45, 1.8, 4.0, 0.9, 0.6, 0.0};
}

int sherd_scales_for_pair(const sherd_params *p, double t, double res, sherd_scales *out) {
  if (!p || !out) return SHERD_E_INVALID;
  auto f = [&](double k, double m) { return std::max(k * t, m * res); };
  out->t = t;
  out->res = res;
  out->coarse = f(p->coarse_delta, p->coarse_res);
  out->stage1 = f(p->stage1_delta, p->stage1_res);
  out->tight = f(p->tight_delta, p->tight_res);
  out->facing = f(p->facing_delta, p->facing_res);
  out->gap = f(p->max_gap, p->gap_res);
  out->seam = f(p->seam_delta, p->seam_res);
  out->near = f(p->near_delta, p->near_res);
  out->pen = f(p->pen_delta, p->pen_res);
  out->nms = p->nms_delta * t;
  out->icp = f(p->icp_delta, p->icp_res) / (p->icp_delta * t);
  return SHERD_OK;
}

uint32_t sherd_accept(const sherd_scores *s, const sherd_params *p, const sherd_scales *sc) {
  if (!s || !p || !sc) return 0;
  return (s->tight >= p->min_tight && s->gap * sc->t <= sc->gap && s->pen <= p->max_pen &&
          s->seam >= p->min_seam && s->cont_n >= p->min_cont_n)
             ? 1u
             : 0u;
}

namespace {

int pair_view(sherd_ctx *ctx, const sherd_surfaces *a, const sherd_surfaces *b, const sherd_scales *sc,
              DBuf<uint32_t> &a_cell, PairView &v) {
  v = PairView{};
  v.a = a->view;
  v.b = b->view;
  v.sc = *sc;
  int rc = seam_cells(ctx, a->brk_p_host, sc->t, a_cell, v.n_cells);
  if (rc) return rc;
  v.a_cell = a_cell.p;
  v.scratch_floats = scratch_words(v);
  return SHERD_OK;
}

}  // namespace

int sherd_verify(sherd_ctx *ctx, const sherd_surfaces *a, const sherd_surfaces *b, const double pose[16],
                 const sherd_scales *sc, int full, sherd_scores *out) {
  if (!ctx || !a || !b || !sc || !out) return fail(ctx, SHERD_E_INVALID, "null argument");
  if (!finite_pose(pose)) return fail(ctx, SHERD_E_INVALID, "pose is not finite");
  if (!(sc->t > 0.0)) return fail(ctx, SHERD_E_INVALID, "scales need t > 0");
  CtxLock lock(ctx);
  int rc = begin(ctx);
  if (rc) return rc;
  DBuf<uint32_t> cells;
  PairView v;
  if ((rc = pair_view(ctx, a, b, sc, cells, v))) return rc;
  DBuf<PairView> dv;
  DBuf<sherd_work_item> di;
  DBuf<sherd_candidate> dc;
  DBuf<uint32_t> order;
  DBuf<unsigned> head, scratch;
  sherd_work_item item{};
  std::memcpy(item.init, pose, sizeof item.init);
  sherd_candidate cand{};
  std::memcpy(cand.rungs[3].transform, pose, sizeof cand.rungs[3].transform);
  uint32_t zero = 0;
  if ((rc = upload(ctx, dv, &v, 1)) || (rc = upload(ctx, di, &item, 1)) || (rc = upload(ctx, dc, &cand, 1)) ||
      (rc = upload(ctx, order, &zero, 1)) || (rc = upload(ctx, head, &zero, 1)))
    return rc;
  CK(scratch.alloc(v.scratch_floats));
  QueueCtl q{head.p, order.p, 1, nullptr, 0};
  sherd_params p;
  sherd_params_default(&p);
  k_verify_items<<<1, VER_BLOCK, 0, ctx->stream>>>(dv.p, di.p, q, p, scratch.p, v.scratch_floats, dc.p,
                                                  full, nullptr, 3, 0, ctx->d_status);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(&cand, dc.p, sizeof cand, cudaMemcpyDeviceToHost, ctx->stream));
  rc = finish(ctx, "verify", 1, true);
  if (rc) return rc;
  *out = cand.scores;
  return SHERD_OK;
}

// ---- the batched stage-2 path ---------------------------------------------------

int sherd_pair_create(sherd_ctx *ctx, const sherd_surfaces *a, const sherd_surfaces *b,
                      const sherd_cloud *reg_target, const sherd_cloud *frac_target,
                      const double *reg_source, uint32_t n_reg, const double *frac_source,
                      uint32_t n_frac, const sherd_scales *sc, sherd_pair **out) {
  if (!ctx || !a || !b || !reg_target || !frac_target || !sc || !out || (!reg_source && n_reg) ||
      (!frac_source && n_frac))
    return fail(ctx, SHERD_E_INVALID, "null argument");
  *out = nullptr;
  if (!(sc->t > 0.0)) return fail(ctx, SHERD_E_INVALID, "scales need t > 0");
  if (!reg_target->view.nrm || !frac_target->view.nrm)
    return fail(ctx, SHERD_E_INVALID, "point-to-plane targets need normals");
  if ((n_reg && has_nan(reg_source, size_t(3) * n_reg)) || (n_frac && has_nan(frac_source, size_t(3) * n_frac)))
    return fail(ctx, SHERD_E_INVALID, "non-finite source point");
  CtxLock lock(ctx);
  CK(cudaSetDevice(ctx->device));
  sherd_pair *p = new sherd_pair;
  p->ctx = ctx;
  p->a = a;
  p->b = b;
  int rc = 0;
  // The moving clouds are stored in Morton order (the LBVH builder's sorted
  // points), so a warp's consecutive source points query nearby targets.
  if (n_reg && (rc = cloud_build(ctx, reg_source, nullptr, n_reg, &p->reg_src))) {
    delete p;
    return rc;
  }
  if (n_frac && (rc = cloud_build(ctx, frac_source, nullptr, n_frac, &p->frac_src))) {
    delete p;
    return rc;
  }
  if ((rc = pair_view(ctx, a, b, sc, p->a_cell, p->view))) {
    delete p;
    return rc;
  }
  p->view.reg_tgt = reg_target->view;
  p->view.frac_tgt = frac_target->view;
  p->view.reg_src = n_reg ? p->reg_src.pts.p : nullptr;
  p->view.n_reg = n_reg;
  p->view.frac_src = n_frac ? p->frac_src.pts.p : nullptr;
  p->view.n_frac = n_frac;
  CK(cudaStreamSynchronize(ctx->stream));
  *out = p;
  return SHERD_OK;
}

int sherd_pair_free(sherd_pair *pair) {
  if (!pair) return SHERD_E_INVALID;
  cudaSetDevice(pair->ctx->device);
  CtxLock lock(pair->ctx);
  delete pair;
  return SHERD_OK;
}

}  // extern "C"

struct sherd_batch {
  sherd_ctx *ctx = nullptr;
  int sched = SHERD_SCHED_BATCHED;
  uint32_t n_pairs = 0, n_items = 0;
  sherd_params params{};
  std::vector<uint32_t> pair_first, pair_count;  // queue segments of the plain schedule
  DBuf<PairView> dv;
  DBuf<sherd_work_item> di;
  DBuf<sherd_candidate> dc;
  DBuf<uint32_t> dorder;
  DBuf<unsigned> heads, scratch;
  // Per ladder CTA, each source point's last match: 16 bits when every target
  // of the batch has fewer than 65535 points, else an int.
  DBuf<unsigned char> hints;
  bool hint16 = true;
  size_t hint_stride = 1;
  // Launches k_ladder variant v (rungs r_lo..r_hi-1) with the batch's hint
  // width, its CTAs using the hint slots from slot0 on.
  template <class H, int MINB>
  void ladder_as(unsigned grid, QueueCtl q, cudaStream_t s, int r_lo, int r_hi, int skip_partial,
                 size_t slot0) {
    H *h = reinterpret_cast<H *>(hints.p) + slot0 * hint_stride;
    k_ladder<H, MINB><<<grid, ICP_BLOCK, 0, s>>>(dv.p, di.p, q, h, hint_stride, dc.p, r_lo, r_hi,
                                                 skip_partial, ctx->d_status);
  }
  template <class H>
  void ladder_h(int v, unsigned grid, QueueCtl q, cudaStream_t s, int r_lo, int r_hi,
                int skip_partial, size_t slot0) {
    if (v == 0)
      ladder_as<H, LADDER_MINB[0]>(grid, q, s, r_lo, r_hi, skip_partial, slot0);
    else if (v == 1)
      ladder_as<H, LADDER_MINB[1]>(grid, q, s, r_lo, r_hi, skip_partial, slot0);
    else
      ladder_as<H, LADDER_MINB[2]>(grid, q, s, r_lo, r_hi, skip_partial, slot0);
  }
  void ladder(unsigned grid, QueueCtl q, cudaStream_t s, int r_lo, int r_hi, int skip_partial,
              int v = LADDER_DEFAULT, size_t slot0 = 0) {
    if (hint16)
      ladder_h<uint16_t>(v, grid, q, s, r_lo, r_hi, skip_partial, slot0);
    else
      ladder_h<int>(v, grid, q, s, r_lo, r_hi, skip_partial, slot0);
  }
  // The ladder's point-count buckets (largest moving clouds first): each is a
  // segment of the queue order, run by its own k_ladder variant (chosen by the
  // autotuner) on a grid of its own, its CTAs on a slice of the hint slots.
  static constexpr int BUCKETS = 3;
  uint32_t seg_first[BUCKETS] = {}, seg_count[BUCKETS] = {};
  int variant[BUCKETS] = {LADDER_DEFAULT, LADDER_DEFAULT, LADDER_DEFAULT};
  size_t slot0[BUCKETS] = {};
  int occ[LADDER_VARIANTS] = {};  // resident k_ladder CTAs per SM of each variant
  DBuf<unsigned> lheads;          // one queue head per bucket
  unsigned bucket_grid(int b) const {
    return std::max(1u, std::min<unsigned>(unsigned(std::max(1, occ[variant[b]]) * ctx->sm_count),
                                           seg_count[b]));
  }
  bool early() const { return params.early_reject_tight > 0.0; }
  // Queue heads per group of items (the whole batch, or one pair of the plain
  // schedule): ladder, verification, early-rejection check, fine ladder.
  static constexpr int HEADS = 4;
  // The penetration wavefront: per item the inverse pose, per (item, side)
  // unit its counters and its first chunk.
  DBuf<double> inv;
  DBuf<unsigned> deeper, deep, best, pen_heads;
  DBuf<uint32_t> chunk0, coarse;
  uint32_t n_chunks = 0;
  unsigned grid_p = 1, grid_m = 1;
  unsigned grid_l = 1, grid_v = 1;
  uint32_t max_scratch = 64;
  static constexpr int STAGES = 5;  // ladder, verify, pen inside, pen min, finalize
  cudaGraph_t graph[STAGES] = {};
  cudaGraphExec_t exec[STAGES] = {};
  uint32_t captured_timeout = 0xFFFFFFFFu;
  cudaEvent_t ev[STAGES + 1] = {};
  ~sherd_batch() {
    for (int k = 0; k < STAGES; ++k) {
      if (exec[k]) cudaGraphExecDestroy(exec[k]);
      if (graph[k]) cudaGraphDestroy(graph[k]);
    }
    for (cudaEvent_t e : ev)
      if (e) cudaEventDestroy(e);
  }
};

namespace {

// The batched schedule as five graphs, one per stage, so that the host can put
// an event between them and every stage's device time is known: the queue
// reset and the persistent ladder kernel; the persistent fracture, seam and
// continuity kernel; the penetration box/parity/depth wavefront; its minimum
// pass; the finalising pass.
// The ladder stage of one group of items (`order[0..n)`, queues at `heads`):
// the four rungs, or, with R 5.6's early rejection, the two pc_reg rungs, the
// fracture and seam scores at rung 1, the marking, and the two pc_frac rungs
// of the items that go on (pair.rs:309-346).
int ladder_stage(sherd_batch *b, cudaStream_t s, unsigned *heads, const uint32_t *order,
                 uint32_t n, unsigned grid) {
  sherd_ctx *ctx = b->ctx;
  unsigned long long budget = (unsigned long long)ctx->timeout_ms * 1000000ULL;
  const bool early = b->early();
  QueueCtl q0{heads, order, n, ctx->abort_dev, budget};
  b->ladder(grid, q0, s, 0, early ? 2 : 4, 0);
  CK(cudaGetLastError());
  if (early) {
    QueueCtl q1{heads + 2, order, n, ctx->abort_dev, budget};
    k_verify_items<<<std::min<unsigned>(b->grid_v, n), VER_BLOCK, 0, s>>>(
        b->dv.p, b->di.p, q1, b->params, b->scratch.p, b->max_scratch, b->dc.p, 0, nullptr, 1, 0,
        ctx->d_status);
    k_early_mark<<<blocks_for(n), 256, 0, s>>>(b->dc.p, order, n, b->params.early_reject_tight);
    CK(cudaGetLastError());
    QueueCtl q2{heads + 3, order, n, ctx->abort_dev, budget};
    b->ladder(grid, q2, s, 2, 4, 1);
    CK(cudaGetLastError());
  }
  return SHERD_OK;
}

// The ladder stage of the batched schedule: one k_ladder launch per
// point-count bucket, the three side by side (the caller's stream and the
// context's two side streams, forked and joined by events, which a stream
// capture records as graph edges), so the buckets share the SMs as one queue
// would. With R 5.6's early rejection the stage stays one queue.
int launch_ladder(sherd_batch *b, cudaStream_t s) {
  sherd_ctx *ctx = b->ctx;
  CK(cudaMemsetAsync(b->heads.p, 0, sherd_batch::HEADS * sizeof(unsigned), s));
  if (b->early())
    return ladder_stage(b, s, b->heads.p, b->dorder.p, b->n_items,
                        std::min<unsigned>(b->grid_l, b->n_items));
  unsigned long long budget = (unsigned long long)ctx->timeout_ms * 1000000ULL;
  CK(cudaMemsetAsync(b->lheads.p, 0, sherd_batch::BUCKETS * sizeof(unsigned), s));
  CK(cudaEventRecord(ctx->fork_ev, s));
  for (int k = 0; k < 2; ++k) CK(cudaStreamWaitEvent(ctx->side[k], ctx->fork_ev, 0));
  for (int bk = 0; bk < sherd_batch::BUCKETS; ++bk) {
    if (!b->seg_count[bk]) continue;
    cudaStream_t on = bk == 0 ? s : ctx->side[bk - 1];
    QueueCtl q{b->lheads.p + bk, b->dorder.p + b->seg_first[bk], b->seg_count[bk], ctx->abort_dev,
               budget};
    b->ladder(b->bucket_grid(bk), q, on, 0, 4, 0, b->variant[bk], b->slot0[bk]);
    CK(cudaGetLastError());
  }
  for (int k = 0; k < 2; ++k) {
    CK(cudaEventRecord(ctx->join_ev[k], ctx->side[k]));
    CK(cudaStreamWaitEvent(s, ctx->join_ev[k], 0));
  }
  return SHERD_OK;
}

// The ladder autotuner: for each point-count bucket with enough items that the
// context has not tuned yet, every k_ladder variant runs the four rungs of the
// bucket's most expensive items (two full grids' worth, the same items for
// every variant, after one untimed run), twice, timed by CUDA events on the
// context's stream; a variant replaces the default (LADDER_DEFAULT) only when
// its faster run beats the default's by TUNE_MARGIN, so
// run-to-run noise does not move the choice. The choice is kept for the bucket
// on this context. The runs write those items' rungs, which every batch run
// writes again.
constexpr float TUNE_MARGIN = 0.05f;
int tune_ladder(sherd_batch *b) {
  sherd_ctx *ctx = b->ctx;
  cudaStream_t s = ctx->stream;
  int max_occ = 1;
  for (int v = 0; v < LADDER_VARIANTS; ++v) max_occ = std::max(max_occ, b->occ[v]);
  for (int bk = 0; bk < sherd_batch::BUCKETS; ++bk) {
    if (ctx->ladder_tuned[bk] >= 0) {
      b->variant[bk] = ctx->ladder_tuned[bk];
      continue;
    }
    const uint32_t need = 2u * uint32_t(max_occ) * uint32_t(ctx->sm_count);
    if (b->seg_count[bk] < need) continue;  // too few items to tell the variants apart
    float ms_of[LADDER_VARIANTS];
    for (int k = 0; k < LADDER_VARIANTS; ++k) ms_of[k] = f_inf();
    for (int t = -1; t < 2 * LADDER_VARIANTS; ++t) {
      const int v = t < 0 ? -1 : t % LADDER_VARIANTS;
      const int run = v < 0 ? LADDER_DEFAULT : v;
      const unsigned grid = std::min<unsigned>(unsigned(b->occ[run] * ctx->sm_count), need);
      QueueCtl q{b->lheads.p + bk, b->dorder.p + b->seg_first[bk], need, ctx->abort_dev, 0ull};
      CK(cudaMemsetAsync(b->lheads.p + bk, 0, sizeof(unsigned), s));
      CK(cudaEventRecord(ctx->ev0, s));
      b->ladder(grid, q, s, 0, 4, 0, run, b->slot0[bk]);
      CK(cudaGetLastError());
      CK(cudaEventRecord(ctx->ev1, s));
      CK(cudaStreamSynchronize(s));
      float ms = 0.0f;
      CK(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
      if (v < 0) continue;  // the untimed first run
      ms_of[v] = std::min(ms_of[v], ms);
    }
    int pick = LADDER_DEFAULT;
    for (int v = 0; v < LADDER_VARIANTS; ++v) {
      ctx->ladder_tune_ms[bk][v] = ms_of[v];
      if (ms_of[v] < ms_of[pick] && ms_of[v] < (1.0f - TUNE_MARGIN) * ms_of[LADDER_DEFAULT])
        pick = v;
    }
    ctx->ladder_tuned[bk] = pick;
    ctx->ladder_tune_items[bk] = need;
    b->variant[bk] = pick;
  }
  return SHERD_OK;
}

int launch_verify_items(sherd_batch *b, cudaStream_t s) {
  sherd_ctx *ctx = b->ctx;
  unsigned long long budget = (unsigned long long)ctx->timeout_ms * 1000000ULL;
  QueueCtl qv{b->heads.p + 1, b->dorder.p, b->n_items, ctx->abort_dev, budget};
  k_verify_items<<<std::min<unsigned>(b->grid_v, b->n_items), VER_BLOCK, 0, s>>>(
      b->dv.p, b->di.p, qv, b->params, b->scratch.p, b->max_scratch, b->dc.p, 1, b->inv.p, 3,
      b->early() ? 1 : 0, ctx->d_status);
  CK(cudaGetLastError());
  return SHERD_OK;
}

PenState pen_state(sherd_batch *b) {
  return PenState{b->deeper.p, b->deep.p, b->best.p, b->chunk0.p, b->coarse.p, 2 * b->n_items,
                  b->n_chunks};
}

int launch_pen_inside(sherd_batch *b, cudaStream_t s) {
  sherd_ctx *ctx = b->ctx;
  unsigned long long budget = (unsigned long long)ctx->timeout_ms * 1000000ULL;
  PenState ps = pen_state(b);
  CK(cudaMemsetAsync(b->pen_heads.p, 0, 2 * sizeof(unsigned), s));
  k_pen_init<<<blocks_for(ps.n_units), 256, 0, s>>>(ps);
  CK(cudaGetLastError());
  if (b->n_chunks) {
    k_pen_inside<<<b->grid_p, 256, 0, s>>>(b->dv.p, b->di.p, b->dc.p, b->inv.p, ps, b->pen_heads.p,
                                         ctx->abort_dev, budget, ctx->d_status);
    CK(cudaGetLastError());
  }
  return SHERD_OK;
}

int launch_pen_min(sherd_batch *b, cudaStream_t s) {
  sherd_ctx *ctx = b->ctx;
  unsigned long long budget = (unsigned long long)ctx->timeout_ms * 1000000ULL;
  PenState ps = pen_state(b);
  if (b->n_chunks) {
    k_pen_seed<<<blocks_for(size_t(ps.n_units) * 32), 256, 0, s>>>(b->dv.p, b->di.p, b->dc.p,
                                                                  b->inv.p, ps, ctx->d_status);
    CK(cudaGetLastError());
    k_pen_min<<<b->grid_m, 256, 0, s>>>(b->dv.p, b->di.p, b->dc.p, b->inv.p, ps,
                                      b->pen_heads.p + 1, ctx->abort_dev, budget, ctx->d_status);
    CK(cudaGetLastError());
  }
  return SHERD_OK;
}

int launch_finalize(sherd_batch *b, cudaStream_t s) {
  sherd_ctx *ctx = b->ctx;
  k_pen_finalize<<<blocks_for(b->n_items), 256, 0, s>>>(b->dv.p, b->di.p, b->dc.p, pen_state(b),
                                                       b->params, b->n_items);
  CK(cudaGetLastError());
  return SHERD_OK;
}

int capture_one(sherd_batch *b, int (*launch)(sherd_batch *, cudaStream_t), cudaGraph_t &graph,
                cudaGraphExec_t &exec) {
  sherd_ctx *ctx = b->ctx;
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  exec = nullptr;
  graph = nullptr;
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  sherd_ctx *held = t_alloc_ctx;  // no pool calls recorded into the graph
  t_alloc_ctx = nullptr;
  int rc = launch(b, ctx->stream);
  t_alloc_ctx = held;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamEndCapture");
  graph = g;
  CK(cudaGraphInstantiate(&exec, graph, 0));
  return SHERD_OK;
}

// Captures every stage's graph (again when the time budget changed).
int capture(sherd_batch *b) {
  if (b->exec[0] && b->captured_timeout == b->ctx->timeout_ms) return SHERD_OK;
  int (*stage[sherd_batch::STAGES])(sherd_batch *, cudaStream_t) = {
      launch_ladder, launch_verify_items, launch_pen_inside, launch_pen_min, launch_finalize};
  for (int k = 0; k < sherd_batch::STAGES; ++k) {
    int rc = capture_one(b, stage[k], b->graph[k], b->exec[k]);
    if (rc) return rc;
  }
  b->captured_timeout = b->ctx->timeout_ms;
  return SHERD_OK;
}

int batch_create(sherd_ctx *ctx, sherd_pair *const *pairs, uint32_t n_pairs,
                 const sherd_work_item *items, uint32_t n_items, const sherd_params *p, int sched,
                 sherd_batch *b) {
  b->ctx = ctx;
  b->sched = sched;
  b->n_pairs = n_pairs;
  b->n_items = n_items;
  b->params = *p;
  // Longest items first: the ladder's point iterations and the sample counts
  // of the verification, per pair.
  std::vector<double> pair_cost(n_pairs);
  for (uint32_t i = 0; i < n_pairs; ++i) {
    const PairView &v = pairs[i]->view;
    pair_cost[i] = 60.0 * (double(v.n_reg) + double(v.n_frac)) + 4.0 * (v.a.n_s + v.b.n_s) +
                   double(v.a.n_pf + v.b.n_pf);
    b->max_scratch = std::max(b->max_scratch, v.scratch_floats);
    b->hint_stride = std::max<size_t>(b->hint_stride, std::max(v.n_reg, v.n_frac));
    if (v.reg_tgt.n >= 0xFFFFu || v.frac_tgt.n >= 0xFFFFu) b->hint16 = false;
  }
  std::vector<PairView> views(n_pairs);
  for (uint32_t i = 0; i < n_pairs; ++i) views[i] = pairs[i]->view;
  std::vector<uint32_t> order(n_items);
  if (sched == SHERD_SCHED_BATCHED) {
    // By point-count bucket of the moving clouds (> 16384, > 4096, the rest),
    // then longest items first within each.
    auto bucket = [&](uint32_t pair) {
      uint32_t m = std::max(views[pair].n_reg, views[pair].n_frac);
      return m > 16384u ? 0 : (m > 4096u ? 1 : 2);
    };
    for (uint32_t i = 0; i < n_items; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
      int bx = bucket(items[x].pair), by = bucket(items[y].pair);
      if (bx != by) return bx < by;
      return pair_cost[items[x].pair] > pair_cost[items[y].pair];
    });
    for (uint32_t k = 0; k < n_items; ++k) b->seg_count[bucket(items[order[k]].pair)]++;
    for (int bk = 1; bk < sherd_batch::BUCKETS; ++bk)
      b->seg_first[bk] = b->seg_first[bk - 1] + b->seg_count[bk - 1];
  } else {
    b->pair_first.assign(n_pairs, 0);
    b->pair_count.assign(n_pairs, 0);
    for (uint32_t i = 0; i < n_items; ++i) b->pair_count[items[i].pair]++;
    uint32_t acc = 0;
    for (uint32_t i = 0; i < n_pairs; ++i) {
      b->pair_first[i] = acc;
      acc += b->pair_count[i];
    }
    std::vector<uint32_t> fill(b->pair_first);
    for (uint32_t i = 0; i < n_items; ++i) order[fill[items[i].pair]++] = i;
  }
  int rc;
  if ((rc = upload(ctx, b->dv, views.data(), n_pairs)) || (rc = upload(ctx, b->di, items, n_items)) ||
      (rc = upload(ctx, b->dorder, order.data(), n_items)))
    return rc;
  CK(b->dc.alloc(n_items));
  CK(cudaMemsetAsync(b->dc.p, 0, sizeof(sherd_candidate) * n_items, ctx->stream));
  CK(b->heads.alloc(sherd_batch::HEADS * size_t(std::max<uint32_t>(n_pairs, 1))));
  int occ_v = 0;
  if (b->hint16) {
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->occ[0], k_ladder<uint16_t, LADDER_MINB[0]>, ICP_BLOCK, 0));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->occ[1], k_ladder<uint16_t, LADDER_MINB[1]>, ICP_BLOCK, 0));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->occ[2], k_ladder<uint16_t, LADDER_MINB[2]>, ICP_BLOCK, 0));
  } else {
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->occ[0], k_ladder<int, LADDER_MINB[0]>, ICP_BLOCK, 0));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->occ[1], k_ladder<int, LADDER_MINB[1]>, ICP_BLOCK, 0));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->occ[2], k_ladder<int, LADDER_MINB[2]>, ICP_BLOCK, 0));
  }
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_v, k_verify_items, VER_BLOCK, 0));
  b->grid_l = unsigned(std::max(1, b->occ[LADDER_DEFAULT]) * ctx->sm_count);
  b->grid_v = unsigned(std::max(1, occ_v) * ctx->sm_count);
  CK(b->scratch.alloc(size_t(b->grid_v) * b->max_scratch));
  if (sched == SHERD_SCHED_BATCHED) {
    // Unit 2i is item i's side 0 (B's samples in A's mesh), 2i+1 its side 1.
    std::vector<uint32_t> chunk0(2 * size_t(n_items) + 1);
    uint64_t acc = 0;
    for (uint32_t i = 0; i < n_items; ++i) {
      const PairView &v = views[items[i].pair];
      bool avail = v.a.has_mesh && v.b.has_mesh && v.a.watertight && v.b.watertight;
      uint32_t ns[2] = {v.b.n_s, v.a.n_s};
      for (int side = 0; side < 2; ++side) {
        chunk0[2 * size_t(i) + side] = uint32_t(acc);
        if (avail) acc += (ns[side] + 31u) / 32u;
      }
    }
    if (acc >= 0xFFFFFFFFull) return fail(ctx, SHERD_E_INVALID, "batch too large for one wavefront");
    chunk0[2 * size_t(n_items)] = uint32_t(acc);
    b->n_chunks = uint32_t(acc);
    if ((rc = upload(ctx, b->chunk0, chunk0.data(), chunk0.size()))) return rc;
    // The unit of every 256th chunk: the last unit starting at or before it.
    std::vector<uint32_t> coarse((size_t(acc) >> 8) + 1);
    uint32_t cu = 0;
    for (size_t k = 0; k < coarse.size(); ++k) {
      uint64_t c = uint64_t(k) << 8;
      while (cu + 1 < 2 * n_items && chunk0[cu + 1] <= c) ++cu;
      coarse[k] = cu;
    }
    if ((rc = upload(ctx, b->coarse, coarse.data(), coarse.size()))) return rc;
    CK(b->inv.alloc(16 * size_t(n_items)));
    CK(b->deeper.alloc(2 * size_t(n_items)));
    CK(b->deep.alloc(2 * size_t(n_items)));
    CK(b->best.alloc(2 * size_t(n_items)));
    CK(b->pen_heads.alloc(2));
    int occ_p = 0, occ_m = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_p, k_pen_inside, 256, 0));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_m, k_pen_min, 256, 0));
    b->grid_p = unsigned(std::max(1, occ_p) * ctx->sm_count);
    b->grid_m = unsigned(std::max(1, occ_m) * ctx->sm_count);
  }
  b->hint_stride = (b->hint_stride + 63) / 64 * 64;
  // The plain schedule launches one CTA per item of a pair, so it needs as many
  // hint slots as the largest pair has items.
  size_t slots = b->grid_l;
  for (uint32_t c : b->pair_count) slots = std::max<size_t>(slots, c);
  if (sched == SHERD_SCHED_BATCHED) {
    // The buckets' launches run side by side, each on its own slice of slots,
    // as wide as the largest grid any variant could take.
    int max_occ = 1;
    for (int v = 0; v < LADDER_VARIANTS; ++v) max_occ = std::max(max_occ, b->occ[v]);
    size_t acc = 0;
    for (int bk = 0; bk < sherd_batch::BUCKETS; ++bk) {
      b->slot0[bk] = acc;
      acc += std::min<size_t>(size_t(max_occ) * ctx->sm_count, b->seg_count[bk]);
    }
    slots = std::max(slots, acc);
    CK(b->lheads.alloc(sherd_batch::BUCKETS));
  }
  CK(b->hints.alloc(slots * b->hint_stride * (b->hint16 ? sizeof(uint16_t) : sizeof(int))));
  for (cudaEvent_t &e : b->ev) CK(cudaEventCreate(&e));
  CK(cudaStreamSynchronize(ctx->stream));
  if (sched == SHERD_SCHED_BATCHED) {
    if (!b->early() && (rc = tune_ladder(b))) return rc;
    return capture(b);
  }
  return SHERD_OK;
}

int batch_run(sherd_batch *b, float *ms) {
  sherd_ctx *ctx = b->ctx;
  __atomic_store_n(ctx->abort_host, 0u, __ATOMIC_SEQ_CST);
  int rc = begin(ctx);
  if (rc) return rc;
  cudaStream_t s = ctx->stream;
  NvtxRange range(b->sched == SHERD_SCHED_BATCHED ? "sherd batch (batched)" : "sherd batch (plain)");
  if (b->sched == SHERD_SCHED_BATCHED) {
    static const char *const kStage[sherd_batch::STAGES] = {
        "sherd stage ladder", "sherd stage verify", "sherd stage pen_inside", "sherd stage pen_min",
        "sherd stage finalize"};
    if ((rc = capture(b))) return rc;
    CK(cudaEventRecord(b->ev[0], s));
    for (int k = 0; k < sherd_batch::STAGES; ++k) {
      NvtxRange stage(kStage[k]);
      CK(cudaGraphLaunch(b->exec[k], s));
      CK(cudaEventRecord(b->ev[k + 1], s));
    }
  } else {
    unsigned long long budget = (unsigned long long)ctx->timeout_ms * 1000000ULL;
    CK(cudaMemsetAsync(b->heads.p, 0, sizeof(unsigned) * sherd_batch::HEADS * b->n_pairs, s));
    CK(cudaEventRecord(b->ev[0], s));
    for (uint32_t i = 0; i < b->n_pairs; ++i) {
      uint32_t cnt = b->pair_count[i];
      if (!cnt) continue;
      unsigned *heads = b->heads.p + sherd_batch::HEADS * size_t(i);
      const uint32_t *order = b->dorder.p + b->pair_first[i];
      if ((rc = ladder_stage(b, s, heads, order, cnt, cnt))) return rc;
      QueueCtl qv{heads + 1, order, cnt, ctx->abort_dev, budget};
      k_verify_items<<<std::min<unsigned>(cnt, b->grid_v), VER_BLOCK, 0, s>>>(
          b->dv.p, b->di.p, qv, b->params, b->scratch.p, b->max_scratch, b->dc.p, 1, nullptr, 3,
          b->early() ? 1 : 0, ctx->d_status);
      CK(cudaGetLastError());
      CK(cudaStreamSynchronize(s));
    }
    CK(cudaEventRecord(b->ev[sherd_batch::STAGES], s));
  }
  rc = finish(ctx, b->sched == SHERD_SCHED_BATCHED ? "batch_batched" : "batch_plain", b->n_items,
              true);
  if (ms) {
    for (int k = 0; k < SHERD_BATCH_TIMES; ++k) ms[k] = -1.0f;
    cudaEventElapsedTime(&ms[SHERD_BATCH_TIMES - 1], b->ev[0], b->ev[sherd_batch::STAGES]);
    if (b->sched == SHERD_SCHED_BATCHED)
      for (int k = 0; k < sherd_batch::STAGES; ++k)
        cudaEventElapsedTime(&ms[k], b->ev[k], b->ev[k + 1]);
    cudaGetLastError();
  }
  return rc;
}

int check_batch_args(sherd_ctx *ctx, sherd_pair *const *pairs, uint32_t n_pairs,
                     const sherd_work_item *items, uint32_t n_items, const sherd_params *p, int sched) {
  if (!ctx || !p || ((!pairs) && n_pairs) || ((!items) && n_items))
    return fail(ctx, SHERD_E_INVALID, "null argument");
  if (sched != SHERD_SCHED_BATCHED && sched != SHERD_SCHED_PLAIN)
    return fail(ctx, SHERD_E_INVALID, "unknown schedule");
  for (uint32_t i = 0; i < n_pairs; ++i)
    if (!pairs[i] || pairs[i]->ctx != ctx) return fail(ctx, SHERD_E_INVALID, "pair of another context");
  for (uint32_t i = 0; i < n_items; ++i) {
    if (items[i].pair >= n_pairs) return fail(ctx, SHERD_E_INVALID, "work item names no pair");
    if (!finite_pose(items[i].init)) return fail(ctx, SHERD_E_INVALID, "work item pose is not finite");
  }
  return SHERD_OK;
}

}  // namespace

extern "C" {

int sherd_batch_create(sherd_ctx *ctx, sherd_pair *const *pairs, uint32_t n_pairs,
                       const sherd_work_item *items, uint32_t n_items, const sherd_params *p,
                       int sched, sherd_batch **out) {
  if (!out) return fail(ctx, SHERD_E_INVALID, "null argument");
  *out = nullptr;
  int rc = check_batch_args(ctx, pairs, n_pairs, items, n_items, p, sched);
  if (rc) return rc;
  if (n_items == 0) return fail(ctx, SHERD_E_EMPTY, "a batch needs at least one work item");
  CtxLock lock(ctx);
  CK(cudaSetDevice(ctx->device));
  sherd_batch *b = new sherd_batch;
  rc = batch_create(ctx, pairs, n_pairs, items, n_items, p, sched, b);
  if (rc) {
    delete b;
    return rc;
  }
  *out = b;
  return SHERD_OK;
}

int sherd_batch_run(sherd_batch *batch, float ms[SHERD_BATCH_TIMES]) {
  if (!batch) return SHERD_E_INVALID;
  CtxLock lock(batch->ctx);
  return batch_run(batch, ms);
}

int sherd_batch_results(sherd_batch *batch, sherd_candidate *out) {
  if (!batch || !out) return SHERD_E_INVALID;
  sherd_ctx *ctx = batch->ctx;
  CtxLock lock(ctx);
  CK(cudaSetDevice(ctx->device));
  CK(cudaMemcpyAsync(out, batch->dc.p, sizeof(sherd_candidate) * batch->n_items,
                     cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return SHERD_OK;
}

int sherd_batch_free(sherd_batch *batch) {
  if (!batch) return SHERD_E_INVALID;
  cudaSetDevice(batch->ctx->device);
  CtxLock lock(batch->ctx);
  delete batch;
  return SHERD_OK;
}

int sherd_ladder_verify_batch(sherd_ctx *ctx, sherd_pair *const *pairs, uint32_t n_pairs,
                              const sherd_work_item *items, uint32_t n_items, const sherd_params *p,
                              int sched, sherd_candidate *out) {
  int rc = check_batch_args(ctx, pairs, n_pairs, items, n_items, p, sched);
  if (rc) return rc;
  if (n_items == 0) return SHERD_OK;
  if (!out) return fail(ctx, SHERD_E_INVALID, "null argument");
  CtxLock lock(ctx);
  CK(cudaSetDevice(ctx->device));
  sherd_batch b;
  if ((rc = batch_create(ctx, pairs, n_pairs, items, n_items, p, sched, &b))) return rc;
  if ((rc = batch_run(&b, nullptr))) return rc;
  CK(cudaMemcpyAsync(out, b.dc.p, sizeof(sherd_candidate) * n_items, cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return SHERD_OK;
}

// ---- differentiation ----------------------------------------------------------

int sherd_adjoint(sherd_ctx *ctx, sherd_pair *const *edges, uint32_t n_edges, const double *poses,
                  const double *inverses, uint32_t n_poses, const sherd_adjoint_options *opt,
                  double *values, double *grads) {
  if (!ctx || !opt) return fail(ctx, SHERD_E_INVALID, "null argument");
  if (n_edges == 0 || n_poses == 0) return SHERD_OK;
  if (!edges || !poses || !inverses || !values || !grads)
    return fail(ctx, SHERD_E_INVALID, "null argument");
  if (!(opt->radius_k > 0.0) || !(opt->width_k > 0.0) || !(opt->window_k >= 0.0) ||
      !std::isfinite(opt->radius_k) || !std::isfinite(opt->width_k) || !std::isfinite(opt->window_k))
    return fail(ctx, SHERD_E_INVALID, "adjoint options must be finite and positive");
  size_t n_pe = size_t(n_poses) * n_edges;
  if (n_pe * 3 > size_t(1u << 31) - 1) return fail(ctx, SHERD_E_INVALID, "too many (pose, edge) units");
  for (size_t i = 0; i < n_pe; ++i)
    if (!finite_pose(poses + 16 * i) || !finite_pose(inverses + 16 * i))
      return fail(ctx, SHERD_E_INVALID, "pose is not finite");
  std::vector<PairView> views(n_edges);
  for (uint32_t e = 0; e < n_edges; ++e) {
    if (!edges[e] || edges[e]->ctx != ctx) return fail(ctx, SHERD_E_INVALID, "edge of another context");
    views[e] = edges[e]->view;
    if (!views[e].frac_tgt.nrm) return fail(ctx, SHERD_E_INVALID, "edge target without normals");
  }
  CtxLock lock(ctx);
  NvtxRange range("sherd adjoint");
  int rc = begin(ctx);
  if (rc) return rc;
  DBuf<PairView> dv;
  DBuf<double> dp, di, dval, dgrad;
  if ((rc = upload(ctx, dv, views.data(), views.size())) ||
      (rc = upload(ctx, dp, poses, 16 * n_pe)) || (rc = upload(ctx, di, inverses, 16 * n_pe)))
    return rc;
  CK(dval.alloc(n_pe * ADJ_VALUES));
  CK(dgrad.alloc(n_pe * ADJ_VALUES * 6));
  AdjointConsts kc{opt->radius_k, opt->width_k, opt->window_k};
  k_adjoint<<<unsigned(n_pe * 3), ADJ_BLOCK, 0, ctx->stream>>>(dv.p, n_edges, dp.p, di.p, kc, dval.p,
                                                              dgrad.p, ctx->d_status);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(values, dval.p, sizeof(double) * n_pe * ADJ_VALUES, cudaMemcpyDeviceToHost,
                     ctx->stream));
  CK(cudaMemcpyAsync(grads, dgrad.p, sizeof(double) * n_pe * ADJ_VALUES * 6,
                     cudaMemcpyDeviceToHost, ctx->stream));
  return finish(ctx, "adjoint", n_pe, true);
}

// ---- segmentation ---------------------------------------------------------------

void sherd_seg_params_default(sherd_seg_params *out) {
  if (!out) return;
  *out = sherd_seg_params{};
  out->smooth_res = 0.0;
  out->coarse_at = 0.1;
  out->boundary_angle = 25.0;
  out->votes = 5;
  out->votes_coarse = 4;
  out->smoothed_hit_normal = 0;
  out->boundary_angle_auto = 0;
}

}  // extern "C"

namespace {

// drop_small_components (components.rs:170-191) on the device mask.
int drop_small(sherd_ctx *ctx, DBuf<uint8_t> &mask, uint8_t target, double min_area,
               const DBuf<uint32_t> &fa, const DBuf<uint32_t> &fb, uint32_t n_pairs,
               const DBuf<double> &areas, uint32_t nf) {
  cudaStream_t s = ctx->stream;
  DBuf<uint32_t> parent, root, face, root2, face2;
  DBuf<double> size;
  CK(parent.alloc(nf));
  CK(root.alloc(nf));
  CK(face.alloc(nf));
  CK(root2.alloc(nf));
  CK(face2.alloc(nf));
  CK(size.alloc(nf));
  k_uf_init<<<blocks_for(nf), 256, 0, s>>>(parent.p, nf);
  k_uf_union<<<std::max(1u, std::min(blocks_for(n_pairs), unsigned(ctx->sm_count) * 16u)), 256, 0,
               s>>>(fa.p, fb.p, n_pairs, mask.p, target, parent.p, ctx->d_status);
  k_uf_roots<<<blocks_for(nf), 256, 0, s>>>(parent.p, mask.p, target, nf, root.p, face.p);
  CK(cudaGetLastError());
  int rc = radix_sort_pairs(ctx, root.p, root2.p, face.p, face2.p, nf, 32);
  if (rc) return rc;
  k_component_areas<<<blocks_for(nf), 256, 0, s>>>(root2.p, face2.p, nf, areas.p, size.p);
  k_drop_small<<<blocks_for(nf), 256, 0, s>>>(mask.p, target, nf, parent.p, size.p, min_area);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s));
  return SHERD_OK;
}

// One radius-ball pass over every representative (k_ball), its shared memory
// sized to the largest ball by a counting pass (k_ball_size).
int ball_pass(sherd_ctx *ctx, const CloudView &all, const double *cent, const uint32_t *rep,
              uint32_t n_rep, double radius, int mode, const double *normals, const double *areas,
              const uint8_t *frac, double *out3, uint8_t *flag) {
  cudaStream_t s = ctx->stream;
  const unsigned grid = std::max(1u, std::min(n_rep, unsigned(ctx->sm_count) * 16u));
  DBuf<uint32_t> mx;
  CK(mx.alloc(2));
  CK(cudaMemsetAsync(mx.p, 0, 8, s));
  k_ball_size<<<std::min(blocks_for(n_rep, 128), unsigned(ctx->sm_count) * 8u), 128, 0, s>>>(
      all, cent, rep, n_rep, radius, mode, frac, mx.p, mx.p + 1, ctx->d_status);
  CK(cudaGetLastError());
  uint32_t h[2];
  CK(cudaMemcpyAsync(h, mx.p, 8, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  uint32_t cap = 1;
  while (cap < h[0]) cap <<= 1;
  const uint32_t rcap = std::max(1u, h[1]);
  const size_t bytes = size_t(cap) * 4 + size_t(rcap) * 8;
  if (bytes > size_t(200) << 10)
    return fail(ctx, SHERD_E_INVALID, "a radius ball holds more faces than shared memory does");
  CK(cudaFuncSetAttribute(k_ball, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
  k_ball<<<grid, BALL_BLOCK, bytes, s>>>(all, cent, rep, n_rep, radius, mode, normals, areas, frac,
                                         out3, flag, cap, rcap, ctx->d_status);
  CK(cudaGetLastError());
  return SHERD_OK;
}

template <typename T>
int to_host(sherd_ctx *ctx, T *host, const T *dev, size_t n) {
  if (host && n) CK(cudaMemcpyAsync(host, dev, sizeof(T) * n, cudaMemcpyDeviceToHost, ctx->stream));
  return SHERD_OK;
}

}  // namespace

namespace {

bool all_finite(const double *p, size_t n);

// refine::vertex_normals (refine.rs:121-151) of a mesh already on the device:
// the corners sorted stably by vertex, so each vertex adds its faces'
// unnormalised normals in ascending face order, as the reference's loop does.
int vertex_normals_dev(sherd_ctx *ctx, const double *dv, uint32_t nv, const uint32_t *df,
                       uint32_t nf, DBuf<double> &dn) {
  cudaStream_t s = ctx->stream;
  const uint32_t nc = 3u * nf;
  DBuf<uint32_t> key, key2, face, face2;
  CK(dn.alloc(size_t(3) * nv));
  if (nc) {
    CK(key.alloc(nc));
    CK(key2.alloc(nc));
    CK(face.alloc(nc));
    CK(face2.alloc(nc));
    k_incidence<<<blocks_for(nc), 256, 0, s>>>(df, nc, key.p, face.p);
    CK(cudaGetLastError());
    int bits = 1;  // vertex ids are below nv <= 2^bits
    while (bits < 32 && (uint64_t(1) << bits) < uint64_t(nv)) ++bits;
    // LSD radix sort is stable: each vertex keeps its faces in ascending order.
    int rc = radix_sort_pairs(ctx, key.p, key2.p, face.p, face2.p, nc, bits);
    if (rc) return rc;
  }
  k_vertex_normals<<<blocks_for(nv), 256, 0, s>>>(dv, df, key2.p, face2.p, nc, nv, dn.p);
  CK(cudaGetLastError());
  return SHERD_OK;
}

}  // namespace

extern "C" {

int sherd_segment(sherd_ctx *ctx, const sherd_mesh *mesh, const double *v, uint32_t nv,
                  const uint32_t *f, uint32_t nf, double thick, double res,
                  const sherd_seg_params *sp_in, uint8_t *labels, sherd_seg_info *info,
                  const sherd_seg_trace *trace) {
  if (!ctx || !mesh || ((!v || !f || !labels) && nf)) return fail(ctx, SHERD_E_INVALID, "null argument");
  if (nf != mesh->view.nf) return fail(ctx, SHERD_E_INVALID, "face count differs from the mesh");
  for (size_t i = 0; i < size_t(3) * nf; ++i)
    if (f[i] >= nv) return fail(ctx, SHERD_E_INVALID, "face index beyond the vertex array");
  sherd_seg_params sp;
  if (sp_in) sp = *sp_in; else sherd_seg_params_default(&sp);
  sherd_seg_info inf{};
  inf.votes = res > sp.coarse_at * thick ? sp.votes_coarse : sp.votes;
  inf.smooth_radius = std::max(thick / 3.0, sp.smooth_res * res);
  inf.boundary_angle = sp.boundary_angle;
  if (nf == 0 || !std::isfinite(thick) || thick <= 0.0) {
    std::fill(labels, labels + nf, uint8_t(0));
    if (info) *info = inf;
    return SHERD_OK;
  }
  double mag = 1.0;
  for (size_t i = 0; i < size_t(3) * nv; ++i) {
    if (!std::isfinite(v[i])) return fail(ctx, SHERD_E_INVALID, "non-finite vertex");
    mag = std::max(mag, std::fabs(v[i]));
  }
  const float pad = float(1e-6 * mag);
  CtxLock lock(ctx);
  NvtxRange range("sherd segment");
  int rc = begin(ctx);
  if (rc) return rc;
  cudaStream_t s = ctx->stream;
  const unsigned grid_sm = unsigned(ctx->sm_count) * 16u;
  DBuf<double> dv, normals, areas, cent;
  DBuf<uint32_t> df;
  if ((rc = upload(ctx, dv, v, size_t(3) * nv)) || (rc = upload(ctx, df, f, size_t(3) * nf))) return rc;
  CK(normals.alloc(size_t(3) * nf));
  CK(areas.alloc(nf));
  CK(cent.alloc(size_t(3) * nf));
  k_face_geometry<<<blocks_for(nf), 256, 0, s>>>(dv.p, df.p, nf, normals.p, areas.p, cent.p);
  CK(cudaGetLastError());

  // 3.4.1 the grid: the lowest face of every t/8 voxel, ascending, and each
  // face's nearest representative.
  DBuf<unsigned long long> mb, keys, keys2;
  DBuf<uint32_t> idx, idx2, rep_unsorted, rep, nrep_dev, near;
  DBuf<uint8_t> heads;
  CK(mb.alloc(3));
  CK(cudaMemsetAsync(mb.p, 0xFF, 3 * sizeof(unsigned long long), s));
  k_min_bound<<<std::min(blocks_for(nf), 1024u), 256, 0, s>>>(cent.p, nf, mb.p);
  CK(keys.alloc(nf));
  CK(keys2.alloc(nf));
  CK(idx.alloc(nf));
  CK(idx2.alloc(nf));
  k_voxel_keys<<<blocks_for(nf), 256, 0, s>>>(cent.p, nf, mb.p, thick * (1.0 / 8.0), keys.p, idx.p,
                                              ctx->d_status);
  CK(cudaGetLastError());
  if ((rc = radix_sort_pairs(ctx, keys.p, keys2.p, idx.p, idx2.p, nf, 63))) return rc;
  CK(heads.alloc(nf));
  k_run_heads<<<blocks_for(nf), 256, 0, s>>>(keys2.p, nf, heads.p);
  CK(rep_unsorted.alloc(nf));
  CK(nrep_dev.alloc(1));
  {
    size_t bytes = 0;
    CK(cub::DeviceSelect::Flagged(nullptr, bytes, idx2.p, heads.p, rep_unsorted.p, nrep_dev.p,
                                  int(nf), s));
    DBuf<unsigned char> tmp;
    CK(tmp.alloc(bytes));
    CK(cub::DeviceSelect::Flagged(tmp.p, bytes, idx2.p, heads.p, rep_unsorted.p, nrep_dev.p,
                                  int(nf), s));
    CK(cudaStreamSynchronize(s));
  }
  uint32_t n_rep = 0;
  CK(cudaMemcpy(&n_rep, nrep_dev.p, 4, cudaMemcpyDeviceToHost));
  inf.n_rep = n_rep;
  CK(rep.alloc(n_rep));
  {
    size_t bytes = 0;
    CK(cub::DeviceRadixSort::SortKeys(nullptr, bytes, rep_unsorted.p, rep.p, int(n_rep), 0, 32, s));
    DBuf<unsigned char> tmp;
    CK(tmp.alloc(bytes));
    CK(cub::DeviceRadixSort::SortKeys(tmp.p, bytes, rep_unsorted.p, rep.p, int(n_rep), 0, 32, s));
    CK(cudaStreamSynchronize(s));
  }
  DBuf<double> rep_pts;
  CK(rep_pts.alloc(size_t(3) * n_rep));
  k_gather_points<<<blocks_for(n_rep), 256, 0, s>>>(cent.p, rep.p, n_rep, rep_pts.p);
  CK(cudaGetLastError());
  sherd_cloud rep_cloud, all;
  if ((rc = cloud_build_dev(ctx, rep_pts.p, nullptr, n_rep, pad, &rep_cloud))) return rc;
  CK(near.alloc(nf));
  k_nearest_rep<<<std::min(blocks_for(nf, 128), grid_sm), 128, 0, s>>>(rep_cloud.view, cent.p, nf,
                                                                       near.p, ctx->d_status);
  CK(cudaGetLastError());
  if ((rc = cloud_build_dev(ctx, cent.p, nullptr, nf, pad, &all))) return rc;

  // 3.4.2 the smoothed normals.
  DBuf<double> g3, ns, ref;
  DBuf<uint8_t> gflag, good, frac, has_ref, cand;
  CK(g3.alloc(size_t(3) * n_rep));
  CK(gflag.alloc(n_rep));
  CK(ns.alloc(size_t(3) * nf));
  if ((rc = ball_pass(ctx, all.view, cent.p, rep.p, n_rep, inf.smooth_radius, BALL_NORMALS,
                      normals.p, areas.p, nullptr, g3.p, gflag.p)))
    return rc;
  k_spread<<<blocks_for(nf), 256, 0, s>>>(near.p, nf, g3.p, gflag.p, ns.p, nullptr);
  CK(cudaGetLastError());

  // 3.4.3 the cone vote.
  CK(good.alloc(nf));
  CK(frac.alloc(nf));
  k_cone_votes<<<blocks_for(nf, 128), 128, 0, s>>>(mesh->view, cent.p, normals.p, ns.p,
                                                  sp.smoothed_hit_normal ? ns.p : normals.p, nf,
                                                  thick, cone_consts(), good.p, ctx->d_status);
  k_votes_to_frac<<<blocks_for(nf), 256, 0, s>>>(good.p, nf, inf.votes, frac.p);
  CK(cudaGetLastError());
  if (trace) {
    if ((rc = to_host(ctx, trace->rep, rep.p, n_rep)) || (rc = to_host(ctx, trace->near, near.p, nf)) ||
        (rc = to_host(ctx, trace->ns, ns.p, size_t(3) * nf)) ||
        (rc = to_host(ctx, trace->good, good.p, nf)) ||
        (rc = to_host(ctx, trace->frac_raw, frac.p, nf)))
      return rc;
  }

  // 3.4.4 the majority filter.
  if ((rc = ball_pass(ctx, all.view, cent.p, rep.p, n_rep, thick * 0.25, BALL_MAJORITY,
                      normals.p, areas.p, frac.p, nullptr, gflag.p)))
    return rc;
  k_spread<<<blocks_for(nf), 256, 0, s>>>(near.p, nf, nullptr, gflag.p, nullptr, frac.p);
  CK(cudaGetLastError());
  if (trace && (rc = to_host(ctx, trace->frac_majority, frac.p, nf))) return rc;

  // 3.4.5-3.4.6 islands, over the face adjacency.
  const uint32_t m = 3 * nf, n_pairs = m - 1;
  DBuf<unsigned long long> ek, ek2;
  DBuf<uint32_t> ep, ep2, fa, fb;
  CK(ek.alloc(m));
  CK(ek2.alloc(m));
  CK(ep.alloc(m));
  CK(ep2.alloc(m));
  k_edge_keys<<<blocks_for(nf), 256, 0, s>>>(df.p, nf, ek.p, ep.p);
  CK(cudaGetLastError());
  if ((rc = radix_sort_pairs(ctx, ek.p, ek2.p, ep.p, ep2.p, m, 64))) return rc;
  CK(fa.alloc(n_pairs));
  CK(fb.alloc(n_pairs));
  k_face_pairs<<<blocks_for(m), 256, 0, s>>>(ek2.p, ep2.p, m, nf, fa.p, fb.p);
  CK(cudaGetLastError());
  const double min_frac = 0.5 * thick * thick, min_shell = 2.0 * thick * thick;
  if ((rc = drop_small(ctx, frac, 1, min_frac, fa, fb, n_pairs, areas, nf)) ||
      (rc = drop_small(ctx, frac, 0, min_shell, fa, fb, n_pairs, areas, nf)))
    return rc;
  if (trace && (rc = to_host(ctx, trace->frac_islands, frac.p, nf))) return rc;

  // 3.4.7 the boundary growth against the fixed shell reference normals.
  if (sp.boundary_angle_auto) {
    DBuf<double> dots;
    CK(dots.alloc(nf));
    k_shell_dots<<<blocks_for(nf), 256, 0, s>>>(frac.p, nf, normals.p, ns.p, dots.p);
    CK(cudaGetLastError());
    std::vector<double> h(nf);
    CK(cudaMemcpyAsync(h.data(), dots.p, sizeof(double) * nf, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    std::vector<double> noise;
    for (double c : h)
      if (c <= 1.0) noise.push_back(std::acos(c) * (180.0 / 3.14159265358979323846));
    if (!noise.empty()) {
      std::sort(noise.begin(), noise.end());
      size_t k = noise.size();
      double med = k % 2 ? noise[k / 2] : (noise[k / 2 - 1] + noise[k / 2]) / 2.0;
      inf.boundary_angle = std::max(inf.boundary_angle, med + 15.0);
    }
  }
  CK(ref.alloc(size_t(3) * nf));
  CK(has_ref.alloc(nf));
  if ((rc = ball_pass(ctx, all.view, cent.p, rep.p, n_rep, thick * 0.5, BALL_SHELL_NORMALS,
                      normals.p, areas.p, frac.p, g3.p, gflag.p)))
    return rc;
  k_spread<<<blocks_for(nf), 256, 0, s>>>(near.p, nf, g3.p, gflag.p, ref.p, has_ref.p);
  CK(cudaGetLastError());
  if (trace && (rc = to_host(ctx, trace->has_ref, has_ref.p, nf))) return rc;
  const double cos_grow = std::cos(inf.boundary_angle * (3.14159265358979323846 / 180.0));
  CK(cand.alloc(nf));
  CK(cudaMemsetAsync(cand.p, 0, nf, s));
  DBuf<uint32_t> flipped;
  CK(flipped.alloc(1));
  for (int pass = 0; pass < 60; ++pass) {
    CK(cudaMemsetAsync(flipped.p, 0, 4, s));
    k_grow_candidates<<<blocks_for(n_pairs), 256, 0, s>>>(fa.p, fb.p, n_pairs, frac.p, cand.p);
    k_grow_flip<<<blocks_for(nf), 256, 0, s>>>(cand.p, frac.p, nf, normals.p, ref.p, has_ref.p,
                                               cos_grow, flipped.p);
    CK(cudaGetLastError());
    uint32_t any = 0;
    CK(cudaMemcpyAsync(&any, flipped.p, 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (!any) break;
  }

  // 3.4.8 one more island pass.
  if ((rc = drop_small(ctx, frac, 1, min_frac, fa, fb, n_pairs, areas, nf))) return rc;
  CK(cudaMemcpyAsync(labels, frac.p, nf, cudaMemcpyDeviceToHost, s));
  rc = finish(ctx, "segment", nf, true);
  if (rc) return rc;
  if (info) *info = inf;
  return SHERD_OK;
}


// ---- R 9: full-resolution join refinement (refine.rs) -------------------------

int sherd_vertex_normals(sherd_ctx *ctx, const double *v, uint32_t nv, const uint32_t *f,
                         uint32_t nf, double *normals) {
  if (!ctx || ((!v || !normals) && nv) || (!f && nf)) return fail(ctx, SHERD_E_INVALID, "null argument");
  if (uint64_t(nf) * 3u >= (uint64_t(1) << 31)) return fail(ctx, SHERD_E_INVALID, "too many faces");
  if (nv == 0 && nf) return fail(ctx, SHERD_E_INVALID, "face index beyond the vertex array");
  if (nv == 0) return SHERD_OK;
  CtxLock lock(ctx);
  NvtxRange range("sherd vertex_normals");
  int rc = begin(ctx);
  if (rc) return rc;
  DBuf<double> dv, dn;
  DBuf<uint32_t> df;
  if ((rc = upload(ctx, dv, v, size_t(3) * nv)) || (rc = upload(ctx, df, f, size_t(3) * nf))) return rc;
  DevInputCheck chk;
  InputCheck got;
  if ((rc = chk.open(ctx, 1)) || (rc = chk.indices(ctx, 0, df.p, size_t(3) * nf, nv)) ||
      (rc = chk.read(ctx, &got)))
    return rc;
  if (got.bad_index) return fail(ctx, SHERD_E_INVALID, "face index beyond the vertex array");
  if ((rc = vertex_normals_dev(ctx, dv.p, nv, df.p, nf, dn))) return rc;
  CK(cudaMemcpyAsync(normals, dn.p, 24 * size_t(nv), cudaMemcpyDeviceToHost, ctx->stream));
  return finish(ctx, "vertex_normals", nv, true);
}

int sherd_fracture_cloud(sherd_ctx *ctx, const double *v, uint32_t nv, const uint32_t *f,
                         uint32_t nf, const double *centroids, const uint8_t *fracture,
                         uint32_t n_cent, double radius, uint32_t cap, uint32_t *idx_out,
                         double *points_out, double *normals_out, uint32_t *n_out) {
  if (!ctx || !n_out || ((!v) && nv) || (!f && nf) || ((!centroids || !fracture) && n_cent) ||
      ((!idx_out || !points_out || !normals_out) && cap))
    return fail(ctx, SHERD_E_INVALID, "null argument");
  *n_out = 0;
  if (uint64_t(nf) * 3u >= (uint64_t(1) << 31)) return fail(ctx, SHERD_E_INVALID, "too many faces");
  CtxLock lock(ctx);
  NvtxRange range("sherd fracture_cloud");
  int rc = begin(ctx);
  if (rc) return rc;
  cudaStream_t s = ctx->stream;
  DBuf<double> dv, dc, dn, dist;
  DBuf<uint32_t> df, near, lin, sel, nsel;
  DBuf<uint8_t> dfrac, flags;
  if ((rc = upload(ctx, dv, v, size_t(3) * nv)) || (rc = upload(ctx, df, f, size_t(3) * nf)) ||
      (rc = upload(ctx, dc, centroids, size_t(3) * n_cent)) ||
      (rc = upload(ctx, dfrac, fracture, size_t(n_cent))))
    return rc;
  // The face indices, and the vertices and centroids finite, checked where
  // they now lie; the centroids' largest magnitude sizes their tree's padding.
  DevInputCheck chk;
  InputCheck got[2];
  if ((rc = chk.open(ctx, 2)) || (rc = chk.indices(ctx, 0, df.p, size_t(3) * nf, nv)) ||
      (rc = chk.coords(ctx, 0, dv.p, size_t(3) * nv)) ||
      (rc = chk.coords(ctx, 1, dc.p, size_t(3) * n_cent)) || (rc = chk.read(ctx, got)))
    return rc;
  if (got[0].bad_index) return fail(ctx, SHERD_E_INVALID, "face index beyond the vertex array");
  if (got[0].non_finite || got[1].non_finite) return fail(ctx, SHERD_E_INVALID, "coordinates must be finite");
  if (nv == 0 || n_cent == 0 || !(radius > 0.0)) return SHERD_OK;
  const double mag = checked_mag(got[1]);
  // The centroids' tree, the nearest centroid of every vertex strictly within
  // the radius (refine.rs:161-178), and the vertices whose nearest is a
  // fracture face, ascending.
  sherd_cloud cent;
  if ((rc = cloud_build_dev(ctx, dc.p, nullptr, n_cent, float(1e-6 * mag), &cent))) return rc;
  CK(near.alloc(nv));
  CK(dist.alloc(nv));
  k_nn_below<<<blocks_for(nv, 128), 128, 0, s>>>(cent.view, dv.p, nv, radius, near.p, dist.p,
                                                 ctx->d_status);
  CK(cudaGetLastError());
  CK(flags.alloc(nv));
  CK(lin.alloc(nv));
  k_fracture_flags<<<blocks_for(nv), 256, 0, s>>>(near.p, dfrac.p, nv, flags.p, lin.p);
  CK(cudaGetLastError());
  CK(sel.alloc(nv));
  CK(nsel.alloc(1));
  size_t bytes = 0;
  CK(cub::DeviceSelect::Flagged(nullptr, bytes, lin.p, flags.p, sel.p, nsel.p, int(nv), s));
  DBuf<unsigned char> tmp;
  CK(tmp.alloc(bytes));
  CK(cub::DeviceSelect::Flagged(tmp.p, bytes, lin.p, flags.p, sel.p, nsel.p, int(nv), s));
  // Every vertex's normal (refine.rs:121-151), then the selected vertices'
  // points and normals gathered in selection order.
  if ((rc = vertex_normals_dev(ctx, dv.p, nv, df.p, nf, dn))) return rc;
  uint32_t count = 0;
  CK(cudaMemcpyAsync(&count, nsel.p, 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  *n_out = count;
  const uint32_t m = std::min(count, cap);
  if (m) {
    DBuf<double> gp, gn;
    CK(gp.alloc(size_t(3) * m));
    CK(gn.alloc(size_t(3) * m));
    k_gather_cloud<<<blocks_for(m), 256, 0, s>>>(dv.p, dn.p, sel.p, m, gp.p, gn.p);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(idx_out, sel.p, 4 * size_t(m), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(points_out, gp.p, 24 * size_t(m), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(normals_out, gn.p, 24 * size_t(m), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
  }
  return finish(ctx, "fracture_cloud", nv, true);
}

}  // extern "C"

namespace {

bool all_finite(const double *p, size_t n) {
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(p[i])) return false;
  return true;
}

// The box padding of a cloud built from `p` placed by the row-major pose t:
// 1e-6 of a bound on the placed coordinates' magnitude (at least 1), the
// padding cloud_build gives a cloud of the placed points themselves.
float placed_pad(const double *p, uint32_t n, const double *t) {
  double m[3] = {0.0, 0.0, 0.0};
  for (size_t i = 0; i < size_t(n); ++i)
    for (int c = 0; c < 3; ++c) m[c] = std::max(m[c], std::fabs(p[3 * i + c]));
  double mag = 1.0;
  for (int r = 0; r < 3; ++r) {
    double b = std::fabs(t[4 * r + 3]);
    for (int c = 0; c < 3; ++c) b += std::fabs(t[4 * r + c]) * m[c];
    mag = std::max(mag, b * (1.0 + 1e-9));
  }
  return float(1e-6 * mag);
}

void identity_registration(sherd_registration &r) {
  std::memset(&r, 0, sizeof r);
  for (int k = 0; k < 16; k += 5) r.transform[k] = 1.0;
}

}  // namespace

extern "C" {

int sherd_refine_join(sherd_ctx *ctx, const double *source, uint32_t n_source,
                      const double *target, const double *target_normals, uint32_t n_target,
                      const double pose_fixed[16], const double pose_moving[16],
                      const double dist[2], int32_t max_iteration, sherd_registration out[2]) {
  if (!ctx || (!source && n_source) || ((!target || !target_normals) && n_target) || !pose_fixed ||
      !pose_moving || !dist || !out)
    return fail(ctx, SHERD_E_INVALID, "null argument");
  if (max_iteration < 0) return fail(ctx, SHERD_E_INVALID, "negative iteration cap");
  if (!finite_pose(pose_fixed) || !finite_pose(pose_moving))
    return fail(ctx, SHERD_E_INVALID, "pose is not finite");
  if (!all_finite(source, size_t(3) * n_source) || !all_finite(target, size_t(3) * n_target) ||
      !all_finite(target_normals, size_t(3) * n_target))
    return fail(ctx, SHERD_E_INVALID, "non-finite point or normal");
  if (n_source == 0 || n_target == 0) {  // nothing to register: both rungs stay at the identity
    identity_registration(out[0]);
    identity_registration(out[1]);
    return SHERD_OK;
  }
  CtxLock lock(ctx);
  NvtxRange range("sherd refine_join");
  int rc = begin(ctx);
  if (rc) return rc;
  cudaStream_t s = ctx->stream;
  const uint32_t ns = n_source, nt = n_target;
  DBuf<double> raw_s, raw_t, raw_n, placed_s, placed_t, placed_n;
  if ((rc = upload(ctx, raw_s, source, size_t(3) * ns)) ||
      (rc = upload(ctx, raw_t, target, size_t(3) * nt)) ||
      (rc = upload(ctx, raw_n, target_normals, size_t(3) * nt)))
    return rc;
  CK(placed_s.alloc(size_t(3) * ns));
  CK(placed_t.alloc(size_t(3) * nt));
  CK(placed_n.alloc(size_t(3) * nt));
  k_place_fused<<<blocks_for(ns), 256, 0, s>>>(raw_s.p, ns, pose_of(pose_moving), 0, placed_s.p);
  k_place_fused<<<blocks_for(nt), 256, 0, s>>>(raw_t.p, nt, pose_of(pose_fixed), 0, placed_t.p);
  k_place_fused<<<blocks_for(nt), 256, 0, s>>>(raw_n.p, nt, pose_of(pose_fixed), 1, placed_n.p);
  CK(cudaGetLastError());
  sherd_cloud src, tgt;
  if ((rc = cloud_build_dev(ctx, placed_s.p, nullptr, ns, placed_pad(source, ns, pose_moving), &src)) ||
      (rc = cloud_build_dev(ctx, placed_t.p, placed_n.p, nt, placed_pad(target, nt, pose_fixed), &tgt)))
    return rc;

  // A slice of about 256 source points per block, at most 4 blocks per SM.
  const uint32_t blocks =
      std::max(1u, std::min<uint32_t>((ns + 255u) / 256u, 4u * uint32_t(std::max(ctx->sm_count, 1))));
  const uint32_t chunk = (ns + blocks - 1u) / blocks;
  DBuf<double> partials, identity;
  DBuf<int> hints;
  DBuf<WideState> state;
  DBuf<sherd_registration> dout;
  CK(partials.alloc(size_t(blocks) * ICP_SUMS));
  CK(hints.alloc(ns));
  CK(state.alloc(1));
  CK(dout.alloc(2));
  static const double kIdentity[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
  if ((rc = upload(ctx, identity, kIdentity, 16))) return rc;
  const double *first_pose = reinterpret_cast<const double *>(
      reinterpret_cast<const char *>(dout.p) + offsetof(sherd_registration, transform));
  // The rungs alone are timed too (method "refine_join_rungs"; items = passes).
  cudaEvent_t rungs_begin = nullptr, rungs_end = nullptr;
  CK(cudaEventCreate(&rungs_begin));
  if (cudaEventCreate(&rungs_end) != cudaSuccess) {
    cudaEventDestroy(rungs_begin);
    return fail(ctx, SHERD_E_DEVICE, "refine_join: cudaEventCreate failed");
  }
  struct EventPair {
    cudaEvent_t a, b;
    ~EventPair() {
      cudaEventDestroy(a);
      cudaEventDestroy(b);
    }
  } events{rungs_begin, rungs_end};
  CK(cudaEventRecord(rungs_begin, s));
  uint32_t done = 0;
  size_t launched = 0;
  for (int r = 0; r < 2; ++r) {
    CK(cudaMemsetAsync(hints.p, 0xFF, sizeof(int) * size_t(ns), s));  // no match yet: -1
    k_wide_reset<<<1, 32, 0, s>>>(state.p, r == 0 ? identity.p : first_pose);
    // max_iteration + 1 passes at most; the state says when the rung ended
    // sooner, looked at every 16 passes.
    for (int64_t pass = 0; pass <= int64_t(max_iteration); ++pass) {
      k_wide_pass<<<blocks, ICP_BLOCK, 0, s>>>(src.pts.p, ns, tgt.view, dist[r], max_iteration,
                                               state.p, hints.p, chunk, partials.p, dout.p + r,
                                               ctx->d_status);
      CK(cudaGetLastError());
      ++launched;
      if (pass % 16 == 15 && pass < int64_t(max_iteration)) {
        CK(cudaMemcpyAsync(&done, reinterpret_cast<const char *>(state.p) + offsetof(WideState, done), 4,
                           cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (done) break;
      }
    }
  }
  CK(cudaEventRecord(rungs_end, s));
  CK(cudaMemcpyAsync(out, dout.p, sizeof(sherd_registration) * 2, cudaMemcpyDeviceToHost, s));
  rc = finish(ctx, "refine_join", ns, true);
  if (rc) return rc;
  float ms = 0.0f;
  MethodStats &m = ctx->stats["refine_join_rungs"];
  m.calls += 1;
  m.items += launched;
  if (cudaEventElapsedTime(&ms, rungs_begin, rungs_end) == cudaSuccess) m.ms += ms;
  return SHERD_OK;
}


// ---- stage 1: hypotheses, coarse score, suppression (R 5.1-5.5) ---------------

int sherd_hypotheses_coarse(sherd_ctx *ctx, const sherd_frames *a, const sherd_frames *b,
                            const uint32_t *ia, uint32_t n_ia, const uint32_t *ib, uint32_t n_ib,
                            double dihedral_tol, const sherd_cloud *target, const double *q,
                            const double *qn, uint32_t n_probe, double delta,
                            double normal_agree, uint32_t capacity, uint32_t *pa, uint32_t *pb,
                            double *poses, double *scores, uint32_t *count) {
  if (!ctx || !a || !b || !target || !count || (!ia && n_ia) || (!ib && n_ib) ||
      ((!q || !qn) && n_probe) || (capacity && (!pa || !pb || !poses || !scores)))
    return fail(ctx, SHERD_E_INVALID, "null argument");
  *count = 0;
  if ((a->n && (!a->p || !a->ns || !a->f || !a->dih)) || (b->n && (!b->p || !b->ns || !b->f || !b->dih)))
    return fail(ctx, SHERD_E_INVALID, "null frame array");
  if (!target->view.nrm) return fail(ctx, SHERD_E_INVALID, "the target carries no normals");
  if (uint64_t(n_ia) * n_ib >= (uint64_t(1) << 31))
    return fail(ctx, SHERD_E_INVALID, "n_ia * n_ib must stay below 2^31");
  for (uint32_t i = 0; i < n_ia; ++i)
    if (ia[i] >= a->n) return fail(ctx, SHERD_E_INVALID, "ia names a point beyond a's frames");
  for (uint32_t j = 0; j < n_ib; ++j)
    if (ib[j] >= b->n) return fail(ctx, SHERD_E_INVALID, "ib names a point beyond b's frames");
  if (n_ia == 0 || n_ib == 0) return SHERD_OK;  // no hypothesis (R 5.1's empty return)
  CtxLock lock(ctx);
  NvtxRange range("sherd hypotheses_coarse");
  int rc = begin(ctx);
  if (rc) return rc;
  cudaStream_t s = ctx->stream;
  DBuf<double> ap, ans, af, adih, bp, bns, bf, bdih, dq, dqn, dposes, dscores;
  DBuf<uint32_t> dia, dib, lin, sel, nsel, dpa, dpb;
  DBuf<uint8_t> flags;
  if ((rc = upload(ctx, ap, a->p, size_t(3) * a->n)) || (rc = upload(ctx, ans, a->ns, size_t(3) * a->n)) ||
      (rc = upload(ctx, af, a->f, size_t(3) * a->n)) || (rc = upload(ctx, adih, a->dih, size_t(a->n))) ||
      (rc = upload(ctx, bp, b->p, size_t(3) * b->n)) || (rc = upload(ctx, bns, b->ns, size_t(3) * b->n)) ||
      (rc = upload(ctx, bf, b->f, size_t(3) * b->n)) || (rc = upload(ctx, bdih, b->dih, size_t(b->n))) ||
      (rc = upload(ctx, dia, ia, size_t(n_ia))) || (rc = upload(ctx, dib, ib, size_t(n_ib))) ||
      (rc = upload(ctx, dq, q, size_t(3) * n_probe)) || (rc = upload(ctx, dqn, qn, size_t(3) * n_probe)))
    return rc;
  const uint32_t grid = n_ia * n_ib;
  CK(flags.alloc(grid));
  CK(lin.alloc(grid));
  CK(sel.alloc(grid));
  CK(nsel.alloc(1));
  k_hyp_flags<<<blocks_for(grid), 256, 0, s>>>(adih.p, dia.p, n_ia, bdih.p, dib.p, n_ib, dihedral_tol,
                                               flags.p, lin.p);
  CK(cudaGetLastError());
  {
    size_t bytes = 0;
    CK(cub::DeviceSelect::Flagged(nullptr, bytes, lin.p, flags.p, sel.p, nsel.p, int(grid), s));
    DBuf<unsigned char> tmp;
    CK(tmp.alloc(bytes));
    CK(cub::DeviceSelect::Flagged(tmp.p, bytes, lin.p, flags.p, sel.p, nsel.p, int(grid), s));
    CK(cudaStreamSynchronize(s));
  }
  uint32_t n = 0;
  CK(cudaMemcpy(&n, nsel.p, 4, cudaMemcpyDeviceToHost));
  *count = n;
  if (n == 0 || capacity == 0) return finish(ctx, "hypotheses_coarse", 0, true);
  if (capacity < n) {
    rc = finish(ctx, "hypotheses_coarse", 0, true);
    if (rc) return rc;
    return fail(ctx, SHERD_E_INVALID, "capacity below the hypothesis count");
  }
  CK(dpa.alloc(n));
  CK(dpb.alloc(n));
  CK(dposes.alloc(size_t(16) * n));
  CK(dscores.alloc(n));
  FramesView fa{ap.p, ans.p, af.p, adih.p, a->n}, fb{bp.p, bns.p, bf.p, bdih.p, b->n};
  k_hyp_poses<<<blocks_for(n), 256, 0, s>>>(fa, fb, dia.p, dib.p, n_ib, sel.p, n, dpa.p, dpb.p,
                                            dposes.p);
  CK(cudaGetLastError());
  if (n_probe) {
    unsigned cgrid = std::min(blocks_for(size_t(n) * 32, 128), unsigned(ctx->sm_count) * 16u);
    k_coarse_scores<<<cgrid, 128, 0, s>>>(target->view, dq.p, dqn.p, n_probe, dposes.p, n, delta,
                                          normal_agree, dscores.p, ctx->d_status);
    CK(cudaGetLastError());
  } else {
    CK(cudaMemsetAsync(dscores.p, 0, sizeof(double) * n, s));  // 0 / 0 probe points: 0
  }
  CK(cudaMemcpyAsync(pa, dpa.p, 4 * size_t(n), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(pb, dpb.p, 4 * size_t(n), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(poses, dposes.p, sizeof(double) * 16 * size_t(n), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(scores, dscores.p, sizeof(double) * size_t(n), cudaMemcpyDeviceToHost, s));
  return finish(ctx, "hypotheses_coarse", size_t(n) * n_probe, true);
}

}  // extern "C"

namespace {

// f64::total_cmp's key (a signed integer order equal to IEEE 754 totalOrder).
int64_t total_key(double x) {
  int64_t bits;
  std::memcpy(&bits, &x, 8);
  return bits ^ int64_t(uint64_t(bits >> 63) >> 1);
}

// nms::trace_of_transpose_product (nms.rs:93-99) on row-major 4x4 poses:
// trace(A^T B) summed over columns i as (a0i b0i + a1i b1i) + a2i b2i.
double trace_tp(const double *a, const double *b) {
  double trace = 0.0;
  for (int i = 0; i < 3; ++i) trace += (a[i] * b[i] + a[4 + i] * b[4 + i]) + a[8 + i] * b[8 + i];
  return trace;
}

}  // namespace

extern "C" {

int sherd_order_by_score(const double *score, uint32_t n, uint32_t limit, uint32_t *order,
                         uint32_t *n_order) {
  if (!n_order || ((!score || (!order && limit)) && n)) return SHERD_E_INVALID;
  // Each score's total-order key computed once, beside its index; the first
  // `limit` of the order selected, then only they sorted. The order is total
  // (no two entries compare equal), so the result is the full sort's head.
  struct Keyed {
    int64_t key;
    uint32_t i;
  };
  std::vector<Keyed> keyed(n);
  for (uint32_t i = 0; i < n; ++i) keyed[i] = {total_key(score[i]), i};
  auto before = [](const Keyed &x, const Keyed &y) { return x.key != y.key ? x.key > y.key : x.i < y.i; };
  const uint32_t m = std::min(n, limit);
  if (m < n) std::nth_element(keyed.begin(), keyed.begin() + m, keyed.end(), before);
  std::sort(keyed.begin(), keyed.begin() + m, before);
  for (uint32_t k = 0; k < m; ++k) order[k] = keyed[k].i;
  *n_order = m;
  return SHERD_OK;
}

int sherd_nms(const uint32_t *order, uint32_t n_order, const double *poses, const double *score,
              uint32_t n_poses, double trans_tol, uint32_t topk, double floor, uint32_t *kept,
              uint32_t *n_kept) {
  if (!n_kept || ((!order || !poses || !score || !kept) && n_order)) return SHERD_E_INVALID;
  for (uint32_t o = 0; o < n_order; ++o)
    if (order[o] >= n_poses) return SHERD_E_INVALID;
  uint32_t m = 0;
  for (uint32_t o = 0; o < n_order; ++o) {
    const uint32_t h = order[o];
    if (score[h] < floor) break;
    const double *t = poses + 16 * size_t(h);
    bool duplicate = false;
    for (uint32_t k = 0; k < m && !duplicate; ++k) {
      const double *u = poses + 16 * size_t(kept[k]);
      const double dx = t[3] - u[3], dy = t[7] - u[7], dz = t[11] - u[11];
      duplicate = std::sqrt((dx * dx + dy * dy) + dz * dz) < trans_tol && trace_tp(t, u) > 2.9;
    }
    if (!duplicate) kept[m++] = h;
    if (m >= topk) break;
  }
  *n_kept = m;
  return SHERD_OK;
}


}  // extern "C"

// ---- R 3.5.3-3.5.5: breaklines and their frames --------------------------------

namespace {

// The entries of `in` (or 0..n-1 when `in` is null) whose flag is set, in
// order; `count` receives how many.
int select_flagged(sherd_ctx *ctx, const uint32_t *in, const uint8_t *flags, uint32_t n,
                   DBuf<uint32_t> &out, uint32_t &count) {
  cudaStream_t s = ctx->stream;
  count = 0;
  CK(out.alloc(std::max<uint32_t>(n, 1)));
  if (n == 0) return SHERD_OK;
  DBuf<uint32_t> iota, cnt;
  if (!in) {
    CK(iota.alloc(n));
    k_iota<<<blocks_for(n), 256, 0, s>>>(iota.p, n);
    CK(cudaGetLastError());
    in = iota.p;
  }
  CK(cnt.alloc(1));
  size_t bytes = 0;
  CK(cub::DeviceSelect::Flagged(nullptr, bytes, in, flags, out.p, cnt.p, int(n), s));
  DBuf<unsigned char> tmp;
  CK(tmp.alloc(std::max<size_t>(bytes, 1)));
  CK(cub::DeviceSelect::Flagged(tmp.p, bytes, in, flags, out.p, cnt.p, int(n), s));
  CK(cudaMemcpyAsync(&count, cnt.p, 4, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return SHERD_OK;
}

// voxel_representatives (segment.rs:217-259) of n device points at `spacing`:
// the lowest index of every occupied voxel, ascending (segmentation's grid).
int voxel_reps(sherd_ctx *ctx, const double *pts, uint32_t n, double spacing,
               DBuf<uint32_t> &rep, uint32_t &n_rep) {
  cudaStream_t s = ctx->stream;
  n_rep = 0;
  CK(rep.alloc(std::max<uint32_t>(n, 1)));
  if (n == 0) return SHERD_OK;
  DBuf<unsigned long long> mb, keys, keys2;
  DBuf<uint32_t> idx, idx2, unsorted;
  DBuf<uint8_t> heads;
  CK(mb.alloc(3));
  CK(cudaMemsetAsync(mb.p, 0xFF, 3 * sizeof(unsigned long long), s));
  k_min_bound<<<std::min(blocks_for(n), 1024u), 256, 0, s>>>(pts, n, mb.p);
  CK(keys.alloc(n));
  CK(keys2.alloc(n));
  CK(idx.alloc(n));
  CK(idx2.alloc(n));
  k_voxel_keys<<<blocks_for(n), 256, 0, s>>>(pts, n, mb.p, spacing, keys.p, idx.p, ctx->d_status);
  CK(cudaGetLastError());
  int rc = radix_sort_pairs(ctx, keys.p, keys2.p, idx.p, idx2.p, n, 63);
  if (rc) return rc;
  CK(heads.alloc(n));
  k_run_heads<<<blocks_for(n), 256, 0, s>>>(keys2.p, n, heads.p);
  CK(cudaGetLastError());
  if ((rc = select_flagged(ctx, idx2.p, heads.p, n, unsorted, n_rep))) return rc;
  if (n_rep == 0) return SHERD_OK;
  size_t bytes = 0;
  CK(cub::DeviceRadixSort::SortKeys(nullptr, bytes, unsorted.p, rep.p, int(n_rep), 0, 32, s));
  DBuf<unsigned char> tmp;
  CK(tmp.alloc(std::max<size_t>(bytes, 1)));
  CK(cub::DeviceRadixSort::SortKeys(tmp.p, bytes, unsorted.p, rep.p, int(n_rep), 0, 32, s));
  CK(cudaStreamSynchronize(s));
  return SHERD_OK;
}

// One macro normal (breakline.rs:307-337) of the n breakline points `p` into
// out3: the area-weighted ball normals over the faces of the mask at distance
// >= inner, then, for the points that got a normal shorter than 0.5, over
// every face of the mask; zeros when the mask is empty.
int macro_normals(sherd_ctx *ctx, const double *p, uint32_t n, const double *cent,
                  const double *normals, const double *areas, const uint8_t *frac, uint32_t nf,
                  const double *dist, uint8_t fracture, double inner, double outer, float pad,
                  double *out3) {
  cudaStream_t s = ctx->stream;
  CK(cudaMemsetAsync(out3, 0, sizeof(double) * 3 * size_t(n), s));
  DBuf<uint8_t> every, far, flag, bad_flag;
  CK(every.alloc(nf));
  CK(far.alloc(nf));
  k_macro_masks<<<blocks_for(nf), 256, 0, s>>>(frac, fracture, dist, inner, nf, every.p, far.p);
  CK(cudaGetLastError());
  DBuf<uint32_t> all_idx, far_idx, queries, bad_idx;
  uint32_t n_all = 0, n_far = 0, n_bad = 0;
  int rc = select_flagged(ctx, nullptr, every.p, nf, all_idx, n_all);
  if (rc) return rc;
  if (n_all == 0) return SHERD_OK;
  if ((rc = select_flagged(ctx, nullptr, far.p, nf, far_idx, n_far))) return rc;
  CK(flag.alloc(n));
  // One ball pass over the faces `sel` (k of them) for the queries q_idx.
  auto pass = [&](const uint32_t *sel, uint32_t k, const uint32_t *q_idx, uint32_t nq,
                  double *res3) -> int {
    DBuf<double> c, nn, a;
    CK(c.alloc(size_t(3) * k));
    CK(nn.alloc(size_t(3) * k));
    CK(a.alloc(k));
    k_gather_points<<<blocks_for(k), 256, 0, s>>>(cent, sel, k, c.p);
    k_gather_points<<<blocks_for(k), 256, 0, s>>>(normals, sel, k, nn.p);
    k_gather1<<<blocks_for(k), 256, 0, s>>>(areas, sel, k, a.p);
    CK(cudaGetLastError());
    sherd_cloud sub;
    int r = cloud_build_dev(ctx, c.p, nullptr, k, pad, &sub);
    if (r) return r;
    if ((r = ball_pass(ctx, sub.view, p, q_idx, nq, outer, BALL_NORMALS, nn.p, a.p, nullptr, res3,
                       flag.p)))
      return r;
    CK(cudaStreamSynchronize(s));
    return SHERD_OK;
  };
  CK(queries.alloc(n));
  k_iota<<<blocks_for(n), 256, 0, s>>>(queries.p, n);
  CK(cudaGetLastError());
  if (n_far && (rc = pass(far_idx.p, n_far, queries.p, n, out3))) return rc;
  CK(bad_flag.alloc(n));
  k_short_normals<<<blocks_for(n), 256, 0, s>>>(out3, n, bad_flag.p);
  CK(cudaGetLastError());
  if ((rc = select_flagged(ctx, nullptr, bad_flag.p, n, bad_idx, n_bad))) return rc;
  if (n_bad == 0) return SHERD_OK;
  DBuf<double> fallback;
  CK(fallback.alloc(size_t(3) * n_bad));
  if ((rc = pass(all_idx.p, n_all, bad_idx.p, n_bad, fallback.p))) return rc;
  k_scatter3<<<blocks_for(n_bad), 256, 0, s>>>(fallback.p, bad_idx.p, n_bad, out3);
  CK(cudaGetLastError());
  return SHERD_OK;
}

}  // namespace

extern "C" {

int sherd_breaklines(sherd_ctx *ctx, const double *v, uint32_t nv, const uint32_t *f, uint32_t nf,
                     const uint8_t *frac, double t, double macro_inner, double macro_outer,
                     double brk_voxel, uint32_t capacity, double *p, double *ns, double *nfr,
                     double *fr, double *dih, uint8_t *valid, uint32_t *sub, uint32_t *n_sub,
                     uint32_t *count) {
  if (!ctx || !count || !n_sub || ((!v || !f || !frac) && nf) ||
      (capacity && (!p || !ns || !nfr || !fr || !dih || !valid || !sub)))
    return fail(ctx, SHERD_E_INVALID, "null argument");
  *count = 0;
  *n_sub = 0;
  if (!(t > 0.0) || !std::isfinite(t) || !(macro_inner >= 0.0) || !(macro_outer > 0.0) ||
      !(brk_voxel > 0.0))
    return fail(ctx, SHERD_E_INVALID, "t, the macro radii and the voxel must be positive");
  if (uint64_t(nf) * 3u >= (uint64_t(1) << 31)) return fail(ctx, SHERD_E_INVALID, "too many faces");
  for (size_t i = 0; i < size_t(3) * nf; ++i)
    if (f[i] >= nv) return fail(ctx, SHERD_E_INVALID, "face index beyond the vertex array");
  double mag = 1.0;
  for (size_t i = 0; i < size_t(3) * nv; ++i) {
    if (!std::isfinite(v[i])) return fail(ctx, SHERD_E_INVALID, "non-finite vertex");
    mag = std::max(mag, std::fabs(v[i]));
  }
  if (nf == 0) return SHERD_OK;
  const float pad = float(1e-6 * mag);
  CtxLock lock(ctx);
  NvtxRange range("sherd breaklines");
  int rc = begin(ctx);
  if (rc) return rc;
  cudaStream_t s = ctx->stream;
  DBuf<double> dv, normals, areas, cent;
  DBuf<uint32_t> df;
  DBuf<uint8_t> dfrac;
  if ((rc = upload(ctx, dv, v, size_t(3) * nv)) || (rc = upload(ctx, df, f, size_t(3) * nf)) ||
      (rc = upload(ctx, dfrac, frac, size_t(nf))))
    return rc;
  CK(normals.alloc(size_t(3) * nf));
  CK(areas.alloc(nf));
  CK(cent.alloc(size_t(3) * nf));
  k_face_geometry<<<blocks_for(nf), 256, 0, s>>>(dv.p, df.p, nf, normals.p, areas.p, cent.p);
  CK(cudaGetLastError());

  // R 3.5.3 the points: the edges whose two faces differ in label, in the
  // adjacency's ascending edge-key order, at their midpoints.
  const uint32_t m = 3 * nf, n_pairs = m - 1;
  DBuf<unsigned long long> ek, ek2;
  DBuf<uint32_t> ep, ep2, fa, fb, edges;
  CK(ek.alloc(m));
  CK(ek2.alloc(m));
  CK(ep.alloc(m));
  CK(ep2.alloc(m));
  k_edge_keys<<<blocks_for(nf), 256, 0, s>>>(df.p, nf, ek.p, ep.p);
  CK(cudaGetLastError());
  if ((rc = radix_sort_pairs(ctx, ek.p, ek2.p, ep.p, ep2.p, m, 64))) return rc;
  CK(fa.alloc(n_pairs));
  CK(fb.alloc(n_pairs));
  k_face_pairs<<<blocks_for(m), 256, 0, s>>>(ek2.p, ep2.p, m, nf, fa.p, fb.p);
  DBuf<uint8_t> bflag;
  CK(bflag.alloc(n_pairs));
  k_brk_flags<<<blocks_for(n_pairs), 256, 0, s>>>(fa.p, fb.p, n_pairs, dfrac.p, bflag.p);
  CK(cudaGetLastError());
  uint32_t n = 0;
  if ((rc = select_flagged(ctx, nullptr, bflag.p, n_pairs, edges, n))) return rc;
  *count = n;
  if (n == 0 || capacity == 0) return finish(ctx, "breaklines", nf, true);
  if (capacity < n) {
    rc = finish(ctx, "breaklines", nf, true);
    if (rc) return rc;
    return fail(ctx, SHERD_E_INVALID, "capacity below the breakline point count");
  }
  DBuf<double> dp, dns, dnf, dfr, ddih, dist;
  DBuf<uint32_t> nn_idx;
  CK(dp.alloc(size_t(3) * n));
  k_brk_points<<<blocks_for(n), 256, 0, s>>>(ek2.p, edges.p, n, dv.p, dp.p);
  CK(cudaGetLastError());

  // R 3.5.4 each centroid's distance to the breakline, needed only below
  // `inner` (the bounded search reports +inf beyond it), then the macro
  // normals of the shell and of the fracture, and the frames.
  const double inner = macro_inner * t, outer = macro_outer * t;
  sherd_cloud brk;
  if ((rc = cloud_build_dev(ctx, dp.p, nullptr, n, pad, &brk))) return rc;
  CK(dist.alloc(nf));
  CK(nn_idx.alloc(nf));
  k_nn_below<<<blocks_for(nf, 128), 128, 0, s>>>(brk.view, cent.p, nf, inner, nn_idx.p, dist.p,
                                                  ctx->d_status);
  CK(cudaGetLastError());
  CK(dns.alloc(size_t(3) * n));
  CK(dnf.alloc(size_t(3) * n));
  if ((rc = macro_normals(ctx, dp.p, n, cent.p, normals.p, areas.p, dfrac.p, nf, dist.p, 0, inner,
                          outer, pad, dns.p)) ||
      (rc = macro_normals(ctx, dp.p, n, cent.p, normals.p, areas.p, dfrac.p, nf, dist.p, 1, inner,
                          outer, pad, dnf.p)))
    return rc;
  DBuf<uint8_t> dvalid, rflag;
  CK(dfr.alloc(size_t(3) * n));
  CK(ddih.alloc(n));
  CK(dvalid.alloc(n));
  k_brk_frames<<<blocks_for(n), 256, 0, s>>>(dns.p, dnf.p, n, dfr.p, dvalid.p, ddih.p);
  CK(cudaGetLastError());

  // R 3.5.5 the hypothesis subset: the valid voxel representatives.
  DBuf<uint32_t> rep, dsub;
  uint32_t n_rep = 0, ns_count = 0;
  if ((rc = voxel_reps(ctx, dp.p, n, brk_voxel * t, rep, n_rep))) return rc;
  CK(rflag.alloc(std::max<uint32_t>(n_rep, 1)));
  if (n_rep) {
    k_valid_reps<<<blocks_for(n_rep), 256, 0, s>>>(rep.p, n_rep, dvalid.p, rflag.p);
    CK(cudaGetLastError());
  }
  if ((rc = select_flagged(ctx, rep.p, rflag.p, n_rep, dsub, ns_count))) return rc;
  *n_sub = ns_count;
  CK(cudaMemcpyAsync(p, dp.p, sizeof(double) * 3 * size_t(n), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(ns, dns.p, sizeof(double) * 3 * size_t(n), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(nfr, dnf.p, sizeof(double) * 3 * size_t(n), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(fr, dfr.p, sizeof(double) * 3 * size_t(n), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(dih, ddih.p, sizeof(double) * size_t(n), cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(valid, dvalid.p, size_t(n), cudaMemcpyDeviceToHost, s));
  if (ns_count) CK(cudaMemcpyAsync(sub, dsub.p, 4 * size_t(ns_count), cudaMemcpyDeviceToHost, s));
  return finish(ctx, "breaklines", nf, true);
}


// ---- io::load_mesh (io/mod.rs:114-137): PLY in, cleaned mesh out -----------------

struct sherd_host_mesh {
  sherd::meshio::HostMesh m;
};

int sherd_mesh_read(const char *path, sherd_host_mesh **out, uint32_t *nv, uint32_t *nf) {
  if (!path || !out || !nv || !nf) return fail(nullptr, SHERD_E_INVALID, "null argument");
  *out = nullptr;
  *nv = 0;
  *nf = 0;
  auto *h = new sherd_host_mesh;
  std::string err;
  try {
    err = sherd::meshio::read_ply(path, h->m);
  } catch (const std::bad_alloc &) {
    err = "out of host memory";
  }
  if (!err.empty()) {
    delete h;
    return fail(nullptr, SHERD_E_INVALID, std::string(path) + ": " + err);
  }
  if (h->m.v.size() / 3 >= (uint64_t(1) << 32) || h->m.f.size() / 3 >= (uint64_t(1) << 32)) {
    delete h;
    return fail(nullptr, SHERD_E_INVALID, std::string(path) + ": more than 2^32 vertices or faces");
  }
  sherd::meshio::clean(h->m);
  if (h->m.f.empty()) {
    delete h;
    return fail(nullptr, SHERD_E_EMPTY, std::string(path) + ": no triangles");
  }
  *nv = uint32_t(h->m.v.size() / 3);
  *nf = uint32_t(h->m.f.size() / 3);
  *out = h;
  return SHERD_OK;
}

int sherd_host_mesh_copy(const sherd_host_mesh *m, double *v, uint32_t *f) {
  if (!m || !v || !f) return fail(nullptr, SHERD_E_INVALID, "null argument");
  std::copy(m->m.v.begin(), m->m.v.end(), v);
  std::copy(m->m.f.begin(), m->m.f.end(), f);
  return SHERD_OK;
}

int sherd_host_mesh_free(sherd_host_mesh *m) {
  delete m;
  return SHERD_OK;
}

}  // extern "C"
