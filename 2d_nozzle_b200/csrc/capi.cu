// capi.cu -- the C ABI: table upload, kernel dispatch, layout conversion,
// norms, and the graph-captured steady-march solver.
//
// Dispatch instantiates the element kernel for triangles p = 0..3 (affine and
// general geometry) and quadrilaterals p = 0..3 (general geometry).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <utility>
#include <vector>

#include "adjoint_dispatch.cuh"
#include "element.cuh"
#include "forward_dispatch.cuh"
#include "split.cuh"
#include "nozzle_b200.h"

namespace nzb {

static thread_local std::string g_err;

static int fail(const std::string& msg) {
  g_err = msg;
  return -1;
}

static int cuda_check(cudaError_t st, const char* what) {
  if (st != cudaSuccess) return fail(std::string(what) + ": " + cudaGetErrorString(st));
  return 0;
}

static int launch_check(const char* what) { return cuda_check(cudaGetLastError(), what); }

static std::mutex g_tab_mu;
static std::set<std::pair<int, int>> g_tab_done;  // (device, kind * 16 + order)

static bool tables_ready(int kind, int order) {
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_tab_mu);
  return g_tab_done.count({dev, kind * 16 + order}) != 0;
}

static int check_mesh(const nzb_mesh* m) {
  if (!m) return fail("mesh is null");
  if (m->kind != NZB_TRI && m->kind != NZB_QUAD) return fail("unknown element kind");
  if (m->order < 0 || m->order > MAX_ORDER) return fail("order must lie in 0..3");
  if (m->affine && m->kind != NZB_TRI) return fail("affine geometry is for straight-sided triangles");
  if (m->n_elem <= 0) return fail("mesh has no elements");
  if (m->split != 0 && m->split != 1 && m->split != SPLIT_T) return fail("split must be 0, 1 or 4 threads per element");
  if (m->vjp_split != 0 && m->vjp_split != 1 && m->vjp_split != SPLIT_T)
    return fail("vjp_split must be 0, 1 or 4 threads per element");
  if (!m->area || !m->face_nbr || !m->face_code || !m->face_edge || !m->edge_geo)
    return fail("mesh arrays area/face_nbr/face_code/face_edge/edge_geo are required");
  if (!m->geo || (!m->affine && !m->minv))
    return fail(m->affine ? "affine mesh needs geo" : "general mesh needs geo (vertices) and minv");
  if (!tables_ready(m->kind, m->order)) return fail("reference tables not uploaded for this kind/order on this device");
  return 0;
}

constexpr int NT = 128;  // threads per block of the helper kernels

static int64_t blocks_for(int64_t n) { return (n + NT - 1) / NT; }
// Element-kernel blocks for (kind, order): one thread per element, 128 per
// block, or 64 for cubic quads.
static int block_threads(int kind, int order) {
  switch (kind * 16 + order) {
#define NZB_BT(K, P) \
  case K * 16 + P: return Launch<K, P>::NT;
    NZB_BT(0, 0) NZB_BT(0, 1) NZB_BT(0, 2) NZB_BT(0, 3) NZB_BT(1, 0) NZB_BT(1, 1) NZB_BT(1, 2) NZB_BT(1, 3)
#undef NZB_BT
  }
  return 128;
}
// Elements per block of the forward element kernel: 32 with four threads per
// element, else one per thread.
static int element_width(const nzb_mesh& m) {
  return (m.split == SPLIT_T && m.order > 0) ? SPLIT_EB : block_threads(m.kind, m.order);
}
// ... and of the adjoint state kernel.
static int adjoint_width(const nzb_mesh& m) {
  return (m.vjp_split == SPLIT_T && m.order > 0) ? SPLIT_EB : block_threads(m.kind, m.order);
}
// Blocks of the forward element kernel (= norm partial slots of stage 1).
static int64_t element_blocks(const nzb_mesh& m) { return (m.n_elem + element_width(m) - 1) / element_width(m); }
// Blocks of the adjoint state kernel (= defect partial slots).
static int64_t adjoint_blocks(const nzb_mesh& m) { return (m.n_elem + adjoint_width(m) - 1) / adjoint_width(m); }

// A block list (fwd_blocks / vjp_blocks) may list each of the mesh's blocks
// at most once, and leaves block-partial norms undefined.
static int check_block_list(const int32_t* list, int64_t n, int64_t blocks, const double* norm_partial,
                            const char* what) {
  if (!list) return 0;
  if (n < 0 || n > blocks) return fail(std::string(what) + ": the block count must lie in [0, blocks of the mesh]");
  if (norm_partial) return fail(std::string(what) + ": block-partial norms need every block (no block list)");
  return 0;
}

// The element kernels live in forward_tri.cu / forward_quad.cu.
static int dispatch(const nzb_mesh& m, const nzb_physics& ph, const Work& w, cudaStream_t st) {
  if (element_blocks(m) > 0x7fffffff || (m.edge_pass && (m.n_edge + 127) / 128 > 0x7fffffff))
    return fail("too many elements for one launch");
  if (m.edge_pass && w.op != OP_LIMIT && (!m.edge_conn || !m.edge_flux || !m.edge_speed))
    return fail("the edge pass needs edge_conn, edge_flux and edge_speed");
  if (m.edge_pass && (reinterpret_cast<uintptr_t>(m.edge_flux) & 15) != 0)
    return fail("edge_flux must be 16-byte aligned");
  if (check_block_list(m.fwd_blocks, m.n_fwd_blocks, element_blocks(m), w.norm_partial, "fwd_blocks")) return -1;
  if (ph.limiter == 2 && m.order > 0 && (w.op == OP_STAGE || w.op == OP_LIMIT)) {
    if (m.elem_inst && (m.n_inst < 1 || !m.inst_status))
      return fail("the Superbee limiter in a batch needs n_inst (lim_scale holds 4 per instance) and inst_status");
    if (!m.elem_share || !m.lim_means || !m.lim_scale)
      return fail("the Superbee limiter needs elem_share, lim_means and lim_scale");
  }
  const cudaError_t e = m.kind == NZB_TRI ? element_launch_tri(m, ph, w, st) : element_launch_quad(m, ph, w, st);
  return cuda_check(e, "element kernel launch");
}

// ---- layout conversion ------------------------------------------------------
__global__ void k_pack(const double* __restrict__ src, double* __restrict__ dst, int64_t E, int np,
                       const int32_t* __restrict__ perm) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= E * np) return;
  const int64_t e = t % E;
  const int i = (int)(t / E);
  const int64_t r = perm ? perm[e] : e;
  const double* p = src + (r * np + i) * 4;
#pragma unroll
  for (int s = 0; s < 4; ++s) dst[((int64_t)s * np + i) * E + e] = p[s];
}

__global__ void k_unpack(const double* __restrict__ src, double* __restrict__ dst, int64_t E, int np,
                         const int32_t* __restrict__ perm) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= E * np) return;
  const int64_t e = t % E;
  const int i = (int)(t / E);
  const int64_t r = perm ? perm[e] : e;
  double* p = dst + (r * np + i) * 4;
#pragma unroll
  for (int s = 0; s < 4; ++s) p[s] = src[((int64_t)s * np + i) * E + e];
}

// ---- norms --------------------------------------------------------------------
__global__ void __launch_bounds__(NT) k_norm_partial(const double* __restrict__ A, int64_t E, int np,
                                                     double w0, double w1, double w2, double w3,
                                                     double* __restrict__ partial) {
  const int64_t e = (int64_t)blockIdx.x * NT + threadIdx.x;
  double acc = 0.0;
  if (e < E) {
    const double w[4] = {w0, w1, w2, w3};
    for (int s = 0; s < 4; ++s)
      for (int i = 0; i < np; ++i) {
        const double v = A[((int64_t)s * np + i) * E + e] * w[s];
        acc = fma(v, v, acc);
      }
  }
  block_sum_store<NT / 32>(acc, partial + blockIdx.x);
}

// One block, fixed order: thread t sums slots t, t + 1024, ...; then a tree.
__global__ void __launch_bounds__(1024) k_norm_finalize(const double* __restrict__ partial, int64_t n,
                                                        double count, double* __restrict__ out) {
  __shared__ double red[1024];
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += 1024) acc += partial[i];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 512; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = sqrt(red[0] / count);
}

__global__ void k_inverse_mass_general(const double* __restrict__ minv, const double* __restrict__ R,
                                       double* __restrict__ out, int64_t E, int np) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  for (int s = 0; s < 4; ++s)
    for (int i = 0; i < np; ++i) {
      double acc = 0.0;
      for (int j = 0; j < np; ++j)
        acc = fma(minv[((int64_t)i * np + j) * E + e], R[((int64_t)s * np + j) * E + e], acc);
      out[((int64_t)s * np + i) * E + e] = acc;
    }
}

template <int K, int P>
__global__ void k_inverse_mass_affine(const double* __restrict__ geo, const double* __restrict__ R,
                                      double* __restrict__ out, int64_t E) {
  using S = Shape<K, P>;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  const double det = geo[4 * E + e];
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    double r[S::NP];
#pragma unroll
    for (int j = 0; j < S::NP; ++j) r[j] = R[((int64_t)s * S::NP + j) * E + e];
#pragma unroll
    for (int i = 0; i < S::NP; ++i) {
      double acc = 0.0;
#pragma unroll
      for (int j = 0; j < S::NP; ++j) acc = fma(tab<K, P>(S::O_MINV + i * S::NP + j), r[j], acc);
      out[((int64_t)s * S::NP + i) * E + e] = acc / det;
    }
  }
}

// ---- solver ---------------------------------------------------------------------
struct Solver {
  nzb_mesh mesh;
  nzb_physics phys;
  nzb_buffers buf;
  int ssprk3;
  double dt_factor;
  int device;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  std::map<int, cudaGraphExec_t> graphs;
};

static int enqueue_step(const Solver& s, cudaStream_t st) {
  Work w{};
  w.op = OP_STAGE;
  w.dt = s.buf.dt;
  w.counters = s.buf.counters;
  w.dt_factor = s.dt_factor;
  // stage 1: S0 -> S2 (ssprk3) or S0 -> S1 (euler), with dt and the norm
  w.V = s.buf.S0;
  w.U0 = nullptr;
  w.out = s.ssprk3 ? s.buf.S2 : s.buf.S1;
  w.norm_partial = s.buf.norm_partial;
  w.stage = 1;
  w.a = 0.0;
  w.b = 1.0;
  if (dispatch(s.mesh, s.phys, w, st)) return -1;
  if (!s.ssprk3) {
    return cuda_check(cudaMemcpyAsync(s.buf.S0, s.buf.S1, sizeof(double) * 4 * s.mesh.n_elem *
                                                              n_basis(s.mesh.kind, s.mesh.order),
                                      cudaMemcpyDeviceToDevice, st),
                      "euler copy-back");
  }
  w.norm_partial = nullptr;
  // stage 2: S1 = limit(3/4 S0 + 1/4 (S2 + dt F(S2)))
  w.V = s.buf.S2;
  w.U0 = s.buf.S0;
  w.out = s.buf.S1;
  w.stage = 2;
  w.a = 0.75;
  w.b = 0.25;
  if (dispatch(s.mesh, s.phys, w, st)) return -1;
  // stage 3: S0 = limit(1/3 S0 + 2/3 (S1 + dt F(S1))), in place over U0
  w.V = s.buf.S1;
  w.U0 = s.buf.S0;
  w.out = s.buf.S0;
  w.stage = 3;
  w.a = 1.0 / 3.0;
  w.b = 2.0 / 3.0;
  return dispatch(s.mesh, s.phys, w, st);
}

static int graph_for(Solver& s, int n, cudaGraphExec_t* out) {
  auto it = s.graphs.find(n);
  if (it != s.graphs.end()) {
    *out = it->second;
    return 0;
  }
  cudaGraph_t g = nullptr;
  if (cuda_check(cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeThreadLocal), "begin capture")) return -1;
  int rc = 0;
  for (int i = 0; i < n && rc == 0; ++i) rc = enqueue_step(s, s.stream);
  const cudaError_t end = cudaStreamEndCapture(s.stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return -1;
  }
  if (cuda_check(end, "end capture")) return -1;
  cudaGraphExec_t ex = nullptr;
  const cudaError_t inst = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (cuda_check(inst, "graph instantiate")) return -1;
  s.graphs[n] = ex;
  *out = ex;
  return 0;
}

// ---- batched march ----------------------------------------------------------------
// Copy S1 -> S0 for the elements of running instances (forward Euler in a batch).
__global__ void k_masked_copy(const double* __restrict__ src, double* __restrict__ dst, int64_t E, int np,
                              const int32_t* __restrict__ elem_inst, const int32_t* __restrict__ status) {
  const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= E * np * 4) return;
  const int64_t e = t % E;
  if (elem_inst && status[elem_inst[e]] != 0) return;
  dst[t] = src[t];
}

// One block per instance: the weighted RMS of its last stage-1 rate, summed in a
// fixed order, then the reference march's tests (src/timestepping/march.py:
// 157-220) on that residual.
__global__ void __launch_bounds__(256) k_batch_check(nzb_batch_march bm, int n_steps, int first) {
  const int64_t inst = blockIdx.x;
  if (inst >= bm.n_inst || bm.status[inst] != 0) return;
  __shared__ double red[256];
  double acc = 0.0;
  for (int64_t e = bm.inst_begin[inst] + threadIdx.x; e < bm.inst_end[inst]; e += 256) acc += bm.elem_norm[e];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const double res = sqrt(red[0] / bm.inst_count[inst]);
  const int done = bm.iterations[inst] + n_steps;
  bm.iterations[inst] = done;
  bm.res[inst] = res;
  int st = 0;
  if (first) {
    bm.res0[inst] = res;
    if (!isfinite(res))
      st = 2;
    else if (res <= bm.inst_tol[inst])
      st = 1;
  } else if (!isfinite(res)) {
    st = 2;
  } else if (res <= bm.inst_tol[inst]) {
    st = 1;
  } else if (res > bm.divergence_factor * bm.res0[inst]) {
    st = 3;
  } else {
    const int W = bm.stall_window;
    const int c = bm.window_count[inst];
    bm.window[inst * W + (c % W)] = res;
    bm.window_count[inst] = c + 1;
    if (c + 1 >= W) {
      double best = 1e300, worst = -1e300;
      for (int k = 0; k < W; ++k) {
        const double v = bm.window[inst * W + k];
        best = v < best ? v : best;
        worst = v > worst ? v : worst;
      }
      if (worst > 0.0 && best / worst > bm.stall_ratio) st = 4;
    }
  }
  if (st == 0 && done >= bm.max_iterations) st = 5;
  bm.status[inst] = st;
  if (st == 0) atomicAdd(bm.n_running, 1);
}

struct Batch {
  std::vector<nzb_mesh> mesh;
  std::vector<nzb_physics> phys;
  std::vector<nzb_buffers> buf;
  std::vector<int64_t> offset;
  std::vector<double> factor;
  nzb_batch_march bm;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  // buckets march concurrently: one capture stream and join event per bucket
  std::vector<cudaStream_t> bstream;
  std::vector<cudaEvent_t> bdone;
  cudaEvent_t fork = nullptr;
  std::map<int, cudaGraphExec_t> graphs;  // key: 2 * n + first
};

static int enqueue_bucket_step(const Batch& B, size_t b, cudaStream_t st) {
  {
    const nzb_mesh& m = B.mesh[b];
    if (m.fwd_blocks && m.n_fwd_blocks == 0) return 0;  // every instance of the bucket has retired
    const nzb_buffers& bf = B.buf[b];
    const bool ssp = m.order > 0;
    Work w{};
    w.op = OP_STAGE;
    w.dt = bf.dt;
    w.dt_factor = B.factor[b];
    w.V = bf.S0;
    w.out = ssp ? bf.S2 : bf.S1;
    w.elem_norm = B.bm.elem_norm + B.offset[b];
    w.stage = 1;
    w.a = 0.0;
    w.b = 1.0;
    if (dispatch(m, B.phys[b], w, st)) return -1;
    if (!ssp) {
      const int np = n_basis(m.kind, m.order);
      const int64_t n = m.n_elem * np * 4;
      k_masked_copy<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(bf.S1, bf.S0, m.n_elem, np, m.elem_inst, m.inst_status);
      return launch_check("masked copy");
    }
    w.elem_norm = nullptr;
    w.V = bf.S2;
    w.U0 = bf.S0;
    w.out = bf.S1;
    w.stage = 2;
    w.a = 0.75;
    w.b = 0.25;
    if (dispatch(m, B.phys[b], w, st)) return -1;
    w.V = bf.S1;
    w.out = bf.S0;
    w.stage = 3;
    w.a = 1.0 / 3.0;
    w.b = 2.0 / 3.0;
    if (dispatch(m, B.phys[b], w, st)) return -1;
  }
  return 0;
}

static int batch_graph(Batch& B, int n, int first, cudaGraphExec_t* out) {
  const int key = 2 * n + (first ? 1 : 0);
  auto it = B.graphs.find(key);
  if (it != B.graphs.end()) {
    *out = it->second;
    return 0;
  }
  cudaGraph_t g = nullptr;
  if (cuda_check(cudaStreamBeginCapture(B.stream, cudaStreamCaptureModeThreadLocal), "begin capture")) return -1;
  // fork: every bucket's n steps on its own stream, then join before the check
  int rc = cuda_check(cudaEventRecord(B.fork, B.stream), "fork record");
  for (size_t b = 0; b < B.mesh.size() && rc == 0; ++b) {
    rc = cuda_check(cudaStreamWaitEvent(B.bstream[b], B.fork, 0), "fork wait");
    for (int i = 0; i < n && rc == 0; ++i) rc = enqueue_bucket_step(B, b, B.bstream[b]);
    if (rc == 0) rc = cuda_check(cudaEventRecord(B.bdone[b], B.bstream[b]), "join record");
    if (rc == 0) rc = cuda_check(cudaStreamWaitEvent(B.stream, B.bdone[b], 0), "join wait");
  }
  if (rc == 0) rc = cuda_check(cudaMemsetAsync(B.bm.n_running, 0, sizeof(int32_t), B.stream), "memset");
  if (rc == 0) {
    k_batch_check<<<(unsigned)B.bm.n_inst, 256, 0, B.stream>>>(B.bm, n, first);
    rc = launch_check("batch check");
  }
  const cudaError_t end = cudaStreamEndCapture(B.stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return -1;
  }
  if (cuda_check(end, "end capture")) return -1;
  cudaGraphExec_t ex = nullptr;
  const cudaError_t inst = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (cuda_check(inst, "graph instantiate")) return -1;
  B.graphs[key] = ex;
  *out = ex;
  return 0;
}

// ---- adjoint ------------------------------------------------------------------
// The adjoint kernels live in adjoint_tri.cu / adjoint_quad.cu.
static int dispatch_vjp(const nzb_mesh& m, const nzb_physics& ph, const AdjWork& w, cudaStream_t st) {
  if (adjoint_blocks(m) > 0x7fffffff) return fail("too many elements for one launch");
  if (check_block_list(m.vjp_blocks, m.n_vjp_blocks, adjoint_blocks(m), w.norm_partial, "vjp_blocks")) return -1;
  const cudaError_t e = m.kind == NZB_TRI ? vjp_launch_tri(m, ph, w, st) : vjp_launch_quad(m, ph, w, st);
  return cuda_check(e, "vjp kernel launch");
}

static int dispatch_vjp_coords(const nzb_mesh& m, const nzb_physics& ph, const CoordWork& w, cudaStream_t st) {
  if ((m.n_elem + 127) / 128 > 0x7fffffff) return fail("too many elements for one launch");
  const cudaError_t e = m.kind == NZB_TRI ? vjp_coords_launch_tri(m, ph, w, st) : vjp_coords_launch_quad(m, ph, w, st);
  return cuda_check(e, "vjp_coords kernel launch");
}

__global__ void k_local_dt(const double* __restrict__ area, const double* __restrict__ wave, int64_t E, double coef,
                           double* __restrict__ dt) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  const double d = wave[e] < FLOOR ? FLOOR : wave[e];
  dt[e] = coef * 2.0 * area[e] / d;
}

// One block per instance: rms of the defect in a fixed order, then the adjoint
// march's tests (src/sensitivity.py:366-383).  n_steps = 0 records res0.
__global__ void __launch_bounds__(256) k_adjoint_check(nzb_adjoint_march am, int n_steps) {
  const int64_t inst = blockIdx.x;
  if (inst >= am.n_inst || am.status[inst] != 0) return;
  __shared__ double red[256];
  double acc = 0.0;
  for (int64_t e = am.inst_begin[inst] + threadIdx.x; e < am.inst_end[inst]; e += 256) acc += am.elem_norm[e];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  const double res = sqrt(red[0] / am.inst_count[inst]);
  int st = 0;
  if (n_steps == 0) {
    am.res0[inst] = res;
    am.res[inst] = res;
    am.iterations[inst] = 0;
    if (!isfinite(res))
      st = 2;
    else if (res == 0.0)
      st = 1;
  } else {
    const int done = am.iterations[inst] + n_steps;
    am.iterations[inst] = done;
    am.res[inst] = res;
    if (!isfinite(res))
      st = 2;
    else if (res <= am.tolerance * am.res0[inst])
      st = 1;
    else if (done >= am.max_iterations)
      st = 5;
  }
  am.status[inst] = st;
  if (st == 0) atomicAdd(am.n_running, 1);
}

struct AdjBatch {
  std::vector<nzb_mesh> mesh;
  std::vector<nzb_physics> phys;
  std::vector<nzb_adjoint_buffers> buf;
  std::vector<int64_t> offset;
  nzb_adjoint_march am;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  std::vector<cudaStream_t> bstream;
  std::vector<cudaEvent_t> bdone;
  cudaEvent_t fork = nullptr;
  std::map<int, cudaGraphExec_t> graphs;  // key: steps per chunk
};

static int enqueue_adjoint_step(const AdjBatch& A, size_t b, cudaStream_t st) {
  const nzb_adjoint_buffers& bf = A.buf[b];
  AdjWork w{};
  w.mode = ADJ_RK4;
  w.U = bf.U;
  w.seed = bf.seed;
  w.lam0 = bf.lam;
  w.dt = bf.dt;
  w.f0 = bf.f0;
  w.f1 = bf.f1;
  w.f2 = bf.f2;
  // stage inputs alternate between two buffers, so no stage reads what it writes
  const double* in[4] = {bf.lam, bf.Y1, bf.Y2, bf.Y1};
  double* outp[4] = {bf.Y1, bf.Y2, bf.Y1, nullptr};
  for (int k = 0; k < 4; ++k) {
    w.stage = k;
    w.lam = in[k];
    w.out = outp[k];
    if (dispatch_vjp(A.mesh[b], A.phys[b], w, st)) return -1;
  }
  return 0;
}

static int enqueue_adjoint_defect(const AdjBatch& A, size_t b, cudaStream_t st) {
  const nzb_adjoint_buffers& bf = A.buf[b];
  AdjWork w{};
  w.mode = ADJ_DEFECT;
  w.U = bf.U;
  w.seed = bf.seed;
  w.lam = bf.lam;
  w.elem_norm = A.am.elem_norm + A.offset[b];
  return dispatch_vjp(A.mesh[b], A.phys[b], w, st);
}

static int adjoint_graph(AdjBatch& A, int n, cudaGraphExec_t* out) {
  auto it = A.graphs.find(n);
  if (it != A.graphs.end()) {
    *out = it->second;
    return 0;
  }
  cudaGraph_t g = nullptr;
  if (cuda_check(cudaStreamBeginCapture(A.stream, cudaStreamCaptureModeThreadLocal), "begin capture")) return -1;
  int rc = cuda_check(cudaEventRecord(A.fork, A.stream), "fork record");
  for (size_t b = 0; b < A.mesh.size() && rc == 0; ++b) {
    rc = cuda_check(cudaStreamWaitEvent(A.bstream[b], A.fork, 0), "fork wait");
    for (int i = 0; i < n && rc == 0; ++i) rc = enqueue_adjoint_step(A, b, A.bstream[b]);
    if (rc == 0) rc = enqueue_adjoint_defect(A, b, A.bstream[b]);
    if (rc == 0) rc = cuda_check(cudaEventRecord(A.bdone[b], A.bstream[b]), "join record");
    if (rc == 0) rc = cuda_check(cudaStreamWaitEvent(A.stream, A.bdone[b], 0), "join wait");
  }
  if (rc == 0) rc = cuda_check(cudaMemsetAsync(A.am.n_running, 0, sizeof(int32_t), A.stream), "memset");
  if (rc == 0) {
    k_adjoint_check<<<(unsigned)A.am.n_inst, 256, 0, A.stream>>>(A.am, n);
    rc = launch_check("adjoint check");
  }
  const cudaError_t end = cudaStreamEndCapture(A.stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return -1;
  }
  if (cuda_check(end, "end capture")) return -1;
  cudaGraphExec_t ex = nullptr;
  const cudaError_t inst = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  if (cuda_check(inst, "graph instantiate")) return -1;
  A.graphs[n] = ex;
  *out = ex;
  return 0;
}

static AdjWork adj_work(const nzb_adjoint_args& a) {
  AdjWork w{};
  w.mode = a.mode;
  w.stage = a.stage;
  w.U = a.U;
  w.lam = a.lam;
  w.seed = a.seed;
  w.out = a.out;
  w.lam0 = a.lam0;
  w.dt = a.dt;
  w.f0 = a.f0;
  w.f1 = a.f1;
  w.f2 = a.f2;
  w.norm_partial = a.norm_partial;
  w.elem_norm = a.elem_norm;
  return w;
}

// ---- the norm without caller-provided scratch ------------------------------------
// Partial sums of nzb_norm_noalloc live in this file-scope array: one slot per
// block of the partial-sum kernel, 128 elements per block.  Every GPU that
// loads the library holds it (512 KiB) until the process exits.
constexpr int64_t NOALLOC_MAX_BLOCKS = 65536;
constexpr int64_t NOALLOC_MAX_ELEMENTS = NOALLOC_MAX_BLOCKS * NT;
static __device__ __align__(256) double g_norm_scratch[NOALLOC_MAX_BLOCKS];

static std::mutex g_scratch_mu;
static std::map<int, double*> g_scratch_addr;  // device -> g_norm_scratch there

// The device address of g_norm_scratch on the current device, looked up once
// per device with that device current.  In host code the symbol itself is only
// a host-side stand-in, never a device address.
static int scratch_address(double** out) {
  int dev = -1;
  if (cuda_check(cudaGetDevice(&dev), "cudaGetDevice")) return -1;
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  auto it = g_scratch_addr.find(dev);
  if (it != g_scratch_addr.end()) {
    *out = it->second;
    return 0;
  }
  double* p = nullptr;
  if (cuda_check(cudaGetSymbolAddress((void**)&p, g_norm_scratch), "cudaGetSymbolAddress(norm scratch)")) return -1;
  g_scratch_addr[dev] = p;
  *out = p;
  return 0;
}

}  // namespace nzb

using namespace nzb;

extern "C" {

int nzb_version(void) { return 1; }

const char* nzb_last_error(void) { return g_err.c_str(); }

int64_t nzb_table_size(int kind, int order) {
  if ((kind != 0 && kind != 1) || order < 0 || order > MAX_ORDER) return -1;
  return slot_size(kind, order);
}

int nzb_upload_tables(int kind, int order, const double* tables, int64_t n) {
  if (nzb_table_size(kind, order) < 0) return fail("unsupported kind/order");
  if (n != slot_size(kind, order)) return fail("table size mismatch");
  if (!tables) return fail("tables is null");
  // every translation unit holds its own copy of the tables
  const size_t off = (size_t)slot_offset(kind, order);
  if (cuda_check(cudaMemcpyToSymbol(c_tab, tables, sizeof(double) * n, sizeof(double) * off), "table upload") ||
      cuda_check(upload_tables_fwd_tri(tables, (size_t)n, off), "table upload (triangles)") ||
      cuda_check(upload_tables_fwd_quad(tables, (size_t)n, off), "table upload (quadrilaterals)") ||
      cuda_check(upload_tables_tri(tables, (size_t)n, off), "table upload (adjoint, triangles)") ||
      cuda_check(upload_tables_quad(tables, (size_t)n, off), "table upload (adjoint, quadrilaterals)") ||
      cuda_check(kind == NZB_TRI ? prepare_split_tri(order) : prepare_split_quad(order), "split kernel attributes") ||
      cuda_check(kind == NZB_TRI ? prepare_vjp_split_tri(order) : prepare_vjp_split_quad(order),
                 "adjoint split kernel attributes"))
    return -1;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lk(g_tab_mu);
  g_tab_done.insert({dev, kind * 16 + order});
  return 0;
}

int nzb_pack_state(const double* src, double* dst, int64_t E, int np, const int32_t* perm, void* stream) {
  if (!src || !dst || E <= 0 || np <= 0) return fail("pack: bad arguments");
  const int64_t n = E * np;
  k_pack<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(src, dst, E, np, perm);
  return launch_check("pack launch");
}

int nzb_unpack_state(const double* src, double* dst, int64_t E, int np, const int32_t* perm, void* stream) {
  if (!src || !dst || E <= 0 || np <= 0) return fail("unpack: bad arguments");
  const int64_t n = E * np;
  k_unpack<<<(unsigned)((n + 255) / 256), 256, 0, (cudaStream_t)stream>>>(src, dst, E, np, perm);
  return launch_check("unpack launch");
}

int nzb_residual(const nzb_mesh* mesh, const nzb_physics* phys, int op, const double* U, double* out,
                 double* wave, void* stream) {
  if (check_mesh(mesh)) return -1;
  if (!phys || !U || !out) return fail("residual: null argument");
  if (op != NZB_OP_RESIDUAL && op != NZB_OP_RATE) return fail("residual: unknown op");
  if (U == out) return fail("residual: out must not alias U");
  Work w{};
  w.op = op == NZB_OP_RESIDUAL ? OP_RESIDUAL : OP_RATE;
  w.V = U;
  w.out = out;
  w.wave = wave;
  return dispatch(*mesh, *phys, w, (cudaStream_t)stream);
}

int nzb_observables(const nzb_mesh* mesh, const nzb_physics* phys, const nzb_obs_args* args, void* stream) {
  if (check_mesh(mesh)) return -1;
  if (!phys || !args || !args->U || !args->bseg || !args->eseg || !args->out) return fail("observables: null argument");
  if (args->n_seg <= 0) return fail("observables: no instances");
  if (!mesh->edge_conn || !mesh->edge_geo || !mesh->area) return fail("observables: the mesh needs edge_conn, edge_geo and area");
  if (!(args->r_gas > 0.0) || !(args->s_t > 0.0)) return fail("observables: r_gas and s_t must be positive");
  const cudaStream_t st = (cudaStream_t)stream;
  const cudaError_t e = mesh->kind == NZB_TRI ? observables_launch_tri(*mesh, *phys, *args, st)
                                              : observables_launch_quad(*mesh, *phys, *args, st);
  return cuda_check(e, "observables launch");
}

int nzb_geometry(const nzb_mesh* mesh, const nzb_geometry_args* args, void* stream) {
  if (check_mesh(mesh)) return -1;
  if (!args || !args->X || !args->elem_nodes || !args->edge_conn || !args->geo || !args->area || !args->edge_geo)
    return fail("geometry: null argument");
  if (!mesh->affine && !args->minv) return fail("geometry: general geometry needs minv");
  if (mesh->n_edge <= 0) return fail("geometry: the mesh has no edges");
  if ((mesh->n_elem + 127) / 128 > 0x7fffffff || (mesh->n_edge + 127) / 128 > 0x7fffffff)
    return fail("geometry: too many elements or edges for one launch");
  const cudaStream_t st = (cudaStream_t)stream;
  const cudaError_t e = mesh->kind == NZB_TRI ? geometry_launch_tri(*mesh, *args, st)
                                              : geometry_launch_quad(*mesh, *args, st);
  return cuda_check(e, "geometry launch");
}

// ---- any order, curved elements (generic.cuh)
static int check_gen(const nzb_gen_mesh* m, const nzb_physics* ph) {
  if (!m || !ph) return fail("generic: null mesh or physics");
  if (m->np < 1 || m->np > 36 || m->nqv < 1 || m->nqf < 1 || (m->nface != 3 && m->nface != 4))
    return fail("generic: sizes out of range (NP 1..36, 3 or 4 faces)");
  if (m->n_elem < 1 || m->n_int < 0 || m->n_bnd < 0 || (m->n_elem + 127) / 128 > 0x7fffffff ||
      (m->n_int + m->n_bnd + 127) / 128 > 0x7fffffff)
    return fail("generic: bad element or edge count");
  if (!m->phi_vol || !m->phi_face || !m->w_face || !m->face_edge || !m->face_side || !m->face_sign || !m->edge_elem ||
      !m->edge_face || (m->n_bnd && !m->edge_tag) || !m->edge_normal || !m->edge_jac || !m->edge_length)
    return fail("generic: missing mesh array");
  return 0;
}

int64_t nzb_gen_blocks(const nzb_gen_mesh* mesh) { return mesh ? (mesh->n_elem + 127) / 128 : -1; }

int nzb_gen_superbee(const nzb_gen_mesh* mesh, const nzb_physics* phys, double* U, const double* share,
                     double* means, double* scale, unsigned long long* counters, void* stream) {
  if (check_gen(mesh, phys)) return -1;
  if (!U || !share || !means || !scale) return fail("gen_superbee: null array");
  if (!mesh->mean_weights) return fail("gen_superbee: the mesh lacks mean_weights");
  return cuda_check(gen_superbee_launch(*mesh, *phys, U, share, means, scale, counters, (cudaStream_t)stream),
                    "generic superbee launch");
}

int nzb_gen_initial_state(const nzb_gen_mesh* mesh, const nzb_physics* phys, const nzb_gen_initial_args* args,
                          void* stream) {
  if (!mesh || !phys || !args) return fail("gen_initial_state: null mesh, physics or arguments");
  const nzb_gen_mesh& m = *mesh;
  const nzb_gen_initial_args& a = *args;
  if (m.np < 1 || m.np > 36 || m.nqv < 1 || m.nqv > 64) return fail("gen_initial_state: sizes out of range");
  if (a.ng < 3 || a.ng > 16) return fail("gen_initial_state: geometry nodes per element out of range (3..16)");
  if (m.n_elem < 1 || m.n_elem > 0x7fffffff) return fail("gen_initial_state: bad element count");
  if (a.n_q1d < 2) return fail("gen_initial_state: the quasi-1D solution needs at least two points");
  if (!m.phi_vol || !a.X || !a.elem_nodes || !a.geom_vol || !a.dgeom_dxi || !a.dgeom_deta || !a.w_vol ||
      !a.inv_mass || !a.wall || !a.q1d || !a.out)
    return fail("gen_initial_state: missing array");
  return cuda_check(gen_initial_launch(m, *phys, a, (cudaStream_t)stream), "generic initial state launch");
}

int nzb_gen_observables(const nzb_gen_mesh* mesh, const nzb_physics* phys, const nzb_gen_obs_args* args,
                        void* stream) {
  if (check_gen(mesh, phys)) return -1;
  if (!args) return fail("gen_observables: null arguments");
  const nzb_gen_obs_args& a = *args;
  if (a.ng < 3 || a.ng > 16) return fail("gen_observables: geometry nodes per element out of range (3..16)");
  if (!a.X || !a.elem_nodes || !a.dgeom_dxi || !a.dgeom_deta || !a.w_vol || !a.U || !a.out || !mesh->elem_area)
    return fail("gen_observables: missing array");
  return cuda_check(gen_observables_launch(*mesh, *phys, a, (cudaStream_t)stream), "generic observables launch");
}

int nzb_gen_geometry(const nzb_gen_mesh* mesh, const nzb_gen_geometry_args* args, void* stream) {
  if (!mesh || !args) return fail("gen_geometry: null mesh or arguments");
  const nzb_gen_mesh& m = *mesh;
  const nzb_gen_geometry_args& a = *args;
  if (m.np < 1 || m.np > 36 || m.nqv < 1 || m.nqv > 64 || m.nqf < 1 || m.nqf > 16 || (m.nface != 3 && m.nface != 4))
    return fail("gen_geometry: sizes out of range (NP 1..36, NQV 1..64, NQF 1..16, 3 or 4 faces)");
  if (a.ng < 3 || a.ng > 16) return fail("gen_geometry: geometry nodes per element out of range (3..16)");
  if (m.n_elem < 1 || m.n_elem > 0x7fffffff || m.n_int < 0 || m.n_bnd < 0 ||
      (m.n_int + m.n_bnd + 127) / 128 > 0x7fffffff)
    return fail("gen_geometry: bad element or edge count");
  if (!m.phi_vol || !m.phi_face || !m.w_face || !m.face_side || !m.edge_elem || !m.edge_face)
    return fail("gen_geometry: missing mesh array");
  if (!a.X || !a.elem_nodes || !a.w_vol || !a.dphi_dxi || !a.dphi_deta || !a.dgeom_dxi || !a.dgeom_deta ||
      !a.dgeom_dsigma || !a.grad_x || !a.grad_y || !a.grad_x_m || !a.grad_y_m || !a.face_basis_m || !a.inv_mass ||
      !a.elem_area || !a.mean_weights || !a.edge_normal || !a.edge_jac || !a.edge_length || !a.bad)
    return fail("gen_geometry: missing argument array");
  if (cuda_check(cudaMemsetAsync(a.bad, 0, sizeof(int32_t), (cudaStream_t)stream), "gen_geometry memset")) return -1;
  return cuda_check(gen_geometry_launch(m, a, (cudaStream_t)stream), "gen_geometry launch");
}

int nzb_gen_rate(const nzb_gen_mesh* mesh, const nzb_physics* phys, int unfolded, const double* U, double* out,
                 double* wave, double* fw, double* smax, void* stream) {
  if (check_gen(mesh, phys)) return -1;
  if (!U || !out || !fw || !smax) return fail("gen_rate: null array");
  if (unfolded ? (!mesh->grad_x || !mesh->grad_y) : (!mesh->grad_x_m || !mesh->grad_y_m || !mesh->face_basis_m))
    return fail("gen_rate: the mesh lacks the operators of this mode");
  return cuda_check(gen_rate_launch(*mesh, *phys, unfolded, U, out, wave, fw, smax, (cudaStream_t)stream),
                    "generic rate launch");
}

int nzb_gen_limit(const nzb_gen_mesh* mesh, const nzb_physics* phys, double* U, unsigned long long* counters,
                  void* stream) {
  if (check_gen(mesh, phys)) return -1;
  if (!U || !mesh->mean_weights) return fail("gen_limit: null array");
  if (phys->limiter != 1) return 0;
  return cuda_check(gen_limit_launch(*mesh, *phys, U, counters, (cudaStream_t)stream), "generic limiter launch");
}

int nzb_gen_update(const nzb_gen_mesh* mesh, const nzb_physics* phys, const nzb_gen_update_args* args, void* stream) {
  if (check_gen(mesh, phys)) return -1;
  if (!args || !args->V || !args->F || !args->dt || !args->out || (args->a != 0.0 && !args->U0) ||
      (args->stage == 1 && (!args->wave || !mesh->elem_area)))
    return fail("gen_update: null array");
  return cuda_check(gen_update_launch(*mesh, *phys, *args, (cudaStream_t)stream), "generic update launch");
}

int nzb_initial_state(const nzb_mesh* mesh, const nzb_physics* phys, const nzb_initial_args* args, void* stream) {
  if (check_mesh(mesh)) return -1;
  if (!phys || !args || !args->verts || !args->wall || !args->q1d || !args->q1d_begin || !args->out)
    return fail("initial_state: null argument");
  if (!mesh->affine && !mesh->minv) return fail("initial_state: general geometry needs the mesh's minv");
  if ((mesh->n_elem + 127) / 128 > 0x7fffffff) return fail("initial_state: too many elements for one launch");
  const cudaStream_t st = (cudaStream_t)stream;
  const cudaError_t e = mesh->kind == NZB_TRI ? initial_launch_tri(*mesh, *phys, *args, st)
                                              : initial_launch_quad(*mesh, *phys, *args, st);
  return cuda_check(e, "initial state launch");
}

int nzb_inverse_mass(const nzb_mesh* mesh, const double* R, double* out, void* stream) {
  if (check_mesh(mesh)) return -1;
  if (!R || !out) return fail("inverse_mass: null argument");
  const int64_t E = mesh->n_elem;
  const unsigned nb = (unsigned)((E + 127) / 128);
  cudaStream_t st = (cudaStream_t)stream;
  if (!mesh->affine) {
    k_inverse_mass_general<<<nb, 128, 0, st>>>(mesh->minv, R, out, E, n_basis(mesh->kind, mesh->order));
    return launch_check("inverse mass launch");
  }
  switch (mesh->order) {
    case 0: k_inverse_mass_affine<0, 0><<<nb, 128, 0, st>>>(mesh->geo, R, out, E); break;
    case 1: k_inverse_mass_affine<0, 1><<<nb, 128, 0, st>>>(mesh->geo, R, out, E); break;
    case 2: k_inverse_mass_affine<0, 2><<<nb, 128, 0, st>>>(mesh->geo, R, out, E); break;
    default: k_inverse_mass_affine<0, 3><<<nb, 128, 0, st>>>(mesh->geo, R, out, E); break;
  }
  return launch_check("inverse mass launch");
}

int nzb_limit(const nzb_mesh* mesh, const nzb_physics* phys, double* U, unsigned long long* counters,
              uint8_t* flags, void* stream) {
  if (check_mesh(mesh)) return -1;
  if (!phys || !U) return fail("limit: null argument");
  Work w{};
  w.op = OP_LIMIT;
  w.V = U;
  w.out = U;
  w.counters = counters;
  w.flags = flags;
  return dispatch(*mesh, *phys, w, (cudaStream_t)stream);
}

int nzb_stage(const nzb_mesh* mesh, const nzb_physics* phys, const nzb_stage_args* a, void* stream) {
  if (check_mesh(mesh)) return -1;
  if (!phys || !a || !a->V || !a->out || !a->dt) return fail("stage: null argument");
  if (a->stage < 1 || a->stage > 3) return fail("stage must be 1, 2 or 3");
  if (a->stage > 1 && !a->U0) return fail("stages 2 and 3 need U0");
  if (a->out == a->V) return fail("stage: out must not alias V");
  Work w{};
  w.op = OP_STAGE;
  w.V = a->V;
  w.U0 = a->U0;
  w.out = a->out;
  w.dt = a->dt;
  w.norm_partial = a->norm_partial;
  w.elem_norm = a->elem_norm;
  w.counters = a->counters;
  w.flags = a->flags;
  w.dt_factor = a->dt_factor;
  w.a = a->a;
  w.b = a->b;
  w.stage = a->stage;
  return dispatch(*mesh, *phys, w, (cudaStream_t)stream);
}

int64_t nzb_norm_blocks(int64_t n_elem) { return n_elem <= 0 ? 0 : (n_elem + SPLIT_EB - 1) / SPLIT_EB; }

int64_t nzb_element_blocks(const nzb_mesh* mesh) { return mesh ? element_blocks(*mesh) : -1; }

int64_t nzb_block_width(const nzb_mesh* mesh, int which) {
  if (!mesh || (which != 0 && which != 1)) return -1;
  return which == 0 ? element_width(*mesh) : adjoint_width(*mesh);
}

int nzb_norm_finalize(const double* partial, int64_t n_partial, double count, double* out, void* stream) {
  if (!partial || !out || n_partial <= 0 || !(count > 0)) return fail("norm_finalize: bad arguments");
  k_norm_finalize<<<1, 1024, 0, (cudaStream_t)stream>>>(partial, n_partial, count, out);
  return launch_check("norm finalize launch");
}

int nzb_norm(const double* A, int64_t E, int np, const double* w4, double* partial, double* out, void* stream) {
  if (!A || !w4 || !partial || !out || E <= 0 || np <= 0) return fail("norm: bad arguments");
  const int64_t nb = blocks_for(E);
  k_norm_partial<<<(unsigned)nb, NT, 0, (cudaStream_t)stream>>>(A, E, np, w4[0], w4[1], w4[2], w4[3], partial);
  if (launch_check("norm launch")) return -1;
  return nzb_norm_finalize(partial, nb, 4.0 * (double)E * np, out, stream);
}

int nzb_norm_noalloc(const double* A, int64_t E, int np, const double* w4, double* out, void* stream) {
  if (!A || !w4 || !out || E <= 0 || np <= 0) return fail("norm_noalloc: bad arguments");
  if (E > NOALLOC_MAX_ELEMENTS)
    return fail("norm_noalloc: n_elem = " + std::to_string(E) + " exceeds its fixed scratch, which holds " +
                std::to_string(NOALLOC_MAX_ELEMENTS) + " elements; use nzb_norm with a caller-provided buffer");
  double* scratch = nullptr;
  if (scratch_address(&scratch)) return -1;
  const int64_t nb = blocks_for(E);
  // every slot the finalize reads is written first, so nothing is cleared
  k_norm_partial<<<(unsigned)nb, NT, 0, (cudaStream_t)stream>>>(A, E, np, w4[0], w4[1], w4[2], w4[3], scratch);
  if (launch_check("norm_noalloc launch")) return -1;
  return nzb_norm_finalize(scratch, nb, 4.0 * (double)E * np, out, stream);
}

int nzb_solver_create(const nzb_mesh* mesh, const nzb_physics* phys, const nzb_buffers* buf, int scheme_ssprk3,
                      double dt_factor, nzb_solver** out) {
  if (!out) return fail("solver_create: out is null");
  *out = nullptr;
  if (check_mesh(mesh)) return -1;
  if (!phys || !buf || !buf->S0 || !buf->S1 || !buf->dt || !buf->norm_partial || !buf->res || !buf->counters)
    return fail("solver_create: missing buffer");
  if (scheme_ssprk3 && !buf->S2) return fail("solver_create: ssprk3 needs S2");
  Solver* s = new Solver();
  s->mesh = *mesh;
  s->phys = *phys;
  s->buf = *buf;
  s->ssprk3 = scheme_ssprk3 ? 1 : 0;
  s->dt_factor = dt_factor;
  cudaGetDevice(&s->device);
  if (cuda_check(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "solver stream") ||
      cuda_check(cudaEventCreateWithFlags(&s->ev_in, cudaEventDisableTiming), "solver event") ||
      cuda_check(cudaEventCreateWithFlags(&s->ev_out, cudaEventDisableTiming), "solver event")) {
    nzb_solver_destroy(reinterpret_cast<nzb_solver*>(s));
    return -1;
  }
  *out = reinterpret_cast<nzb_solver*>(s);
  return 0;
}

int nzb_solver_run(nzb_solver* solver, int n_steps, void* stream) {
  Solver* s = reinterpret_cast<Solver*>(solver);
  if (!s) return fail("solver is null");
  if (n_steps < 1) return fail("n_steps must be at least 1");
  cudaStream_t caller = (cudaStream_t)stream;
  if (cuda_check(cudaEventRecord(s->ev_in, caller), "event record") ||
      cuda_check(cudaStreamWaitEvent(s->stream, s->ev_in, 0), "stream wait"))
    return -1;
  // chunks of up to 64 steps share one captured graph per size
  int left = n_steps;
  while (left > 0) {
    const int n = left > 64 ? 64 : left;
    cudaGraphExec_t ex = nullptr;
    if (graph_for(*s, n, &ex)) return -1;
    if (cuda_check(cudaGraphLaunch(ex, s->stream), "graph launch")) return -1;
    left -= n;
  }
  const int np = n_basis(s->mesh.kind, s->mesh.order);
  if (nzb_norm_finalize(s->buf.norm_partial, element_blocks(s->mesh), 4.0 * (double)s->mesh.n_elem * np,
                        s->buf.res, s->stream))
    return -1;
  if (cuda_check(cudaEventRecord(s->ev_out, s->stream), "event record") ||
      cuda_check(cudaStreamWaitEvent(caller, s->ev_out, 0), "stream wait"))
    return -1;
  return 0;
}

int nzb_batch_create(int n_buckets, const nzb_mesh* meshes, const nzb_physics* phys, const nzb_buffers* buffers,
                     const int64_t* elem_offset, const double* dt_factor, const nzb_batch_march* march,
                     nzb_batch** out) {
  if (!out) return fail("batch_create: out is null");
  *out = nullptr;
  if (n_buckets < 1 || !meshes || !phys || !buffers || !elem_offset || !dt_factor || !march)
    return fail("batch_create: null argument");
  const nzb_batch_march& bm = *march;
  if (bm.n_inst < 1 || !bm.inst_begin || !bm.inst_end || !bm.inst_count || !bm.inst_tol || !bm.elem_norm ||
      !bm.status || !bm.iterations || !bm.res0 || !bm.res || !bm.window || !bm.window_count || !bm.n_running)
    return fail("batch_create: missing march array");
  if (bm.stall_window < 2 || bm.max_iterations < 1) return fail("batch_create: bad march parameters");
  if (bm.n_inst > 0x7fffffff) return fail("batch_create: too many instances");
  Batch* B = new Batch();
  for (int b = 0; b < n_buckets; ++b) {
    if (check_mesh(&meshes[b])) {
      delete B;
      return -1;
    }
    if (!meshes[b].elem_inst || !meshes[b].inst_status) {
      delete B;
      return fail("batch_create: bucket meshes need elem_inst and inst_status");
    }
    const nzb_buffers& bf = buffers[b];
    if (!bf.S0 || !bf.S1 || !bf.dt || (meshes[b].order > 0 && !bf.S2)) {
      delete B;
      return fail("batch_create: missing bucket buffer");
    }
    B->mesh.push_back(meshes[b]);
    B->phys.push_back(phys[b]);
    B->buf.push_back(bf);
    B->offset.push_back(elem_offset[b]);
    B->factor.push_back(dt_factor[b]);
  }
  B->bm = bm;
  if (cuda_check(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking), "batch stream") ||
      cuda_check(cudaEventCreateWithFlags(&B->ev_in, cudaEventDisableTiming), "batch event") ||
      cuda_check(cudaEventCreateWithFlags(&B->ev_out, cudaEventDisableTiming), "batch event") ||
      cuda_check(cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming), "batch event")) {
    nzb_batch_destroy(reinterpret_cast<nzb_batch*>(B));
    return -1;
  }
  for (int b = 0; b < n_buckets; ++b) {
    cudaStream_t s = nullptr;
    cudaEvent_t ev = nullptr;
    const int rc = cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "bucket stream") ||
                   cuda_check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "bucket event");
    if (s) B->bstream.push_back(s);
    if (ev) B->bdone.push_back(ev);
    if (rc) {
      nzb_batch_destroy(reinterpret_cast<nzb_batch*>(B));
      return -1;
    }
  }
  *out = reinterpret_cast<nzb_batch*>(B);
  return 0;
}

int nzb_batch_run(nzb_batch* batch, int n_steps, int first, void* stream) {
  Batch* B = reinterpret_cast<Batch*>(batch);
  if (!B) return fail("batch is null");
  if (n_steps < 1 || (first && n_steps != 1)) return fail("batch_run: n_steps >= 1, and 1 for the first chunk");
  cudaStream_t caller = (cudaStream_t)stream;
  if (cuda_check(cudaEventRecord(B->ev_in, caller), "event record") ||
      cuda_check(cudaStreamWaitEvent(B->stream, B->ev_in, 0), "stream wait"))
    return -1;
  cudaGraphExec_t ex = nullptr;
  if (batch_graph(*B, n_steps, first, &ex)) return -1;
  if (cuda_check(cudaGraphLaunch(ex, B->stream), "graph launch")) return -1;
  if (cuda_check(cudaEventRecord(B->ev_out, B->stream), "event record") ||
      cuda_check(cudaStreamWaitEvent(caller, B->ev_out, 0), "stream wait"))
    return -1;
  return 0;
}

int nzb_batch_destroy(nzb_batch* batch) {
  Batch* B = reinterpret_cast<Batch*>(batch);
  if (!B) return 0;
  for (auto& kv : B->graphs) cudaGraphExecDestroy(kv.second);
  if (B->ev_in) cudaEventDestroy(B->ev_in);
  if (B->ev_out) cudaEventDestroy(B->ev_out);
  if (B->fork) cudaEventDestroy(B->fork);
  for (auto ev : B->bdone) cudaEventDestroy(ev);
  for (auto s : B->bstream) cudaStreamDestroy(s);
  if (B->stream) cudaStreamDestroy(B->stream);
  delete B;
  return 0;
}

int nzb_vjp(const nzb_mesh* mesh, const nzb_physics* phys, const nzb_adjoint_args* a, void* stream) {
  if (check_mesh(mesh)) return -1;
  if (!phys || !a || !a->U || !a->lam) return fail("vjp: null argument");
  switch (a->mode) {
    case NZB_ADJ_VJP:
    case NZB_ADJ_RATE:
      if (!a->out) return fail("vjp: out is null");
      if (a->mode == NZB_ADJ_RATE && !a->seed) return fail("vjp: rate needs seed");
      if (a->out == a->lam || a->out == a->U) return fail("vjp: out must not alias lam or U");
      break;
    case NZB_ADJ_DEFECT:
      if (!a->seed) return fail("vjp: defect needs seed");
      if (a->out && (a->out == a->lam || a->out == a->U)) return fail("vjp: out must not alias lam or U");
      break;
    case NZB_ADJ_RK4:
      if (!a->seed || !a->lam0 || !a->dt || !a->f0 || !a->f1 || !a->f2)
        return fail("vjp: rk4 needs seed, lam0, dt, f0..f2");
      if (a->stage < 0 || a->stage > 3) return fail("vjp: rk4 stage must be 0..3");
      if (a->stage < 3 && (!a->out || a->out == a->lam || a->out == a->lam0))
        return fail("vjp: rk4 out missing or aliased");
      if (a->stage == 3 && a->lam == a->lam0) return fail("vjp: rk4 stage 3 input must not alias lam0");
      break;
    default:
      return fail("vjp: unknown mode");
  }
  return dispatch_vjp(*mesh, *phys, adj_work(*a), (cudaStream_t)stream);
}

int nzb_vjp_coords(const nzb_mesh* mesh, const nzb_physics* phys, const double* U, const double* lam,
                   const double* verts, const double* dgs, double* gvert, double* gpb, void* stream) {
  if (check_mesh(mesh)) return -1;
  if (!phys || !U || !lam || !verts || !dgs || !gvert) return fail("vjp_coords: null argument");
  CoordWork w{};
  w.U = U;
  w.lam = lam;
  w.verts = verts;
  w.gvert = gvert;
  w.gpb = gpb;
  for (int f = 0; f < 4; ++f)
    for (int v = 0; v < 4; ++v) w.dgs[f][v] = dgs[4 * f + v];
  return dispatch_vjp_coords(*mesh, *phys, w, (cudaStream_t)stream);
}

int nzb_local_dt(const nzb_mesh* mesh, const double* wave, double coefficient, double* dt, void* stream) {
  if (check_mesh(mesh)) return -1;
  if (!wave || !dt) return fail("local_dt: null argument");
  const int64_t E = mesh->n_elem;
  k_local_dt<<<(unsigned)((E + 127) / 128), 128, 0, (cudaStream_t)stream>>>(mesh->area, wave, E, coefficient, dt);
  return launch_check("local dt launch");
}

int nzb_adjoint_create(int n_buckets, const nzb_mesh* meshes, const nzb_physics* phys,
                       const nzb_adjoint_buffers* buffers, const int64_t* elem_offset,
                       const nzb_adjoint_march* march, nzb_adjoint** out) {
  if (!out) return fail("adjoint_create: out is null");
  *out = nullptr;
  if (n_buckets < 1 || !meshes || !phys || !buffers || !elem_offset || !march)
    return fail("adjoint_create: null argument");
  const nzb_adjoint_march& am = *march;
  if (am.n_inst < 1 || !am.inst_begin || !am.inst_end || !am.inst_count || !am.elem_norm || !am.status ||
      !am.iterations || !am.res0 || !am.res || !am.n_running)
    return fail("adjoint_create: missing march array");
  if (am.max_iterations < 1 || !(am.tolerance >= 0.0)) return fail("adjoint_create: bad march parameters");
  if (am.n_inst > 0x7fffffff) return fail("adjoint_create: too many instances");
  AdjBatch* A = new AdjBatch();
  for (int b = 0; b < n_buckets; ++b) {
    if (check_mesh(&meshes[b])) {
      delete A;
      return -1;
    }
    if (am.n_inst > 1 && (!meshes[b].elem_inst || !meshes[b].inst_status)) {
      delete A;
      return fail("adjoint_create: several instances need elem_inst and inst_status");
    }
    const nzb_adjoint_buffers& bf = buffers[b];
    if (!bf.U || !bf.seed || !bf.lam || !bf.Y1 || !bf.Y2 || !bf.f0 || !bf.f1 || !bf.f2 || !bf.dt) {
      delete A;
      return fail("adjoint_create: missing bucket buffer");
    }
    A->mesh.push_back(meshes[b]);
    A->phys.push_back(phys[b]);
    A->buf.push_back(bf);
    A->offset.push_back(elem_offset[b]);
  }
  A->am = am;
  if (cuda_check(cudaStreamCreateWithFlags(&A->stream, cudaStreamNonBlocking), "adjoint stream") ||
      cuda_check(cudaEventCreateWithFlags(&A->ev_in, cudaEventDisableTiming), "adjoint event") ||
      cuda_check(cudaEventCreateWithFlags(&A->ev_out, cudaEventDisableTiming), "adjoint event") ||
      cuda_check(cudaEventCreateWithFlags(&A->fork, cudaEventDisableTiming), "adjoint event")) {
    nzb_adjoint_destroy(reinterpret_cast<nzb_adjoint*>(A));
    return -1;
  }
  for (int b = 0; b < n_buckets; ++b) {
    cudaStream_t s = nullptr;
    cudaEvent_t ev = nullptr;
    const int rc = cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "bucket stream") ||
                   cuda_check(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "bucket event");
    if (s) A->bstream.push_back(s);
    if (ev) A->bdone.push_back(ev);
    if (rc) {
      nzb_adjoint_destroy(reinterpret_cast<nzb_adjoint*>(A));
      return -1;
    }
  }
  *out = reinterpret_cast<nzb_adjoint*>(A);
  return 0;
}

int nzb_adjoint_run(nzb_adjoint* adjoint, int n_steps, void* stream) {
  AdjBatch* A = reinterpret_cast<AdjBatch*>(adjoint);
  if (!A) return fail("adjoint is null");
  if (n_steps < 0) return fail("adjoint_run: n_steps must be >= 0");
  cudaStream_t caller = (cudaStream_t)stream;
  if (cuda_check(cudaEventRecord(A->ev_in, caller), "event record") ||
      cuda_check(cudaStreamWaitEvent(A->stream, A->ev_in, 0), "stream wait"))
    return -1;
  cudaGraphExec_t ex = nullptr;
  if (adjoint_graph(*A, n_steps, &ex)) return -1;
  if (cuda_check(cudaGraphLaunch(ex, A->stream), "graph launch")) return -1;
  if (cuda_check(cudaEventRecord(A->ev_out, A->stream), "event record") ||
      cuda_check(cudaStreamWaitEvent(caller, A->ev_out, 0), "stream wait"))
    return -1;
  return 0;
}

int nzb_adjoint_destroy(nzb_adjoint* adjoint) {
  AdjBatch* A = reinterpret_cast<AdjBatch*>(adjoint);
  if (!A) return 0;
  for (auto& kv : A->graphs) cudaGraphExecDestroy(kv.second);
  if (A->ev_in) cudaEventDestroy(A->ev_in);
  if (A->ev_out) cudaEventDestroy(A->ev_out);
  if (A->fork) cudaEventDestroy(A->fork);
  for (auto ev : A->bdone) cudaEventDestroy(ev);
  for (auto s : A->bstream) cudaStreamDestroy(s);
  if (A->stream) cudaStreamDestroy(A->stream);
  delete A;
  return 0;
}

int nzb_solver_destroy(nzb_solver* solver) {
  Solver* s = reinterpret_cast<Solver*>(solver);
  if (!s) return 0;
  for (auto& kv : s->graphs) cudaGraphExecDestroy(kv.second);
  if (s->ev_in) cudaEventDestroy(s->ev_in);
  if (s->ev_out) cudaEventDestroy(s->ev_out);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return 0;
}

}  // extern "C"
