// C ABI (include/bem_b200.h): solver context, device upload, mat-vec orchestration
// (CUDA-graph captured) and the device-resident GMRES driver.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <map>
#include <mutex>
#include <tuple>
#include <string>
#include <vector>

#include "../../include/bem_b200.h"
#include "fmm_math.cuh"
#include "kernels.cuh"
#include "tree_dev.hpp"
#include "plan.hpp"

using namespace bemb200;

namespace {

// Device buffer that keeps its allocation across set-ups: alloc() only reallocates when the
// new size exceeds the capacity (a repeated set-up of the same or a smaller problem, e.g. the
// time steps of one simulation, allocates nothing).
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0, cap = 0;
  int64_t* acct = nullptr;  // the owner's running total of allocated device bytes
  DBuf() = default;
  explicit DBuf(int64_t* a) : acct(a) {}
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    if (acct) *acct -= (int64_t)(sizeof(T) * cap);
    p = nullptr;
    n = cap = 0;
  }
  cudaError_t alloc(size_t count) {
    n = count;
    if (count <= cap) return cudaSuccess;
    release();
    n = count;
    const cudaError_t e = cudaMalloc((void**)&p, sizeof(T) * count);
    if (e == cudaSuccess) {
      cap = count;
      if (acct) *acct += (int64_t)(sizeof(T) * cap);
    }
    return e;
  }
};

// Pinned host staging area for the set-up uploads: host arrays are copied into it and sent
// with asynchronous copies, so the upload runs at pinned-memory bandwidth instead of through
// the driver's pageable bounce buffer.  Grown on demand (after draining the stream).
struct PinnedStage {
  unsigned char* p = nullptr;
  size_t cap = 0, off = 0, used = 0;  // used: bytes staged since begin()
  ~PinnedStage() {
    if (p) cudaFreeHost(p);
  }
  // start of a set-up's uploads: the area from its beginning, grown to `bytes` (the previous
  // set-up's total) so that the uploads of one set-up do not wait for each other
  cudaError_t begin(size_t bytes, cudaStream_t s) {
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    off = used = 0;
    if (bytes <= cap) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    const size_t want = bytes + bytes / 4;  // headroom: pinning is slow, the next mesh may be a little larger
    e = cudaHostAlloc((void**)&p, want, cudaHostAllocDefault);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  // space for `bytes`, synchronising `s` when the area must be reused or grown
  cudaError_t reserve(size_t bytes, cudaStream_t s, unsigned char** out) {
    if (off + bytes > cap) {
      cudaError_t e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) return e;
      off = 0;
      if (bytes > cap) {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        const size_t want = std::max<size_t>(bytes, size_t(64) << 20);
        e = cudaHostAlloc((void**)&p, want, cudaHostAllocDefault);
        if (e != cudaSuccess) return e;
        cap = want;
      }
    }
    *out = p + off;
    off += (bytes + 255) & ~size_t(255);
    used += (bytes + 255) & ~size_t(255);
    return cudaSuccess;
  }
};

double now_s() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }

}  // namespace

constexpr int kErrRing = 8;  // residual estimates in flight (>= the read-back lag + 1)
constexpr int kMaxPolyDegree = 24;
// pairs per tensor-core work item tried by the autotuner: orders <= 10 have a kernel variant for
// items of up to 128 pairs (one table slot in shared memory), higher orders up to 80
constexpr int kTuneCandWide[4] = {64, 80, 112, 128};
constexpr int kTuneCandNarrow[4] = {32, 48, 64, 80};
inline const int* tune_cand(int p) { return p <= 10 ? kTuneCandWide : kTuneCandNarrow; }
inline int poly_degree(const bem_gpu_opts& o) { return o.poly_degree > 0 ? o.poly_degree : 8; }

// M2L pair slots of bem_gpu_matvec_device_noalloc: a fixed area in this file's device image,
// reserved on every device that loads the module and held until the process exits.
constexpr size_t kNoAllocSlotBytes = size_t(32) << 20;  // 32 MiB: m2l_pairs * 2 * ncoef(p) * 16 B must fit
static __device__ __align__(256) unsigned char g_m2l_slot_scratch[kNoAllocSlotBytes];

struct bem_gpu_ctx {
  bem_gpu_opts opts{};
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;                         // near field of the low-precision A.x
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;    // fork / join of the side stream
  std::string err;
  Plan plan, plan_spare;
  bool ready = false;
  double time_setup = 0.0;
  // device address of g_m2l_slot_scratch on this context's device, looked up at the first
  // set-up with the device current (nullptr: not looked up yet, or the lookup failed)
  void* noalloc_slots = nullptr;
  cudaError_t noalloc_lookup = cudaSuccess;
  uint32_t tc_wait_tries = tc_default_wait_tries();  // bem_gpu_set_wait_limit

  // geometry / tree
  int64_t dev_bytes = 0;  // device bytes held by the DBuf members below (declared first: destroyed last)
  DBuf<double> Xs{&dev_bytes}, e_q{&dev_bytes}, e_W{&dev_bytes}, e_n{&dev_bytes}, e_near{&dev_bytes}, node_X{&dev_bytes}, WG{&dev_bytes}, WGn{&dev_bytes}, Wc{&dev_bytes}, diag{&dev_bytes};
  DBuf<float> Wc32{&dev_bytes};  // combined near weights of A.x in FP32 (mixed precision, polynomial preconditioner)
  DBuf<int> leaf_dof_off{&dev_bytes}, leaf_dof{&dev_bytes}, e_slot{&dev_bytes};  // P2M operator of A.x: DOFs per leaf
  DBuf<int> near_counter{&dev_bytes};  // next near block of the near-field quadrature
  // near-block preconditioner (preconditioner = 3): core DOFs per near block and the inverses
  DBuf<int> bj_doff{&dev_bytes}, bj_dofs{&dev_bytes};
  DBuf<int64_t> bj_ioff{&dev_bytes};
  DBuf<double> bj_inv{&dev_bytes}, bj_tmp{&dev_bytes};
  DBuf<double2> p2m_C{&dev_bytes};                       // [(leaf, DOF)][NC]
  DBuf<float2> p2m_C32{&dev_bytes};                      // its FP32 copy (mixed precision)
  DBuf<double2> near_scratch{&dev_bytes};                // element values of the near-weight kernel
  DBuf<int> e_dof{&dev_bytes}, e_vtx{&dev_bytes}, node_fb{&dev_bytes}, node_fe{&dev_bytes}, leaves{&dev_bytes}, child_begin{&dev_bytes}, child_end{&dev_bytes}, node_children{&dev_bytes};
  // tree passes, one launch per level: upward-pass nodes and the parent each hands its multipole
  // to, the multipoles shifted to the parent, downward-pass (parent, child) pairs
  DBuf<int> m2m_nodes{&dev_bytes}, node_up{&dev_bytes}, m2m_nodes_nl{&dev_bytes}, leaf_level{&dev_bytes};
  DBuf<double2> Yup{&dev_bytes};
  DBuf<int2> l2l_pairs{&dev_bytes};
  DBuf<int> blk_path_off{&dev_bytes}, blk_path{&dev_bytes};  // near block -> its bucket's M2L-target path
  int max_path = 0;
  std::vector<int> h_tc_src, h_tc_pos, h_tc_tgt;  // host staging of the tensor-core work-item arrays
  std::vector<int> m2m_level_off, m2m_level_off_nl, l2l_level_off;
  int n_tree_levels = 0;
  DBuf<int> m2l_targets{&dev_bytes}, m2l_off{&dev_bytes}, m2l_src{&dev_bytes}, nb_dofs{&dev_bytes}, nb_targets{&dev_bytes}, nb_ranges{&dev_bytes}, dof_inc_off{&dev_bytes}, dof_inc{&dev_bytes};
  DBuf<int> block_of_point{&dev_bytes}, row_of_point{&dev_bytes}, self_col{&dev_bytes};  // right-Jacobi inputs
  DBuf<int> point_dof_off{&dev_bytes}, point_dof{&dev_bytes}, dof_kind{&dev_bytes}, dof_point{&dev_bytes};
  DBuf<NearBlockDev> blocks{&dev_bytes};
  DBuf<int> chunk_grp{&dev_bytes}, chunk_begin{&dev_bytes}, chunk_cnt{&dev_bytes}, grp_pair{&dev_bytes};
  DBuf<double> grp_vec{&dev_bytes};
  DBuf<double2> Sg{&dev_bytes}, Y{&dev_bytes}, Ftab{&dev_bytes};
  DBuf<double> ftab_vec{&dev_bytes};
  DBuf<double2> M{&dev_bytes}, L{&dev_bytes};
  int n_m2l_targets = 0, max_ntgt = 0, chunk = 0;
  int64_t w4_total = 0;  // size of the row-padded FP32 near weights
  int n_tc_items = 0;    // tensor-core work items (every table-row-tile image's pair chunks)
  // state
  DBuf<double> phi{&dev_bytes}, phin{&dev_bytes}, known_s{&dev_bytes}, rows{&dev_bytes}, GPhin{&dev_bytes}, GnPhi{&dev_bytes};
  // graph-captured A.x : mv_in -> mv_out
  DBuf<double> mv_in{&dev_bytes}, mv_out{&dev_bytes};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  // Krylov
  DBuf<double> V{&dev_bytes}, w{&dev_bytes}, hdev{&dev_bytes}, partial{&dev_bytes}, xdev{&dev_bytes}, bdev{&dev_bytes}, rdev{&dev_bytes}, ydev{&dev_bytes}, tmp{&dev_bytes}, dinv{&dev_bytes};
  int V_cols = 0;
  int graph_kernels = 0;
  // mixed precision: tensor-core M2L tables and buffers; graph of the low-precision A.x
  bool mixed = false;
  DBuf<int> tc_item_tab{&dev_bytes}, tc_item_begin{&dev_bytes}, tc_item_cnt{&dev_bytes}, tc_pos{&dev_bytes}, tc_src{&dev_bytes}, tc_err{&dev_bytes};
  DBuf<double> near_sum{&dev_bytes};  // near sums of A.x by target slot
  DBuf<double> tc_tabvec{&dev_bytes}, tc_alpha{&dev_bytes}, node_dL{&dev_bytes};
  DBuf<uint16_t> tc_T{&dev_bytes}, tc_Mt{&dev_bytes};
  DBuf<float> tc_escale{&dev_bytes};
  DBuf<int> tc_tgt{&dev_bytes};    // [pairs] compact target index of each work-item-ordered pair
  DBuf<float> tc_acc{&dev_bytes};  // [n_m2l_targets][KPO] FP32 accumulators of the fused reduction (zero between launches)
  DBuf<unsigned int> tc_max{&dev_bytes};
  int tc_grid = 148;
  int tc_tune = 0;                 // pairs per tensor-core work item in use
  bool tc_tuned_here = false;      // this set-up ran the tuning
  float tc_tune_ms[4] = {0, 0, 0, 0};
  std::vector<unsigned char> tc_map;  // TMA tensor map over tc_Mt (host copy, passed by value)
  cudaGraph_t graph_lo = nullptr;
  cudaGraphExec_t graph_exec_lo = nullptr;
  int graph_kernels_lo = 0;
  // device-resident Arnoldi: state, rotations, g, R; one graph per step; pinned ring of
  // residual estimates with an event per slot
  DBuf<ArnoldiState> arn_state{&dev_bytes};
  DBuf<double> arn_g{&dev_bytes}, arn_cs{&dev_bytes}, arn_sn{&dev_bytes}, arn_R{&dev_bytes}, xbase{&dev_bytes};
  cudaGraph_t arn_graph = nullptr;
  cudaGraphExec_t arn_exec = nullptr;
  int arn_kernels = 0;
  const void* arn_key_V = nullptr;
  int arn_key_cols = 0, arn_key_prec = -1, arn_key_mixed = -1;
  // polynomial preconditioner: roots (from the set-up), Arnoldi basis of the root run,
  // apply scratch, and Z = M V (the iterate is updated from Z)
  PolyRoots poly;
  DBuf<double> poly_V{&dev_bytes}, poly_h{&dev_bytes}, poly_part{&dev_bytes}, poly_prod{&dev_bytes}, poly_y{&dev_bytes}, Z{&dev_bytes};
  double* arn_err_host = nullptr;
  cudaEvent_t arn_ev[kErrRing] = {};
  // accounting of the current setup + solve
  int64_t h2d = 0, d2h = 0, launches = 0;
  int64_t setup_h2d = 0, setup_launches = 0;
  // set-up device window start/end, solve start/end, near-field quadrature start/end
  cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  float setup_dev_ms = 0.f;
  float near_weights_ms = 0.f;  // the near-field quadrature's part of setup_dev_ms
  double time_plan = 0.0, time_upload = 0.0;
  // the upload part of the set-up by step (host time; the copies are asynchronous): [0] node and
  // level arrays, [1] near blocks and element/tree arrays, [2] tensor-core items, [3] P2M operator
  // lists, [4] remaining arrays, [5] unused (0)
  double upload_part_s[6] = {0, 0, 0, 0, 0, 0};

  DeviceTree* dtree = nullptr;  // octree growth on the device (set-up)
  PinnedStage stage;  // set-up uploads
  size_t stage_bytes = 0;  // staged bytes of the last set-up (with alignment padding)
  ~bem_gpu_ctx() {
    if (stream) cudaStreamSynchronize(stream);
    for (auto& e : ev)
      if (e) cudaEventDestroy(e);
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    if (graph_exec_lo) cudaGraphExecDestroy(graph_exec_lo);
    if (graph_lo) cudaGraphDestroy(graph_lo);
    if (arn_exec) cudaGraphExecDestroy(arn_exec);
    if (arn_graph) cudaGraphDestroy(arn_graph);
    for (auto& e : arn_ev)
      if (e) cudaEventDestroy(e);
    if (arn_err_host) cudaFreeHost(arn_err_host);
    if (dtree) dtree_destroy(dtree);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (side) cudaStreamDestroy(side);
    if (stream) cudaStreamDestroy(stream);
  }
  MatvecArgs args(const double* d_phi, const double* d_phin, double* d_rows, double* d_gphin, double* d_gnphi) const {
    MatvecArgs a;
    a.n_nodes = (int)plan.nodes.size();
    a.n_levels = n_tree_levels;
    a.n_leaves = (int)plan.leaves.size();
    a.leaves = leaves.p;
    a.node_fb = node_fb.p;
    a.node_fe = node_fe.p;
    a.node_X = node_X.p;
    a.e_q = e_q.p;
    a.e_W = e_W.p;
    a.e_n = e_n.p;
    a.e_dof = e_dof.p;
    a.child_begin = child_begin.p;
    a.child_end = child_end.p;
    a.node_children = node_children.p;
    a.Ftab = Ftab.p;
    a.m2m_level_off = m2m_level_off.empty() ? nullptr : m2m_level_off.data();
    a.m2m_nodes = m2m_nodes.p;
    a.node_up = node_up.p;
    a.Yup = Yup.p;
    a.m2m_level_off_nl = m2m_level_off_nl.empty() ? nullptr : m2m_level_off_nl.data();
    a.m2m_nodes_nl = m2m_nodes_nl.p;
    a.leaf_level = leaf_level.p;
    a.l2l_level_off = l2l_level_off.empty() ? nullptr : l2l_level_off.data();
    a.l2l_pairs = l2l_pairs.p;
    a.blk_path_off = blk_path_off.p;
    a.max_path = max_path;
    a.blk_path = blk_path.p;

    a.n_m2l_targets = n_m2l_targets;
    a.m2l_targets = m2l_targets.p;
    a.m2l_off = m2l_off.p;
    a.m2l_src = m2l_src.p;
    a.n_chunks = (int)plan.chunk_grp.size();
    a.chunk_grp = chunk_grp.p;
    a.chunk_begin = chunk_begin.p;
    a.chunk_cnt = chunk_cnt.p;
    a.grp_pair = grp_pair.p;
    a.Sg = Sg.p;
    a.Y = Y.p;
    a.M = M.p;
    a.L = L.p;
    a.n_blocks = (int)plan.blocks.size();
    a.chunk = chunk;
    a.near_sum = near_sum.p;
    a.max_ntgt = max_ntgt;
    a.blocks = blocks.p;
    a.nb_dofs = nb_dofs.p;
    a.nb_targets = nb_targets.p;
    a.WG = WG.p;
    a.WGn = WGn.p;
    a.Xs = Xs.p;
    a.point_dof_off = point_dof_off.p;
    a.point_dof = point_dof.p;
    a.dof_kind = dof_kind.p;
    a.diag = diag.p;
    a.phi = d_phi;
    a.phin = d_phin;
    a.rows = d_rows;
    a.GPhin = d_gphin;
    a.GnPhi = d_gnphi;
    return a;
  }
  NearBjArgs bj_args() const {
    NearBjArgs a;
    if (opts.preconditioner != 3) return a;
    a.nblocks = (int)plan.blocks.size();
    a.blocks = blocks.p;
    a.doff = bj_doff.p;
    a.dofs = bj_dofs.p;
    a.ioff = bj_ioff.p;
    a.inv = bj_inv.p;
    return a;
  }
  // marks an argument set as A.x of mv_in (combined near weights, FP32 ones when lowp)
  void set_ax(MatvecArgs& a, bool lowp) const {
    a.ax = mv_in.p;
    a.leaf_dof_off = leaf_dof_off.p;
    a.leaf_dof = leaf_dof.p;
    a.p2m_C = p2m_C.p;
    a.p2m_C32 = lowp ? p2m_C32.p : nullptr;
    a.Wc = lowp ? nullptr : Wc.p;
    a.Wc32 = lowp ? Wc32.p : nullptr;
    if (opts.overlap_near == 1) {  // near-field sums on the side stream, concurrent with the FMM passes
      a.side = side;
      a.ev_fork = ev_fork;
      a.ev_join = ev_join;
    }
  }
  // the near-field part of A.x (FP32 weights where built): mv_in -> mv_out
  MatvecArgs near_args() const {
    MatvecArgs a = args(nullptr, nullptr, mv_out.p, nullptr, nullptr);
    set_ax(a, Wc32.p != nullptr);
    return a;
  }
  // switches an argument set to the tensor-core M2L
  void set_tc(MatvecArgs& a) const {
    a.use_tc = 1;
    a.n_tc_items = n_tc_items;
    a.tc_grid = tc_grid;
    a.tc_item_tab = tc_item_tab.p;
    a.tc_item_begin = tc_item_begin.p;
    a.tc_item_cnt = tc_item_cnt.p;
    a.tc_pos = tc_pos.p;
    a.n_tc_pairs = (int)plan.tc_pair.size();
    a.tc_item_pairs = tc_tune > 0 ? tc_tune : 80;
    a.tc_src = tc_src.p;
    a.tc_tab = tc_T.p;
    a.tc_Mt = tc_Mt.p;
    a.tc_escale = tc_escale.p;
    a.tc_Y = reinterpret_cast<float*>(Y.p);
    a.tc_tgt = tc_tgt.p;
    a.tc_acc = opts.tc_deterministic ? nullptr : tc_acc.p;
    a.tc_err = tc_err.p;
    a.tc_wait_tries = tc_wait_tries;
    a.node_dL = node_dL.p;
    a.tc_alpha = tc_alpha.p;
    a.tc_rows_map = tc_map.data();
  }
};

#define CK(call)                                                               \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      ctx->err = std::string(#call) + ": " + cudaGetErrorString(e_);            \
      return e_ == cudaErrorMemoryAllocation ? BEM_ERR_OUT_OF_MEMORY : BEM_ERR_DEVICE; \
    }                                                                          \
  } while (0)

namespace {

int fill_quadrature(bem_gpu_ctx* ctx) {
  const double dv[6][4] = {{0.816847572980459, 0.091576213509771, 0.091576213509771, 0.054975871827661},
                           {0.091576213509771, 0.816847572980459, 0.091576213509771, 0.054975871827661},
                           {0.091576213509771, 0.091576213509771, 0.816847572980459, 0.054975871827661},
                           {0.108103018168070, 0.445948490915965, 0.445948490915965, 0.111690794839006},
                           {0.445948490915965, 0.108103018168070, 0.445948490915965, 0.111690794839006},
                           {0.445948490915965, 0.445948490915965, 0.108103018168070, 0.111690794839006}};
  // 5x5 Gauss-Legendre product rule on [0,1]^2 with the reference's own 15-digit constants
  // (__array_GW5xGW5__, lib/include/basic_constants.hpp:1326-1350), which the near-field
  // weights must share to agree with the reference beyond ~1e-12.  Symmetric table: node a,
  // weight class c(a) = {0, 1, 2, 1, 0}, w(a, b) = wc[c(a)][c(b)].
  const double xs[5] = {0.046910077030668, 0.230765344947158, 0.5, 0.769234655052841, 0.953089922969332};
  const int cls[5] = {0, 1, 2, 1, 0};
  const double wc[3][3] = {{0.0140335872156063, 0.0283499999999991, 0.0336962680968792},
                           {0.0283499999999991, 0.0572713510559978, 0.0680716331376877},
                           {0.0336962680968792, 0.0680716331376877, 0.0809086419753086}};
  double gw[25][3];
  for (int a = 0; a < 5; ++a)
    for (int b = 0; b < 5; ++b) {
      gw[5 * a + b][0] = xs[a];
      gw[5 * a + b][1] = xs[b];
      gw[5 * a + b][2] = wc[cls[a]][cls[b]];
    }
  upload_quadrature(dv, gw, ctx->stream);
  CK(cudaGetLastError());
  return BEM_OK;
}

// one operator application on device state: densities already in ctx->phi/phin
void run_fmm(bem_gpu_ctx* ctx, double* rows, double* gphin, double* gnphi) {
  ctx->launches += launch_matvec(ctx->plan.opt.p, ctx->args(ctx->phi.p, ctx->phin.p, rows, gphin, gnphi), ctx->stream);
}

template <typename T>
cudaError_t up(bem_gpu_ctx* ctx, DBuf<T>& b, const std::vector<T>& v) {
  const size_t bytes = sizeof(T) * v.size();
  ctx->h2d += (int64_t)bytes;
  cudaError_t e = b.alloc(v.size());
  if (e != cudaSuccess || v.empty()) return e;
  unsigned char* h = nullptr;
  if ((e = ctx->stage.reserve(bytes, ctx->stream, &h)) != cudaSuccess) return e;
  parallel_copy(h, v.data(), bytes);
  return cudaMemcpyAsync(b.p, h, bytes, cudaMemcpyHostToDevice, ctx->stream);
}

// Captures A.x (mv_in -> mv_out) as a graph; tc selects the tensor-core M2L.
int capture_matvec(bem_gpu_ctx* ctx, bool tc, cudaGraph_t& graph, cudaGraphExec_t& exec, int& kernels) {
  if (exec) {
    cudaGraphExecDestroy(exec);
    exec = nullptr;
  }
  if (graph) {
    cudaGraphDestroy(graph);
    graph = nullptr;
  }
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  launch_densities(ctx->plan.ndof, 0, ctx->mv_in.p, nullptr, ctx->dof_kind.p, ctx->phi.p, ctx->phin.p, ctx->stream);
  MatvecArgs a = ctx->args(ctx->phi.p, ctx->phin.p, ctx->mv_out.p, nullptr, nullptr);
  ctx->set_ax(a, tc);
  if (tc) ctx->set_tc(a);
  launch_matvec(ctx->plan.opt.p, a, ctx->stream);
  CK(cudaStreamEndCapture(ctx->stream, &graph));
  CK(cudaGraphInstantiate(&exec, graph, 0));
  size_t nn = 0;
  CK(cudaGraphGetNodes(graph, nullptr, &nn));
  std::vector<cudaGraphNode_t> nodes(nn);
  if (nn) CK(cudaGraphGetNodes(graph, nodes.data(), &nn));
  kernels = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType ty;
    CK(cudaGraphNodeGetType(nd, &ty));
    if (ty == cudaGraphNodeTypeKernel) ++kernels;
  }
  return BEM_OK;
}

int build_graph(bem_gpu_ctx* ctx) {
  ctx->arn_key_V = nullptr;  // the Arnoldi step graph holds this set-up's buffers: recapture at the next solve
  int rc = capture_matvec(ctx, false, ctx->graph, ctx->graph_exec, ctx->graph_kernels);
  if (rc != BEM_OK || !ctx->mixed) return rc;
  return capture_matvec(ctx, true, ctx->graph_lo, ctx->graph_exec_lo, ctx->graph_kernels_lo);
}

// (Re)captures the Arnoldi step graph when the basis, its capacity, the operator or the
// preconditioner (0 none, 1 Jacobi, 2 polynomial) changed.
int ensure_arnoldi_graph(bem_gpu_ctx* ctx, int prec, bool lowp, int cols) {
  const int N = ctx->plan.ndof;
  if (ctx->arn_cs.n < (size_t)cols) {
    CK(ctx->arn_state.alloc(1));
    CK(ctx->arn_g.alloc((size_t)cols + 1));
    CK(ctx->arn_cs.alloc(cols));
    CK(ctx->arn_sn.alloc(cols));
    CK(ctx->arn_R.alloc((size_t)cols * cols));
  }
  if (ctx->xbase.n < (size_t)N) CK(ctx->xbase.alloc(N));
  if (!ctx->arn_err_host) {
    CK(cudaHostAlloc((void**)&ctx->arn_err_host, sizeof(double) * kErrRing, cudaHostAllocDefault));
    for (auto& e : ctx->arn_ev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  if (prec == 2 && ctx->poly_prod.n < (size_t)N) {
    CK(ctx->poly_prod.alloc(N));
    CK(ctx->poly_y.alloc(N));
  }
  if (ctx->arn_exec && ctx->arn_key_V == ctx->V.p && ctx->arn_key_cols == cols && ctx->arn_key_prec == prec &&
      ctx->arn_key_mixed == (int)lowp)
    return BEM_OK;
  if (ctx->arn_exec) {
    cudaGraphExecDestroy(ctx->arn_exec);
    ctx->arn_exec = nullptr;
  }
  if (ctx->arn_graph) {
    cudaGraphDestroy(ctx->arn_graph);
    ctx->arn_graph = nullptr;
  }
  ArnoldiArgs a;
  a.nrow = N;
  a.cols = cols;
  a.p = ctx->plan.opt.p;
  a.V = ctx->V.p;
  a.dinv = (prec == 1 || prec == 2) ? ctx->dinv.p : nullptr;
  if (prec == 3) a.bj = ctx->bj_args();
  a.state = ctx->arn_state.p;
  a.x = ctx->mv_in.p;
  a.w = ctx->mv_out.p;
  a.mv = ctx->args(ctx->phi.p, ctx->phin.p, ctx->mv_out.p, nullptr, nullptr);
  ctx->set_ax(a.mv, lowp);
  if (lowp) ctx->set_tc(a.mv);
  a.h = ctx->hdev.p;
  a.partial = ctx->partial.p;
  a.cs = ctx->arn_cs.p;
  a.sn = ctx->arn_sn.p;
  a.g = ctx->arn_g.p;
  a.R = ctx->arn_R.p;
  if (prec == 2) {
    a.poly = &ctx->poly;
    a.near = ctx->near_args();
    a.prod = ctx->poly_prod.p;
    a.y = ctx->poly_y.p;
    a.Z = ctx->Z.p;
  }
  if (configure_arnoldi(cols) != 0) {
    ctx->err = "GMRES basis too large for the on-device Givens step (max_iter > 9000)";
    return BEM_ERR_UNSUPPORTED;
  }
  CK(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  launch_arnoldi_step(a, ctx->stream);
  CK(cudaStreamEndCapture(ctx->stream, &ctx->arn_graph));
  CK(cudaGraphInstantiate(&ctx->arn_exec, ctx->arn_graph, 0));
  size_t nn = 0;
  CK(cudaGraphGetNodes(ctx->arn_graph, nullptr, &nn));
  std::vector<cudaGraphNode_t> nodes(nn);
  if (nn) CK(cudaGraphGetNodes(ctx->arn_graph, nodes.data(), &nn));
  ctx->arn_kernels = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType ty;
    CK(cudaGraphNodeGetType(nd, &ty));
    if (ty == cudaGraphNodeTypeKernel) ++ctx->arn_kernels;
  }
  ctx->arn_key_V = ctx->V.p;
  ctx->arn_key_cols = cols;
  ctx->arn_key_prec = prec;
  ctx->arn_key_mixed = (int)lowp;
  return BEM_OK;
}

// y = A_lo x on device buffers (tensor-core M2L), on the context's stream
int matvec_lo(bem_gpu_ctx* ctx, const double* d_x, double* d_y) {
  const int N = ctx->plan.ndof;
  cudaStream_t s = ctx->stream;
  if (d_x != ctx->mv_in.p) CK(cudaMemcpyAsync(ctx->mv_in.p, d_x, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
  CK(cudaGraphLaunch(ctx->graph_exec_lo, s));
  if (d_y != ctx->mv_out.p) CK(cudaMemcpyAsync(d_y, ctx->mv_out.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
  return BEM_OK;
}

}  // namespace

extern "C" {

int bem_gpu_is_available(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return 0;
  for (int d = 0; d < n; ++d) {
    cudaDeviceProp pr{};
    if (cudaGetDeviceProperties(&pr, d) == cudaSuccess && pr.major == 10) return 1;
  }
  return 0;
}

void bem_gpu_default_opts(bem_gpu_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->expansion_order = 10;
  o->mac_theta = 0.25;
  o->leaf_max_elements = 30;
  o->max_level = 7;
  o->tol = 1e-9;
  o->max_iter = 500;
  o->device = 0;
  o->overlap_near = 1;
}

bem_gpu_ctx* bem_gpu_create(const bem_gpu_opts* opts) {
  if (!opts || opts->expansion_order < 1 || opts->expansion_order > 12 || !(opts->mac_theta > 0) || opts->leaf_max_elements < 1 ||
      opts->max_level < 1 || opts->max_level > 20 || opts->max_iter < 1 || !(opts->refine_rtol >= 0.0 && opts->refine_rtol < 1.0))
    return nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || opts->device < 0 || opts->device >= ndev) return nullptr;
  if (cudaSetDevice(opts->device) != cudaSuccess) return nullptr;
  auto* ctx = new (std::nothrow) bem_gpu_ctx();
  if (!ctx) return nullptr;
  ctx->opts = *opts;
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    delete ctx;
    return nullptr;
  }
  if (fill_quadrature(ctx) != BEM_OK) {
    delete ctx;
    return nullptr;
  }
  for (auto& e : ctx->ev)
    if (cudaEventCreate(&e) != cudaSuccess) {
      delete ctx;
      return nullptr;
    }
  return ctx;
}

void bem_gpu_destroy(bem_gpu_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->opts.device);
  delete ctx;
}

const char* bem_gpu_last_error(const bem_gpu_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int bem_gpu_build_dofs(int32_t n_points, const double* X, int32_t n_faces, const int32_t* tri, const uint8_t* face_dirichlet,
                       int32_t* dof_point, int32_t* dof_face, int32_t* dof_kind, int32_t* face_dof, uint8_t* point_flags) {
  if (!dof_point || !dof_face || !dof_kind || !face_dof) return BEM_ERR_INVALID_ARGUMENT;
  const int n = build_dofs(n_points, X, n_faces, tri, face_dirichlet, dof_point, dof_face, dof_kind, face_dof, point_flags);
  return n < 0 ? BEM_ERR_INVALID_ARGUMENT : n;
}

// Roots of the near-field polynomial preconditioner: k Arnoldi steps (classical Gram-Schmidt
// twice) on B = A_near D^{-1} from a fixed pseudo-random start, the Hessenberg matrix read
// back after each step; harmonic Ritz values of the run in Leja order.  A breakdown ends the
// run early (lower degree); roots that cannot be formed leave the polynomial empty and the
// solve falls back to the Jacobi scaling.
static int build_poly(bem_gpu_ctx* ctx) {
  const int N = ctx->plan.ndof, k = poly_degree(ctx->opts), p = ctx->plan.opt.p;
  cudaStream_t s = ctx->stream;
  const MatvecArgs nm = ctx->near_args();
  double* Vp = ctx->poly_V.p;
  double* hd = ctx->poly_h.p;
  std::vector<double> H((size_t)(k + 1) * k, 0.0), hh((size_t)3 * (k + 1));
  launch_hash_fill(N, 0x5eedULL, ctx->mv_out.p, s);
  launch_mdot(ctx->mv_out.p, N, 1, ctx->mv_out.p, N, ctx->poly_part.p, hd, s);
  CK(cudaMemcpyAsync(hh.data(), hd, sizeof(double), cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  launch_axpby(N, 1.0 / std::sqrt(hh[0]), ctx->mv_out.p, 0.0, Vp, s);
  ctx->launches += 4;
  int steps = 0;
  double hscale = 0.0;
  for (int j = 0; j < k; ++j) {
    launch_mul(N, ctx->dinv.p, Vp + (size_t)j * N, ctx->mv_in.p, s);
    ctx->launches += 1 + launch_near_only(p, nm, s);
    double* w = ctx->mv_out.p;
    for (int pass = 0; pass < 2; ++pass) {
      launch_mdot(Vp, N, j + 1, w, N, ctx->poly_part.p, hd + pass * (k + 1), s);
      launch_maxpy(Vp, N, j + 1, hd + pass * (k + 1), w, N, s);
    }
    launch_mdot(w, N, 1, w, N, ctx->poly_part.p, hd + 2 * (k + 1), s);
    ctx->launches += 8;
    CK(cudaMemcpyAsync(hh.data(), hd, sizeof(double) * hh.size(), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    for (int i = 0; i <= j; ++i) {
      H[(size_t)i * k + j] = hh[i] + hh[(k + 1) + i];
      hscale = std::max(hscale, std::abs(H[(size_t)i * k + j]));
    }
    const double hn = std::sqrt(std::max(hh[2 * (k + 1)], 0.0));
    H[(size_t)(j + 1) * k + j] = hn;
    steps = j + 1;
    if (!std::isfinite(hn) || !(hn > 1e-12 * hscale)) break;  // (near-)invariant subspace
    if (j + 1 < k) {
      launch_axpby(N, 1.0 / hn, w, 0.0, Vp + (size_t)(j + 1) * N, s);
      ctx->launches += 1;
    }
  }
  CK(cudaGetLastError());
  if (steps < k) {  // the leading steps x steps block with its own subdiagonal entry
    std::vector<double> Hs((size_t)(steps + 1) * steps);
    for (int i = 0; i <= steps; ++i)
      for (int j = 0; j < steps; ++j) Hs[(size_t)i * steps + j] = H[(size_t)i * k + j];
    H.swap(Hs);
  }
  if (poly_roots_from_hessenberg(steps, H.data(), steps, ctx->poly) != 0) ctx->poly.n = 0;
  return BEM_OK;
}

int bem_gpu_tc_tuning(bem_gpu_ctx* ctx, int32_t* pairs_in_use, int32_t* candidates, double* ms) {
  if (!ctx || !pairs_in_use || !candidates || !ms) return BEM_ERR_INVALID_ARGUMENT;
  if (!ctx->ready) return BEM_ERR_NOT_READY;
  *pairs_in_use = ctx->mixed ? ctx->tc_tune : 0;
  for (int c = 0; c < 4; ++c) {
    candidates[c] = tune_cand(ctx->plan.opt.p)[c];
    ms[c] = ctx->tc_tune_ms[c];
  }
  return ctx->tc_tuned_here ? 1 : 0;
}

int bem_gpu_setup_phases(bem_gpu_ctx* ctx, double* out) {
  if (!ctx || !out) return BEM_ERR_INVALID_ARGUMENT;
  if (!ctx->ready) return BEM_ERR_NOT_READY;
  for (int k = 0; k < 7; ++k) out[k] = ctx->plan.phase_s[k];
  out[7] = ctx->time_upload;
  out[8] = 1e-3 * ctx->setup_dev_ms;
  out[9] = (ctx->plan.tree_on_device ? 1 : 0) + (ctx->plan.lists_on_device ? 2 : 0);
  for (int k = 0; k < 5; ++k) out[10 + k] = ctx->upload_part_s[k];
  out[15] = 1e-3 * ctx->near_weights_ms;
  return BEM_OK;
}

int bem_gpu_poly_roots(bem_gpu_ctx* ctx, int32_t cap, double* re, double* im) {
  if (!ctx || cap < 0 || (cap > 0 && (!re || !im))) return BEM_ERR_INVALID_ARGUMENT;
  if (!ctx->ready) return BEM_ERR_NOT_READY;
  for (int i = 0; i < ctx->poly.n && i < cap; ++i) {
    re[i] = ctx->poly.re[i];
    im[i] = ctx->poly.im[i];
  }
  return ctx->poly.n;
}

// Set-up of a BVP (refresh: same mesh as the last set-up at new coordinates; see
// bem_gpu_setup_refresh).  With an unchanged structure only the geometry-dependent arrays are
// uploaded and only the geometry-dependent device tables rebuilt.
// Work items of the tensor-core M2L over table images: every item once per row tile, the row
// tiles of a table consecutive (image = table * tiles + tile), so each image is loaded once
// per CTA range.
static cudaError_t upload_tc_items(bem_gpu_ctx* ctx, bool skip) {
  const Plan& P = ctx->plan;
  const int rt = tc_row_tiles(P.opt.p);
  std::vector<int> itab, ibeg, icnt;
  const size_t ni = P.tc_item_tab.size();
  for (size_t i0 = 0; i0 < ni;) {
    size_t i1 = i0;
    while (i1 < ni && P.tc_item_tab[i1] == P.tc_item_tab[i0]) ++i1;
    for (int r = 0; r < rt; ++r)
      for (size_t i = i0; i < i1; ++i) {
        itab.push_back(P.tc_item_tab[i] * rt + r);
        ibeg.push_back(P.tc_item_begin[i]);
        icnt.push_back(P.tc_item_cnt[i]);
      }
    i0 = i1;
  }
  ctx->n_tc_items = (int)itab.size();
  if (skip) return cudaSuccess;
  cudaError_t e;
  if ((e = up(ctx, ctx->tc_item_tab, itab)) != cudaSuccess || (e = up(ctx, ctx->tc_item_begin, ibeg)) != cudaSuccess) return e;
  return up(ctx, ctx->tc_item_cnt, icnt);
}

// Autotuning of the tensor-core M2L work-item size (pairs per item = the MMA's N, 16..80):
// each candidate's items are timed on the contraction kernel alone (CUDA events, after a
// warm-up launch), once per process for each device, expansion order and problem-size class
// (powers of two of the pair count); the best is cached.  The item size changes which CTA
// computes a pair, not the pair's arithmetic: the M2L result is the same bit for bit.
struct TuneEntry {
  int best = 0;
  float ms[4] = {0, 0, 0, 0};
};
static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int>, TuneEntry> g_tune;

static std::tuple<int, int, int> tune_key(const bem_gpu_ctx* ctx) {
  int lg = 0;
  for (int64_t n = ctx->plan.m2l_pairs; n > 1; n >>= 1) ++lg;
  return {ctx->opts.device, ctx->plan.opt.p, lg};
}

static int tune_tc_items(bem_gpu_ctx* ctx) {
  cudaStream_t s = ctx->stream;
  const int p = ctx->plan.opt.p;
  MatvecArgs a = ctx->args(ctx->phi.p, ctx->phin.p, ctx->mv_out.p, nullptr, nullptr);
  ctx->set_ax(a, true);
  ctx->set_tc(a);
  launch_m2l_tc(p, a, s, TC_EXPAND, 1);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  TuneEntry t;
  float best = 1e30f;
  const int* cand = tune_cand(p);
  for (int c = 0; c < 4; ++c) {
    retile_tc_items(ctx->plan, cand[c]);
    ctx->tc_tune = cand[c];
    CK(upload_tc_items(ctx, false));
    ctx->set_tc(a);
    launch_m2l_tc(p, a, s, TC_CONTRACT, 1);
    CK(cudaEventRecord(e0, s));
    for (int r = 0; r < 5; ++r) launch_m2l_tc(p, a, s, TC_CONTRACT, 1);
    CK(cudaEventRecord(e1, s));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    t.ms[c] = ms / 5;
    if (t.ms[c] < best) {
      best = t.ms[c];
      t.best = cand[c];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // the timed contractions added into the fused accumulators without a finalize: clear them
  CK(cudaMemsetAsync(ctx->tc_acc.p, 0, sizeof(float) * ctx->tc_acc.n, s));
  retile_tc_items(ctx->plan, t.best);
  CK(upload_tc_items(ctx, false));
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[tune_key(ctx)] = t;
  }
  ctx->tc_tune = t.best;
  ctx->tc_tuned_here = true;
  for (int c = 0; c < 4; ++c) ctx->tc_tune_ms[c] = t.ms[c];
  return BEM_OK;
}

static int setup_impl(bem_gpu_ctx* ctx, const bem_bvp_desc* d, bool refresh) {
  if (!ctx || !d) return BEM_ERR_INVALID_ARGUMENT;
  CK(cudaSetDevice(ctx->opts.device));
  if (!ctx->noalloc_slots) {
    // the no-alloc mat-vec's slot area: its name is a host-side handle only, the kernels need
    // its address on this device.  The lookup allocates nothing (the area comes with the
    // module, which this loads if nothing of it ran yet); a failure only disables that entry.
    ctx->noalloc_lookup = cudaGetSymbolAddress(&ctx->noalloc_slots, g_m2l_slot_scratch);
    if (ctx->noalloc_lookup != cudaSuccess) {
      ctx->noalloc_slots = nullptr;
      (void)cudaGetLastError();
    }
  }
  const bool had_plan = ctx->ready;
  ctx->ready = false;
  ctx->h2d = ctx->d2h = ctx->launches = 0;
  const double t0 = now_s();
  if (ctx->opts.precision == 1 && !tc_supported(ctx->opts.expansion_order)) {
    ctx->err = "mixed precision needs expansion_order <= 12";
    return BEM_ERR_UNSUPPORTED;
  }
  if (ctx->opts.precision != 0 && ctx->opts.precision != 1) {
    ctx->err = "precision must be 0 (fp64) or 1 (mixed)";
    return BEM_ERR_INVALID_ARGUMENT;
  }
  if (ctx->opts.tc_item_pairs < 0 || ctx->opts.tc_item_pairs > tc_max_pairs(ctx->opts.expansion_order)) {
    ctx->err = "tc_item_pairs must be 0 (autotuned) or 1..128 (p <= 10), 1..80 (p 11, 12)";
    return BEM_ERR_INVALID_ARGUMENT;
  }
  if (ctx->opts.preconditioner < 0 || ctx->opts.preconditioner > 3 || ctx->opts.poly_degree < 0 ||
      ctx->opts.poly_degree > kMaxPolyDegree) {
    ctx->err = "preconditioner must be 0 (none), 1 (Jacobi), 2 (near-field polynomial, degree 0..24; 0: 8) or 3 (near blocks)";
    return BEM_ERR_INVALID_ARGUMENT;
  }
  PlanOptions po;
  po.p = ctx->opts.expansion_order;
  po.theta = ctx->opts.mac_theta;
  po.leaf_max = ctx->opts.leaf_max_elements;
  po.max_level = ctx->opts.max_level;
  if (ctx->opts.tree_on_host == 0) {
    if (!ctx->dtree) ctx->dtree = dtree_create(ctx->stream);
    po.device_tree = ctx->dtree;
  }
  // built into the spare plan (the one before the current: its arrays' memory is reused), then
  // swapped in; the current plan is the refresh's previous plan
  if (!build_plan(ctx->plan_spare, po, d->n_points, d->X, d->n_faces, d->tri, d->face_dirichlet, d->n_dof, d->dof_point, d->dof_face,
                  d->dof_kind, d->face_dof, refresh && had_plan ? &ctx->plan : nullptr, /*defer_m2l_groups=*/true)) {
    ctx->err = ctx->plan_spare.error;
    return BEM_ERR_INVALID_ARGUMENT;
  }
  std::swap(ctx->plan, ctx->plan_spare);
  ctx->time_plan = now_s() - t0;
  double t_part = now_s();
  auto part_done = [&](int k) {
    const double t = now_s();
    ctx->upload_part_s[k] = t - t_part;
    t_part = t;
  };
  Plan& P = ctx->plan;
  ctx->launches += P.device_launches;  // octree and list kernels of the plan
  // a refresh that kept the tree and lists (reuse) and the L2P targets (reuse_near) skips the
  // uploads of what it kept: the buffers still hold the same data
  const bool reuse = P.reused_m2l, reuse_near = P.reused_near;
  {  // pinned area for this set-up's uploads: the previous set-up's total, or an estimate from the
     // plan's array sizes for the first one (pinning a larger area later is slow)
    const size_t ne = (size_t)P.nf, pairs = (size_t)P.m2l_pairs;
    const size_t est = ne * (18 + 6 + 3 + 8) * 8 + ne * 3 * 4 * 4 + (size_t)P.np * 3 * 8 + P.nb_dofs.size() * 4 +
                       pairs * 4 * (ctx->opts.precision == 1 ? 4 : 2) + pairs * 2 + P.dof_inc.size() * 4 +
                       P.blocks.size() * sizeof(NearBlockDev) + P.nb_targets.size() * 8 + P.nb_ranges.size() * 4 +
                       (size_t)P.ndof * 16 + (size_t)P.np * 12 + P.nodes.size() * 64 + (size_t)(4 << 20);
    CK(ctx->stage.begin(std::max(ctx->stage_bytes, reuse ? 0 : est), ctx->stream));
  }
  auto ups = [&](auto& buf, const auto& v) -> cudaError_t { return reuse ? cudaSuccess : up(ctx, buf, v); };
  auto upn = [&](auto& buf, const auto& v) -> cudaError_t { return reuse_near ? cudaSuccess : up(ctx, buf, v); };
  cudaStream_t s = ctx->stream;
  const int NC = ncoef(P.opt.p);
  const int nb = (int)P.nodes.size();
  // node arrays
  std::vector<double> nX(3 * nb);
  std::vector<int> nfb(nb), nfe(nb), cb(nb), ce(nb);
  for (int i = 0; i < nb; ++i) {
    for (int a = 0; a < 3; ++a) nX[3 * i + a] = P.nodes[i].X[a];
    nfb[i] = P.nodes[i].fb;
    nfe[i] = P.nodes[i].fe;
    cb[i] = P.nodes[i].child_begin;
    ce[i] = P.nodes[i].child_end;
  }
  // parents per level (non-empty nodes with children)
  std::vector<int> lp_all, lp_all_off(1, 0);
  for (int l = 0; l < (int)P.level_nodes.size(); ++l) {
    for (int i : P.level_nodes[l])
      if (P.nodes[i].child_end > P.nodes[i].child_begin) lp_all.push_back(i);
    lp_all_off.push_back((int)lp_all.size());
  }
  // Passes that cannot change a result are left out (exactly: the values they skip are zero or
  // never read).  node_up[i]: the parent, or -1 at the root.  M of a node is needed when the
  // node is an M2L source or its parent's M is needed (M2M builds a parent from its children);
  // the local expansion of a node is non-zero only when the node or an ancestor is an M2L
  // target, so the downward pass starts below the levels without targets.
  std::vector<int> node_up(nb, -1);
  std::vector<char> m_needed(nb, 0), l_nonzero(nb, 0);
  for (int i = 0; i < nb; ++i)
    for (int ci = P.nodes[i].child_begin; ci < P.nodes[i].child_end; ++ci) node_up[P.node_children[ci]] = i;
  {
    std::vector<char> is_src(nb, 0);
    for (int32_t s2 : P.m2l_src) is_src[s2] = 1;
    for (int l = 0; l < (int)P.level_nodes.size(); ++l)
      for (int i : P.level_nodes[l]) {
        const int up = node_up[i];
        m_needed[i] = is_src[i] || (up >= 0 && m_needed[up]);
        l_nonzero[i] = (P.m2l_off[i + 1] > P.m2l_off[i]) || (up >= 0 && l_nonzero[up]);
      }
  }
  {  // per-level lists of the tree passes
    const int nlev = (int)P.level_nodes.size();
    ctx->n_tree_levels = nlev;
    std::vector<int> up_needed(nb, -1), mnodes;
    for (int i = 0; i < nb; ++i) up_needed[i] = (node_up[i] >= 0 && m_needed[node_up[i]]) ? node_up[i] : -1;
    // upward: nodes that build a needed multipole from their children or hand theirs up; the
    // same without the leaves (the A.x P2M kernel shifts the leaves' multipoles itself)
    std::vector<int> mnodes_nl, llev(std::max<size_t>(P.leaves.size(), 1), 0);
    ctx->m2m_level_off.assign(1, 0);
    ctx->m2m_level_off_nl.assign(1, 0);
    for (int l = 0; l < nlev; ++l) {
      for (int i : P.level_nodes[l]) {
        const bool parent = P.nodes[i].child_end > P.nodes[i].child_begin;
        if ((parent && m_needed[i]) || up_needed[i] >= 0) mnodes.push_back(i);
        if (parent && (m_needed[i] || up_needed[i] >= 0)) mnodes_nl.push_back(i);
      }
      ctx->m2m_level_off.push_back((int)mnodes.size());
      ctx->m2m_level_off_nl.push_back((int)mnodes_nl.size());
    }
    for (size_t li = 0; li < P.leaves.size(); ++li) llev[li] = P.nodes[P.leaves[li]].level;
    // downward: (parent, child) pairs of the parents with a non-zero local expansion
    std::vector<int2> pairs;
    ctx->l2l_level_off.assign(1, 0);
    for (int l = 0; l < nlev; ++l) {
      for (int i : P.level_nodes[l])
        if (l_nonzero[i])
          for (int ci = P.nodes[i].child_begin; ci < P.nodes[i].child_end; ++ci) pairs.push_back(make_int2(i, P.node_children[ci]));
      ctx->l2l_level_off.push_back((int)pairs.size());
    }
    if (mnodes.empty()) mnodes.push_back(0);  // keep the device arrays non-empty
    if (mnodes_nl.empty()) mnodes_nl.push_back(0);
    if (pairs.empty()) pairs.push_back(make_int2(0, 0));
    CK(ups(ctx->m2m_nodes, mnodes));
    CK(ups(ctx->node_up, up_needed));
    CK(ups(ctx->m2m_nodes_nl, mnodes_nl));
    CK(ups(ctx->leaf_level, llev));
    CK(ups(ctx->l2l_pairs, pairs));
    CK(ctx->Yup.alloc((size_t)std::max(nb, 1) * 2 * ncoef(P.opt.p)));
  }
  {  // parent-to-child F tables per (level, octant), from the first pair met of each
    const int nlev = (int)lp_all_off.size() - 1;
    std::vector<double> fv((size_t)std::max(nlev, 1) * 8 * 3, 0.0);
    std::vector<char> seen((size_t)std::max(nlev, 1) * 8, 0);
    for (int l = 0; l < nlev; ++l)
      for (int q = lp_all_off[l]; q < lp_all_off[l + 1]; ++q) {
        const int par = lp_all[q];
        for (int ci = P.nodes[par].child_begin; ci < P.nodes[par].child_end; ++ci) {
          const int c = P.node_children[ci];
          double d[3];
          for (int a2 = 0; a2 < 3; ++a2) d[a2] = P.nodes[c].X[a2] - P.nodes[par].X[a2];
          const int o = (d[0] > 0 ? 1 : 0) | (d[1] > 0 ? 2 : 0) | (d[2] > 0 ? 4 : 0);
          if (!seen[l * 8 + o]) {
            seen[l * 8 + o] = 1;
            for (int a2 = 0; a2 < 3; ++a2) fv[(l * 8 + o) * 3 + a2] = d[a2];
          }
        }
      }
    if (!reuse) {
      CK(up(ctx, ctx->ftab_vec, fv));
      const int NFt = (P.opt.p + 1) * (P.opt.p + 1);
      CK(ctx->Ftab.alloc((size_t)std::max(nlev, 1) * 8 * NFt));
      launch_f_tables(P.opt.p, std::max(nlev, 1) * 8, ctx->ftab_vec.p, ctx->Ftab.p, s);
      ctx->launches += 1;
    }
  }
  std::vector<NearBlockDev> bd(P.blocks.size());
  ctx->max_ntgt = 1;
  int max_ndof = 1;
  int64_t w4_total = 0;
  for (size_t i = 0; i < P.blocks.size(); ++i) {
    const auto& b = P.blocks[i];
    bd[i].w_off = b.w_off;
    bd[i].w4_off = w4_total;
    w4_total += (int64_t)b.ntgt * ((b.ndof + 3) & ~3);
    bd[i].node = b.node;
    bd[i].dof_off = b.dof_off;
    bd[i].ndof = b.ndof;
    bd[i].tgt_off = b.tgt_off;
    bd[i].ntgt = b.ntgt;
    bd[i].rng_off = b.rng_off;
    bd[i].nrng = b.nrng;
    ctx->max_ntgt = std::max(ctx->max_ntgt, b.ntgt);
    max_ndof = std::max(max_ndof, b.ndof);
  }
  ctx->w4_total = w4_total;
  {  // per near block: its bucket and the bucket's ancestors that are M2L targets, deepest first
    std::vector<int> off(1, 0), path;
    for (const auto& b : P.blocks) {
      for (int a = b.node; a >= 0; a = node_up[a])
        if (P.m2l_off[a + 1] > P.m2l_off[a]) path.push_back(a);
      off.push_back((int)path.size());
    }
    ctx->max_path = 0;
    for (size_t b = 0; b + 1 < off.size(); ++b) ctx->max_path = std::max(ctx->max_path, off[b + 1] - off[b]);
    if (configure_target_rows_smem(P.opt.p, ctx->max_path, ctx->max_ntgt) != 0) {
      ctx->err = "too many targets in one bucket for the rows kernel";
      return BEM_ERR_UNSUPPORTED;
    }
    if (path.empty()) path.push_back(0);
    CK(up(ctx, ctx->blk_path_off, off));
    CK(up(ctx, ctx->blk_path, path));
  }
  // shared memory budget of k_targets: chunk of (phi, phin) + per-target sums
  const int smem_cap = 160 * 1024;
  if (ctx->max_ntgt * 16 > smem_cap / 2) {
    ctx->err = "too many targets in one bucket";
    return BEM_ERR_UNSUPPORTED;
  }
  // a multiple of 4 columns (the FP32 rows are read 4 columns at a time)
  ctx->chunk = std::min((max_ndof + 3) & ~3, ((smem_cap - ctx->max_ntgt * 16) / 16) & ~3);
  configure_targets_smem(P.opt.p, (ctx->chunk + ctx->max_ntgt) * 16);
  if (configure_targets_ax_smem(ctx->max_ntgt) != 0) {
    ctx->err = "too many targets in one bucket for the near-field kernel";
    return BEM_ERR_UNSUPPORTED;
  }
  configure_m2l_smem(P.opt.p);


  part_done(0);
  // The near-field quadrature needs only the near blocks and the element geometry: those go up
  // first and the quadrature runs on the device while the host groups the M2L pairs.  Its
  // device time is counted into the set-up's (a window of its own: the uploads around it are
  // not device work).
  CK(up(ctx, ctx->Xs, P.Xs));
  CK(up(ctx, ctx->e_near, P.e_near));
  CK(ups(ctx->e_vtx, P.e_vtx));
  CK(upn(ctx->nb_dofs, P.nb_dofs));
  CK(upn(ctx->nb_targets, P.nb_targets));
  CK(upn(ctx->nb_ranges, P.nb_ranges));
  CK(ups(ctx->dof_inc_off, P.dof_inc_off));
  CK(ups(ctx->dof_inc, P.dof_inc));
  CK(upn(ctx->blocks, bd));
  CK(ctx->WG.alloc(std::max<int64_t>(P.nnz, 1)));
  CK(ctx->WGn.alloc(std::max<int64_t>(P.nnz, 1)));
  NearArgs na;
  na.n_blocks = (int)P.blocks.size();
  na.blocks = ctx->blocks.p;
  na.nb_dofs = ctx->nb_dofs.p;
  na.nb_targets = ctx->nb_targets.p;
  na.nb_ranges = ctx->nb_ranges.p;
  na.dof_inc_off = ctx->dof_inc_off.p;
  na.dof_inc = ctx->dof_inc.p;
  na.Xs = ctx->Xs.p;
  na.e_vtx = ctx->e_vtx.p;
  na.e_near = ctx->e_near.p;
  na.near_region = P.near_region;
  na.WG = ctx->WG.p;
  na.WGn = ctx->WGn.p;
  {
    int mr = 0;
    int64_t mel = 1;
    for (int bi = 0; bi < (int)P.blocks.size(); ++bi) {
      const auto& nbk = P.blocks[bi];
      mr = std::max(mr, nbk.nrng);
      int64_t ne = 0;
      for (int r = 0; r < nbk.nrng; ++r) ne += P.nb_ranges[2 * (nbk.rng_off + r) + 1] - P.nb_ranges[2 * (nbk.rng_off + r)];
      mel = std::max(mel, ne);
    }
    na.n_slots = (int)P.nb_targets.size();
    CK(ctx->near_counter.alloc(1));
    na.next_block = ctx->near_counter.p;
    na.max_nrng = mr;
    na.scratch_stride = 3 * mel;
    CK(ctx->near_scratch.alloc((size_t)near_weights_grid() * na.scratch_stride));
    na.scratch = ctx->near_scratch.p;
  }
  CK(cudaEventRecord(ctx->ev[4], s));
  if (launch_near_weights(na, s) != 0) {
    ctx->err = "near-field quadrature: block element ranges exceed the kernel's shared memory";
    return BEM_ERR_UNSUPPORTED;
  }
  CK(cudaEventRecord(ctx->ev[5], s));
  CK(cudaGetLastError());
  if (!P.reused_m2l) {  // M2L grouping on the host meanwhile
    const double tg = now_s();
    if (!build_m2l_groups(P)) {
      ctx->err = P.error;
      return BEM_ERR_INVALID_ARGUMENT;
    }
    P.phase_s[4] += now_s() - tg;
    ctx->time_plan += now_s() - tg;  // host plan work, not upload
  }
  t_part = now_s();
  const std::vector<int>& mt = P.m2l_targets;
  ctx->n_m2l_targets = (int)mt.size();
  CK(up(ctx, ctx->e_q, P.e_q));
  CK(up(ctx, ctx->e_W, P.e_W));
  CK(up(ctx, ctx->e_n, P.e_n));
  CK(ups(ctx->e_dof, P.e_dof));
  CK(ups(ctx->node_X, nX));
  CK(ups(ctx->node_fb, nfb));
  CK(ups(ctx->node_fe, nfe));
  CK(ups(ctx->child_begin, cb));
  CK(ups(ctx->child_end, ce));
  CK(ups(ctx->node_children, P.node_children));
  CK(ups(ctx->leaves, P.leaves));
  CK(ups(ctx->m2l_targets, mt));
  CK(ups(ctx->m2l_off, P.m2l_off));
  CK(ups(ctx->m2l_src, P.m2l_src));
  CK(ups(ctx->point_dof_off, P.point_dof_off));
  CK(ups(ctx->point_dof, P.point_dof));
  CK(ups(ctx->dof_kind, P.dof_kind));
  CK(ups(ctx->dof_point, P.dof_point));
  CK(ups(ctx->chunk_grp, P.chunk_grp));
  CK(ups(ctx->chunk_begin, P.chunk_begin));
  CK(ups(ctx->chunk_cnt, P.chunk_cnt));
  CK(ups(ctx->grp_pair, P.grp_pair));
  CK(ups(ctx->grp_vec, P.grp_vec));
  {
    const int ngroups = (int)P.grp_off.size() - 1;
    const int Q = 2 * P.opt.p;
    CK(ctx->Sg.alloc((size_t)std::max(ngroups, 1) * (Q + 1) * (Q + 1)));
    // per-pair slots; the tensor-core path stores tc_kpo floats per pair in the same buffer
    const size_t y64 = (size_t)std::max<int64_t>(P.m2l_pairs, 1) * 2 * NC;
    const size_t ytc = ((size_t)std::max<int64_t>(P.m2l_pairs, 1) * tc_kpo(P.opt.p) * sizeof(float) + sizeof(double2) - 1) / sizeof(double2);
    CK(ctx->Y.alloc(ctx->opts.precision == 1 ? std::max(y64, ytc) : y64));
  }
  ctx->mixed = ctx->opts.precision == 1;
  part_done(1);
  if (ctx->mixed) {  // tensor-core M2L: translation tables, multipole rows, work items
    const int p = P.opt.p, kp = tc_kp(p);
    if (!reuse) {  // item size: forced, tuned earlier for this class, or the kernel's maximum until tuned
      int mp = 80;
      ctx->tc_tuned_here = false;
      if (ctx->opts.tc_item_pairs > 0) {
        mp = std::min(ctx->opts.tc_item_pairs, tc_max_pairs(P.opt.p));
      } else {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(tune_key(ctx));
        if (it != g_tune.end()) {
          mp = it->second.best;
          for (int c = 0; c < 4; ++c) ctx->tc_tune_ms[c] = it->second.ms[c];
        }
      }
      ctx->tc_tune = mp;
      build_tc_groups(P, mp);
    }
    const int ntab = (int)(P.tc_tab.size() / 4);
    std::vector<double> dl(nb), al(kp);
    for (int i = 0; i < nb; ++i) dl[i] = P.nodes[i].dL;
    tc_alpha_host(p, al.data());
    CK(upload_tc_items(ctx, reuse));
    {  // work-item order j -> source bucket and compact target index; pair slot k -> its position j
       // (the row of its partial)
      std::vector<int>&src = ctx->h_tc_src, &pos = ctx->h_tc_pos, &tgt = ctx->h_tc_tgt;  // kept across set-ups
      tc_item_arrays(P, src, pos, tgt);
      CK(ups(ctx->tc_src, src));
      CK(ups(ctx->tc_pos, pos));
      CK(ups(ctx->tc_tgt, tgt));
    }
    CK(ctx->tc_acc.alloc((size_t)std::max<size_t>(P.m2l_targets.size(), 1) * tc_kpo(p)));
    CK(ups(ctx->tc_tabvec, P.tc_tab));
    CK(ups(ctx->tc_alpha, al));
    CK(ups(ctx->node_dL, dl));
    CK(ctx->tc_T.alloc((size_t)std::max(ntab, 1) * tc_row_tiles(p) * tc_table_bytes(p) / 2));
    CK(ctx->tc_Mt.alloc((size_t)(nb + 1) * 2 * kp));
    ctx->tc_map.assign(tc_rows_map_bytes(), 0);
    if (tc_make_rows_map(ctx->tc_map.data(), ctx->tc_Mt.p, 2 * (nb + 1), p) != 0) {
      ctx->err = "mixed precision: could not encode the TMA tensor map of the multipole rows";
      return BEM_ERR_DEVICE;
    }
    CK(ctx->tc_escale.alloc((size_t)nb + 1));
    CK(ctx->tc_err.alloc(1));
    CK(ctx->tc_max.alloc(1));
    int sms = 148;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->opts.device));
    ctx->tc_grid = sms;
  }
  part_done(2);
  {  // P2M operator of A.x: the DOFs of each leaf's elements, and the slot of every vertex
    const int nl = (int)P.leaves.size();
    std::vector<int> ldo(nl + 1, 0), ld, es(3 * (size_t)P.nf, 0);
    std::vector<int> seen(P.ndof, -1);
    for (int li = 0; li < nl; ++li) {
      const auto& Nd = P.nodes[P.leaves[li]];
      for (int s2 = Nd.fb; s2 < Nd.fe; ++s2)
        for (int a = 0; a < 3; ++a) {
          const int d = P.e_dof[3 * s2 + a];
          if (seen[d] < ldo[li]) {  // first time in this leaf
            seen[d] = (int)ld.size();
            ld.push_back(d);
          }
          es[3 * s2 + a] = seen[d] - ldo[li];
        }
      ldo[li + 1] = (int)ld.size();
    }
    CK(ups(ctx->leaf_dof_off, ldo));
    CK(ups(ctx->leaf_dof, ld));
    CK(ups(ctx->e_slot, es));
    CK(ctx->p2m_C.alloc(std::max<size_t>(ld.size(), 1) * NC));
    if (ctx->mixed) CK(ctx->p2m_C32.alloc(std::max<size_t>(ld.size(), 1) * NC));
  }
  part_done(3);
  CK(ctx->M.alloc((size_t)nb * 2 * NC));
  CK(ctx->L.alloc((size_t)nb * 2 * NC));
  CK(ctx->Wc.alloc(std::max<int64_t>(ctx->w4_total, 1)));  // rows padded to 4 columns, as the FP32 copy
  const bool want_w32 = ctx->opts.precision == 1 || ctx->opts.preconditioner == 2;
  if (want_w32) CK(ctx->Wc32.alloc(std::max<int64_t>(ctx->w4_total, 1)));
  const int N = P.ndof;
  if (ctx->opts.preconditioner == 2) {
    const int k = poly_degree(ctx->opts);
    CK(ctx->poly_V.alloc((size_t)(k + 1) * N));
    CK(ctx->poly_h.alloc((size_t)3 * (k + 1)));
    CK(ctx->poly_part.alloc((size_t)mdot_blocks(N) * (k + 1)));
  }
  CK(ctx->phi.alloc(N));
  CK(ctx->phin.alloc(N));
  CK(ctx->known_s.alloc(N));
  CK(ctx->rows.alloc(N));
  CK(ctx->diag.alloc(N));
  CK(ctx->GPhin.alloc(P.np));
  CK(ctx->GnPhi.alloc(P.np));
  CK(ctx->mv_in.alloc(N));
  CK(ctx->mv_out.alloc(N));
  {  // right-Jacobi scaling inputs: each point's near-field block row
    std::vector<int> bop(P.np), rop(P.np);
    for (int p = 0; p < P.np; ++p) {
      bop[p] = std::max(P.block_of_point[p], 0);
      rop[p] = std::max(P.row_of_point[p], 0);
    }
    CK(upn(ctx->block_of_point, bop));
    CK(upn(ctx->row_of_point, rop));
    CK(upn(ctx->self_col, P.self_col));
    CK(ctx->dinv.alloc(N));
  }
  part_done(4);
  // no wait here: the device part follows the copies (and the near-field quadrature) in stream
  // order, and its events time only device work
  ctx->time_upload = now_s() - t0 - ctx->time_plan;
  ctx->stage_bytes = std::max(ctx->stage_bytes, ctx->stage.used);
  // device part of the set-up starts here (inputs resident): every kernel that derives the
  // operator's tables and weights from the uploaded plan
  CK(cudaEventRecord(ctx->ev[0], s));
  CK(cudaMemsetAsync(ctx->GPhin.p, 0, sizeof(double) * P.np, s));
  CK(cudaMemsetAsync(ctx->GnPhi.p, 0, sizeof(double) * P.np, s));
  CK(cudaMemsetAsync(ctx->M.p, 0, sizeof(double2) * ctx->M.n, s));
  CK(cudaMemsetAsync(ctx->p2m_C.p, 0, sizeof(double2) * ctx->p2m_C.n, s));
  if (!reuse) {  // translation tables depend on the bucket geometry alone
    launch_s_tables(P.opt.p, (int)P.grp_off.size() - 1, ctx->grp_vec.p, ctx->Sg.p, s);
    ctx->launches += 1;
  }
  CK(ctx->near_sum.alloc(std::max<size_t>(P.nb_targets.size(), 1)));
  if (ctx->mixed) {
    CK(cudaMemsetAsync(ctx->tc_Mt.p, 0, sizeof(uint16_t) * ctx->tc_Mt.n, s));
    CK(cudaMemsetAsync(ctx->tc_acc.p, 0, sizeof(float) * ctx->tc_acc.n, s));
    CK(cudaMemsetAsync(ctx->tc_err.p, 0, sizeof(int), s));
    if (!reuse) {
      CK(cudaMemsetAsync(ctx->tc_max.p, 0, sizeof(unsigned int), s));
      launch_tc_tables(P.opt.p, (int)(P.tc_tab.size() / 4), ctx->tc_tabvec.p, ctx->tc_alpha.p, ctx->tc_T.p, ctx->tc_max.p, s);
      ctx->launches += 1;
    }
  }
  {
    MatvecArgs pa = ctx->args(nullptr, nullptr, nullptr, nullptr, nullptr);
    ctx->set_ax(pa, false);
    launch_p2m_op(P.opt.p, pa, ctx->e_slot.p, s);
    ctx->launches += 1;
    if (ctx->mixed) {
      launch_to_float2(ctx->p2m_C.n, ctx->p2m_C.p, ctx->p2m_C32.p, s);
      ctx->launches += 1;
    }
  }
  launch_combine_weights((int)P.blocks.size(), ctx->blocks.p, ctx->nb_dofs.p, ctx->dof_kind.p, ctx->WG.p, ctx->WGn.p, ctx->Wc.p,
                         want_w32 ? ctx->Wc32.p : nullptr, s);
  ctx->launches += want_w32 ? 2 : 1;
  CK(cudaGetLastError());
  // rigid-mode diagonal (BEM_solveBVP_GMRES_FMM.hpp:2661-2716)
  launch_densities(N, 2, nullptr, nullptr, ctx->dof_kind.p, ctx->phi.p, ctx->phin.p, s);  // phi = 1, phin = 0
  run_fmm(ctx, nullptr, nullptr, ctx->GnPhi.p);
  launch_diag(N, ctx->dof_point.p, ctx->GnPhi.p, ctx->diag.p, s);
  ctx->launches += 3;
  CK(cudaGetLastError());
  // right-Jacobi scaling from the near-field diagonal entries
  launch_jacobi(N, ctx->dof_point.p, ctx->dof_kind.p, ctx->diag.p, ctx->block_of_point.p, ctx->row_of_point.p, ctx->blocks.p,
                ctx->self_col.p, ctx->WG.p, ctx->WGn.p, ctx->dinv.p, s);
  ctx->launches += 1;
  CK(cudaGetLastError());
  if (ctx->opts.preconditioner == 3) {  // near-block preconditioner: cores = the DOFs of each block's targets
    const int nb = (int)P.blocks.size();
    std::vector<int> doff(nb + 1, 0), cdofs;
    std::vector<int64_t> ioff(nb + 1, 0);
    cdofs.reserve(N);
    for (int b = 0; b < nb; ++b) {
      const auto& B = P.blocks[b];
      for (int tl = 0; tl < B.ntgt; ++tl) {
        const int p = P.nb_targets[B.tgt_off + tl];
        for (int k = P.point_dof_off[p]; k < P.point_dof_off[p + 1]; ++k) cdofs.push_back(P.point_dof[k]);
      }
      doff[b + 1] = (int)cdofs.size();
      const int64_t m = doff[b + 1] - doff[b];
      ioff[b + 1] = ioff[b] + (m <= kBjMaxCore ? m * m : m);
    }
    if ((int)cdofs.size() != N) {
      ctx->err = "near-block preconditioner: the blocks' targets do not cover every DOF once";
      return BEM_ERR_INVALID_ARGUMENT;
    }
    CK(ctx->bj_doff.alloc(nb + 1));
    CK(ctx->bj_dofs.alloc(std::max(N, 1)));
    CK(ctx->bj_ioff.alloc(nb + 1));
    CK(ctx->bj_inv.alloc(std::max<int64_t>(ioff[nb], 1)));
    CK(ctx->bj_tmp.alloc(std::max(N, 1)));
    CK(cudaMemcpyAsync(ctx->bj_doff.p, doff.data(), sizeof(int) * (nb + 1), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->bj_dofs.p, cdofs.data(), sizeof(int) * N, cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(ctx->bj_ioff.p, ioff.data(), sizeof(int64_t) * (nb + 1), cudaMemcpyHostToDevice, s));
    CK(cudaStreamSynchronize(s));  // the host vectors go out of scope
    launch_bj_setup(ctx->bj_args(), ctx->nb_dofs.p, ctx->dof_point.p, ctx->row_of_point.p, ctx->dof_kind.p, ctx->diag.p, ctx->Wc.p,
                    ctx->dinv.p, s);
    ctx->launches += 1;
    CK(cudaGetLastError());
  }
  ctx->poly.n = 0;
  if (ctx->opts.preconditioner == 2) {
    const int rc = build_poly(ctx);
    if (rc != BEM_OK) return rc;
  }
  CK(cudaEventRecord(ctx->ev[1], s));
  if (ctx->mixed && !reuse) {  // FP16 tables must stay far from the FP16 range limit (65504)
    unsigned int bits = 0;
    CK(cudaMemcpyAsync(&bits, ctx->tc_max.p, sizeof(bits), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    float mx;
    std::memcpy(&mx, &bits, sizeof(mx));
    if (!(mx < 1024.f)) {
      ctx->err = "mixed precision: translation table entry " + std::to_string(mx) + " too large for FP16 operands";
      return BEM_ERR_UNSUPPORTED;
    }
  }
  if (ctx->mixed && !reuse && ctx->opts.tc_item_pairs <= 0) {
    bool known;
    {
      std::lock_guard<std::mutex> lk(g_tune_mu);
      known = g_tune.count(tune_key(ctx)) > 0;
    }
    if (!known) {  // once per process and problem class, after the device-time window
      const int trc = tune_tc_items(ctx);
      if (trc != BEM_OK) return trc;
    }
  }
  int rc = build_graph(ctx);
  if (rc != BEM_OK) return rc;
  CK(cudaStreamSynchronize(s));
  CK(cudaEventElapsedTime(&ctx->setup_dev_ms, ctx->ev[0], ctx->ev[1]));
  {
    float nw_ms = 0.f;
    CK(cudaEventElapsedTime(&nw_ms, ctx->ev[4], ctx->ev[5]));
    ctx->setup_dev_ms += nw_ms;
    ctx->near_weights_ms = nw_ms;
  }
  ctx->setup_h2d = ctx->h2d;
  ctx->setup_launches = ctx->launches;
  ctx->time_setup = now_s() - t0;
  ctx->ready = true;
  return BEM_OK;
}

int bem_gpu_setup(bem_gpu_ctx* ctx, const bem_bvp_desc* d) { return setup_impl(ctx, d, false); }

int bem_gpu_setup_refresh(bem_gpu_ctx* ctx, const bem_bvp_desc* d) {
  const int rc = setup_impl(ctx, d, true);
  return rc != BEM_OK ? rc : (int)ctx->plan.reused_m2l + (int)ctx->plan.reused_near;
}

int bem_gpu_apply(bem_gpu_ctx* ctx, const double* phi, const double* phin, double* Av) {
  if (!ctx || !phi || !phin || !Av) return BEM_ERR_INVALID_ARGUMENT;
  if (!ctx->ready) return BEM_ERR_NOT_READY;
  CK(cudaSetDevice(ctx->opts.device));
  const int N = ctx->plan.ndof;
  cudaStream_t s = ctx->stream;
  CK(cudaMemcpyAsync(ctx->phi.p, phi, sizeof(double) * N, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(ctx->phin.p, phin, sizeof(double) * N, cudaMemcpyHostToDevice, s));
  run_fmm(ctx, ctx->rows.p, nullptr, nullptr);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(Av, ctx->rows.p, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return BEM_OK;
}

int bem_gpu_point_integrals(bem_gpu_ctx* ctx, const double* phi, const double* phin, double* GPhin, double* GnPhi) {
  if (!ctx || !phi || !phin || !GPhin || !GnPhi) return BEM_ERR_INVALID_ARGUMENT;
  if (!ctx->ready) return BEM_ERR_NOT_READY;
  CK(cudaSetDevice(ctx->opts.device));
  const int N = ctx->plan.ndof;
  cudaStream_t s = ctx->stream;
  CK(cudaMemcpyAsync(ctx->phi.p, phi, sizeof(double) * N, cudaMemcpyHostToDevice, s));
  CK(cudaMemcpyAsync(ctx->phin.p, phin, sizeof(double) * N, cudaMemcpyHostToDevice, s));
  CK(cudaMemsetAsync(ctx->GPhin.p, 0, sizeof(double) * ctx->plan.np, s));
  CK(cudaMemsetAsync(ctx->GnPhi.p, 0, sizeof(double) * ctx->plan.np, s));
  run_fmm(ctx, nullptr, ctx->GPhin.p, ctx->GnPhi.p);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(GPhin, ctx->GPhin.p, sizeof(double) * ctx->plan.np, cudaMemcpyDeviceToHost, s));
  CK(cudaMemcpyAsync(GnPhi, ctx->GnPhi.p, sizeof(double) * ctx->plan.np, cudaMemcpyDeviceToHost, s));
  CK(cudaStreamSynchronize(s));
  return BEM_OK;
}

int bem_gpu_matvec_device(bem_gpu_ctx* ctx, const double* d_x, double* d_y) {
  if (!ctx || !d_x || !d_y) return BEM_ERR_INVALID_ARGUMENT;
  if (!ctx->ready) return BEM_ERR_NOT_READY;
  const int N = ctx->plan.ndof;
  cudaStream_t s = ctx->stream;
  if (d_x != ctx->mv_in.p) CK(cudaMemcpyAsync(ctx->mv_in.p, d_x, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
  CK(cudaGraphLaunch(ctx->graph_exec, s));
  if (d_y != ctx->mv_out.p) CK(cudaMemcpyAsync(d_y, ctx->mv_out.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
  return BEM_OK;
}

int bem_gpu_get_diag(bem_gpu_ctx* ctx, double* diag) {
  if (!ctx || !diag) return BEM_ERR_INVALID_ARGUMENT;
  if (!ctx->ready) return BEM_ERR_NOT_READY;
  CK(cudaMemcpyAsync(diag, ctx->diag.p, sizeof(double) * ctx->plan.ndof, cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  return BEM_OK;
}

double bem_gpu_scale_factor(const bem_gpu_ctx* ctx) { return ctx ? ctx->plan.L : 0.0; }

int bem_gpu_near_row(bem_gpu_ctx* ctx, int32_t point, int32_t cap, int32_t* dof, double* wG, double* wGn) {
  if (!ctx || point < 0 || point >= ctx->plan.np || cap < 0) return BEM_ERR_INVALID_ARGUMENT;
  if (!ctx->ready) return BEM_ERR_NOT_READY;
  const Plan& P = ctx->plan;
  const int bi = P.block_of_point[point];
  if (bi < 0) return 0;
  const auto& b = P.blocks[bi];
  const int n = std::min(cap, b.ndof);
  if (n > 0) {
    if (!dof || !wG || !wGn) return BEM_ERR_INVALID_ARGUMENT;
    // the row in ascending DOF order (the block keeps its DOFs in first-appearance order)
    const int64_t off = b.w_off + (int64_t)P.row_of_point[point] * b.ndof;
    std::vector<double> g(b.ndof), gn(b.ndof);
    CK(cudaMemcpyAsync(g.data(), ctx->WG.p + off, sizeof(double) * b.ndof, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaMemcpyAsync(gn.data(), ctx->WGn.p + off, sizeof(double) * b.ndof, cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    std::vector<int> ord(b.ndof);
    for (int j = 0; j < b.ndof; ++j) ord[j] = j;
    std::sort(ord.begin(), ord.end(), [&](int x, int y) { return P.nb_dofs[b.dof_off + x] < P.nb_dofs[b.dof_off + y]; });
    for (int j = 0; j < n; ++j) {
      dof[j] = P.nb_dofs[b.dof_off + ord[j]];
      wG[j] = g[ord[j]];
      wGn[j] = gn[ord[j]];
    }
  }
  return b.ndof;
}

int bem_gpu_face_leaf(bem_gpu_ctx* ctx, int32_t* level, double* corner) {
  if (!ctx || !level || !corner) return BEM_ERR_INVALID_ARGUMENT;
  if (!ctx->ready) return BEM_ERR_NOT_READY;
  const Plan& P = ctx->plan;
  for (int f = 0; f < P.nf; ++f) {
    level[f] = -1;
    corner[3 * f] = corner[3 * f + 1] = corner[3 * f + 2] = 0.0;
    const int s = P.pos_of_face[f];
    if (s < 0) continue;
    const int o = P.owner_of_pos[s];
    if (o < 0 || P.nodes[o].child_end > P.nodes[o].child_begin) continue;
    level[f] = P.nodes[o].level;
    for (int a = 0; a < 3; ++a) corner[3 * f + a] = P.nodes[o].lo[a];
  }
  return BEM_OK;
}

int bem_gpu_near_stats(bem_gpu_ctx* ctx, int64_t* out) {
  if (!ctx || !out) return BEM_ERR_INVALID_ARGUMENT;
  if (!ctx->ready) return BEM_ERR_NOT_READY;
  const Plan& P = ctx->plan;
  int64_t w = 0, w4 = 0, cols = 0, tg = 0;
  for (const Plan::NearBlock& b : P.blocks) {
    w += (int64_t)b.ntgt * b.ndof;
    w4 += (int64_t)b.ntgt * ((b.ndof + 3) & ~3);
    cols += b.ndof;
    tg += b.ntgt;
  }
  out[0] = w;
  out[1] = w4;
  out[2] = cols;
  out[3] = (int64_t)P.blocks.size();
  out[4] = tg;
  out[5] = P.ndof;
  return BEM_OK;
}

int64_t bem_gpu_device_bytes(const bem_gpu_ctx* ctx) { return ctx ? ctx->dev_bytes : 0; }

// Device memory of one BVP from its sizes alone (no plan is built): near-field weights (two FP64
// arrays, the combined FP64 copy and, mixed, the FP32 copy; about 52 nonzeros per point per
// element of the leaf size on these meshes, at most one per DOF), the M2L pair slots (about 11
// pairs per element), the P2M operator, the Krylov basis (twice with the polynomial
// preconditioner's flexible vectors) and the per-element arrays, plus 64 MB for the rest.
int64_t bem_gpu_estimate_bytes(const bem_gpu_opts* o, const bem_bvp_desc* d) {
  if (!o || !d || d->n_points <= 0 || d->n_faces <= 0) return 0;
  const int64_t np = d->n_points, nf = d->n_faces, ndof = std::max(d->n_dof, 1);
  const int p = std::max(1, std::min(o->expansion_order, 12));
  const int64_t nc = (int64_t)(p + 1) * (p + 2) / 2, kp = ((int64_t)(p + 1) * (p + 1) + 63) / 64 * 64;
  const int64_t nnz = std::min<int64_t>(np * 52 * std::max(o->leaf_max_elements, 1), np * ndof);
  const int64_t pairs = 11 * nf;
  int64_t b = nnz * (8 + 8 + 8 + (o->precision == 1 ? 4 : 0));
  b += pairs * 2 * nc * 16 + (o->precision == 1 ? pairs * (kp * 4 / 8 + 8) : 0);
  b += nf * 2 * nc * 16 + (o->precision == 1 ? nf * 2 * nc * 8 : 0);  // P2M operator columns (and their FP32 copy)
  b += (int64_t)(std::max(o->max_iter, 1) + 2) * ndof * 8 * (o->preconditioner == 2 ? 2 : 1);
  b += nf * (18 + 6 + 3 + 8) * 8 + nf * 3 * 4 * 4 + np * 64 + ndof * 160;
  if (o->preconditioner == 3) b += ndof * (64 * 8 + 16);  // near-block inverses (cores of <= 64 DOFs) and core lists
  return b + ((int64_t)64 << 20);
}

int bem_gpu_tree_stats(bem_gpu_ctx* ctx, int64_t* out) {
  if (!ctx || !out) return BEM_ERR_INVALID_ARGUMENT;
  if (!ctx->ready) return BEM_ERR_NOT_READY;
  const Plan& P = ctx->plan;
  int64_t nodes = 0;
  int depth = 0;
  for (size_t l = 0; l < P.level_nodes.size(); ++l) {
    nodes += (int64_t)P.level_nodes[l].size();
    if (!P.level_nodes[l].empty()) depth = (int)l;
  }
  out[0] = nodes;
  out[1] = (int64_t)P.leaves.size();
  out[2] = depth;
  out[3] = P.n_added;
  out[4] = P.m2l_pairs;
  out[5] = P.near_pairs;
  out[6] = P.nnz;
  out[7] = (int64_t)P.blocks.size();
  out[8] = (int64_t)P.chunk_grp.size();
  out[9] = (int64_t)P.grp_off.size() - 1;
  return BEM_OK;
}

static int64_t plan_diffs(const Plan& a1, const Plan& b1);

int bem_gpu_tree_check(const bem_gpu_opts* opts, const bem_bvp_desc* d, int64_t* out) {
  if (!opts || !d || !out) return BEM_ERR_INVALID_ARGUMENT;
  cudaStream_t st = nullptr;
  if (cudaSetDevice(opts->device) != cudaSuccess || cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess)
    return BEM_ERR_DEVICE;
  DeviceTree* dt = dtree_create(st);
  PlanOptions po;
  po.p = opts->expansion_order;
  po.theta = opts->mac_theta;
  po.leaf_max = opts->leaf_max_elements;
  po.max_level = opts->max_level;
  Plan host, dev;
  bool ok = build_plan(host, po, d->n_points, d->X, d->n_faces, d->tri, d->face_dirichlet, d->n_dof, d->dof_point, d->dof_face,
                       d->dof_kind, d->face_dof);
  po.device_tree = dt;
  ok = ok && build_plan(dev, po, d->n_points, d->X, d->n_faces, d->tri, d->face_dirichlet, d->n_dof, d->dof_point, d->dof_face,
                        d->dof_kind, d->face_dof);
  dtree_destroy(dt);
  cudaStreamDestroy(st);
  if (!ok) return BEM_ERR_INVALID_ARGUMENT;
  out[0] = (int)dev.tree_on_device + 2 * (int)dev.lists_on_device;
  out[1] = plan_diffs(host, dev) + (host.n_child_drops != dev.n_child_drops) + (host.n_added != dev.n_added);
  out[2] = (int64_t)dev.nodes.size();
  out[3] = dev.n_child_drops;
  return BEM_OK;
}

static int64_t plan_diffs(const Plan& a1, const Plan& b1) {
  int64_t diff = 0;
#define BEMB200_CMP(f) diff += (a1.f == b1.f) ? 0 : 1;
  BEMB200_CMP(Xs) BEMB200_CMP(L) BEMB200_CMP(scale) BEMB200_CMP(near_region) BEMB200_CMP(face_of_pos) BEMB200_CMP(pos_of_face)
  BEMB200_CMP(owner_of_pos) BEMB200_CMP(e_q) BEMB200_CMP(e_W) BEMB200_CMP(e_n) BEMB200_CMP(e_dof) BEMB200_CMP(e_vtx)
  BEMB200_CMP(e_near) BEMB200_CMP(node_children) BEMB200_CMP(level_nodes) BEMB200_CMP(leaves) BEMB200_CMP(m2l_off)
  BEMB200_CMP(m2l_src) BEMB200_CMP(near_off) BEMB200_CMP(near_nodes) BEMB200_CMP(m2l_pairs) BEMB200_CMP(near_pairs)
  BEMB200_CMP(grp_vec) BEMB200_CMP(grp_off) BEMB200_CMP(grp_pair) BEMB200_CMP(chunk_grp) BEMB200_CMP(chunk_begin)
  BEMB200_CMP(chunk_cnt) BEMB200_CMP(m2l_targets) BEMB200_CMP(m2l_key_sorted) BEMB200_CMP(tc_tab) BEMB200_CMP(tc_pair)
  BEMB200_CMP(tc_item_tab) BEMB200_CMP(tc_item_begin) BEMB200_CMP(tc_item_cnt) BEMB200_CMP(target_box) BEMB200_CMP(nb_dofs)
  BEMB200_CMP(nb_targets) BEMB200_CMP(nb_ranges) BEMB200_CMP(block_of_point) BEMB200_CMP(row_of_point) BEMB200_CMP(self_col)
  BEMB200_CMP(nnz) BEMB200_CMP(dof_inc_off) BEMB200_CMP(dof_inc)
#undef BEMB200_CMP
  diff += a1.nodes.size() != b1.nodes.size() || a1.blocks.size() != b1.blocks.size();
  for (size_t i = 0; i < a1.nodes.size() && i < b1.nodes.size(); ++i)
    diff += std::memcmp(&a1.nodes[i], &b1.nodes[i], sizeof(Plan::Node)) != 0;
  for (size_t i = 0; i < a1.blocks.size() && i < b1.blocks.size(); ++i) {
    const auto &x = a1.blocks[i], &y = b1.blocks[i];
    diff += x.node != y.node || x.w_off != y.w_off || x.dof_off != y.dof_off || x.ndof != y.ndof || x.tgt_off != y.tgt_off ||
            x.ntgt != y.ntgt || x.rng_off != y.rng_off || x.nrng != y.nrng;
  }
  return diff;
}

int bem_plan_refresh_inspect(const bem_gpu_opts* opts, const bem_bvp_desc* d0, const bem_bvp_desc* d1, int64_t* out) {
  if (!opts || !d0 || !d1 || !out) return BEM_ERR_INVALID_ARGUMENT;
  PlanOptions po;
  po.p = opts->expansion_order;
  po.theta = opts->mac_theta;
  po.leaf_max = opts->leaf_max_elements;
  po.max_level = opts->max_level;
  auto build = [&](Plan& P, const bem_bvp_desc* d, Plan* prev, bool take) {
    PlanOptions o = po;
    o.take_structure = take;
    if (!build_plan(P, o, d->n_points, d->X, d->n_faces, d->tri, d->face_dirichlet, d->n_dof, d->dof_point, d->dof_face, d->dof_kind,
                    d->face_dof, prev))
      return false;
    if (!P.reused_m2l) build_tc_groups(P, 80);
    return true;
  };
  Plan a0, b0, a1, b1;
  if (!build(a0, d0, nullptr, true) || !build(b0, d0, nullptr, true)) return BEM_ERR_INVALID_ARGUMENT;
  if (!build(a1, d1, &a0, true) || !build(b1, d1, &b0, false)) return BEM_ERR_INVALID_ARGUMENT;
  const int64_t diff = plan_diffs(a1, b1);
  bool same_root = true;
  for (int k = 0; k < 3; ++k) same_root = same_root && a1.root_C[k] == a0.root_C[k];
  out[0] = same_root && a1.root_R == a0.root_R;
  out[1] = (int)a1.reused_m2l + (int)a1.reused_near;
  out[2] = diff;
  return BEM_OK;
}

int bem_plan_inspect(const bem_gpu_opts* opts, const bem_bvp_desc* d, int32_t* face_level, double* face_corner, int64_t* stats) {
  if (!opts || !d) return BEM_ERR_INVALID_ARGUMENT;
  PlanOptions po;
  po.p = opts->expansion_order;
  po.theta = opts->mac_theta;
  po.leaf_max = opts->leaf_max_elements;
  po.max_level = opts->max_level;
  Plan P;
  if (!build_plan(P, po, d->n_points, d->X, d->n_faces, d->tri, d->face_dirichlet, d->n_dof, d->dof_point, d->dof_face, d->dof_kind,
                  d->face_dof))
    return BEM_ERR_INVALID_ARGUMENT;
  if (face_level && face_corner)
    for (int f = 0; f < P.nf; ++f) {
      face_level[f] = -1;
      face_corner[3 * f] = face_corner[3 * f + 1] = face_corner[3 * f + 2] = 0.0;
      const int s = P.pos_of_face[f];
      if (s < 0) continue;
      const int o = P.owner_of_pos[s];
      if (o < 0 || P.nodes[o].child_end > P.nodes[o].child_begin) continue;
      face_level[f] = P.nodes[o].level;
      for (int a = 0; a < 3; ++a) face_corner[3 * f + a] = P.nodes[o].lo[a];
    }
  if (stats) {
    int64_t nodes = 0;
    int depth = 0;
    for (size_t l = 0; l < P.level_nodes.size(); ++l) {
      nodes += (int64_t)P.level_nodes[l].size();
      if (!P.level_nodes[l].empty()) depth = (int)l;
    }
    stats[0] = nodes;
    stats[1] = (int64_t)P.leaves.size();
    stats[2] = depth;
    stats[3] = P.n_added;
    stats[4] = P.m2l_pairs;
    stats[5] = P.near_pairs;
    stats[6] = P.nnz;
    stats[7] = (int64_t)P.blocks.size();
    stats[8] = (int64_t)P.chunk_grp.size();
    stats[9] = (int64_t)P.grp_off.size() - 1;
  }
  return BEM_OK;
}

// GMRES with the reference's driver logic (run_gmres, BEM_solveBVP_GMRES_FMM.hpp:2275-2355):
// single Arnoldi cycle with incremental Givens QR; once the estimate is within 10*tol the
// true residual is checked every step; six failed checks end the cycle and GMRES restarts
// from the current iterate.  Orthogonalisation is classical Gram-Schmidt applied twice
// (the reference uses one pass of modified Gram-Schmidt; both are FP64-stable here).
int bem_gpu_solve(bem_gpu_ctx* ctx, const double* known, const double* x0, double* out_phi, double* out_phin, bem_gpu_stats* stats) {
  if (!ctx || !known || !out_phi || !out_phin) return BEM_ERR_INVALID_ARGUMENT;
  if (!ctx->ready) return BEM_ERR_NOT_READY;
  CK(cudaSetDevice(ctx->opts.device));
  const double t0 = now_s();
  const Plan& P = ctx->plan;
  const int N = P.ndof;
  cudaStream_t s = ctx->stream;
  ctx->h2d = ctx->setup_h2d;
  ctx->d2h = 0;
  ctx->launches = ctx->setup_launches;
  // preconditioner: 2 falls back to the Jacobi scaling when the set-up formed no polynomial
  const int prec = (ctx->opts.preconditioner == 2 && ctx->poly.n == 0) ? 1 : ctx->opts.preconditioner;
  const bool jacobi = prec == 1;
  double tol = ctx->opts.tol;
  const int max_iter = ctx->opts.max_iter;
  for (int i = 0; i < N; ++i)
    if (!std::isfinite(known[i])) {
      ctx->err = "non-finite boundary value";
      return BEM_ERR_NAN;
    }
  // known values in scaled units (copyToFMM: Neumann phin x L)
  std::vector<double> ks(N);
  for (int i = 0; i < N; ++i) ks[i] = (P.dof_kind[i] == 0) ? known[i] : known[i] * P.L;
  CK(cudaMemcpyAsync(ctx->known_s.p, ks.data(), sizeof(double) * N, cudaMemcpyHostToDevice, s));
  ctx->h2d += 8LL * N;
  CK(cudaEventRecord(ctx->ev[2], s));
  const int cols = max_iter + 2;
  if (ctx->V_cols < cols || ctx->V.n < (size_t)cols * N || (prec == 2 && ctx->Z.n < (size_t)cols * N)) {
    CK(ctx->V.alloc((size_t)cols * N));
    if (prec == 2) CK(ctx->Z.alloc((size_t)cols * N));
    ctx->V_cols = cols;
  }
  if (ctx->w.n < (size_t)N) {
    CK(ctx->w.alloc(N));
    CK(ctx->xdev.alloc(N));
    CK(ctx->bdev.alloc(N));
    CK(ctx->rdev.alloc(N));
    CK(ctx->tmp.alloc(N));
  }
  CK(ctx->hdev.alloc((size_t)3 * cols + 8));
  CK(ctx->ydev.alloc(cols));
  CK(ctx->partial.alloc((size_t)std::max(mdot_blocks(N), arnoldi_dot_blocks(N)) * cols));
  int matvecs = 0;
  // b = -(A*0 - b) with corner rows replaced by the point's phi (:2025-2047)
  launch_densities(N, 1, nullptr, ctx->known_s.p, ctx->dof_kind.p, ctx->phi.p, ctx->phin.p, s);
  run_fmm(ctx, ctx->rows.p, nullptr, nullptr);
  ctx->launches += 1;
  ++matvecs;
  std::vector<double> b(N);
  CK(cudaMemcpyAsync(b.data(), ctx->rows.p, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
  ctx->d2h += 8LL * N;
  CK(cudaStreamSynchronize(s));
  for (int i = 0; i < N; ++i) {
    b[i] = -b[i];
    if (P.dof_kind[i] == 2) b[i] = (P.corner_src_dof[i] >= 0) ? known[P.corner_src_dof[i]] : 0.0;
  }
  CK(cudaMemcpyAsync(ctx->bdev.p, b.data(), sizeof(double) * N, cudaMemcpyHostToDevice, s));
  ctx->h2d += 8LL * N;
  double bn = 0.0;
  for (int i = 0; i < N; ++i) bn = std::fma(b[i], b[i], bn);
  const double rhs_norm = std::sqrt(bn);
  if (ctx->opts.tol_relative) tol *= rhs_norm;
  std::vector<double> x0s;
  if (x0) {  // initial guess in physical units (phin for Dirichlet DOFs, phi otherwise) -> scaled
    x0s.resize(N);
    for (int i = 0; i < N; ++i) {
      if (!std::isfinite(x0[i])) {
        ctx->err = "non-finite initial guess";
        return BEM_ERR_NAN;
      }
      x0s[i] = (P.dof_kind[i] == 0) ? x0[i] * P.L : x0[i];
    }
    CK(cudaMemcpyAsync(ctx->xdev.p, x0s.data(), sizeof(double) * N, cudaMemcpyHostToDevice, s));
    ctx->h2d += 8LL * N;
  } else
    CK(cudaMemsetAsync(ctx->xdev.p, 0, sizeof(double) * N, s));

  auto matvec = [&](const double* din, double* dout) -> int {
    ++matvecs;
    ctx->launches += ctx->graph_kernels;
    return bem_gpu_matvec_device(ctx, din, dout);
  };
  const bool mixed = ctx->mixed;
  int matvecs_lo = 0;
  // Mixed precision is iterative refinement: each GMRES cycle solves A_lo d = r to
  // max(tol, kInnerRtol |r|) and the cycle ends with the FP64 true residual, from which the
  // next cycle starts (that residual is reused, not recomputed).
  const double kInnerRtol = ctx->opts.refine_rtol > 0.0 ? ctx->opts.refine_rtol : 1e-6;
  bool have_res = false;
  auto norm_of = [&](const double* v, double* out) -> int {
    launch_mdot(v, N, 1, v, N, ctx->partial.p, ctx->hdev.p, s);
    ctx->launches += 2;
    ctx->d2h += 8;
    CK(cudaMemcpyAsync(out, ctx->hdev.p, sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    *out = std::sqrt(*out);
    return BEM_OK;
  };
  int iters = 0, rc = BEM_OK;
  double r_true = 1e300, err = 1e300;
  bool x_zero = (x0 == nullptr);
  // Arnoldi steps run as one graph each (operator + orthogonalisation + Givens update, all
  // state on the device); the host reads each step's residual estimate kLag steps behind.
  if ((rc = ensure_arnoldi_graph(ctx, prec, mixed, cols)) != BEM_OK) return rc;
  constexpr int kLag = 3;
  auto x_update = [&]() -> int {  // x = x_base + M V R^{-1} g over the cycle's steps (M V = Z stored)
    CK(cudaMemcpyAsync(ctx->xdev.p, ctx->xbase.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
    launch_arnoldi_solve_y(ctx->arn_state.p, ctx->arn_R.p, cols, ctx->arn_g.p, ctx->ydev.p, s);
    if (prec == 2) {
      launch_arnoldi_update(ctx->Z.p, N, cols, ctx->arn_state.p, ctx->ydev.p, ctx->xdev.p, s);
      ctx->launches += 2;
    } else if (prec == 3) {  // x += M^{-1} (V R^{-1} g)
      CK(cudaMemsetAsync(ctx->tmp.p, 0, sizeof(double) * N, s));
      launch_arnoldi_update(ctx->V.p, N, cols, ctx->arn_state.p, ctx->ydev.p, ctx->tmp.p, s);
      launch_bj_apply(ctx->bj_args(), ctx->tmp.p, N, nullptr, ctx->bj_tmp.p, s);
      launch_axpby(N, 1.0, ctx->bj_tmp.p, 1.0, ctx->xdev.p, s);
      ctx->launches += 4;
    } else if (!jacobi) {
      launch_arnoldi_update(ctx->V.p, N, cols, ctx->arn_state.p, ctx->ydev.p, ctx->xdev.p, s);
      ctx->launches += 2;
    } else {
      CK(cudaMemsetAsync(ctx->tmp.p, 0, sizeof(double) * N, s));
      launch_arnoldi_update(ctx->V.p, N, cols, ctx->arn_state.p, ctx->ydev.p, ctx->tmp.p, s);
      launch_add_mul(N, ctx->xdev.p, ctx->dinv.p, ctx->tmp.p, ctx->xdev.p, s);
      ctx->launches += 3;
    }
    return BEM_OK;
  };
  auto true_res = [&](double* out) -> int {
    int r;
    if ((r = matvec(ctx->xdev.p, ctx->rdev.p)) != BEM_OK) return r;
    launch_axpby(N, -1.0, ctx->bdev.p, 1.0, ctx->rdev.p, s);
    ctx->launches += 1;
    return norm_of(ctx->rdev.p, out);
  };
  while (iters < max_iter && r_true > tol) {
    double beta = 0.0;
    if (have_res) {  // rdev = A x - b from the true-residual check that ended the last cycle
      launch_axpby(N, 0.0, ctx->bdev.p, -1.0, ctx->rdev.p, s);
      ctx->launches += 1;
      beta = r_true;
      have_res = false;
    } else if (x_zero) {  // r0 = b for the zero start: no operator application
      CK(cudaMemcpyAsync(ctx->rdev.p, ctx->bdev.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
      if ((rc = norm_of(ctx->rdev.p, &beta)) != BEM_OK) return rc;
    } else {
      // r0 = b - A x
      if ((rc = matvec(ctx->xdev.p, ctx->rdev.p)) != BEM_OK) return rc;
      launch_axpby(N, 1.0, ctx->bdev.p, -1.0, ctx->rdev.p, s);  // r = b - r
      ctx->launches += 1;
      if ((rc = norm_of(ctx->rdev.p, &beta)) != BEM_OK) return rc;
    }
    if (!std::isfinite(beta)) {
      ctx->err = "non-finite residual";
      return BEM_ERR_NAN;
    }
    if (beta <= tol) {  // the iterate (a good initial guess, or zero data) already meets the tolerance
      r_true = beta;
      err = beta;
      break;
    }
    x_zero = false;
    launch_axpby(N, 1.0 / beta, ctx->rdev.p, 0.0, ctx->V.p, s);
    launch_arnoldi_init(ctx->arn_state.p, ctx->arn_g.p, beta, s);
    launch_arnoldi_prep(N, ctx->V.p, (prec == 1 || prec == 2) ? ctx->dinv.p : nullptr, ctx->arn_state.p, ctx->mv_in.p, s);
    // x_base: the iterate this cycle's corrections start from
    CK(cudaMemcpyAsync(ctx->xbase.p, ctx->xdev.p, sizeof(double) * N, cudaMemcpyDeviceToDevice, s));
    ctx->launches += 3;
    const int cycle_cap = std::min(cols - 2, max_iter - iters);  // steps this cycle may take
    const double check_at = mixed ? std::max(tol, kInnerRtol * beta) : tol * 10.;
    int launched = 0, done = 0, sat = 0;
    auto launch_step = [&]() -> int {
      CK(cudaGraphLaunch(ctx->arn_exec, s));
      const int slot = launched % kErrRing;
      CK(cudaMemcpyAsync(ctx->arn_err_host + slot, &ctx->arn_state.p->err, sizeof(double), cudaMemcpyDeviceToHost, s));
      CK(cudaEventRecord(ctx->arn_ev[slot], s));
      ctx->launches += ctx->arn_kernels;
      ctx->d2h += 8;
      ++launched;
      if (mixed)
        ++matvecs_lo;
      else
        ++matvecs;
      return BEM_OK;
    };
    auto drain = [&]() -> int {  // all launched steps finished; err of the last one
      CK(cudaStreamSynchronize(s));
      err = ctx->arn_err_host[(launched - 1) % kErrRing];
      iters += launched - done;
      done = launched;
      return BEM_OK;
    };
    while (true) {
      while (launched - done < kLag && launched < cycle_cap)
        if ((rc = launch_step()) != BEM_OK) return rc;
      CK(cudaEventSynchronize(ctx->arn_ev[done % kErrRing]));
      err = ctx->arn_err_host[done % kErrRing];
      ++done;
      ++iters;
      if (!std::isfinite(err)) {
        ctx->err = "non-finite Arnoldi vector";
        return BEM_ERR_NAN;
      }
      if (done > 1 && err <= check_at) {
        if ((rc = drain()) != BEM_OK) return rc;
        if ((rc = x_update()) != BEM_OK) return rc;
        if ((rc = true_res(&r_true)) != BEM_OK) return rc;
        if (r_true <= tol) break;
        if (mixed) {  // refine: next cycle from this residual
          have_res = true;
          break;
        }
        if (sat++ >= 5) break;
        if (launched >= cycle_cap) break;
        // the check's operator application overwrote the next step's input: write it again
        launch_arnoldi_prep(N, ctx->V.p, (prec == 1 || prec == 2) ? ctx->dinv.p : nullptr, ctx->arn_state.p, ctx->mv_in.p, s);
        ctx->launches += 1;
        continue;
      }
      if (done >= cycle_cap) {  // basis full or iteration cap: finish the cycle at this iterate
        if ((rc = drain()) != BEM_OK) return rc;
        if ((rc = x_update()) != BEM_OK) return rc;
        if (err <= tol * 10.) {
          if ((rc = true_res(&r_true)) != BEM_OK) return rc;
        } else
          r_true = err;
        break;
      }
    }
  }
  CK(cudaEventRecord(ctx->ev[3], s));
  if ((rc = bem_gpu_check_device_status(ctx)) != BEM_OK) return rc;
  std::vector<double> x(N);
  CK(cudaMemcpyAsync(x.data(), ctx->xdev.p, sizeof(double) * N, cudaMemcpyDeviceToHost, s));
  ctx->d2h += 8LL * N;
  CK(cudaStreamSynchronize(s));
  float solve_dev_ms = 0.f;
  CK(cudaEventElapsedTime(&solve_dev_ms, ctx->ev[2], ctx->ev[3]));
  bool finite = true;
  for (int i = 0; i < N; ++i) {
    finite = finite && std::isfinite(x[i]);
    if (P.dof_kind[i] == 0) {  // unscale phin (BEM_solveBVP_GMRES_FMM.hpp:3462-3486)
      out_phi[i] = known[i];
      out_phin[i] = x[i] / P.L;
    } else {
      out_phi[i] = x[i];
      out_phin[i] = known[i];
    }
  }
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->iterations = iters;
    stats->converged = r_true <= tol;
    stats->residual = r_true;
    stats->residual_est = err;
    stats->time_setup_s = ctx->time_setup;
    stats->time_solve_s = now_s() - t0;
    stats->nnz_near = P.nnz;
    stats->m2l_pairs = P.m2l_pairs;
    int64_t nodes = 0;
    for (auto& lv : P.level_nodes) nodes += (int64_t)lv.size();
    stats->n_nodes = (int)nodes;
    stats->n_leaves = (int)P.leaves.size();
    stats->matvecs = matvecs;
    stats->matvecs_lo = matvecs_lo;
    stats->time_device_s = 1e-3 * ((double)ctx->setup_dev_ms + (double)solve_dev_ms);
    stats->h2d_bytes = ctx->h2d;
    stats->d2h_bytes = ctx->d2h;
    stats->kernel_launches = ctx->launches;
    stats->time_plan_s = ctx->time_plan;
    stats->time_upload_s = ctx->time_upload;
    stats->time_setup_device_s = 1e-3 * (double)ctx->setup_dev_ms;
    stats->rhs_norm = rhs_norm;
    stats->tol_abs = tol;
  }
  if (!finite) {
    ctx->err = "non-finite solution";
    return BEM_ERR_NAN;
  }
  return (r_true <= tol) ? BEM_OK : BEM_ERR_NOT_CONVERGED;
}

int bem_gpu_solve_bvp(bem_gpu_ctx* ctx, const bem_bvp_desc* desc, const double* known, const double* x0, double* out_phi, double* out_phin,
                      bem_gpu_stats* stats) {
  int rc = bem_gpu_setup(ctx, desc);
  if (rc != BEM_OK) return rc;
  return bem_gpu_solve(ctx, known, x0, out_phi, out_phin, stats);
}

namespace {
int profile_matvec(bem_gpu_ctx* ctx, int repeats, bool tc, double* stage_ms) {
  CK(cudaSetDevice(ctx->opts.device));
  cudaStream_t s = ctx->stream;
  const int N = ctx->plan.ndof;
  // representative input: unit unknowns
  std::vector<double> one(N, 1.0);
  CK(cudaMemcpyAsync(ctx->mv_in.p, one.data(), sizeof(double) * N, cudaMemcpyHostToDevice, s));
  launch_densities(N, 0, ctx->mv_in.p, nullptr, ctx->dof_kind.p, ctx->phi.p, ctx->phin.p, s);
  run_fmm(ctx, ctx->mv_out.p, nullptr, nullptr);
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const int stages[5] = {STAGE_P2M, STAGE_M2M, STAGE_M2L, STAGE_L2L, STAGE_TARGETS};
  MatvecArgs a = ctx->args(ctx->phi.p, ctx->phin.p, ctx->mv_out.p, nullptr, nullptr);
  ctx->set_ax(a, tc);
  if (tc) ctx->set_tc(a);
  for (int k = 0; k < 6; ++k) {
    CK(cudaEventRecord(e0, s));
    for (int r = 0; r < repeats; ++r) {
      if (k < 5)
        launch_matvec(ctx->plan.opt.p, a, s, stages[k]);
      else
        CK(cudaGraphLaunch(tc ? ctx->graph_exec_lo : ctx->graph_exec, s));
    }
    CK(cudaEventRecord(e1, s));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    stage_ms[k] = ms / repeats;
  }
  if (tc) {  // the three kernels of the tensor-core M2L on their own
    const int parts[3] = {TC_EXPAND, TC_CONTRACT, TC_REDUCE};
    for (int k = 0; k < 3; ++k) {
      CK(cudaEventRecord(e0, s));
      for (int r = 0; r < repeats; ++r) launch_m2l_tc(ctx->plan.opt.p, a, s, parts[k], 1);
      CK(cudaEventRecord(e1, s));
      CK(cudaEventSynchronize(e1));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      stage_ms[6 + k] = ms / repeats;
    }
    CK(cudaEventRecord(e0, s));
    for (int r = 0; r < repeats; ++r) launch_near_sums(a, s);
    CK(cudaEventRecord(e1, s));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    stage_ms[9] = ms / repeats;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return BEM_OK;
}
}  // namespace

int bem_gpu_profile_matvec(bem_gpu_ctx* ctx, int repeats, double* stage_ms) {
  if (!ctx || !stage_ms || repeats < 1) return BEM_ERR_INVALID_ARGUMENT;
  if (!ctx->ready) return BEM_ERR_NOT_READY;
  return profile_matvec(ctx, repeats, false, stage_ms);
}

int bem_gpu_profile_matvec_mixed(bem_gpu_ctx* ctx, int repeats, double* stage_ms) {
  if (!ctx || !stage_ms || repeats < 1) return BEM_ERR_INVALID_ARGUMENT;
  if (!ctx->ready) return BEM_ERR_NOT_READY;
  if (!ctx->mixed) {
    ctx->err = "context was not set up with precision = 1";
    return BEM_ERR_UNSUPPORTED;
  }
  return profile_matvec(ctx, repeats, true, stage_ms);
}

int bem_gpu_matvec_device_mixed(bem_gpu_ctx* ctx, const double* d_x, double* d_y) {
  if (!ctx || !d_x || !d_y) return BEM_ERR_INVALID_ARGUMENT;
  if (!ctx->ready) return BEM_ERR_NOT_READY;
  if (!ctx->mixed) {
    ctx->err = "context was not set up with precision = 1";
    return BEM_ERR_UNSUPPORTED;
  }
  return matvec_lo(ctx, d_x, d_y);
}

int bem_gpu_set_wait_limit(bem_gpu_ctx* ctx, int64_t tries) {
  if (!ctx) return BEM_ERR_INVALID_ARGUMENT;
  ctx->tc_wait_tries = tries < 0 ? tc_default_wait_tries() : (uint32_t)std::min<int64_t>(tries, 0xffffffffLL);
  if (!ctx->ready) return BEM_OK;
  CK(cudaSetDevice(ctx->opts.device));
  CK(cudaStreamSynchronize(ctx->stream));
  if (ctx->mixed) CK(cudaMemsetAsync(ctx->tc_err.p, 0, sizeof(int), ctx->stream));
  // the limit is a kernel argument: recapture the operator graphs that launch the contraction
  return build_graph(ctx);
}

int bem_gpu_check_device_status(bem_gpu_ctx* ctx) {
  if (!ctx) return BEM_ERR_INVALID_ARGUMENT;
  if (!ctx->ready) return BEM_OK;
  if (!ctx->mixed) return BEM_OK;  // only the tensor-core M2L waits on the device
  int flag = 0;
  CK(cudaMemcpyAsync(&flag, ctx->tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  CK(cudaStreamSynchronize(ctx->stream));
  if (flag) {
    ctx->err = "tensor-core M2L: a bounded wait on the MMA completion gave up";
    return BEM_ERR_DEVICE;
  }
  return BEM_OK;
}

// ---- mat-vec that allocates nothing ------------------------------------------------
// The M2L stage writes one translated expansion per (target, source) pair into a slot
// buffer and then sums each target's slots in a fixed order.  This entry point takes that
// slot buffer from a file-scope device array instead of the context.  The array is part of
// this library's device image: the driver reserves it on each device when the module is
// loaded, so no call ever allocates for it.  Callers that must not allocate device memory
// while they apply the operator (a time integrator or outer solver running out of a fixed
// device-memory reservation, a server holding many small problems on one device that wants
// one shared slot area rather than one per problem) use this entry point.
int bem_gpu_matvec_device_noalloc(bem_gpu_ctx* ctx, const double* d_x, double* d_y) {
  if (!ctx || !d_x || !d_y) return BEM_ERR_INVALID_ARGUMENT;
  if (!ctx->ready) return BEM_ERR_NOT_READY;
  const Plan& P = ctx->plan;
  const size_t need = (size_t)P.m2l_pairs * 2 * ncoef(P.opt.p) * sizeof(double2);
  if (need > kNoAllocSlotBytes) {
    ctx->err = "no-alloc mat-vec: M2L slot scratch of " + std::to_string(need) + " bytes (" + std::to_string(P.m2l_pairs) +
               " pairs at order " + std::to_string(P.opt.p) + ") exceeds the fixed " + std::to_string(kNoAllocSlotBytes) + " bytes";
    return BEM_ERR_UNSUPPORTED;
  }
  if (!ctx->noalloc_slots) {
    ctx->err = std::string("no-alloc mat-vec: the slot area's device address could not be looked up at set-up: ") +
               cudaGetErrorString(ctx->noalloc_lookup);
    return BEM_ERR_DEVICE;
  }
  int prev_dev = -1;
  CK(cudaGetDevice(&prev_dev));
  const int dev = ctx->opts.device;
  if (dev != prev_dev) CK(cudaSetDevice(dev));
  // every slot of the m2l_pairs in use is overwritten before the reduction reads it, so the
  // area needs no clearing; the local expansions L are zeroed inside the launch sequence as
  // on the graph path.  One area per device: calls that may overlap on one device (other
  // streams, other threads, other contexts) race on it and must be ordered by the caller.
  // The FP64 operator, also on a mixed-precision context.
  MatvecArgs a = ctx->args(ctx->phi.p, ctx->phin.p, d_y, nullptr, nullptr);
  a.Y = static_cast<double2*>(ctx->noalloc_slots);
  launch_densities(P.ndof, 0, d_x, nullptr, ctx->dof_kind.p, ctx->phi.p, ctx->phin.p, ctx->stream);
  ctx->launches += 1 + launch_matvec(P.opt.p, a, ctx->stream);
  const cudaError_t e = cudaGetLastError();
  if (dev != prev_dev) cudaSetDevice(prev_dev);
  if (e != cudaSuccess) {
    ctx->err = std::string("no-alloc mat-vec: ") + cudaGetErrorString(e);
    return BEM_ERR_DEVICE;
  }
  return BEM_OK;
}

double bem_gpu_fp64_peak_tflops(int32_t device) {
  if (cudaSetDevice(device) != cudaSuccess) return 0.0;
  cudaStream_t s;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return 0.0;
  double* sink = nullptr;
  if (cudaMalloc(&sink, sizeof(double)) != cudaSuccess) return 0.0;
  const double tf = fp64_probe_tflops(s, sink);
  cudaStreamSynchronize(s);
  cudaFree(sink);
  cudaStreamDestroy(s);
  return tf;
}

}  // extern "C"
