// Launch interface of the FMM / near-field / Krylov kernels (kernels.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include <utility>

#include "poly.hpp"

namespace bemb200 {

// devices tracked by the per-device launch bookkeeping (shared-memory permissions)
constexpr int kMaxDevices = 64;

// Programmatic dependent launch for the kernels of an operator application: each is launched
// with programmatic stream serialisation and starts with pdl_enter(), which waits until the
// previous kernel in the stream has completed and its writes are visible, then lets the next
// kernel's blocks be scheduled while this one runs.  The chain stays ordered (every kernel
// waits for its predecessor before touching memory); only the launch latency between
// consecutive kernels is hidden.  Kernels launched this way must call pdl_enter() first.
#ifdef __CUDACC__
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
#endif
// BEMB200_NO_PDL=1 in the environment launches the same kernels without the programmatic
// serialisation attribute (plain stream order; for tools that do not follow dependent launches)
bool pdl_enabled();

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

struct NearBlockDev {
  int64_t w_off;   // first weight of this block's rows
  int64_t w4_off;  // same in the FP32 copy, whose rows are padded to a multiple of 4 columns
  int node;       // deepest bucket shared by the block's targets
  int dof_off, ndof;
  int tgt_off, ntgt;
  int rng_off, nrng;
};

struct MatvecArgs {
  int n_nodes = 0, n_levels = 0;  // n_levels: tree levels (rows of the per-level lists below)
  // P2M
  int n_leaves = 0;
  const int* leaves = nullptr;
  const int* node_fb = nullptr;
  const int* node_fe = nullptr;
  const double* node_X = nullptr;
  const double* e_q = nullptr;
  const double* e_W = nullptr;
  const double* e_n = nullptr;
  const int* e_dof = nullptr;
  // tree passes
  const int* child_begin = nullptr;
  const int* child_end = nullptr;
  const int* node_children = nullptr;
  const double2* Ftab = nullptr;           // [level][octant][(P+1)^2] parent-to-child F tables
  // upward pass, one launch per level: the level's nodes that build or hand up a multipole
  const int* m2m_level_off = nullptr;      // host [n_levels+1] into m2m_nodes
  const int* m2m_nodes = nullptr;          // device
  const int* node_up = nullptr;            // [n_nodes] parent whose multipole is needed, else -1
  double2* Yup = nullptr;                  // [n_nodes][2][NC] multipoles shifted to the parent's centre
  const int* m2m_level_off_nl = nullptr;   // host [n_levels+1]: the same lists without the leaves
  const int* m2m_nodes_nl = nullptr;       // device
  const int* leaf_level = nullptr;         // [n_leaves] level of each leaf (A.x: k_p2m_leaf shifts the leaves)
  // downward pass, one launch per parent level: (parent, child) pairs of parents with a local expansion
  const int* l2l_level_off = nullptr;      // host [n_levels+1] into l2l_pairs
  const int2* l2l_pairs = nullptr;         // device

  int n_m2l_targets = 0;
  const int* m2l_targets = nullptr;
  const int* m2l_off = nullptr;
  const int* m2l_src = nullptr;
  int n_chunks = 0;
  const int* chunk_grp = nullptr;
  const int* chunk_begin = nullptr;
  const int* chunk_cnt = nullptr;
  const int* grp_pair = nullptr;
  const double2* Sg = nullptr;  // per-group S tables
  double2* Y = nullptr;         // per-pair partial locals
  double2* M = nullptr;
  double2* L = nullptr;
  // tensor-core M2L (mixed precision); used instead of the FP64 M2L when use_tc != 0
  int use_tc = 0;
  int n_tc_items = 0, tc_grid = 0;
  const int* tc_item_tab = nullptr;
  const int* tc_item_begin = nullptr;
  const int* tc_item_cnt = nullptr;
  int n_tc_pairs = 0;
  int tc_item_pairs = 80;  // largest item (selects the tensor-core kernel variant)
  // overlap of the near field with the FMM passes (low-precision A.x): a second stream and the
  // two events that fork it from and join it to the launching stream; null: one stream
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  const int* tc_pos = nullptr;   // [pairs] position of pair slot k in work-item order
  const int* tc_src = nullptr;   // [pairs] source bucket, in work-item order
  const void* tc_tab = nullptr;  // FP16 hi/lo table images
  void* tc_Mt = nullptr;         // FP16 hi/lo rows of M[0] - M[1] [n_nodes+1][2][KP]
  float* tc_escale = nullptr;    // [n_nodes] power-of-two column scales
  float* tc_Y = nullptr;         // per-pair partial locals [pairs][KPO], in work-item order
  // fused reduction (tc_acc set): the contraction adds each pair into its target's FP32
  // accumulator [n_m2l_targets][KPO] in L2 instead of writing partials; a finalize kernel
  // converts and clears them (summation order varies between runs)
  const int* tc_tgt = nullptr;   // [pairs] compact target index (into m2l_targets), in work-item order
  float* tc_acc = nullptr;
  int* tc_err = nullptr;         // set when a bounded wait gave up
  uint32_t tc_wait_tries = 0;    // iteration limit of the contraction's pipeline waits
  const double* node_dL = nullptr;
  const double* tc_alpha = nullptr;  // [KP] sqrt((n+m)!(n-m)!) per real coefficient
  const void* tc_rows_map = nullptr; // host copy of the TMA tensor map over tc_Mt
  // targets
  int n_blocks = 0, chunk = 0, max_ntgt = 0;
  double* near_sum = nullptr;  // [targets] near sums of A.x by target slot (blocks' tgt_off order)
  // per near block, its bucket and the bucket's ancestors that are M2L targets, deepest first
  // (the A.x rows sum their L2Ps instead of a downward pass)
  int max_path = 0;                   // longest path
  const int* blk_path_off = nullptr;  // [n_blocks + 1]
  const int* blk_path = nullptr;
  const NearBlockDev* blocks = nullptr;
  const int* nb_dofs = nullptr;
  const int* nb_targets = nullptr;
  const double* WG = nullptr;
  const double* WGn = nullptr;
  const double* Xs = nullptr;
  const int* point_dof_off = nullptr;
  const int* point_dof = nullptr;
  const int* dof_kind = nullptr;
  const double* diag = nullptr;
  // state
  const double* phi = nullptr;
  const double* phin = nullptr;
  double* rows = nullptr;   // may be null
  double* GPhin = nullptr;  // may be null
  double* GnPhi = nullptr;
  // A.x application (rows only): unknown vector and combined near weights (either precision)
  const double* ax = nullptr;
  const double* Wc = nullptr;
  const float* Wc32 = nullptr;
  // P2M operator of A.x: per leaf, the DOFs of its elements (CSR over leaf index) and the
  // multipole column of each (leaf, DOF)
  const int* leaf_dof_off = nullptr;
  const int* leaf_dof = nullptr;
  double2* p2m_C = nullptr;
  const float2* p2m_C32 = nullptr;  // FP32 copy of the P2M operator (low-precision A.x), or null
};

struct NearArgs {
  int n_blocks = 0;
  int n_slots = 0;                  // targets over all blocks (rows of the weight arrays)
  int* next_block = nullptr;        // device counter of the blocks taken (zeroed at launch)
  int max_nrng = 0;                 // most element ranges of one block
  double2* scratch = nullptr;       // near_weights_grid() rows of 3 x scratch_stride/3 element values
  int64_t scratch_stride = 0;       // >= 3 x most near elements of one block
  const NearBlockDev* blocks = nullptr;
  const int* nb_dofs = nullptr;
  const int* nb_targets = nullptr;
  const int* nb_ranges = nullptr;
  const int* dof_inc_off = nullptr;
  const int* dof_inc = nullptr;
  const double* Xs = nullptr;
  const int* e_vtx = nullptr;
  const double* e_near = nullptr;
  double near_region = 0.0;
  double* WG = nullptr;
  double* WGn = nullptr;
};

int near_weights_grid();  // CTAs of the near-weight kernel (one scratch row each)
void upload_quadrature(const double dv[6][4], const double gw[25][3], cudaStream_t s);
void configure_targets_smem(int p, int bytes);
int configure_target_rows_smem(int p, int max_path, int max_ntgt);  // -1: does not fit an SM
void configure_m2l_smem(int p);
void launch_s_tables(int p, int ngroups, const double* gvec, double2* Sg, cudaStream_t st);
// F(child - parent) per (level, octant) from one representative offset each: vec [ntab][3]
void launch_f_tables(int p, int ntab, const double* vec, double2* Ftab, cudaStream_t st);
enum { STAGE_P2M = 1, STAGE_M2M = 2, STAGE_M2L = 4, STAGE_L2L = 8, STAGE_TARGETS = 16, STAGE_ALL = 31 };
// returns the number of kernels launched
// One operator application; returns the number of kernel launches.  A call that asks for
// GPhin carries both densities through the tree; any other call carries their difference
// only (half the P2M, M2M, M2L, L2L and L2P work) -- a call for GnPhi alone must then have
// phin = 0 (the rigid-mode diagonal).
int launch_matvec(int p, const MatvecArgs& a, cudaStream_t st, int stages = STAGE_ALL);
int launch_near_only(int p, const MatvecArgs& a, cudaStream_t st);  // a.rows = A_near a.ax (no far field)
int launch_near_sums(const MatvecArgs& a, cudaStream_t st);          // a.near_sum = per-target near sums of a.ax

// tensor-core M2L (m2l_tc.cu)
int tc_supported(int p);            // 1 for 1 <= p <= 12
uint32_t tc_default_wait_tries();   // iteration limit of the contraction's pipeline waits
// k_near_sums: sets its dynamic shared-memory permission for the largest near block of a problem
// (max_ntgt targets) on the current device; -1 when that does not fit an SM
int configure_targets_ax_smem(int max_ntgt);
int tc_kp(int p);                   // real coefficients per row, padded to 64
size_t tc_rows_map_bytes();         // size of the TMA tensor map over the multipole rows
int tc_make_rows_map(void* map_out, void* Mt, int nrows, int p);
size_t tc_table_bytes(int p);       // bytes of one table image (hi + lo, one row tile of 128 outputs)
int tc_row_tiles(int p);            // table images per translation (1 for p <= 10, 2 for p = 11, 12)
int tc_kpo(int p);                  // floats per pair partial
int tc_max_pairs(int p);            // largest pairs per work item at order p
void tc_alpha_host(int p, double* alpha /*[tc_kp(p)]*/);
void launch_tc_tables(int p, int ntab, const double* tab, const double* alpha, void* T, unsigned int* maxbits, cudaStream_t st);
constexpr int TC_EXPAND = 1, TC_CONTRACT = 2, TC_REDUCE = 4, TC_ALL = 7;
// nd = 2: M[0], M[1] separate, their difference is translated; nd = 1: M[0] already holds it
int launch_m2l_tc(int p, const MatvecArgs& a, cudaStream_t st, int parts = TC_ALL, int nd = 2);
// builds the P2M operator (a.p2m_C zeroed beforehand); e_slot[3 s + a]: slot of the DOF of
// vertex a of element s within its leaf's DOF list
void launch_p2m_op(int p, const MatvecArgs& a, const int* e_slot, cudaStream_t st);
// FP32 copy of a complex FP64 array (the low-precision operator's P2M operator)
void launch_to_float2(size_t n, const double2* src, float2* dst, cudaStream_t st);
void launch_combine_weights(int nblocks, const NearBlockDev* blocks, const int* nb_dofs, const int* dof_kind, const double* WG,
                            const double* WGn, double* Wc, float* Wc32, cudaStream_t st);
void launch_densities(int n, int mode, const double* x, const double* known, const int* kind, double* phi, double* phin, cudaStream_t st);
int launch_near_weights(const NearArgs& a, cudaStream_t st);  // -1 if the block ranges exceed shared memory
void launch_diag(int n, const int* dof_point, const double* GnPhi, double* diag, cudaStream_t st);
int mdot_blocks(int n);
void launch_mdot(const double* V, int ldv, int k, const double* w, int n, double* partial, double* out, cudaStream_t st);
void launch_maxpy(const double* V, int ldv, int k, const double* h, double* w, int n, cudaStream_t st);
void launch_axpby(int n, double a, const double* x, double b, double* y, cudaStream_t st);
void launch_scale_inv(int n, const double* x, const double* s, double* y, cudaStream_t st);
void launch_mul(int n, const double* a, const double* x, double* y, cudaStream_t st);
void launch_hash_fill(int n, unsigned long long seed, double* y, cudaStream_t st);  // fixed pseudo-random [-0.5, 0.5)
void launch_add_mul(int n, const double* xb, const double* a, const double* u, double* y, cudaStream_t st);
struct ArnoldiState;
// near-block (block-Jacobi) preconditioner: per near block the DOFs of its targets (the core)
// and the column-major inverse of the core's near-field matrix (m^2 values); a core of more
// than kBjMaxCore DOFs keeps the point-Jacobi scaling as m diagonal values
constexpr int kBjMaxCore = 64;
struct NearBjArgs {
  int nblocks = 0;
  const NearBlockDev* blocks = nullptr;
  const int* doff = nullptr;      // [nblocks + 1] into dofs
  const int* dofs = nullptr;      // core DOFs, block by block
  const int64_t* ioff = nullptr;  // [nblocks + 1] into inv (m^2 per block, m above kBjMaxCore)
  double* inv = nullptr;
};
void launch_bj_setup(const NearBjArgs& a, const int* nb_dofs, const int* dof_point, const int* row_of_point, const int* dof_kind,
                     const double* diag, const double* Wc, const double* dinv, cudaStream_t st);
void launch_bj_apply(const NearBjArgs& a, const double* y, int ldy, const ArnoldiState* st, double* z, cudaStream_t s);
void launch_jacobi(int n, const int* dof_point, const int* dof_kind, const double* diag, const int* block_of_point, const int* row_of_point,
                   const NearBlockDev* blocks, const int* self_col, const double* WG, const double* WGn, double* dinv, cudaStream_t st);
double fp64_probe_tflops(cudaStream_t st, double* sink);

// ---- device-resident Arnoldi step (gmres.cu) ----
struct ArnoldiState {
  int n;         // basis vectors beyond V[:, 0] in this cycle
  int bad;       // a non-finite Arnoldi vector was met
  double err;    // |g[n]|: the GMRES residual estimate
  double inv_h;  // 1 / h_{n, n-1} of the last step
};
struct ArnoldiArgs {
  int nrow = 0, cols = 0, p = 0;  // unknowns, basis capacity (columns), expansion order
  double* V = nullptr;            // [cols][nrow] basis
  const double* dinv = nullptr;   // right Jacobi scaling or null
  ArnoldiState* state = nullptr;
  double* x = nullptr;            // operator input (the mat-vec's ax)
  double* w = nullptr;            // operator output (the mat-vec's rows)
  MatvecArgs mv;                  // the operator
  double* h = nullptr;            // [3][cols]: the two Gram-Schmidt passes (third column unused)
  double* partial = nullptr;      // [cols][arnoldi_dot_blocks(nrow)] per-slice partial dots
  double* cs = nullptr;           // [cols] rotations
  double* sn = nullptr;
  double* g = nullptr;            // [cols + 1] rotated right-hand side
  double* R = nullptr;            // [cols][cols] triangular factor, column j at R + j * cols
  // polynomial preconditioner: x = D^{-1} p(B) V[:, n] with B = A_near D^{-1}, written to the
  // operator input and to Z[:, n] (flexible storage: the iterate is updated from Z)
  const PolyRoots* poly = nullptr;  // null: x = (D^{-1}) V[:, n]
  NearBjArgs bj;                    // nblocks > 0: x = M^{-1} V[:, n] with the near-block preconditioner
  MatvecArgs near;                  // B: a.x (with D^{-1} applied) -> a.w, near field only
  double* prod = nullptr;           // [nrow] running product of the root factors
  double* y = nullptr;              // [nrow] polynomial accumulator
  double* Z = nullptr;              // [cols][nrow]
};
int arnoldi_dot_blocks(int nrow);
int configure_arnoldi(int cols);  // before capture: shared memory of the orthogonalisation kernels; -1 if cols is too large
int launch_arnoldi_step(const ArnoldiArgs& a, cudaStream_t st);  // returns kernel launches
void launch_arnoldi_init(ArnoldiState* state, double* g, double beta, cudaStream_t st);
// the first operator input of a cycle, x = (dinv .*) V[:, 0] (each step writes the next one's)
void launch_arnoldi_prep(int nrow, const double* V, const double* dinv, const ArnoldiState* state, double* x, cudaStream_t st);
void launch_arnoldi_solve_y(const ArnoldiState* state, const double* R, int ldr, const double* g, double* y, cudaStream_t st);
void launch_arnoldi_update(const double* V, int nrow, int cols, const ArnoldiState* state, const double* y, double* w, cudaStream_t st);

}  // namespace bemb200
