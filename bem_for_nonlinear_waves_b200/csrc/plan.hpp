// Host-side set-up plan of one boundary-value problem: coordinate scaling, element
// sources, the bucket octree, MAC interaction lists, L2P targets and the near-field
// sparsity.  Everything the device kernels need is flattened into index arrays here.
//
// The octree must reproduce the reference's Buckets tree exactly (same leaves for
// every element), so the floating-point expressions that place an element or size a
// bucket are the reference's own (lib/include/lib_spatial_partitioning.hpp:295-400,
// 1078-1111) and this file is compiled without fast-math.
#pragma once
#include <array>
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace bemb200 {

struct PlanOptions {
  int p = 10;
  double theta = 0.25;
  int leaf_max = 30;
  int max_level = 7;
  bool take_structure = true;  // refresh: take over the previous plan's unchanged structure (false: rebuild it)
  void* device_tree = nullptr;  // DeviceTree (tree_dev.hpp): grow the octree on the device; null: on the host
};

struct Plan {
  PlanOptions opt;
  int np = 0, nf = 0, ndof = 0;
  double L = 1.0;      // coordinate scale factor (bounding-box diagonal)
  double scale = 1.0;  // diagonal of the scaled bounding box
  double near_region = 0.0;
  std::vector<double> Xs;  // [3*np] scaled coordinates

  // DOF table
  std::vector<int32_t> dof_point, dof_face, dof_kind, face_dof;  // face_dof [3*nf] by face id
  std::vector<int32_t> point_dof_off, point_dof;                  // CSR point -> DOFs
  std::vector<int32_t> corner_src_dof;  // [ndof] for kind-2 rows: the point's Dirichlet DOF (or -1)

  // elements in tree order (position s = 0..nf-1)
  std::vector<int32_t> face_of_pos;   // [nf] face id at position s
  std::vector<int32_t> pos_of_face;   // [nf]
  std::vector<int32_t> owner_of_pos;  // [ne] deepest bucket holding the element
  std::vector<double> e_q;            // [nf*18] P2M points (6 x xyz), scaled
  std::vector<double> e_W;            // [nf*6] J * w_q
  std::vector<double> e_n;            // [nf*3] unit normal of the P2M points
  std::vector<int32_t> e_dof;         // [nf*3] face-vertex DOFs
  std::vector<int32_t> e_vtx;         // [nf*3] face vertices (point ids)
  std::vector<double> e_near;         // [nf*8]: J_near, cross_near xyz, centroid xyz, unused

  // octree nodes (every created bucket, DFS pre-order)
  struct Node {
    double lo[3], hi[3];
    double X[3];
    double dL, inv_dL;
    int size[3];
    int level;
    int parent;
    int child_begin, child_end;  // into node_children
    int fb, fe;                  // element range [fb, fe) in tree order (subtree, incl. orphans)
    int n_data;                  // elements held (data1D size)
    bool empty() const { return n_data == 0; }
    double max_internal_offset;
  };
  std::vector<Node> nodes;
  std::vector<int32_t> node_children;
  std::vector<std::vector<int32_t>> level_nodes;  // non-empty nodes per level (reference order)
  std::vector<int32_t> leaves;                    // non-empty childless nodes
  int n_added = 0;
  int n_child_drops = 0;  // elements a child bucket refused (reference edge case, counted)

  // lists
  std::vector<int32_t> m2l_off, m2l_src;  // CSR over nodes: sources of each target's M2L
  std::vector<int32_t> near_off, near_nodes;  // CSR over nodes: same-level near buckets
  int64_t m2l_pairs = 0, near_pairs = 0;
  // M2L grouped by translation vector: pairs of one level whose target - source offset is
  // the same lattice vector share one irregular-harmonic table.  Pair k is the k-th entry of
  // the target-major CSR (m2l_off / m2l_src); its partial local goes to slot k.
  std::vector<double> grp_vec;       // [groups*3] translation (target - source) of each group
  std::vector<int32_t> grp_off;      // [groups+1] CSR into grp_pair
  std::vector<int32_t> grp_pair;     // pair slots k, grouped
  std::vector<int32_t> chunk_grp;    // work chunks of <= 8 pairs: group
  std::vector<int32_t> chunk_begin;  // first index into grp_pair
  std::vector<int32_t> chunk_cnt;    // pairs in the chunk
  std::vector<int32_t> m2l_targets;  // targets with at least one pair
  // pairs in group order as packed values (offset key << 33 | level << 29 | slot; bit 63 set
  // for a pair off the lattice), kept for the tensor-core grouping
  std::vector<uint64_t> m2l_key_sorted;
  // tensor-core M2L (mixed precision): pairs grouped by their translation measured in
  // target-bucket sizes, so one table serves a lattice offset on every level; work items of
  // at most tc_item_max pairs of one table.  Filled by build_tc_groups().
  std::vector<double> tc_tab;        // [ntab*4]: (X_t - X_s) / dL_t, dL_s / dL_t
  std::vector<int32_t> tc_pair;      // pair slots k ordered by table
  std::vector<int32_t> tc_item_tab;  // table of each work item
  std::vector<int32_t> tc_item_begin;
  std::vector<int32_t> tc_item_cnt;

  // L2P / near targets: one target per point with DOFs
  std::vector<int32_t> target_box;     // [np] node of the point, -1 if the point has no DOF
  // near-field blocks: one per distinct target node
  struct NearBlock {
    int node;
    int64_t w_off;      // offset of this block's rows in the weight arrays
    int dof_off, ndof;  // into nb_dofs
    int tgt_off, ntgt;  // into nb_targets
    int rng_off, nrng;  // into nb_ranges (element ranges [a,b) in tree order, sorted)
  };
  std::vector<NearBlock> blocks;
  std::vector<int32_t> nb_dofs, nb_targets, nb_ranges;  // nb_dofs: per block, in first-appearance order
  std::vector<int32_t> block_of_point, row_of_point;  // [np]
  std::vector<int32_t> self_col;  // [ndof] column of the DOF in its point's block row, -1 if none
  int64_t nnz = 0;

  // DOF -> incident (element position, vertex slot)
  std::vector<int32_t> dof_inc_off, dof_inc;  // dof_inc = pos*3 + slot

  double phase_s[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // host set-up phase timings
  // per-face source data by face id before the element order is known (scratch kept across
  // set-ups with its size: a set-up of the same mesh writes it without new pages or clearing)
  struct SourceScratch {
    std::vector<std::array<double, 3>> pole;
    std::vector<double> q, W, en, enear, offs;
  } src_scratch;
  // scratch of the M2L grouping and of the tensor-core item arrays, kept the same way
  std::vector<int32_t> scratch_pair_tgt, scratch_slot_tgt;
  std::vector<std::vector<int32_t>> scratch_blk_dofs, scratch_blk_rng;  // per-thread near-block buffers

  // root bucket (centre, half-width) the tree was grown in; a refresh keeps it
  double root_C[3] = {0, 0, 0}, root_R = 0.0;
  // set by a refresh whose tree and lists came out identical to the previous plan's: the M2L
  // grouping and tensor-core items were taken over from it; reused_near: the L2P targets too,
  // and with them the near-field blocks
  bool reused_m2l = false, reused_near = false;
  bool tree_on_device = false;   // the octree was grown on the device
  bool lists_on_device = false;  // and the interaction lists built there
  int device_launches = 0;       // kernels those two launched (during the host plan)

  std::string error;
};

// every array member of Plan (build_plan reuses their capacity from the plan it overwrites)
#define BEMB200_PLAN_ARRAYS(X) X(Xs) X(dof_point) X(dof_face) X(dof_kind) X(face_dof) X(point_dof_off) X(point_dof) X(corner_src_dof) X(face_of_pos) X(pos_of_face) X(owner_of_pos) X(e_dof) X(e_vtx) X(nodes) X(node_children) X(level_nodes) X(leaves) X(m2l_off) X(m2l_src) X(near_off) X(near_nodes) X(grp_vec) X(grp_off) X(grp_pair) X(chunk_grp) X(chunk_begin) X(chunk_cnt) X(m2l_targets) X(m2l_key_sorted) X(tc_tab) X(tc_pair) X(tc_item_tab) X(tc_item_begin) X(tc_item_cnt) X(target_box) X(blocks) X(nb_dofs) X(nb_targets) X(nb_ranges) X(block_of_point) X(row_of_point) X(self_col) X(dof_inc_off) X(dof_inc)

// Fills dof tables from face flags with the reference's key rules; returns n_dof or -1.
int build_dofs(int np, const double* X, int nf, const int32_t* tri, const uint8_t* fdir, int32_t* dof_point, int32_t* dof_face,
               int32_t* dof_kind, int32_t* face_dof, uint8_t* point_flags);

// Builds the plan; returns false and sets plan.error on invalid input.
//
// prev (refresh): the previous plan of the same mesh (same options, DOF tables and faces) at
// other coordinates.  The tree is then grown in prev's root bucket, as the reference keeps its
// Buckets root across time steps and rebins the moved sources into it
// (bem/BEM_solveBVP_GMRES_FMM.hpp:3125-3346: initializeBucket once, rebin when the topology is
// unchanged); a fresh root is taken only if an element centroid left the old one.  When the
// tree and lists come out identical to prev's, the M2L structure is moved out of prev (prev is
// left partly empty; plan.reused_m2l), and with identical L2P targets the near-field blocks too
// (plan.reused_near).
// defer_m2l_groups: leave the M2L grouping (build_m2l_groups) to the caller, who can run it while
// the device works on what the plan already holds (it is skipped anyway when reused_m2l).
bool build_plan(Plan& plan, const PlanOptions& opt, int np, const double* X, int nf, const int32_t* tri, const uint8_t* fdir, int ndof,
                const int32_t* dof_point, const int32_t* dof_face, const int32_t* dof_kind, const int32_t* face_dof,
                Plan* prev = nullptr, bool defer_m2l_groups = false);
// the M2L grouping of build_plan (FP64 groups, chunks, targets with pairs)
bool build_m2l_groups(Plan& plan);

// memcpy in 1 MiB pieces over the OpenMP threads (staging of the set-up uploads)
void parallel_copy(void* dst, const void* src, size_t bytes);

// Groups the M2L pairs for the tensor-core path (tc_* fields); items hold <= max_pairs pairs.
void build_tc_groups(Plan& plan, int max_pairs);
// per tensor-core pair (work-item order j): its source bucket and compact target index (into
// m2l_targets); per pair slot k: its position j
void tc_item_arrays(Plan& plan, std::vector<int>& src, std::vector<int>& pos, std::vector<int>& tgt);
// Re-splits the tensor-core work items of build_tc_groups into items of <= max_pairs pairs
// (tables and pair order unchanged).
void retile_tc_items(Plan& plan, int max_pairs);

}  // namespace bemb200
