// ============================================================================
// ORACLE — test infrastructure only.  Not part of the product.
//
// A single-threaded-by-default CPU restatement (OpenMP where noted) of the
// reference's GMRES + FMM Laplace BVP path for linear triangle elements:
//   bem/BEM_setBoundaryTypes.hpp           DOF keys (isNeumannID/isDirichletID/pf2Index)
//   bem/BEM_solveBVP_GMRES_FMM.hpp         scaling, sources, tree set-up, mat-vec, GMRES driver
//   lib/include/lib_spatial_partitioning.hpp  Buckets octree (cell floor rule, 0.5+1e-13 child size)
//   lib/include/moments.hpp                P2M/M2M/M2L/L2L, MAC, interaction lists
//   lib/include/lib_multipole_expansion.hpp   SphericalCoordinates, near-field weights, L2P
//   lib/include/basic_linear_systems.hpp   gmres / ArnoldiProcess (MGS + Givens)
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it,
// as the checker.  The product path (the CUDA library) never links it.
//
// Deviation (documented): the dipole P2M coefficient n.grad(rho^n Y_n^{-m}) is
// evaluated with a Cartesian recurrence of the regular solid harmonics instead
// of the reference's spherical-coordinate formula (lib_multipole_expansion.hpp:
// 996-1010), which divides by r2D and by P_n^{|m|} and is NaN on the box axis or
// in the box mid-plane.  Where the reference is finite both agree to rounding.
// ============================================================================
#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <memory>
#include <numeric>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "aaa_coeffs.hpp"

namespace {

using cd = std::complex<double>;
using V3 = std::array<double, 3>;

// ---- numerics mirrored from the reference's helpers ------------------------

// libstdc++ 3-argument std::hypot (used by Norm(Tddd), basic_arithmetic_array_operations.hpp:860)
inline double hypot3(double x, double y, double z) {
  x = std::abs(x);
  y = std::abs(y);
  z = std::abs(z);
  if (double a = x < y ? y < z ? z : y : x < z ? z : x)
    return a * std::sqrt((x / a) * (x / a) + (y / a) * (y / a) + (z / a) * (z / a));
  return 0.0;
}
inline double norm3(const V3& a) { return hypot3(a[0], a[1], a[2]); }
inline V3 sub(const V3& a, const V3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
inline V3 add(const V3& a, const V3& b) { return {a[0] + b[0], a[1] + b[1], a[2] + b[2]}; }
inline V3 mul(double s, const V3& a) { return {s * a[0], s * a[1], s * a[2]}; }
// Dot(double3, double3): fma chain (basic_arithmetic_array_operations.hpp:593)
inline double dot3(const V3& a, const V3& b) { return std::fma(a[0], b[0], std::fma(a[1], b[1], a[2] * b[2])); }
// Dot(weights[3], X012[3]) : ret[j] = fma(w_i, X_i[j], ret[j]) (basic_arithmetic_array_operations.hpp:639-657)
inline V3 wsum3(const V3& w, const V3& X0, const V3& X1, const V3& X2) {
  V3 r{0, 0, 0};
  for (int j = 0; j < 3; ++j) r[j] = std::fma(w[0], X0[j], r[j]);
  for (int j = 0; j < 3; ++j) r[j] = std::fma(w[1], X1[j], r[j]);
  for (int j = 0; j < 3; ++j) r[j] = std::fma(w[2], X2[j], r[j]);
  return r;
}
// Cross in float128 then rounded (basic_arithmetic_array_operations.hpp:906-920)
inline V3 cross_hp(const V3& A, const V3& B) {
  __float128 ax = A[0], ay = A[1], az = A[2], bx = B[0], by = B[1], bz = B[2];
  return {(double)(ay * bz - az * by), (double)(az * bx - ax * bz), (double)(ax * by - ay * bx)};
}
// Normalize: fma-accumulated squared norm (basic_arithmetic_array_operations.hpp:837-850)
inline V3 normalize(V3 a) {
  double n = 0.;
  for (double v : a) n = std::fma(v, v, n);
  if (n == 0.) return a;
  n = std::sqrt(n);
  for (auto& v : a) v /= n;
  return a;
}
// TriangleNormalHP (basic_arithmetic_array_operations.hpp:961-986)
inline V3 tri_normal_hp(const V3& a, const V3& b, const V3& c) {
  __float128 ax = a[0], ay = a[1], az = a[2];
  __float128 bax = (__float128)b[0] - ax, bay = (__float128)b[1] - ay, baz = (__float128)b[2] - az;
  __float128 cax = (__float128)c[0] - ax, cay = (__float128)c[1] - ay, caz = (__float128)c[2] - az;
  __float128 nx = bay * caz - baz * cay, ny = baz * cax - bax * caz, nz = bax * cay - bay * cax;
  __float128 n2 = nx * nx + ny * ny + nz * nz;
  if (n2 == 0) return {0, 0, 0};
  __float128 inv = (__float128)1 / (__float128)std::sqrt((double)n2);
  return {(double)(nx * inv), (double)(ny * inv), (double)(nz * inv)};
}

// ---- quadrature tables ---------------------------------------------------
// 5x5 Gauss-Legendre product rule on [0,1]^2 with the reference's own 15-digit constants
// (__array_GW5xGW5__, lib/include/basic_constants.hpp:1326-1350): the near-field weights must
// share them to agree with the reference beyond ~1e-12.  The table is symmetric: node a and
// weight class c(a) = {0, 1, 2, 1, 0}, w(a, b) = kGW5W[c(a)][c(b)].
struct GW {
  double t0, t1, w;
};
std::vector<GW> make_gw5x5() {
  static const double x[5] = {0.046910077030668, 0.230765344947158, 0.5, 0.769234655052841, 0.953089922969332};
  static const int c[5] = {0, 1, 2, 1, 0};
  static const double w[3][3] = {{0.0140335872156063, 0.0283499999999991, 0.0336962680968792},
                                 {0.0283499999999991, 0.0572713510559978, 0.0680716331376877},
                                 {0.0336962680968792, 0.0680716331376877, 0.0809086419753086}};
  std::vector<GW> r;
  for (int a = 0; a < 5; ++a)
    for (int b = 0; b < 5; ++b) r.push_back({x[a], x[b], w[c[a]][c[b]]});
  return r;
}
// Dunavant degree-4 6-point rule (barycentrics, weight incl. the 1/2 area factor)
// (reference: __dunavant_p2m_6__, lib/include/dunavant_rules.hpp:36-42)
struct DV {
  double b0, b1, b2, w;
};
const DV kDunavant6[6] = {{0.816847572980459, 0.091576213509771, 0.091576213509771, 0.054975871827661},
                          {0.091576213509771, 0.816847572980459, 0.091576213509771, 0.054975871827661},
                          {0.091576213509771, 0.091576213509771, 0.816847572980459, 0.054975871827661},
                          {0.108103018168070, 0.445948490915965, 0.445948490915965, 0.111690794839006},
                          {0.445948490915965, 0.108103018168070, 0.445948490915965, 0.111690794839006},
                          {0.445948490915965, 0.445948490915965, 0.108103018168070, 0.111690794839006}};

// ModTriShape<3>(t0,t1) (basic_arithmetic_array_operations.hpp:1591)
inline V3 mod_tri_shape(double t0, double t1) { return {t0, t1 * (1. - t0), (t0 - 1.) * (t1 - 1.)}; }

// ---- spherical harmonics, reference conventions ---------------------------
// SphericalCoordinates (lib_multipole_expansion.hpp:779-800)
struct Sph {
  double rho, theta, phi;
  explicit Sph(const V3& X) {
    double r2D = std::hypot(X[0], X[1]);
    rho = hypot3(X[0], X[1], X[2]);
    phi = std::atan2(X[1], X[0]);
    theta = std::atan2(r2D, X[2]);
  }
  // Y_n^m = sqrt(4pi/(2n+1)) sph_legendre(n,|m|,theta) e^{i m phi}  (:878-890)
  cd Y(int n, int m) const {
    int am = std::abs(m);
    if (am > n) return 0.0;
    double s = std::sqrt(2.0 * M_PI) / std::sqrt(n + 0.5);
    return std::polar(std::sph_legendre(n, am, theta) * s, m * phi);
  }
  cd Y_rho(int n, int m) const { return Y(n, m) * std::pow(rho, n); }
  cd Y_div_rhon1(int n, int m) const { return Y(n, m) / (std::pow(rho, n) * rho); }
};

// Regular solid harmonics without Condon-Shortley phase, F_n^m = rho^n P_n^m e^{im phi}/(n+m)!,
// m >= 0, by the standard three-term recurrences; F[n*(n+1)/2 + m].
void solid_F(const V3& v, int p, std::vector<cd>& F) {
  const double x = v[0], y = v[1], z = v[2];
  const double r2 = x * x + y * y + z * z;
  F.assign((p + 2) * (p + 3) / 2, 0.0);
  auto idx = [](int n, int m) { return n * (n + 1) / 2 + m; };
  F[0] = 1.0;
  for (int m = 0; m <= p; ++m) {
    if (m > 0) F[idx(m, m)] = F[idx(m - 1, m - 1)] * cd(x, y) / (2.0 * m);
    if (m + 1 <= p) F[idx(m + 1, m)] = z * F[idx(m, m)];
    for (int n = m + 1; n < p; ++n)
      F[idx(n + 1, m)] = ((2.0 * n + 1.0) * z * F[idx(n, m)] - r2 * F[idx(n - 1, m)]) / double((n + 1) * (n + 1) - m * m);
  }
}
inline cd getF(const std::vector<cd>& F, int n, int m) {
  if (n < 0 || std::abs(m) > n) return 0.0;
  if (m >= 0) return F[n * (n + 1) / 2 + m];
  cd c = std::conj(F[n * (n + 1) / 2 - m]);
  return ((-m) & 1) ? -c : c;
}

// ---- data --------------------------------------------------------------------
struct Node {
  double bmin[3], bmax[3];
  double xmin, ymin, zmin;
  double dL, inv_dL;
  int size[3];
  V3 X;  // centre = Mean(Transpose(bounds))
  int level;
  Node* parent = nullptr;
  std::vector<Node*> children;          // xsize*ysize*zsize slots (nullptr = none)
  std::vector<std::vector<int>> cells;  // face ids per cell
  std::vector<int> data;                // data1D_vector (faces in this subtree, insertion order)
  std::vector<Node*> near, m2l, l2m;
  double max_internal_offset = 0.0;
  int id = -1;  // DFS pre-order id among non-empty nodes
  // moments: [(p+1)^2][2]
  std::vector<std::array<cd, 2>> MM, LL;
  bool has_children() const {
    for (auto* c : children)
      if (c) return true;
    return false;
  }
  void init(const double lo[3], const double hi[3], double dL_in) {
    for (int a = 0; a < 3; ++a) {
      bmin[a] = lo[a];
      bmax[a] = hi[a];
    }
    X = {(lo[0] + hi[0]) / 2., (lo[1] + hi[1]) / 2., (lo[2] + hi[2]) / 2.};
    dL = dL_in;
    inv_dL = 1.0 / dL_in;
    xmin = lo[0];
    ymin = lo[1];
    zmin = lo[2];
    for (int a = 0; a < 3; ++a) {
      double s = std::ceil((bmax[a] - bmin[a]) / dL);
      if (s <= 0.) s = 1.;
      size[a] = (int)s;
    }
    cells.assign(size[0] * size[1] * size[2], {});
  }
  int cell_id(int i, int j, int k) const { return (i * size[1] + j) * size[2] + k; }
  void indices_no_clamp(const V3& x, int ijk[3]) const {
    ijk[0] = (int)std::floor((x[0] - xmin) * inv_dL);
    ijk[1] = (int)std::floor((x[1] - ymin) * inv_dL);
    ijk[2] = (int)std::floor((x[2] - zmin) * inv_dL);
  }
  bool inside(const V3& x) const {
    int ijk[3];
    indices_no_clamp(x, ijk);
    return ijk[0] >= 0 && ijk[0] < size[0] && ijk[1] >= 0 && ijk[1] < size[1] && ijk[2] >= 0 && ijk[2] < size[2];
  }
  void indices(const V3& x, int ijk[3]) const {
    indices_no_clamp(x, ijk);
    for (int a = 0; a < 3; ++a) ijk[a] = std::clamp(ijk[a], 0, size[a] - 1);
  }
};

struct Source {  // one linear element (lib_multipole_expansion.hpp:675-775)
  V3 X;           // tree position Dot({1/3,1/3,1/3}, X012)
  V3 normal;      // Normalize(cross)
  V3 q[6];        // P2M points
  double W[6];    // J_det * w_q
  double N[6][3]; // barycentrics
  double max_source_offset;
  int v[3];       // point ids
  int dof[3];     // face-vertex DOF (pf2Index)
  // near-field data (BEM_solveBVP_GMRES_FMM.hpp:1832-1891)
  double J_near;  // 2*area
  V3 cross_near;  // 2*area*normal_hp
  V3 centroid;    // (a+b+c)/3
};

}  // namespace

struct OracleCtx {
  int near_stride = 1;  // near-field rows computed for every near_stride-th point only (timing samples)
  double t_tree = 0.0, t_near = 0.0;
  int p = 8;
  double theta = 0.25;
  int max_points = 30;
  int max_level = 7;
  int np = 0, nf = 0, ndof = 0;
  std::vector<V3> Xs;  // scaled points
  std::vector<int> tri;
  std::vector<uint8_t> fdir;
  std::vector<int> dof_point, dof_face, dof_kind;  // kind 0 Dir, 1 Neu, 2 corner-Neumann constraint
  std::vector<int> face_dof;                       // nf*3
  std::vector<std::vector<int>> point_dofs;        // DOFs per point
  double L = 1.0;  // coordinate scale factor
  double scale = 1.0;
  V3 center{};
  double near_region = 0;
  std::vector<Source> src;
  std::unique_ptr<Node> root;
  std::vector<std::unique_ptr<Node>> pool;
  std::vector<std::vector<Node*>> level_nodes;
  std::vector<Node*> leaves;
  int n_added = 0;
  // targets (one per point)
  std::vector<Node*> tgt_leaf;
  std::vector<std::vector<int>> near_idx;
  std::vector<std::vector<double>> near_wG, near_wGn;  // wG multiplies phin, wGn multiplies phi
  std::vector<double> diag;
  // AAA tables flattened [j][k+p][n][m+p]
  std::vector<double> aaa_m2m, aaa_m2l, aaa_l2l;
  int ncoef() const { return (p + 1) * (p + 1); }
  size_t aidx(int j, int k, int n, int m) const {
    int w = 2 * p + 1;
    return (((size_t)j * w + (k + p)) * (p + 1) + n) * w + (m + p);
  }
};

namespace {

// ---- DOF keys (BEM_setBoundaryTypes.hpp:29-100, 134-254, 434-441, 573-579) ----
struct PointFlags {
  std::vector<uint8_t> neu, dir, corner, multiple;
};

PointFlags point_flags(int np, const double* X, int nf, const int* tri, const uint8_t* fdir, std::vector<std::vector<int>>& pf) {
  pf.assign(np, {});
  for (int f = 0; f < nf; ++f)
    for (int a = 0; a < 3; ++a) pf[tri[3 * f + a]].push_back(f);
  PointFlags fl;
  fl.neu.assign(np, 0);
  fl.dir.assign(np, 0);
  fl.corner.assign(np, 0);
  fl.multiple.assign(np, 0);
  std::vector<V3> fn(nf);
  std::vector<double> fa(nf);
  for (int f = 0; f < nf; ++f) {
    V3 a{X[3 * tri[3 * f]], X[3 * tri[3 * f] + 1], X[3 * tri[3 * f] + 2]};
    V3 b{X[3 * tri[3 * f + 1]], X[3 * tri[3 * f + 1] + 1], X[3 * tri[3 * f + 1] + 2]};
    V3 c{X[3 * tri[3 * f + 2]], X[3 * tri[3 * f + 2] + 1], X[3 * tri[3 * f + 2] + 2]};
    fn[f] = tri_normal_hp(a, b, c);
    fa[f] = 0.5 * norm3(cross_hp(sub(b, a), sub(c, a)));
  }
  const double lim = 20. * M_PI / 180.;
  for (int p = 0; p < np; ++p) {
    if (pf[p].empty()) continue;
    bool alln = true, alld = true;
    for (int f : pf[p]) {
      alln = alln && !fdir[f];
      alld = alld && fdir[f];
    }
    fl.neu[p] = alln;
    fl.dir[p] = alld;
    fl.corner[p] = !alln && !alld;
    if (fl.corner[p]) {
      fl.multiple[p] = 1;
    } else {
      V3 n{0, 0, 0};
      for (int f : pf[p]) n = add(n, mul(fa[f], fn[f]));
      n = normalize(n);
      bool any_not_flat = false;
      for (int f : pf[p]) {
        bool flat = dot3(n, fn[f]) > std::cos(lim) * std::sqrt(dot3(n, n)) * std::sqrt(dot3(fn[f], fn[f]));
        if (!flat) any_not_flat = true;
      }
      fl.multiple[p] = any_not_flat;
    }
  }
  return fl;
}

inline bool isNeumannID(const PointFlags& fl, const std::vector<uint8_t>& fdir, int p, int f) {
  if (fl.neu[p] || fl.corner[p]) {
    if (fl.multiple[p]) return f >= 0 && !fdir[f];
    return f < 0;
  }
  return false;
}
inline bool isDirichletID(const PointFlags& fl, int p, int f) { return (fl.dir[p] || fl.corner[p]) && f < 0; }

}  // namespace

extern "C" {

// Builds the DOF table with the reference's key rules.  DOFs are numbered point by
// point (point order), key (p,null) first then (p,f) in ascending face order; the
// reference renumbers by Morton order (BEM_solveBVP_GMRES_FMM.hpp:3152-3305), which
// is a permutation and leaves every solution value unchanged.
// Returns n_dof; arrays must hold up to np + 3*nf entries; face_dof holds nf*3.
int oracle_build_dofs(int np, const double* X, int nf, const int* tri, const uint8_t* face_dirichlet, int* dof_point, int* dof_face,
                      int* dof_kind, int* face_dof, uint8_t* point_flags_out) {
  std::vector<std::vector<int>> pf;
  std::vector<uint8_t> fdir(face_dirichlet, face_dirichlet + nf);
  PointFlags fl = point_flags(np, X, nf, tri, face_dirichlet, pf);
  int n = 0;
  std::vector<int> null_dof(np, -1);
  std::vector<std::vector<std::pair<int, int>>> face_keys(np);
  for (int p = 0; p < np; ++p) {
    if (pf[p].empty()) continue;
    if (isNeumannID(fl, fdir, p, -1) || isDirichletID(fl, p, -1)) {
      dof_point[n] = p;
      dof_face[n] = -1;
      dof_kind[n] = isDirichletID(fl, p, -1) ? 0 : 1;
      null_dof[p] = n++;
    }
    std::vector<int> fs = pf[p];
    std::sort(fs.begin(), fs.end());
    for (int f : fs)
      if (isNeumannID(fl, fdir, p, f) || isDirichletID(fl, p, f)) {
        dof_point[n] = p;
        dof_face[n] = f;
        dof_kind[n] = fl.corner[p] ? 2 : 1;
        face_keys[p].push_back({f, n});
        ++n;
      }
  }
  for (int f = 0; f < nf; ++f)
    for (int a = 0; a < 3; ++a) {
      int p = tri[3 * f + a];
      int d = -1;
      if (!fl.multiple[p] || fdir[f]) {
        d = null_dof[p];
      } else {
        for (auto& kv : face_keys[p])
          if (kv.first == f) d = kv.second;
      }
      face_dof[3 * f + a] = d;
    }
  if (point_flags_out)
    for (int p = 0; p < np; ++p)
      point_flags_out[p] = (fl.neu[p] ? 1 : 0) | (fl.dir[p] ? 2 : 0) | (fl.corner[p] ? 4 : 0) | (fl.multiple[p] ? 8 : 0);
  return n;
}

}  // extern "C"

namespace {

// ---- tree (lib_spatial_partitioning.hpp) ------------------------------------
Node* new_node(OracleCtx& C) {
  C.pool.emplace_back(new Node());
  return C.pool.back().get();
}

// Buckets::add(x,p): InsideQ (no clamp) then insert into the clamped cell.
bool node_add(Node* b, const V3& x, int s) {
  if (!b->inside(x)) return false;
  int ijk[3];
  b->indices(x, ijk);
  b->cells[b->cell_id(ijk[0], ijk[1], ijk[2])].push_back(s);
  b->data.push_back(s);
  return true;
}

// Buckets::generateTree with newChild (lib_spatial_partitioning.hpp:1078-1111)
void generate_tree(OracleCtx& C, Node* b) {
  bool cond = !b->data.empty() && ((int)b->data.size() > C.max_points && b->level < C.max_level);
  if (cond && b->level < C.max_level) {
    b->children.assign(b->size[0] * b->size[1] * b->size[2], nullptr);
    for (int i = 0; i < b->size[0]; ++i)
      for (int j = 0; j < b->size[1]; ++j)
        for (int k = 0; k < b->size[2]; ++k) {
          auto& cell = b->cells[b->cell_id(i, j, k)];
          if (cell.empty()) continue;
          Node* c = new_node(C);
          double lo[3] = {b->dL * i + b->xmin, b->dL * j + b->ymin, b->dL * k + b->zmin};
          double hi[3] = {b->dL * (i + 1) + b->xmin, b->dL * (j + 1) + b->ymin, b->dL * (k + 1) + b->zmin};
          c->init(lo, hi, b->dL * (0.5 + 1e-13));
          c->parent = b;
          for (int s : cell) node_add(c, C.src[s].X, s);
          c->level = b->level + 1;
          b->children[b->cell_id(i, j, k)] = c;
          generate_tree(C, c);
        }
  }
}

void traverse_tree(Node* b, const std::function<void(Node*)>& f) {
  for (auto* c : b->children)
    if (c) {
      f(c);
      traverse_tree(c, f);
    }
}

Node* bucket_at_deepest(Node* root, const V3& x) {
  Node* cur = root;
  while (cur->has_children()) {
    int ijk[3];
    cur->indices(x, ijk);
    Node* nx = cur->children[cur->cell_id(ijk[0], ijk[1], ijk[2])];
    if (!nx) return cur;
    cur = nx;
  }
  return cur;
}

// MAC (moments.hpp:950-956)
bool is_far(const OracleCtx& C, const Node* A, const Node* B) {
  double eff = std::max(A->dL + 2.0 * A->max_internal_offset, B->dL + 2.0 * B->max_internal_offset);
  return C.theta > std::sqrt(3.0) * eff / norm3(sub(B->X, A->X));
}

// buildNearAndM2LLists (moments.hpp:967-979)
void build_lists(const OracleCtx& C, Node* A, Node* B) {
  if (!is_far(C, A, B)) {
    if (A != B) A->near.push_back(B);
    for (auto* Ac : A->children) {
      if (!Ac) continue;
      for (auto* Bc : B->children) {
        if (!Bc) continue;
        if (Ac != Bc && is_far(C, Ac, Bc))
          Ac->m2l.push_back(Bc);
        else
          build_lists(C, Ac, Bc);
      }
    }
  }
}

// ---- FMM kernels in the reference's G&R form ----------------------------------
// p2mFunction(n,m,normal) -> {rho^n Y_n^{-m}, normal.grad(rho^n Y_n^{-m})}
// (lib_multipole_expansion.hpp:996-1010) via F recurrences:
//   rho^n Y_n^{m} = (-1)^m sqrt((n-m)!(n+m)!) F_n^m for m>=0, Y_n^{-m} = conj(Y_n^m).
void p2m_point(const OracleCtx& C, const V3& v, const V3& nu, double w_phin, double w_phi, std::vector<std::array<cd, 2>>& MM) {
  const int p = C.p;
  std::vector<cd> F;
  solid_F(v, p, F);
  for (int n = 0; n <= p; ++n)
    for (int m = -n; m <= n; ++m) {
      int am = std::abs(m);
      double c = ((am & 1) ? -1.0 : 1.0) * std::sqrt(std::tgamma(n - am + 1.0) * std::tgamma(n + am + 1.0));
      // gradient of F_n^{am}
      cd g = nu[2] * getF(F, n - 1, am) + 0.5 * cd(nu[0], nu[1]) * getF(F, n - 1, am - 1) - 0.5 * cd(nu[0], -nu[1]) * getF(F, n - 1, am + 1);
      cd f = getF(F, n, am);
      cd R, G;
      if (m >= 0) {  // rho^n Y_n^{-m} = conj(rho^n Y_n^m)
        R = c * std::conj(f);
        G = c * std::conj(g);
      } else {  // rho^n Y_n^{|m|}
        R = c * f;
        G = c * g;
      }
      int ind = n * (n + 1) + m;
      MM[ind][0] += w_phin * R;
      MM[ind][1] += w_phi * G;
    }
}

void conj_fill(int p, std::vector<std::array<cd, 2>>& A) {  // enforce_conjugate_m_symmetry (moments.hpp:287-298)
  for (int n = 0; n <= p; ++n)
    for (int m = 1; m <= n; ++m) {
      A[n * (n + 1) - m][0] = std::conj(A[n * (n + 1) + m][0]);
      A[n * (n + 1) - m][1] = std::conj(A[n * (n + 1) + m][1]);
    }
}

}  // namespace

extern "C" {

// Set-up: scaling, sources, tree, lists, L2P targets, near-field weights, diagonal.
// desc arrays: X[np*3] physical, tri[nf*3], face_dirichlet[nf], DOF table.
void* oracle_create_sampled(int np, const double* X, int nf, const int* tri, const uint8_t* face_dirichlet, int ndof, const int* dof_point,
                            const int* dof_face, const int* dof_kind, const int* face_dof, int p, double theta, int max_points, int max_level,
                            int near_stride) {
  auto* Cp = new OracleCtx();
  OracleCtx& C = *Cp;
  C.near_stride = near_stride < 1 ? 1 : near_stride;
  const double wt0 = omp_get_wtime();
  C.p = p;
  C.theta = theta;
  C.max_points = max_points;
  C.max_level = max_level;
  C.np = np;
  C.nf = nf;
  C.ndof = ndof;
  C.tri.assign(tri, tri + 3 * nf);
  C.fdir.assign(face_dirichlet, face_dirichlet + nf);
  C.dof_point.assign(dof_point, dof_point + ndof);
  C.dof_face.assign(dof_face, dof_face + ndof);
  C.dof_kind.assign(dof_kind, dof_kind + ndof);
  C.face_dof.assign(face_dof, face_dof + 3 * nf);
  C.point_dofs.assign(np, {});
  for (int i = 0; i < ndof; ++i) C.point_dofs[dof_point[i]].push_back(i);

  // coordinate scaling (Network.hpp:3215-3245; BEM_solveBVP_GMRES_FMM.hpp:3076-3091)
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (int i = 0; i < np; ++i)
    for (int a = 0; a < 3; ++a) {
      mn[a] = std::min(mn[a], X[3 * i + a]);
      mx[a] = std::max(mx[a], X[3 * i + a]);
    }
  double Lx = std::abs(mx[0] - mn[0]), Ly = std::abs(mx[1] - mn[1]), Lz = std::abs(mx[2] - mn[2]);
  C.L = std::sqrt(Lx * Lx + Ly * Ly + Lz * Lz);
  if (!(C.L > 1e-10)) C.L = 1.0;
  C.Xs.resize(np);
  for (int i = 0; i < np; ++i) C.Xs[i] = {X[3 * i] / C.L, X[3 * i + 1] / C.L, X[3 * i + 2] / C.L};
  for (int a = 0; a < 3; ++a) {
    mn[a] = 1e300;
    mx[a] = -1e300;
  }
  for (int i = 0; i < np; ++i)
    for (int a = 0; a < 3; ++a) {
      mn[a] = std::min(mn[a], C.Xs[i][a]);
      mx[a] = std::max(mx[a], C.Xs[i][a]);
    }
  C.scale = hypot3(mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]);
  C.center = {(mn[0] + mx[0]) / 2., (mn[1] + mx[1]) / 2., (mn[2] + mx[2]) / 2.};
  C.near_region = C.scale / 25.;

  // sources (BEM_solveBVP_GMRES_FMM.hpp:1799-1937)
  C.src.resize(nf);
  for (int f = 0; f < nf; ++f) {
    Source& s = C.src[f];
    for (int a = 0; a < 3; ++a) {
      s.v[a] = tri[3 * f + a];
      s.dof[a] = face_dof[3 * f + a];
    }
    const V3 &X0 = C.Xs[s.v[0]], &X1 = C.Xs[s.v[1]], &X2 = C.Xs[s.v[2]];
    V3 cr = cross_hp(sub(X1, X0), sub(X2, X0));
    s.normal = normalize(cr);
    double J = norm3(cr);
    s.X = wsum3({1. / 3., 1. / 3., 1. / 3.}, X0, X1, X2);
    s.max_source_offset = 0.0;
    for (int q = 0; q < 6; ++q) {
      const DV& d = kDunavant6[q];
      s.q[q] = wsum3({d.b0, d.b1, d.b2}, X0, X1, X2);
      s.W[q] = J * d.w;
      s.N[q][0] = d.b0;
      s.N[q][1] = d.b1;
      s.N[q][2] = d.b2;
      s.max_source_offset = std::max(s.max_source_offset, norm3(sub(s.q[q], s.X)));
    }
    double area = 0.5 * norm3(cross_hp(sub(X1, X0), sub(X2, X0)));
    V3 nhp = tri_normal_hp(X0, X1, X2);
    s.J_near = 2. * area;
    s.cross_near = mul(2. * area, nhp);
    s.centroid = {(X0[0] + X1[0] + X2[0]) / 3., (X0[1] + X1[1] + X2[1]) / 3., (X0[2] + X1[2] + X2[2]) / 3.};
  }

  // root bucket (BEM_solveBVP_GMRES_FMM.hpp:1178-1201)
  double dLr = 1.05 * C.scale / 2.;
  C.root.reset(new Node());
  Node* R = C.root.get();
  double lo[3] = {C.center[0] - dLr, C.center[1] - dLr, C.center[2] - dLr};
  double hi[3] = {C.center[0] + dLr, C.center[1] + dLr, C.center[2] + dLr};
  R->init(lo, hi, dLr);
  R->level = 0;
  C.n_added = 0;
  for (int f = 0; f < nf; ++f) C.n_added += node_add(R, C.src[f].X, f);
  generate_tree(C, R);
  // rebuildHierarchyLists (lib_spatial_partitioning.hpp:966-984)
  C.level_nodes.assign(C.max_level + 1, {});
  C.leaves.clear();
  int idc = 0;
  auto visit = [&](Node* b) {
    if (!b->data.empty()) {
      b->id = idc++;
      C.level_nodes[b->level].push_back(b);
      if (!b->has_children()) C.leaves.push_back(b);
    }
  };
  visit(R);
  traverse_tree(R, visit);

  // max_internal_offset (moments.hpp:1336-1349)
  for (auto* b : C.leaves) {
    b->max_internal_offset = 0.0;
    for (int s : b->data) b->max_internal_offset = std::max(b->max_internal_offset, C.src[s].max_source_offset);
  }
  for (int level = C.max_level - 1; level >= 0; --level)
    for (auto* b : C.level_nodes[level]) {
      if (!b->has_children()) continue;
      b->max_internal_offset = 0.0;
      for (auto* c : b->children)
        if (c) b->max_internal_offset = std::max(b->max_internal_offset, c->max_internal_offset);
    }

  // lists (moments.hpp:983-997)
  for (auto* A : R->children)
    if (A)
      for (auto* B : R->children)
        if (B) build_lists(C, A, B);
  for (auto& lv : C.level_nodes)
    for (auto* A : lv)
      for (auto* B : A->m2l) B->l2m.push_back(A);

  // AAA tables
  const int w = 2 * p + 1;
  size_t asz = (size_t)(p + 1) * w * (p + 1) * w;
  C.aaa_m2m.assign(asz, 0.);
  C.aaa_m2l.assign(asz, 0.);
  C.aaa_l2l.assign(asz, 0.);
  for (int j = 0; j <= p; ++j)
    for (int k = -j; k <= j; ++k)
      for (int n = 0; n <= p; ++n)
        for (int m = -n; m <= n; ++m) {
          C.aaa_m2m[C.aidx(j, k, n, m)] = bem_oracle_aaa::m2m(j, k, n, m);
          C.aaa_m2l[C.aidx(j, k, n, m)] = bem_oracle_aaa::m2l(j, k, n, m);
          C.aaa_l2l[C.aidx(j, k, n, m)] = bem_oracle_aaa::l2l(j, k, n, m);
        }

  C.t_tree = omp_get_wtime() - wt0;
  const double wt1 = omp_get_wtime();
  // targets: leaf + near-field weights (lib_multipole_expansion.hpp:1130-1271)
  C.tgt_leaf.assign(np, nullptr);
  C.near_idx.assign(np, {});
  C.near_wG.assign(np, {});
  C.near_wGn.assign(np, {});
  static const std::vector<GW> gw = make_gw5x5();
#pragma omp parallel for schedule(dynamic, 16)
  for (int t = 0; t < np; ++t) {
    if (C.point_dofs[t].empty()) continue;
    const V3 xt = C.Xs[t];
    Node* bd = bucket_at_deepest(R, xt);
    C.tgt_leaf[t] = bd;
    if (t % C.near_stride != 0) continue;
    std::vector<double> accG(ndof, 0.0), accGn(ndof, 0.0);
    std::vector<uint8_t> touched(ndof, 0);
    std::vector<int> tl;
    auto addw = [&](int idx, double g, double gn) {
      accG[idx] += g;
      accGn[idx] += gn;
      if (!touched[idx]) {
        touched[idx] = 1;
        tl.push_back(idx);
      }
    };
    auto setNear = [&](const Node* B) {
      for (int sidx : B->data) {
        const Source& s = C.src[sidx];
        bool adj = (s.v[0] == t || s.v[1] == t || s.v[2] == t);
        if (adj) {  // fill_direct_linear
          int pv[3] = {s.v[0], s.v[1], s.v[2]};
          int idx[3] = {0, 1, 2};
          if (s.v[1] == t) {
            pv[0] = s.v[1];
            pv[1] = s.v[2];
            pv[2] = s.v[0];
            idx[0] = 2;
            idx[1] = 0;
            idx[2] = 1;
          } else if (s.v[2] == t) {
            pv[0] = s.v[2];
            pv[1] = s.v[0];
            pv[2] = s.v[1];
            idx[0] = 1;
            idx[1] = 2;
            idx[2] = 0;
          }
          const V3 &X0 = C.Xs[pv[0]], &X1 = C.Xs[pv[1]], &X2 = C.Xs[pv[2]];
          V3 WG{0, 0, 0}, WGn{0, 0, 0};
          for (const auto& g : gw) {
            V3 Ng = mod_tri_shape(g.t0, g.t1);
            V3 Rv = sub(wsum3(Ng, X0, X1, X2), xt);
            double nr_inv = 1. / norm3(Rv);
            V3 tmp = mul(g.w * (1. - g.t0) * nr_inv, Ng);
            WG = add(WG, mul(s.J_near, tmp));
            double dn = -dot3(mul(nr_inv, Rv), s.cross_near);
            WGn = add(WGn, mul(nr_inv, mul(dn, tmp)));
          }
          addw(s.dof[0], WG[idx[0]], 0.0);
          addw(s.dof[1], WG[idx[1]], WGn[idx[1]]);
          addw(s.dof[2], WG[idx[2]], WGn[idx[2]]);
        } else {  // fill_nonadj_linear
          const V3 &X0 = C.Xs[s.v[0]], &X1 = C.Xs[s.v[1]], &X2 = C.Xs[s.v[2]];
          V3 WG{0, 0, 0}, WGn{0, 0, 0};
          if (norm3(sub(s.centroid, xt)) < C.near_region) {
            for (const auto& g : gw) {
              V3 Ng = mod_tri_shape(g.t0, g.t1);
              V3 Rv = sub(wsum3(Ng, X0, X1, X2), xt);
              double nr_inv = 1. / norm3(Rv);
              V3 tmp = mul(nr_inv, mul(g.w * (1. - g.t0), Ng));
              WG = add(WG, mul(s.J_near, tmp));
              double dn = dot3(mul(nr_inv, Rv), s.cross_near);
              WGn = sub(WGn, mul(dn, mul(nr_inv, tmp)));
            }
          } else {
            for (int q = 0; q < 6; ++q) {
              const DV& d = kDunavant6[q];
              V3 Ng{d.b0, d.b1, d.b2};
              V3 Rv = sub(wsum3(Ng, X0, X1, X2), xt);
              double nr_inv = 1. / norm3(Rv);
              V3 tmp = mul(nr_inv, mul(d.w, Ng));
              WG = add(WG, mul(s.J_near, tmp));
              double dn = dot3(mul(nr_inv, Rv), s.cross_near);
              WGn = sub(WGn, mul(dn, mul(nr_inv, tmp)));
            }
          }
          for (int a = 0; a < 3; ++a) addw(s.dof[a], WG[a], WGn[a]);
        }
      }
    };
    setNear(bd);
    for (auto* b : bd->near) setNear(b);
    for (Node* a = bd->parent; a; a = a->parent)
      for (auto* b : a->near)
        if (!b->has_children()) setNear(b);
    std::sort(tl.begin(), tl.end());
    C.near_idx[t] = tl;
    C.near_wG[t].resize(tl.size());
    C.near_wGn[t].resize(tl.size());
    for (size_t i = 0; i < tl.size(); ++i) {
      C.near_wG[t][i] = accG[tl[i]];
      C.near_wGn[t][i] = accGn[tl[i]];
    }
  }

  C.t_near = omp_get_wtime() - wt1;
  int nc = C.ncoef();
  for (auto& up : C.pool) {
    up->MM.assign(nc, {0., 0.});
    up->LL.assign(nc, {0., 0.});
  }
  R->MM.assign(nc, {0., 0.});
  R->LL.assign(nc, {0., 0.});
  return Cp;
}

void* oracle_create(int np, const double* X, int nf, const int* tri, const uint8_t* face_dirichlet, int ndof, const int* dof_point,
                    const int* dof_face, const int* dof_kind, const int* face_dof, int p, double theta, int max_points, int max_level) {
  return oracle_create_sampled(np, X, nf, tri, face_dirichlet, ndof, dof_point, dof_face, dof_kind, face_dof, p, theta, max_points,
                               max_level, 1);
}

void oracle_destroy(void* h) { delete (OracleCtx*)h; }

}  // extern "C"

namespace {

std::vector<Node*> all_nodes(OracleCtx& C) {
  std::vector<Node*> v;
  v.push_back(C.root.get());
  traverse_tree(C.root.get(), [&](Node* b) { v.push_back(b); });
  return v;
}

// One FMM update + per-point (near + far) integrals for given per-DOF phi/phin
// (moments.hpp:1547-1574; lib_multipole_expansion.hpp:1143-1150,1273-1302).
// stages: bit k runs stage k (0 P2M, 1 M2M, 2 M2L, 3 L2L, 4 near sums, 5 L2P); a stage that is
// skipped leaves the expansions and point sums of the previous call as they were.
void fmm_point_integrals(OracleCtx& C, const double* phi, const double* phin, std::vector<double>& GPhin, std::vector<double>& GnPhi,
                         int m2l_stride = 1, double* tstage = nullptr, unsigned stages = 0x3fu) {
  const int p = C.p;
  double tw = omp_get_wtime();
  auto lap = [&](int k) {
    const double n = omp_get_wtime();
    if (tstage) tstage[k] += n - tw;
    tw = n;
  };
  const int nc = C.ncoef();
  auto nodes = all_nodes(C);
  for (auto* b : nodes) {
    if (stages & 1u) std::fill(b->MM.begin(), b->MM.end(), std::array<cd, 2>{0., 0.});
    if (stages & 4u) std::fill(b->LL.begin(), b->LL.end(), std::array<cd, 2>{0., 0.});
  }
  // P2M at leaves (increment_M, moments.hpp:307-356)
#pragma omp parallel for schedule(dynamic, 4)
  for (size_t li = 0; li < ((stages & 1u) ? C.leaves.size() : 0); ++li) {
    Node* b = C.leaves[li];
    for (int sidx : b->data) {
      const Source& s = C.src[sidx];
      for (int q = 0; q < 6; ++q) {
        double w_phi = s.W[q] * (s.N[q][0] * phi[s.dof[0]] + s.N[q][1] * phi[s.dof[1]] + s.N[q][2] * phi[s.dof[2]]);
        double w_phin = s.W[q] * (s.N[q][0] * phin[s.dof[0]] + s.N[q][1] * phin[s.dof[1]] + s.N[q][2] * phin[s.dof[2]]);
        p2m_point(C, sub(s.q[q], b->X), s.normal, w_phin, w_phi, b->MM);
      }
    }
    conj_fill(p, b->MM);
  }
  lap(0);
  // M2M bottom-up (moments.hpp:401-436, 912-915)
  for (int level = C.max_level - 1; level >= 0 && (stages & 2u); --level) {
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t bi = 0; bi < C.level_nodes[level].size(); ++bi) {
      Node* b = C.level_nodes[level][bi];
      for (auto* c : b->children) {
        if (!c) continue;
        Sph S(sub(c->X, b->X));
        std::vector<cd> Yr(nc);
        for (int n = 0; n <= p; ++n)
          for (int m = -n; m <= n; ++m) Yr[n * (n + 1) + m] = S.Y_rho(n, m);
        for (int j = p; j >= 0; --j)
          for (int k = 0; k <= j; ++k)
            for (int n = j; n >= 0; --n)
              for (int m = -n; m <= n; ++m) {
                double a = C.aaa_m2m[C.aidx(j, k, n, m)];
                if (a == 0.0) continue;
                cd Rv = a * Yr[n * (n + 1) - m];
                int src = (j - n) * ((j - n) + 1) + (k - m);
                b->MM[j * (j + 1) + k][0] += Rv * c->MM[src][0];
                b->MM[j * (j + 1) + k][1] += Rv * c->MM[src][1];
              }
      }
      conj_fill(p, b->MM);
    }
  }
  lap(1);
  // M2L (moments.hpp:492-598, 732-764)
  for (auto& lv : C.level_nodes) {
    if (!(stages & 4u)) break;
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t ai = 0; ai < lv.size(); ++ai) {
      Node* A = lv[ai];
      if (A->l2m.empty()) continue;
      if (m2l_stride > 1 && (ai % m2l_stride) != 0) continue;
      std::vector<std::array<cd, 2>> acc(nc, {0., 0.});
      std::vector<cd> Ys((2 * p + 1) * (2 * p + 1));
      for (auto* B : A->l2m) {
        Sph S(sub(B->X, A->X));
        for (int l = 0; l <= 2 * p; ++l)
          for (int q = -l; q <= l; ++q) Ys[l * (l + 1) + q] = S.Y_div_rhon1(l, q);
        for (int j = 0; j <= p; ++j)
          for (int k = 0; k <= j; ++k) {
            cd s0 = 0., s1 = 0.;
            for (int n = 0; n <= p; ++n)
              for (int m = -n; m <= n; ++m) {
                double a = C.aaa_m2l[C.aidx(j, k, n, m)];
                if (a == 0.0) continue;
                int l = j + n, q = m - k;
                cd t = a * Ys[l * (l + 1) + q];
                s0 += t * B->MM[n * (n + 1) + m][0];
                s1 += t * B->MM[n * (n + 1) + m][1];
              }
            acc[j * (j + 1) + k][0] += s0;
            acc[j * (j + 1) + k][1] += s1;
          }
      }
      for (int i = 0; i < nc; ++i) {
        A->LL[i][0] += acc[i][0];
        A->LL[i][1] += acc[i][1];
      }
      conj_fill(p, A->LL);
    }
  }
  lap(2);
  // L2L top-down (moments.hpp:862-884, 925-929)
  for (auto& lv : C.level_nodes) {
    if (!(stages & 8u)) break;
#pragma omp parallel for schedule(dynamic, 1)
    for (size_t bi = 0; bi < lv.size(); ++bi) {
      Node* par = lv[bi];
      for (auto* c : par->children) {
        if (!c) continue;
        Sph S(sub(par->X, c->X));
        for (int j = p; j >= 0; --j)
          for (int k = 0; k <= j; ++k)
            for (int n = p; n >= j; --n)
              for (int m = -n; m <= n; ++m) {
                double a = C.aaa_l2l[C.aidx(j, k, n, m)];
                if (a == 0.0) continue;
                cd Rv = a * S.Y_rho(n - j, m - k);
                c->LL[j * (j + 1) + k][0] += Rv * par->LL[n * (n + 1) + m][0];
                c->LL[j * (j + 1) + k][1] += Rv * par->LL[n * (n + 1) + m][1];
              }
        conj_fill(p, c->LL);
      }
    }
  }
  lap(3);
  // per point near + far
  GPhin.assign(C.np, 0.0);
  GnPhi.assign(C.np, 0.0);
#pragma omp parallel for schedule(dynamic, 32)
  for (int t = 0; t < ((stages & 16u) ? C.np : 0); ++t) {
    double r0 = 0, r1 = 0;
    for (size_t i = 0; i < C.near_idx[t].size(); ++i) {
      r0 += phin[C.near_idx[t][i]] * C.near_wG[t][i];
      r1 += phi[C.near_idx[t][i]] * C.near_wGn[t][i];
    }
    GPhin[t] = r0;
    GnPhi[t] = r1;
  }
  lap(4);
#pragma omp parallel for schedule(dynamic, 32)
  for (int t = 0; t < ((stages & 32u) ? C.np : 0); ++t) {
    if (!C.tgt_leaf[t]) continue;
    Node* b = C.tgt_leaf[t];
    Sph S(sub(C.Xs[t], b->X));
    cd f0 = 0., f1 = 0.;
    for (int n = 0; n <= p; ++n)
      for (int m = -n; m <= n; ++m) {
        cd y = S.Y_rho(n, m);
        f0 += y * b->LL[n * (n + 1) + m][0];
        f1 += y * b->LL[n * (n + 1) + m][1];
      }
    GPhin[t] += f0.real();
    GnPhi[t] += f1.real();
  }
  lap(5);
}

void apply_rows(OracleCtx& C, const double* phi, const double* phin, double* Av) {
  std::vector<double> GPhin, GnPhi;
  fmm_point_integrals(C, phi, phin, GPhin, GnPhi);
  for (int i = 0; i < C.ndof; ++i) {
    int t = C.dof_point[i];
    if (C.dof_kind[i] == 2)
      Av[i] = phi[i];
    else
      Av[i] = GPhin[t] - (GnPhi[t] + C.diag[i] * phi[i]);
  }
}

}  // namespace

extern "C" {

// Rigid-mode diagonal (BEM_solveBVP_GMRES_FMM.hpp:2661-2716).
void oracle_compute_diag(void* h) {
  OracleCtx& C = *(OracleCtx*)h;
  std::vector<double> phi(C.ndof, 1.0), phin(C.ndof, 0.0), GPhin, GnPhi;
  fmm_point_integrals(C, phi.data(), phin.data(), GPhin, GnPhi);
  C.diag.assign(C.ndof, 1.0);
  for (int i = 0; i < C.ndof; ++i) {
    C.diag[i] = -GnPhi[C.dof_point[i]];
    if (std::abs(C.diag[i]) < 1e-15) C.diag[i] = 1.0;
  }
}

void oracle_get_diag(void* h, double* out) {
  OracleCtx& C = *(OracleCtx*)h;
  std::copy(C.diag.begin(), C.diag.end(), out);
}

// Per-point near+far integrals for arbitrary per-DOF phi/phin (scaled units).
void oracle_point_integrals(void* h, const double* phi, const double* phin, double* GPhin_out, double* GnPhi_out) {
  OracleCtx& C = *(OracleCtx*)h;
  std::vector<double> a, b;
  fmm_point_integrals(C, phi, phin, a, b);
  std::copy(a.begin(), a.end(), GPhin_out);
  std::copy(b.begin(), b.end(), GnPhi_out);
}

// Rows of the operator for per-DOF phi/phin (compute_Ax_minus_b, BEM_solveBVP_GMRES_FMM.hpp:34-158).
void oracle_apply(void* h, const double* phi, const double* phin, double* Av) { apply_rows(*(OracleCtx*)h, phi, phin, Av); }

// Direct (no FMM) evaluation of the far part: every non-near source by its 6 P2M points.
// Used to validate the regenerated translation operators (FMM vs direct).
void oracle_point_integrals_direct(void* h, const double* phi, const double* phin, double* GPhin_out, double* GnPhi_out) {
  OracleCtx& C = *(OracleCtx*)h;
#pragma omp parallel for schedule(dynamic, 16)
  for (int t = 0; t < C.np; ++t) {
    if (!C.tgt_leaf[t]) {
      GPhin_out[t] = GnPhi_out[t] = 0;
      continue;
    }
    // near set of faces
    std::vector<uint8_t> isnear(C.nf, 0);
    Node* bd = C.tgt_leaf[t];
    auto mark = [&](const Node* B) {
      for (int s : B->data) isnear[s] = 1;
    };
    mark(bd);
    for (auto* b : bd->near) mark(b);
    for (Node* a = bd->parent; a; a = a->parent)
      for (auto* b : a->near)
        if (!b->has_children()) mark(b);
    double r0 = 0, r1 = 0;
    for (size_t i = 0; i < C.near_idx[t].size(); ++i) {
      r0 += phin[C.near_idx[t][i]] * C.near_wG[t][i];
      r1 += phi[C.near_idx[t][i]] * C.near_wGn[t][i];
    }
    const V3 xt = C.Xs[t];
    for (int f = 0; f < C.nf; ++f) {
      if (isnear[f]) continue;
      const Source& s = C.src[f];
      for (int q = 0; q < 6; ++q) {
        double w_phi = s.W[q] * (s.N[q][0] * phi[s.dof[0]] + s.N[q][1] * phi[s.dof[1]] + s.N[q][2] * phi[s.dof[2]]);
        double w_phin = s.W[q] * (s.N[q][0] * phin[s.dof[0]] + s.N[q][1] * phin[s.dof[1]] + s.N[q][2] * phin[s.dof[2]]);
        V3 Rv = sub(s.q[q], xt);
        double r = std::sqrt(Rv[0] * Rv[0] + Rv[1] * Rv[1] + Rv[2] * Rv[2]);
        r0 += w_phin / r;
        r1 += w_phi * (-(Rv[0] * s.normal[0] + Rv[1] * s.normal[1] + Rv[2] * s.normal[2]) / (r * r * r));
      }
    }
    GPhin_out[t] = r0;
    GnPhi_out[t] = r1;
  }
}

struct OracleStats {
  int n_nodes, n_leaves, depth, n_added;
  long long m2l_pairs, near_pairs, nnz;
  double L, scale;
};

void oracle_stats(void* h, long long* out /*[8]*/, double* dout /*[2]*/, long long* per_level /*[max_level+1][3]*/) {
  OracleCtx& C = *(OracleCtx*)h;
  long long nodes = 0, m2l = 0, nearp = 0, nnz = 0;
  int depth = 0;
  for (size_t l = 0; l < C.level_nodes.size(); ++l) {
    long long lm = 0, ln = 0;
    for (auto* b : C.level_nodes[l]) {
      lm += b->l2m.size();
      ln += b->near.size();
    }
    if (per_level) {
      per_level[3 * l] = C.level_nodes[l].size();
      per_level[3 * l + 1] = lm;
      per_level[3 * l + 2] = ln;
    }
    nodes += C.level_nodes[l].size();
    m2l += lm;
    nearp += ln;
    if (!C.level_nodes[l].empty()) depth = (int)l;
  }
  for (auto& v : C.near_idx) nnz += v.size();
  out[0] = nodes;
  out[1] = C.leaves.size();
  out[2] = depth;
  out[3] = C.n_added;
  out[4] = m2l;
  out[5] = nearp;
  out[6] = nnz;
  out[7] = 0;
  dout[0] = C.L;
  dout[1] = C.scale;
}

// Per-face leaf identification: level and lower corner of the leaf that holds it
// (-1 if the face was dropped by the root InsideQ test).
void oracle_face_leaf(void* h, int* level, double* corner) {
  OracleCtx& C = *(OracleCtx*)h;
  for (int f = 0; f < C.nf; ++f) {
    level[f] = -1;
    corner[3 * f] = corner[3 * f + 1] = corner[3 * f + 2] = 0;
  }
  for (auto* b : C.leaves)
    for (int s : b->data) {
      level[s] = b->level;
      corner[3 * s] = b->bmin[0];
      corner[3 * s + 1] = b->bmin[1];
      corner[3 * s + 2] = b->bmin[2];
    }
}

// Near-field row of point t: returns length; copies up to cap entries.
int oracle_near_row(void* h, int t, int cap, int* idx, double* wG, double* wGn) {
  OracleCtx& C = *(OracleCtx*)h;
  int n = (int)C.near_idx[t].size();
  for (int i = 0; i < std::min(n, cap); ++i) {
    idx[i] = C.near_idx[t][i];
    wG[i] = C.near_wG[t][i];
    wGn[i] = C.near_wGn[t][i];
  }
  return n;
}

double oracle_scale_factor(void* h) { return ((OracleCtx*)h)->L; }

// Timing sample for the CPU baseline: set-up parts and one FMM mat-vec with M2L run for
// every m2l_stride-th target bucket (times scaled by the pair counts).  t[0..5]: P2M, M2M,
// M2L (scaled), L2L, near sums (scaled by near_stride), L2P; t[6]: tree+lists set-up,
// t[7]: near-field quadrature (scaled by near_stride); t[8]: OpenMP threads.
void oracle_time_sample(void* h, int m2l_stride, double* t) {
  OracleCtx& C = *(OracleCtx*)h;
  std::vector<double> phi(C.ndof, 1.0), phin(C.ndof, 0.5), a, b;
  for (int k = 0; k < 9; ++k) t[k] = 0.0;
  fmm_point_integrals(C, phi.data(), phin.data(), a, b, m2l_stride, t);
  long long all = 0, sampled = 0;
  for (auto& lv : C.level_nodes)
    for (size_t ai = 0; ai < lv.size(); ++ai) {
      all += lv[ai]->l2m.size();
      if (m2l_stride <= 1 || ai % m2l_stride == 0) sampled += lv[ai]->l2m.size();
    }
  if (sampled > 0) t[2] *= (double)all / (double)sampled;
  t[4] *= C.near_stride;
  t[6] = C.t_tree;
  t[7] = C.t_near * C.near_stride;
  t[8] = omp_get_max_threads();
}

// Wall time (s) of ONE whole stage of the mat-vec on the whole problem (stage as in
// fmm_point_integrals: 0 P2M, 1 M2M, 2 M2L, 3 L2L, 4 near sums, 5 L2P), with all OpenMP
// threads; the stage reads the expansions the previous call left.  For the CPU baseline.
double oracle_time_stage(void* h, int stage) {
  OracleCtx& C = *(OracleCtx*)h;
  if (stage < 0 || stage > 5) return -1.0;
  std::vector<double> phi(C.ndof, 1.0), phin(C.ndof, 0.5), a, b;
  double t[9] = {0};
  fmm_point_integrals(C, phi.data(), phin.data(), a, b, 1, t, 1u << stage);
  return t[stage];
}

// Wall time (s) of the set-up parts that were measured when the context was created:
// out[0] tree + lists, out[1] near-field quadrature (every point; the context must have been
// created with near_stride 1), out[2] OpenMP threads.
void oracle_setup_times(void* h, double* out) {
  OracleCtx& C = *(OracleCtx*)h;
  out[0] = C.t_tree;
  out[1] = C.t_near * C.near_stride;
  out[2] = omp_get_max_threads();
}

// GMRES solve (BEM_solveBVP_GMRES_FMM.hpp:2007-2400; basic_linear_systems.hpp:3137-3451).
// known[i]: phi (Dirichlet DOF) or phin (Neumann DOFs) in physical units;
// corner_phi[i]: phi of the point for corner-Neumann rows.  Outputs per-DOF phi and
// phin in physical units.  stats: [iters, r_true, r_est, converged].
int oracle_solve(void* h, const double* known, const double* x0_in, double tol, int max_iter, double* out_phi, double* out_phin, double* stats) {
  OracleCtx& C = *(OracleCtx*)h;
  const int N = C.ndof;
  if (C.diag.empty()) oracle_compute_diag(h);
  // copyToFMM: Neumann phin scaled by L
  std::vector<double> kphi(N, 0.0), kphin(N, 0.0), corner_rhs(N, 0.0);
  std::vector<int> point_dir_dof(C.np, -1);
  for (int i = 0; i < N; ++i)
    if (C.dof_kind[i] == 0) point_dir_dof[C.dof_point[i]] = i;
  for (int i = 0; i < N; ++i) {
    if (C.dof_kind[i] == 0)
      kphi[i] = known[i];
    else
      kphin[i] = known[i] * C.L;
  }
  auto Aop = [&](const std::vector<double>& v) {
    std::vector<double> phi(N), phin(N), out(N);
    for (int i = 0; i < N; ++i) {
      if (C.dof_kind[i] == 0) {
        phin[i] = v[i];
        phi[i] = 0.0;
      } else {
        phi[i] = v[i];
        phin[i] = 0.0;
      }
    }
    apply_rows(C, phi.data(), phin.data(), out.data());
    return out;
  };
  // b = -(A*0 - b)
  std::vector<double> b(N);
  {
    std::vector<double> phi(N), phin(N);
    for (int i = 0; i < N; ++i) {
      phi[i] = (C.dof_kind[i] == 0) ? kphi[i] : 0.0;
      phin[i] = (C.dof_kind[i] == 0) ? 0.0 : kphin[i];
    }
    apply_rows(C, phi.data(), phin.data(), b.data());
    for (auto& x : b) x = -x;
    for (int i = 0; i < N; ++i)
      if (C.dof_kind[i] == 2) {
        int d = point_dir_dof[C.dof_point[i]];
        b[i] = (d >= 0) ? known[d] : 0.0;
      }
  }
  auto dot = [](const std::vector<double>& a, const std::vector<double>& c) {
    double s = 0;
    for (size_t i = 0; i < a.size(); ++i) s = std::fma(a[i], c[i], s);
    return s;
  };
  auto nrm = [&](const std::vector<double>& a) { return std::sqrt(dot(a, a)); };
  std::vector<double> x(N, 0.0);
  if (x0_in) x.assign(x0_in, x0_in + N);
  // run_gmres: restart from the current x after a saturation break
  // (BEM_solveBVP_GMRES_FMM.hpp:2275-2355, gmres ctor basic_linear_systems.hpp:3339)
  int iters = 0;
  double r_true = 1e300, err = 1e300;
  const int restart_max = 100;  // solver_restart default (main_time_domain.cpp:51)
  while (iters < max_iter && r_true > tol) {
    const int remaining = max_iter - iters;
    const int k_cycle_max = std::min(restart_max, remaining);
    std::vector<double> xb = x;
    std::vector<double> r0 = Aop(xb);
    for (int i = 0; i < N; ++i) r0[i] = b[i] - r0[i];
    double beta = nrm(r0);
    if (beta == 0.0) {
      r_true = 0.0;
      err = 0.0;
      break;
    }
    std::vector<std::vector<double>> V;
    std::vector<double> v0(N);
    for (int i = 0; i < N; ++i) v0[i] = r0[i] / beta;
    V.push_back(v0);
    std::vector<double> cs, sn, g{beta};
    std::vector<std::vector<double>> Rm;  // columns of R
    auto add_basis = [&]() {
      std::vector<double> w = Aop(V.back());
      int n = (int)V.size();
      std::vector<double> hcol(n + 1, 0.0);
      for (int i = 0; i < n; ++i) {
        double hh = dot(V[i], w);
        hcol[i] = hh;
        for (int k = 0; k < N; ++k) w[k] = std::fma(-hh, V[i][k], w[k]);
      }
      hcol[n] = nrm(w);
      for (int k = 0; k < N; ++k) w[k] /= hcol[n];
      V.push_back(w);
      for (int i = 0; i < n - 1; ++i) {
        double t = std::fma(cs[i], hcol[i], sn[i] * hcol[i + 1]);
        hcol[i + 1] = std::fma(cs[i], hcol[i + 1], -sn[i] * hcol[i]);
        hcol[i] = t;
      }
      double a = hcol[n - 1], bb = hcol[n];
      double r = std::hypot(a, bb), c = 1.0, s = 0.0;
      if (r != 0.0) {
        c = a / r;
        s = bb / r;
      }
      cs.push_back(c);
      sn.push_back(s);
      {
        double t = std::fma(c, hcol[n - 1], s * hcol[n]);
        hcol[n] = std::fma(c, hcol[n], -s * hcol[n - 1]);
        hcol[n - 1] = t;
      }
      g.push_back(0.0);
      {
        double t = std::fma(c, g[n - 1], s * g[n]);
        g[n] = std::fma(c, g[n], -s * g[n - 1]);
        g[n - 1] = t;
      }
      Rm.push_back(hcol);
      err = std::abs(g.back());
    };
    auto update_solution = [&]() {
      int n = (int)Rm.size();
      std::vector<double> y(n, 0.0);
      for (int i = n - 1; i >= 0; --i) {
        double s = g[i];
        for (int j = i + 1; j < n; ++j) s -= Rm[j][i] * y[j];
        y[i] = s / Rm[i][i];
      }
      x = xb;
      for (int i = 0; i < n; ++i)
        for (int k = 0; k < N; ++k) x[k] = std::fma(y[i], V[i][k], x[k]);
    };
    auto true_residual = [&]() {
      std::vector<double> ax = Aop(x);
      for (int i = 0; i < N; ++i) ax[i] -= b[i];
      return nrm(ax);
    };
    add_basis();
    iters += 1;
    int sat = 0;
    while (true) {
      add_basis();
      ++iters;
      if (err <= tol * 10.) {
        update_solution();
        r_true = true_residual();
        if (r_true <= tol) break;
        if (sat++ >= 5) break;
      }
      if (iters >= max_iter && (int)Rm.size() >= k_cycle_max) {
        update_solution();
        r_true = (err <= tol * 10.) ? true_residual() : err;
        break;
      }
    }
  }
  for (int i = 0; i < N; ++i) {
    if (C.dof_kind[i] == 0) {
      out_phi[i] = known[i];
      out_phin[i] = x[i] / C.L;
    } else {
      out_phi[i] = x[i];
      out_phin[i] = known[i];
    }
  }
  if (stats) {
    stats[0] = iters;
    stats[1] = r_true;
    stats[2] = err;
    stats[3] = (r_true <= tol) ? 1.0 : 0.0;
  }
  return 0;
}

}  // extern "C"
