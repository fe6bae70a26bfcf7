// Test infrastructure only: drives the UNMODIFIED reference BEM_BVP GMRES-FMM path
// (bem/BEM_solveBVP.hpp, bem/BEM_solveBVP_GMRES_FMM.hpp) on a mesh given as flat arrays,
// and dumps its intermediate and final results for the oracle's parity tests.
//
// It replaces the reference's application driver (bem/main_time_domain.cpp): it defines
// the globals that BEM_solveBVP.hpp declares extern (main_time_domain.cpp:25-62), builds a
// Network from an OBJ file, sets face/point boundary flags the way setBoundaryTypes does
// (BEM_setBoundaryTypes.hpp:555-562, 434-441), assigns phi/phin per DOF key (the analytic
// linear Stokes potential; the reference's own setPhiPhinOnFace would take phin from the
// contact velocity, which is zero for a fixed tank), then runs the body of BEM_BVP::solve()
// for solver_type == "GMRES" (BEM_solveBVP.hpp:565-630).
//
// Usage: ref_harness INPUT.bin OUTPUT.txt WORKDIR
#include "pch.hpp"

bool use_linear_element = true;
bool use_pseudo_quadratic_element = false;
bool use_true_quadratic_element = false;
std::string solver_type = "GMRES";
std::string coupling_type = "NONE";
double coupling_tol = 1e-10;
std::vector<double> coupling_params;
std::string preconditioner_type = "NONE";
std::string ilu_neighborhood_type = "BUCKETS";
int ilu_kring_num = 1;
double milu_omega = 1.0;
double ilut_drop_tol = 1e-3;
int ilut_max_entries_per_row = 50;
double ilut_pivot_min = 1e-12;
int schwarz_core_k = 1;
int schwarz_overlap_k = 1;
int schwarz_max_core_size = 64;
int schwarz_max_block_size = 128;
double schwarz_pivot_min = 1e-12;
double schwarz_diag_shift = 0.0;
double solver_tol = 1e-10;
int solver_max_iter = 500;
int solver_restart = 100;
int fmm_max_level = 7;
int fmm_bucket_max_points = 30;
std::string nearfield_mode = "scalar";
int g_p2m_quadrature_points = 6;
double g_mac_theta = 0.25;
int time_step;
double simulation_time = 0;

#define BEM
#define simulation
#include "Network.hpp"
#include "BEM_BoundaryValues.hpp"
#include "BEM_setBoundaryTypes.hpp"
#include "BEM_solveBVP.hpp"

#include <cstdio>
#include <map>

struct Input {
  int np = 0, nf = 0, max_iter = 500;
  double A = 0, k = 0, depth = 0, g = 9.81, tol = 1e-10;
  std::vector<double> X;
  std::vector<int> tri;
  std::vector<unsigned char> fdir;
  std::vector<double> v_phi, v_phin;  // optional test vector per (point, face-slot) for a mat-vec dump
};

static Input read_input(const char* path) {
  Input in;
  FILE* fp = std::fopen(path, "rb");
  if (!fp) throw std::runtime_error("cannot open input");
  auto rd = [&](void* p, size_t sz) {
    if (std::fread(p, 1, sz, fp) != sz) throw std::runtime_error("short read");
  };
  rd(&in.np, 4);
  rd(&in.nf, 4);
  rd(&in.max_iter, 4);
  double prm[5];
  rd(prm, sizeof prm);
  in.A = prm[0];
  in.k = prm[1];
  in.depth = prm[2];
  in.g = prm[3];
  in.tol = prm[4];
  in.X.resize(3 * in.np);
  in.tri.resize(3 * in.nf);
  in.fdir.resize(in.nf);
  rd(in.X.data(), 8 * in.X.size());
  rd(in.tri.data(), 4 * in.tri.size());
  rd(in.fdir.data(), in.fdir.size());
  std::fclose(fp);
  return in;
}

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s INPUT.bin OUTPUT.txt WORKDIR\n", argv[0]);
    return 2;
  }
  Input in = read_input(argv[1]);
  solver_tol = in.tol;
  solver_max_iter = in.max_iter;
  std::string work = argv[3];
  std::filesystem::create_directories(work);
  std::string obj = work + "/mesh.obj";
  {
    FILE* fp = std::fopen(obj.c_str(), "w");
    for (int i = 0; i < in.np; ++i) std::fprintf(fp, "v %.17g %.17g %.17g\n", in.X[3 * i], in.X[3 * i + 1], in.X[3 * i + 2]);
    for (int f = 0; f < in.nf; ++f) std::fprintf(fp, "f %d %d %d\n", in.tri[3 * f] + 1, in.tri[3 * f + 1] + 1, in.tri[3 * f + 2] + 1);
    std::fclose(fp);
  }
  auto* water = new Network(obj, "water");

  // map reference points/faces back to input indices by exact coordinates
  std::map<std::array<double, 3>, int> pmap;
  for (int i = 0; i < in.np; ++i) pmap[{in.X[3 * i], in.X[3 * i + 1], in.X[3 * i + 2]}] = i;
  std::unordered_map<networkPoint*, int> pid;
  for (auto* p : water->getPoints()) {
    auto it = pmap.find(p->X);
    if (it == pmap.end()) throw std::runtime_error("point not matched");
    pid[p] = it->second;
  }
  std::map<std::array<int, 3>, int> fmap;
  for (int f = 0; f < in.nf; ++f) {
    std::array<int, 3> key{in.tri[3 * f], in.tri[3 * f + 1], in.tri[3 * f + 2]};
    std::sort(key.begin(), key.end());
    fmap[key] = f;
  }
  std::unordered_map<networkFace*, int> fid;
  for (auto* f : water->getFaces()) {
    auto [p0, p1, p2] = f->getPoints();
    std::array<int, 3> key{pid[p0], pid[p1], pid[p2]};
    std::sort(key.begin(), key.end());
    fid[f] = fmap.at(key);
  }

  // boundary flags: face from input, point/line by the reference's step3/step4 rules
  water->setGeometricPropertiesForce();
  for (auto* f : water->getBoundaryFaces()) {
    f->Dirichlet = in.fdir[fid[f]] != 0;
    f->Neumann = !f->Dirichlet;
    f->isLinearElement = true;
    f->isPseudoQuadraticElement = false;
    f->isTrueQuadraticElement = false;
  }
  for (auto* l : water->getLines()) {
    l->Neumann = std::ranges::all_of(l->getBoundaryFaces(), [](const auto& f) { return f->Neumann; });
    bool hd = std::ranges::any_of(l->getBoundaryFaces(), [](const auto& f) { return f->Dirichlet; });
    bool hn = std::ranges::any_of(l->getBoundaryFaces(), [](const auto& f) { return f->Neumann; });
    l->CORNER = !l->Neumann && hd && hn;
    l->Dirichlet = !l->Neumann && !l->CORNER;
  }
  for (auto* p : water->getPoints()) {
    p->Neumann = std::ranges::all_of(p->getBoundaryFaces(), [](const auto& f) { return f->Neumann; });
    p->Dirichlet = std::ranges::all_of(p->getBoundaryFaces(), [](const auto& f) { return f->Dirichlet; });
    p->CORNER = (!p->Neumann && !p->Dirichlet);
    setIsMultipleNode(p);
  }

  const double omega = std::sqrt(in.g * in.k * std::tanh(in.k * in.depth));
  const double c = in.g * in.A / omega / std::cosh(in.k * in.depth);
  auto phi_at = [&](const Tddd& X) { return c * std::cosh(in.k * (X[2] + in.depth)) * std::sin(in.k * X[0]); };
  auto grad_at = [&](const Tddd& X) {
    return Tddd{c * in.k * std::cosh(in.k * (X[2] + in.depth)) * std::cos(in.k * X[0]), 0.0,
                c * in.k * std::sinh(in.k * (X[2] + in.depth)) * std::sin(in.k * X[0])};
  };
  auto pnormal = [](networkPoint* p) {
    Tddd n = {0., 0., 0.};
    for (auto* f : p->getBoundaryFaces()) n += f->area * f->normal;
    return Normalize(n);
  };

  std::vector<Network*> WATERS{water};
  BEM_BVP bvp(WATERS);
  bvp.output_directory = work;
  // BEM_BVP::solve() body (BEM_solveBVP.hpp:565-630), GMRES branch
  bvp.matrix_size = setNodeFaceIndices(WATERS);
  for (auto* p : water->getPoints()) {
    p->phiOnFace.clear();
    p->phinOnFace.clear();
    p->phitOnFace.clear();
    p->phintOnFace.clear();
    const double ph = phi_at(p->X);
    std::get<0>(p->phiphin) = ph;
    for (const auto& [f, i] : p->f2Index) {
      if (isDirichletID_BEM(p, f)) {
        p->phiOnFace[f] = ph;
        p->phinOnFace[f] = 0.0;  // initial guess of the unknown
      } else {
        Tddd n = f ? f->normal : pnormal(p);
        p->phinOnFace[f] = Dot(grad_at(p->X), n);
        p->phiOnFace[f] = 0.0;  // initial guess of the unknown
      }
      p->phitOnFace[f] = 1E+30;
      p->phintOnFace[f] = 1E+30;
    }
  }
  TimeWatch watch;
  double t_setup = 0, t_solve = 0;
  bvp.solveGMRES(watch, t_setup, t_solve);

  FILE* out = std::fopen(argv[2], "w");
  std::fprintf(out, "time_setup %.6f\ntime_solve %.6f\n", t_setup, t_solve);
  std::fprintf(out, "gmres_iter %d\n", bvp.last_gmres_total_iter);
  std::fprintf(out, "matrix_size %d\n", (int)bvp.matrix_size);
  // DOF key -> index, and solution (physical units)
  std::vector<std::tuple<int, int, int>> keys;  // point, face, index
  for (auto* p : water->getPoints())
    for (const auto& [f, i] : p->f2Index) keys.emplace_back(pid[p], f ? fid[f] : -1, i);
  std::sort(keys.begin(), keys.end());
  std::fprintf(out, "dofs %zu\n", keys.size());
  for (auto& [pp, ff, ii] : keys) std::fprintf(out, "%d %d %d %.17g %.17g\n", pp, ff, ii, bvp.ans[ii], bvp.diag_coeffs[ii]);
  // tree: leaf of each source
  std::fprintf(out, "leaves %zu\n", bvp.B_poles.deepest_level_buckets.size());
  std::vector<std::tuple<int, int, double, double, double>> leafs;
  for (auto* b : bvp.B_poles.deepest_level_buckets)
    for (auto& s : b->data1D_vector) {
      // identify the source's face by its tree position
      (void)s;
    }
  {
    std::unordered_map<const void*, int> src_face;
    for (auto* f : water->getBoundaryFaces())
      for (auto& s : f->sources) src_face[s.get()] = fid[f];
    for (auto* b : bvp.B_poles.deepest_level_buckets)
      for (auto& s : b->data1D_vector) leafs.emplace_back(src_face[s.get()], b->level, b->xmin, b->ymin, b->zmin);
    std::sort(leafs.begin(), leafs.end());
    std::fprintf(out, "face_leaf %zu\n", leafs.size());
    for (auto& [f, l, x, y, z] : leafs) std::fprintf(out, "%d %d %.17g %.17g %.17g\n", f, l, x, y, z);
  }
  // near rows per point: (dof index, wG, wGn)
  {
    std::fprintf(out, "near_rows %zu\n", water->getPoints().size());
    for (auto* p : water->getPoints()) {
      std::fprintf(out, "%d %zu\n", pid[p], p->near_indices.size());
      for (size_t i = 0; i < p->near_indices.size(); ++i)
        std::fprintf(out, "%d %.17g %.17g\n", p->near_indices[i], p->near_weights_phi[i], p->near_weights_phin[i]);
    }
  }
  // one mat-vec with a deterministic unknown vector v_i = sin(1.7 i + 0.3) (index space)
  {
    std::vector<double> v(bvp.matrix_size);
    for (size_t i = 0; i < v.size(); ++i) v[i] = std::sin(1.7 * (double)i + 0.3);
    bvp.setUnknowns(v);
    bvp.setKnowns(0.);
    auto Av = bvp.compute_Ax_minus_b();
    std::fprintf(out, "matvec %zu\n", Av.size());
    for (size_t i = 0; i < Av.size(); ++i) std::fprintf(out, "%.17g\n", Av[i]);
  }
  std::fprintf(out, "L %.17g\n", water->getScaleFactor());
  // the MEL stage quantities of the solution: point phi (storePhiPhin), the velocity gradPhi
  // (BEM_BoundaryValues.hpp:565, set as set_u_potential_BEM does, BEM_calculateVelocities.hpp:
  // 1027-1031) and Dphi/Dt with the node moving with the fluid and zero pressure
  // (Network.hpp:224-235); physical units
  {
    for (auto* p : water->getPoints()) p->u_potential_BEM = gradPhi(p);  // the point loop of set_u_potential_BEM
    std::vector<std::tuple<int, double, Tddd, double>> mel;
    for (auto* p : water->getPoints())
      mel.emplace_back(pid[p], std::get<0>(p->phiphin), p->u_potential_BEM, p->DphiDt(p->u_potential_BEM, 0.));
    std::sort(mel.begin(), mel.end(), [](const auto& a, const auto& b) { return std::get<0>(a) < std::get<0>(b); });
    std::fprintf(out, "mel %zu\n", mel.size());
    for (auto& [pp, ph, u, dd] : mel) std::fprintf(out, "%d %.17g %.17g %.17g %.17g %.17g\n", pp, ph, u[0], u[1], u[2], dd);
  }
  std::fclose(out);
  return 0;
}
