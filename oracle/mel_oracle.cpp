// Oracle (test infrastructure): CPU restatement of the reference's MEL stage update that
// follows each boundary-value solve, for linear triangles.  Checker only: imported by tests.
//
//   storePhiPhinCommon point averaging   bem/BEM_setBoundaryTypes.hpp:952-983
//   gradPhi(const networkPoint*)         bem/BEM_BoundaryValues.hpp:500-563
//   gradP1 (triangle)                     lib/include/basic_vectors.hpp:2112-2128
//   optimalVector                         lib/include/rootFinding.hpp:119-205
//   DphiDt / DphiDt_damped                lib/include/Network.hpp:224-235
//   RungeKuttaCommon::push (steps = 4)    lib/include/integrationOfODE.hpp:227-300
//   pushPhi / pushPosition guards         bem/main_time_domain.cpp:2410-2440
#include <array>
#include <cmath>
#include <cstdint>
#include <vector>

namespace {

using V3 = std::array<double, 3>;
V3 sub(const V3& a, const V3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
V3 cross(const V3& a, const V3& b) { return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]}; }
double dot(const V3& a, const V3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
V3 normalize(V3 a) {
  const double n = std::sqrt(dot(a, a));
  if (n > 0)
    for (auto& v : a) v /= n;
  return a;
}

struct Surface {
  int np, nf;
  const double* X;
  const int32_t* tri;
  const uint8_t* fdir;
  const uint8_t* flags;
  const int32_t* face_dof;
  const double* phi;
  const double* phin;
  std::vector<std::vector<std::pair<int, int>>> pfaces;  // (face, vertex slot), ascending face
  std::vector<V3> normal;
  std::vector<double> area;
  V3 x(int p) const { return {X[3 * p], X[3 * p + 1], X[3 * p + 2]}; }
  void build() {
    pfaces.assign(np, {});
    normal.resize(nf);
    area.resize(nf);
    for (int f = 0; f < nf; ++f) {
      for (int a = 0; a < 3; ++a) pfaces[tri[3 * f + a]].push_back({f, a});
      const V3 c = cross(sub(x(tri[3 * f + 1]), x(tri[3 * f])), sub(x(tri[3 * f + 2]), x(tri[3 * f])));
      area[f] = 0.5 * std::sqrt(dot(c, c));
      normal[f] = normalize(c);
    }
  }
  // point phi after storePhiPhin: all-Neumann points average phiOnFace by face area
  double point_phi(int p) const {
    if (flags[p] & 1) {
      double tot = 0, s = 0;
      for (auto [f, a] : pfaces[p]) {
        tot += area[f];
        s += phi[face_dof[3 * f + a]] * area[f];
      }
      return pfaces[p].empty() ? 0.0 : s / tot;
    }
    for (auto [f, a] : pfaces[p])
      if (fdir[f]) return phi[face_dof[3 * f + a]];
    return 0.0;
  }
};

V3 grad_p1(const V3& X0, const V3& X1, const V3& X2, double v0, double v1, double v2) {
  const V3 ex = normalize(sub(X1, X0)), ez = normalize(cross(sub(X1, X0), sub(X2, X0))), ey = normalize(cross(ez, ex));
  const double x1 = std::sqrt(dot(sub(X1, X0), sub(X1, X0))), x2 = dot(sub(X2, X0), ex), y2 = dot(sub(X2, X0), ey);
  const double a = (-v0 + v1) / x1, b = (v2 * x1 - v1 * x2 + v0 * (-x1 + x2)) / (x1 * y2);
  return {a * ex[0] + b * ey[0], a * ex[1] + b * ey[1], a * ex[2] + b * ey[2]};
}

// the weighted least-squares vector the Newton iteration of optimalVector converges to, by
// Gaussian elimination with partial pivoting on the normal equations
V3 optimal_vector(const std::vector<double>& v, const std::vector<V3>& d, const std::vector<double>& w) {
  double mean = 0;
  for (double s : v) mean += std::abs(s);
  if (mean == 0) return {0, 0, 0};
  double M[3][4] = {};
  for (size_t i = 0; i < v.size(); ++i) {
    const V3 n = normalize(d[i]);
    for (int r = 0; r < 3; ++r) {
      for (int c = 0; c < 3; ++c) M[r][c] += w[i] * n[r] * n[c];
      M[r][3] += w[i] * n[r] * v[i];
    }
  }
  for (int c = 0; c < 3; ++c) {
    int piv = c;
    for (int r = c + 1; r < 3; ++r)
      if (std::abs(M[r][c]) > std::abs(M[piv][c])) piv = r;
    for (int k = 0; k < 4; ++k) std::swap(M[c][k], M[piv][k]);
    for (int r = c + 1; r < 3; ++r) {
      const double f = M[r][c] / M[c][c];
      for (int k = c; k < 4; ++k) M[r][k] -= f * M[c][k];
    }
  }
  V3 u{};
  for (int r = 2; r >= 0; --r) {
    double s = M[r][3];
    for (int k = r + 1; k < 3; ++k) s -= M[r][k] * u[k];
    u[r] = s / M[r][r];
  }
  return u;
}

V3 grad_phi(const Surface& S, const std::vector<double>& pphi, int p) {
  if (S.pfaces[p].empty()) return {0, 0, 0};
  std::vector<double> vs, W;
  std::vector<V3> dirs;
  const V3 E[3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
  for (auto [f, a] : S.pfaces[p]) {
    const int* t = S.tri + 3 * f;
    V3 u = grad_p1(S.x(t[0]), S.x(t[1]), S.x(t[2]), pphi[t[0]], pphi[t[1]], pphi[t[2]]);
    const double pn = S.phin[S.face_dof[3 * f + a]];
    for (int j = 0; j < 3; ++j) u[j] += pn * S.normal[f][j];
    for (int j = 0; j < 3; ++j) {
      vs.push_back(dot(u, E[j]));
      dirs.push_back(E[j]);
      W.push_back(S.area[f]);
    }
  }
  double meanW = 0;
  for (double w : W) meanW += w;
  meanW /= W.size();
  if (S.flags[p] & 4)
    for (auto [f, a] : S.pfaces[p]) {
      if (S.fdir[f] || !(S.area[f] > 0)) continue;
      vs.push_back(S.phin[S.face_dof[3 * f + a]]);
      dirs.push_back(S.normal[f]);
      W.push_back(10. * meanW);
    }
  return optimal_vector(vs, dirs, W);
}

// RK4 (steps = 4) with the list of increments f dt, as RungeKuttaCommon keeps it
double rk4_x(int stage, double dt, double x0, const std::vector<double>& dX, double f) {
  switch (stage) {
    case 0:
    case 1:
      return x0 + f * (dt / 2.0);
    case 2:
      return x0 + f * dt;
    default:
      return x0 + (dX[0] + 2.0 * dX[1] + 2.0 * dX[2] + dX[3]) / 6.0;
  }
}

}  // namespace

extern "C" {

int oracle_mel_velocity(int np, const double* X, int nf, const int32_t* tri, const uint8_t* fdir, const uint8_t* flags, const int32_t* face_dof,
                        const double* phi, const double* phin, double* out_phi_point, double* out_u) {
  Surface S{np, nf, X, tri, fdir, flags, face_dof, phi, phin, {}, {}, {}};
  S.build();
  std::vector<double> pphi(np);
  for (int p = 0; p < np; ++p) pphi[p] = S.point_phi(p);
  for (int p = 0; p < np; ++p) {
    const V3 u = grad_phi(S, pphi, p);
    for (int j = 0; j < 3; ++j) out_u[3 * p + j] = u[j];
    if (out_phi_point) out_phi_point[p] = pphi[p];
  }
  return 0;
}

// rk_dX: the caller's list of increments, [4][n_points][4] (x, y, z, phi) per stage
int oracle_mel_stage(int np, const double* X, int nf, const int32_t* tri, const uint8_t* fdir, const uint8_t* flags, const int32_t* face_dof,
                     const double* phi, const double* phin, int stage, double dt, double gravity, double* rk_X0, double* rk_phi0,
                     double* rk_dX, double* out_X, double* out_phi, double* out_u, double* out_dphidt) {
  Surface S{np, nf, X, tri, fdir, flags, face_dof, phi, phin, {}, {}, {}};
  S.build();
  std::vector<double> pphi(np);
  for (int p = 0; p < np; ++p) pphi[p] = S.point_phi(p);
  for (int p = 0; p < np; ++p) {
    if (stage == 0) {
      for (int j = 0; j < 3; ++j) rk_X0[3 * p + j] = X[3 * p + j];
      rk_phi0[p] = pphi[p];
    }
    const V3 u = grad_phi(S, pphi, p);
    auto incr = [&](int k) { return rk_dX + (size_t)k * np * 4 + (size_t)p * 4; };  // stage k, point p
    double rate = 0;
    if (!(flags[p] & 1)) {
      rate = -0.5 * dot(u, u) - gravity * X[3 * p + 2] - 0.0 + dot(u, u);  // pressure 0, u_node = u
      if (!std::isfinite(rate)) rate = 0;
      incr(stage)[3] = rate * dt;
      std::vector<double> l(4);
      for (int k = 0; k < 4; ++k) l[k] = incr(k)[3];
      out_phi[p] = rk4_x(stage, dt, rk_phi0[p], l, rate);
    } else {
      out_phi[p] = pphi[p];
    }
    for (int j = 0; j < 3; ++j) {
      incr(stage)[j] = u[j] * dt;
      std::vector<double> l(4);
      for (int k = 0; k < 4; ++k) l[k] = incr(k)[j];
      out_X[3 * p + j] = rk4_x(stage, dt, rk_X0[3 * p + j], l, u[j]);
    }
    for (int j = 0; j < 3; ++j) out_u[3 * p + j] = u[j];
    out_dphidt[p] = rate;
  }
  return 0;
}

}  // extern "C"
