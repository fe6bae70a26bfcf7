// Mixed-Eulerian-Lagrangian stage update on the device: the step of a BEM-MEL time step that
// follows each boundary-value solve (set_u_potential_BEM, DphiDt_damped, pushPhi and
// pushPosition; bem/BEM_calculateVelocities.hpp:1027-1044, lib/include/Network.hpp:224-235,
// bem/main_time_domain.cpp:2410-2510).
//
//   k_face_geom    unit normal and area of every surface triangle
//   k_point_phi    phi of every point from the per-DOF solution (storePhiPhin,
//                  bem/BEM_setBoundaryTypes.hpp:952-983): all-Neumann points take the
//                  area-weighted mean of their face DOFs, the others their point DOF
//   k_grad_phi     velocity of every point (gradPhi(p), bem/BEM_BoundaryValues.hpp:500-563):
//                  per adjacent face the linear-triangle surface gradient of phi plus phin
//                  times the face normal, combined by the area-weighted least-squares fit that
//                  optimalVector (lib/include/rootFinding.hpp:119-205) converges to; CORNER
//                  points add the Neumann faces' phin along their normals with weight 10x the
//                  mean face area
//   k_mel_push     Dphi/Dt = -|u|^2/2 - g z + u_node . u - gamma (phi - phi_ref) on points that
//                  are not all-Neumann, then the classical RK4 stage update of phi and of the
//                  point position (RungeKuttaCommon::push, lib/include/integrationOfODE.hpp:227-300)
//
// Thread per face or per point; all FP64.  Host arrays in and out (bem_gpu_mel_stage), the
// device buffers belong to a bem_gpu_mel context and keep their allocation between calls.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/bem_b200.h"

namespace {

template <typename T>
struct MBuf {
  T* p = nullptr;
  size_t cap = 0;
  ~MBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t reserve(size_t n) {
    if (n <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void**)&p, sizeof(T) * std::max<size_t>(n, 1));
    if (e == cudaSuccess) cap = n;
    return e;
  }
};

__device__ __forceinline__ void v3cross(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ __forceinline__ double v3dot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
__device__ __forceinline__ void v3unit(double* a) {
  const double n = sqrt(v3dot(a, a));
  if (n > 0.0) {
    a[0] /= n;
    a[1] /= n;
    a[2] /= n;
  }
}

__global__ void k_face_geom(int nf, const int32_t* __restrict__ tri, const double* __restrict__ X, double* __restrict__ normal,
                            double* __restrict__ area) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= nf) return;
  const double* a = X + 3 * tri[3 * f];
  const double* b = X + 3 * tri[3 * f + 1];
  const double* c = X + 3 * tri[3 * f + 2];
  double ba[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, ca[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]}, n[3];
  v3cross(ba, ca, n);
  area[f] = 0.5 * sqrt(v3dot(n, n));
  v3unit(n);
  normal[3 * f] = n[0];
  normal[3 * f + 1] = n[1];
  normal[3 * f + 2] = n[2];
}

// point flags: 1 all-Neumann, 2 all-Dirichlet, 4 CORNER
__global__ void k_point_phi(int np, const int32_t* __restrict__ pf_off, const int32_t* __restrict__ pf_face,
                            const int8_t* __restrict__ pf_slot, const int32_t* __restrict__ face_dof, const uint8_t* __restrict__ face_dir,
                            const uint8_t* __restrict__ flags, const double* __restrict__ area, const double* __restrict__ phi_dof,
                            double* __restrict__ phi_pt) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int k0 = pf_off[p], k1 = pf_off[p + 1];
  double v = 0.0;
  if (flags[p] & 1) {
    double tot = 0.0;
    for (int k = k0; k < k1; ++k) {
      const int f = pf_face[k];
      tot += area[f];
      v += phi_dof[face_dof[3 * f + pf_slot[k]]] * area[f];
    }
    if (k1 > k0) v /= tot;
  } else {
    for (int k = k0; k < k1; ++k)
      if (face_dir[pf_face[k]]) {
        v = phi_dof[face_dof[3 * pf_face[k] + pf_slot[k]]];
        break;
      }
  }
  phi_pt[p] = v;
}

// surface gradient of the linear interpolant of (v0, v1, v2) on triangle (X0, X1, X2), in the
// local frame x along X1 - X0 (gradP1, lib/include/basic_vectors.hpp:2112-2128)
__device__ __forceinline__ void grad_p1(const double* X0, const double* X1, const double* X2, double v0, double v1, double v2,
                                        double* g) {
  double e1[3] = {X1[0] - X0[0], X1[1] - X0[1], X1[2] - X0[2]}, e2[3] = {X2[0] - X0[0], X2[1] - X0[1], X2[2] - X0[2]};
  double ex[3] = {e1[0], e1[1], e1[2]}, ez[3], ey[3];
  v3unit(ex);
  v3cross(e1, e2, ez);
  v3unit(ez);
  v3cross(ez, ex, ey);
  v3unit(ey);
  const double x1 = sqrt(v3dot(e1, e1)), x2 = v3dot(e2, ex), y2 = v3dot(e2, ey);
  const double a = (-v0 + v1) / x1, b = (v2 * x1 - v1 * x2 + v0 * (-x1 + x2)) / (x1 * y2);
  for (int j = 0; j < 3; ++j) g[j] = a * ex[j] + b * ey[j];
}

__global__ void k_grad_phi(int np, const int32_t* __restrict__ pf_off, const int32_t* __restrict__ pf_face,
                           const int8_t* __restrict__ pf_slot, const int32_t* __restrict__ tri, const int32_t* __restrict__ face_dof,
                           const uint8_t* __restrict__ face_dir, const uint8_t* __restrict__ flags, const double* __restrict__ X,
                           const double* __restrict__ normal, const double* __restrict__ area, const double* __restrict__ phi_pt,
                           const double* __restrict__ phin_dof, double* __restrict__ u) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int k0 = pf_off[p], k1 = pf_off[p + 1];
  double H[6] = {0, 0, 0, 0, 0, 0};  // xx xy xz yy yz zz
  double g[3] = {0, 0, 0};
  double sum_abs = 0.0, wsum = 0.0;
  int nsamp = 0;
  for (int k = k0; k < k1; ++k) {
    const int f = pf_face[k];
    const int* t = tri + 3 * f;
    double uf[3];
    grad_p1(X + 3 * t[0], X + 3 * t[1], X + 3 * t[2], phi_pt[t[0]], phi_pt[t[1]], phi_pt[t[2]], uf);
    const double pn = phin_dof[face_dof[3 * f + pf_slot[k]]];
    const double* n = normal + 3 * f;
    const double A = area[f];
    for (int j = 0; j < 3; ++j) {
      uf[j] += pn * n[j];
      g[j] += A * uf[j];  // samples along ex, ey, ez
      sum_abs += fabs(uf[j]);
    }
    H[0] += A;
    H[3] += A;
    H[5] += A;
    wsum += 3.0 * A;
    nsamp += 3;
  }
  if (nsamp == 0) {
    u[3 * p] = u[3 * p + 1] = u[3 * p + 2] = 0.0;
    return;
  }
  if (flags[p] & 4) {  // CORNER: phin of the Neumann faces along their normals
    const double w = 10.0 * (wsum / nsamp);
    for (int k = k0; k < k1; ++k) {
      const int f = pf_face[k];
      if (face_dir[f] || !(area[f] > 0.0)) continue;  // Neumann faces with a normal
      const double* n = normal + 3 * f;
      const double pn = phin_dof[face_dof[3 * f + pf_slot[k]]];
      H[0] += w * n[0] * n[0];
      H[1] += w * n[0] * n[1];
      H[2] += w * n[0] * n[2];
      H[3] += w * n[1] * n[1];
      H[4] += w * n[1] * n[2];
      H[5] += w * n[2] * n[2];
      for (int j = 0; j < 3; ++j) g[j] += w * pn * n[j];
      sum_abs += fabs(pn);
      ++nsamp;
    }
  }
  if (sum_abs == 0.0) {
    u[3 * p] = u[3 * p + 1] = u[3 * p + 2] = 0.0;
    return;
  }
  // minimiser of sum w (d . U - v)^2: H U = g, H symmetric positive definite (adjugate)
  const double a = H[0], b = H[1], c = H[2], d = H[3], e = H[4], ff = H[5];
  const double A00 = d * ff - e * e, A01 = c * e - b * ff, A02 = b * e - c * d;
  const double A11 = a * ff - c * c, A12 = b * c - a * e, A22 = a * d - b * b;
  const double det = a * A00 + b * A01 + c * A02;
  u[3 * p] = (A00 * g[0] + A01 * g[1] + A02 * g[2]) / det;
  u[3 * p + 1] = (A01 * g[0] + A11 * g[1] + A12 * g[2]) / det;
  u[3 * p + 2] = (A02 * g[0] + A12 * g[1] + A22 * g[2]) / det;
}

// one RK4 stage of RungeKuttaCommon<T> with steps = 4: stage k adds f dt to the weighted sum
// (weights 1, 2, 2, 1 in that order) and sets x = x_init + f dt/2 (k = 0, 1), x_init + f dt
// (k = 2), x_init + sum / 6 (k = 3)
__device__ __forceinline__ double rk4(int k, double dt, double x0, double f, double& acc) {
  const double dx = f * dt;
  switch (k) {
    case 0:
      acc = dx;
      return x0 + f * (dt / 2.0);
    case 1:
      acc = acc + 2.0 * dx;
      return x0 + f * (dt / 2.0);
    case 2:
      acc = acc + 2.0 * dx;
      return x0 + f * dt;
    default:
      return x0 + (acc + dx) / 6.0;
  }
}

__global__ void k_mel_push(int np, int stage, double dt, double gravity, const uint8_t* __restrict__ flags, const double* __restrict__ X,
                           const double* __restrict__ phi_pt, const double* __restrict__ u, const double* __restrict__ u_node,
                           const double* __restrict__ damping, double* __restrict__ X0, double* __restrict__ phi0, double* __restrict__ accX,
                           double* __restrict__ accphi, double* __restrict__ Xout, double* __restrict__ phiout,
                           double* __restrict__ dphidt_out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  if (stage == 0) {  // the RK state starts from the current point state
    for (int j = 0; j < 3; ++j) X0[3 * p + j] = X[3 * p + j];
    phi0[p] = phi_pt[p];
  }
  const double* up = u + 3 * p;
  const double* un = u_node ? u_node + 3 * p : up;
  double rate = 0.0;
  if (!(flags[p] & 1)) {
    const double gam = damping ? damping[2 * p] : 0.0, ref = damping ? damping[2 * p + 1] : 0.0;
    rate = -gam * (phi_pt[p] - ref) + (-0.5 * v3dot(up, up) - gravity * X[3 * p + 2] + v3dot(un, up));
    if (!isfinite(rate)) rate = 0.0;  // pushPhi's guard
    double a = accphi[p];
    double ph = rk4(stage, dt, phi0[p], rate, a);
    if (!isfinite(ph)) {
      a = accphi[p];
      ph = rk4(stage, dt, phi0[p], 0.0, a);
      if (!isfinite(ph)) ph = 0.0;
    }
    accphi[p] = a;
    phiout[p] = ph;
  } else {
    phiout[p] = phi_pt[p];
  }
  dphidt_out[p] = rate;
  double xn[3], an[3];
  bool fin = true;
  for (int j = 0; j < 3; ++j) {
    an[j] = accX[3 * p + j];
    xn[j] = rk4(stage, dt, X0[3 * p + j], un[j], an[j]);
    fin = fin && isfinite(xn[j]);
  }
  if (!fin) {  // pushPosition's guard: the stage again with zero velocity, else stay
    fin = true;
    for (int j = 0; j < 3; ++j) {
      an[j] = accX[3 * p + j];
      xn[j] = rk4(stage, dt, X0[3 * p + j], 0.0, an[j]);
      fin = fin && isfinite(xn[j]);
    }
    if (!fin)
      for (int j = 0; j < 3; ++j) xn[j] = X[3 * p + j];
  }
  for (int j = 0; j < 3; ++j) {
    accX[3 * p + j] = an[j];
    Xout[3 * p + j] = xn[j];
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Known values of the phi_t boundary-value problem (setPhiPhin_t,
// bem/BEM_setBoundaryTypes.hpp:858-935).

// gradient, within the triangle's plane, of the linear function taking v[k] at x[k] (the three
// vertices): with e = x1 - x0, f = x2 - x0 and the in-plane frame ex = e/|e|,
// ey = (ez x ex), ez the unit normal of e x f, the function is v0 + a (p . ex) + b (p . ey) with
// a = (v1 - v0)/|e| and b fixed by the third vertex (gradP1, lib/include/basic_vectors.hpp:2112-2128)
__device__ void grad_linear_tri(const double x[3][3], const double v[3], double g[3]) {
  double e[3] = {x[1][0] - x[0][0], x[1][1] - x[0][1], x[1][2] - x[0][2]};
  double f[3] = {x[2][0] - x[0][0], x[2][1] - x[0][1], x[2][2] - x[0][2]};
  double ex[3] = {e[0], e[1], e[2]}, ez[3], ey[3];
  v3unit(ex);
  v3cross(e, f, ez);
  v3unit(ez);
  v3cross(ez, ex, ey);
  v3unit(ey);
  const double x1 = sqrt(v3dot(e, e)), x2 = v3dot(f, ex), y2 = v3dot(f, ey);
  const double a = (v[1] - v[0]) / x1;
  const double b = (v[2] * x1 - v[1] * x2 + v[0] * (x2 - x1)) / (x1 * y2);
  for (int k = 0; k < 3; ++k) g[k] = a * ex[k] + b * ey[k];
}

// phin_t at point p on the Neumann face F (phint_Neumann(p, F), bem/BEM_BoundaryValues.hpp:701-728):
// 0 on a face of no body; on a face of rigid body b (bodies[15 b ..]: centre c, velocity U,
// angular velocity W, acceleration A, angular acceleration Al; RigidBodyDynamics.hpp:84-89)
//   v = U + W x r, a = A + Al x r + W x (W x r), r = x_p - c,
//   phin_t = n.a + (W x n).(v - u_p) - (B v).H0,
// B = {n, s0, s1} (OrthogonalBasis, :307-315) and H0 the first row of HessianOfPhi (:653-672):
// with the vertices and their velocities in that basis and g_ij = component j of the in-plane
// gradient of component i of the velocity, H0 = (-g11 - g22, (g01 + g10)/2, (g02 + g20)/2).
__device__ double phint_face(int p, int F, const int32_t* __restrict__ tri, const double* __restrict__ X, const double* __restrict__ normal,
                             const double* __restrict__ u, const int32_t* __restrict__ face_body, const double* __restrict__ bodies) {
  const int b = face_body[F];
  if (b < 0) return 0.0;
  const double* B = bodies + 15 * b;
  const double n[3] = {normal[3 * F], normal[3 * F + 1], normal[3 * F + 2]};
  const double r[3] = {X[3 * p] - B[0], X[3 * p + 1] - B[1], X[3 * p + 2] - B[2]};
  double wr[3], wwr[3], alr[3], wn[3];
  v3cross(B + 6, r, wr);
  v3cross(B + 6, wr, wwr);
  v3cross(B + 12, r, alr);
  v3cross(B + 6, n, wn);
  double v[3], a[3];
  for (int k = 0; k < 3; ++k) {
    v[k] = B[3 + k] + wr[k];
    a[k] = B[9 + k] + alr[k] + wwr[k];
  }
  // basis {n, s0, s1}: s0 = the part of ex (or ey, when ex is almost normal) off n
  double s0[3] = {1.0 - n[0] * n[0], -n[0] * n[1], -n[0] * n[2]};
  if (sqrt(v3dot(s0, s0)) < 1e-3) {
    s0[0] = -n[1] * n[0];
    s0[1] = 1.0 - n[1] * n[1];
    s0[2] = -n[1] * n[2];
  }
  v3unit(s0);
  double s1[3];
  v3cross(n, s0, s1);
  v3unit(s1);
  const double* basis[3] = {n, s0, s1};
  double xr[3][3], ur[3][3];  // [vertex][basis component]
  for (int k = 0; k < 3; ++k) {
    const int q = tri[3 * F + k];
    for (int i = 0; i < 3; ++i) {
      xr[k][i] = v3dot(basis[i], X + 3 * q);
      ur[k][i] = v3dot(basis[i], u + 3 * q);
    }
  }
  double g[3][3];  // g[i][j]: in-plane gradient (component j) of velocity component i
  for (int i = 0; i < 3; ++i) {
    const double vi[3] = {ur[0][i], ur[1][i], ur[2][i]};
    grad_linear_tri(xr, vi, g[i]);
  }
  const double H0[3] = {-g[1][1] - g[2][2], 0.5 * (g[0][1] + g[1][0]), 0.5 * (g[0][2] + g[2][0])};
  const double tmp[3] = {v3dot(n, v), v3dot(s0, v), v3dot(s1, v)};
  const double du[3] = {v[0] - u[3 * p], v[1] - u[3 * p + 1], v[2] - u[3 * p + 2]};
  return v3dot(n, a) + v3dot(wn, du) - v3dot(tmp, H0);
}

// per DOF: Dirichlet (kind 0) phi_t = -|u|^2/2 - gravity z (aphiat(0), lib/include/Network.hpp:971-976);
// Neumann (kinds 1, 2) phin_t of its face, or for a point DOF the area-weighted mean over the
// point's Neumann faces (phint_Neumann(p), bem/BEM_BoundaryValues.hpp:751-779)
__global__ void k_phit_known(int ndof, const int32_t* __restrict__ dof_point, const int32_t* __restrict__ dof_face,
                             const int32_t* __restrict__ dof_kind, const int32_t* __restrict__ pf_off, const int32_t* __restrict__ pf_face,
                             const int32_t* __restrict__ tri, const uint8_t* __restrict__ face_dir, const double* __restrict__ X,
                             const double* __restrict__ normal, const double* __restrict__ area, const double* __restrict__ u,
                             const int32_t* __restrict__ face_body, const double* __restrict__ bodies, double gravity,
                             double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ndof) return;
  const int p = dof_point[i];
  if (dof_kind[i] == 0) {
    const double* up = u + 3 * p;
    out[i] = -0.5 * v3dot(up, up) - gravity * X[3 * p + 2];
    return;
  }
  const int F = dof_face[i];
  if (F >= 0) {
    out[i] = phint_face(p, F, tri, X, normal, u, face_body, bodies);
    return;
  }
  double s = 0.0, w = 0.0;
  for (int k = pf_off[p]; k < pf_off[p + 1]; ++k) {
    const int f = pf_face[k];
    if (face_dir[f]) continue;
    s += phint_face(p, f, tri, X, normal, u, face_body, bodies) * area[f];
    w += area[f];
  }
  out[i] = w > 0.0 ? s / w : 0.0;
}

struct bem_gpu_mel {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  MBuf<double> X, normal, area, phi_dof, phin_dof, phi_pt, u, u_node, damping, X0, phi0, accX, accphi, Xout, phiout, dphidt, bodies, known_t;
  MBuf<int32_t> tri, face_dof, pf_off, pf_face, dof_point, dof_face, dof_kind, face_body;
  MBuf<int8_t> pf_slot;
  MBuf<uint8_t> flags, face_dir;
  ~bem_gpu_mel() {
    if (stream) cudaStreamDestroy(stream);
  }
};

#define MK(call)                                                                \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      m->err = std::string(#call) + ": " + cudaGetErrorString(e_);              \
      return e_ == cudaErrorMemoryAllocation ? BEM_ERR_OUT_OF_MEMORY : BEM_ERR_DEVICE; \
    }                                                                           \
  } while (0)

namespace {

template <typename T>
cudaError_t put(bem_gpu_mel* m, MBuf<T>& b, const T* src, size_t n) {
  cudaError_t e = b.reserve(n);
  if (e != cudaSuccess || n == 0) return e;
  return cudaMemcpyAsync(b.p, src, sizeof(T) * n, cudaMemcpyHostToDevice, m->stream);
}

// uploads the surface and derives the per-face and per-point data every kernel needs
int mel_prepare(bem_gpu_mel* m, const bem_mel_surface* s) {
  const int np = s->n_points, nf = s->n_faces;
  if (np <= 0 || nf <= 0 || !s->X || !s->tri || !s->point_flags || !s->face_dirichlet || !s->face_dof || !s->phi || !s->phin ||
      s->n_dof <= 0) {
    m->err = "invalid MEL surface";
    return BEM_ERR_INVALID_ARGUMENT;
  }
  std::vector<int32_t> off(np + 1, 0);
  for (int i = 0; i < 3 * nf; ++i) {
    const int p = s->tri[i];
    if (p < 0 || p >= np || s->face_dof[i] < 0 || s->face_dof[i] >= s->n_dof) {
      m->err = "invalid MEL connectivity";
      return BEM_ERR_INVALID_ARGUMENT;
    }
    ++off[p + 1];
  }
  for (int p = 0; p < np; ++p) off[p + 1] += off[p];
  std::vector<int32_t> pff(3 * (size_t)nf);
  std::vector<int8_t> pfs(3 * (size_t)nf);
  {
    std::vector<int32_t> fill(off.begin(), off.end() - 1);
    for (int f = 0; f < nf; ++f)  // ascending face order per point
      for (int a = 0; a < 3; ++a) {
        const int k = fill[s->tri[3 * f + a]]++;
        pff[k] = f;
        pfs[k] = (int8_t)a;
      }
  }
  MK(cudaSetDevice(m->device));
  MK(put(m, m->X, s->X, 3 * (size_t)np));
  MK(put(m, m->tri, s->tri, 3 * (size_t)nf));
  MK(put(m, m->face_dof, s->face_dof, 3 * (size_t)nf));
  MK(put(m, m->flags, s->point_flags, (size_t)np));
  MK(put(m, m->face_dir, s->face_dirichlet, (size_t)nf));
  MK(put(m, m->phi_dof, s->phi, (size_t)s->n_dof));
  MK(put(m, m->phin_dof, s->phin, (size_t)s->n_dof));
  MK(put(m, m->pf_off, off.data(), off.size()));
  MK(put(m, m->pf_face, pff.data(), pff.size()));
  MK(put(m, m->pf_slot, pfs.data(), pfs.size()));
  MK(m->normal.reserve(3 * (size_t)nf));
  MK(m->area.reserve((size_t)nf));
  MK(m->phi_pt.reserve((size_t)np));
  MK(m->u.reserve(3 * (size_t)np));
  const int gf = (nf + 255) / 256, gp = (np + 255) / 256;
  k_face_geom<<<gf, 256, 0, m->stream>>>(nf, m->tri.p, m->X.p, m->normal.p, m->area.p);
  k_point_phi<<<gp, 256, 0, m->stream>>>(np, m->pf_off.p, m->pf_face.p, m->pf_slot.p, m->face_dof.p, m->face_dir.p, m->flags.p,
                                         m->area.p, m->phi_dof.p, m->phi_pt.p);
  k_grad_phi<<<gp, 256, 0, m->stream>>>(np, m->pf_off.p, m->pf_face.p, m->pf_slot.p, m->tri.p, m->face_dof.p, m->face_dir.p,
                                        m->flags.p, m->X.p, m->normal.p, m->area.p, m->phi_pt.p, m->phin_dof.p, m->u.p);
  MK(cudaGetLastError());
  return BEM_OK;
}

}  // namespace

extern "C" {

bem_gpu_mel* bem_gpu_mel_create(int32_t device) {
  if (cudaSetDevice(device) != cudaSuccess) return nullptr;
  auto* m = new bem_gpu_mel();
  m->device = device;
  if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete m;
    return nullptr;
  }
  return m;
}

void bem_gpu_mel_destroy(bem_gpu_mel* m) {
  if (!m) return;
  cudaSetDevice(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  delete m;
}

const char* bem_gpu_mel_last_error(const bem_gpu_mel* m) { return m ? m->err.c_str() : "null MEL context"; }

int bem_gpu_mel_velocity(bem_gpu_mel* m, const bem_mel_surface* s, double* out_phi_point, double* out_u) {
  if (!m || !s || !out_u) return BEM_ERR_INVALID_ARGUMENT;
  int rc = mel_prepare(m, s);
  if (rc != BEM_OK) return rc;
  const size_t np = (size_t)s->n_points;
  if (out_phi_point) MK(cudaMemcpyAsync(out_phi_point, m->phi_pt.p, sizeof(double) * np, cudaMemcpyDeviceToHost, m->stream));
  MK(cudaMemcpyAsync(out_u, m->u.p, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost, m->stream));
  MK(cudaStreamSynchronize(m->stream));
  return BEM_OK;
}

int bem_gpu_mel_stage(bem_gpu_mel* m, const bem_mel_surface* s, int32_t stage, double dt, double gravity, const double* u_node,
                      const double* damping, double* rk_X0, double* rk_phi0, double* rk_accX, double* rk_accphi, double* out_X,
                      double* out_phi, double* out_u, double* out_dphidt) {
  if (!m || !s || stage < 0 || stage > 3 || !(dt > 0) || !std::isfinite(gravity) || !rk_X0 || !rk_phi0 || !rk_accX || !rk_accphi ||
      !out_X || !out_phi)
    return BEM_ERR_INVALID_ARGUMENT;
  int rc = mel_prepare(m, s);
  if (rc != BEM_OK) return rc;
  const size_t np = (size_t)s->n_points;
  MK(put(m, m->X0, rk_X0, 3 * np));
  MK(put(m, m->phi0, rk_phi0, np));
  MK(put(m, m->accX, rk_accX, 3 * np));
  MK(put(m, m->accphi, rk_accphi, np));
  if (u_node) MK(put(m, m->u_node, u_node, 3 * np));
  if (damping) MK(put(m, m->damping, damping, 2 * np));
  MK(m->Xout.reserve(3 * np));
  MK(m->phiout.reserve(np));
  MK(m->dphidt.reserve(np));
  k_mel_push<<<(int)((np + 255) / 256), 256, 0, m->stream>>>((int)np, stage, dt, gravity, m->flags.p, m->X.p, m->phi_pt.p, m->u.p,
                                                             u_node ? m->u_node.p : nullptr, damping ? m->damping.p : nullptr, m->X0.p,
                                                             m->phi0.p, m->accX.p, m->accphi.p, m->Xout.p, m->phiout.p, m->dphidt.p);
  MK(cudaGetLastError());
  MK(cudaMemcpyAsync(rk_X0, m->X0.p, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost, m->stream));
  MK(cudaMemcpyAsync(rk_phi0, m->phi0.p, sizeof(double) * np, cudaMemcpyDeviceToHost, m->stream));
  MK(cudaMemcpyAsync(rk_accX, m->accX.p, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost, m->stream));
  MK(cudaMemcpyAsync(rk_accphi, m->accphi.p, sizeof(double) * np, cudaMemcpyDeviceToHost, m->stream));
  MK(cudaMemcpyAsync(out_X, m->Xout.p, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost, m->stream));
  MK(cudaMemcpyAsync(out_phi, m->phiout.p, sizeof(double) * np, cudaMemcpyDeviceToHost, m->stream));
  if (out_u) MK(cudaMemcpyAsync(out_u, m->u.p, sizeof(double) * 3 * np, cudaMemcpyDeviceToHost, m->stream));
  if (out_dphidt) MK(cudaMemcpyAsync(out_dphidt, m->dphidt.p, sizeof(double) * np, cudaMemcpyDeviceToHost, m->stream));
  MK(cudaStreamSynchronize(m->stream));
  return BEM_OK;
}

int bem_gpu_mel_phit_known(bem_gpu_mel* m, const bem_mel_surface* s, const int32_t* dof_point, const int32_t* dof_face,
                           const int32_t* dof_kind, const int32_t* face_body, int32_t n_bodies, const double* bodies, double gravity,
                           const double* u, double* out_known) {
  if (!m || !s || !dof_point || !dof_face || !dof_kind || !face_body || n_bodies < 0 || (n_bodies > 0 && !bodies) ||
      !std::isfinite(gravity) || !out_known)
    return BEM_ERR_INVALID_ARGUMENT;
  const int nd = s->n_dof, nf = s->n_faces;
  for (int i = 0; i < nd; ++i)
    if (dof_point[i] < 0 || dof_point[i] >= s->n_points || dof_kind[i] < 0 || dof_kind[i] > 2 || dof_face[i] < -1 || dof_face[i] >= nf) {
      m->err = "invalid DOF table";
      return BEM_ERR_INVALID_ARGUMENT;
    }
  for (int f = 0; f < nf; ++f)
    if (face_body[f] < -1 || face_body[f] >= n_bodies) {
      m->err = "face_body out of range";
      return BEM_ERR_INVALID_ARGUMENT;
    }
  int rc = mel_prepare(m, s);
  if (rc != BEM_OK) return rc;
  if (u) MK(put(m, m->u, u, 3 * (size_t)s->n_points));  // the caller's velocities replace the computed ones
  MK(put(m, m->dof_point, dof_point, (size_t)nd));
  MK(put(m, m->dof_face, dof_face, (size_t)nd));
  MK(put(m, m->dof_kind, dof_kind, (size_t)nd));
  MK(put(m, m->face_body, face_body, (size_t)nf));
  MK(m->bodies.reserve(15 * (size_t)std::max(n_bodies, 1)));
  if (n_bodies > 0) MK(cudaMemcpyAsync(m->bodies.p, bodies, sizeof(double) * 15 * n_bodies, cudaMemcpyHostToDevice, m->stream));
  MK(m->known_t.reserve((size_t)nd));
  k_phit_known<<<(nd + 255) / 256, 256, 0, m->stream>>>(nd, m->dof_point.p, m->dof_face.p, m->dof_kind.p, m->pf_off.p, m->pf_face.p, m->tri.p,
                                                         m->face_dir.p, m->X.p, m->normal.p, m->area.p, m->u.p, m->face_body.p,
                                                         m->bodies.p, gravity, m->known_t.p);
  MK(cudaGetLastError());
  MK(cudaMemcpyAsync(out_known, m->known_t.p, sizeof(double) * nd, cudaMemcpyDeviceToHost, m->stream));
  MK(cudaStreamSynchronize(m->stream));
  return BEM_OK;
}

}  // extern "C"
