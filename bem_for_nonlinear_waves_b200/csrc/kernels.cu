// FP64 FMM mat-vec and near-field kernels for sm_100a.
//
// Per mat-vec (return_A_dot_v, bem/BEM_solveBVP_GMRES_FMM.hpp:2124-2155):
//   k_densities   per-DOF phi/phin from the unknown vector (setUnknowns/setKnowns, :1142-1176)
//   k_p2m         leaf multipoles from the 6 Dunavant points of every element (moments.hpp:307-368)
//   k_m2m_level   one launch per level from the deepest: multipoles summed from the children's
//                 shifted ones, then shifted to the parent (moments.hpp:419-436, 912-915)
//   k_m2l         every M2L pair of every level in one launch (moments.hpp:732-764)
//   k_l2l_pairs   one launch per level, top-down, a CTA per (parent, child) (moments.hpp:869-884, 925-929)
//   k_targets     near-field block SpMV + L2P + BIE rows (compute_Ax_minus_b, :34-158)
// Set-up:
//   k_near_weights  near-field quadrature into per-block dense rows (target4FMM::setDirectIntegration,
//                   lib_multipole_expansion.hpp:1180-1271 with fill_direct_linear / fill_nonadj_linear,
//                   BEM_solveBVP_GMRES_FMM.hpp:1824-1891)
#include <cuda_runtime.h>

#include <cstdlib>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <type_traits>

#include "fmm_math.cuh"
#include "kernels.cuh"
#include "tc_sm100.cuh"

namespace bemb200 {

__constant__ double c_dv[6][4];   // Dunavant 6-point rule: b0, b1, b2, w
__constant__ double c_gw[25][3];  // 5x5 Gauss-Legendre on [0,1]^2: t0, t1, w

void upload_quadrature(const double dv[6][4], const double gw[25][3], cudaStream_t s) {
  cudaMemcpyToSymbolAsync(c_dv, dv, sizeof(double) * 24, 0, cudaMemcpyHostToDevice, s);
  cudaMemcpyToSymbolAsync(c_gw, gw, sizeof(double) * 75, 0, cudaMemcpyHostToDevice, s);
}

// ---------------------------------------------------------------------------
// per-DOF phi / phin.  mode 0: unknowns = x, knowns = 0 (A.x);  mode 1: unknowns = 0,
// knowns = known (right-hand side);  mode 2: phi = 1, phin = 0 (rigid mode);  mode 3:
// phi/phin given directly (x = phi, known = phin).
__global__ void k_densities(int n, int mode, const double* __restrict__ x, const double* __restrict__ known, const int* __restrict__ kind,
                            double* __restrict__ phi, double* __restrict__ phin) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const bool dir = kind[i] == 0;
    double a, b;
    if (mode == 0) {
      a = dir ? 0.0 : x[i];
      b = dir ? x[i] : 0.0;
    } else if (mode == 1) {
      a = dir ? known[i] : 0.0;
      b = dir ? 0.0 : known[i];
    } else if (mode == 2) {
      a = 1.0;
      b = 0.0;
    } else {
      a = x[i];
      b = known[i];
    }
    phi[i] = a;
    phin[i] = b;
  }
}

// ---------------------------------------------------------------------------
// P2M: one block (4 warps) per leaf; each half-warp carries one P2M point, lane m its
// column m of F_n^m, advanced degree by degree in lock-step so that the gradient
// terms F_{n-1}^{m-1}, F_{n-1}^{m+1} come from the neighbouring lanes by shuffles.
// ND = 2: the monopole (phin) and dipole (phi) expansions M[0], M[1] separately; ND = 1: only
// their difference M[0] - M[1] (in M[0]), all that a mat-vec row GPhin - GnPhi needs.
template <int P, int ND>
__global__ void __launch_bounds__(128) k_p2m(const int* __restrict__ leaves, const int* __restrict__ node_fb, const int* __restrict__ node_fe,
                                             const double* __restrict__ node_X, const double* __restrict__ e_q,
                                             const double* __restrict__ e_W, const double* __restrict__ e_n,
                                             const int* __restrict__ e_dof, const double* __restrict__ phi,
                                             const double* __restrict__ phin, double2* __restrict__ M) {
  constexpr int NC = ncoef(P);
  static_assert(P <= 14, "column lanes live in a half warp");
  __shared__ double2 red[4][ND][NC];
  const int leaf = leaves[blockIdx.x];
  const int fb = node_fb[leaf], fe = node_fe[leaf];
  const double cx = node_X[3 * leaf], cy = node_X[3 * leaf + 1], cz = node_X[3 * leaf + 2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int half = lane >> 4, m = lane & 15;
  double2 accM[P + 1], accD[P + 1];
#pragma unroll
  for (int n = 0; n <= P; ++n) {
    accM[n] = make_double2(0.0, 0.0);
    accD[n] = make_double2(0.0, 0.0);
  }
  const int npts = (fe - fb) * 6;
  for (int base = 0; base < npts; base += 8) {
    const int pt = base + warp * 2 + half;
    double x = 0, y = 0, z = 0, wphi = 0, wphin = 0, nx = 0, ny = 0, nz = 0;
    if (pt < npts) {
      const int s = fb + pt / 6, k = pt % 6;
      x = e_q[s * 18 + 3 * k] - cx;
      y = e_q[s * 18 + 3 * k + 1] - cy;
      z = e_q[s * 18 + 3 * k + 2] - cz;
      const int d0 = e_dof[3 * s], d1 = e_dof[3 * s + 1], d2 = e_dof[3 * s + 2];
      const double W = e_W[s * 6 + k];
      // closure get_weighted_source_densities (BEM_solveBVP_GMRES_FMM.hpp:1915-1922)
      wphi = W * (c_dv[k][0] * phi[d0] + c_dv[k][1] * phi[d1] + c_dv[k][2] * phi[d2]);
      wphin = W * (c_dv[k][0] * phin[d0] + c_dv[k][1] * phin[d1] + c_dv[k][2] * phin[d2]);
      nx = e_n[3 * s];
      ny = e_n[3 * s + 1];
      nz = e_n[3 * s + 2];
    }
    const double r2 = x * x + y * y + z * z;
    double2 diag = make_double2(1.0, 0.0);
    for (int k = 1; k <= m && k <= P; ++k) diag = cscale(cmul(diag, make_double2(x, y)), 1.0 / (2.0 * k));
    double2 prev = make_double2(0.0, 0.0), prev2 = make_double2(0.0, 0.0);
#pragma unroll
    for (int n = 0; n <= P; ++n) {
      double2 cur;
      if (n < m)
        cur = make_double2(0.0, 0.0);
      else if (n == m)
        cur = diag;
      else {
        const double inv = 1.0 / double(n * n - m * m);
        cur = make_double2(((2 * n - 1) * z * prev.x - r2 * prev2.x) * inv, ((2 * n - 1) * z * prev.y - r2 * prev2.y) * inv);
      }
      double2 up = shfl_up2(prev, 1, 16);    // F_{n-1}^{m-1}
      double2 dn = shfl_down2(prev, 1, 16);  // F_{n-1}^{m+1}
      if (m == 0) up = make_double2(-dn.x, dn.y);  // F^{-1} = -conj(F^{1})
      if (m == 15) dn = make_double2(0.0, 0.0);
      // g = nu_z F^m + 1/2 (nu_x + i nu_y) F^{m-1} - 1/2 (nu_x - i nu_y) F^{m+1}
      double2 g = cscale(prev, nz);
      g = cadd(g, cscale(cmul(make_double2(nx, ny), up), 0.5));
      g = csub(g, cscale(cmul(make_double2(nx, -ny), dn), 0.5));
      if (n >= m) {
        if (ND == 2) {
          accM[n].x += wphin * cur.x;
          accM[n].y -= wphin * cur.y;
          accD[n].x += wphi * g.x;
          accD[n].y -= wphi * g.y;
        } else {
          accM[n].x += wphin * cur.x - wphi * g.x;
          accM[n].y -= wphin * cur.y - wphi * g.y;
        }
      }
      prev2 = prev;
      prev = cur;
    }
  }
#pragma unroll
  for (int n = 0; n <= P; ++n) {
    accM[n] = cadd(accM[n], shfl_down2(accM[n], 16, 32));
    if (ND == 2) accD[n] = cadd(accD[n], shfl_down2(accD[n], 16, 32));
  }
  if (half == 0 && m <= P) {
#pragma unroll
    for (int n = 0; n <= P; ++n)
      if (n >= m) {
        red[warp][0][cidx(n, m)] = accM[n];
        if (ND == 2) red[warp][ND - 1][cidx(n, m)] = accD[n];
      }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < ND * NC; t += blockDim.x) {
    const int d = t / NC, c = t % NC;
    double2 s = red[0][d][c];
    s = cadd(s, red[1][d][c]);
    s = cadd(s, red[2][d][c]);
    s = cadd(s, red[3][d][c]);
    M[(size_t)leaf * 2 * NC + t] = s;
  }
}

__device__ __forceinline__ void decode_nm(int t, int& n, int& m) {
  n = 0;
  while ((n + 1) * (n + 2) / 2 <= t) ++n;
  m = t - n * (n + 1) / 2;
}

// P2M of A.x as a precomputed operator.  With the known values zero, a DOF d of a leaf enters
// the leaf's combined multipole M[0] - M[1] linearly through its unknown x_d:
//   C_{leaf,d} = sum over the leaf's element vertices a with DOF d and P2M points k of
//                W_k N_a(k) conj(F(y_k - c))      (Dirichlet DOF: phin = x_d)
//             or -W_k N_a(k) conj(nu . grad F)    (otherwise: phi = x_d)
// so each A.x computes M_leaf = sum_d x_d C_{leaf,d}: one pass over C (a few bytes per
// source point) instead of the harmonics of every P2M point (k_p2m_leaf, with the leaf's first
// M2M shift).  k_p2m_op builds C at set-up:
// block per leaf, four points at a time (a warp fills the F table of one point), thread per
// coefficient adding the points in order into its own entries of C (deterministic).
template <int P>
__global__ void __launch_bounds__(128) k_p2m_op(const int* __restrict__ leaves, const int* __restrict__ node_fb, const int* __restrict__ node_fe,
                                                const double* __restrict__ node_X, const double* __restrict__ e_q,
                                                const double* __restrict__ e_W, const double* __restrict__ e_n,
                                                const int* __restrict__ e_dof, const int* __restrict__ e_slot,
                                                const int* __restrict__ dof_kind, const int* __restrict__ leaf_dof_off,
                                                double2* __restrict__ C) {
  constexpr int NC = ncoef(P), NF = (P + 1) * (P + 1);
  __shared__ double2 sF[4][NF];
  __shared__ double spt[4][8];  // W, nx, ny, nz, element, point of each staged point
  const int li = blockIdx.x, leaf = leaves[li];
  const int fb = node_fb[leaf], fe = node_fe[leaf];
  const double cx = node_X[3 * leaf], cy = node_X[3 * leaf + 1], cz = node_X[3 * leaf + 2];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, t = threadIdx.x;
  double2* Cl = C + (size_t)leaf_dof_off[li] * NC;
  int n = 0, m = 0;
  if (t < NC) decode_nm(t, n, m);
  const int npts = (fe - fb) * 6;
  for (int base = 0; base < npts; base += 4) {
    const int pt = base + warp;
    if (pt < npts) {
      const int s = fb + pt / 6, k = pt % 6;
      F_full_column<P>(lane, e_q[s * 18 + 3 * k] - cx, e_q[s * 18 + 3 * k + 1] - cy, e_q[s * 18 + 3 * k + 2] - cz, sF[warp]);
      if (lane == 0) {
        spt[warp][0] = e_W[s * 6 + k];
        spt[warp][1] = e_n[3 * s];
        spt[warp][2] = e_n[3 * s + 1];
        spt[warp][3] = e_n[3 * s + 2];
      }
    }
    __syncthreads();
    if (t < NC) {
      for (int w = 0; w < 4; ++w) {
        const int q = base + w;
        if (q >= npts) break;
        const int s = fb + q / 6, k = q % 6;
        const double2* T = sF[w];
        const double2 F = T[n * (n + 1) + m];
        // nu . grad F_n^m = nu_z F_{n-1}^m + 1/2 (nu_x + i nu_y) F_{n-1}^{m-1} - 1/2 (nu_x - i nu_y) F_{n-1}^{m+1}
        double2 g = make_double2(0.0, 0.0);
        if (n >= 1) {
          const double nx = spt[w][1], ny = spt[w][2], nz = spt[w][3];
          const int b = (n - 1) * n;
          if (m <= n - 1) g = cscale(T[b + m], nz);
          if (m - 1 >= -(n - 1)) g = cadd(g, cscale(cmul(make_double2(nx, ny), T[b + m - 1]), 0.5));
          if (m + 1 <= n - 1) g = csub(g, cscale(cmul(make_double2(nx, -ny), T[b + m + 1]), 0.5));
        }
        const double W = spt[w][0];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          const int d = e_dof[3 * s + a];
          const double wa = W * c_dv[k][a];
          const double2 v = dof_kind[d] == 0 ? make_double2(wa * F.x, -wa * F.y) : make_double2(-wa * g.x, wa * g.y);
          double2* c = Cl + (size_t)e_slot[3 * s + a] * NC + t;
          *c = cadd(*c, v);
        }
      }
    }
    __syncthreads();
  }
}

// M_leaf[0] = sum_d x_d C_{leaf,d} (block per leaf, thread per coefficient)

// ---------------------------------------------------------------------------
// Parent-to-child translation tables.  A child bucket sits at one of eight offsets from its
// parent, the same on a level up to rounding, so F(c - c') is tabulated once per (level,
// octant) at set-up; the tree passes read the table instead of running the recurrence.
template <int P>
__global__ void k_ftab(int ntab, const double* __restrict__ vec, double2* __restrict__ Ftab) {
  constexpr int NF = (P + 1) * (P + 1);
  const int t = blockIdx.x;
  if (t < ntab && threadIdx.x < 32) F_full_column<P>(threadIdx.x, vec[3 * t], vec[3 * t + 1], vec[3 * t + 2], Ftab + (size_t)t * NF);
}

__device__ __forceinline__ int child_octant(const double* __restrict__ node_X, int c, int par) {
  return (node_X[3 * c] > node_X[3 * par] ? 1 : 0) | (node_X[3 * c + 1] > node_X[3 * par + 1] ? 2 : 0) |
         (node_X[3 * c + 2] > node_X[3 * par + 2] ? 4 : 0);
}

// half-stored [ND][NC] -> full [ND][(P+1)^2] by the threads [0, nthr) of a group
template <int P, int ND, bool kThroughL2>
__device__ __forceinline__ void expand_full_group(const double2* __restrict__ src, double2* dst, int tid, int nthr) {
  constexpr int NC = ncoef(P), NF = (P + 1) * (P + 1);
  for (int t = tid; t < ND * NF; t += nthr) {
    const int d = t / NF, i = t % NF;
    int n = 0;
    while ((n + 1) * (n + 1) <= i) ++n;
    const int m = i - n * (n + 1);
    const double2* q = src + d * NC + cidx(n, m < 0 ? -m : m);
    double2 v = kThroughL2 ? __ldcg(q) : *q;
    if (m < 0) v = ((-m) & 1) ? make_double2(-v.x, v.y) : make_double2(v.x, -v.y);
    dst[t] = v;
  }
}

// Tree translations with kTreeLanes lanes per output coefficient: lane q sums the rows
// (source degree) q, q + kTreeLanes, ... of the coefficient's terms in two interleaved chains,
// and the lanes' partial sums are added by warp shuffles in a fixed order (every lane ends with
// the same sum).  The longest coefficient (121 terms at p = 10) then takes about a third of the
// dependent adds, and the row bookkeeping is not repeated across lanes.  One CTA per
// translation (a child and its parent).
constexpr int kTreeLanes = 4;
template <int P>
constexpr int tree_threads() { return (kTreeLanes * ncoef(P) + 31) / 32 * 32; }

__device__ __forceinline__ double2 tree_lanes_sum(double2 v) {
#pragma unroll
  for (int o = 1; o < kTreeLanes; o <<= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}

// conj(f) * x added to a
__device__ __forceinline__ void cmac_conj(double2& a, const double2 f, const double2 x) {
  a.x += f.x * x.x + f.y * x.y;
  a.y += f.x * x.y - f.y * x.x;
}

// lane q's rows of the M2M output (n, m): sum conj(F_{n1}^{m1}) M_{n-n1}^{m-m1}, n1 = q, q + 4, ...
template <int P, int ND>
__device__ __forceinline__ void m2m_terms(int n, int m, int q, const double2* __restrict__ sF, const double2* __restrict__ sM, double2& o0,
                                          double2& o1) {
  constexpr int NF = (P + 1) * (P + 1);
  double2 a0 = make_double2(0.0, 0.0), b0 = a0, a1 = a0, b1 = a0;
  for (int n1 = q; n1 <= n; n1 += kTreeLanes) {
    const int n2 = n - n1;
    const int lo = max(-n1, m - n2), hi = min(n1, m + n2);
    const double2* f = sF + n1 * (n1 + 1);
    const double2* x = sM + n2 * (n2 + 1) + m;
    int m1 = lo;
    for (; m1 < hi; m1 += 2) {
      cmac_conj(a0, f[m1], x[-m1]);
      cmac_conj(b0, f[m1 + 1], x[-m1 - 1]);
      if (ND == 2) {
        cmac_conj(a1, f[m1], x[NF - m1]);
        cmac_conj(b1, f[m1 + 1], x[NF - m1 - 1]);
      }
    }
    if (m1 == hi) {
      cmac_conj(a0, f[m1], x[-m1]);
      if (ND == 2) cmac_conj(a1, f[m1], x[NF - m1]);
    }
  }
  o0 = cadd(a0, b0);
  if (ND == 2) o1 = cadd(a1, b1);
}

// lane q's rows of the L2L output (k, j): sum_{n>=k} L_n^m conj(F_{n-k}^{m-j}), n = k + q, k + q + 4, ...
template <int P, int ND>
__device__ __forceinline__ void l2l_terms(int k, int j, int q, const double2* __restrict__ sF, const double2* __restrict__ sL, double2& o0,
                                          double2& o1) {
  constexpr int NF = (P + 1) * (P + 1);
  double2 a0 = make_double2(0.0, 0.0), b0 = a0, a1 = a0, b1 = a0;
  for (int n = k + q; n <= P; n += kTreeLanes) {
    const int dn = n - k;
    const int lo = max(-n, j - dn), hi = min(n, j + dn);
    const double2* f = sF + dn * (dn + 1) - j;
    const double2* x = sL + n * (n + 1);
    int m = lo;
    for (; m < hi; m += 2) {
      cmac_conj(a0, f[m], x[m]);
      cmac_conj(b0, f[m + 1], x[m + 1]);
      if (ND == 2) {
        cmac_conj(a1, f[m], x[NF + m]);
        cmac_conj(b1, f[m + 1], x[NF + m + 1]);
      }
    }
    if (m == hi) {
      cmac_conj(a0, f[m], x[m]);
      if (ND == 2) cmac_conj(a1, f[m], x[NF + m]);
    }
  }
  o0 = cadd(a0, b0);
  if (ND == 2) o1 = cadd(a1, b1);
}

// M2M, one launch per level from the deepest (moments.hpp:419-436): a CTA per node c of the
// level that either builds a multipole (a non-leaf whose multipole is needed: the sum of its
// children's translated multipoles Yup, in child order) or hands its multipole up (its parent's
// multipole is needed: Yup[c] = the multipole shifted to the parent's centre).  A leaf's
// multipole comes from the P2M.  Fup: the F tables of the parent level [8 octants][(P+1)^2].
template <int P, int ND>
__global__ void __launch_bounds__(tree_threads<P>(), 5) k_m2m_level(const int* __restrict__ nodes, const int* __restrict__ node_up,
                                                                 const int* __restrict__ child_begin, const int* __restrict__ child_end,
                                                                 const int* __restrict__ node_children, const double* __restrict__ node_X,
                                                                 const double2* __restrict__ Fup, double2* __restrict__ M,
                                                                 double2* __restrict__ Yup) {
  pdl_enter();
  constexpr int NC = ncoef(P), NF = (P + 1) * (P + 1);
  __shared__ double2 sF[NF];
  __shared__ double2 sHalf[ND * NC];
  __shared__ double2 sM[ND * NF];
  const int c = nodes[blockIdx.x];
  const int cb = child_begin[c], ce = child_end[c], up = node_up[c];
  double2* Mc = M + (size_t)c * 2 * NC;
  if (ce > cb) {
    for (int i = threadIdx.x; i < ND * NC; i += blockDim.x) {
      double2 s = make_double2(0.0, 0.0);
      for (int ci = cb; ci < ce; ++ci) s = cadd(s, Yup[(size_t)node_children[ci] * 2 * NC + i]);
      Mc[i] = s;
      sHalf[i] = s;
    }
  } else {
    for (int i = threadIdx.x; i < ND * NC; i += blockDim.x) sHalf[i] = Mc[i];
  }
  if (up < 0) return;  // uniform over the CTA
  const double2* Ft = Fup + (size_t)child_octant(node_X, c, up) * NF;
  for (int i = threadIdx.x; i < NF; i += blockDim.x) sF[i] = Ft[i];
  __syncthreads();
  expand_full_group<P, ND, false>(sHalf, sM, threadIdx.x, blockDim.x);
  __syncthreads();
  const int o = threadIdx.x / kTreeLanes, q = threadIdx.x % kTreeLanes;
  double2 a0 = make_double2(0.0, 0.0), a1 = a0;
  if (o < NC) {
    int n = 0, m = 0;
    decode_nm(o, n, m);
    m2m_terms<P, ND>(n, m, q, sF, sM, a0, a1);
  }
  a0 = tree_lanes_sum(a0);
  if (ND == 2) a1 = tree_lanes_sum(a1);
  if (o < NC && q == 0) {
    double2* y = Yup + (size_t)c * 2 * NC;
    y[o] = a0;
    if (ND == 2) y[NC + o] = a1;
  }
}

// P2M of A.x fused with the leaf's first M2M shift: a CTA per leaf computes
// M_leaf = sum_d x_d C_{leaf,d} (kTreeLanes lanes per coefficient over interleaved DOFs, lane
// sums added by shuffles in a fixed order) and, when its parent's multipole is needed, shifts
// it to the parent's centre into Yup (the same shift as k_m2m_level), so the upward pass
// starts at the leaves' parents.  Fl: the F tables of every level, leaf_level: each leaf's level.
template <typename CT>
__device__ __forceinline__ double2 load_c2(const CT* c) {
  const CT v = *c;
  return make_double2((double)v.x, (double)v.y);
}

template <int P, typename CT>
__global__ void __launch_bounds__(tree_threads<P>(), 5) k_p2m_leaf(const int* __restrict__ leaves, const int* __restrict__ leaf_dof_off,
                                                                   const int* __restrict__ leaf_dof, const CT* __restrict__ C,
                                                                   const double* __restrict__ x, const int* __restrict__ node_up,
                                                                   const int* __restrict__ leaf_level, const double* __restrict__ node_X,
                                                                   const double2* __restrict__ Ftab, double2* __restrict__ M,
                                                                   double2* __restrict__ Yup) {
  pdl_enter();
  constexpr int NC = ncoef(P), NF = (P + 1) * (P + 1);
  __shared__ double2 sF[NF];
  __shared__ double2 sHalf[NC];
  __shared__ double2 sM[NF];
  const int li = blockIdx.x, leaf = leaves[li];
  const int o = threadIdx.x / kTreeLanes, q = threadIdx.x % kTreeLanes;
  const int up = node_up[leaf];
  if (up >= 0) {  // the shift's table, loaded while the multipole is summed
    const double2* Ft = Ftab + ((size_t)(leaf_level[li] - 1) * 8 + child_octant(node_X, leaf, up)) * NF;
    for (int i = threadIdx.x; i < NF; i += blockDim.x) sF[i] = Ft[i];
  }
  const int d0 = leaf_dof_off[li], d1 = leaf_dof_off[li + 1];
  double2 acc = make_double2(0.0, 0.0);
  if (o < NC)
    for (int j = d0 + q; j < d1; j += kTreeLanes) {
      const double xv = x[leaf_dof[j]];
      const double2 c = load_c2(C + (size_t)j * NC + o);
      acc.x = fma(xv, c.x, acc.x);
      acc.y = fma(xv, c.y, acc.y);
    }
  acc = tree_lanes_sum(acc);
  if (o < NC && q == 0) {
    M[(size_t)leaf * 2 * NC + o] = acc;
    sHalf[o] = acc;
  }
  if (up < 0) return;  // uniform over the CTA
  __syncthreads();
  expand_full_group<P, 1, false>(sHalf, sM, threadIdx.x, blockDim.x);
  __syncthreads();
  double2 a0 = make_double2(0.0, 0.0), a1 = a0;
  if (o < NC) {
    int n = 0, m = 0;
    decode_nm(o, n, m);
    m2m_terms<P, 1>(n, m, q, sF, sM, a0, a1);
  }
  a0 = tree_lanes_sum(a0);
  if (o < NC && q == 0) Yup[(size_t)leaf * 2 * NC + o] = a0;
}

// ---------------------------------------------------------------------------
// M2L grouped by translation vector.
//   k_s_tables    (set-up) one irregular-harmonic table S(d_g) per group, all orders
//   k_m2l_grp     block per chunk of <= 8 pairs of one group: the group's table in shared
//                 memory is applied to the 8 source multipoles (one S load feeds 8 pairs);
//                 partial locals to slot k of each pair
//   k_m2l_reduce  per target bucket: L = sum of its slots (CSR order, deterministic)
template <int P>
__global__ void k_s_tables(int ngroups, const double* __restrict__ gvec, double2* __restrict__ Sg) {
  constexpr int Q = 2 * P, NS = (Q + 1) * (Q + 1);
  const int g = blockIdx.x;
  if (g < ngroups && threadIdx.x < 32) S_full_column<Q>(threadIdx.x, gvec[3 * g], gvec[3 * g + 1], gvec[3 * g + 2], Sg + (size_t)g * NS);
}


template <int P>
constexpr int m2l_grp_smem_bytes() {
  return (int)sizeof(double2) * ((2 * P + 1) * (2 * P + 1) + 8 * 2 * ncoef(P));
}

// Thread per output coefficient L_n^m (m >= 0) of one density, applied to the chunk's <= 8
// source multipoles in their m >= 0 half: with M^{-m'} = (-1)^{m'} conj(M^{m'}) the terms of
// m' and -m' combine into one real 2x2 block on (Re M^{m'}, Im M^{m'}),
//   [[Re(S+ + s S-), -Im(S+) + s Im(S-)], [Im(S+ + s S-), Re(S+ - s S-)]],
// S+- = S_{n+n'}^{m+-m'}, s = (-1)^{m'}: 4 real multiply-adds per term and pair instead of 8.
template <int P, int ND>
__global__ void __launch_bounds__(((2 * ncoef(P) + 31) / 32) * 32) k_m2l_grp(const int* __restrict__ chunk_grp, const int* __restrict__ chunk_begin,
                                                                             const int* __restrict__ chunk_cnt, const int* __restrict__ grp_pair,
                                                                             const int* __restrict__ m2l_src, const double2* __restrict__ Sg,
                                                                             const double2* __restrict__ M, double2* __restrict__ Y) {
  constexpr int NC = ncoef(P), Q = 2 * P, NS = (Q + 1) * (Q + 1);
  extern __shared__ double2 smem_grp[];
  double2* sS = smem_grp;        // [NS]
  double2* sM = smem_grp + NS;   // [8][ND][NC] half-stored multipoles
  const int c = blockIdx.x;
  const int g = chunk_grp[c], b0 = chunk_begin[c], cnt = chunk_cnt[c];
  const int t = threadIdx.x;
  {
    const double2* src = Sg + (size_t)g * NS;
    for (int i = t; i < NS; i += blockDim.x) sS[i] = src[i];
    for (int j = 0; j < cnt; ++j) {
      const double2* mp = M + (size_t)m2l_src[grp_pair[b0 + j]] * 2 * NC;
      for (int i = t; i < ND * NC; i += blockDim.x) sM[j * ND * NC + i] = mp[i];
    }
    for (int j = cnt; j < 8; ++j)
      for (int i = t; i < ND * NC; i += blockDim.x) sM[j * ND * NC + i] = make_double2(0.0, 0.0);
  }
  __syncthreads();
  if (t >= ND * NC) return;
  const int dd = (t < NC) ? 0 : 1;
  const int o = t - dd * NC;
  int n = 0, m = 0;
  decode_nm(o, n, m);
  double2 acc[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) acc[j] = make_double2(0.0, 0.0);
  const double2* sMd = sM + dd * NC;
  for (int n1 = 0; n1 <= P; ++n1) {
    const int l = n + n1;
    const double2* Srow = sS + l * (l + 1) + m;
    const int cb = n1 * (n1 + 1) / 2;
    {
      const double2 s0 = Srow[0];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const double a = sMd[j * ND * NC + cb].x;
        acc[j].x = fma(s0.x, a, acc[j].x);
        acc[j].y = fma(s0.y, a, acc[j].y);
      }
    }
    for (int m1 = 1; m1 <= n1; ++m1) {
      const double2 sp = Srow[m1], sm = Srow[-m1];
      const double sg = (m1 & 1) ? -1.0 : 1.0;
      const double b00 = sp.x + sg * sm.x, b01 = -sp.y + sg * sm.y;
      const double b10 = sp.y + sg * sm.y, b11 = sp.x - sg * sm.x;
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const double2 x = sMd[j * ND * NC + cb + m1];
        acc[j].x = fma(b00, x.x, fma(b01, x.y, acc[j].x));
        acc[j].y = fma(b10, x.x, fma(b11, x.y, acc[j].y));
      }
    }
  }
  const double sg = (n & 1) ? -1.0 : 1.0;
#pragma unroll
  for (int j = 0; j < 8; ++j)
    if (j < cnt) Y[(size_t)grp_pair[b0 + j] * 2 * NC + t] = make_double2(sg * acc[j].x, sg * acc[j].y);
}

template <int P, int ND>
__global__ void k_m2l_reduce(int ntargets, const int* __restrict__ targets, const int* __restrict__ m2l_off, const double2* __restrict__ Y,
                             double2* __restrict__ L) {
  constexpr int NC = ncoef(P);
  const int64_t total = (int64_t)ntargets * ND * NC;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int ti = (int)(e / (ND * NC));
    const int r = (int)(e - (int64_t)ti * ND * NC);
    const int tgt = targets[ti];
    double2 s = make_double2(0.0, 0.0);
    for (int k = m2l_off[tgt]; k < m2l_off[tgt + 1]; ++k) s = cadd(s, Y[(size_t)k * 2 * NC + r]);
    L[(size_t)tgt * 2 * NC + r] = s;
  }
}

// ---------------------------------------------------------------------------
// L2L: one launch per level, top-down (moments.hpp:869-884), a CTA per (parent, child) pair of
// the level: L'_k^j += sum_{n>=k} L_n^m conj(F_{n-k}^{m-j}), kTreeLanes lanes per output.  Only
// the child's CTA writes the child in this launch, and parents are only read.
template <int P, int ND>
__global__ void __launch_bounds__(tree_threads<P>(), 5) k_l2l_pairs(const int2* __restrict__ pairs, const double* __restrict__ node_X,
                                                                 const double2* __restrict__ Fl, double2* __restrict__ L) {
  pdl_enter();
  constexpr int NC = ncoef(P), NF = (P + 1) * (P + 1);
  __shared__ double2 sF[NF];
  __shared__ double2 sL[ND * NF];
  const int2 pc = pairs[blockIdx.x];
  const int par = pc.x, c = pc.y;
  const double2* Ft = Fl + (size_t)child_octant(node_X, c, par) * NF;
  for (int i = threadIdx.x; i < NF; i += blockDim.x) sF[i] = Ft[i];
  expand_full_group<P, ND, false>(L + (size_t)par * 2 * NC, sL, threadIdx.x, blockDim.x);
  __syncthreads();
  const int o = threadIdx.x / kTreeLanes, q = threadIdx.x % kTreeLanes;
  double2 a0 = make_double2(0.0, 0.0), a1 = a0;
  if (o < NC) {
    int k = 0, j = 0;
    decode_nm(o, k, j);
    l2l_terms<P, ND>(k, j, q, sF, sL, a0, a1);
  }
  a0 = tree_lanes_sum(a0);
  if (ND == 2) a1 = tree_lanes_sum(a1);
  if (o < NC && q == 0) {
    double2* dst = L + (size_t)c * 2 * NC;
    dst[o] = cadd(dst[o], a0);
    if (ND == 2) dst[NC + o] = cadd(dst[NC + o], a1);
  }
}

// ---------------------------------------------------------------------------
// Targets: one block per near block (targets sharing a deepest bucket).  The block
// stages (phi, phin) of its DOF set in shared memory chunk by chunk, each warp reduces
// the cached weight rows of its targets, then evaluates L2P and writes the BIE rows.
template <int P, int ND>
__global__ void __launch_bounds__(128) k_targets(const NearBlockDev* __restrict__ blocks, const int* __restrict__ nb_dofs,
                                                 const int* __restrict__ nb_targets, const double* __restrict__ WG,
                                                 const double* __restrict__ WGn, const double* __restrict__ Xs,
                                                 const double* __restrict__ node_X, const double2* __restrict__ L,
                                                 const double* __restrict__ phi, const double* __restrict__ phin,
                                                 const int* __restrict__ point_dof_off, const int* __restrict__ point_dof,
                                                 const int* __restrict__ dof_kind, const double* __restrict__ diag,
                                                 double* __restrict__ rows, double* __restrict__ GPhin_out,
                                                 double* __restrict__ GnPhi_out, int chunk) {
  constexpr int NC = ncoef(P);
  extern __shared__ double2 smem[];
  double2* xs = smem;                   // [chunk] (phi, phin)
  double2* accs = smem + chunk;         // [ntgt] near sums (G.phin, Gn.phi)
  __shared__ double2 sL[2 * NC];
  __shared__ double sHalf[P + 1], sRec[(P + 1) * (P + 1)];  // 1/(2k), 1/(n^2 - m^2) of the L2P recurrence
  for (int i = threadIdx.x; i < (P + 1) * (P + 1); i += blockDim.x) {
    const int n = i / (P + 1), m = i - n * (P + 1);
    sRec[i] = n > m ? 1.0 / double(n * n - m * m) : 0.0;
    if (i <= P) sHalf[i] = i > 0 ? 1.0 / (2.0 * i) : 0.0;
  }
  const NearBlockDev B = blocks[blockIdx.x];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nwarp = blockDim.x >> 5;
  for (int i = threadIdx.x; i < ND * NC; i += blockDim.x) sL[i] = L[(size_t)B.node * 2 * NC + i];
  for (int i = threadIdx.x; i < B.ntgt; i += blockDim.x) accs[i] = make_double2(0, 0);
  for (int c0 = 0; c0 < B.ndof; c0 += chunk) {
    const int cn = min(chunk, B.ndof - c0);
    __syncthreads();
    for (int i = threadIdx.x; i < cn; i += blockDim.x) {
      const int d = nb_dofs[B.dof_off + c0 + i];
      xs[i] = make_double2(phi[d], phin[d]);
    }
    __syncthreads();
    for (int tl = warp; tl < B.ntgt; tl += nwarp) {
      const double* wg = WG + B.w_off + (int64_t)tl * B.ndof + c0;
      const double* wgn = WGn + B.w_off + (int64_t)tl * B.ndof + c0;
      double s0 = 0.0, s1 = 0.0;
      for (int i = lane; i < cn; i += 32) {
        const double2 v = xs[i];
        s0 = fma(wg[i], v.y, s0);
        s1 = fma(wgn[i], v.x, s1);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      }
      if (lane == 0) {
        accs[tl].x += s0;
        accs[tl].y += s1;
      }
    }
  }
  __syncthreads();
  const double cx = node_X[3 * B.node], cy = node_X[3 * B.node + 1], cz = node_X[3 * B.node + 2];
  for (int tl = warp; tl < B.ntgt; tl += nwarp) {
    const int p = nb_targets[B.tgt_off + tl];
    const double x = Xs[3 * p] - cx, y = Xs[3 * p + 1] - cy, z = Xs[3 * p + 2] - cz;
    // L2P: lane m owns column m of F_n^m(x - c)
    double f0 = 0.0, f1 = 0.0;
    const int m = lane;
    if (m <= P) {
      const double r2 = x * x + y * y + z * z;
      double2 cur = make_double2(1.0, 0.0);
      for (int k = 1; k <= m; ++k) cur = cscale(cmul(cur, make_double2(x, y)), sHalf[k]);
      double2 prev = make_double2(0.0, 0.0);
      const double w = (m == 0) ? 1.0 : 2.0;
      for (int n = m; n <= P; ++n) {
        if (n > m) {
          const double inv = sRec[n * (P + 1) + m];
          double2 nx = make_double2(((2 * n - 1) * z * cur.x - r2 * prev.x) * inv, ((2 * n - 1) * z * cur.y - r2 * prev.y) * inv);
          prev = cur;
          cur = nx;
        }
        // Re(L conj(F))
        const double2 l0 = sL[cidx(n, m)];
        f0 += w * (l0.x * cur.x + l0.y * cur.y);
        if (ND == 2) {
          const double2 l1 = sL[NC + cidx(n, m)];
          f1 += w * (l1.x * cur.x + l1.y * cur.y);
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      f0 += __shfl_xor_sync(0xffffffffu, f0, o);
      if (ND == 2) f1 += __shfl_xor_sync(0xffffffffu, f1, o);
    }
    const double GPhin = accs[tl].x + f0, GnPhi = accs[tl].y + f1;
    if (lane == 0) {
      if (ND == 2) {
        if (GPhin_out) GPhin_out[p] = GPhin;
        if (GnPhi_out) GnPhi_out[p] = GnPhi;
      } else if (GnPhi_out) {
        // GnPhi alone from the combined expansion: valid when phin = 0 (far of M[0] - M[1] = -far of M[1])
        GnPhi_out[p] = accs[tl].y - f0;
      }
    }
    if (rows) {
      for (int k = point_dof_off[p] + lane; k < point_dof_off[p + 1]; k += 32) {
        const int i = point_dof[k];
        rows[i] = (dof_kind[i] == 2) ? phi[i] : GPhin - (GnPhi + diag[i] * phi[i]);
      }
    }
  }
}

// Targets for A.x (the Krylov operator): with the known values zero, each DOF enters the
// rows through one weight only -- WG (times phin = x) for a Dirichlet DOF, -WGn (times
// phi = x) otherwise -- so the near sum of a row is one dot product with the combined weights
// Wc = [Dirichlet] WG - [other] WGn (half the weight bytes of the general kernel), read
// straight from the unknown vector x; a CORNER row is its own unknown (phi_i = x_i).
//
// HBM-bound: every weight is read once per application (369 MB in FP32 at tank_60k: 5,476
// blocks of ~12 rows x ~1,570 columns).  One small CTA per near block, many resident per SM,
// so that one CTA's gather of x (a dependent load through the block's DOF list) overlaps the
// weight streams of the others: the block's x values go to shared memory in chunks of kNsXCap
// columns, then warp tl % kNsWarps streams row tl, every lane kNsUnroll 16-byte loads ahead
// of its FMAs, and reduces it by a warp shuffle in a fixed order (the result does not depend
// on timing).  Weight rows are padded with zeros to a multiple of 4 columns in both precisions
// (16-byte aligned loads); x past the block's last column is 0.  FP32: x in four planes, column
// c at xs[(c % 4) * q + c / 4] (q = chunk / 4), so lanes reading consecutive column groups hit
// consecutive words.  The near sum of each target goes to its target slot; the rows (near sum
// + the far field of the bucket's local expansion - diag x, or x on a CORNER row) are written
// by k_target_rows afterwards.
constexpr int kNsThreads = 128;
constexpr int kNsWarps = kNsThreads / 32;
constexpr int kNsXCap = 2048;  // x values per chunk (a multiple of 4)
constexpr int kNsUnroll = 4;   // 16-byte weight loads in flight per lane

// dynamic shared memory of k_near_sums: one x chunk and a running sum per target
inline size_t ns_smem_bytes(int max_ntgt) { return sizeof(double) * (kNsXCap + (size_t)std::max(max_ntgt, 1)); }

template <typename WT>
__global__ void __launch_bounds__(kNsThreads) k_near_sums(const NearBlockDev* __restrict__ blocks, const int* __restrict__ nb_dofs,
                                                          const WT* __restrict__ Wc, const double* __restrict__ x,
                                                          double* __restrict__ near_sum) {
  pdl_enter();
  constexpr int VC = 16 / (int)sizeof(WT);  // columns per 16-byte load
  extern __shared__ __align__(16) double ns_smem[];
  double* xs = ns_smem;          // [kNsXCap]
  double* run = xs + kNsXCap;    // [ntgt] sums over the previous chunks
  const NearBlockDev B = blocks[blockIdx.x];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int stride = (B.ndof + 3) & ~3;
  if (B.ntgt <= 0) return;
  if (stride == 0) {
    for (int tl = threadIdx.x; tl < B.ntgt; tl += kNsThreads) near_sum[B.tgt_off + tl] = 0.0;
    return;
  }
  for (int c0 = 0; c0 < stride; c0 += kNsXCap) {
    const int cn = min(kNsXCap, stride - c0);  // a multiple of 4
    const int real = min(cn, B.ndof - c0);
    const bool last = c0 + cn >= stride;
    if (c0 > 0) __syncthreads();  // every warp is done with the previous chunk
    const int* idx = nb_dofs + B.dof_off + c0;
    if constexpr (VC == 4) {
      const int q = cn >> 2;
      for (int i = threadIdx.x; i < cn; i += kNsThreads) xs[(i & 3) * q + (i >> 2)] = i < real ? x[idx[i]] : 0.0;
    } else {
      for (int i = threadIdx.x; i < cn; i += kNsThreads) xs[i] = i < real ? x[idx[i]] : 0.0;
    }
    __syncthreads();
    const int ng = cn / VC;  // 16-byte groups of a row in this chunk
    for (int tl = warp; tl < B.ntgt; tl += kNsWarps) {
      const WT* wrow = Wc + B.w4_off + (int64_t)tl * stride + c0;
      double s0 = 0.0, s1 = 0.0;
      if constexpr (VC == 4) {
        const float4* w4 = reinterpret_cast<const float4*>(wrow);
        const int q = ng;
        int g = lane;
        for (; g + 32 * (kNsUnroll - 1) < ng; g += 32 * kNsUnroll) {
          float4 v[kNsUnroll];
#pragma unroll
          for (int u = 0; u < kNsUnroll; ++u) v[u] = __ldcs(w4 + g + 32 * u);
#pragma unroll
          for (int u = 0; u < kNsUnroll; ++u) {
            const int gg = g + 32 * u;
            s0 = fma((double)v[u].x, xs[gg], s0);
            s1 = fma((double)v[u].y, xs[q + gg], s1);
            s0 = fma((double)v[u].z, xs[2 * q + gg], s0);
            s1 = fma((double)v[u].w, xs[3 * q + gg], s1);
          }
        }
        for (; g < ng; g += 32) {
          const float4 v = __ldcs(w4 + g);
          s0 = fma((double)v.x, xs[g], s0);
          s1 = fma((double)v.y, xs[q + g], s1);
          s0 = fma((double)v.z, xs[2 * q + g], s0);
          s1 = fma((double)v.w, xs[3 * q + g], s1);
        }
      } else {
        const double2* w2 = reinterpret_cast<const double2*>(wrow);
        const double2* x2 = reinterpret_cast<const double2*>(xs);
        int g = lane;
        for (; g + 32 * (kNsUnroll - 1) < ng; g += 32 * kNsUnroll) {
          double2 v[kNsUnroll];
#pragma unroll
          for (int u = 0; u < kNsUnroll; ++u) v[u] = __ldcs(w2 + g + 32 * u);
#pragma unroll
          for (int u = 0; u < kNsUnroll; ++u) {
            const double2 xv = x2[g + 32 * u];
            s0 = fma(v[u].x, xv.x, s0);
            s1 = fma(v[u].y, xv.y, s1);
          }
        }
        for (; g < ng; g += 32) {
          const double2 v = __ldcs(w2 + g), xv = x2[g];
          s0 = fma(v.x, xv.x, s0);
          s1 = fma(v.y, xv.y, s1);
        }
      }
      double s = s0 + s1;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
      if (lane == 0) {
        // row tl stays on this warp in every chunk: its running sum needs no synchronisation
        const double tot = (c0 > 0 ? run[tl] : 0.0) + s;
        if (last)
          near_sum[B.tgt_off + tl] = tot;
        else
          run[tl] = tot;
      }
    }
  }
}

// L2P of one local expansion (shared memory, read at the same address by every thread: a
// broadcast) at the point d from its centre: the expansion against the regular solid harmonics
// of d, column m by column from R_m^m = (x + iy)^m / (2^m m!) with
// (n - m)(n + m) R_n^m = (2n - 1) z R_{n-1}^m - r^2 R_{n-2}^m, fully unrolled so that the
// recurrence constants fold at compile time.
template <int P>
__device__ __forceinline__ double l2p_point(const double2* __restrict__ sL, double px, double py, double pz) {
  const double r2 = px * px + py * py + pz * pz;
  double far = 0.0;
  double2 rmm = make_double2(1.0, 0.0);  // R_m^m
#pragma unroll
  for (int m = 0; m <= P; ++m) {
    if (m > 0) rmm = cscale(cmul(rmm, make_double2(px, py)), 1.0 / (2.0 * m));
    double2 prev = make_double2(0.0, 0.0), cur = rmm;
    double fm = 0.0;
#pragma unroll
    for (int n = m; n <= P; ++n) {
      if (n > m) {
        const double inv = 1.0 / double(n * n - m * m);
        const double2 nx = make_double2(((2 * n - 1) * pz * cur.x - r2 * prev.x) * inv, ((2 * n - 1) * pz * cur.y - r2 * prev.y) * inv);
        prev = cur;
        cur = nx;
      }
      const double2 l0 = sL[cidx(n, m)];
      fm += l0.x * cur.x + l0.y * cur.y;
    }
    far += (m == 0 ? 1.0 : 2.0) * fm;
    // keep the next column's expansion loads below this column (bounded register use)
    asm volatile("" ::: "memory");
  }
  return far;
}

// Rows of A.x from the near sums k_near_sums left per target slot: rows[i] = near + far -
// diag_i x_i (a CORNER row: x_i).  far = the L2P at the point of the local expansion its bucket
// would hold after the downward pass.  L2L is exact for a truncated local expansion (it
// re-expands the same degree-P harmonic polynomial about another centre), so that equals the sum
// of the L2Ps of the M2L locals of the bucket and of its ancestors, each about its own centre:
// with the block's path (the bucket and its ancestors that are M2L targets, deepest first) the
// downward pass is not needed.  One CTA per near block (= target bucket): the path's locals go
// to shared memory, a thread per (path node, target) pair evaluates one L2P (pairs node-major,
// so a warp reads few distinct expansions), and thread t adds its target's L2Ps in path order.
// L null: no far field (the near-field operator alone).  Dynamic shared memory:
// target_rows_smem_bytes(P, max_path, max_ntgt).
constexpr int kRowsThreads = 64;
inline size_t target_rows_smem_bytes(int p, int max_path, int max_ntgt) {
  return sizeof(double2) * (size_t)ncoef(p) * std::max(max_path, 1) + sizeof(double) * (size_t)std::max(max_path, 1) * std::max(max_ntgt, 1);
}

template <int P>
__global__ void __launch_bounds__(kRowsThreads) k_target_rows(const NearBlockDev* __restrict__ blocks, const int* __restrict__ nb_targets,
                                                              const double* __restrict__ Xs, const double* __restrict__ node_X,
                                                              const double2* __restrict__ L, const int* __restrict__ path_off,
                                                              const int* __restrict__ path, const double* __restrict__ near_sum,
                                                              const double* __restrict__ x, const int* __restrict__ point_dof_off,
                                                              const int* __restrict__ point_dof, const int* __restrict__ dof_kind,
                                                              const double* __restrict__ diag, double* __restrict__ rows) {
  pdl_enter();
  constexpr int NC = ncoef(P);
  extern __shared__ __align__(16) double2 rows_smem[];
  const NearBlockDev B = blocks[blockIdx.x];
  const int k0 = L ? path_off[blockIdx.x] : 0, np = L ? path_off[blockIdx.x + 1] - k0 : 0;
  double2* sL = rows_smem;                                            // [np][NC]
  double* part = reinterpret_cast<double*>(rows_smem + (size_t)np * NC);  // [ntgt][np]
  for (int i = threadIdx.x; i < np * NC; i += kRowsThreads) {
    const int k = i / NC;
    sL[i] = L[(size_t)path[k0 + k] * 2 * NC + (i - k * NC)];
  }
  __syncthreads();
  for (int j = threadIdx.x; j < np * B.ntgt; j += kRowsThreads) {
    const int k = j / B.ntgt, tl = j - k * B.ntgt;
    const int a = path[k0 + k], p = nb_targets[B.tgt_off + tl];
    part[tl * np + k] = l2p_point<P>(sL + (size_t)k * NC, Xs[3 * p] - node_X[3 * a], Xs[3 * p + 1] - node_X[3 * a + 1],
                                     Xs[3 * p + 2] - node_X[3 * a + 2]);
  }
  __syncthreads();
  for (int tl = threadIdx.x; tl < B.ntgt; tl += kRowsThreads) {
    const int p = nb_targets[B.tgt_off + tl];
    double far = 0.0;
    for (int k = 0; k < np; ++k) far += part[tl * np + k];
    const double g = near_sum[B.tgt_off + tl] + far;
    const int d1 = point_dof_off[p + 1];
    for (int d = point_dof_off[p]; d < d1; ++d) {
      const int i = point_dof[d];
      const int kd = dof_kind[i];
      rows[i] = (kd == 2) ? x[i] : g - (kd == 0 ? 0.0 : diag[i] * x[i]);
    }
  }
}

// Combined near weights of A.x (set-up): Wc = WG for a Dirichlet DOF column, -WGn otherwise.
template <typename WT>
__global__ void k_combine_weights(const NearBlockDev* __restrict__ blocks, const int* __restrict__ nb_dofs, const int* __restrict__ dof_kind,
                                  const double* __restrict__ WG, const double* __restrict__ WGn, WT* __restrict__ Wc) {
  // each row padded with zeros to a multiple of 4 columns (16-byte aligned rows for the vector
  // loads of k_near_sums), from the block's own offset w4_off, in both precisions
  const NearBlockDev B = blocks[blockIdx.x];
  const int stride = (B.ndof + 3) & ~3;
  const int64_t base = B.w4_off;
  const int64_t total = (int64_t)B.ntgt * stride;
  for (int64_t e = threadIdx.x; e < total; e += blockDim.x) {
    const int64_t tl = e / stride;
    const int j = (int)(e - tl * stride);
    if (j < B.ndof) {
      const int64_t w = B.w_off + tl * B.ndof + j;
      Wc[base + e] = (WT)(dof_kind[nb_dofs[B.dof_off + j]] == 0 ? WG[w] : -WGn[w]);
    } else {
      Wc[base + e] = (WT)0;
    }
  }
}

// ---------------------------------------------------------------------------
// Near-field quadrature (set-up): the weights of a target over the DOFs of its near block,
// summing every incident element vertex whose element lies in the block's near element ranges.
__device__ __forceinline__ double dnorm3(double x, double y, double z) { return sqrt(x * x + y * y + z * z); }

// All three vertex weights of element s for target t at once (the kernel evaluations at the
// quadrature points are shared).  Adjacent element (target is a vertex): rotated so the
// target is vertex 0, Duffy-collapsed 5x5 Gauss rule, and the Gn weight of the element's first
// vertex dropped (rigid-mode diagonal); near element (centroid within near_region): 5x5 rule;
// otherwise the Dunavant 6-point rule (fill_direct_linear / fill_nonadj_linear,
// BEM_solveBVP_GMRES_FMM.hpp:1824-1891).
__device__ void elem_weights3(int s, int t, const double* __restrict__ Xs, const int* __restrict__ e_vtx,
                              const double* __restrict__ e_near, double near_region, double wG[3], double wGn[3]) {
  const int v[3] = {e_vtx[3 * s], e_vtx[3 * s + 1], e_vtx[3 * s + 2]};
  const double J = e_near[8 * s];
  const double crx = e_near[8 * s + 1], cry = e_near[8 * s + 2], crz = e_near[8 * s + 3];
  const double xt = Xs[3 * t], yt = Xs[3 * t + 1], zt = Xs[3 * t + 2];
  double G[3] = {0.0, 0.0, 0.0}, Gn[3] = {0.0, 0.0, 0.0};
  if (v[0] == t || v[1] == t || v[2] == t) {
    const int o = (v[0] == t) ? 0 : (v[1] == t ? 1 : 2);
    const int r0 = v[o], r1 = v[(o + 1) % 3], r2 = v[(o + 2) % 3];
    const double X0[3] = {Xs[3 * r0], Xs[3 * r0 + 1], Xs[3 * r0 + 2]};
    const double X1[3] = {Xs[3 * r1], Xs[3 * r1 + 1], Xs[3 * r1 + 2]};
    const double X2[3] = {Xs[3 * r2], Xs[3 * r2 + 1], Xs[3 * r2 + 2]};
    for (int g = 0; g < 25; ++g) {
      const double t0 = c_gw[g][0], t1 = c_gw[g][1], ww = c_gw[g][2];
      const double N[3] = {t0, t1 * (1. - t0), (t0 - 1.) * (t1 - 1.)};
      const double Rx = N[0] * X0[0] + N[1] * X1[0] + N[2] * X2[0] - xt;
      const double Ry = N[0] * X0[1] + N[1] * X1[1] + N[2] * X2[1] - yt;
      const double Rz = N[0] * X0[2] + N[1] * X1[2] + N[2] * X2[2] - zt;
      const double nr_inv = rsqrt(Rx * Rx + Ry * Ry + Rz * Rz);
      const double base = ww * (1. - t0) * nr_inv;
      const double dn = -((Rx * crx + Ry * cry + Rz * crz) * nr_inv);
      const double bn = dn * base * nr_inv;
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        const double Na = N[(a - o + 3) % 3];
        G[a] += base * Na;  // times J after the loop
        Gn[a] += bn * Na;
      }
    }
    Gn[0] = 0.0;  // the element's first vertex: dropped (rigid-mode diagonal)
  } else {
    const double X0[3] = {Xs[3 * v[0]], Xs[3 * v[0] + 1], Xs[3 * v[0] + 2]};
    const double X1[3] = {Xs[3 * v[1]], Xs[3 * v[1] + 1], Xs[3 * v[1] + 2]};
    const double X2[3] = {Xs[3 * v[2]], Xs[3 * v[2] + 1], Xs[3 * v[2] + 2]};
    const double dcx = e_near[8 * s + 4] - xt, dcy = e_near[8 * s + 5] - yt, dcz = e_near[8 * s + 6] - zt;
    if (dnorm3(dcx, dcy, dcz) < near_region) {
      for (int g = 0; g < 25; ++g) {
        const double t0 = c_gw[g][0], t1 = c_gw[g][1], ww = c_gw[g][2];
        const double N[3] = {t0, t1 * (1. - t0), (t0 - 1.) * (t1 - 1.)};
        const double Rx = N[0] * X0[0] + N[1] * X1[0] + N[2] * X2[0] - xt;
        const double Ry = N[0] * X0[1] + N[1] * X1[1] + N[2] * X2[1] - yt;
        const double Rz = N[0] * X0[2] + N[1] * X1[2] + N[2] * X2[2] - zt;
        const double nr_inv = rsqrt(Rx * Rx + Ry * Ry + Rz * Rz);
        const double sw = ww * (1. - t0) * nr_inv;
        const double dn = (Rx * crx + Ry * cry + Rz * crz) * nr_inv;
        const double tw = dn * sw * nr_inv;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          G[a] += sw * N[a];  // times J after the loop
          Gn[a] -= tw * N[a];
        }
      }
    } else {
      for (int q = 0; q < 6; ++q) {
        const double N[3] = {c_dv[q][0], c_dv[q][1], c_dv[q][2]};
        const double Rx = N[0] * X0[0] + N[1] * X1[0] + N[2] * X2[0] - xt;
        const double Ry = N[0] * X0[1] + N[1] * X1[1] + N[2] * X2[1] - yt;
        const double Rz = N[0] * X0[2] + N[1] * X1[2] + N[2] * X2[2] - zt;
        const double nr_inv = rsqrt(Rx * Rx + Ry * Ry + Rz * Rz);
        const double dn = (Rx * crx + Ry * cry + Rz * crz) * nr_inv;
        const double sw = c_dv[q][3] * nr_inv, tw = dn * sw * nr_inv;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          G[a] += sw * N[a];  // times J after the loop
          Gn[a] -= tw * N[a];
        }
      }
    }
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    wG[a] = J * G[a];  // every rule's single-layer sum carries the factor J once
    wGn[a] = Gn[a];
  }
}

// Near-field weights.  Persistent CTAs take whole near blocks from a counter; for a block the
// CTA stages its element ranges and, where it fits in shared memory, the block's element list
// and the map from each DOF column's incidences (in incidence order) to the element-vertex
// slot they read (or "not near").  Then for each target of the block it integrates every near
// element once for its three vertices into a per-CTA scratch row in global memory
// (L2-resident), and each thread sums, for the DOF columns it owns, its incidences' slots in
// incidence order.  The searches of an element in the block's ranges are done once per block
// instead of once per target; a block whose map does not fit searches per target.  The
// quadrature work is one evaluation per (target, element) instead of one per (target, DOF,
// element).
constexpr int kNearThreads = 256;
constexpr int kNearMapBytes = 70 * 1024;  // element list, column offsets and incidence map of one block
constexpr unsigned short kNotNear = 0xFFFFu;

// the range r of the sorted half-open ranges holding element s, or -1
__device__ __forceinline__ int find_range(const int* sRng, int nrng, int s) {
  int lo = 0, hi = nrng - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    if (s < sRng[2 * mid])
      hi = mid - 1;
    else if (s >= sRng[2 * mid + 1])
      lo = mid + 1;
    else
      return mid;
  }
  return -1;
}

// the range r with sR[r] <= li < sR[r + 1]
__device__ __forceinline__ int range_of_local(const int* sR, int nrng, int li) {
  int lo = 0, hi = nrng - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (sR[mid] <= li)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

__global__ void __launch_bounds__(kNearThreads, 3) k_near_weights(int nblocks, int* __restrict__ next_block, int max_nrng,
                                                              const NearBlockDev* __restrict__ blocks, const int* __restrict__ nb_dofs,
                                                              const int* __restrict__ nb_targets, const int* __restrict__ nb_ranges,
                                                              const int* __restrict__ dof_inc_off, const int* __restrict__ dof_inc,
                                                              const double* __restrict__ Xs, const int* __restrict__ e_vtx,
                                                              const double* __restrict__ e_near, double near_region, double2* __restrict__ scratch,
                                                              int64_t scratch_stride, double* __restrict__ WG, double* __restrict__ WGn) {
  // shared: ranges [2 max_nrng], prefix [max_nrng + 1], then (map mode) element list [nel],
  // column offsets [ndof + 1] and the incidence map [total incidences] (16-bit slots)
  extern __shared__ int sm_near[];
  __shared__ int s_bi, s_total;
  __shared__ int s_warp[kNearThreads / 32];
  double2* E = scratch + (int64_t)blockIdx.x * scratch_stride;  // [3 * near elements] (G, Gn)
  int* sRng = sm_near;
  int* sR = sm_near + 2 * max_nrng;
  int* sMap0 = sR + max_nrng + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  while (true) {
    __syncthreads();  // the previous block's shared data are no longer read
    if (threadIdx.x == 0) s_bi = atomicAdd(next_block, 1);
    __syncthreads();
    const int bi = s_bi;
    if (bi >= nblocks) return;
    const NearBlockDev B = blocks[bi];
    const int nrng = B.nrng, ndof = B.ndof;
    const int* rng = nb_ranges + 2 * B.rng_off;
    for (int i = threadIdx.x; i < 2 * nrng; i += blockDim.x) sRng[i] = rng[i];
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int r = 0; r < nrng; ++r) {
        sR[r] = acc;
        acc += sRng[2 * r + 1] - sRng[2 * r];
      }
      sR[nrng] = acc;
    }
    // incidences of the block's columns: a contiguous run of columns per thread, block scan
    const int per = (ndof + blockDim.x - 1) / blockDim.x;
    const int j0 = min(ndof, (int)threadIdx.x * per), j1 = min(ndof, j0 + per);
    int local = 0;
    for (int j = j0; j < j1; ++j) {
      const int d = nb_dofs[B.dof_off + j];
      local += dof_inc_off[d + 1] - dof_inc_off[d];
    }
    int incl = local;
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
        const int v = s_warp[w];
        s_warp[w] = acc;
        acc += v;
      }
      s_total = acc;
    }
    __syncthreads();
    const int nel = sR[nrng], total = s_total;
    // map mode when the element list, the column offsets and the map fit
    const int map_words = nel + (ndof + 1) + (total + 1) / 2;
    const bool use_map = map_words * 4 <= kNearMapBytes;
    int* sElem = sMap0;                                                  // [nel] element of local index li
    int* sCol = sElem + nel;                                             // [ndof + 1]
    unsigned short* sMap = reinterpret_cast<unsigned short*>(sCol + ndof + 1);  // [total]
    if (use_map) {
      for (int li = threadIdx.x; li < nel; li += blockDim.x) {
        const int r = range_of_local(sR, nrng, li);
        sElem[li] = sRng[2 * r] + (li - sR[r]);
      }
      int off = s_warp[warp] + incl - local;  // exclusive prefix of this thread's run
      for (int j = j0; j < j1; ++j) {
        sCol[j] = off;
        const int d = nb_dofs[B.dof_off + j];
        for (int k = dof_inc_off[d]; k < dof_inc_off[d + 1]; ++k) {
          const int s = dof_inc[k] / 3, a = dof_inc[k] % 3;
          const int r = find_range(sRng, nrng, s);
          sMap[off++] = r < 0 ? kNotNear : (unsigned short)(3 * (sR[r] + (s - sRng[2 * r])) + a);
        }
      }
      if (threadIdx.x == 0) sCol[ndof] = total;
    }
    __syncthreads();
    for (int tl = 0; tl < B.ntgt; ++tl) {
      const int t = nb_targets[B.tgt_off + tl];
      for (int li = threadIdx.x; li < nel; li += blockDim.x) {
        int s;
        if (use_map) {
          s = sElem[li];
        } else {
          const int r = range_of_local(sR, nrng, li);
          s = sRng[2 * r] + (li - sR[r]);
        }
        double g[3], gn[3];
        elem_weights3(s, t, Xs, e_vtx, e_near, near_region, g, gn);
#pragma unroll
        for (int a = 0; a < 3; ++a) E[3 * li + a] = make_double2(g[a], gn[a]);
      }
      __syncthreads();
      for (int j = threadIdx.x; j < ndof; j += blockDim.x) {
        double G = 0.0, Gn = 0.0;
        if (use_map) {
          for (int q = sCol[j]; q < sCol[j + 1]; ++q) {
            const unsigned short m = sMap[q];
            if (m != kNotNear) {
              const double2 w = E[m];
              G += w.x;
              Gn += w.y;
            }
          }
        } else {
          const int d = nb_dofs[B.dof_off + j];
          for (int k = dof_inc_off[d]; k < dof_inc_off[d + 1]; ++k) {
            const int s = dof_inc[k] / 3, a = dof_inc[k] % 3;
            const int r = find_range(sRng, nrng, s);
            if (r >= 0) {
              const double2 w = E[3 * (sR[r] + (s - sRng[2 * r])) + a];
              G += w.x;
              Gn += w.y;
            }
          }
        }
        WG[B.w_off + (int64_t)tl * ndof + j] = G;
        WGn[B.w_off + (int64_t)tl * ndof + j] = Gn;
      }
      __syncthreads();  // E is rewritten by the next target
    }
  }
}

// rigid-mode diagonal: diag_i = -GnPhi(point of i), 1 if |.| < 1e-15
__global__ void k_diag(int n, const int* __restrict__ dof_point, const double* __restrict__ GnPhi, double* __restrict__ diag) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d = -GnPhi[dof_point[i]];
    if (fabs(d) < 1e-15) d = 1.0;
    diag[i] = d;
  }
}

// ---------------------------------------------------------------------------
// Krylov helpers (FP64).  Dot products of w with columns V[0..k) in two deterministic
// stages: per-block partials, then one block per column.
__global__ void k_mdot_partial(const double* __restrict__ V, int ldv, int k, const double* __restrict__ w, int n,
                               double* __restrict__ partial /*[gridDim.x][k]*/) {
  extern __shared__ double red[];
  const int nw = blockDim.x >> 5, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int c = 0; c < k; ++c) {
    const double* v = V + (size_t)c * ldv;
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s = fma(v[i], w[i], s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int i = 0; i < nw; ++i) t += red[i];
      partial[(size_t)blockIdx.x * k + c] = t;
    }
    __syncthreads();
  }
}

__global__ void k_mdot_final(const double* __restrict__ partial, int nblk, int k, double* __restrict__ out) {
  const int c = blockIdx.x;
  __shared__ double red[32];
  double s = 0.0;
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += partial[(size_t)b * k + c];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    out[c] = t;
  }
}

// w -= V[:, 0:k] h   (h on device)
__global__ void k_maxpy(const double* __restrict__ V, int ldv, int k, const double* __restrict__ h, double* __restrict__ w, int n) {
  extern __shared__ double sh[];
  for (int c = threadIdx.x; c < k; c += blockDim.x) sh[c] = h[c];
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = w[i];
    for (int c = 0; c < k; ++c) s = fma(-sh[c], V[(size_t)c * ldv + i], s);
    w[i] = s;
  }
}

// y = a*x (+ y if accumulate)
__global__ void k_axpby(int n, double a, const double* __restrict__ x, double b, double* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = a * x[i] + (b == 0.0 ? 0.0 : b * y[i]);
}

// y = x * (1/s), s read from device memory
__global__ void k_scale_inv(int n, const double* __restrict__ x, const double* __restrict__ s, double* __restrict__ y) {
  const double inv = 1.0 / s[0];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = x[i] * inv;
}

// y = a .* x
__global__ void k_mul(int n, const double* __restrict__ a, const double* __restrict__ x, double* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = a[i] * x[i];
}

// y = xb + a .* u
__global__ void k_add_mul(int n, const double* __restrict__ xb, const double* __restrict__ a, const double* __restrict__ u,
                          double* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = xb[i] + a[i] * u[i];
}

// Inverse of the operator's diagonal entries A_ii, read from the cached near-field row of
// the DOF's own point: Dirichlet rows (unknown phin) w_G(i,i); Neumann rows (unknown phi)
// -(w_Gn(i,i) + diag_i); constraint rows 1.
__global__ void k_jacobi(int n, const int* __restrict__ dof_point, const int* __restrict__ dof_kind, const double* __restrict__ diag,
                         const int* __restrict__ block_of_point, const int* __restrict__ row_of_point, const NearBlockDev* __restrict__ blocks,
                         const int* __restrict__ self_col, const double* __restrict__ WG, const double* __restrict__ WGn,
                         double* __restrict__ dinv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int k = dof_kind[i];
    double a = 1.0;
    if (k != 2) {
      const int t = dof_point[i];
      const NearBlockDev B = blocks[block_of_point[t]];
      const int j = self_col[i];
      const int64_t w = B.w_off + (int64_t)row_of_point[t] * B.ndof + j;
      if (j >= 0) a = (k == 0) ? WG[w] : -(WGn[w] + diag[i]);
    }
    dinv[i] = (fabs(a) > 1e-300) ? 1.0 / a : 1.0;
  }
}

// Near-block preconditioner: block Jacobi (non-overlapping additive Schwarz) whose cores are
// the DOFs of each near block's targets (the points of one deepest bucket), the counterpart of
// the reference's additive Schwarz on the near-field matrix (SchwarzAdditive_CRS built at
// bem/BEM_solveBVP_GMRES_FMM.hpp:899-1013, cores grown by BFS over the near-field graph; here
// the cores are the buckets and there is no overlap).  The core matrix holds the operator's
// near-field entries among the core's DOFs: combined weight Wc of the row's point and the
// column DOF, minus diag_i on the diagonal of a Neumann row, unit rows for constraint rows.
// One CTA per block inverts it by Gauss-Jordan elimination with partial pivoting in shared
// memory and stores the inverse column-major; a core whose elimination meets a zero pivot
// keeps the point-Jacobi scaling on the diagonal of its m x m slot, and a core larger than
// kBjMax keeps it as m diagonal entries only (its slot holds m values, not m^2).
constexpr int kBjMax = kBjMaxCore;
constexpr int kBjThreads = 256;

size_t bj_setup_smem() { return sizeof(double) * (2 * (size_t)kBjMax * kBjMax + kBjMax); }

__global__ void __launch_bounds__(kBjThreads) k_bj_setup(const NearBlockDev* __restrict__ blocks, const int* __restrict__ bj_doff,
                                                        const int* __restrict__ bj_dofs, const int64_t* __restrict__ bj_ioff,
                                                        const int* __restrict__ nb_dofs, const int* __restrict__ dof_point,
                                                        const int* __restrict__ row_of_point, const int* __restrict__ dof_kind,
                                                        const double* __restrict__ diag, const double* __restrict__ Wc,
                                                        const double* __restrict__ dinv, double* __restrict__ inv) {
  extern __shared__ double bj_sm[];
  __shared__ int s_piv, s_ok;
  __shared__ int s_col[kBjMax];  // column of each core DOF in the block's DOF set
  const int b = blockIdx.x;
  const NearBlockDev B = blocks[b];
  const int d0 = bj_doff[b], m = bj_doff[b + 1] - d0;
  const int* core = bj_dofs + d0;
  double* out = inv + bj_ioff[b];  // column-major m x m
  if (m > kBjMax) {  // diagonal slot
    for (int a = threadIdx.x; a < m; a += blockDim.x) out[a] = dinv[core[a]];
    return;
  }
  bool ok = true;
  {
    double* A = bj_sm;                         // [m][m] row-major
    double* X = bj_sm + kBjMax * kBjMax;        // [m][m] inverse being formed
    double* f = bj_sm + 2 * kBjMax * kBjMax;    // [m] elimination factors
    const int stride = (B.ndof + 3) & ~3;
    for (int c = threadIdx.x; c < m; c += blockDim.x) s_col[c] = -1;
    __syncthreads();
    {  // the block's DOF set is in first-appearance order: scan it once for the core's DOFs
      const int* cols = nb_dofs + B.dof_off;
      for (int k = threadIdx.x; k < B.ndof; k += blockDim.x) {
        const int d = cols[k];
        for (int c = 0; c < m; ++c)
          if (core[c] == d) s_col[c] = k;
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
      const int a = e / m, c = e - a * m;
      const int i = core[a];
      const int k = dof_kind[i];
      double v;
      if (k == 2) {
        v = (a == c) ? 1.0 : 0.0;
      } else {
        const int col = s_col[c];
        v = col < 0 ? 0.0 : Wc[B.w4_off + (int64_t)row_of_point[dof_point[i]] * stride + col];
        if (k == 1 && a == c) v -= diag[i];
      }
      A[e] = v;
      X[e] = (a == c) ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int kk = 0; kk < m; ++kk) {
      if (threadIdx.x == 0) {
        int p = kk;
        double best = fabs(A[kk * m + kk]);
        for (int r = kk + 1; r < m; ++r)
          if (fabs(A[r * m + kk]) > best) {
            best = fabs(A[r * m + kk]);
            p = r;
          }
        s_piv = p;
        s_ok = best > 1e-300;
      }
      __syncthreads();
      if (!s_ok) {
        ok = false;
        break;
      }
      const int p = s_piv;
      if (p != kk)
        for (int c = threadIdx.x; c < m; c += blockDim.x) {
          double t = A[kk * m + c];
          A[kk * m + c] = A[p * m + c];
          A[p * m + c] = t;
          t = X[kk * m + c];
          X[kk * m + c] = X[p * m + c];
          X[p * m + c] = t;
        }
      __syncthreads();
      const double ip = 1.0 / A[kk * m + kk];
      __syncthreads();
      for (int c = threadIdx.x; c < m; c += blockDim.x) {
        A[kk * m + c] *= ip;
        X[kk * m + c] *= ip;
      }
      for (int r = threadIdx.x; r < m; r += blockDim.x) f[r] = (r == kk) ? 0.0 : A[r * m + kk];
      __syncthreads();
      for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
        const int r = e / m, c = e - r * m;
        if (r != kk) {
          A[e] = fma(-f[r], A[kk * m + c], A[e]);
          X[e] = fma(-f[r], X[kk * m + c], X[e]);
        }
      }
      __syncthreads();
    }
    if (ok)
      for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
        const int a = e / m, c = e - a * m;
        out[(int64_t)c * m + a] = X[e];
      }
  }
  if (!ok)  // point-Jacobi scaling on the diagonal
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
      const int a = e / m, c = e - a * m;
      out[(int64_t)c * m + a] = (a == c) ? dinv[core[a]] : 0.0;
    }
}

// z = M^{-1} y: a warp per block, lane per core row (the inverse column-major: the lanes read
// consecutive entries); the core's y values are gathered 32 at a time, one per lane, and
// broadcast by shuffles, so the gathers are not chained through the sum.  With st, y is the
// basis column V[:, st->n].
__global__ void k_bj_apply(int nblocks, const int* __restrict__ bj_doff, const int* __restrict__ bj_dofs, const int64_t* __restrict__ bj_ioff,
                           const double* __restrict__ inv, const double* __restrict__ y, int ldy, const ArnoldiState* __restrict__ st,
                           double* __restrict__ z) {
  pdl_enter();
  const int b = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (b >= nblocks) return;
  const double* yc = st ? y + (size_t)st->n * ldy : y;
  const int d0 = bj_doff[b], m = bj_doff[b + 1] - d0;
  const int* core = bj_dofs + d0;
  const double* M = inv + bj_ioff[b];
  if (m > kBjMax) {  // a core kept diagonal: m entries
    for (int a = lane; a < m; a += 32) z[core[a]] = M[a] * yc[core[a]];
    return;
  }
  for (int a0 = 0; a0 < m; a0 += 32) {  // rows a0 .. a0 + 31
    const int a = a0 + lane;
    double s = 0.0;
    for (int c0 = 0; c0 < m; c0 += 32) {  // columns c0 .. c0 + 31, in order
      const double yv = (c0 + lane < m) ? yc[core[c0 + lane]] : 0.0;
      const int cn = min(32, m - c0);
      for (int k = 0; k < cn; ++k) {
        const double yk = __shfl_sync(0xffffffffu, yv, k);
        if (a < m) s = fma(M[(int64_t)(c0 + k) * m + a], yk, s);
      }
    }
    if (a < m) z[core[a]] = s;
  }
}

// FP64 FMA throughput probe: 8 independent FMA chains per thread.
__global__ void k_fp64_probe(int iters, double seed, double* __restrict__ sink) {
  double a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
  const double m = 0.999999, c = 1e-7;
  for (int i = 0; i < iters; ++i) {
    a0 = fma(a0, m, c);
    a1 = fma(a1, m, c);
    a2 = fma(a2, m, c);
    a3 = fma(a3, m, c);
    a4 = fma(a4, m, c);
    a5 = fma(a5, m, c);
    a6 = fma(a6, m, c);
    a7 = fma(a7, m, c);
  }
  const double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
  if (s == 12345.678) sink[0] = s;
}

// ---------------------------------------------------------------------------
// launchers
// the near-field SpMV of A.x: per-target near sums (one CTA per near block)
int launch_near_sums(const MatvecArgs& a, cudaStream_t st) {
  const size_t shm = ns_smem_bytes(a.max_ntgt);
  if (a.Wc32)
    launch_pdl(k_near_sums<float>, a.n_blocks, kNsThreads, shm, st, a.blocks, a.nb_dofs, a.Wc32, a.ax, a.near_sum);
  else
    launch_pdl(k_near_sums<double>, a.n_blocks, kNsThreads, shm, st, a.blocks, a.nb_dofs, a.Wc, a.ax, a.near_sum);
  return 1;
}

// the rows of A.x from the near sums, with the far field of L (none when L is null)
template <int P>
int launch_target_rows(const MatvecArgs& a, cudaStream_t st, const double2* L) {
  launch_pdl(k_target_rows<P>, a.n_blocks, kRowsThreads, target_rows_smem_bytes(P, a.max_path, a.max_ntgt), st, a.blocks, a.nb_targets, a.Xs, a.node_X, a.blk_path ? L : nullptr, a.blk_path_off,
             a.blk_path, a.near_sum, a.ax, a.point_dof_off, a.point_dof, a.dof_kind, a.diag, a.rows);
  return 1;
}

template <int P>
int launch_targets_ax(const MatvecArgs& a, cudaStream_t st, const double2* L) {
  return launch_near_sums(a, st) + launch_target_rows<P>(a, st, L);
}

template <int P, int ND>
int launch_matvec_fmm(const MatvecArgs& a, cudaStream_t st, int stages) {
  constexpr int NC = ncoef(P);
  int launches = 0;
  // overlap: the near-field part of the rows (HBM-bound) runs on the side stream while the FMM
  // passes run here; the far-field part is added once both are done
  const bool overlap = stages == STAGE_ALL && ND == 1 && a.side && a.ev_fork && a.ev_join && (a.Wc32 || a.Wc) && a.ax && a.n_blocks > 0;
  if (overlap) {
    cudaEventRecord(a.ev_fork, st);
    cudaStreamWaitEvent(a.side, a.ev_fork, 0);
    launches += launch_near_sums(a, a.side);
    cudaEventRecord(a.ev_join, a.side);
    stages &= ~STAGE_TARGETS;
  }
  // A.x: the P2M operator, each leaf's multipole shifted to its parent in the same kernel, and
  // an upward pass over the non-leaf nodes only
  const bool ax_p2m = ND == 1 && a.ax && a.p2m_C && a.leaf_level && a.m2m_level_off_nl;
  if ((stages & STAGE_P2M) && a.n_leaves > 0 && ax_p2m) {
    if (a.p2m_C32)  // low-precision operator: the FP32 copy (half the bytes of the kernel's dominant read)
      launch_pdl(k_p2m_leaf<P, float2>, a.n_leaves, tree_threads<P>(), 0, st, a.leaves, a.leaf_dof_off, a.leaf_dof, a.p2m_C32, a.ax,
                 a.node_up, a.leaf_level, a.node_X, a.Ftab, a.M, a.Yup);
    else
      launch_pdl(k_p2m_leaf<P, double2>, a.n_leaves, tree_threads<P>(), 0, st, a.leaves, a.leaf_dof_off, a.leaf_dof,
                 (const double2*)a.p2m_C, a.ax, a.node_up, a.leaf_level, a.node_X, a.Ftab, a.M, a.Yup);
    ++launches;

  } else if ((stages & STAGE_P2M) && a.n_leaves > 0) {
    k_p2m<P, ND><<<a.n_leaves, 128, 0, st>>>(a.leaves, a.node_fb, a.node_fe, a.node_X, a.e_q, a.e_W, a.e_n, a.e_dof, a.phi, a.phin, a.M);
    ++launches;
  }
  constexpr int NF = (P + 1) * (P + 1);
  if ((stages & STAGE_M2M) && a.m2m_level_off) {
    const int* off = ax_p2m ? a.m2m_level_off_nl : a.m2m_level_off;  // without the leaves when k_p2m_leaf shifted them
    const int* nodes = ax_p2m ? a.m2m_nodes_nl : a.m2m_nodes;
    for (int l = a.n_levels - 1; l >= 0; --l) {
      const int cnt = off[l + 1] - off[l];
      if (cnt <= 0) continue;
      const double2* Fup = a.Ftab + (size_t)std::max(l - 1, 0) * 8 * NF;  // tables of the parent level
      launch_pdl(k_m2m_level<P, ND>, cnt, tree_threads<P>(), 0, st, nodes + off[l], a.node_up, a.child_begin, a.child_end, a.node_children,
                 a.node_X, Fup, a.M, a.Yup);
      ++launches;
    }
  }
  if (stages & STAGE_M2L) {
    cudaMemsetAsync(a.L, 0, sizeof(double2) * 2 * NC * (size_t)a.n_nodes, st);
    if (a.use_tc) {
      launches += launch_m2l_tc(P, a, st, TC_ALL, ND);
    } else if (a.n_chunks > 0) {
      const int tpb2 = ((ND * NC + 31) / 32) * 32;
      k_m2l_grp<P, ND><<<a.n_chunks, tpb2, m2l_grp_smem_bytes<P>(), st>>>(a.chunk_grp, a.chunk_begin, a.chunk_cnt, a.grp_pair, a.m2l_src,
                                                                        a.Sg, a.M, a.Y);
      const int64_t tr = (int64_t)a.n_m2l_targets * ND * NC;
      int gr = (int)std::min<int64_t>((tr + 255) / 256, 148 * 16);
      k_m2l_reduce<P, ND><<<gr, 256, 0, st>>>(a.n_m2l_targets, a.m2l_targets, a.m2l_off, a.Y, a.L);
      launches += 2;
    }
  }
  // the A.x rows sum the L2Ps along each target bucket's path instead (k_target_rows)
  const bool ax_rows = ND == 1 && a.ax && (a.Wc || a.Wc32) && a.blk_path;
  if ((stages & STAGE_L2L) && a.l2l_level_off && !ax_rows)
    for (int l = 0; l < a.n_levels; ++l) {
      const int cnt = a.l2l_level_off[l + 1] - a.l2l_level_off[l];
      if (cnt <= 0) continue;
      launch_pdl(k_l2l_pairs<P, ND>, cnt, tree_threads<P>(), 0, st, a.l2l_pairs + a.l2l_level_off[l], a.node_X, a.Ftab + (size_t)l * 8 * NF,
                 a.L);
      ++launches;
    }
  if ((stages & STAGE_TARGETS) && a.n_blocks > 0 && ND == 1 && a.ax && (a.Wc || a.Wc32)) {
    launches += launch_targets_ax<P>(a, st, a.L);
  } else if ((stages & STAGE_TARGETS) && a.n_blocks > 0) {
    const size_t shm = sizeof(double2) * (size_t)(a.chunk + a.max_ntgt);
    k_targets<P, ND><<<a.n_blocks, 128, shm, st>>>(a.blocks, a.nb_dofs, a.nb_targets, a.WG, a.WGn, a.Xs, a.node_X, a.L, a.phi, a.phin,
                                               a.point_dof_off, a.point_dof, a.dof_kind, a.diag, a.rows, a.GPhin, a.GnPhi, a.chunk);
    ++launches;
  }
  if (overlap) {
    cudaStreamWaitEvent(st, a.ev_join, 0);
    launches += launch_target_rows<P>(a, st, a.L);
  }
  return launches;
}

template <int P>
void set_target_smem(int bytes) {
  // the permission only grows: contexts of different problems (batch workers on other
  // threads) may launch these kernels with their own sizes at any time.  The attribute
  // belongs to the current device, so the bookkeeping is per device.
  static std::mutex mu;
  static int granted[kMaxDevices] = {};
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
  const bool tracked = dev >= 0 && dev < kMaxDevices;  // untracked devices: set every time
  std::lock_guard<std::mutex> lk(mu);
  if (tracked && bytes <= granted[dev]) return;
  if (tracked) granted[dev] = bytes;
  cudaFuncSetAttribute(k_targets<P, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  cudaFuncSetAttribute(k_targets<P, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

// k_near_sums's dynamic shared memory (an x chunk and a running sum per target): the permission
// only grows, per device, as for the other targets kernels
int configure_targets_ax_smem(int max_ntgt) {
  const size_t bytes = ns_smem_bytes(max_ntgt);
  if (bytes > 200 * 1024) return -1;
  static std::mutex mu;
  static int granted[kMaxDevices] = {};
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
  const bool tracked = dev >= 0 && dev < kMaxDevices;
  std::lock_guard<std::mutex> lk(mu);
  if (tracked && (int)bytes <= granted[dev]) return 0;
  if (tracked) granted[dev] = (int)bytes;
  cudaFuncSetAttribute(k_near_sums<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  cudaFuncSetAttribute(k_near_sums<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  return 0;
}

int launch_matvec(int p, const MatvecArgs& a, cudaStream_t st, int stages) {
  switch (p) {
#define BEMB200_CASE(PP) \
  case PP:               \
    return a.GPhin ? launch_matvec_fmm<PP, 2>(a, st, stages) : launch_matvec_fmm<PP, 1>(a, st, stages);
    BEMB200_CASE(1) BEMB200_CASE(2) BEMB200_CASE(3) BEMB200_CASE(4) BEMB200_CASE(5) BEMB200_CASE(6)
    BEMB200_CASE(7) BEMB200_CASE(8) BEMB200_CASE(9) BEMB200_CASE(10) BEMB200_CASE(11) BEMB200_CASE(12)
#undef BEMB200_CASE
    default: break;
  }
  return 0;
}

// y = A_near x: the near-field rows of the A.x operator (combined weights, diagonal and
// constraint rows as k_near_sums + k_target_rows, no far field); a.ax -> a.rows, FP32 weights when present
template <int P>
int launch_near_only_t(const MatvecArgs& a, cudaStream_t st) {
  if (a.n_blocks <= 0 || !a.ax || !(a.Wc || a.Wc32)) return 0;
  return launch_targets_ax<P>(a, st, nullptr);
}

int launch_near_only(int p, const MatvecArgs& a, cudaStream_t st) {
  switch (p) {
#define BEMB200_CASE(PP) \
  case PP:               \
    return launch_near_only_t<PP>(a, st);
    BEMB200_CASE(1) BEMB200_CASE(2) BEMB200_CASE(3) BEMB200_CASE(4) BEMB200_CASE(5) BEMB200_CASE(6)
    BEMB200_CASE(7) BEMB200_CASE(8) BEMB200_CASE(9) BEMB200_CASE(10) BEMB200_CASE(11) BEMB200_CASE(12)
#undef BEMB200_CASE
    default: break;
  }
  return 0;
}

template <int P>
void set_m2l_smem() {
  cudaFuncSetAttribute(k_m2l_grp<P, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, m2l_grp_smem_bytes<P>());
  cudaFuncSetAttribute(k_m2l_grp<P, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, m2l_grp_smem_bytes<P>());
}

template <int P>
void f_tables(int ntab, const double* vec, double2* Ftab, cudaStream_t st) {
  if (ntab > 0) k_ftab<P><<<ntab, 32, 0, st>>>(ntab, vec, Ftab);
}

void launch_f_tables(int p, int ntab, const double* vec, double2* Ftab, cudaStream_t st) {
  switch (p) {
#define BEMB200_CASE(PP) \
  case PP:               \
    f_tables<PP>(ntab, vec, Ftab, st); break;
    BEMB200_CASE(1) BEMB200_CASE(2) BEMB200_CASE(3) BEMB200_CASE(4) BEMB200_CASE(5) BEMB200_CASE(6)
    BEMB200_CASE(7) BEMB200_CASE(8) BEMB200_CASE(9) BEMB200_CASE(10) BEMB200_CASE(11) BEMB200_CASE(12)
#undef BEMB200_CASE
    default: break;
  }
}

template <int P>
void s_tables(int ngroups, const double* gvec, double2* Sg, cudaStream_t st) {
  if (ngroups > 0) k_s_tables<P><<<ngroups, 32, 0, st>>>(ngroups, gvec, Sg);
}

void launch_s_tables(int p, int ngroups, const double* gvec, double2* Sg, cudaStream_t st) {
  switch (p) {
#define BEMB200_CASE(PP) \
  case PP:               \
    s_tables<PP>(ngroups, gvec, Sg, st); break;
    BEMB200_CASE(1) BEMB200_CASE(2) BEMB200_CASE(3) BEMB200_CASE(4) BEMB200_CASE(5) BEMB200_CASE(6)
    BEMB200_CASE(7) BEMB200_CASE(8) BEMB200_CASE(9) BEMB200_CASE(10) BEMB200_CASE(11) BEMB200_CASE(12)
#undef BEMB200_CASE
    default: break;
  }
}

void configure_m2l_smem(int p) {
  switch (p) {
#define BEMB200_CASE(PP) \
  case PP:               \
    set_m2l_smem<PP>(); break;
    BEMB200_CASE(1) BEMB200_CASE(2) BEMB200_CASE(3) BEMB200_CASE(4) BEMB200_CASE(5) BEMB200_CASE(6)
    BEMB200_CASE(7) BEMB200_CASE(8) BEMB200_CASE(9) BEMB200_CASE(10) BEMB200_CASE(11) BEMB200_CASE(12)
#undef BEMB200_CASE
    default: break;
  }
}

void configure_targets_smem(int p, int bytes) {
  switch (p) {
#define BEMB200_CASE(PP) \
  case PP:               \
    set_target_smem<PP>(bytes); break;
    BEMB200_CASE(1) BEMB200_CASE(2) BEMB200_CASE(3) BEMB200_CASE(4) BEMB200_CASE(5) BEMB200_CASE(6)
    BEMB200_CASE(7) BEMB200_CASE(8) BEMB200_CASE(9) BEMB200_CASE(10) BEMB200_CASE(11) BEMB200_CASE(12)
#undef BEMB200_CASE
    default: break;
  }
}

template <int P>
void set_rows_smem(int bytes) {
  static std::mutex mu;
  static int granted[kMaxDevices] = {};
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
  const bool tracked = dev >= 0 && dev < kMaxDevices;
  std::lock_guard<std::mutex> lk(mu);
  if (tracked && bytes <= granted[dev]) return;
  if (tracked) granted[dev] = bytes;
  cudaFuncSetAttribute(k_target_rows<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

// k_target_rows's dynamic shared memory (the path's locals and the per-(target, node) L2Ps);
// -1 when it does not fit an SM
int configure_target_rows_smem(int p, int max_path, int max_ntgt) {
  const size_t bytes = target_rows_smem_bytes(p, max_path, max_ntgt);
  if (bytes > 200 * 1024) return -1;
  switch (p) {
#define BEMB200_CASE(PP) \
  case PP:               \
    set_rows_smem<PP>((int)bytes); break;
    BEMB200_CASE(1) BEMB200_CASE(2) BEMB200_CASE(3) BEMB200_CASE(4) BEMB200_CASE(5) BEMB200_CASE(6)
    BEMB200_CASE(7) BEMB200_CASE(8) BEMB200_CASE(9) BEMB200_CASE(10) BEMB200_CASE(11) BEMB200_CASE(12)
#undef BEMB200_CASE
    default: break;
  }
  return 0;
}

template <int P>
void p2m_op(const MatvecArgs& a, const int* e_slot, cudaStream_t st) {
  if (a.n_leaves > 0)
    k_p2m_op<P><<<a.n_leaves, 128, 0, st>>>(a.leaves, a.node_fb, a.node_fe, a.node_X, a.e_q, a.e_W, a.e_n, a.e_dof, e_slot, a.dof_kind,
                                            a.leaf_dof_off, a.p2m_C);
}

void launch_p2m_op(int p, const MatvecArgs& a, const int* e_slot, cudaStream_t st) {
  switch (p) {
#define BEMB200_CASE(PP) \
  case PP:               \
    p2m_op<PP>(a, e_slot, st); break;
    BEMB200_CASE(1) BEMB200_CASE(2) BEMB200_CASE(3) BEMB200_CASE(4) BEMB200_CASE(5) BEMB200_CASE(6)
    BEMB200_CASE(7) BEMB200_CASE(8) BEMB200_CASE(9) BEMB200_CASE(10) BEMB200_CASE(11) BEMB200_CASE(12)
#undef BEMB200_CASE
    default: break;
  }
}

__global__ void k_to_float2(size_t n, const double2* __restrict__ src, float2* __restrict__ dst) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = make_float2((float)src[i].x, (float)src[i].y);
}

void launch_to_float2(size_t n, const double2* src, float2* dst, cudaStream_t st) {
  if (n == 0) return;
  const size_t g = std::min<size_t>((n + 255) / 256, 148 * 16);
  k_to_float2<<<(int)g, 256, 0, st>>>(n, src, dst);
}

void launch_combine_weights(int nblocks, const NearBlockDev* blocks, const int* nb_dofs, const int* dof_kind, const double* WG,
                            const double* WGn, double* Wc, float* Wc32, cudaStream_t st) {
  if (nblocks <= 0) return;
  if (Wc) k_combine_weights<double><<<nblocks, 256, 0, st>>>(blocks, nb_dofs, dof_kind, WG, WGn, Wc);
  if (Wc32) k_combine_weights<float><<<nblocks, 256, 0, st>>>(blocks, nb_dofs, dof_kind, WG, WGn, Wc32);
}

void launch_densities(int n, int mode, const double* x, const double* known, const int* kind, double* phi, double* phin, cudaStream_t st) {
  const int g = (n + 255) / 256;
  k_densities<<<g > 0 ? g : 1, 256, 0, st>>>(n, mode, x, known, kind, phi, phin);
}

int near_weights_grid() { return 148 * 3; }  // three 256-thread CTAs per SM (80 registers a thread)

int launch_near_weights(const NearArgs& a, cudaStream_t st) {
  if (a.n_blocks <= 0 || a.n_slots <= 0) return 0;
  const size_t shm = sizeof(int) * (size_t)(3 * a.max_nrng + 1) + kNearMapBytes;
  if (shm > 200 * 1024) return -1;
  {  // the permission only grows, per device (contexts of other threads launch it too)
    static std::mutex mu;
    static size_t granted[kMaxDevices] = {};
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
    const bool tracked = dev >= 0 && dev < kMaxDevices;
    std::lock_guard<std::mutex> lk(mu);
    if (!tracked || shm > granted[dev]) {
      if (cudaFuncSetAttribute(k_near_weights, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm) != cudaSuccess) return -1;
      if (tracked) granted[dev] = shm;
    }
  }
  if (cudaMemsetAsync(a.next_block, 0, sizeof(int), st) != cudaSuccess) return -1;
  k_near_weights<<<std::min(a.n_blocks, near_weights_grid()), kNearThreads, shm, st>>>(
      a.n_blocks, a.next_block, a.max_nrng, a.blocks, a.nb_dofs, a.nb_targets, a.nb_ranges, a.dof_inc_off, a.dof_inc, a.Xs, a.e_vtx,
      a.e_near, a.near_region, a.scratch, a.scratch_stride, a.WG, a.WGn);
  return 0;
}

void launch_diag(int n, const int* dof_point, const double* GnPhi, double* diag, cudaStream_t st) {
  const int g = (n + 255) / 256;
  k_diag<<<g > 0 ? g : 1, 256, 0, st>>>(n, dof_point, GnPhi, diag);
}

int mdot_blocks(int n) {
  int b = (n + 1023) / 1024;
  return b < 1 ? 1 : (b > 296 ? 296 : b);
}

void launch_mdot(const double* V, int ldv, int k, const double* w, int n, double* partial, double* out, cudaStream_t st) {
  const int nb = mdot_blocks(n);
  k_mdot_partial<<<nb, 256, 8 * sizeof(double), st>>>(V, ldv, k, w, n, partial);
  k_mdot_final<<<k, 256, 0, st>>>(partial, nb, k, out);
}

void launch_maxpy(const double* V, int ldv, int k, const double* h, double* w, int n, cudaStream_t st) {
  int g = (n + 255) / 256;
  if (g > 1184) g = 1184;
  k_maxpy<<<g > 0 ? g : 1, 256, sizeof(double) * (k > 0 ? k : 1), st>>>(V, ldv, k, h, w, n);
}

void launch_axpby(int n, double a, const double* x, double b, double* y, cudaStream_t st) {
  int g = (n + 255) / 256;
  if (g > 1184) g = 1184;
  k_axpby<<<g > 0 ? g : 1, 256, 0, st>>>(n, a, x, b, y);
}

bool pdl_enabled() {
  static const bool on = [] {
    const char* v = std::getenv("BEMB200_NO_PDL");
    return !(v && v[0] && v[0] != '0');
  }();
  return on;
}

// y[i] in [-0.5, 0.5): a fixed pseudo-random vector (splitmix64 of seed + i)
__global__ void k_hash_fill(int n, unsigned long long seed, double* __restrict__ y) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    unsigned long long z = seed + 0x9e3779b97f4a7c15ull * (unsigned long long)(i + 1);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    z ^= z >> 31;
    y[i] = (double)(z >> 11) * 0x1.0p-53 - 0.5;
  }
}

void launch_hash_fill(int n, unsigned long long seed, double* y, cudaStream_t st) {
  int g = (n + 255) / 256;
  if (g > 1184) g = 1184;
  k_hash_fill<<<g > 0 ? g : 1, 256, 0, st>>>(n, seed, y);
}

void launch_mul(int n, const double* a, const double* x, double* y, cudaStream_t st) {
  int g = (n + 255) / 256;
  if (g > 1184) g = 1184;
  k_mul<<<g > 0 ? g : 1, 256, 0, st>>>(n, a, x, y);
}

void launch_add_mul(int n, const double* xb, const double* a, const double* u, double* y, cudaStream_t st) {
  int g = (n + 255) / 256;
  if (g > 1184) g = 1184;
  k_add_mul<<<g > 0 ? g : 1, 256, 0, st>>>(n, xb, a, u, y);
}

void launch_bj_setup(const NearBjArgs& a, const int* nb_dofs, const int* dof_point, const int* row_of_point, const int* dof_kind,
                     const double* diag, const double* Wc, const double* dinv, cudaStream_t st) {
  if (a.nblocks <= 0) return;
  static std::mutex mu;
  static bool granted[kMaxDevices] = {};
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (dev < 0 || dev >= kMaxDevices || !granted[dev]) {
      cudaFuncSetAttribute(k_bj_setup, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bj_setup_smem());
      if (dev >= 0 && dev < kMaxDevices) granted[dev] = true;
    }
  }
  k_bj_setup<<<a.nblocks, kBjThreads, bj_setup_smem(), st>>>(a.blocks, a.doff, a.dofs, a.ioff, nb_dofs, dof_point, row_of_point, dof_kind,
                                                               diag, Wc, dinv, a.inv);
}

void launch_bj_apply(const NearBjArgs& a, const double* y, int ldy, const ArnoldiState* st, double* z, cudaStream_t s) {
  if (a.nblocks <= 0) return;
  const int warps_per_cta = 8;
  launch_pdl(k_bj_apply, (a.nblocks + warps_per_cta - 1) / warps_per_cta, 32 * warps_per_cta, 0, s, a.nblocks, (const int*)a.doff,
             (const int*)a.dofs, (const int64_t*)a.ioff, (const double*)a.inv, y, ldy, st, z);
}

void launch_jacobi(int n, const int* dof_point, const int* dof_kind, const double* diag, const int* block_of_point, const int* row_of_point,
                   const NearBlockDev* blocks, const int* self_col, const double* WG, const double* WGn, double* dinv, cudaStream_t st) {
  int g = (n + 255) / 256;
  k_jacobi<<<g > 0 ? g : 1, 256, 0, st>>>(n, dof_point, dof_kind, diag, block_of_point, row_of_point, blocks, self_col, WG, WGn, dinv);
}

double fp64_probe_tflops(cudaStream_t st, double* sink) {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int iters = 1 << 14, blocks = sms * 8, threads = 256;
  k_fp64_probe<<<blocks, threads, 0, st>>>(iters, 1.0, sink);  // warm-up
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  k_fp64_probe<<<blocks, threads, 0, st>>>(iters, 2.0, sink);
  cudaEventRecord(e1, st);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const double flops = 2.0 * 8.0 * (double)iters * blocks * threads;
  return flops / (ms * 1e-3) / 1e12;
}

void launch_scale_inv(int n, const double* x, const double* s, double* y, cudaStream_t st) {
  int g = (n + 255) / 256;
  if (g > 1184) g = 1184;
  k_scale_inv<<<g > 0 ? g : 1, 256, 0, st>>>(n, x, s, y);
}

}  // namespace bemb200
