// Device-resident Arnoldi step of the GMRES driver (solveSystemGMRES,
// bem/BEM_solveBVP_GMRES_FMM.hpp:2007-2649; ArnoldiProcess::AddBasisVector and the Givens
// update of gmres, lib/include/basic_linear_systems.hpp:3242-3260, 3369-3433).
//
// One step = prepare the operator input from basis column n, apply the operator (the mat-vec
// kernels are captured into the same graph), orthogonalise against columns 0..n by classical
// Gram-Schmidt applied twice, normalise into column n+1, and update the QR factor of the
// Hessenberg matrix by Givens rotations.  The step count n, the rotations, the rotated
// right-hand side g and the triangular factor R live in device memory, so consecutive steps
// are graph launches with no host round trip; the host reads the residual estimate |g[n]|
// a few steps behind.  The arithmetic of the rotations is the reference's, term by term.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>

#include "kernels.cuh"

namespace bemb200 {
namespace {

// Orthogonalisation kernels.  Each CTA owns a contiguous slice of rows (the same slices in
// every kernel of a step); a dot product over the basis is a per-slice partial written
// column-major (partial[c * nslice + b]) and summed over the slices by a CTA per column in a
// fixed order, so the sums are deterministic.  A step is: the operator, k_arn_dots, k_arn_sum,
// k_arn_orth_dots (first correction fused with the second pass's dots), k_arn_sum,
// k_arn_orth_norm (second correction fused with |w|^2), k_arn_givens, k_arn_next.
constexpr int kArnThreads = 256;
constexpr int kArnRowsMax = 2048;  // rows per slice at most (shared-memory copy of the slice)

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// partial[c * nb + b] = V[rows of b, c] . ws for c < ncol: warp per column, lanes along the rows
__device__ __forceinline__ void slice_dots(const double* __restrict__ V, int ldv, int ncol, int row0, int nr, const double* ws,
                                           double* __restrict__ partial, int nb) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int c = warp; c < ncol; c += nw) {
    const double* v = V + (size_t)c * ldv + row0;
    double s = 0.0;
    for (int i = lane; i < nr; i += 32) s = fma(v[i], ws[i], s);
    s = warp_sum(s);
    if (lane == 0) partial[(size_t)c * nb + blockIdx.x] = s;
  }
}

// partial dots of the first pass: V[:, 0..n]^T w per slice
__global__ void __launch_bounds__(kArnThreads) k_arn_dots(const double* __restrict__ V, int ldv, const ArnoldiState* __restrict__ st,
                                                          const double* __restrict__ w, int nrow, int rows, double* __restrict__ partial) {
  pdl_enter();
  extern __shared__ double arn_sm[];
  const int ncol = st->n + 1;
  const int row0 = blockIdx.x * rows, nr = min(rows, nrow - row0);
  double* ws = arn_sm;
  for (int i = threadIdx.x; i < nr; i += blockDim.x) ws[i] = w[row0 + i];
  __syncthreads();
  slice_dots(V, ldv, ncol, row0, nr, ws, partial, gridDim.x);
}

// out[c] = sum over the nb slices of partial[c * nb + b]: a CTA per column
__global__ void __launch_bounds__(kArnThreads) k_arn_sum(const double* __restrict__ partial, int nb, const ArnoldiState* __restrict__ st,
                                                         double* __restrict__ out) {
  pdl_enter();
  __shared__ double red[kArnThreads / 32];
  const int c = blockIdx.x;
  if (c > st->n) return;
  double s = 0.0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) s += partial[(size_t)c * nb + b];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[q];
    out[c] = t;
  }
}

// w -= V[:, 0..n] h1 on the slice, then the second pass's partial dots on the corrected slice
__global__ void __launch_bounds__(kArnThreads) k_arn_orth_dots(const double* __restrict__ V, int ldv, const ArnoldiState* __restrict__ st,
                                                               const double* __restrict__ h1, double* __restrict__ w, int nrow, int rows,
                                                               double* __restrict__ partial, int cols) {
  pdl_enter();
  extern __shared__ double arn_sm[];
  const int ncol = st->n + 1;
  const int row0 = blockIdx.x * rows, nr = min(rows, nrow - row0);
  double* sh = arn_sm;         // [cols]
  double* ws = arn_sm + cols;  // [rows]
  for (int c = threadIdx.x; c < ncol; c += blockDim.x) sh[c] = h1[c];
  __syncthreads();
  for (int i = threadIdx.x; i < nr; i += blockDim.x) {
    double s = w[row0 + i];
    for (int c = 0; c < ncol; ++c) s = fma(-sh[c], V[(size_t)c * ldv + row0 + i], s);
    w[row0 + i] = s;
    ws[i] = s;
  }
  __syncthreads();
  slice_dots(V, ldv, ncol, row0, nr, ws, partial, gridDim.x);
}

// w -= V[:, 0..n] h2 on the slice, and the slice's |w|^2 into partial[b]
__global__ void __launch_bounds__(kArnThreads) k_arn_orth_norm(const double* __restrict__ V, int ldv, const ArnoldiState* __restrict__ st,
                                                               const double* __restrict__ h2, double* __restrict__ w, int nrow, int rows,
                                                               double* __restrict__ partial) {
  pdl_enter();
  extern __shared__ double arn_sm[];  // h2 [n + 1]
  __shared__ double red[kArnThreads / 32];
  const int ncol = st->n + 1;
  const int row0 = blockIdx.x * rows, nr = min(rows, nrow - row0);
  double* sh = arn_sm;
  for (int c = threadIdx.x; c < ncol; c += blockDim.x) sh[c] = h2[c];
  __syncthreads();
  double ss = 0.0;
  for (int i = threadIdx.x; i < nr; i += blockDim.x) {
    double s = w[row0 + i];
    for (int c = 0; c < ncol; ++c) s = fma(-sh[c], V[(size_t)c * ldv + row0 + i], s);
    w[row0 + i] = s;
    ss = fma(s, s, ss);
  }
  ss = warp_sum(ss);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ss;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[q];
    partial[blockIdx.x] = t;
  }
}

// One warp: |w| from the slice partials, the Hessenberg column h1 + h2 with h_{n+1,n} = |w|,
// the previous rotations applied, the new rotation, g rotated, the R column stored, the
// residual estimate |g[n+1]|, and n advanced (the reference's Givens update,
// basic_linear_systems.hpp:3369-3433, term by term)
__global__ void k_arn_givens(ArnoldiState* __restrict__ st, const double* __restrict__ h1, const double* __restrict__ h2,
                             const double* __restrict__ partial, int nb, double* __restrict__ cs, double* __restrict__ sn,
                             double* __restrict__ g, double* __restrict__ R, int ldr) {
  pdl_enter();
  extern __shared__ double sg[];  // h [k+1], cs [k], sn [k]
  const int n = st->n, k = n + 1;
  const int lane = threadIdx.x;
  double hn = 0.0;
  for (int b = lane; b < nb; b += 32) hn += partial[b];
  hn = warp_sum(hn);
  double* h = sg;
  double* c_ = sg + k + 1;
  double* s_ = c_ + k;
  for (int i = lane; i < k; i += 32) {
    h[i] = h1[i] + h2[i];
    c_[i] = cs[i];
    s_[i] = sn[i];
  }
  __syncwarp();
  if (lane == 0) {
    h[k] = sqrt(hn);
    st->inv_h = h[k] > 0.0 ? 1.0 / h[k] : 0.0;
    if (!isfinite(h[k])) st->bad = 1;
    for (int i = 0; i < k - 1; ++i) {
      const double t = fma(c_[i], h[i], s_[i] * h[i + 1]);
      h[i + 1] = fma(c_[i], h[i + 1], -s_[i] * h[i]);
      h[i] = t;
    }
    const double a = h[k - 1], bb = h[k];
    const double rr = hypot(a, bb);
    double c = 1.0, sv = 0.0;
    if (rr != 0.0) {
      c = a / rr;
      sv = bb / rr;
    }
    cs[k - 1] = c;
    sn[k - 1] = sv;
    {
      const double t = fma(c, h[k - 1], sv * h[k]);
      h[k] = fma(c, h[k], -sv * h[k - 1]);
      h[k - 1] = t;
    }
    g[k] = 0.0;
    {
      const double t = fma(c, g[k - 1], sv * g[k]);
      g[k] = fma(c, g[k], -sv * g[k - 1]);
      g[k - 1] = t;
    }
    st->err = fabs(g[k]);
    st->n = k;
  }
  __syncwarp();
  double* Rc = R + (size_t)n * ldr;
  for (int i = lane; i <= k; i += 32) Rc[i] = h[i];
}

// V[:, n] = w / h_{n,n-1} (n already advanced) and the next step's operator input
// x = (dinv .*) V[:, n]
__global__ void k_arn_next(int nrow, const double* __restrict__ w, const ArnoldiState* __restrict__ st, double* __restrict__ V,
                           const double* __restrict__ dinv, double* __restrict__ x) {
  pdl_enter();
  double* v = V + (size_t)st->n * nrow;
  const double s = st->inv_h;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrow; i += gridDim.x * blockDim.x) {
    const double vi = w[i] * s;
    v[i] = vi;
    x[i] = dinv ? dinv[i] * vi : vi;
  }
}

// operator input: x = (dinv .*) V[:, n]
__global__ void k_arn_prep(int nrow, const double* __restrict__ V, const double* __restrict__ dinv, const ArnoldiState* __restrict__ st,
                           double* __restrict__ x) {
  pdl_enter();
  const double* v = V + (size_t)st->n * nrow;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrow; i += gridDim.x * blockDim.x) x[i] = dinv ? dinv[i] * v[i] : v[i];
}

// One factor of the polynomial preconditioner p(B) applied to u = V[:, n] (B = A_near D^{-1},
// 1 - B p(B) = prod over roots of (1 - B / theta)); r = B(prod) or B(w) from the launch before.
//   mode 0, real root:        y += prod / theta; prod -= r / theta             (c = 1 / theta)
//   mode 1, pair, first half: w = 2a prod - r; y += w / |theta|^2; next B input w  (c = 1 / |theta|^2)
//   mode 2, pair, second half: prod -= r / |theta|^2
// first: prod is V[:, n] and y starts at zero.  last: no further B; x = Z[:, n] = D^{-1} y.
// Otherwise x = D^{-1} (next B input).
__global__ void k_poly_factor(int nrow, int mode, int first, int last, double c, double two_a, const double* __restrict__ V,
                              const ArnoldiState* __restrict__ st, double* __restrict__ prod, const double* __restrict__ r,
                              double* __restrict__ y, const double* __restrict__ dinv, double* __restrict__ x, double* __restrict__ Z) {
  pdl_enter();
  const size_t col = (size_t)st->n * nrow;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrow; i += gridDim.x * blockDim.x) {
    const double p = first ? V[col + i] : prod[i];
    double yi = first ? 0.0 : y[i];
    double nxt = 0.0;
    if (mode == 0) {
      yi = fma(p, c, yi);
      if (!last) {
        nxt = fma(-r[i], c, p);
        prod[i] = nxt;
      }
    } else if (mode == 1) {
      const double w = fma(two_a, p, -r[i]);
      yi = fma(w, c, yi);
      nxt = w;
      if (first && !last) prod[i] = p;
    } else {
      nxt = fma(-r[i], c, p);
      prod[i] = nxt;
    }
    const double d = dinv ? dinv[i] : 1.0;
    if (last) {
      const double z = d * yi;
      x[i] = z;
      Z[col + i] = z;
    } else {
      if (mode != 2) y[i] = yi;
      x[i] = d * nxt;
    }
  }
}

// start of a cycle: g = (beta, 0, ...), n = 0
__global__ void k_arn_init(ArnoldiState* __restrict__ st, double* __restrict__ g, double beta) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    st->n = 0;
    st->err = beta;
    st->inv_h = 0.0;
    st->bad = 0;
    g[0] = beta;
  }
}

// y = -R^{-1} g over the cycle's n steps (negated: the update subtracts V y)
__global__ void k_arn_backsub(const ArnoldiState* __restrict__ st, const double* __restrict__ R, int ldr, const double* __restrict__ g,
                              double* __restrict__ y) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int k = st->n;
  for (int i = k - 1; i >= 0; --i) {
    double sum = g[i];
    for (int j = i + 1; j < k; ++j) sum -= R[(size_t)j * ldr + i] * y[j];
    y[i] = sum / R[(size_t)i * ldr + i];
  }
  for (int i = 0; i < k; ++i) y[i] = -y[i];
}

// w -= V[:, 0..n-1] y over the cycle's n columns (x update from the basis)
__global__ void k_maxpy_steps(const double* __restrict__ V, int ldv, const ArnoldiState* __restrict__ st, const double* __restrict__ y,
                              double* __restrict__ w, int nrow) {
  extern __shared__ double sh[];
  const int ncol = st->n;
  for (int c = threadIdx.x; c < ncol; c += blockDim.x) sh[c] = y[c];
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nrow; i += gridDim.x * blockDim.x) {
    double s = w[i];
    for (int c = 0; c < ncol; ++c) s = fma(-sh[c], V[(size_t)c * ldv + i], s);
    w[i] = s;
  }
}

int grid_rows(int n) {
  const int b = (n + 255) / 256;
  return b < 1 ? 1 : (b > 148 * 4 ? 148 * 4 : b);
}

}  // namespace

namespace {
// rows per slice of the orthogonalisation kernels: about 256, at most two slices per SM, and
// at most kArnRowsMax rows (the slice's shared-memory copy)
int arnoldi_rows(int n) {
  int nb = (n + 255) / 256;
  nb = nb < 1 ? 1 : (nb > 2 * 148 ? 2 * 148 : nb);
  int rows = (n + nb - 1) / nb;
  if (rows > kArnRowsMax) rows = kArnRowsMax;
  return rows < 1 ? 1 : rows;
}
}  // namespace

int arnoldi_dot_blocks(int n) {
  const int rows = arnoldi_rows(n);
  const int nb = (n + rows - 1) / rows;
  return nb < 1 ? 1 : nb;
}

// x = Z[:, n] = D^{-1} p(B) V[:, n]: d - 1 applications of the near-field operator for a
// polynomial of degree d (a conjugate pair takes two, the last factor none after it)
int launch_poly_apply(const ArnoldiArgs& a, cudaStream_t st) {
  const int g = grid_rows(a.nrow);
  const PolyRoots& R = *a.poly;
  launch_pdl(k_arn_prep, g, 256, 0, st, a.nrow, a.V, a.dinv, a.state, a.x);  // x = D^{-1} V[:, n]
  int launches = 1;
  bool first = true;
  for (int k = 0; k < R.n; ++k) {
    const bool last = k == R.n - 1;
    const double re = R.re[k], im = R.im[k];
    if (im == 0.0) {
      if (!last) launches += launch_near_only(a.p, a.near, st);
      launch_pdl(k_poly_factor, g, 256, 0, st, a.nrow, 0, (int)first, (int)last, 1.0 / re, 0.0, (const double*)a.V,
                 (const ArnoldiState*)a.state, a.prod, (const double*)a.w, a.y, a.dinv, a.x, a.Z);
      ++launches;
    } else {
      const double c = 1.0 / (re * re + im * im);
      launches += launch_near_only(a.p, a.near, st);
      launch_pdl(k_poly_factor, g, 256, 0, st, a.nrow, 1, (int)first, (int)last, c, 2.0 * re, (const double*)a.V,
                 (const ArnoldiState*)a.state, a.prod, (const double*)a.w, a.y, a.dinv, a.x, a.Z);
      ++launches;
      if (!last) {
        launches += launch_near_only(a.p, a.near, st);
        launch_pdl(k_poly_factor, g, 256, 0, st, a.nrow, 2, 0, 0, c, 0.0, (const double*)a.V, (const ArnoldiState*)a.state, a.prod,
                   (const double*)a.w, a.y, a.dinv, a.x, a.Z);
        ++launches;
      }
    }
    first = false;
  }
  return launches;
}

// bytes of dynamic shared memory of the kernels whose size grows with the basis capacity
size_t orth_dots_smem(int cols, int rows) { return sizeof(double) * ((size_t)cols + rows); }
size_t givens_smem(int cols) { return sizeof(double) * (3 * (size_t)cols + 1); }

int launch_arnoldi_step(const ArnoldiArgs& a, cudaStream_t st) {
  const int g = grid_rows(a.nrow);
  const int rows = arnoldi_rows(a.nrow);
  const int nb = arnoldi_dot_blocks(a.nrow);
  int launches = 0;
  if (a.poly && a.poly->n > 0) {
    launches = launch_poly_apply(a, st);
  } else if (a.bj.nblocks > 0) {  // x = M^{-1} V[:, n] (block Jacobi)
    launch_bj_apply(a.bj, a.V, a.nrow, a.state, a.x, st);
    launches = 1;
  }  // else x was written by the previous step's k_arn_next
  launches += launch_matvec(a.p, a.mv, st);
  double* h1 = a.h;
  double* h2 = a.h + a.cols;
  const ArnoldiState* cst = a.state;
  launch_pdl(k_arn_dots, nb, kArnThreads, sizeof(double) * rows, st, (const double*)a.V, a.nrow, cst, (const double*)a.w, a.nrow, rows,
             a.partial);
  launch_pdl(k_arn_sum, a.cols, kArnThreads, 0, st, (const double*)a.partial, nb, cst, h1);
  launch_pdl(k_arn_orth_dots, nb, kArnThreads, orth_dots_smem(a.cols, rows), st, (const double*)a.V, a.nrow, cst, (const double*)h1, a.w,
             a.nrow, rows, a.partial, a.cols);
  launch_pdl(k_arn_sum, a.cols, kArnThreads, 0, st, (const double*)a.partial, nb, cst, h2);
  launch_pdl(k_arn_orth_norm, nb, kArnThreads, sizeof(double) * a.cols, st, (const double*)a.V, a.nrow, cst, (const double*)h2, a.w,
             a.nrow, rows, a.partial);
  launch_pdl(k_arn_givens, 1, 32, givens_smem(a.cols), st, a.state, (const double*)h1, (const double*)h2, (const double*)a.partial, nb,
             a.cs, a.sn, a.g, a.R, a.cols);
  launch_pdl(k_arn_next, g, 256, 0, st, a.nrow, (const double*)a.w, cst, a.V, a.dinv, a.x);
  return launches + 7;
}

int configure_arnoldi(int cols) {
  // the permission only grows (contexts on other threads may use larger bases); it belongs
  // to the current device, so the bookkeeping is per device
  static std::mutex mu;
  static size_t granted[kMaxDevices] = {};
  const size_t b1 = orth_dots_smem(cols, kArnRowsMax), b2 = givens_smem(cols);
  const size_t bytes = b1 > b2 ? b1 : b2;
  if (bytes > 227 * 1024) return -1;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = -1;
  const bool tracked = dev >= 0 && dev < kMaxDevices;  // untracked devices: set every time
  std::lock_guard<std::mutex> lk(mu);
  if (tracked && bytes <= granted[dev]) return 0;
  if (cudaFuncSetAttribute(k_arn_orth_dots, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess) return -1;
  if (cudaFuncSetAttribute(k_arn_orth_norm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess) return -1;
  if (cudaFuncSetAttribute(k_arn_givens, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess) return -1;
  if (tracked) granted[dev] = bytes;
  return 0;
}

void launch_arnoldi_prep(int nrow, const double* V, const double* dinv, const ArnoldiState* state, double* x, cudaStream_t st) {
  k_arn_prep<<<grid_rows(nrow), 256, 0, st>>>(nrow, V, dinv, state, x);
}

void launch_arnoldi_init(ArnoldiState* state, double* g, double beta, cudaStream_t st) { k_arn_init<<<1, 32, 0, st>>>(state, g, beta); }

void launch_arnoldi_solve_y(const ArnoldiState* state, const double* R, int ldr, const double* g, double* y, cudaStream_t st) {
  k_arn_backsub<<<1, 32, 0, st>>>(state, R, ldr, g, y);
}

void launch_arnoldi_update(const double* V, int n, int cols, const ArnoldiState* state, const double* y, double* w, cudaStream_t st) {
  k_maxpy_steps<<<grid_rows(n), 256, sizeof(double) * cols, st>>>(V, n, state, y, w, n);
}

}  // namespace bemb200
