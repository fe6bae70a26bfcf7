// Mixed-precision M2L on the Blackwell tensor cores (tcgen05, FP16 operands, FP32 accumulate
// in tensor memory).  Used by the mixed-precision solve for its inner (correction) mat-vecs;
// the FP64 M2L in kernels.cu stays the reference-parity path.
//
// Real form.  For degree n and order m >= 0 the complex local coefficient is split into
// Re, and Im for m > 0 (Im L_n^0 = 0 for a real field), so the (p+1)(p+2)/2 complex
// coefficients become NR = (p+1)^2 real ones, in the order
//   (0,0,re), (1,0,re), (1,1,re), (1,1,im), (2,0,re), (2,1,re), (2,1,im), ...
// i.e. degree n starts at n^2.  The same order is used for multipoles.  With
// M^{-m} = (-1)^m conj(M^m) the M2L L_n^m = (-1)^n sum S_{n+n'}^{m+m'}(d) M_{n'}^{m'} is a real
// NR x NR matrix T(d) applied to the real multipole vector.
//
// Scaling.  With a_t, a_s the target and source bucket sizes and d^ = d / a_t:
//   S_j^k(d) = a_t^{-(j+1)} S_j^k(d^)    (homogeneity),
//   M^_n' = M_n' / a_s^n',  L^_n = L_n a_t^{n+1}  =>  L^ = T(d^) diag((a_s/a_t)^n') M^,
// so one table serves every level for a lattice offset d^ = r.  Each coefficient is further
// normalised by alpha(n,m) = sqrt((n+m)!(n-m)!):  M~ = alpha M^,  L~ = L^ / alpha, so
// T~ = T / (alpha_i alpha_k), whose entries are bounded by 2^j / |d^|^{j+1} <= 1 for
// well-separated buckets.  Each multipole column is finally scaled by a power of two so
// that its largest entry lies in [0.5, 1), and the scale is undone in FP32 after the MMA.
//
// Precision.  Every operand x is split into FP16 hi = fp16(x), lo = fp16(x - hi) (22
// significant bits together); the product uses three MMA passes hi*hi + hi*lo + lo*hi
// accumulated in FP32, so each translated coefficient carries an error of about 2^-22 of
// the largest term of its column.
//
// GEMM shape per work item: D[128 rows (output coefficients) x N (2 x pairs: both
// densities)] = T~[128 x KP] * B[N x KP]^T, A = the table (one per item), B = gathered
// multipole rows; K-major, no swizzle, operands staged in shared memory by cp.async,
// D in tensor memory, one thread issues the MMAs and commits to an mbarrier.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

#include "fmm_math.cuh"
#include "kernels.cuh"
#include "tc_sm100.cuh"

namespace bemb200 {
namespace {

constexpr int kRows = 128;          // MMA M: output coefficients (NR <= 128, p <= 10)
constexpr int kMaxPairs = 128;      // pairs per work item
constexpr int kMaxCols = 2 * kMaxPairs;  // MMA N (two densities per pair)
constexpr uint32_t kWaitTries = 1u << 22;

template <int P>
struct TcDims {
  static constexpr int NR = (P + 1) * (P + 1);
  static constexpr int KP = (NR + 15) / 16 * 16;  // K padded to the MMA K step (16)
  static constexpr int KC = KP / 8;               // 16-byte chunks per operand row
  static constexpr int TAB_BYTES = 2 * kRows * KP * 2;    // hi + lo images of one table
  static constexpr int B_BYTES = 2 * kMaxCols * KP * 2;   // hi + lo gathered rows
  // at least half the SM's shared memory, so one CTA (and one TMEM allocation) per SM
  static constexpr int SMEM = (TAB_BYTES + B_BYTES) > 116 * 1024 ? (TAB_BYTES + B_BYTES) : 116 * 1024;
  static_assert(NR <= kRows, "tensor-core M2L needs (p+1)^2 <= 128");
};

// real index i -> (n, m, part) with part 0 = Re, 1 = Im
__device__ __forceinline__ void decode_real(int i, int& n, int& m, int& part) {
  n = (int)sqrtf((float)i);
  while (n * n > i) --n;
  while ((n + 1) * (n + 1) <= i) ++n;
  const int o = i - n * n;
  m = (o + 1) >> 1;
  part = (o > 0 && (o & 1) == 0) ? 1 : 0;
}

__device__ __forceinline__ void cp_async16(void* s, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// ---------------------------------------------------------------------------
// Set-up: one normalised table per translation, as hi/lo FP16 images in the shared-memory
// (core-matrix) layout so a work item copies it with straight 16-byte chunks.
template <int P>
__global__ void __launch_bounds__(128) k_tc_tables(int ntab, const double* __restrict__ tab, const double* __restrict__ alpha,
                                                   __half* __restrict__ T, unsigned int* __restrict__ maxbits) {
  using D = TcDims<P>;
  constexpr int Q = 2 * P, NS = (Q + 1) * (Q + 1);
  __shared__ double2 sS[NS];
  __shared__ float red[4];
  const int g = blockIdx.x;
  if (g >= ntab) return;
  const double x = tab[4 * g], y = tab[4 * g + 1], z = tab[4 * g + 2], ratio = tab[4 * g + 3];
  if (threadIdx.x < 32) S_full_column<Q>(threadIdx.x, x, y, z, sS);
  __syncthreads();
  unsigned char* base = reinterpret_cast<unsigned char*>(T) + (size_t)g * D::TAB_BYTES;
  float vmax = 0.f;
  for (int e = threadIdx.x; e < kRows * D::KP; e += blockDim.x) {
    const int i = e / D::KP, k = e - (e / D::KP) * D::KP;
    double v = 0.0;
    if (i < D::NR && k < D::NR) {
      int n, m, po, n1, m1, pi;
      decode_real(i, n, m, po);
      decode_real(k, n1, m1, pi);
      const int j = n + n1;
      const double2 Sp = sS[j * (j + 1) + m + m1];
      double val;
      if (m1 == 0) {
        val = po ? Sp.y : Sp.x;
      } else {
        const double2 Sm = sS[j * (j + 1) + m - m1];
        const double sg = (m1 & 1) ? -1.0 : 1.0;
        if (pi == 0)
          val = po ? (Sp.y + sg * Sm.y) : (Sp.x + sg * Sm.x);
        else
          val = po ? (Sp.x - sg * Sm.x) : (-Sp.y + sg * Sm.y);
      }
      double rp = 1.0;
      for (int q = 0; q < n1; ++q) rp *= ratio;
      v = ((n & 1) ? -val : val) * rp / (alpha[i] * alpha[k]);
    }
    const __half h = __double2half(v);
    const __half l = __double2half(v - (double)__half2float(h));
    const uint32_t off = kmajor_offset(i, k, D::KP);
    *reinterpret_cast<__half*>(base + off) = h;
    *reinterpret_cast<__half*>(base + kRows * D::KP * 2 + off) = l;
    vmax = fmaxf(vmax, (float)fabs(v));
  }
  for (int o = 16; o > 0; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = vmax;
  __syncthreads();
  if (threadIdx.x == 0) {
    float mx = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) mx = fmaxf(mx, red[w]);
    atomicMax(maxbits, __float_as_uint(mx));
  }
}

// ---------------------------------------------------------------------------
// Per mat-vec: FP64 multipoles -> normalised, power-of-two scaled FP16 hi/lo rows.
// One warp per (bucket, density); row layout [hi KP][lo KP] halves.
template <int P>
__global__ void k_tc_expand(int nnodes, const double2* __restrict__ M, const double* __restrict__ node_dL,
                            const double* __restrict__ alpha, __half* __restrict__ Mt, float* __restrict__ escale) {
  using D = TcDims<P>;
  constexpr int NC = ncoef(P), PER = (D::KP + 31) / 32;
  const int lane = threadIdx.x & 31;
  const int w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int nd = w0; nd < 2 * nnodes; nd += nw) {
    const int node = nd >> 1;
    const double inv_a = 1.0 / node_dL[node];
    const double2* Mc = M + (size_t)nd * NC;  // [node][d][NC] with nd = 2 node + d
    double v[PER];
    double mx = 0.0;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int k = lane + 32 * q;
      double x = 0.0;
      if (k < D::NR) {
        int n1, m1, part;
        decode_real(k, n1, m1, part);
        const double2 c = Mc[cidx(n1, m1)];
        double ip = 1.0;
        for (int t = 0; t < n1; ++t) ip *= inv_a;
        x = (part ? c.y : c.x) * alpha[k] * ip;
      }
      v[q] = x;
      mx = fmax(mx, fabs(x));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    int E = 0;
    if (mx > 0.0 && mx < 1e300) frexp(mx, &E);  // mx = f 2^E, f in [0.5, 1)
    const double s = ldexp(1.0, -E);
    __half* row = Mt + (size_t)nd * 2 * D::KP;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int k = lane + 32 * q;
      if (k < D::KP) {
        const double x = v[q] * s;
        const __half h = __double2half(x);
        row[k] = h;
        row[D::KP + k] = __double2half(x - (double)__half2float(h));
      }
    }
    if (lane == 0) escale[nd] = ldexpf(1.f, E);
  }
}

// ---------------------------------------------------------------------------
// The contraction.  Persistent CTAs of 4 warps walk the work items; per item:
//   1. pair metadata to shared memory, 2. cp.async the table image and gather the
//   multipole rows of the item's sources (both densities, zero rows as padding),
//   3. thread 0 issues 3 x KP/16 MMAs (hi*hi, hi*lo, lo*hi) into one TMEM accumulator
//   and commits to an mbarrier, 4. each warp reads its 32 TMEM lanes (= 32 output
//   coefficients) and writes the partial locals of every pair to its slot, scaled back.
// Every wait is bounded; a timeout sets *err, skips the remaining items and frees TMEM.
template <int P>
__global__ void __launch_bounds__(128, 1)
    k_m2l_tc(int nitems, const int* __restrict__ item_tab, const int* __restrict__ item_begin, const int* __restrict__ item_cnt,
             const int* __restrict__ tc_pair, const int* __restrict__ m2l_src, const __half* __restrict__ Ttab,
             const __half* __restrict__ Mt, const float* __restrict__ escale, int zero_row, float* __restrict__ Y, int* __restrict__ err) {
  using D = TcDims<P>;
  extern __shared__ __align__(128) unsigned char sm_tc[];
  unsigned char* sT = sm_tc;                 // [hi | lo] table images
  unsigned char* sB = sm_tc + D::TAB_BYTES;  // [hi | lo] gathered rows, kMaxCols each
  __shared__ int s_row[kMaxCols];
  __shared__ float s_sc[kMaxCols];
  __shared__ int s_slot[kMaxPairs];
  __shared__ uint64_t bar;
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) tmem_alloc(&tslot, 256);
  if (tid == 0) mbar_init(&bar, 1);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tslot;
  uint32_t phase = 0;
  bool failed = false;
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int tab = item_tab[item], b0 = item_begin[item], cnt = item_cnt[item];
    const int ncol = 2 * cnt, npad = (ncol + 15) & ~15;
    for (int c = tid; c < npad; c += blockDim.x) {
      if (c < ncol) {
        const int j = c >> 1, d = c & 1;
        const int slot = tc_pair[b0 + j];
        const int src = m2l_src[slot];
        s_row[c] = 2 * src + d;
        s_sc[c] = escale[2 * src + d];
        if (d == 0) s_slot[j] = slot;
      } else {
        s_row[c] = zero_row;
        s_sc[c] = 0.f;
      }
    }
    __syncthreads();
    {
      const unsigned char* gT = reinterpret_cast<const unsigned char*>(Ttab) + (size_t)tab * D::TAB_BYTES;
      for (int q = tid; q < D::TAB_BYTES / 16; q += blockDim.x) cp_async16(sT + 16 * q, gT + 16 * q);
      const int per_part = npad * D::KC;
      for (int q = tid; q < 2 * per_part; q += blockDim.x) {
        const int part = q >= per_part ? 1 : 0;
        const int qq = q - part * per_part;
        const int rg = qq / (8 * D::KC), kc = (qq >> 3) % D::KC, r8 = qq & 7;
        const int c = rg * 8 + r8;
        const __half* src = Mt + ((size_t)s_row[c] * 2 + part) * D::KP + kc * 8;
        cp_async16(sB + part * (kMaxCols * D::KP * 2) + kmajor_offset(c, kc * 8, D::KP), src);
      }
      cp_async_wait_all();
      fence_proxy_async_smem();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0) {
      const uint32_t idesc = make_idesc_f16_f32(kRows, npad);
      const uint32_t aH = smem_u32(sT), aL = aH + kRows * D::KP * 2;
      const uint32_t bH = smem_u32(sB), bL = bH + kMaxCols * D::KP * 2;
      constexpr uint32_t SBO = D::KP * 16;
#pragma unroll 1
      for (int k = 0; k < D::KP / 16; ++k)
        tc_mma_f16(tbase, make_smem_desc(aH + 256 * k, 128, SBO), make_smem_desc(bH + 256 * k, 128, SBO), idesc, k > 0 ? 1u : 0u);
#pragma unroll 1
      for (int k = 0; k < D::KP / 16; ++k)
        tc_mma_f16(tbase, make_smem_desc(aH + 256 * k, 128, SBO), make_smem_desc(bL + 256 * k, 128, SBO), idesc, 1u);
#pragma unroll 1
      for (int k = 0; k < D::KP / 16; ++k)
        tc_mma_f16(tbase, make_smem_desc(aL + 256 * k, 128, SBO), make_smem_desc(bH + 256 * k, 128, SBO), idesc, 1u);
      tc_commit(&bar);
    }
    const bool ok = mbar_wait(&bar, phase, kWaitTries);
    phase ^= 1u;
    if (__syncthreads_or(ok ? 0 : 1)) {
      failed = true;
      break;
    }
    tc_fence_after();
    const int i = warp * 32 + lane;  // output coefficient of this thread's TMEM lane
    for (int c0 = 0; c0 < npad; c0 += 8) {
      float v[8];
      tmem_ld8(tbase + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (i < D::KP) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int c = c0 + q;
          if (c < ncol) Y[((size_t)s_slot[c >> 1] * 2 + (c & 1)) * D::KP + i] = v[q] * s_sc[c];
        }
      }
    }
    tc_fence_before();
    __syncthreads();
  }
  if (failed && tid == 0) atomicExch(err, 1);
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tbase, 256);
  }
}

// Per target bucket: L = sum of its slots (target-major CSR order, deterministic), back to
// the FP64 complex layout [node][density][NC] with the normalisation and a_t^{n+1} undone.
template <int P>
__global__ void k_m2l_tc_reduce(int ntargets, const int* __restrict__ targets, const int* __restrict__ m2l_off,
                                const double* __restrict__ node_dL, const double* __restrict__ alpha, const float* __restrict__ Y,
                                double2* __restrict__ L) {
  using D = TcDims<P>;
  constexpr int NC = ncoef(P);
  const int64_t total = (int64_t)ntargets * 2 * NC;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
    const int ti = (int)(e / (2 * NC));
    const int r = (int)(e - (int64_t)ti * 2 * NC);
    const int d = r / NC, o = r - d * NC;
    int n = 0;
    while ((n + 1) * (n + 2) / 2 <= o) ++n;
    const int m = o - n * (n + 1) / 2;
    const int ire = n * n + (m == 0 ? 0 : 2 * m - 1);
    const int tgt = targets[ti];
    double sr = 0.0, si = 0.0;
    for (int k = m2l_off[tgt]; k < m2l_off[tgt + 1]; ++k) {
      const float* y = Y + ((size_t)k * 2 + d) * D::KP;
      sr += (double)y[ire];
      if (m > 0) si += (double)y[ire + 1];
    }
    const double a = node_dL[tgt];
    double ap = a;
    for (int t = 0; t < n; ++t) ap *= a;
    const double f = alpha[ire] / ap;
    L[((size_t)tgt * 2 + d) * NC + o] = make_double2(sr * f, si * f);
  }
}

template <int P>
int m2l_tc_launch(const MatvecArgs& a, cudaStream_t st) {
  using D = TcDims<P>;
  if (a.n_tc_items <= 0) return 0;
  const int nd = 2 * a.n_nodes;
  const int ge = (int)std::min<int64_t>(((int64_t)nd * 32 + 255) / 256, 148 * 8);
  __half* Mt = static_cast<__half*>(a.tc_Mt);
  k_tc_expand<P><<<ge, 256, 0, st>>>(a.n_nodes, a.M, a.node_dL, a.tc_alpha, Mt, a.tc_escale);
  const int grid = a.n_tc_items < a.tc_grid ? a.n_tc_items : a.tc_grid;
  k_m2l_tc<P><<<grid, 128, D::SMEM, st>>>(a.n_tc_items, a.tc_item_tab, a.tc_item_begin, a.tc_item_cnt, a.tc_pair, a.m2l_src,
                                           static_cast<const __half*>(a.tc_tab), Mt, a.tc_escale, nd, a.tc_Y, a.tc_err);
  const int64_t tr = (int64_t)a.n_m2l_targets * 2 * ncoef(P);
  const int gr = (int)std::min<int64_t>((tr + 255) / 256, 148 * 16);
  k_m2l_tc_reduce<P><<<gr, 256, 0, st>>>(a.n_m2l_targets, a.m2l_targets, a.m2l_off, a.node_dL, a.tc_alpha, a.tc_Y, a.L);
  return 3;
}

template <int P>
void tc_tables_launch(int ntab, const double* tab, const double* alpha, __half* T, unsigned int* maxbits, cudaStream_t st) {
  cudaFuncSetAttribute(k_m2l_tc<P>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcDims<P>::SMEM);
  if (ntab > 0) k_tc_tables<P><<<ntab, 128, 0, st>>>(ntab, tab, alpha, T, maxbits);
}

}  // namespace

int tc_supported(int p) { return p >= 1 && (p + 1) * (p + 1) <= kRows; }
int tc_kp(int p) { return ((p + 1) * (p + 1) + 15) / 16 * 16; }
size_t tc_table_bytes(int p) { return (size_t)2 * kRows * tc_kp(p) * 2; }
int tc_max_pairs() { return kMaxPairs; }

void tc_alpha_host(int p, double* alpha) {
  // alpha(i) = sqrt((n+m)! (n-m)!) for the real index i of (n, m, part)
  double fact[64];
  fact[0] = 1.0;
  for (int i = 1; i < 64; ++i) fact[i] = fact[i - 1] * i;
  const int kp = tc_kp(p);
  for (int i = 0; i < kp; ++i) alpha[i] = 1.0;
  for (int n = 0; n <= p; ++n)
    for (int m = 0; m <= n; ++m) {
      const double v = std::sqrt(fact[n + m] * fact[n - m]);
      const int ire = n * n + (m == 0 ? 0 : 2 * m - 1);
      alpha[ire] = v;
      if (m > 0) alpha[ire + 1] = v;
    }
}

void launch_tc_tables(int p, int ntab, const double* tab, const double* alpha, void* T, unsigned int* maxbits, cudaStream_t st) {
  __half* t = static_cast<__half*>(T);
  switch (p) {
#define BEMB200_CASE(PP) \
  case PP:               \
    tc_tables_launch<PP>(ntab, tab, alpha, t, maxbits, st); break;
    BEMB200_CASE(1) BEMB200_CASE(2) BEMB200_CASE(3) BEMB200_CASE(4) BEMB200_CASE(5)
    BEMB200_CASE(6) BEMB200_CASE(7) BEMB200_CASE(8) BEMB200_CASE(9) BEMB200_CASE(10)
#undef BEMB200_CASE
    default: break;
  }
}

int launch_m2l_tc(int p, const MatvecArgs& a, cudaStream_t st) {
  switch (p) {
#define BEMB200_CASE(PP) \
  case PP:               \
    return m2l_tc_launch<PP>(a, st);
    BEMB200_CASE(1) BEMB200_CASE(2) BEMB200_CASE(3) BEMB200_CASE(4) BEMB200_CASE(5)
    BEMB200_CASE(6) BEMB200_CASE(7) BEMB200_CASE(8) BEMB200_CASE(9) BEMB200_CASE(10)
#undef BEMB200_CASE
    default: break;
  }
  return 0;
}

}  // namespace bemb200
