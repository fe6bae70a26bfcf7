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
// Densities.  A mat-vec row needs only GPhin - GnPhi, and the far field of both comes from
// the same L2P, so the M2L here translates the combined multipole M[0] - M[1] into L[0] and
// leaves L[1] = 0: one column per pair instead of two.
//
// GEMM shape per work item (<= 256 pairs of one table): D[128 coefficients x pairs] =
// T~[128 x KP] * B[pairs x KP]^T, B = gathered multipole rows, T~ = the table; both K-major,
// staged in shared memory by the TMA unit, D in tensor memory, one thread issues the MMAs
// and commits to mbarriers.
#include <cuda.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>

#include "fmm_math.cuh"
#include "kernels.cuh"
#include "tc_sm100.cuh"

namespace bemb200 {
namespace {

constexpr int kRows = 128;          // table rows = MMA N: output coefficients (NR <= 128, p <= 10)
// pairs per work item = gathered rows (one per pair) = MMA N: at most 80 with two table slots
// in shared memory, at most 128 with one (p <= 10; the kernel variant is chosen per launch)
constexpr int kMaxPairs = 80;
constexpr int kMaxPairsWide = 128;
// Bounded waits: the pipeline waits use the launch's wait_tries (kWaitTries unless a caller set
// a test limit); after a wait gave up, the waits that drain the CTA's own copies and MMAs still
// in flight always use kDrainTries, so a CTA never leaves with asynchronous work pending.
constexpr uint32_t kWaitTries = 1u << 22;
constexpr uint32_t kDrainTries = 1u << 22;

template <int P, int MC = kMaxPairs>
struct TcDims {
  static constexpr int NR = (P + 1) * (P + 1);
  static constexpr int KP = (NR + 63) / 64 * 64;  // K padded to whole 128-byte swizzle atoms
  static constexpr int KA = KP / 64;              // K atoms (64 halves) per operand row
  static constexpr int RT = (NR + kRows - 1) / kRows;  // row tiles of 128 output coefficients per table
  // floats per pair partial: the padded coefficient count (a multiple of 64, so every lane of
  // the reduction reads an even number of floats at an 8-byte aligned offset)
  static constexpr int KPO = KP;
  static constexpr int TAB_BYTES = 2 * kRows * KP * 2;    // hi + lo images of one row tile of a table
  static constexpr int REGION = MC * 128;                 // one (part, atom) region of gathered rows
  static constexpr int B_BYTES = 2 * KA * REGION;         // hi + lo gathered rows
  // two table slots when they fit beside two stages of gathered rows (one slot for the
  // 96 KB images of p = 11, 12), plus 1 KB to align them to the 1024-byte swizzle atom; at
  // least half the SM's shared memory, so one CTA (and one TMEM allocation) per SM
  static constexpr int TAB_SLOTS = 2 * TAB_BYTES + 2 * B_BYTES + 1024 + 4096 <= 227 * 1024 ? 2 : 1;
  static constexpr int NEED = TAB_SLOTS * TAB_BYTES + 2 * B_BYTES + 1024;
  static constexpr int SMEM = NEED > 116 * 1024 ? NEED : 116 * 1024;
  static_assert(RT <= 2, "tensor-core M2L needs (p+1)^2 <= 256");
  static_assert(KPO % 64 == 0 && KPO / 32 <= 6, "partial rows of 64, 128 or 192 floats");
  static_assert(TAB_BYTES % 1024 == 0 && B_BYTES % 1024 == 0, "gathered rows must start on a swizzle atom");
  static_assert(NEED + 4096 <= 227 * 1024, "shared memory of one CTA");
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
  const int g = blockIdx.x;  // image: table g / RT, output rows [128 (g % RT), 128 (g % RT) + 128)
  if (g >= ntab * D::RT) return;
  const int tb = g / D::RT, r0 = (g % D::RT) * kRows;
  const double x = tab[4 * tb], y = tab[4 * tb + 1], z = tab[4 * tb + 2], ratio = tab[4 * tb + 3];
  if (threadIdx.x < 32) S_full_column<Q>(threadIdx.x, x, y, z, sS);
  __syncthreads();
  unsigned char* base = reinterpret_cast<unsigned char*>(T) + (size_t)g * D::TAB_BYTES;
  float vmax = 0.f;
  for (int e = threadIdx.x; e < kRows * D::KP; e += blockDim.x) {
    const int il = e / D::KP, k = e - (e / D::KP) * D::KP, i = r0 + il;
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
    const uint32_t off = kmajor_offset(il, k, D::KP);
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
// Per mat-vec: FP64 multipoles -> combined M[0] - M[1] (ND = 2) or M[0] as given (ND = 1),
// normalised, power-of-two scaled FP16 hi/lo rows.  One warp per bucket; row layout
// [hi KP][lo KP] halves.
template <int P, int ND>
__global__ void k_tc_expand(int nnodes, const double2* __restrict__ M, const double* __restrict__ node_dL,
                            const double* __restrict__ alpha, __half* __restrict__ Mt, float* __restrict__ escale) {
  pdl_enter();
  using D = TcDims<P>;
  constexpr int NC = ncoef(P), PER = (D::KP + 31) / 32;
  const int lane = threadIdx.x & 31;
  const int w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int node = w0; node < nnodes; node += nw) {
    const double inv_a = 1.0 / node_dL[node];
    const double2* M0 = M + (size_t)node * 2 * NC;
    double v[PER];
    double mx = 0.0;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int k = lane + 32 * q;
      double x = 0.0;
      if (k < D::NR) {
        int n1, m1, part;
        decode_real(k, n1, m1, part);
        const double2 c0 = M0[cidx(n1, m1)];
        const double2 c1 = ND == 2 ? M0[NC + cidx(n1, m1)] : make_double2(0.0, 0.0);
        double ip = 1.0;
        for (int t = 0; t < n1; ++t) ip *= inv_a;
        x = (part ? (c0.y - c1.y) : (c0.x - c1.x)) * alpha[k] * ip;
      }
      v[q] = x;
      mx = fmax(mx, fabs(x));
    }
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    int E = 0;
    if (mx > 0.0 && mx < 1e300) frexp(mx, &E);  // mx = f 2^E, f in [0.5, 1)
    const double sc = ldexp(1.0, -E);
    __half* row = Mt + (size_t)node * 2 * D::KP;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
      const int k = lane + 32 * q;
      if (k < D::KP) {
        const double x = v[q] * sc;
        const __half h = __double2half(x);
        row[k] = h;
        row[D::KP + k] = __double2half(x - (double)__half2float(h));
      }
    }
    if (lane == 0) escale[node] = ldexpf(1.f, E);
  }
}

// ---------------------------------------------------------------------------
// The contraction: persistent, warp-specialised CTAs, each over a contiguous range of work
// items (consecutive items mostly share a table, which then stays in shared memory).
//   warps 0-7   epilogue: TMEM lane = output coefficient, column = pair; warp w reads lane
//               quadrant w % 4 and every other 32-column chunk (w / 4 picks which); for
//               each pair it stores 32 consecutive coefficients (one 128-byte line) of the
//               pair's partial.  Partials are stored in work-item order, so a CTA writes one
//               contiguous stream; the reduction gathers them per target and undoes the
//               column scales.  The next chunk's TMEM load is in flight while the current
//               chunk is stored.
//   warps 8-11  producers (thread = gathered row): metadata is loaded two items ahead;
//               TMA: one bulk copy of the table image when the table changes, and
//               tile::gather4 loads of the multipole rows of the item's sources into
//               128-byte swizzled K-major tiles
//   warp 12     MMA issuer (one elected lane)
// MMA per item: D[128 coefficients x N pairs] = T~ * B^T with A = T~ (no swizzle, K-major)
// and B = gathered rows (SW128 K-major), N = pairs rounded up to 16, three passes
// hi*hi + hi*lo + lo*hi.  Shared memory holds two table images and two item stages of
// gathered rows, TMEM four accumulators (128 columns each): the loads of item i+1 (and of
// its table, when it differs) overlap the MMAs of item i, and the epilogue of item i
// overlaps both.
// Barriers (s = item stage = i % 2, t = table slot, b = accumulator = i % 4):
//   full[s]    all TMA bytes of the item landed                   -> MMA issuer
//   bfree[s]   MMAs of the item finished reading its gathered rows -> producers
//   tfree[t]   MMAs of every item of the table in slot t finished  -> producers
//   accf[b]    accumulator b written                               -> epilogue
//   acce[b]    epilogue drained accumulator b                      -> producers, MMA issuer
//   meta[b]    epilogue metadata of accumulator b published        -> epilogue
// Every wait is bounded; a timeout records *err and ends the waiting role's loop, and the
// roles waiting on it then time out as well rather than wait forever.
constexpr int kProducers = 128;
constexpr int kEpilogue = 256;
constexpr int kIssuer = 32;
constexpr int kStages = 2;
constexpr int kAcc = 4;
constexpr int kAccCols = 128;
static_assert(kMaxPairsWide <= kAccCols, "one accumulator holds an item");
static_assert(kMaxPairsWide <= kProducers, "one producer thread per gathered row");

template <int P, int MC, bool FUSED>
__global__ void __launch_bounds__(kEpilogue + kProducers + kIssuer, 1)
    k_m2l_tc(const __grid_constant__ CUtensorMap rows_map, int nitems, const int* __restrict__ item_tab, const int* __restrict__ item_begin,
             const int* __restrict__ item_cnt, int npairs, const int* __restrict__ tc_src, const __half* __restrict__ Ttab,
             const __half* __restrict__ Mt, float* __restrict__ Y, int* __restrict__ err, uint32_t wait_tries,
             const int* __restrict__ tc_tgt, const float* __restrict__ escale, float* __restrict__ acc) {
  pdl_enter();
  using D = TcDims<P, MC>;
  extern __shared__ __align__(128) unsigned char sm_raw[];
  unsigned char* sm_tc = sm_raw + ((1024u - (smem_u32(sm_raw) & 1023u)) & 1023u);
  constexpr int NS = D::TAB_SLOTS;
  unsigned char* sT = sm_tc;                      // table slots: [hi | lo] images, kRows rows each
  unsigned char* sB = sm_tc + NS * D::TAB_BYTES;  // kStages stages of regions (part, atom): MC rows x 128 B
  __shared__ int s_row[MC];
  __shared__ int s_ncol[kAcc], s_b0[kAcc], s_rt[kAcc];
  // FUSED: per accumulator, the target (compact index) and source column scale of each pair
  __shared__ int s_tgt[FUSED ? kAcc : 1][FUSED ? MC : 1];
  __shared__ float s_sc[FUSED ? kAcc : 1][FUSED ? MC : 1];
  __shared__ int s_tsl[kStages], s_icol[kStages], s_last[kStages];
  __shared__ uint64_t bar_full[kStages], bar_bfree[kStages], bar_tfree[2], bar_accf[kAcc], bar_acce[kAcc], bar_meta[kAcc];
  __shared__ uint32_t tslot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int i0 = (int)((int64_t)nitems * blockIdx.x / gridDim.x);
  const int i1 = (int)((int64_t)nitems * (blockIdx.x + 1) / gridDim.x);
  if (warp == 0) tmem_alloc(&tslot, kAcc * kAccCols);
  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&bar_full[s], 1);
      mbar_init(&bar_bfree[s], 1);
    }
    for (int t = 0; t < NS; ++t) mbar_init(&bar_tfree[t], 1);
    for (int b = 0; b < kAcc; ++b) {
      mbar_init(&bar_accf[b], 1);
      mbar_init(&bar_acce[b], kEpilogue);
      mbar_init(&bar_meta[b], 1);
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tslot;
  if (tid >= kEpilogue + kProducers) {
    // MMA issuer
    if (lane == 0) {
      int issued = 0;
      bool ok = true;
      for (int it = i0; it < i1; ++it) {
        const int li = it - i0, s = li % kStages, b = li % kAcc;
        ok = mbar_wait(&bar_full[s], (li / kStages) & 1, wait_tries);
        if (ok && li >= kAcc) ok = mbar_wait(&bar_acce[b], ((li / kAcc) - 1) & 1, wait_tries);
        if (!ok) break;
        tc_fence_after();
        const int tsl = s_tsl[s], ncol = s_icol[s], last = s_last[s];
        const int npad = (ncol + 15) & ~15;
        const uint32_t idesc = make_idesc_f16_f32(kRows, npad);
        constexpr uint32_t SBO_T = D::KP * 16;
        const uint32_t bBase = smem_u32(sB + s * D::B_BYTES);
        const uint32_t aH = smem_u32(sT + tsl * D::TAB_BYTES), aL = aH + kRows * D::KP * 2;
        const uint32_t dt = tbase + (uint32_t)(b * kAccCols);
        // descriptors of the item's operands; every MMA's start address is a compile-time
        // offset from them (the address field counts 16-byte units and cannot carry: shared
        // memory is below 256 KB)
        const uint64_t dAh = make_smem_desc(aH, 128, SBO_T), dAl = make_smem_desc(aL, 128, SBO_T);
        const uint64_t dB = make_smem_desc_sw128(bBase, 1024);
#pragma unroll
        for (int pass = 0; pass < 3; ++pass) {
          const uint64_t a0 = pass == 2 ? dAl : dAh;                                     // T: hi, hi, lo
          const uint64_t b0 = dB + (pass == 1 ? (uint64_t)((D::KA * D::REGION) >> 4) : 0);  // rows: hi, lo, hi
#pragma unroll
          for (int k = 0; k < D::KP / 16; ++k)
            tc_mma_f16(dt, a0 + (uint64_t)(16 * k), b0 + (uint64_t)((((k >> 2) * D::REGION) + (k & 3) * 32) >> 4), idesc,
                       (pass > 0 || k > 0) ? 1u : 0u);
        }
        tc_commit(&bar_bfree[s]);
        tc_commit(&bar_accf[b]);
        if (last) tc_commit(&bar_tfree[tsl]);  // the table's last item: its slot is free once these MMAs end
        ++issued;
      }
      if (!ok) {
        atomicExch(err, 1);
        // let MMAs already issued finish before the CTA leaves
        if (issued > 0) mbar_wait(&bar_bfree[(issued - 1) % kStages], ((issued - 1) / kStages) & 1, kDrainTries);
      }
    }
    __syncwarp();
  } else if (tid >= kEpilogue) {
    const int pt = tid - kEpilogue;  // producer thread = gathered row
    int last_tab = -1, ntab_loaded = 0;
    int armed[kStages];  // item (local index) whose loads were last started on each stage, -1: none
#pragma unroll
    for (int q = 0; q < kStages; ++q) armed[q] = -1;
    bool ok = true;
    // metadata of the current item (c_) and of the next one (n_), loaded two items ahead;
    // an item's first pair (nn_b0) is loaded one iteration before its rows are, so no load
    // waits on another inside the loop
    int c_tab = 0, c_b0 = 0, c_n = 0, c_src = 0, n_tab = 0, n_b0 = 0, n_n = 0, n_src = 0, nn_b0 = 0;
    int c_tgt = 0, n_tgt = 0;  // FUSED: target of this thread's pair, and its source's column scale
    float c_sc = 0.f;
    auto load_item = [&](int it, int b0, int& tb, int& n, int& src, int& tgt) {
      tb = item_tab[it];
      n = item_cnt[it];
      src = tc_src[min(b0 + pt, npairs - 1)];
      if constexpr (FUSED) tgt = tc_tgt[min(b0 + pt, npairs - 1)];
    };
    if (i0 < i1) {
      c_b0 = item_begin[i0];
      load_item(i0, c_b0, c_tab, c_n, c_src, c_tgt);
      if constexpr (FUSED) c_sc = escale[c_src];
    }
    if (i0 + 1 < i1) {
      n_b0 = item_begin[i0 + 1];
      load_item(i0 + 1, n_b0, n_tab, n_n, n_src, n_tgt);
    }
    if (i0 + 2 < i1) nn_b0 = item_begin[i0 + 2];
    for (int it = i0; it < i1; ++it) {
      const int li = it - i0, s = li % kStages, b = li % kAcc;
      const bool load_tab = c_tab != last_tab;
      const int tsl = load_tab ? (ntab_loaded % NS) : ((ntab_loaded - 1) % NS);
      if (ok && li >= kStages) ok = mbar_wait(&bar_bfree[s], ((li / kStages) - 1) & 1, wait_tries);
      if (ok && li >= kAcc) ok = mbar_wait(&bar_acce[b], ((li / kAcc) - 1) & 1, wait_tries);
      if (ok && load_tab && ntab_loaded >= NS) ok = mbar_wait(&bar_tfree[tsl], ((ntab_loaded / NS) - 1) & 1, wait_tries);
      if (named_bar_or(1, kProducers, ok ? 0 : 1)) {
        ok = false;
        break;
      }
      if (pt < c_n) {
        s_row[pt] = c_src;
        if constexpr (FUSED) {
          s_tgt[b][pt] = c_tgt;
          s_sc[b][pt] = c_sc;
        }
      }
      const int cur_tab = c_tab, cur_ncol = c_n;
      const int nquad = (cur_ncol + 3) >> 2;
      if (load_tab) ++ntab_loaded;
      last_tab = cur_tab;
      if (pt == 0) {
        s_ncol[b] = cur_ncol;
        s_b0[b] = c_b0;
        s_rt[b] = cur_tab % D::RT;
        s_tsl[s] = tsl;
        s_icol[s] = cur_ncol;
        s_last[s] = (it + 1 >= i1) || (n_tab != cur_tab);
        const uint32_t bytes = (load_tab ? (uint32_t)D::TAB_BYTES : 0u) + (uint32_t)nquad * 4u * 128u * 2u * D::KA;
        mbar_arrive_expect_tx(&bar_full[s], bytes);
      }
      named_bar_sync(1, kProducers);
      armed[s] = li;
      if (pt == 0) {
        mbar_arrive(&bar_meta[b]);
        if (load_tab)
          bulk_copy_g2s(sT + tsl * D::TAB_BYTES, reinterpret_cast<const unsigned char*>(Ttab) + (size_t)cur_tab * D::TAB_BYTES,
                        D::TAB_BYTES, &bar_full[s]);
      }
      // gather4: quad q of rows, part (hi/lo), atom a -> region (part, a), rows 4q..4q+3
      unsigned char* sBs = sB + s * D::B_BYTES;
      for (int g = pt; g < nquad * 2 * D::KA; g += kProducers) {
        const int q = g / (2 * D::KA), pa = g - q * (2 * D::KA);
        const int part = pa / D::KA, a = pa - part * D::KA;
        int y[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) y[i] = s_row[min(4 * q + i, cur_ncol - 1)] * 2 + part;
        tma_gather4(sBs + (part * D::KA + a) * D::REGION + q * 4 * 128, &rows_map, a * 64, y[0], y[1], y[2], y[3], &bar_full[s]);
      }
      if constexpr (FUSED) c_sc = (it + 1 < i1) ? escale[n_src] : 0.f;  // the next item's scale, one iteration ahead
      c_tab = n_tab;
      c_b0 = n_b0;
      c_n = n_n;
      c_src = n_src;
      c_tgt = n_tgt;
      if (it + 2 < i1) {
        n_b0 = nn_b0;
        load_item(it + 2, n_b0, n_tab, n_n, n_src, n_tgt);
        if (it + 3 < i1) nn_b0 = item_begin[it + 3];
      }
    }
    if (!ok) {
      atomicExch(err, 1);
      // the loads already started land in this CTA's shared memory: wait for each stage's last
      // armed item (its transaction bytes complete on full[s]) before the CTA may leave
      if (pt == 0)
#pragma unroll
        for (int q = 0; q < kStages; ++q)
          if (armed[q] >= 0) mbar_wait(&bar_full[q], (armed[q] / kStages) & 1, kDrainTries);
    }
  } else {
    const int quad = warp & 3, half = warp >> 2;  // TMEM lane quad * 32 + lane: output row of the tile
    const uint32_t lane_base = tbase + ((uint32_t)(quad * 32) << 16);
    for (int it = i0; it < i1; ++it) {
      const int li = it - i0, b = li % kAcc;
      bool ok = mbar_wait(&bar_meta[b], (li / kAcc) & 1, wait_tries);
      if (ok) ok = mbar_wait(&bar_accf[b], (li / kAcc) & 1, wait_tries);
      if (!__all_sync(0xffffffffu, ok ? 1 : 0)) {
        if (lane == 0) atomicExch(err, 1);
        break;
      }
      tc_fence_after();
      const int ncol = s_ncol[b];
      const int row0 = s_rt[b] * kRows + quad * 32;  // first output coefficient of this warp's lanes
      float* Yb = Y + (size_t)s_b0[b] * D::KPO + row0 + lane;
      if (row0 < D::KPO) {
        const uint32_t col0 = (uint32_t)(b * kAccCols);
        uint32_t ra[32], rb[32];
        int c0 = half * 32;
        if (c0 < ncol) {
          tmem_ld32_issue(lane_base + col0 + c0, ra);
          tmem_ld32_wait(ra);
        }
        auto store = [&](const uint32_t* r, int cbase) {
          if constexpr (FUSED) {
            // the pair's coefficients, its source's column scale undone, added into the
            // target's FP32 accumulator in L2 (one coalesced 128-byte reduction per warp)
            const bool live = row0 + lane < D::NR;
#pragma unroll
            for (int q = 0; q < 32; ++q) {
              const int j = cbase + q;
              if (j < ncol && live) {
                float* dst = acc + (size_t)s_tgt[b][j] * D::KPO + row0 + lane;
                asm volatile("red.global.add.f32 [%0], %1;" ::"l"(dst), "f"(__uint_as_float(r[q]) * s_sc[b][j]) : "memory");
              }
            }
          } else {
#pragma unroll
            for (int q = 0; q < 32; ++q) {
              const int j = cbase + q;
              if (j < ncol) Yb[(size_t)j * D::KPO] = __uint_as_float(r[q]);
            }
          }
        };
        while (c0 < ncol) {
          const int c1 = c0 + 64;
          if (c1 < ncol) tmem_ld32_issue(lane_base + col0 + c1, rb);
          store(ra, c0);
          if (c1 >= ncol) break;
          tmem_ld32_wait(rb);
          const int c2 = c1 + 64;
          if (c2 < ncol) tmem_ld32_issue(lane_base + col0 + c2, ra);
          store(rb, c1);
          if (c2 >= ncol) break;
          tmem_ld32_wait(ra);
          c0 = c2;
        }
      }
      tc_fence_before();
      mbar_arrive(&bar_acce[b]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tbase, kAcc * kAccCols);
  }
}

// Per target bucket: L[0] = sum of its pair partials (target-major CSR order of the pairs,
// deterministic), each with its source's column scale undone, back to the FP64 complex
// layout [node][density][NC] with the normalisation and a_t^{n+1} undone; L[1] stays zero
// (the combined density carries both; L is cleared before the M2L).  One warp per target:
// lane l sums real coefficients [l*V, l*V+V) of every partial with vector loads (a warp
// reads one whole partial row per instruction), eight partials in flight.
template <int P>
__global__ void k_m2l_tc_reduce(int ntargets, const int* __restrict__ targets, const int* __restrict__ m2l_off,
                                const int* __restrict__ m2l_src, const int* __restrict__ pos, const float* __restrict__ escale,
                                const double* __restrict__ node_dL, const double* __restrict__ alpha, const float* __restrict__ Y,
                                double2* __restrict__ L) {
  pdl_enter();
  using D = TcDims<P>;
  constexpr int NC = ncoef(P), V = D::KPO / 32;
  const int lane = threadIdx.x & 31;
  const int w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int ti = w0; ti < ntargets; ti += nw) {
    const int tgt = targets[ti];
    const int k0 = m2l_off[tgt], k1 = m2l_off[tgt + 1];
    double acc[V];
#pragma unroll
    for (int v = 0; v < V; ++v) acc[v] = 0.0;
    auto load = [&](int r, float out[V]) {
      const float* row = Y + (size_t)r * D::KPO + lane * V;
      if constexpr (V == 4) {
        const float4 q = __ldcs(reinterpret_cast<const float4*>(row));
        out[0] = q.x; out[1] = q.y; out[2] = q.z; out[3] = q.w;
      } else {
#pragma unroll
        for (int h = 0; h < V / 2; ++h) {
          const float2 q = __ldcs(reinterpret_cast<const float2*>(row) + h);
          out[2 * h] = q.x;
          out[2 * h + 1] = q.y;
        }
      }
    };
    // 32 partials at a time: lane l fetches the row position and column scale of partial
    // kb + l (one coalesced load each), then the warp walks them eight rows in flight
    for (int kb = k0; kb < k1; kb += 32) {
      const int nk = min(32, k1 - kb);
      int my_row = 0;
      double my_sc = 0.0;
      if (lane < nk) {
        my_row = pos[kb + lane];
        my_sc = escale[m2l_src[kb + lane]];
      }
      int j = 0;
      for (; j + 8 <= nk; j += 8) {
        float a[8][V];
        double sc[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          load(__shfl_sync(0xffffffffu, my_row, j + u), a[u]);
          sc[u] = __shfl_sync(0xffffffffu, my_sc, j + u);
        }
#pragma unroll
        for (int v = 0; v < V; ++v)
          acc[v] += (((double)a[0][v] * sc[0] + (double)a[1][v] * sc[1]) + ((double)a[2][v] * sc[2] + (double)a[3][v] * sc[3])) +
                    (((double)a[4][v] * sc[4] + (double)a[5][v] * sc[5]) + ((double)a[6][v] * sc[6] + (double)a[7][v] * sc[7]));
      }
      for (; j < nk; ++j) {
        float a0[V];
        load(__shfl_sync(0xffffffffu, my_row, j), a0);
        const double s0 = __shfl_sync(0xffffffffu, my_sc, j);
#pragma unroll
        for (int v = 0; v < V; ++v) acc[v] += (double)a0[v] * s0;
      }
    }
    const double a = node_dL[tgt];
    double* Lr = reinterpret_cast<double*>(L + (size_t)tgt * 2 * NC);
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const int i = lane * V + v;
      if (i < D::NR) {
        int n, m, part;
        decode_real(i, n, m, part);
        double ap = a;
        for (int t = 0; t < n; ++t) ap *= a;
        Lr[2 * cidx(n, m) + part] = acc[v] * alpha[i] / ap;
      }
    }
  }
}

// FUSED path: per target, the FP32 accumulator the contraction reduced into, back to the FP64
// complex layout [node][density][NC] with the normalisation and a_t^{n+1} undone (L[1] stays
// zero), and the accumulator cleared for the next launch.  One warp per target.
template <int P>
__global__ void k_m2l_tc_finalize(int ntargets, const int* __restrict__ targets, const double* __restrict__ node_dL,
                                  const double* __restrict__ alpha, float* __restrict__ acc, double2* __restrict__ L) {
  pdl_enter();
  using D = TcDims<P>;
  constexpr int NC = ncoef(P), V = D::KPO / 32;
  const int lane = threadIdx.x & 31;
  const int w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int ti = w0; ti < ntargets; ti += nw) {
    const int tgt = targets[ti];
    float* row = acc + (size_t)ti * D::KPO + lane * V;
    float v[V];
#pragma unroll
    for (int q = 0; q < V; ++q) {
      v[q] = row[q];
      row[q] = 0.f;
    }
    const double a = node_dL[tgt];
    double* Lr = reinterpret_cast<double*>(L + (size_t)tgt * 2 * NC);
#pragma unroll
    for (int q = 0; q < V; ++q) {
      const int i = lane * V + q;
      if (i < D::NR) {
        int n, m, part;
        decode_real(i, n, m, part);
        double ap = a;
        for (int t = 0; t < n; ++t) ap *= a;
        Lr[2 * cidx(n, m) + part] = (double)v[q] * alpha[i] / ap;
      }
    }
  }
}

template <int P>
int m2l_tc_launch(const MatvecArgs& a, cudaStream_t st, int parts, int nd) {
  using D = TcDims<P>;
  if (a.n_tc_items <= 0) return 0;
  int launches = 0;
  __half* Mt = static_cast<__half*>(a.tc_Mt);
  if (parts & TC_EXPAND) {
    const int ge = (int)std::min<int64_t>(((int64_t)a.n_nodes * 32 + 255) / 256, 148 * 8);
    if (nd == 1)
      launch_pdl(k_tc_expand<P, 1>, ge, 256, 0, st, a.n_nodes, (const double2*)a.M, (const double*)a.node_dL, (const double*)a.tc_alpha,
                 Mt, a.tc_escale);
    else
      launch_pdl(k_tc_expand<P, 2>, ge, 256, 0, st, a.n_nodes, (const double2*)a.M, (const double*)a.node_dL, (const double*)a.tc_alpha,
                 Mt, a.tc_escale);
    ++launches;
  }
  if (parts & TC_CONTRACT) {
    const int grid = a.n_tc_items < a.tc_grid ? a.n_tc_items : a.tc_grid;
    CUtensorMap map;
    std::memcpy(&map, a.tc_rows_map, sizeof(map));
    bool wide = false;
    if constexpr (P <= 10) wide = a.tc_item_pairs > kMaxPairs;
    const bool fused = a.tc_acc != nullptr;
    auto go = [&](auto kern, int smem) {
      launch_pdl(kern, grid, kEpilogue + kProducers + kIssuer, smem, st, map, a.n_tc_items, a.tc_item_tab, a.tc_item_begin, a.tc_item_cnt,
                 a.n_tc_pairs, a.tc_src, static_cast<const __half*>(a.tc_tab), static_cast<const __half*>(a.tc_Mt), a.tc_Y, a.tc_err,
                 a.tc_wait_tries, a.tc_tgt, static_cast<const float*>(a.tc_escale), a.tc_acc);
    };
    if (wide) {
      if constexpr (P <= 10) {
        if (fused)
          go(k_m2l_tc<P, kMaxPairsWide, true>, TcDims<P, kMaxPairsWide>::SMEM);
        else
          go(k_m2l_tc<P, kMaxPairsWide, false>, TcDims<P, kMaxPairsWide>::SMEM);
      }
    } else {
      if (fused)
        go(k_m2l_tc<P, kMaxPairs, true>, D::SMEM);
      else
        go(k_m2l_tc<P, kMaxPairs, false>, D::SMEM);
    }
    ++launches;
  }
  if ((parts & TC_REDUCE) && a.tc_acc) {
    const int gr = (int)std::min<int64_t>(((int64_t)a.n_m2l_targets * 32 + 255) / 256, 148 * 16);
    launch_pdl(k_m2l_tc_finalize<P>, gr, 256, 0, st, a.n_m2l_targets, a.m2l_targets, a.node_dL, a.tc_alpha, a.tc_acc, a.L);
    ++launches;
  } else if (parts & TC_REDUCE) {
    const int gr = (int)std::min<int64_t>(((int64_t)a.n_m2l_targets * 32 + 255) / 256, 148 * 16);
    launch_pdl(k_m2l_tc_reduce<P>, gr, 256, 0, st, a.n_m2l_targets, a.m2l_targets, a.m2l_off, a.m2l_src, a.tc_pos, a.tc_escale, a.node_dL,
                                           a.tc_alpha, a.tc_Y, a.L);
    ++launches;
  }
  return launches;
}

template <int P>
void tc_tables_launch(int ntab, const double* tab, const double* alpha, __half* T, unsigned int* maxbits, cudaStream_t st) {
  cudaFuncSetAttribute(k_m2l_tc<P, kMaxPairs, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcDims<P>::SMEM);
  cudaFuncSetAttribute(k_m2l_tc<P, kMaxPairs, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcDims<P>::SMEM);
  if constexpr (P <= 10) {
    cudaFuncSetAttribute(k_m2l_tc<P, kMaxPairsWide, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcDims<P, kMaxPairsWide>::SMEM);
    cudaFuncSetAttribute(k_m2l_tc<P, kMaxPairsWide, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, TcDims<P, kMaxPairsWide>::SMEM);
  }
  if (ntab > 0) k_tc_tables<P><<<ntab * TcDims<P>::RT, 128, 0, st>>>(ntab, tab, alpha, T, maxbits);
}

}  // namespace

int tc_supported(int p) { return p >= 1 && p <= 12; }
uint32_t tc_default_wait_tries() { return kWaitTries; }
int tc_kp(int p) { return ((p + 1) * (p + 1) + 63) / 64 * 64; }

size_t tc_rows_map_bytes() { return sizeof(CUtensorMap); }

// Tensor map over the multipole rows Mt viewed as [rows = 2 (n_nodes + 1)][tc_kp halves]:
// boxes of 64 halves x 1 row, 128-byte swizzle, for tile::gather4.
int tc_make_rows_map(void* map_out, void* Mt, int nrows, int p) {
  using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                                const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static const EncodeFn encode = [] {  // thread-safe one-time lookup
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
      return static_cast<EncodeFn>(nullptr);
    return reinterpret_cast<EncodeFn>(fn);
  }();
  if (!encode) return -1;
  const int kp = tc_kp(p);
  const cuuint64_t dims[2] = {(cuuint64_t)kp, (cuuint64_t)nrows};
  const cuuint64_t strides[1] = {(cuuint64_t)kp * 2};
  const cuuint32_t box[2] = {64, 1};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = encode(static_cast<CUtensorMap*>(map_out), CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, Mt, dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -1;
}
size_t tc_table_bytes(int p) { return (size_t)2 * kRows * tc_kp(p) * 2; }
int tc_row_tiles(int p) { return ((p + 1) * (p + 1) + kRows - 1) / kRows; }
int tc_kpo(int p) { return tc_kp(p); }
int tc_max_pairs(int p) { return p <= 10 ? kMaxPairsWide : kMaxPairs; }

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
    BEMB200_CASE(11) BEMB200_CASE(12)
#undef BEMB200_CASE
    default: break;
  }
}

int launch_m2l_tc(int p, const MatvecArgs& a, cudaStream_t st, int parts, int nd) {
  switch (p) {
#define BEMB200_CASE(PP) \
  case PP:               \
    return m2l_tc_launch<PP>(a, st, parts, nd);
    BEMB200_CASE(1) BEMB200_CASE(2) BEMB200_CASE(3) BEMB200_CASE(4) BEMB200_CASE(5)
    BEMB200_CASE(6) BEMB200_CASE(7) BEMB200_CASE(8) BEMB200_CASE(9) BEMB200_CASE(10)
    BEMB200_CASE(11) BEMB200_CASE(12)
#undef BEMB200_CASE
    default: break;
  }
  return 0;
}

}  // namespace bemb200
