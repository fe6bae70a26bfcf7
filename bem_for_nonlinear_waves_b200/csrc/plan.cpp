// Host-side set-up plan (see plan.hpp).  Compiled with g++ -O2 -march=x86-64-v3,
// no fast-math: the element positions and bucket bounds must round like the
// reference's so that the octree is the same tree.
#include "plan.hpp"

#include "tree_dev.hpp"

#include <algorithm>
#include <parallel/algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <chrono>
#include <numeric>
#include <omp.h>

namespace bemb200 {
namespace {

using V3 = std::array<double, 3>;

// std::hypot(x, y, z) as libstdc++ implements it (Norm(Tddd),
// lib/include/basic_arithmetic_array_operations.hpp:860).
inline double hypot3(double x, double y, double z) {
  x = std::abs(x);
  y = std::abs(y);
  z = std::abs(z);
  if (double a = x < y ? y < z ? z : y : x < z ? z : x)
    return a * std::sqrt((x / a) * (x / a) + (y / a) * (y / a) + (z / a) * (z / a));
  return 0.0;
}
inline V3 sub(const V3& a, const V3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
inline double nrm(const V3& a) { return hypot3(a[0], a[1], a[2]); }
// Dot(weights[3], X[3]): fma into a zero accumulator per component (basic_arithmetic_array_operations.hpp:639-657)
inline V3 bary(const double w0, const double w1, const double w2, const V3& a, const V3& b, const V3& c) {
  V3 r{0, 0, 0};
  for (int j = 0; j < 3; ++j) r[j] = std::fma(w0, a[j], r[j]);
  for (int j = 0; j < 3; ++j) r[j] = std::fma(w1, b[j], r[j]);
  for (int j = 0; j < 3; ++j) r[j] = std::fma(w2, c[j], r[j]);
  return r;
}
// Double-double arithmetic (Dekker's and Knuth's error-free transformations, ~106 significant
// bits) in place of the reference's binary128 for the element normals and Jacobians: each
// result is rounded to double once, as the reference's is, and agrees with it except where the
// exact value lies within ~2^-104 of a rounding boundary.
struct DD {
  double hi, lo;
};
inline DD two_sum(double a, double b) {
  const double s = a + b, bb = s - a;
  return {s, (a - (s - bb)) + (b - bb)};
}
inline DD quick_two_sum(double a, double b) {
  const double s = a + b;
  return {s, b - (s - a)};
}
inline DD two_prod(double a, double b) {
  const double p = a * b;
  return {p, std::fma(a, b, -p)};
}
inline DD dd_add(DD x, DD y) {
  DD s = two_sum(x.hi, y.hi);
  const DD t = two_sum(x.lo, y.lo);
  s.lo += t.hi;
  s = quick_two_sum(s.hi, s.lo);
  s.lo += t.lo;
  return quick_two_sum(s.hi, s.lo);
}
inline DD dd_neg(DD x) { return {-x.hi, -x.lo}; }
inline DD dd_mul(DD x, DD y) {
  DD p = two_prod(x.hi, y.hi);
  p.lo += x.hi * y.lo + x.lo * y.hi;
  return quick_two_sum(p.hi, p.lo);
}
inline DD dd_mul_d(DD x, double y) {
  DD p = two_prod(x.hi, y);
  p.lo += x.lo * y;
  return quick_two_sum(p.hi, p.lo);
}
// 1 / s for a double s: q + (1 - q s) / s
inline DD dd_recip(double s) {
  const double q = 1.0 / s;
  return quick_two_sum(q, std::fma(-q, s, 1.0) / s);
}
// Cross(), products exact and differences to ~106 bits, rounded once
// (basic_arithmetic_array_operations.hpp:906-920)
inline V3 cross_dd(const V3& A, const V3& B) {
  return {dd_add(two_prod(A[1], B[2]), dd_neg(two_prod(A[2], B[1]))).hi, dd_add(two_prod(A[2], B[0]), dd_neg(two_prod(A[0], B[2]))).hi,
          dd_add(two_prod(A[0], B[1]), dd_neg(two_prod(A[1], B[0]))).hi};
}
// TriangleNormalHP (…:961-986) in double-double: edge vectors exact, the cross product and its
// squared norm to ~106 bits, 1/sqrt of the norm rounded to double as the reference does
inline V3 normal_dd(const V3& a, const V3& b, const V3& c) {
  const DD bax = two_sum(b[0], -a[0]), bay = two_sum(b[1], -a[1]), baz = two_sum(b[2], -a[2]);
  const DD cax = two_sum(c[0], -a[0]), cay = two_sum(c[1], -a[1]), caz = two_sum(c[2], -a[2]);
  const DD nx = dd_add(dd_mul(bay, caz), dd_neg(dd_mul(baz, cay)));
  const DD ny = dd_add(dd_mul(baz, cax), dd_neg(dd_mul(bax, caz)));
  const DD nz = dd_add(dd_mul(bax, cay), dd_neg(dd_mul(bay, cax)));
  const DD n2 = dd_add(dd_add(dd_mul(nx, nx), dd_mul(ny, ny)), dd_mul(nz, nz));
  if (n2.hi == 0.0) return {0, 0, 0};
  const DD inv = dd_recip(std::sqrt(n2.hi));
  return {dd_mul(nx, inv).hi, dd_mul(ny, inv).hi, dd_mul(nz, inv).hi};
}
inline V3 unit(V3 a) {  // Normalize (basic_arithmetic_array_operations.hpp:837-850)
  double n = 0.;
  for (double v : a) n = std::fma(v, v, n);
  if (n == 0.) return a;
  n = std::sqrt(n);
  for (auto& v : a) v /= n;
  return a;
}
inline double dotfma(const V3& a, const V3& b) { return std::fma(a[0], b[0], std::fma(a[1], b[1], a[2] * b[2])); }

// Dunavant degree-4 rule (lib/include/dunavant_rules.hpp:36-42): barycentrics + weight
const double kDv[6][4] = {{0.816847572980459, 0.091576213509771, 0.091576213509771, 0.054975871827661},
                          {0.091576213509771, 0.816847572980459, 0.091576213509771, 0.054975871827661},
                          {0.091576213509771, 0.091576213509771, 0.816847572980459, 0.054975871827661},
                          {0.108103018168070, 0.445948490915965, 0.445948490915965, 0.111690794839006},
                          {0.445948490915965, 0.108103018168070, 0.445948490915965, 0.111690794839006},
                          {0.445948490915965, 0.445948490915965, 0.108103018168070, 0.111690794839006}};

struct Bucket {
  double lo[3], hi[3], X[3];
  double dL, inv_dL, xmin[3];
  int size[3];
  int level = 0, parent = -1;
  std::vector<int> kids;                  // created children, cell order
  std::vector<std::vector<int>> cell;     // elements per cell
  std::vector<int> data;                  // data1D
  std::vector<int> kid_of_cell;
  double off = 0.0;
  std::vector<int> near, m2l;
};

void bucket_init(Bucket& b, const double lo[3], const double hi[3], double dL) {
  for (int a = 0; a < 3; ++a) {
    b.lo[a] = lo[a];
    b.hi[a] = hi[a];
    b.X[a] = (lo[a] + hi[a]) / 2.;  // Mean(Transpose(bounds))
    b.xmin[a] = lo[a];
  }
  b.dL = dL;
  b.inv_dL = 1.0 / dL;
  for (int a = 0; a < 3; ++a) {
    double s = std::ceil((b.hi[a] - b.lo[a]) / dL);  // calculate_size
    if (s <= 0.) s = 1.;
    b.size[a] = (int)s;
  }
  b.cell.assign(b.size[0] * b.size[1] * b.size[2], {});
  b.kid_of_cell.assign(b.size[0] * b.size[1] * b.size[2], -1);
}

inline void cell_index(const Bucket& b, const double* x, int ijk[3]) {
  for (int a = 0; a < 3; ++a) ijk[a] = (int)std::floor((x[a] - b.xmin[a]) * b.inv_dL);
}
inline bool inside(const Bucket& b, const double* x) {
  int ijk[3];
  cell_index(b, x, ijk);
  for (int a = 0; a < 3; ++a)
    if (ijk[a] < 0 || ijk[a] >= b.size[a]) return false;
  return true;
}
inline int cell_of(const Bucket& b, const double* x) {
  int ijk[3];
  cell_index(b, x, ijk);
  for (int a = 0; a < 3; ++a) ijk[a] = std::clamp(ijk[a], 0, b.size[a] - 1);
  return (ijk[0] * b.size[1] + ijk[1]) * b.size[2] + ijk[2];
}

struct TreeBuilder {
  const PlanOptions& opt;
  const std::vector<V3>& pole;
  std::vector<Bucket> B;
  int drops = 0;
  explicit TreeBuilder(const PlanOptions& o, const std::vector<V3>& p) : opt(o), pole(p) {}

  bool add(int bi, int e) {  // Buckets::add: InsideQ without clamp, then the clamped cell
    Bucket& b = B[bi];
    if (!inside(b, pole[e].data())) return false;
    b.cell[cell_of(b, pole[e].data())].push_back(e);
    b.data.push_back(e);
    return true;
  }
  // Buckets::generateTree with newChild (lib_spatial_partitioning.hpp:1078-1111)
  void grow(int bi) {
    const bool cond = !B[bi].data.empty() && (int)B[bi].data.size() > opt.leaf_max && B[bi].level < opt.max_level;
    if (!cond) return;
    const int nc = B[bi].size[0] * B[bi].size[1] * B[bi].size[2];
    for (int c = 0; c < nc; ++c) {
      if (B[bi].cell[c].empty()) continue;
      const int i = c / (B[bi].size[1] * B[bi].size[2]);
      const int j = (c / B[bi].size[2]) % B[bi].size[1];
      const int k = c % B[bi].size[2];
      double lo[3], hi[3];
      const int ijk[3] = {i, j, k};
      for (int a = 0; a < 3; ++a) {  // getBounds({i,j,k})
        lo[a] = B[bi].dL * ijk[a] + B[bi].xmin[a];
        hi[a] = B[bi].dL * (ijk[a] + 1) + B[bi].xmin[a];
      }
      const double dLc = B[bi].dL * (0.5 + 1e-13);
      Bucket child;
      bucket_init(child, lo, hi, dLc);
      child.level = B[bi].level + 1;
      child.parent = bi;
      B.push_back(std::move(child));
      const int ci = (int)B.size() - 1;
      B[bi].kids.push_back(ci);
      B[bi].kid_of_cell[c] = ci;
      for (int e : B[bi].cell[c])
        if (!add(ci, e)) ++drops;
      grow(ci);
    }
  }
};

// The same growth with the element classification on the device (tree.cu), level by level:
// buckets are created per level (breadth first) and renumbered depth first at the end, which
// is the order grow() creates them in.  The root holds its elements already.  Returns false
// (tree left as the root alone) if a device step fails or a bucket is not 2x2x2 cells.
bool grow_on_device(TreeBuilder& T, DeviceTree* dt, int nf, const std::vector<V3>& pole) {
  std::vector<Bucket>& B = T.B;
  const PlanOptions& opt = T.opt;
  if (B.size() != 1) return false;
  std::vector<double> P3(3 * (size_t)nf);
  for (int f = 0; f < nf; ++f)
    for (int a = 0; a < 3; ++a) P3[3 * (size_t)f + a] = pole[f][a];
  const std::vector<int> root_data = B[0].data;
  if (!dtree_begin(dt, nf, P3.data(), (int)root_data.size(), root_data.data(), opt.max_level)) return false;
  // breadth-first buckets: index 0 = root; per bucket its segment in its level's array
  std::vector<Bucket> Q;
  Q.push_back(B[0]);
  std::vector<int> seg_b{0}, seg_e{(int)root_data.size()}, level_of{0};
  std::vector<size_t> level_base{0};
  std::vector<int> cur{0};
  size_t base = 0, cur_n = root_data.size();
  int drops = 0;
  while (!cur.empty()) {
    std::vector<int> split;
    for (int q : cur) {
      const int n = seg_e[q] - seg_b[q];
      if (n > 0 && n > opt.leaf_max && Q[q].level < opt.max_level) split.push_back(q);
    }
    if (split.empty()) break;
    const int ns = (int)split.size();
    std::vector<int> sb(ns), se(ns), ca(8 * (size_t)ns), cp(8 * (size_t)ns);
    std::vector<double> geo(63 * (size_t)ns);
    std::vector<Bucket> kid(8 * (size_t)ns);
    for (int k = 0; k < ns; ++k) {
      const Bucket& b = Q[split[k]];
      if (b.size[0] != 2 || b.size[1] != 2 || b.size[2] != 2) return false;
      sb[k] = seg_b[split[k]];
      se[k] = seg_e[split[k]];
      double* g = &geo[63 * (size_t)k];
      for (int a = 0; a < 3; ++a) {
        g[a] = b.xmin[a];
        g[4 + a] = b.size[a];
      }
      g[3] = b.inv_dL;
      for (int c = 0; c < 8; ++c) {  // the child grow() would create for cell c
        const int i = c / (b.size[1] * b.size[2]), j = (c / b.size[2]) % b.size[1], kk = c % b.size[2];
        const int ijk[3] = {i, j, kk};
        double lo[3], hi[3];
        for (int a = 0; a < 3; ++a) {
          lo[a] = b.dL * ijk[a] + b.xmin[a];
          hi[a] = b.dL * (ijk[a] + 1) + b.xmin[a];
        }
        Bucket& ch = kid[8 * (size_t)k + c];
        bucket_init(ch, lo, hi, b.dL * (0.5 + 1e-13));
        double* gc = g + 7 * (1 + c);
        for (int a = 0; a < 3; ++a) {
          gc[a] = ch.xmin[a];
          gc[4 + a] = ch.size[a];
        }
        gc[3] = ch.inv_dL;
      }
    }
    if (!dtree_count(dt, ns, sb.data(), se.data(), geo.data(), ca.data(), cp.data())) return false;
    std::vector<int> off(8 * (size_t)ns, 0);
    int total = 0;
    std::vector<int> next;
    for (int k = 0; k < ns; ++k)
      for (int c = 0; c < 8; ++c) {
        const size_t kc = 8 * (size_t)k + c;
        off[kc] = total;
        if (ca[kc] == 0) continue;
        Bucket ch = std::move(kid[kc]);
        ch.level = Q[split[k]].level + 1;
        ch.parent = split[k];
        const int qi = (int)Q.size();
        Q.push_back(std::move(ch));
        Q[split[k]].kids.push_back(qi);
        Q[split[k]].kid_of_cell[c] = qi;
        seg_b.push_back(total);
        seg_e.push_back(total + cp[kc]);
        level_of.push_back(Q[qi].level);
        next.push_back(qi);
        drops += ca[kc] - cp[kc];
        total += cp[kc];
      }
    if (!dtree_scatter(dt, ns, off.data(), total)) return false;
    base += cur_n;
    cur_n = (size_t)total;
    level_base.push_back(base);
    cur.swap(next);
  }
  std::vector<int> all(base + cur_n);
  if (!dtree_download(dt, all.data(), all.size())) return false;
  for (size_t q = 1; q < Q.size(); ++q) {
    const size_t lb = level_base[level_of[q]];
    Q[q].data.assign(all.begin() + lb + seg_b[q], all.begin() + lb + seg_e[q]);
  }
  // depth-first renumbering (grow() creates a bucket, then its subtree, then its next sibling)
  std::vector<int> id(Q.size(), -1), order;
  order.reserve(Q.size());
  std::vector<int> stack{0};
  while (!stack.empty()) {
    const int q = stack.back();
    stack.pop_back();
    id[q] = (int)order.size();
    order.push_back(q);
    for (auto it = Q[q].kids.rbegin(); it != Q[q].kids.rend(); ++it) stack.push_back(*it);
  }
  B.clear();
  B.reserve(Q.size());
  for (int q : order) {
    Bucket b = std::move(Q[q]);
    if (b.parent >= 0) b.parent = id[b.parent];
    for (int& k : b.kids) k = id[k];
    for (int& k : b.kid_of_cell)
      if (k >= 0) k = id[k];
    B.push_back(std::move(b));
  }
  T.drops = drops;
  return true;
}

// Sorts the packed M2L pair keys (offset key << 33 | level << 29 | slot; bit 63 for a pair off
// the lattice).  The slots are unique and the keys arrive in slot order, so the sorted order is
// a stable sort by the part above the slot: a counting sort over a dense table of lattice
// offsets |r| <= 31 and levels, with the off-lattice pairs last.  Falls back to a comparison
// sort for larger offsets.
// The positions i in [0, n) where head(i) holds, in increasing order, found in parallel
// (per-thread counts, an exclusive scan, then per-thread writes).
template <typename F>
static void parallel_heads(int64_t n, F head, std::vector<int64_t>& out) {
  const int nt = std::max(1, omp_get_max_threads());
  std::vector<int64_t> cnt(nt + 1, 0);
#pragma omp parallel num_threads(nt)
  {
    const int t = omp_get_thread_num(), T = omp_get_num_threads();
    const int64_t lo = n * t / T, hi = n * (t + 1) / T;
    int64_t c = 0;
    for (int64_t i = lo; i < hi; ++i) c += head(i) ? 1 : 0;
    cnt[t + 1] = c;
#pragma omp barrier
#pragma omp single
    {
      for (int k = 0; k < T; ++k) cnt[k + 1] += cnt[k];
      out.resize(cnt[T]);
    }
    int64_t w = cnt[t];
    for (int64_t i = lo; i < hi; ++i)
      if (head(i)) out[w++] = i;
  }
}

// target bucket of every M2L pair slot (the target-major CSR m2l_off / m2l_src)
static void pair_targets(const Plan& P, std::vector<int>& pair_tgt) {
  const int nb = (int)P.nodes.size();
  pair_tgt.resize(P.m2l_off.empty() ? 0 : P.m2l_off[nb]);
#pragma omp parallel for schedule(static)
  for (int t = 0; t < nb; ++t)
    for (int k = P.m2l_off[t]; k < P.m2l_off[t + 1]; ++k) pair_tgt[k] = t;
}

void sort_pair_keys(std::vector<uint64_t>& keyed) {
  constexpr int R = 31, W = 2 * R + 1;
  constexpr int64_t kOff = (int64_t)W * W * W * 16;  // dense bucket index; kOff = off the lattice
  const int64_t n = (int64_t)keyed.size();
  std::vector<int32_t> bucket(n);
  bool dense = true;
#pragma omp parallel for schedule(static) reduction(&& : dense)
  for (int64_t k = 0; k < n; ++k) {
    const uint64_t v = keyed[k];
    if (v >> 63) {
      bucket[k] = (int32_t)kOff;
      continue;
    }
    const int lev = (int)((v >> 29) & 15);
    const uint64_t rk = v >> 33;
    const int r0 = (int)((rk >> 20) & 1023) - 512, r1 = (int)((rk >> 10) & 1023) - 512, r2 = (int)(rk & 1023) - 512;
    if (std::abs(r0) > R || std::abs(r1) > R || std::abs(r2) > R) {
      dense = false;
      bucket[k] = 0;
      continue;
    }
    bucket[k] = (int32_t)((((int64_t)(r0 + R) * W + (r1 + R)) * W + (r2 + R)) * 16 + lev);
  }
  if (!dense || n < 4096) {
    __gnu_parallel::sort(keyed.begin(), keyed.end());
    return;
  }
  // ranks of the used buckets, in bucket order: a bitmap of the used ones and per-word prefix
  // counts (rank = used buckets before b)
  const int64_t nw = kOff / 64 + 1;
  std::vector<uint64_t> used(nw, 0);
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < n; ++k) {
    const int64_t b = bucket[k];
    const uint64_t bit = uint64_t(1) << (b & 63);
    if (!(used[b >> 6] & bit)) __atomic_fetch_or(&used[b >> 6], bit, __ATOMIC_RELAXED);
  }
  std::vector<int32_t> wpre(nw + 1, 0);
  for (int64_t w = 0; w < nw; ++w) wpre[w + 1] = wpre[w] + __builtin_popcountll(used[w]);
  const int32_t nr = wpre[nw];
  auto rank_of = [&](int64_t b) {
    const uint64_t below = used[b >> 6] & ((uint64_t(1) << (b & 63)) - 1);
    return wpre[b >> 6] + __builtin_popcountll(below);
  };
  std::vector<int32_t> rank(n);
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < n; ++k) rank[k] = rank_of(bucket[k]);
  // stable scatter: histograms over contiguous slot ranges (slices), prefix in (rank, slice) order
  const int ns = std::max(1, std::min(omp_get_max_threads(), 64));
  std::vector<int64_t> hist((size_t)ns * nr, 0);
#pragma omp parallel for schedule(static)
  for (int t = 0; t < ns; ++t) {
    int64_t* h = &hist[(size_t)t * nr];
    for (int64_t k = n * t / ns, e = n * (t + 1) / ns; k < e; ++k) ++h[rank[k]];
  }
  int64_t run = 0;
  for (int32_t r = 0; r < nr; ++r)
    for (int t = 0; t < ns; ++t) {
      const int64_t c = hist[(size_t)t * nr + r];
      hist[(size_t)t * nr + r] = run;
      run += c;
    }
  std::vector<uint64_t> out(n);
#pragma omp parallel for schedule(static)
  for (int t = 0; t < ns; ++t) {
    int64_t* h = &hist[(size_t)t * nr];
    for (int64_t k = n * t / ns, e = n * (t + 1) / ns; k < e; ++k) out[h[rank[k]]++] = keyed[k];
  }
  keyed.swap(out);
}

bool is_far(const PlanOptions& o, const Bucket& A, const Bucket& Bk) {  // moments.hpp:950-956
  const double eff = std::max(A.dL + 2.0 * A.off, Bk.dL + 2.0 * Bk.off);
  const V3 d{Bk.X[0] - A.X[0], Bk.X[1] - A.X[1], Bk.X[2] - A.X[2]};
  // clear-cut cases by squared distance; only pairs within 1e-9 of the threshold go
  // through the reference's exact expression (identical decisions, fewer hypot calls)
  const double thr = std::sqrt(3.0) * eff / o.theta;
  const double d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  if (d2 > thr * thr * (1.0 + 1e-9)) return true;
  if (d2 < thr * thr * (1.0 - 1e-9)) return false;
  return o.theta > std::sqrt(3.0) * eff / nrm(d);
}

void lists(const PlanOptions& o, std::vector<Bucket>& B, int a, int b) {  // moments.hpp:967-979
  if (is_far(o, B[a], B[b])) return;
  if (a != b) B[a].near.push_back(b);
  for (int ac : B[a].kids)
    for (int bc : B[b].kids) {
      if (ac != bc && is_far(o, B[ac], B[bc]))
        B[ac].m2l.push_back(bc);
      else
        lists(o, B, ac, bc);
    }
}

}  // namespace

void parallel_copy(void* dst, const void* src, size_t bytes) {
  constexpr size_t kPiece = size_t(1) << 20;
  if (bytes < 4 * kPiece) {
    std::memcpy(dst, src, bytes);
    return;
  }
  const int64_t n = (int64_t)((bytes + kPiece - 1) / kPiece);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const size_t a = (size_t)i * kPiece, b = std::min(bytes, a + kPiece);
    std::memcpy(static_cast<char*>(dst) + a, static_cast<const char*>(src) + a, b - a);
  }
}

int build_dofs(int np, const double* X, int nf, const int32_t* tri, const uint8_t* fdir, int32_t* dof_point, int32_t* dof_face,
               int32_t* dof_kind, int32_t* face_dof, uint8_t* point_flags) {
  if (np <= 0 || nf <= 0 || !X || !tri || !fdir) return -1;
  std::vector<int> cnt(np + 1, 0);
  for (int f = 0; f < nf; ++f)
    for (int a = 0; a < 3; ++a) {
      int p = tri[3 * f + a];
      if (p < 0 || p >= np) return -1;
      ++cnt[p + 1];
    }
  for (int p = 0; p < np; ++p) cnt[p + 1] += cnt[p];
  std::vector<int> pf(cnt[np]);
  {
    std::vector<int> fill(cnt.begin(), cnt.end() - 1);
    for (int f = 0; f < nf; ++f)
      for (int a = 0; a < 3; ++a) pf[fill[tri[3 * f + a]]++] = f;  // ascending face order per point
  }
  std::vector<V3> fn(nf);
  std::vector<double> fa(nf);
  auto P = [&](int i) { return V3{X[3 * i], X[3 * i + 1], X[3 * i + 2]}; };
  for (int f = 0; f < nf; ++f) {
    V3 a = P(tri[3 * f]), b = P(tri[3 * f + 1]), c = P(tri[3 * f + 2]);
    fn[f] = normal_dd(a, b, c);
    fa[f] = 0.5 * nrm(cross_dd(sub(b, a), sub(c, a)));
  }
  std::vector<uint8_t> neu(np, 0), dir(np, 0), cor(np, 0), mult(np, 0);
  const double lim = 20. * M_PI / 180.;  // setIsMultipleNode (BEM_setBoundaryTypes.hpp:434-441)
  for (int p = 0; p < np; ++p) {
    if (cnt[p] == cnt[p + 1]) continue;
    bool alln = true, alld = true;
    for (int k = cnt[p]; k < cnt[p + 1]; ++k) {
      alln = alln && !fdir[pf[k]];
      alld = alld && fdir[pf[k]];
    }
    neu[p] = alln;
    dir[p] = alld;
    cor[p] = !alln && !alld;
    if (cor[p]) {
      mult[p] = 1;
      continue;
    }
    V3 n{0, 0, 0};
    for (int k = cnt[p]; k < cnt[p + 1]; ++k)
      for (int a = 0; a < 3; ++a) n[a] += fa[pf[k]] * fn[pf[k]][a];
    n = unit(n);
    for (int k = cnt[p]; k < cnt[p + 1]; ++k) {
      const V3& m = fn[pf[k]];
      if (!(dotfma(n, m) > std::cos(lim) * std::sqrt(dotfma(n, n)) * std::sqrt(dotfma(m, m)))) mult[p] = 1;
    }
  }
  auto isNeu = [&](int p, int f) {  // isNeumannID_BEM (BEM_setBoundaryTypes.hpp:29-37)
    if (neu[p] || cor[p]) return mult[p] ? (f >= 0 && !fdir[f]) : (f < 0);
    return false;
  };
  auto isDir = [&](int p, int f) { return (dir[p] || cor[p]) && f < 0; };
  int n = 0;
  std::vector<int> null_dof(np, -1);
  std::vector<std::vector<std::pair<int, int>>> fkeys(np);
  for (int p = 0; p < np; ++p) {
    if (cnt[p] == cnt[p + 1]) continue;
    if (isNeu(p, -1) || isDir(p, -1)) {
      dof_point[n] = p;
      dof_face[n] = -1;
      dof_kind[n] = isDir(p, -1) ? 0 : 1;
      null_dof[p] = n++;
    }
    for (int k = cnt[p]; k < cnt[p + 1]; ++k) {
      const int f = pf[k];
      if (isNeu(p, f) || isDir(p, f)) {
        dof_point[n] = p;
        dof_face[n] = f;
        dof_kind[n] = cor[p] ? 2 : 1;
        fkeys[p].push_back({f, n});
        ++n;
      }
    }
  }
  for (int f = 0; f < nf; ++f)
    for (int a = 0; a < 3; ++a) {  // pf2Index (BEM_setBoundaryTypes.hpp:83-95)
      const int p = tri[3 * f + a];
      int d = -1;
      if (!mult[p] || fdir[f])
        d = null_dof[p];
      else
        for (auto& kv : fkeys[p])
          if (kv.first == f) d = kv.second;
      if (d < 0) return -1;
      face_dof[3 * f + a] = d;
    }
  if (point_flags)
    for (int p = 0; p < np; ++p) point_flags[p] = (neu[p] ? 1 : 0) | (dir[p] ? 2 : 0) | (cor[p] ? 4 : 0) | (mult[p] ? 8 : 0);
  return n;
}

// the tree, element order and interaction lists a refresh must reproduce to take over the
// previous plan's M2L structure
static bool same_tree(const Plan& a, const Plan& b) {
  if (a.nodes.size() != b.nodes.size()) return false;
  for (size_t i = 0; i < a.nodes.size(); ++i) {
    const Plan::Node &x = a.nodes[i], &y = b.nodes[i];
    if (x.level != y.level || x.parent != y.parent || x.child_begin != y.child_begin || x.child_end != y.child_end || x.fb != y.fb ||
        x.fe != y.fe || x.n_data != y.n_data)
      return false;
  }
  return a.node_children == b.node_children && a.face_of_pos == b.face_of_pos && a.m2l_off == b.m2l_off && a.m2l_src == b.m2l_src &&
         a.near_off == b.near_off && a.near_nodes == b.near_nodes && a.e_vtx == b.e_vtx && a.e_dof == b.e_dof &&
         a.leaves == b.leaves && a.level_nodes == b.level_nodes;
}

// M2L grouped by lattice offset r = (X_t - X_s) / dL_t and level; groups ordered by key,
// pairs within a group in slot order.  One parallel sort of packed 64-bit values
// (offset key | level | slot; a pair off the lattice gets a value of its own, sorted last)
// serves both the FP64 groups (level, r) and the tensor-core tables (r on every level).  Fills
// the groups, their chunks of <= 8 pairs and the targets with at least one pair.
bool build_m2l_groups(Plan& P) {
  const int nb = (int)P.nodes.size();
  const int64_t npair = P.m2l_pairs;
  if (npair >= (int64_t(1) << 29)) {
    P.error = "too many M2L pairs";
    return false;
  }
  std::vector<int>& pair_tgt = P.scratch_pair_tgt;
  pair_targets(P, pair_tgt);
  std::vector<uint64_t>& keyed = P.m2l_key_sorted;
  keyed.resize(npair);
  std::vector<double> bx(4 * (size_t)nb);  // bucket centre and size, packed (the pair loop reads them at random)
  for (int i = 0; i < nb; ++i) {
    for (int a = 0; a < 3; ++a) bx[4 * (size_t)i + a] = P.nodes[i].X[a];
    bx[4 * (size_t)i + 3] = P.nodes[i].dL;
  }
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < npair; ++k) {
    const int t = pair_tgt[k], s = P.m2l_src[k];
    const double* xt = &bx[4 * (size_t)t];
    const double* xs = &bx[4 * (size_t)s];
    bool lattice = std::abs(xs[3] - xt[3]) <= 1e-12 * xt[3];
    long long r[3];
    for (int a = 0; a < 3; ++a) {
      const double q = (xt[a] - xs[a]) / xt[3];
      r[a] = std::llround(q);
      if (std::abs(q - (double)r[a]) > 1e-9 || std::abs(r[a]) > 500) lattice = false;
    }
    const uint64_t rkey = (uint64_t)(((r[0] + 512) << 20) | ((r[1] + 512) << 10) | (r[2] + 512));
    keyed[k] = lattice ? ((((rkey << 4) | (uint64_t)P.nodes[t].level) << 29) | (uint64_t)k) : ((uint64_t(1) << 63) | (uint64_t)k);
  }
  sort_pair_keys(keyed);
  // groups: runs of one (offset, level) key; a pair off the lattice is a group of its own
  const uint64_t kmask = (uint64_t(1) << 29) - 1;
  std::vector<int64_t> gs;
  parallel_heads(
      npair, [&](int64_t i) { return i == 0 || (keyed[i] >> 63) || (keyed[i - 1] >> 63) || (keyed[i] >> 29) != (keyed[i - 1] >> 29); },
      gs);
  const int ng = (int)gs.size();
  P.grp_off.resize(ng + 1);
  P.grp_vec.resize(3 * (size_t)ng);
  P.grp_pair.resize(npair);
  std::vector<int> nch(ng + 1, 0);  // chunks of <= 8 pairs per group, then their offsets
#pragma omp parallel for schedule(static)
  for (int g = 0; g < ng; ++g) {
    const int64_t b = gs[g], e = g + 1 < ng ? gs[g + 1] : npair;
    P.grp_off[g] = (int)b;
    const int k0 = (int)(keyed[b] & kmask);
    const int t0 = pair_tgt[k0], s0 = P.m2l_src[k0];
    for (int a = 0; a < 3; ++a) P.grp_vec[3 * (size_t)g + a] = P.nodes[t0].X[a] - P.nodes[s0].X[a];
    nch[g + 1] = (int)((e - b + 7) / 8);
  }
  P.grp_off[ng] = (int)npair;
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < npair; ++j) P.grp_pair[j] = (int)(keyed[j] & kmask);
  for (int g = 0; g < ng; ++g) nch[g + 1] += nch[g];
  P.chunk_grp.resize(nch[ng]);
  P.chunk_begin.resize(nch[ng]);
  P.chunk_cnt.resize(nch[ng]);
#pragma omp parallel for schedule(static)
  for (int g = 0; g < ng; ++g)
    for (int c = nch[g], b = P.grp_off[g]; c < nch[g + 1]; ++c, b += 8) {
      P.chunk_grp[c] = g;
      P.chunk_begin[c] = b;
      P.chunk_cnt[c] = std::min(8, P.grp_off[g + 1] - b);
    }
  P.m2l_targets.clear();
  for (int t = 0; t < nb; ++t)
    if (P.m2l_off[t + 1] > P.m2l_off[t]) P.m2l_targets.push_back(t);

  return true;
}

bool build_plan(Plan& P, const PlanOptions& opt, int np, const double* X, int nf, const int32_t* tri, const uint8_t* fdir, int ndof,
                const int32_t* dof_point, const int32_t* dof_face, const int32_t* dof_kind, const int32_t* face_dof, Plan* prev,
                bool defer_m2l_groups) {
  {  // start from an empty plan that keeps the capacity of P's arrays: a plan of similar size
     // then reuses memory whose pages are already mapped
    Plan fresh;
#define BEMB200_KEEP(v) \
  fresh.v.swap(P.v);    \
  fresh.v.clear();
    BEMB200_PLAN_ARRAYS(BEMB200_KEEP)
#undef BEMB200_KEEP
    fresh.src_scratch = std::move(P.src_scratch);  // kept with their sizes
    // per-element source arrays: resized and overwritten in full, so kept with their sizes too
    fresh.e_q.swap(P.e_q);
    fresh.e_W.swap(P.e_W);
    fresh.e_n.swap(P.e_n);
    fresh.e_near.swap(P.e_near);
    fresh.scratch_blk_dofs.swap(P.scratch_blk_dofs);
    fresh.scratch_blk_rng.swap(P.scratch_blk_rng);
    fresh.scratch_pair_tgt = std::move(P.scratch_pair_tgt);
    fresh.scratch_slot_tgt = std::move(P.scratch_slot_tgt);
    P = std::move(fresh);
  }
  P.opt = opt;
  auto clk = std::chrono::steady_clock::now();
  auto lap = [&](int k) {
    const auto n = std::chrono::steady_clock::now();
    P.phase_s[k] += std::chrono::duration<double>(n - clk).count();
    clk = n;
  };
  if (np <= 0 || nf <= 0 || ndof <= 0 || !X || !tri || !fdir || !dof_point || !dof_face || !dof_kind || !face_dof) {
    P.error = "invalid BVP description";
    return false;
  }
  if (opt.p < 1 || opt.p > 12 || opt.max_level < 1 || opt.max_level > 20 || opt.leaf_max < 1 || !(opt.theta > 0)) {
    P.error = "invalid options";
    return false;
  }
  P.np = np;
  P.nf = nf;
  P.ndof = ndof;
  P.dof_point.assign(dof_point, dof_point + ndof);
  P.dof_face.assign(dof_face, dof_face + ndof);
  P.dof_kind.assign(dof_kind, dof_kind + ndof);
  P.face_dof.assign(face_dof, face_dof + 3 * nf);
  for (int i = 0; i < ndof; ++i)
    if (dof_point[i] < 0 || dof_point[i] >= np || dof_kind[i] < 0 || dof_kind[i] > 2) {
      P.error = "invalid DOF table";
      return false;
    }
  for (int i = 0; i < 3 * nf; ++i)
    if (tri[i] < 0 || tri[i] >= np || face_dof[i] < 0 || face_dof[i] >= ndof) {
      P.error = "invalid connectivity";
      return false;
    }
  for (int i = 0; i < 3 * np; ++i)
    if (!std::isfinite(X[i])) {
      P.error = "non-finite coordinates";
      return false;
    }
  // point -> DOFs
  P.point_dof_off.assign(np + 1, 0);
  for (int i = 0; i < ndof; ++i) ++P.point_dof_off[dof_point[i] + 1];
  for (int p = 0; p < np; ++p) P.point_dof_off[p + 1] += P.point_dof_off[p];
  P.point_dof.resize(ndof);
  {
    std::vector<int> fill(P.point_dof_off.begin(), P.point_dof_off.end() - 1);
    for (int i = 0; i < ndof; ++i) P.point_dof[fill[dof_point[i]]++] = i;
  }
  P.corner_src_dof.assign(ndof, -1);
  for (int i = 0; i < ndof; ++i)
    if (dof_kind[i] == 2) {
      const int p = dof_point[i];
      for (int k = P.point_dof_off[p]; k < P.point_dof_off[p + 1]; ++k)
        if (dof_kind[P.point_dof[k]] == 0) P.corner_src_dof[i] = P.point_dof[k];
    }

  // coordinate scaling (Network.hpp:3215-3245, BEM_solveBVP_GMRES_FMM.hpp:3076-3091)
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (int i = 0; i < np; ++i)
    for (int a = 0; a < 3; ++a) {
      mn[a] = std::min(mn[a], X[3 * i + a]);
      mx[a] = std::max(mx[a], X[3 * i + a]);
    }
  const double Lx = std::abs(mx[0] - mn[0]), Ly = std::abs(mx[1] - mn[1]), Lz = std::abs(mx[2] - mn[2]);
  P.L = std::sqrt(Lx * Lx + Ly * Ly + Lz * Lz);
  if (!(P.L > 1e-10)) P.L = 1.0;
  P.Xs.resize(3 * np);
  for (int i = 0; i < 3 * np; ++i) P.Xs[i] = X[i] / P.L;
  for (int a = 0; a < 3; ++a) {
    mn[a] = 1e300;
    mx[a] = -1e300;
  }
  for (int i = 0; i < np; ++i)
    for (int a = 0; a < 3; ++a) {
      mn[a] = std::min(mn[a], P.Xs[3 * i + a]);
      mx[a] = std::max(mx[a], P.Xs[3 * i + a]);
    }
  P.scale = hypot3(mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]);
  const double C[3] = {(mn[0] + mx[0]) / 2., (mn[1] + mx[1]) / 2., (mn[2] + mx[2]) / 2.};
  bool keep_root = prev && !prev->nodes.empty() && prev->np == np && prev->nf == nf && prev->ndof == ndof && prev->opt.p == opt.p &&
                   prev->opt.theta == opt.theta && prev->opt.leaf_max == opt.leaf_max && prev->opt.max_level == opt.max_level &&
                   prev->dof_point == P.dof_point && prev->dof_face == P.dof_face && prev->dof_kind == P.dof_kind &&
                   prev->face_dof == P.face_dof;
  P.near_region = P.scale / 25.;

  // element sources (BEM_solveBVP_GMRES_FMM.hpp:1799-1937)
  auto XP = [&](int i) { return V3{P.Xs[3 * i], P.Xs[3 * i + 1], P.Xs[3 * i + 2]}; };
  Plan::SourceScratch& S = P.src_scratch;
  S.pole.resize(nf);
  S.q.resize(nf * 18);
  S.W.resize(nf * 6);
  S.en.resize(nf * 3);
  S.enear.resize(nf * 8);
  S.offs.resize(nf);
  std::vector<V3>& pole = S.pole;
  std::vector<double>&q = S.q, &W = S.W, &en = S.en, &enear = S.enear, &offs = S.offs;
#pragma omp parallel for schedule(static)
  for (int f = 0; f < nf; ++f) {
    const V3 a = XP(tri[3 * f]), b = XP(tri[3 * f + 1]), c = XP(tri[3 * f + 2]);
    const V3 cr = cross_dd(sub(b, a), sub(c, a));
    const V3 n = unit(cr);
    const double J = nrm(cr);
    pole[f] = bary(1. / 3., 1. / 3., 1. / 3., a, b, c);
    double off = 0.0;
    for (int k = 0; k < 6; ++k) {
      const V3 x = bary(kDv[k][0], kDv[k][1], kDv[k][2], a, b, c);
      for (int d = 0; d < 3; ++d) q[f * 18 + 3 * k + d] = x[d];
      W[f * 6 + k] = J * kDv[k][3];
      off = std::max(off, nrm(sub(x, pole[f])));
    }
    offs[f] = off;
    for (int d = 0; d < 3; ++d) en[3 * f + d] = n[d];
    const double area = 0.5 * nrm(cr);
    const V3 nh = normal_dd(a, b, c);
    enear[8 * f + 0] = 2. * area;
    for (int d = 0; d < 3; ++d) {
      enear[8 * f + 1 + d] = 2. * area * nh[d];
      enear[8 * f + 4 + d] = (a[d] + b[d] + c[d]) / 3.;
    }
    enear[8 * f + 7] = 0.0;
  }

  lap(0);
  // octree (BEM_solveBVP_GMRES_FMM.hpp:1178-1201; lib_spatial_partitioning.hpp)
  TreeBuilder T(opt, pole);
  auto grow_from = [&](const double* rc, double dLr) {
    T.B.clear();
    T.drops = 0;
    P.n_added = 0;
    double lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = rc[a] - dLr;
      hi[a] = rc[a] + dLr;
      P.root_C[a] = rc[a];
    }
    P.root_R = dLr;
    Bucket root;
    bucket_init(root, lo, hi, dLr);
    T.B.push_back(std::move(root));
    for (int f = 0; f < nf; ++f) P.n_added += T.add(0, f);
    if (opt.device_tree && grow_on_device(T, static_cast<DeviceTree*>(opt.device_tree), nf, pole)) {
      P.tree_on_device = true;
      return;
    }
    P.tree_on_device = false;
    if (T.B.size() != 1) {  // a device step failed part-way: grow on the host from the root alone
      T.B.resize(1);
      T.B[0].kids.clear();
      T.B[0].kid_of_cell.assign(T.B[0].kid_of_cell.size(), -1);
    }
    T.grow(0);
  };
  if (keep_root) {
    grow_from(prev->root_C, prev->root_R);
    if (P.n_added != nf) keep_root = false;  // a centroid left the old root: the reference re-initialises
  }
  if (!keep_root) grow_from(C, 1.05 * P.scale / 2.);
  P.n_child_drops = T.drops;
  std::vector<Bucket>& B = T.B;
  const int nb = (int)B.size();

  lap(1);
  // offsets (moments.hpp:1336-1349): leaves from their elements, parents from children
  std::vector<std::vector<int>> lvl(opt.max_level + 1);
  for (int i = 0; i < nb; ++i)
    if (!B[i].data.empty()) lvl[B[i].level].push_back(i);
  for (int i = 0; i < nb; ++i)
    if (!B[i].data.empty() && B[i].kids.empty()) {
      B[i].off = 0.0;
      for (int e : B[i].data) B[i].off = std::max(B[i].off, offs[e]);
    }
  for (int l = opt.max_level - 1; l >= 0; --l)
    for (int i : lvl[l]) {
      if (B[i].kids.empty()) continue;
      B[i].off = 0.0;
      for (int c : B[i].kids) B[i].off = std::max(B[i].off, B[c].off);
    }
  // lists (moments.hpp:983-997).  lists(a, b) only appends to the lists of a and of a's
  // descendants, so the traversal runs serially down to the calls whose target is at level
  // kSplit, records those calls in order, and then runs each such target's calls (in the
  // recorded order) in parallel: every list ends up in the serial order.
  bool lists_done = false;
  if (opt.device_tree) {  // level by level on the device (tree.cu), same lists in the same order
    std::vector<double> nXv(3 * (size_t)nb), ndl(nb), nof(nb);
    std::vector<int> cbv(nb), cev(nb), chv;
    for (int i = 0; i < nb; ++i) {
      for (int a = 0; a < 3; ++a) nXv[3 * (size_t)i + a] = B[i].X[a];
      ndl[i] = B[i].dL;
      nof[i] = B[i].off;
      cbv[i] = (int)chv.size();
      chv.insert(chv.end(), B[i].kids.begin(), B[i].kids.end());
      cev[i] = (int)chv.size();
    }
    std::vector<std::vector<int>> nr, ml;
    if (dtree_lists(static_cast<DeviceTree*>(opt.device_tree), nb, nXv.data(), ndl.data(), nof.data(), cbv.data(), cev.data(), chv.data(),
                    (int)chv.size(), opt.theta, nr, ml)) {
      for (int i = 0; i < nb; ++i) {
        B[i].near.swap(nr[i]);
        B[i].m2l.swap(ml[i]);
      }
      lists_done = true;
      P.lists_on_device = true;
    }
    P.device_launches = dtree_take_launches(static_cast<DeviceTree*>(opt.device_tree));
  }
  if (!lists_done) {
    constexpr int kSplit = 2;
    std::vector<std::pair<int, int>> tasks;
    std::function<void(int, int)> top = [&](int a, int b) {
      if (B[a].level >= kSplit) {
        tasks.push_back({a, b});
        return;
      }
      if (is_far(opt, B[a], B[b])) return;
      if (a != b) B[a].near.push_back(b);
      for (int ac : B[a].kids)
        for (int bc : B[b].kids) {
          if (ac != bc && is_far(opt, B[ac], B[bc]))
            B[ac].m2l.push_back(bc);
          else
            top(ac, bc);
        }
    };
    for (int a : B[0].kids)
      for (int b : B[0].kids) top(a, b);
    std::vector<int> torder(tasks.size());
    std::iota(torder.begin(), torder.end(), 0);
    std::stable_sort(torder.begin(), torder.end(), [&](int x, int y) { return tasks[x].first < tasks[y].first; });
    std::vector<int> starts;
    for (size_t i = 0; i < torder.size(); ++i)
      if (i == 0 || tasks[torder[i]].first != tasks[torder[i - 1]].first) starts.push_back((int)i);
    starts.push_back((int)torder.size());
#pragma omp parallel for schedule(dynamic, 1)
    for (int g = 0; g < (int)starts.size() - 1; ++g)
      for (int i = starts[g]; i < starts[g + 1]; ++i) lists(opt, B, tasks[torder[i]].first, tasks[torder[i]].second);
  }
  // the M2L sources of every target b, in the order the traversal (level by level) meets them:
  // the inverse of the m2l lists as a CSR, built by a parallel counting sort over the sources
  // taken in that order (per-thread counts per target, then a scan over (target, thread))
  std::vector<int> l2m_off(nb + 1, 0), l2m_src;
  {
    std::vector<int> order;
    for (auto& lv : lvl) order.insert(order.end(), lv.begin(), lv.end());
    const int na = (int)order.size();
    const int nt = std::max(1, omp_get_max_threads());
    std::vector<int> cnt((size_t)nt * nb, 0);
    int T = 1;
#pragma omp parallel num_threads(nt)
    {
      const int t = omp_get_thread_num();
#pragma omp single
      T = omp_get_num_threads();
      const int lo = (int)((int64_t)na * t / T), hi = (int)((int64_t)na * (t + 1) / T);
      int* c = &cnt[(size_t)t * nb];
      for (int i = lo; i < hi; ++i)
        for (int b : B[order[i]].m2l) ++c[b];
#pragma omp barrier
#pragma omp single
      {
        int run = 0;
        for (int b = 0; b < nb; ++b) {
          l2m_off[b] = run;
          for (int u = 0; u < T; ++u) {
            const int k = cnt[(size_t)u * nb + b];
            cnt[(size_t)u * nb + b] = run;
            run += k;
          }
        }
        l2m_off[nb] = run;
        l2m_src.resize(run);
      }
      for (int i = lo; i < hi; ++i)
        for (int b : B[order[i]].m2l) l2m_src[c[b]++] = order[i];
    }
  }

  lap(2);
  // element order: DFS pre-order of the deepest bucket holding each element
  // (the buckets of one level hold disjoint elements, and a deeper bucket is created after its
  // ancestors: assigning level by level leaves each element with the last bucket in creation
  // order that holds it)
  std::vector<int> owner(nf, -1);
  {
    int maxl = 0;
    for (int i = 0; i < nb; ++i) maxl = std::max(maxl, B[i].level);
    std::vector<std::vector<int>> by_level(maxl + 1);
    for (int i = 0; i < nb; ++i) by_level[B[i].level].push_back(i);
    for (const auto& lv : by_level) {
#pragma omp parallel for schedule(dynamic, 16)
      for (int k = 0; k < (int)lv.size(); ++k)
        for (int e : B[lv[k]].data) owner[e] = lv[k];
    }
  }
  std::vector<std::vector<int>> owned(nb);
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nb; ++i)
    for (int e : B[i].data)
      if (owner[e] == i) owned[i].push_back(e);
  std::vector<int> subtree_end(nb);
  for (int i = nb - 1; i >= 0; --i) {
    subtree_end[i] = i + 1;
    for (int c : B[i].kids) subtree_end[i] = std::max(subtree_end[i], subtree_end[c]);
  }
  P.face_of_pos.clear();
  std::vector<int> start(nb + 1);
  for (int i = 0; i < nb; ++i) {
    start[i] = (int)P.face_of_pos.size();
    for (int e : owned[i]) P.face_of_pos.push_back(e);
  }
  start[nb] = (int)P.face_of_pos.size();
  P.owner_of_pos.assign(P.face_of_pos.size(), -1);
  for (int i = 0; i < nb; ++i)
    for (int s = start[i]; s < start[i] + (int)owned[i].size(); ++s) P.owner_of_pos[s] = i;
  const int ne = (int)P.face_of_pos.size();
  P.pos_of_face.assign(nf, -1);
  for (int s = 0; s < ne; ++s) P.pos_of_face[P.face_of_pos[s]] = s;
  P.e_q.resize(ne * 18);
  P.e_W.resize(ne * 6);
  P.e_n.resize(ne * 3);
  P.e_dof.resize(ne * 3);
  P.e_vtx.resize(ne * 3);
  P.e_near.resize(ne * 8);
#pragma omp parallel for schedule(static)
  for (int s = 0; s < ne; ++s) {
    const int f = P.face_of_pos[s];
    std::memcpy(&P.e_q[s * 18], &q[f * 18], 18 * sizeof(double));
    std::memcpy(&P.e_W[s * 6], &W[f * 6], 6 * sizeof(double));
    std::memcpy(&P.e_n[s * 3], &en[f * 3], 3 * sizeof(double));
    std::memcpy(&P.e_near[s * 8], &enear[f * 8], 8 * sizeof(double));
    for (int a = 0; a < 3; ++a) {
      P.e_dof[s * 3 + a] = face_dof[3 * f + a];
      P.e_vtx[s * 3 + a] = tri[3 * f + a];
    }
  }
  P.nodes.resize(nb);
  P.node_children.clear();
  for (int i = 0; i < nb; ++i) {
    Plan::Node& N = P.nodes[i];
    for (int a = 0; a < 3; ++a) {
      N.lo[a] = B[i].lo[a];
      N.hi[a] = B[i].hi[a];
      N.X[a] = B[i].X[a];
    }
    N.dL = B[i].dL;
    N.inv_dL = B[i].inv_dL;
    for (int a = 0; a < 3; ++a) N.size[a] = B[i].size[a];
    N.level = B[i].level;
    N.parent = B[i].parent;
    N.child_begin = (int)P.node_children.size();
    for (int c : B[i].kids) P.node_children.push_back(c);
    N.child_end = (int)P.node_children.size();
    N.fb = start[i];
    N.fe = start[subtree_end[i]];
    N.n_data = (int)B[i].data.size();
    N.max_internal_offset = B[i].off;
  }
  P.level_nodes = lvl;
  P.leaves.clear();
  for (auto& lv : lvl)
    for (int i : lv)
      if (B[i].kids.empty()) P.leaves.push_back(i);
  // M2L sources per target node (non-empty targets only), near lists
  P.m2l_off.assign(nb + 1, 0);
  P.near_off.assign(nb + 1, 0);
  for (int i = 0; i < nb; ++i) {
    P.m2l_off[i + 1] = P.m2l_off[i] + (B[i].data.empty() ? 0 : l2m_off[i + 1] - l2m_off[i]);
    P.near_off[i + 1] = P.near_off[i] + (int)B[i].near.size();
  }
  P.m2l_src.resize(P.m2l_off[nb]);
  P.near_nodes.resize(P.near_off[nb]);
  for (int i = 0; i < nb; ++i) {
    if (!B[i].data.empty()) std::copy(l2m_src.begin() + l2m_off[i], l2m_src.begin() + l2m_off[i + 1], P.m2l_src.begin() + P.m2l_off[i]);
    std::copy(B[i].near.begin(), B[i].near.end(), P.near_nodes.begin() + P.near_off[i]);
  }
  P.m2l_pairs = P.m2l_off[nb];
  // targets (target4FMM::setL2P / setDirectIntegration: getBucketAtDeepest)
  P.target_box.assign(np, -1);
#pragma omp parallel for schedule(static)
  for (int p = 0; p < np; ++p) {
    if (P.point_dof_off[p] == P.point_dof_off[p + 1]) continue;
    const double* x = &P.Xs[3 * p];
    int cur = 0;
    while (!B[cur].kids.empty()) {
      const int nx = B[cur].kid_of_cell[cell_of(B[cur], x)];
      if (nx < 0) break;
      cur = nx;
    }
    P.target_box[p] = cur;
  }
  lap(3);
  P.reused_m2l = keep_root && opt.take_structure && same_tree(P, *prev);
  if (P.reused_m2l) {  // refresh, unchanged tree and lists: the M2L grouping is the previous one
    P.m2l_key_sorted = std::move(prev->m2l_key_sorted);
    P.grp_vec = std::move(prev->grp_vec);
    P.grp_off = std::move(prev->grp_off);
    P.grp_pair = std::move(prev->grp_pair);
    P.chunk_grp = std::move(prev->chunk_grp);
    P.chunk_begin = std::move(prev->chunk_begin);
    P.chunk_cnt = std::move(prev->chunk_cnt);
    P.m2l_targets = std::move(prev->m2l_targets);
    P.tc_tab = std::move(prev->tc_tab);
    P.tc_pair = std::move(prev->tc_pair);
    P.tc_item_tab = std::move(prev->tc_item_tab);
    P.tc_item_begin = std::move(prev->tc_item_begin);
    P.tc_item_cnt = std::move(prev->tc_item_cnt);
  }
  if (!P.reused_m2l && !defer_m2l_groups && !build_m2l_groups(P)) return false;
  P.near_pairs = P.near_off[nb];
  for (int i = 0; i < nb; ++i)
    if (B[i].data.empty()) P.near_pairs -= (int)B[i].near.size();
  lap(4);
  P.reused_near = P.reused_m2l && P.target_box == prev->target_box;
  if (P.reused_near) {  // and the same L2P targets: the near-field blocks are the previous ones
    P.blocks = std::move(prev->blocks);
    P.nb_dofs = std::move(prev->nb_dofs);
    P.nb_targets = std::move(prev->nb_targets);
    P.nb_ranges = std::move(prev->nb_ranges);
    P.block_of_point = std::move(prev->block_of_point);
    P.row_of_point = std::move(prev->row_of_point);
    P.self_col = std::move(prev->self_col);
    P.nnz = prev->nnz;
    P.dof_inc_off = std::move(prev->dof_inc_off);
    P.dof_inc = std::move(prev->dof_inc);
    return true;
  }
  // near blocks (lib_multipole_expansion.hpp:1180-1213)
  std::vector<int> block_of_node(nb, -1);
  P.blocks.clear();
  P.block_of_point.assign(np, -1);
  P.row_of_point.assign(np, -1);
  std::vector<std::vector<int>> btargets;
  for (int p = 0; p < np; ++p) {
    const int t = P.target_box[p];
    if (t < 0) continue;
    if (block_of_node[t] < 0) {
      block_of_node[t] = (int)P.blocks.size();
      Plan::NearBlock nbk{};
      nbk.node = t;
      P.blocks.push_back(nbk);
      btargets.emplace_back();
    }
    const int bi = block_of_node[t];
    P.block_of_point[p] = bi;
    P.row_of_point[p] = (int)btargets[bi].size();
    btargets[bi].push_back(p);
  }
  P.nb_dofs.clear();
  P.nb_targets.clear();
  P.nb_ranges.clear();
  const int nblk = (int)P.blocks.size();
  // each thread appends its blocks' merged element ranges and DOF lists to buffers of its own
  // (kept across set-ups), then every block is copied to its place
  struct BlkRec {
    int th;
    int nd, nr;
    int64_t d0, r0;
  };
  std::vector<BlkRec> rec(nblk);
  const int nthr = std::max(1, omp_get_max_threads());
  if ((int)P.scratch_blk_dofs.size() < nthr) {
    P.scratch_blk_dofs.resize(nthr);
    P.scratch_blk_rng.resize(nthr);
  }
#pragma omp parallel num_threads(nthr)
  {
    const int th = omp_get_thread_num();
    // the buffers on this thread's stack while it appends (their headers would otherwise share
    // cache lines between threads), back in the plan afterwards
    std::vector<int32_t> bd = std::move(P.scratch_blk_dofs[th]), br = std::move(P.scratch_blk_rng[th]);
    bd.clear();
    br.clear();
    std::vector<int> mark(ndof, -1);
    std::vector<std::pair<int, int>> rng, merged;
#pragma omp for schedule(dynamic, 8)
    for (int bi = 0; bi < nblk; ++bi) {
      const int t = P.blocks[bi].node;
      rng.clear();
      merged.clear();
      auto addr = [&](int n) {
        if (P.nodes[n].fe > P.nodes[n].fb) rng.push_back({P.nodes[n].fb, P.nodes[n].fe});
      };
      addr(t);
      for (int n : B[t].near) addr(n);
      for (int a = B[t].parent; a >= 0; a = B[a].parent)
        for (int n : B[a].near)
          if (B[n].kids.empty()) addr(n);
      std::sort(rng.begin(), rng.end());
      for (auto& r : rng) {
        if (!merged.empty() && r.first <= merged.back().second)
          merged.back().second = std::max(merged.back().second, r.second);
        else
          merged.push_back(r);
      }
      BlkRec& R = rec[bi];
      R.th = th;
      R.d0 = (int64_t)bd.size();
      R.r0 = (int64_t)br.size();
      for (auto& r : merged) {
        br.push_back(r.first);
        br.push_back(r.second);
        for (int s = r.first; s < r.second; ++s)
          for (int a = 0; a < 3; ++a) {
            const int d = P.e_dof[s * 3 + a];
            if (mark[d] != bi) {
              mark[d] = bi;
              bd.push_back(d);
            }
          }
      }
      R.nd = (int)((int64_t)bd.size() - R.d0);
      R.nr = (int)(((int64_t)br.size() - R.r0) / 2);
    }
    P.scratch_blk_dofs[th] = std::move(bd);
    P.scratch_blk_rng[th] = std::move(br);
  }
  // offsets first, then one parallel copy into arrays sized once
  int64_t woff = 0, roff = 0, doff = 0, toff = 0;
  for (int bi = 0; bi < nblk; ++bi) {
    Plan::NearBlock& nbk = P.blocks[bi];
    nbk.rng_off = (int)(roff / 2);
    nbk.nrng = rec[bi].nr;
    roff += 2 * (int64_t)rec[bi].nr;
    nbk.dof_off = (int)doff;
    nbk.ndof = rec[bi].nd;
    doff += nbk.ndof;
    nbk.tgt_off = (int)toff;
    nbk.ntgt = (int)btargets[bi].size();
    toff += nbk.ntgt;
    nbk.w_off = woff;
    woff += (int64_t)nbk.ntgt * nbk.ndof;
  }
  P.nb_ranges.resize(roff);
  P.nb_dofs.resize(doff);
  P.nb_targets.resize(toff);
#pragma omp parallel for schedule(dynamic, 16)
  for (int bi = 0; bi < nblk; ++bi) {
    const Plan::NearBlock& nbk = P.blocks[bi];
    const BlkRec& R = rec[bi];
    const std::vector<int32_t>& bd = P.scratch_blk_dofs[R.th];
    const std::vector<int32_t>& br = P.scratch_blk_rng[R.th];
    std::copy(br.begin() + R.r0, br.begin() + R.r0 + 2 * (int64_t)R.nr, P.nb_ranges.begin() + 2 * (int64_t)nbk.rng_off);
    std::copy(bd.begin() + R.d0, bd.begin() + R.d0 + R.nd, P.nb_dofs.begin() + nbk.dof_off);
    std::copy(btargets[bi].begin(), btargets[bi].end(), P.nb_targets.begin() + nbk.tgt_off);
  }
  P.nnz = woff;
  // column of each DOF in its own point's block row (the diagonal entry of the operator)
  P.self_col.assign(ndof, -1);
#pragma omp parallel for schedule(dynamic, 16)
  for (int bi = 0; bi < nblk; ++bi) {
    const Plan::NearBlock& nbk = P.blocks[bi];
    for (int j = 0; j < nbk.ndof; ++j) {
      const int d = P.nb_dofs[nbk.dof_off + j];
      if (P.block_of_point[dof_point[d]] == bi) P.self_col[d] = j;
    }
  }
  lap(5);
  // DOF -> incident element vertices
  P.dof_inc_off.assign(ndof + 1, 0);
  for (int s = 0; s < ne; ++s)
    for (int a = 0; a < 3; ++a) ++P.dof_inc_off[P.e_dof[s * 3 + a] + 1];
  for (int i = 0; i < ndof; ++i) P.dof_inc_off[i + 1] += P.dof_inc_off[i];
  P.dof_inc.resize(P.dof_inc_off[ndof]);
  {
    std::vector<int> fill(P.dof_inc_off.begin(), P.dof_inc_off.end() - 1);
    for (int s = 0; s < ne; ++s)
      for (int a = 0; a < 3; ++a) P.dof_inc[fill[P.e_dof[s * 3 + a]]++] = s * 3 + a;
  }
  lap(6);
  return true;
}

void retile_tc_items(Plan& P, int max_pairs) {
  std::vector<int32_t> tab, beg, cnt;
  const size_t n = P.tc_item_tab.size();
  for (size_t i = 0; i < n;) {  // the items of one table cover one run of tc_pair
    size_t j = i;
    int64_t total = 0;
    while (j < n && P.tc_item_tab[j] == P.tc_item_tab[i]) total += P.tc_item_cnt[j++];
    for (int64_t b = 0; b < total; b += max_pairs) {
      tab.push_back(P.tc_item_tab[i]);
      beg.push_back(P.tc_item_begin[i] + (int)b);
      cnt.push_back((int)std::min<int64_t>(max_pairs, total - b));
    }
    i = j;
  }
  P.tc_item_tab.swap(tab);
  P.tc_item_begin.swap(beg);
  P.tc_item_cnt.swap(cnt);
}

void build_tc_groups(Plan& P, int max_pairs) {
  // tables = runs of one lattice offset over all levels in the sorted pair order of the FP64
  // groups (the pairs of one offset are contiguous there); pairs off the lattice get one each
  const int64_t npair = (int64_t)P.m2l_key_sorted.size();
  const std::vector<uint64_t>& keyed = P.m2l_key_sorted;
  const uint64_t kmask = (uint64_t(1) << 29) - 1;
  std::vector<int>& pair_tgt = P.scratch_pair_tgt;
  pair_targets(P, pair_tgt);
  std::vector<int64_t> rs;
  parallel_heads(
      npair, [&](int64_t i) { return i == 0 || (keyed[i] >> 63) || (keyed[i - 1] >> 63) || (keyed[i] >> 33) != (keyed[i - 1] >> 33); }, rs);
  const int nt = (int)rs.size();
  P.tc_tab.resize(4 * (size_t)nt);
  P.tc_pair.resize(npair);
  std::vector<int> nit(nt + 1, 0);  // items per table, then their offsets
#pragma omp parallel for schedule(static)
  for (int t = 0; t < nt; ++t) {
    const int64_t b = rs[t], e = t + 1 < nt ? rs[t + 1] : npair;
    const bool lattice = (keyed[b] >> 63) == 0;
    const int k0 = (int)(keyed[b] & kmask);
    const auto& T = P.nodes[pair_tgt[k0]];
    const auto& S = P.nodes[P.m2l_src[k0]];
    for (int a = 0; a < 3; ++a) {
      const double q = (T.X[a] - S.X[a]) / T.dL;
      P.tc_tab[4 * (size_t)t + a] = lattice ? (double)std::llround(q) : q;
    }
    P.tc_tab[4 * (size_t)t + 3] = lattice ? 1.0 : S.dL / T.dL;
    nit[t + 1] = (int)((e - b + max_pairs - 1) / max_pairs);
  }
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < npair; ++j) P.tc_pair[j] = (int)(keyed[j] & kmask);
  for (int t = 0; t < nt; ++t) nit[t + 1] += nit[t];
  P.tc_item_tab.resize(nit[nt]);
  P.tc_item_begin.resize(nit[nt]);
  P.tc_item_cnt.resize(nit[nt]);
#pragma omp parallel for schedule(static)
  for (int t = 0; t < nt; ++t) {
    const int64_t e = t + 1 < nt ? rs[t + 1] : npair;
    int64_t b = rs[t];
    for (int i = nit[t]; i < nit[t + 1]; ++i, b += max_pairs) {
      P.tc_item_tab[i] = t;
      P.tc_item_begin[i] = (int)b;
      P.tc_item_cnt[i] = (int)std::min<int64_t>(max_pairs, e - b);
    }
  }
}

void tc_item_arrays(Plan& P, std::vector<int>& src, std::vector<int>& pos, std::vector<int>& tgt) {
  const size_t n = P.tc_pair.size();
  src.resize(n);
  pos.resize(n);
  tgt.resize(n);
  std::vector<int32_t>& tgt_of_slot = P.scratch_slot_tgt;
  tgt_of_slot.resize((size_t)P.m2l_pairs);
  const int nt = (int)P.m2l_targets.size();
#pragma omp parallel for schedule(static)
  for (int ti = 0; ti < nt; ++ti) {
    const int t = P.m2l_targets[ti];
    for (int k = P.m2l_off[t]; k < P.m2l_off[t + 1]; ++k) tgt_of_slot[k] = ti;
  }
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < (int64_t)n; ++j) {
    const int k = P.tc_pair[j];
    src[j] = P.m2l_src[k];
    pos[k] = (int)j;
    tgt[j] = tgt_of_slot[k];
  }
}

}  // namespace bemb200
