// Octree growth on the device: the element-parallel part of Buckets::generateTree
// (lib/include/lib_spatial_partitioning.hpp:1078-1111, Buckets::add :295-350).
//
// The tree grows level by level.  For every bucket of the level that splits, each of its
// elements (in the bucket's data order) is classified into one of the bucket's 2x2x2 cells by
// the reference's floor((x - xmin) / dL) with clamping, and kept in the child of that cell only
// if the child's own InsideQ (no clamping) accepts it; the children's data are the kept
// elements in the parent's order (a stable partition).  Bucket geometry stays on the host
// (plan.cpp computes every child's bounds with the reference's expressions), so the device
// evaluates only subtractions, products and floors of the host's numbers: the classification is
// bit-identical to the host's.  Node numbering (creation order, depth first) is done on the host
// from the per-level results.
#include <cuda_runtime.h>

#include <cstdint>
#include <algorithm>
#include <vector>

#include "tree_dev.hpp"

namespace bemb200 {
namespace {

// per splitting bucket: parent geometry then the 8 children's (xmin[3], inv_dL, size[3]) as
// doubles, 7 + 8 * 7 values
constexpr int kGeo = 7 * 9;
constexpr int kChunk = 4096;  // elements per CTA of the classification and the scatter

__device__ __forceinline__ int cell_index_clamped(const double* g, const double* x) {
  int ijk[3];
  for (int a = 0; a < 3; ++a) {
    int v = (int)floor((x[a] - g[a]) * g[3]);
    const int sz = (int)g[4 + a];
    v = v < 0 ? 0 : (v > sz - 1 ? sz - 1 : v);
    ijk[a] = v;
  }
  return (ijk[0] * (int)g[5] + ijk[1]) * (int)g[6] + ijk[2];
}

__device__ __forceinline__ bool inside_box(const double* g, const double* x) {
  for (int a = 0; a < 3; ++a) {
    const int v = (int)floor((x[a] - g[a]) * g[3]);
    if (v < 0 || v >= (int)g[4 + a]) return false;
  }
  return true;
}

// one CTA per chunk of a splitting bucket's elements (at most kChunk, in order): cell and inside
// flag of each element; counts per cell of the chunk
__global__ void __launch_bounds__(256) k_tree_count(const int* __restrict__ seg_beg, const int* __restrict__ seg_end,
                                                    const int* __restrict__ seg_geo, const double* __restrict__ geo,
                                                    const int* __restrict__ elems,
                                                    const double* __restrict__ poles, int tag_base, uint8_t* __restrict__ tag,
                                                    int* __restrict__ cnt_all, int* __restrict__ cnt_pass) {
  __shared__ double g[kGeo];
  __shared__ int ca[8], cp[8];
  const int node = blockIdx.x;
  for (int i = threadIdx.x; i < kGeo; i += blockDim.x) g[i] = geo[(size_t)seg_geo[node] * kGeo + i];
  if (threadIdx.x < 8) ca[threadIdx.x] = cp[threadIdx.x] = 0;
  __syncthreads();
  for (int i = seg_beg[node] + threadIdx.x; i < seg_end[node]; i += blockDim.x) {
    const int e = elems[i];
    const double x[3] = {poles[3 * (size_t)e], poles[3 * (size_t)e + 1], poles[3 * (size_t)e + 2]};
    const int c = cell_index_clamped(g, x);
    const bool in = inside_box(g + 7 * (1 + c), x);
    tag[i - tag_base] = (uint8_t)(c | (in ? 8 : 0));
    atomicAdd(&ca[c], 1);
    if (in) atomicAdd(&cp[c], 1);
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    cnt_all[node * 8 + threadIdx.x] = ca[threadIdx.x];
    cnt_pass[node * 8 + threadIdx.x] = cp[threadIdx.x];
  }
}

// stable scatter of the kept elements of each (chunk, cell) to off[chunk * 8 + cell] onwards (the
// chunks of a bucket follow each other, so the bucket's partition is stable as a whole)
__global__ void __launch_bounds__(256) k_tree_scatter(const int* __restrict__ seg_beg, const int* __restrict__ seg_end,
                                                      const int* __restrict__ elems, int tag_base, const uint8_t* __restrict__ tag,
                                                      const int* __restrict__ off, int* __restrict__ next) {
  __shared__ int run[8];
  __shared__ int wcnt[8][8];  // [warp][cell]
  const int node = blockIdx.x, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x < 8) run[threadIdx.x] = 0;
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  for (int base = seg_beg[node]; base < seg_end[node]; base += blockDim.x) {
    const int i = base + threadIdx.x;
    int c = 8;
    if (i < seg_end[node]) {
      const int t = tag[i - tag_base];
      if (t & 8) c = t & 7;
    }
    int rank = 0;
    for (int k = 0; k < 8; ++k) {
      const unsigned m = __ballot_sync(0xffffffffu, c == k);
      if (c == k) rank = __popc(m & lt);
      if (lane == 0) wcnt[warp][k] = __popc(m);
    }
    __syncthreads();
    if (c < 8) {
      int o = run[c];
      for (int w = 0; w < warp; ++w) o += wcnt[w][c];
      next[off[node * 8 + c] + o + rank] = elems[i];
    }
    __syncthreads();
    if (threadIdx.x < 8) {
      int s = 0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += wcnt[w][threadIdx.x];
      run[threadIdx.x] += s;
    }
    __syncthreads();
  }
}

// ---- interaction lists (moments.hpp:950-997) ----
// isFar with the host's arithmetic (plan.cpp is_far as g++ compiles it: the squared distance and
// the hypot sum contracted as fma(z, z, fma(y, y, x * x)), eff as dL + 2 off), so the decisions
// are the host's, including the pairs within 1e-9 of the threshold that take the exact form
struct NodeGeo {
  const double* X;  // [3 * nb]
  const double* dL;
  const double* off;
  const int* cb;  // children of node i: children[cb[i] .. ce[i])
  const int* ce;
  const int* children;
};

__device__ __forceinline__ double hypot3_dev(double x, double y, double z) {
  x = fabs(x);
  y = fabs(y);
  z = fabs(z);
  const double a = x < y ? (y < z ? z : y) : (x < z ? z : x);
  if (a == 0.0) return 0.0;
  const double xa = __ddiv_rn(x, a), ya = __ddiv_rn(y, a), za = __ddiv_rn(z, a);
  return __dmul_rn(a, __dsqrt_rn(fma(za, za, fma(ya, ya, __dmul_rn(xa, xa)))));
}

__device__ __forceinline__ bool is_far_dev(const NodeGeo& g, double theta, int a, int b) {
  const double ea = fma(2.0, g.off[a], g.dL[a]), eb = fma(2.0, g.off[b], g.dL[b]);
  const double eff = ea > eb ? ea : eb;  // std::max(ea, eb)
  const double d0 = __dsub_rn(g.X[3 * b], g.X[3 * a]), d1 = __dsub_rn(g.X[3 * b + 1], g.X[3 * a + 1]),
               d2 = __dsub_rn(g.X[3 * b + 2], g.X[3 * a + 2]);
  const double s3e = __dmul_rn(1.7320508075688772, eff);
  const double thr = __ddiv_rn(s3e, theta);
  const double dd = fma(d2, d2, fma(d1, d1, __dmul_rn(d0, d0)));
  const double t2 = __dmul_rn(thr, thr);
  if (dd > __dmul_rn(t2, 1.0 + 1e-9)) return true;
  if (dd < __dmul_rn(t2, 1.0 - 1e-9)) return false;
  return theta > __ddiv_rn(s3e, hypot3_dev(d0, d1, d2));
}

// one warp per target x: for each candidate b (lists(x, b) calls, in order) that is not far:
// near[x] += b (b != x); for each child pair (ac, bc) of (x, b): far -> m2l[ac] += bc, else
// lists(ac, bc) is called (candidate of ac at the next level).  fill = 0: counts only.
template <bool kFill>
__global__ void __launch_bounds__(128) k_lists(int n, const int* __restrict__ tgt, const int* __restrict__ cand_off,
                                               const int* __restrict__ cand, NodeGeo g, double theta, int* __restrict__ cnt_near,
                                               int* __restrict__ cnt_m2l, int* __restrict__ cnt_next, const int* __restrict__ near_off,
                                               const int* __restrict__ m2l_off, const int* __restrict__ next_off,
                                               int* __restrict__ near_out, int* __restrict__ m2l_out, int* __restrict__ next_out) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= n) return;
  const unsigned lt = (1u << lane) - 1u;
  const int x = tgt[w];
  const int kx0 = g.cb[x], nkx = g.ce[x] - g.cb[x];
  int cn = 0, rm[8], rn[8];
#pragma unroll
  for (int s = 0; s < 8; ++s) rm[s] = rn[s] = 0;
  for (int k = cand_off[w]; k < cand_off[w + 1]; ++k) {
    const int b = cand[k];
    if (is_far_dev(g, theta, x, b)) continue;
    if (x != b) {
      if (kFill && lane == 0) near_out[near_off[w] + cn] = b;
      ++cn;
    }
    const int kb0 = g.cb[b], nkb = g.ce[b] - g.cb[b];
    const int combos = nkx * nkb;
    for (int base = 0; base < combos; base += 32) {
      const int j = base + lane;
      const bool valid = j < combos;
      int ai = -1, bc = -1;
      bool f = false;
      if (valid) {
        ai = j / nkb;
        const int ac = g.children[kx0 + ai];
        bc = g.children[kb0 + (j - ai * nkb)];
        f = ac != bc && is_far_dev(g, theta, ac, bc);
      }
#pragma unroll
      for (int s = 0; s < 8; ++s) {
        const unsigned mm = __ballot_sync(0xffffffffu, valid && ai == s && f);
        const unsigned mn = __ballot_sync(0xffffffffu, valid && ai == s && !f);
        if (kFill && valid && ai == s) {
          if (f)
            m2l_out[m2l_off[8 * w + s] + rm[s] + __popc(mm & lt)] = bc;
          else
            next_out[next_off[8 * w + s] + rn[s] + __popc(mn & lt)] = bc;
        }
        rm[s] += __popc(mm);
        rn[s] += __popc(mn);
      }
    }
  }
  if (!kFill && lane == 0) {
    cnt_near[w] = cn;
#pragma unroll
    for (int s = 0; s < 8; ++s) {
      cnt_m2l[8 * w + s] = rm[s];
      cnt_next[8 * w + s] = rn[s];
    }
  }
}

template <typename T>
struct Buf {
  T* p = nullptr;
  size_t cap = 0;
  ~Buf() {
    if (p) cudaFree(p);
  }
  bool fit(size_t n) {
    if (n <= cap) return true;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (cudaMalloc((void**)&p, sizeof(T) * (n ? n : 1)) != cudaSuccess) return false;
    cap = n ? n : 1;
    return true;
  }
};

}  // namespace

struct DeviceTree {
  cudaStream_t stream = nullptr;
  Buf<double> poles, geo;
  Buf<int> elems, seg_beg, seg_end, seg_geo, cnt, off;  // elems: every level's array, back to back; segments = chunks
  Buf<uint8_t> tag;
  Buf<double> nX, ndL, noff;                              // interaction lists: node geometry
  Buf<int> ncb, nce, nch, lt, lco, lc, lcnt, loff, lno, lmo, lxo;  // and per-level work arrays
  size_t cur = 0, cur_n = 0;  // current level: offset into elems, length
  int launches = 0;
  std::vector<int> h_beg, h_end, h_geo, h_cnt;  // chunks of the current level and their counts
};

DeviceTree* dtree_create(void* stream) {
  auto* t = new DeviceTree();
  if (t) t->stream = static_cast<cudaStream_t>(stream);
  return t;
}

void dtree_destroy(DeviceTree* t) { delete t; }

bool dtree_begin(DeviceTree* t, int nf, const double* poles, int n_root, const int* root_elems, int max_level) {
  // every level holds at most the root's elements
  const size_t total = (size_t)n_root * (size_t)(max_level + 1);
  if (!t->poles.fit((size_t)3 * nf) || !t->elems.fit(total) || !t->tag.fit((size_t)n_root)) return false;
  cudaStream_t s = t->stream;
  if (cudaMemcpyAsync(t->poles.p, poles, sizeof(double) * 3 * nf, cudaMemcpyHostToDevice, s) != cudaSuccess) return false;
  if (n_root && cudaMemcpyAsync(t->elems.p, root_elems, sizeof(int) * n_root, cudaMemcpyHostToDevice, s) != cudaSuccess) return false;
  t->cur = 0;
  t->cur_n = (size_t)n_root;
  return true;
}

bool dtree_count(DeviceTree* t, int n, const int* seg_beg, const int* seg_end, const double* geo, int* cnt_all, int* cnt_pass) {
  if (n <= 0) return true;
  cudaStream_t s = t->stream;
  // chunks of at most kChunk elements, in bucket order and, within a bucket, in element order
  t->h_beg.clear();
  t->h_end.clear();
  t->h_geo.clear();
  for (int i = 0; i < n; ++i) {  // segments are offsets into the current level's array
    if (seg_beg[i] < 0 || seg_end[i] < seg_beg[i] || (size_t)seg_end[i] > t->cur_n) return false;
    for (int b = seg_beg[i]; b < seg_end[i]; b += kChunk) {
      t->h_beg.push_back(b + (int)t->cur);
      t->h_end.push_back(std::min(b + kChunk, seg_end[i]) + (int)t->cur);
      t->h_geo.push_back(i);
    }
  }
  const int nc = (int)t->h_beg.size();
  std::fill(cnt_all, cnt_all + 8 * (size_t)n, 0);
  std::fill(cnt_pass, cnt_pass + 8 * (size_t)n, 0);
  t->h_cnt.assign(16 * (size_t)nc, 0);
  if (nc == 0) return true;
  if (!t->seg_beg.fit(nc) || !t->seg_end.fit(nc) || !t->seg_geo.fit(nc) || !t->geo.fit((size_t)n * kGeo) || !t->cnt.fit((size_t)16 * nc) ||
      !t->off.fit((size_t)8 * nc))
    return false;
  if (cudaMemcpyAsync(t->seg_beg.p, t->h_beg.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(t->seg_end.p, t->h_end.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(t->seg_geo.p, t->h_geo.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(t->geo.p, geo, sizeof(double) * kGeo * n, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return false;
  // tags are indexed by position in the elems buffer relative to the current level
  ++t->launches;
  k_tree_count<<<nc, 256, 0, s>>>(t->seg_beg.p, t->seg_end.p, t->seg_geo.p, t->geo.p, t->elems.p, t->poles.p, (int)t->cur, t->tag.p,
                                  t->cnt.p, t->cnt.p + 8 * nc);
  if (cudaGetLastError() != cudaSuccess) return false;
  if (cudaMemcpyAsync(t->h_cnt.data(), t->cnt.p, sizeof(int) * 16 * nc, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return false;
  for (int c = 0; c < nc; ++c)
    for (int k = 0; k < 8; ++k) {
      cnt_all[8 * t->h_geo[c] + k] += t->h_cnt[8 * (size_t)c + k];
      cnt_pass[8 * t->h_geo[c] + k] += t->h_cnt[8 * (size_t)nc + 8 * (size_t)c + k];
    }
  return true;
}

bool dtree_scatter(DeviceTree* t, int n, const int* off, int total) {
  cudaStream_t s = t->stream;
  const size_t next = t->cur + t->cur_n;
  if (next + (size_t)total > t->elems.cap) return false;
  const int nc = (int)t->h_beg.size();
  if (n > 0 && nc > 0) {
    // each chunk's kept elements of cell k start after those of the bucket's earlier chunks
    for (int i = 0; i < 8 * n; ++i)
      if (off[i] < 0 || off[i] > total) return false;
    std::vector<int> o(8 * (size_t)nc), run(off, off + 8 * (size_t)n);
    for (int c = 0; c < nc; ++c)
      for (int k = 0; k < 8; ++k) {
        int& r = run[8 * (size_t)t->h_geo[c] + k];
        o[8 * (size_t)c + k] = r + (int)next;
        r += t->h_cnt[8 * (size_t)nc + 8 * (size_t)c + k];
        if (r > total) return false;
      }
    if (cudaMemcpyAsync(t->off.p, o.data(), sizeof(int) * 8 * nc, cudaMemcpyHostToDevice, s) != cudaSuccess) return false;
    ++t->launches;
    k_tree_scatter<<<nc, 256, 0, s>>>(t->seg_beg.p, t->seg_end.p, t->elems.p, (int)t->cur, t->tag.p, t->off.p, t->elems.p);
    if (cudaGetLastError() != cudaSuccess) return false;
    if (cudaStreamSynchronize(s) != cudaSuccess) return false;  // o is freed on return
  }
  t->cur = next;
  t->cur_n = (size_t)total;
  return true;
}

bool dtree_lists(DeviceTree* t, int nb, const double* X, const double* dL, const double* off, const int* cb, const int* ce,
                 const int* children, int n_children, double theta, std::vector<std::vector<int>>& near,
                 std::vector<std::vector<int>>& m2l) {
  cudaStream_t s = t->stream;
  near.assign(nb, {});
  m2l.assign(nb, {});
  if (nb <= 0) return true;
  for (int i = 0; i < nb; ++i)
    if (cb[i] < 0 || ce[i] < cb[i] || ce[i] - cb[i] > 8 || ce[i] > n_children) return false;
  for (int i = 0; i < n_children; ++i)
    if (children[i] < 0 || children[i] >= nb) return false;
  if (!t->nX.fit((size_t)3 * nb) || !t->ndL.fit(nb) || !t->noff.fit(nb) || !t->ncb.fit(nb) || !t->nce.fit(nb) ||
      !t->nch.fit((size_t)std::max(n_children, 1)))
    return false;
  if (cudaMemcpyAsync(t->nX.p, X, sizeof(double) * 3 * nb, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(t->ndL.p, dL, sizeof(double) * nb, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(t->noff.p, off, sizeof(double) * nb, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(t->ncb.p, cb, sizeof(int) * nb, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(t->nce.p, ce, sizeof(int) * nb, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      (n_children && cudaMemcpyAsync(t->nch.p, children, sizeof(int) * n_children, cudaMemcpyHostToDevice, s) != cudaSuccess))
    return false;
  const NodeGeo g{t->nX.p, t->ndL.p, t->noff.p, t->ncb.p, t->nce.p, t->nch.p};
  // level 1: every child of the root against every child of the root, in order
  std::vector<int> tg(children + cb[0], children + ce[0]), coff(1, 0), cd;
  for (size_t i = 0; i < tg.size(); ++i) {
    cd.insert(cd.end(), children + cb[0], children + ce[0]);
    coff.push_back((int)cd.size());
  }
  while (!tg.empty()) {
    const int n = (int)tg.size();
    if (!t->lt.fit(n) || !t->lco.fit((size_t)n + 1) || !t->lc.fit(std::max<size_t>(cd.size(), 1)) || !t->lcnt.fit((size_t)17 * n) ||
        !t->loff.fit((size_t)17 * n + 1))
      return false;
    if (cudaMemcpyAsync(t->lt.p, tg.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
        cudaMemcpyAsync(t->lco.p, coff.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, s) != cudaSuccess ||
        (!cd.empty() && cudaMemcpyAsync(t->lc.p, cd.data(), sizeof(int) * cd.size(), cudaMemcpyHostToDevice, s) != cudaSuccess))
      return false;
    const int blocks = (n + 3) / 4;  // 4 warps per block
    int* cnt = t->lcnt.p;
    t->launches += 2;
    k_lists<false><<<blocks, 128, 0, s>>>(n, t->lt.p, t->lco.p, t->lc.p, g, theta, cnt, cnt + n, cnt + 9 * n, nullptr, nullptr, nullptr,
                                          nullptr, nullptr, nullptr);
    if (cudaGetLastError() != cudaSuccess) return false;
    std::vector<int> hc((size_t)17 * n);
    if (cudaMemcpyAsync(hc.data(), cnt, sizeof(int) * 17 * n, cudaMemcpyDeviceToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
      return false;
    // offsets: near per target, m2l and next candidates per (target, child slot)
    std::vector<int> ho((size_t)17 * n);
    int tn = 0, tm = 0, tx = 0;
    for (int w = 0; w < n; ++w) {
      ho[w] = tn;
      tn += hc[w];
    }
    for (int i = 0; i < 8 * n; ++i) {
      ho[n + i] = tm;
      tm += hc[n + i];
      ho[9 * n + i] = tx;
      tx += hc[9 * n + i];
    }
    if (!t->lno.fit(std::max(tn, 1)) || !t->lmo.fit(std::max(tm, 1)) || !t->lxo.fit(std::max(tx, 1))) return false;
    if (cudaMemcpyAsync(t->loff.p, ho.data(), sizeof(int) * 17 * n, cudaMemcpyHostToDevice, s) != cudaSuccess) return false;
    k_lists<true><<<blocks, 128, 0, s>>>(n, t->lt.p, t->lco.p, t->lc.p, g, theta, nullptr, nullptr, nullptr, t->loff.p, t->loff.p + n,
                                         t->loff.p + 9 * n, t->lno.p, t->lmo.p, t->lxo.p);
    if (cudaGetLastError() != cudaSuccess) return false;
    std::vector<int> hn(tn), hm(tm), hx(tx);
    if ((tn && cudaMemcpyAsync(hn.data(), t->lno.p, sizeof(int) * tn, cudaMemcpyDeviceToHost, s) != cudaSuccess) ||
        (tm && cudaMemcpyAsync(hm.data(), t->lmo.p, sizeof(int) * tm, cudaMemcpyDeviceToHost, s) != cudaSuccess) ||
        (tx && cudaMemcpyAsync(hx.data(), t->lxo.p, sizeof(int) * tx, cudaMemcpyDeviceToHost, s) != cudaSuccess) ||
        cudaStreamSynchronize(s) != cudaSuccess)
      return false;
    std::vector<int> ntg, ncoff(1, 0), ncd;
    for (int w = 0; w < n; ++w) {
      const int x = tg[w];
      near[x].insert(near[x].end(), hn.begin() + ho[w], hn.begin() + ho[w] + hc[w]);
      for (int sl = 0; sl < ce[x] - cb[x]; ++sl) {
        const int ac = children[cb[x] + sl], i = 8 * w + sl;
        m2l[ac].insert(m2l[ac].end(), hm.begin() + ho[n + i], hm.begin() + ho[n + i] + hc[n + i]);
        if (hc[9 * n + i] == 0) continue;
        ntg.push_back(ac);
        ncd.insert(ncd.end(), hx.begin() + ho[9 * n + i], hx.begin() + ho[9 * n + i] + hc[9 * n + i]);
        ncoff.push_back((int)ncd.size());
      }
    }
    tg.swap(ntg);
    coff.swap(ncoff);
    cd.swap(ncd);
  }
  return true;
}

int dtree_take_launches(DeviceTree* t) {
  const int n = t ? t->launches : 0;
  if (t) t->launches = 0;
  return n;
}

bool dtree_download(DeviceTree* t, int* out, size_t count) {
  if (count > t->cur + t->cur_n) return false;
  if (count && cudaMemcpyAsync(out, t->elems.p, sizeof(int) * count, cudaMemcpyDeviceToHost, t->stream) != cudaSuccess) return false;
  return cudaStreamSynchronize(t->stream) == cudaSuccess;
}

}  // namespace bemb200
