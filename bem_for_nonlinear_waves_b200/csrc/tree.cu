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
#include <vector>

#include "tree_dev.hpp"

namespace bemb200 {
namespace {

// per splitting bucket: parent geometry then the 8 children's (xmin[3], inv_dL, size[3]) as
// doubles, 7 + 8 * 7 values
constexpr int kGeo = 7 * 9;

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

// one CTA per splitting bucket: cell and inside flag of each element; counts per cell
__global__ void __launch_bounds__(256) k_tree_count(const int* __restrict__ seg_beg, const int* __restrict__ seg_end,
                                                    const double* __restrict__ geo, const int* __restrict__ elems,
                                                    const double* __restrict__ poles, int tag_base, uint8_t* __restrict__ tag,
                                                    int* __restrict__ cnt_all, int* __restrict__ cnt_pass) {
  __shared__ double g[kGeo];
  __shared__ int ca[8], cp[8];
  const int node = blockIdx.x;
  for (int i = threadIdx.x; i < kGeo; i += blockDim.x) g[i] = geo[(size_t)node * kGeo + i];
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

// stable scatter of the kept elements of each (bucket, cell) to off[bucket * 8 + cell] onwards
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
  Buf<int> elems, seg_beg, seg_end, cnt, off;  // elems: every level's array, back to back
  Buf<uint8_t> tag;
  size_t cur = 0, cur_n = 0;  // current level: offset into elems, length
  std::vector<int> h_beg, h_end;
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
  if (!t->seg_beg.fit(n) || !t->seg_end.fit(n) || !t->geo.fit((size_t)n * kGeo) || !t->cnt.fit((size_t)16 * n) || !t->off.fit((size_t)8 * n))
    return false;
  t->h_beg.assign(seg_beg, seg_beg + n);
  t->h_end.assign(seg_end, seg_end + n);
  for (int i = 0; i < n; ++i) {  // segments are offsets into the current level's array
    if (seg_beg[i] < 0 || seg_end[i] < seg_beg[i] || (size_t)seg_end[i] > t->cur_n) return false;
    t->h_beg[i] += (int)t->cur;
    t->h_end[i] += (int)t->cur;
  }
  if (cudaMemcpyAsync(t->seg_beg.p, t->h_beg.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(t->seg_end.p, t->h_end.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(t->geo.p, geo, sizeof(double) * kGeo * n, cudaMemcpyHostToDevice, s) != cudaSuccess)
    return false;
  // tags are indexed by position in the elems buffer relative to the current level
  k_tree_count<<<n, 256, 0, s>>>(t->seg_beg.p, t->seg_end.p, t->geo.p, t->elems.p, t->poles.p, (int)t->cur, t->tag.p, t->cnt.p,
                                 t->cnt.p + 8 * n);
  if (cudaGetLastError() != cudaSuccess) return false;
  if (cudaMemcpyAsync(cnt_all, t->cnt.p, sizeof(int) * 8 * n, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaMemcpyAsync(cnt_pass, t->cnt.p + 8 * n, sizeof(int) * 8 * n, cudaMemcpyDeviceToHost, s) != cudaSuccess)
    return false;
  return cudaStreamSynchronize(s) == cudaSuccess;
}

bool dtree_scatter(DeviceTree* t, int n, const int* off, int total) {
  cudaStream_t s = t->stream;
  const size_t next = t->cur + t->cur_n;
  if (next + (size_t)total > t->elems.cap) return false;
  if (n > 0) {
    std::vector<int> o(off, off + 8 * (size_t)n);
    for (auto& v : o) {
      if (v < 0 || v > total) return false;
      v += (int)next;
    }
    if (cudaMemcpyAsync(t->off.p, o.data(), sizeof(int) * 8 * n, cudaMemcpyHostToDevice, s) != cudaSuccess) return false;
    k_tree_scatter<<<n, 256, 0, s>>>(t->seg_beg.p, t->seg_end.p, t->elems.p, (int)t->cur, t->tag.p, t->off.p, t->elems.p);
    if (cudaGetLastError() != cudaSuccess) return false;
    if (cudaStreamSynchronize(s) != cudaSuccess) return false;  // o is freed on return
  }
  t->cur = next;
  t->cur_n = (size_t)total;
  return true;
}

bool dtree_download(DeviceTree* t, int* out, size_t count) {
  if (count > t->cur + t->cur_n) return false;
  if (count && cudaMemcpyAsync(out, t->elems.p, sizeof(int) * count, cudaMemcpyDeviceToHost, t->stream) != cudaSuccess) return false;
  return cudaStreamSynchronize(t->stream) == cudaSuccess;
}

}  // namespace bemb200
