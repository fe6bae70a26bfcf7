// Octree growth on the device (tree.cu), driven level by level from plan.cpp.  No CUDA types:
// plan.cpp is host C++.
#pragma once
#include <cstddef>
#include <vector>

namespace bemb200 {

struct DeviceTree;
DeviceTree* dtree_create(void* stream);  // stream: a cudaStream_t
void dtree_destroy(DeviceTree* t);
// poles [3*nf]; the root bucket's elements in data order; levels below the root <= max_level
bool dtree_begin(DeviceTree* t, int nf, const double* poles, int n_root, const int* root_elems, int max_level);
// n splitting buckets of the current level: segments into the level's element array and the
// geometry of each (parent, then its 8 children: xmin[3], 1/dL, size[3]); per (bucket, cell)
// the elements of the cell (cnt_all) and those the child keeps (cnt_pass)
bool dtree_count(DeviceTree* t, int n, const int* seg_beg, const int* seg_end, const double* geo, int* cnt_all, int* cnt_pass);
// the next level's array: kept elements of (bucket, cell) at off[bucket * 8 + cell], stable
bool dtree_scatter(DeviceTree* t, int n, const int* off, int total);
// interaction lists of lists() (moments.hpp:967-997) from the level-1 pairs, level by level on
// the device: near[x], m2l[x] in the order the reference's recursion appends them.  Nodes in
// creation order; children[cb[i] .. ce[i]) in cell order (at most 8)
bool dtree_lists(DeviceTree* t, int nb, const double* X, const double* dL, const double* off, const int* cb, const int* ce,
                 const int* children, int n_children, double theta, std::vector<std::vector<int>>& near,
                 std::vector<std::vector<int>>& m2l);
// kernels launched since the last call (octree growth and lists)
int dtree_take_launches(DeviceTree* t);
// every level's array, back to back from the root's
bool dtree_download(DeviceTree* t, int* out, size_t count);

}  // namespace bemb200
