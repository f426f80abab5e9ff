// 2^N-tree build on the GPU (SpatialSubdivisionTree::decompose, src/painter/space/tree.h:327-387,
// 466-525): the same level-by-level construction as the host build, with every box-simplex overlap
// decided on the device by the same code (geometry.hpp), so the tree is the host's, node for node.
#pragma once

#include "geometry.hpp"

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace ntrace
{
struct TreeResult
{
        std::vector<int32_t> nodes;     // int2 per node: internal {first child, -1}, leaf {offset, count}
        std::vector<int32_t> leaf_idx;  // facet indices of the leaves, in node order
        long long leaf_count = 0;
        long long overlap_tests = 0;
        cudaError_t error = cudaSuccess;
        std::string message;
};

// shapes: the facets' overlap data; root_org and level_sizes ((max_depth + 1) x N) as the host build
// computes them; boxes with more than min_objects facets are split until max_depth.
template <int N>
void build_tree_gpu(const std::vector<SimplexShape<N, float>>& shapes, const Vec<N, float>& root_org,
                    const std::vector<float>& level_sizes, int max_depth, int min_objects, cudaStream_t st,
                    TreeResult* out);
}
