// ogx_tree_common.cuh -- device helpers shared by the tree and list kernels.
#pragma once

#include "ogx_internal.cuh"

namespace ogx {

// AdaptiveOctree::adjacent (src3d/AdaptiveOctree.hpp:58-62), same FP64 operation order
__device__ __forceinline__ bool adjacent64(const double* ctr, int a, int b, double tol) {
    const double s = __dadd_rn(__dadd_rn(ctr[4 * a + 3], ctr[4 * b + 3]), tol);
    return fabs(__dsub_rn(ctr[4 * a], ctr[4 * b])) <= s && fabs(__dsub_rn(ctr[4 * a + 1], ctr[4 * b + 1])) <= s &&
           fabs(__dsub_rn(ctr[4 * a + 2], ctr[4 * b + 2])) <= s;
}

// slot of a same-level neighbour at integer offset (ox, oy, oz) in [-1, 1]^3
__device__ __forceinline__ int colleague_slot(int ox, int oy, int oz) { return (ox + 1) + 3 * (oy + 1) + 9 * (oz + 1); }

}  // namespace ogx
