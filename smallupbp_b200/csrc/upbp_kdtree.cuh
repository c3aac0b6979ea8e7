// The reference's k-nearest-neighbour search for the KNN radii (upbp_kdtree.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "upbp_kernels.cuh"

namespace upbp {

// Builds the reference's kd-tree (Jensen's left-balanced tree, heap order, node 1 the root) over the
// n points pos[idx[i]] (idx NULL: pos[i]) in that order, bbox = their bounding box ([lo xyz, hi
// xyz]).  Scratch: org and tree n + 1 float4, boxes 6 (n + 1) floats, pa and pb n + 1 ints.
void launch_kd_build(const float4* pos, const int32_t* idx, int n, const float* bbox, float4* org, float4* tree,
                     float* boxes, int* pa, int* pb, cudaStream_t stream);
// number of kernels launch_kd_build launches for n points
int kd_build_launches(int n);
// PB2D photon radii^2 from the reference's search: query i at queries[i].xyz
void launch_kd_photon_r2(const float4* tree, int n, const float4* queries, int nq, int k, float r, float* r2,
                         cudaStream_t stream);
// BB1D beam radii from the reference's search, in three steps: the 2 nb query points (the beams'
// origins, then their end points), the searches in a given order of the points (a Morton order
// keeps a warp's walks alike; d2 indexed by point), and the start radius, radius change and max
// radius^2 of every beam
void launch_kd_beam_points(const float* origin, const float* dir, const float* length, int nb, float4* pts,
                           cudaStream_t stream);
void launch_kd_knn_sorted(const float4* tree, int n, const float4* pts, const int32_t* order, int nq, int k,
                          float* d2, cudaStream_t stream);
void launch_kd_beam_finish(const float* d2, const float* length, int nb, float r, float* rstart, float* rchange,
                           float* r2max, cudaStream_t stream);

}  // namespace upbp
