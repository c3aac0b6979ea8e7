// Host-side interface of the generic-precision gathers (upbp_generic.cu): the FP64 evaluation
// mode and the adjoint with respect to one medium's parameters.
#pragma once

#include <cuda_runtime.h>

#include "upbp_kernels.cuh"
#include "upbp_mis_prep.cuh"

namespace upbp {
namespace gen {

struct GenConsts {
    upbp_medium raw[UPBP_MAX_MEDIA];  // the media as given (sigma_a, sigma_s, g, continuation)
    int n_media;
    int grad_medium;                  // medium whose parameters carry tangents (adjoint), else -1
};

struct GenOut {
    float* rgb;                  // FP64 mode: per-query result [n][3] (rounded to FP32), or null
    float* image;                // FP64 mode: framebuffer [H*W][3], or null
    uint32_t* count;             // FP64 mode: accepted candidates per query, or null
    unsigned long long* hash;    // FP64 mode: order-independent candidate hash per query, or null
    const float* grad_image;     // adjoint: dL/d framebuffer [H*W][3]
    double* grad;                // adjoint: accumulated dL/d(sigma_a rgb, sigma_s rgb, g) [7]
};

struct GenLaunch {
    GatherConsts K;
    GenConsts G;
    LightSoA L;
    PhotonBVH photons;
    BeamBVH beams;
    BeamSoA bs;
    HashGridDev hash;
    SegQueriesDev sq;
    PointQueriesDev pq;
    const upbp_mis* cam;
    const CamSum* cs_seg;
    const CamSum* cs_pt;
    GenOut out_pb2d, out_bb1d, out_pp3d, out_bp2d;
    unsigned int* work;  // work counters, [0] BB1D, [1] PB2D and [2] B-P2D (zeroed by the caller)
    int* status;         // traversal status (zeroed by the caller)
    int bb1d_grid;
    int pb2d_grid;
    int bp2d_grid;
    const int32_t* order;  // segment queries in Morton order of their midpoints, or nullptr
};

void launch_generic(const GenLaunch& A, bool adjoint, cudaStream_t stream);
int generic_bb1d_blocks_per_sm(bool adjoint);
int generic_pb2d_blocks_per_sm(bool adjoint);
int generic_bp2d_blocks_per_sm(bool adjoint);

}  // namespace gen
}  // namespace upbp
