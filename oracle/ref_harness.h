/*
 * C API of the reference harness (test infrastructure only).
 *
 * ref_run() evaluates one iteration's estimator calls with the reference's
 * own estimator code (compiled from the reference sources by
 * oracle/build_ref.py into oracle/_ref/libupbp_ref.so), on the same arrays
 * the CUDA path consumes (include/upbp_gpu.h).  Only tests, the smoke check
 * and the CPU-baseline leg of bench.py load it.
 */
#ifndef UPBP_REF_HARNESS_H
#define UPBP_REF_HARNESS_H

#include <stdint.h>
#include "../include/upbp_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* what ref_run evaluates */
#define REF_PB2D 1        /* EmbreeBre::evalBre (Embree BVH, MIS callback)               */
#define REF_BB1D_GRID 2   /* PhotonBeamsEvaluator::evalBeamBeamEstimate, USE_GRID (default) */
#define REF_BB1D_BRUTE 4  /* same with the reference's brute-force AccelStruct (PhBrute.hxx) */
#define REF_PP3D 8        /* HashGrid::Process with UPBP::RangeQuery                      */
#define REF_CANDIDATES 16 /* per-query candidate counts and hashes                         */

typedef struct ref_outputs {
    float* pb2d_rgb;       /* [nq][3] */
    float* bb1d_rgb;       /* [nq][3] grid */
    float* bb1d_brute_rgb; /* [nq][3] brute force */
    float* pp3d_rgb;       /* [np][3] */
    uint32_t* count_pb2d; uint64_t* hash_pb2d;
    uint32_t* count_bb1d; uint64_t* hash_bb1d;
    uint32_t* count_pp3d; uint64_t* hash_pp3d;
    float* image;          /* [H*W][3], += mult * contrib for every evaluated estimator */
    double build_ms;       /* wall time of the structure builds */
    double gather_ms;      /* wall time of the query evaluation */
} ref_outputs;

/* Evaluate queries q with q % stride == 0 (stride >= 1; the others are left
 * untouched) on `threads` OpenMP threads (0 = all), each thread owning its
 * own copy of the structures as the reference keeps one renderer per thread.
 * Returns 0 on success. */
int ref_run(const upbp_params* params, const upbp_medium* media, int32_t n_media,
            const upbp_light_vertices* lv, const upbp_beams* beams,
            const upbp_mis* cam_mis, int64_t n_cam_mis,
            const upbp_segment_queries* sq, const upbp_point_queries* pq,
            int32_t what, int64_t stride, int32_t threads, ref_outputs* out);

/* The same in three steps, so that a caller can time the per-thread builds once and then
 * evaluate several query subsets (q = offset + k*stride) on the built structures. */
void* ref_prepare(const upbp_params* params, const upbp_medium* media, int32_t n_media,
                  const upbp_light_vertices* lv, const upbp_beams* beams, const upbp_mis* cam_mis,
                  const upbp_segment_queries* sq, const upbp_point_queries* pq, int32_t what, int32_t threads);
int ref_eval(void* session, int64_t offset, int64_t stride, ref_outputs* out);
void ref_release(void* session);

/* The reference's BB1D grid options, set from the command line in the renderer
 * (-gridres / -gridmax / -gridred, Misc/Config.hxx:1964-1966): statics of
 * PhotonBeamsEvaluator (Beams/PhBeams.cxx:44-46). */
void ref_set_grid_options(uint32_t grid_size, uint32_t max_beams_in_cell, uint32_t reduction_type);

#ifdef __cplusplus
}
#endif

#endif
