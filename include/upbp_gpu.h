/*
 * upbp_gpu.h -- C ABI of the B200 volumetric estimator stage (PP3D, PB2D, BB1D).
 *
 * This is the drop-in boundary for SmallUPBP's estimator interface.  The
 * reference renderer calls, per iteration,
 *
 *   HashGrid::Reserve/Build            (Misc/HashGrid.hxx:41-126)      PP3D build
 *   EmbreeBre::build                   (Bre/Bre.hxx:93-99, Bre.cxx:649-755)  PB2D build
 *   PhotonBeamsEvaluator::build        (Beams/PhBeams.hxx:71-76, PhBeams.cxx:66-148) BB1D build
 *   EmbreeBre::evalBre                 (Bre/Bre.hxx:125-131, Bre.cxx:812-964) per camera segment
 *   PhotonBeamsEvaluator::evalBeamBeamEstimate (PhBeams.hxx:96-113, PhBeams.cxx:177-324) per camera segment
 *   HashGrid::Process + UPBP::RangeQuery (HashGrid.hxx:129-188, Renderers/UPBP.hxx:86-133) per camera medium vertex
 *   EmbreeBre::destroy / PhotonBeamsEvaluator::destroy (UPBP.hxx:1172-1181)
 *
 * one query at a time and adds each returned Rgb into the pixel colour
 * (UPBP.hxx:782-783, 795-796, 890-891, 908-909, 1120; Framebuffer::AddColor
 * at UPBP.hxx:1162).  No control flow depends on the returned value, so the
 * calls can be RECORDED during the camera pass and evaluated in one batch at
 * the end of the iteration: that batch is what this library evaluates.
 *
 * Data crosses the boundary as plain arrays (host or device pointers; the
 * library copies them).  The light-vertex, beam and MIS records carry exactly
 * the fields the reference estimators read from UPBPLightVertex
 * (Path/UPBPLightVertex.hxx:32-78), PhotonBeam (Beams/PhotonBeam.hxx:40-64),
 * VolumeSegment (Path/Ray.hxx:131-227) and AdditionalRayDataForMis
 * (embree-2.0/embree/common/ray.h:31-99).
 *
 * Every entry point returns an int status: UPBP_OK (0) or a negative
 * UPBP_ERR_* code; upbp_last_error() gives the message.  The reference has no
 * error returns (it calls exit(2) on failed asserts, Misc/Defs.hxx:96-97).
 * One context per host thread, as the reference keeps one renderer (and so
 * one set of estimator structures) per OpenMP thread (SmallUPBP.cxx:66-79).
 */
#ifndef UPBP_GPU_H
#define UPBP_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define UPBP_OK 0
#define UPBP_ERR_INVALID_ARG (-1)
#define UPBP_ERR_OUT_OF_MEMORY (-2)
#define UPBP_ERR_CUDA (-3)
#define UPBP_ERR_NOT_BUILT (-4)
#define UPBP_ERR_WATCHDOG (-5)
#define UPBP_ERR_CAPACITY (-6)

/* ---- flags: values identical to the reference enums (Misc/Defs.hxx:140-194,
 *      Scene/Media.hxx:44-48) ------------------------------------------- */
#define UPBP_SHORT_BEAM 1u
#define UPBP_LONG_BEAM 2u
#define UPBP_BPT 4u
#define UPBP_SURF 8u
#define UPBP_PP3D 16u
#define UPBP_PB2D 32u
#define UPBP_BB1D 64u
#define UPBP_NO_SINE_IN_WEIGHTS 128u
#define UPBP_PREVIOUS 256u
#define UPBP_COMPATIBLE 512u
#define UPBP_BB1D_PREVIOUS 1024u
#define UPBP_BP2D 65536u /* extension, not a reference technique (above every reference flag; 2048 is
                         * SPECULAR_ONLY): B-P2D, photon beams x camera medium points with a 2-D
                         * kernel, as a standalone estimator with MIS weight 1 */
/* Estimators without MIS, as VolLightTracer's pure algorithms run them (`-a pb2d`, `-a bb1d`,
 * Renderers/VolLightTracer.hxx:296-412): EmbreeBre::build over VltLightVertex records
 * (Bre.cxx:526-614) with evalBre and no AdditionalRayDataForMis, whose photons take the callback
 * breIntersectFuncHomogeneous (Bre.cxx:239-291), and evalBeamBeamEstimate(..., BB1D, 0, NULL),
 * which takes PhotonBeam::accumulate (Beams/PhotonBeam.hxx:315-367).  Every candidate then adds
 * its unweighted contribution: no path-length or minimum-distance rejects and no MIS weight.  The
 * caller sets norm_pb2d = 1 / mLightSubPathCount, norm_bb1d = 1 / mBB1DUsedLightSubPathCount and
 * the query throughput to 1 (VolLightTracer.hxx:378, 384).  The MIS inputs may then be NULL:
 * upbp_light_vertices.mis, path_idx, cont_prob and path_ends (n_paths 0); upbp_beams.ray_sample_pdf,
 * ray_sample_rev_pdf, ray_sampling_flags, last_pdf_w_inv and light_vertex; upbp_segment_queries
 * .last_pdf_w_inv and cam_mis_begin; and no camera MIS records.  The reference has no pure PP3D
 * algorithm: UPBP_PP3D together with this bit is rejected.  (Not a reference flag: above every
 * reference flag and UPBP_BP2D.) */
#define UPBP_NO_MIS 131072u
#define UPBP_ORIGIN_IN_MEDIUM 1u /* AbstractMedium::kOriginInMedium */
#define UPBP_END_IN_MEDIUM 2u    /* AbstractMedium::kEndInMedium */

/* upbp_mis.flags bits (the four bools of MisData) */
#define UPBP_MIS_IS_DELTA 1u
#define UPBP_MIS_ON_LIGHT_SOURCE 2u
#define UPBP_MIS_IS_SPECULAR 4u
#define UPBP_MIS_IN_MEDIUM_WITH_BEAMS 8u

/* light-vertex flags */
#define UPBP_LV_IN_MEDIUM 1u
#define UPBP_LV_CONNECTABLE 2u
#define UPBP_LV_IS_FINITE 4u

/* segment-query flags */
#define UPBP_Q_ORIGIN_IN_MEDIUM 1u /* raySamplingFlags of the call */
#define UPBP_Q_LITE 2u             /* segments are LiteVolumeSegments: pdfs and attenuation come from the medium */
#define UPBP_Q_PB2D 4u             /* evaluate evalBre for this segment */
#define UPBP_Q_BB1D 8u             /* evaluate evalBeamBeamEstimate for this segment */

/* evaluation modes */
#define UPBP_MODE_PLAIN 0 /* all-FP32, MIS walks the stored subpaths per candidate (reference order) */
#define UPBP_MODE_MIXED 1 /* FP32 bulk, FP64 near-parallel BB1D solve and FP64 MIS suffix sums */
#define UPBP_MODE_FP64 2  /* FP64 oracle on the GPU: the same FP32 candidate predicates, candidate
                                * geometry re-solved in FP64, all contribution and MIS arithmetic FP64 */

/* ---- records ------------------------------------------------------------ */

/* Homogeneous medium (Scene/Media.hxx:129-159).  Derived quantities
 * (sigma_t, min positive sigma_t component, MFP) are computed by the library
 * exactly as the reference constructor does. */
typedef struct upbp_medium {
    float absorption[3];     /* sigma_a */
    float scattering[3];     /* sigma_s */
    float mean_cosine;       /* HG g */
    float continuation_prob; /* MEDIUM_SURVIVAL_PROB 0.8 for scene media, 1.0 for the clear medium */
} upbp_medium;

/* MisData (Path/UPBPLightVertex.hxx:32-52): 14 floats + 4 bools as flags. 60 bytes. */
typedef struct upbp_mis {
    float pdf_a_inv;
    float rev_pdf_a;
    float rev_pdf_a_without_bsdf;
    float ray_sample_pdf_inv;
    float ray_sample_rev_pdf_inv;
    float ray_sample_pdfs_ratio;
    float ray_sample_rev_pdfs_ratio;
    float sin_theta;
    float cos_theta_out;
    float surf_factor;
    float pp3d_factor;
    float pb2d_factor;
    float bb1d_factor;
    float bb1d_beam_selection_pdf;
    uint32_t flags; /* UPBP_MIS_* */
} upbp_mis;

/* Per-iteration constants (Renderers/UPBP.hxx:415-460) and options. */
typedef struct upbp_params {
    uint32_t techniques;        /* mEstimatorTechniques: UPBP_BPT|SURF|PP3D|PB2D|BB1D|NO_SINE|PREVIOUS|BB1D_PREVIOUS */
    uint32_t query_beam_type;   /* mQueryBeamType  */
    uint32_t photon_beam_type;  /* mPhotonBeamType */
    uint32_t min_path_length;
    uint32_t max_path_length;
    float radius_pp3d;
    float radius_pb2d;
    float radius_bb1d;
    float mis_factor_surf;      /* etaSurf */
    float mis_factor_pp3d;      /* etaPP3D */
    float mis_factor_pb2d;      /* etaPB2D */
    float mis_factor_bb1d;      /* etaBB1D */
    float norm_pp3d;            /* mPP3DNormalization */
    float norm_pb2d;            /* mPB2DNormalization */
    float norm_bb1d;            /* mBB1DNormalization */
    float bb1d_min_mfp;         /* mBB1DMinMFP */
    float min_dist_to_med;      /* mMinDistToMed */
    int32_t hash_cells;         /* PP3D HashGrid::Reserve(pathCountL) */
    int32_t image_width;
    int32_t image_height;
    /* KNN radii (RadiusCalculation KNN_RADIUS): 0 = constant radius.  k > 0: each PB2D photon's
     * radius is radius_pb2d * 2 * (distance to its k-th nearest photon, itself included)
     * (EmbreeBre::build, Bre.cxx:685-725); each beam's start / end radius is
     * max(2 * (distance from its origin / end to the k-th nearest beam origin) * radius_bb1d, 0.001),
     * varying linearly along the beam (PhotonBeamsEvaluator::build, PhBeams.cxx:72-123). */
    int32_t pb2d_knn;           /* mPB2DRadiusKNN when mPB2DRadiusCalculation == KNN_RADIUS, else 0 */
    int32_t bb1d_knn;           /* mBB1DRadiusKNN when mBB1DRadiusCalculation == KNN_RADIUS, else 0 */
    /* How the KNN radii find "the k-th nearest": 0 (default) as the reference does, with its
     * kd-tree search (KdTreeTmplPtr::KNNQuery, Misc/KdTmpl.hxx), so that the radii equal the
     * reference's bit for bit; that search is approximate (its heap bound stays unset until k points
     * are held, the (k+1)-th then replaces the farthest whatever its distance, and its descent treats
     * the nodes from n/2 - 1 on as leaves).  1: the exact distance to the k-th nearest point. */
    int32_t knn_exact;
} upbp_params;

/* Light vertices (mLightVertices): n entries, stored per light path in
 * increasing path length, path p occupying [path_ends[p-1], path_ends[p]). */
typedef struct upbp_light_vertices {
    int64_t n;
    const float* position;   /* [n][3] mHitpoint */
    const float* throughput; /* [n][3] mThroughput */
    const float* dir_fix;    /* [n][3] mBSDF.WorldDirFix() */
    const float* cont_prob;  /* [n]    mBSDF.ContinuationProb() */
    const int32_t* path_idx;    /* [n] mPathIdx */
    const int32_t* path_length; /* [n] mPathLength */
    const int32_t* medium_id;   /* [n] medium of mBSDF (-1 on surface) */
    const uint32_t* flags;      /* [n] UPBP_LV_* */
    const upbp_mis* mis;        /* [n] mMisData */
    int32_t n_paths;
    const int32_t* path_ends;   /* [n_paths] mPathEnds */
} upbp_light_vertices;

/* Photon beams (mPhotonBeamsArray, filled by UPBP::AddBeams, UPBP.hxx:1783-1870). */
typedef struct upbp_beams {
    int64_t n;
    const float* origin;          /* [n][3] mRay.origin */
    const float* direction;       /* [n][3] mRay.direction */
    const float* length;          /* [n] mLength */
    const float* throughput;      /* [n][3] mThroughputAtOrigin */
    const uint32_t* flags;        /* [n] mFlags (SHORT/LONG) */
    const float* ray_sample_pdf;  /* [n] mRaySamplePdf */
    const float* ray_sample_rev_pdf; /* [n] mRaySampleRevPdf */
    const uint32_t* ray_sampling_flags; /* [n] mRaySamplingFlags */
    const float* last_pdf_w_inv;  /* [n] mLastPdfWInv */
    const int32_t* medium_id;     /* [n] mMedium */
    const int32_t* light_vertex;  /* [n] mLightVertex as an index into the light vertices */
} upbp_beams;

/* Camera segment queries: one entry per evalBre/evalBeamBeamEstimate call
 * pair at a camera path length L.  cam_mis[cam_mis_begin .. +L) is the
 * snapshot of mCameraVerticesMisData[0..L-1] taken at the call. */
typedef struct upbp_segment_queries {
    int64_t n;
    const float* origin;        /* [n][3] ray.origin */
    const float* direction;     /* [n][3] ray.direction */
    const int32_t* seg_begin;   /* [n] first segment in the segment arrays */
    const int32_t* seg_count;   /* [n] number of segments */
    const uint32_t* flags;      /* [n] UPBP_Q_* */
    const int32_t* path_length; /* [n] cameraState.mPathLength */
    const float* last_pdf_w_inv;/* [n] cameraState.mLastPdfWInv */
    const float* throughput;    /* [n][3] cameraState.mThroughput */
    const int32_t* pixel;       /* [n] framebuffer index (y*W+x) or -1 */
    const int64_t* cam_mis_begin; /* [n] */
    int64_t n_segments;
    const float* seg_dist_min;  /* [s] mDistMin */
    const float* seg_dist_max;  /* [s] mDistMax */
    const float* seg_pdf;       /* [s] mRaySamplePdf */
    const float* seg_rev_pdf;   /* [s] mRaySampleRevPdf */
    const float* seg_attenuation; /* [s][3] mAttenuation */
    const int32_t* seg_medium;  /* [s] mMediumID */
} upbp_segment_queries;

/* Camera point queries (PP3D RangeQuery at a camera medium vertex).
 * cam_mis[cam_mis_begin .. +L+1) is mCameraVerticesMisData[0..L]. */
typedef struct upbp_point_queries {
    int64_t n;
    const float* position;      /* [n][3] hitPoint */
    const float* dir_fix;       /* [n][3] camera bsdf WorldDirFix */
    const int32_t* medium_id;   /* [n] camera bsdf medium */
    const int32_t* path_length; /* [n] cameraState.mPathLength */
    const float* throughput;    /* [n][3] cameraState.mThroughput */
    const int32_t* pixel;       /* [n] */
    const int64_t* cam_mis_begin; /* [n] */
} upbp_point_queries;

/* Per-query candidate statistics for candidate-set parity.  A candidate is a
 * (query, photon|beam) pair that passes the reference's geometric test:
 * testIntersectionBre (Bre.cxx:199-223) for PB2D, testIntersectionBeamBeam
 * plus same medium and radius >= distance (PhotonBeam.hxx:238-296, 390-413)
 * for BB1D, and distSqr <= r^2 over the 8 hashed cells (HashGrid.hxx:177-185,
 * counted with multiplicity) for PP3D.  hash = sum over candidates of
 * mix64(id) (wrapping), which is order independent. */
typedef struct upbp_query_stats {
    uint32_t* count_pb2d; uint64_t* hash_pb2d; /* [n_segment_queries] or NULL */
    uint32_t* count_bb1d; uint64_t* hash_bb1d; /* [n_segment_queries] or NULL */
    uint32_t* count_pp3d; uint64_t* hash_pp3d; /* [n_point_queries]  or NULL */
} upbp_query_stats;

typedef struct upbp_ctx upbp_ctx;

/* ---- entry points ------------------------------------------------------- */

/* Create a context on CUDA device `device`.  Replaces the construction of
 * EmbreeBre(scene) / PhotonBeamsEvaluator(scene) / HashGrid in the UPBP ctor
 * (Renderers/UPBP.hxx:160-216). */
int upbp_ctx_create(upbp_ctx** out, int device);
/* Replaces EmbreeBre::~EmbreeBre / PhotonBeamsEvaluator destructor. */
int upbp_ctx_destroy(upbp_ctx* ctx);
const char* upbp_last_error(const upbp_ctx* ctx);

/* Evaluation mode (UPBP_MODE_*). */
int upbp_set_mode(upbp_ctx* ctx, int mode);
/* Tunables (picked by smallupbp_b200.autotune): LBVH leaf sizes (powers of two), the block size
 * of the thread-per-query gathers, the BB1D beam-piece length in beam radii, and the BB1D
 * gather variant (0: thread per query, 1: warp-cooperative persistent work queue at 6 blocks of
 * 4 warps per SM, 2: the same kernel compiled for 7 blocks per SM, 3 and 4: one persistent
 * work-queue kernel for all camera segments that evaluates PB2D and BB1D per query, at 5 or 6
 * blocks per SM; the PB2D phase of upbp_last_timings is then 0 and the BB1D phase covers both).
 * pb2d_kernel picks the PB2D gather when it runs on its own (bb1d_kernel 0-2), and the B-P2D
 * gather (bb1d_kernel 1-4): 0 one thread per query, 1 one warp per query from a persistent work
 * queue with the candidate queue.
 * Defaults: photon leaves of 4, beam-piece leaves of 8, 128 threads, pieces of 6 radii, variant 2,
 * PB2D variant 1. */
typedef struct upbp_tuning {
    int32_t pb2d_leaf;
    int32_t bb1d_leaf;
    int32_t block_threads;
    float beam_piece_radii;
    int32_t bb1d_kernel;
    int32_t pb2d_kernel;
    /* order in which the persistent gathers draw the segment queries: 0 along a Morton curve of
     * their midpoints; 1 the camera rays (path length 1) along a Morton curve of their pixels,
     * then the other segments by midpoint; 2 along a 5-D Morton curve of midpoint and direction */
    int32_t query_order;
} upbp_tuning;
int upbp_set_tuning(upbp_ctx* ctx, const upbp_tuning* tuning);
int upbp_get_tuning(const upbp_ctx* ctx, upbp_tuning* tuning);

/* BB1D over the reference's uniform grid of beams (Beams/PhGrid.hxx, Beams/Grid.hxx: the
 * evaluator of the reference's default USE_GRID build, PhBeams.hxx:30-34) instead of the LBVH over
 * beam pieces.  The grid has the reference's resolution, cell lists and cell order, and its DDA
 * walk tests the beams of each visited cell with the query restricted to the cell's t range
 * (Grid.hxx:322-398), so a pair whose closest point lies on a cell boundary is found in both cells
 * or in neither, as in the reference.  Optionally the reference's beam reduction (-gridmax,
 * -gridred; Grid.hxx:453-631) tests max_beams_in_cell beams of each over-full cell and divides the
 * contribution by the cell's selection pdf max_beams / beams.  The build's draws are the
 * reference's own (std::mt19937_64 seeded with `seed`, through std::uniform_real_distribution<float>
 * as libstdc++ defines it): PRESAMPLE (0, the reference's default) is reproduced exactly, and
 * OFFSET (1) shuffles each over-full cell as the reference does.  The per-query draws of OFFSET,
 * RESAMPLE_FIXED (2) and SAMPLED (3) come in the reference from the same stream in the order the
 * queries are made, which a parallel evaluation cannot follow; here they are a function of (seed,
 * query, segment, cell, draw) with the same distributions.  As in the reference
 * (Config.hxx:1111-1112), the reduction is for the estimator without MIS (UPBP_NO_MIS) only.
 * Plain and mixed modes (not UPBP_MODE_FP64, not the adjoint).  The grid build reads its sizes
 * on the host (three synchronisations: the cell entries, the unique ones, the random draws); a
 * CUDA graph from upbp_capture_graph replays the build with the sizes of the build before it.
 * grid_res 0 (the default) switches the grid off. */
typedef struct upbp_bb1d_grid {
    uint32_t grid_res;          /* -gridres: PhotonBeamsEvaluator::sGridSize (reference default 256) */
    uint32_t max_beams_in_cell; /* -gridmax: sMaxBeamsInCell (0: no reduction) */
    uint32_t reduction;         /* -gridred: sReductionType (0 PRESAMPLE, 1 OFFSET, 2 RESAMPLE_FIXED, 3 SAMPLED) */
    int32_t seed;               /* PhotonBeamsEvaluator::mSeed (UPBP.hxx:417: base seed + iteration) */
} upbp_bb1d_grid;
int upbp_set_bb1d_grid(upbp_ctx* ctx, const upbp_bb1d_grid* grid);
/* CUDA stream (cudaStream_t as void*) used by all later calls; NULL = the context's own stream. */
int upbp_set_stream(upbp_ctx* ctx, void* stream);

/* Scene media table: scene.mMedia (Scene/Scene.hxx).  Replaces the
 * `scene` member read by EmbreeBre / PhotonBeamsEvaluator. */
int upbp_set_media(upbp_ctx* ctx, const upbp_medium* media, int32_t n_media);
/* Per-iteration constants (Renderers/UPBP.hxx:415-460). */
int upbp_set_params(upbp_ctx* ctx, const upbp_params* params);

/* Upload mLightVertices + mPathEnds.  Together with upbp_build this replaces
 * HashGrid::Reserve/Build (UPBP.hxx:699-704) and EmbreeBre::build
 * (Bre.cxx:649-755). */
int upbp_set_light_vertices(upbp_ctx* ctx, const upbp_light_vertices* lv);
/* Upload mPhotonBeamsArray.  With upbp_build replaces
 * PhotonBeamsEvaluator::build (PhBeams.cxx:66-148). */
int upbp_set_beams(upbp_ctx* ctx, const upbp_beams* beams);
/* Build every acceleration structure for the uploaded photons and beams:
 * PP3D hash grid, PB2D photon LBVH, BB1D beam LBVH, MIS suffix sums. */
int upbp_build(upbp_ctx* ctx);

/* Upload the recorded camera MIS snapshots and queries of this iteration. */
int upbp_set_camera_mis(upbp_ctx* ctx, const upbp_mis* records, int64_t n_records);
int upbp_set_segment_queries(upbp_ctx* ctx, const upbp_segment_queries* q);
int upbp_set_point_queries(upbp_ctx* ctx, const upbp_point_queries* q);

/* Evaluate all recorded queries: the batched equivalent of every
 * evalBre / evalBeamBeamEstimate / HashGrid::Process call of the iteration,
 * with the contributions splatted into the device framebuffer
 * (color += throughput * normalisation * contrib, UPBP.hxx:782-796, 890-909, 1120). */
int upbp_evaluate(upbp_ctx* ctx);

/* Results. */
int upbp_read_segment_results(upbp_ctx* ctx, float* pb2d_rgb, float* bb1d_rgb); /* [n][3] each, may be NULL */
int upbp_read_point_results(upbp_ctx* ctx, float* pp3d_rgb);                    /* [n][3] */
int upbp_read_query_stats(upbp_ctx* ctx, const upbp_query_stats* stats);
/* CUDA graph of one iteration's estimator stage: upbp_capture_graph records clear image + build
 * + evaluate for the inputs of the last upbp_build / upbp_evaluate (which must have run, so that
 * every buffer is sized and the photon and beam-piece counts are known) without executing it;
 * upbp_launch_graph replays it on the context's stream, asynchronously, with the same results
 * as those three calls.  Any upload, upbp_set_* or reallocation discards the graph (launch then
 * returns UPBP_ERR_NOT_BUILT).  The stream must not be the legacy default stream. */
int upbp_capture_graph(upbp_ctx* ctx);
int upbp_launch_graph(upbp_ctx* ctx);

/* Adjoint of the estimator sum with respect to the parameters of media[medium]: given
 * grad_image = dL/d(framebuffer) ([H*W][3] floats, host or device pointer), writes
 * grad[0..6] = dL/d(sigma_a r,g,b, sigma_s r,g,b, g) for the structures and queries of the last
 * build / upload, holding the candidate sets and the choice of the minimal sigma_t component
 * fixed.  Transmittance is recomputed, not stored.  Needs UPBP_MODE_MIXED or UPBP_MODE_FP64.
 * No counterpart in the reference (it has no derivatives); this is the backward of the
 * differentiable estimator (smallupbp_b200.autograd). */
int upbp_adjoint(upbp_ctx* ctx, const float* grad_image, int32_t medium, double* grad);

/* B-P2D results of the last evaluate (extension; needs UPBP_BP2D in params.techniques): per
 * point query the contribution [n][3] (before throughput and normalisation), the number of
 * accepted beams and the order-independent hash of their indices.  Any pointer may be NULL.
 * The point-query phase of upbp_last_timings (pp3d_ms) includes the B-P2D gather. */
int upbp_read_bp2d_results(upbp_ctx* ctx, float* rgb, uint32_t* count, uint64_t* hash);

/* Device memory the context holds (its grow-only buffers), in bytes. */
int upbp_device_bytes(const upbp_ctx* ctx, uint64_t* bytes);

/* Candidates tested by the last evaluate, summed over all queries: [0] PB2D photons, [1] BB1D beam
 * pieces, [2] PP3D photons (diagnostics of culling quality; accepted counts are in the query stats). */
int upbp_read_tested_counts(upbp_ctx* ctx, uint64_t* tested);
int upbp_clear_image(upbp_ctx* ctx); /* zeroes the framebuffer and the per-query results */
int upbp_read_image(upbp_ctx* ctx, float* rgb); /* [H*W][3] accumulated */
/* Device-side counters: number of kernels launched by the last upbp_build and upbp_evaluate. */
int upbp_last_launch_count(const upbp_ctx* ctx, int* build_launches, int* evaluate_launches);
/* Average duration (ms) of the last evaluate's dominant gather kernel, measured with CUDA events. */
int upbp_last_timings(const upbp_ctx* ctx, float* build_ms, float* pp3d_ms, float* pb2d_ms, float* bb1d_ms);

/* Allocation-free PP3D evaluation.  No counterpart in the reference: its HashGrid::Build and
 * HashGrid::Process with UPBP::RangeQuery (plain FP32 mode) for callers that cannot allocate
 * device memory -- a renderer plug-in inside a host application that owns the device memory
 * budget and forbids plug-ins to allocate, or an embedded caller that reserves all memory up
 * front.  All pointers inside lv / pq and cam_mis / out_rgb ([pq->n][3]) are device pointers the
 * caller owns; a null array for a non-empty count returns UPBP_ERR_INVALID_ARG; nothing is
 * allocated.  The scratch memory is one fixed array of about 18 MiB inside the library, held on
 * every GPU that loads it until the process exits; it limits lv->n to
 * UPBP_NOALLOC_MAX_LIGHT_VERTICES and params->hash_cells to UPBP_NOALLOC_MAX_HASH_CELLS (larger
 * sizes return UPBP_ERR_CAPACITY).  The first call on a device looks up that device's scratch
 * address, so make the first call before any stream capture.  The call reads the photon count and
 * the hash grid's bounds back to the host, so it waits for `stream`.  Every call shares the
 * scratch array: calls that overlap on the GPU (other streams, other host threads) race, so
 * serialise them.  stream = cudaStream_t or NULL. */
#define UPBP_NOALLOC_MAX_LIGHT_VERTICES (1 << 17)
#define UPBP_NOALLOC_MAX_HASH_CELLS (1 << 17)
int upbp_pp3d_evaluate_noalloc(const upbp_params* params, const upbp_medium* media, int32_t n_media,
                               const upbp_light_vertices* lv, const upbp_mis* cam_mis,
                               const upbp_point_queries* pq, float* out_rgb, void* stream);

/* ---- device-side light and camera passes -------------------------------- */

/* The estimator stage's inputs can also be produced on the device: the light pass of
 * UPBP::RunIteration (Renderers/UPBP.hxx:501-674, with UPBP::AddBeams :1783-1870) and its camera
 * pass (:742-1160), for scenes of nested axis-aligned boxes of homogeneous media with imaginary
 * boundaries, an area quad light and a pinhole camera.  The passes compute in FP64.  Random
 * numbers are per path: Philox4x64-10 with key (seed, iteration) and counter (path or pixel index,
 * bounce, block, stream 0 = light / 1 = camera), four uniforms (x >> 11) * 2^-53 per counter.
 * Light path p draws its emission from block 0 of bounce 0 (position x, position z, two
 * direction samples); the ray of bounce L (leaving vertex L-1) draws the free flight of its k-th
 * medium segment from block 1 + k / 4, word k % 4, and the scattering at vertex L its phase
 * function and Russian roulette samples from block 0, words 0-2.  Camera paths draw the pixel
 * jitter from block 0 of bounce 0, words 0-1, and bounce as light paths do. */
#define UPBP_MAX_BOXES 8
#define UPBP_SCENE_MAX_MEDIA 16

typedef struct upbp_scene_medium {
    double absorption[3];
    double scattering[3];
    double mean_cosine;
    double continuation_prob;
} upbp_scene_medium;

/* Box i+1 lies inside box i; a point takes the medium of the last box that contains it (bounds
 * included) and medium 0 outside every box.  The light is a square of side light_size centred on
 * the top face (y = box_hi[0][1]) of box 0, emitting with a cosine distribution downwards, with
 * radiance light_intensity.  The camera at camera_pos looks along +z, x right and y up, with a
 * horizontal field of view fov_deg over width pixels.  width, height, max_path_length and
 * techniques must equal the upbp_params given to upbp_set_params, which must come first (the
 * records take its MIS factors). */
typedef struct upbp_scene {
    int32_t n_media;
    upbp_scene_medium media[UPBP_SCENE_MAX_MEDIA];
    int32_t n_boxes;
    double box_lo[UPBP_MAX_BOXES][3];
    double box_hi[UPBP_MAX_BOXES][3];
    int32_t box_medium[UPBP_MAX_BOXES];
    double camera_pos[3];
    double fov_deg;
    int32_t width;
    int32_t height;
    int32_t light_paths;        /* N_L */
    int32_t max_path_length;    /* at most 16 */
    double light_size;
    double light_intensity;
    uint32_t techniques;        /* UPBP_PB2D decides where beams are stored (bb1d_min_mfp) */
    uint32_t query_beam_type;   /* UPBP_SHORT_BEAM / UPBP_LONG_BEAM */
    uint32_t photon_beam_type;
    double beam_length_cap;     /* cap on LONG photon beams beyond MaxBeamLength; +inf for none */
    double min_dist_to_med;     /* mMinDistToMed: no PP3D query at a first camera vertex closer than this */
    double bb1d_min_mfp;        /* mBB1DMinMFP */
    uint64_t seed;
} upbp_scene;

/* Trace the light sub-paths of iteration `iteration` on the device and store their light vertices
 * and photon beams in the context, as upbp_set_light_vertices and upbp_set_beams would: vertex
 * records per path in increasing path length, beams per path in the order AddBeams emits them. */
int upbp_trace_light_paths(upbp_ctx* ctx, const upbp_scene* scene, uint32_t iteration);
/* Trace the camera sub-paths (one per pixel) of iteration `iteration` on the device and store the
 * estimator calls they make, as upbp_set_camera_mis, upbp_set_segment_queries and
 * upbp_set_point_queries would: per pixel in call order, for each camera path length the segment
 * query, then the point query, each with its snapshot of the camera MIS records. */
int upbp_trace_camera_paths(upbp_ctx* ctx, const upbp_scene* scene, uint32_t iteration);
/* Copy one stored input array to dst (host or device memory; capacity in bytes).  name is one of
 * the C ABI's record arrays: lv_position, lv_throughput, lv_dir_fix, lv_cont_prob, lv_path_idx,
 * lv_path_length, lv_medium_id, lv_flags, lv_mis, lv_path_ends, beam_origin, beam_direction,
 * beam_length, beam_throughput, beam_flags, beam_ray_sample_pdf, beam_ray_sample_rev_pdf,
 * beam_ray_sampling_flags, beam_last_pdf_w_inv, beam_medium_id, beam_light_vertex, cam_mis,
 * sq_origin, sq_direction, sq_seg_begin, sq_seg_count, sq_flags, sq_path_length,
 * sq_last_pdf_w_inv, sq_throughput, sq_pixel, sq_cam_mis_begin, seg_dist_min, seg_dist_max,
 * seg_pdf, seg_rev_pdf, seg_attenuation, seg_medium, pq_position, pq_dir_fix, pq_medium_id,
 * pq_path_length, pq_throughput, pq_pixel, pq_cam_mis_begin; and after a build over the beam grid
 * (upbp_set_bb1d_grid) its structure as the reference holds it (Grid.hxx:644-646):
 * bb1d_grid_cells (mCells, uint32), bb1d_grid_beams (mPointers as beam indices, int32) and, with a
 * reduction, bb1d_grid_pdfs (mPdfs, float).  *bytes receives the array's size; dst may be NULL to
 * query it. */
int upbp_read_input(upbp_ctx* ctx, const char* name, void* dst, int64_t capacity_bytes, int64_t* bytes);

/* Releases the per-iteration structures; replaces EmbreeBre::destroy and
 * PhotonBeamsEvaluator::destroy (UPBP.hxx:1172-1181).  Device buffers are
 * kept for reuse by the next iteration. */
int upbp_destroy_structures(upbp_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* UPBP_GPU_H */
