// Kernel interfaces of the B200 estimator stage (device data layout in HBM).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "upbp_device.cuh"

namespace upbp {

// BVH2 node with both child boxes (64 B, one 4x16-byte load per visit).
// Children: >= 0 internal node index, < 0 leaf ~index.
struct __align__(16) BNode {
    float4 a;  // left.lo.xyz, left.hi.x
    float4 b;  // left.hi.yz, right.lo.xy
    float4 c;  // right.lo.z, right.hi.xyz
    int4 d;    // left, right, -, -
};

struct Box {
    float lo[3], hi[3];
};

// Light vertices, packed for the gathers (index = light vertex index).
struct LightSoA {
    const float4* pos;      // xyz, continuation prob of its BSDF
    const float4* dir;      // dir_fix xyz, -
    const float4* thr;      // throughput rgb, -
    const int4* info;       // path_idx, path_length, flags, medium_id
    const upbp_mis* mis;    // MisData
    const int32_t* path_ends;
    const struct LightSum* sums;  // mixed mode: FP64 partial sums of the light walks
    int64_t n;
};

// Photon LBVH (PB2D): photons in leaf order, leaf k = photons [k*leaf, min((k+1)*leaf, n)).
struct PhotonBVH {
    const float4* pos;   // xyz, light-vertex index (int bits)
    const BNode* nodes;  // n_leaves - 1 internal nodes, root 0
    const float* r2;     // KNN radii: photon radius^2 in leaf order (NULL: radius_pb2d^2)
    int n;
    int leaf;
    int n_leaves;
};

// Payload of the beam a piece belongs to, packed per piece (mixed mode): everything an accepted
// candidate reads besides the piece geometry, so it comes from the lines the warp just tested.
// The light vertex's partial sums d, e are the FP64 LightSum values rounded to FP32 for the
// per-candidate combination (the FP64 mode reads LightSum itself).
struct __align__(16) PiecePayload {
    float4 thr;   // beam throughput at origin rgb, light vertex partial sum d
    float4 pdf;   // beam ray_sample_pdf, ray_sample_rev_pdf, last_pdf_w_inv, light vertex partial sum e
    float4 lv;    // light vertex |cos_theta_out| (0 on a delta light), bptb, radius, bits (payload_* below)
};
// bits of PiecePayload::lv.w: the light vertex's path length, whether it is finite, and the two beam
// flags the contribution reads
constexpr int kPayPathMask = 0x1fffffff;
constexpr int kPayFinite = 1 << 29;
constexpr int kPayShortBeam = 1 << 30;
constexpr unsigned kPayOriginInMedium = 1u << 31;

// Beam pieces (BB1D) in leaf order.  Piece = beam sub-interval [t_lo, t_hi).
struct BeamBVH {
    const float4* pa;    // beam origin xyz, beam length
    const float4* pb;    // beam direction xyz, max radius^2   (pa, pb: all the predicate reads)
    const float4* pc;    // t_lo, t_hi, beam id (int bits), medium (int bits)
    const BNode* nodes;
    const PiecePayload* pay;  // mixed mode, per piece
    int n;
    int leaf;
    int n_leaves;
};

// The reference's uniform grid of beams (Beams/Grid.hxx:222-279, built by upbp_grid.cu): its
// box, cell size and resolution, and the cell lists in the reference's order.
struct GridHeader {
    float lo[3], hi[3];          // mAABB
    float cell[3], inv_cell[3];  // mCellSize, mInvCellSize
    int res[3];                  // mRes
    uint32_t shift[3];           // mIndexShift
    uint32_t n_cells;            // mCells.size(): (res0 + 1)(res1 + 1)(res2 + 1) + 1
    uint32_t max_beams;          // mMaxBeamsInCell (0: no reduction)
    uint32_t reduction;          // mReductionType: 0 PRESAMPLE, 1 OFFSET, 2 RESAMPLE_FIXED, 3 SAMPLED
    int32_t seed;                // the evaluator's seed (the per-query draws of reductions 1-3)
};
struct BeamGrid {
    const GridHeader* hdr;
    const uint32_t* cells;  // mCells: the first entry of every cell's list (n_cells entries)
    const float* pdf;       // mPdfs, NULL: 1 in every cell (no reduction)
    const int32_t* ptr;     // mPointers: beam ids, each cell's beams in descending id order
    const float4* rec_a;    // per entry of ptr: the beam's origin xyz, length
    const float4* rec_b;    // per entry of ptr: the beam's direction xyz, mMaxRadiusSqr
    const int32_t* medium;  // per beam, as uploaded
    const PiecePayload* pay;  // mixed mode: the contribution's inputs per beam (PiecePayload layout)
};

// Beam payload (index = beam id).
struct BeamSoA {
    const float4* thr;   // throughput at origin rgb, flags (int bits)
    const float4* pdf;   // ray_sample_pdf, ray_sample_rev_pdf, last_pdf_w_inv, ray_sampling_flags (int bits)
    const int2* link;    // light vertex, medium
    const float* radius; // start radius (the constant radius, or the KNN start radius)
    const float* rchange; // KNN radii: radius change per unit length (NULL: constant radius)
    float radius_const;   // every beam's radius when rchange is NULL
    int64_t n;
};

// Start radius of a beam: the constant radius, or with KNN radii the beam's own, loaded from
// `start` only then.
__device__ __forceinline__ float beam_start_radius(const BeamSoA& S, const float* start)
{
    return S.rchange ? __ldg(start) : S.radius_const;
}

// Radius of a beam at t (PhotonBeam.hxx:411: mStartRadius + t * mRadiusChange).
__device__ __forceinline__ float beam_radius_at(const BeamSoA& S, int beam, float start, float t)
{
    return S.rchange ? __fadd_rn(start, __fmul_rn(t, __ldg(&S.rchange[beam]))) : start;
}

// PP3D hash grid (Misc/HashGrid.hxx), photons sorted by bucket, stable in light-vertex order.
struct HashGridDev {
    const float4* pos;      // xyz, light-vertex index (int bits)
    const int32_t* start;   // [cells]
    const int32_t* end;     // [cells]
    float bbox_min[3], bbox_max[3];
    float inv_cell;
    float r2;
    int cells;
    int n;
};

struct SegQueriesDev {
    const float* origin;
    const float* direction;
    const int32_t* seg_begin;
    const int32_t* seg_count;
    const uint32_t* flags;
    const int32_t* path_length;
    const float* last_pdf_w_inv;
    const float* throughput;
    const int32_t* pixel;
    const int64_t* cam_mis_begin;
    const float* seg_dist_min;
    const float* seg_dist_max;
    const float* seg_pdf;
    const float* seg_rev_pdf;
    const float* seg_attenuation;
    const int32_t* seg_medium;
    int64_t n;
};

struct PointQueriesDev {
    const float* position;
    const float* dir_fix;
    const int32_t* medium_id;
    const int32_t* path_length;
    const float* throughput;
    const int32_t* pixel;
    const int64_t* cam_mis_begin;
    int64_t n;
};

struct Outputs {
    float* rgb;                 // [n][3]
    float* image;               // [H*W][3] or null
    uint32_t* count;            // [n] or null
    unsigned long long* hash;   // [n] or null
    unsigned long long* tested; // total candidates tested (diagnostic), or null
};

struct GatherConsts {
    upbp_params P;
    DMedium media[UPBP_MAX_MEDIA];
    int n_media;
    int has_bb1d_beams;  // PB2D: mBB1DPhotonBeams != NULL
    float eps;           // conservative box slack for traversal
    float bb1d_extra;    // reach margin of the BB1D candidate rule (bb1d_reach_extra)
};

constexpr int kMaxKnn = 64;  // largest k of the KNN radii

// ---- launches (all asynchronous on `stream`) ----------------------------------------
void launch_photon_knn_r2(const float4* pts, int n, const BNode* nodes, int n_leaves, int leaf, int k, float r,
                          float* r2, int* status, cudaStream_t stream);
void launch_photon_leaf_boxes_r2(const float4* pos, const float* r2, int n, int leaf, float eps, Box* leaf_boxes,
                                 cudaStream_t stream);
void launch_beam_origins(const float* origin, int n, float4* out, cudaStream_t stream);
void launch_beam_knn(const float* origin, const float* dir, const float* length, int n, const BNode* nodes,
                     int n_leaves, const float4* pts, int leaf, int k, float r, float* rstart, float* rchange,
                     float* r2max, int* status, cudaStream_t stream);
void launch_pack_lights(const float* pos, const float* thr, const float* dir, const float* cont,
                        const int32_t* path_idx, const int32_t* path_length, const int32_t* medium,
                        const uint32_t* flags, int64_t n, float4* o_pos, float4* o_dir, float4* o_thr, int4* o_info,
                        uint32_t* o_in_medium, cudaStream_t stream);

void launch_bbox_partial(const float4* pts, const int32_t* idx, int n, float* partial, int blocks,
                         cudaStream_t stream);
void launch_bbox_final(const float* partial, int blocks, float* out, cudaStream_t stream);

void launch_hash_keys(const float4* lv_pos, const int32_t* ph_lv, int n, const float* bbox, float inv_cell, int cells,
                      uint32_t* keys, cudaStream_t stream);
void launch_hash_ranges(const uint32_t* keys_sorted, const int32_t* lv_sorted, const float4* lv_pos, int n,
                        int32_t* start, int32_t* end, float4* out_pos, cudaStream_t stream);

void launch_morton_points(const float4* lv_pos, const int32_t* ph_lv, int n, const float* bbox, uint32_t* codes,
                          cudaStream_t stream);
void launch_gather_photons(const int32_t* lv_sorted, const float4* lv_pos, int n, float4* out_pos,
                           cudaStream_t stream);
void launch_leaf_codes(const uint32_t* codes_sorted, int n, int leaf, uint32_t* leaf_codes, cudaStream_t stream);
void launch_karras(const uint32_t* leaf_codes, int n_leaves, BNode* nodes, int32_t* parent_int,
                   int32_t* parent_leaf, cudaStream_t stream);
void launch_photon_leaf_boxes(const float4* pos, int n, int leaf, float r, float eps, Box* leaf_boxes,
                              cudaStream_t stream);
void launch_bottom_up(const Box* leaf_boxes, int n_leaves, BNode* nodes, const int32_t* parent_int,
                      const int32_t* parent_leaf, Box* node_boxes, int32_t* flags, cudaStream_t stream);

void launch_pack_beams(const float* thr, const uint32_t* flags, const float* rsp, const float* rsr, const float* lpw,
                       const uint32_t* rsf, const int32_t* lv, const int32_t* medium, int64_t n, float radius,
                       float4* o_thr, float4* o_pdf, int2* o_link, float* o_radius, cudaStream_t stream);
void launch_piece_counts(const float* length, int64_t n, float piece_len, int32_t* counts, cudaStream_t stream);
void launch_bbox_beams_partial(const float* origin, const float* dir, const float* length, int64_t n, float* partial,
                               int blocks, cudaStream_t s);
void launch_piece_codes(const float* origin, const float* dir, const float* length, int64_t nb, const int32_t* offsets,
                        int np, const float* bbox, uint32_t* codes, int32_t* perm, cudaStream_t s);
void launch_emit_sorted(const float* origin, const float* dir, const float* length, const int32_t* medium, int64_t nb,
                        const int32_t* offsets, const int32_t* perm, int np, float radius, float eps,
                        const float* rstart, const float* rchange, const float* r2max, float4* pa, float4* pb,
                        float4* pc, Box* boxes, cudaStream_t s);
void launch_box_leaf_boxes(const Box* boxes, int n, int leaf, Box* leaf_boxes, cudaStream_t stream);

struct CamSum;
void launch_gather_pb2d(const GatherConsts& K, const LightSoA& L, const PhotonBVH& B, const SegQueriesDev& Q,
                        const upbp_mis* cam, const CamSum* cs, const Outputs& O, int block, bool mixed,
                        cudaStream_t stream, const int32_t* order = nullptr);
void launch_gather_bb1d(const GatherConsts& K, const LightSoA& L, const BeamBVH& B, const BeamSoA& S,
                        const SegQueriesDev& Q, const upbp_mis* cam, const CamSum* cs, const Outputs& O, int block,
                        bool mixed, cudaStream_t stream);
void launch_piece_payload(const float4* pc, int n, const float4* bm_thr, const float4* bm_pdf, const int2* bm_link,
                          const float* bm_radius, const int4* lv_info, const upbp_mis* lv_mis,
                          const struct LightSum* sums, PiecePayload* out, cudaStream_t stream);
void launch_query_keys(const SegQueriesDev& Q, const float* bbox, int mode, int image_width, uint32_t* keys,
                       int32_t* iota, cudaStream_t stream);
// keys that put the queries with more than `factor` x the mean PB2D candidate count first, each
// group in the given Morton order; *sum must be zero on entry
void launch_heavy_keys(const uint32_t* cnt, int64_t n, unsigned long long* sum, unsigned factor,
                       const uint32_t* morton, uint32_t* keys, int32_t* iota, cudaStream_t stream);
int bb1d_warp_blocks_per_sm(bool mixed, int variant);
int pb2d_warp_blocks_per_sm(bool mixed);
void launch_pb2d_warp(const GatherConsts& K, const LightSoA& L, const PhotonBVH& P, const SegQueriesDev& Q,
                      const upbp_mis* cam, const CamSum* cs, const Outputs& O, int grid, bool mixed,
                      unsigned int* work, int* status, const int32_t* order, cudaStream_t stream);
int segments_warp_blocks_per_sm(bool mixed, int variant);
void launch_segments_warp(const GatherConsts& K, const LightSoA& L, const PhotonBVH& P, const BeamBVH& B,
                          const BeamSoA& S, const SegQueriesDev& Q, const upbp_mis* cam, const CamSum* cs,
                          const Outputs& Opb, const Outputs& Obb, int grid, bool mixed, unsigned int* work,
                          int* status, const int32_t* order, cudaStream_t stream, int variant);
// BB1D over the reference's uniform grid (upbp_set_bb1d_grid): warp per query, persistent.
int bb1d_grid_blocks_per_sm(bool mixed);
void launch_bb1d_grid(const GatherConsts& K, const LightSoA& L, const BeamGrid& G, const BeamSoA& S,
                      const SegQueriesDev& Q, const upbp_mis* cam, const CamSum* cs, const Outputs& O, int grid,
                      bool mixed, unsigned int* work, const int32_t* order, cudaStream_t stream);
// Grid build steps (upbp_grid.cu): the beams' boxes and the grid header; the (cell, beam) pairs of
// every beam's rasterisation, counted and then written as sort keys; the cell lists from the
// sorted, unique keys; the PRESAMPLE reduction from the reference's random stream.
void launch_grid_header(const float* origin, const float* dir, const float* length, const float* rstart,
                        const float* rchange, float radius, int64_t nb, uint32_t grid_res, uint32_t max_beams,
                        uint32_t reduction, int32_t seed, float* partial, int blocks, GridHeader* hdr,
                        cudaStream_t s);
void launch_grid_count(const float* origin, const float* dir, const float* length, const float* rstart,
                       const float* rchange, float radius, int64_t nb, const GridHeader* hdr,
                       unsigned long long* counts, cudaStream_t s);
void launch_grid_emit(const float* origin, const float* dir, const float* length, const float* rstart,
                      const float* rchange, float radius, int64_t nb, const GridHeader* hdr,
                      const unsigned long long* offsets, unsigned long long* keys, cudaStream_t s);
void launch_grid_lists(const unsigned long long* keys, int64_t n, uint32_t* counts, int32_t* ptr, cudaStream_t s);
void launch_grid_records(const int32_t* ptr, int64_t n, const float* origin, const float* dir, const float* length,
                         const float* r2max, float r2c, float4* rec_a, float4* rec_b, cudaStream_t s);
void launch_grid_draws(const uint32_t* cells, uint32_t n_cells, uint32_t max_beams, uint32_t reduction,
                       uint32_t* draws, cudaStream_t s);
void launch_mt64_floats(unsigned long long seed, int64_t n, float* out, cudaStream_t s);
void launch_grid_reduce(const uint32_t* cells, uint32_t n_cells, uint32_t max_beams, uint32_t reduction,
                        const uint32_t* draw_off, const float* rnd, int32_t* ptr, float* pdf, cudaStream_t s);

void launch_bb1d_warp(const GatherConsts& K, const LightSoA& L, const BeamBVH& B, const BeamSoA& S,
                      const SegQueriesDev& Q, const upbp_mis* cam, const CamSum* cs, const Outputs& O, int grid,
                      bool mixed, unsigned int* work, int* status, const int32_t* order, cudaStream_t stream,
                      int variant);
void launch_gather_bp2d(const GatherConsts& K, const BeamBVH& B, const BeamSoA& S, const PointQueriesDev& Q,
                        const Outputs& O, int block, cudaStream_t stream);
int bp2d_warp_blocks_per_sm();
void launch_bp2d_warp(const GatherConsts& K, const BeamBVH& B, const BeamSoA& S, const PointQueriesDev& Q,
                      const Outputs& O, int grid, unsigned int* work, int* status, cudaStream_t stream);
void launch_gather_pp3d(const GatherConsts& K, const LightSoA& L, const HashGridDev& G, const PointQueriesDev& Q,
                        const upbp_mis* cam, const CamSum* cs, const Outputs& O, int block, bool mixed,
                        cudaStream_t stream);
void launch_light_sums(const upbp_mis* mis, const int32_t* path_ends, int n_paths, uint32_t tech, uint32_t qbt,
                       uint32_t pbt, struct LightSum* out, cudaStream_t s);
void launch_cam_sums(const upbp_mis* cam, const int64_t* begin, const int32_t* path_length, int64_t n, uint32_t tech,
                     uint32_t qbt, uint32_t pbt, CamSum* out, cudaStream_t s);

}  // namespace upbp
