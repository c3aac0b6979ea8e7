// Device-side light and camera passes of one UPBP iteration: the scene as the kernels see it and
// the output arrays they fill (the layout of the C ABI's input records, upbp_gpu.h).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/upbp_gpu.h"

namespace upbp {
namespace trace {

constexpr int kMaxSegments = 2 * UPBP_MAX_BOXES;  // every box face can split a ray
constexpr int kMaxTracePath = 16;                 // longest camera / light path the passes trace

// One homogeneous medium with the quantities the HomogeneousMedium constructor derives
// (Scene/Media.hxx:129-159), in FP64.
struct TraceMedium {
    double st[3];     // sigma_t = sigma_a + sigma_s
    double ss[3];     // sigma_s
    double smin;      // smallest positive sigma_t component (the free-flight sampling coefficient)
    double mfp;       // 1 / max sigma_t (inf without extinction)
    double g;         // HG mean cosine
    double cont;      // continuation probability
    double maxlen;    // MaxBeamLength = -ln(1e-9) / max sigma_t (inf without extinction)
    int scat;         // any sigma_s > 0
    int beams_ok;     // photon beams are stored in this medium (scattering, and mfp > bb1d_min_mfp under PB2D)
    int in_beams;     // MisData::mInMediumWithBeams of a vertex in this medium
};

struct TraceScene {
    TraceMedium media[UPBP_SCENE_MAX_MEDIA];
    int n_boxes;
    double lo[UPBP_MAX_BOXES][3], hi[UPBP_MAX_BOXES][3];
    int box_medium[UPBP_MAX_BOXES];
    double cam[3];
    double ipd;  // image plane distance: width / (2 tan(fov / 2))
    int width, height;
    int light_paths;
    int max_path_length;
    double light_size, light_intensity;
    unsigned techniques, query_beam_type, photon_beam_type;
    double beam_length_cap, min_dist_to_med;
    float eta_pp3d, eta_pb2d, eta_bb1d;  // MIS factors as stored in the records (upbp_params)
    uint64_t seed, iteration;
};

struct LightOut {
    int* v_count;  // count pass: vertices per path
    int* b_count;  // count pass: beams per path
    const int* v_off;  // write pass: first vertex of each path
    const int* b_off;  // write pass: first beam of each path
    float *pos, *thr, *dir, *cont;
    int *pidx, *plen, *med, *path_ends;
    uint32_t* flags;
    upbp_mis* mis;
    float *b_origin, *b_dir, *b_len, *b_thr, *b_rsp, *b_rsr, *b_lpw;
    uint32_t *b_flags, *b_rsf;
    int *b_med, *b_lv;
    int* status;  // write pass: set when a path would write past its counted records
};

struct CameraOut {
    int *q_count, *s_count, *p_count, *c_count;  // count pass, per pixel
    const int *q_off, *s_off, *p_off, *c_off;    // write pass, per pixel
    float *sq_origin, *sq_dir, *sq_lpw, *sq_thr;
    int *sq_seg_begin, *sq_seg_count, *sq_plen, *sq_pixel;
    uint32_t* sq_flags;
    int64_t* sq_cam_begin;
    float *seg_dmin, *seg_dmax, *seg_pdf, *seg_rev, *seg_att;
    int* seg_med;
    float *pq_pos, *pq_dir, *pq_thr;
    int *pq_med, *pq_plen, *pq_pixel;
    int64_t* pq_cam_begin;
    upbp_mis* cam;
    int* status;  // write pass: set when a pixel would write past its counted records
};

// Derive the device scene from the C ABI's description (host side; FP64 as the generator).
// Returns nullptr on success, else a message naming the invalid field.
const char* make_scene(const upbp_scene& in, const upbp_params& P, uint32_t iteration, TraceScene* out);

void launch_light(const TraceScene& S, bool write, const LightOut& O, cudaStream_t s);
void launch_camera(const TraceScene& S, bool write, const CameraOut& O, cudaStream_t s);

// Exclusive prefix sum of n ints (CUB) with tmp_bytes >= scan_temp_bytes(n) of temporary storage.
size_t scan_temp_bytes(int n);
void exclusive_scan(const int* in, int* out, int n, void* tmp, size_t tmp_bytes, cudaStream_t s);

}  // namespace trace
}  // namespace upbp
