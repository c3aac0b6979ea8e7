/*
 * upbp_gpu.hpp -- C++ host-side mirror of SmallUPBP's estimator interface over the C ABI.
 *
 * The reference renderer owns three estimator objects per UPBP instance
 * (Renderers/UPBP.hxx:2005-2030) and calls them synchronously, one query at a
 * time.  These classes keep the reference names and argument meanings but
 * RECORD the calls during the camera pass; Batch::evaluate() runs all of them
 * on the GPU at the end of the iteration and the recorded calls' results (the
 * Rgb each evalBre / evalBeamBeamEstimate / RangeQuery would have returned)
 * are then available by ticket.
 *
 *   reference                                     this header
 *   --------------------------------------------  ------------------------------------------
 *   HashGrid::Reserve / Build (HashGrid.hxx:41-126)    Batch::set_light_vertices + Batch::build
 *   EmbreeBre::build (Bre.hxx:93-99)                   (same)
 *   PhotonBeamsEvaluator::build (PhBeams.hxx:71-76)    Batch::set_beams + Batch::build
 *   EmbreeBre::evalBre + PhotonBeamsEvaluator::        Batch::record_segment -> ticket
 *     evalBeamBeamEstimate (UPBP.hxx:775-798, 879-911)
 *   HashGrid::Process(RangeQuery) (UPBP.hxx:1114-1122)  Batch::record_point -> ticket
 *   Framebuffer::AddColor of those contributions       Batch::image()
 *   EmbreeBre::destroy / PhotonBeamsEvaluator::destroy Batch::clear
 *
 * Errors: every C-ABI status other than UPBP_OK throws upbp_gpu::Error
 * carrying the code and upbp_last_error().  (The reference exits with
 * status 2 on failed assertions, Misc/Defs.hxx:96-97.)
 */
#ifndef UPBP_GPU_HPP
#define UPBP_GPU_HPP

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "upbp_gpu.h"

namespace upbp_gpu {

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

/* One volume segment of a query ray: VolumeSegment (Path/Ray.hxx:131-140). */
struct Segment {
    float dist_min, dist_max;
    float ray_sample_pdf, ray_sample_rev_pdf;
    float attenuation[3];
    int32_t medium_id;
};

/* Records one iteration's estimator calls and evaluates them in one batch. */
class Batch {
public:
    explicit Batch(int device = 0, int mode = UPBP_MODE_MIXED)
    {
        check(upbp_ctx_create(&ctx_, device));
        check(upbp_set_mode(ctx_, mode));
    }
    ~Batch() { upbp_ctx_destroy(ctx_); }
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;

    void set_media(const std::vector<upbp_medium>& media) { check(upbp_set_media(ctx_, media.data(), (int32_t)media.size())); }
    void set_params(const upbp_params& p)
    {
        params_ = p;
        check(upbp_set_params(ctx_, &p));
    }
    void set_light_vertices(const upbp_light_vertices& lv) { check(upbp_set_light_vertices(ctx_, &lv)); }
    void set_beams(const upbp_beams& b) { check(upbp_set_beams(ctx_, &b)); }
    /* PhotonBeamsEvaluator::sGridSize / sMaxBeamsInCell / sReductionType and mSeed (the -gridres,
     * -gridmax and -gridred options): BB1D over the reference's uniform beam grid. */
    void set_bb1d_grid(uint32_t grid_res, uint32_t max_beams_in_cell = 0, uint32_t reduction = 0,
                       int32_t seed = 1234)
    {
        const upbp_bb1d_grid g{grid_res, max_beams_in_cell, reduction, seed};
        check(upbp_set_bb1d_grid(ctx_, &g));
    }
    /* HashGrid::Build + EmbreeBre::build + PhotonBeamsEvaluator::build for the uploaded records. */
    void build() { check(upbp_build(ctx_)); }

    /* One evalBre/evalBeamBeamEstimate call pair at camera path length L.  cam_mis points at
     * mCameraVerticesMisData[0..L-1] as it is at the call, or is NULL for the calls without MIS
     * data of VolLightTracer's pure PB2D / BB1D (UPBP_NO_MIS in the params' techniques, where
     * last_pdf_w_inv is not read either).  `flags` = UPBP_Q_* (which estimators, origin in medium,
     * lite segments).  Returns the ticket of the call. */
    int64_t record_segment(const float origin[3], const float direction[3], const std::vector<Segment>& segs,
                           uint32_t flags, int path_length, float last_pdf_w_inv, const float throughput[3],
                           int32_t pixel, const upbp_mis* cam_mis)
    {
        const int64_t t = (int64_t)sq_path_length_.size();
        for (int k = 0; k < 3; ++k) {
            sq_origin_.push_back(origin[k]);
            sq_dir_.push_back(direction[k]);
            sq_thr_.push_back(throughput[k]);
        }
        sq_seg_begin_.push_back((int32_t)seg_dmin_.size());
        sq_seg_count_.push_back((int32_t)segs.size());
        for (const Segment& s : segs) {
            seg_dmin_.push_back(s.dist_min);
            seg_dmax_.push_back(s.dist_max);
            seg_pdf_.push_back(s.ray_sample_pdf);
            seg_rev_.push_back(s.ray_sample_rev_pdf);
            for (int k = 0; k < 3; ++k) seg_att_.push_back(s.attenuation[k]);
            seg_med_.push_back(s.medium_id);
        }
        sq_flags_.push_back(flags);
        sq_path_length_.push_back(path_length);
        sq_lpw_.push_back(last_pdf_w_inv);
        sq_pixel_.push_back(pixel);
        sq_cam_begin_.push_back((int64_t)cam_.size());
        if (cam_mis) cam_.insert(cam_.end(), cam_mis, cam_mis + path_length);
        return t;
    }

    /* One HashGrid::Process(RangeQuery) call at a camera medium vertex; cam_mis points at
     * mCameraVerticesMisData[0..L].  Returns the ticket of the call. */
    int64_t record_point(const float position[3], const float dir_fix[3], int32_t medium_id, int path_length,
                         const float throughput[3], int32_t pixel, const upbp_mis* cam_mis)
    {
        const int64_t t = (int64_t)pq_path_length_.size();
        for (int k = 0; k < 3; ++k) {
            pq_pos_.push_back(position[k]);
            pq_dir_.push_back(dir_fix[k]);
            pq_thr_.push_back(throughput[k]);
        }
        pq_med_.push_back(medium_id);
        pq_path_length_.push_back(path_length);
        pq_pixel_.push_back(pixel);
        pq_cam_begin_.push_back((int64_t)cam_.size());
        cam_.insert(cam_.end(), cam_mis, cam_mis + path_length + 1);
        return t;
    }

    /* Evaluate every recorded call; the framebuffer accumulates the normalised contributions. */
    void evaluate()
    {
        check(upbp_set_camera_mis(ctx_, cam_.data(), (int64_t)cam_.size()));
        upbp_segment_queries q{};
        q.n = (int64_t)sq_path_length_.size();
        q.origin = sq_origin_.data();
        q.direction = sq_dir_.data();
        q.seg_begin = sq_seg_begin_.data();
        q.seg_count = sq_seg_count_.data();
        q.flags = sq_flags_.data();
        q.path_length = sq_path_length_.data();
        q.last_pdf_w_inv = sq_lpw_.data();
        q.throughput = sq_thr_.data();
        q.pixel = sq_pixel_.data();
        q.cam_mis_begin = sq_cam_begin_.data();
        q.n_segments = (int64_t)seg_dmin_.size();
        q.seg_dist_min = seg_dmin_.data();
        q.seg_dist_max = seg_dmax_.data();
        q.seg_pdf = seg_pdf_.data();
        q.seg_rev_pdf = seg_rev_.data();
        q.seg_attenuation = seg_att_.data();
        q.seg_medium = seg_med_.data();
        check(upbp_set_segment_queries(ctx_, &q));
        upbp_point_queries p{};
        p.n = (int64_t)pq_path_length_.size();
        p.position = pq_pos_.data();
        p.dir_fix = pq_dir_.data();
        p.medium_id = pq_med_.data();
        p.path_length = pq_path_length_.data();
        p.throughput = pq_thr_.data();
        p.pixel = pq_pixel_.data();
        p.cam_mis_begin = pq_cam_begin_.data();
        check(upbp_set_point_queries(ctx_, &p));
        check(upbp_clear_image(ctx_));
        check(upbp_evaluate(ctx_));
    }

    /* Rgb the reference's evalBre / evalBeamBeamEstimate returned for segment ticket t. */
    void segment_results(std::vector<float>& pb2d_rgb, std::vector<float>& bb1d_rgb)
    {
        pb2d_rgb.resize(3 * sq_path_length_.size());
        bb1d_rgb.resize(3 * sq_path_length_.size());
        check(upbp_read_segment_results(ctx_, pb2d_rgb.data(), bb1d_rgb.data()));
    }
    /* RangeQuery::GetContrib() for point ticket t. */
    void point_results(std::vector<float>& pp3d_rgb)
    {
        pp3d_rgb.resize(3 * pq_path_length_.size());
        check(upbp_read_point_results(ctx_, pp3d_rgb.data()));
    }
    std::vector<float> image()
    {
        std::vector<float> img(3 * (size_t)params_.image_width * (size_t)params_.image_height);
        check(upbp_read_image(ctx_, img.data()));
        return img;
    }

    /* B-P2D contributions per point ticket (extension, UPBP_BP2D in the techniques). */
    void bp2d_results(std::vector<float>& bp2d_rgb)
    {
        bp2d_rgb.resize(3 * pq_path_length_.size());
        check(upbp_read_bp2d_results(ctx_, bp2d_rgb.data(), nullptr, nullptr));
    }

    /* dL/d(sigma_a rgb, sigma_s rgb, g) of media[medium] for dL/d framebuffer (H*W*3 floats), after
     * evaluate() in UPBP_MODE_MIXED or UPBP_MODE_FP64 (no counterpart in the reference). */
    std::vector<double> adjoint(const std::vector<float>& grad_image, int medium)
    {
        std::vector<double> g(7);
        check(upbp_adjoint(ctx_, grad_image.data(), medium, g.data()));
        return g;
    }

    /* Record build + evaluate of the current recording as a CUDA graph (after one evaluate()), and
     * replay it (asynchronously; results as from build() + evaluate()). */
    void capture_graph() { check(upbp_capture_graph(ctx_)); }
    void launch_graph() { check(upbp_launch_graph(ctx_)); }

    /* End of the iteration: EmbreeBre::destroy / PhotonBeamsEvaluator::destroy and a new recording. */
    void clear()
    {
        check(upbp_destroy_structures(ctx_));
        sq_origin_.clear(); sq_dir_.clear(); sq_thr_.clear(); sq_seg_begin_.clear(); sq_seg_count_.clear();
        sq_flags_.clear(); sq_path_length_.clear(); sq_lpw_.clear(); sq_pixel_.clear(); sq_cam_begin_.clear();
        seg_dmin_.clear(); seg_dmax_.clear(); seg_pdf_.clear(); seg_rev_.clear(); seg_att_.clear(); seg_med_.clear();
        pq_pos_.clear(); pq_dir_.clear(); pq_thr_.clear(); pq_med_.clear(); pq_path_length_.clear();
        pq_pixel_.clear(); pq_cam_begin_.clear(); cam_.clear();
    }

    upbp_ctx* handle() { return ctx_; }

private:
    void check(int rc)
    {
        if (rc != UPBP_OK) throw Error(rc, std::string("upbp_gpu: ") + upbp_last_error(ctx_));
    }

    upbp_ctx* ctx_ = nullptr;
    upbp_params params_{};
    std::vector<float> sq_origin_, sq_dir_, sq_thr_, sq_lpw_, seg_dmin_, seg_dmax_, seg_pdf_, seg_rev_, seg_att_,
        pq_pos_, pq_dir_, pq_thr_;
    std::vector<int32_t> sq_seg_begin_, sq_seg_count_, sq_path_length_, sq_pixel_, seg_med_, pq_med_,
        pq_path_length_, pq_pixel_;
    std::vector<uint32_t> sq_flags_;
    std::vector<int64_t> sq_cam_begin_, pq_cam_begin_;
    std::vector<upbp_mis> cam_;
};

}  // namespace upbp_gpu

#endif
