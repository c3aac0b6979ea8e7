// Replays a recorded iteration through the C++ mirror of the estimator interface
// (include/upbp_gpu.hpp) the way the binding in UPBP::RunIteration would drive it: set the media,
// params, light vertices and beams, build, then one Batch::record_segment per evalBre /
// evalBeamBeamEstimate call pair and one Batch::record_point per HashGrid::Process call, each with
// its own segment list and its snapshot of the camera MIS records, then evaluate and read the
// framebuffer and the per-ticket results.  Built as a shared library by the test, which passes
// the arrays of a golden fixture.
#include <cstring>
#include <vector>

#include "upbp_gpu.hpp"

extern "C" int replay_through_batch(int mode, const upbp_params* params, const upbp_medium* media, int32_t n_media,
                                    const upbp_light_vertices* lv, const upbp_beams* beams, const upbp_mis* cam,
                                    const upbp_segment_queries* sq, const upbp_point_queries* pq, float* image,
                                    float* pb2d, float* bb1d, float* pp3d, char* err, int err_len)
{
    try {
        upbp_gpu::Batch batch(0, mode);
        batch.set_media(std::vector<upbp_medium>(media, media + n_media));
        batch.set_params(*params);
        batch.set_light_vertices(*lv);
        batch.set_beams(*beams);
        batch.build();
        std::vector<upbp_gpu::Segment> segs;
        for (int64_t q = 0; q < sq->n; ++q) {
            segs.clear();
            for (int32_t s = sq->seg_begin[q]; s < sq->seg_begin[q] + sq->seg_count[q]; ++s) {
                upbp_gpu::Segment g{};
                g.dist_min = sq->seg_dist_min[s];
                g.dist_max = sq->seg_dist_max[s];
                g.ray_sample_pdf = sq->seg_pdf[s];
                g.ray_sample_rev_pdf = sq->seg_rev_pdf[s];
                for (int k = 0; k < 3; ++k) g.attenuation[k] = sq->seg_attenuation[3 * s + k];
                g.medium_id = sq->seg_medium[s];
                segs.push_back(g);
            }
            const upbp_mis* snap = (cam && sq->cam_mis_begin) ? cam + sq->cam_mis_begin[q] : nullptr;
            const int64_t ticket = batch.record_segment(
                sq->origin + 3 * q, sq->direction + 3 * q, segs, sq->flags[q], sq->path_length[q],
                sq->last_pdf_w_inv ? sq->last_pdf_w_inv[q] : 0.f, sq->throughput + 3 * q, sq->pixel[q], snap);
            if (ticket != q) throw upbp_gpu::Error(-1, "segment ticket out of order");
        }
        for (int64_t q = 0; q < pq->n; ++q) {
            const int64_t ticket =
                batch.record_point(pq->position + 3 * q, pq->dir_fix + 3 * q, pq->medium_id[q], pq->path_length[q],
                                   pq->throughput + 3 * q, pq->pixel[q], cam + pq->cam_mis_begin[q]);
            if (ticket != q) throw upbp_gpu::Error(-1, "point ticket out of order");
        }
        batch.evaluate();
        std::vector<float> a, b, c;
        batch.segment_results(a, b);
        batch.point_results(c);
        const std::vector<float> img = batch.image();
        std::memcpy(pb2d, a.data(), sizeof(float) * a.size());
        std::memcpy(bb1d, b.data(), sizeof(float) * b.size());
        std::memcpy(pp3d, c.data(), sizeof(float) * c.size());
        std::memcpy(image, img.data(), sizeof(float) * img.size());
        batch.clear();
        return 0;
    } catch (const upbp_gpu::Error& e) {
        std::strncpy(err, e.what(), (size_t)err_len - 1);
        err[err_len - 1] = 0;
        return e.code();
    }
}
