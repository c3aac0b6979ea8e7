/*
 * Reference harness (test infrastructure only; never linked into the product).
 *
 * Drives the reference SmallUPBP estimator objects exactly as
 * UPBP::RunIteration does (Renderers/UPBP.hxx:682-730 builds, 775-798 and
 * 879-911 segment estimators, 1114-1122 PP3D), on the neutral arrays of
 * include/upbp_gpu.h:
 *   - the UPBP object's own mPP3DHashGrid (Misc/HashGrid.hxx), mPB2DEmbreeBre
 *     (Bre/Bre.cxx, with the reference's Embree 2.0 BVH) and mBB1DPhotonBeams
 *     (Beams/PhBeams.cxx, USE_GRID) are built and queried;
 *   - PP3D queries use the reference's nested UPBP::RangeQuery (UPBP.hxx:63-143);
 *   - the brute-force BB1D evaluator (PhBrute.hxx) is compiled in its own TU.
 * The camera MIS array mCameraVerticesMisData is loaded from the recorded
 * snapshot before every call, which is its state at the call in the renderer.
 *
 * With UPBP_NO_MIS in the techniques the harness runs the estimators as
 * VolLightTracer's pure algorithms do (Renderers/VolLightTracer.hxx:296-412):
 * EmbreeBre::build over VltLightVertex records (photons with the callback
 * breIntersectFuncHomogeneous), evalBre and evalBeamBeamEstimate with no
 * AdditionalRayDataForMis (PhotonBeam::accumulate), beams without light vertices.
 */
#include <vector>
#include <list>
#include <forward_list>
#include <string>
#include <sstream>
#include <iostream>
#include <fstream>
#include <iomanip>
#include <algorithm>
#include <cmath>
#include <set>
#include <map>
#include <memory>
#include <chrono>
#include <mutex>
#include <omp.h>

#define private public
#define protected public
#include "Renderers/UPBP.hxx"
#undef private
#undef protected

#include "ref_harness.h"
#include "ref_internal.h"

void* ref_brute_create(const Scene& scene, PhotonBeamsArray& beams, float radius, int knn);
void ref_bre_radii(const EmbreeBre& bre, const UPBPLightVertex* base, int64_t n, float* r2);
void ref_bre_link_photons(EmbreeBre& bre, const UPBPLightVertex* base, int64_t n);
Rgb ref_brute_eval(void* h, BeamType bt, const Ray& ray, const VolumeSegments& segs, uint tech, uint rsf,
                   embree::AdditionalRayDataForMis* data);
Rgb ref_brute_eval_lite(void* h, BeamType bt, const Ray& ray, const LiteVolumeSegments& segs, uint tech, uint rsf,
                        embree::AdditionalRayDataForMis* data);
void ref_brute_destroy(void* h);

/* the seed of the grid's beam reduction (PhotonBeamsEvaluator::mSeed; the evaluator's own default
 * is 1234, PhBeams.hxx:56) */
static int g_grid_seed = 1234;

namespace {

struct World {
    Scene scene;
    UPBP* upbp = nullptr;
    void* brute = nullptr;
    std::vector<VltLightVertex> vlt;  // VolLightTracer's light vertices (UPBP_NO_MIS)
    ~World()
    {
        if (upbp) {
            if (upbp->mMergeWithLightVerticesPB2D) upbp->mPB2DEmbreeBre.destroy();
            if (upbp->mBB1DPhotonBeams.accelStruct) upbp->mBB1DPhotonBeams.destroy();
            delete upbp;
        }
        if (brute) ref_brute_destroy(brute);
    }
};

inline Pos P3(const float* v) { return Pos(v[0], v[1], v[2]); }
inline Dir D3(const float* v) { return Dir(v[0], v[1], v[2]); }
inline Rgb C3(const float* v) { return Rgb(v[0], v[1], v[2]); }

MisData to_mis(const upbp_mis& m)
{
    MisData d;
    d.mPdfAInv = m.pdf_a_inv;
    d.mRevPdfA = m.rev_pdf_a;
    d.mRevPdfAWithoutBsdf = m.rev_pdf_a_without_bsdf;
    d.mRaySamplePdfInv = m.ray_sample_pdf_inv;
    d.mRaySampleRevPdfInv = m.ray_sample_rev_pdf_inv;
    d.mRaySamplePdfsRatio = m.ray_sample_pdfs_ratio;
    d.mRaySampleRevPdfsRatio = m.ray_sample_rev_pdfs_ratio;
    d.mSinTheta = m.sin_theta;
    d.mCosThetaOut = m.cos_theta_out;
    d.mSurfMisWeightFactor = m.surf_factor;
    d.mPP3DMisWeightFactor = m.pp3d_factor;
    d.mPB2DMisWeightFactor = m.pb2d_factor;
    d.mBB1DMisWeightFactor = m.bb1d_factor;
    d.mBB1DBeamSelectionPdf = m.bb1d_beam_selection_pdf;
    d.mIsDelta = (m.flags & UPBP_MIS_IS_DELTA) != 0;
    d.mIsOnLightSource = (m.flags & UPBP_MIS_ON_LIGHT_SOURCE) != 0;
    d.mIsSpecular = (m.flags & UPBP_MIS_IS_SPECULAR) != 0;
    d.mInMediumWithBeams = (m.flags & UPBP_MIS_IN_MEDIUM_WITH_BEAMS) != 0;
    return d;
}

/* BSDF of a medium vertex, through the reference constructor (Path/Bsdf.hxx:95-152). */
BSDF medium_bsdf(const Scene& scene, const float* dir_fix, int medium, BSDF::Direction from)
{
    Ray ray(Pos(0.f), -D3(dir_fix));
    Isect isect(1.0f);
    isect.mMatID = -1;
    isect.mMedID = medium;
    return BSDF(ray, isect, scene, from, -1.0f);
}

void setup_world(World& w, const upbp_params& P, const upbp_medium* media, int n_media,
                 const upbp_light_vertices* lv, const upbp_beams* bm, int what)
{
    for (int i = 0; i < n_media; ++i) {
        const upbp_medium& m = media[i];
        w.scene.mMedia.push_back(new HomogeneousMedium(C3(m.absorption), Rgb(0.f), C3(m.scattering),
                                                       m.continuation_prob, m.mean_cosine));
    }
    const float nl = (float)P.hash_cells;
    const bool nomis = (P.techniques & UPBP_NO_MIS) != 0;
    w.scene.mCamera.mResolution = Vec2f(1.f, 1.f);
    w.upbp = new UPBP(w.scene, UPBP::kCustom, P.techniques & ~UPBP_NO_MIS,
                      P.radius_pp3d, 1.f, P.radius_pp3d, 1.f, P.radius_pb2d, 1.f,
                      P.pb2d_knn > 0 ? KNN_RADIUS : CONSTANT_RADIUS, P.pb2d_knn,
                      (BeamType)P.query_beam_type, P.radius_bb1d, 1.f,
                      P.bb1d_knn > 0 ? KNN_RADIUS : CONSTANT_RADIUS, P.bb1d_knn,
                      (BeamType)P.photon_beam_type, nl, 0.f, nl, nl, P.min_dist_to_med,
                      (size_t)1 << 30, 1234, 1234, false, false);
    UPBP& U = *w.upbp;
    U.mMaxPathLength = P.max_path_length;
    U.mMinPathLength = P.min_path_length;
    U.mDebugImages.Setup((int)P.max_path_length + 1, Vec2f((float)P.image_width, (float)P.image_height),
                         DebugImages::NONE, DebugImages::DO_NOT_OUTPUT_WEIGHTS, DebugImages::MULTIPLY_BY_WEIGHTS);
    U.mLightSubPathCount = nl;
    U.mBB1DUsedLightSubPathCount = nl;
    U.mSurfMisWeightFactor = P.mis_factor_surf;
    U.mPP3DMisWeightFactor = P.mis_factor_pp3d;
    U.mPB2DMisWeightFactor = P.mis_factor_pb2d;
    U.mBB1DMisWeightFactor = P.mis_factor_bb1d;
    U.mPP3DNormalization = P.norm_pp3d;
    U.mPB2DNormalization = P.norm_pb2d;
    U.mBB1DNormalization = P.norm_bb1d;
    U.mBB1DMinMFP = P.bb1d_min_mfp;

    // light vertices (UPBP.hxx:573-655 record layout)
    U.mLightVertices.clear();
    U.mLightVertices.resize((size_t)lv->n);
    size_t in_medium = 0, on_surface = 0;
    for (int64_t i = 0; i < lv->n; ++i) {
        UPBPLightVertex& v = U.mLightVertices[(size_t)i];
        v.mHitpoint = P3(lv->position + 3 * i);
        v.mThroughput = C3(lv->throughput + 3 * i);
        v.mPathIdx = lv->path_idx ? lv->path_idx[i] : 0;
        v.mPathLength = (uint)lv->path_length[i];
        v.mInMedium = (lv->flags[i] & UPBP_LV_IN_MEDIUM) != 0;
        v.mConnectable = (lv->flags[i] & UPBP_LV_CONNECTABLE) != 0;
        v.mIsFinite = (lv->flags[i] & UPBP_LV_IS_FINITE) != 0;
        v.mBehindSurf = false;
        if (v.mInMedium) {
            v.mBSDF = medium_bsdf(w.scene, lv->dir_fix + 3 * i, lv->medium_id[i], BSDF::kFromLight);
            ++in_medium;
        } else {
            ++on_surface;
        }
        if (lv->mis) v.mMisData = to_mis(lv->mis[i]);
    }
    U.mLightVerticesInMediumCount = in_medium;
    U.mLightVerticesOnSurfaceCount = on_surface;
    if (lv->path_ends) U.mPathEnds.assign(lv->path_ends, lv->path_ends + lv->n_paths);
    if (nomis) {
        // VolLightTracer's records (VolLightTracer.hxx:241-250): hitpoint, throughput, path
        // length, in-medium flag and the BSDF, no MIS data
        w.vlt.resize((size_t)lv->n);
        for (int64_t i = 0; i < lv->n; ++i) {
            VltLightVertex& v = w.vlt[(size_t)i];
            const UPBPLightVertex& u = U.mLightVertices[(size_t)i];
            v.mHitpoint = u.mHitpoint;
            v.mThroughput = u.mThroughput;
            v.mPrevThroughput = u.mThroughput;
            v.mIncEdgeLength = 0.f;
            v.mPathLength = u.mPathLength;
            v.mIsInMedium = u.mInMedium ? 1 : 0;
            v.mBSDF = u.mBSDF;
        }
    }

    // photon beams (UPBP::AddBeams record layout, UPBP.hxx:1783-1870)
    U.mPhotonBeamsArray.clear();
    if (bm && bm->n > 0) {
        U.mPhotonBeamsArray.resize((size_t)bm->n);
        for (int64_t i = 0; i < bm->n; ++i) {
            PhotonBeam& b = U.mPhotonBeamsArray[(size_t)i];
            b.mThroughputAtOrigin = C3(bm->throughput + 3 * i);
            b.mRay = Ray(P3(bm->origin + 3 * i), D3(bm->direction + 3 * i));
            b.mLength = bm->length[i];
            b.mFlags = bm->flags[i];
            b.mRaySamplePdf = bm->ray_sample_pdf ? bm->ray_sample_pdf[i] : 0.f;
            b.mRaySampleRevPdf = bm->ray_sample_rev_pdf ? bm->ray_sample_rev_pdf[i] : 0.f;
            b.mRaySamplingFlags = bm->ray_sampling_flags ? bm->ray_sampling_flags[i] : 0u;
            b.mLastPdfWInv = bm->last_pdf_w_inv ? bm->last_pdf_w_inv[i] : 0.f;
            b.mIsFirstSegment = false;
            b.mMedium = w.scene.mMedia[bm->medium_id[i]];
            // VolLightTracer::AddBeams stores no light vertex (VolLightTracer.hxx:586-640)
            b.mLightVertex = (nomis || !bm->light_vertex) ? NULL : &U.mLightVertices[(size_t)bm->light_vertex[i]];
        }
    }

    // builds, as UPBP::RunIteration (UPBP.hxx:689-730)
    if ((what & (REF_PP3D | REF_CANDIDATES)) && U.mMergeWithLightVerticesPP3D && in_medium) {
        U.mPP3DHashGrid.Reserve(P.hash_cells);
        U.mPP3DHashGrid.Build(U.mLightVertices, P.radius_pp3d, PP3D);
    }
    if ((what & (REF_PB2D | REF_CANDIDATES)) && U.mMergeWithLightVerticesPB2D && !U.mLightVertices.empty()) {
        if (nomis) {
            // the VolLightTracer overload (Bre.cxx:526-614); the photons' light-vertex links, which
            // that build leaves unset and its callback never reads, are filled for the candidate
            // enumeration and the radii
            U.mPB2DEmbreeBre.build(&w.vlt[0], (int)w.vlt.size(), P.pb2d_knn > 0 ? KNN_RADIUS : CONSTANT_RADIUS,
                                   P.radius_pb2d, P.pb2d_knn, false);
            ref_bre_link_photons(U.mPB2DEmbreeBre, &U.mLightVertices[0], (int64_t)U.mLightVertices.size());
        } else {
            U.mPB2DEmbreeBre.build(&U.mLightVertices[0], (int)U.mLightVertices.size(),
                                   P.pb2d_knn > 0 ? KNN_RADIUS : CONSTANT_RADIUS, P.radius_pb2d, P.pb2d_knn, false);
        }
    }
    if ((what & REF_BB1D_GRID) && U.mMergeWithLightVerticesBB1D && !U.mPhotonBeamsArray.empty()) {
        U.mBB1DPhotonBeams.mSeed = g_grid_seed;
        U.mBB1DPhotonBeams.build(U.mPhotonBeamsArray, P.bb1d_knn > 0 ? KNN_RADIUS : CONSTANT_RADIUS, P.radius_bb1d,
                                 P.bb1d_knn, false);
    }
    if ((what & (REF_BB1D_BRUTE | REF_CANDIDATES)) && U.mMergeWithLightVerticesBB1D && !U.mPhotonBeamsArray.empty())
        w.brute = ref_brute_create(w.scene, U.mPhotonBeamsArray, P.radius_bb1d, P.bb1d_knn);
}

void load_camera(UPBP& U, const upbp_mis* cam_mis, int64_t begin, int count)
{
    for (int i = 0; i < count; ++i) U.mCameraVerticesMisData[i] = to_mis(cam_mis[begin + i]);
}

/* PP3D candidate counter with the HashGrid query interface (HashGrid.hxx:129-188). */
struct CountQuery {
    Pos pos;
    const UPBPLightVertex* base;
    uint32_t count = 0;
    uint64_t hash = 0;
    const Pos& GetPosition() const { return pos; }
    void Process(const UPBPLightVertex& v)
    {
        ++count;
        hash += ref_mix64((uint64_t)(&v - base));
    }
};

/* BB1D candidate test, full-interval form (the brute-force AccelStruct passes
 * the segment [mint, maxt) as the cell interval, PhBrute.hxx:77-85). */
void bb1d_candidates(const UPBP& U, const Ray& ray, float dmin, float dmax, const AbstractMedium* medium,
                     uint32_t& count, uint64_t& hash)
{
    const PhotonBeamsArray& beams = U.mPhotonBeamsArray;
    for (size_t i = 0; i < beams.size(); ++i) {
        const PhotonBeam& b = beams[i];
        float dist, sinTheta, t1, t2;
        if (b.mMedium == medium &&
            PhotonBeam::testIntersectionBeamBeam(ray.origin, ray.direction, dmin, dmax, b.mRay.origin, b.mRay.direction,
                                                 0, b.mLength, b.mMaxRadiusSqr, dist, sinTheta, t1, t2)) {
            const float radius = b.mStartRadius + t2 * b.mRadiusChange;
            if (radius < dist) continue;
            ++count;
            hash += ref_mix64((uint64_t)i);
        }
    }
}

/* UPBP::RangeQuery and UPBP::SubPathState are private nested types of the
 * renderer.  Names used in an explicit instantiation are not access checked
 * ([temp.explicit]), so this instantiation exposes one function that runs the
 * reference's own RangeQuery over the reference's HashGrid (UPBP.hxx:1114-1122). */
typedef Rgb (*pp3d_fn_t)(UPBP&, const Pos&, const BSDF&, int);
pp3d_fn_t g_pp3d_fn = nullptr;
template <typename RQ, typename SS>
struct PP3DExposer {
    static Rgb run(UPBP& U, const Pos& hit, const BSDF& bsdf, int L)
    {
        SS cs;
        cs.mPathLength = (uint)L;
        RQ query(U, hit, bsdf, cs, U.mDebugImages);
        U.mPP3DHashGrid.Process(U.mLightVertices, query);
        return query.GetContrib();
    }
    struct Init {
        Init() { g_pp3d_fn = &run; }
    };
    static Init init;
};
template <typename RQ, typename SS>
typename PP3DExposer<RQ, SS>::Init PP3DExposer<RQ, SS>::init;
template struct PP3DExposer<UPBP::RangeQuery, UPBP::SubPathState>;

}  // namespace

extern "C" void ref_set_grid_options(uint32_t grid_size, uint32_t max_beams_in_cell, uint32_t reduction_type)
{
    PhotonBeamsEvaluator::sGridSize = grid_size;
    PhotonBeamsEvaluator::sMaxBeamsInCell = max_beams_in_cell;
    PhotonBeamsEvaluator::sReductionType = reduction_type;
}

extern "C" void ref_set_grid_seed(int32_t seed) { g_grid_seed = seed; }

struct RefSession {
    upbp_params P;
    const upbp_medium* media;
    int32_t n_media;
    const upbp_light_vertices* lv;
    const upbp_beams* beams;
    const upbp_mis* cam_mis;
    const upbp_segment_queries* sq;
    const upbp_point_queries* pq;
    int32_t what;
    int nthreads;
    std::vector<std::unique_ptr<World>> worlds;
    double build_ms;
};

extern "C" void* ref_prepare(const upbp_params* params, const upbp_medium* media, int32_t n_media,
                             const upbp_light_vertices* lv, const upbp_beams* beams, const upbp_mis* cam_mis,
                             const upbp_segment_queries* sq, const upbp_point_queries* pq, int32_t what,
                             int32_t threads)
{
    if (!params || !media || !lv) return nullptr;
    // Embree library init, as EmbreeAcc::initLib (Bre/EmbreeAcc.hxx:42-49).
    static std::once_flag embree_once;
    std::call_once(embree_once, [] {
        embree::rtcInit();
        embree::rtcSetVerbose(0);
        embree::rtcStartThreads(0);
    });
    RefSession* S = new RefSession();
    S->P = *params;
    S->media = media;
    S->n_media = n_media;
    S->lv = lv;
    S->beams = beams;
    S->cam_mis = cam_mis;
    S->sq = sq;
    S->pq = pq;
    S->what = what;
    S->nthreads = threads > 0 ? threads : omp_get_max_threads();
    S->worlds.resize(S->nthreads);
    auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel num_threads(S->nthreads)
    {
        const int tid = omp_get_thread_num();
        S->worlds[tid].reset(new World());
        setup_world(*S->worlds[tid], S->P, media, n_media, lv, beams, what);
    }
    S->build_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return S;
}

extern "C" void ref_release(void* h) { delete static_cast<RefSession*>(h); }

/* The radii the reference's builds assigned (session prepared with PB2D and BB1D_BRUTE):
 * ph_r2[light vertex] = EmbreePhoton::radiusSqr (0 for vertices that are no photon), and per beam
 * mStartRadius, mEndRadius, mMaxRadiusSqr.  Any pointer may be NULL. */
extern "C" int ref_radii(void* h, float* ph_r2, float* bm_start, float* bm_end, float* bm_r2)
{
    RefSession* S = static_cast<RefSession*>(h);
    if (!S || S->worlds.empty() || !S->worlds[0]) return -1;
    UPBP& U = *S->worlds[0]->upbp;
    if (ph_r2 && !U.mLightVertices.empty())
        ref_bre_radii(U.mPB2DEmbreeBre, &U.mLightVertices[0], (int64_t)U.mLightVertices.size(), ph_r2);
    for (size_t b = 0; b < U.mPhotonBeamsArray.size(); ++b) {
        const PhotonBeam& pb = U.mPhotonBeamsArray[b];
        if (bm_start) bm_start[b] = pb.mStartRadius;
        if (bm_end) bm_end[b] = pb.mEndRadius;
        if (bm_r2) bm_r2[b] = pb.mMaxRadiusSqr;
    }
    return 0;
}

/* The reference grid of a session prepared with REF_BB1D_GRID: mCells, mPointers as beam indices
 * and mPdfs (ref_beams.cpp:ref_grid_export, where the grid class is visible).  NULL outputs only
 * report the sizes. */
int ref_grid_export(const PhotonBeamsEvaluator& e, const PhotonBeam* base, uint32_t* cells, int32_t* beams, float* pdfs,
                    int64_t* n_cells, int64_t* n_entries);

extern "C" int ref_grid_structure(void* h, uint32_t* cells, int32_t* beams, float* pdfs, int64_t* n_cells,
                                  int64_t* n_entries)
{
    RefSession* S = static_cast<RefSession*>(h);
    if (!S || S->worlds.empty() || !S->worlds[0]) return -1;
    UPBP& U = *S->worlds[0]->upbp;
    if (!U.mBB1DPhotonBeams.accelStruct || U.mPhotonBeamsArray.empty()) return -2;
    return ref_grid_export(U.mBB1DPhotonBeams, &U.mPhotonBeamsArray[0], cells, beams, pdfs, n_cells, n_entries);
}

/* Evaluate queries q = offset + k*stride; returns the wall time in ms through out->gather_ms. */
extern "C" int ref_eval(void* h, int64_t offset, int64_t stride, ref_outputs* out)
{
    RefSession* S = static_cast<RefSession*>(h);
    if (!S || !out || stride < 1 || offset < 0) return -1;
    const upbp_params& P = S->P;
    const int nthreads = S->nthreads;
    const int32_t what = S->what;
    const upbp_segment_queries* sq = S->sq;
    const upbp_point_queries* pq = S->pq;
    const upbp_mis* cam_mis = S->cam_mis;
    const int64_t npix = (int64_t)P.image_width * P.image_height;
    std::vector<std::vector<float>> images(out->image ? nthreads : 0, std::vector<float>(out->image ? 3 * npix : 0, 0.f));
    std::vector<std::unique_ptr<World>>& worlds = S->worlds;
    auto t1 = std::chrono::steady_clock::now();
    const int64_t nq = sq ? sq->n : 0;
    const int64_t np = pq ? pq->n : 0;
#pragma omp parallel num_threads(nthreads)
    {
        const int tid = omp_get_thread_num();
        World& w = *worlds[tid];
        UPBP& U = *w.upbp;
        float* img = out->image ? images[tid].data() : nullptr;
        const uint tech = P.techniques;
        const uint rsf_in = AbstractMedium::kOriginInMedium;
#pragma omp for schedule(dynamic, 16)
        for (int64_t q = offset; q < nq; q += stride) {
            const int L = sq->path_length[q];
            const uint qf = sq->flags[q];
            const bool lite = (qf & UPBP_Q_LITE) != 0;
            const uint rsf = (qf & UPBP_Q_ORIGIN_IN_MEDIUM) ? rsf_in : 0;
            const Ray ray(P3(sq->origin + 3 * q), D3(sq->direction + 3 * q));
            VolumeSegments segs;
            LiteVolumeSegments lsegs;
            const int sb = sq->seg_begin[q], sc = sq->seg_count[q];
            for (int s = sb; s < sb + sc; ++s) {
                if (lite) {
                    VolumeSegmentLite l;
                    l.mDistMin = sq->seg_dist_min[s];
                    l.mDistMax = sq->seg_dist_max[s];
                    l.mMediumID = sq->seg_medium[s];
                    lsegs.push_back(l);
                } else {
                    VolumeSegment v;
                    v.mDistMin = sq->seg_dist_min[s];
                    v.mDistMax = sq->seg_dist_max[s];
                    v.mRaySamplePdf = sq->seg_pdf[s];
                    v.mRaySampleRevPdf = sq->seg_rev_pdf[s];
                    v.mAttenuation = C3(sq->seg_attenuation + 3 * s);
                    v.mEmission = Rgb(0.f);
                    v.mMediumID = sq->seg_medium[s];
                    segs.push_back(v);
                }
            }
            const Rgb thr = C3(sq->throughput + 3 * q);
            const BeamType qbt = (BeamType)P.query_beam_type;
            // PB2D, UPBP.hxx:775-785 / 879-893
            const bool nomis = (P.techniques & UPBP_NO_MIS) != 0;
            if ((qf & UPBP_Q_PB2D) && U.mMergeWithLightVerticesPB2D && !U.mLightVertices.empty()) {
                if ((what & REF_PB2D) && nomis) {
                    // VolLightTracer.hxx:378: evalBre(mPB2DBeamType, ray, mVolumeSegments)
                    const Rgb c = lite ? U.mPB2DEmbreeBre.evalBre(qbt, ray, lsegs, PB2D, 0, NULL)
                                       : U.mPB2DEmbreeBre.evalBre(qbt, ray, segs, PB2D, 0, NULL);
                    if (out->pb2d_rgb) for (int k = 0; k < 3; ++k) out->pb2d_rgb[3 * q + k] = c[k];
                    const int px = sq->pixel[q];
                    if (img && px >= 0) {
                        const Rgb add = thr * U.mPB2DNormalization * c;
                        for (int k = 0; k < 3; ++k) img[3 * px + k] += add[k];
                    }
                } else if (what & REF_PB2D) {
                    load_camera(U, cam_mis, sq->cam_mis_begin[q], L);
                    embree::AdditionalRayDataForMis data(
                        &U.mLightVertices, &U.mPathEnds, &U.mCameraVerticesMisData, L, U.mMinPathLength,
                        U.mMaxPathLength, U.mQueryBeamType, U.mPhotonBeamType, sq->last_pdf_w_inv[q],
                        U.mSurfMisWeightFactor, U.mPP3DMisWeightFactor, U.mPB2DMisWeightFactor, U.mBB1DMisWeightFactor,
                        (U.mMergeWithLightVerticesBB1D && !U.mPhotonBeamsArray.empty()) ? &U.mBB1DPhotonBeams : NULL,
                        U.mBB1DMinMFP, U.mLightSubPathCount, U.mMinDistToMed, 0.0f, 0.0f, 0, &U.mDebugImages);
                    const Rgb c = lite ? U.mPB2DEmbreeBre.evalBre(qbt, ray, lsegs, tech, rsf, &data)
                                       : U.mPB2DEmbreeBre.evalBre(qbt, ray, segs, tech, rsf, &data);
                    if (out->pb2d_rgb) for (int k = 0; k < 3; ++k) out->pb2d_rgb[3 * q + k] = c[k];
                    const int px = sq->pixel[q];
                    if (img && px >= 0) {
                        const Rgb add = thr * U.mPB2DNormalization * c;
                        for (int k = 0; k < 3; ++k) img[3 * px + k] += add[k];
                    }
                }
                if ((what & REF_CANDIDATES) && out->count_pb2d) {
                    uint32_t cnt = 0;
                    uint64_t h = 0;
                    Rgb att(1.f);
                    for (int s = sb; s < sb + sc; ++s) {
                        const AbstractMedium* m = w.scene.mMedia[sq->seg_medium[s]];
                        if (m->HasScattering())
                            ref_bre_candidates(U.mPB2DEmbreeBre, sq->origin + 3 * q, sq->direction + 3 * q,
                                               sq->seg_dist_min[s], sq->seg_dist_max[s], &U.mLightVertices[0], cnt, h);
                        if (lite) att *= m->EvalAttenuation(ray, sq->seg_dist_min[s], sq->seg_dist_max[s]);
                        else att *= qbt == SHORT_BEAM ? C3(sq->seg_attenuation + 3 * s) / sq->seg_pdf[s]
                                                      : C3(sq->seg_attenuation + 3 * s);
                        if (!att.isPositive()) break;
                    }
                    out->count_pb2d[q] = cnt;
                    out->hash_pb2d[q] = h;
                }
            }
            // BB1D, UPBP.hxx:788-798 / 897-911
            if ((qf & UPBP_Q_BB1D) && U.mMergeWithLightVerticesBB1D && !U.mPhotonBeamsArray.empty()) {
                for (int variant = 0; variant < 2; ++variant) {
                    if (variant == 0 && !(what & REF_BB1D_GRID)) continue;
                    if (variant == 1 && !(what & REF_BB1D_BRUTE)) continue;
                    Rgb c;
                    if (nomis) {
                        // VolLightTracer.hxx:384: evalBeamBeamEstimate(..., BB1D, 0, NULL, &gridStats)
                        GridStats gs;
                        if (variant == 0)
                            c = lite ? U.mBB1DPhotonBeams.evalBeamBeamEstimate(qbt, ray, lsegs, BB1D, 0, NULL, &gs)
                                     : U.mBB1DPhotonBeams.evalBeamBeamEstimate(qbt, ray, segs, BB1D, 0, NULL, &gs);
                        else
                            c = lite ? ref_brute_eval_lite(w.brute, qbt, ray, lsegs, BB1D, 0, NULL)
                                     : ref_brute_eval(w.brute, qbt, ray, segs, BB1D, 0, NULL);
                    } else {
                        load_camera(U, cam_mis, sq->cam_mis_begin[q], L);
                        embree::AdditionalRayDataForMis data(
                            &U.mLightVertices, &U.mPathEnds, &U.mCameraVerticesMisData, L, U.mMinPathLength,
                            U.mMaxPathLength, U.mQueryBeamType, U.mPhotonBeamType, sq->last_pdf_w_inv[q],
                            U.mSurfMisWeightFactor, U.mPP3DMisWeightFactor, U.mPB2DMisWeightFactor,
                            U.mBB1DMisWeightFactor, &U.mBB1DPhotonBeams, U.mBB1DMinMFP, U.mBB1DUsedLightSubPathCount,
                            U.mMinDistToMed, 0.0f, 0.0f, 0, &U.mDebugImages);
                        if (variant == 0)
                            c = lite ? U.mBB1DPhotonBeams.evalBeamBeamEstimate(qbt, ray, lsegs, tech, rsf, &data)
                                     : U.mBB1DPhotonBeams.evalBeamBeamEstimate(qbt, ray, segs, tech, rsf, &data);
                        else
                            c = lite ? ref_brute_eval_lite(w.brute, qbt, ray, lsegs, tech, rsf, &data)
                                     : ref_brute_eval(w.brute, qbt, ray, segs, tech, rsf, &data);
                    }
                    float* dst = variant == 0 ? out->bb1d_rgb : out->bb1d_brute_rgb;
                    if (dst) for (int k = 0; k < 3; ++k) dst[3 * q + k] = c[k];
                    const int px = sq->pixel[q];
                    // The image follows the brute-force estimate when it is computed: it
                    // defines the candidate set (the grid can differ where t1 falls on a
                    // DDA cell boundary, Grid.hxx:359-364).
                    const bool splat = variant == 1 || !(what & REF_BB1D_BRUTE);
                    if (img && px >= 0 && splat) {
                        const Rgb add = thr * U.mBB1DNormalization * c;
                        for (int k = 0; k < 3; ++k) img[3 * px + k] += add[k];
                    }
                }
                if ((what & REF_CANDIDATES) && out->count_bb1d) {
                    uint32_t cnt = 0;
                    uint64_t h = 0;
                    Rgb att(1.f);
                    for (int s = sb; s < sb + sc; ++s) {
                        const AbstractMedium* m = w.scene.mMedia[sq->seg_medium[s]];
                        if (m->HasScattering())
                            bb1d_candidates(U, ray, sq->seg_dist_min[s], sq->seg_dist_max[s], m, cnt, h);
                        if (lite) att *= m->EvalAttenuation(ray, sq->seg_dist_min[s], sq->seg_dist_max[s]);
                        else att *= qbt == SHORT_BEAM ? C3(sq->seg_attenuation + 3 * s) / sq->seg_pdf[s]
                                                      : C3(sq->seg_attenuation + 3 * s);
                        if (!att.isPositive()) break;
                    }
                    out->count_bb1d[q] = cnt;
                    out->hash_bb1d[q] = h;
                }
            }
        }
        // PP3D, UPBP.hxx:1114-1122
#pragma omp for schedule(dynamic, 16)
        for (int64_t q = offset; q < np; q += stride) {
            if (!U.mMergeWithLightVerticesPP3D || U.mLightVerticesInMediumCount == 0) continue;
            const int L = pq->path_length[q];
            const Pos hit = P3(pq->position + 3 * q);
            if (what & REF_PP3D) {
                load_camera(U, cam_mis, pq->cam_mis_begin[q], L + 1);
                const BSDF bsdf = medium_bsdf(w.scene, pq->dir_fix + 3 * q, pq->medium_id[q], BSDF::kFromCamera);
                const Rgb c = g_pp3d_fn(U, hit, bsdf, L);
                if (out->pp3d_rgb) for (int k = 0; k < 3; ++k) out->pp3d_rgb[3 * q + k] = c[k];
                const int px = pq->pixel[q];
                if (img && px >= 0) {
                    const Rgb add = C3(pq->throughput + 3 * q) * U.mPP3DNormalization * c;
                    for (int k = 0; k < 3; ++k) img[3 * px + k] += add[k];
                }
            }
            if ((what & REF_CANDIDATES) && out->count_pp3d) {
                CountQuery cq;
                cq.pos = hit;
                cq.base = &U.mLightVertices[0];
                U.mPP3DHashGrid.Process(U.mLightVertices, cq);
                out->count_pp3d[q] = cq.count;
                out->hash_pp3d[q] = cq.hash;
            }
        }
    }
    auto t2 = std::chrono::steady_clock::now();
    out->gather_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
    out->build_ms = S->build_ms;
    if (out->image) {
        for (int t = 0; t < nthreads; ++t)
            for (int64_t i = 0; i < 3 * npix; ++i) out->image[i] += images[t][i];
    }
    return 0;
}

extern "C" int ref_run(const upbp_params* params, const upbp_medium* media, int32_t n_media,
                       const upbp_light_vertices* lv, const upbp_beams* beams, const upbp_mis* cam_mis,
                       int64_t n_cam_mis, const upbp_segment_queries* sq, const upbp_point_queries* pq, int32_t what,
                       int64_t stride, int32_t threads, ref_outputs* out)
{
    (void)n_cam_mis;
    if (!out || stride < 1) return -1;
    void* h = ref_prepare(params, media, n_media, lv, beams, cam_mis, sq, pq, what, threads);
    if (!h) return -1;
    const int rc = ref_eval(h, 0, stride, out);
    ref_release(h);
    return rc;
}
