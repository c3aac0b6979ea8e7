// Gather kernels of the B200 estimator stage: one thread per recorded query.
//
//  * PB2D  : EmbreeBre::evalBre + breIntersectFuncHomogeneous2 (Bre/Bre.cxx:293-464, 812-964)
//  * BB1D  : PhotonBeamsEvaluator::evalBeamBeamEstimate + PhotonBeam::accumulate2
//            (Beams/PhBeams.cxx:177-324, Beams/PhotonBeam.hxx:386-607)
//  * PP3D  : HashGrid::Process + UPBP::RangeQuery::Process (Misc/HashGrid.hxx:129-188,
//            Renderers/UPBP.hxx:86-133)
// Candidate predicates use the reference operation order (upbp_device.cuh); the MIS weights
// walk the stored camera snapshot and light subpath exactly as Path/PathWeight.hxx does.
#include <cfloat>
#include <cstdint>

#include "upbp_kernels.cuh"
#include "upbp_mis_prep.cuh"
#include "upbp_traverse.cuh"

namespace upbp {

namespace {

// Camera MisData as the reference array holds it during an estimator call at path length L:
// entries < L-1 from the snapshot, entry L-1 from the snapshot with mRaySampleRevPdfInv set by
// the estimator, entry L written by the estimator for the candidate.
struct CamView {
    const upbp_mis* snap;
    int L;
    const upbp_mis* cand;
    float prev_ray_rev_inv;
    __device__ upbp_mis operator()(int k) const
    {
        if (k == L) return *cand;
        upbp_mis m = load_mis(snap + k);
        if (k == L - 1) m.ray_sample_rev_pdf_inv = prev_ray_rev_inv;
        return m;
    }
};

struct CamSnap {
    const upbp_mis* snap;
    __device__ upbp_mis operator()(int k) const { return load_mis(snap + k); }
};

struct LightView {
    const upbp_mis* mis;
    int override_idx;
    float override_ray_rev_inv;
    __device__ upbp_mis operator()(int k) const
    {
        upbp_mis m = load_mis(mis + k);
        if (k == override_idx) m.ray_sample_rev_pdf_inv = override_ray_rev_inv;
        return m;
    }
};

// Per-segment state that evalBre / evalBeamBeamEstimate hand to the callbacks through
// AdditionalRayDataForMis (Bre.cxx:839-850, PhBeams.cxx:198-210).
struct SegCtx {
    V3 o, d;
    float dmin, dmax;
    float rs_pdf, rs_rev_pdf;  // mRaySamplePdf / mRaySampleRevPdf accumulated over earlier segments
    uint32_t rsf;              // mRaySamplingFlags
    int L;
    float last_pdf_w_inv;
    uint32_t ray_flags;        // beamType | estimatorTechniques
    const upbp_mis* cam;
    // mixed mode: camera entry L-1 and the FP64 suffix of the camera walk (the warp kernel keeps
    // them in shared memory: they are the same for the whole warp)
    const upbp_mis* e;
    const CamSum* cs;
};

__device__ __forceinline__ void fill_cand(upbp_mis& c, const upbp_params& P, float pdf_a_inv, float rsp_inv,
                                          float ratio, float sel_pdf, uint32_t flags)
{
    c.pdf_a_inv = pdf_a_inv;
    c.rev_pdf_a = 1.f;
    c.rev_pdf_a_without_bsdf = 1.f;
    c.ray_sample_pdf_inv = rsp_inv;
    c.ray_sample_rev_pdf_inv = 1.f;
    c.ray_sample_pdfs_ratio = ratio;
    c.ray_sample_rev_pdfs_ratio = 0.f;
    c.sin_theta = 0.f;
    c.cos_theta_out = 0.f;
    c.surf_factor = 0.f;
    c.pp3d_factor = P.mis_factor_pp3d;
    c.pb2d_factor = P.mis_factor_pb2d;
    c.bb1d_factor = P.mis_factor_bb1d;
    c.bb1d_beam_selection_pdf = sel_pdf;
    c.flags = flags;
}

// ----------------------------------------------------------------- estimators without MIS
// breIntersectFuncHomogeneous (Bre.cxx:239-291), the callback of VolLightTracer's pure PB2D: the
// photon's flux (its light vertex's throughput) x transmittance to the photon (over the
// free-flight pdf for SHORT query beams) x sigma_s x HG x the 2-D Epanechnikov kernel, with no
// rejects and no MIS weight.  The reference's expression divides the product by r^2 pi / 2.
__device__ __forceinline__ Rgb pb2d_contrib_nomis(const DMedium& m, const LightSoA& Lv, const SegCtx& s, int lv,
                                                  float t, float d2, float r2)
{
    Rgb att = eval_att(m, t - s.dmin);
    if (s.ray_flags & UPBP_SHORT_BEAM) att = att / comp(att, m.min_idx);
    const float4 ld = __ldg(&Lv.dir[lv]);
    const float4 th = __ldg(&Lv.thr[lv]);
    float sinT;
    const float phase = hg_pdf(s.d, neg3(v3(ld.x, ld.y, ld.z)), m.g, &sinT);
    const Rgb ss{m.ss[0], m.ss[1], m.ss[2]};
    return (Rgb{th.x, th.y, th.z} * att * ss * phase * (1.f - d2 / r2)) / (r2 * UPBP_PI_F * 0.5f);
}

// PhotonBeam::accumulate without MIS data (PhotonBeam.hxx:315-367), VolLightTracer's pure BB1D:
// (1 / beam selection pdf, 1 without beam reduction) x the beam's throughput x sigma_s x the query
// and beam transmittances (each over its free-flight pdf for SHORT beams) x HG x the 1-D kernel.
// The candidate test and the radius test are the caller's, as for accumulate2.
__device__ __forceinline__ Rgb bb1d_contrib_nomis(const DMedium& m, const SegCtx& s, float4 bthr, bool beam_short,
                                                  V3 bdir, float radius, float dist, float sinTheta, float t1,
                                                  float t2)
{
    Rgb att = eval_att(m, t1 - s.dmin);
    const Rgb batt = eval_att(m, t2);
    if (s.ray_flags & UPBP_SHORT_BEAM) att = att / comp(att, m.min_idx);
    att = att * batt;
    if (beam_short) att = att / comp(batt, m.min_idx);
    float sinDummy;
    const float phase = hg_pdf(s.d, bdir, m.g, &sinDummy);
    const Rgb ss{m.ss[0], m.ss[1], m.ss[2]};
    return ((1.0f * Rgb{bthr.x, bthr.y, bthr.z} * ss * att * phase * (1.f - dist * dist / (radius * radius))) * 3.f) /
           (4.f * radius * sinTheta);
}

// ----------------------------------------------------------------- PB2D contribution
// breIntersectFuncHomogeneous2 after testIntersectionBre accepted photon `lv` at (t, d2).
template <bool kMixed>
__device__ Rgb pb2d_contrib(const GatherConsts& K, const DMedium& m, const LightSoA& Lv, const SegCtx& s, int lv,
                            float t, float d2, float r2)
{
    const upbp_params& P = K.P;
    if (P.techniques & UPBP_NO_MIS) return pb2d_contrib_nomis(m, Lv, s, lv, t, d2, r2);
    const int4 info = __ldg(&Lv.info[lv]);
    const int pl = info.y;
    if ((uint32_t)(pl + s.L) > P.max_path_length || (uint32_t)(pl + s.L) < P.min_path_length) return rgb(0.f);
    if (s.L == 1 && t < P.min_dist_to_med) return rgb(0.f);
    Rgb att = eval_att(m, t - s.dmin);
    const float pdf = comp(att, m.min_idx);
    if (s.ray_flags & UPBP_SHORT_BEAM) att = att / pdf;
    float rsp = m.min_st * pdf;
    float rsr = (s.rsf & UPBP_ORIGIN_IN_MEDIUM) ? rsp : pdf;
    const float ratio = 1.0f / m.min_st;
    if (!rgb_positive(att)) return rgb(0.f);
    rsp *= s.rs_pdf;
    rsr *= s.rs_rev_pdf;
    const float4 ld = __ldg(&Lv.dir[lv]);
    float sinT;
    const float phase = hg_pdf(neg3(s.d), v3(ld.x, ld.y, ld.z), m.g, &sinT);
    if (phase <= 0.f) return rgb(0.f);
    const float camDirPdfW = phase * m.cont;
    const float camRevPdfW = phase * __ldg(&Lv.pos[lv]).w;
    const float kernel = (1.f - d2 / r2) / (r2 * UPBP_PI_F * 0.5f);  // the photon's radiusSqr
    if (!is_pos(kernel)) return rgb(0.f);
    const float4 th = __ldg(&Lv.thr[lv]);
    const Rgb ss{m.ss[0], m.ss[1], m.ss[2]};
    const Rgb unweighted = Rgb{th.x, th.y, th.z} * att * ss * phase * kernel;
    if (rgb_black_or_neg(unweighted)) return rgb(0.f);
    const float distSq = t * t;
    const float rspInv = 1.0f / rsp;
    upbp_mis cand;
    fill_cand(cand, P, s.last_pdf_w_inv * distSq * rspInv, rspInv, ratio, K.has_bb1d_beams ? 1.f : 0.f,
              (m.mfp > P.bb1d_min_mfp) ? UPBP_MIS_IN_MEDIUM_WITH_BEAMS : 0u);
    const float last = (s.ray_flags & UPBP_SHORT_BEAM) ? (float)(1.0 / (double)(ratio * cand.pb2d_factor))
                                                       : rsp / cand.pb2d_factor;
    const upbp_mis lvm = load_mis(Lv.mis + lv);
    if (kMixed) {
        const float wc = camera_weight_fast(s.L, cand, last, sinT, lvm.ray_sample_pdf_inv, lvm.ray_sample_pdfs_ratio,
                                            camRevPdfW * rsr / distSq, *s.e, 1.0f / rsr, *s.cs, s.ray_flags,
                                            P.query_beam_type, P.photon_beam_type);
        const LightSum ls = Lv.sums[lv];
        const float wl = last * ((float)ls.a + camDirPdfW * (float)ls.c);
        return (1.0f / (wl + wc)) * unweighted;
    }
    const CamView cam{s.cam, s.L, &cand, 1.0f / rsr};
    const float wCamera = camera_path_weight(s.L, last, sinT, lvm.ray_sample_pdf_inv, lvm.ray_sample_pdfs_ratio,
                                             camRevPdfW * rsr / distSq, P.query_beam_type, P.photon_beam_type,
                                             s.ray_flags, cam);
    const LightView lview{Lv.mis, -1, 0.f};
    const float wLight = light_path_weight(info.x, pl, last, 0.f, 0.f, 0.f, camDirPdfW, UPBP_PB2D, P.query_beam_type,
                                           P.photon_beam_type, s.ray_flags, Lv.path_ends, lview, nullptr);
    const float w = 1.f / (wLight + wCamera);
    return w * unweighted;
}

// ----------------------------------------------------------------- BB1D contribution
// PhotonBeam::accumulate2 after testIntersectionBeamBeam and the radius test accepted `beam`.
// FP64 closest approach of the query line and the beam line (unit directions), used in mixed
// mode for near-parallel pairs where the FP32 solve of PhotonBeam.hxx:253-293 cancels.
__device__ __forceinline__ void closest_approach_f64(V3 O1, V3 d1, V3 O2, V3 d2, float& dist, float& sinT, float& t1,
                                                     float& t2)
{
    const double ax = d1.x, ay = d1.y, az = d1.z, bx = d2.x, by = d2.y, bz = d2.z;
    const double wx = (double)O1.x - O2.x, wy = (double)O1.y - O2.y, wz = (double)O1.z - O2.z;
    const double cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
    const double s2 = cx * cx + cy * cy + cz * cz;
    const double b = ax * bx + ay * by + az * bz;
    const double dd = ax * wx + ay * wy + az * wz;
    const double ee = bx * wx + by * wy + bz * wz;
    const double aa = ax * ax + ay * ay + az * az, cc = bx * bx + by * by + bz * bz;
    const double den = aa * cc - b * b;
    const double s = sqrt(s2);
    t1 = (float)((b * ee - cc * dd) / den);
    t2 = (float)((aa * ee - b * dd) / den);
    dist = (float)(fabs(-wx * cx - wy * cy - wz * cz) / s);
    sinT = (float)s;
}

template <bool kMixed>
__device__ Rgb bb1d_contrib(const GatherConsts& K, const DMedium& m, const LightSoA& Lv, const BeamSoA& Bs,
                            const SegCtx& s, int beam, V3 bo, V3 bdir, float radius, float dist, float sinTheta,
                            float t1, float t2)
{
    if (kMixed) {
        // near-parallel lines: 1 - (d1.d2)^2 small (PhotonBeam.hxx:267-273 rejects only below 1e-5)
        const float c = s.d.x * bdir.x + s.d.y * bdir.y + s.d.z * bdir.z;
        if (1.f - c * c < 1e-2f) closest_approach_f64(s.o, s.d, bo, bdir, dist, sinTheta, t1, t2);
    }
    const upbp_params& P = K.P;
    if (P.techniques & UPBP_NO_MIS) {
        const float4 bthr = __ldg(&Bs.thr[beam]);
        const bool bshort = ((uint32_t)__float_as_int(bthr.w) & UPBP_SHORT_BEAM) != 0;
        return bb1d_contrib_nomis(m, s, bthr, bshort, bdir, radius, dist, sinTheta, t1, t2);
    }
    const int2 link = __ldg(&Bs.link[beam]);
    const int lvi = link.x;
    const int4 info = __ldg(&Lv.info[lvi]);
    const int pl = info.y;
    if ((uint32_t)(pl + 1 + s.L) > P.max_path_length || (uint32_t)(pl + 1 + s.L) < P.min_path_length) return rgb(0.f);
    if (s.L == 1 && t1 < P.min_dist_to_med) return rgb(0.f);
    const float4 bthr = __ldg(&Bs.thr[beam]);
    const float4 bpdf = __ldg(&Bs.pdf[beam]);
    const uint32_t bflags = (uint32_t)__float_as_int(bthr.w);
    const uint32_t brsf = (uint32_t)__float_as_int(bpdf.w);
    // query side
    Rgb att = eval_att(m, t1 - s.dmin);
    const float pfdQ = comp(att, m.min_idx);
    if (s.ray_flags & UPBP_SHORT_BEAM) att = att / pfdQ;
    float rspQ = m.min_st * pfdQ;
    float rsrQ = (s.rsf & UPBP_ORIGIN_IN_MEDIUM) ? rspQ : pfdQ;
    const float ratioQ = 1.0f / m.min_st;
    // beam side
    const Rgb batt = eval_att(m, t2);
    att = att * batt;
    const float pfdB = comp(batt, m.min_idx);
    if (bflags & UPBP_SHORT_BEAM) att = att / pfdB;
    float rspB = m.min_st * pfdB;
    float rsrB = (brsf & UPBP_ORIGIN_IN_MEDIUM) ? rspB : pfdB;
    const float ratioB = 1.0f / m.min_st;
    if (!rgb_positive(att)) return rgb(0.f);
    rspQ *= s.rs_pdf;
    rsrQ *= s.rs_rev_pdf;
    rspB *= bpdf.x;
    rsrB *= bpdf.y;
    float sinDummy;
    const float phase = hg_pdf(neg3(s.d), neg3(bdir), m.g, &sinDummy);
    if (phase <= 0.f) return rgb(0.f);
    const float bsdfDirPdfW = phase * m.cont;
    const float bsdfRevPdfW = phase * m.cont;
    const float sel = 1.0f;  // no beam reduction (sMaxBeamsInCell == 0)
    const Rgb ss{m.ss[0], m.ss[1], m.ss[2]};
    const Rgb unweighted = ((1.0f / sel) * Rgb{bthr.x, bthr.y, bthr.z} * ss * att * phase *
                            (1.f - dist * dist / (radius * radius))) * 3.f / (4.f * radius * sinTheta);
    if (rgb_black_or_neg(unweighted)) return rgb(0.f);
    const float distSqQ = t1 * t1;
    const float rspInvQ = 1.0f / rspQ;
    upbp_mis cand;
    fill_cand(cand, P, s.last_pdf_w_inv * distSqQ * rspInvQ, rspInvQ, ratioQ, sel, UPBP_MIS_IN_MEDIUM_WITH_BEAMS);
    const bool finite = (info.z & UPBP_LV_IS_FINITE) != 0;
    const float distSqB = finite ? t2 * t2 : 1.0f;
    const float rspInvB = 1.0f / rspB;
    upbp_mis brec;
    fill_cand(brec, P, bpdf.z * distSqB * rspInvB, rspInvB, ratioB, sel, UPBP_MIS_IN_MEDIUM_WITH_BEAMS);
    float sinT = sinTheta;
    if (s.ray_flags & UPBP_NO_SINE_IN_WEIGHTS) sinT = 1.0f;
    const float f = cand.bb1d_factor;
    float last;
    if (s.ray_flags & UPBP_SHORT_BEAM)
        last = (bflags & UPBP_SHORT_BEAM) ? (float)(1.0 / (double)(ratioQ * ratioB * f * sel * sinT))
                                          : rspB / (ratioQ * f * sel * sinT);
    else
        last = (bflags & UPBP_SHORT_BEAM) ? rspQ / (ratioB * f * sel * sinT) : rspQ * rspB / (f * sel * sinT);
    const upbp_mis lvm = load_mis(Lv.mis + lvi);
    const bool onDeltaLight = (lvm.flags & UPBP_MIS_ON_LIGHT_SOURCE) && (lvm.flags & UPBP_MIS_IS_DELTA);
    const float ntl = onDeltaLight ? 0.f : bsdfDirPdfW * rsrB * fabsf(lvm.cos_theta_out) / distSqB;
    if (kMixed) {
        const float wc = camera_weight_fast(s.L, cand, last, sinT, rspInvB, ratioB, bsdfRevPdfW * rsrQ / distSqQ, *s.e,
                                            1.0f / rsrQ, *s.cs, s.ray_flags, P.query_beam_type, P.photon_beam_type);
        const LightSum ls = Lv.sums[lvi];
        float inner = ls.bptb;
        if (!(s.ray_flags & UPBP_PREVIOUS)) inner += ntl * ((float)ls.d + (float)ls.e / rsrB);
        const float wl = last * brec.pdf_a_inv * inner;
        return (1.0f / (wl + wc)) * unweighted;
    }
    const CamView cam{s.cam, s.L, &cand, 1.0f / rsrQ};
    const float wCamera = camera_path_weight(s.L, last, sinT, rspInvB, ratioB, bsdfRevPdfW * rsrQ / distSqQ,
                                             P.query_beam_type, P.photon_beam_type, s.ray_flags, cam);
    const LightView lview{Lv.mis, lvi, 1.0f / rsrB};
    const float wLight = light_path_weight(info.x, pl + 1, last, 0.f, 0.f, 0.f, ntl, UPBP_BB1D, P.query_beam_type,
                                           P.photon_beam_type, s.ray_flags, Lv.path_ends, lview, &brec);
    const float w = 1.f / (wLight + wCamera);
    return w * unweighted;
}

// PhotonBeam::accumulate2 (mixed mode) with the beam's payload packed per piece.
__device__ Rgb bb1d_contrib_packed(const GatherConsts& K, const DMedium& m, const SegCtx& s, const PiecePayload& py,
                                   V3 bo, V3 bdir, float dist, float sinTheta, float t1, float t2, float radius)
{
    const upbp_params& P = K.P;
    const unsigned lvbits = (unsigned)__float_as_int(py.lv.w);
    if (P.techniques & UPBP_NO_MIS)
        return bb1d_contrib_nomis(m, s, py.thr, (lvbits & kPayShortBeam) != 0, bdir, radius, dist, sinTheta, t1, t2);
    const int pl = (int)(lvbits & kPayPathMask);
    const bool finite = (lvbits & kPayFinite) != 0;
    if ((uint32_t)(pl + 1 + s.L) > P.max_path_length || (uint32_t)(pl + 1 + s.L) < P.min_path_length) return rgb(0.f);

    if (s.L == 1 && t1 < P.min_dist_to_med) return rgb(0.f);
    const uint32_t bflags = (lvbits & kPayShortBeam) ? UPBP_SHORT_BEAM : 0u;
    const uint32_t brsf = (lvbits & kPayOriginInMedium) ? UPBP_ORIGIN_IN_MEDIUM : 0u;
    Rgb att = eval_att(m, t1 - s.dmin);
    const float pfdQ = comp(att, m.min_idx);
    if (s.ray_flags & UPBP_SHORT_BEAM) att = att / pfdQ;
    float rspQ = m.min_st * pfdQ;
    float rsrQ = (s.rsf & UPBP_ORIGIN_IN_MEDIUM) ? rspQ : pfdQ;
    const float ratioQ = 1.0f / m.min_st;
    const Rgb batt = eval_att(m, t2);
    att = att * batt;
    const float pfdB = comp(batt, m.min_idx);
    if (bflags & UPBP_SHORT_BEAM) att = att / pfdB;
    float rspB = m.min_st * pfdB;
    float rsrB = (brsf & UPBP_ORIGIN_IN_MEDIUM) ? rspB : pfdB;
    const float ratioB = ratioQ;
    if (!rgb_positive(att)) return rgb(0.f);
    rspQ *= s.rs_pdf;
    rsrQ *= s.rs_rev_pdf;
    rspB *= py.pdf.x;
    rsrB *= py.pdf.y;
    float sinDummy;
    const float phase = hg_pdf(neg3(s.d), neg3(bdir), m.g, &sinDummy);
    if (phase <= 0.f) return rgb(0.f);
    const float bsdfPdfW = phase * m.cont;
    const Rgb ss{m.ss[0], m.ss[1], m.ss[2]};
    const Rgb unweighted = (Rgb{py.thr.x, py.thr.y, py.thr.z} * ss * att * phase *
                            (1.f - dist * dist / (radius * radius))) * 3.f / (4.f * radius * sinTheta);
    if (rgb_black_or_neg(unweighted)) return rgb(0.f);
    const float distSqQ = t1 * t1;
    const float rspInvQ = 1.0f / rspQ;
    upbp_mis cand;
    fill_cand(cand, P, s.last_pdf_w_inv * distSqQ * rspInvQ, rspInvQ, ratioQ, 1.0f, UPBP_MIS_IN_MEDIUM_WITH_BEAMS);
    const float distSqB = finite ? t2 * t2 : 1.0f;
    const float rspInvB = 1.0f / rspB;
    const float brecPdfAInv = py.pdf.z * distSqB * rspInvB;
    const float sinT = (s.ray_flags & UPBP_NO_SINE_IN_WEIGHTS) ? 1.0f : sinTheta;
    const float f = cand.bb1d_factor;
    float last;
    if (s.ray_flags & UPBP_SHORT_BEAM)
        last = (bflags & UPBP_SHORT_BEAM) ? (float)(1.0 / (double)(ratioQ * ratioB * f * sinT))
                                          : rspB / (ratioQ * f * sinT);
    else
        last = (bflags & UPBP_SHORT_BEAM) ? rspQ / (ratioB * f * sinT) : rspQ * rspB / (f * sinT);
    const float wc = camera_weight_fast(s.L, cand, last, sinT, rspInvB, ratioB, bsdfPdfW * rsrQ / distSqQ, *s.e,
                                        1.0f / rsrQ, *s.cs, s.ray_flags, P.query_beam_type, P.photon_beam_type);
    const float ntl = bsdfPdfW * rsrB * py.lv.x / distSqB;
    float inner = py.lv.y;
    if (!(s.ray_flags & UPBP_PREVIOUS)) inner += ntl * (py.thr.w + py.pdf.w / rsrB);
    const float wl = last * brecPdfAInv * inner;
    return (1.0f / (wl + wc)) * unweighted;
}

// ----------------------------------------------------------------- segment loop
// The per-segment driver of evalBre / evalBeamBeamEstimate (full and lite segments).
template <class PerSegment>
__device__ __forceinline__ Rgb segment_loop(const GatherConsts& K, const DMedium* media, const SegQueriesDev& Q,
                                            int64_t q, SegCtx& s, PerSegment&& per_segment)
{
    const uint32_t qf = Q.flags[q];
    const bool lite = (qf & UPBP_Q_LITE) != 0;
    const uint32_t qrsf = (qf & UPBP_Q_ORIGIN_IN_MEDIUM) ? UPBP_ORIGIN_IN_MEDIUM : 0u;
    const uint32_t bt = K.P.query_beam_type;
    Rgb result = rgb(0.f), attn = rgb(1.f);
    float rsp = 1.f, rsr = 1.f;
    const int sb = Q.seg_begin[q], sc = Q.seg_count[q];
    for (int i = 0; i < sc; ++i) {
        const int sg = sb + i;
        const DMedium& m = media[Q.seg_medium[sg]];
        const float dmin = Q.seg_dist_min[sg], dmax = Q.seg_dist_max[sg];
        Rgb seg = rgb(0.f);
        if (m.has_scat) {
            s.dmin = dmin;
            s.dmax = dmax;
            s.rs_pdf = rsp;
            s.rs_rev_pdf = rsr;
            s.rsf = UPBP_END_IN_MEDIUM | (i == 0 ? qrsf : 0u);
            seg = per_segment(m);
        }
        result = result + attn * seg;
        if (lite) {
            attn = attn * eval_att(m, dmax - dmin);
            float srev;
            const float spdf = ray_sample_pdf(m, dmin, dmax, i == 0 ? qrsf : 0u, &srev);
            if (!rgb_positive(attn)) break;
            rsp *= spdf;
            rsr *= srev;
        } else {
            const Rgb sa{Q.seg_attenuation[3 * sg], Q.seg_attenuation[3 * sg + 1], Q.seg_attenuation[3 * sg + 2]};
            attn = attn * (bt == UPBP_SHORT_BEAM ? sa / Q.seg_pdf[sg] : sa);
            if (!rgb_positive(attn)) break;
            rsp *= Q.seg_pdf[sg];
            rsr *= Q.seg_rev_pdf[sg];
        }
    }
    return result;
}

template <bool kMixed>
__device__ __forceinline__ void init_seg_ctx(SegCtx& s, const GatherConsts& K, const SegQueriesDev& Q,
                                             const upbp_mis* cam, const CamSum* cs, int64_t q, upbp_mis* e_store,
                                             CamSum* cs_store, bool leader = true)
{
    s.o = v3(Q.origin[3 * q], Q.origin[3 * q + 1], Q.origin[3 * q + 2]);
    s.d = v3(Q.direction[3 * q], Q.direction[3 * q + 1], Q.direction[3 * q + 2]);
    s.L = Q.path_length[q];
    s.last_pdf_w_inv = Q.last_pdf_w_inv[q];
    s.ray_flags = K.P.query_beam_type | K.P.techniques;
    s.cam = cam + Q.cam_mis_begin[q];
    s.e = e_store;
    s.cs = cs_store;
    if (kMixed && leader && !(K.P.techniques & UPBP_NO_MIS)) {
        if (s.L >= 2) *e_store = load_mis(s.cam + s.L - 1);
        *cs_store = cs[q];
    }
}

__device__ __forceinline__ void write_out(const Outputs& O, int64_t q, Rgb v, uint32_t cnt, unsigned long long h,
                                          const SegQueriesDev& Q, float norm)
{
    O.rgb[3 * q + 0] = v.r;
    O.rgb[3 * q + 1] = v.g;
    O.rgb[3 * q + 2] = v.b;
    if (O.count) O.count[q] = cnt;
    if (O.hash) O.hash[q] = h;
    const Rgb thr{Q.throughput[3 * q], Q.throughput[3 * q + 1], Q.throughput[3 * q + 2]};
    splat(O.image, Q.pixel[q], thr * norm * v);
}

// ----------------------------------------------------------------- kernels
template <bool kMixed>
__global__ void __launch_bounds__(256) k_gather_pb2d(const __grid_constant__ GatherConsts K, const LightSoA Lv,
                                                     const PhotonBVH B, const SegQueriesDev Q,
                                                     const upbp_mis* __restrict__ cam, const CamSum* __restrict__ cs,
                                                     const Outputs O, const int32_t* __restrict__ order)
{
    __shared__ DMedium media[UPBP_MAX_MEDIA];
    stage_media(K, media);
    const int64_t item = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (item >= Q.n) return;
    const int64_t q = order ? (int64_t)__ldg(&order[item]) : item;
    uint32_t cnt = 0;
    unsigned long long h = 0, tested = 0;
    Rgb res = rgb(0.f);
    if ((Q.flags[q] & UPBP_Q_PB2D) && (K.P.techniques & UPBP_PB2D) && B.n > 0) {
        SegCtx s;
        upbp_mis e_store;
        CamSum cs_store;
        init_seg_ctx<kMixed>(s, K, Q, cam, cs, q, &e_store, &cs_store);
        const V3 inv = v3(safe_inv(s.d.x), safe_inv(s.d.y), safe_inv(s.d.z));
        const float r2 = K.P.radius_pb2d * K.P.radius_pb2d;
        res = segment_loop(K, media, Q, q, s, [&](const DMedium& m) {
            Rgb acc = rgb(0.f);
            traverse(B.nodes, B.n_leaves, s.o, inv, s.dmin - K.eps, s.dmax + K.eps, [&](int leaf) {
                const int e = min(B.n, (leaf + 1) * B.leaf);
                for (int i = leaf * B.leaf; i < e; ++i) {
                    const float4 p = __ldg(&B.pos[i]);
                    ++tested;
                    float t, d2;
                    const float r2i = B.r2 ? __ldg(&B.r2[i]) : r2;
                    if (test_bre(s.o, s.d, s.dmin, s.dmax, v3(p.x, p.y, p.z), r2i, &t, &d2)) {
                        const int lv = __float_as_int(p.w);
                        ++cnt;
                        h += mix64((unsigned long long)lv);
                        acc = acc + pb2d_contrib<kMixed>(K, m, Lv, s, lv, t, d2, r2i);
                    }
                }
            });
            return acc;
        });
    }
    write_out(O, q, res, cnt, h, Q, K.P.norm_pb2d);
    if (O.tested) atomicAdd(O.tested, tested);
}

template <bool kMixed>
__global__ void __launch_bounds__(256) k_gather_bb1d(const __grid_constant__ GatherConsts K, const LightSoA Lv,
                                                     const BeamBVH B, const BeamSoA Bs, const SegQueriesDev Q,
                                                     const upbp_mis* __restrict__ cam, const CamSum* __restrict__ cs,
                                                     const Outputs O)
{
    __shared__ DMedium media[UPBP_MAX_MEDIA];
    stage_media(K, media);
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= Q.n) return;
    uint32_t cnt = 0;
    unsigned long long h = 0, tested = 0;
    Rgb res = rgb(0.f);
    if ((Q.flags[q] & UPBP_Q_BB1D) && (K.P.techniques & UPBP_BB1D) && B.n > 0) {
        SegCtx s;
        upbp_mis e_store;
        CamSum cs_store;
        init_seg_ctx<kMixed>(s, K, Q, cam, cs, q, &e_store, &cs_store);
        const V3 inv = v3(safe_inv(s.d.x), safe_inv(s.d.y), safe_inv(s.d.z));
        res = segment_loop(K, media, Q, q, s, [&](const DMedium& m) {
            Rgb acc = rgb(0.f);
            const int mid = (int)(&m - media);
            traverse(B.nodes, B.n_leaves, s.o, inv, s.dmin - K.eps, s.dmax + K.eps, [&](int leaf) {
                const int e = min(B.n, (leaf + 1) * B.leaf);
                for (int i = leaf * B.leaf; i < e; ++i) {
                    const float4 pc = __ldg(&B.pc[i]);
                    if (__float_as_int(pc.w) != mid) continue;  // mMedium == medium (PhotonBeam.hxx:390)
                    const float4 pa = __ldg(&B.pa[i]);
                    const float4 pb = __ldg(&B.pb[i]);
                    ++tested;
                    float dist, sinT, t1, t2, bb, ee;
                    if (!test_beam_beam(s.o, s.d, s.dmin, s.dmax, v3(pa.x, pa.y, pa.z), v3(pb.x, pb.y, pb.z), 0.f, pa.w,
                                        pb.w, &dist, &sinT, &t1, &t2, &bb, &ee))
                        continue;
                    const int beam = __float_as_int(pc.z);
                    const float rs = beam_start_radius(Bs, &Bs.radius[beam]);
                    const float radius = beam_radius_at(Bs, beam, rs, t2);
                    if (radius < dist) continue;  // PhotonBeam.hxx:411-413
                    if (!piece_takes(s.o, s.d, s.dmin, s.dmax, v3(pa.x, pa.y, pa.z), v3(pb.x, pb.y, pb.z), pa.w, pc.x,
                                     pc.y, t1, bb, ee, dist, rs, Bs.rchange ? __ldg(&Bs.rchange[beam]) : 0.f,
                                     K.bb1d_extra))
                        continue;
                    ++cnt;
                    h += mix64((unsigned long long)beam);
                    acc = acc + bb1d_contrib<kMixed>(K, m, Lv, Bs, s, beam, v3(pa.x, pa.y, pa.z), v3(pb.x, pb.y, pb.z), radius,
                                                          dist, sinT, t1, t2);
                }
            });
            return acc;
        });
    }
    write_out(O, q, res, cnt, h, Q, K.P.norm_bb1d);
    if (O.tested) atomicAdd(O.tested, tested);
}

// Accepted candidates of one warp waiting for evaluation: the piece and its closest approach.
constexpr int kCandQueue = 64;
struct CandQueue {
    int piece[kCandQueue];
    float4 geo[kCandQueue];  // dist, sin(theta), t1 (query), t2 (beam)
    int near[kCandQueue];    // BB1D: pieces past the predicate's first check, waiting for the rest
};

// Per-warp scratch of the warp-cooperative gathers (shared memory).
struct WarpScratch {
    int* stack;
    int* leaves;
    CandQueue* cq;
    int lane;
    unsigned lt;  // lanes below this one
};

// BB1D of one query by one warp: the lanes test 32 beam pieces at a time; the accepted ones go to
// the warp's candidate queue, and whenever it holds 32 they are evaluated one per lane, so the
// contribution (transmittance, phase function, MIS weight) runs with every lane busy although
// only a fraction of the tested pieces is accepted.  Returns this lane's share of the result.
template <bool kMixed>
__device__ __forceinline__ Rgb bb1d_query_warp(const GatherConsts& K, const DMedium* media, const LightSoA& Lv,
                                               const BeamBVH& B, const BeamSoA& Bs, const SegQueriesDev& Q,
                                               int64_t q, SegCtx& s, V3 inv, const WarpScratch& ws,
                                               unsigned long long& cnt, unsigned long long& h,
                                               unsigned long long& tested, int* status)
{
    const int lane = ws.lane;
    const unsigned lt = ws.lt;
    CandQueue& cq = *ws.cq;
    const int leaf_shift = __ffs(B.leaf) - 1;
    unsigned cnt32 = 0, tested32 = 0;  // per query: below 2^32
    const Rgb res = segment_loop(K, media, Q, q, s, [&](const DMedium& m) {
        Rgb part = rgb(0.f);
        const int mid = (int)(&m - media);
        int qn = 0;  // entries in the candidate queue (warp-uniform)
        // evaluates queue entry e (one lane, one accepted candidate)
        auto eval = [&](int e) {
            const int i = cq.piece[e];
            const float4 g = cq.geo[e];
            const float4 pa = __ldg(&B.pa[i]);
            const float4 pb = __ldg(&B.pb[i]);
            const float4 pc = __ldg(&B.pc[i]);
            ++cnt32;
            h += mix64((unsigned long long)__float_as_int(pc.z));
            const int beam = __float_as_int(pc.z);
            if (kMixed) {
                const PiecePayload py = B.pay[i];
                part = part + bb1d_contrib_packed(K, m, s, py, v3(pa.x, pa.y, pa.z), v3(pb.x, pb.y, pb.z), g.x, g.y,
                                                  g.z, g.w, beam_radius_at(Bs, beam, py.lv.z, g.w));
            } else {
                part = part + bb1d_contrib<false>(K, m, Lv, Bs, s, beam, v3(pa.x, pa.y, pa.z), v3(pb.x, pb.y, pb.z),
                                                  beam_radius_at(Bs, beam, beam_start_radius(Bs, &Bs.radius[beam]), g.w), g.x, g.y,
                                                  g.z, g.w);
            }
        };
        // the rest of the predicate for one piece per lane (i < 0: none) that passed its first
        // check, with the ownership decision (in FP64 where the FP32 values cannot take it) and, in
        // mixed mode, the FP64 closest approach of near-parallel pairs; both run here rather than
        // in the evaluation, where the payload and the MIS inputs keep many more registers live.
        // Accepted candidates go to the candidate queue.
        auto full = [&](int i) {
            bool hit = false;
            float dist = 0.f, sinT = 0.f, t1 = 0.f, t2 = 0.f, bb = 0.f, ee = 0.f;
            if (i >= 0) {
                // the predicate reads only pa and pb; pc (piece interval, beam, medium) is loaded for
                // the pieces that pass it
                const float4 pa = __ldg(&B.pa[i]);
                const float4 pb = __ldg(&B.pb[i]);
                if (test_beam_beam(s.o, s.d, s.dmin, s.dmax, v3(pa.x, pa.y, pa.z), v3(pb.x, pb.y, pb.z), 0.f, pa.w,
                                   pb.w, &dist, &sinT, &t1, &t2, &bb, &ee)) {
                    const float4 pc = __ldg(&B.pc[i]);
                    if (__float_as_int(pc.w) == mid) {  // mMedium == medium (PhotonBeam.hxx:390)
                        // the radius test (PhotonBeam.hxx:411-413), then the reach rule and the owner
                        const int beam = __float_as_int(pc.z);
                        const float rs = beam_start_radius(Bs, kMixed ? &B.pay[i].lv.z : &Bs.radius[beam]);
                        const float rc = Bs.rchange ? __ldg(&Bs.rchange[beam]) : 0.f;
                        const float radius = beam_radius_at(Bs, beam, rs, t2);
                        hit = !(radius < dist);
                        if (hit) {
                            const int own = piece_takes_fast(s.o, s.d, s.dmin, s.dmax, v3(pa.x, pa.y, pa.z), pa.w,
                                                             pc.x, pc.y, t1, bb, ee, dist, rs, rc, K.bb1d_extra);
                            // the FP32 values cannot decide: the FP64 closest points of the segments
                            hit = own >= 0 ? own == 1
                                           : piece_takes_f64(s.o, s.d, s.dmin, s.dmax, v3(pa.x, pa.y, pa.z),
                                                             v3(pb.x, pb.y, pb.z), pa.w, pc.x, pc.y, rs, rc,
                                                             K.bb1d_extra);
                        }
                        if (kMixed && hit) {
                            // near-parallel lines, 1 - (d1.d2)^2 small: the FP32 solve of
                            // PhotonBeam.hxx:253-293 cancels, so the contribution gets the FP64
                            // closest approach (the candidate decision above stays FP32)
                            const float c = s.d.x * pb.x + s.d.y * pb.y + s.d.z * pb.z;
                            if (1.f - c * c < 1e-2f)
                                closest_approach_f64(s.o, s.d, v3(pa.x, pa.y, pa.z), v3(pb.x, pb.y, pb.z), dist,
                                                     sinT, t1, t2);
                        }
                    }
                }
            }
            const unsigned vote = __ballot_sync(kFull, hit);
            if (vote == 0u) return;
            if (hit) {
                const int pos = qn + __popc(vote & lt);
                cq.piece[pos] = i;
                cq.geo[pos] = make_float4(dist, sinT, t1, t2);
            }
            qn += __popc(vote);
            __syncwarp();
            if (qn >= 32) {  // the newest 32 entries, one per lane
                eval(qn - 32 + lane);
                qn -= 32;
                __syncwarp();
            }
        };
        // about a third of the tested pieces pass the predicate's first check (the distance of the
        // lines); they are queued and the rest of the predicate runs 32 at a time
        int pn = 0;  // entries in the near queue (warp-uniform)
        const bool ok = warp_traverse(B.nodes, B.n_leaves, B.n, leaf_shift, s.o, inv, s.dmin - K.eps, s.dmax + K.eps,
                                      ws.stack, ws.leaves, lane, [&](int i) {
            bool near = false;
            if (i >= 0) {
                const float4 pa = __ldg(&B.pa[i]);
                const float4 pb = __ldg(&B.pb[i]);
                ++tested32;
                near = beam_beam_near(s.o, s.d, v3(pa.x, pa.y, pa.z), v3(pb.x, pb.y, pb.z), pb.w);
            }
            const unsigned vote = __ballot_sync(kFull, near);
            if (vote == 0u) return;
            if (near) cq.near[pn + __popc(vote & lt)] = i;
            pn += __popc(vote);
            __syncwarp();
            if (pn >= 32) {
                full(cq.near[pn - 32 + lane]);
                pn -= 32;
                __syncwarp();
            }
        });
        if (pn > 0) {
            full(lane < pn ? cq.near[lane] : -1);
            __syncwarp();
        }
        if (lane < qn) eval(lane);
        __syncwarp();
        if (!ok && lane == 0) atomicOr(status, 1);
        return part;
    });
    cnt += cnt32;
    tested += tested32;
    return res;
}

// PB2D of one query by one warp over the photon LBVH, with the same candidate queue.
template <bool kMixed>
__device__ __forceinline__ Rgb pb2d_query_warp(const GatherConsts& K, const DMedium* media, const LightSoA& Lv,
                                               const PhotonBVH& P, const SegQueriesDev& Q, int64_t q, SegCtx& s,
                                               V3 inv, const WarpScratch& ws, unsigned long long& cnt,
                                               unsigned long long& h, unsigned long long& tested, int* status)
{
    const int lane = ws.lane;
    const unsigned lt = ws.lt;
    CandQueue& cq = *ws.cq;
    const int leaf_shift = __ffs(P.leaf) - 1;
    const float r2 = K.P.radius_pb2d * K.P.radius_pb2d;
    return segment_loop(K, media, Q, q, s, [&](const DMedium& m) {
        Rgb part = rgb(0.f);
        int qn = 0;
        auto eval = [&](int e) {
            const float4 g = cq.geo[e];
            part = part + pb2d_contrib<kMixed>(K, m, Lv, s, cq.piece[e], g.x, g.y, g.z);
        };
        const bool ok = warp_traverse(P.nodes, P.n_leaves, P.n, leaf_shift, s.o, inv, s.dmin - K.eps, s.dmax + K.eps,
                                      ws.stack, ws.leaves, lane, [&](int i) {
            bool hit = false;
            float t = 0.f, d2 = 0.f, r2i = r2;
            int lv = 0;
            if (i >= 0) {
                const float4 p = __ldg(&P.pos[i]);
                ++tested;
                if (P.r2) r2i = __ldg(&P.r2[i]);
                if (test_bre(s.o, s.d, s.dmin, s.dmax, v3(p.x, p.y, p.z), r2i, &t, &d2)) {
                    lv = __float_as_int(p.w);
                    hit = true;
                    ++cnt;
                    h += mix64((unsigned long long)lv);
                }
            }
            const unsigned vote = __ballot_sync(kFull, hit);
            if (vote == 0u) return;
            if (hit) {
                const int pos = qn + __popc(vote & lt);
                cq.piece[pos] = lv;
                cq.geo[pos] = make_float4(t, d2, r2i, 0.f);
            }
            qn += __popc(vote);
            __syncwarp();
            if (qn >= 32) {
                eval(qn - 32 + lane);
                qn -= 32;
                __syncwarp();
            }
        });
        if (lane < qn) eval(lane);
        __syncwarp();
        if (!ok && lane == 0) atomicOr(status, 1);
        return part;
    });
}

// BB1D, warp per query, persistent: warps draw query indices (in Morton order of the query
// midpoints) from an atomic counter.
template <bool kMixed, int kWarps, int kMinBlocks>
__global__ void __launch_bounds__(kWarps * 32, kMinBlocks) k_bb1d_warp(const __grid_constant__ GatherConsts K, const LightSoA Lv,
                                                          const BeamBVH B, const BeamSoA Bs, const SegQueriesDev Q,
                                                          const upbp_mis* __restrict__ cam,
                                                          const CamSum* __restrict__ cs, const Outputs O,
                                                          unsigned int* __restrict__ work, int* __restrict__ status,
                                                          const int32_t* __restrict__ order)
{
    __shared__ DMedium media[UPBP_MAX_MEDIA];
    __shared__ int s_stack[kWarps][kWarpStack];
    __shared__ int s_leaves[kWarps][kWarpLeaves];
    __shared__ CandQueue s_queue[kWarps];
    __shared__ upbp_mis s_e[kWarps];
    __shared__ CamSum s_cs[kWarps];
    stage_media(K, media);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const WarpScratch ws{s_stack[warp], s_leaves[warp], &s_queue[warp], lane, (1u << lane) - 1u};
    for (;;) {
        unsigned qq = 0;
        if (lane == 0) qq = atomicAdd(work, 1u);
        const int64_t item = (int64_t)__shfl_sync(kFull, qq, 0);
        if (item >= Q.n) break;
        const int64_t q = order ? (int64_t)__ldg(&order[item]) : item;
        Rgb acc = rgb(0.f);
        unsigned long long cnt = 0, h = 0, tested = 0;
        if ((Q.flags[q] & UPBP_Q_BB1D) && (K.P.techniques & UPBP_BB1D) && B.n > 0) {
            SegCtx s;
            init_seg_ctx<kMixed>(s, K, Q, cam, cs, q, &s_e[warp], &s_cs[warp], lane == 0);
            __syncwarp();
            const V3 inv = v3(safe_inv(s.d.x), safe_inv(s.d.y), safe_inv(s.d.z));
            acc = bb1d_query_warp<kMixed>(K, media, Lv, B, Bs, Q, q, s, inv, ws, cnt, h, tested, status);
        }
        const float r = warp_sum(acc.r), g = warp_sum(acc.g), b = warp_sum(acc.b);
        cnt = warp_sum_u64(cnt);
        h = warp_sum_u64(h);
        tested = warp_sum_u64(tested);
        if (lane == 0) {
            O.rgb[3 * q + 0] = r;
            O.rgb[3 * q + 1] = g;
            O.rgb[3 * q + 2] = b;
            if (O.count) O.count[q] = (uint32_t)cnt;
            if (O.hash) O.hash[q] = h;
            const Rgb thr{Q.throughput[3 * q], Q.throughput[3 * q + 1], Q.throughput[3 * q + 2]};
            splat(O.image, Q.pixel[q], thr * K.P.norm_bb1d * Rgb{r, g, b});
            if (O.tested) atomicAdd(O.tested, tested);
        }
    }
}

// PB2D, warp per query, persistent (the BB1D kernel's scheme over the photon LBVH): the lanes
// test 32 photons at a time and evaluate the accepted ones 32 at a time from the candidate queue.
template <bool kMixed, int kWarps, int kMinBlocks>
__global__ void __launch_bounds__(kWarps * 32, kMinBlocks) k_pb2d_warp(const __grid_constant__ GatherConsts K,
                                                                     const LightSoA Lv, const PhotonBVH P,
                                                                     const SegQueriesDev Q,
                                                                     const upbp_mis* __restrict__ cam,
                                                                     const CamSum* __restrict__ cs, const Outputs O,
                                                                     unsigned int* __restrict__ work,
                                                                     int* __restrict__ status,
                                                                     const int32_t* __restrict__ order)
{
    __shared__ DMedium media[UPBP_MAX_MEDIA];
    __shared__ int s_stack[kWarps][kWarpStack];
    __shared__ int s_leaves[kWarps][kWarpLeaves];
    __shared__ CandQueue s_queue[kWarps];
    __shared__ upbp_mis s_e[kWarps];
    __shared__ CamSum s_cs[kWarps];
    stage_media(K, media);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const WarpScratch ws{s_stack[warp], s_leaves[warp], &s_queue[warp], lane, (1u << lane) - 1u};
    for (;;) {
        unsigned qq = 0;
        if (lane == 0) qq = atomicAdd(work, 1u);
        const int64_t item = (int64_t)__shfl_sync(kFull, qq, 0);
        if (item >= Q.n) break;
        const int64_t q = order ? (int64_t)__ldg(&order[item]) : item;
        Rgb acc = rgb(0.f);
        unsigned long long cnt = 0, h = 0, tested = 0;
        if ((Q.flags[q] & UPBP_Q_PB2D) && (K.P.techniques & UPBP_PB2D) && P.n > 0) {
            SegCtx s;
            init_seg_ctx<kMixed>(s, K, Q, cam, cs, q, &s_e[warp], &s_cs[warp], lane == 0);
            __syncwarp();
            const V3 inv = v3(safe_inv(s.d.x), safe_inv(s.d.y), safe_inv(s.d.z));
            acc = pb2d_query_warp<kMixed>(K, media, Lv, P, Q, q, s, inv, ws, cnt, h, tested, status);
        }
        const float r = warp_sum(acc.r), g = warp_sum(acc.g), b = warp_sum(acc.b);
        cnt = warp_sum_u64(cnt);
        h = warp_sum_u64(h);
        tested = warp_sum_u64(tested);
        if (lane == 0) {
            O.rgb[3 * q + 0] = r;
            O.rgb[3 * q + 1] = g;
            O.rgb[3 * q + 2] = b;
            if (O.count) O.count[q] = (uint32_t)cnt;
            if (O.hash) O.hash[q] = h;
            const Rgb thr{Q.throughput[3 * q], Q.throughput[3 * q + 1], Q.throughput[3 * q + 2]};
            splat(O.image, Q.pixel[q], thr * K.P.norm_pb2d * Rgb{r, g, b});
            if (O.tested) atomicAdd(O.tested, tested);
        }
    }
}

// All camera segments of an iteration in one persistent work-queue kernel: a warp takes the next
// query (Morton order) and evaluates both segment estimators for it, PB2D over the photon LBVH
// and BB1D over the beam-piece LBVH, with one camera context and one splat per query.
template <bool kMixed, int kWarps, int kMinBlocks>
__global__ void __launch_bounds__(kWarps * 32, kMinBlocks) k_segments_warp(
    const __grid_constant__ GatherConsts K, const LightSoA Lv, const PhotonBVH P, const BeamBVH B, const BeamSoA Bs,
    const SegQueriesDev Q, const upbp_mis* __restrict__ cam, const CamSum* __restrict__ cs, const Outputs Opb,
    const Outputs Obb, unsigned int* __restrict__ work, int* __restrict__ status, const int32_t* __restrict__ order)
{
    __shared__ DMedium media[UPBP_MAX_MEDIA];
    __shared__ int s_stack[kWarps][kWarpStack];
    __shared__ int s_leaves[kWarps][kWarpLeaves];
    __shared__ CandQueue s_queue[kWarps];
    __shared__ upbp_mis s_e[kWarps];
    __shared__ CamSum s_cs[kWarps];
    stage_media(K, media);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const WarpScratch ws{s_stack[warp], s_leaves[warp], &s_queue[warp], lane, (1u << lane) - 1u};
    for (;;) {
        unsigned qq = 0;
        if (lane == 0) qq = atomicAdd(work, 1u);
        const int64_t item = (int64_t)__shfl_sync(kFull, qq, 0);
        if (item >= Q.n) break;
        const int64_t q = order ? (int64_t)__ldg(&order[item]) : item;
        const uint32_t qf = Q.flags[q];
        const bool do_pb = (qf & UPBP_Q_PB2D) && (K.P.techniques & UPBP_PB2D) && P.n > 0;
        const bool do_bb = (qf & UPBP_Q_BB1D) && (K.P.techniques & UPBP_BB1D) && B.n > 0;
        Rgb apb = rgb(0.f), abb = rgb(0.f);
        unsigned long long cpb = 0, hpb = 0, tpb = 0, cbb = 0, hbb = 0, tbb = 0;
        if (do_pb || do_bb) {
            SegCtx s;
            init_seg_ctx<kMixed>(s, K, Q, cam, cs, q, &s_e[warp], &s_cs[warp], lane == 0);
            __syncwarp();
            const V3 inv = v3(safe_inv(s.d.x), safe_inv(s.d.y), safe_inv(s.d.z));
            if (do_pb) apb = pb2d_query_warp<kMixed>(K, media, Lv, P, Q, q, s, inv, ws, cpb, hpb, tpb, status);
            if (do_bb) abb = bb1d_query_warp<kMixed>(K, media, Lv, B, Bs, Q, q, s, inv, ws, cbb, hbb, tbb, status);
        }
        const Rgb vpb{warp_sum(apb.r), warp_sum(apb.g), warp_sum(apb.b)};
        const Rgb vbb{warp_sum(abb.r), warp_sum(abb.g), warp_sum(abb.b)};
        cpb = warp_sum_u64(cpb);
        hpb = warp_sum_u64(hpb);
        tpb = warp_sum_u64(tpb);
        cbb = warp_sum_u64(cbb);
        hbb = warp_sum_u64(hbb);
        tbb = warp_sum_u64(tbb);
        if (lane == 0) {
            Opb.rgb[3 * q + 0] = vpb.r;
            Opb.rgb[3 * q + 1] = vpb.g;
            Opb.rgb[3 * q + 2] = vpb.b;
            Obb.rgb[3 * q + 0] = vbb.r;
            Obb.rgb[3 * q + 1] = vbb.g;
            Obb.rgb[3 * q + 2] = vbb.b;
            if (Opb.count) Opb.count[q] = (uint32_t)cpb;
            if (Opb.hash) Opb.hash[q] = hpb;
            if (Obb.count) Obb.count[q] = (uint32_t)cbb;
            if (Obb.hash) Obb.hash[q] = hbb;
            const Rgb thr{Q.throughput[3 * q], Q.throughput[3 * q + 1], Q.throughput[3 * q + 2]};
            splat(Obb.image, Q.pixel[q], thr * (vpb * K.P.norm_pb2d + vbb * K.P.norm_bb1d));
            if (Opb.tested) atomicAdd(Opb.tested, tpb);
            if (Obb.tested) atomicAdd(Obb.tested, tbb);
        }
    }
}

template <bool kMixed>
__global__ void __launch_bounds__(256) k_gather_pp3d(const __grid_constant__ GatherConsts K, const LightSoA Lv,
                                                     const HashGridDev G, const PointQueriesDev Q,
                                                     const upbp_mis* __restrict__ cam, const CamSum* __restrict__ cs,
                                                     const Outputs O)
{
    __shared__ DMedium media[UPBP_MAX_MEDIA];
    stage_media(K, media);
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= Q.n) return;
    const upbp_params& P = K.P;
    uint32_t cnt = 0;
    unsigned long long h = 0, tested = 0;
    Rgb res = rgb(0.f);
    const V3 qp = v3(Q.position[3 * q], Q.position[3 * q + 1], Q.position[3 * q + 2]);
    bool inside = (P.techniques & UPBP_PP3D) && G.n > 0;
    V3 dmin{0.f, 0.f, 0.f};
    if (inside) {
        dmin = xsub3(qp, v3(G.bbox_min[0], G.bbox_min[1], G.bbox_min[2]));
        const V3 dmax = xsub3(v3(G.bbox_max[0], G.bbox_max[1], G.bbox_max[2]), qp);
        inside = !(dmin.x < 0.f || dmin.y < 0.f || dmin.z < 0.f || dmax.x < 0.f || dmax.y < 0.f || dmax.z < 0.f);
    }
    if (inside) {
        const DMedium& m = media[Q.medium_id[q]];
        const V3 cfix = v3(Q.dir_fix[3 * q], Q.dir_fix[3 * q + 1], Q.dir_fix[3 * q + 2]);
        const int L = Q.path_length[q];
        const CamSnap camv{cam + Q.cam_mis_begin[q]};
        upbp_mis eL, eL1;
        CamSum csq;
        if (kMixed) {
            eL = load_mis(camv.snap + L);
            if (L >= 2) eL1 = load_mis(camv.snap + L - 1);
            csq = cs[q];
        }
        const bool scat_pos = !(m.ss[0] <= 0.f && m.ss[1] <= 0.f && m.ss[2] <= 0.f);
        const V3 cell = v3(xmul(G.inv_cell, dmin.x), xmul(G.inv_cell, dmin.y), xmul(G.inv_cell, dmin.z));
        const V3 cf = v3(floorf(cell.x), floorf(cell.y), floorf(cell.z));
        const int px = (int)cf.x, py = (int)cf.y, pz = (int)cf.z;
        const int pxo = px + (xsub(cell.x, cf.x) < 0.5f ? -1 : 1);
        const int pyo = py + (xsub(cell.y, cf.y) < 0.5f ? -1 : 1);
        const int pzo = pz + (xsub(cell.z, cf.z) < 0.5f ? -1 : 1);
        for (int j = 0; j < 8; ++j) {
            const int cx = (j & 4) ? pxo : px, cy = (j & 2) ? pyo : py, cz = (j & 1) ? pzo : pz;
            const uint32_t c = hash_cell(cx, cy, cz, G.cells);
            const int e = __ldg(&G.end[c]);
            for (int i = __ldg(&G.start[c]); i < e; ++i) {
                const float4 p = __ldg(&G.pos[i]);
                ++tested;
                const V3 dd = xsub3(qp, v3(p.x, p.y, p.z));
                if (!(xdot3(dd, dd) <= G.r2)) continue;
                const int lv = __float_as_int(p.w);
                ++cnt;
                h += mix64((unsigned long long)lv);
                // UPBP::RangeQuery::Process (UPBP.hxx:86-133)
                const int4 info = __ldg(&Lv.info[lv]);
                if (!(info.z & UPBP_LV_CONNECTABLE)) continue;
                const int pl = info.y;
                if ((uint32_t)(pl + L) > P.max_path_length || (uint32_t)(pl + L) < P.min_path_length) continue;
                if (!scat_pos) continue;
                const float4 ld = __ldg(&Lv.dir[lv]);
                float sinT;
                const float phase = hg_pdf(cfix, v3(ld.x, ld.y, ld.z), m.g, &sinT);
                const Rgb factor = Rgb{m.ss[0], m.ss[1], m.ss[2]} * phase;
                if (rgb_black_or_neg(factor)) continue;
                const float dirPdf = phase * m.cont;
                const float revPdf = phase * __ldg(&Lv.pos[lv]).w;
                const upbp_mis lvm = load_mis(Lv.mis + lv);
                const float mwfInv = 1.0f / lvm.pp3d_factor;
                float wCamera, wLight;
                if (kMixed) {
                    wCamera = camera_weight_fast(L, eL, mwfInv, sinT, lvm.ray_sample_pdf_inv,
                                                 lvm.ray_sample_pdfs_ratio, revPdf, eL1, eL1.ray_sample_rev_pdf_inv,
                                                 csq, P.techniques, P.query_beam_type, P.photon_beam_type);
                    const LightSum ls = Lv.sums[lv];
                    wLight = mwfInv * ((float)ls.a + dirPdf * (float)ls.c);
                } else {
                    wCamera = camera_path_weight(L, mwfInv, sinT, lvm.ray_sample_pdf_inv, lvm.ray_sample_pdfs_ratio,
                                                 revPdf, P.query_beam_type, P.photon_beam_type, P.techniques, camv);
                    const LightView lview{Lv.mis, -1, 0.f};
                    wLight = light_path_weight(info.x, pl, mwfInv, 0.f, 0.f, 0.f, dirPdf, UPBP_PP3D,
                                               P.query_beam_type, P.photon_beam_type, P.techniques, Lv.path_ends,
                                               lview, nullptr);
                }
                const float w = 1.f / (wLight + wCamera);
                const float4 th = __ldg(&Lv.thr[lv]);
                res = res + w * (factor * Rgb{th.x, th.y, th.z});
            }
        }
    }
    O.rgb[3 * q + 0] = res.r;
    O.rgb[3 * q + 1] = res.g;
    O.rgb[3 * q + 2] = res.b;
    if (O.count) O.count[q] = cnt;
    if (O.hash) O.hash[q] = h;
    const Rgb thr{Q.throughput[3 * q], Q.throughput[3 * q + 1], Q.throughput[3 * q + 2]};
    splat(O.image, Q.pixel[q], thr * P.norm_pp3d * res);
    if (O.tested) atomicAdd(O.tested, tested);
}

// B-P2D (extension; the reference has no beam x point estimator): photon beams queried at the
// camera medium vertices with a 2-D kernel, MIS weight 1.  Candidate: testIntersectionBre with
// the beam as the ray and the query point as the photon; the piece containing the foot point
// takes it.  Value: beam throughput x transmittance to the foot point (divided by the free-flight
// pdf for SHORT beams) x sigma_s x HG phase x (1 - d^2/r^2) / (pi r^2 / 2).
// B-P2D contribution of one accepted (point, beam) pair: beam throughput x transmittance to the
// foot point t (divided by the free-flight pdf for SHORT beams) x sigma_s x HG x the 2-D kernel.
__device__ __forceinline__ Rgb bp2d_contrib(const DMedium& m, const BeamSoA& Bs, int beam, V3 cfix, V3 bdir, float t,
                                            float d2, float r2)
{
    const float4 bthr = __ldg(&Bs.thr[beam]);
    Rgb att = eval_att(m, t);
    const float pfd = comp(att, m.min_idx);
    if ((uint32_t)__float_as_int(bthr.w) & UPBP_SHORT_BEAM) att = att / pfd;
    if (!rgb_positive(att)) return rgb(0.f);
    float sinT;
    const float phase = hg_pdf(cfix, neg3(bdir), m.g, &sinT);
    if (phase <= 0.f) return rgb(0.f);
    const float kernel = (1.f - d2 / r2) / (r2 * UPBP_PI_F * 0.5f);
    if (!is_pos(kernel)) return rgb(0.f);
    const Rgb ss{m.ss[0], m.ss[1], m.ss[2]};
    return Rgb{bthr.x, bthr.y, bthr.z} * att * ss * (phase * kernel);
}

// B-P2D, warp per point query, persistent: the lanes test 32 beam pieces at a time (the zero-length
// ray at the point makes the slab test a point-in-box test); accepted pairs go to the candidate
// queue and are evaluated 32 at a time.
template <int kWarps, int kMinBlocks>
__global__ void __launch_bounds__(kWarps * 32, kMinBlocks) k_bp2d_warp(const __grid_constant__ GatherConsts K,
                                                                     const BeamBVH B, const BeamSoA Bs,
                                                                     const PointQueriesDev Q, const Outputs O,
                                                                     unsigned int* __restrict__ work,
                                                                     int* __restrict__ status)
{
    __shared__ DMedium media[UPBP_MAX_MEDIA];
    __shared__ int s_stack[kWarps][kWarpStack];
    __shared__ int s_leaves[kWarps][kWarpLeaves];
    __shared__ CandQueue s_queue[kWarps];
    stage_media(K, media);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    int* stack = s_stack[warp];
    int* leaves = s_leaves[warp];
    CandQueue& cq = s_queue[warp];
    const int leaf_shift = __ffs(B.leaf) - 1;
    for (;;) {
        unsigned qq = 0;
        if (lane == 0) qq = atomicAdd(work, 1u);
        const int64_t q = (int64_t)__shfl_sync(kFull, qq, 0);
        if (q >= Q.n) break;
        Rgb part = rgb(0.f);
        unsigned long long cnt = 0, h = 0, tested = 0;
        const int mid = Q.medium_id[q];
        const DMedium& m = media[mid];
        if ((K.P.techniques & UPBP_BP2D) && m.has_scat && B.n > 0) {
            const V3 x = v3(Q.position[3 * q], Q.position[3 * q + 1], Q.position[3 * q + 2]);
            const V3 cfix = v3(Q.dir_fix[3 * q], Q.dir_fix[3 * q + 1], Q.dir_fix[3 * q + 2]);
            int qn = 0;
            auto eval = [&](int e) {
                const int i = cq.piece[e];
                const float4 g = cq.geo[e];  // t, d^2, r^2, -
                const float4 pb = __ldg(&B.pb[i]);
                const float4 pc = __ldg(&B.pc[i]);
                part = part + bp2d_contrib(m, Bs, __float_as_int(pc.z), cfix, v3(pb.x, pb.y, pb.z), g.x, g.y, g.z);
            };
            const bool ok = warp_traverse(B.nodes, B.n_leaves, B.n, leaf_shift, x, v3(1.f, 1.f, 1.f), 0.f, 0.f, stack,
                                          leaves, lane, [&](int i) {
                bool hit = false;
                float t = 0.f, d2 = 0.f, r2 = 0.f;
                if (i >= 0) {
                    const float4 pc = __ldg(&B.pc[i]);
                    if (__float_as_int(pc.w) == mid) {
                        const float4 pa = __ldg(&B.pa[i]);
                        const float4 pb = __ldg(&B.pb[i]);
                        ++tested;
                        // bound: the beam's largest radius^2; then the radius at the foot point
                        if (test_bre(v3(pa.x, pa.y, pa.z), v3(pb.x, pb.y, pb.z), 0.f, pa.w, x, pb.w, &t, &d2) &&
                            t >= pc.x && t < pc.y) {  // the piece containing the foot point
                            const int beam = __float_as_int(pc.z);
                            const float rt = beam_radius_at(Bs, beam, beam_start_radius(Bs, &Bs.radius[beam]), t);
                            r2 = rt * rt;
                            if (!(Bs.rchange && d2 > r2)) {
                                hit = true;
                                ++cnt;
                                h += mix64((unsigned long long)beam);
                            }
                        }
                    }
                }
                const unsigned vote = __ballot_sync(kFull, hit);
                if (vote == 0u) return;
                if (hit) {
                    const int pos = qn + __popc(vote & lt);
                    cq.piece[pos] = i;
                    cq.geo[pos] = make_float4(t, d2, r2, 0.f);
                }
                qn += __popc(vote);
                __syncwarp();
                if (qn >= 32) {
                    eval(qn - 32 + lane);
                    qn -= 32;
                    __syncwarp();
                }
            });
            if (lane < qn) eval(lane);
            __syncwarp();
            if (!ok && lane == 0) atomicOr(status, 1);
        }
        const float r = warp_sum(part.r), g = warp_sum(part.g), b = warp_sum(part.b);
        cnt = warp_sum_u64(cnt);
        h = warp_sum_u64(h);
        tested = warp_sum_u64(tested);
        if (lane == 0) {
            O.rgb[3 * q + 0] = r;
            O.rgb[3 * q + 1] = g;
            O.rgb[3 * q + 2] = b;
            if (O.count) O.count[q] = (uint32_t)cnt;
            if (O.hash) O.hash[q] = h;
            const Rgb thr{Q.throughput[3 * q], Q.throughput[3 * q + 1], Q.throughput[3 * q + 2]};
            splat(O.image, Q.pixel[q], thr * K.P.norm_bb1d * Rgb{r, g, b});
            if (O.tested) atomicAdd(O.tested, tested);
        }
    }
}

__global__ void __launch_bounds__(256) k_gather_bp2d(const __grid_constant__ GatherConsts K, const BeamBVH B,
                                                     const BeamSoA Bs, const PointQueriesDev Q, const Outputs O)
{
    __shared__ DMedium media[UPBP_MAX_MEDIA];
    stage_media(K, media);
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= Q.n) return;
    uint32_t cnt = 0;
    unsigned long long h = 0, tested = 0;
    Rgb res = rgb(0.f);
    const V3 x = v3(Q.position[3 * q], Q.position[3 * q + 1], Q.position[3 * q + 2]);
    const int mid = Q.medium_id[q];
    const DMedium& m = media[mid];
    if ((K.P.techniques & UPBP_BP2D) && m.has_scat && B.n > 0) {
        const V3 cfix = v3(Q.dir_fix[3 * q], Q.dir_fix[3 * q + 1], Q.dir_fix[3 * q + 2]);
        // a zero-length ray at x: the slab test becomes point-in-box
        traverse(B.nodes, B.n_leaves, x, v3(1.f, 1.f, 1.f), 0.f, 0.f, [&](int leaf) {
            const int e = min(B.n, (leaf + 1) * B.leaf);
            for (int i = leaf * B.leaf; i < e; ++i) {
                const float4 pc = __ldg(&B.pc[i]);
                if (__float_as_int(pc.w) != mid) continue;
                const float4 pa = __ldg(&B.pa[i]);
                const float4 pb = __ldg(&B.pb[i]);
                ++tested;
                float t, d2;
                // bound: the beam's largest radius^2; then the radius at the foot point
                if (!test_bre(v3(pa.x, pa.y, pa.z), v3(pb.x, pb.y, pb.z), 0.f, pa.w, x, pb.w, &t, &d2)) continue;
                if (!(t >= pc.x && t < pc.y)) continue;  // the piece containing the foot point
                const int beam = __float_as_int(pc.z);
                const float rt = beam_radius_at(Bs, beam, beam_start_radius(Bs, &Bs.radius[beam]), t), r2 = rt * rt;
                if (Bs.rchange && d2 > r2) continue;
                ++cnt;
                h += mix64((unsigned long long)beam);
                res = res + bp2d_contrib(m, Bs, beam, cfix, v3(pb.x, pb.y, pb.z), t, d2, r2);
            }
        });
    }
    O.rgb[3 * q + 0] = res.r;
    O.rgb[3 * q + 1] = res.g;
    O.rgb[3 * q + 2] = res.b;
    if (O.count) O.count[q] = cnt;
    if (O.hash) O.hash[q] = h;
    const Rgb thr{Q.throughput[3 * q], Q.throughput[3 * q + 1], Q.throughput[3 * q + 2]};
    splat(O.image, Q.pixel[q], thr * K.P.norm_bb1d * res);
    if (O.tested) atomicAdd(O.tested, tested);
}

// ----------------------------------------------------------------- BB1D over the beam grid
// SSE min_ps / max_ps: the second operand unless the first compares below / above it
__device__ __forceinline__ float sse_min(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float sse_max(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float pick3(int k, float a, float b, float c) { return k == 0 ? a : (k == 1 ? b : c); }

// Grid::intersect (Grid.hxx:322-398): the DDA walk of one segment [mint, maxt] of the query ray
// through the reference's grid, with the reference's float operations (the box test of
// BoundingBox3::intersect, Structs/BoundingBox.hxx:218-272, with its SSE operand order, which
// turns the NaN of a zero direction component into an unbounded slab).  visit(cell, cell_mint,
// cell_maxt) for every visited cell, in order; the walk leaves the grid after at most
// res0 + res1 + res2 cells.
template <class Visit>
__device__ __forceinline__ void grid_walk(const GridHeader& h, V3 o, V3 d, float mint, float maxt, Visit&& visit)
{
    const float ix = __fdiv_rn(1.f, d.x), iy = __fdiv_rn(1.f, d.y), iz = __fdiv_rn(1.f, d.z);
    float lmax = 0.f, lmin = 0.f;
    for (int k = 0; k < 3; ++k) {
        const float ok = pick3(k, o.x, o.y, o.z), ik = pick3(k, ix, iy, iz);
        const float l1 = __fmul_rn(__fsub_rn(h.lo[k], ok), ik);
        const float l2 = __fmul_rn(__fsub_rn(h.hi[k], ok), ik);
        const float mx = sse_max(sse_min(l1, INFINITY), sse_min(l2, INFINITY));
        const float mn = sse_min(sse_max(l1, -INFINITY), sse_max(l2, -INFINITY));
        lmax = k == 0 ? mx : sse_min(lmax, mx);
        lmin = k == 0 ? mn : sse_max(lmin, mn);
    }
    if (!(lmax >= lmin)) return;
    const float tmn = lmin < mint ? mint : lmin;
    const float tmx = lmax > maxt ? maxt : lmax;
    if (!(tmx > tmn)) return;
    float dx = __fmul_rn(h.cell[0], ix), dy = __fmul_rn(h.cell[1], iy), dz = __fmul_rn(h.cell[2], iz);
    const float ex = __fmul_rn(__fsub_rn(__fadd_rn(o.x, __fmul_rn(d.x, tmn)), h.lo[0]), h.inv_cell[0]);
    const float ey = __fmul_rn(__fsub_rn(__fadd_rn(o.y, __fmul_rn(d.y, tmn)), h.lo[1]), h.inv_cell[1]);
    const float ez = __fmul_rn(__fsub_rn(__fadd_rn(o.z, __fmul_rn(d.z, tmn)), h.lo[2]), h.inv_cell[2]);
    // Grid::posToVoxel: Utils::clamp((int)pos, 0, res - 1)
    int px = max(0, min((int)ex, h.res[0] - 1));
    int py = max(0, min((int)ey, h.res[1] - 1));
    int pz = max(0, min((int)ez, h.res[2] - 1));
    uint32_t cell = (uint32_t)px + (uint32_t)h.res[0] * ((uint32_t)py + (uint32_t)h.res[1] * (uint32_t)pz);
    int sx = 1, sy = 1, sz = 1, cx = h.res[0], cy = h.res[1], cz = h.res[2];
    if (!(d.x >= 0.f)) { sx = -1; cx = -1; dx = -dx; }
    if (!(d.y >= 0.f)) { sy = -1; cy = -1; dy = -dy; }
    if (!(d.z >= 0.f)) { sz = -1; cz = -1; dz = -dz; }
    float lx = __fmul_rn(__fmul_rn(__fsub_rn((float)(px + (sx > 0 ? 1 : 0)), ex), ix), h.cell[0]);
    float ly = __fmul_rn(__fmul_rn(__fsub_rn((float)(py + (sy > 0 ? 1 : 0)), ey), iy), h.cell[1]);
    float lz = __fmul_rn(__fmul_rn(__fsub_rn((float)(pz + (sz > 0 ? 1 : 0)), ez), iz), h.cell[2]);
    float t = tmn;
    const int steps = h.res[0] + h.res[1] + h.res[2] + 3;
    for (int it = 0; it < steps; ++it) {
        // Vector3::argMin (Structs/Vector3.hxx:473-475)
        const int ax = (lx < ly) ? ((lx < lz) ? 0 : 2) : ((ly < lz) ? 1 : 2);
        const float la = pick3(ax, lx, ly, lz);
        const float tn = __fadd_rn(t, la);
        visit(cell, t, tmx < tn ? tmx : tn);  // std::min(t + l[minAxis], _maxt)
        t = tn;
        lx = __fsub_rn(lx, la);
        ly = __fsub_rn(ly, la);
        lz = __fsub_rn(lz, la);
        if (ax == 0) {
            lx = dx;
            cell += h.shift[0] * (uint32_t)sx;
            px += sx;
            if (px == cx) return;
        } else if (ax == 1) {
            ly = dy;
            cell += h.shift[1] * (uint32_t)sy;
            py += sy;
            if (py == cy) return;
        } else {
            lz = dz;
            cell += h.shift[2] * (uint32_t)sz;
            pz += sz;
            if (pz == cz) return;
        }
        if (!(t < tmx)) return;
    }
}

// The cells of one warp's walk waiting for their beams to be tested, and the (cell, entry) items
// past the first check of the predicate waiting for the rest of it.
constexpr int kGridQueue = 32, kGridNear = 64;
struct GridQueue {
    float tmin[kGridQueue], tmax[kGridQueue], pdf[kGridQueue];
    uint32_t begin[kGridQueue], beams[kGridQueue];
    unsigned long long key[kGridQueue];  // the cell's draws (reductions 1-3)
    uint32_t first[kGridQueue + 1];      // the first item of every queued cell; first[n] = all items
    float ntmin[kGridNear], ntmax[kGridNear], npdf[kGridNear];
    uint32_t nat[kGridNear];             // the item's entry in the cell lists
};

// The per-query draws of the OFFSET, RESAMPLE_FIXED and SAMPLED reductions (Grid.hxx:466-548).  The
// reference takes them from the grid's one sequential stream in the order the queries are made;
// here each is a function of (seed, query, segment, cell, draw), the same uniform distribution
// whatever the order of evaluation: a SplitMix64 finaliser, 24 bits to [0, 1).
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ float grid_draw(unsigned long long key, uint32_t j)
{
    return (float)(splitmix64(key + (unsigned long long)j * 0xD1B54A32D192ED03ull) >> 40) * 0x1p-24f;
}

// BB1D of one query by one warp over the beam grid.  The walk runs on every lane alike and queues
// the visited cells that hold beams (max_beams_in_cell items of an over-full cell of a reduced
// grid, Grid.hxx:453-548); once 32 or more (cell, beam) items wait, the lanes take them 32 at a
// time through the first checks of PhotonBeam::testIntersectionBeamBeam (the distance of the two
// lines, then the closest point's t1 within the cell's t range), from the entries' packed geometry.
// The items that pass them go to a second queue, whose 32-wide batches run the rest: the medium,
// the whole predicate, the radius, and PhotonBeam::accumulate / accumulate2 (PhotonBeam.hxx:315-367,
// 375-480) divided by the cell's selection pdf.
template <bool kMixed>
__device__ __forceinline__ Rgb bb1d_query_grid(const GatherConsts& K, const DMedium* media, const LightSoA& Lv,
                                               const BeamGrid& G, const GridHeader& hdr, const BeamSoA& Bs,
                                               const SegQueriesDev& Q, int64_t q, SegCtx& s, GridQueue& gq,
                                               int lane, unsigned long long& cnt, unsigned long long& h,
                                               unsigned long long& tested)
{
    const unsigned lt = (1u << lane) - 1u;
    unsigned cnt32 = 0, tested32 = 0;
    const Rgb res = segment_loop(K, media, Q, q, s, [&](const DMedium& m) {
        Rgb part = rgb(0.f);
        const int mid = (int)(&m - media);
        int qc = 0, nq = 0;  // queued cells and items past the first check (warp-uniform)
        auto finish = [&](int k) {
            const uint32_t at = gq.nat[k];
            const int b = __ldg(&G.ptr[at]);
            if (__ldg(&G.medium[b]) != mid) return;  // mMedium == medium
            const float4 a = __ldg(&G.rec_a[at]), bd = __ldg(&G.rec_b[at]);
            const V3 o2 = v3(a.x, a.y, a.z), d2 = v3(bd.x, bd.y, bd.z);
            float dist, sinT, t1, t2;
            if (!test_beam_beam(s.o, s.d, gq.ntmin[k], gq.ntmax[k], o2, d2, 0.f, a.w, bd.w, &dist, &sinT, &t1, &t2))
                return;
            const float rs = beam_start_radius(Bs, kMixed ? &G.pay[b].lv.z : &Bs.radius[b]);
            const float radius = beam_radius_at(Bs, b, rs, t2);
            if (radius < dist) return;  // PhotonBeam.hxx:334-336 / 411-413
            ++cnt32;
            h += mix64((unsigned long long)b);
            Rgb c;
            if (kMixed) {
                // the beam's packed payload, and the FP64 closest approach of near-parallel lines
                // (the candidate decision above stays FP32)
                const float cb = s.d.x * d2.x + s.d.y * d2.y + s.d.z * d2.z;
                if (1.f - cb * cb < 1e-2f) closest_approach_f64(s.o, s.d, o2, d2, dist, sinT, t1, t2);
                c = bb1d_contrib_packed(K, m, s, G.pay[b], o2, d2, dist, sinT, t1, t2, beam_radius_at(Bs, b, rs, t2));
            } else {
                c = bb1d_contrib<false>(K, m, Lv, Bs, s, b, o2, d2, radius, dist, sinT, t1, t2);
            }
            const float pdf = gq.npdf[k];
            if (pdf != 1.f) c = c * __fdiv_rn(1.f, pdf);
            part = part + c;
        };
        // the queued cells' items; final: also the last items past the first check
        auto flush = [&](bool final) {
            const uint32_t total = qc > 0 ? gq.first[qc] : 0u;
            for (uint32_t base = 0; base < total || (final && nq > 0); base += 32) {
                const uint32_t it = base + (uint32_t)lane;
                bool near = false;
                int e = 0;
                uint32_t at = 0;
                if (it < total) {
                    while (e + 1 < qc && gq.first[e + 1] <= it) ++e;
                    const uint32_t j = it - gq.first[e], begin = gq.begin[e], beams = gq.beams[e];
                    // the entry of item j: intersectPresampled / intersectOffsetted / intersectFixedSampled /
                    // intersectSampled (Grid.hxx:453-548); unreduced cells and PRESAMPLE: the j-th of the list
                    at = begin + j;
                    bool take = true;
                    if (gq.pdf[e] != 1.f && hdr.reduction != 0) {
                        if (hdr.reduction == 1) {
                            const uint32_t off = (uint32_t)__fmul_rn(grid_draw(gq.key[e], 0), (float)beams);
                            const uint32_t k = min(hdr.max_beams, beams - min(off, beams));
                            at = j < k ? begin + off + j : begin + (j - k);
                        } else if (hdr.reduction == 2) {
                            at = begin + min((uint32_t)__fmul_rn(grid_draw(gq.key[e], j), (float)beams), beams - 1);
                        } else {
                            take = grid_draw(gq.key[e], j) < gq.pdf[e];
                        }
                    }
                    if (take) {
                        ++tested32;
                        const float4 a = __ldg(&G.rec_a[at]), bd = __ldg(&G.rec_b[at]);
                        const V3 o2 = v3(a.x, a.y, a.z), d2 = v3(bd.x, bd.y, bd.z);
                        if (beam_beam_near(s.o, s.d, o2, d2, bd.w)) {
                            // a beam near the query's line is listed in every cell it crosses along the
                            // walk; only the cell holding the lines' closest point accepts it
                            float b12, b1o1, b1o2, be, t1;
                            near = beam_beam_t1(s.o, s.d, o2, d2, b12, b1o1, b1o2, be, t1) &&
                                   !(t1 <= gq.tmin[e] || t1 >= gq.tmax[e]);
                        }
                    }
                }
                const unsigned bal = __ballot_sync(kFull, near);
                if (near) {
                    const int slot = nq + __popc(bal & lt);
                    gq.ntmin[slot] = gq.tmin[e];
                    gq.ntmax[slot] = gq.tmax[e];
                    gq.npdf[slot] = gq.pdf[e];
                    gq.nat[slot] = at;
                }
                nq += __popc(bal);
                __syncwarp();
                if (nq >= 32 || (final && base + 32 >= total && nq > 0)) {
                    const int n = min(nq, 32);
                    nq -= n;
                    if (lane < n) finish(nq + lane);
                    __syncwarp();
                }
            }
            qc = 0;
            __syncwarp();
        };
        // the reductions' draws of this query and segment
        const unsigned long long qkey =
            splitmix64(((unsigned long long)(uint32_t)hdr.seed << 32) ^ (unsigned long long)q) ^
            ((unsigned long long)__float_as_uint(s.dmin) * 0x94D049BB133111EBull);
        grid_walk(hdr, s.o, s.d, s.dmin, s.dmax, [&](uint32_t cell, float cmin, float cmax) {
            const uint32_t begin = __ldg(&G.cells[cell]);
            const uint32_t beams = __ldg(&G.cells[cell + 1]) - begin;
            const float pdf = G.pdf ? __ldg(&G.pdf[cell]) : 1.f;
            // a reduced cell tests max_beams beams, SAMPLED draws for each of them
            const uint32_t n = (pdf != 1.f && hdr.reduction != 3) ? hdr.max_beams : beams;
            if (n == 0) return;
            if (lane == 0) {
                if (qc == 0) gq.first[0] = 0;
                gq.tmin[qc] = cmin;
                gq.tmax[qc] = cmax;
                gq.pdf[qc] = pdf;
                gq.begin[qc] = begin;
                gq.beams[qc] = beams;
                gq.key[qc] = splitmix64(qkey + (unsigned long long)cell * 0x9E3779B97F4A7C15ull);
                gq.first[qc + 1] = gq.first[qc] + n;
            }
            __syncwarp();
            ++qc;
            if (qc == kGridQueue || gq.first[qc] >= 32) flush(false);
        });
        if (qc > 0 || nq > 0) flush(true);
        return part;
    });
    cnt += cnt32;
    tested += tested32;
    return res;
}

// Persistent, one warp per query from the atomic work queue.  Compiled for 7 blocks of 4 warps per
// SM (72 registers): the walk and the first checks stream the cell entries and wait on their loads,
// so resident warps matter more than the spills of the rare contribution path.
template <bool kMixed>
__global__ void __launch_bounds__(128, 7) k_bb1d_grid(const __grid_constant__ GatherConsts K, const LightSoA Lv,
                                                  const BeamGrid G, const BeamSoA Bs, const SegQueriesDev Q,
                                                  const upbp_mis* __restrict__ cam, const CamSum* __restrict__ cs,
                                                  const Outputs O, unsigned int* __restrict__ work,
                                                  const int32_t* __restrict__ order)
{
    constexpr int kWarps = 4;
    __shared__ DMedium media[UPBP_MAX_MEDIA];
    __shared__ GridHeader s_hdr;
    __shared__ GridQueue s_q[kWarps];
    __shared__ upbp_mis s_e[kWarps];
    __shared__ CamSum s_cs[kWarps];
    if (threadIdx.x == 0) s_hdr = *G.hdr;
    stage_media(K, media);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (;;) {
        unsigned qq = 0;
        if (lane == 0) qq = atomicAdd(work, 1u);
        const int64_t item = (int64_t)__shfl_sync(kFull, qq, 0);
        if (item >= Q.n) break;
        const int64_t q = order ? (int64_t)__ldg(&order[item]) : item;
        Rgb acc = rgb(0.f);
        unsigned long long cnt = 0, h = 0, tested = 0;
        if ((Q.flags[q] & UPBP_Q_BB1D) && (K.P.techniques & UPBP_BB1D)) {
            SegCtx s;
            init_seg_ctx<kMixed>(s, K, Q, cam, cs, q, &s_e[warp], &s_cs[warp], lane == 0);
            __syncwarp();
            acc = bb1d_query_grid<kMixed>(K, media, Lv, G, s_hdr, Bs, Q, q, s, s_q[warp], lane, cnt, h, tested);
        }
        const float r = warp_sum(acc.r), g = warp_sum(acc.g), b = warp_sum(acc.b);
        cnt = warp_sum_u64(cnt);
        h = warp_sum_u64(h);
        tested = warp_sum_u64(tested);
        if (lane == 0) {
            if (O.tested && tested) atomicAdd(O.tested, tested);
            O.rgb[3 * q + 0] = r;
            O.rgb[3 * q + 1] = g;
            O.rgb[3 * q + 2] = b;
            if (O.count) O.count[q] = (uint32_t)cnt;
            if (O.hash) O.hash[q] = h;
            const Rgb thr{Q.throughput[3 * q], Q.throughput[3 * q + 1], Q.throughput[3 * q + 2]};
            splat(O.image, Q.pixel[q], thr * K.P.norm_bb1d * Rgb{r, g, b});
        }
    }
}

}  // namespace

int bb1d_grid_blocks_per_sm(bool mixed)
{
    int nb = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_bb1d_grid<true>, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_bb1d_grid<false>, 128, 0);
    return nb > 0 ? nb : 1;
}

void launch_bb1d_grid(const GatherConsts& K, const LightSoA& L, const BeamGrid& G, const BeamSoA& S,
                      const SegQueriesDev& Q, const upbp_mis* cam, const CamSum* cs, const Outputs& O, int grid,
                      bool mixed, unsigned int* work, const int32_t* order, cudaStream_t stream)
{
    if (Q.n <= 0) return;
    if (mixed) k_bb1d_grid<true><<<grid, 128, 0, stream>>>(K, L, G, S, Q, cam, cs, O, work, order);
    else k_bb1d_grid<false><<<grid, 128, 0, stream>>>(K, L, G, S, Q, cam, cs, O, work, order);
}

void launch_gather_bp2d(const GatherConsts& K, const BeamBVH& B, const BeamSoA& S, const PointQueriesDev& Q,
                        const Outputs& O, int block, cudaStream_t stream)
{
    if (Q.n <= 0) return;
    const int grid = (int)((Q.n + block - 1) / block);
    k_gather_bp2d<<<grid, block, 0, stream>>>(K, B, S, Q, O);
}

int bp2d_warp_blocks_per_sm()
{
    int nb = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_bp2d_warp<4, 6>, 128, 0);
    return nb > 0 ? nb : 1;
}

void launch_bp2d_warp(const GatherConsts& K, const BeamBVH& B, const BeamSoA& S, const PointQueriesDev& Q,
                      const Outputs& O, int grid, unsigned int* work, int* status, cudaStream_t stream)
{
    if (Q.n > 0) k_bp2d_warp<4, 6><<<grid, 128, 0, stream>>>(K, B, S, Q, O, work, status);
}

void launch_gather_pb2d(const GatherConsts& K, const LightSoA& L, const PhotonBVH& B, const SegQueriesDev& Q,
                        const upbp_mis* cam, const CamSum* cs, const Outputs& O, int block, bool mixed,
                        cudaStream_t stream, const int32_t* order)
{
    if (Q.n <= 0) return;
    const int grid = (int)((Q.n + block - 1) / block);
    if (mixed) k_gather_pb2d<true><<<grid, block, 0, stream>>>(K, L, B, Q, cam, cs, O, order);
    else k_gather_pb2d<false><<<grid, block, 0, stream>>>(K, L, B, Q, cam, cs, O, order);
}

void launch_gather_bb1d(const GatherConsts& K, const LightSoA& L, const BeamBVH& B, const BeamSoA& S,
                        const SegQueriesDev& Q, const upbp_mis* cam, const CamSum* cs, const Outputs& O, int block,
                        bool mixed, cudaStream_t stream)
{
    if (Q.n <= 0) return;
    const int grid = (int)((Q.n + block - 1) / block);
    if (mixed) k_gather_bb1d<true><<<grid, block, 0, stream>>>(K, L, B, S, Q, cam, cs, O);
    else k_gather_bb1d<false><<<grid, block, 0, stream>>>(K, L, B, S, Q, cam, cs, O);
}

// The fused segment kernel at 5 (variant 3) or 6 (variant 4) blocks of 4 warps per SM.
int segments_warp_blocks_per_sm(bool mixed, int variant)
{
    int nb = 0;
    const bool six = variant == 4;
    if (mixed) {
        if (six) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_segments_warp<true, 4, 6>, 128, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_segments_warp<true, 4, 5>, 128, 0);
    } else {
        if (six) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_segments_warp<false, 4, 6>, 128, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_segments_warp<false, 4, 5>, 128, 0);
    }
    return nb > 0 ? nb : 1;
}

void launch_segments_warp(const GatherConsts& K, const LightSoA& L, const PhotonBVH& P, const BeamBVH& B,
                          const BeamSoA& S, const SegQueriesDev& Q, const upbp_mis* cam, const CamSum* cs,
                          const Outputs& Opb, const Outputs& Obb, int grid, bool mixed, unsigned int* work,
                          int* status, const int32_t* order, cudaStream_t stream, int variant)
{
    if (Q.n <= 0) return;
    const bool six = variant == 4;
#define UPBP_SEG_LAUNCH(M, N) \
    k_segments_warp<M, 4, N><<<grid, 128, 0, stream>>>(K, L, P, B, S, Q, cam, cs, Opb, Obb, work, status, order)
    if (mixed) {
        if (six) UPBP_SEG_LAUNCH(true, 6);
        else UPBP_SEG_LAUNCH(true, 5);
    } else {
        if (six) UPBP_SEG_LAUNCH(false, 6);
        else UPBP_SEG_LAUNCH(false, 5);
    }
#undef UPBP_SEG_LAUNCH
}

// Two instantiations of the warp kernel differ only in the occupancy the compiler is asked to
// reach: 5 blocks of 4 warps per SM (up to 96 registers) or 6 (up to 80 registers, more warps to
// hide load latency, some spills); the tuning's bb1d_kernel picks 1 or 2.
template <bool kMixed>
static int blocks_for(int variant)
{
    int nb = 0;
    if (variant == 2) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_bb1d_warp<kMixed, 4, 7>, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_bb1d_warp<kMixed, 4, 6>, 128, 0);
    return nb > 0 ? nb : 1;
}

int pb2d_warp_blocks_per_sm(bool mixed)
{
    int nb = 0;
    if (mixed) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_pb2d_warp<true, 4, 6>, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_pb2d_warp<false, 4, 6>, 128, 0);
    return nb > 0 ? nb : 1;
}

void launch_pb2d_warp(const GatherConsts& K, const LightSoA& L, const PhotonBVH& P, const SegQueriesDev& Q,
                      const upbp_mis* cam, const CamSum* cs, const Outputs& O, int grid, bool mixed,
                      unsigned int* work, int* status, const int32_t* order, cudaStream_t stream)
{
    if (Q.n <= 0) return;
    if (mixed) k_pb2d_warp<true, 4, 6><<<grid, 128, 0, stream>>>(K, L, P, Q, cam, cs, O, work, status, order);
    else k_pb2d_warp<false, 4, 6><<<grid, 128, 0, stream>>>(K, L, P, Q, cam, cs, O, work, status, order);
}

int bb1d_warp_blocks_per_sm(bool mixed, int variant)
{
    return mixed ? blocks_for<true>(variant) : blocks_for<false>(variant);
}

void launch_bb1d_warp(const GatherConsts& K, const LightSoA& L, const BeamBVH& B, const BeamSoA& S,
                      const SegQueriesDev& Q, const upbp_mis* cam, const CamSum* cs, const Outputs& O, int grid,
                      bool mixed, unsigned int* work, int* status, const int32_t* order, cudaStream_t stream,
                      int variant)
{
    if (Q.n <= 0) return;
    if (variant == 2) {
        if (mixed) k_bb1d_warp<true, 4, 7><<<grid, 128, 0, stream>>>(K, L, B, S, Q, cam, cs, O, work, status, order);
        else k_bb1d_warp<false, 4, 7><<<grid, 128, 0, stream>>>(K, L, B, S, Q, cam, cs, O, work, status, order);
    } else {
        if (mixed) k_bb1d_warp<true, 4, 6><<<grid, 128, 0, stream>>>(K, L, B, S, Q, cam, cs, O, work, status, order);
        else k_bb1d_warp<false, 4, 6><<<grid, 128, 0, stream>>>(K, L, B, S, Q, cam, cs, O, work, status, order);
    }
}

namespace {
__global__ void k_piece_payload(const float4* __restrict__ pc, int n, const float4* __restrict__ bm_thr,
                                const float4* __restrict__ bm_pdf, const int2* __restrict__ bm_link,
                                const float* __restrict__ bm_radius, const int4* __restrict__ lv_info,
                                const upbp_mis* __restrict__ lv_mis, const LightSum* __restrict__ sums,
                                PiecePayload* __restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int beam = pc ? __float_as_int(pc[i].z) : i;  // pc == NULL: one payload per beam
    const int lv = bm_link[beam].x;
    // without MIS (lv_info == nullptr) the beams need not have light vertices
    upbp_mis m{};
    int4 info = make_int4(0, 0, 0, 0);
    LightSum ls{};
    if (lv_info) {
        m = load_mis(lv_mis + lv);
        info = lv_info[lv];
        ls = sums[lv];
    }
    const bool onDelta = (m.flags & UPBP_MIS_ON_LIGHT_SOURCE) && (m.flags & UPBP_MIS_IS_DELTA);
    const float4 thr = bm_thr[beam], pdf = bm_pdf[beam];
    const uint32_t bflags = (uint32_t)__float_as_int(thr.w), brsf = (uint32_t)__float_as_int(pdf.w);
    PiecePayload p;
    p.thr = make_float4(thr.x, thr.y, thr.z, (float)ls.d);
    p.pdf = make_float4(pdf.x, pdf.y, pdf.z, (float)ls.e);
    const unsigned bits = (unsigned)(info.y & kPayPathMask) | ((info.z & UPBP_LV_IS_FINITE) ? (unsigned)kPayFinite : 0u) |
                          ((bflags & UPBP_SHORT_BEAM) ? (unsigned)kPayShortBeam : 0u) |
                          ((brsf & UPBP_ORIGIN_IN_MEDIUM) ? kPayOriginInMedium : 0u);
    p.lv = make_float4(onDelta ? 0.f : fabsf(m.cos_theta_out), ls.bptb, bm_radius[beam], __int_as_float((int)bits));
    out[i] = p;
}

// Morton code of the middle of a segment query's span (10 bits per axis in the given box).
// Spreads the low 10 bits of v to every third bit (3-D Morton interleave).
__device__ __forceinline__ uint32_t spread3(uint32_t v)
{
    uint32_t r = 0;
    for (int b = 0; b < 10; ++b) r |= ((v >> b) & 1u) << (3 * b);
    return r;
}
// Spreads the low 14 bits of v to every second bit (2-D Morton interleave).
__device__ __forceinline__ uint32_t spread2(uint32_t v)
{
    uint32_t r = 0;
    for (int b = 0; b < 14; ++b) r |= ((v >> b) & 1u) << (2 * b);
    return r;
}

// Sort key of a segment query (30 bits), by `mode` (upbp_tuning.query_order):
//  0: 3-D Morton code of the midpoint of the query's span;
//  1: camera rays (path length 1) first, along a 2-D Morton curve of their pixels (neighbouring
//     pixels' rays cross nearly the same beam pieces), then the other segments by midpoint;
//  2: 5-D Morton code of the midpoint (6 bits per axis) and the direction (octahedral map, 6 bits
//     per axis).
__global__ void k_query_keys(const SegQueriesDev Q, const float* __restrict__ bb, int mode, int width, uint32_t* keys,
                             int32_t* iota)
{
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= Q.n) return;
    const int sb = Q.seg_begin[q], sc = Q.seg_count[q];
    const float t = sc > 0 ? 0.5f * (Q.seg_dist_min[sb] + Q.seg_dist_max[sb + sc - 1]) : 0.f;
    const float tm = isfinite(t) ? t : (sc > 0 ? Q.seg_dist_min[sb] : 0.f);
    float p[3];
    for (int c = 0; c < 3; ++c) p[c] = Q.origin[3 * q + c] + Q.direction[3 * q + c] * tm;
    uint32_t ix[3];
    for (int c = 0; c < 3; ++c) {
        const float ext = bb[3 + c] - bb[c];
        const float u = ext > 0.f ? (p[c] - bb[c]) / ext : 0.f;
        ix[c] = (uint32_t)fminf(fmaxf(u * 1024.f, 0.f), 1023.f);
    }
    uint32_t code = (spread3(ix[0]) << 2) | (spread3(ix[1]) << 1) | spread3(ix[2]);
    if (mode == 1) {
        const int px = Q.pixel[q];
        if (Q.path_length[q] == 1 && px >= 0 && width > 0)
            code = spread2((uint32_t)(px % width) & 0x3fffu) | (spread2((uint32_t)(px / width) & 0x3fffu) << 1);
        else
            code = (1u << 29) | (code >> 1);
    } else if (mode == 2) {
        // octahedral map of the direction to [0, 1)^2
        const float dx = Q.direction[3 * q], dy = Q.direction[3 * q + 1], dz = Q.direction[3 * q + 2];
        const float n = fabsf(dx) + fabsf(dy) + fabsf(dz);
        float ox = n > 0.f ? dx / n : 0.f, oy = n > 0.f ? dy / n : 0.f;
        if (dz < 0.f) {
            const float tx = (1.f - fabsf(oy)) * (ox >= 0.f ? 1.f : -1.f);
            oy = (1.f - fabsf(ox)) * (oy >= 0.f ? 1.f : -1.f);
            ox = tx;
        }
        const uint32_t a[5] = {ix[0] >> 4, ix[1] >> 4, ix[2] >> 4,
                               (uint32_t)fminf(fmaxf((ox * 0.5f + 0.5f) * 64.f, 0.f), 63.f),
                               (uint32_t)fminf(fmaxf((oy * 0.5f + 0.5f) * 64.f, 0.f), 63.f)};
        code = 0;
        for (int b = 5; b >= 0; --b)
            for (int k = 0; k < 5; ++k) code = (code << 1) | ((a[k] >> b) & 1u);
    }
    keys[q] = code;
    iota[q] = (int32_t)q;
}
// Sum of the per-query PB2D candidate counts (integer, so the order of the atomics does not matter).
__global__ void k_sum_counts(const uint32_t* __restrict__ cnt, int64_t n, unsigned long long* sum)
{
    unsigned long long v = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        v += cnt[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(sum, v);
}

// BB1D work order: the queries whose PB2D candidate count exceeds `factor` times the mean come
// first (they are the heaviest BB1D queries too), each group in Morton order of the midpoints.
__global__ void k_heavy_keys(const uint32_t* __restrict__ cnt, int64_t n, const unsigned long long* __restrict__ sum,
                             unsigned factor, const uint32_t* __restrict__ morton, uint32_t* keys, int32_t* iota)
{
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= n) return;
    const bool heavy = (unsigned long long)cnt[q] * (unsigned long long)n > (unsigned long long)factor * *sum;
    keys[q] = (heavy ? 0u : (1u << 30)) | morton[q];
    iota[q] = (int32_t)q;
}
}  // namespace

void launch_heavy_keys(const uint32_t* cnt, int64_t n, unsigned long long* sum, unsigned factor,
                       const uint32_t* morton, uint32_t* keys, int32_t* iota, cudaStream_t stream)
{
    if (n <= 0) return;
    k_sum_counts<<<148 * 4, 256, 0, stream>>>(cnt, n, sum);
    k_heavy_keys<<<(int)((n + 255) / 256), 256, 0, stream>>>(cnt, n, sum, factor, morton, keys, iota);
}

void launch_piece_payload(const float4* pc, int n, const float4* bm_thr, const float4* bm_pdf, const int2* bm_link,
                          const float* bm_radius, const int4* lv_info, const upbp_mis* lv_mis, const LightSum* sums,
                          PiecePayload* out, cudaStream_t stream)
{
    if (n > 0)
        k_piece_payload<<<(n + 255) / 256, 256, 0, stream>>>(pc, n, bm_thr, bm_pdf, bm_link, bm_radius, lv_info, lv_mis,
                                                             sums, out);
}

void launch_query_keys(const SegQueriesDev& Q, const float* bbox, int mode, int image_width, uint32_t* keys,
                       int32_t* iota, cudaStream_t stream)
{
    if (Q.n > 0) k_query_keys<<<(int)((Q.n + 255) / 256), 256, 0, stream>>>(Q, bbox, mode, image_width, keys, iota);
}

void launch_gather_pp3d(const GatherConsts& K, const LightSoA& L, const HashGridDev& G, const PointQueriesDev& Q,
                        const upbp_mis* cam, const CamSum* cs, const Outputs& O, int block, bool mixed,
                        cudaStream_t stream)
{
    if (Q.n <= 0) return;
    const int grid = (int)((Q.n + block - 1) / block);
    if (mixed) k_gather_pp3d<true><<<grid, block, 0, stream>>>(K, L, G, Q, cam, cs, O);
    else k_gather_pp3d<false><<<grid, block, 0, stream>>>(K, L, G, Q, cam, cs, O);
}

}  // namespace upbp
