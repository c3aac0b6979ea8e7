// Generic-precision gathers: the FP64 evaluation mode and the adjoint (dL/d medium parameters).
//
// Candidate enumeration is the one of the FP32 kernels (same traversals, same FP32 predicates,
// so the same candidate sets); the contributions are the scalar-generic versions of
// breIntersectFuncHomogeneous2 (Bre/Bre.cxx:293-464), PhotonBeam::accumulate2
// (Beams/PhotonBeam.hxx:386-607) and UPBP::RangeQuery::Process (Renderers/UPBP.hxx:86-133) with
// the O(1) MIS weights of the FP64 partial sums (upbp_mis_prep.cuh).  With T = double every
// result is an FP64 oracle computed on the GPU; with T = DualF every candidate also carries the
// derivatives (FP32 tangents) of its contribution with respect to one medium's sigma_a, sigma_s
// and g, and the kernels accumulate sum_pixels dL/dI . dI/dtheta in FP64 -- the adjoint of the
// estimator sum.
#include <cfloat>
#include <cstdint>

#include "upbp_generic.cuh"
#include "upbp_generic_api.cuh"
#include "upbp_kernels.cuh"
#include "upbp_mis_prep.cuh"
#include "upbp_traverse.cuh"

namespace upbp {
namespace gen {
namespace {

template <class T>
struct SegCtx {
    V3 of, df;       // query ray in FP32 (predicates)
    V3d o, d;        // the same in FP64 (contribution geometry)
    double dmin, dmax;
    T rs_pdf, rs_rev_pdf;
    uint32_t rsf;
    int L;
    double lpw;
    uint32_t ray_flags;
    const upbp_mis* e;  // camera entry L-1 (L >= 2)
    const CamSum* cs;
};

template <class T>
__device__ __forceinline__ void stage_media_t(const GenConsts& G, MedT<T>* s)
{
    for (int i = threadIdx.x; i < G.n_media; i += blockDim.x) s[i] = make_med<T>(G.raw[i], i == G.grad_medium);
    __syncthreads();
}

// evalBre / evalBeamBeamEstimate segment loop (Bre.cxx:812-964, PhBeams.cxx:177-324) in T.
template <class T, class PerSeg>
__device__ __forceinline__ RgbT<T> seg_loop(const GatherConsts& K, const MedT<T>* media, const SegQueriesDev& Q,
                                            int64_t q, SegCtx<T>& s, PerSeg&& per)
{
    const uint32_t qf = Q.flags[q];
    const bool lite = (qf & UPBP_Q_LITE) != 0;
    const uint32_t qrsf = (qf & UPBP_Q_ORIGIN_IN_MEDIUM) ? UPBP_ORIGIN_IN_MEDIUM : 0u;
    const uint32_t bt = K.P.query_beam_type;
    RgbT<T> result = rgb_zero<T>(), attn = rgbt<T>(cst<T>(1.0));
    T rsp = cst<T>(1.0), rsr = cst<T>(1.0);
    const int sb = Q.seg_begin[q], sc = Q.seg_count[q];
    for (int i = 0; i < sc; ++i) {
        const int sg = sb + i;
        const int mid = Q.seg_medium[sg];
        const MedT<T>& m = media[mid];
        const float dminf = Q.seg_dist_min[sg], dmaxf = Q.seg_dist_max[sg];
        const double dmin = dminf, dmax = dmaxf;
        if (m.has_scat) {
            s.dmin = dmin;
            s.dmax = dmax;
            s.rs_pdf = rsp;
            s.rs_rev_pdf = rsr;
            s.rsf = UPBP_END_IN_MEDIUM | (i == 0 ? qrsf : 0u);
            result = result + attn * per(m, mid, dminf, dmaxf);
        }
        if (lite) {
            attn = attn * eval_att(m, dmax - dmin);
            T srev;
            const T spdf = ray_sample_pdf(m, dmin, dmax, i == 0 ? qrsf : 0u, &srev);
            if (!positive(attn)) break;
            rsp = rsp * spdf;
            rsr = rsr * srev;
        } else {
            const double pdf = Q.seg_pdf[sg];
            RgbT<T> sa = RgbT<T>{cst<T>(Q.seg_attenuation[3 * sg]), cst<T>(Q.seg_attenuation[3 * sg + 1]),
                                 cst<T>(Q.seg_attenuation[3 * sg + 2])};
            if (bt == UPBP_SHORT_BEAM) sa = sa / pdf;
            attn = attn * sa;
            if (!positive(attn)) break;
            rsp = rsp * pdf;
            rsr = rsr * (double)Q.seg_rev_pdf[sg];
        }
    }
    return result;
}

template <class T>
__device__ __forceinline__ void init_ctx(SegCtx<T>& s, const GatherConsts& K, const SegQueriesDev& Q,
                                         const upbp_mis* cam, const CamSum* cs, int64_t q)
{
    s.of = v3(Q.origin[3 * q], Q.origin[3 * q + 1], Q.origin[3 * q + 2]);
    s.df = v3(Q.direction[3 * q], Q.direction[3 * q + 1], Q.direction[3 * q + 2]);
    s.o = v3d(s.of);
    s.d = v3d(s.df);
    s.L = Q.path_length[q];
    s.lpw = Q.last_pdf_w_inv[q];
    s.ray_flags = K.P.query_beam_type | K.P.techniques;
    s.e = cam + Q.cam_mis_begin[q] + (s.L >= 1 ? s.L - 1 : 0);
    s.cs = cs + q;
}

// ------------------------------------------------------------------ PB2D (Bre.cxx:293-464)
// Without MIS (UPBP_NO_MIS): breIntersectFuncHomogeneous (Bre.cxx:239-291), every accepted photon's
// unweighted contribution, the candidate geometry re-solved in FP64.
template <class T>
__device__ RgbT<T> pb2d_contrib_nomis(const MedT<T>& m, const LightSoA& Lv, const SegCtx<T>& s, int lv, double r2)
{
    const float4 lp = __ldg(&Lv.pos[lv]);
    const V3d p = v3d(lp.x, lp.y, lp.z);
    const double t = dot(sub(p, s.o), s.d);
    const V3d qv = V3d{s.o.x + s.d.x * t - p.x, s.o.y + s.d.y * t - p.y, s.o.z + s.d.z * t - p.z};
    const double d2 = dot(qv, qv);
    RgbT<T> att = eval_att(m, t - s.dmin);
    if (s.ray_flags & UPBP_SHORT_BEAM) att = att / comp(att, m.min_idx);
    const float4 ld = __ldg(&Lv.dir[lv]);
    const float4 th = __ldg(&Lv.thr[lv]);
    double sinT;
    const T phase = hg_pdf(s.d, neg(v3d(ld.x, ld.y, ld.z)), m.g, &sinT);
    const double kernel = (1.0 - d2 / r2) / (r2 * 3.14159265358979323846 * 0.5);
    return RgbT<T>{att.r * (double)th.x, att.g * (double)th.y, att.b * (double)th.z} *
           RgbT<T>{m.ss[0], m.ss[1], m.ss[2]} * (phase * kernel);
}

template <class T>
__device__ RgbT<T> pb2d_contrib(const GatherConsts& K, const MedT<T>& m, const LightSoA& Lv, const SegCtx<T>& s,
                                int lv, float r2f)
{
    const upbp_params& P = K.P;
    if (P.techniques & UPBP_NO_MIS) return pb2d_contrib_nomis<T>(m, Lv, s, lv, (double)r2f);
    const int4 info = __ldg(&Lv.info[lv]);
    const int pl = info.y;
    if ((uint32_t)(pl + s.L) > P.max_path_length || (uint32_t)(pl + s.L) < P.min_path_length) return rgb_zero<T>();
    const float4 lp = __ldg(&Lv.pos[lv]);
    // the candidate geometry re-solved in FP64
    const V3d p = v3d(lp.x, lp.y, lp.z);
    const double t = dot(sub(p, s.o), s.d);
    const V3d qv = V3d{s.o.x + s.d.x * t - p.x, s.o.y + s.d.y * t - p.y, s.o.z + s.d.z * t - p.z};
    const double d2 = dot(qv, qv);
    if (s.L == 1 && t < P.min_dist_to_med) return rgb_zero<T>();
    RgbT<T> att = eval_att(m, t - s.dmin);
    const T pdf = comp(att, m.min_idx);
    if (s.ray_flags & UPBP_SHORT_BEAM) att = att / pdf;
    T rsp = m.min_st * pdf;
    T rsr = (s.rsf & UPBP_ORIGIN_IN_MEDIUM) ? rsp : pdf;
    const T ratio = 1.0 / m.min_st;
    if (!positive(att)) return rgb_zero<T>();
    rsp = rsp * s.rs_pdf;
    rsr = rsr * s.rs_rev_pdf;
    const float4 ld = __ldg(&Lv.dir[lv]);
    double sinT;
    const T phase = hg_pdf(neg(s.d), v3d(ld.x, ld.y, ld.z), m.g, &sinT);
    if (!(val(phase) > 0.0)) return rgb_zero<T>();
    const T camDirPdfW = phase * m.cont;
    const T camRevPdfW = phase * (double)lp.w;
    const double r2 = r2f;  // the photon's radiusSqr
    const double kernel = (1.0 - d2 / r2) / (r2 * 3.14159265358979323846 * 0.5);
    if (!(kernel > 1e-20)) return rgb_zero<T>();
    const float4 th = __ldg(&Lv.thr[lv]);
    const RgbT<T> unweighted =
        RgbT<T>{att.r * (double)th.x, att.g * (double)th.y, att.b * (double)th.z} * RgbT<T>{m.ss[0], m.ss[1], m.ss[2]} *
        (phase * kernel);
    if (black_or_neg(unweighted)) return rgb_zero<T>();
    const double distSq = t * t;
    const T rspInv = 1.0 / rsp;
    CandT<T> cand;
    cand.f = Factors{0.f, P.mis_factor_pp3d, P.mis_factor_pb2d, P.mis_factor_bb1d, K.has_bb1d_beams ? 1.f : 0.f,
                     (m.mfp > P.bb1d_min_mfp) ? UPBP_MIS_IN_MEDIUM_WITH_BEAMS : 0u};
    cand.pdf_a_inv = rspInv * (s.lpw * distSq);
    cand.rsp_inv = rspInv;
    cand.ratio = ratio;
    const T last = (s.ray_flags & UPBP_SHORT_BEAM) ? 1.0 / (ratio * (double)P.mis_factor_pb2d)
                                                   : rsp / (double)P.mis_factor_pb2d;
    const upbp_mis lvm = load_mis(Lv.mis + lv);
    const T wc = camera_weight(P, s.L, cand, last, sinT, cst<T>((double)lvm.ray_sample_pdf_inv),
                               cst<T>((double)lvm.ray_sample_pdfs_ratio), camRevPdfW * rsr / distSq, *s.e, 1.0 / rsr,
                               *s.cs, s.ray_flags);
    const LightSum ls = Lv.sums[lv];
    const T wl = last * (camDirPdfW * ls.c + ls.a);
    return unweighted / (wl + wc);
}

// ------------------------------------------------------------------ BB1D (PhotonBeam.hxx:386-607)
__device__ __forceinline__ void closest_f64(V3d O1, V3d d1, V3d O2, V3d d2, double& dist, double& sinT, double& t1,
                                            double& t2)
{
    const double wx = O1.x - O2.x, wy = O1.y - O2.y, wz = O1.z - O2.z;
    const double cx = d1.y * d2.z - d1.z * d2.y, cy = d1.z * d2.x - d1.x * d2.z, cz = d1.x * d2.y - d1.y * d2.x;
    const double aa = d1.x * d1.x + d1.y * d1.y + d1.z * d1.z;
    const double cc = d2.x * d2.x + d2.y * d2.y + d2.z * d2.z;
    const double b = d1.x * d2.x + d1.y * d2.y + d1.z * d2.z;
    const double dd = d1.x * wx + d1.y * wy + d1.z * wz;
    const double ee = d2.x * wx + d2.y * wy + d2.z * wz;
    const double den = aa * cc - b * b;
    const double s = sqrt(cx * cx + cy * cy + cz * cz);
    t1 = (b * ee - cc * dd) / den;
    t2 = (aa * ee - b * dd) / den;
    dist = fabs(wx * cx + wy * cy + wz * cz) / s;
    sinT = s;
}

// Without MIS (UPBP_NO_MIS): PhotonBeam::accumulate (PhotonBeam.hxx:315-367), the unweighted
// contribution in FP64.
template <class T>
__device__ RgbT<T> bb1d_contrib_nomis(const MedT<T>& m, const SegCtx<T>& s, const PiecePayload& py, V3d bo,
                                      V3d bdir, double rchange)
{
    double dist, sinTheta, t1, t2;
    closest_f64(s.o, s.d, bo, bdir, dist, sinTheta, t1, t2);
    const double radius = (double)py.lv.z + t2 * rchange;
    const unsigned lvbits = (unsigned)__float_as_int(py.lv.w);
    RgbT<T> att = eval_att(m, t1 - s.dmin);
    const RgbT<T> batt = eval_att(m, t2);
    if (s.ray_flags & UPBP_SHORT_BEAM) att = att / comp(att, m.min_idx);
    att = att * batt;
    if (lvbits & kPayShortBeam) att = att / comp(batt, m.min_idx);
    double sinDummy;
    const T phase = hg_pdf(s.d, bdir, m.g, &sinDummy);
    const double kern = (1.0 - dist * dist / (radius * radius)) * 3.0 / (4.0 * radius * sinTheta);
    return RgbT<T>{att.r * (double)py.thr.x, att.g * (double)py.thr.y, att.b * (double)py.thr.z} *
           RgbT<T>{m.ss[0], m.ss[1], m.ss[2]} * (phase * kern);
}

template <class T>
__device__ RgbT<T> bb1d_contrib(const GatherConsts& K, const MedT<T>& m, const SegCtx<T>& s, const PiecePayload& py,
                                const LightSum& ls, V3d bo, V3d bdir, double rchange)
{
    const upbp_params& P = K.P;
    if (P.techniques & UPBP_NO_MIS) return bb1d_contrib_nomis<T>(m, s, py, bo, bdir, rchange);
    const unsigned lvbits = (unsigned)__float_as_int(py.lv.w);
    const int pl = (int)(lvbits & kPayPathMask);
    const bool finite = (lvbits & kPayFinite) != 0;
    if ((uint32_t)(pl + 1 + s.L) > P.max_path_length || (uint32_t)(pl + 1 + s.L) < P.min_path_length)
        return rgb_zero<T>();
    double dist, sinTheta, t1, t2;
    closest_f64(s.o, s.d, bo, bdir, dist, sinTheta, t1, t2);
    if (s.L == 1 && t1 < P.min_dist_to_med) return rgb_zero<T>();
    const double radius = (double)py.lv.z + t2 * rchange;  // mStartRadius + t2 * mRadiusChange
    const uint32_t bflags = (lvbits & kPayShortBeam) ? UPBP_SHORT_BEAM : 0u;
    const uint32_t brsf = (lvbits & kPayOriginInMedium) ? UPBP_ORIGIN_IN_MEDIUM : 0u;
    RgbT<T> att = eval_att(m, t1 - s.dmin);
    const T pfdQ = comp(att, m.min_idx);
    if (s.ray_flags & UPBP_SHORT_BEAM) att = att / pfdQ;
    T rspQ = m.min_st * pfdQ;
    T rsrQ = (s.rsf & UPBP_ORIGIN_IN_MEDIUM) ? rspQ : pfdQ;
    const T ratio = 1.0 / m.min_st;
    const RgbT<T> batt = eval_att(m, t2);
    att = att * batt;
    const T pfdB = comp(batt, m.min_idx);
    if (bflags & UPBP_SHORT_BEAM) att = att / pfdB;
    T rspB = m.min_st * pfdB;
    T rsrB = (brsf & UPBP_ORIGIN_IN_MEDIUM) ? rspB : pfdB;
    if (!positive(att)) return rgb_zero<T>();
    rspQ = rspQ * s.rs_pdf;
    rsrQ = rsrQ * s.rs_rev_pdf;
    rspB = rspB * (double)py.pdf.x;
    rsrB = rsrB * (double)py.pdf.y;
    double sinDummy;
    const T phase = hg_pdf(neg(s.d), neg(bdir), m.g, &sinDummy);
    if (!(val(phase) > 0.0)) return rgb_zero<T>();
    const T pdfW = phase * m.cont;
    const double kern = (1.0 - dist * dist / (radius * radius)) * 3.0 / (4.0 * radius * sinTheta);
    const RgbT<T> unweighted = RgbT<T>{att.r * (double)py.thr.x, att.g * (double)py.thr.y, att.b * (double)py.thr.z} *
                               RgbT<T>{m.ss[0], m.ss[1], m.ss[2]} * (phase * kern);
    if (black_or_neg(unweighted)) return rgb_zero<T>();
    const double distSqQ = t1 * t1;
    const T rspInvQ = 1.0 / rspQ;
    CandT<T> cand;
    cand.f = Factors{0.f, P.mis_factor_pp3d, P.mis_factor_pb2d, P.mis_factor_bb1d, 1.f, UPBP_MIS_IN_MEDIUM_WITH_BEAMS};
    cand.pdf_a_inv = rspInvQ * (s.lpw * distSqQ);
    cand.rsp_inv = rspInvQ;
    cand.ratio = ratio;
    const double distSqB = finite ? t2 * t2 : 1.0;
    const T rspInvB = 1.0 / rspB;
    const T brecPdfAInv = rspInvB * ((double)py.pdf.z * distSqB);
    const double sinT = (s.ray_flags & UPBP_NO_SINE_IN_WEIGHTS) ? 1.0 : sinTheta;
    const double f = P.mis_factor_bb1d;
    T last;
    if (s.ray_flags & UPBP_SHORT_BEAM)
        last = (bflags & UPBP_SHORT_BEAM) ? 1.0 / (ratio * ratio * (f * sinT)) : rspB / (ratio * (f * sinT));
    else
        last = (bflags & UPBP_SHORT_BEAM) ? rspQ / (ratio * (f * sinT)) : rspQ * rspB / (f * sinT);
    const T wc = camera_weight(P, s.L, cand, last, sinT, rspInvB, ratio, pdfW * rsrQ / distSqQ, *s.e, 1.0 / rsrQ,
                               *s.cs, s.ray_flags);
    const T ntl = pdfW * rsrB * ((double)py.lv.x / distSqB);
    T inner = cst<T>((double)ls.bptb);
    if (!(s.ray_flags & UPBP_PREVIOUS)) inner = inner + ntl * (ls.e / rsrB + ls.d);
    const T wl = last * brecPdfAInv * inner;
    return unweighted / (wl + wc);
}

// ------------------------------------------------------------------ epilogues
// Per-query result of one lane (its share of the query's candidates): FP64 mode writes values,
// the adjoint contracts the tangents with the framebuffer gradient of the query's pixel.
template <class T>
__device__ __forceinline__ void lane_grad(const RgbT<T>& v, const double w[3], double g[kNT])
{
    if constexpr (is_dual<T>::value) {
#pragma unroll
        for (int i = 0; i < kNT; ++i) g[i] += w[0] * v.r.d[i] + w[1] * v.g.d[i] + w[2] * v.b.d[i];
    }
}

__device__ __forceinline__ double wsum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// weights dL/dI(pixel) * throughput * normalisation, per channel
__device__ __forceinline__ void pixel_weights(const GenOut& O, int px, const float* thr, double norm, double w[3])
{
    w[0] = w[1] = w[2] = 0.0;
    if (!O.grad_image || px < 0) return;
    for (int c = 0; c < 3; ++c) w[c] = (double)O.grad_image[3 * px + c] * (double)thr[c] * norm;
}

template <class T>
__device__ __forceinline__ void finish_thread(const GenOut& O, int64_t q, const RgbT<T>& v, int px, const float* thr,
                                              double norm, uint32_t cnt, unsigned long long h)
{
    if constexpr (is_dual<T>::value) {
        double w[3], g[kNT];
        pixel_weights(O, px, thr, norm, w);
        for (int i = 0; i < kNT; ++i) g[i] = 0.0;
        lane_grad(v, w, g);
        for (int i = 0; i < kNT; ++i)
            if (g[i] != 0.0) atomicAdd(&O.grad[i], g[i]);
    } else {
        if (O.rgb) {
            O.rgb[3 * q + 0] = (float)v.r;
            O.rgb[3 * q + 1] = (float)v.g;
            O.rgb[3 * q + 2] = (float)v.b;
        }
        if (O.count) O.count[q] = cnt;
        if (O.hash) O.hash[q] = h;
        if (O.image && px >= 0) {
            atomicAdd(&O.image[3 * px + 0], (float)(v.r * (double)thr[0] * norm));
            atomicAdd(&O.image[3 * px + 1], (float)(v.g * (double)thr[1] * norm));
            atomicAdd(&O.image[3 * px + 2], (float)(v.b * (double)thr[2] * norm));
        }
    }
}

// Thread-per-query epilogue: every lane of the warp calls it (valid = the lane has a query), so
// the adjoint can reduce over the warp before its atomics.
template <class T>
__device__ __forceinline__ void finish_lanes(const GenOut& O, bool valid, int64_t q, const RgbT<T>& v, int px,
                                             const float* thr, double norm, uint32_t cnt, unsigned long long h)
{
    if constexpr (is_dual<T>::value) {
        double w[3] = {0.0, 0.0, 0.0}, g[kNT];
        for (int i = 0; i < kNT; ++i) g[i] = 0.0;
        if (valid) {
            pixel_weights(O, px, thr, norm, w);
            lane_grad(v, w, g);
        }
        for (int i = 0; i < kNT; ++i) g[i] = wsum(g[i]);
        if ((threadIdx.x & 31) == 0)
            for (int i = 0; i < kNT; ++i)
                if (g[i] != 0.0) atomicAdd(&O.grad[i], g[i]);
    } else {
        if (valid) finish_thread<T>(O, q, v, px, thr, norm, cnt, h);
    }
}

// End of a warp's query (the warp kernels): the adjoint adds the lanes' gradient terms of this
// query's pixel weight; otherwise the lanes' partial results, counts and hashes are reduced and
// lane 0 writes the query's outputs.
template <class T>
__device__ __forceinline__ void finish_warp(const GenOut& O, int64_t q, const RgbT<T>& acc, int px, const float* thr,
                                            double norm, unsigned long long cnt, unsigned long long h, int lane)
{
    if constexpr (is_dual<T>::value) {
        double w[3], g[kNT];
        pixel_weights(O, px, thr, norm, w);
        for (int i = 0; i < kNT; ++i) g[i] = 0.0;
        lane_grad(acc, w, g);
        for (int i = 0; i < kNT; ++i) g[i] = wsum(g[i]);
        if (lane == 0)
            for (int i = 0; i < kNT; ++i)
                if (g[i] != 0.0) atomicAdd(&O.grad[i], g[i]);
    } else {
        RgbT<T> v{wsum(acc.r), wsum(acc.g), wsum(acc.b)};
        for (int o = 16; o > 0; o >>= 1) {
            cnt += __shfl_xor_sync(kFull, cnt, o);
            h += __shfl_xor_sync(kFull, h, o);
        }
        if (lane == 0) finish_thread<T>(O, q, v, px, thr, norm, (uint32_t)cnt, h);
    }
}

// ------------------------------------------------------------------ kernels
constexpr int kGenQueue = 64;

// PB2D, warp per query with a candidate queue (the scheme of the BB1D kernel below, over the
// photon LBVH): the lanes test 32 photons at a time and evaluate the accepted ones 32 at a time.
template <class T>
__device__ __forceinline__ void gen_pb2d_body(const GatherConsts& K, const GenConsts& G, const LightSoA Lv,
                                                  const PhotonBVH B, const SegQueriesDev Q,
                                                  const upbp_mis* __restrict__ cam, const CamSum* __restrict__ cs,
                                                  const GenOut O, unsigned int* __restrict__ work,
                                                  int* __restrict__ status, const int32_t* __restrict__ order)
{
    constexpr int kWarps = 4;
    __shared__ MedT<T> media[UPBP_MAX_MEDIA];
    __shared__ int s_stack[kWarps][kWarpStack];
    __shared__ int s_leaves[kWarps][kWarpLeaves];
    __shared__ int s_photon[kWarps][kGenQueue];
    stage_media_t<T>(G, media);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    int* stack = s_stack[warp];
    int* leaves = s_leaves[warp];
    int* cq = s_photon[warp];
    const int leaf_shift = __ffs(B.leaf) - 1;
    const float r2 = K.P.radius_pb2d * K.P.radius_pb2d;
    for (;;) {
        unsigned qq = 0;
        if (lane == 0) qq = atomicAdd(work, 1u);
        const int64_t item = (int64_t)__shfl_sync(kFull, qq, 0);
        if (item >= Q.n) break;
        const int64_t q = order ? (int64_t)__ldg(&order[item]) : item;
        RgbT<T> acc = rgb_zero<T>();
        unsigned long long cnt = 0, h = 0;
        if ((Q.flags[q] & UPBP_Q_PB2D) && (K.P.techniques & UPBP_PB2D) && B.n > 0) {
            SegCtx<T> s;
            init_ctx(s, K, Q, cam, cs, q);
            const V3 inv = v3(safe_inv(s.df.x), safe_inv(s.df.y), safe_inv(s.df.z));
            acc = seg_loop<T>(K, media, Q, q, s, [&](const MedT<T>& m, int, float dminf, float dmaxf) {
                RgbT<T> part = rgb_zero<T>();
                int qn = 0;
                auto eval = [&](int e) {
                    const int i = cq[e];
                    const float4 p = __ldg(&B.pos[i]);
                    const float r2i = B.r2 ? __ldg(&B.r2[i]) : r2;
                    part = part + pb2d_contrib<T>(K, m, Lv, s, __float_as_int(p.w), r2i);
                };
                const bool ok = warp_traverse(B.nodes, B.n_leaves, B.n, leaf_shift, s.of, inv, dminf - K.eps,
                                              dmaxf + K.eps, stack, leaves, lane, [&](int i) {
                    bool hit = false;
                    if (i >= 0) {
                        const float4 p = __ldg(&B.pos[i]);
                        const float r2i = B.r2 ? __ldg(&B.r2[i]) : r2;
                        float t, d2;
                        if (test_bre(s.of, s.df, dminf, dmaxf, v3(p.x, p.y, p.z), r2i, &t, &d2)) {
                            hit = true;
                            ++cnt;
                            h += mix64((unsigned long long)__float_as_int(p.w));
                        }
                    }
                    const unsigned vote = __ballot_sync(kFull, hit);
                    if (vote == 0u) return;
                    if (hit) cq[qn + __popc(vote & lt)] = i;
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
        finish_warp<T>(O, q, acc, Q.pixel[q], Q.throughput + 3 * q, K.P.norm_pb2d, cnt, h, lane);
    }
}



// BB1D, warp per query with the two queues of the FP32 warp kernel: pieces past the predicate's
// first check, then accepted candidates.
template <class T>
__device__ __forceinline__ void gen_bb1d_body(const GatherConsts& K, const GenConsts& G, const BeamBVH B,
                                                  const BeamSoA Bs, const LightSum* __restrict__ lsums,
                                                  const SegQueriesDev Q,
                                                  const upbp_mis* __restrict__ cam, const CamSum* __restrict__ cs,
                                                  const GenOut O, unsigned int* __restrict__ work,
                                                  int* __restrict__ status, const int32_t* __restrict__ order)
{
    constexpr int kWarps = 4;
    __shared__ MedT<T> media[UPBP_MAX_MEDIA];
    __shared__ int s_stack[kWarps][kWarpStack];
    __shared__ int s_leaves[kWarps][kWarpLeaves];
    __shared__ int s_piece[kWarps][kGenQueue];
    __shared__ int s_near[kWarps][kGenQueue];
    stage_media_t<T>(G, media);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    int* stack = s_stack[warp];
    int* leaves = s_leaves[warp];
    int* cq = s_piece[warp];
    int* nq = s_near[warp];
    const int leaf_shift = __ffs(B.leaf) - 1;
    for (;;) {
        unsigned qq = 0;
        if (lane == 0) qq = atomicAdd(work, 1u);
        const int64_t item = (int64_t)__shfl_sync(kFull, qq, 0);
        if (item >= Q.n) break;
        const int64_t q = order ? (int64_t)__ldg(&order[item]) : item;
        RgbT<T> acc = rgb_zero<T>();
        unsigned long long cnt = 0, h = 0;
        if ((Q.flags[q] & UPBP_Q_BB1D) && (K.P.techniques & UPBP_BB1D) && B.n > 0) {
            SegCtx<T> s;
            init_ctx(s, K, Q, cam, cs, q);
            const V3 inv = v3(safe_inv(s.df.x), safe_inv(s.df.y), safe_inv(s.df.z));
            acc = seg_loop<T>(K, media, Q, q, s, [&](const MedT<T>& m, int mid, float dminf, float dmaxf) {
                RgbT<T> part = rgb_zero<T>();
                int qn = 0;
                auto eval = [&](int e) {
                    const int i = cq[e];
                    const float4 pa = __ldg(&B.pa[i]);
                    const float4 pb = __ldg(&B.pb[i]);
                    const PiecePayload py = B.pay[i];
                    const int beam = __float_as_int(__ldg(&B.pc[i]).z);
                    const double rchg = Bs.rchange ? (double)__ldg(&Bs.rchange[beam]) : 0.0;
                    const LightSum ls =
                        (K.P.techniques & UPBP_NO_MIS) ? LightSum{} : lsums[__ldg(&Bs.link[beam]).x];
                    part = part + bb1d_contrib<T>(K, m, s, py, ls, v3d(pa.x, pa.y, pa.z), v3d(pb.x, pb.y, pb.z), rchg);
                };
                // the rest of the predicate for one piece per lane (i < 0: none)
                auto full = [&](int i) {
                    bool hit = false;
                    if (i >= 0) {
                        const float4 pc = __ldg(&B.pc[i]);
                        if (__float_as_int(pc.w) == mid) {
                            const float4 pa = __ldg(&B.pa[i]);
                            const float4 pb = __ldg(&B.pb[i]);
                            float dist, sinT, t1, t2, bb, ee;
                            if (test_beam_beam(s.of, s.df, dminf, dmaxf, v3(pa.x, pa.y, pa.z), v3(pb.x, pb.y, pb.z),
                                               0.f, pa.w, pb.w, &dist, &sinT, &t1, &t2, &bb, &ee)) {
                                const int beam = __float_as_int(pc.z);
                                const float rs = beam_start_radius(Bs, &B.pay[i].lv.z);
                                const float radius = beam_radius_at(Bs, beam, rs, t2);
                                // the radius test (PhotonBeam.hxx:411-413), the reach rule and the owner
                                if (!(radius < dist) &&
                                    piece_takes(s.of, s.df, dminf, dmaxf, v3(pa.x, pa.y, pa.z), v3(pb.x, pb.y, pb.z),
                                                pa.w, pc.x, pc.y, t1, bb, ee, dist, rs,
                                                Bs.rchange ? __ldg(&Bs.rchange[beam]) : 0.f, K.bb1d_extra)) {
                                    hit = true;
                                    ++cnt;
                                    h += mix64((unsigned long long)beam);
                                }
                            }
                        }
                    }
                    const unsigned vote = __ballot_sync(kFull, hit);
                    if (vote == 0u) return;
                    if (hit) cq[qn + __popc(vote & lt)] = i;
                    qn += __popc(vote);
                    __syncwarp();
                    if (qn >= 32) {
                        eval(qn - 32 + lane);
                        qn -= 32;
                        __syncwarp();
                    }
                };
                int pn = 0;  // entries in the near queue
                const bool ok = warp_traverse(B.nodes, B.n_leaves, B.n, leaf_shift, s.of, inv, dminf - K.eps,
                                              dmaxf + K.eps, stack, leaves, lane, [&](int i) {
                    bool near = false;
                    if (i >= 0) {
                        const float4 pa = __ldg(&B.pa[i]);
                        const float4 pb = __ldg(&B.pb[i]);
                        near = beam_beam_near(s.of, s.df, v3(pa.x, pa.y, pa.z), v3(pb.x, pb.y, pb.z), pb.w);
                    }
                    const unsigned vote = __ballot_sync(kFull, near);
                    if (vote == 0u) return;
                    if (near) nq[pn + __popc(vote & lt)] = i;
                    pn += __popc(vote);
                    __syncwarp();
                    if (pn >= 32) {
                        full(nq[pn - 32 + lane]);
                        pn -= 32;
                        __syncwarp();
                    }
                });
                if (pn > 0) {
                    full(lane < pn ? nq[lane] : -1);
                    __syncwarp();
                }
                if (lane < qn) eval(lane);
                __syncwarp();
                if (!ok && lane == 0) atomicOr(status, 1);
                return part;
            });
        }
        finish_warp<T>(O, q, acc, Q.pixel[q], Q.throughput + 3 * q, K.P.norm_bb1d, cnt, h, lane);
    }
}

// PP3D: HashGrid::Process + UPBP::RangeQuery::Process (HashGrid.hxx:129-188, UPBP.hxx:86-133).
template <class T>
__global__ void __launch_bounds__(128) k_gen_pp3d(const __grid_constant__ GatherConsts K,
                                                  const __grid_constant__ GenConsts G, const LightSoA Lv,
                                                  const HashGridDev H, const PointQueriesDev Q,
                                                  const upbp_mis* __restrict__ cam, const CamSum* __restrict__ cs,
                                                  const GenOut O)
{
    __shared__ MedT<T> media[UPBP_MAX_MEDIA];
    stage_media_t<T>(G, media);
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const bool valid = q < Q.n;
    const upbp_params& P = K.P;
    uint32_t cnt = 0;
    unsigned long long h = 0;
    RgbT<T> res = rgb_zero<T>();
    const int64_t qs = valid ? q : 0;
    const V3 qp = v3(Q.position[3 * qs], Q.position[3 * qs + 1], Q.position[3 * qs + 2]);
    bool inside = valid && (P.techniques & UPBP_PP3D) && H.n > 0;
    V3 dmin{0.f, 0.f, 0.f};
    if (inside) {
        dmin = xsub3(qp, v3(H.bbox_min[0], H.bbox_min[1], H.bbox_min[2]));
        const V3 dmax = xsub3(v3(H.bbox_max[0], H.bbox_max[1], H.bbox_max[2]), qp);
        inside = !(dmin.x < 0.f || dmin.y < 0.f || dmin.z < 0.f || dmax.x < 0.f || dmax.y < 0.f || dmax.z < 0.f);
    }
    if (inside) {
        const MedT<T>& m = media[Q.medium_id[q]];
        const V3d cfix = v3d(Q.dir_fix[3 * q], Q.dir_fix[3 * q + 1], Q.dir_fix[3 * q + 2]);
        const int L = Q.path_length[q];
        const upbp_mis* snap = cam + Q.cam_mis_begin[q];
        const upbp_mis eL = load_mis(snap + L);
        upbp_mis eL1 = eL;
        if (L >= 2) eL1 = load_mis(snap + L - 1);
        const CamSum csq = cs[q];
        const bool scat_pos = !(val(m.ss[0]) <= 0.0 && val(m.ss[1]) <= 0.0 && val(m.ss[2]) <= 0.0);
        CandT<T> cand;
        cand.f = factors_of(eL);
        cand.pdf_a_inv = cst<T>((double)eL.pdf_a_inv);
        cand.rsp_inv = cst<T>((double)eL.ray_sample_pdf_inv);
        cand.ratio = cst<T>((double)eL.ray_sample_pdfs_ratio);
        const V3 cell = v3(xmul(H.inv_cell, dmin.x), xmul(H.inv_cell, dmin.y), xmul(H.inv_cell, dmin.z));
        const V3 cf = v3(floorf(cell.x), floorf(cell.y), floorf(cell.z));
        const int px = (int)cf.x, py = (int)cf.y, pz = (int)cf.z;
        const int pxo = px + (xsub(cell.x, cf.x) < 0.5f ? -1 : 1);
        const int pyo = py + (xsub(cell.y, cf.y) < 0.5f ? -1 : 1);
        const int pzo = pz + (xsub(cell.z, cf.z) < 0.5f ? -1 : 1);
        for (int j = 0; j < 8; ++j) {
            const int cx = (j & 4) ? pxo : px, cy = (j & 2) ? pyo : py, cz = (j & 1) ? pzo : pz;
            const uint32_t c = hash_cell(cx, cy, cz, H.cells);
            const int e = __ldg(&H.end[c]);
            for (int i = __ldg(&H.start[c]); i < e; ++i) {
                const float4 p = __ldg(&H.pos[i]);
                const V3 dd = xsub3(qp, v3(p.x, p.y, p.z));
                if (!(xdot3(dd, dd) <= H.r2)) continue;
                const int lv = __float_as_int(p.w);
                ++cnt;
                h += mix64((unsigned long long)lv);
                const int4 info = __ldg(&Lv.info[lv]);
                if (!(info.z & UPBP_LV_CONNECTABLE)) continue;
                const int pl = info.y;
                if ((uint32_t)(pl + L) > P.max_path_length || (uint32_t)(pl + L) < P.min_path_length) continue;
                if (!scat_pos) continue;
                const float4 ld = __ldg(&Lv.dir[lv]);
                double sinT;
                const T phase = hg_pdf(cfix, v3d(ld.x, ld.y, ld.z), m.g, &sinT);
                const RgbT<T> factor = RgbT<T>{m.ss[0], m.ss[1], m.ss[2]} * phase;
                if (black_or_neg(factor)) continue;
                const T dirPdf = phase * m.cont;
                const T revPdf = phase * (double)__ldg(&Lv.pos[lv]).w;
                const upbp_mis lvm = load_mis(Lv.mis + lv);
                const double mwfInv = 1.0 / (double)lvm.pp3d_factor;
                const T wc = camera_weight(P, L, cand, cst<T>(mwfInv), sinT, cst<T>((double)lvm.ray_sample_pdf_inv),
                                           cst<T>((double)lvm.ray_sample_pdfs_ratio), revPdf, eL1,
                                           cst<T>((double)eL1.ray_sample_rev_pdf_inv), csq, P.techniques);
                const LightSum ls = Lv.sums[lv];
                const T wl = (dirPdf * ls.c + ls.a) * mwfInv;
                const float4 th = __ldg(&Lv.thr[lv]);
                res = res + RgbT<T>{factor.r * (double)th.x, factor.g * (double)th.y, factor.b * (double)th.z} /
                                (wl + wc);
            }
        }
    }
    finish_lanes<T>(O, valid, q, res, valid ? Q.pixel[q] : -1, valid ? Q.throughput + 3 * q : nullptr, P.norm_pp3d,
                    cnt, h);
}

// B-P2D contribution (extension, standalone, MIS weight 1) in T of an accepted (point x, piece)
// pair: the foot point re-solved in FP64.  r2d is the radius^2 the FP32 predicate accepted with.
template <class T>
__device__ __forceinline__ RgbT<T> bp2d_contrib_t(const MedT<T>& m, const BeamSoA& Bs, float4 pa, float4 pb, int beam,
                                                  V3 x, const V3d& cfix, double r2d)
{
    const V3d o = v3d(pa.x, pa.y, pa.z), d = v3d(pb.x, pb.y, pb.z), p = v3d(x);
    const double t = dot(sub(p, o), d);
    const V3d qv = V3d{o.x + d.x * t - p.x, o.y + d.y * t - p.y, o.z + d.z * t - p.z};
    const double d2 = dot(qv, qv);
    const float4 bthr = __ldg(&Bs.thr[beam]);
    RgbT<T> att = eval_att(m, t);
    const T pfd = comp(att, m.min_idx);
    if ((uint32_t)__float_as_int(bthr.w) & UPBP_SHORT_BEAM) att = att / pfd;
    if (!positive(att)) return rgb_zero<T>();
    double sinT;
    const T phase = hg_pdf(cfix, neg(d), m.g, &sinT);
    if (!(val(phase) > 0.0)) return rgb_zero<T>();
    const double kernel = (1.0 - d2 / r2d) / (r2d * 3.14159265358979323846 * 0.5);
    if (!(kernel > 1e-20)) return rgb_zero<T>();
    return RgbT<T>{att.r * (double)bthr.x, att.g * (double)bthr.y, att.b * (double)bthr.z} *
           RgbT<T>{m.ss[0], m.ss[1], m.ss[2]} * (phase * kernel);
}

// B-P2D in T, warp per point query from the persistent work queue: the lanes test 32 beam pieces
// at a time with the FP32 predicate (a zero-length ray at the point: the slab test is
// point-in-box) and evaluate the accepted ones 32 at a time from the candidate queue.
template <class T>
__global__ void __launch_bounds__(128) k_gen_bp2d(const __grid_constant__ GatherConsts K,
                                                  const __grid_constant__ GenConsts G, const BeamBVH B,
                                                  const BeamSoA Bs, const PointQueriesDev Q, const GenOut O,
                                                  unsigned int* __restrict__ work, int* __restrict__ status)
{
    constexpr int kWarps = 4;
    __shared__ MedT<T> media[UPBP_MAX_MEDIA];
    __shared__ int s_stack[kWarps][kWarpStack];
    __shared__ int s_leaves[kWarps][kWarpLeaves];
    __shared__ int s_piece[kWarps][kGenQueue];
    __shared__ float s_r2[kWarps][kGenQueue];
    stage_media_t<T>(G, media);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    int* stack = s_stack[warp];
    int* leaves = s_leaves[warp];
    int* cq = s_piece[warp];
    float* cr2 = s_r2[warp];
    const int leaf_shift = __ffs(B.leaf) - 1;
    for (;;) {
        unsigned qq = 0;
        if (lane == 0) qq = atomicAdd(work, 1u);
        const int64_t q = (int64_t)__shfl_sync(kFull, qq, 0);
        if (q >= Q.n) break;
        RgbT<T> acc = rgb_zero<T>();
        unsigned long long cnt = 0, h = 0;
        const int mid = Q.medium_id[q];
        const MedT<T>& m = media[mid];
        if ((K.P.techniques & UPBP_BP2D) && m.has_scat && B.n > 0) {
            const V3 x = v3(Q.position[3 * q], Q.position[3 * q + 1], Q.position[3 * q + 2]);
            const V3d cfix = v3d(Q.dir_fix[3 * q], Q.dir_fix[3 * q + 1], Q.dir_fix[3 * q + 2]);
            int qn = 0;
            auto eval = [&](int e) {
                const int i = cq[e];
                const float4 pc = __ldg(&B.pc[i]);
                acc = acc + bp2d_contrib_t<T>(m, Bs, __ldg(&B.pa[i]), __ldg(&B.pb[i]), __float_as_int(pc.z), x, cfix,
                                              (double)cr2[e]);
            };
            const bool ok = warp_traverse(B.nodes, B.n_leaves, B.n, leaf_shift, x, v3(1.f, 1.f, 1.f), 0.f, 0.f, stack,
                                          leaves, lane, [&](int i) {
                bool hit = false;
                float r2 = 0.f;
                if (i >= 0) {
                    const float4 pc = __ldg(&B.pc[i]);
                    if (__float_as_int(pc.w) == mid) {
                        const float4 pa = __ldg(&B.pa[i]);
                        const float4 pb = __ldg(&B.pb[i]);
                        float tf, d2f;
                        if (test_bre(v3(pa.x, pa.y, pa.z), v3(pb.x, pb.y, pb.z), 0.f, pa.w, x, pb.w, &tf, &d2f) &&
                            tf >= pc.x && tf < pc.y) {
                            const int beam = __float_as_int(pc.z);
                            const float rt = beam_radius_at(Bs, beam, beam_start_radius(Bs, &Bs.radius[beam]), tf);
                            r2 = rt * rt;
                            if (!(Bs.rchange && d2f > r2)) {
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
                    cq[pos] = i;
                    cr2[pos] = r2;
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
        finish_warp<T>(O, q, acc, Q.pixel[q], Q.throughput + 3 * q, K.P.norm_bb1d, cnt, h, lane);
    }
}

// The warp gathers as kernels.  The adjoint's dual-number instantiations would take every register a
// thread can have, which leaves 2 blocks of 128 threads per SM; asking for 3 blocks costs some
// spills and runs the diff512 adjoint 8 % faster (4 spills more than it gains).  The FP64 ones keep
// the compiler's own choice (156 and 126 registers, no spills): a minimum of blocks changes it.
template <class T>
__global__ void __launch_bounds__(128) k_gen_pb2d(const __grid_constant__ GatherConsts K,
                                                  const __grid_constant__ GenConsts G, const LightSoA Lv,
                                                  const PhotonBVH B, const SegQueriesDev Q,
                                                  const upbp_mis* __restrict__ cam, const CamSum* __restrict__ cs,
                                                  const GenOut O, unsigned int* __restrict__ work,
                                                  int* __restrict__ status, const int32_t* __restrict__ order)
{
    gen_pb2d_body<T>(K, G, Lv, B, Q, cam, cs, O, work, status, order);
}
__global__ void __launch_bounds__(128, 3) k_gen_pb2d_dual(const __grid_constant__ GatherConsts K,
                                                          const __grid_constant__ GenConsts G, const LightSoA Lv,
                                                          const PhotonBVH B, const SegQueriesDev Q,
                                                          const upbp_mis* __restrict__ cam,
                                                          const CamSum* __restrict__ cs, const GenOut O,
                                                          unsigned int* __restrict__ work, int* __restrict__ status,
                                                          const int32_t* __restrict__ order)
{
    gen_pb2d_body<DualF>(K, G, Lv, B, Q, cam, cs, O, work, status, order);
}
template <class T>
__global__ void __launch_bounds__(128) k_gen_bb1d(const __grid_constant__ GatherConsts K,
                                                  const __grid_constant__ GenConsts G, const BeamBVH B,
                                                  const BeamSoA Bs, const LightSum* __restrict__ lsums,
                                                  const SegQueriesDev Q,
                                                  const upbp_mis* __restrict__ cam, const CamSum* __restrict__ cs,
                                                  const GenOut O, unsigned int* __restrict__ work,
                                                  int* __restrict__ status, const int32_t* __restrict__ order)
{
    gen_bb1d_body<T>(K, G, B, Bs, lsums, Q, cam, cs, O, work, status, order);
}
__global__ void __launch_bounds__(128, 3) k_gen_bb1d_dual(const __grid_constant__ GatherConsts K,
                                                          const __grid_constant__ GenConsts G, const BeamBVH B,
                                                          const BeamSoA Bs, const LightSum* __restrict__ lsums,
                                                          const SegQueriesDev Q, const upbp_mis* __restrict__ cam,
                                                          const CamSum* __restrict__ cs, const GenOut O,
                                                          unsigned int* __restrict__ work, int* __restrict__ status,
                                                          const int32_t* __restrict__ order)
{
    gen_bb1d_body<DualF>(K, G, B, Bs, lsums, Q, cam, cs, O, work, status, order);
}

}  // namespace

template <class T>
static void launch_all(const GenLaunch& A, cudaStream_t s)
{
    if (A.pq.n > 0 && A.hash.n > 0)
        k_gen_pp3d<T><<<(unsigned)((A.pq.n + 127) / 128), 128, 0, s>>>(A.K, A.G, A.L, A.hash, A.pq, A.cam, A.cs_pt,
                                                                        A.out_pp3d);
    if (A.pq.n > 0 && A.beams.n > 0 && (A.K.P.techniques & UPBP_BP2D))
        k_gen_bp2d<T><<<A.bp2d_grid, 128, 0, s>>>(A.K, A.G, A.beams, A.bs, A.pq, A.out_bp2d, A.work + 2, A.status);
    if (A.sq.n > 0 && A.photons.n > 0)
    {
        if constexpr (is_dual<T>::value)
            k_gen_pb2d_dual<<<A.pb2d_grid, 128, 0, s>>>(A.K, A.G, A.L, A.photons, A.sq, A.cam, A.cs_seg, A.out_pb2d,
                                                        A.work + 1, A.status, A.order);
        else
            k_gen_pb2d<T><<<A.pb2d_grid, 128, 0, s>>>(A.K, A.G, A.L, A.photons, A.sq, A.cam, A.cs_seg, A.out_pb2d,
                                                      A.work + 1, A.status, A.order);
    }
    if (A.sq.n > 0 && A.beams.n > 0)
    {
        if constexpr (is_dual<T>::value)
            k_gen_bb1d_dual<<<A.bb1d_grid, 128, 0, s>>>(A.K, A.G, A.beams, A.bs, A.L.sums, A.sq, A.cam, A.cs_seg,
                                                        A.out_bb1d, A.work, A.status, A.order);
        else
            k_gen_bb1d<T><<<A.bb1d_grid, 128, 0, s>>>(A.K, A.G, A.beams, A.bs, A.L.sums, A.sq, A.cam, A.cs_seg,
                                                      A.out_bb1d, A.work, A.status, A.order);
    }
}

void launch_generic(const GenLaunch& A, bool adjoint, cudaStream_t stream)
{
    if (adjoint) launch_all<DualF>(A, stream);
    else launch_all<double>(A, stream);
}

int generic_pb2d_blocks_per_sm(bool adjoint)
{
    int nb = 0;
    if (adjoint) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_gen_pb2d_dual, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_gen_pb2d<double>, 128, 0);
    return nb > 0 ? nb : 1;
}

int generic_bp2d_blocks_per_sm(bool adjoint)
{
    int nb = 0;
    if (adjoint) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_gen_bp2d<DualF>, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_gen_bp2d<double>, 128, 0);
    return nb > 0 ? nb : 1;
}

int generic_bb1d_blocks_per_sm(bool adjoint)
{
    int nb = 0;
    if (adjoint) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_gen_bb1d_dual, 128, 0);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_gen_bb1d<double>, 128, 0);
    return nb > 0 ? nb : 1;
}

}  // namespace gen
}  // namespace upbp
