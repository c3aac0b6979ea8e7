// FP64 partial sums of the UPBP MIS walks (Path/PathWeight.hxx:33-270).
//
// AccumulateLightPathWeight and AccumulateCameraPathWeight walk the whole light / camera
// subpath for every accepted candidate.  Only the first two walk steps depend on the
// candidate: index 0 (the merged vertex) takes the candidate's pdfs, index 1 (the vertex
// before it) takes the candidate's next-to-last reverse pdf and, for BB1D, a reverse ray
// sampling pdf written by the estimator.  Everything from index 2 on reads records that are
// final when the estimators run, so it is precomputed once per light vertex and once per
// query, in FP64, and each candidate combines them in O(1).
//
// Light side, for light vertex u as the "index >= 2" vertex of a walk:
//   G(u) = rev_u == 0 ? 0 : rev_u * (Mfix(u) + rayRev_u * Mr(u) + pdfAInv_u * (B(u) + G(u-1)))
// with M(u) = Mfix(u) + rayRev * Mr(u) the merging terms (SURF, PP3D, PB2D, BB1D) and B(u)
// the BPT term of the walk loop; G(start-1) = 0 (the walk ends at the light source).
// Per light vertex we keep
//   a = pdfAInv_u * B0(u)                                  (index 0 BPT term, PB2D/PP3D photon u)
//   c = pdfAInv_u * revWB_{u-1} * (M(u-1) + T(u-1))         (index 1 onward, PB2D/PP3D photon u)
//   d = Mfix(u) + T(u),  e = Mr(u)                          (u as index 1 of a BB1D walk)
//   bptb = BPT term of index 0 of a BB1D walk whose beam starts at u
// where T(u) = pdfAInv_u * (B(u) + G(u-1)).  Then
//   PB2D / PP3D: wLight = last * (a_j + ntl * c_j)
//   BB1D:        wLight = last * pdfAInv_beam * (bptb_u + ntl * (d_u + e_u / revRaySamplePdf))
//
// Camera side, per query: S_other / S_bb1d = the walk's sums over entries L-2 .. 1 relative to
// the product after index 1, with the BB1D_PREVIOUS resets folded in (reset = a reset
// happened inside that suffix, which discards the index 0/1 BB1D terms).
#pragma once

#include "upbp_device.cuh"

namespace upbp {

struct __align__(8) LightSum {
    double a, c, d, e;
    float bptb;
    uint32_t pad;
};

struct __align__(8) CamSum {
    double s_other, s_bb1d;
    float f_other, f_bb1d;  // the same sums rounded to FP32, for the per-candidate combination
    uint32_t flags;  // bit0: reset inside the suffix, bit1: entry L-2 (or L-1 when L == 2) is specular
    uint32_t pad;
};

// Merging terms of one walk vertex split into the part without and the coefficient of
// the reverse ray-sampling pdf (the only field the BB1D estimator overrides at index 1).
__device__ __forceinline__ void light_merge_terms(const upbp_mis& m, uint32_t tech, uint32_t qbt, uint32_t pbt,
                                                  double& fix, double& rcoef)
{
    fix = 0.0;
    rcoef = 0.0;
    const bool usable = !(m.flags & UPBP_MIS_IS_SPECULAR);
    if ((tech & UPBP_SURF) && usable) fix += (double)m.surf_factor;
    if (tech & UPBP_PP3D) fix += (double)m.pp3d_factor;
    if (tech & UPBP_PB2D) {
        if (qbt & UPBP_LONG_BEAM) rcoef += (double)m.pb2d_factor;
        else fix += (double)m.pb2d_factor * m.ray_sample_rev_pdfs_ratio;
    }
    if ((tech & UPBP_BB1D) && !(tech & UPBP_BB1D_PREVIOUS) && (m.flags & UPBP_MIS_IN_MEDIUM_WITH_BEAMS)) {
        const double sinT = (tech & UPBP_NO_SINE_IN_WEIGHTS) ? 1.0 : (double)m.sin_theta;
        const double b = (pbt & UPBP_LONG_BEAM) ? (double)m.ray_sample_pdf_inv : (double)m.ray_sample_pdfs_ratio;
        const double k = (double)m.bb1d_factor * m.bb1d_beam_selection_pdf * sinT * b;
        if (qbt & UPBP_LONG_BEAM) rcoef += k;
        else fix += k * m.ray_sample_rev_pdfs_ratio;
    }
}

// Camera-walk merging terms of one entry (PathWeight.hxx:88-126) with explicit ray reverse pdfs,
// accumulated in R (double for the FP64 partial sums, float for the per-candidate combination).
template <class R>
__device__ __forceinline__ void cam_merge_terms(const upbp_mis& m, bool usable, float sinT, float rayRev,
                                                float rayRevRatio, uint32_t tech, uint32_t qbt, uint32_t pbt,
                                                R& other, R& bb1d)
{
    other = 0;
    bb1d = 0;
    if ((tech & UPBP_SURF) && usable) other += (R)m.surf_factor;
    if (tech & UPBP_PP3D) other += (R)m.pp3d_factor;
    if (tech & UPBP_PB2D)
        other += (R)m.pb2d_factor * (R)((qbt & UPBP_LONG_BEAM) ? m.ray_sample_pdf_inv : m.ray_sample_pdfs_ratio);
    if ((tech & UPBP_BB1D) && (m.flags & UPBP_MIS_IN_MEDIUM_WITH_BEAMS)) {
        const R s = (tech & UPBP_NO_SINE_IN_WEIGHTS) ? (R)1 : (R)sinT;
        const R a = (qbt & UPBP_LONG_BEAM) ? (R)m.ray_sample_pdf_inv : (R)m.ray_sample_pdfs_ratio;
        const R b = (pbt & UPBP_LONG_BEAM) ? (R)rayRev : (R)rayRevRatio;
        bb1d += (R)m.bb1d_factor * (R)m.bb1d_beam_selection_pdf * a * s * b;
    }
}

// Camera weight from the candidate's index-0 record, entry L-1 (index 1, with the reverse
// ray pdf the estimator writes) and the precomputed FP64 suffix.  The candidate's terms are
// combined in FP32: every term is a non-negative product of pdfs, so the sum has no cancellation
// and FP32 carries the weight to a few ulp; the recursive sums over the rest of the path are the
// FP64 ones, rounded once (CamSum::f_other, f_bb1d).
__device__ __forceinline__ float camera_weight_fast(int L, const upbp_mis& cand, float lastRev, float lastSin,
                                                    float lastRayRev, float lastRayRevRatio, float ntl,
                                                    const upbp_mis& e, float e_ray_rev, const CamSum& cs,
                                                    uint32_t tech, uint32_t qbt, uint32_t pbt)
{
    float prod = lastRev;
    float o0, b0;
    cam_merge_terms<float>(cand, true, lastSin, lastRayRev, lastRayRevRatio, tech, qbt, pbt, o0, b0);
    float w_o = prod * o0, w_b = prod * b0;
    prod *= cand.pdf_a_inv;
    const bool next0_spec = L >= 2 ? (e.flags & UPBP_MIS_IS_SPECULAR) != 0 : (cand.flags & UPBP_MIS_IS_SPECULAR) != 0;
    if ((tech & UPBP_BPT) && !next0_spec) w_o += prod;
    if (L >= 2) {
        const bool espec = (e.flags & UPBP_MIS_IS_SPECULAR) != 0;
        if ((tech & UPBP_BB1D_PREVIOUS) && !espec) w_b = 0.f;
        prod *= e.rev_pdf_a * ntl;
        float o1, b1;
        cam_merge_terms<float>(e, !espec, e.sin_theta, e_ray_rev, e.ray_sample_rev_pdfs_ratio, tech, qbt, pbt, o1, b1);
        w_o += prod * o1;
        w_b += prod * b1;
        prod *= e.pdf_a_inv;
        if ((tech & UPBP_BPT) && !espec && !(cs.flags & 2u)) w_o += prod;
        w_o += prod * cs.f_other;
        w_b = (cs.flags & 1u) ? prod * cs.f_bb1d : w_b + prod * cs.f_bb1d;
    }
    return w_o + w_b;
}

}  // namespace upbp
