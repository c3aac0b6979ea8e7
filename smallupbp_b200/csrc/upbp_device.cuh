// Device-side building blocks of the B200 estimator stage.
//
// Predicates that decide candidate sets are evaluated with the reference's
// exact FP32 operation order and no FMA contraction (__fmul_rn/__fadd_rn),
// so that the accepted (query, photon|beam) pairs are bit-identical:
//   dot   = (x*x' + y*y') + z*z'       (_mm_dp_ps mask 0x71, Structs/Vector3.hxx:518-546)
//   cross = a.yzx*b.zxy - a.zxy*b.yzx  (Structs/Vector3.hxx:513-516)
// Contribution arithmetic (transmittance, phase, kernels, MIS) is ordinary
// FP32 and matches the reference within 1e-4 relative.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/upbp_gpu.h"

#define UPBP_PI_F 3.141592653589793238462643383279f
#define UPBP_MAX_MEDIA 16
#define UPBP_MAX_CAM 64

namespace upbp {

// ------------------------------------------------------------------ exact float ops
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float xsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float xdiv(float a, float b) { return __fdiv_rn(a, b); }

struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 xsub3(V3 a, V3 b) { return V3{xsub(a.x, b.x), xsub(a.y, b.y), xsub(a.z, b.z)}; }
__device__ __forceinline__ V3 xadd3(V3 a, V3 b) { return V3{xadd(a.x, b.x), xadd(a.y, b.y), xadd(a.z, b.z)}; }
__device__ __forceinline__ V3 xscale3(V3 a, float s) { return V3{xmul(a.x, s), xmul(a.y, s), xmul(a.z, s)}; }
__device__ __forceinline__ float xdot3(V3 a, V3 b) { return xadd(xadd(xmul(a.x, b.x), xmul(a.y, b.y)), xmul(a.z, b.z)); }
__device__ __forceinline__ V3 xcross3(V3 a, V3 b)
{
    return V3{xsub(xmul(a.y, b.z), xmul(a.z, b.y)), xsub(xmul(a.z, b.x), xmul(a.x, b.z)),
              xsub(xmul(a.x, b.y), xmul(a.y, b.x))};
}
__device__ __forceinline__ V3 neg3(V3 a) { return V3{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ V3 ld3(const float* p) { return V3{p[0], p[1], p[2]}; }

struct Rgb {
    float r, g, b;
};
__device__ __forceinline__ Rgb rgb(float v) { return Rgb{v, v, v}; }
__device__ __forceinline__ Rgb operator*(Rgb a, Rgb b) { return Rgb{a.r * b.r, a.g * b.g, a.b * b.b}; }
__device__ __forceinline__ Rgb operator*(Rgb a, float s) { return Rgb{a.r * s, a.g * s, a.b * s}; }
__device__ __forceinline__ Rgb operator*(float s, Rgb a) { return Rgb{a.r * s, a.g * s, a.b * s}; }
__device__ __forceinline__ Rgb operator/(Rgb a, float s) { return Rgb{a.r / s, a.g / s, a.b / s}; }
__device__ __forceinline__ Rgb operator+(Rgb a, Rgb b) { return Rgb{a.r + b.r, a.g + b.g, a.b + b.b}; }
__device__ __forceinline__ float comp(Rgb a, int i) { return i == 0 ? a.r : (i == 1 ? a.g : a.b); }
// Utils.hxx:109 Float::isPositive: x > 1e-20; Rgb.hxx:213-222
__device__ __forceinline__ bool is_pos(float x) { return x > 1e-20f; }
__device__ __forceinline__ bool rgb_positive(Rgb a) { return is_pos(a.r) && is_pos(a.g) && is_pos(a.b); }
__device__ __forceinline__ bool rgb_black_or_neg(Rgb a) { return a.r <= 0.f && a.g <= 0.f && a.b <= 0.f; }

// ------------------------------------------------------------------ media
// HomogeneousMedium with its derived quantities (Scene/Media.hxx:129-159)
struct DMedium {
    float st[3];    // mAttenuationCoef
    float ss[3];    // mScatteringCoef
    float g;        // mMeanCosine
    float cont;     // mContinuationProb
    float min_st;   // mMinPositiveAttenuationCoefComp
    int min_idx;    // mMinAttenuationCoefIndex
    float mfp;      // mMFP
    int has_scat;   // kHasScattering
    int gray;       // sigma_t equal in all channels: one exp per attenuation
};

// EvalAttenuation(dist) = exp(-sigma_t * dist) per channel (Media.hxx:216-229)
__device__ __forceinline__ Rgb eval_att(const DMedium& m, float dist)
{
    if (m.gray) {
        const float a = expf(-m.st[0] * dist);
        return Rgb{a, a, a};
    }
    return Rgb{expf(-m.st[0] * dist), expf(-m.st[1] * dist), expf(-m.st[2] * dist)};
}
template <typename R>
__device__ __forceinline__ R eval_att_t(const DMedium& m, R dist, int c)
{
    return exp(-(R)m.st[c] * dist);
}

// RaySamplePdf (Media.hxx:294-323)
__device__ __forceinline__ float ray_sample_pdf(const DMedium& m, float dmin, float dmax, uint32_t flags, float* rev)
{
    float pdf = 1.f;
    *rev = 1.f;
    if (m.min_st != 0.f && m.has_scat) {
        const float att = fmaxf(expf(-m.min_st * (dmax - dmin)), 1e-35f);
        const float minatt = m.min_st * att;
        pdf = (flags & UPBP_END_IN_MEDIUM) ? minatt : att;
        *rev = (flags & UPBP_ORIGIN_IN_MEDIUM) ? minatt : att;
    }
    return pdf;
}

// PhaseFunction::Pdf (Path/PhaseFunction.hxx:50-80); UniformSpherePdfW = INV_PI_F * 0.25
__device__ __forceinline__ float hg_pdf(V3 fix, V3 gen, float g, float* sin_theta)
{
    const float inv4pi = (1.f / UPBP_PI_F) * 0.25f;
    const float cos_t = -xdot3(gen, fix);
    *sin_theta = sqrtf(fmaxf(0.f, 1.f - cos_t * cos_t));
    if (fabsf(g) < 1e-3f) return inv4pi;
    const float g2 = g * g;
    const float d = 1.f + g2 - (g + g) * cos_t;
    return d > 0.f ? (inv4pi * (1.f - g2) / (d * sqrtf(d))) : 0.f;
}

// ------------------------------------------------------------------ candidate predicates
// EmbreePhoton::testIntersectionBre (Bre/Bre.cxx:199-223)
__device__ __forceinline__ bool test_bre(V3 o, V3 d, float tmin, float tmax, V3 p, float r2, float* t_out,
                                         float* d2_out)
{
    const V3 op = xsub3(p, o);
    const float t = xdot3(op, d);
    if (t > tmin && t < tmax) {
        const V3 q = xsub3(xadd3(o, xscale3(d, t)), p);
        const float d2 = xdot3(q, q);
        if (d2 <= r2) {
            *t_out = t;
            *d2_out = d2;
            return true;
        }
    }
    return false;
}

// The first check of test_beam_beam: false where it rejects by the distance of the lines alone.
__device__ __forceinline__ bool beam_beam_near(V3 O1, V3 d1, V3 O2, V3 d2, float maxDistSqr)
{
    const V3 c = xcross3(d1, d2);
    const float sinThetaSqr = xdot3(c, c);
    const float ad = xdot3(xsub3(O2, O1), c);
    return !(xmul(ad, ad) >= xmul(maxDistSqr, sinThetaSqr));
}

// The second part of test_beam_beam: the near-parallel rejection and the query parameter t1 of the
// lines' closest points, with d1.d2, d1.O2 and e = d2.O1 - d2.O2 (false: near-parallel).
__device__ __forceinline__ bool beam_beam_t1(V3 O1, V3 d1, V3 O2, V3 d2, float& d1d2, float& d1O1, float& d1O2,
                                             float& e, float& t1)
{
    d1d2 = xdot3(d1, d2);
    const float d1d2Sqr = xmul(d1d2, d1d2);
    const float d1d2SqrMinus1 = xsub(d1d2Sqr, 1.0f);
    if (d1d2SqrMinus1 < 1e-5f && d1d2SqrMinus1 > -1e-5f) return false;
    d1O1 = xdot3(d1, O1);
    d1O2 = xdot3(d1, O2);
    e = xsub(xdot3(d2, O1), xdot3(d2, O2));
    t1 = xdiv(xsub(xsub(d1O1, d1O2), xmul(d1d2, e)), d1d2SqrMinus1);
    return true;
}

// PhotonBeam::testIntersectionBeamBeam (Beams/PhotonBeam.hxx:238-296).  On acceptance it can also
// return b = d1.d2 and e = d2.O1 - d2.O2, the terms of the line solution that piece_takes_fast uses.
__device__ __forceinline__ bool test_beam_beam(V3 O1, V3 d1, float minT1, float maxT1, V3 O2, V3 d2, float minT2,
                                               float maxT2, float maxDistSqr, float* oDist, float* oSin, float* oT1,
                                               float* oT2, float* oB = nullptr, float* oE = nullptr)
{
    const V3 c = xcross3(d1, d2);
    const float sinThetaSqr = xdot3(c, c);
    const float ad = xdot3(xsub3(O2, O1), c);
    if (xmul(ad, ad) >= xmul(maxDistSqr, sinThetaSqr)) return false;
    float d1d2, d1O1, d1O2, e, t1;
    if (!beam_beam_t1(O1, d1, O2, d2, d1d2, d1O1, d1O2, e, t1)) return false;
    if (t1 <= minT1 || t1 >= maxT1) return false;
    const float t2 = xdiv(xsub(xadd(t1, d1O1), d1O2), d1d2);
    if (t2 <= minT2 || t2 >= maxT2 || isnan(t2)) return false;
    const float s = __fsqrt_rn(sinThetaSqr);
    *oDist = xdiv(fabsf(ad), s);
    *oSin = s;
    *oT1 = t1;
    *oT2 = t2;
    if (oB) *oB = d1d2;
    if (oE) *oE = e;
    return true;
}

// Which BB1D candidates are taken, and by which piece of the beam.
//
// The reference predicate (PhotonBeam.hxx:238-296) tests the whole beam; the beam is split into
// pieces here only for culling, so exactly one piece must take each candidate, and whether a
// candidate is found must not depend on the tree, the leaf size or the piece length.  The FP32 t2
// = (t1 + d1.O1 - d1.O2) / (d1.d2) of the predicate is ill-conditioned for nearly perpendicular
// pairs (and t1, t2 for nearly parallel ones): it can accept a pair whose true closest point lies
// outside the beam segment, far from any box the query crosses, so no spatial search (nor the
// reference's own grid, Grid.hxx) finds every such pair.  The candidate set is therefore defined
// by a reach rule that every implementation here applies (the CUDA kernels and the C oracle):
//
//   taken  <=>  the FP32 predicate and the radius test accept the pair (reference order), and
//               the FP64 distance D of the query segment [dmin, dmax] and the beam segment
//               [0, len] satisfies D <= r(u) + e, where u is the beam parameter of their closest
//               point, r(u) the beam radius there and e = bb1d_reach_extra(r).
//
// The rule keeps every pair whose segments really pass within the radius; it drops only pairs
// that the FP32 predicate accepts through rounding.  The owner is the piece containing u.  Its box
// contains every point within r(u) + e of the owned part of the segment -- for a u inside (0, len)
// that point lies in the disc perpendicular to the beam, for u = 0 or len in the ball about the
// end point, which the end pieces' boxes include -- so the traversal reaches the owner of every
// taken pair, whatever the tree.
__host__ __device__ __forceinline__ float bb1d_reach_extra(float r) { return 2e-5f + 1e-3f * r; }
// slack of the piece boxes: the reach margin plus the rounding of the slab test
__host__ __device__ __forceinline__ float bb1d_box_eps(float r) { return bb1d_reach_extra(r) + 1e-5f; }

// FP64 closest points of the query segment [dmin, dmax] and the beam segment [0, len]: the beam
// parameter u and the squared distance.
struct SegClosest {
    double u, d2;
};
__device__ __forceinline__ SegClosest seg_closest_f64(V3 O1, V3 d1, float dminf, float dmaxf, V3 O2, V3 d2, float lenf)
{
    const double wx = (double)O1.x - O2.x, wy = (double)O1.y - O2.y, wz = (double)O1.z - O2.z;
    const double ax = d1.x, ay = d1.y, az = d1.z, bx = d2.x, by = d2.y, bz = d2.z;
    const double aa = ax * ax + ay * ay + az * az, cc = bx * bx + by * by + bz * bz, b = ax * bx + ay * by + az * bz;
    const double dd = ax * wx + ay * wy + az * wz, ee = bx * wx + by * wy + bz * wz;
    const double den = aa * cc - b * b;
    const double dmin = dminf, dmax = dmaxf, len = lenf;
    double t = dmin, u = 0.0;
    bool inside = false;
    if (den > 1e-300) {
        const double inv = 1.0 / den;
        t = (b * ee - cc * dd) * inv;
        u = (aa * ee - b * dd) * inv;
        inside = t >= dmin && t <= dmax && u >= 0.0 && u <= len;  // closest points inside both
    }
    if (!inside) {
        t = fmin(fmax(t, dmin), dmax);
        u = fmin(fmax((b * t + ee) / cc, 0.0), len);
        t = fmin(fmax((b * u - dd) / aa, dmin), dmax);
        u = fmin(fmax((b * t + ee) / cc, 0.0), len);
    }
    const double rx = wx + t * ax - u * bx, ry = wy + t * ay - u * by, rz = wz + t * az - u * bz;
    return SegClosest{u, rx * rx + ry * ry + rz * rz};
}

// 1: this piece takes the candidate, 0: it does not (another piece owns it), -1: undecided in
// FP32 (use piece_takes_f64).  Called after the predicate and the radius test accepted the pair,
// with b = d1.d2, e = d2.O1 - d2.O2 and t1 from the predicate; rs, rc = the beam radius at 0 and
// its change per unit t.  The reference's own t2 = (t1 + d1.O1 - d1.O2) / b is ill-conditioned for
// nearly perpendicular pairs, so the beam parameter of the lines' closest points is taken as
// u = e + b t1 instead, which is well-conditioned whenever the lines are not nearly parallel.
// The rounding error of t1 and u grows as 1 / (1 - b^2) (t1 divides by b^2 - 1): it stays below
// 39 ulp x scale / (1 - b^2), under m = 6e-6 x scale / (1 - b^2), so t1 and u more than m inside
// their ranges put the exact closest points inside both segments: u is the owner's parameter, and
// D is the distance of the lines, which the FP32 dist approximates within errb (|ad| carries at
// most 6 ulp of |O2 - O1|_1 and is divided by sin(theta); errb is twice that bound).  Below
// 1 - b^2 = 0.002 (the lines within 2.6 degrees of parallel) the FP64 solve decides.  (Checked on
// the CPU against the FP64 rule over 64 M piece decisions of pairs concentrated at 1 - b^2 in
// [0.0006, 0.12]: none differs.)
__device__ __forceinline__ int piece_takes_fast(V3 O1, V3 d1, float dmin, float dmax, V3 O2, float len, float t_lo,
                                                float t_hi, float t1, float b, float e, float dist, float rs,
                                                float rc, float extra)
{
    const float om = 1.f - b * b;
    if (om > 0.002f) {
        const float scale = fmaxf(fmaxf(fmaxf(fabsf(O1.x), fabsf(O1.y)), fmaxf(fabsf(O1.z), fabsf(O2.x))),
                                  fmaxf(fmaxf(fabsf(O2.y), fabsf(O2.z)), fmaxf(fmaxf(len, fabsf(dmax)), 1.f)));
        const float m = __fdividef(6e-6f * scale, om);
        const float u = e + b * t1;
        if (t1 > dmin + m && t1 < dmax - m && u > m && u < len - m) {
            if (u < t_lo - m || u >= t_hi + m) return 0;
            if (u >= t_lo + m && u < t_hi - m) {
                const float w1 = fabsf(O2.x - O1.x) + fabsf(O2.y - O1.y) + fabsf(O2.z - O1.z);
                const float errb = 8e-7f * w1 * rsqrtf(om) + 3e-6f * dist + 1e-8f;
                if (dist + errb + fabsf(rc) * m <= rs + u * rc + extra) return 1;
            }
        }
    }
    return -1;
}

// The reach rule and the owner in FP64: rs, rc = the beam radius at 0 and its change per unit t.
__device__ __forceinline__ bool piece_takes_f64(V3 O1, V3 d1, float dmin, float dmax, V3 O2, V3 d2, float len,
                                                float t_lo, float t_hi, float rs, float rc, float extra)
{
    const SegClosest sc = seg_closest_f64(O1, d1, dmin, dmax, O2, d2, len);
    if (!(sc.u >= (double)t_lo && (sc.u < (double)t_hi || t_hi >= len))) return false;
    const double rho = (double)rs + sc.u * (double)rc + (double)extra;
    return sc.d2 <= rho * rho;
}

__device__ __forceinline__ bool piece_takes(V3 O1, V3 d1, float dmin, float dmax, V3 O2, V3 d2, float len,
                                            float t_lo, float t_hi, float t1, float b, float e, float dist, float rs,
                                            float rc, float extra)
{
    const int f = piece_takes_fast(O1, d1, dmin, dmax, O2, len, t_lo, t_hi, t1, b, e, dist, rs, rc, extra);
    return f >= 0 ? f == 1 : piece_takes_f64(O1, d1, dmin, dmax, O2, d2, len, t_lo, t_hi, rs, rc, extra);
}

// ------------------------------------------------------------------ MIS walks
__device__ __forceinline__ bool mis_spec(const upbp_mis& m) { return (m.flags & UPBP_MIS_IS_SPECULAR) != 0; }

// AccumulateCameraPathWeight (Path/PathWeight.hxx:33-142).  cam(k) returns the
// camera MisData entry k as the reference array holds it during the call.
template <class Cam>
__device__ float camera_path_weight(int L, float lastRev, float lastSin, float lastRayRev, float lastRayRevRatio,
                                    float ntlPartialRevPdfW, uint32_t qbt, uint32_t pbt, uint32_t tech, const Cam& cam)
{
    float weight = 0.f, product = 1.f, weightBB1D = 0.f;
    const int lastIndex = L;
    for (int index = 0; index < L; ++index) {
        const upbp_mis cur = cam(lastIndex - index);
        const bool nextSpec = index < L - 1 ? mis_spec(cam(lastIndex - index - 1)) : mis_spec(cur);
        if ((tech & UPBP_BB1D_PREVIOUS) && !mis_spec(cur)) weightBB1D = 0.f;
        float rev = cur.rev_pdf_a, sinT = cur.sin_theta, rayRev = cur.ray_sample_rev_pdf_inv,
              rayRevRatio = cur.ray_sample_rev_pdfs_ratio;
        if (index == 0) {
            rev = lastRev;
            sinT = lastSin;
            rayRev = lastRayRev;
            rayRevRatio = lastRayRevRatio;
        } else if (index == 1) {
            rev *= ntlPartialRevPdfW;
        }
        product *= rev;
        const bool usable = index == 0 || !mis_spec(cur);
        if ((tech & UPBP_SURF) && usable) weight += product * cur.surf_factor;
        if (tech & UPBP_PP3D) weight += product * cur.pp3d_factor;
        if (tech & UPBP_PB2D) {
            if (qbt & UPBP_LONG_BEAM) weight += product * cur.pb2d_factor * cur.ray_sample_pdf_inv;
            else weight += product * cur.pb2d_factor * cur.ray_sample_pdfs_ratio;
        }
        if ((tech & UPBP_BB1D) && (cur.flags & UPBP_MIS_IN_MEDIUM_WITH_BEAMS)) {
            if (tech & UPBP_NO_SINE_IN_WEIGHTS) sinT = 1.f;
            const float a = (qbt & UPBP_LONG_BEAM) ? cur.ray_sample_pdf_inv : cur.ray_sample_pdfs_ratio;
            const float b = (pbt & UPBP_LONG_BEAM) ? rayRev : rayRevRatio;
            weightBB1D += product * cur.bb1d_factor * cur.bb1d_beam_selection_pdf * a * sinT * b;
        }
        product *= cur.pdf_a_inv;
        if ((tech & UPBP_BPT) && usable && !nextSpec) weight += product;
    }
    return weight + weightBB1D;
}

// AccumulateLightPathWeight (Path/PathWeight.hxx:145-270).  lv(k) returns the
// MisData of light vertex k; for BB1D, beam_rec replaces the index-0 entry.
template <class Lv>
__device__ float light_path_weight(int pathIdx, int pathLength, float lastRev, float lastSin, float lastRayRev,
                                   float lastRayRevRatio, float ntlPartialRevPdfW, uint32_t technique, uint32_t qbt,
                                   uint32_t pbt, uint32_t tech, const int32_t* pathEnds, const Lv& lv,
                                   const upbp_mis* beam_rec)
{
    float weight = 0.f, product = 1.f;
    const int lastIndex = (pathIdx == 0) ? pathLength : pathEnds[pathIdx - 1] + pathLength;
    for (int index = 0; index <= pathLength; ++index) {
        const upbp_mis cur = (technique == UPBP_BB1D && index == 0) ? *beam_rec : lv(lastIndex - index);
        const bool nextSpec = index < pathLength ? mis_spec(lv(lastIndex - index - 1)) : mis_spec(cur);
        float rev = cur.rev_pdf_a, sinT = cur.sin_theta, rayRev = cur.ray_sample_rev_pdf_inv,
              rayRevRatio = cur.ray_sample_rev_pdfs_ratio;
        if (index == 0) {
            rev = lastRev;
            sinT = lastSin;
            rayRev = lastRayRev;
            rayRevRatio = lastRayRevRatio;
        } else if (index == 1) {
            rev = technique == UPBP_BB1D ? ntlPartialRevPdfW : cur.rev_pdf_a_without_bsdf * ntlPartialRevPdfW;
        }
        if (rev == 0.f) break;
        product *= rev;
        const bool usable = index == 0 || !mis_spec(cur);
        if (index != 0 || technique == UPBP_BPT) {
            if ((tech & UPBP_SURF) && usable) weight += product * cur.surf_factor;
            if (tech & UPBP_PP3D) weight += product * cur.pp3d_factor;
            if (tech & UPBP_PB2D) {
                if (qbt & UPBP_LONG_BEAM) weight += product * cur.pb2d_factor * rayRev;
                else weight += product * cur.pb2d_factor * rayRevRatio;
            }
            if ((tech & UPBP_BB1D) && !(tech & UPBP_BB1D_PREVIOUS) && (cur.flags & UPBP_MIS_IN_MEDIUM_WITH_BEAMS)) {
                if (tech & UPBP_NO_SINE_IN_WEIGHTS) sinT = 1.f;
                const float a = (qbt & UPBP_LONG_BEAM) ? rayRev : rayRevRatio;
                const float b = (pbt & UPBP_LONG_BEAM) ? cur.ray_sample_pdf_inv : cur.ray_sample_pdfs_ratio;
                weight += product * cur.bb1d_factor * cur.bb1d_beam_selection_pdf * a * sinT * b;
            }
        }
        product *= cur.pdf_a_inv;
        if ((tech & UPBP_BPT) && usable && !nextSpec) weight += product;
        if (tech & UPBP_PREVIOUS) break;
    }
    return weight;
}

__device__ __forceinline__ upbp_mis load_mis(const upbp_mis* p)
{
    upbp_mis m;
    const float* f = reinterpret_cast<const float*>(p);
    m.pdf_a_inv = __ldg(f + 0);
    m.rev_pdf_a = __ldg(f + 1);
    m.rev_pdf_a_without_bsdf = __ldg(f + 2);
    m.ray_sample_pdf_inv = __ldg(f + 3);
    m.ray_sample_rev_pdf_inv = __ldg(f + 4);
    m.ray_sample_pdfs_ratio = __ldg(f + 5);
    m.ray_sample_rev_pdfs_ratio = __ldg(f + 6);
    m.sin_theta = __ldg(f + 7);
    m.cos_theta_out = __ldg(f + 8);
    m.surf_factor = __ldg(f + 9);
    m.pp3d_factor = __ldg(f + 10);
    m.pb2d_factor = __ldg(f + 11);
    m.bb1d_factor = __ldg(f + 12);
    m.bb1d_beam_selection_pdf = __ldg(f + 13);
    m.flags = __ldg(reinterpret_cast<const uint32_t*>(p) + 14);
    return m;
}

// splitmix64 finaliser of (id+1): order-independent candidate-set hash term
__device__ __forceinline__ unsigned long long mix64(unsigned long long id)
{
    unsigned long long z = id + 1ull + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

}  // namespace upbp
