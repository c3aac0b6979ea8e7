// Scalar-generic estimator arithmetic: the contributions of PB2D, BB1D and PP3D written once over a
// scalar type T, instantiated as
//   * double -- the FP64 evaluation mode (an FP64 oracle on the GPU: the candidate sets come from
//     the same FP32 predicates, the candidate geometry is re-solved in FP64 and all contribution
//     and MIS arithmetic is FP64), and
//   * DualF  -- forward-mode tangents (FP32) with respect to one medium's sigma_a (rgb),
//     sigma_s (rgb) and g, used by the adjoint kernels (the vector-Jacobian product of the
//     estimator sum).
// Transmittance is recomputed from the medium at every use, never stored.
#pragma once

#include <type_traits>

#include "upbp_device.cuh"
#include "upbp_mis_prep.cuh"

namespace upbp {
namespace gen {

constexpr int kNT = 7;  // tangent slots: sigma_a r,g,b, sigma_s r,g,b, g

// Forward-mode number: a value and its kNT tangents, in scalar S.  The adjoint runs in
// DualF (FP32 value and tangents: half the registers of FP64, within the 1e-3 gradient bound);
// DualD keeps FP64 for checks of the tangent arithmetic itself.
template <class S>
struct DualS {
    S v;
    S d[kNT];
};
using DualD = DualS<double>;
using DualF = DualS<float>;
template <class T> struct is_dual : std::false_type {};
template <class S> struct is_dual<DualS<S>> : std::true_type {};

template <class S>
__device__ __forceinline__ DualS<S> dual(S v)
{
    DualS<S> r;
    r.v = v;
#pragma unroll
    for (int i = 0; i < kNT; ++i) r.d[i] = S(0);
    return r;
}
template <class S>
__device__ __forceinline__ DualS<S> operator+(const DualS<S>& a, const DualS<S>& b)
{
    DualS<S> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < kNT; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <class S>
__device__ __forceinline__ DualS<S> operator-(const DualS<S>& a, const DualS<S>& b)
{
    DualS<S> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < kNT; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <class S>
__device__ __forceinline__ DualS<S> operator-(const DualS<S>& a)
{
    DualS<S> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < kNT; ++i) r.d[i] = -a.d[i];
    return r;
}
template <class S>
__device__ __forceinline__ DualS<S> operator*(const DualS<S>& a, const DualS<S>& b)
{
    DualS<S> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < kNT; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <class S>
__device__ __forceinline__ DualS<S> operator/(const DualS<S>& a, const DualS<S>& b)
{
    DualS<S> r;
    const S ib = S(1) / b.v;
    r.v = a.v * ib;
#pragma unroll
    for (int i = 0; i < kNT; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
    return r;
}
template <class S>
__device__ __forceinline__ DualS<S> operator+(const DualS<S>& a, double b)
{
    DualS<S> r = a;
    r.v += (S)b;
    return r;
}
template <class S>
__device__ __forceinline__ DualS<S> operator+(double a, const DualS<S>& b) { return b + a; }
template <class S>
__device__ __forceinline__ DualS<S> operator-(const DualS<S>& a, double b)
{
    DualS<S> r = a;
    r.v -= (S)b;
    return r;
}
template <class S>
__device__ __forceinline__ DualS<S> operator-(double a, const DualS<S>& b)
{
    DualS<S> r = -b;
    r.v += (S)a;
    return r;
}
template <class S>
__device__ __forceinline__ DualS<S> operator*(const DualS<S>& a, double b)
{
    DualS<S> r;
    const S sb = (S)b;
    r.v = a.v * sb;
#pragma unroll
    for (int i = 0; i < kNT; ++i) r.d[i] = a.d[i] * sb;
    return r;
}
template <class S>
__device__ __forceinline__ DualS<S> operator*(double a, const DualS<S>& b) { return b * a; }
template <class S>
__device__ __forceinline__ DualS<S> operator/(const DualS<S>& a, double b) { return a * (1.0 / b); }
template <class S>
__device__ __forceinline__ DualS<S> operator/(double a, const DualS<S>& b)
{
    DualS<S> r;
    const S ib = S(1) / b.v;
    r.v = (S)a * ib;
#pragma unroll
    for (int i = 0; i < kNT; ++i) r.d[i] = -r.v * ib * b.d[i];
    return r;
}
template <class S>
__device__ __forceinline__ DualS<S>& operator+=(DualS<S>& a, const DualS<S>& b) { return a = a + b; }
template <class S>
__device__ __forceinline__ DualS<S>& operator*=(DualS<S>& a, const DualS<S>& b) { return a = a * b; }

__device__ __forceinline__ double val(double x) { return x; }
template <class S>
__device__ __forceinline__ double val(const DualS<S>& x) { return (double)x.v; }

template <class T> __device__ __forceinline__ T cst(double v);
template <> __device__ __forceinline__ double cst<double>(double v) { return v; }
template <> __device__ __forceinline__ DualD cst<DualD>(double v) { return dual<double>(v); }
template <> __device__ __forceinline__ DualF cst<DualF>(double v) { return dual<float>((float)v); }

__device__ __forceinline__ double t_exp(double x) { return exp(x); }
__device__ __forceinline__ float t_exp_s(float x) { return expf(x); }
__device__ __forceinline__ double t_exp_s(double x) { return exp(x); }
template <class S>
__device__ __forceinline__ DualS<S> t_exp(const DualS<S>& x)
{
    DualS<S> r;
    r.v = t_exp_s(x.v);
#pragma unroll
    for (int i = 0; i < kNT; ++i) r.d[i] = r.v * x.d[i];
    return r;
}
__device__ __forceinline__ double t_sqrt(double x) { return sqrt(x); }
template <class S>
__device__ __forceinline__ DualS<S> t_sqrt(const DualS<S>& x)
{
    DualS<S> r;
    r.v = sqrt(x.v);
    const S k = r.v > S(0) ? S(0.5) / r.v : S(0);
#pragma unroll
    for (int i = 0; i < kNT; ++i) r.d[i] = k * x.d[i];
    return r;
}

template <class T>
struct RgbT {
    T r, g, b;
};
template <class T> __device__ __forceinline__ RgbT<T> rgbt(const T& v) { return RgbT<T>{v, v, v}; }
template <class T> __device__ __forceinline__ RgbT<T> rgb_zero() { return rgbt<T>(cst<T>(0.0)); }
template <class T>
__device__ __forceinline__ RgbT<T> operator*(const RgbT<T>& a, const RgbT<T>& b)
{
    return RgbT<T>{a.r * b.r, a.g * b.g, a.b * b.b};
}
template <class T, class S>
__device__ __forceinline__ RgbT<T> operator*(const RgbT<T>& a, const S& s)
{
    return RgbT<T>{a.r * s, a.g * s, a.b * s};
}
template <class T>
__device__ __forceinline__ RgbT<T> operator+(const RgbT<T>& a, const RgbT<T>& b)
{
    return RgbT<T>{a.r + b.r, a.g + b.g, a.b + b.b};
}
template <class T, class S>
__device__ __forceinline__ RgbT<T> operator/(const RgbT<T>& a, const S& s)
{
    return RgbT<T>{a.r / s, a.g / s, a.b / s};
}
template <class T> __device__ __forceinline__ const T& comp(const RgbT<T>& a, int i)
{
    return i == 0 ? a.r : (i == 1 ? a.g : a.b);
}
template <class T> __device__ __forceinline__ bool positive(const RgbT<T>& a)
{
    return val(a.r) > 1e-20 && val(a.g) > 1e-20 && val(a.b) > 1e-20;  // Utils.hxx:109 isPositive
}
template <class T> __device__ __forceinline__ bool black_or_neg(const RgbT<T>& a)
{
    return val(a.r) <= 0.0 && val(a.g) <= 0.0 && val(a.b) <= 0.0;
}

struct V3d {
    double x, y, z;
};
__device__ __forceinline__ V3d v3d(V3 a) { return V3d{a.x, a.y, a.z}; }
__device__ __forceinline__ V3d v3d(float x, float y, float z) { return V3d{x, y, z}; }
__device__ __forceinline__ V3d sub(V3d a, V3d b) { return V3d{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ V3d neg(V3d a) { return V3d{-a.x, -a.y, -a.z}; }
__device__ __forceinline__ double dot(V3d a, V3d b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

// HomogeneousMedium (Scene/Media.hxx:129-159) in T.  For the medium the tangents belong to,
// sigma_t = |sigma_a| + |sigma_s| and sigma_s carry unit tangents (signs of the inputs); the
// index of the minimal attenuation component is a discrete choice and is held fixed.
template <class T>
struct MedT {
    T st[3], ss[3], g, min_st;
    double cont, mfp;
    int min_idx, has_scat;
};

template <class T>
__device__ __forceinline__ MedT<T> make_med(const upbp_medium& raw, bool seed)
{
    MedT<T> m;
    double st[3];
    for (int c = 0; c < 3; ++c) {
        const double a = fabs((double)raw.absorption[c]), s = fabs((double)raw.scattering[c]);
        st[c] = a + s;
        m.st[c] = cst<T>(st[c]);
        m.ss[c] = cst<T>(s);
    }
    double mn = st[0];
    int idx = 0;
    if (st[1] > 0 && (mn == 0 || st[1] < mn)) mn = st[1], idx = 1;
    if (st[2] > 0 && (mn == 0 || st[2] < mn)) mn = st[2], idx = 2;
    m.min_idx = idx;
    m.has_scat = (val(m.ss[0]) > 0 || val(m.ss[1]) > 0 || val(m.ss[2]) > 0) ? 1 : 0;
    const double mx = fmax(st[0], fmax(st[1], st[2]));
    m.mfp = (st[0] > 0 || st[1] > 0 || st[2] > 0) ? 1.0 / mx : INFINITY;
    m.g = cst<T>((double)raw.mean_cosine);
    m.cont = raw.continuation_prob;
    if constexpr (is_dual<T>::value) {
        if (seed) {
            for (int c = 0; c < 3; ++c) {
                const double sa = raw.absorption[c] < 0.f ? -1.0 : 1.0, ss = raw.scattering[c] < 0.f ? -1.0 : 1.0;
                m.st[c].d[c] = sa;
                m.st[c].d[3 + c] = ss;
                m.ss[c].d[3 + c] = ss;
            }
            m.g.d[6] = 1.0;
        }
    }
    m.min_st = m.st[idx];
    return m;
}

// EvalAttenuation (Media.hxx:216-229)
template <class T>
__device__ __forceinline__ RgbT<T> eval_att(const MedT<T>& m, double dist)
{
    return RgbT<T>{t_exp(m.st[0] * (-dist)), t_exp(m.st[1] * (-dist)), t_exp(m.st[2] * (-dist))};
}

// RaySamplePdf (Media.hxx:294-323)
template <class T>
__device__ __forceinline__ T ray_sample_pdf(const MedT<T>& m, double dmin, double dmax, uint32_t flags, T* rev)
{
    T pdf = cst<T>(1.0);
    *rev = cst<T>(1.0);
    if (val(m.min_st) != 0.0 && m.has_scat) {
        T att = t_exp(m.min_st * (-(dmax - dmin)));
        if (val(att) < 1e-35) att = cst<T>(1e-35);
        const T minatt = m.min_st * att;
        pdf = (flags & UPBP_END_IN_MEDIUM) ? minatt : att;
        *rev = (flags & UPBP_ORIGIN_IN_MEDIUM) ? minatt : att;
    }
    return pdf;
}

// PhaseFunction::Pdf (Path/PhaseFunction.hxx:50-80), Henyey-Greenstein in T (through g).
template <class T>
__device__ __forceinline__ T hg_pdf(V3d fix, V3d gen, const T& g, double* sin_theta)
{
    const double inv4pi = 0.25 / 3.14159265358979323846;
    const double cos_t = -dot(gen, fix);
    const double s = 1.0 - cos_t * cos_t;
    *sin_theta = sqrt(s > 0.0 ? s : 0.0);
    if (fabs(val(g)) < 1e-3) return cst<T>(inv4pi);
    const T g2 = g * g;
    const T d = (g2 + 1.0) - (g + g) * cos_t;
    if (!(val(d) > 0.0)) return cst<T>(0.0);
    return (1.0 - g2) * inv4pi / (d * t_sqrt(d));
}

// UPBP camera-walk merging terms (PathWeight.hxx:88-126) of one record; the ray-sampling fields
// that may depend on the medium are passed explicitly.
struct Factors {
    float surf, pp3d, pb2d, bb1d, sel_pdf;
    uint32_t flags;
};
__device__ __forceinline__ Factors factors_of(const upbp_mis& m)
{
    return Factors{m.surf_factor, m.pp3d_factor, m.pb2d_factor, m.bb1d_factor, m.bb1d_beam_selection_pdf, m.flags};
}

template <class T>
__device__ __forceinline__ void cam_merge(const upbp_params& P, const Factors& f, bool usable, const T& rsp_inv,
                                          const T& rsp_ratio, double sinT, const T& rayRev, const T& rayRevRatio,
                                          uint32_t tech, T& other, T& bb1d)
{
    const uint32_t qbt = P.query_beam_type, pbt = P.photon_beam_type;
    double o = 0.0;
    if ((tech & UPBP_SURF) && usable) o += (double)f.surf;
    if (tech & UPBP_PP3D) o += (double)f.pp3d;
    other = cst<T>(o);
    if (tech & UPBP_PB2D) other = other + ((qbt & UPBP_LONG_BEAM) ? rsp_inv : rsp_ratio) * (double)f.pb2d;
    bb1d = cst<T>(0.0);
    if ((tech & UPBP_BB1D) && (f.flags & UPBP_MIS_IN_MEDIUM_WITH_BEAMS)) {
        const double s = (tech & UPBP_NO_SINE_IN_WEIGHTS) ? 1.0 : sinT;
        const T& a = (qbt & UPBP_LONG_BEAM) ? rsp_inv : rsp_ratio;
        const T& b = (pbt & UPBP_LONG_BEAM) ? rayRev : rayRevRatio;
        bb1d = a * b * ((double)f.bb1d * (double)f.sel_pdf * s);
    }
}

// The candidate's camera record (index 0 of the camera walk): its factors and the fields that
// may depend on the medium.
template <class T>
struct CandT {
    Factors f;
    T pdf_a_inv, rsp_inv, ratio;
};

// camera_weight_fast (upbp_mis_prep.cuh) in T: index 0 = the candidate, index 1 = camera entry
// L-1 with the reverse ray pdf the estimator writes, the rest from the FP64 suffix sums.
template <class T>
__device__ __forceinline__ T camera_weight(const upbp_params& P, int L, const CandT<T>& cand, const T& lastRev,
                                           double lastSin, const T& lastRayRev, const T& lastRayRevRatio,
                                           const T& ntl, const upbp_mis& e, const T& e_ray_rev, const CamSum& cs,
                                           uint32_t tech)
{
    T prod = lastRev;
    T o0, b0;
    cam_merge(P, cand.f, true, cand.rsp_inv, cand.ratio, lastSin, lastRayRev, lastRayRevRatio, tech, o0, b0);
    T w_o = prod * o0, w_b = prod * b0;
    prod = prod * cand.pdf_a_inv;
    const bool next0_spec = L >= 2 ? (e.flags & UPBP_MIS_IS_SPECULAR) != 0 : (cand.f.flags & UPBP_MIS_IS_SPECULAR) != 0;
    if ((tech & UPBP_BPT) && !next0_spec) w_o = w_o + prod;
    if (L >= 2) {
        const bool espec = (e.flags & UPBP_MIS_IS_SPECULAR) != 0;
        if ((tech & UPBP_BB1D_PREVIOUS) && !espec) w_b = cst<T>(0.0);
        prod = prod * ntl * (double)e.rev_pdf_a;
        T o1, b1;
        cam_merge(P, factors_of(e), !espec, cst<T>((double)e.ray_sample_pdf_inv),
                  cst<T>((double)e.ray_sample_pdfs_ratio), (double)e.sin_theta, e_ray_rev,
                  cst<T>((double)e.ray_sample_rev_pdfs_ratio), tech, o1, b1);
        w_o = w_o + prod * o1;
        w_b = w_b + prod * b1;
        prod = prod * (double)e.pdf_a_inv;
        if ((tech & UPBP_BPT) && !espec && !(cs.flags & 2u)) w_o = w_o + prod;
        w_o = w_o + prod * cs.s_other;
        w_b = (cs.flags & 1u) ? prod * cs.s_bb1d : w_b + prod * cs.s_bb1d;
    }
    return w_o + w_b;
}

}  // namespace gen
}  // namespace upbp
