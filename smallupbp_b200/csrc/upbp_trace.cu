// Device-side light and camera passes of one UPBP iteration, for scenes of nested axis-aligned
// boxes of homogeneous media with imaginary boundaries, an area quad light and a pinhole camera:
//   * light sub-paths: emission from the quad light (cosine-weighted), free-flight sampling in
//     each medium segment (HomogeneousMedium::SampleRay, Scene/Media.hxx:240-290), photon beams
//     (UPBP::AddBeams, Renderers/UPBP.hxx:1783-1870), light vertices with their MIS records
//     (UPBP.hxx:560-655), Henyey-Greenstein scattering (PhaseFunction::Sample,
//     Path/PhaseFunction.hxx:82-137) and Russian roulette (UPBP::SampleScattering, :1908-1969);
//   * camera sub-paths: one per pixel; each traced ray that crosses a scattering medium makes one
//     segment query (the evalBre / evalBeamBeamEstimate calls, UPBP.hxx:775-798, 879-911), each
//     camera medium vertex one PP3D point query (:1102-1118), both with the snapshot of
//     mCameraVerticesMisData at the call.
// One thread per path.  A count pass sizes every path's records, an exclusive scan places them,
// and a write pass traces the same path again (the random numbers are counter-based) and stores
// them in path order.  All arithmetic is FP64 in the operation order of the host generator
// (smallupbp_b200/workload.py); this file is compiled with -fmad=false, so no multiply-add is
// contracted, and the records agree with the generator's up to the last bit of log, exp, sin and
// cos.
#include <cub/device/device_scan.cuh>

#include <cmath>
#include <cstdint>

#include "upbp_trace.cuh"

namespace upbp {
namespace trace {

namespace {

constexpr double kInvPi = 0.3183098861837907;        // 1 / pi
constexpr double kTwoPi = 6.283185307179586;         // 2 pi
constexpr double kEpsCosine = 1e-6;
constexpr uint32_t kLightStream = 0, kCameraStream = 1;

// ------------------------------------------------------------------ random numbers
// Philox4x64-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11).
__device__ __forceinline__ void philox4x64(uint64_t c[4], uint64_t k0, uint64_t k1)
{
    const uint64_t m0 = 0xD2E7470EE14C6C93ull, m1 = 0xCA5A826395121157ull;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) {
            k0 += 0x9E3779B97F4A7C15ull;
            k1 += 0xBB67AE8584CAA73Bull;
        }
        const uint64_t hi0 = __umul64hi(m0, c[0]), lo0 = m0 * c[0];
        const uint64_t hi1 = __umul64hi(m1, c[2]), lo1 = m1 * c[2];
        const uint64_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
    }
}

// Four uniforms in [0, 1) of counter (id, bounce, block, stream).
__device__ __forceinline__ void uniforms(const TraceScene& S, uint32_t stream, uint64_t id, uint64_t bounce,
                                         uint64_t block, double u[4])
{
    uint64_t c[4] = {id, bounce, block, stream};
    philox4x64(c, S.seed, S.iteration);
#pragma unroll
    for (int i = 0; i < 4; ++i) u[i] = (double)(c[i] >> 11) * (1.0 / 9007199254740992.0);
}

__device__ __forceinline__ double np_min(double a, double b)  // np.minimum: NaN propagates
{
    return (isnan(a) || isnan(b)) ? __longlong_as_double(0x7ff8000000000000ll) : fmin(a, b);
}
__device__ __forceinline__ double np_max(double a, double b)
{
    return (isnan(a) || isnan(b)) ? __longlong_as_double(0x7ff8000000000000ll) : fmax(a, b);
}

// ------------------------------------------------------------------ ray through the boxes
// The ray split at every box face into medium segments, with one free flight sampled per
// scattering medium in order until one scatters (Scene::Intersect with imaginary boundaries).
struct Ray {
    int K;
    double start[kMaxSegments], end[kMaxSegments];  // segment k = [start, end): the break distances
    double dmax_full[kMaxSegments];                 // end of the VolumeSegment (the scattering point)
    double pdf[kMaxSegments], rev[kMaxSegments];    // free-flight pdf and reverse pdf of the segment
    double att[kMaxSegments][3];                    // transmittance over the VolumeSegment
    int med[kMaxSegments];
    bool full[kMaxSegments];  // VolumeSegment: up to the scattering point, clear segments included
    bool lite[kMaxSegments];  // LiteVolumeSegment: every scattering medium on the ray
    double scatter_t;         // +inf when the ray leaves the scene
};

__device__ int medium_at(const TraceScene& S, const double p[3])
{
    int m = 0;
    for (int b = 0; b < S.n_boxes; ++b) {
        bool inside = true;
        for (int c = 0; c < 3; ++c) inside = inside && p[c] >= S.lo[b][c] && p[c] <= S.hi[b][c];
        if (inside) m = S.box_medium[b];
    }
    return m;
}

__device__ void trace_ray(const TraceScene& S, uint32_t stream, uint64_t id, int bounce, const double o[3],
                          const double d[3], bool origin_in_medium, Ray& R)
{
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    const int K = 2 * S.n_boxes;
    R.K = K;
    double br[kMaxSegments];
    double inv[3];
    for (int c = 0; c < 3; ++c) inv[c] = 1.0 / d[c];
    for (int b = 0; b < S.n_boxes; ++b) {
        double tmin = 0.0, tmax = 0.0;
        bool have_min = false, have_max = false;  // np.nanmax / np.nanmin over the three slabs
        for (int c = 0; c < 3; ++c) {
            const double t0 = (S.lo[b][c] - o[c]) * inv[c];
            const double t1 = (S.hi[b][c] - o[c]) * inv[c];
            const double mn = np_min(t0, t1), mx = np_max(t0, t1);
            if (!isnan(mn)) {
                tmin = have_min ? fmax(tmin, mn) : mn;
                have_min = true;
            }
            if (!isnan(mx)) {
                tmax = have_max ? fmin(tmax, mx) : mx;
                have_max = true;
            }
        }
        const double nan = __longlong_as_double(0x7ff8000000000000ll);
        if (!have_min) tmin = nan;
        if (!have_max) tmax = nan;
        const bool hit = tmax >= np_max(tmin, 0.0);
        br[2 * b] = (hit && tmin > 0) ? tmin : inf;
        br[2 * b + 1] = (hit && tmax > 0) ? tmax : inf;
    }
    for (int i = 1; i < K; ++i) {  // ascending
        const double v = br[i];
        int j = i;
        for (; j > 0 && br[j - 1] > v; --j) br[j] = br[j - 1];
        br[j] = v;
    }
    double u[kMaxSegments];
    for (int blk = 0; blk < (K + 3) / 4; ++blk) {
        double w[4];
        uniforms(S, stream, id, bounce, 1 + blk, w);
        for (int i = 0; i < 4 && 4 * blk + i < K; ++i) u[4 * blk + i] = w[i];
    }
    bool alive = true;
    R.scatter_t = inf;
    for (int k = 0; k < K; ++k) {
        const double s0 = k ? br[k - 1] : 0.0, e0 = br[k];
        const bool valid = isfinite(e0) && e0 > s0;
        const double mid = valid ? 0.5 * (s0 + e0) : 0.0;
        double p[3];
        for (int c = 0; c < 3; ++c) p[c] = o[c] + d[c] * mid;
        const int m = medium_at(S, p);
        const TraceMedium& M = S.media[m];
        R.start[k] = s0;
        R.end[k] = e0;
        R.med[k] = m;
        const double seglen = valid ? e0 - s0 : 0.0;
        const double smin = M.smin;
        const bool sampled = valid && alive && M.scat && smin > 0;
        R.full[k] = valid && alive;
        R.lite[k] = valid && M.scat;
        const bool first = k == 0 && origin_in_medium;
        const double s = -log(fmax(u[k], 1e-300)) / (smin > 0 ? smin : 1.0);
        const bool hit = sampled && s < seglen;
        const bool through = sampled && !hit;
        double pdf = 1.0, rev = 1.0;
        if (hit) {
            const double a = exp(-smin * s);
            pdf = smin * a;
            rev = first ? smin * a : a;
        } else if (through) {
            const double a = exp(-smin * seglen);
            pdf = a;
            rev = first ? smin * a : a;
        }
        R.pdf[k] = pdf;
        R.rev[k] = rev;
        const double ln = hit ? s : seglen;
        for (int c = 0; c < 3; ++c) R.att[k][c] = exp(-M.st[c] * ln);
        R.dmax_full[k] = hit ? s0 + s : e0;
        if (hit) R.scatter_t = s0 + s;
        alive = alive && !hit;
    }
}

// Products of pdf, reverse pdf and transmittance over the VolumeSegments; medium of the last one.
__device__ void full_products(const Ray& R, double& rsp, double& rsr, double att[3], int& last_med)
{
    rsp = 1.0;
    rsr = 1.0;
    att[0] = att[1] = att[2] = 1.0;
    last_med = 0;
    for (int k = 0; k < R.K; ++k) {
        if (!R.full[k]) continue;
        rsp = rsp * R.pdf[k];
        rsr = rsr * R.rev[k];
        for (int c = 0; c < 3; ++c) att[c] = att[c] * R.att[k][c];
        last_med = R.med[k];
    }
}

__device__ __forceinline__ void normalize3(double v[3])
{
    const double n = sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
    for (int c = 0; c < 3; ++c) v[c] = v[c] / n;
}

// HG sampling around the propagation direction z (PhaseFunction::Sample): new direction w, pdf,
// sin theta.
__device__ void hg_sample(double u1, double u2, const double z[3], double g, double w[3], double& pdf, double& sin_t)
{
    const bool iso = fabs(g) < 1e-3;
    const double g2 = g * g, twog = g + g;
    double cos_t;
    if (iso) {
        cos_t = 1 - 2 * u1;
    } else {
        const double sq = (1 - g2) / ((1 - g) + twog * u1);
        cos_t = ((1 + g2) - sq * sq) / twog;
    }
    cos_t = fmin(fmax(cos_t, -1.0), 1.0);
    sin_t = sqrt(fmax(0.0, 1 - cos_t * cos_t));
    const double phi = kTwoPi * u2;
    const double a[3] = {fabs(z[0]) > 0.99 ? 0.0 : 1.0, fabs(z[0]) > 0.99 ? 1.0 : 0.0, 0.0};
    double x[3] = {a[1] * z[2] - a[2] * z[1], a[2] * z[0] - a[0] * z[2], a[0] * z[1] - a[1] * z[0]};
    normalize3(x);
    const double y[3] = {z[1] * x[2] - z[2] * x[1], z[2] * x[0] - z[0] * x[2], z[0] * x[1] - z[1] * x[0]};
    const double cp = cos(phi) * sin_t, sp = sin(phi) * sin_t;
    for (int c = 0; c < 3; ++c) w[c] = (x[c] * cp + y[c] * sp) + z[c] * cos_t;
    normalize3(w);
    if (iso) {
        pdf = 0.25 * kInvPi;
    } else {
        const double dd = (1 + g2) - twog * cos_t;
        pdf = ((0.25 * kInvPi) * (1 - g2)) / (dd * sqrt(fmax(dd, 1e-30)));
    }
}

__device__ __forceinline__ upbp_mis zero_mis()
{
    upbp_mis m;
    m.pdf_a_inv = m.rev_pdf_a = m.rev_pdf_a_without_bsdf = m.ray_sample_pdf_inv = m.ray_sample_rev_pdf_inv = 0.f;
    m.ray_sample_pdfs_ratio = m.ray_sample_rev_pdfs_ratio = m.sin_theta = m.cos_theta_out = m.surf_factor = 0.f;
    m.pp3d_factor = m.pb2d_factor = m.bb1d_factor = m.bb1d_beam_selection_pdf = 0.f;
    m.flags = 0;
    return m;
}

// MIS record of a vertex created by a free flight (light and camera passes alike).
__device__ __forceinline__ upbp_mis medium_vertex_mis(const TraceScene& S, double lpw, double dist2, double rsp,
                                                      int mid)
{
    upbp_mis m = zero_mis();
    m.pdf_a_inv = (float)((lpw * dist2) / rsp);
    m.rev_pdf_a = 1.f;
    m.ray_sample_pdf_inv = (float)(1.0 / rsp);
    m.ray_sample_rev_pdf_inv = 1.f;
    m.pp3d_factor = S.eta_pp3d;
    m.pb2d_factor = S.eta_pb2d;
    m.bb1d_factor = S.eta_bb1d;
    m.bb1d_beam_selection_pdf = 1.f;
    const float ratio = (float)(1.0 / S.media[mid].smin);
    m.ray_sample_pdfs_ratio = ratio;
    m.ray_sample_rev_pdfs_ratio = ratio;
    m.flags = S.media[mid].in_beams ? UPBP_MIS_IN_MEDIUM_WITH_BEAMS : 0u;
    return m;
}

__device__ __forceinline__ void store3(float* a, int64_t i, const double v[3])
{
    a[3 * i] = (float)v[0];
    a[3 * i + 1] = (float)v[1];
    a[3 * i + 2] = (float)v[2];
}

// ------------------------------------------------------------------ light pass
template <bool kWrite>
__device__ void light_path(const TraceScene& S, int p, const LightOut& O)
{
    const int v0 = kWrite ? O.v_off[p] : 0;
    const int b0 = kWrite ? O.b_off[p] : 0;
    // the write pass retraces the counted path; every store stays inside the counted records
    const int vcap = kWrite ? O.v_off[p + 1] - v0 : 0;
    const int bcap = kWrite ? O.b_off[p + 1] - b0 : 0;
    int nv = 0, nb = 0;

    double ue[4];
    uniforms(S, kLightStream, (uint64_t)p, 0, 0, ue);
    const double half = S.light_size * 0.5, area = S.light_size * S.light_size;
    const double cx = 0.5 * (S.lo[0][0] + S.hi[0][0]), cz = 0.5 * (S.lo[0][2] + S.hi[0][2]);
    double o[3] = {(cx - half) + S.light_size * ue[0], S.hi[0][1], (cz - half) + S.light_size * ue[1]};
    const double u1 = ue[2], u2 = ue[3];
    const double r = sqrt(u1), phi = kTwoPi * u2;
    const double cos_l = fmax(sqrt(fmax(0.0, 1 - u1)), kEpsCosine);
    double d[3] = {r * cos(phi), -cos_l, r * sin(phi)};
    normalize3(d);
    const double emission_pdf_w = (cos_l * kInvPi) / area;
    const double direct_pdf_a = 1.0 / area;
    double thr[3];
    for (int c = 0; c < 3; ++c) thr[c] = (S.light_intensity * cos_l) / emission_pdf_w;
    double lpw = direct_pdf_a / emission_pdf_w;

    // vertex 0: on the light source
    upbp_mis prev = zero_mis();
    prev.pdf_a_inv = (float)(1.0 / direct_pdf_a);
    prev.rev_pdf_a = (float)cos_l;
    prev.rev_pdf_a_without_bsdf = (float)cos_l;
    prev.ray_sample_rev_pdf_inv = 1.f;
    prev.cos_theta_out = (float)cos_l;
    prev.flags = UPBP_MIS_ON_LIGHT_SOURCE;
    if (kWrite && vcap < 1) {
        atomicOr(O.status, 1);
        return;
    }
    if (kWrite) {
        const int64_t i = v0;
        store3(O.pos, i, o);
        const double one[3] = {1.0, 1.0, 1.0}, zero[3] = {0.0, 0.0, 0.0};
        store3(O.thr, i, one);
        store3(O.dir, i, zero);
        O.cont[i] = 1.f;
        O.pidx[i] = p;
        O.plen[i] = 0;
        O.med[i] = -1;
        O.flags[i] = UPBP_LV_IS_FINITE;
        O.mis[i] = prev;
    }
    nv = 1;
    bool oim = false;
    Ray R;
    for (int L = 1; S.max_path_length > 1; ++L) {
        trace_ray(S, kLightStream, (uint64_t)p, L, o, d, oim, R);
        // photon beams of this ray (UPBP::AddBeams)
        double t3[3] = {thr[0], thr[1], thr[2]};
        double rsp = 1.0, rsr = 1.0;
        int last_beam = -1;
        double last_len = 0.0;
        int last_med = 0;
        const bool is_long = S.photon_beam_type == UPBP_LONG_BEAM;
        int first_lite = 0;
        if (is_long)
            for (int k = R.K - 1; k >= 0; --k)
                if (R.lite[k]) first_lite = k;
        for (int k = 0; k < R.K; ++k) {
            const int mk = R.med[k];
            const TraceMedium& M = S.media[mk];
            const bool f = is_long ? R.lite[k] : R.full[k];
            const bool ok = f && M.beams_ok;
            const double len = is_long ? R.end[k] - R.start[k] : R.dmax_full[k] - R.start[k];
            const bool isfirst = is_long ? (first_lite == k && oim) : (k == 0 && oim);
            if (ok) {
                if (kWrite && nb >= bcap) {
                    atomicOr(O.status, 1);
                    return;
                }
                if (kWrite) {
                    const int64_t j = b0 + nb;
                    const double org[3] = {o[0] + d[0] * R.start[k], o[1] + d[1] * R.start[k],
                                           o[2] + d[2] * R.start[k]};
                    store3(O.b_origin, j, org);
                    store3(O.b_dir, j, d);
                    O.b_len[j] = (float)len;
                    store3(O.b_thr, j, t3);
                    O.b_flags[j] = is_long ? UPBP_LONG_BEAM : UPBP_SHORT_BEAM;
                    O.b_rsp[j] = (float)rsp;
                    O.b_rsr[j] = (float)rsr;
                    O.b_rsf[j] = UPBP_END_IN_MEDIUM | (isfirst ? UPBP_ORIGIN_IN_MEDIUM : 0u);
                    O.b_lpw[j] = (float)lpw;
                    O.b_med[j] = mk;
                    O.b_lv[j] = v0 + L - 1;
                }
                last_beam = nb;
                last_len = len;
                last_med = mk;
                ++nb;
            }
            if (is_long) {
                if (f) {
                    for (int c = 0; c < 3; ++c) t3[c] = t3[c] * exp(-M.st[c] * len);
                    const double a1 = fmax(exp(-M.smin * len), 1e-35);
                    if (M.smin > 0 && M.scat) {
                        rsp = rsp * a1;
                        rsr = rsr * (isfirst ? M.smin * a1 : a1);
                    }
                }
            } else if (f) {
                for (int c = 0; c < 3; ++c) t3[c] = (t3[c] * R.att[k][c]) / R.pdf[k];
                rsp = rsp * R.pdf[k];
                rsr = rsr * R.rev[k];
            }
        }
        if (is_long && last_beam >= 0 && kWrite) {  // the ray's last beam is capped (UPBP.hxx:1867-1868)
            const double cap = fmin(S.media[last_med].maxlen, S.beam_length_cap);
            O.b_len[b0 + last_beam] = (float)fmin(last_len, cap);
        }
        // scattering vertex (UPBP.hxx:560-655)
        if (!isfinite(R.scatter_t)) break;
        double rsp_s, rsr_s, att_s[3];
        int mid;
        full_products(R, rsp_s, rsr_s, att_s, mid);
        double nthr[3];
        for (int c = 0; c < 3; ++c) nthr[c] = (thr[c] * att_s[c]) / rsp_s;
        if (!(nthr[0] > 0 || nthr[1] > 0 || nthr[2] > 0)) break;
        for (int c = 0; c < 3; ++c) thr[c] = nthr[c];
        const double st = R.scatter_t;
        const double hit[3] = {o[0] + d[0] * st, o[1] + d[1] * st, o[2] + d[2] * st};
        const double dist2 = st * st;
        upbp_mis cur = medium_vertex_mis(S, lpw, dist2, rsp_s, mid);
        cur.rev_pdf_a_without_bsdf = 1.f;
        prev.rev_pdf_a = (float)(((double)prev.rev_pdf_a * rsr_s) / dist2);
        prev.rev_pdf_a_without_bsdf = prev.rev_pdf_a;
        prev.ray_sample_rev_pdf_inv = (float)(1.0 / rsr_s);
        const int64_t vi = v0 + nv;
        if (kWrite && nv >= vcap) {
            atomicOr(O.status, 1);
            return;
        }
        if (kWrite) {
            O.mis[vi - 1] = prev;
            store3(O.pos, vi, hit);
            store3(O.thr, vi, nthr);
            const double fix[3] = {-d[0], -d[1], -d[2]};
            store3(O.dir, vi, fix);
            O.cont[vi] = (float)S.media[mid].cont;
            O.pidx[vi] = p;
            O.plen[vi] = L;
            O.med[vi] = mid;
            O.flags[vi] = UPBP_LV_IN_MEDIUM | UPBP_LV_CONNECTABLE | UPBP_LV_IS_FINITE;
            O.mis[vi] = cur;
        }
        ++nv;
        for (int c = 0; c < 3; ++c) o[c] = hit[c];
        oim = true;
        if (!(L + 2 <= S.max_path_length)) break;
        // UPBP::SampleScattering: HG direction, Russian roulette
        double us[4];
        uniforms(S, kLightStream, (uint64_t)p, L, 0, us);
        double wnew[3], pdfw, sin_t;
        hg_sample(us[0], us[1], d, S.media[mid].g, wnew, pdfw, sin_t);
        const double cont = S.media[mid].cont;
        if (cont == 0 || (cont < 1 && us[2] > cont)) break;
        const double dir_pdf = pdfw * cont;
        for (int c = 0; c < 3; ++c) thr[c] = (thr[c] * S.media[mid].ss[c]) * (pdfw / dir_pdf);
        lpw = 1.0 / dir_pdf;
        cur.rev_pdf_a_without_bsdf = cur.rev_pdf_a;
        cur.sin_theta = (float)sin_t;
        cur.cos_theta_out = 1.f;
        prev.rev_pdf_a = (float)((double)prev.rev_pdf_a * dir_pdf);  // HG is symmetric
        if (kWrite) {
            O.mis[vi - 1] = prev;
            O.mis[vi] = cur;
        }
        prev = cur;
        for (int c = 0; c < 3; ++c) d[c] = wnew[c];
    }
    if (kWrite) {
        if (nv != vcap || nb != bcap) atomicOr(O.status, 1);
        O.path_ends[p] = v0 + nv;
    } else {
        O.v_count[p] = nv;
        O.b_count[p] = nb;
    }
}

__global__ void __launch_bounds__(128) k_light(const TraceScene S, const LightOut O, int write)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= S.light_paths) return;
    if (write) light_path<true>(S, p, O);
    else light_path<false>(S, p, O);
}

// ------------------------------------------------------------------ camera pass
template <bool kWrite>
__device__ void camera_path(const TraceScene& S, int pix, const CameraOut& O)
{
    int nq = 0, ns = 0, np = 0, nc = 0;
    const int q0 = kWrite ? O.q_off[pix] : 0, s0 = kWrite ? O.s_off[pix] : 0, p0 = kWrite ? O.p_off[pix] : 0;
    const int64_t c0 = kWrite ? (int64_t)O.c_off[pix] : 0;
    const int qcap = kWrite ? O.q_off[pix + 1] - q0 : 0, scap = kWrite ? O.s_off[pix + 1] - s0 : 0;
    const int pcap = kWrite ? O.p_off[pix + 1] - p0 : 0, ccap = kWrite ? O.c_off[pix + 1] - (int)c0 : 0;
    const int W = S.width, H = S.height;
    const int maxL = S.max_path_length;
    double uj[4];
    uniforms(S, kCameraStream, (uint64_t)pix, 0, 0, uj);
    const double sx = ((double)(pix % W) + uj[0]) - W * 0.5;
    const double sy = ((double)(pix / W) + uj[1]) - H * 0.5;
    double d[3] = {sx, -sy, S.ipd};
    normalize3(d);
    const double cos_cam = d[2];
    const double tt = S.ipd / cos_cam;
    const double cam_pdf_w = (tt * tt) / cos_cam;
    double o[3] = {S.cam[0], S.cam[1], S.cam[2]};
    double thr[3] = {1.0, 1.0, 1.0};
    double lpw = (double)(W * H) / cam_pdf_w;
    bool oim = false, stop_bb1d = false;
    upbp_mis table[kMaxTracePath + 1];
    for (int i = 0; i <= maxL; ++i) table[i] = zero_mis();
    table[0].rev_pdf_a = 1.f;
    Ray R;
    for (int L = 1;; ++L) {
        trace_ray(S, kCameraStream, (uint64_t)pix, L, o, d, oim, R);
        const bool scattered = isfinite(R.scatter_t);
        const bool use_lite = scattered && S.query_beam_type == UPBP_LONG_BEAM;
        bool has_med = false;
        int cnt = 0;
        for (int k = 0; k < R.K; ++k) {
            const bool sm = use_lite ? R.lite[k] : R.full[k];
            cnt += sm;
            has_med = has_med || (sm && S.media[R.med[k]].scat);
        }
        if (has_med) {
            if (kWrite && (nq >= qcap || ns + cnt > scap || nc + L > ccap)) {
                atomicOr(O.status, 1);
                return;
            }
            uint32_t qf = (oim ? UPBP_Q_ORIGIN_IN_MEDIUM : 0u) | (use_lite ? UPBP_Q_LITE : 0u);
            if (S.techniques & UPBP_PB2D) qf |= UPBP_Q_PB2D;
            if ((S.techniques & UPBP_BB1D) && !stop_bb1d) qf |= UPBP_Q_BB1D;
            if (kWrite) {
                const int64_t qi = q0 + nq;
                store3(O.sq_origin, qi, o);
                store3(O.sq_dir, qi, d);
                O.sq_seg_begin[qi] = s0 + ns;
                O.sq_seg_count[qi] = cnt;
                O.sq_flags[qi] = qf;
                O.sq_plen[qi] = L;
                O.sq_lpw[qi] = (float)lpw;
                store3(O.sq_thr, qi, thr);
                O.sq_pixel[qi] = pix;
                O.sq_cam_begin[qi] = c0 + nc;
                int j = s0 + ns;
                for (int k = 0; k < R.K; ++k) {
                    if (!(use_lite ? R.lite[k] : R.full[k])) continue;
                    O.seg_dmin[j] = (float)R.start[k];
                    O.seg_dmax[j] = (float)(use_lite ? R.end[k] : R.dmax_full[k]);
                    O.seg_pdf[j] = (float)(use_lite ? 1.0 : R.pdf[k]);
                    O.seg_rev[j] = (float)(use_lite ? 1.0 : R.rev[k]);
                    const double one[3] = {1.0, 1.0, 1.0};
                    store3(O.seg_att, j, use_lite ? one : R.att[k]);
                    O.seg_med[j] = R.med[k];
                    ++j;
                }
                for (int i = 0; i < L; ++i) O.cam[c0 + nc + i] = table[i];
            }
            ++nq;
            ns += cnt;
            nc += L;
        }
        if (!scattered) break;
        double rsp, rsr, att[3];
        int mid;
        full_products(R, rsp, rsr, att, mid);
        double nthr[3];
        for (int c = 0; c < 3; ++c) nthr[c] = (thr[c] * att[c]) / rsp;
        if (!(nthr[0] > 0 || nthr[1] > 0 || nthr[2] > 0)) break;
        for (int c = 0; c < 3; ++c) thr[c] = nthr[c];
        const double st = R.scatter_t;
        const double hit[3] = {o[0] + d[0] * st, o[1] + d[1] * st, o[2] + d[2] * st};
        const double dist2 = st * st;
        table[L] = medium_vertex_mis(S, lpw, dist2, rsp, mid);
        table[L - 1].rev_pdf_a = (float)(((double)table[L - 1].rev_pdf_a * rsr) / dist2);
        table[L - 1].ray_sample_rev_pdf_inv = (float)(1.0 / rsr);
        if (L >= maxL) break;
        if ((S.techniques & UPBP_PP3D) && (L > 1 || st >= S.min_dist_to_med)) {
            if (kWrite && (np >= pcap || nc + L + 1 > ccap)) {
                atomicOr(O.status, 1);
                return;
            }
            if (kWrite) {
                const int64_t pi = p0 + np;
                store3(O.pq_pos, pi, hit);
                const double fix[3] = {-d[0], -d[1], -d[2]};
                store3(O.pq_dir, pi, fix);
                O.pq_med[pi] = mid;
                O.pq_plen[pi] = L;
                store3(O.pq_thr, pi, nthr);
                O.pq_pixel[pi] = pix;
                O.pq_cam_begin[pi] = c0 + nc;
                for (int i = 0; i <= L; ++i) O.cam[c0 + nc + i] = table[i];
            }
            ++np;
            nc += L + 1;
        }
        double us[4];
        uniforms(S, kCameraStream, (uint64_t)pix, L, 0, us);
        double wnew[3], pdfw, sin_t;
        hg_sample(us[0], us[1], d, S.media[mid].g, wnew, pdfw, sin_t);
        const double cont = S.media[mid].cont;
        if (cont == 0 || (cont < 1 && us[2] > cont)) break;
        const double dir_pdf = pdfw * cont;
        for (int c = 0; c < 3; ++c) thr[c] = (thr[c] * S.media[mid].ss[c]) * (pdfw / dir_pdf);
        table[L].sin_theta = (float)sin_t;
        table[L].cos_theta_out = 1.f;
        table[L - 1].rev_pdf_a = (float)((double)table[L - 1].rev_pdf_a * dir_pdf);
        if (S.techniques & UPBP_BB1D_PREVIOUS) stop_bb1d = true;
        lpw = 1.0 / dir_pdf;
        for (int c = 0; c < 3; ++c) {
            o[c] = hit[c];
            d[c] = wnew[c];
        }
        oim = true;
    }
    if (kWrite && (nq != qcap || ns != scap || np != pcap || nc != ccap)) atomicOr(O.status, 1);
    if (!kWrite) {
        O.q_count[pix] = nq;
        O.s_count[pix] = ns;
        O.p_count[pix] = np;
        O.c_count[pix] = nc;
    }
}

__global__ void __launch_bounds__(128) k_camera(const TraceScene S, const CameraOut O, int write)
{
    const int pix = blockIdx.x * blockDim.x + threadIdx.x;
    if (pix >= S.width * S.height) return;
    if (write) camera_path<true>(S, pix, O);
    else camera_path<false>(S, pix, O);
}

}  // namespace

const char* make_scene(const upbp_scene& in, const upbp_params& P, uint32_t iteration, TraceScene* out)
{
    TraceScene& S = *out;
    S = TraceScene{};
    if (in.n_media < 1 || in.n_media > UPBP_SCENE_MAX_MEDIA) return "n_media out of range";
    if (in.n_boxes < 1 || in.n_boxes > UPBP_MAX_BOXES) return "n_boxes out of range";
    if (in.width < 1 || in.height < 1 || (int64_t)in.width * in.height > (int64_t)1 << 28) return "bad image size";
    if (in.light_paths < 0) return "negative light_paths";
    if (in.max_path_length < 1 || in.max_path_length > kMaxTracePath) return "max_path_length out of range";
    if (in.width != P.image_width || in.height != P.image_height) return "image size differs from the params";
    if ((uint32_t)in.max_path_length != P.max_path_length) return "max_path_length differs from the params";
    if (in.techniques != P.techniques) return "techniques differ from the params";
    if (!(in.fov_deg > 0 && in.fov_deg < 180)) return "fov_deg out of range";
    const bool merge_pb2d = (in.techniques & UPBP_PB2D) != 0;
    for (int m = 0; m < in.n_media; ++m) {
        const upbp_scene_medium& a = in.media[m];
        TraceMedium& M = S.media[m];
        double mx = 0.0;
        M.scat = 0;
        for (int c = 0; c < 3; ++c) {
            M.st[c] = a.absorption[c] + a.scattering[c];
            M.ss[c] = a.scattering[c];
            mx = c ? std::fmax(mx, M.st[c]) : M.st[c];
            M.scat |= a.scattering[c] > 0;
        }
        double best = M.st[0];  // smallest positive component (HomogeneousMedium ctor, Media.hxx:142-145)
        for (int c = 1; c < 3; ++c)
            if (M.st[c] > 0 && (best == 0 || M.st[c] < best)) best = M.st[c];
        M.smin = best;
        M.mfp = mx > 0 ? 1.0 / mx : INFINITY;
        M.maxlen = mx > 0 ? -std::log(1e-9) / mx : INFINITY;
        M.g = a.mean_cosine;
        M.cont = a.continuation_prob;
        M.beams_ok = M.scat && (!merge_pb2d || M.mfp > in.bb1d_min_mfp);
        M.in_beams = !merge_pb2d || M.mfp > in.bb1d_min_mfp;
    }
    S.n_boxes = in.n_boxes;
    for (int b = 0; b < in.n_boxes; ++b) {
        if (in.box_medium[b] < 0 || in.box_medium[b] >= in.n_media) return "box_medium out of range";
        S.box_medium[b] = in.box_medium[b];
        for (int c = 0; c < 3; ++c) {
            S.lo[b][c] = in.box_lo[b][c];
            S.hi[b][c] = in.box_hi[b][c];
        }
    }
    for (int c = 0; c < 3; ++c) S.cam[c] = in.camera_pos[c];
    const double deg_to_rad = M_PI / 180.0;
    S.ipd = in.width / (2.0 * std::tan(in.fov_deg * deg_to_rad * 0.5));
    S.width = in.width;
    S.height = in.height;
    S.light_paths = in.light_paths;
    S.max_path_length = in.max_path_length;
    S.light_size = in.light_size;
    S.light_intensity = in.light_intensity;
    S.techniques = in.techniques;
    S.query_beam_type = in.query_beam_type;
    S.photon_beam_type = in.photon_beam_type;
    S.beam_length_cap = in.beam_length_cap;
    S.min_dist_to_med = in.min_dist_to_med;
    S.eta_pp3d = P.mis_factor_pp3d;
    S.eta_pb2d = P.mis_factor_pb2d;
    S.eta_bb1d = P.mis_factor_bb1d;
    S.seed = in.seed;
    S.iteration = iteration;
    return nullptr;
}

void launch_light(const TraceScene& S, bool write, const LightOut& O, cudaStream_t s)
{
    if (S.light_paths > 0) k_light<<<(S.light_paths + 127) / 128, 128, 0, s>>>(S, O, write ? 1 : 0);
}

void launch_camera(const TraceScene& S, bool write, const CameraOut& O, cudaStream_t s)
{
    const int n = S.width * S.height;
    if (n > 0) k_camera<<<(n + 127) / 128, 128, 0, s>>>(S, O, write ? 1 : 0);
}

size_t scan_temp_bytes(int n)
{
    size_t b = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b, (const int*)nullptr, (int*)nullptr, n);
    return b;
}

void exclusive_scan(const int* in, int* out, int n, void* tmp, size_t tmp_bytes, cudaStream_t s)
{
    cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, in, out, n, s);
}

}  // namespace trace
}  // namespace upbp
