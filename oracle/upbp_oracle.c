/*
 * upbp_oracle.c -- CPU restatement of SmallUPBP's volumetric estimator stage.
 *
 * TEST INFRASTRUCTURE ONLY.  Used as the checker by tests/, by the smoke
 * check and by the CPU-baseline leg of bench.py where the reference build
 * (oracle/_ref) is absent.  Never linked into, or called by, the product.
 *
 * Parity pinned: tests/test_oracle_cpu.py checks every function here against
 * the golden fixtures in tests/golden/, which hold outputs of the reference's
 * own code (oracle/build_ref.py + oracle/ref_harness.cpp).
 *
 * Restated from (paths inside the reference project):
 *   dot / cross order            SmallUPBP/src/Structs/Vector3.hxx:513-546
 *   HomogeneousMedium            SmallUPBP/src/Scene/Media.hxx:129-159, 216-229, 294-323
 *   PhaseFunction::Pdf           SmallUPBP/src/Path/PhaseFunction.hxx:36-80
 *   AccumulateCameraPathWeight   SmallUPBP/src/Path/PathWeight.hxx:33-142
 *   AccumulateLightPathWeight    SmallUPBP/src/Path/PathWeight.hxx:145-270
 *   testIntersectionBre          SmallUPBP/src/Bre/Bre.cxx:199-223
 *   breIntersectFuncHomogeneous2 SmallUPBP/src/Bre/Bre.cxx:293-464
 *   EmbreeBre::evalBre           SmallUPBP/src/Bre/Bre.cxx:812-964
 *   testIntersectionBeamBeam     SmallUPBP/src/Beams/PhotonBeam.hxx:238-296
 *   PhotonBeam::accumulate2      SmallUPBP/src/Beams/PhotonBeam.hxx:386-607
 *   evalBeamBeamEstimate         SmallUPBP/src/Beams/PhBeams.cxx:177-324 (brute force, PhBrute.hxx:77-85)
 *   HashGrid::Build / Process    SmallUPBP/src/Misc/HashGrid.hxx:47-188
 *   UPBP::RangeQuery::Process    SmallUPBP/src/Renderers/UPBP.hxx:86-133
 *
 * Compiled with -O2 -ffp-contract=off so that float operations round like the
 * reference's SSE build (no FMA).  Candidates are enumerated by brute force.
 *
 * Two builds: ORACLE_REAL=float (liboracle.so, the FP32 restatement) and
 * ORACLE_REAL=double (liboracle64.so, the FP64 oracle).  Candidate predicates
 * are always evaluated in the reference's exact FP32 order, so both builds
 * accept the same candidates; in the FP64 build the candidate geometry
 * (distances along the rays, closest approach, sin theta) is re-solved in FP64
 * and all contribution and MIS arithmetic is FP64.
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/upbp_gpu.h"

#define PI_F 3.141592653589793238462643383279f
#define ORACLE_MAX_MEDIA 64

#ifndef ORACLE_REAL
#define ORACLE_REAL float
#endif
typedef ORACLE_REAL real;
#define IS_F64 (sizeof(real) == sizeof(double))

static real rexp(real x) { return IS_F64 ? (real)exp((double)x) : (real)expf((float)x); }
static real rsqrt(real x) { return IS_F64 ? (real)sqrt((double)x) : (real)sqrtf((float)x); }
static real rabs(real x) { return x < 0 ? -x : x; }

/* float vectors: the candidate predicates, in the reference's exact operation order */
typedef struct { float x, y, z; } v3f;
static v3f Vf(const float* p) { v3f v = {p[0], p[1], p[2]}; return v; }
static v3f subf(v3f a, v3f b) { v3f v = {a.x - b.x, a.y - b.y, a.z - b.z}; return v; }
static v3f addf(v3f a, v3f b) { v3f v = {a.x + b.x, a.y + b.y, a.z + b.z}; return v; }
static v3f scalef(v3f a, float s) { v3f v = {a.x * s, a.y * s, a.z * s}; return v; }
/* _mm_dp_ps(a, b, 0x71): (x*x' + y*y') + (z*z' + 0) */
static float dotf(v3f a, v3f b) { float xy = a.x * b.x + a.y * b.y; float z = a.z * b.z; return xy + z; }
static v3f crossf(v3f a, v3f b)
{
    v3f v = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return v;
}

/* real vectors / colours: contribution arithmetic */
typedef struct { real x, y, z; } v3;
typedef struct { real r, g, b; } rgb;
static v3 V(const float* p) { v3 v = {p[0], p[1], p[2]}; return v; }
static v3 sub(v3 a, v3 b) { v3 v = {a.x - b.x, a.y - b.y, a.z - b.z}; return v; }
static v3 neg(v3 a) { v3 v = {-a.x, -a.y, -a.z}; return v; }
static real dot(v3 a, v3 b) { real xy = a.x * b.x + a.y * b.y; real z = a.z * b.z; return xy + z; }
static v3 cross(v3 a, v3 b)
{
    v3 v = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return v;
}
static rgb C3(const float* p) { rgb c = {p[0], p[1], p[2]}; return c; }
static rgb Cr(const real* p) { rgb c = {p[0], p[1], p[2]}; return c; }
static rgb cs(real v) { rgb c = {v, v, v}; return c; }
static rgb cmul(rgb a, rgb b) { rgb c = {a.r * b.r, a.g * b.g, a.b * b.b}; return c; }
static rgb cscale(rgb a, real s) { rgb c = {a.r * s, a.g * s, a.b * s}; return c; }
static rgb cdiv(rgb a, real s) { rgb c = {a.r / s, a.g / s, a.b / s}; return c; }
static rgb cadd(rgb a, rgb b) { rgb c = {a.r + b.r, a.g + b.g, a.b + b.b}; return c; }
static real comp(rgb a, int i) { return i == 0 ? a.r : (i == 1 ? a.g : a.b); }
static int is_pos(real x) { return x > 1e-20f; }                        /* Utils.hxx:109 */

typedef struct {
    real st[3], ss[3], g, cont, min_st, mfp;
    int min_idx, has_scat;
} medium;

/* MisData with real fields (the candidate records are computed in `real`) */
typedef struct {
    real pdf_a_inv, rev_pdf_a, rev_pdf_a_without_bsdf, ray_sample_pdf_inv, ray_sample_rev_pdf_inv,
        ray_sample_pdfs_ratio, ray_sample_rev_pdfs_ratio, sin_theta, cos_theta_out, surf_factor, pp3d_factor,
        pb2d_factor, bb1d_factor, bb1d_beam_selection_pdf;
    uint32_t flags;
} rmis;

static rmis R(const upbp_mis* m)
{
    rmis r;
    r.pdf_a_inv = m->pdf_a_inv; r.rev_pdf_a = m->rev_pdf_a; r.rev_pdf_a_without_bsdf = m->rev_pdf_a_without_bsdf;
    r.ray_sample_pdf_inv = m->ray_sample_pdf_inv; r.ray_sample_rev_pdf_inv = m->ray_sample_rev_pdf_inv;
    r.ray_sample_pdfs_ratio = m->ray_sample_pdfs_ratio; r.ray_sample_rev_pdfs_ratio = m->ray_sample_rev_pdfs_ratio;
    r.sin_theta = m->sin_theta; r.cos_theta_out = m->cos_theta_out; r.surf_factor = m->surf_factor;
    r.pp3d_factor = m->pp3d_factor; r.pb2d_factor = m->pb2d_factor; r.bb1d_factor = m->bb1d_factor;
    r.bb1d_beam_selection_pdf = m->bb1d_beam_selection_pdf; r.flags = m->flags;
    return r;
}
static int c_positive(rgb a) { return is_pos(a.r) && is_pos(a.g) && is_pos(a.b); }
static int c_black_neg(rgb a) { return a.r <= 0.f && a.g <= 0.f && a.b <= 0.f; }

/* ---------------------------------------------------------------- media */
static medium make_medium(const upbp_medium* m)
{
    medium d;
    real mn;
    int c, idx = 0;
    memset(&d, 0, sizeof d);
    for (c = 0; c < 3; ++c) {
        d.ss[c] = fabsf(m->scattering[c]);
        d.st[c] = (real)fabsf(m->absorption[c]) + d.ss[c];
    }
    mn = d.st[0];
    if (d.st[1] > 0 && (mn == 0 || d.st[1] < mn)) { mn = d.st[1]; idx = 1; }
    if (d.st[2] > 0 && (mn == 0 || d.st[2] < mn)) { mn = d.st[2]; idx = 2; }
    d.min_st = mn;
    d.min_idx = idx;
    d.has_scat = d.ss[0] > 0 || d.ss[1] > 0 || d.ss[2] > 0;
    {
        real mx = d.st[0] > d.st[1] ? d.st[0] : d.st[1];
        mx = mx > d.st[2] ? mx : d.st[2];
        d.mfp = (d.st[0] > 0 || d.st[1] > 0 || d.st[2] > 0) ? (real)1 / mx : (real)INFINITY;
    }
    d.g = m->mean_cosine;
    d.cont = m->continuation_prob;
    return d;
}

static rgb eval_att(const medium* m, real dist)
{
    rgb c = {rexp(-m->st[0] * dist), rexp(-m->st[1] * dist), rexp(-m->st[2] * dist)};
    return c;
}

static real ray_sample_pdf(const medium* m, real dmin, real dmax, uint32_t flags, real* rev)
{
    real pdf = 1.f;
    *rev = 1.f;
    if (m->min_st != 0.f && m->has_scat) {
        real att = rexp(-m->min_st * (dmax - dmin));
        real minatt;
        if (att < 1e-35f) att = 1e-35f;
        minatt = m->min_st * att;
        pdf = (flags & UPBP_END_IN_MEDIUM) ? minatt : att;
        *rev = (flags & UPBP_ORIGIN_IN_MEDIUM) ? minatt : att;
    }
    return pdf;
}

static real hg_pdf(v3 fix, v3 gen, real g, real* sin_theta)
{
    const real inv4pi = IS_F64 ? (real)(0.25 / 3.14159265358979323846) : (real)((1.f / PI_F) * 0.25f);
    const real cos_t = -dot(gen, fix);
    real s = 1 - cos_t * cos_t;
    *sin_theta = rsqrt(s > 0 ? s : 0);
    if (rabs(g) < 1e-3f) return inv4pi;
    {
        const real g2 = g * g;
        const real d = 1 + g2 - (g + g) * cos_t;
        return d > 0 ? (inv4pi * (1 - g2) / (d * rsqrt(d))) : 0;
    }
}

/* ---------------------------------------------------------------- predicates */
static int test_bre(v3f o, v3f d, float tmin, float tmax, v3f p, float r2, float* t_out, float* d2_out)
{
    const v3f op = subf(p, o);
    const float t = dotf(op, d);
    if (t > tmin && t < tmax) {
        const v3f q = subf(addf(o, scalef(d, t)), p);
        const float d2 = dotf(q, q);
        if (d2 <= r2) { *t_out = t; *d2_out = d2; return 1; }
    }
    return 0;
}

static int test_beam_beam(v3f O1, v3f d1, float minT1, float maxT1, v3f O2, v3f d2, float minT2, float maxT2,
                          float maxDistSqr, float* oDist, float* oSin, float* oT1, float* oT2)
{
    const v3f c = crossf(d1, d2);
    const float sinThetaSqr = dotf(c, c);
    const float ad = dotf(subf(O2, O1), c);
    float d1d2, d1d2SqrMinus1, d1O1, d1O2, t1, t2, s;
    if (ad * ad >= maxDistSqr * sinThetaSqr) return 0;
    d1d2 = dotf(d1, d2);
    d1d2SqrMinus1 = d1d2 * d1d2 - 1.0f;
    if (d1d2SqrMinus1 < 1e-5f && d1d2SqrMinus1 > -1e-5f) return 0;
    d1O1 = dotf(d1, O1);
    d1O2 = dotf(d1, O2);
    t1 = (d1O1 - d1O2 - d1d2 * (dotf(d2, O1) - dotf(d2, O2))) / d1d2SqrMinus1;
    if (t1 <= minT1 || t1 >= maxT1) return 0;
    t2 = (t1 + d1O1 - d1O2) / d1d2;
    if (t2 <= minT2 || t2 >= maxT2 || isnan(t2)) return 0;
    s = sqrtf(sinThetaSqr);
    *oDist = fabsf(ad) / s;
    *oSin = s;
    *oT1 = t1;
    *oT2 = t2;
    return 1;
}

/* ---------------------------------------------------------------- MIS walks */
typedef struct {
    const upbp_mis* snap; /* camera snapshot (entries 0..) */
    int L;
    const rmis* cand;      /* entry L during an estimator call, or NULL (read from snapshot) */
    int prev_override;
    real prev_ray_rev_inv;
} cam_view;

static rmis cam_at(const cam_view* c, int k)
{
    rmis m;
    if (c->cand && k == c->L) return *c->cand;
    m = R(&c->snap[k]);
    if (c->prev_override && k == c->L - 1) m.ray_sample_rev_pdf_inv = c->prev_ray_rev_inv;
    return m;
}

static int spec(const rmis* m) { return (m->flags & UPBP_MIS_IS_SPECULAR) != 0; }

static real camera_path_weight(int L, real lastRev, real lastSin, real lastRayRev, real lastRayRevRatio,
                               real ntl, uint32_t qbt, uint32_t pbt, uint32_t tech, const cam_view* cam)
{
    real weight = 0, product = 1, weightBB1D = 0;
    int index;
    for (index = 0; index < L; ++index) {
        const rmis cur = cam_at(cam, L - index);
        rmis nx = index < L - 1 ? cam_at(cam, L - index - 1) : cur;
        real rev = cur.rev_pdf_a, sinT = cur.sin_theta, rayRev = cur.ray_sample_rev_pdf_inv,
              rayRevRatio = cur.ray_sample_rev_pdfs_ratio;
        int usable;
        if ((tech & UPBP_BB1D_PREVIOUS) && !spec(&cur)) weightBB1D = 0.f;
        if (index == 0) { rev = lastRev; sinT = lastSin; rayRev = lastRayRev; rayRevRatio = lastRayRevRatio; }
        else if (index == 1) rev *= ntl;
        product *= rev;
        usable = index == 0 || !spec(&cur);
        if ((tech & UPBP_SURF) && usable) weight += product * cur.surf_factor;
        if (tech & UPBP_PP3D) weight += product * cur.pp3d_factor;
        if (tech & UPBP_PB2D) {
            if (qbt & UPBP_LONG_BEAM) weight += product * cur.pb2d_factor * cur.ray_sample_pdf_inv;
            else weight += product * cur.pb2d_factor * cur.ray_sample_pdfs_ratio;
        }
        if ((tech & UPBP_BB1D) && (cur.flags & UPBP_MIS_IN_MEDIUM_WITH_BEAMS)) {
            real a, b;
            if (tech & UPBP_NO_SINE_IN_WEIGHTS) sinT = 1.f;
            a = (qbt & UPBP_LONG_BEAM) ? cur.ray_sample_pdf_inv : cur.ray_sample_pdfs_ratio;
            b = (pbt & UPBP_LONG_BEAM) ? rayRev : rayRevRatio;
            weightBB1D += product * cur.bb1d_factor * cur.bb1d_beam_selection_pdf * a * sinT * b;
        }
        product *= cur.pdf_a_inv;
        if ((tech & UPBP_BPT) && usable && !spec(&nx)) weight += product;
    }
    return weight + weightBB1D;
}

typedef struct {
    const upbp_mis* mis;
    int override_idx;
    real override_ray_rev_inv;
} light_view;

static rmis lv_at(const light_view* l, int k)
{
    rmis m = R(&l->mis[k]);
    if (k == l->override_idx) m.ray_sample_rev_pdf_inv = l->override_ray_rev_inv;
    return m;
}

static real light_path_weight(int pathIdx, int pathLength, real lastRev, real lastSin, real lastRayRev,
                              real lastRayRevRatio, real ntl, uint32_t technique, uint32_t qbt, uint32_t pbt,
                              uint32_t tech, const int32_t* pathEnds, const light_view* lv, const rmis* beam_rec)
{
    real weight = 0, product = 1;
    const int lastIndex = (pathIdx == 0) ? pathLength : pathEnds[pathIdx - 1] + pathLength;
    int index;
    for (index = 0; index <= pathLength; ++index) {
        const rmis cur = (technique == UPBP_BB1D && index == 0) ? *beam_rec : lv_at(lv, lastIndex - index);
        rmis nx = index < pathLength ? lv_at(lv, lastIndex - index - 1) : cur;
        real rev = cur.rev_pdf_a, sinT = cur.sin_theta, rayRev = cur.ray_sample_rev_pdf_inv,
              rayRevRatio = cur.ray_sample_rev_pdfs_ratio;
        int usable;
        if (index == 0) { rev = lastRev; sinT = lastSin; rayRev = lastRayRev; rayRevRatio = lastRayRevRatio; }
        else if (index == 1) rev = technique == UPBP_BB1D ? ntl : cur.rev_pdf_a_without_bsdf * ntl;
        if (rev == 0.f) break;
        product *= rev;
        usable = index == 0 || !spec(&cur);
        if (index != 0 || technique == UPBP_BPT) {
            if ((tech & UPBP_SURF) && usable) weight += product * cur.surf_factor;
            if (tech & UPBP_PP3D) weight += product * cur.pp3d_factor;
            if (tech & UPBP_PB2D) {
                if (qbt & UPBP_LONG_BEAM) weight += product * cur.pb2d_factor * rayRev;
                else weight += product * cur.pb2d_factor * rayRevRatio;
            }
            if ((tech & UPBP_BB1D) && !(tech & UPBP_BB1D_PREVIOUS) && (cur.flags & UPBP_MIS_IN_MEDIUM_WITH_BEAMS)) {
                real a, b;
                if (tech & UPBP_NO_SINE_IN_WEIGHTS) sinT = 1.f;
                a = (qbt & UPBP_LONG_BEAM) ? rayRev : rayRevRatio;
                b = (pbt & UPBP_LONG_BEAM) ? cur.ray_sample_pdf_inv : cur.ray_sample_pdfs_ratio;
                weight += product * cur.bb1d_factor * cur.bb1d_beam_selection_pdf * a * sinT * b;
            }
        }
        product *= cur.pdf_a_inv;
        if ((tech & UPBP_BPT) && usable && !spec(&nx)) weight += product;
        if (tech & UPBP_PREVIOUS) break;
    }
    return weight;
}

static uint64_t mix64(uint64_t id)
{
    uint64_t z = id + 1 + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static void fill_cand(rmis* c, const upbp_params* P, real pdf_a_inv, real rsp_inv, real ratio, real sel,
                      uint32_t flags)
{
    memset(c, 0, sizeof *c);
    c->pdf_a_inv = pdf_a_inv;
    c->rev_pdf_a = 1.f;
    c->rev_pdf_a_without_bsdf = 1.f;
    c->ray_sample_pdf_inv = rsp_inv;
    c->ray_sample_rev_pdf_inv = 1.f;
    c->ray_sample_pdfs_ratio = ratio;
    c->pp3d_factor = P->mis_factor_pp3d;
    c->pb2d_factor = P->mis_factor_pb2d;
    c->bb1d_factor = P->mis_factor_bb1d;
    c->bb1d_beam_selection_pdf = sel;
    c->flags = flags;
}

/* ---------------------------------------------------------------- oracle state */
typedef struct {
    const upbp_params* P;
    medium media[ORACLE_MAX_MEDIA];
    int n_media;
    const upbp_light_vertices* lv;
    const upbp_beams* bm;
    const upbp_mis* cam;
    int has_beams;
    float* ph_r2;      /* KNN photon radius^2 per light vertex (NULL: constant radius_pb2d) */
    float* bm_start;   /* KNN beam start radius, radius change per unit length, max radius^2 */
    float* bm_change;  /* (NULL: constant radius_bb1d) */
    float* bm_r2;
} oracle;

/* ---------------------------------------------------------------- KNN radii */
/* k-th smallest squared distance from q to the n points pts[idx[i]] (idx NULL: pts[i]).  This is
 * the dist2[1] that KdTree::KNNQuery leaves for a query with k nearest (Misc/KdTmpl.hxx:600-680):
 * the root of the max-heap of the k nearest found, each distance ((dx*dx + dy*dy) + dz*dz) in FP32
 * with d = point - query.  With n <= k the reference's value depends on its tree order; the
 * largest distance is used then. */
static float knn_d2(const float* pts, const int64_t* idx, int64_t n, const float* q, int k)
{
    float best[256];
    int nb = 0, a;
    int64_t i;
    if (k > 256) k = 256;
    for (i = 0; i < n; ++i) {
        const float* p = pts + 3 * (idx ? idx[i] : i);
        float d1 = p[0] - q[0];
        float d2 = d1 * d1;
        d1 = p[1] - q[1];
        d2 += d1 * d1;
        d1 = p[2] - q[2];
        d2 += d1 * d1;
        if (nb < k) {
            for (a = nb++; a > 0 && best[a - 1] > d2; --a) best[a] = best[a - 1];
            best[a] = d2;
        } else if (d2 < best[k - 1]) {
            for (a = k - 1; a > 0 && best[a - 1] > d2; --a) best[a] = best[a - 1];
            best[a] = d2;
        }
    }
    return nb > 0 ? best[nb - 1] : 0.f;
}

/* The reference's own search (KdTreeTmplPtr, Misc/KdTmpl.hxx), restated step for step: it is
 * approximate, and its radii are what the reference renders with.  Jensen's left-balanced kd-tree
 * in heap order (node i has children 2i and 2i+1), built by recursive median splits along the
 * longest side of the current box (BuildUp and _balanceSegment, KdTmpl.hxx:321-468) with
 * Sedgewick's in-place partition (_medianSplit, :354-383); the query walks it with an explicit
 * stack (KNNQuery, :692-760) and keeps the candidates in a max-heap that is built only once k
 * points are held (_checkAddNearest, :600-687).  Two properties make it approximate: the heap
 * bound stays at the initial radius until the heap is built, and the (k+1)-th point then replaces
 * the largest held one whatever its distance; and the descent treats nodes from n/2 - 1 on as
 * leaves, so some points are never visited.  The radius the builds use is dist2[1] afterwards:
 * the heap root, or with at most k points found the first one found. */
typedef struct {
    float p[3];
    int plane;
} kd_node;

/* _medianSplit: partition a[start..end] along `axis` so that a[median] holds its sorted value */
static void kd_split(kd_node* a, int start, int end, int median, int axis)
{
    int left = start, right = end;
    while (right > left) {
        const float v = a[right].p[axis];
        int i = left - 1, j = right;
        kd_node t;
        for (;;) {
            while (a[++i].p[axis] < v) {
            }
            while (a[--j].p[axis] > v && j > left) {
            }
            if (i >= j) break;
            t = a[i]; a[i] = a[j]; a[j] = t;
        }
        t = a[i]; a[i] = a[right]; a[right] = t;
        if (i >= median) right = i - 1;
        if (i <= median) left = i + 1;
    }
}

/* _balanceSegment: node `index` of the balanced tree from org[start..end] in the box lo..hi */
static void kd_balance(kd_node* bal, kd_node* org, int index, int start, int end, float lo[3], float hi[3])
{
    const int n = end - start + 1;
    int median = 1, axis = 2;
    while (4 * median <= n) median += median;
    if (3 * median <= n) median = median + median + start - 1;
    else median = end - median + 1;
    if (hi[0] - lo[0] > hi[1] - lo[1] && hi[0] - lo[0] > hi[2] - lo[2]) axis = 0;
    else if (hi[1] - lo[1] > hi[2] - lo[2]) axis = 1;
    kd_split(org, start, end, median, axis);
    bal[index] = org[median];
    bal[index].plane = axis;
    if (median > start) {
        if (start < median - 1) {
            const float keep = hi[axis];
            hi[axis] = bal[index].p[axis];
            kd_balance(bal, org, 2 * index, start, median - 1, lo, hi);
            hi[axis] = keep;
        } else {
            bal[2 * index] = org[start];
        }
    }
    if (median < end) {
        if (median + 1 < end) {
            const float keep = lo[axis];
            lo[axis] = bal[index].p[axis];
            kd_balance(bal, org, 2 * index + 1, median + 1, end, lo, hi);
            lo[axis] = keep;
        } else {
            bal[2 * index + 1] = org[end];
        }
    }
}

/* AddItem + BuildUp over pts[idx[i]] (idx NULL: pts[i]) in that order; returns the tree, node 1
 * the root, or NULL on allocation failure */
static kd_node* kd_build(const float* pts, const int64_t* idx, int64_t n)
{
    kd_node* org = (kd_node*)malloc(sizeof(kd_node) * (size_t)(n + 1));
    kd_node* bal = (kd_node*)malloc(sizeof(kd_node) * (size_t)(n + 1));
    float lo[3] = {1e18f, 1e18f, 1e18f}, hi[3] = {-1e18f, -1e18f, -1e18f};
    int64_t i;
    int a;
    if (!org || !bal) { free(org); free(bal); return NULL; }
    memset(org, 0, sizeof(kd_node) * (size_t)(n + 1));
    for (i = 0; i < n; ++i) {
        const float* p = pts + 3 * (idx ? idx[i] : i);
        for (a = 0; a < 3; ++a) {
            org[i + 1].p[a] = p[a];
            if (p[a] < lo[a]) lo[a] = p[a];
            if (p[a] > hi[a]) hi[a] = p[a];
        }
    }
    if (n > 1) {
        memset(bal, 0, sizeof(kd_node) * (size_t)(n + 1));
        kd_balance(bal, org, 1, 1, (int)n, lo, hi);
        free(org);
        return bal;
    }
    free(bal);
    return org;
}

/* _checkAddNearest for one node */
static void kd_add(const kd_node* p, const float* q, float* heap, int k, int* found, int* got_heap, float* maxd)
{
    float d1 = p->p[0] - q[0];
    float d2 = d1 * d1;
    d1 = p->p[1] - q[1];
    d2 += d1 * d1;
    d1 = p->p[2] - q[2];
    d2 += d1 * d1;
    if (!(d2 < heap[0])) return;
    if (*found < k) {
        heap[++*found] = d2;
        if (*maxd < d2) *maxd = d2;
        return;
    }
    if (!*got_heap) { /* heapify heap[1..found] (largest at 1) */
        const int half = *found >> 1;
        int kk;
        for (kk = half; kk >= 1; --kk) {
            int parent = kk, j;
            const float v = heap[kk];
            while (parent <= half) {
                j = parent + parent;
                if (j < *found && heap[j] < heap[j + 1]) ++j;
                if (v >= heap[j]) break;
                heap[parent] = heap[j];
                parent = j;
            }
            heap[parent] = v;
        }
        *got_heap = 1;
    }
    {   /* the root leaves, d2 sinks from the top */
        int parent = 1, j = 2;
        while (j <= *found) {
            if (j < *found && heap[j] < heap[j + 1]) ++j;
            if (d2 > heap[j]) break;
            heap[parent] = heap[j];
            parent = j;
            j += j;
        }
        heap[parent] = d2;
        heap[0] = *maxd = heap[1];
    }
}

/* KNNQuery with the initial radius sqrt(FLT_MAX) of the builds (Bre.cxx:44, PhBeams.cxx:48); returns
 * dist2[1] */
static float kd_knn_d2(const kd_node* t, int64_t n, const float* q, int k)
{
    float heap[257];
    struct { int index; float d2; } stack[64];
    const int half = (int)(n / 2 - 1);
    const float r0 = sqrtf(FLT_MAX);
    int found = 0, got_heap = 0, level = 0, index = 1, camefrom;
    float maxd = 0.0f;
    if (k > 256) k = 256;
    heap[0] = r0 * r0;
    heap[1] = 0.0f;
    if (n < 1) return 0.0f;
    for (;;) {
        while (index < half) {
            const kd_node* p = &t[index];
            const float d1 = q[p->plane] - p->p[p->plane];
            index *= 2;
            if (d1 > 0.0f) ++index;
            stack[level].index = index;
            stack[level].d2 = d1 * d1;
            ++level;
        }
        kd_add(&t[index], q, heap, k, &found, &got_heap, &maxd);
        do {
            camefrom = index;
            index /= 2;
            --level;
            if (index == 0) return heap[1];
        } while (stack[level].d2 >= heap[0] || camefrom != stack[level].index);
        kd_add(&t[index], q, heap, k, &found, &got_heap, &maxd);
        index = stack[level].index ^ 1;
        ++level;
    }
}

/* The k-NN distance the radius builds use: the reference's search, or (exact) the k-th smallest */
static float knn_dist2(const kd_node* tree, const float* pts, const int64_t* idx, int64_t n, const float* q, int k,
                       int exact)
{
    return exact ? knn_d2(pts, idx, n, q, k) : kd_knn_d2(tree, n, q, k);
}

/* Radii given from outside instead of the KNN search (tests inject the radii the reference's own
 * builds produced, so that everything but the search is compared with the reference).  Per light
 * vertex photon radius^2; per beam start and end radius.  NULL pointers: compute by KNN. */
static const float* g_ph_r2;
static const float* g_bm_start;
static const float* g_bm_end;
void upbp_oracle_set_radii(const float* ph_r2, const float* bm_start, const float* bm_end)
{
    g_ph_r2 = ph_r2;
    g_bm_start = bm_start;
    g_bm_end = bm_end;
}

/* The BB1D reach rule (not in the reference; the CUDA path defines its candidate set by it).  The
 * reference predicate's FP32 t2 = (t1 + d1.O1 - d1.O2) / (d1.d2) (PhotonBeam.hxx:290) is
 * ill-conditioned for nearly perpendicular pairs, so it accepts a few pairs whose segments do not
 * come within the radius at all: the true closest point lies beyond the beam's end.  No spatial
 * structure finds those reliably (the reference's own grid, Grid.hxx, misses them too).  With the
 * rule on, a pair that the predicate and the radius test accept is kept only if the FP64 distance
 * D of the query segment [dmin, dmax] and the beam segment [0, len] is at most r(u) + e, u being
 * the beam parameter of the closest points, r(u) the radius there and e = 2e-5 + 1e-3 r.  With
 * the rule off this is the reference's brute-force evaluator (Beams/PhBrute.hxx:77-85). */
static int g_reach = 1;
void upbp_oracle_set_reach(int on) { g_reach = on; }

static int reach_ok(v3f O1, v3f d1, float dminf, float dmaxf, v3f O2, v3f d2, float lenf, float rs, float rc,
                    float r)
{
    const double wx = (double)O1.x - O2.x, wy = (double)O1.y - O2.y, wz = (double)O1.z - O2.z;
    const double ax = d1.x, ay = d1.y, az = d1.z, bx = d2.x, by = d2.y, bz = d2.z;
    const double aa = ax * ax + ay * ay + az * az, cc = bx * bx + by * by + bz * bz, b = ax * bx + ay * by + az * bz;
    const double dd = ax * wx + ay * wy + az * wz, ee = bx * wx + by * wy + bz * wz;
    const double den = aa * cc - b * b, dmin = dminf, dmax = dmaxf, len = lenf;
    const float extra = 2e-5f + 1e-3f * r;
    double t = dmin, u = 0.0, rx, ry, rz, rho;
    int inside = 0;
    if (den > 1e-300) {
        const double inv = 1.0 / den;
        t = (b * ee - cc * dd) * inv;
        u = (aa * ee - b * dd) * inv;
        inside = t >= dmin && t <= dmax && u >= 0.0 && u <= len;
    }
    if (!inside) { /* clamp to the segments (the closest points of two segments) */
        t = fmin(fmax(t, dmin), dmax);
        u = fmin(fmax((b * t + ee) / cc, 0.0), len);
        t = fmin(fmax((b * u - dd) / aa, dmin), dmax);
        u = fmin(fmax((b * t + ee) / cc, 0.0), len);
    }
    rx = wx + t * ax - u * bx;
    ry = wy + t * ay - u * by;
    rz = wz + t * az - u * bz;
    rho = (double)rs + u * (double)rc + (double)extra;
    return rx * rx + ry * ry + rz * rz <= rho * rho;
}

/* EmbreeBre::build with KNN_RADIUS (Bre.cxx:685-725): radius = r * (2 * sqrt(d2_k)) over the
 * photons (light vertices in media); EmbreePhoton::set keeps radius * radius. */
static float* knn_photon_r2(const upbp_light_vertices* lv, float r, int k, int exact)
{
    int64_t i, n = 0;
    int64_t* idx = (int64_t*)malloc(sizeof(int64_t) * (size_t)(lv->n > 0 ? lv->n : 1));
    float* r2 = (float*)calloc((size_t)(lv->n > 0 ? lv->n : 1), sizeof(float));
    if (!idx || !r2) { free(idx); free(r2); return NULL; }
    for (i = 0; i < lv->n; ++i)
        if (lv->flags[i] & UPBP_LV_IN_MEDIUM) idx[n++] = i;
    {
        kd_node* tree = exact ? NULL : kd_build(lv->position, idx, n);
        if (!exact && !tree && n > 0) { free(idx); free(r2); return NULL; }
#pragma omp parallel for schedule(dynamic, 64)
        for (i = 0; i < n; ++i) {
            const int64_t j = idx[i];
            const float radius =
                r * (2.0f * sqrtf(knn_dist2(tree, lv->position, idx, n, lv->position + 3 * j, k, exact)));
            r2[j] = radius * radius;
        }
        free(tree);
    }
    free(idx);
    return r2;
}

/* PhotonBeamsEvaluator::build with KNN_RADIUS (PhBeams.cxx:77-123): start / end radius from the
 * k-th nearest beam origin to the beam's origin / end, max(2 * sqrt(d2_k) * r, 0.001). */
static int knn_beam_radii(const upbp_beams* bm, float r, int k, int exact, float** start, float** change, float** r2,
                          float* end_out)
{
    int64_t b;
    kd_node* tree = NULL;
    *start = (float*)malloc(sizeof(float) * (size_t)(bm->n > 0 ? bm->n : 1));
    *change = (float*)malloc(sizeof(float) * (size_t)(bm->n > 0 ? bm->n : 1));
    *r2 = (float*)malloc(sizeof(float) * (size_t)(bm->n > 0 ? bm->n : 1));
    if (!*start || !*change || !*r2) return -1;
    if (!exact && bm->n > 0 && !(tree = kd_build(bm->origin, NULL, bm->n))) return -1;
#pragma omp parallel for schedule(dynamic, 64)
    for (b = 0; b < bm->n; ++b) {
        const float* o = bm->origin + 3 * b;
        const float* d = bm->direction + 3 * b;
        const float len = bm->length[b];
        const float end[3] = {o[0] + d[0] * len, o[1] + d[1] * len, o[2] + d[2] * len};
        float rs = 2.0f * sqrtf(knn_dist2(tree, bm->origin, NULL, bm->n, o, k, exact)) * r;
        float re = 2.0f * sqrtf(knn_dist2(tree, bm->origin, NULL, bm->n, end, k, exact)) * r;
        float mx;
        rs = rs > 0.001f ? rs : 0.001f;
        re = re > 0.001f ? re : 0.001f;
        mx = rs > re ? rs : re;
        (*start)[b] = rs;
        (*r2)[b] = mx * mx;
        (*change)[b] = (re - rs) / len;
        if (end_out) end_out[b] = re;
    }
    free(tree);
    return 0;
}

typedef struct {
    v3f of, df;   /* query ray, float (predicates) */
    v3 o, d;      /* the same in `real` (contributions) */
    real dmin, dmax, rs_pdf, rs_rev;
    uint32_t rsf, ray_flags;
    int L;
    real lpw;
    const upbp_mis* snap;
} seg_ctx;

/* breIntersectFuncHomogeneous2 after testIntersectionBre accepted light vertex j (the FP64
 * build re-solves t and d2 from the inputs). */
static rgb pb2d_contrib(const oracle* O, const medium* m, const seg_ctx* s, int64_t j, real t, real d2)
{
    const upbp_params* P = O->P;
    const upbp_light_vertices* lv = O->lv;
    const int pl = (P->techniques & UPBP_NO_MIS) ? 0 : lv->path_length[j];
    rgb att, un;
    real pdf, rsp, rsr, ratio, sinT, phase, dirPdf, revPdf, r2, kernel, distSq, rspInv, last, wc, wl;
    rmis cand, lvm;
    cam_view cv;
    light_view lview;
    if (IS_F64) {
        const v3 p = V(lv->position + 3 * j);
        const v3 op = sub(p, s->o);
        v3 q;
        t = dot(op, s->d);
        q.x = s->o.x + s->d.x * t - p.x; q.y = s->o.y + s->d.y * t - p.y; q.z = s->o.z + s->d.z * t - p.z;
        d2 = dot(q, q);
    }
    if (P->techniques & UPBP_NO_MIS) {
        /* breIntersectFuncHomogeneous (Bre.cxx:239-291): VolLightTracer's pure PB2D, no rejects, no MIS:
         * flux * attenuation * sigma_s * HG * (1 - d2/r2), divided by r2 pi / 2 */
        att = eval_att(m, t - s->dmin);
        if (s->ray_flags & UPBP_SHORT_BEAM) att = cdiv(att, comp(att, m->min_idx));
        phase = hg_pdf(s->d, neg(V(lv->dir_fix + 3 * j)), m->g, &sinT);
        r2 = O->ph_r2 ? (real)O->ph_r2[j] : (real)P->radius_pb2d * P->radius_pb2d;
        un = cscale(cscale(cmul(cmul(C3(lv->throughput + 3 * j), att), Cr(m->ss)), phase), 1 - d2 / r2);
        return cdiv(un, r2 * (IS_F64 ? (real)3.14159265358979323846 : (real)PI_F) * (real)0.5);
    }
    if ((uint32_t)(pl + s->L) > P->max_path_length || (uint32_t)(pl + s->L) < P->min_path_length) return cs(0);
    if (s->L == 1 && t < P->min_dist_to_med) return cs(0);
    att = eval_att(m, t - s->dmin);
    pdf = comp(att, m->min_idx);
    if (s->ray_flags & UPBP_SHORT_BEAM) att = cdiv(att, pdf);
    rsp = m->min_st * pdf;
    rsr = (s->rsf & UPBP_ORIGIN_IN_MEDIUM) ? rsp : pdf;
    ratio = (real)1 / m->min_st;
    if (!c_positive(att)) return cs(0);
    rsp *= s->rs_pdf;
    rsr *= s->rs_rev;
    phase = hg_pdf(neg(s->d), V(lv->dir_fix + 3 * j), m->g, &sinT);
    if (phase <= 0) return cs(0);
    dirPdf = phase * m->cont;
    revPdf = phase * lv->cont_prob[j];
    r2 = O->ph_r2 ? (real)O->ph_r2[j] : (real)P->radius_pb2d * P->radius_pb2d;
    kernel = (1 - d2 / r2) / (r2 * (IS_F64 ? (real)3.14159265358979323846 : (real)PI_F) * (real)0.5);
    if (!is_pos(kernel)) return cs(0);
    un = cscale(cscale(cmul(cmul(C3(lv->throughput + 3 * j), att), Cr(m->ss)), phase), kernel);
    if (c_black_neg(un)) return cs(0);
    distSq = t * t;
    rspInv = (real)1 / rsp;
    fill_cand(&cand, P, s->lpw * distSq * rspInv, rspInv, ratio, O->has_beams ? 1 : 0,
              m->mfp > P->bb1d_min_mfp ? UPBP_MIS_IN_MEDIUM_WITH_BEAMS : 0u);
    last = (s->ray_flags & UPBP_SHORT_BEAM) ? (real)(1.0 / (double)(ratio * cand.pb2d_factor)) : rsp / cand.pb2d_factor;
    cv.snap = s->snap; cv.L = s->L; cv.cand = &cand; cv.prev_override = 1; cv.prev_ray_rev_inv = (real)1 / rsr;
    lvm = R(&lv->mis[j]);
    wc = camera_path_weight(s->L, last, sinT, lvm.ray_sample_pdf_inv, lvm.ray_sample_pdfs_ratio,
                            revPdf * rsr / distSq, P->query_beam_type, P->photon_beam_type, s->ray_flags, &cv);
    lview.mis = lv->mis; lview.override_idx = -1; lview.override_ray_rev_inv = 0;
    wl = light_path_weight(lv->path_idx[j], pl, last, 0, 0, 0, dirPdf, UPBP_PB2D, P->query_beam_type,
                           P->photon_beam_type, s->ray_flags, lv->path_ends, &lview, NULL);
    return cscale(un, (real)1 / (wl + wc));
}

/* FP64 closest approach of two lines with unit directions (the FP64 build re-solves the
 * candidate geometry that PhotonBeam::testIntersectionBeamBeam computed in FP32). */
static void closest_f64(v3 O1, v3 d1, v3 O2, v3 d2, real* dist, real* sinT, real* t1, real* t2)
{
    const double wx = (double)O1.x - O2.x, wy = (double)O1.y - O2.y, wz = (double)O1.z - O2.z;
    const double cx = (double)d1.y * d2.z - (double)d1.z * d2.y, cy = (double)d1.z * d2.x - (double)d1.x * d2.z,
                 cz = (double)d1.x * d2.y - (double)d1.y * d2.x;
    const double aa = (double)d1.x * d1.x + (double)d1.y * d1.y + (double)d1.z * d1.z;
    const double cc = (double)d2.x * d2.x + (double)d2.y * d2.y + (double)d2.z * d2.z;
    const double b = (double)d1.x * d2.x + (double)d1.y * d2.y + (double)d1.z * d2.z;
    const double dd = (double)d1.x * wx + (double)d1.y * wy + (double)d1.z * wz;
    const double ee = (double)d2.x * wx + (double)d2.y * wy + (double)d2.z * wz;
    const double den = aa * cc - b * b;
    const double s = sqrt(cx * cx + cy * cy + cz * cz);
    *t1 = (real)((b * ee - cc * dd) / den);
    *t2 = (real)((aa * ee - b * dd) / den);
    *dist = (real)(fabs(wx * cx + wy * cy + wz * cz) / s);
    *sinT = (real)s;
}

/* PhotonBeam::accumulate2 after the test and the radius check accepted beam b. */
static rgb bb1d_contrib(const oracle* O, const medium* m, const seg_ctx* s, int64_t b, real dist, real sinTheta,
                        real t1, real t2, real rstart, real rchange)
{
    real radius;
    const upbp_params* P = O->P;
    const upbp_beams* B = O->bm;
    const upbp_light_vertices* lv = O->lv;
    const int nomis = (P->techniques & UPBP_NO_MIS) != 0;
    const int lvi = nomis ? -1 : B->light_vertex[b];
    const int pl = nomis ? 0 : lv->path_length[lvi];
    const uint32_t bflags = B->flags[b], brsf = nomis ? 0u : B->ray_sampling_flags[b];
    rgb att, batt, un;
    real pfdQ, rspQ, rsrQ, ratioQ, pfdB, rspB, rsrB, ratioB, phase, sinDummy, dirPdf, revPdf, sel = 1;
    real distSqQ, rspInvQ, distSqB, rspInvB, sinT, f, last, wc, wl, ntl;
    rmis cand, brec, lvm;
    cam_view cv;
    light_view lview;
    if (IS_F64) closest_f64(s->o, s->d, V(B->origin + 3 * b), V(B->direction + 3 * b), &dist, &sinTheta, &t1, &t2);
    radius = rstart + t2 * rchange;
    if (nomis) {
        /* PhotonBeam::accumulate without MIS data (PhotonBeam.hxx:315-367): VolLightTracer's pure BB1D */
        att = eval_att(m, t1 - s->dmin);
        batt = eval_att(m, t2);
        if (s->ray_flags & UPBP_SHORT_BEAM) att = cdiv(att, comp(att, m->min_idx));
        att = cmul(att, batt);
        if (bflags & UPBP_SHORT_BEAM) att = cdiv(att, comp(batt, m->min_idx));
        phase = hg_pdf(s->d, V(B->direction + 3 * b), m->g, &sinDummy);
        return cdiv(cscale(cscale(cscale(cmul(cmul(cscale(C3(B->throughput + 3 * b), (real)1 / sel), Cr(m->ss)), att),
                                         phase),
                                  1 - dist * dist / (radius * radius)),
                           3),
                    4 * radius * sinTheta);
    }
    if ((uint32_t)(pl + 1 + s->L) > P->max_path_length || (uint32_t)(pl + 1 + s->L) < P->min_path_length) return cs(0);
    if (s->L == 1 && t1 < P->min_dist_to_med) return cs(0);
    att = eval_att(m, t1 - s->dmin);
    pfdQ = comp(att, m->min_idx);
    if (s->ray_flags & UPBP_SHORT_BEAM) att = cdiv(att, pfdQ);
    rspQ = m->min_st * pfdQ;
    rsrQ = (s->rsf & UPBP_ORIGIN_IN_MEDIUM) ? rspQ : pfdQ;
    ratioQ = (real)1 / m->min_st;
    batt = eval_att(m, t2);
    att = cmul(att, batt);
    pfdB = comp(batt, m->min_idx);
    if (bflags & UPBP_SHORT_BEAM) att = cdiv(att, pfdB);
    rspB = m->min_st * pfdB;
    rsrB = (brsf & UPBP_ORIGIN_IN_MEDIUM) ? rspB : pfdB;
    ratioB = (real)1 / m->min_st;
    if (!c_positive(att)) return cs(0);
    rspQ *= s->rs_pdf;
    rsrQ *= s->rs_rev;
    rspB *= B->ray_sample_pdf[b];
    rsrB *= B->ray_sample_rev_pdf[b];
    phase = hg_pdf(neg(s->d), neg(V(B->direction + 3 * b)), m->g, &sinDummy);
    if (phase <= 0) return cs(0);
    dirPdf = phase * m->cont;
    revPdf = phase * m->cont;
    un = cdiv(cscale(cscale(cscale(cmul(cmul(cscale(C3(B->throughput + 3 * b), (real)1 / sel), Cr(m->ss)), att), phase),
                            1 - dist * dist / (radius * radius)), 3),
              4 * radius * sinTheta);
    if (c_black_neg(un)) return cs(0);
    distSqQ = t1 * t1;
    rspInvQ = (real)1 / rspQ;
    fill_cand(&cand, P, s->lpw * distSqQ * rspInvQ, rspInvQ, ratioQ, sel, UPBP_MIS_IN_MEDIUM_WITH_BEAMS);
    distSqB = (lv->flags[lvi] & UPBP_LV_IS_FINITE) ? t2 * t2 : 1;
    rspInvB = (real)1 / rspB;
    fill_cand(&brec, P, (real)B->last_pdf_w_inv[b] * distSqB * rspInvB, rspInvB, ratioB, sel,
              UPBP_MIS_IN_MEDIUM_WITH_BEAMS);
    sinT = (s->ray_flags & UPBP_NO_SINE_IN_WEIGHTS) ? 1 : sinTheta;
    f = cand.bb1d_factor;
    if (s->ray_flags & UPBP_SHORT_BEAM)
        last = (bflags & UPBP_SHORT_BEAM) ? (real)(1.0 / (double)(ratioQ * ratioB * f * sel * sinT))
                                          : rspB / (ratioQ * f * sel * sinT);
    else
        last = (bflags & UPBP_SHORT_BEAM) ? rspQ / (ratioB * f * sel * sinT) : rspQ * rspB / (f * sel * sinT);
    cv.snap = s->snap; cv.L = s->L; cv.cand = &cand; cv.prev_override = 1; cv.prev_ray_rev_inv = (real)1 / rsrQ;
    wc = camera_path_weight(s->L, last, sinT, rspInvB, ratioB, revPdf * rsrQ / distSqQ, P->query_beam_type,
                            P->photon_beam_type, s->ray_flags, &cv);
    lvm = R(&lv->mis[lvi]);
    ntl = ((lvm.flags & UPBP_MIS_ON_LIGHT_SOURCE) && (lvm.flags & UPBP_MIS_IS_DELTA))
              ? 0 : dirPdf * rsrB * rabs(lvm.cos_theta_out) / distSqB;
    lview.mis = lv->mis; lview.override_idx = lvi; lview.override_ray_rev_inv = (real)1 / rsrB;
    wl = light_path_weight(lv->path_idx[lvi], pl + 1, last, 0, 0, 0, ntl, UPBP_BB1D, P->query_beam_type,
                           P->photon_beam_type, s->ray_flags, lv->path_ends, &lview, &brec);
    return cscale(un, (real)1 / (wl + wc));
}

/* evalBre / evalBeamBeamEstimate segment loop for one query; est = UPBP_PB2D or UPBP_BB1D. */
static rgb eval_segments(const oracle* O, const upbp_segment_queries* Q, int64_t q, uint32_t est, uint32_t* cnt,
                         uint64_t* hash)
{
    const upbp_params* P = O->P;
    const uint32_t qf = Q->flags[q];
    const int lite = (qf & UPBP_Q_LITE) != 0;
    const uint32_t qrsf = (qf & UPBP_Q_ORIGIN_IN_MEDIUM) ? UPBP_ORIGIN_IN_MEDIUM : 0u;
    const uint32_t bt = P->query_beam_type;
    rgb result = cs(0), attn = cs(1);
    real rsp = 1, rsr = 1;
    seg_ctx s;
    int i;
    s.of = Vf(Q->origin + 3 * q);
    s.df = Vf(Q->direction + 3 * q);
    s.o = V(Q->origin + 3 * q);
    s.d = V(Q->direction + 3 * q);
    s.L = Q->path_length[q];
    s.lpw = Q->last_pdf_w_inv ? Q->last_pdf_w_inv[q] : 0; /* NULL only without MIS (UPBP_NO_MIS) */
    s.ray_flags = bt | P->techniques;
    s.snap = (O->cam && Q->cam_mis_begin) ? O->cam + Q->cam_mis_begin[q] : NULL;
    for (i = 0; i < Q->seg_count[q]; ++i) {
        const int sg = Q->seg_begin[q] + i;
        const medium* m = &O->media[Q->seg_medium[sg]];
        const float dminf = Q->seg_dist_min[sg], dmaxf = Q->seg_dist_max[sg];
        const real dmin = dminf, dmax = dmaxf;
        rgb seg = cs(0);
        if (m->has_scat) {
            s.dmin = dmin;
            s.dmax = dmax;
            s.rs_pdf = rsp;
            s.rs_rev = rsr;
            s.rsf = UPBP_END_IN_MEDIUM | (i == 0 ? qrsf : 0u);
            if (est == UPBP_PB2D) {
                const upbp_light_vertices* lv = O->lv;
                const float r2c = P->radius_pb2d * P->radius_pb2d;
                int64_t j;
                for (j = 0; j < lv->n; ++j) {
                    float t, d2;
                    const float r2 = O->ph_r2 ? O->ph_r2[j] : r2c;
                    if (!(lv->flags[j] & UPBP_LV_IN_MEDIUM)) continue;
                    if (!test_bre(s.of, s.df, dminf, dmaxf, Vf(lv->position + 3 * j), r2, &t, &d2)) continue;
                    ++*cnt;
                    *hash += mix64((uint64_t)j);
                    seg = cadd(seg, pb2d_contrib(O, m, &s, j, t, d2));
                }
            } else {
                const upbp_beams* B = O->bm;
                const float rc = P->radius_bb1d, r2c = rc * rc;
                int64_t b;
                for (b = 0; b < B->n; ++b) {
                    float dist, sinT, t1, t2, radius;
                    const float rs = O->bm_start ? O->bm_start[b] : rc, rd = O->bm_change ? O->bm_change[b] : 0.f;
                    if (&O->media[B->medium_id[b]] != m) continue;
                    if (!test_beam_beam(s.of, s.df, dminf, dmaxf, Vf(B->origin + 3 * b), Vf(B->direction + 3 * b), 0.f,
                                        B->length[b], O->bm_r2 ? O->bm_r2[b] : r2c, &dist, &sinT, &t1, &t2))
                        continue;
                    radius = rs + t2 * rd; /* mStartRadius + t2 * mRadiusChange (PhotonBeam.hxx:411) */
                    if (radius < dist) continue;
                    if (g_reach && !reach_ok(s.of, s.df, dminf, dmaxf, Vf(B->origin + 3 * b), Vf(B->direction + 3 * b),
                                             B->length[b], rs, rd, P->radius_bb1d))
                        continue;
                    ++*cnt;
                    *hash += mix64((uint64_t)b);
                    seg = cadd(seg, bb1d_contrib(O, m, &s, b, dist, sinT, t1, t2, rs, rd));
                }
            }
        }
        result = cadd(result, cmul(attn, seg));
        if (lite) {
            real srev, spdf;
            attn = cmul(attn, eval_att(m, dmax - dmin));
            spdf = ray_sample_pdf(m, dmin, dmax, i == 0 ? qrsf : 0u, &srev);
            if (!c_positive(attn)) break;
            rsp *= spdf;
            rsr *= srev;
        } else {
            const rgb sa = C3(Q->seg_attenuation + 3 * sg);
            attn = cmul(attn, bt == UPBP_SHORT_BEAM ? cdiv(sa, Q->seg_pdf[sg]) : sa);
            if (!c_positive(attn)) break;
            rsp *= Q->seg_pdf[sg];
            rsr *= Q->seg_rev_pdf[sg];
        }
    }
    return result;
}

/* ---------------------------------------------------------------- PP3D hash grid */
typedef struct {
    float bmin[3], bmax[3], inv_cell, r2;
    int cells;
    int32_t* start; /* per bucket, into idx */
    int32_t* end;
    int32_t* idx;   /* light-vertex indices, bucket-sorted, stable */
} hashgrid;

static uint32_t hash_cell(int x, int y, int z, int cells)
{
    return ((uint32_t)x * 73856093u ^ (uint32_t)y * 19349663u ^ (uint32_t)z * 83492791u) % (uint32_t)cells;
}

static uint32_t point_bucket(const hashgrid* g, const float* p)
{
    const int x = (int)floorf(g->inv_cell * (p[0] - g->bmin[0]));
    const int y = (int)floorf(g->inv_cell * (p[1] - g->bmin[1]));
    const int z = (int)floorf(g->inv_cell * (p[2] - g->bmin[2]));
    return hash_cell(x, y, z, g->cells);
}

static int hashgrid_build(hashgrid* g, const upbp_light_vertices* lv, float radius, int cells)
{
    int64_t i, n = 0;
    int32_t* count;
    int c, sum = 0;
    memset(g, 0, sizeof *g);
    g->cells = cells > 0 ? cells : 1;
    g->r2 = radius * radius;
    g->inv_cell = 1.f / (radius * 2.f);
    for (c = 0; c < 3; ++c) { g->bmin[c] = 1e36f; g->bmax[c] = -1e36f; }
    for (i = 0; i < lv->n; ++i) {
        if (!(lv->flags[i] & UPBP_LV_IN_MEDIUM)) continue;
        for (c = 0; c < 3; ++c) {
            const float v = lv->position[3 * i + c];
            if (v > g->bmax[c]) g->bmax[c] = v;
            if (v < g->bmin[c]) g->bmin[c] = v;
        }
        ++n;
    }
    g->start = (int32_t*)calloc((size_t)g->cells, sizeof(int32_t));
    g->end = (int32_t*)calloc((size_t)g->cells, sizeof(int32_t));
    g->idx = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
    count = (int32_t*)calloc((size_t)g->cells, sizeof(int32_t));
    if (!g->start || !g->end || !g->idx || !count) { free(count); return -1; }
    for (i = 0; i < lv->n; ++i)
        if (lv->flags[i] & UPBP_LV_IN_MEDIUM) ++count[point_bucket(g, lv->position + 3 * i)];
    for (c = 0; c < g->cells; ++c) { g->start[c] = sum; sum += count[c]; g->end[c] = g->start[c]; }
    for (i = 0; i < lv->n; ++i)
        if (lv->flags[i] & UPBP_LV_IN_MEDIUM) {
            const uint32_t b = point_bucket(g, lv->position + 3 * i);
            g->idx[g->end[b]++] = (int32_t)i;
        }
    free(count);
    return 0;
}

static rgb pp3d_query(const oracle* O, const hashgrid* g, const upbp_point_queries* Q, int64_t q, uint32_t* cnt,
                      uint64_t* hash)
{
    const upbp_params* P = O->P;
    const upbp_light_vertices* lv = O->lv;
    rgb res = cs(0.f);
    const v3f qp = Vf(Q->position + 3 * q);
    const float qa[3] = {qp.x, qp.y, qp.z};
    const medium* m = &O->media[Q->medium_id[q]];
    const v3 cfix = V(Q->dir_fix + 3 * q);
    const int L = Q->path_length[q];
    float dmin[3], cell[3], cf[3];
    int c, j, p[3], po[3];
    cam_view cv;
    light_view lview;
    for (c = 0; c < 3; ++c) {
        dmin[c] = qa[c] - g->bmin[c];
        if (dmin[c] < 0.f || g->bmax[c] - qa[c] < 0.f) return res;
    }
    for (c = 0; c < 3; ++c) {
        cell[c] = g->inv_cell * dmin[c];
        cf[c] = floorf(cell[c]);
        p[c] = (int)cf[c];
        po[c] = p[c] + (cell[c] - cf[c] < 0.5f ? -1 : 1);
    }
    cv.snap = O->cam + Q->cam_mis_begin[q]; cv.L = L; cv.cand = NULL; cv.prev_override = 0; cv.prev_ray_rev_inv = 0;
    lview.mis = lv->mis; lview.override_idx = -1; lview.override_ray_rev_inv = 0;
    for (j = 0; j < 8; ++j) {
        const uint32_t b = hash_cell((j & 4) ? po[0] : p[0], (j & 2) ? po[1] : p[1], (j & 1) ? po[2] : p[2], g->cells);
        int k;
        for (k = g->start[b]; k < g->end[b]; ++k) {
            const int32_t i = g->idx[k];
            const v3f dd = subf(qp, Vf(lv->position + 3 * i));
            real sinT, phase, dirPdf, revPdf, mwfInv, wc, wl;
            rmis lvm;
            rgb factor;
            int pl;
            if (!(dotf(dd, dd) <= g->r2)) continue;
            ++*cnt;
            *hash += mix64((uint64_t)i);
            if (!(lv->flags[i] & UPBP_LV_CONNECTABLE)) continue;
            pl = lv->path_length[i];
            if ((uint32_t)(pl + L) > P->max_path_length || (uint32_t)(pl + L) < P->min_path_length) continue;
            if (m->ss[0] <= 0.f && m->ss[1] <= 0.f && m->ss[2] <= 0.f) continue;
            phase = hg_pdf(cfix, V(lv->dir_fix + 3 * i), m->g, &sinT);
            factor = cscale(Cr(m->ss), phase);
            if (c_black_neg(factor)) continue;
            dirPdf = phase * m->cont;
            revPdf = phase * lv->cont_prob[i];
            lvm = R(&lv->mis[i]);
            mwfInv = (real)1 / lvm.pp3d_factor;
            wc = camera_path_weight(L, mwfInv, sinT, lvm.ray_sample_pdf_inv, lvm.ray_sample_pdfs_ratio,
                                    revPdf, P->query_beam_type, P->photon_beam_type, P->techniques, &cv);
            wl = light_path_weight(lv->path_idx[i], pl, mwfInv, 0, 0, 0, dirPdf, UPBP_PP3D, P->query_beam_type,
                                   P->photon_beam_type, P->techniques, lv->path_ends, &lview, NULL);
            res = cadd(res, cscale(cmul(factor, C3(lv->throughput + 3 * i)), (real)1 / (wl + wc)));
        }
    }
    return res;
}

/* The KNN radii the oracle's builds use (params.knn_exact picks the search): photon radius^2 per
 * light vertex (0 off the media), beam start and end radius (mStartRadius, mEndRadius).  Any
 * output may be NULL. */
int upbp_oracle_knn_radii(const upbp_params* P, const upbp_light_vertices* lv, const upbp_beams* bm, float* ph_r2,
                          float* bm_start, float* bm_end)
{
    if (!P) return -1;
    if (ph_r2 && lv && P->pb2d_knn > 0) {
        float* r2 = knn_photon_r2(lv, P->radius_pb2d, P->pb2d_knn, P->knn_exact);
        if (!r2) return -1;
        memcpy(ph_r2, r2, sizeof(float) * (size_t)lv->n);
        free(r2);
    }
    if ((bm_start || bm_end) && bm && P->bb1d_knn > 0) {
        float *rs = NULL, *rc = NULL, *r2 = NULL;
        int64_t b;
        if (knn_beam_radii(bm, P->radius_bb1d, P->bb1d_knn, P->knn_exact, &rs, &rc, &r2, bm_end) != 0) return -1;
        for (b = 0; b < bm->n; ++b)
            if (bm_start) bm_start[b] = rs[b];
        free(rs); free(rc); free(r2);
    }
    return 0;
}

/* ---------------------------------------------------------------- entry point */
/*
 * Evaluate queries with index % stride == 0.  Any output pointer may be NULL.
 * image (H*W*3) is accumulated with throughput * normalisation * contribution.
 * Returns 0, or -1 on allocation failure / bad medium table.
 */
int upbp_oracle_run(const upbp_params* P, const upbp_medium* media, int32_t n_media, const upbp_light_vertices* lv,
                    const upbp_beams* bm, const upbp_mis* cam, const upbp_segment_queries* sq,
                    const upbp_point_queries* pq, int64_t stride, float* pb2d_rgb, float* bb1d_rgb, float* pp3d_rgb,
                    uint32_t* cnt_pb2d, uint64_t* hash_pb2d, uint32_t* cnt_bb1d, uint64_t* hash_bb1d,
                    uint32_t* cnt_pp3d, uint64_t* hash_pp3d, float* image)
{
    oracle O;
    hashgrid g;
    int64_t q;
    int i, have_grid = 0;
    if (!P || !media || n_media <= 0 || n_media > ORACLE_MAX_MEDIA || !lv || stride < 1) return -1;
    memset(&O, 0, sizeof O);
    O.P = P;
    O.n_media = n_media;
    for (i = 0; i < n_media; ++i) O.media[i] = make_medium(&media[i]);
    O.lv = lv;
    O.bm = bm;
    O.cam = cam;
    O.has_beams = (P->techniques & UPBP_BB1D) && bm && bm->n > 0;
    if (P->pb2d_knn > 0 && (P->techniques & UPBP_PB2D)) {
        O.ph_r2 = knn_photon_r2(lv, P->radius_pb2d, P->pb2d_knn, P->knn_exact);
        if (!O.ph_r2) return -1;
        if (g_ph_r2) memcpy(O.ph_r2, g_ph_r2, sizeof(float) * (size_t)lv->n);
    }
    if (P->bb1d_knn > 0 && O.has_beams) {
        if (knn_beam_radii(bm, P->radius_bb1d, P->bb1d_knn, P->knn_exact, &O.bm_start, &O.bm_change, &O.bm_r2, NULL) != 0)
            return -1;
        if (g_bm_start && g_bm_end) {
            int64_t b;
            for (b = 0; b < bm->n; ++b) {  /* PhBeams.cxx:117-121 from the given start / end */
                const float rs = g_bm_start[b], re = g_bm_end[b], mx = rs > re ? rs : re;
                O.bm_start[b] = rs;
                O.bm_r2[b] = mx * mx;
                O.bm_change[b] = (re - rs) / bm->length[b];
            }
        }
    }
    if (pq && pq->n > 0 && (P->techniques & UPBP_PP3D)) {
        int64_t nin = 0;
        for (q = 0; q < lv->n; ++q) nin += (lv->flags[q] & UPBP_LV_IN_MEDIUM) != 0;
        if (nin > 0) {
            if (hashgrid_build(&g, lv, P->radius_pp3d, P->hash_cells) != 0) return -1;
            have_grid = 1;
        }
    }
    if (sq) {
#pragma omp parallel for schedule(dynamic, 8)
        for (q = 0; q < sq->n; q += stride) {
            const float norm_pb = P->norm_pb2d, norm_bb = P->norm_bb1d;
            const int px = sq->pixel[q];
            const rgb thr = C3(sq->throughput + 3 * q);
            rgb v;
            uint32_t c = 0;
            uint64_t h = 0;
            int k;
            v = cs(0.f);
            if ((sq->flags[q] & UPBP_Q_PB2D) && (P->techniques & UPBP_PB2D) && lv->n > 0)
                v = eval_segments(&O, sq, q, UPBP_PB2D, &c, &h);
            if (pb2d_rgb) { pb2d_rgb[3 * q] = v.r; pb2d_rgb[3 * q + 1] = v.g; pb2d_rgb[3 * q + 2] = v.b; }
            if (cnt_pb2d) cnt_pb2d[q] = c;
            if (hash_pb2d) hash_pb2d[q] = h;
            if (image && px >= 0) {
                const rgb a = cscale(cmul(thr, cs(norm_pb)), 1.f);
                for (k = 0; k < 3; ++k) {
#pragma omp atomic
                    image[3 * px + k] += comp(a, k) * comp(v, k);
                }
            }
            c = 0;
            h = 0;
            v = cs(0.f);
            if ((sq->flags[q] & UPBP_Q_BB1D) && O.has_beams) v = eval_segments(&O, sq, q, UPBP_BB1D, &c, &h);
            if (bb1d_rgb) { bb1d_rgb[3 * q] = v.r; bb1d_rgb[3 * q + 1] = v.g; bb1d_rgb[3 * q + 2] = v.b; }
            if (cnt_bb1d) cnt_bb1d[q] = c;
            if (hash_bb1d) hash_bb1d[q] = h;
            if (image && px >= 0) {
                for (k = 0; k < 3; ++k) {
#pragma omp atomic
                    image[3 * px + k] += comp(thr, k) * norm_bb * comp(v, k);
                }
            }
        }
    }
    if (pq) {
#pragma omp parallel for schedule(dynamic, 8)
        for (q = 0; q < pq->n; q += stride) {
            rgb v = cs(0.f);
            uint32_t c = 0;
            uint64_t h = 0;
            int k;
            const int px = pq->pixel[q];
            if (have_grid) v = pp3d_query(&O, &g, pq, q, &c, &h);
            if (pp3d_rgb) { pp3d_rgb[3 * q] = v.r; pp3d_rgb[3 * q + 1] = v.g; pp3d_rgb[3 * q + 2] = v.b; }
            if (cnt_pp3d) cnt_pp3d[q] = c;
            if (hash_pp3d) hash_pp3d[q] = h;
            if (image && px >= 0)
                for (k = 0; k < 3; ++k) {
#pragma omp atomic
                    image[3 * px + k] += pq->throughput[3 * q + k] * P->norm_pp3d * comp(v, k);
                }
        }
    }
    if (have_grid) { free(g.start); free(g.end); free(g.idx); }
    free(O.ph_r2);
    free(O.bm_start);
    free(O.bm_change);
    free(O.bm_r2);
    return 0;
}

/* ---------------------------------------------------------------- B-P2D (extension) */
/*
 * Beam x point, 2-D kernel: photon beams queried at the camera medium vertices (the PP3D
 * queries).  The reference has no B-P2D estimator, so this is the definition the CUDA path is
 * checked against (parity unpinned by the reference):
 *   candidate  the beam's ray [0, len) passes within r = radius_bb1d of the point, tested with
 *              testIntersectionBre (Bre.cxx:199-223) with the beam as the ray and the query point
 *              as the photon (FP32, reference operation order), beam medium == point medium;
 *   value      beam throughput x exp(-sigma_t t) (divided by the free-flight pdf of the minimum
 *              component for SHORT beams, as accumulate2 does on the beam side) x sigma_s x
 *              HG phase(camera dir_fix, -beam dir) x (1 - d^2 / r^2) / (pi r^2 / 2);
 *   weight     1: the reference's MIS records carry no B-P2D terms, so B-P2D is a standalone
 *              estimator outside the UPBP combination;
 *   image      += camera throughput x norm_bb1d (1 / light paths) x value.
 * Point queries with index % stride == 0; any output pointer may be NULL.
 */
int upbp_oracle_bp2d(const upbp_params* P, const upbp_medium* media, int32_t n_media, const upbp_beams* bm,
                     const upbp_point_queries* pq, int64_t stride, float* bp2d_rgb, uint32_t* cnt, uint64_t* hash,
                     float* image)
{
    medium M[ORACLE_MAX_MEDIA];
    int64_t q;
    int i;
    float *bs = NULL, *bc = NULL, *br2 = NULL; /* KNN beam radii */
    if (!P || !media || n_media <= 0 || n_media > ORACLE_MAX_MEDIA || !bm || !pq || stride < 1) return -1;
    for (i = 0; i < n_media; ++i) M[i] = make_medium(&media[i]);
    if (P->bb1d_knn > 0 && (P->techniques & UPBP_BP2D) &&
        knn_beam_radii(bm, P->radius_bb1d, P->bb1d_knn, P->knn_exact, &bs, &bc, &br2, NULL))
        return -1;
#pragma omp parallel for schedule(dynamic, 8)
    for (q = 0; q < pq->n; q += stride) {
        const int px = pq->pixel[q];
        const v3f x = Vf(pq->position + 3 * q);
        const v3 cfix = V(pq->dir_fix + 3 * q);
        const int mid = pq->medium_id[q];
        const medium* m = &M[mid];
        const float r = P->radius_bb1d, r2c = r * r;
        rgb v = cs(0.f);
        uint32_t c = 0;
        uint64_t h = 0;
        int64_t b;
        int k;
        if ((P->techniques & UPBP_BP2D) && m->has_scat) {
            for (b = 0; b < bm->n; ++b) {
                float tf, d2f;
                real t, d2, pfd, phase, sinT, kernel;
                rgb att, val;
                float rt, r2;
                if (bm->medium_id[b] != mid) continue;
                /* bound: the beam's largest radius^2; then the radius at the foot point (KNN radii) */
                if (!test_bre(Vf(bm->origin + 3 * b), Vf(bm->direction + 3 * b), 0.f, bm->length[b], x,
                              br2 ? br2[b] : r2c, &tf, &d2f))
                    continue;
                rt = bs ? bs[b] + tf * bc[b] : r;
                r2 = rt * rt;
                if (bs && d2f > r2) continue;
                ++c;
                h += mix64((uint64_t)b);
                t = tf;
                d2 = d2f;
                if (IS_F64) { /* re-solve the foot point in FP64 */
                    const v3 o = V(bm->origin + 3 * b), d = V(bm->direction + 3 * b), p = V(pq->position + 3 * q);
                    v3 qv;
                    t = dot(sub(p, o), d);
                    qv.x = o.x + d.x * t - p.x; qv.y = o.y + d.y * t - p.y; qv.z = o.z + d.z * t - p.z;
                    d2 = dot(qv, qv);
                }
                att = eval_att(m, t);
                pfd = comp(att, m->min_idx);
                if (bm->flags[b] & UPBP_SHORT_BEAM) att = cdiv(att, pfd);
                if (!c_positive(att)) continue;
                phase = hg_pdf(cfix, neg(V(bm->direction + 3 * b)), m->g, &sinT);
                if (phase <= 0) continue;
                kernel = (1 - d2 / (real)r2) / ((real)r2 * (IS_F64 ? (real)3.14159265358979323846 : (real)PI_F) * (real)0.5);
                if (!is_pos(kernel)) continue;
                val = cscale(cmul(cmul(C3(bm->throughput + 3 * b), att), Cr(m->ss)), phase * kernel);
                v = cadd(v, val);
            }
        }
        if (bp2d_rgb) { bp2d_rgb[3 * q] = v.r; bp2d_rgb[3 * q + 1] = v.g; bp2d_rgb[3 * q + 2] = v.b; }
        if (cnt) cnt[q] = c;
        if (hash) hash[q] = h;
        if (image && px >= 0)
            for (k = 0; k < 3; ++k) {
#pragma omp atomic
                image[3 * px + k] += pq->throughput[3 * q + k] * P->norm_bb1d * comp(v, k);
            }
    }
    free(bs);
    free(bc);
    free(br2);
    return 0;
}
