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
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/upbp_gpu.h"

#define PI_F 3.141592653589793238462643383279f
#define ORACLE_MAX_MEDIA 64

typedef struct { float x, y, z; } v3;
typedef struct { float r, g, b; } rgb;

typedef struct {
    float st[3], ss[3], g, cont, min_st, mfp;
    int min_idx, has_scat;
} medium;

/* ---------------------------------------------------------------- vectors */
static v3 V(const float* p) { v3 v = {p[0], p[1], p[2]}; return v; }
static v3 sub(v3 a, v3 b) { v3 v = {a.x - b.x, a.y - b.y, a.z - b.z}; return v; }
static v3 add(v3 a, v3 b) { v3 v = {a.x + b.x, a.y + b.y, a.z + b.z}; return v; }
static v3 scale(v3 a, float s) { v3 v = {a.x * s, a.y * s, a.z * s}; return v; }
static v3 neg(v3 a) { v3 v = {-a.x, -a.y, -a.z}; return v; }
/* _mm_dp_ps(a, b, 0x71): (x*x' + y*y') + (z*z' + 0) */
static float dot(v3 a, v3 b) { float xy = a.x * b.x + a.y * b.y; float z = a.z * b.z; return xy + z; }
static v3 cross(v3 a, v3 b)
{
    v3 v = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return v;
}
static rgb C3(const float* p) { rgb c = {p[0], p[1], p[2]}; return c; }
static rgb cs(float v) { rgb c = {v, v, v}; return c; }
static rgb cmul(rgb a, rgb b) { rgb c = {a.r * b.r, a.g * b.g, a.b * b.b}; return c; }
static rgb cscale(rgb a, float s) { rgb c = {a.r * s, a.g * s, a.b * s}; return c; }
static rgb cdiv(rgb a, float s) { rgb c = {a.r / s, a.g / s, a.b / s}; return c; }
static rgb cadd(rgb a, rgb b) { rgb c = {a.r + b.r, a.g + b.g, a.b + b.b}; return c; }
static float comp(rgb a, int i) { return i == 0 ? a.r : (i == 1 ? a.g : a.b); }
static int is_pos(float x) { return x > 1e-20f; }                       /* Utils.hxx:109 */
static int c_positive(rgb a) { return is_pos(a.r) && is_pos(a.g) && is_pos(a.b); }
static int c_black_neg(rgb a) { return a.r <= 0.f && a.g <= 0.f && a.b <= 0.f; }

/* ---------------------------------------------------------------- media */
static medium make_medium(const upbp_medium* m)
{
    medium d;
    float mn;
    int c, idx = 0;
    memset(&d, 0, sizeof d);
    for (c = 0; c < 3; ++c) {
        d.ss[c] = fabsf(m->scattering[c]);
        d.st[c] = fabsf(m->absorption[c]) + d.ss[c];
    }
    mn = d.st[0];
    if (d.st[1] > 0 && (mn == 0 || d.st[1] < mn)) { mn = d.st[1]; idx = 1; }
    if (d.st[2] > 0 && (mn == 0 || d.st[2] < mn)) { mn = d.st[2]; idx = 2; }
    d.min_st = mn;
    d.min_idx = idx;
    d.has_scat = d.ss[0] > 0 || d.ss[1] > 0 || d.ss[2] > 0;
    {
        float mx = d.st[0] > d.st[1] ? d.st[0] : d.st[1];
        mx = mx > d.st[2] ? mx : d.st[2];
        d.mfp = (d.st[0] > 0 || d.st[1] > 0 || d.st[2] > 0) ? 1.0f / mx : INFINITY;
    }
    d.g = m->mean_cosine;
    d.cont = m->continuation_prob;
    return d;
}

static rgb eval_att(const medium* m, float dist)
{
    rgb c = {expf(-m->st[0] * dist), expf(-m->st[1] * dist), expf(-m->st[2] * dist)};
    return c;
}

static float ray_sample_pdf(const medium* m, float dmin, float dmax, uint32_t flags, float* rev)
{
    float pdf = 1.f;
    *rev = 1.f;
    if (m->min_st != 0.f && m->has_scat) {
        float att = expf(-m->min_st * (dmax - dmin));
        float minatt;
        if (att < 1e-35f) att = 1e-35f;
        minatt = m->min_st * att;
        pdf = (flags & UPBP_END_IN_MEDIUM) ? minatt : att;
        *rev = (flags & UPBP_ORIGIN_IN_MEDIUM) ? minatt : att;
    }
    return pdf;
}

static float hg_pdf(v3 fix, v3 gen, float g, float* sin_theta)
{
    const float inv4pi = (1.f / PI_F) * 0.25f;
    const float cos_t = -dot(gen, fix);
    float s = 1.f - cos_t * cos_t;
    *sin_theta = sqrtf(s > 0.f ? s : 0.f);
    if (fabsf(g) < 1e-3f) return inv4pi;
    {
        const float g2 = g * g;
        const float d = 1.f + g2 - (g + g) * cos_t;
        return d > 0.f ? (inv4pi * (1.f - g2) / (d * sqrtf(d))) : 0.f;
    }
}

/* ---------------------------------------------------------------- predicates */
static int test_bre(v3 o, v3 d, float tmin, float tmax, v3 p, float r2, float* t_out, float* d2_out)
{
    const v3 op = sub(p, o);
    const float t = dot(op, d);
    if (t > tmin && t < tmax) {
        const v3 q = sub(add(o, scale(d, t)), p);
        const float d2 = dot(q, q);
        if (d2 <= r2) { *t_out = t; *d2_out = d2; return 1; }
    }
    return 0;
}

static int test_beam_beam(v3 O1, v3 d1, float minT1, float maxT1, v3 O2, v3 d2, float minT2, float maxT2,
                          float maxDistSqr, float* oDist, float* oSin, float* oT1, float* oT2)
{
    const v3 c = cross(d1, d2);
    const float sinThetaSqr = dot(c, c);
    const float ad = dot(sub(O2, O1), c);
    float d1d2, d1d2SqrMinus1, d1O1, d1O2, t1, t2, s;
    if (ad * ad >= maxDistSqr * sinThetaSqr) return 0;
    d1d2 = dot(d1, d2);
    d1d2SqrMinus1 = d1d2 * d1d2 - 1.0f;
    if (d1d2SqrMinus1 < 1e-5f && d1d2SqrMinus1 > -1e-5f) return 0;
    d1O1 = dot(d1, O1);
    d1O2 = dot(d1, O2);
    t1 = (d1O1 - d1O2 - d1d2 * (dot(d2, O1) - dot(d2, O2))) / d1d2SqrMinus1;
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
    const upbp_mis* cand; /* entry L during an estimator call, or NULL (read from snapshot) */
    int prev_override;
    float prev_ray_rev_inv;
} cam_view;

static upbp_mis cam_at(const cam_view* c, int k)
{
    upbp_mis m;
    if (c->cand && k == c->L) return *c->cand;
    m = c->snap[k];
    if (c->prev_override && k == c->L - 1) m.ray_sample_rev_pdf_inv = c->prev_ray_rev_inv;
    return m;
}

static int spec(const upbp_mis* m) { return (m->flags & UPBP_MIS_IS_SPECULAR) != 0; }

static float camera_path_weight(int L, float lastRev, float lastSin, float lastRayRev, float lastRayRevRatio,
                                float ntl, uint32_t qbt, uint32_t pbt, uint32_t tech, const cam_view* cam)
{
    float weight = 0.f, product = 1.f, weightBB1D = 0.f;
    int index;
    for (index = 0; index < L; ++index) {
        const upbp_mis cur = cam_at(cam, L - index);
        upbp_mis nx = index < L - 1 ? cam_at(cam, L - index - 1) : cur;
        float rev = cur.rev_pdf_a, sinT = cur.sin_theta, rayRev = cur.ray_sample_rev_pdf_inv,
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
            float a, b;
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
    float override_ray_rev_inv;
} light_view;

static upbp_mis lv_at(const light_view* l, int k)
{
    upbp_mis m = l->mis[k];
    if (k == l->override_idx) m.ray_sample_rev_pdf_inv = l->override_ray_rev_inv;
    return m;
}

static float light_path_weight(int pathIdx, int pathLength, float lastRev, float lastSin, float lastRayRev,
                               float lastRayRevRatio, float ntl, uint32_t technique, uint32_t qbt, uint32_t pbt,
                               uint32_t tech, const int32_t* pathEnds, const light_view* lv, const upbp_mis* beam_rec)
{
    float weight = 0.f, product = 1.f;
    const int lastIndex = (pathIdx == 0) ? pathLength : pathEnds[pathIdx - 1] + pathLength;
    int index;
    for (index = 0; index <= pathLength; ++index) {
        const upbp_mis cur = (technique == UPBP_BB1D && index == 0) ? *beam_rec : lv_at(lv, lastIndex - index);
        upbp_mis nx = index < pathLength ? lv_at(lv, lastIndex - index - 1) : cur;
        float rev = cur.rev_pdf_a, sinT = cur.sin_theta, rayRev = cur.ray_sample_rev_pdf_inv,
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
                float a, b;
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

static void fill_cand(upbp_mis* c, const upbp_params* P, float pdf_a_inv, float rsp_inv, float ratio, float sel,
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
} oracle;

typedef struct {
    v3 o, d;
    float dmin, dmax, rs_pdf, rs_rev;
    uint32_t rsf, ray_flags;
    int L;
    float lpw;
    const upbp_mis* snap;
} seg_ctx;

/* breIntersectFuncHomogeneous2 after testIntersectionBre accepted light vertex j. */
static rgb pb2d_contrib(const oracle* O, const medium* m, const seg_ctx* s, int64_t j, float t, float d2)
{
    const upbp_params* P = O->P;
    const upbp_light_vertices* lv = O->lv;
    const int pl = lv->path_length[j];
    rgb att, un;
    float pdf, rsp, rsr, ratio, sinT, phase, dirPdf, revPdf, r2, kernel, distSq, rspInv, last, wc, wl;
    upbp_mis cand;
    cam_view cv;
    light_view lview;
    if ((uint32_t)(pl + s->L) > P->max_path_length || (uint32_t)(pl + s->L) < P->min_path_length) return cs(0.f);
    if (s->L == 1 && t < P->min_dist_to_med) return cs(0.f);
    att = eval_att(m, t - s->dmin);
    pdf = comp(att, m->min_idx);
    if (s->ray_flags & UPBP_SHORT_BEAM) att = cdiv(att, pdf);
    rsp = m->min_st * pdf;
    rsr = (s->rsf & UPBP_ORIGIN_IN_MEDIUM) ? rsp : pdf;
    ratio = 1.0f / m->min_st;
    if (!c_positive(att)) return cs(0.f);
    rsp *= s->rs_pdf;
    rsr *= s->rs_rev;
    phase = hg_pdf(neg(s->d), V(lv->dir_fix + 3 * j), m->g, &sinT);
    if (phase <= 0.f) return cs(0.f);
    dirPdf = phase * m->cont;
    revPdf = phase * lv->cont_prob[j];
    r2 = P->radius_pb2d * P->radius_pb2d;
    kernel = (1.f - d2 / r2) / (r2 * PI_F * 0.5f);
    if (!is_pos(kernel)) return cs(0.f);
    un = cscale(cscale(cmul(cmul(C3(lv->throughput + 3 * j), att), C3(m->ss)), phase), kernel);
    if (c_black_neg(un)) return cs(0.f);
    distSq = t * t;
    rspInv = 1.0f / rsp;
    fill_cand(&cand, P, s->lpw * distSq * rspInv, rspInv, ratio, O->has_beams ? 1.f : 0.f,
              m->mfp > P->bb1d_min_mfp ? UPBP_MIS_IN_MEDIUM_WITH_BEAMS : 0u);
    last = (s->ray_flags & UPBP_SHORT_BEAM) ? (float)(1.0 / (double)(ratio * cand.pb2d_factor)) : rsp / cand.pb2d_factor;
    cv.snap = s->snap; cv.L = s->L; cv.cand = &cand; cv.prev_override = 1; cv.prev_ray_rev_inv = 1.0f / rsr;
    wc = camera_path_weight(s->L, last, sinT, lv->mis[j].ray_sample_pdf_inv, lv->mis[j].ray_sample_pdfs_ratio,
                            revPdf * rsr / distSq, P->query_beam_type, P->photon_beam_type, s->ray_flags, &cv);
    lview.mis = lv->mis; lview.override_idx = -1; lview.override_ray_rev_inv = 0.f;
    wl = light_path_weight(lv->path_idx[j], pl, last, 0.f, 0.f, 0.f, dirPdf, UPBP_PB2D, P->query_beam_type,
                           P->photon_beam_type, s->ray_flags, lv->path_ends, &lview, NULL);
    return cscale(un, 1.f / (wl + wc));
}

/* PhotonBeam::accumulate2 after the test and the radius check accepted beam b. */
static rgb bb1d_contrib(const oracle* O, const medium* m, const seg_ctx* s, int64_t b, float dist, float sinTheta,
                        float t1, float t2, float radius)
{
    const upbp_params* P = O->P;
    const upbp_beams* B = O->bm;
    const upbp_light_vertices* lv = O->lv;
    const int lvi = B->light_vertex[b];
    const int pl = lv->path_length[lvi];
    const uint32_t bflags = B->flags[b], brsf = B->ray_sampling_flags[b];
    rgb att, batt, un;
    float pfdQ, rspQ, rsrQ, ratioQ, pfdB, rspB, rsrB, ratioB, phase, sinDummy, dirPdf, revPdf, sel = 1.0f;
    float distSqQ, rspInvQ, distSqB, rspInvB, sinT, f, last, wc, wl, ntl;
    upbp_mis cand, brec;
    cam_view cv;
    light_view lview;
    const upbp_mis* lvm;
    if ((uint32_t)(pl + 1 + s->L) > P->max_path_length || (uint32_t)(pl + 1 + s->L) < P->min_path_length) return cs(0.f);
    if (s->L == 1 && t1 < P->min_dist_to_med) return cs(0.f);
    att = eval_att(m, t1 - s->dmin);
    pfdQ = comp(att, m->min_idx);
    if (s->ray_flags & UPBP_SHORT_BEAM) att = cdiv(att, pfdQ);
    rspQ = m->min_st * pfdQ;
    rsrQ = (s->rsf & UPBP_ORIGIN_IN_MEDIUM) ? rspQ : pfdQ;
    ratioQ = 1.0f / m->min_st;
    batt = eval_att(m, t2);
    att = cmul(att, batt);
    pfdB = comp(batt, m->min_idx);
    if (bflags & UPBP_SHORT_BEAM) att = cdiv(att, pfdB);
    rspB = m->min_st * pfdB;
    rsrB = (brsf & UPBP_ORIGIN_IN_MEDIUM) ? rspB : pfdB;
    ratioB = 1.0f / m->min_st;
    if (!c_positive(att)) return cs(0.f);
    rspQ *= s->rs_pdf;
    rsrQ *= s->rs_rev;
    rspB *= B->ray_sample_pdf[b];
    rsrB *= B->ray_sample_rev_pdf[b];
    phase = hg_pdf(neg(s->d), neg(V(B->direction + 3 * b)), m->g, &sinDummy);
    if (phase <= 0.f) return cs(0.f);
    dirPdf = phase * m->cont;
    revPdf = phase * m->cont;
    un = cdiv(cscale(cscale(cscale(cmul(cmul(cscale(C3(B->throughput + 3 * b), 1.0f / sel), C3(m->ss)), att), phase),
                            1.f - dist * dist / (radius * radius)), 3.f),
              4.f * radius * sinTheta);
    if (c_black_neg(un)) return cs(0.f);
    distSqQ = t1 * t1;
    rspInvQ = 1.0f / rspQ;
    fill_cand(&cand, P, s->lpw * distSqQ * rspInvQ, rspInvQ, ratioQ, sel, UPBP_MIS_IN_MEDIUM_WITH_BEAMS);
    distSqB = (lv->flags[lvi] & UPBP_LV_IS_FINITE) ? t2 * t2 : 1.0f;
    rspInvB = 1.0f / rspB;
    fill_cand(&brec, P, B->last_pdf_w_inv[b] * distSqB * rspInvB, rspInvB, ratioB, sel, UPBP_MIS_IN_MEDIUM_WITH_BEAMS);
    sinT = (s->ray_flags & UPBP_NO_SINE_IN_WEIGHTS) ? 1.0f : sinTheta;
    f = cand.bb1d_factor;
    if (s->ray_flags & UPBP_SHORT_BEAM)
        last = (bflags & UPBP_SHORT_BEAM) ? (float)(1.0 / (double)(ratioQ * ratioB * f * sel * sinT))
                                          : rspB / (ratioQ * f * sel * sinT);
    else
        last = (bflags & UPBP_SHORT_BEAM) ? rspQ / (ratioB * f * sel * sinT) : rspQ * rspB / (f * sel * sinT);
    cv.snap = s->snap; cv.L = s->L; cv.cand = &cand; cv.prev_override = 1; cv.prev_ray_rev_inv = 1.0f / rsrQ;
    wc = camera_path_weight(s->L, last, sinT, rspInvB, ratioB, revPdf * rsrQ / distSqQ, P->query_beam_type,
                            P->photon_beam_type, s->ray_flags, &cv);
    lvm = &lv->mis[lvi];
    ntl = ((lvm->flags & UPBP_MIS_ON_LIGHT_SOURCE) && (lvm->flags & UPBP_MIS_IS_DELTA))
              ? 0.f : dirPdf * rsrB * fabsf(lvm->cos_theta_out) / distSqB;
    lview.mis = lv->mis; lview.override_idx = lvi; lview.override_ray_rev_inv = 1.0f / rsrB;
    wl = light_path_weight(lv->path_idx[lvi], pl + 1, last, 0.f, 0.f, 0.f, ntl, UPBP_BB1D, P->query_beam_type,
                           P->photon_beam_type, s->ray_flags, lv->path_ends, &lview, &brec);
    return cscale(un, 1.f / (wl + wc));
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
    rgb result = cs(0.f), attn = cs(1.f);
    float rsp = 1.f, rsr = 1.f;
    seg_ctx s;
    int i;
    s.o = V(Q->origin + 3 * q);
    s.d = V(Q->direction + 3 * q);
    s.L = Q->path_length[q];
    s.lpw = Q->last_pdf_w_inv[q];
    s.ray_flags = bt | P->techniques;
    s.snap = O->cam + Q->cam_mis_begin[q];
    for (i = 0; i < Q->seg_count[q]; ++i) {
        const int sg = Q->seg_begin[q] + i;
        const medium* m = &O->media[Q->seg_medium[sg]];
        const float dmin = Q->seg_dist_min[sg], dmax = Q->seg_dist_max[sg];
        rgb seg = cs(0.f);
        if (m->has_scat) {
            s.dmin = dmin;
            s.dmax = dmax;
            s.rs_pdf = rsp;
            s.rs_rev = rsr;
            s.rsf = UPBP_END_IN_MEDIUM | (i == 0 ? qrsf : 0u);
            if (est == UPBP_PB2D) {
                const upbp_light_vertices* lv = O->lv;
                const float r2 = P->radius_pb2d * P->radius_pb2d;
                int64_t j;
                for (j = 0; j < lv->n; ++j) {
                    float t, d2;
                    if (!(lv->flags[j] & UPBP_LV_IN_MEDIUM)) continue;
                    if (!test_bre(s.o, s.d, dmin, dmax, V(lv->position + 3 * j), r2, &t, &d2)) continue;
                    ++*cnt;
                    *hash += mix64((uint64_t)j);
                    seg = cadd(seg, pb2d_contrib(O, m, &s, j, t, d2));
                }
            } else {
                const upbp_beams* B = O->bm;
                const float radius = P->radius_bb1d, r2 = radius * radius;
                int64_t b;
                for (b = 0; b < B->n; ++b) {
                    float dist, sinT, t1, t2;
                    if (&O->media[B->medium_id[b]] != m) continue;
                    if (!test_beam_beam(s.o, s.d, dmin, dmax, V(B->origin + 3 * b), V(B->direction + 3 * b), 0.f,
                                        B->length[b], r2, &dist, &sinT, &t1, &t2))
                        continue;
                    if (radius < dist) continue;
                    ++*cnt;
                    *hash += mix64((uint64_t)b);
                    seg = cadd(seg, bb1d_contrib(O, m, &s, b, dist, sinT, t1, t2, radius));
                }
            }
        }
        result = cadd(result, cmul(attn, seg));
        if (lite) {
            float srev, spdf;
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
    const v3 qp = V(Q->position + 3 * q);
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
    cv.snap = O->cam + Q->cam_mis_begin[q]; cv.L = L; cv.cand = NULL; cv.prev_override = 0; cv.prev_ray_rev_inv = 0.f;
    lview.mis = lv->mis; lview.override_idx = -1; lview.override_ray_rev_inv = 0.f;
    for (j = 0; j < 8; ++j) {
        const uint32_t b = hash_cell((j & 4) ? po[0] : p[0], (j & 2) ? po[1] : p[1], (j & 1) ? po[2] : p[2], g->cells);
        int k;
        for (k = g->start[b]; k < g->end[b]; ++k) {
            const int32_t i = g->idx[k];
            const v3 dd = sub(qp, V(lv->position + 3 * i));
            float sinT, phase, dirPdf, revPdf, mwfInv, wc, wl;
            rgb factor;
            int pl;
            if (!(dot(dd, dd) <= g->r2)) continue;
            ++*cnt;
            *hash += mix64((uint64_t)i);
            if (!(lv->flags[i] & UPBP_LV_CONNECTABLE)) continue;
            pl = lv->path_length[i];
            if ((uint32_t)(pl + L) > P->max_path_length || (uint32_t)(pl + L) < P->min_path_length) continue;
            if (m->ss[0] <= 0.f && m->ss[1] <= 0.f && m->ss[2] <= 0.f) continue;
            phase = hg_pdf(cfix, V(lv->dir_fix + 3 * i), m->g, &sinT);
            factor = cscale(C3(m->ss), phase);
            if (c_black_neg(factor)) continue;
            dirPdf = phase * m->cont;
            revPdf = phase * lv->cont_prob[i];
            mwfInv = 1.0f / lv->mis[i].pp3d_factor;
            wc = camera_path_weight(L, mwfInv, sinT, lv->mis[i].ray_sample_pdf_inv, lv->mis[i].ray_sample_pdfs_ratio,
                                    revPdf, P->query_beam_type, P->photon_beam_type, P->techniques, &cv);
            wl = light_path_weight(lv->path_idx[i], pl, mwfInv, 0.f, 0.f, 0.f, dirPdf, UPBP_PP3D, P->query_beam_type,
                                   P->photon_beam_type, P->techniques, lv->path_ends, &lview, NULL);
            res = cadd(res, cscale(cmul(factor, C3(lv->throughput + 3 * i)), 1.f / (wl + wc)));
        }
    }
    return res;
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
    return 0;
}
