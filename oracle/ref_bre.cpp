/*
 * Reference harness TU for PB2D (test infrastructure): compiles the
 * reference's Bre/Bre.cxx unchanged (EmbreeBre::build / evalBre / destroy and
 * the BRE callbacks) and adds the candidate enumerator used for
 * candidate-set parity.
 */
#include <vector>
#include <list>
#include <forward_list>
#include <string>
#include <sstream>
#include <iostream>
#include <iomanip>
#include <algorithm>
#include <cmath>
#define private public
#define protected public
#include "Bre/Bre.cxx"
#undef private
#undef protected

#include "ref_internal.h"

void ref_bre_candidates(const EmbreeBre& bre, const float* origin, const float* dir, float tnear, float tfar,
                        const UPBPLightVertex* lv_base, uint32_t& count, uint64_t& hash)
{
    Ray ray(Pos(origin[0], origin[1], origin[2]), Dir(dir[0], dir[1], dir[2]));
    for (int i = 0; i < bre.numEmbreePhotons; ++i) {
        const EmbreePhoton& ph = bre.embreePhotons[i];
        float t, d2;
        if (EmbreePhoton::testIntersectionBre(t, d2, ray, tnear, tfar, ph.lightVertex->mHitpoint, ph.radiusSqr)) {
            ++count;
            hash += ref_mix64((uint64_t)(ph.lightVertex - lv_base));
        }
    }
}

void ref_bre_radii(const EmbreeBre& bre, const UPBPLightVertex* base, int64_t n, float* r2)
{
    for (int64_t i = 0; i < n; ++i) r2[i] = 0.f;
    for (int i = 0; i < bre.numEmbreePhotons; ++i) {
        const EmbreePhoton& ph = bre.embreePhotons[i];
        r2[ph.lightVertex - base] = ph.radiusSqr;
    }
}

/* Links the photons of a VltLightVertex build (Bre.cxx:526-614, which stores position, radius,
 * direction and flux but no light vertex) to the light vertices they were made from: the build
 * takes the in-medium vertices in order.  Only the candidate enumeration and the radii read it. */
void ref_bre_link_photons(EmbreeBre& bre, const UPBPLightVertex* base, int64_t n)
{
    int k = 0;
    for (int64_t i = 0; i < n && k < bre.numEmbreePhotons; ++i)
        if (base[i].mInMedium) bre.embreePhotons[k++].lightVertex = base + i;
}
