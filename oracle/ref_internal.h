/*
 * Cross-translation-unit helpers of the reference harness (test infrastructure).
 * Each reference .cxx is compiled in its own TU (they define the same
 * file-scope constants), so the harness reaches them through these functions.
 */
#pragma once

#include <cstdint>

struct UPBPLightVertex;
class EmbreeBre;
class Scene;
namespace SmallUPBP_ref_fwd {}

/* splitmix64 finaliser of (id+1): order-independent candidate-set hash term */
static inline uint64_t ref_mix64(uint64_t id) {
    uint64_t z = id + 1 + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

/* ref_bre.cpp: PB2D candidates of one query segment, by the reference's
 * EmbreePhoton::testIntersectionBre (Bre.cxx:199-223) over every photon of `bre`. */
void ref_bre_candidates(const EmbreeBre& bre, const float* origin, const float* dir, float tnear, float tfar,
                        const UPBPLightVertex* lv_base, uint32_t& count, uint64_t& hash);
