"""BB1D closest-approach precision stress: photon beams and query rays with origins uniform in the
unit cube, half of each within 1e-4 rad of a common axis and half isotropic, lengths ~Exp(2),
r = 0.002 (``workload.beam_stress``).

The reference rejects a pair as parallel when |d1.d2|^2 - 1 is within 1e-5 (PhotonBeam.hxx:267-273),
so all near-parallel/near-parallel pairs are rejected by every implementation; the pairs that stay
are isotropic/isotropic and isotropic/near-parallel, some of them close enough to parallel for the
FP32 closest-approach solve to lose digits.  Candidate sets must be bit-exact against the oracle,
which applies the same BB1D reach rule as the CUDA path: a pair the reference's FP32 predicate
accepts is kept when the FP64 distance of the two segments is within the radius at the closest
point plus 2e-5 + 1e-3 r.  The pairs the rule removes from the reference's brute-force set are
checked one by one on the CPU (``rule_removed``).  Contributions are compared against the FP64
oracle with per-query relative-error histograms.

Run as a script on a GPU machine to print the histograms as JSON:
    python tests/test_beam_stress.py [n_beams n_queries]
"""
import json
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))

import golden_io as G  # noqa: E402
from smallupbp_b200 import workload as W  # noqa: E402

N_BEAMS, N_QUERIES = 100000, 20000
BINS = [0.0, 1e-7, 1e-6, 1e-5, 1e-4, 1e-3, 1e-2, np.inf]


@pytest.fixture(scope="module")
def stress():
    return W.beam_stress(N_BEAMS, N_QUERIES)


def per_query_rel(got: np.ndarray, want: np.ndarray) -> np.ndarray:
    """Max over RGB of |got - want| / |want| for queries whose FP64 contribution is nonzero."""
    g, w = got.astype(np.float64), want.astype(np.float64)
    mag = np.abs(w).max(axis=1)
    m = mag > 0
    return np.abs(g - w).max(axis=1)[m] / mag[m]


def histogram(rel: np.ndarray) -> dict:
    h, _ = np.histogram(rel, bins=BINS)
    labels = ["<1e-7", "1e-7..1e-6", "1e-6..1e-5", "1e-5..1e-4", "1e-4..1e-3", "1e-3..1e-2", ">=1e-2"]
    return {"queries": int(len(rel)), "median": float(np.median(rel)) if len(rel) else 0.0,
            "p99": float(np.percentile(rel, 99)) if len(rel) else 0.0, "max": float(rel.max()) if len(rel) else 0.0,
            "histogram": dict(zip(labels, [int(x) for x in h]))}


def test_stress_geometry(stress):
    w = stress
    for key in ("beam_direction", "sq_direction"):
        d = w[key].astype(np.float64)
        assert np.allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-6)
        par = d[:, 2] > np.cos(1e-4) - 1e-7
        assert 0.45 < par.mean() < 0.55
    assert 0.4 < w["beam_length"].mean() < 0.6 and 0.4 < w["seg_dist_max"].mean() < 0.6
    assert (w["beam_origin"] >= 0).all() and (w["beam_origin"] < 1).all()
    assert len(w["pq_path_length"]) == 0
    assert ((w["sq_flags"] & W.Q_BB1D) != 0).all() and ((w["sq_flags"] & (W.Q_PB2D | W.Q_LITE)) == 0).all()
    assert w["beam_light_vertex"].max() < len(w["lv_path_idx"])


def test_oracles_share_candidates(stress):
    from oracle import port

    a, b = port.run(stress), port.run(stress, fp64=True)
    assert a["count_bb1d"].sum() > 1000
    np.testing.assert_array_equal(a["count_bb1d"], b["count_bb1d"])
    np.testing.assert_array_equal(a["hash_bb1d"], b["hash_bb1d"])


M64 = (1 << 64) - 1


def mix64(i: int) -> int:
    """The order-independent candidate hash term of the CUDA path and the oracle (splitmix64)."""
    z = (i + 1 + 0x9E3779B97F4A7C15) & M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


def _dotf(a, b):  # the reference's _mm_dp_ps order in FP32: (x*x' + y*y') + z*z'
    return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]


def _crossf(a, b):
    return np.stack([a[..., 1] * b[..., 2] - a[..., 2] * b[..., 1], a[..., 2] * b[..., 0] - a[..., 0] * b[..., 2],
                     a[..., 0] * b[..., 1] - a[..., 1] * b[..., 0]], -1)


def fp32_accepted(w, q):
    """Beams that PhotonBeam::testIntersectionBeamBeam + the radius test accept for query q (one
    segment), evaluated in FP32 numpy (no FMA, the reference's operation order)."""
    f = np.float32
    O1, d1 = w["sq_origin"][q][None], w["sq_direction"][q][None]
    mn, mx = w["seg_dist_min"][q], w["seg_dist_max"][q]
    O2, d2, ln = w["beam_origin"], w["beam_direction"], w["beam_length"]
    r = f(w["params"]["radius_bb1d"][0])
    c = _crossf(d1, d2)
    s2 = _dotf(c, c)
    ad = _dotf(O2 - O1, c)
    ok = ad * ad < (r * r) * s2
    d1d2 = _dotf(d1, d2)
    m1 = d1d2 * d1d2 - f(1)
    ok &= ~((m1 < f(1e-5)) & (m1 > f(-1e-5)))
    with np.errstate(all="ignore"):
        t1 = (_dotf(d1, O1) - _dotf(d1, O2) - d1d2 * (_dotf(d2, O1) - _dotf(d2, O2))) / m1
        ok &= (t1 > mn) & (t1 < mx)
        t2 = (t1 + _dotf(d1, O1) - _dotf(d1, O2)) / d1d2
        ok &= (t2 > 0) & (t2 < ln) & ~np.isnan(t2)
        dist = np.abs(ad) / np.sqrt(s2)
    ok &= ~(r < dist)
    return np.nonzero(ok)[0]


def rule_rejects(w, q, b) -> bool:
    """The BB1D reach rule, restated in FP64 numpy: True when the segments of query q and beam b are
    farther apart than r(u) + 2e-5 + 1e-3 r, u being the beam parameter of their closest points."""
    O1, d1 = w["sq_origin"][q].astype(float), w["sq_direction"][q].astype(float)
    a1, b1 = float(w["seg_dist_min"][q]), float(w["seg_dist_max"][q])
    O2, d2, ln = w["beam_origin"][b].astype(float), w["beam_direction"][b].astype(float), float(w["beam_length"][b])
    r = float(np.float32(w["params"]["radius_bb1d"][0]))
    wv = O1 - O2
    bb, dd, ee, aa, cc = d1 @ d2, d1 @ wv, d2 @ wv, d1 @ d1, d2 @ d2
    den = aa * cc - bb * bb
    t, u, inside = a1, 0.0, False
    if den > 1e-300:
        t, u = (bb * ee - cc * dd) / den, (aa * ee - bb * dd) / den
        inside = a1 <= t <= b1 and 0.0 <= u <= ln
    if not inside:
        t = min(max(t, a1), b1)
        u = min(max((bb * t + ee) / cc, 0.0), ln)
        t = min(max((bb * u - dd) / aa, a1), b1)
        u = min(max((bb * t + ee) / cc, 0.0), ln)
    dist = float(np.linalg.norm(wv + t * d1 - u * d2))
    extra = float(np.float32(2e-5) + np.float32(1e-3) * np.float32(r))
    return dist > r + extra


def rule_removed(w, rule_count, rule_hash, ref_count, ref_hash) -> dict:
    """For every query whose candidate set under the reach rule differs from the reference's
    brute-force set, enumerate the FP32-accepted beams and check that the difference is exactly the
    beams the rule rejects: the counts and the order-independent hashes must agree.  These are pairs
    the FP32 predicate accepts only through rounding (a nearly perpendicular pair's FP32 t2 lands
    inside the beam while the true closest point lies beyond its end)."""
    bad = np.nonzero((rule_count != ref_count) | (rule_hash != ref_hash))[0]
    removed = 0
    for q in bad:
        acc = fp32_accepted(w, q)
        assert len(acc) == ref_count[q], ("emulation", q, len(acc), ref_count[q])
        assert sum(mix64(int(b)) for b in acc) & M64 == int(ref_hash[q]), ("emulation hash", q)
        gone = [int(b) for b in acc if rule_rejects(w, q, int(b))]
        kept_hash = (int(ref_hash[q]) - sum(mix64(b) for b in gone)) & M64
        assert len(acc) - len(gone) == int(rule_count[q]) and kept_hash == int(rule_hash[q]), \
            ("difference not explained by the reach rule", int(q), int(rule_count[q]), int(ref_count[q]), gone)
        removed += len(gone)
    return {"queries_differing": int(len(bad)), "pairs_removed": removed}


def test_reach_rule_removes_only_rounding_pairs(stress):
    """The oracle with the reach rule against the reference's brute-force definition (the oracle
    with the rule off): every removed pair is one that the rule rejects, none is added."""
    from oracle import port

    a, b = port.run(stress), port.run(stress, reach=False)
    assert (a["count_bb1d"] <= b["count_bb1d"]).all()
    rep = rule_removed(stress, a["count_bb1d"], a["hash_bb1d"], b["count_bb1d"], b["hash_bb1d"])
    assert rep["pairs_removed"] <= 1e-5 * b["count_bb1d"].astype(np.int64).sum() + 1, rep


def test_rule_check_catches_a_planted_difference(stress):
    """The checker itself: remove an ordinary pair from a copy of the oracle's counts and hashes (on
    the CPU) and check that rule_removed rejects the difference."""
    from oracle import port

    w = stress
    o = port.run(w, reach=False)
    q = next(q for q in range(len(o["count_bb1d"])) if o["count_bb1d"][q] >= 1)
    b = int(fp32_accepted(w, q)[0])
    assert not rule_rejects(w, q, b)
    cnt, h = o["count_bb1d"].copy(), o["hash_bb1d"].copy()
    cnt[q] -= 1
    h[q] = np.uint64((int(h[q]) - mix64(b)) & M64)
    with pytest.raises(AssertionError, match="not explained"):
        rule_removed(w, cnt, h, o["count_bb1d"], o["hash_bb1d"])
    assert rule_removed(w, o["count_bb1d"], o["hash_bb1d"], o["count_bb1d"], o["hash_bb1d"])["queries_differing"] == 0


def gpu_report(w) -> dict:
    from oracle import port
    from smallupbp_b200 import engine

    o32, o64 = port.run(w), port.run(w, fp64=True)
    out = {"beams": int(len(w["beam_length"])), "queries": int(len(w["sq_path_length"])),
           "accepted": int(o64["count_bb1d"].astype(np.int64).sum())}
    for name, mode in (("plain", engine.MODE_PLAIN), ("mixed", engine.MODE_MIXED)):
        with engine.EstimatorStage(0, mode) as st:
            st.run(w)
            _, bb1d = st.segment_results()
            stats = st.query_stats()
            img = st.image()
        out[name] = {"candidates_equal_oracle": bool(np.array_equal(stats["count_bb1d"], o64["count_bb1d"]) and
                                                     np.array_equal(stats["hash_bb1d"], o64["hash_bb1d"])),
                     "queries_differing": int(((stats["count_bb1d"] != o64["count_bb1d"]) |
                                               (stats["hash_bb1d"] != o64["hash_bb1d"])).sum()),
                     "vs_fp64": histogram(per_query_rel(bb1d, o64["bb1d"])),
                     "image_rel_l2_vs_fp64": G.image_rel_l2(img, o64["image"]),
                     "_bb1d": bb1d}
    out["fp32_oracle"] = {"vs_fp64": histogram(per_query_rel(o32["bb1d"], o64["bb1d"])),
                          "image_rel_l2_vs_fp64": G.image_rel_l2(o32["image"], o64["image"])}
    out["_o32"] = o32["bb1d"]
    return out


@pytest.mark.gpu
def test_gpu_stress_against_fp64_oracle(stress):
    rep = gpu_report(stress)
    for name in ("plain", "mixed"):
        # bit-exact: every query's count and candidate hash equal the oracle's (reach rule applied)
        assert rep[name]["candidates_equal_oracle"], (name, rep[name]["queries_differing"])
        assert rep[name]["image_rel_l2_vs_fp64"] <= 1e-3, (name, rep[name]["image_rel_l2_vs_fp64"])
    # plain FP32 follows the FP32 reference arithmetic
    G.assert_close(rep["plain"]["_bb1d"], rep["_o32"], "plain BB1D vs FP32 oracle")
    # the FP64 solve of near-parallel pairs: mixed is never worse than FP32 at the tail
    assert rep["mixed"]["vs_fp64"]["max"] <= rep["plain"]["vs_fp64"]["max"] + 1e-6
    assert rep["mixed"]["vs_fp64"]["p99"] <= 1e-4


if __name__ == "__main__":
    nb = int(sys.argv[1]) if len(sys.argv) > 1 else N_BEAMS
    nq = int(sys.argv[2]) if len(sys.argv) > 2 else N_QUERIES
    r = gpu_report(W.beam_stress(nb, nq))
    print(json.dumps({k: ({kk: vv for kk, vv in v.items() if not kk.startswith("_")} if isinstance(v, dict) else v)
                      for k, v in r.items() if not k.startswith("_")}, indent=1))
