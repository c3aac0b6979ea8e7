"""Seeded synthetic UPBP iteration data for the volumetric estimator stage.

The estimator stage consumes what one ``UPBP::RunIteration`` produces on the
host: light vertices with their MIS records (``Renderers/UPBP.hxx:501-674``),
photon beams (``UPBP::AddBeams``, ``UPBP.hxx:1783-1870``) and, per camera
segment / camera medium vertex, the estimator calls with a snapshot of the
camera MIS records (``UPBP.hxx:742-1160``).  This module produces exactly
those records for scenes made of nested axis-aligned boxes of homogeneous
media (imaginary boundaries, no surfaces), an area quad light on the top face
of the outer box and a pinhole camera, following the reference formulas for
free-flight sampling (``Scene/Media.hxx:240-323``), Henyey-Greenstein
sampling (``Path/PhaseFunction.hxx:82-137``), Russian roulette with the
medium continuation probability, and the MIS bookkeeping of the light and
camera passes (``UPBP.hxx:600-645, 940-975, 1908-1969``).

No public dataset is involved; the inputs are generated from a Philox
counter-based generator with a fixed seed.  Both the oracle and the CUDA path
consume the same arrays (layout of ``include/upbp_gpu.h``).

Random numbers are per path: Philox4x64-10 (Salmon et al., "Parallel random
numbers: as easy as 1, 2, 3", SC'11) with key (seed, iteration) and counter
(path or pixel index, bounce, block, stream) gives four uniforms
``(x >> 11) * 2^-53`` per counter.  Light path p: the emission draws are block 0
of bounce 0 (position x, position z, two direction samples); the ray of bounce L
(from vertex L-1) takes its free-flight draws for medium segment k from block
1 + k // 4, word k % 4, and the scattering at vertex L its phase-function and
Russian-roulette draws from block 0, words 0-2.  Camera path of pixel p: the
pixel jitter is block 0 of bounce 0, words 0-1; bounces as for light paths.
Every path therefore draws the same numbers whatever the others do, and the
device-side light and camera passes (``upbp_trace_light_paths`` /
``upbp_trace_camera_paths``) trace the same paths.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, List, Sequence, Tuple

import numpy as np

# flags, identical to include/upbp_gpu.h (and the reference enums)
SHORT_BEAM, LONG_BEAM = 1, 2
BPT, SURF, PP3D, PB2D, BB1D = 4, 8, 16, 32, 64
BP2D = 65536  # extension: B-P2D (standalone, MIS weight 1); not a reference technique
NO_SINE_IN_WEIGHTS, PREVIOUS, COMPATIBLE, BB1D_PREVIOUS = 128, 256, 512, 1024
NO_MIS = 131072  # the estimators without MIS of VolLightTracer's pure -a pb2d / -a bb1d (upbp_gpu.h)

# MIS inputs that the estimators without MIS never read: without_mis() leaves them out, and the C
# ABI receives them as NULL
MIS_ONLY_INPUTS = ("lv_mis", "lv_path_idx", "lv_cont_prob", "lv_path_ends", "beam_ray_sample_pdf",
                   "beam_ray_sample_rev_pdf", "beam_ray_sampling_flags", "beam_last_pdf_w_inv", "beam_light_vertex",
                   "sq_last_pdf_w_inv", "sq_cam_mis_begin", "cam_mis")
ORIGIN_IN_MEDIUM, END_IN_MEDIUM = 1, 2
MIS_IS_DELTA, MIS_ON_LIGHT_SOURCE, MIS_IS_SPECULAR, MIS_IN_MEDIUM_WITH_BEAMS = 1, 2, 4, 8
LV_IN_MEDIUM, LV_CONNECTABLE, LV_IS_FINITE = 1, 2, 4
Q_ORIGIN_IN_MEDIUM, Q_LITE, Q_PB2D, Q_BB1D = 1, 2, 4, 8

# upbp_mis layout: 14 float32 + 1 uint32 (60 bytes)
MIS_FIELDS = (
    "pdf_a_inv", "rev_pdf_a", "rev_pdf_a_without_bsdf", "ray_sample_pdf_inv", "ray_sample_rev_pdf_inv",
    "ray_sample_pdfs_ratio", "ray_sample_rev_pdfs_ratio", "sin_theta", "cos_theta_out", "surf_factor",
    "pp3d_factor", "pb2d_factor", "bb1d_factor", "bb1d_beam_selection_pdf",
)
MIS_DTYPE = np.dtype([(f, "<f4") for f in MIS_FIELDS] + [("flags", "<u4")])
assert MIS_DTYPE.itemsize == 60

MEDIUM_DTYPE = np.dtype([("absorption", "<f4", (3,)), ("scattering", "<f4", (3,)),
                         ("mean_cosine", "<f4"), ("continuation_prob", "<f4")])

PARAMS_FIELDS = (
    ("techniques", "<u4"), ("query_beam_type", "<u4"), ("photon_beam_type", "<u4"),
    ("min_path_length", "<u4"), ("max_path_length", "<u4"),
    ("radius_pp3d", "<f4"), ("radius_pb2d", "<f4"), ("radius_bb1d", "<f4"),
    ("mis_factor_surf", "<f4"), ("mis_factor_pp3d", "<f4"), ("mis_factor_pb2d", "<f4"), ("mis_factor_bb1d", "<f4"),
    ("norm_pp3d", "<f4"), ("norm_pb2d", "<f4"), ("norm_bb1d", "<f4"),
    ("bb1d_min_mfp", "<f4"), ("min_dist_to_med", "<f4"),
    ("hash_cells", "<i4"), ("image_width", "<i4"), ("image_height", "<i4"),
    ("pb2d_knn", "<i4"), ("bb1d_knn", "<i4"), ("knn_exact", "<i4"),
)
PARAMS_DTYPE = np.dtype(list(PARAMS_FIELDS))

EPS_COSINE = 1e-6
INV_PI = 1.0 / math.pi


LIGHT_STREAM, CAMERA_STREAM = 0, 1
_PHILOX_M = (np.uint64(0xD2E7470EE14C6C93), np.uint64(0xCA5A826395121157))
_PHILOX_W = (np.uint64(0x9E3779B97F4A7C15), np.uint64(0xBB67AE8584CAA73B))
_MASK32 = np.uint64(0xFFFFFFFF)
_S32 = np.uint64(32)


def _mulhilo64(a: np.ndarray, b: np.uint64):
    """(high, low) 64-bit halves of the 128-bit product a * b, elementwise."""
    a0, a1 = a & _MASK32, a >> _S32
    b0, b1 = b & _MASK32, b >> _S32
    p00, p01, p10, p11 = a0 * b0, a0 * b1, a1 * b0, a1 * b1
    mid = (p00 >> _S32) + (p01 & _MASK32) + (p10 & _MASK32)
    return p11 + (p01 >> _S32) + (p10 >> _S32) + (mid >> _S32), a * b


def philox4x64(counter, key):
    """Philox4x64-10 block function: counter = 4 uint64 arrays, key = 2 uint64 -> 4 uint64 arrays."""
    c = [np.asarray(x, np.uint64) for x in counter]
    k0, k1 = np.uint64(key[0]), np.uint64(key[1])
    with np.errstate(over="ignore"):
        for rnd in range(10):
            if rnd:
                k0, k1 = k0 + _PHILOX_W[0], k1 + _PHILOX_W[1]
            hi0, lo0 = _mulhilo64(c[0], _PHILOX_M[0])
            hi1, lo1 = _mulhilo64(c[2], _PHILOX_M[1])
            c = [hi1 ^ c[1] ^ k0, lo1, hi0 ^ c[3] ^ k1, lo0]
    return c


def uniforms(key, stream: int, ids: np.ndarray, bounce: int, block: int) -> np.ndarray:
    """(n, 4) uniforms in [0, 1) of counter (ids, bounce, block, stream) under key (seed, iteration)."""
    ids = np.asarray(ids, np.uint64)
    z = np.zeros_like(ids)
    words = philox4x64((ids, z + np.uint64(bounce), z + np.uint64(block), z + np.uint64(stream)), key)
    return np.stack([(w >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0) for w in words], axis=1)


def flight_uniforms(key, stream: int, ids: np.ndarray, bounce: int, n_segments: int) -> np.ndarray:
    """(n, n_segments) free-flight uniforms of one bounce: segment k is word k % 4 of block 1 + k // 4."""
    blocks = [uniforms(key, stream, ids, bounce, 1 + b) for b in range((n_segments + 3) // 4)]
    if not blocks:
        return np.zeros((len(ids), 0))
    return np.concatenate(blocks, axis=1)[:, :n_segments]


@dataclasses.dataclass
class Medium:
    absorption: Tuple[float, float, float]
    scattering: Tuple[float, float, float]
    mean_cosine: float = 0.0
    continuation_prob: float = 0.8

    @property
    def sigma_t(self) -> np.ndarray:
        return np.asarray(self.absorption, np.float64) + np.asarray(self.scattering, np.float64)

    @property
    def min_pos_sigma_t(self) -> float:
        # HomogeneousMedium ctor (Scene/Media.hxx:142-145): smallest positive component
        st = self.sigma_t
        best = st[0]
        for c in (1, 2):
            if st[c] > 0 and (best == 0 or st[c] < best):
                best = st[c]
        return float(best)

    @property
    def has_scattering(self) -> bool:
        return bool(np.any(np.asarray(self.scattering) > 0))

    @property
    def mfp(self) -> float:
        st = self.sigma_t
        return float(1.0 / st.max()) if st.max() > 0 else math.inf


CLEAR = Medium((0.0, 0.0, 0.0), (0.0, 0.0, 0.0), 0.0, 1.0)


@dataclasses.dataclass
class SceneConfig:
    """Nested boxes of media; boxes[i] = (lo, hi, medium index); later boxes are inside earlier ones."""
    name: str
    media: List[Medium]
    boxes: List[Tuple[Tuple[float, float, float], Tuple[float, float, float], int]]
    width: int
    height: int
    light_paths: int
    max_path_length: int
    radius: float
    camera_pos: Tuple[float, float, float] = (0.5, 0.5, -1.5)
    fov_deg: float = 45.0
    light_size: float = 0.2
    light_intensity: float = 25.0
    techniques: int = BPT | SURF | PP3D | PB2D | BB1D
    query_beam_type: int = LONG_BEAM
    photon_beam_type: int = SHORT_BEAM
    beam_length_cap: float = math.inf
    min_path_length: int = 0
    min_dist_to_med: float = 0.0
    bb1d_storage_factor: float = 0.0
    pb2d_knn: int = 0   # KNN photon radius (0: constant radius)
    bb1d_knn: int = 0   # KNN beam radius (0: constant radius)
    seed: int = 1234


def cube_scene(name="cube128", width=128, height=128, light_paths=16384, max_path_length=6, radius=0.01,
               **kw) -> SceneConfig:
    media = [CLEAR, Medium((0.1, 0.1, 0.1), (0.5, 0.5, 0.5), 0.3, 0.8)]
    return SceneConfig(name, media, [((0, 0, 0), (1, 1, 1), 1)], width, height, light_paths, max_path_length,
                       radius, **kw)


def nested_boxes_scene(name="boxes3", width=1024, height=1024, light_paths=2_097_152, max_path_length=6,
                       radius=0.005, **kw) -> SceneConfig:
    albedo = 0.8
    mk = lambda st, g: Medium(tuple([st * (1 - albedo)] * 3), tuple([st * albedo] * 3), g, 0.8)
    media = [CLEAR, mk(0.05, -0.5), mk(1.0, 0.0), mk(10.0, 0.7)]
    boxes = [((0, 0, 0), (1, 1, 1), 1), ((0.2, 0.2, 0.2), (0.8, 0.8, 0.8), 2), ((0.35, 0.35, 0.35), (0.65, 0.65, 0.65), 3)]
    return SceneConfig(name, media, boxes, width, height, light_paths, max_path_length, radius, **kw)


def config(name: str) -> SceneConfig:
    """The workloads of the five estimator-stage configurations (names used by tests and bench)."""
    if name == "cube128":      # CPU-runnable case: 128^2, 16384 light paths, r=0.01
        return cube_scene()
    if name == "cube1024":     # 1024^2, 1,048,576 light paths, r=0.005, LONG photon beams capped at 2.0
        return cube_scene("cube1024", 1024, 1024, 1_048_576, 6, 0.005, photon_beam_type=LONG_BEAM,
                          beam_length_cap=2.0)
    if name == "cube512":      # quarter-size cube1024 (profiling case): 512^2, 262,144 light paths
        return cube_scene("cube512", 512, 512, 262_144, 6, 0.005, photon_beam_type=LONG_BEAM, beam_length_cap=2.0)
    if name == "boxes3":       # heavy-tailed: nested sigma_t 0.05 / 1 / 10
        return nested_boxes_scene()
    if name == "diff512":      # differentiable-estimator scene: 512^2, 262,144 light paths
        return cube_scene("diff512", 512, 512, 262_144, 6, 0.01)
    if name == "beamstress":   # BB1D closest-approach stress: 2M beams x 2M query rays (see beam_stress)
        ss = 1.6
        return SceneConfig("beamstress", [CLEAR, Medium((0.4,) * 3, (ss,) * 3, 0.3, 0.8)], [((0, 0, 0), (1, 1, 1), 1)],
                           64, 64, 4096, 6, 0.002)
    if name.startswith("cube") and "x" in name[4:]:
        # cube<W>x<N_L>, e.g. cube64x4096 (small parity cases)
        w, nl = name[4:].split("x")
        return cube_scene(name, int(w), int(w), int(nl), 6, 0.02 if int(nl) < 8192 else 0.01)
    raise KeyError(name)


# ----------------------------------------------------------------------------------------------
# Geometry helpers (vectorised over rays)

def _box_breaks(cfg: SceneConfig, o: np.ndarray, d: np.ndarray):
    """Return sorted break distances t>0 (n, K) with +inf padding, from all box slabs."""
    n = o.shape[0]
    ts = []
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = 1.0 / d
        for lo, hi, _m in cfg.boxes:
            lo = np.asarray(lo, np.float64)
            hi = np.asarray(hi, np.float64)
            t0 = (lo - o) * inv
            t1 = (hi - o) * inv
            tmin = np.nanmax(np.minimum(t0, t1), axis=1)
            tmax = np.nanmin(np.maximum(t0, t1), axis=1)
            hit = tmax >= np.maximum(tmin, 0.0)
            a = np.where(hit & (tmin > 0), tmin, np.inf)
            b = np.where(hit & (tmax > 0), tmax, np.inf)
            ts += [a, b]
    t = np.stack(ts, axis=1) if ts else np.zeros((n, 0))
    t.sort(axis=1)
    return t


def _medium_at(cfg: SceneConfig, p: np.ndarray) -> np.ndarray:
    m = np.zeros(p.shape[0], np.int32)
    for lo, hi, mid in cfg.boxes:
        inside = np.all((p >= np.asarray(lo)) & (p <= np.asarray(hi)), axis=1)
        m = np.where(inside, mid, m)
    return m


def _trace(cfg: SceneConfig, u: np.ndarray, o: np.ndarray, d: np.ndarray, origin_in_medium: np.ndarray):
    """Scene::Intersect for imaginary-boundary media, vectorised over rays.

    The ray is split at every box face into medium segments; a free-flight distance is sampled in
    each scattering medium in order (HomogeneousMedium::SampleRay, Scene/Media.hxx:240-290) until
    one scatters; ``u`` (n, K) holds the free-flight uniforms of the K possible segments.  Returns
    a dict of (n, K) arrays: ``full`` marks the VolumeSegments (up to the
    scattering point, clear-medium segments included), ``lite`` the LiteVolumeSegments (every
    scattering medium on the ray), with distances, pdfs, attenuation and medium ids, plus the
    scattering distance per ray (inf when the ray leaves the scene).
    """
    n = o.shape[0]
    breaks = _box_breaks(cfg, o, d)
    K = breaks.shape[1]
    starts = np.concatenate([np.zeros((n, 1)), breaks[:, :-1]], axis=1)
    ends = breaks.copy()
    valid = np.isfinite(ends) & (ends > starts)
    mids = np.where(valid, 0.5 * (starts + np.where(np.isfinite(ends), ends, starts)), 0.0)
    med = np.zeros((n, K), np.int32)
    for k in range(K):
        med[:, k] = _medium_at(cfg, o + d * mids[:, k:k + 1])
    st_tab = np.array([m.sigma_t for m in cfg.media])                 # (M, 3)
    smin_tab = np.array([m.min_pos_sigma_t for m in cfg.media])
    scat_tab = np.array([m.has_scattering for m in cfg.media])
    assert u.shape == (n, K)
    np.seterr(invalid="ignore")
    alive = np.ones(n, bool)
    full = np.zeros((n, K), bool)
    dmax = ends.copy()
    pdf = np.ones((n, K))
    rev = np.ones((n, K))
    att = np.ones((n, K, 3))
    scatter_t = np.full(n, np.inf)
    for k in range(K):
        v = valid[:, k]
        m = med[:, k]
        seglen = np.where(v, ends[:, k] - starts[:, k], 0.0)
        smin = smin_tab[m]
        sampled = v & alive & scat_tab[m] & (smin > 0)
        full[:, k] = v & alive
        first = np.full(n, k == 0) & origin_in_medium
        with np.errstate(divide="ignore", invalid="ignore"):
            s = -np.log(np.maximum(u[:, k], 1e-300)) / np.where(smin > 0, smin, 1.0)
        hit = sampled & (s < seglen)
        through = sampled & ~hit
        a_hit = np.exp(-smin * s)
        a_thr = np.exp(-smin * seglen)
        pdf[:, k] = np.where(hit, smin * a_hit, np.where(through, a_thr, 1.0))
        rev[:, k] = np.where(hit, np.where(first, smin * a_hit, a_hit),
                             np.where(through, np.where(first, smin * a_thr, a_thr), 1.0))
        ln = np.where(hit, s, seglen)
        att[:, k, :] = np.exp(-st_tab[m] * ln[:, None])
        dmax[:, k] = np.where(hit, starts[:, k] + s, ends[:, k])
        scatter_t = np.where(hit, starts[:, k] + s, scatter_t)
        alive &= ~hit
    lite = valid & scat_tab[med]
    return dict(K=K, dmin=starts, dmax_full=dmax, dmax_lite=ends, pdf=pdf, rev=rev, att=att, med=med, full=full,
                lite=lite, scatter_t=scatter_t)


def _hg_sample(u1: np.ndarray, u2: np.ndarray, wfix: np.ndarray, g: np.ndarray):
    """PhaseFunction::Sample (Path/PhaseFunction.hxx:82-137): returns (direction, pdf, sinTheta)."""
    iso = np.abs(g) < 1e-3
    g2 = g * g
    twog = g + g
    with np.errstate(divide="ignore", invalid="ignore"):
        sq = (1 - g2) / (1 - g + twog * u1)
        cos_hg = (1 + g2 - sq * sq) / twog
    cos_iso = 1 - 2 * u1
    cos_t = np.clip(np.where(iso, cos_iso, cos_hg), -1, 1)
    sin_t = np.sqrt(np.maximum(0.0, 1 - cos_t * cos_t))
    phi = 2 * math.pi * u2
    # frame with z = -wfix (the propagation direction)
    z = -wfix
    a = np.where(np.abs(z[:, :1]) > 0.99, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
    x = np.cross(a, z)
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    y = np.cross(z, x)
    w = x * (np.cos(phi) * sin_t)[:, None] + y * (np.sin(phi) * sin_t)[:, None] + z * cos_t[:, None]
    w /= np.linalg.norm(w, axis=1, keepdims=True)
    d = 1 + g2 - twog * cos_t
    pdf = np.where(iso, 0.25 * INV_PI, 0.25 * INV_PI * (1 - g2) / (d * np.sqrt(np.maximum(d, 1e-30))))
    return w, pdf, sin_t


def iteration_constants(cfg: SceneConfig, iteration: int = 0) -> Dict[str, float]:
    """UPBP::RunIteration per-iteration constants (Renderers/UPBP.hxx:422-460) with alpha=1 radii."""
    nl = float(cfg.light_paths)
    r = cfg.radius
    eta_surf = math.pi * r * r * nl
    eta_pp3d = (4.0 / 3.0) * math.pi * r ** 3 * nl
    eta_pb2d = math.pi * r * r * nl
    eta_bb1d = 0.5 * r * nl
    return dict(radius=r, eta_surf=eta_surf, eta_pp3d=eta_pp3d, eta_pb2d=eta_pb2d, eta_bb1d=eta_bb1d,
                norm_pp3d=1.0 / eta_pp3d, norm_pb2d=1.0 / nl, norm_bb1d=1.0 / nl,
                bb1d_min_mfp=cfg.bb1d_storage_factor * 0.5 * math.pi * r)


def _mis_record(**kw) -> tuple:
    vals = [float(kw.get(f, 0.0)) for f in MIS_FIELDS]
    return tuple(vals) + (int(kw.get("flags", 0)),)


def _media_tables(cfg: SceneConfig):
    M = cfg.media
    return dict(st=np.array([m.sigma_t for m in M]), ss=np.array([np.asarray(m.scattering, float) for m in M]),
                smin=np.array([m.min_pos_sigma_t for m in M]), scat=np.array([m.has_scattering for m in M]),
                mfp=np.array([m.mfp for m in M]), g=np.array([m.mean_cosine for m in M]),
                cont=np.array([m.continuation_prob for m in M]),
                maxlen=np.array([(-math.log(1e-9) / m.sigma_t.max()) if m.sigma_t.max() > 0 else math.inf for m in M]))


def _new_mis(n: int) -> np.ndarray:
    return np.zeros(n, MIS_DTYPE)


def _full_products(tr, sel: np.ndarray):
    """Products over the VolumeSegments of rays `sel`: pdf, rev pdf and attenuation."""
    f = tr["full"][sel]
    rsp = np.prod(np.where(f, tr["pdf"][sel], 1.0), axis=1)
    rsr = np.prod(np.where(f, tr["rev"][sel], 1.0), axis=1)
    att = np.prod(np.where(f[:, :, None], tr["att"][sel], 1.0), axis=1)
    return rsp, rsr, att


def _last_full_medium(tr, sel: np.ndarray) -> np.ndarray:
    f = tr["full"][sel]
    last = f.shape[1] - 1 - np.argmax(f[:, ::-1], axis=1)
    return tr["med"][sel][np.arange(len(last)), last]


def generate(cfg: SceneConfig, iteration: int = 0) -> Dict[str, np.ndarray]:
    """Run the light and camera passes of one iteration and return the estimator-stage inputs."""
    key = (cfg.seed, iteration)
    k = iteration_constants(cfg, iteration)
    tech = cfg.techniques
    merge_pb2d = bool(tech & PB2D)
    T = _media_tables(cfg)
    maxL = cfg.max_path_length
    min_mfp = k["bb1d_min_mfp"]
    beam_ok_med = T["scat"] & (~np.bool_(merge_pb2d) | (T["mfp"] > min_mfp))
    in_beams_med = (~np.bool_(merge_pb2d)) | (T["mfp"] > min_mfp)

    # ------------------------------------------------------------------ light pass
    NL = cfg.light_paths
    half = cfg.light_size * 0.5
    area = cfg.light_size * cfg.light_size
    lo_box, hi_box = np.asarray(cfg.boxes[0][0], float), np.asarray(cfg.boxes[0][1], float)
    cx, cz = 0.5 * (lo_box[0] + hi_box[0]), 0.5 * (lo_box[2] + hi_box[2])
    ue = uniforms(key, LIGHT_STREAM, np.arange(NL), 0, 0)
    pos0 = np.stack([cx - half + cfg.light_size * ue[:, 0], np.full(NL, hi_box[1]),
                     cz - half + cfg.light_size * ue[:, 1]], axis=1)
    u1, u2 = ue[:, 2], ue[:, 3]
    r_ = np.sqrt(u1)
    phi = 2 * math.pi * u2
    cos_l = np.maximum(np.sqrt(np.maximum(0.0, 1 - u1)), EPS_COSINE)   # SampleCosHemisphereW around -y
    dirs = np.stack([r_ * np.cos(phi), -cos_l, r_ * np.sin(phi)], axis=1)
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    emission_pdf_w = cos_l * INV_PI / area
    direct_pdf_a = np.full(NL, 1.0 / area)

    # vertex records per bounce; bounce b holds the vertices of path length b
    V: List[Dict[str, np.ndarray]] = []
    m0 = _new_mis(NL)
    m0["pdf_a_inv"] = 1.0 / direct_pdf_a
    m0["rev_pdf_a"] = cos_l
    m0["rev_pdf_a_without_bsdf"] = cos_l
    m0["ray_sample_rev_pdf_inv"] = 1.0
    m0["cos_theta_out"] = cos_l
    m0["flags"] = MIS_ON_LIGHT_SOURCE
    V.append(dict(path=np.arange(NL), pos=pos0, thr=np.ones((NL, 3)), dir_fix=np.zeros((NL, 3)), cont=np.ones(NL),
                  med=np.full(NL, -1, np.int32), flags=np.full(NL, LV_IS_FINITE, np.uint32), mis=m0))
    B: List[Dict[str, np.ndarray]] = []   # beams per bounce
    act = np.arange(NL)
    origin = pos0.copy()
    direction = dirs.copy()
    thr = np.tile(np.full(3, cfg.light_intensity), (NL, 1)) * cos_l[:, None] / emission_pdf_w[:, None]
    lpw = direct_pdf_a / emission_pdf_w
    oim = np.zeros(NL, bool)
    prev_row = np.arange(NL)          # row of each active path's last vertex in V[L-1]
    L = 1
    while act.size and maxL > 1:
        o, d = origin[act], direction[act]
        tr = _trace(cfg, flight_uniforms(key, LIGHT_STREAM, act, L, 2 * len(cfg.boxes)), o, d, oim[act])
        K = tr["K"]
        # ---- UPBP::AddBeams (UPBP.hxx:1783-1870) for the ray of this segment
        bl = []
        t3 = thr[act].copy()
        rsp = np.ones(len(act))
        rsr = np.ones(len(act))
        if cfg.photon_beam_type == SHORT_BEAM:
            for kk in range(K):
                f = tr["full"][:, kk]
                mk = tr["med"][:, kk]
                ok = f & beam_ok_med[mk]
                bl.append(dict(sel=np.nonzero(ok)[0], kk=kk, origin=o + d * tr["dmin"][:, kk:kk + 1],
                               length=tr["dmax_full"][:, kk] - tr["dmin"][:, kk], thr=t3.copy(), rsp=rsp.copy(),
                               rsr=rsr.copy(), flags=SHORT_BEAM,
                               rsf=END_IN_MEDIUM | np.where((kk == 0) & oim[act], ORIGIN_IN_MEDIUM, 0), med=mk))
                t3 = np.where(f[:, None], t3 * tr["att"][:, kk] / tr["pdf"][:, kk:kk + 1], t3)
                rsp = np.where(f, rsp * tr["pdf"][:, kk], rsp)
                rsr = np.where(f, rsr * tr["rev"][:, kk], rsr)
        else:
            first_lite = np.argmax(tr["lite"], axis=1)
            for kk in range(K):
                f = tr["lite"][:, kk]
                mk = tr["med"][:, kk]
                ok = f & beam_ok_med[mk]
                seglen = tr["dmax_lite"][:, kk] - tr["dmin"][:, kk]
                isfirst = (first_lite == kk) & oim[act]
                bl.append(dict(sel=np.nonzero(ok)[0], kk=kk, origin=o + d * tr["dmin"][:, kk:kk + 1],
                               length=seglen.copy(), thr=t3.copy(), rsp=rsp.copy(), rsr=rsr.copy(), flags=LONG_BEAM,
                               rsf=END_IN_MEDIUM | np.where(isfirst, ORIGIN_IN_MEDIUM, 0), med=mk))
                with np.errstate(invalid="ignore"):
                    t3 = np.where(f[:, None], t3 * np.exp(-T["st"][mk] * np.where(f, seglen, 0.0)[:, None]), t3)
                smin = T["smin"][mk]
                a1 = np.maximum(np.exp(-smin * np.where(f, seglen, 0.0)), 1e-35)
                samp = f & (smin > 0) & T["scat"][mk]
                rsp = np.where(samp, rsp * a1, rsp)
                rsr = np.where(samp, rsr * np.where(isfirst, smin * a1, a1), rsr)
            # cap the last beam of the ray (UPBP.hxx:1867-1868) and the configured cap
            last_k = np.full(len(act), -1)
            for e in bl:
                last_k[e["sel"]] = e["kk"]
            for e in bl:
                s = e["sel"][last_k[e["sel"]] == e["kk"]]
                cap = np.minimum(T["maxlen"][e["med"][s]], cfg.beam_length_cap)
                e["length"][s] = np.minimum(e["length"][s], cap)
        for e in bl:
            s = e["sel"]
            if s.size == 0:
                continue
            B.append(dict(path=act[s], lvlen=np.full(s.size, L - 1), kk=np.full(s.size, e["kk"]),
                          origin=e["origin"][s], direction=d[s], length=e["length"][s], thr=e["thr"][s],
                          flags=np.full(s.size, e["flags"], np.uint32), rsp=e["rsp"][s], rsr=e["rsr"][s],
                          rsf=np.asarray(e["rsf"])[s].astype(np.uint32) if np.ndim(e["rsf"]) else np.full(s.size, e["rsf"], np.uint32),
                          lpw=lpw[act[s]], med=e["med"][s]))
        # ---- scattering vertices (UPBP.hxx:560-655)
        sc = np.nonzero(np.isfinite(tr["scatter_t"]))[0]
        rsp_s, rsr_s, att_s = _full_products(tr, sc)
        pth = act[sc]
        new_thr = thr[pth] * att_s / rsp_s[:, None]
        ok = np.any(new_thr > 0, axis=1)
        sc, pth, rsp_s, rsr_s, new_thr = sc[ok], pth[ok], rsp_s[ok], rsr_s[ok], new_thr[ok]
        thr[pth] = new_thr
        st = tr["scatter_t"][sc]
        hit = o[sc] + d[sc] * st[:, None]
        mid = _last_full_medium(tr, sc)
        dist2 = st * st
        mis = _new_mis(len(sc))
        mis["pdf_a_inv"] = lpw[pth] * dist2 / rsp_s
        mis["rev_pdf_a"] = 1.0
        mis["rev_pdf_a_without_bsdf"] = 1.0
        mis["ray_sample_pdf_inv"] = 1.0 / rsp_s
        mis["ray_sample_rev_pdf_inv"] = 1.0
        mis["pp3d_factor"] = k["eta_pp3d"]
        mis["pb2d_factor"] = k["eta_pb2d"]
        mis["bb1d_factor"] = k["eta_bb1d"]
        mis["bb1d_beam_selection_pdf"] = 1.0
        mis["ray_sample_pdfs_ratio"] = 1.0 / T["smin"][mid]
        mis["ray_sample_rev_pdfs_ratio"] = 1.0 / T["smin"][mid]
        mis["flags"] = np.where(in_beams_med[mid], MIS_IN_MEDIUM_WITH_BEAMS, 0)
        pm = V[L - 1]["mis"]
        pr = prev_row[sc]
        pm["rev_pdf_a"][pr] = pm["rev_pdf_a"][pr] * rsr_s / dist2
        pm["rev_pdf_a_without_bsdf"][pr] = pm["rev_pdf_a"][pr]
        pm["ray_sample_rev_pdf_inv"][pr] = 1.0 / rsr_s
        V.append(dict(path=pth, pos=hit, thr=new_thr.copy(), dir_fix=-d[sc], cont=T["cont"][mid], med=mid.astype(np.int32),
                      flags=np.full(len(sc), LV_IN_MEDIUM | LV_CONNECTABLE | LV_IS_FINITE, np.uint32), mis=mis))
        origin[pth] = hit
        oim[pth] = True
        cont_ok = np.full(len(sc), L + 2 <= maxL)
        rows = np.nonzero(cont_ok)[0]
        if rows.size == 0:
            break
        # ---- SampleScattering (UPBP.hxx:1908-1969): HG direction, Russian roulette
        gvals = T["g"][mid[rows]]
        us = uniforms(key, LIGHT_STREAM, pth[rows], L, 0)
        wnew, pdfw, sin_t = _hg_sample(us[:, 0], us[:, 1], -d[sc[rows]], gvals)
        rr = us[:, 2]
        cont = T["cont"][mid[rows]]
        keep = ~((cont == 0) | ((cont < 1) & (rr > cont)))
        rows, wnew, pdfw, sin_t, cont = rows[keep], wnew[keep], pdfw[keep], sin_t[keep], cont[keep]
        p2 = pth[rows]
        dir_pdf = pdfw * cont
        thr[p2] = thr[p2] * T["ss"][mid[rows]] * (pdfw / dir_pdf)[:, None]
        lpw[p2] = 1.0 / dir_pdf
        cm = V[L]["mis"]
        cm["rev_pdf_a_without_bsdf"][rows] = cm["rev_pdf_a"][rows]
        cm["sin_theta"][rows] = sin_t
        cm["cos_theta_out"][rows] = 1.0
        pm["rev_pdf_a"][prev_row[sc[rows]]] *= dir_pdf   # reverse pdf of the previous vertex (HG is symmetric)
        direction[p2] = wnew
        act = p2
        prev_row = rows  # row of each surviving path's vertex in V[L], by position in act
        L += 1

    # ---- flatten light vertices in path order (path p, increasing path length)
    keys = np.concatenate([v["path"].astype(np.int64) * maxL + b for b, v in enumerate(V)])
    order = np.argsort(keys, kind="stable")
    cat = lambda f: np.concatenate([v[f] for v in V])[order]
    out: Dict[str, np.ndarray] = {}
    out["lv_position"] = cat("pos").astype(np.float32)
    out["lv_throughput"] = cat("thr").astype(np.float32)
    out["lv_dir_fix"] = cat("dir_fix").astype(np.float32)
    out["lv_cont_prob"] = cat("cont").astype(np.float32)
    out["lv_path_idx"] = cat("path").astype(np.int32)
    out["lv_path_length"] = np.concatenate([np.full(len(v["path"]), b) for b, v in enumerate(V)])[order].astype(np.int32)
    out["lv_medium_id"] = cat("med").astype(np.int32)
    out["lv_flags"] = cat("flags").astype(np.uint32)
    out["lv_mis"] = np.concatenate([v["mis"] for v in V])[order]
    out["lv_path_ends"] = np.cumsum(np.bincount(out["lv_path_idx"], minlength=NL)).astype(np.int32)
    skeys = keys[order]
    if B:
        bk = np.concatenate([b["path"].astype(np.int64) * maxL + b["lvlen"] for b in B])
        bkk = np.concatenate([b["kk"] for b in B])
        border = np.lexsort((bkk, bk))
        bcat = lambda f: np.concatenate([b[f] for b in B])[border]
        out["beam_origin"] = bcat("origin").astype(np.float32)
        out["beam_direction"] = bcat("direction").astype(np.float32)
        out["beam_length"] = bcat("length").astype(np.float32)
        out["beam_throughput"] = bcat("thr").astype(np.float32)
        out["beam_flags"] = bcat("flags").astype(np.uint32)
        out["beam_ray_sample_pdf"] = bcat("rsp").astype(np.float32)
        out["beam_ray_sample_rev_pdf"] = bcat("rsr").astype(np.float32)
        out["beam_ray_sampling_flags"] = bcat("rsf").astype(np.uint32)
        out["beam_last_pdf_w_inv"] = bcat("lpw").astype(np.float32)
        out["beam_medium_id"] = bcat("med").astype(np.int32)
        out["beam_light_vertex"] = np.searchsorted(skeys, bk[border]).astype(np.int32)
    else:
        for f, dt, sh in (("origin", np.float32, 3), ("direction", np.float32, 3), ("length", np.float32, 0),
                          ("throughput", np.float32, 3), ("flags", np.uint32, 0), ("ray_sample_pdf", np.float32, 0),
                          ("ray_sample_rev_pdf", np.float32, 0), ("ray_sampling_flags", np.uint32, 0),
                          ("last_pdf_w_inv", np.float32, 0), ("medium_id", np.int32, 0), ("light_vertex", np.int32, 0)):
            out["beam_" + f] = np.zeros((0, 3) if sh else 0, dt)

    _camera_pass(cfg, key, k, T, out)
    out["media"], out["params"] = stage_constants(cfg, iteration)
    return out


def stage_constants(cfg: SceneConfig, iteration: int = 0):
    """The media table and the per-iteration params of the estimator stage (no tracing)."""
    k = iteration_constants(cfg, iteration)
    tech = cfg.techniques
    NL = cfg.light_paths
    med = np.zeros(len(cfg.media), MEDIUM_DTYPE)
    for mi, m in enumerate(cfg.media):
        med[mi] = (m.absorption, m.scattering, m.mean_cosine, m.continuation_prob)
    prm = np.zeros(1, PARAMS_DTYPE)
    prm["techniques"] = tech
    prm["query_beam_type"] = cfg.query_beam_type
    prm["photon_beam_type"] = cfg.photon_beam_type
    prm["min_path_length"] = cfg.min_path_length
    prm["max_path_length"] = cfg.max_path_length
    prm["radius_pp3d"] = prm["radius_pb2d"] = prm["radius_bb1d"] = k["radius"]
    prm["mis_factor_surf"] = k["eta_surf"]
    prm["mis_factor_pp3d"] = k["eta_pp3d"]
    prm["mis_factor_pb2d"] = k["eta_pb2d"]
    prm["mis_factor_bb1d"] = k["eta_bb1d"]
    prm["norm_pp3d"] = k["norm_pp3d"]
    prm["norm_pb2d"] = k["norm_pb2d"]
    prm["norm_bb1d"] = k["norm_bb1d"]
    prm["bb1d_min_mfp"] = k["bb1d_min_mfp"]
    prm["min_dist_to_med"] = cfg.min_dist_to_med
    prm["hash_cells"] = NL
    prm["image_width"] = cfg.width
    prm["image_height"] = cfg.height
    prm["pb2d_knn"] = cfg.pb2d_knn
    prm["bb1d_knn"] = cfg.bb1d_knn
    return med, prm


def _camera_pass(cfg: SceneConfig, key, k: Dict[str, float], T, out: Dict[str, np.ndarray]):
    """Camera sub-paths (UPBP.hxx:742-1160): one segment query per traced ray that crosses a scattering
    medium and one PP3D point query per camera medium vertex, each with the snapshot of
    mCameraVerticesMisData at the call.  The records are stored per pixel in call order: for
    each camera path length L, the segment query, then the point query (and their snapshots)."""
    W_, H_ = cfg.width, cfg.height
    npix = W_ * H_
    tech = cfg.techniques
    merge_pb2d = bool(tech & PB2D)
    maxL = cfg.max_path_length
    in_beams_med = (~np.bool_(merge_pb2d)) | (T["mfp"] > k["bb1d_min_mfp"])
    cam = np.asarray(cfg.camera_pos, np.float64)
    tan_half = math.tan(math.radians(cfg.fov_deg) * 0.5)
    ipd = W_ / (2.0 * tan_half)
    pix = np.arange(npix)
    uj = uniforms(key, CAMERA_STREAM, pix, 0, 0)
    sx = (pix % W_ + uj[:, 0]) - W_ * 0.5
    sy = (pix // W_ + uj[:, 1]) - H_ * 0.5
    d_all = np.stack([sx, -sy, np.full(npix, ipd)], axis=1)
    d_all /= np.linalg.norm(d_all, axis=1, keepdims=True)
    cos_cam = d_all[:, 2]
    cam_pdf_w = (ipd / cos_cam) ** 2 / cos_cam
    # active state
    act = pix.copy()
    d = d_all
    o = np.tile(cam, (npix, 1))
    thr = np.ones((npix, 3))
    lpw = float(npix) / cam_pdf_w
    oim = np.zeros(npix, bool)
    stop_bb1d = np.zeros(npix, bool)
    table = np.zeros((npix, maxL + 1), MIS_DTYPE)
    table["rev_pdf_a"][:, 0] = 1.0
    Q: List[dict] = []
    S: List[dict] = []
    PQ: List[dict] = []
    CR: List[np.ndarray] = []
    n_cam = 0
    n_seg = 0
    kstride = 2 * (maxL + 2)  # record order key: pixel, path length, segment before point query
    L = 1
    while act.size:
        tr = _trace(cfg, flight_uniforms(key, CAMERA_STREAM, act, L, 2 * len(cfg.boxes)), o, d, oim)
        sc_mask = np.isfinite(tr["scatter_t"])
        use_lite = sc_mask & (cfg.query_beam_type == LONG_BEAM)
        seg_mask = np.where(use_lite[:, None], tr["lite"], tr["full"])
        dmax = np.where(use_lite[:, None], tr["dmax_lite"], tr["dmax_full"])
        has_med = np.any(seg_mask & T["scat"][tr["med"]], axis=1)
        qr = np.nonzero(has_med)[0]
        if qr.size:
            qf = (np.where(oim[qr], Q_ORIGIN_IN_MEDIUM, 0) | np.where(use_lite[qr], Q_LITE, 0)).astype(np.uint32)
            if tech & PB2D:
                qf |= Q_PB2D
            if tech & BB1D:
                qf |= np.where(stop_bb1d[qr], 0, Q_BB1D).astype(np.uint32)
            cnt = seg_mask[qr].sum(axis=1)
            sm = seg_mask[qr]
            ii, kk = np.nonzero(sm)
            rows = qr[ii]
            lite_rows = use_lite[rows]
            S.append(dict(dmin=tr["dmin"][rows, kk], dmax=dmax[rows, kk],
                          pdf=np.where(lite_rows, 1.0, tr["pdf"][rows, kk]),
                          rev=np.where(lite_rows, 1.0, tr["rev"][rows, kk]),
                          att=np.where(lite_rows[:, None], 1.0, tr["att"][rows, kk]), med=tr["med"][rows, kk]))
            begin = n_seg + np.concatenate([[0], np.cumsum(cnt)[:-1]])
            n_seg += int(cnt.sum())
            snap = table[qr, :L].reshape(-1)
            CR.append(snap)
            Q.append(dict(origin=o[qr], direction=d[qr], seg_begin=begin, seg_count=cnt, flags=qf,
                          path_length=np.full(qr.size, L), lpw=lpw[qr], thr=thr[qr], pixel=act[qr],
                          cam_begin=n_cam + np.arange(qr.size) * L, key=act[qr].astype(np.int64) * kstride + 2 * L))
            n_cam += snap.size
        # scattering events: camera vertex in a medium
        sc = np.nonzero(sc_mask)[0]
        if sc.size == 0:
            break
        rsp, rsr, att = _full_products(tr, sc)
        nthr = thr[sc] * att / rsp[:, None]
        ok = np.any(nthr > 0, axis=1)
        sc, rsp, rsr, nthr = sc[ok], rsp[ok], rsr[ok], nthr[ok]
        thr[sc] = nthr
        st = tr["scatter_t"][sc]
        hit = o[sc] + d[sc] * st[:, None]
        mid = _last_full_medium(tr, sc)
        dist2 = st * st
        rec = table[sc, L]
        rec["pdf_a_inv"] = lpw[sc] * dist2 / rsp
        rec["rev_pdf_a"] = 1.0
        rec["ray_sample_pdf_inv"] = 1.0 / rsp
        rec["ray_sample_rev_pdf_inv"] = 1.0
        rec["ray_sample_pdfs_ratio"] = 1.0 / T["smin"][mid]
        rec["ray_sample_rev_pdfs_ratio"] = 1.0 / T["smin"][mid]
        rec["pp3d_factor"] = k["eta_pp3d"]
        rec["pb2d_factor"] = k["eta_pb2d"]
        rec["bb1d_factor"] = k["eta_bb1d"]
        rec["bb1d_beam_selection_pdf"] = 1.0
        rec["flags"] = np.where(in_beams_med[mid], MIS_IN_MEDIUM_WITH_BEAMS, 0)
        table[sc, L] = rec
        prev = table[sc, L - 1]
        prev["rev_pdf_a"] = prev["rev_pdf_a"] * rsr / dist2
        prev["ray_sample_rev_pdf_inv"] = 1.0 / rsr
        table[sc, L - 1] = prev
        if L >= maxL:
            break
        pq_ok = (L > 1) | (st >= cfg.min_dist_to_med)
        if tech & PP3D:
            r = np.nonzero(pq_ok)[0]
            if r.size:
                snap = table[sc[r], :L + 1].reshape(-1)
                CR.append(snap)
                PQ.append(dict(position=hit[r], dir_fix=-d[sc[r]], medium=mid[r], path_length=np.full(r.size, L),
                               thr=nthr[r], pixel=act[sc[r]], cam_begin=n_cam + np.arange(r.size) * (L + 1),
                               key=act[sc[r]].astype(np.int64) * kstride + 2 * L + 1))
                n_cam += snap.size
        # SampleScattering at the camera vertex
        us = uniforms(key, CAMERA_STREAM, act[sc], L, 0)
        wnew, pdfw, sin_t = _hg_sample(us[:, 0], us[:, 1], -d[sc], T["g"][mid])
        rr = us[:, 2]
        cont = T["cont"][mid]
        keep = ~((cont == 0) | ((cont < 1) & (rr > cont)))
        sc, mid, wnew, pdfw, sin_t, cont, hit = sc[keep], mid[keep], wnew[keep], pdfw[keep], sin_t[keep], cont[keep], hit[keep]
        dir_pdf = pdfw * cont
        thr[sc] = thr[sc] * T["ss"][mid] * (pdfw / dir_pdf)[:, None]
        cur = table[sc, L]
        cur["sin_theta"] = sin_t
        cur["cos_theta_out"] = 1.0
        table[sc, L] = cur
        prev = table[sc, L - 1]
        prev["rev_pdf_a"] = prev["rev_pdf_a"] * dir_pdf
        table[sc, L - 1] = prev
        if tech & BB1D_PREVIOUS:
            stop_bb1d[sc] = True
        # compact the active set
        act, table, thr, stop_bb1d = act[sc], table[sc], thr[sc], stop_bb1d[sc]
        lpw = 1.0 / dir_pdf
        o, d, oim = hit, wnew, np.ones(sc.size, bool)
        L += 1

    cat = lambda lst, f, dt: (np.concatenate([x[f] for x in lst]) if lst else np.zeros(0)).astype(dt)
    nq = sum(len(x["flags"]) for x in Q)
    npq = sum(len(x["pixel"]) for x in PQ)
    # per-pixel call order (the records were produced bounce by bounce)
    qkey, pqkey = cat(Q, "key", np.int64), cat(PQ, "key", np.int64)
    oq, opq = np.argsort(qkey, kind="stable"), np.argsort(pqkey, kind="stable")
    cam_all = np.concatenate(CR) if CR else np.zeros(0, MIS_DTYPE)
    bkey = np.concatenate([qkey, pqkey])
    blen = np.concatenate([cat(Q, "path_length", np.int64), cat(PQ, "path_length", np.int64) + 1])
    bbeg = np.concatenate([cat(Q, "cam_begin", np.int64), cat(PQ, "cam_begin", np.int64)])
    ob = np.argsort(bkey, kind="stable")
    nb_sorted = np.concatenate([[0], np.cumsum(blen[ob])[:-1]]).astype(np.int64) if ob.size else np.zeros(0, np.int64)
    new_beg = np.empty_like(nb_sorted)
    new_beg[ob] = nb_sorted
    out["cam_mis"] = cam_all[np.repeat(bbeg[ob] - nb_sorted, blen[ob]) + np.arange(int(blen.sum()))]
    sbeg, scnt = cat(Q, "seg_begin", np.int64)[oq], cat(Q, "seg_count", np.int64)[oq]
    nsb = np.concatenate([[0], np.cumsum(scnt)[:-1]]).astype(np.int64) if nq else np.zeros(0, np.int64)
    sidx = np.repeat(sbeg - nsb, scnt) + np.arange(int(scnt.sum()))
    qcat = lambda f, dt: cat(Q, f, dt)[oq]
    q3 = lambda f: (np.concatenate([x[f] for x in Q])[oq] if Q else np.zeros((0, 3))).astype(np.float32).reshape(nq, 3)
    out["sq_origin"] = q3("origin")
    out["sq_direction"] = q3("direction")
    out["sq_seg_begin"] = nsb.astype(np.int32)
    out["sq_seg_count"] = scnt.astype(np.int32)
    out["sq_flags"] = qcat("flags", np.uint32)
    out["sq_path_length"] = qcat("path_length", np.int32)
    out["sq_last_pdf_w_inv"] = qcat("lpw", np.float32)
    out["sq_throughput"] = q3("thr")
    out["sq_pixel"] = qcat("pixel", np.int32)
    out["sq_cam_mis_begin"] = new_beg[:nq][oq].astype(np.int64)
    ns = int(scnt.sum())
    scat = lambda f, dt: cat(S, f, dt)[sidx]
    out["seg_dist_min"] = scat("dmin", np.float32)
    out["seg_dist_max"] = scat("dmax", np.float32)
    out["seg_pdf"] = scat("pdf", np.float32)
    out["seg_rev_pdf"] = scat("rev", np.float32)
    out["seg_attenuation"] = (np.concatenate([x["att"] for x in S])[sidx] if S else np.zeros((0, 3))).astype(np.float32).reshape(ns, 3)
    out["seg_medium"] = scat("med", np.int32)
    pcat = lambda f, dt: cat(PQ, f, dt)[opq]
    p3 = lambda f: (np.concatenate([x[f] for x in PQ])[opq] if PQ else np.zeros((0, 3))).astype(np.float32).reshape(npq, 3)
    out["pq_position"] = p3("position")
    out["pq_dir_fix"] = p3("dir_fix")
    out["pq_medium_id"] = pcat("medium", np.int32)
    out["pq_path_length"] = pcat("path_length", np.int32)
    out["pq_throughput"] = p3("thr")
    out["pq_pixel"] = pcat("pixel", np.int32)
    out["pq_cam_mis_begin"] = new_beg[nq:][opq].astype(np.int64)


# ----------------------------------------------------------------------------------------------
# Closest-approach precision stress (beam-beam geometry only)

def _stress_directions(rng: np.random.Generator, n: int, parallel_fraction: float, max_angle: float):
    """Unit directions: a ``parallel_fraction`` share within ``max_angle`` (uniform angle) of +z, the
    rest uniform on the sphere."""
    par = rng.random(n) < parallel_fraction
    theta = np.where(par, rng.random(n) * max_angle, np.arccos(1.0 - 2.0 * rng.random(n)))
    phi = 2.0 * math.pi * rng.random(n)
    st = np.sin(theta)
    d = np.stack([st * np.cos(phi), st * np.sin(phi), np.cos(theta)], axis=1)
    return d, par


def beam_stress(n_beams: int, n_queries: int, radius: float = 0.002, sigma_t: float = 2.0,
                parallel_fraction: float = 0.5, max_angle: float = 1e-4, seed: int = 1234,
                base_light_paths: int = 4096, base_size: int = 64) -> Dict[str, np.ndarray]:
    """BB1D closest-approach stress workload: ``n_beams`` photon beams and ``n_queries`` query rays
    with origins uniform in [0,1]^3, half of both (``parallel_fraction``) within ``max_angle`` rad of
    a common axis and half isotropic, lengths exponential with rate ``sigma_t``, radius ``radius``.

    The geometry is the stress; every other record comes from one ordinary cube iteration (radius
    ``radius``, medium with sigma_t = ``sigma_t``), whose beam and query records are reused
    cyclically: beam throughputs, pdfs, flags and light-vertex links (so the light-side MIS records
    stay valid), and the queries' camera MIS snapshots, path lengths, throughputs and pixels.  Each
    query becomes one full segment [0, length) in the medium with only BB1D enabled; there are no
    point queries.
    """
    ss = 0.8 * sigma_t
    med = Medium((sigma_t - ss,) * 3, (ss,) * 3, 0.3, 0.8)
    cfg = SceneConfig("stress_base", [CLEAR, med], [((0, 0, 0), (1, 1, 1), 1)], base_size, base_size,
                      base_light_paths, 6, radius, seed=seed)
    w = generate(cfg, 0)
    rng = np.random.Generator(np.random.Philox(key=seed + 7919))
    nb0, nq0 = len(w["beam_length"]), len(w["sq_path_length"])
    if nb0 == 0 or nq0 == 0:
        raise ValueError("base iteration has no beams or no segment queries")
    bi = np.arange(n_beams) % nb0
    for k in [k for k in w if k.startswith("beam_")]:
        w[k] = np.ascontiguousarray(w[k][bi])
    w["beam_origin"] = rng.random((n_beams, 3)).astype(np.float32)
    d, _ = _stress_directions(rng, n_beams, parallel_fraction, max_angle)
    w["beam_direction"] = d.astype(np.float32)
    w["beam_length"] = (-np.log1p(-rng.random(n_beams)) / sigma_t).astype(np.float32)
    w["beam_medium_id"] = np.ones(n_beams, np.int32)

    qi = np.arange(n_queries) % nq0
    for k in ("sq_path_length", "sq_last_pdf_w_inv", "sq_throughput", "sq_pixel", "sq_cam_mis_begin"):
        w[k] = np.ascontiguousarray(w[k][qi])
    w["sq_flags"] = ((w["sq_flags"][qi] & Q_ORIGIN_IN_MEDIUM) | Q_BB1D).astype(np.uint32)
    w["sq_origin"] = rng.random((n_queries, 3)).astype(np.float32)
    d, _ = _stress_directions(rng, n_queries, parallel_fraction, max_angle)
    w["sq_direction"] = d.astype(np.float32)
    w["sq_seg_begin"] = np.arange(n_queries, dtype=np.int32)
    w["sq_seg_count"] = np.ones(n_queries, np.int32)
    length = (-np.log1p(-rng.random(n_queries)) / sigma_t).astype(np.float32)
    w["seg_dist_min"] = np.zeros(n_queries, np.float32)
    w["seg_dist_max"] = length
    w["seg_pdf"] = np.exp(-sigma_t * length.astype(np.float64)).astype(np.float32)
    w["seg_rev_pdf"] = w["seg_pdf"].copy()
    w["seg_attenuation"] = np.repeat(w["seg_pdf"][:, None], 3, axis=1).astype(np.float32)
    w["seg_medium"] = np.ones(n_queries, np.int32)
    for k in ("pq_position", "pq_dir_fix", "pq_throughput"):
        w[k] = np.zeros((0, 3), np.float32)
    for k, dt in (("pq_medium_id", np.int32), ("pq_path_length", np.int32), ("pq_pixel", np.int32),
                  ("pq_cam_mis_begin", np.int64)):
        w[k] = np.zeros(0, dt)
    return w


def make(cfg: SceneConfig, iteration: int = 0) -> Dict[str, np.ndarray]:
    """The estimator-stage inputs of one iteration of configuration ``cfg``."""
    if cfg.name == "beamstress":
        return beam_stress(2_000_000, 2_000_000, radius=cfg.radius, seed=cfg.seed + iteration)
    return generate(cfg, iteration)


def without_mis(w: Dict[str, np.ndarray], techniques: int = PB2D | BB1D) -> Dict[str, np.ndarray]:
    """The workload as VolLightTracer's pure algorithms query it (Renderers/VolLightTracer.hxx:296-412):
    the same photons, beams and camera segments, the estimators without MIS (``NO_MIS`` with PB2D
    and/or BB1D), no point queries (the reference has no pure PP3D), and the MIS-only arrays left
    out."""
    out = {k: v for k, v in w.items() if k not in MIS_ONLY_INPUTS and not k.startswith("pq_")}
    p = w["params"].copy()
    p["techniques"] = (int(techniques) & (PB2D | BB1D | BP2D)) | NO_MIS
    out["params"] = p
    out["pq_position"] = np.zeros((0, 3), np.float32)
    out["pq_dir_fix"] = np.zeros((0, 3), np.float32)
    for k in ("pq_medium_id", "pq_path_length", "pq_pixel"):
        out[k] = np.zeros(0, np.int32)
    out["pq_throughput"] = np.zeros((0, 3), np.float32)
    out["pq_cam_mis_begin"] = np.zeros(0, np.int64)
    return out
