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
"""
from __future__ import annotations

import dataclasses
import math
from typing import Dict, List, Sequence, Tuple

import numpy as np

# flags, identical to include/upbp_gpu.h (and the reference enums)
SHORT_BEAM, LONG_BEAM = 1, 2
BPT, SURF, PP3D, PB2D, BB1D = 4, 8, 16, 32, 64
NO_SINE_IN_WEIGHTS, PREVIOUS, COMPATIBLE, BB1D_PREVIOUS = 128, 256, 512, 1024
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
)
PARAMS_DTYPE = np.dtype(list(PARAMS_FIELDS))

EPS_COSINE = 1e-6
INV_PI = 1.0 / math.pi


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
    if name == "boxes3":       # heavy-tailed: nested sigma_t 0.05 / 1 / 10
        return nested_boxes_scene()
    if name == "diff512":      # differentiable-estimator scene: 512^2, 262,144 light paths
        return cube_scene("diff512", 512, 512, 262_144, 6, 0.01)
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


def _trace(cfg: SceneConfig, rng: np.random.Generator, o: np.ndarray, d: np.ndarray, origin_in_medium: np.ndarray):
    """Scene::Intersect for imaginary-boundary media: split the ray into medium segments and sample a
    free-flight distance in each scattering medium in order (HomogeneousMedium::SampleRay,
    Scene/Media.hxx:240-290).  Returns per-ray lists of full segments (up to the scattering point)
    and lite segments (the whole traversal), plus the scattering distance (inf when the ray leaves).
    """
    n = o.shape[0]
    breaks = _box_breaks(cfg, o, d)
    K = breaks.shape[1]
    starts = np.concatenate([np.zeros((n, 1)), breaks[:, :-1]], axis=1) if K else np.zeros((n, 0))
    ends = breaks
    full: List[list] = [[] for _ in range(n)]
    lite: List[list] = [[] for _ in range(n)]
    scatter_t = np.full(n, np.inf)
    alive = np.ones(n, bool)
    first = np.ones(n, bool)
    for k in range(K):
        s0 = starts[:, k]
        s1 = ends[:, k]
        valid = np.isfinite(s1) & (s1 > s0)
        mid = o + d * ((s0 + np.where(np.isfinite(s1), s1, s0 + 1.0)) * 0.5)[:, None]
        med = _medium_at(cfg, mid)
        u = rng.random(n)
        for i in np.nonzero(valid)[0]:
            m = cfg.media[med[i]]
            seglen = s1[i] - s0[i]
            if med[i] == 0 and not m.has_scattering:
                flags_first = first[i]
                if alive[i]:
                    full[i].append((s0[i], s1[i], 1.0, 1.0, (1.0, 1.0, 1.0), int(med[i])))
                first[i] = False
                continue
            lite[i].append((s0[i], s1[i], int(med[i])))
            if not alive[i]:
                first[i] = False
                continue
            st = m.sigma_t
            smin = m.min_pos_sigma_t
            rflags = ORIGIN_IN_MEDIUM if (first[i] and origin_in_medium[i]) else 0
            if smin > 0 and m.has_scattering:
                s = -math.log(max(u[i], 1e-300)) / smin
                if s < seglen:
                    att1 = math.exp(-smin * s)
                    pdf = smin * att1
                    rev = pdf if rflags & ORIGIN_IN_MEDIUM else att1
                    a = tuple(np.exp(-st * s))
                    full[i].append((s0[i], s0[i] + s, pdf, rev, a, int(med[i])))
                    scatter_t[i] = s0[i] + s
                    alive[i] = False
                else:
                    att1 = math.exp(-smin * seglen)
                    pdf = att1
                    rev = smin * att1 if rflags & ORIGIN_IN_MEDIUM else att1
                    a = tuple(np.exp(-st * seglen))
                    full[i].append((s0[i], s1[i], pdf, rev, a, int(med[i])))
            else:
                a = tuple(np.exp(-st * seglen))
                full[i].append((s0[i], s1[i], 1.0, 1.0, a, int(med[i])))
            first[i] = False
    return full, lite, scatter_t


def _hg_sample(rng: np.random.Generator, wfix: np.ndarray, g: np.ndarray):
    """PhaseFunction::Sample (Path/PhaseFunction.hxx:82-137): returns (direction, pdf, sinTheta)."""
    n = wfix.shape[0]
    u1, u2 = rng.random(n), rng.random(n)
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


def generate(cfg: SceneConfig, iteration: int = 0) -> Dict[str, np.ndarray]:
    """Run the light and camera passes of one iteration and return the estimator-stage inputs."""
    rng = np.random.Generator(np.random.Philox(key=cfg.seed + iteration))
    k = iteration_constants(cfg, iteration)
    tech = cfg.techniques
    merge_pb2d = bool(tech & PB2D)
    media = cfg.media

    # ------------------------------------------------------------------ light pass
    NL = cfg.light_paths
    half = cfg.light_size * 0.5
    area = cfg.light_size * cfg.light_size
    lo_box, hi_box = np.asarray(cfg.boxes[0][0], float), np.asarray(cfg.boxes[0][1], float)
    cx, cz = 0.5 * (lo_box[0] + hi_box[0]), 0.5 * (lo_box[2] + hi_box[2])
    pos = np.stack([cx - half + cfg.light_size * rng.random(NL), np.full(NL, hi_box[1]),
                    cz - half + cfg.light_size * rng.random(NL)], axis=1)
    u1, u2 = rng.random(NL), rng.random(NL)
    # SampleCosHemisphereW around the light normal (-y)
    r_ = np.sqrt(u1)
    phi = 2 * math.pi * u2
    cos_l = np.maximum(np.sqrt(np.maximum(0.0, 1 - u1)), EPS_COSINE)
    dirs = np.stack([r_ * np.cos(phi), -cos_l, r_ * np.sin(phi)], axis=1)
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    emission_pdf_w = cos_l * INV_PI / area
    direct_pdf_a = np.full(NL, 1.0 / area)

    lv: Dict[str, list] = {k_: [] for k_ in ("position", "throughput", "dir_fix", "cont_prob", "path_idx",
                                              "path_length", "medium_id", "flags", "mis")}
    beams: Dict[str, list] = {k_: [] for k_ in ("origin", "direction", "length", "throughput", "flags",
                                                 "ray_sample_pdf", "ray_sample_rev_pdf", "ray_sampling_flags",
                                                 "last_pdf_w_inv", "medium_id", "light_vertex")}
    path_ends = np.zeros(NL, np.int32)

    # per-path state arrays
    thr = np.tile(np.full(3, cfg.light_intensity), (NL, 1)) * cos_l[:, None] / emission_pdf_w[:, None]
    last_pdf_w_inv = direct_pdf_a / emission_pdf_w
    origin = pos.copy()
    direction = dirs.copy()
    origin_in_med = np.zeros(NL, bool)
    # records are appended path by path; to keep paths contiguous we build per-path lists first
    per_path_lv: List[list] = [[] for _ in range(NL)]
    per_path_beams: List[list] = [[] for _ in range(NL)]
    for p in range(NL):
        per_path_lv[p].append(dict(
            position=pos[p], throughput=(1.0, 1.0, 1.0), dir_fix=(0.0, 0.0, 0.0), cont_prob=1.0, path_idx=p,
            path_length=0, medium_id=-1, flags=LV_IS_FINITE,
            mis=dict(pdf_a_inv=1.0 / direct_pdf_a[p], rev_pdf_a=cos_l[p], rev_pdf_a_without_bsdf=cos_l[p],
                     ray_sample_pdf_inv=0.0, ray_sample_rev_pdf_inv=1.0, cos_theta_out=cos_l[p],
                     flags=MIS_ON_LIGHT_SOURCE)))
    active = np.arange(NL)
    path_len = 1
    while active.size and cfg.max_path_length > 1:
        o = origin[active]
        d = direction[active]
        full, lite, st = _trace(cfg, rng, o, d, origin_in_med[active])
        # AddBeams (UPBP.hxx:532-535 -> 1783-1870) from the ray of this segment
        for j, p in enumerate(active):
            prev_idx = len(per_path_lv[p]) - 1
            oflag = ORIGIN_IN_MEDIUM if origin_in_med[p] else 0
            t3 = np.array(thr[p], np.float64)
            rsp, rsr = 1.0, 1.0
            if cfg.photon_beam_type == SHORT_BEAM:
                for si, (d0, d1, pdf, rev, att, mid) in enumerate(full[j]):
                    m = media[mid]
                    if m.has_scattering and (not merge_pb2d or m.mfp > k["bb1d_min_mfp"]):
                        per_path_beams[p].append(dict(
                            origin=o[j] + d[j] * d0, direction=d[j], length=d1 - d0, throughput=t3.copy(),
                            flags=SHORT_BEAM, ray_sample_pdf=rsp, ray_sample_rev_pdf=rsr,
                            ray_sampling_flags=END_IN_MEDIUM | (oflag if si == 0 else 0),
                            last_pdf_w_inv=last_pdf_w_inv[p], medium_id=mid, light_vertex=prev_idx))
                    t3 = t3 * np.asarray(att) / pdf
                    rsp *= pdf
                    rsr *= rev
            else:
                lite_all = [(s0, s1, mid) for (s0, s1, mid) in lite[j]]
                for si, (d0, d1, mid) in enumerate(lite_all):
                    m = media[mid]
                    added = False
                    if m.has_scattering and (not merge_pb2d or m.mfp > k["bb1d_min_mfp"]):
                        per_path_beams[p].append(dict(
                            origin=o[j] + d[j] * d0, direction=d[j], length=d1 - d0, throughput=t3.copy(),
                            flags=LONG_BEAM, ray_sample_pdf=rsp, ray_sample_rev_pdf=rsr,
                            ray_sampling_flags=END_IN_MEDIUM | (oflag if si == 0 else 0),
                            last_pdf_w_inv=last_pdf_w_inv[p], medium_id=mid, light_vertex=prev_idx))
                        added = True
                    seglen = d1 - d0
                    t3 = t3 * np.exp(-m.sigma_t * seglen)
                    smin = m.min_pos_sigma_t
                    if smin > 0 and m.has_scattering:
                        att1 = max(math.exp(-smin * seglen), 1e-35)
                        spdf = att1
                        srev = smin * att1 if (si == 0 and oflag) else att1
                    else:
                        spdf = srev = 1.0
                    rsp *= spdf
                    rsr *= srev
                # cap the last beam of this ray (UPBP.hxx:1867-1868; config cap on top)
                if per_path_beams[p] and per_path_beams[p][-1]["light_vertex"] == prev_idx:
                    b = per_path_beams[p][-1]
                    cap = min(media[b["medium_id"]].sigma_t.max() and (-math.log(1e-9) / media[b["medium_id"]].sigma_t.max()) or math.inf,
                              cfg.beam_length_cap)
                    if b["length"] > cap:
                        b["length"] = cap
        # intersect: scattering vertices
        nxt = []
        scattered = np.isfinite(st)
        for j, p in enumerate(active):
            if not scattered[j]:
                continue
            segs = full[j]
            rsp = float(np.prod([s[2] for s in segs])) if segs else 1.0
            rsr = float(np.prod([s[3] for s in segs])) if segs else 1.0
            att = np.prod(np.asarray([s[4] for s in segs]), axis=0) if segs else np.ones(3)
            thr[p] = thr[p] * att / rsp
            if not np.any(thr[p] > 0):
                continue
            mid = segs[-1][5]
            m = media[mid]
            hit = o[j] + d[j] * st[j]
            dist2 = st[j] * st[j]
            rsp_inv = 1.0 / rsp
            flags = 0
            if (not merge_pb2d) or m.mfp > k["bb1d_min_mfp"]:
                flags |= MIS_IN_MEDIUM_WITH_BEAMS
            ratio = 1.0 / m.min_pos_sigma_t
            rec = dict(pdf_a_inv=last_pdf_w_inv[p] * dist2 * rsp_inv, rev_pdf_a=1.0, rev_pdf_a_without_bsdf=1.0,
                       ray_sample_pdf_inv=rsp_inv, ray_sample_rev_pdf_inv=1.0, sin_theta=0.0, cos_theta_out=0.0,
                       surf_factor=0.0, pp3d_factor=k["eta_pp3d"], pb2d_factor=k["eta_pb2d"],
                       bb1d_factor=k["eta_bb1d"], bb1d_beam_selection_pdf=1.0,
                       ray_sample_pdfs_ratio=ratio, ray_sample_rev_pdfs_ratio=ratio, flags=flags)
            prev = per_path_lv[p][-1]["mis"]
            prev["rev_pdf_a"] = prev.get("rev_pdf_a", 0.0) * rsr / dist2
            prev["rev_pdf_a_without_bsdf"] = prev["rev_pdf_a"]
            prev["ray_sample_rev_pdf_inv"] = 1.0 / rsr
            per_path_lv[p].append(dict(position=hit, throughput=thr[p].copy(), dir_fix=-d[j],
                                       cont_prob=m.continuation_prob, path_idx=p, path_length=path_len,
                                       medium_id=mid, flags=LV_IN_MEDIUM | LV_CONNECTABLE | LV_IS_FINITE, mis=rec))
            origin[p] = hit
            origin_in_med[p] = True
            if path_len + 2 > cfg.max_path_length:
                continue
            nxt.append((j, p))
        if not nxt:
            break
        js = np.array([j for j, _ in nxt])
        ps = np.array([p for _, p in nxt])
        gs = np.array([media[per_path_lv[p][-1]["medium_id"]].mean_cosine for p in ps])
        wfix = -d[js]
        wnew, pdfw, sin_t = _hg_sample(rng, wfix, gs)
        rr = rng.random(len(ps))
        cont = np.array([media[per_path_lv[p][-1]["medium_id"]].continuation_prob for p in ps])
        keep = ~((cont == 0) | ((cont < 1) & (rr > cont)))
        survivors = []
        for t_, p in enumerate(ps):
            if not keep[t_]:
                continue
            m = media[per_path_lv[p][-1]["medium_id"]]
            dir_pdf = pdfw[t_] * cont[t_]
            rev_pdf = pdfw[t_] * cont[t_]  # HG is symmetric: reverse pdf equals forward pdf
            thr[p] = thr[p] * np.asarray(m.scattering) * pdfw[t_] / dir_pdf
            last_pdf_w_inv[p] = 1.0 / dir_pdf
            cur = per_path_lv[p][-1]["mis"]
            cur["rev_pdf_a_without_bsdf"] = cur["rev_pdf_a"]
            cur["sin_theta"] = sin_t[t_]
            cur["cos_theta_out"] = 1.0
            per_path_lv[p][-2]["mis"]["rev_pdf_a"] *= rev_pdf
            direction[p] = wnew[t_]
            survivors.append(p)
        active = np.array(survivors, dtype=np.int64)
        path_len += 1

    # flatten light vertices and beams
    lv_base = np.zeros(NL + 1, np.int64)
    for p in range(NL):
        lv_base[p + 1] = lv_base[p] + len(per_path_lv[p])
    n_lv = int(lv_base[-1])
    out: Dict[str, np.ndarray] = {}
    out["lv_position"] = np.zeros((n_lv, 3), np.float32)
    out["lv_throughput"] = np.zeros((n_lv, 3), np.float32)
    out["lv_dir_fix"] = np.zeros((n_lv, 3), np.float32)
    out["lv_cont_prob"] = np.zeros(n_lv, np.float32)
    out["lv_path_idx"] = np.zeros(n_lv, np.int32)
    out["lv_path_length"] = np.zeros(n_lv, np.int32)
    out["lv_medium_id"] = np.zeros(n_lv, np.int32)
    out["lv_flags"] = np.zeros(n_lv, np.uint32)
    mis = np.zeros(n_lv, MIS_DTYPE)
    bl = []
    i = 0
    for p in range(NL):
        for v in per_path_lv[p]:
            out["lv_position"][i] = v["position"]
            out["lv_throughput"][i] = v["throughput"]
            out["lv_dir_fix"][i] = v["dir_fix"]
            out["lv_cont_prob"][i] = v["cont_prob"]
            out["lv_path_idx"][i] = v["path_idx"]
            out["lv_path_length"][i] = v["path_length"]
            out["lv_medium_id"][i] = v["medium_id"]
            out["lv_flags"][i] = v["flags"]
            mis[i] = _mis_record(**v["mis"])
            i += 1
        path_ends[p] = i
        for b in per_path_beams[p]:
            b = dict(b)
            b["light_vertex"] = int(lv_base[p] + b["light_vertex"])
            bl.append(b)
    out["lv_mis"] = mis
    out["lv_path_ends"] = path_ends
    nb = len(bl)
    out["beam_origin"] = np.array([b["origin"] for b in bl], np.float32).reshape(nb, 3)
    out["beam_direction"] = np.array([b["direction"] for b in bl], np.float32).reshape(nb, 3)
    out["beam_length"] = np.array([b["length"] for b in bl], np.float32)
    out["beam_throughput"] = np.array([b["throughput"] for b in bl], np.float32).reshape(nb, 3)
    out["beam_flags"] = np.array([b["flags"] for b in bl], np.uint32)
    out["beam_ray_sample_pdf"] = np.array([b["ray_sample_pdf"] for b in bl], np.float32)
    out["beam_ray_sample_rev_pdf"] = np.array([b["ray_sample_rev_pdf"] for b in bl], np.float32)
    out["beam_ray_sampling_flags"] = np.array([b["ray_sampling_flags"] for b in bl], np.uint32)
    out["beam_last_pdf_w_inv"] = np.array([b["last_pdf_w_inv"] for b in bl], np.float32)
    out["beam_medium_id"] = np.array([b["medium_id"] for b in bl], np.int32)
    out["beam_light_vertex"] = np.array([b["light_vertex"] for b in bl], np.int32)

    # ------------------------------------------------------------------ camera pass
    _camera_pass(cfg, rng, k, out)

    # ------------------------------------------------------------------ media / params
    med = np.zeros(len(media), MEDIUM_DTYPE)
    for mi, m in enumerate(media):
        med[mi] = (m.absorption, m.scattering, m.mean_cosine, m.continuation_prob)
    out["media"] = med
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
    out["params"] = prm
    return out


def _camera_pass(cfg: SceneConfig, rng: np.random.Generator, k: Dict[str, float], out: Dict[str, np.ndarray]):
    """Camera sub-paths (UPBP.hxx:742-1160): record one segment query per traced ray and one PP3D point
    query per medium vertex, each with the snapshot of the camera MIS records at the call."""
    W, H = cfg.width, cfg.height
    npix = W * H
    media = cfg.media
    tech = cfg.techniques
    merge_pb2d = bool(tech & PB2D)
    cam = np.asarray(cfg.camera_pos, np.float64)
    tan_half = math.tan(math.radians(cfg.fov_deg) * 0.5)
    image_plane_dist = W / (2.0 * tan_half)
    pix = np.arange(npix)
    px, py = pix % W, pix // W
    jx, jy = rng.random(npix), rng.random(npix)
    sx = (px + jx) - W * 0.5
    sy = (py + jy) - H * 0.5
    d = np.stack([sx, -sy, np.full(npix, image_plane_dist)], axis=1)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    cos_cam = d[:, 2]
    cam_pdf_w = (image_plane_dist / cos_cam) ** 2 / cos_cam
    last_pdf_w_inv = float(npix) / cam_pdf_w
    origin = np.tile(cam, (npix, 1))
    thr = np.ones((npix, 3))
    origin_in_med = np.zeros(npix, bool)
    stop_bb1d = np.zeros(npix, bool)
    # per-path camera MIS arrays (list of dict records, index = path length)
    cmis: List[list] = [[dict(pdf_a_inv=0.0, rev_pdf_a=1.0, flags=0)] for _ in range(npix)]

    sq: Dict[str, list] = {k_: [] for k_ in ("origin", "direction", "seg_begin", "seg_count", "flags", "path_length",
                                             "last_pdf_w_inv", "throughput", "pixel", "cam_mis_begin")}
    seg: Dict[str, list] = {k_: [] for k_ in ("dist_min", "dist_max", "pdf", "rev_pdf", "attenuation", "medium")}
    pq: Dict[str, list] = {k_: [] for k_ in ("position", "dir_fix", "medium_id", "path_length", "throughput",
                                             "pixel", "cam_mis_begin")}
    cam_records: List[tuple] = []

    def snapshot(p, count):
        b = len(cam_records)
        for rec in cmis[p][:count]:
            cam_records.append(_mis_record(**rec))
        return b

    active = np.arange(npix)
    L = 1
    while active.size:
        o = origin[active]
        dd = d[active]
        full, lite, st = _trace(cfg, rng, o, dd, origin_in_med[active])
        for j, p in enumerate(active):
            scattered = np.isfinite(st[j])
            use_lite = scattered and cfg.query_beam_type == LONG_BEAM
            if use_lite:
                segs = [(s0, s1, 1.0, 1.0, (1.0, 1.0, 1.0), mid) for (s0, s1, mid) in lite[j]]
            else:
                segs = full[j]
            has_medium = any(media[s[5]].has_scattering for s in segs)
            if has_medium:
                qf = (Q_ORIGIN_IN_MEDIUM if origin_in_med[p] else 0) | (Q_LITE if use_lite else 0)
                if tech & PB2D:
                    qf |= Q_PB2D
                if (tech & BB1D) and not stop_bb1d[p]:
                    qf |= Q_BB1D
                sq["origin"].append(o[j])
                sq["direction"].append(dd[j])
                sq["seg_begin"].append(len(seg["dist_min"]))
                sq["seg_count"].append(len(segs))
                for (s0, s1, pdf, rev, att, mid) in segs:
                    seg["dist_min"].append(s0)
                    seg["dist_max"].append(s1)
                    seg["pdf"].append(pdf)
                    seg["rev_pdf"].append(rev)
                    seg["attenuation"].append(att)
                    seg["medium"].append(mid)
                sq["flags"].append(qf)
                sq["path_length"].append(L)
                sq["last_pdf_w_inv"].append(last_pdf_w_inv[p])
                sq["throughput"].append(thr[p].copy())
                sq["pixel"].append(p)
                sq["cam_mis_begin"].append(snapshot(p, L))
        nxt = []
        for j, p in enumerate(active):
            if not np.isfinite(st[j]):
                continue
            segs = full[j]
            rsp = float(np.prod([s[2] for s in segs]))
            rsr = float(np.prod([s[3] for s in segs]))
            att = np.prod(np.asarray([s[4] for s in segs]), axis=0)
            thr[p] = thr[p] * att / rsp
            if not np.any(thr[p] > 0):
                continue
            mid = segs[-1][5]
            m = media[mid]
            hit = o[j] + dd[j] * st[j]
            dist2 = st[j] * st[j]
            ratio = 1.0 / m.min_pos_sigma_t
            flags = 0
            if (not merge_pb2d) or m.mfp > k["bb1d_min_mfp"]:
                flags |= MIS_IN_MEDIUM_WITH_BEAMS
            rec = dict(pdf_a_inv=last_pdf_w_inv[p] * dist2 / rsp, rev_pdf_a=1.0, ray_sample_pdf_inv=1.0 / rsp,
                       ray_sample_rev_pdf_inv=1.0, ray_sample_pdfs_ratio=ratio, ray_sample_rev_pdfs_ratio=ratio,
                       pp3d_factor=k["eta_pp3d"], pb2d_factor=k["eta_pb2d"], bb1d_factor=k["eta_bb1d"],
                       bb1d_beam_selection_pdf=1.0, flags=flags)
            prev = cmis[p][L - 1]
            prev["rev_pdf_a"] = prev.get("rev_pdf_a", 0.0) * rsr / dist2
            prev["ray_sample_rev_pdf_inv"] = 1.0 / rsr
            cmis[p].append(rec)
            if L >= cfg.max_path_length:
                continue
            if L > 1 or st[j] >= cfg.min_dist_to_med:
                if tech & PP3D:
                    pq["position"].append(hit)
                    pq["dir_fix"].append(-dd[j])
                    pq["medium_id"].append(mid)
                    pq["path_length"].append(L)
                    pq["throughput"].append(thr[p].copy())
                    pq["pixel"].append(p)
                    pq["cam_mis_begin"].append(snapshot(p, L + 1))
            origin[p] = hit
            origin_in_med[p] = True
            nxt.append((j, p))
        if not nxt:
            break
        js = np.array([j for j, _ in nxt])
        ps = np.array([p for _, p in nxt])
        gvals = np.array([cfg.media[_medium_of(cfg, origin[p])].mean_cosine for p in ps])
        wnew, pdfw, sin_t = _hg_sample(rng, -dd[js], gvals)
        rr = rng.random(len(ps))
        survivors = []
        for t_, p in enumerate(ps):
            m = cfg.media[_medium_of(cfg, origin[p])]
            cont = m.continuation_prob
            if cont == 0 or (cont < 1 and rr[t_] > cont):
                continue
            dir_pdf = pdfw[t_] * cont
            thr[p] = thr[p] * np.asarray(m.scattering) * pdfw[t_] / dir_pdf
            last_pdf_w_inv[p] = 1.0 / dir_pdf
            cur = cmis[p][L]
            cur["sin_theta"] = sin_t[t_]
            cur["cos_theta_out"] = 1.0
            cmis[p][L - 1]["rev_pdf_a"] = cmis[p][L - 1].get("rev_pdf_a", 0.0) * dir_pdf
            d[p] = wnew[t_]
            if tech & BB1D_PREVIOUS:
                stop_bb1d[p] = True
            survivors.append(p)
        active = np.array(survivors, dtype=np.int64)
        L += 1

    nq = len(sq["origin"])
    out["sq_origin"] = np.asarray(sq["origin"], np.float32).reshape(nq, 3)
    out["sq_direction"] = np.asarray(sq["direction"], np.float32).reshape(nq, 3)
    out["sq_seg_begin"] = np.asarray(sq["seg_begin"], np.int32)
    out["sq_seg_count"] = np.asarray(sq["seg_count"], np.int32)
    out["sq_flags"] = np.asarray(sq["flags"], np.uint32)
    out["sq_path_length"] = np.asarray(sq["path_length"], np.int32)
    out["sq_last_pdf_w_inv"] = np.asarray(sq["last_pdf_w_inv"], np.float32)
    out["sq_throughput"] = np.asarray(sq["throughput"], np.float32).reshape(nq, 3)
    out["sq_pixel"] = np.asarray(sq["pixel"], np.int32)
    out["sq_cam_mis_begin"] = np.asarray(sq["cam_mis_begin"], np.int64)
    ns = len(seg["dist_min"])
    out["seg_dist_min"] = np.asarray(seg["dist_min"], np.float32)
    out["seg_dist_max"] = np.asarray(seg["dist_max"], np.float32)
    out["seg_pdf"] = np.asarray(seg["pdf"], np.float32)
    out["seg_rev_pdf"] = np.asarray(seg["rev_pdf"], np.float32)
    out["seg_attenuation"] = np.asarray(seg["attenuation"], np.float32).reshape(ns, 3)
    out["seg_medium"] = np.asarray(seg["medium"], np.int32)
    npq = len(pq["position"])
    out["pq_position"] = np.asarray(pq["position"], np.float32).reshape(npq, 3)
    out["pq_dir_fix"] = np.asarray(pq["dir_fix"], np.float32).reshape(npq, 3)
    out["pq_medium_id"] = np.asarray(pq["medium_id"], np.int32)
    out["pq_path_length"] = np.asarray(pq["path_length"], np.int32)
    out["pq_throughput"] = np.asarray(pq["throughput"], np.float32).reshape(npq, 3)
    out["pq_pixel"] = np.asarray(pq["pixel"], np.int32)
    out["pq_cam_mis_begin"] = np.asarray(pq["cam_mis_begin"], np.int64)
    cm = np.zeros(len(cam_records), MIS_DTYPE)
    if cam_records:
        cm[:] = cam_records
    out["cam_mis"] = cm


def _medium_of(cfg: SceneConfig, p: np.ndarray) -> int:
    return int(_medium_at(cfg, p[None, :])[0])
