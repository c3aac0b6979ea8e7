// Per-iteration builds of the B200 estimator stage:
//   * light-vertex packing into float4 SoA,
//   * the PP3D hash grid, bit-compatible with Misc/HashGrid.hxx:47-126,
//   * LBVHs (Morton codes, CUB radix sort, Karras hierarchy, bottom-up boxes)
//     over photon spheres (PB2D) and over beam pieces (BB1D).
#include <cfloat>
#include <cstdint>

#include "upbp_kernels.cuh"

namespace upbp {

namespace {

constexpr int kThreads = 256;
inline int blocks_for(int64_t n, int t = kThreads) { return (int)((n + t - 1) / t); }

__global__ void k_pack_lights(const float* __restrict__ pos, const float* __restrict__ thr,
                              const float* __restrict__ dir, const float* __restrict__ cont,
                              const int32_t* __restrict__ path_idx, const int32_t* __restrict__ path_length,
                              const int32_t* __restrict__ medium, const uint32_t* __restrict__ flags, int64_t n,
                              float4* o_pos, float4* o_dir, float4* o_thr, int4* o_info, uint32_t* o_in_medium)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    o_pos[i] = make_float4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], cont[i]);
    o_dir[i] = make_float4(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2], 0.f);
    o_thr[i] = make_float4(thr[3 * i], thr[3 * i + 1], thr[3 * i + 2], 0.f);
    o_info[i] = make_int4(path_idx[i], path_length[i], (int)flags[i], medium[i]);
    o_in_medium[i] = (flags[i] & UPBP_LV_IN_MEDIUM) ? 1u : 0u;
}

// ---------------------------------------------------------------- bounding boxes
__global__ void k_bbox_partial(const float4* __restrict__ pts, const int32_t* __restrict__ idx, int n, float* partial)
{
    __shared__ float s[6][kThreads];
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = pts[idx ? idx[i] : i];
        lo[0] = fminf(lo[0], p.x); lo[1] = fminf(lo[1], p.y); lo[2] = fminf(lo[2], p.z);
        hi[0] = fmaxf(hi[0], p.x); hi[1] = fmaxf(hi[1], p.y); hi[2] = fmaxf(hi[2], p.z);
    }
    for (int c = 0; c < 3; ++c) { s[c][threadIdx.x] = lo[c]; s[3 + c][threadIdx.x] = hi[c]; }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int c = 0; c < 3; ++c) {
                s[c][threadIdx.x] = fminf(s[c][threadIdx.x], s[c][threadIdx.x + w]);
                s[3 + c][threadIdx.x] = fmaxf(s[3 + c][threadIdx.x], s[3 + c][threadIdx.x + w]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 6; ++c) partial[6 * blockIdx.x + c] = s[c][0];
}

__global__ void k_bbox_final(const float* partial, int blocks, float* out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float v[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int b = 0; b < blocks; ++b)
        for (int c = 0; c < 3; ++c) {
            v[c] = fminf(v[c], partial[6 * b + c]);
            v[3 + c] = fmaxf(v[3 + c], partial[6 * b + 3 + c]);
        }
    for (int c = 0; c < 6; ++c) out[c] = v[c];
}

// ---------------------------------------------------------------- PP3D hash grid
// HashGrid::GetCellIndex (Misc/HashGrid.hxx:198-218), same float operations.
__device__ __forceinline__ uint32_t hash_cell(int x, int y, int z, int cells)
{
    const uint32_t ux = (uint32_t)x, uy = (uint32_t)y, uz = (uint32_t)z;
    return ((ux * 73856093u) ^ (uy * 19349663u) ^ (uz * 83492791u)) % (uint32_t)cells;
}

__global__ void k_hash_keys(const float4* __restrict__ lv_pos, const int32_t* __restrict__ ph_lv, int n,
                            const float* __restrict__ bbox, float inv_cell, int cells, uint32_t* keys)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = lv_pos[ph_lv[i]];
    const int x = (int)floorf(__fmul_rn(inv_cell, __fsub_rn(p.x, bbox[0])));
    const int y = (int)floorf(__fmul_rn(inv_cell, __fsub_rn(p.y, bbox[1])));
    const int z = (int)floorf(__fmul_rn(inv_cell, __fsub_rn(p.z, bbox[2])));
    keys[i] = hash_cell(x, y, z, cells);
}

__global__ void k_hash_ranges(const uint32_t* __restrict__ keys, const int32_t* __restrict__ lv_sorted,
                              const float4* __restrict__ lv_pos, int n, int32_t* start, int32_t* end, float4* out_pos)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t k = keys[i];
    if (i == 0 || keys[i - 1] != k) start[k] = i;
    if (i == n - 1 || keys[i + 1] != k) end[k] = i + 1;
    const int lv = lv_sorted[i];
    const float4 p = lv_pos[lv];
    out_pos[i] = make_float4(p.x, p.y, p.z, __int_as_float(lv));
}

// ---------------------------------------------------------------- Morton / LBVH
__device__ __forceinline__ uint32_t expand_bits(uint32_t v)
{
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

__device__ __forceinline__ uint32_t morton3(float x, float y, float z, const float* bb)
{
    const float sx = bb[3] - bb[0], sy = bb[4] - bb[1], sz = bb[5] - bb[2];
    const float nx = sx > 0.f ? (x - bb[0]) / sx : 0.f;
    const float ny = sy > 0.f ? (y - bb[1]) / sy : 0.f;
    const float nz = sz > 0.f ? (z - bb[2]) / sz : 0.f;
    const uint32_t ix = (uint32_t)fminf(fmaxf(nx * 1024.f, 0.f), 1023.f);
    const uint32_t iy = (uint32_t)fminf(fmaxf(ny * 1024.f, 0.f), 1023.f);
    const uint32_t iz = (uint32_t)fminf(fmaxf(nz * 1024.f, 0.f), 1023.f);
    return (expand_bits(ix) << 2) | (expand_bits(iy) << 1) | expand_bits(iz);
}

__global__ void k_morton_points(const float4* __restrict__ lv_pos, const int32_t* __restrict__ ph_lv, int n,
                                const float* __restrict__ bbox, uint32_t* codes)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = lv_pos[ph_lv[i]];
    codes[i] = morton3(p.x, p.y, p.z, bbox);
}

__global__ void k_gather_photons(const int32_t* __restrict__ lv_sorted, const float4* __restrict__ lv_pos, int n,
                                 float4* out_pos)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int lv = lv_sorted[i];
    const float4 p = lv_pos[lv];
    out_pos[i] = make_float4(p.x, p.y, p.z, __int_as_float(lv));
}

__global__ void k_leaf_codes(const uint32_t* __restrict__ codes, int n, int leaf, uint32_t* leaf_codes)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int nl = (n + leaf - 1) / leaf;
    if (k >= nl) return;
    leaf_codes[k] = codes[k * leaf];
}

// Karras 2012, "Maximizing parallelism in the construction of BVHs": common-prefix length
// of leaves i and j, with the index as tie breaker for equal codes.
__device__ __forceinline__ int delta(const uint32_t* codes, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    const uint32_t a = codes[i], b = codes[j];
    if (a == b) return 32 + __clz((uint32_t)i ^ (uint32_t)j);
    return __clz(a ^ b);
}

__global__ void k_karras(const uint32_t* __restrict__ codes, int n, BNode* nodes, int32_t* parent_int,
                         int32_t* parent_leaf)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    const int d = (delta(codes, n, i, i + 1) - delta(codes, n, i, i - 1)) >= 0 ? 1 : -1;
    const int dmin = delta(codes, n, i, i - d);
    int lmax = 2;
    while (delta(codes, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(codes, n, i, i + (l + t) * d) > dmin) l += t;
    const int j = i + l * d;
    const int dnode = delta(codes, n, i, j);
    int s = 0;
    int t = l;
    for (;;) {
        t = (t + 1) >> 1;
        if (delta(codes, n, i, i + (s + t) * d) > dnode) s += t;
        if (t <= 1) break;
    }
    const int gamma = i + s * d + min(d, 0);
    const int left = (min(i, j) == gamma) ? ~gamma : gamma;
    const int right = (max(i, j) == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    nodes[i].d = make_int4(left, right, 0, 0);
    if (left < 0) parent_leaf[~left] = i; else parent_int[left] = i;
    if (right < 0) parent_leaf[~right] = i; else parent_int[right] = i;
    if (i == 0) parent_int[0] = -1;
}

__global__ void k_photon_leaf_boxes(const float4* __restrict__ pos, int n, int leaf, float r, float eps, Box* out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int nl = (n + leaf - 1) / leaf;
    if (k >= nl) return;
    Box b;
    for (int c = 0; c < 3; ++c) { b.lo[c] = FLT_MAX; b.hi[c] = -FLT_MAX; }
    const int e = min(n, (k + 1) * leaf);
    for (int i = k * leaf; i < e; ++i) {
        const float4 p = pos[i];
        b.lo[0] = fminf(b.lo[0], p.x); b.lo[1] = fminf(b.lo[1], p.y); b.lo[2] = fminf(b.lo[2], p.z);
        b.hi[0] = fmaxf(b.hi[0], p.x); b.hi[1] = fmaxf(b.hi[1], p.y); b.hi[2] = fmaxf(b.hi[2], p.z);
    }
    for (int c = 0; c < 3; ++c) { b.lo[c] -= r + eps; b.hi[c] += r + eps; }
    out[k] = b;
}

__global__ void k_box_leaf_boxes(const Box* __restrict__ boxes, int n, int leaf, Box* out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int nl = (n + leaf - 1) / leaf;
    if (k >= nl) return;
    Box b;
    for (int c = 0; c < 3; ++c) { b.lo[c] = FLT_MAX; b.hi[c] = -FLT_MAX; }
    const int e = min(n, (k + 1) * leaf);
    for (int i = k * leaf; i < e; ++i)
        for (int c = 0; c < 3; ++c) {
            b.lo[c] = fminf(b.lo[c], boxes[i].lo[c]);
            b.hi[c] = fmaxf(b.hi[c], boxes[i].hi[c]);
        }
    out[k] = b;
}

__device__ __forceinline__ Box load_box_volatile(const Box* p)
{
    const volatile float* f = reinterpret_cast<const volatile float*>(p);
    Box b;
    for (int c = 0; c < 3; ++c) { b.lo[c] = f[c]; b.hi[c] = f[3 + c]; }
    return b;
}

// Bottom-up boxes: the second child to arrive at a node computes it (atomic flag per node).
__global__ void k_bottom_up(const Box* leaf_boxes, int n_leaves, BNode* nodes, const int32_t* __restrict__ parent_int,
                            const int32_t* __restrict__ parent_leaf, Box* node_boxes, int32_t* flags)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_leaves || n_leaves < 2) return;
    int node = parent_leaf[k];
    while (node >= 0) {
        __threadfence();
        if (atomicAdd(&flags[node], 1) == 0) return;
        __threadfence();
        const int4 ch = nodes[node].d;
        const Box l = ch.x < 0 ? load_box_volatile(&leaf_boxes[~ch.x]) : load_box_volatile(&node_boxes[ch.x]);
        const Box r = ch.y < 0 ? load_box_volatile(&leaf_boxes[~ch.y]) : load_box_volatile(&node_boxes[ch.y]);
        BNode nd;
        nd.a = make_float4(l.lo[0], l.lo[1], l.lo[2], l.hi[0]);
        nd.b = make_float4(l.hi[1], l.hi[2], r.lo[0], r.lo[1]);
        nd.c = make_float4(r.lo[2], r.hi[0], r.hi[1], r.hi[2]);
        nd.d = ch;
        nodes[node] = nd;
        Box u;
        for (int c = 0; c < 3; ++c) { u.lo[c] = fminf(l.lo[c], r.lo[c]); u.hi[c] = fmaxf(l.hi[c], r.hi[c]); }
        volatile float* f = reinterpret_cast<volatile float*>(&node_boxes[node]);
        for (int c = 0; c < 3; ++c) { f[c] = u.lo[c]; f[3 + c] = u.hi[c]; }
        node = parent_int[node];
    }
}

// ---------------------------------------------------------------- beams
__global__ void k_pack_beams(const float* __restrict__ thr, const uint32_t* __restrict__ flags,
                             const float* __restrict__ rsp, const float* __restrict__ rsr,
                             const float* __restrict__ lpw, const uint32_t* __restrict__ rsf,
                             const int32_t* __restrict__ lv, const int32_t* __restrict__ medium, int64_t n,
                             float radius, float4* o_thr, float4* o_pdf, int2* o_link, float* o_radius)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    o_thr[i] = make_float4(thr[3 * i], thr[3 * i + 1], thr[3 * i + 2], __int_as_float((int)flags[i]));
    o_pdf[i] = make_float4(rsp[i], rsr[i], lpw[i], __int_as_float((int)rsf[i]));
    o_link[i] = make_int2(lv[i], medium[i]);
    o_radius[i] = radius;  // PhotonBeamsEvaluator::build, CONSTANT_RADIUS (PhBeams.cxx:117-121)
}

__global__ void k_piece_counts(const float* __restrict__ length, int64_t n, float piece_len, int32_t* counts)
{
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float len = length[i];
    int c = (int)ceilf(len / piece_len);
    counts[i] = max(1, min(c, 1 << 16));
}

// Piece k of beam b covers [t(k), t(k+1)) with t(k) = k*len/cnt and t(cnt) = len, so
// consecutive pieces share their boundary value exactly and every t2 in (0, len)
// belongs to exactly one piece.
__device__ __forceinline__ float piece_t(int k, int cnt, float len)
{
    return k >= cnt ? len : __fmul_rn((float)k, __fdiv_rn(len, (float)cnt));
}

// Beam of piece p: offsets (nb + 1 entries, every beam has at least one piece) are strictly
// increasing, so the beam is the last one whose first piece is <= p.
__device__ __forceinline__ int piece_beam(const int32_t* __restrict__ offsets, int64_t nb, int p)
{
    int lo = 0, hi = (int)nb - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&offsets[mid]) <= p) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Bounding box of the beam segments (both end points of every beam): the frame of the pieces'
// Morton codes.
__global__ void k_bbox_beams_partial(const float* __restrict__ origin, const float* __restrict__ dir,
                                     const float* __restrict__ length, int64_t n, float* partial)
{
    __shared__ float s[6][kThreads];
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float len = length[i];
        for (int c = 0; c < 3; ++c) {
            const float a = origin[3 * i + c], b = a + dir[3 * i + c] * len;
            lo[c] = fminf(lo[c], fminf(a, b));
            hi[c] = fmaxf(hi[c], fmaxf(a, b));
        }
    }
    for (int c = 0; c < 3; ++c) { s[c][threadIdx.x] = lo[c]; s[3 + c][threadIdx.x] = hi[c]; }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int c = 0; c < 3; ++c) {
                s[c][threadIdx.x] = fminf(s[c][threadIdx.x], s[c][threadIdx.x + w]);
                s[3 + c][threadIdx.x] = fmaxf(s[3 + c][threadIdx.x], s[3 + c][threadIdx.x + w]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int c = 0; c < 6; ++c) partial[6 * blockIdx.x + c] = s[c][0];
}

// Morton code of every piece's midpoint (one thread per piece); perm = the identity.
__global__ void k_piece_codes(const float* __restrict__ origin, const float* __restrict__ dir,
                              const float* __restrict__ length, int64_t nb, const int32_t* __restrict__ offsets,
                              int np, const float* __restrict__ bbox, uint32_t* codes, int32_t* perm)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    const int b = piece_beam(offsets, nb, p);
    const int first = offsets[b], cnt = offsets[b + 1] - first, k = p - first;
    const float len = length[b];
    const float t0 = piece_t(k, cnt, len), t1 = piece_t(k + 1, cnt, len), tm = 0.5f * (t0 + t1);
    codes[p] = morton3(origin[3 * b] + dir[3 * b] * tm, origin[3 * b + 1] + dir[3 * b + 1] * tm,
                       origin[3 * b + 2] + dir[3 * b + 2] * tm, bbox);
    perm[p] = p;
}

// The records of the pieces in Morton order (one thread per sorted position): piece perm[i] of
// its beam, at position i.  rstart / rchange / r2max (KNN radii, or NULL for the constant radius):
// beam radius at t is rstart + t * rchange, the predicate's bound is r2max (PhotonBeam.hxx:238-296,
// 411).
__global__ void k_emit_sorted(const float* __restrict__ origin, const float* __restrict__ dir,
                              const float* __restrict__ length, const int32_t* __restrict__ medium, int64_t nb,
                              const int32_t* __restrict__ offsets, const int32_t* __restrict__ perm, int np,
                              float radius, float eps, const float* __restrict__ rstart,
                              const float* __restrict__ rchange, const float* __restrict__ r2max, float4* pa,
                              float4* pb, float4* pc, Box* boxes)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const int p = perm[i];
    const int b = piece_beam(offsets, nb, p);
    const int first = offsets[b], cnt = offsets[b + 1] - first, k = p - first;
    const float ox = origin[3 * b], oy = origin[3 * b + 1], oz = origin[3 * b + 2];
    const float dx = dir[3 * b], dy = dir[3 * b + 1], dz = dir[3 * b + 2];
    const float len = length[b];
    // disc of radius r perpendicular to the beam: extent r*sqrt(1-d_i^2) per axis
    const float ex = sqrtf(fmaxf(0.f, 1.f - dx * dx)), ey = sqrtf(fmaxf(0.f, 1.f - dy * dy));
    const float ez = sqrtf(fmaxf(0.f, 1.f - dz * dz));
    const float rs = rstart ? rstart[b] : radius, rc = rchange ? rchange[b] : 0.f;
    const float r2 = r2max ? r2max[b] : radius * radius;
    const float t0 = piece_t(k, cnt, len), t1 = piece_t(k + 1, cnt, len);
    // the largest radius on the piece (the radius is linear in t)
    const float rp = rchange ? fmaxf(rs + t0 * rc, rs + t1 * rc) * 1.000001f : radius;
    const float mx = rp * ex + eps, my = rp * ey + eps, mz = rp * ez + eps;
    const float ax = ox + dx * t0, ay = oy + dy * t0, az = oz + dz * t0;
    const float bx = ox + dx * t1, by = oy + dy * t1, bz = oz + dz * t1;
    Box bx_;
    bx_.lo[0] = fminf(ax, bx) - mx; bx_.hi[0] = fmaxf(ax, bx) + mx;
    bx_.lo[1] = fminf(ay, by) - my; bx_.hi[1] = fmaxf(ay, by) + my;
    bx_.lo[2] = fminf(az, bz) - mz; bx_.hi[2] = fmaxf(az, bz) + mz;
    // The first and the last piece own the pairs whose closest point is clamped to the beam's
    // start or end; the query then passes within the reach of the end point in any direction, so
    // those pieces' boxes hold the ball of radius r(end) + eps about it (the reach rule of
    // piece_takes_f64).
    if (k == 0) {
        const float re = (rchange ? rs * 1.000001f : radius) + eps;
        bx_.lo[0] = fminf(bx_.lo[0], ax - re); bx_.hi[0] = fmaxf(bx_.hi[0], ax + re);
        bx_.lo[1] = fminf(bx_.lo[1], ay - re); bx_.hi[1] = fmaxf(bx_.hi[1], ay + re);
        bx_.lo[2] = fminf(bx_.lo[2], az - re); bx_.hi[2] = fmaxf(bx_.hi[2], az + re);
    }
    if (k == cnt - 1) {
        const float re = (rchange ? fmaxf(rs + len * rc, 0.f) * 1.000001f : radius) + eps;
        bx_.lo[0] = fminf(bx_.lo[0], bx - re); bx_.hi[0] = fmaxf(bx_.hi[0], bx + re);
        bx_.lo[1] = fminf(bx_.lo[1], by - re); bx_.hi[1] = fmaxf(bx_.hi[1], by + re);
        bx_.lo[2] = fminf(bx_.lo[2], bz - re); bx_.hi[2] = fmaxf(bx_.hi[2], bz + re);
    }
    pa[i] = make_float4(ox, oy, oz, len);
    pb[i] = make_float4(dx, dy, dz, r2);
    pc[i] = make_float4(t0, t1, __int_as_float(b), __int_as_float(medium[b]));
    boxes[i] = bx_;
}

}  // namespace

// ---------------------------------------------------------------- launch wrappers
void launch_pack_lights(const float* pos, const float* thr, const float* dir, const float* cont,
                        const int32_t* path_idx, const int32_t* path_length, const int32_t* medium,
                        const uint32_t* flags, int64_t n, float4* o_pos, float4* o_dir, float4* o_thr, int4* o_info,
                        uint32_t* o_in_medium, cudaStream_t stream)
{
    if (n <= 0) return;
    k_pack_lights<<<blocks_for(n), kThreads, 0, stream>>>(pos, thr, dir, cont, path_idx, path_length, medium, flags,
                                                          n, o_pos, o_dir, o_thr, o_info, o_in_medium);
}
void launch_bbox_partial(const float4* pts, const int32_t* idx, int n, float* partial, int blocks, cudaStream_t s)
{
    k_bbox_partial<<<blocks, kThreads, 0, s>>>(pts, idx, n, partial);
}
void launch_bbox_final(const float* partial, int blocks, float* out, cudaStream_t s)
{
    k_bbox_final<<<1, 32, 0, s>>>(partial, blocks, out);
}
void launch_hash_keys(const float4* lv_pos, const int32_t* ph_lv, int n, const float* bbox, float inv_cell, int cells,
                      uint32_t* keys, cudaStream_t s)
{
    if (n > 0) k_hash_keys<<<blocks_for(n), kThreads, 0, s>>>(lv_pos, ph_lv, n, bbox, inv_cell, cells, keys);
}
void launch_hash_ranges(const uint32_t* keys_sorted, const int32_t* lv_sorted, const float4* lv_pos, int n,
                        int32_t* start, int32_t* end, float4* out_pos, cudaStream_t s)
{
    if (n > 0) k_hash_ranges<<<blocks_for(n), kThreads, 0, s>>>(keys_sorted, lv_sorted, lv_pos, n, start, end, out_pos);
}
void launch_morton_points(const float4* lv_pos, const int32_t* ph_lv, int n, const float* bbox, uint32_t* codes,
                          cudaStream_t s)
{
    if (n > 0) k_morton_points<<<blocks_for(n), kThreads, 0, s>>>(lv_pos, ph_lv, n, bbox, codes);
}
void launch_gather_photons(const int32_t* lv_sorted, const float4* lv_pos, int n, float4* out_pos, cudaStream_t s)
{
    if (n > 0) k_gather_photons<<<blocks_for(n), kThreads, 0, s>>>(lv_sorted, lv_pos, n, out_pos);
}
void launch_leaf_codes(const uint32_t* codes_sorted, int n, int leaf, uint32_t* leaf_codes, cudaStream_t s)
{
    const int nl = (n + leaf - 1) / leaf;
    if (nl > 0) k_leaf_codes<<<blocks_for(nl), kThreads, 0, s>>>(codes_sorted, n, leaf, leaf_codes);
}
void launch_karras(const uint32_t* leaf_codes, int n_leaves, BNode* nodes, int32_t* parent_int, int32_t* parent_leaf,
                   cudaStream_t s)
{
    if (n_leaves > 1)
        k_karras<<<blocks_for(n_leaves - 1), kThreads, 0, s>>>(leaf_codes, n_leaves, nodes, parent_int, parent_leaf);
}
void launch_photon_leaf_boxes(const float4* pos, int n, int leaf, float r, float eps, Box* leaf_boxes, cudaStream_t s)
{
    const int nl = (n + leaf - 1) / leaf;
    if (nl > 0) k_photon_leaf_boxes<<<blocks_for(nl), kThreads, 0, s>>>(pos, n, leaf, r, eps, leaf_boxes);
}
void launch_box_leaf_boxes(const Box* boxes, int n, int leaf, Box* leaf_boxes, cudaStream_t s)
{
    const int nl = (n + leaf - 1) / leaf;
    if (nl > 0) k_box_leaf_boxes<<<blocks_for(nl), kThreads, 0, s>>>(boxes, n, leaf, leaf_boxes);
}
void launch_bottom_up(const Box* leaf_boxes, int n_leaves, BNode* nodes, const int32_t* parent_int,
                      const int32_t* parent_leaf, Box* node_boxes, int32_t* flags, cudaStream_t s)
{
    if (n_leaves > 1)
        k_bottom_up<<<blocks_for(n_leaves), kThreads, 0, s>>>(leaf_boxes, n_leaves, nodes, parent_int, parent_leaf,
                                                              node_boxes, flags);
}
void launch_pack_beams(const float* thr, const uint32_t* flags, const float* rsp, const float* rsr, const float* lpw,
                       const uint32_t* rsf, const int32_t* lv, const int32_t* medium, int64_t n, float radius,
                       float4* o_thr, float4* o_pdf, int2* o_link, float* o_radius, cudaStream_t s)
{
    if (n > 0)
        k_pack_beams<<<blocks_for(n), kThreads, 0, s>>>(thr, flags, rsp, rsr, lpw, rsf, lv, medium, n, radius, o_thr,
                                                        o_pdf, o_link, o_radius);
}
void launch_piece_counts(const float* length, int64_t n, float piece_len, int32_t* counts, cudaStream_t s)
{
    if (n > 0) k_piece_counts<<<blocks_for(n), kThreads, 0, s>>>(length, n, piece_len, counts);
}
void launch_bbox_beams_partial(const float* origin, const float* dir, const float* length, int64_t n, float* partial,
                               int blocks, cudaStream_t s)
{
    k_bbox_beams_partial<<<blocks, kThreads, 0, s>>>(origin, dir, length, n, partial);
}
void launch_piece_codes(const float* origin, const float* dir, const float* length, int64_t nb, const int32_t* offsets,
                        int np, const float* bbox, uint32_t* codes, int32_t* perm, cudaStream_t s)
{
    if (np > 0) k_piece_codes<<<blocks_for(np), kThreads, 0, s>>>(origin, dir, length, nb, offsets, np, bbox, codes, perm);
}
void launch_emit_sorted(const float* origin, const float* dir, const float* length, const int32_t* medium, int64_t nb,
                        const int32_t* offsets, const int32_t* perm, int np, float radius, float eps,
                        const float* rstart, const float* rchange, const float* r2max, float4* pa, float4* pb,
                        float4* pc, Box* boxes, cudaStream_t s)
{
    if (np > 0)
        k_emit_sorted<<<blocks_for(np), kThreads, 0, s>>>(origin, dir, length, medium, nb, offsets, perm, np, radius,
                                                          eps, rstart, rchange, r2max, pa, pb, pc, boxes);
}

}  // namespace upbp
