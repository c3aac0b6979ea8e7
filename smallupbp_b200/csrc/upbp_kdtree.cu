// The reference's own k-nearest-neighbour search for the KNN radii (upbp_params.knn_exact = 0), so
// that the radii equal the reference's bit for bit.
//
// The reference builds Jensen's left-balanced kd-tree over the points in insertion order
// (KdTreeTmplPtr::AddItem / BuildUp / _balanceSegment / _medianSplit, Misc/KdTmpl.hxx:300-468) and
// runs KNNQuery (:692-760) with _checkAddNearest (:600-687).  That search is approximate -- its
// heap bound stays at the initial radius until k points are held, the (k+1)-th point then replaces
// the farthest held one whatever its distance, and the descent treats the nodes from n/2 - 1 on as
// leaves -- so its result depends on the exact tree, and the tree on the exact in-place partition
// of every median split, ties included.
//
// The build here produces that tree level by level.  Node i (heap order, root 1) covers a segment
// [start, end] of the working array that depends only on n (the median rule of _balanceSegment);
// its splitting axis is the longest side of its box (the root's: the points' bounding box; a
// child's: its parent's box cut at the parent's split value).  Each level partitions all of its
// segments in one launch:
//   * a segment of more than kBigSeg points is split by one block, which reproduces Sedgewick's
//     sequential partition exactly: with pivot v = a[right], the k-th swap of the sequential loop
//     exchanges the k-th element >= v counted from the left (A[k]) with the k-th element <= v counted
//     from the right (B[k]), for as long as A[k] < B[k]; the pivot then goes to min(A[m], B[m-1]) (m
//     swaps).  So one partition is two block-wide compactions of positions and m parallel swaps;
//   * smaller segments are split by one thread each, running the sequential loop itself.
// The query is one thread per point, the reference's stack walk and heap, in FP32 without
// contraction.
#include <cfloat>
#include <cstdint>

#include <cub/block/block_scan.cuh>

#include "upbp_kdtree.cuh"

namespace upbp {

namespace {

constexpr int kBigSeg = 4096;
constexpr int kWarpSeg = 64;
constexpr int kSplitThreads = 1024;
constexpr unsigned kAllLanes = 0xffffffffu;

__host__ __device__ __forceinline__ int kd_median(int start, int end)
{
    const int n = end - start + 1;
    int m = 1;
    while (4 * m <= n) m += m;
    return (3 * m <= n) ? m + m + start - 1 : end - m + 1;
}

// Segment [start, end] of heap node idx (1-based) of the tree over n points; false if the node does
// not exist.
__device__ __forceinline__ bool kd_segment(int idx, int n, int& start, int& end)
{
    start = 1;
    end = n;
    const int level = 31 - __clz(idx);
    for (int b = level - 1; b >= 0; --b) {
        if (start >= end) return false;  // a single point has no children
        const int m = kd_median(start, end);
        if ((idx >> b) & 1) start = m + 1;
        else end = m - 1;
    }
    return start <= end;
}

__device__ __forceinline__ float axis_of(const float4& p, int axis) { return axis == 0 ? p.x : (axis == 1 ? p.y : p.z); }

// _balanceSegment's choice of the splitting axis from the node's box
__device__ __forceinline__ int kd_axis(const float* box)
{
    const float ex = box[3] - box[0], ey = box[4] - box[1], ez = box[5] - box[2];
    if (ex > ey && ex > ez) return 0;
    return ey > ez ? 1 : 2;
}

__device__ __forceinline__ void kd_swap(float4* a, int i, int j)
{
    const float4 t = a[i];
    a[i] = a[j];
    a[j] = t;
}

// node idx takes its median point (and its axis in w), and its children's boxes are written
__device__ __forceinline__ void kd_emit(float4* tree, float* boxes, const float4* org, int idx, int n, int median,
                                        int axis, const float* box)
{
    const float4 p = org[median];
    tree[idx] = make_float4(p.x, p.y, p.z, __int_as_float(axis));
    const float v = axis_of(p, axis);
    if (2 * idx <= n)
        for (int c = 0; c < 6; ++c) boxes[6 * (2 * idx) + c] = (c == 3 + axis) ? v : box[c];
    if (2 * idx + 1 <= n)
        for (int c = 0; c < 6; ++c) boxes[6 * (2 * idx + 1) + c] = (c == axis) ? v : box[c];
}

__global__ void k_kd_gather(const float4* __restrict__ pos, const int32_t* __restrict__ idx, int n, float4* org)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[idx ? idx[i] : i];
    org[i + 1] = make_float4(p.x, p.y, p.z, 0.f);
}

// the root's box: the points' bounding box (AddItem)
__global__ void k_kd_root_box(const float* __restrict__ bbox, float* boxes)
{
    if (threadIdx.x < 6 && blockIdx.x == 0) boxes[6 + threadIdx.x] = bbox[threadIdx.x];
}

// one level, the segments of at most kBigSeg points: one thread each, the sequential partition
__global__ void k_kd_level_small(float4* __restrict__ org, float4* __restrict__ tree, float* __restrict__ boxes, int n,
                                 int first, int count)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const int idx = first + t;
    int start, end;
    if (idx > n || !kd_segment(idx, n, start, end)) return;
    if (start == end) {  // a single point: copied (its plane is never read by the query)
        const float4 p = org[start];
        tree[idx] = make_float4(p.x, p.y, p.z, __int_as_float(0));
        return;
    }
    if (end - start + 1 > kWarpSeg) return;  // k_kd_level_warp, k_kd_level_big
    float box[6];
    for (int c = 0; c < 6; ++c) box[c] = boxes[6 * idx + c];
    const int axis = kd_axis(box);
    const int median = kd_median(start, end);
    int left = start, right = end;
    while (right > left) {
        const float v = axis_of(org[right], axis);
        int i = left - 1, j = right;
        for (;;) {
            while (axis_of(org[++i], axis) < v) {
            }
            while (axis_of(org[--j], axis) > v && j > left) {
            }
            if (i >= j) break;
            kd_swap(org, i, j);
        }
        kd_swap(org, i, right);
        if (i >= median) right = i - 1;
        if (i <= median) left = i + 1;
    }
    kd_emit(tree, boxes, org, idx, n, median, axis, box);
}

// one level, the segments of kWarpSeg + 1 to kBigSeg points: one warp each, the partition of
// k_kd_level_big (below) with ballots in place of the block scans.  The sequential loop's pivots
// make some segments take many partition passes (up to one per element on ordered input); each
// pass then costs a warp sweep of the segment instead of one thread's.
__global__ void k_kd_level_warp(float4* __restrict__ org, float4* __restrict__ tree, float* __restrict__ boxes,
                                int* __restrict__ pa, int* __restrict__ pb, int n, int first, int count)
{
    const int w = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (w >= count) return;  // the whole warp: w is the same on its lanes
    const int idx = first + w;
    int start, end;
    if (idx > n || !kd_segment(idx, n, start, end)) return;
    if (end - start + 1 <= kWarpSeg || end - start + 1 > kBigSeg) return;
    float box[6];
    for (int c = 0; c < 6; ++c) box[c] = boxes[6 * idx + c];
    const int axis = kd_axis(box);
    const int median = kd_median(start, end);
    const unsigned lt = (1u << lane) - 1u;
    int left = start, right = end;
    while (right > left) {
        const float v = axis_of(org[right], axis);
        // A: ascending positions in [left, right] with key >= v; B: ascending positions in
        // (left, right) with key <= v
        int na = 0, nb = 0;
        for (int base = left; base <= right; base += 32) {
            const int i = base + lane;
            const float key = i <= right ? axis_of(org[i], axis) : 0.f;
            const bool fa = i <= right && key >= v;
            const bool fb = i > left && i < right && key <= v;
            const unsigned ba = __ballot_sync(kAllLanes, fa), bb = __ballot_sync(kAllLanes, fb);
            if (fa) pa[start + na + __popc(ba & lt)] = i;
            if (fb) pb[start + nb + __popc(bb & lt)] = i;
            na += __popc(ba);
            nb += __popc(bb);
        }
        __syncwarp();
        // m = the first k with A[k] >= B'[k] (B'[k]: the k-th of B from the right, then `left`);
        // A ascends and B' descends, so the test turns true once, at the latest at A's last entry
        int m = na - 1;
        for (int k0 = 0; k0 < na; k0 += 32) {
            const int k = k0 + lane;
            bool hit = false;
            if (k < na) hit = pa[start + k] >= (k < nb ? pb[start + nb - 1 - k] : left);
            const unsigned bh = __ballot_sync(kAllLanes, hit);
            if (bh) {
                m = k0 + __ffs(bh) - 1;
                break;
            }
        }
        for (int k = lane; k < m; k += 32) kd_swap(org, pa[start + k], pb[start + nb - 1 - k]);
        __syncwarp();
        int i = 0;
        if (lane == 0) {
            const int a = pa[start + m];
            i = m == 0 ? a : min(a, pb[start + nb - m]);
            kd_swap(org, i, right);
        }
        i = __shfl_sync(kAllLanes, i, 0);
        __syncwarp();
        if (i >= median) right = i - 1;
        if (i <= median) left = i + 1;
    }
    if (lane == 0) kd_emit(tree, boxes, org, idx, n, median, axis, box);
}

// one level, the segments of more than kBigSeg points: one block each.  pa, pb: position scratch
// (the segment's own range of it).
__global__ void __launch_bounds__(kSplitThreads) k_kd_level_big(float4* __restrict__ org, float4* __restrict__ tree,
                                                                float* __restrict__ boxes, int* __restrict__ pa,
                                                                int* __restrict__ pb, int n, int first)
{
    using Scan = cub::BlockScan<int, kSplitThreads>;
    __shared__ typename Scan::TempStorage scan_tmp;
    __shared__ int s_left, s_right, s_m;
    const int idx = first + blockIdx.x;
    int start, end;
    if (idx > n || !kd_segment(idx, n, start, end) || end - start + 1 <= kBigSeg) return;
    float box[6];
    for (int c = 0; c < 6; ++c) box[c] = boxes[6 * idx + c];
    const int axis = kd_axis(box);
    const int median = kd_median(start, end);
    const int tid = threadIdx.x;
    if (tid == 0) {
        s_left = start;
        s_right = end;
    }
    __syncthreads();
    for (;;) {
        const int left = s_left, right = s_right;
        if (!(right > left)) break;
        const float v = axis_of(org[right], axis);
        // A: ascending positions in [left, right] with key >= v (right is the last);
        // B: ascending positions in (left, right) with key <= v (the sequential loop takes them
        // from the right)
        int na = 0, nb = 0;
        for (int base = left; base <= right; base += kSplitThreads) {
            const int i = base + tid;
            const float key = i <= right ? axis_of(org[i], axis) : 0.f;
            const int fa = (i <= right && key >= v) ? 1 : 0;
            const int fb = (i > left && i < right && key <= v) ? 1 : 0;
            int ra, rb, ta, tb;
            Scan(scan_tmp).ExclusiveSum(fa, ra, ta);
            __syncthreads();
            Scan(scan_tmp).ExclusiveSum(fb, rb, tb);
            __syncthreads();
            if (fa) pa[start + na + ra] = i;
            if (fb) pb[start + nb + rb] = i;
            na += ta;
            nb += tb;
        }
        if (tid == 0) s_m = na;
        __syncthreads();
        // m = the first k with A[k] >= B'[k], B'[k] = the k-th from the right of B, then `left`
        for (int k = tid; k < na; k += kSplitThreads) {
            const int bk = k < nb ? pb[start + nb - 1 - k] : left;
            if (pa[start + k] >= bk) atomicMin(&s_m, k);
        }
        __syncthreads();
        const int m = s_m;
        for (int k = tid; k < m; k += kSplitThreads) kd_swap(org, pa[start + k], pb[start + nb - 1 - k]);
        __syncthreads();
        if (tid == 0) {
            const int a = pa[start + m];
            const int i = m == 0 ? a : min(a, pb[start + nb - m]);
            kd_swap(org, i, right);
            int l = left, r = right;
            if (i >= median) r = i - 1;
            if (i <= median) l = i + 1;
            s_left = l;
            s_right = r;
        }
        __syncthreads();
    }
    if (tid == 0) kd_emit(tree, boxes, org, idx, n, median, axis, box);
}

// KNNQuery (KdTmpl.hxx:692-760) with _checkAddNearest (:600-687) and the builds' initial radius
// sqrt(FLT_MAX) (Bre.cxx:44, PhBeams.cxx:48); returns dist2[1]
__device__ float kd_knn_d2(const float4* __restrict__ tree, int n, V3 q, int k)
{
    float heap[kMaxKnn + 1];
    int s_index[64];
    float s_d2[64];
    const int half = n / 2 - 1;
    const float r0 = __fsqrt_rn(FLT_MAX);
    heap[0] = __fmul_rn(r0, r0);
    heap[1] = 0.f;
    if (n < 1) return 0.f;
    int found = 0, got_heap = 0, level = 0, index = 1;
    float maxd = 0.f;
    auto add = [&](int node) {
        const float4 p = __ldg(&tree[node]);
        float d1 = __fsub_rn(p.x, q.x);
        float d2 = __fmul_rn(d1, d1);
        d1 = __fsub_rn(p.y, q.y);
        d2 = __fadd_rn(d2, __fmul_rn(d1, d1));
        d1 = __fsub_rn(p.z, q.z);
        d2 = __fadd_rn(d2, __fmul_rn(d1, d1));
        if (!(d2 < heap[0])) return;
        if (found < k) {
            heap[++found] = d2;
            if (maxd < d2) maxd = d2;
            return;
        }
        if (!got_heap) {  // the max-heap over heap[1..found]
            const int h = found >> 1;
            for (int kk = h; kk >= 1; --kk) {
                int parent = kk;
                const float v = heap[kk];
                while (parent <= h) {
                    int j = parent + parent;
                    if (j < found && heap[j] < heap[j + 1]) ++j;
                    if (v >= heap[j]) break;
                    heap[parent] = heap[j];
                    parent = j;
                }
                heap[parent] = v;
            }
            got_heap = 1;
        }
        int parent = 1, j = 2;  // the root leaves, d2 sinks from the top
        while (j <= found) {
            if (j < found && heap[j] < heap[j + 1]) ++j;
            if (d2 > heap[j]) break;
            heap[parent] = heap[j];
            parent = j;
            j += j;
        }
        heap[parent] = d2;
        heap[0] = maxd = heap[1];
    };
    for (;;) {
        while (index < half) {
            const float4 p = __ldg(&tree[index]);
            const int plane = __float_as_int(p.w);
            const float d1 = __fsub_rn(plane == 0 ? q.x : (plane == 1 ? q.y : q.z), axis_of(p, plane));
            index *= 2;
            if (d1 > 0.f) ++index;
            s_index[level] = index;
            s_d2[level] = __fmul_rn(d1, d1);
            ++level;
        }
        add(index);
        int camefrom;
        do {
            camefrom = index;
            index /= 2;
            --level;
            if (index == 0) return heap[1];
        } while (s_d2[level] >= heap[0] || camefrom != s_index[level]);
        add(index);
        index = s_index[level] ^ 1;
        ++level;
    }
}

__global__ void k_kd_photon_r2(const float4* __restrict__ tree, int n, const float4* __restrict__ queries, int nq, int k,
                               float r, float* __restrict__ r2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nq) return;
    const float4 p = queries[i];
    const float d2 = kd_knn_d2(tree, n, v3(p.x, p.y, p.z), k);
    const float radius = __fmul_rn(r, __fmul_rn(2.0f, __fsqrt_rn(d2)));  // radius *= 2 * sqrt(dist2[1])
    r2[i] = __fmul_rn(radius, radius);                                     // EmbreePhoton::set
}

__device__ __forceinline__ float kd_beam_radius(float d2, float r)
{
    return fmaxf(__fmul_rn(__fmul_rn(2.0f, __fsqrt_rn(d2)), r), 0.001f);  // PhBeams.cxx:100, 105
}

// The beams' two query points (PhBeams.cxx:94-115): j < nb the origin of beam j, j >= nb the end
// point of beam j - nb, mRay.target(mLength).
__global__ void k_kd_beam_points(const float* __restrict__ origin, const float* __restrict__ dir,
                                 const float* __restrict__ length, int nb, float4* __restrict__ pts)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= 2 * nb) return;
    const int b = j < nb ? j : j - nb;
    const V3 o = v3(origin[3 * b], origin[3 * b + 1], origin[3 * b + 2]);
    if (j < nb) {
        pts[j] = make_float4(o.x, o.y, o.z, 0.f);
        return;
    }
    const V3 d = v3(dir[3 * b], dir[3 * b + 1], dir[3 * b + 2]);
    const float len = length[b];
    pts[j] = make_float4(__fadd_rn(o.x, __fmul_rn(d.x, len)), __fadd_rn(o.y, __fmul_rn(d.y, len)),
                         __fadd_rn(o.z, __fmul_rn(d.z, len)), 0.f);
}

// KNNQuery at the query points in the given order (neighbouring threads on neighbouring points, so
// that a warp's walks through the tree stay alike): d2[j] = dist2[1] of point order[i]
__global__ void k_kd_knn_sorted(const float4* __restrict__ tree, int n, const float4* __restrict__ pts,
                                const int32_t* __restrict__ order, int nq, int k, float* __restrict__ d2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nq) return;
    const int j = order[i];
    const float4 p = pts[j];
    d2[j] = kd_knn_d2(tree, n, v3(p.x, p.y, p.z), k);
}

// the beam's radii from its two searches (PhBeams.cxx:94-115)
__global__ void k_kd_beam_finish(const float* __restrict__ d2, const float* __restrict__ length, int nb, float r,
                                 float* rstart, float* rchange, float* r2max)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    const float rs = kd_beam_radius(d2[b], r);
    const float re = kd_beam_radius(d2[nb + b], r);
    const float mx = fmaxf(rs, re);
    rstart[b] = rs;
    r2max[b] = __fmul_rn(mx, mx);
    rchange[b] = __fdiv_rn(__fsub_rn(re, rs), length[b]);
}

constexpr int kThreads = 128;
inline int blocks_for(int64_t n) { return (int)((n + kThreads - 1) / kThreads); }

// the largest segment of each level of the tree over n points (the segments depend on n only)
void level_max_sizes(int n, int* out, int max_levels)
{
    // segment sizes of a level with their counts; every level has at most a few distinct sizes
    struct Sz {
        int size;
        long long count;
    };
    Sz cur[8], nxt[8];
    int nc = 1, nn;
    cur[0] = Sz{n, 1};
    for (int L = 0; L < max_levels; ++L) {
        int mx = 0;
        nn = 0;
        for (int a = 0; a < nc; ++a) {
            mx = cur[a].size > mx ? cur[a].size : mx;
            if (cur[a].size < 2) continue;
            const int m = kd_median(1, cur[a].size);
            const int ls = m - 1, rs = cur[a].size - m;
            for (int side = 0; side < 2; ++side) {
                const int s = side ? rs : ls;
                if (s < 1) continue;
                int f = 0;
                while (f < nn && nxt[f].size != s) ++f;
                if (f == nn) {
                    if (nn == 8) {  // never seen (a level has at most 3 sizes): split every later level by blocks
                        for (int l = L; l < max_levels; ++l) out[l] = 1 << 30;
                        return;
                    }
                    nxt[nn++] = Sz{s, 0};
                }
                nxt[f].count += cur[a].count;
            }
        }
        out[L] = mx;
        for (int a = 0; a < nn; ++a) cur[a] = nxt[a];
        nc = nn;
    }
}

}  // namespace

void launch_kd_build(const float4* pos, const int32_t* idx, int n, const float* bbox, float4* org, float4* tree,
                     float* boxes, int* pa, int* pb, cudaStream_t s)
{
    if (n < 1) return;
    k_kd_gather<<<blocks_for(n), kThreads, 0, s>>>(pos, idx, n, org);
    if (n == 1) {  // BuildUp leaves a single point in place
        cudaMemcpyAsync(tree + 1, org + 1, sizeof(float4), cudaMemcpyDeviceToDevice, s);
        return;
    }
    k_kd_root_box<<<1, 32, 0, s>>>(bbox, boxes);
    constexpr int kMaxLevels = 32;
    int sizes[kMaxLevels];
    level_max_sizes(n, sizes, kMaxLevels);
    for (int L = 0; L < kMaxLevels; ++L) {
        const int first = 1 << L;
        if (first > n) break;
        const int count = min(first, n - first + 1);
        if (sizes[L] > kBigSeg)
            k_kd_level_big<<<count, kSplitThreads, 0, s>>>(org, tree, boxes, pa, pb, n, first);
        if (sizes[L] > kWarpSeg)
            k_kd_level_warp<<<blocks_for(32LL * count), kThreads, 0, s>>>(org, tree, boxes, pa, pb, n, first, count);
        k_kd_level_small<<<blocks_for(count), kThreads, 0, s>>>(org, tree, boxes, n, first, count);
    }
}

int kd_build_launches(int n)
{
    if (n < 2) return n;
    int sizes[32], c = 2;
    level_max_sizes(n, sizes, 32);
    for (int L = 0; L < 32 && (1 << L) <= n; ++L) c += 1 + (sizes[L] > kBigSeg ? 1 : 0) + (sizes[L] > kWarpSeg ? 1 : 0);
    return c;
}

void launch_kd_photon_r2(const float4* tree, int n, const float4* queries, int nq, int k, float r, float* r2,
                         cudaStream_t s)
{
    if (nq > 0) k_kd_photon_r2<<<blocks_for(nq), kThreads, 0, s>>>(tree, n, queries, nq, k, r, r2);
}

void launch_kd_beam_points(const float* origin, const float* dir, const float* length, int nb, float4* pts,
                           cudaStream_t s)
{
    if (nb > 0) k_kd_beam_points<<<blocks_for(2LL * nb), kThreads, 0, s>>>(origin, dir, length, nb, pts);
}
void launch_kd_knn_sorted(const float4* tree, int n, const float4* pts, const int32_t* order, int nq, int k,
                          float* d2, cudaStream_t s)
{
    if (nq > 0) k_kd_knn_sorted<<<blocks_for(nq), kThreads, 0, s>>>(tree, n, pts, order, nq, k, d2);
}
void launch_kd_beam_finish(const float* d2, const float* length, int nb, float r, float* rstart, float* rchange,
                           float* r2max, cudaStream_t s)
{
    if (nb > 0) k_kd_beam_finish<<<blocks_for(nb), kThreads, 0, s>>>(d2, length, nb, r, rstart, rchange, r2max);
}

}  // namespace upbp
