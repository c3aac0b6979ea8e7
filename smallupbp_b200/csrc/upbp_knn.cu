// KNN radii (RadiusCalculation KNN_RADIUS of the reference):
//   * PB2D: each photon's radius is radius_pb2d * 2 * (distance to its k-th nearest photon, itself
//     included) (EmbreeBre::build, Bre/Bre.cxx:685-725);
//   * BB1D: each beam's start / end radius is max(2 * (distance from its origin / end to the k-th
//     nearest beam origin) * radius_bb1d, 0.001), varying linearly along the beam
//     (PhotonBeamsEvaluator::build, Beams/PhBeams.cxx:72-123).
// The distance is the exact k-th smallest of ((dx*dx + dy*dy) + dz*dz) in FP32 with d = point -
// query, the operation order of the reference's KdTree (Misc/KdTmpl.hxx:604-610).  (The
// reference's kd-tree search itself is approximate and can return a larger value.)  One thread
// per query walks an LBVH over the points with a sorted list of the k best distances.
#include <cfloat>
#include <cstdint>

#include "upbp_kernels.cuh"

namespace upbp {

namespace {

constexpr int kThreads = 128;
inline int blocks_for(int64_t n) { return (int)((n + kThreads - 1) / kThreads); }

__device__ __forceinline__ float point_d2(float4 p, V3 q)
{
    const float dx = __fsub_rn(p.x, q.x), dy = __fsub_rn(p.y, q.y), dz = __fsub_rn(p.z, q.z);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)), __fmul_rn(dz, dz));
}

// Squared distance from q to a box (a lower bound for every point inside the box).
__device__ __forceinline__ float box_d2(float lx, float ly, float lz, float hx, float hy, float hz, V3 q)
{
    const float dx = fmaxf(fmaxf(lx - q.x, 0.f), q.x - hx);
    const float dy = fmaxf(fmaxf(ly - q.y, 0.f), q.y - hy);
    const float dz = fmaxf(fmaxf(lz - q.z, 0.f), q.z - hz);
    return dx * dx + dy * dy + dz * dz;
}

// k-th smallest squared distance from q to the points (largest found if fewer than k); sets
// *overflow when the traversal stack would overflow (the result is then incomplete).
__device__ float kth_d2(V3 q, const BNode* __restrict__ nodes, int n_leaves, const float4* __restrict__ pts, int n,
                        int leaf, int k, int* overflow)
{
    float best[kMaxKnn];
    int nb = 0;
    auto consider = [&](float d2) {
        if (nb == k && !(d2 < best[k - 1])) return;
        int a = nb < k ? nb++ : k - 1;
        for (; a > 0 && best[a - 1] > d2; --a) best[a] = best[a - 1];
        best[a] = d2;
    };
    auto leaf_points = [&](int l) {
        const int e = min(n, (l + 1) * leaf);
        for (int i = l * leaf; i < e; ++i) consider(point_d2(__ldg(&pts[i]), q));
    };
    // a box is skipped only if even its (rounded) lower bound is clearly beyond the k-th best
    auto prune = [&](float lb) { return nb == k && lb * 0.999998f > best[k - 1]; };
    if (n_leaves == 1) {
        leaf_points(0);
    } else if (n_leaves > 1) {
        constexpr int kStack = 96;
        int stack[kStack];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            const int node = stack[--sp];
            const float4 a = __ldg(&nodes[node].a);
            const float4 b = __ldg(&nodes[node].b);
            const float4 c = __ldg(&nodes[node].c);
            const int4 d = __ldg(&nodes[node].d);
            const float ll = box_d2(a.x, a.y, a.z, a.w, b.x, b.y, q);
            const float lr = box_d2(b.z, b.w, c.x, c.y, c.z, c.w, q);
            // visit the nearer child first: push it last
            const bool left_first = ll <= lr;
            const int first = left_first ? d.x : d.y, second = left_first ? d.y : d.x;
            const float lf = left_first ? ll : lr, ls = left_first ? lr : ll;
            if (!prune(ls)) {
                if (second < 0) leaf_points(~second);
                else if (sp < kStack) stack[sp++] = second;
                else *overflow = 1;
            }
            if (!prune(lf)) {
                if (first < 0) leaf_points(~first);
                else if (sp < kStack) stack[sp++] = first;
                else *overflow = 1;
            }
        }
    }
    return nb > 0 ? best[nb - 1] : 0.f;
}

__global__ void k_photon_knn_r2(const float4* __restrict__ pts, int n, const BNode* __restrict__ nodes, int n_leaves,
                                int leaf, int k, float r, float* __restrict__ r2, int* status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pts[i];
    int overflow = 0;
    const float d2 = kth_d2(v3(p.x, p.y, p.z), nodes, n_leaves, pts, n, leaf, k, &overflow);
    const float radius = __fmul_rn(r, __fmul_rn(2.0f, __fsqrt_rn(d2)));  // radius *= 2 * sqrt(dist2[1])
    r2[i] = __fmul_rn(radius, radius);                                     // EmbreePhoton::set
    if (overflow) atomicOr(status, 2);
}

// Leaf boxes of photon spheres with per-photon radius (sqrt of r2, plus eps).
__global__ void k_photon_leaf_boxes_r2(const float4* __restrict__ pos, const float* __restrict__ r2, int n, int leaf,
                                       float eps, Box* out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int nl = (n + leaf - 1) / leaf;
    if (k >= nl) return;
    Box b;
    for (int c = 0; c < 3; ++c) { b.lo[c] = FLT_MAX; b.hi[c] = -FLT_MAX; }
    const int e = min(n, (k + 1) * leaf);
    for (int i = k * leaf; i < e; ++i) {
        const float4 p = pos[i];
        const float m = sqrtf(r2[i]) * 1.000001f + eps;
        b.lo[0] = fminf(b.lo[0], p.x - m); b.lo[1] = fminf(b.lo[1], p.y - m); b.lo[2] = fminf(b.lo[2], p.z - m);
        b.hi[0] = fmaxf(b.hi[0], p.x + m); b.hi[1] = fmaxf(b.hi[1], p.y + m); b.hi[2] = fmaxf(b.hi[2], p.z + m);
    }
    out[k] = b;
}

__global__ void k_beam_origins(const float* __restrict__ origin, int n, float4* out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = make_float4(origin[3 * i], origin[3 * i + 1], origin[3 * i + 2], __int_as_float(i));
}

__device__ __forceinline__ float beam_radius(float d2, float r)
{
    const float v = __fmul_rn(__fmul_rn(2.0f, __fsqrt_rn(d2)), r);  // 2 * sqrt(dist2[1]) * beamRadius
    return fmaxf(v, 0.001f);                                       // SMALLEST_RADIUS
}

// Per beam: start radius, radius change per unit length, max radius^2 (PhBeams.cxx:94-115).
__global__ void k_beam_knn(const float* __restrict__ origin, const float* __restrict__ dir,
                           const float* __restrict__ length, int n, const BNode* __restrict__ nodes, int n_leaves,
                           const float4* __restrict__ pts, int leaf, int k, float r, float* rstart, float* rchange,
                           float* r2max, int* status)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    const V3 o = v3(origin[3 * b], origin[3 * b + 1], origin[3 * b + 2]);
    const V3 d = v3(dir[3 * b], dir[3 * b + 1], dir[3 * b + 2]);
    const float len = length[b];
    const V3 e = v3(__fadd_rn(o.x, __fmul_rn(d.x, len)), __fadd_rn(o.y, __fmul_rn(d.y, len)),
                    __fadd_rn(o.z, __fmul_rn(d.z, len)));  // mRay.target(mLength)
    int overflow = 0;
    const float rs = beam_radius(kth_d2(o, nodes, n_leaves, pts, n, leaf, k, &overflow), r);
    const float re = beam_radius(kth_d2(e, nodes, n_leaves, pts, n, leaf, k, &overflow), r);
    const float mx = fmaxf(rs, re);
    rstart[b] = rs;
    r2max[b] = __fmul_rn(mx, mx);
    rchange[b] = __fdiv_rn(__fsub_rn(re, rs), len);
    if (overflow) atomicOr(status, 2);
}

}  // namespace

void launch_photon_knn_r2(const float4* pts, int n, const BNode* nodes, int n_leaves, int leaf, int k, float r,
                          float* r2, int* status, cudaStream_t s)
{
    if (n > 0) k_photon_knn_r2<<<blocks_for(n), kThreads, 0, s>>>(pts, n, nodes, n_leaves, leaf, k, r, r2, status);
}
void launch_photon_leaf_boxes_r2(const float4* pos, const float* r2, int n, int leaf, float eps, Box* leaf_boxes,
                                 cudaStream_t s)
{
    const int nl = (n + leaf - 1) / leaf;
    if (nl > 0) k_photon_leaf_boxes_r2<<<blocks_for(nl), kThreads, 0, s>>>(pos, r2, n, leaf, eps, leaf_boxes);
}
void launch_beam_origins(const float* origin, int n, float4* out, cudaStream_t s)
{
    if (n > 0) k_beam_origins<<<blocks_for(n), kThreads, 0, s>>>(origin, n, out);
}
void launch_beam_knn(const float* origin, const float* dir, const float* length, int n, const BNode* nodes,
                     int n_leaves, const float4* pts, int leaf, int k, float r, float* rstart, float* rchange,
                     float* r2max, int* status, cudaStream_t s)
{
    if (n > 0)
        k_beam_knn<<<blocks_for(n), kThreads, 0, s>>>(origin, dir, length, n, nodes, n_leaves, pts, leaf, k, r, rstart,
                                                      rchange, r2max, status);
}

}  // namespace upbp
