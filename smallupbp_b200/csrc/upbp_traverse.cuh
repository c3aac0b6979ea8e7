// BVH traversal, warp helpers and splatting shared by the gather kernels of every precision.
#pragma once

#include "upbp_kernels.cuh"

namespace upbp {

__device__ __forceinline__ void stage_media(const GatherConsts& K, DMedium* s)
{
    for (int i = threadIdx.x; i < K.n_media; i += blockDim.x) s[i] = K.media[i];
    __syncthreads();
}

__device__ __forceinline__ bool slab(float lx, float ly, float lz, float hx, float hy, float hz, V3 o, V3 inv,
                                     float tmin, float tmax)
{
    const float tx0 = (lx - o.x) * inv.x, tx1 = (hx - o.x) * inv.x;
    const float ty0 = (ly - o.y) * inv.y, ty1 = (hy - o.y) * inv.y;
    const float tz0 = (lz - o.z) * inv.z, tz1 = (hz - o.z) * inv.z;
    const float tn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
    const float tf = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fminf(fmaxf(tz0, tz1), tmax));
    return tn <= tf;
}

// IEEE reciprocal whatever the file's division flags: the slab tests of the traversal use it
__device__ __forceinline__ float safe_inv(float d) { return __frcp_rn(d == 0.f ? copysignf(1e-30f, d) : d); }

// Stack traversal of a BVH2 with child boxes; calls leaf(k) for every leaf whose box the
// segment [tmin, tmax] overlaps.  Returns false on stack overflow (reported through the
// status word).  The stack holds at most one entry per tree level, and the LBVH has at most 63
// (see kMaxTreeDepth below), so the 96 entries do not overflow.
template <class LeafFn>
__device__ __forceinline__ bool traverse(const BNode* __restrict__ nodes, int n_leaves, V3 o, V3 inv, float tmin,
                                         float tmax, LeafFn&& leaf)
{
    if (n_leaves <= 0) return true;
    if (n_leaves == 1) {
        leaf(0);
        return true;
    }
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
        const bool hl = slab(a.x, a.y, a.z, a.w, b.x, b.y, o, inv, tmin, tmax);
        const bool hr = slab(b.z, b.w, c.x, c.y, c.z, c.w, o, inv, tmin, tmax);
        if (hl) {
            if (d.x < 0) leaf(~d.x);
            else if (sp < kStack) stack[sp++] = d.x;
            else return false;
        }
        if (hr) {
            if (d.y < 0) leaf(~d.y);
            else if (sp < kStack) stack[sp++] = d.y;
            else return false;
        }
    }
    return true;
}

__device__ __forceinline__ void splat(float* image, int px, Rgb v)
{
    if (!image || px < 0) return;
    atomicAdd(&image[3 * px + 0], v.r);
    atomicAdd(&image[3 * px + 1], v.g);
    atomicAdd(&image[3 * px + 2], v.b);
}

// ----------------------------------------------------------------- warp-cooperative traversal
// One warp per query.  Each step pops up to 32 BVH nodes from the warp's shared-memory stack
// (one per lane), tests both child boxes, pushes internal hits (ballot + prefix counts) and
// appends leaf hits to the warp's leaf list; once 32 leaves are gathered (or the traversal is
// done) the warp tests the leaves' primitives 32 at a time, consecutive primitives to
// consecutive lanes.  Returns false if the stack overflowed (the status word records it).
//
// The stack cannot overflow.  A step pops `take` nodes and pushes at most 2 x take children, so it
// grows by at most `take`.  Up to kWarpStack - kMaxTreeDepth entries the warp pops as many as keep
// it there (32 at most); above that it pops one node per step, a depth-first walk that adds at
// most one entry per tree level below the popped node.  An LBVH over keys of 62 bits (30-bit
// Morton code, 32-bit index tie-break) is at most 63 levels deep.
constexpr int kWarpStack = 1024;
constexpr int kMaxTreeDepth = 64;
constexpr int kWarpLeaves = 96;
constexpr unsigned kFull = 0xffffffffu;

template <class PrimFn>
__device__ __forceinline__ bool warp_traverse(const BNode* __restrict__ nodes, int n_leaves, int n_prims, int leaf_shift,
                                              V3 o, V3 inv, float tmin, float tmax, int* stack, int* leaves, int lane,
                                              PrimFn&& prim)
{
    if (n_leaves <= 0) return true;
    const unsigned lt = (1u << lane) - 1u;
    int sp = 0, nleaf = 0;
    bool ok = true;
    if (n_leaves == 1) {
        if (lane == 0) leaves[0] = 0;
        nleaf = 1;
    } else {
        if (lane == 0) stack[0] = 0;
        sp = 1;
    }
    __syncwarp();
    while (sp > 0 || nleaf > 0) {
        if (sp > 0 && nleaf < 32) {
            const int take = min(min(sp, 32), max(1, kWarpStack - kMaxTreeDepth - sp));
            const int node = lane < take ? stack[sp - 1 - lane] : -1;
            sp -= take;
            __syncwarp();
            bool hl = false, hr = false;
            int cl = 0, cr = 0;
            if (node >= 0) {
                const float4 a = __ldg(&nodes[node].a);
                const float4 b = __ldg(&nodes[node].b);
                const float4 c = __ldg(&nodes[node].c);
                const int4 d = __ldg(&nodes[node].d);
                hl = slab(a.x, a.y, a.z, a.w, b.x, b.y, o, inv, tmin, tmax);
                hr = slab(b.z, b.w, c.x, c.y, c.z, c.w, o, inv, tmin, tmax);
                cl = d.x;
                cr = d.y;
            }
            const bool pl = hl && cl >= 0, pr = hr && cr >= 0, ll = hl && cl < 0, lr = hr && cr < 0;
            const unsigned bpl = __ballot_sync(kFull, pl), bpr = __ballot_sync(kFull, pr);
            const unsigned bll = __ballot_sync(kFull, ll), blr = __ballot_sync(kFull, lr);
            const int npush = __popc(bpl) + __popc(bpr);
            if (sp + npush > kWarpStack) {
                ok = false;  // cannot happen (see above); kept as a guard
                break;
            }
            const int ppos = sp + __popc(bpl & lt) + __popc(bpr & lt);
            if (pl) stack[ppos] = cl;
            if (pr) stack[ppos + (pl ? 1 : 0)] = cr;
            sp += npush;
            const int lpos = nleaf + __popc(bll & lt) + __popc(blr & lt);
            if (ll) leaves[lpos] = ~cl;
            if (lr) leaves[lpos + (ll ? 1 : 0)] = ~cr;
            nleaf += __popc(bll) + __popc(blr);
            __syncwarp();
        }
        if (nleaf >= 32 || (sp == 0 && nleaf > 0)) {
            // every lane calls prim (p < 0: nothing to test), so prim may use warp-wide votes
            const int total = nleaf << leaf_shift;
            for (int base = 0; base < total; base += 32) {
                const int idx = base + lane;
                int p = -1;
                if (idx < total) {
                    p = (leaves[idx >> leaf_shift] << leaf_shift) + (idx & ((1 << leaf_shift) - 1));
                    if (p >= n_prims) p = -1;
                }
                prim(p);
            }
            nleaf = 0;
            __syncwarp();
        }
    }
    return ok;
}

__device__ __forceinline__ float warp_sum(float v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ __forceinline__ uint32_t hash_cell(int x, int y, int z, int cells)
{
    const uint32_t ux = (uint32_t)x, uy = (uint32_t)y, uz = (uint32_t)z;
    return ((ux * 73856093u) ^ (uy * 19349663u) ^ (uz * 83492791u)) % (uint32_t)cells;
}

}  // namespace upbp
