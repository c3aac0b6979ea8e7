// The reference's uniform grid of photon beams (Beams/Grid.hxx, Beams/PhGrid.hxx), built on the
// GPU with the reference's float operations, so that every beam lands in the same cells, in the same
// order, as in the reference:
//  * the beams' boxes (PhotonBeam::getAABB / getSegmentAABB, PhotonBeam.hxx:71-84, 186-198) and
//    their union, then the grid header (Grid::build, Grid.hxx:222-241);
//  * the rasterisation of every beam in chops along its major axis (Grid::buildloop,
//    Grid.hxx:177-219), a cell entered once per beam: each (cell, beam) pair becomes a 64-bit key
//    cell << 32 | ~beam, and sorted unique keys give the cell lists with every cell's beams in
//    descending id order, the order in which Grid's Store pass fills them;
//  * the reductions' build (Grid::reduceBeams, Grid.hxx:558-631): the over-full cells, in cell
//    order, take their draws from the reference's stream, std::mt19937_64 (Rng.hxx:51-62) through
//    std::uniform_real_distribution<float>, which libstdc++ computes as float(x) / 2^64 from one
//    64-bit output, clamped below 1: PRESAMPLE shuffles the first max_beams entries of a cell
//    (max_beams draws), OFFSET all of them (beams - 1 draws).
// The float operations are the reference's (SSE, no fused multiply-add), written with the _rn
// intrinsics so that the compiler does not contract them.
#include <cfloat>
#include <cstdint>

#include "upbp_kernels.cuh"

namespace upbp {

namespace {

constexpr int kThreads = 256;
// every kernel below loops over its items with the grid's stride
inline int blocks_for(int64_t n) { return (int)std::min<int64_t>((n + kThreads - 1) / kThreads, 1 << 20); }

// SSE min_ps / max_ps: the second operand unless the first compares below / above it
__device__ __forceinline__ float sse_min(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float sse_max(float a, float b) { return a > b ? a : b; }

struct BeamGeo {
    float o[3], d[3], len, rs, rc, m[3];
};

// PhotonBeam::getAABB's margins (PhotonBeam.hxx:74-80): sqrt of the squared direction's other two
// components, per axis.
__device__ __forceinline__ BeamGeo load_beam(const float* origin, const float* dir, const float* length,
                                             const float* rstart, const float* rchange, float radius, int64_t b)
{
    BeamGeo g;
    for (int k = 0; k < 3; ++k) {
        g.o[k] = origin[3 * b + k];
        g.d[k] = dir[3 * b + k];
    }
    g.len = length[b];
    g.rs = rstart ? rstart[b] : radius;
    g.rc = rchange ? rchange[b] : 0.f;
    const float x2 = __fmul_rn(g.d[0], g.d[0]), y2 = __fmul_rn(g.d[1], g.d[1]), z2 = __fmul_rn(g.d[2], g.d[2]);
    g.m[0] = __fsqrt_rn(__fadd_rn(y2, z2));
    g.m[1] = __fsqrt_rn(__fadd_rn(x2, z2));
    g.m[2] = __fsqrt_rn(__fadd_rn(x2, y2));
    return g;
}

// PhotonBeam::getSegmentAABB (PhotonBeam.hxx:186-198)
__device__ __forceinline__ void segment_aabb(const BeamGeo& g, float smin, float smax, float lo[3], float hi[3])
{
    smin = __fmul_rn(smin, g.len);
    smax = __fmul_rn(smax, g.len);
    const float rS = __fadd_rn(g.rs, __fmul_rn(smin, g.rc));
    const float rE = __fadd_rn(g.rs, __fmul_rn(smax, g.rc));
    for (int k = 0; k < 3; ++k) {
        const float s = __fadd_rn(g.o[k], __fmul_rn(g.d[k], smin));
        const float e = __fadd_rn(g.o[k], __fmul_rn(g.d[k], smax));
        const float sm = __fmul_rn(rS, g.m[k]), em = __fmul_rn(rE, g.m[k]);
        lo[k] = sse_min(__fsub_rn(s, sm), __fsub_rn(e, em));
        hi[k] = sse_max(__fadd_rn(s, sm), __fadd_rn(e, em));
    }
}

__global__ void k_grid_boxes_partial(const float* __restrict__ origin, const float* __restrict__ dir,
                                     const float* __restrict__ length, const float* __restrict__ rstart,
                                     const float* __restrict__ rchange, float radius, int64_t n, float* partial)
{
    __shared__ float s[6][kThreads];
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < n; b += (int64_t)gridDim.x * blockDim.x) {
        const BeamGeo g = load_beam(origin, dir, length, rstart, rchange, radius, b);
        float l[3], h[3];
        segment_aabb(g, 0.f, 1.f, l, h);
        for (int k = 0; k < 3; ++k) {
            lo[k] = fminf(lo[k], l[k]);
            hi[k] = fmaxf(hi[k], h[k]);
        }
    }
    for (int k = 0; k < 3; ++k) {
        s[k][threadIdx.x] = lo[k];
        s[3 + k][threadIdx.x] = hi[k];
    }
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 3; ++k) {
                s[k][threadIdx.x] = fminf(s[k][threadIdx.x], s[k][threadIdx.x + w]);
                s[3 + k][threadIdx.x] = fmaxf(s[3 + k][threadIdx.x], s[3 + k][threadIdx.x + w]);
            }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < 6; ++k) partial[6 * blockIdx.x + k] = s[k][0];
}

// Grid::build (Grid.hxx:222-241): the resolution from the box's largest extent, the cell size and
// its inverse, the index shifts.
__global__ void k_grid_header(const float* __restrict__ partial, int blocks, uint32_t grid_res, uint32_t max_beams,
                              uint32_t reduction, int32_t seed, GridHeader* hdr)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    GridHeader h;
    for (int k = 0; k < 3; ++k) {
        h.lo[k] = FLT_MAX;
        h.hi[k] = -FLT_MAX;
    }
    for (int b = 0; b < blocks; ++b)
        for (int k = 0; k < 3; ++k) {
            h.lo[k] = fminf(h.lo[k], partial[6 * b + k]);
            h.hi[k] = fmaxf(h.hi[k], partial[6 * b + 3 + k]);
        }
    float ext[3];
    for (int k = 0; k < 3; ++k) ext[k] = __fsub_rn(h.hi[k], h.lo[k]);
    const float size = __fdiv_rn(fmaxf(fmaxf(ext[0], ext[1]), ext[2]), (float)grid_res);
    for (int k = 0; k < 3; ++k) {
        h.res[k] = (int)((uint32_t)__fdiv_rn(ext[k], size) + 1u);
        h.cell[k] = __fdiv_rn(ext[k], (float)(uint32_t)h.res[k]);
        h.inv_cell[k] = __fdiv_rn(1.f, h.cell[k]);
    }
    h.shift[0] = 1u;
    h.shift[1] = (uint32_t)h.res[0];
    h.shift[2] = (uint32_t)h.res[0] * (uint32_t)h.res[1];
    h.n_cells = ((uint32_t)h.res[0] + 1u) * ((uint32_t)h.res[1] + 1u) * ((uint32_t)h.res[2] + 1u) + 1u;
    h.max_beams = max_beams;
    h.reduction = reduction;
    h.seed = seed;
    // a box without extent along an axis (or not finite) has no cells: n_cells 0 stops the
    // rasterisation kernels and the host rejects the build
    bool ok = true;
    for (int k = 0; k < 3; ++k)
        ok = ok && ext[k] > 0.f && isfinite(ext[k]) && isfinite(h.inv_cell[k]) && h.res[k] >= 1 &&
             h.res[k] <= (int)grid_res + 1;
    if (!ok) h.n_cells = 0u;
    *hdr = h;
}

// Grid::buildloop for one beam (Grid.hxx:177-219): calls visit(cell) for the cells of its chops in
// the reference's loop order, with the reference's index arithmetic (cell = x + res0 (y + res1 z)
// in unsigned arithmetic, rows that run past the last cell cut short).  A cell that the previous
// chop's box holds is skipped: that chop visited it (the index depends on the cell alone).  The
// bounds of a straight beam's chop boxes change monotonically from chop to chop, so a cell shared
// with any earlier chop is shared with the previous one; where rounding breaks that, the sorted
// keys' uniqueness still removes the repeat, as testDuplicates does.
template <class Visit>
__device__ __forceinline__ void rasterise(const BeamGeo& g, const GridHeader& h, Visit&& visit)
{
    float lo[3], hi[3];
    segment_aabb(g, 0.f, 1.f, lo, hi);
    const float ad[3] = {fabsf(g.d[0]), fabsf(g.d[1]), fabsf(g.d[2])};
    // Vector3::argMax (Structs/Vector3.hxx:208-210)
    const int ax = (ad[0] > ad[1]) ? ((ad[0] > ad[2]) ? 0 : 2) : ((ad[1] > ad[2]) ? 1 : 2);
    const float ext = __fsub_rn(hi[ax], lo[ax]);
    const int chops = (int)__fmul_rn(ext, h.inv_cell[ax]) + 1;
    const float inv_chops = __fdiv_rn(1.f, (float)chops);
    const int64_t size = (int64_t)h.n_cells;  // testDuplicates.size()
    int ps[3] = {1, 1, 1}, pe[3] = {0, 0, 0};  // the previous chop's cells (none at first)
    for (int c = 0; c < chops; ++c) {
        float a[3], b[3];
        segment_aabb(g, __fmul_rn((float)c, inv_chops), __fmul_rn((float)(c + 1), inv_chops), a, b);
        int is[3], ie[3];
        for (int k = 0; k < 3; ++k) {
            is[k] = (int)__fmul_rn(__fsub_rn(a[k], h.lo[k]), h.inv_cell[k]);
            ie[k] = (int)__fmul_rn(__fsub_rn(b[k], h.lo[k]), h.inv_cell[k]);
        }
        // Grid::index: unsigned arithmetic
        uint32_t id = (uint32_t)is[0] + (uint32_t)h.res[0] * ((uint32_t)is[1] + (uint32_t)h.res[1] * (uint32_t)is[2]);
        for (int z = is[2]; z <= ie[2]; ++z, id += h.shift[2]) {
            int idy = (int)id;
            for (int y = is[1]; y <= ie[1]; ++y, idy = (int)((uint32_t)idy + h.shift[1])) {
                const bool row_prev = y >= ps[1] && y <= pe[1] && z >= ps[2] && z <= pe[2];
                int idx = idy;
                for (int x = is[0]; x <= ie[0]; ++x, ++idx) {
                    if (row_prev && x >= ps[0] && x <= pe[0]) {  // jump over the previous chop's cells
                        const int nx = min(pe[0], ie[0]) + 1;
                        idx += nx - x - 1;
                        x = nx - 1;
                        continue;
                    }
                    if (idx < 0) continue;
                    if ((int64_t)idx >= size) break;
                    visit((uint32_t)idx);
                }
            }
        }
        for (int k = 0; k < 3; ++k) {
            ps[k] = is[k];
            pe[k] = ie[k];
        }
    }
}

__global__ void k_grid_count(const float* __restrict__ origin, const float* __restrict__ dir,
                             const float* __restrict__ length, const float* __restrict__ rstart,
                             const float* __restrict__ rchange, float radius, int64_t nb,
                             const GridHeader* __restrict__ hdr, unsigned long long* counts)
{
    const GridHeader h = *hdr;
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nb; b += (int64_t)gridDim.x * blockDim.x) {
        unsigned long long n = 0;
        if (h.n_cells >= 2u) {
            const BeamGeo g = load_beam(origin, dir, length, rstart, rchange, radius, b);
            rasterise(g, h, [&](uint32_t) { ++n; });
        }
        counts[b] = n;
    }
}

__global__ void k_grid_emit(const float* __restrict__ origin, const float* __restrict__ dir,
                            const float* __restrict__ length, const float* __restrict__ rstart,
                            const float* __restrict__ rchange, float radius, int64_t nb,
                            const GridHeader* __restrict__ hdr, const unsigned long long* __restrict__ offsets,
                            unsigned long long* keys)
{
    const GridHeader h = *hdr;
    if (h.n_cells < 2u) return;
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nb; b += (int64_t)gridDim.x * blockDim.x) {
        const BeamGeo g = load_beam(origin, dir, length, rstart, rchange, radius, b);
        unsigned long long at = offsets[b];
        const unsigned long long end = offsets[b + 1];
        const unsigned long long low = (unsigned long long)(~(uint32_t)b);
        rasterise(g, h, [&](uint32_t cell) {
            if (at < end) keys[at++] = ((unsigned long long)cell << 32) | low;
        });
    }
}

// counts per cell and the beam of every sorted unique key.  The keys are sorted, so the lanes of a
// warp mostly share a cell: one atomic per cell and warp (the lanes with the same cell counted by
// __match_any_sync) instead of one per entry on the same address.
__global__ void k_grid_lists(const unsigned long long* __restrict__ keys, int64_t n, uint32_t* counts, int32_t* ptr)
{
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t first = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    // every lane of a warp runs the same number of iterations, so the match is over full warps
    const int64_t warp0 = first - (threadIdx.x & 31);
    for (int64_t w = warp0; w < n; w += stride) {
        const int64_t i = w + (threadIdx.x & 31);
        const bool in = i < n;
        const unsigned long long k = in ? keys[i] : ~0ull;
        const uint32_t cell = (uint32_t)(k >> 32);
        const unsigned peers = __match_any_sync(0xffffffffu, cell);
        if (in && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&counts[cell], (uint32_t)__popc(peers));
        if (in) ptr[i] = (int32_t)(~(uint32_t)k);
    }
}

// The beam geometry of every cell entry, in the cells' (final, shuffled) order: (origin, length) and
// (direction, maximal radius squared).  The gather reads 32 consecutive entries with two coalesced
// 16-byte loads per lane instead of scattered loads through the beam id.
__global__ void k_grid_records(const int32_t* __restrict__ ptr, int64_t n, const float* __restrict__ origin,
                               const float* __restrict__ dir, const float* __restrict__ length,
                               const float* __restrict__ r2max, float r2c, float4* __restrict__ rec_a,
                               float4* __restrict__ rec_b)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int b = ptr[i];
        rec_a[i] = make_float4(origin[3 * b], origin[3 * b + 1], origin[3 * b + 2], length[b]);
        rec_b[i] = make_float4(dir[3 * b], dir[3 * b + 1], dir[3 * b + 2], r2max ? r2max[b] : r2c);
    }
}

// the build's draws of every cell (Grid.hxx:571-631): PRESAMPLE max_beams and OFFSET beams - 1 for
// an over-full cell, the resampling reductions none
__global__ void k_grid_draws(const uint32_t* __restrict__ cells, uint32_t n_cells, uint32_t max_beams,
                             uint32_t reduction, uint32_t* draws)
{
    // mPdfs covers the cells 0 .. n_cells - 2 (reduceBeams: cells = mCells.size() - 1)
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (int64_t)n_cells;
         i += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t beams = i + 1 < (int64_t)n_cells ? cells[i + 1] - cells[i] : 0u;
        draws[i] = beams <= max_beams ? 0u : (reduction == 0 ? max_beams : (reduction == 1 ? beams - 1 : 0u));
    }
}

// std::mt19937_64 (the 64-bit Mersenne Twister: n = 312, m = 156, r = 31, a = 0xb5026f5aa96619e9,
// tempering u = 29 / d = 0x5555555555555555, s = 17 / b = 0x71d67fffeda60000, t = 37 /
// c = 0xfff7eee000000000, l = 43, initialisation multiplier f = 6364136223846793005), its
// outputs x mapped to float(x) / 2^64 and clamped below 1.  One block of 312 threads: each round
// regenerates the state in two halves (the first half reads only the old state, the second half
// the first half's new values) and tempers 312 outputs.
constexpr int kMtN = 312, kMtM = 156;
__global__ void __launch_bounds__(kMtN) k_mt64_floats(unsigned long long seed, int64_t n, float* out)
{
    __shared__ unsigned long long mt[kMtN];
    const unsigned long long kUpper = 0xFFFFFFFF80000000ull, kLower = 0x7FFFFFFFull, kA = 0xB5026F5AA96619E9ull;
    const int i = threadIdx.x;
    if (i == 0) {
        mt[0] = seed;
        for (int k = 1; k < kMtN; ++k) mt[k] = 6364136223846793005ull * (mt[k - 1] ^ (mt[k - 1] >> 62)) + (unsigned long long)k;
    }
    __syncthreads();
    for (int64_t base = 0; base < n; base += kMtN) {
        // first half: entries 0 .. n - m - 1 from the old state
        {
            const unsigned long long a0 = mt[i], a1 = mt[(i + 1) % kMtN], am = mt[(i + kMtM) % kMtN];
            __syncthreads();
            if (i < kMtN - kMtM) {
                const unsigned long long x = (a0 & kUpper) | (a1 & kLower);
                mt[i] = am ^ (x >> 1) ^ ((x & 1ull) ? kA : 0ull);
            }
            __syncthreads();
        }
        // second half: entries n - m .. n - 1 from the new first half (the last one wraps to entry 0)
        {
            const unsigned long long b0 = mt[i], b1 = mt[(i + 1) % kMtN], bm = mt[(i + kMtM) % kMtN];
            __syncthreads();
            if (i >= kMtN - kMtM) {
                const unsigned long long x = (b0 & kUpper) | (b1 & kLower);
                mt[i] = bm ^ (x >> 1) ^ ((x & 1ull) ? kA : 0ull);
            }
            __syncthreads();
        }
        unsigned long long y = mt[i];
        y ^= (y >> 29) & 0x5555555555555555ull;
        y ^= (y << 17) & 0x71D67FFFEDA60000ull;
        y ^= (y << 37) & 0xFFF7EEE000000000ull;
        y ^= y >> 43;
        if (base + i < n) {
            const float f = __fmul_rn(__ull2float_rn(y), 5.42101086242752217e-20f);  // 2^-64
            out[base + i] = f >= 1.f ? 0x1.fffffep-1f : f;
        }
        __syncthreads();
    }
}

// Grid::reduceBeams (Grid.hxx:558-631): every cell's selection pdf, max_beams / beams for an
// over-full cell; PRESAMPLE shuffles the first max_beams entries of such a cell (a partial
// Fisher-Yates from the front), OFFSET shuffles all of them (from the back).
__global__ void k_grid_reduce(const uint32_t* __restrict__ cells, uint32_t n_cells, uint32_t max_beams,
                              uint32_t reduction, const uint32_t* __restrict__ draw_off, const float* __restrict__ rnd,
                              int32_t* ptr, float* pdf)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c + 1 < (int64_t)n_cells;
         c += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t begin = cells[c], beams = cells[c + 1] - begin;
        if (beams <= max_beams) {
            pdf[c] = 1.f;
            continue;
        }
        pdf[c] = __fdiv_rn((float)max_beams, (float)beams);
        const float* r = rnd + draw_off[c];
        if (reduction == 0) {
            for (uint32_t i = 0; i < max_beams; ++i) {
                const uint32_t j = i + (uint32_t)__fmul_rn(r[i], (float)(beams - i));
                if (j < beams) {  // r < 1: always
                    const int32_t t = ptr[begin + i];
                    ptr[begin + i] = ptr[begin + j];
                    ptr[begin + j] = t;
                }
            }
        } else if (reduction == 1) {
            for (uint32_t i = beams - 1, k = 0; i > 0; --i, ++k) {
                const uint32_t j = (uint32_t)__fmul_rn(r[k], (float)(i + 1));
                if (j <= i) {  // r < 1: always
                    const int32_t t = ptr[begin + i];
                    ptr[begin + i] = ptr[begin + j];
                    ptr[begin + j] = t;
                }
            }
        }
    }
}

}  // namespace

void launch_grid_header(const float* origin, const float* dir, const float* length, const float* rstart,
                        const float* rchange, float radius, int64_t nb, uint32_t grid_res, uint32_t max_beams,
                        uint32_t reduction, int32_t seed, float* partial, int blocks, GridHeader* hdr,
                        cudaStream_t s)
{
    k_grid_boxes_partial<<<blocks, kThreads, 0, s>>>(origin, dir, length, rstart, rchange, radius, nb, partial);
    k_grid_header<<<1, 32, 0, s>>>(partial, blocks, grid_res, max_beams, reduction, seed, hdr);
}
void launch_grid_count(const float* origin, const float* dir, const float* length, const float* rstart,
                       const float* rchange, float radius, int64_t nb, const GridHeader* hdr,
                       unsigned long long* counts, cudaStream_t s)
{
    if (nb > 0)
        k_grid_count<<<blocks_for(nb), kThreads, 0, s>>>(origin, dir, length, rstart, rchange, radius, nb, hdr,
                                                         counts);
}
void launch_grid_emit(const float* origin, const float* dir, const float* length, const float* rstart,
                      const float* rchange, float radius, int64_t nb, const GridHeader* hdr,
                      const unsigned long long* offsets, unsigned long long* keys, cudaStream_t s)
{
    if (nb > 0)
        k_grid_emit<<<blocks_for(nb), kThreads, 0, s>>>(origin, dir, length, rstart, rchange, radius, nb, hdr,
                                                        offsets, keys);
}
void launch_grid_lists(const unsigned long long* keys, int64_t n, uint32_t* counts, int32_t* ptr, cudaStream_t s)
{
    if (n > 0) k_grid_lists<<<blocks_for(n), kThreads, 0, s>>>(keys, n, counts, ptr);
}
void launch_grid_records(const int32_t* ptr, int64_t n, const float* origin, const float* dir, const float* length,
                         const float* r2max, float r2c, float4* rec_a, float4* rec_b, cudaStream_t s)
{
    if (n > 0) k_grid_records<<<blocks_for(n), kThreads, 0, s>>>(ptr, n, origin, dir, length, r2max, r2c, rec_a, rec_b);
}
void launch_grid_draws(const uint32_t* cells, uint32_t n_cells, uint32_t max_beams, uint32_t reduction,
                       uint32_t* draws, cudaStream_t s)
{
    if (n_cells > 0)
        k_grid_draws<<<blocks_for(n_cells), kThreads, 0, s>>>(cells, n_cells, max_beams, reduction, draws);
}
void launch_mt64_floats(unsigned long long seed, int64_t n, float* out, cudaStream_t s)
{
    if (n > 0) k_mt64_floats<<<1, kMtN, 0, s>>>(seed, n, out);
}
void launch_grid_reduce(const uint32_t* cells, uint32_t n_cells, uint32_t max_beams, uint32_t reduction,
                        const uint32_t* draw_off, const float* rnd, int32_t* ptr, float* pdf, cudaStream_t s)
{
    if (n_cells > 1)
        k_grid_reduce<<<blocks_for(n_cells), kThreads, 0, s>>>(cells, n_cells, max_beams, reduction, draw_off, rnd,
                                                               ptr, pdf);
}

}  // namespace upbp
