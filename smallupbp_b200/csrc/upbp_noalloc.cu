// Allocation-free PP3D evaluation: upbp_pp3d_evaluate_noalloc (include/upbp_gpu.h).
//
// Some callers cannot call cudaMalloc: a renderer plug-in running inside a host application
// that owns the device memory budget (and forbids allocations from plug-ins), or an embedded
// caller that reserves all device memory up front.  This entry point builds the PP3D hash grid
// and evaluates the point queries without allocating anything: its scratch memory is the
// file-scope device array below, a fixed size held by every GPU that loads the library until
// the process exits.
//
// The caller passes device pointers for every input and output.  The call reads two small
// values back to the host (the photon count and the hash grid's bounding box), so it waits for
// its stream.  The scratch array is shared by all calls: it keeps the last call's contents,
// everything that must start at zero is cleared by each call, and calls that overlap on the
// GPU (different streams or host threads) race on it.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>

#include "upbp_kernels.cuh"

using namespace upbp;

namespace {

// HomogeneousMedium's derived coefficients (Scene/Media.hxx:129-159), as the context path
// computes them.
DMedium derive_medium_noalloc(const upbp_medium& m)
{
    DMedium d{};
    for (int c = 0; c < 3; ++c) {
        d.ss[c] = std::fabs(m.scattering[c]);
        d.st[c] = std::fabs(m.absorption[c]) + d.ss[c];
    }
    float mn = d.st[0];
    int idx = 0;
    if (d.st[1] > 0 && (mn == 0 || d.st[1] < mn)) mn = d.st[1], idx = 1;
    if (d.st[2] > 0 && (mn == 0 || d.st[2] < mn)) mn = d.st[2], idx = 2;
    d.min_st = mn;
    d.min_idx = idx;
    d.has_scat = (d.ss[0] > 0 || d.ss[1] > 0 || d.ss[2] > 0) ? 1 : 0;
    const bool has_att = d.st[0] > 0 || d.st[1] > 0 || d.st[2] > 0;
    const float mx = std::max(d.st[0], std::max(d.st[1], d.st[2]));
    d.mfp = has_att ? 1.0f / mx : INFINITY;
    d.g = m.mean_cosine;
    d.cont = m.continuation_prob;
    d.gray = (d.st[0] == d.st[1] && d.st[1] == d.st[2]) ? 1 : 0;
    return d;
}

constexpr int64_t kMaxLv = UPBP_NOALLOC_MAX_LIGHT_VERTICES;
constexpr int64_t kMaxCells = UPBP_NOALLOC_MAX_HASH_CELLS;
constexpr size_t kCubBytes = size_t(4) << 20;  // radix sort / select temporary storage

constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }
// Layout of the scratch array (bytes).
constexpr size_t kOffPos = 0;
constexpr size_t kOffDir = kOffPos + align256(16 * kMaxLv);
constexpr size_t kOffThr = kOffDir + align256(16 * kMaxLv);
constexpr size_t kOffInfo = kOffThr + align256(16 * kMaxLv);
constexpr size_t kOffInMed = kOffInfo + align256(16 * kMaxLv);
constexpr size_t kOffIota = kOffInMed + align256(4 * kMaxLv);
constexpr size_t kOffPhLv = kOffIota + align256(4 * kMaxLv);
constexpr size_t kOffPhLvSorted = kOffPhLv + align256(4 * kMaxLv);
constexpr size_t kOffKeys = kOffPhLvSorted + align256(4 * kMaxLv);
constexpr size_t kOffKeysSorted = kOffKeys + align256(4 * kMaxLv);
constexpr size_t kOffHgPos = kOffKeysSorted + align256(4 * kMaxLv);
constexpr size_t kOffStart = kOffHgPos + align256(16 * kMaxLv);
constexpr size_t kOffEnd = kOffStart + align256(4 * kMaxCells);
constexpr size_t kOffPartial = kOffEnd + align256(4 * kMaxCells);
constexpr size_t kOffBbox = kOffPartial + align256(4 * 8 + 4 * 6 * 1024);
constexpr size_t kOffCub = kOffBbox + align256(4 * 8);
constexpr size_t kScratchBytes = kOffCub + kCubBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Device address of g_noalloc_scratch per device, looked up on the first call on that device
// with the device current (the host-side name of the array is only a stand-in and must never be
// passed to a kernel).  Only a successful lookup is kept: after a failure the next call tries
// again.
constexpr int kMaxDevices = 64;
unsigned char* g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

unsigned char* scratch_address(int dev)
{
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        g_scratch_addr[dev] = static_cast<unsigned char*>(p);
    }
    return g_scratch_addr[dev];
}

__global__ void k_iota_noalloc(int32_t* v, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

int bits_for_cells(uint32_t maxv)
{
    int b = 1;
    while (b < 32 && (maxv >> b)) ++b;
    return b;
}

}  // namespace

extern "C" int upbp_pp3d_evaluate_noalloc(const upbp_params* params, const upbp_medium* media, int32_t n_media,
                                          const upbp_light_vertices* lv, const upbp_mis* cam_mis,
                                          const upbp_point_queries* pq, float* out_rgb, void* stream_ptr)
{
    if (!params || !media || n_media <= 0 || n_media > UPBP_MAX_MEDIA || !lv || !pq || (pq->n > 0 && !out_rgb))
        return UPBP_ERR_INVALID_ARG;
    // every array the call reads must be given for a non-empty count (a null pointer would fault
    // on the device instead of returning an error)
    if (lv->n > 0 && (!lv->position || !lv->throughput || !lv->dir_fix || !lv->cont_prob || !lv->path_idx ||
                      !lv->path_length || !lv->medium_id || !lv->flags || !lv->mis || !lv->path_ends))
        return UPBP_ERR_INVALID_ARG;
    if (pq->n > 0 && (!cam_mis || !pq->position || !pq->dir_fix || !pq->medium_id || !pq->path_length ||
                      !pq->throughput || !pq->pixel || !pq->cam_mis_begin))
        return UPBP_ERR_INVALID_ARG;
    if (lv->n < 0 || lv->n > kMaxLv || params->hash_cells < 1 || params->hash_cells > kMaxCells || pq->n < 0)
        return UPBP_ERR_CAPACITY;
    if (!(params->radius_pp3d > 0.f)) return UPBP_ERR_INVALID_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return UPBP_ERR_CUDA;
    unsigned char* base = scratch_address(dev);
    if (!base) return UPBP_ERR_CUDA;
    cudaStream_t s = static_cast<cudaStream_t>(stream_ptr);
    const upbp_params& P = *params;
    const int n = (int)lv->n;
    if (pq->n == 0) return UPBP_OK;
    float4* pos = reinterpret_cast<float4*>(base + kOffPos);
    float4* dir = reinterpret_cast<float4*>(base + kOffDir);
    float4* thr = reinterpret_cast<float4*>(base + kOffThr);
    int4* info = reinterpret_cast<int4*>(base + kOffInfo);
    uint32_t* inmed = reinterpret_cast<uint32_t*>(base + kOffInMed);
    int32_t* iota = reinterpret_cast<int32_t*>(base + kOffIota);
    int32_t* ph_lv = reinterpret_cast<int32_t*>(base + kOffPhLv);
    int32_t* ph_lv_sorted = reinterpret_cast<int32_t*>(base + kOffPhLvSorted);
    uint32_t* keys = reinterpret_cast<uint32_t*>(base + kOffKeys);
    uint32_t* keys_sorted = reinterpret_cast<uint32_t*>(base + kOffKeysSorted);
    float4* hg_pos = reinterpret_cast<float4*>(base + kOffHgPos);
    int32_t* hg_start = reinterpret_cast<int32_t*>(base + kOffStart);
    int32_t* hg_end = reinterpret_cast<int32_t*>(base + kOffEnd);
    int32_t* d_nsel = reinterpret_cast<int32_t*>(base + kOffPartial);
    float* partial = reinterpret_cast<float*>(base + kOffPartial + 32);
    float* bbox = reinterpret_cast<float*>(base + kOffBbox);
    void* cub_tmp = base + kOffCub;
#define NA_CK(x)                                           \
    do {                                                   \
        if ((x) != cudaSuccess) {                          \
            cudaGetLastError();                            \
            return UPBP_ERR_CUDA;                          \
        }                                                  \
    } while (0)
    int nph = 0;
    float hbbox[6] = {0, 0, 0, 0, 0, 0};
    if (n > 0) {
        launch_pack_lights(lv->position, lv->throughput, lv->dir_fix, lv->cont_prob, lv->path_idx, lv->path_length,
                           lv->medium_id, lv->flags, n, pos, dir, thr, info, inmed, s);
        k_iota_noalloc<<<(n + 255) / 256, 256, 0, s>>>(iota, n);
        size_t bytes = 0;
        NA_CK(cub::DeviceSelect::Flagged(nullptr, bytes, iota, inmed, ph_lv, d_nsel, n, s));
        if (bytes > kCubBytes) return UPBP_ERR_CAPACITY;
        NA_CK(cub::DeviceSelect::Flagged(cub_tmp, bytes, iota, inmed, ph_lv, d_nsel, n, s));
        NA_CK(cudaMemcpyAsync(&nph, d_nsel, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
        NA_CK(cudaStreamSynchronize(s));
    }
    const int cells = P.hash_cells;
    NA_CK(cudaMemsetAsync(hg_start, 0, sizeof(int32_t) * cells, s));
    NA_CK(cudaMemsetAsync(hg_end, 0, sizeof(int32_t) * cells, s));
    const float inv_cell = 1.f / (P.radius_pp3d * 2.f);
    if (nph > 0) {
        const int blocks = std::max(1, std::min(1024, (nph + 255) / 256));
        launch_bbox_partial(pos, ph_lv, nph, partial, blocks, s);
        launch_bbox_final(partial, blocks, bbox, s);
        NA_CK(cudaMemcpyAsync(hbbox, bbox, sizeof(float) * 6, cudaMemcpyDeviceToHost, s));
        launch_hash_keys(pos, ph_lv, nph, bbox, inv_cell, cells, keys, s);
        size_t bytes = 0;
        const int end_bit = bits_for_cells((uint32_t)cells - 1);
        NA_CK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys, keys_sorted, ph_lv, ph_lv_sorted, nph, 0, end_bit,
                                              s));
        if (bytes > kCubBytes) return UPBP_ERR_CAPACITY;
        NA_CK(cub::DeviceRadixSort::SortPairs(cub_tmp, bytes, keys, keys_sorted, ph_lv, ph_lv_sorted, nph, 0, end_bit,
                                              s));
        launch_hash_ranges(keys_sorted, ph_lv_sorted, pos, nph, hg_start, hg_end, hg_pos, s);
        NA_CK(cudaStreamSynchronize(s));  // hbbox is read below
    }
    GatherConsts K{};
    K.P = P;
    K.n_media = n_media;
    for (int i = 0; i < n_media; ++i) K.media[i] = derive_medium_noalloc(media[i]);
    K.has_bb1d_beams = 0;
    K.eps = 1e-4f;
    LightSoA L{};
    L.pos = pos;
    L.dir = dir;
    L.thr = thr;
    L.info = info;
    L.mis = lv->mis;
    L.path_ends = lv->path_ends;
    L.sums = nullptr;
    L.n = n;
    HashGridDev G{};
    G.pos = hg_pos;
    G.start = hg_start;
    G.end = hg_end;
    for (int k = 0; k < 3; ++k) {
        G.bbox_min[k] = hbbox[k];
        G.bbox_max[k] = hbbox[3 + k];
    }
    G.inv_cell = inv_cell;
    G.r2 = P.radius_pp3d * P.radius_pp3d;
    G.cells = cells;
    G.n = (P.techniques & UPBP_PP3D) ? nph : 0;
    PointQueriesDev Q{};
    Q.position = pq->position;
    Q.dir_fix = pq->dir_fix;
    Q.medium_id = pq->medium_id;
    Q.path_length = pq->path_length;
    Q.throughput = pq->throughput;
    Q.pixel = pq->pixel;
    Q.cam_mis_begin = pq->cam_mis_begin;
    Q.n = pq->n;
    Outputs O{out_rgb, nullptr, nullptr, nullptr, nullptr};
    launch_gather_pp3d(K, L, G, Q, cam_mis, nullptr, O, 128, false, s);
    NA_CK(cudaGetLastError());
#undef NA_CK
    return UPBP_OK;
}
