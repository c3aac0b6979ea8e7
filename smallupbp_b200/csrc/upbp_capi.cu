// C ABI of the B200 estimator stage (include/upbp_gpu.h): context, uploads, builds, evaluation.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "upbp_generic_api.cuh"
#include "upbp_kdtree.cuh"
#include "upbp_kdtree.cuh"
#include "upbp_kernels.cuh"
#include "upbp_mis_prep.cuh"
#include "upbp_trace.cuh"

using namespace upbp;

namespace {

// Grow-only device buffer.
struct DBuf {
    void* p = nullptr;
    size_t cap = 0;
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

struct Error {
    int code;
};

}  // namespace

struct upbp_ctx {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int mode = UPBP_MODE_PLAIN;
    int pb2d_leaf = 4;
    int bb1d_leaf = 8;
    int block = 128;
    float piece_len_r = 6.f;  // beam piece length in units of the beam radius
    std::string err;
    upbp_params P{};
    bool have_params = false;
    std::vector<DMedium> media;
    std::vector<upbp_medium> media_raw;
    size_t bytes = 0;

    // inputs
    int64_t n_lv = 0;
    int32_t n_paths = 0;
    DBuf lv_pos_in, lv_thr_in, lv_dir_in, lv_cont_in, lv_pidx_in, lv_plen_in, lv_med_in, lv_flags_in, lv_mis,
        path_ends;
    int64_t n_beams = 0;
    DBuf b_origin, b_dir, b_len, b_thr_in, b_flags_in, b_rsp_in, b_rsr_in, b_rsf_in, b_lpw_in, b_med_in, b_lv_in;
    int64_t n_cam = 0;
    DBuf cam_mis;
    int64_t n_sq = 0, n_seg = 0;
    DBuf sq_origin, sq_dir, sq_seg_begin, sq_seg_count, sq_flags, sq_plen, sq_lpw, sq_thr, sq_pixel, sq_cam_begin,
        seg_dmin, seg_dmax, seg_pdf, seg_rev, seg_att, seg_med;
    int64_t n_pq = 0;
    DBuf pq_pos, pq_dir, pq_med, pq_plen, pq_thr, pq_pixel, pq_cam_begin;
    // the first MIS input given as NULL (allowed only with UPBP_NO_MIS), per upload; nullptr: none
    const char* lv_mis_missing = nullptr;
    const char* beam_mis_missing = nullptr;
    const char* sq_mis_missing = nullptr;

    // packed light vertices
    DBuf lv_pos4, lv_dir4, lv_thr4, lv_info4, lv_inmed;
    // photons
    int n_ph = 0;
    DBuf ph_lv, ph_lv_sorted, ph_keys, ph_keys_sorted, bbox_partial, bbox_ph;
    // hash grid
    DBuf hg_start, hg_end, hg_pos;
    float hg_bbox[6] = {0, 0, 0, 0, 0, 0};
    float hg_inv_cell = 0.f;
    // photon LBVH
    DBuf pb_pos, pb_leaf_codes, pb_nodes, pb_parent_int, pb_parent_leaf, pb_leaf_boxes, pb_node_boxes, pb_flags;
    int pb_n_leaves = 0;
    // beams
    DBuf bm_thr4, bm_pdf4, bm_link, bm_radius, bm_counts, bm_offsets, pc_a2, pc_b2, pc_c2,
        pc_boxes2, pc_codes, pc_codes_sorted, pc_perm, pc_perm_sorted, bbox_pc;
    int n_pieces = 0;
    DBuf bm_leaf_codes, bm_nodes, bm_parent_int, bm_parent_leaf, bm_leaf_boxes, bm_node_boxes, bm_flagsbuf;
    DBuf pc_pay;  // mixed mode: beam payload packed per piece
    // BB1D over the reference's uniform grid (upbp_set_bb1d_grid)
    upbp_bb1d_grid bgrid{};
    DBuf gr_hdr, gr_partial, gr_counts, gr_offsets, gr_keys, gr_keys_sorted, gr_keys_unique, gr_num, gr_cellcount,
        gr_cells, gr_ptr, gr_pdf, gr_draws, gr_draw_off, gr_rnd, gr_rec_a, gr_rec_b, gr_pay;
    GridHeader gr_host{};           // the last build's header
    int64_t gr_raw = 0, gr_pairs = 0, gr_draws_total = 0;  // its sizes (a replay reuses them)
    bool gr_valid = false;
    // KNN radii: per-photon radius^2 (leaf order); per-beam radius change and max radius^2 (the
    // start radius goes to bm_radius); the LBVH over beam origins for the beam KNN search
    DBuf pb_r2, bm_rchange, bm_r2max, knn_status;
    // the reference's kd-tree search for the KNN radii (knn_exact = 0): working array, tree, node
    // boxes, partition scratch
    DBuf kd_org, kd_tree, kd_boxes, kd_pa, kd_pb, kd_qpts, kd_qcodes, kd_qcodes_sorted, kd_qidx, kd_qidx_sorted,
        kd_qd2;
    DBuf bo_pos, bo_pts, bo_codes, bo_codes_sorted, bo_idx, bo_idx_sorted, bo_bbox, bo_leaf_codes, bo_nodes,
        bo_parent_int, bo_parent_leaf, bo_leaf_boxes, bo_node_boxes, bo_flags;
    int bo_n_leaves = 0;
    // query order (Morton code of the query span's midpoint)
    DBuf q_keys, q_keys_sorted, q_iota, q_order;
    // BB1D work order: the heavy queries (by PB2D candidate count) first
    DBuf bb_keys, bb_keys_sorted, bb_iota, bb_order, bb_sum;
    bool order_queries = true;
    int bm_n_leaves = 0;
    // mixed mode: FP64 partial sums of the MIS walks
    DBuf light_sums, cam_sums_seg, cam_sums_pt;
    // temp storage for CUB
    DBuf cub_tmp;
    // outputs
    DBuf work, status;
    DBuf grad_img, grad_acc;  // adjoint: dL/d framebuffer, dL/d medium parameters
    int* status_host = nullptr;   // page-locked copy of status[0] after the last evaluate
    // CUDA graph of clear + build + evaluate for the current inputs (upbp_capture_graph)
    cudaGraphExec_t graph_exec = nullptr;
    bool replay = false;     // capturing: reuse the last build's counts, allocate nothing, no host syncs
    bool evaluated = false;  // an evaluate ran after the last build (every buffer is sized)
    bool graph_status = false;  // the graph copies the warp gathers' traversal status back
    bool status_pending = false;  // status_host holds the last evaluate's warp-gather status flag
    int num_sms = 0;
    int bb1d_kernel = 2;  // 0: thread per query, 1-2: warp-cooperative BB1D, 3-4: fused segment kernel
    int pb2d_kernel = 1;  // PB2D on its own: 0 thread per query, 1 warp-cooperative persistent
    int query_order = 1;  // segment query order of the persistent gathers (upbp_tuning.query_order)
    DBuf out_bp2d, cnt_bp2d, hash_bp2d;  // B-P2D (extension) per point query
    DBuf tr_cnt, tr_off, tr_status;  // device-side light / camera passes: per-path record counts and offsets
    DBuf out_pb2d, out_bb1d, out_pp3d, image, cnt_pb2d, cnt_bb1d, cnt_pp3d, hash_pb2d, hash_bb1d, hash_pp3d, tested;
    bool built = false;
    int build_launches = 0, eval_launches = 0;
    float t_build = 0.f, t_pp3d = 0.f, t_pb2d = 0.f, t_bb1d = 0.f;
    cudaEvent_t ev[8] = {};
};

namespace {

void fail(upbp_ctx* c, int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    throw Error{code};
}

void ck(upbp_ctx* c, cudaError_t e, const char* what)
{
    if (e != cudaSuccess) {
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            fail(c, UPBP_ERR_OUT_OF_MEMORY, "%s: %s", what, cudaGetErrorString(e));
        }
        fail(c, UPBP_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    }
}

// After a synchronisation of the context's stream: the warp gathers (PB2D, BB1D, B-P2D) set
// status[0] when a query's traversal stack would overflow; its candidate set is then incomplete,
// which is an error.
void check_status(upbp_ctx* c)
{
    if (c->status_pending && c->status_host && *c->status_host != 0)
        fail(c, UPBP_ERR_CAPACITY, "traversal stack overflow in the last evaluate: a candidate set is "
                                   "incomplete (use a larger leaf size or beam_piece_radii)");
}

// Timing event; inside a graph capture it must be an external event record node, or the
// captured record would only order the graph's own nodes and never time anything.
void mark(upbp_ctx* c, int k, cudaStream_t s)
{
    ck(c, c->replay ? cudaEventRecordWithFlags(c->ev[k], s, cudaEventRecordExternal) : cudaEventRecord(c->ev[k], s),
       "event");
}

void drop_graph(upbp_ctx* c)
{
    if (c->graph_exec) {
        cudaGraphExecDestroy(c->graph_exec);
        c->graph_exec = nullptr;
    }
}

void ensure(upbp_ctx* c, DBuf& b, size_t bytes)
{
    if (bytes <= b.cap) return;
    if (c->replay) fail(c, UPBP_ERR_INVALID_ARG, "graph capture needs buffers sized by a build and an evaluate");
    drop_graph(c);  // a reallocation moves a buffer the graph may hold
    if (b.p) {
        ck(c, cudaFreeAsync(b.p, c->stream), "cudaFreeAsync");
        c->bytes -= b.cap;
        b.p = nullptr;
        b.cap = 0;
    }
    const size_t want = std::max<size_t>(bytes + bytes / 4, 256);
    ck(c, cudaMallocAsync(&b.p, want, c->stream), "cudaMallocAsync");
    b.cap = want;
    c->bytes += want;
}

template <class T>
void upload(upbp_ctx* c, DBuf& b, const T* src, int64_t count, const char* name)
{
    if (count <= 0) return;
    if (!src) fail(c, UPBP_ERR_INVALID_ARG, "%s is NULL", name);
    ensure(c, b, sizeof(T) * (size_t)count);
    ck(c, cudaMemcpyAsync(b.p, src, sizeof(T) * (size_t)count, cudaMemcpyDefault, c->stream), name);
}

// An MIS input, which the estimators without MIS (UPBP_NO_MIS) never read: a NULL array is
// stored as `count` elements of the byte `fill` (zeros, or -1 for indices) and its name recorded
// in *missing, so that a build or evaluate that needs it fails.
template <class T>
void upload_mis(upbp_ctx* c, DBuf& b, const T* src, int64_t count, const char* name, int fill, const char** missing)
{
    if (count <= 0) return;
    if (src) {
        upload(c, b, src, count, name);
        return;
    }
    ensure(c, b, sizeof(T) * (size_t)count);
    ck(c, cudaMemsetAsync(b.p, fill, sizeof(T) * (size_t)count, c->stream), name);
    if (!*missing) *missing = name;
}

void free_buf(DBuf& b)
{
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
}

DMedium derive_medium(const upbp_medium& m)
{
    // HomogeneousMedium ctor (Scene/Media.hxx:129-159), same float operations.
    DMedium d{};
    for (int c = 0; c < 3; ++c) {
        const float a = std::fabs(m.absorption[c]);
        const float s = std::fabs(m.scattering[c]);
        d.ss[c] = s;
        d.st[c] = a + s;
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

void sort_pairs(upbp_ctx* c, const uint32_t* kin, uint32_t* kout, const int32_t* vin, int32_t* vout, int n,
                int end_bit)
{
    size_t b = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, b, kin, kout, vin, vout, n, 0, end_bit, c->stream);
    ensure(c, c->cub_tmp, b);
    ck(c, cub::DeviceRadixSort::SortPairs(c->cub_tmp.p, b, kin, kout, vin, vout, n, 0, end_bit, c->stream),
       "SortPairs");
    c->build_launches += 4;
}

int bits_for(uint32_t maxv);

// The reference's uniform grid of beams (upbp_grid.cu).  Three host synchronisations read the
// sizes that the next steps allocate (the raw and the unique (cell, beam) pairs, the random draws);
// a replay under graph capture reuses the last build's.
void build_grid(upbp_ctx* c, cudaStream_t s, float radius, const float* rstart, const float* rchange)
{
    const int64_t nb = c->n_beams;
    const upbp_bb1d_grid& g = c->bgrid;
    const float* org = c->b_origin.as<float>();
    const float* dir = c->b_dir.as<float>();
    const float* len = c->b_len.as<float>();
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>(1024, (nb + 255) / 256));
    ensure(c, c->gr_hdr, sizeof(GridHeader));
    ensure(c, c->gr_partial, sizeof(float) * 6 * blocks);
    GridHeader* hdr = c->gr_hdr.as<GridHeader>();
    launch_grid_header(org, dir, len, rstart, rchange, radius, nb, g.grid_res, g.max_beams_in_cell, g.reduction, g.seed,
                       c->gr_partial.as<float>(), blocks, hdr, s);
    ensure(c, c->gr_counts, sizeof(unsigned long long) * (nb + 1));
    ensure(c, c->gr_offsets, sizeof(unsigned long long) * (nb + 1));
    unsigned long long* cnt = c->gr_counts.as<unsigned long long>();
    unsigned long long* off = c->gr_offsets.as<unsigned long long>();
    launch_grid_count(org, dir, len, rstart, rchange, radius, nb, hdr, cnt, s);
    ck(c, cudaMemsetAsync(cnt + nb, 0, sizeof(unsigned long long), s), "memset");
    size_t b = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b, cnt, off, (int)(nb + 1), s);
    ensure(c, c->cub_tmp, b);
    ck(c, cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, b, cnt, off, (int)(nb + 1), s), "ExclusiveSum");
    if (!c->replay) {
        unsigned long long raw = 0;
        ck(c, cudaMemcpyAsync(&raw, off + nb, sizeof(raw), cudaMemcpyDeviceToHost, s), "copy grid pairs");
        ck(c, cudaMemcpyAsync(&c->gr_host, hdr, sizeof(GridHeader), cudaMemcpyDeviceToHost, s), "copy grid header");
        ck(c, cudaStreamSynchronize(s), "sync");
        if (c->gr_host.n_cells < 2)
            fail(c, UPBP_ERR_INVALID_ARG, "the beams' box has no extent along an axis: no beam grid");
        if (raw >= (1ull << 31))
            fail(c, UPBP_ERR_CAPACITY, "the beam grid holds %llu cell entries (at most 2^31 - 1)", raw);
        c->gr_raw = (int64_t)raw;
    }
    const int64_t raw = c->gr_raw;
    const uint32_t nc = c->gr_host.n_cells;
    ensure(c, c->gr_keys, sizeof(unsigned long long) * std::max<int64_t>(raw, 1));
    ensure(c, c->gr_keys_sorted, sizeof(unsigned long long) * std::max<int64_t>(raw, 1));
    ensure(c, c->gr_keys_unique, sizeof(unsigned long long) * std::max<int64_t>(raw, 1));
    ensure(c, c->gr_num, sizeof(int64_t));
    launch_grid_emit(org, dir, len, rstart, rchange, radius, nb, hdr, off, c->gr_keys.as<unsigned long long>(), s);
    const int end_bit = 32 + bits_for(nc);
    b = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, b, c->gr_keys.as<unsigned long long>(),
                                   c->gr_keys_sorted.as<unsigned long long>(), (int)raw, 0, end_bit, s);
    ensure(c, c->cub_tmp, b);
    ck(c, cub::DeviceRadixSort::SortKeys(c->cub_tmp.p, b, c->gr_keys.as<unsigned long long>(),
                                         c->gr_keys_sorted.as<unsigned long long>(), (int)raw, 0, end_bit, s),
       "SortKeys");
    b = 0;
    cub::DeviceSelect::Unique(nullptr, b, c->gr_keys_sorted.as<unsigned long long>(),
                              c->gr_keys_unique.as<unsigned long long>(), c->gr_num.as<int64_t>(), (int64_t)raw, s);
    ensure(c, c->cub_tmp, b);
    ck(c, cub::DeviceSelect::Unique(c->cub_tmp.p, b, c->gr_keys_sorted.as<unsigned long long>(),
                                    c->gr_keys_unique.as<unsigned long long>(), c->gr_num.as<int64_t>(), (int64_t)raw,
                                    s),
       "Unique");
    if (!c->replay) {
        int64_t n = 0;
        ck(c, cudaMemcpyAsync(&n, c->gr_num.p, sizeof(int64_t), cudaMemcpyDeviceToHost, s), "copy grid pairs");
        ck(c, cudaStreamSynchronize(s), "sync");
        c->gr_pairs = n;
    }
    const int64_t np = c->gr_pairs;
    ensure(c, c->gr_cellcount, sizeof(uint32_t) * nc);
    ensure(c, c->gr_cells, sizeof(uint32_t) * nc);
    ensure(c, c->gr_ptr, sizeof(int32_t) * std::max<int64_t>(np, 1));
    ck(c, cudaMemsetAsync(c->gr_cellcount.p, 0, sizeof(uint32_t) * nc, s), "memset");
    launch_grid_lists(c->gr_keys_unique.as<unsigned long long>(), np, c->gr_cellcount.as<uint32_t>(),
                      c->gr_ptr.as<int32_t>(), s);
    b = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b, c->gr_cellcount.as<uint32_t>(), c->gr_cells.as<uint32_t>(), (int)nc, s);
    ensure(c, c->cub_tmp, b);
    ck(c, cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, b, c->gr_cellcount.as<uint32_t>(), c->gr_cells.as<uint32_t>(),
                                        (int)nc, s),
       "ExclusiveSum");
    c->build_launches += 12;
    if (g.max_beams_in_cell > 0) {
        ensure(c, c->gr_draws, sizeof(uint32_t) * nc);
        ensure(c, c->gr_draw_off, sizeof(uint32_t) * nc);
        ensure(c, c->gr_pdf, sizeof(float) * nc);
        launch_grid_draws(c->gr_cells.as<uint32_t>(), nc, g.max_beams_in_cell, g.reduction, c->gr_draws.as<uint32_t>(),
                          s);
        b = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, b, c->gr_draws.as<uint32_t>(), c->gr_draw_off.as<uint32_t>(), (int)nc,
                                      s);
        ensure(c, c->cub_tmp, b);
        ck(c, cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, b, c->gr_draws.as<uint32_t>(), c->gr_draw_off.as<uint32_t>(),
                                            (int)nc, s),
           "ExclusiveSum");
        if (!c->replay) {  // the last cell (the sentinel) draws nothing: the total is its offset
            uint32_t t = 0;
            ck(c, cudaMemcpyAsync(&t, c->gr_draw_off.as<uint32_t>() + nc - 1, sizeof(uint32_t),
                                  cudaMemcpyDeviceToHost, s),
               "copy grid draws");
            ck(c, cudaStreamSynchronize(s), "sync");
            c->gr_draws_total = t;
        }
        ensure(c, c->gr_rnd, sizeof(float) * std::max<int64_t>(c->gr_draws_total, 1));
        // std::mt19937_64 takes the int seed converted to its 64-bit result type
        launch_mt64_floats((unsigned long long)(long long)g.seed, c->gr_draws_total, c->gr_rnd.as<float>(), s);
        launch_grid_reduce(c->gr_cells.as<uint32_t>(), nc, g.max_beams_in_cell, g.reduction,
                           c->gr_draw_off.as<uint32_t>(), c->gr_rnd.as<float>(), c->gr_ptr.as<int32_t>(),
                           c->gr_pdf.as<float>(), s);
        c->build_launches += 5;
    }
    // the entries' beam geometry in the final cell order (after the shuffles)
    ensure(c, c->gr_rec_a, sizeof(float4) * std::max<int64_t>(np, 1));
    ensure(c, c->gr_rec_b, sizeof(float4) * std::max<int64_t>(np, 1));
    launch_grid_records(c->gr_ptr.as<int32_t>(), np, org, dir, len,
                        (c->P.bb1d_knn > 0) ? c->bm_r2max.as<float>() : nullptr, radius * radius,
                        c->gr_rec_a.as<float4>(), c->gr_rec_b.as<float4>(), s);
    c->build_launches += 1;
    c->gr_valid = true;
}

int bits_for(uint32_t maxv)
{
    int b = 1;
    while (b < 32 && (maxv >> b)) ++b;
    return b;
}

__global__ void k_iota(int32_t* v, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = i;
}

void build_lbvh(upbp_ctx* c, const uint32_t* codes_sorted, int n, int leaf, DBuf& leaf_codes, DBuf& nodes,
                DBuf& parent_int, DBuf& parent_leaf, DBuf& leaf_boxes, DBuf& node_boxes, DBuf& flags, int& n_leaves)
{
    n_leaves = (n + leaf - 1) / leaf;
    const int ni = std::max(1, n_leaves - 1);
    ensure(c, leaf_codes, sizeof(uint32_t) * n_leaves);
    ensure(c, nodes, sizeof(BNode) * ni);
    ensure(c, parent_int, sizeof(int32_t) * ni);
    ensure(c, parent_leaf, sizeof(int32_t) * n_leaves);
    ensure(c, node_boxes, sizeof(Box) * ni);
    ensure(c, flags, sizeof(int32_t) * ni);
    launch_leaf_codes(codes_sorted, n, leaf, leaf_codes.as<uint32_t>(), c->stream);
    launch_karras(leaf_codes.as<uint32_t>(), n_leaves, nodes.as<BNode>(), parent_int.as<int32_t>(),
                  parent_leaf.as<int32_t>(), c->stream);
    ck(c, cudaMemsetAsync(flags.p, 0, sizeof(int32_t) * ni, c->stream), "memset");
    launch_bottom_up(leaf_boxes.as<Box>(), n_leaves, nodes.as<BNode>(), parent_int.as<int32_t>(),
                     parent_leaf.as<int32_t>(), node_boxes.as<Box>(), flags.as<int32_t>(), c->stream);
    c->build_launches += 3;
}

// The reference's kd-tree over n points pos[idx[i]] in that order (launch_kd_build) in the context's
// kd buffers; bbox = the points' bounding box on the device.
void build_kd_tree(upbp_ctx* c, const float4* pos, const int32_t* idx, int n, const float* bbox)
{
    ensure(c, c->kd_org, sizeof(float4) * (n + 1));
    ensure(c, c->kd_tree, sizeof(float4) * (n + 1));
    ensure(c, c->kd_boxes, sizeof(float) * 6 * (n + 1));
    ensure(c, c->kd_pa, sizeof(int) * (n + 1));
    ensure(c, c->kd_pb, sizeof(int) * (n + 1));
    launch_kd_build(pos, idx, n, bbox, c->kd_org.as<float4>(), c->kd_tree.as<float4>(), c->kd_boxes.as<float>(),
                    c->kd_pa.as<int>(), c->kd_pb.as<int>(), c->stream);
    c->build_launches += kd_build_launches(n);
}

void do_build(upbp_ctx* c)
{
    if (!c->have_params) fail(c, UPBP_ERR_INVALID_ARG, "upbp_set_params was not called");
    if (c->media.empty()) fail(c, UPBP_ERR_INVALID_ARG, "upbp_set_media was not called");
    cudaStream_t s = c->stream;
    c->build_launches = 0;
    mark(c, 0, s);
    const bool knn = (c->P.pb2d_knn > 0 && (c->P.techniques & UPBP_PB2D)) ||
                     (c->P.bb1d_knn > 0 && (c->P.techniques & UPBP_BB1D));
    if (knn) {
        ensure(c, c->knn_status, sizeof(int) * 4);
        ck(c, cudaMemsetAsync(c->knn_status.p, 0, sizeof(int) * 4, s), "memset");
    }
    const upbp_params& P = c->P;
    const int64_t n = c->n_lv;
    const bool mis = !(P.techniques & UPBP_NO_MIS);
    if (mis && n > 0 && c->lv_mis_missing)
        fail(c, UPBP_ERR_INVALID_ARG, "light vertex %s is NULL (only UPBP_NO_MIS runs without it)", c->lv_mis_missing);
    if (mis && c->n_beams > 0 && (P.techniques & UPBP_BB1D) && c->beam_mis_missing)
        fail(c, UPBP_ERR_INVALID_ARG, "%s is NULL (only UPBP_NO_MIS runs without it)", c->beam_mis_missing);
    if (c->bgrid.grid_res > 0) {
        if (c->mode == UPBP_MODE_FP64)
            fail(c, UPBP_ERR_INVALID_ARG, "the beam grid (upbp_set_bb1d_grid) runs in plain and mixed mode");
        if (c->bgrid.max_beams_in_cell > 0 && mis)
            fail(c, UPBP_ERR_INVALID_ARG,
                 "beam reduction (max_beams_in_cell) works only for the estimator without MIS (UPBP_NO_MIS), "
                 "as in the reference");
    }
    // ---- light vertices
    ensure(c, c->lv_pos4, sizeof(float4) * std::max<int64_t>(n, 1));
    ensure(c, c->lv_dir4, sizeof(float4) * std::max<int64_t>(n, 1));
    ensure(c, c->lv_thr4, sizeof(float4) * std::max<int64_t>(n, 1));
    ensure(c, c->lv_info4, sizeof(int4) * std::max<int64_t>(n, 1));
    ensure(c, c->lv_inmed, sizeof(uint32_t) * std::max<int64_t>(n, 1));
    ensure(c, c->ph_lv, sizeof(int32_t) * std::max<int64_t>(n, 1));
    launch_pack_lights(c->lv_pos_in.as<float>(), c->lv_thr_in.as<float>(), c->lv_dir_in.as<float>(),
                       c->lv_cont_in.as<float>(), c->lv_pidx_in.as<int32_t>(), c->lv_plen_in.as<int32_t>(),
                       c->lv_med_in.as<int32_t>(), c->lv_flags_in.as<uint32_t>(), n, c->lv_pos4.as<float4>(),
                       c->lv_dir4.as<float4>(), c->lv_thr4.as<float4>(), c->lv_info4.as<int4>(),
                       c->lv_inmed.as<uint32_t>(), s);
    c->build_launches += 1;
    if (c->mode != UPBP_MODE_PLAIN && n > 0 && mis) {
        ensure(c, c->light_sums, sizeof(LightSum) * n);
        // the PB2D / BB1D walks see beamType | techniques, PP3D the techniques: same terms
        launch_light_sums(c->lv_mis.as<upbp_mis>(), c->path_ends.as<int32_t>(), c->n_paths, P.techniques,
                          P.query_beam_type, P.photon_beam_type, c->light_sums.as<LightSum>(), s);
        c->build_launches += 1;
    }
    // ---- photons = light vertices in media (stable compaction keeps light-vertex order)
    if (!c->replay) c->n_ph = 0;
    if (n > 0) {
        ensure(c, c->bbox_partial, sizeof(int32_t) * 8 + sizeof(float) * 6 * 1024);
        int32_t* d_nsel = c->bbox_partial.as<int32_t>();
        ensure(c, c->ph_lv_sorted, sizeof(int32_t) * n);
        {
            ensure(c, c->ph_keys, sizeof(int32_t) * n);
            k_iota<<<(int)((n + 255) / 256), 256, 0, s>>>(c->ph_keys.as<int32_t>(), (int)n);
            size_t b = 0;
            cub::DeviceSelect::Flagged(nullptr, b, c->ph_keys.as<int32_t>(), c->lv_inmed.as<uint32_t>(),
                                       c->ph_lv.as<int32_t>(), d_nsel, (int)n, s);
            ensure(c, c->cub_tmp, b);
            ck(c, cub::DeviceSelect::Flagged(c->cub_tmp.p, b, c->ph_keys.as<int32_t>(), c->lv_inmed.as<uint32_t>(),
                                             c->ph_lv.as<int32_t>(), d_nsel, (int)n, s),
               "DeviceSelect");
            c->build_launches += 2;
        }
        if (!c->replay) {  // a replay reuses the count of the build it repeats
            int32_t h_nsel = 0;
            ck(c, cudaMemcpyAsync(&h_nsel, d_nsel, sizeof(int32_t), cudaMemcpyDeviceToHost, s), "copy n_sel");
            ck(c, cudaStreamSynchronize(s), "sync");
            c->n_ph = h_nsel;
        }
    }
    const int nph = c->n_ph;
    const int blocks = std::max(1, std::min(1024, (nph + 255) / 256));
    if (nph > 0) {
        ensure(c, c->bbox_ph, sizeof(float) * 6);
        float* partial = reinterpret_cast<float*>(c->bbox_partial.as<int32_t>() + 8);
        launch_bbox_partial(c->lv_pos4.as<float4>(), c->ph_lv.as<int32_t>(), nph, partial, blocks, s);
        launch_bbox_final(partial, blocks, c->bbox_ph.as<float>(), s);
        if (!c->replay)
            ck(c, cudaMemcpyAsync(c->hg_bbox, c->bbox_ph.p, sizeof(float) * 6, cudaMemcpyDeviceToHost, s), "bbox");
        c->build_launches += 2;
    }
    // ---- PP3D hash grid (HashGrid::Build, Misc/HashGrid.hxx:47-126)
    if (nph > 0 && (P.techniques & UPBP_PP3D)) {
        const int cells = std::max(1, P.hash_cells);
        const float cell_size = P.radius_pp3d * 2.f;
        c->hg_inv_cell = 1.f / cell_size;
        ensure(c, c->ph_keys, sizeof(uint32_t) * nph);
        ensure(c, c->ph_keys_sorted, sizeof(uint32_t) * nph);
        ensure(c, c->hg_start, sizeof(int32_t) * cells);
        ensure(c, c->hg_end, sizeof(int32_t) * cells);
        ensure(c, c->hg_pos, sizeof(float4) * nph);
        launch_hash_keys(c->lv_pos4.as<float4>(), c->ph_lv.as<int32_t>(), nph, c->bbox_ph.as<float>(),
                         c->hg_inv_cell, cells, c->ph_keys.as<uint32_t>(), s);
        sort_pairs(c, c->ph_keys.as<uint32_t>(), c->ph_keys_sorted.as<uint32_t>(), c->ph_lv.as<int32_t>(),
                   c->ph_lv_sorted.as<int32_t>(), nph, bits_for((uint32_t)cells - 1));
        ck(c, cudaMemsetAsync(c->hg_start.p, 0, sizeof(int32_t) * cells, s), "memset");
        ck(c, cudaMemsetAsync(c->hg_end.p, 0, sizeof(int32_t) * cells, s), "memset");
        launch_hash_ranges(c->ph_keys_sorted.as<uint32_t>(), c->ph_lv_sorted.as<int32_t>(), c->lv_pos4.as<float4>(),
                           nph, c->hg_start.as<int32_t>(), c->hg_end.as<int32_t>(), c->hg_pos.as<float4>(), s);
        c->build_launches += 2;
    }
    // ---- PB2D photon LBVH
    c->pb_n_leaves = 0;
    if (nph > 0 && (P.techniques & UPBP_PB2D)) {
        ensure(c, c->ph_keys, sizeof(uint32_t) * nph);
        ensure(c, c->ph_keys_sorted, sizeof(uint32_t) * nph);
        ensure(c, c->pb_pos, sizeof(float4) * nph);
        launch_morton_points(c->lv_pos4.as<float4>(), c->ph_lv.as<int32_t>(), nph, c->bbox_ph.as<float>(),
                             c->ph_keys.as<uint32_t>(), s);
        sort_pairs(c, c->ph_keys.as<uint32_t>(), c->ph_keys_sorted.as<uint32_t>(), c->ph_lv.as<int32_t>(),
                   c->ph_lv_sorted.as<int32_t>(), nph, 30);
        launch_gather_photons(c->ph_lv_sorted.as<int32_t>(), c->lv_pos4.as<float4>(), nph, c->pb_pos.as<float4>(), s);
        const int leaf = std::max(1, c->pb2d_leaf);
        const int nl = (nph + leaf - 1) / leaf;
        ensure(c, c->pb_leaf_boxes, sizeof(Box) * nl);
        const float eps = 1e-5f + 1e-3f * P.radius_pb2d;
        launch_photon_leaf_boxes(c->pb_pos.as<float4>(), nph, leaf, P.radius_pb2d, eps, c->pb_leaf_boxes.as<Box>(), s);
        build_lbvh(c, c->ph_keys_sorted.as<uint32_t>(), nph, leaf, c->pb_leaf_codes, c->pb_nodes, c->pb_parent_int,
                   c->pb_parent_leaf, c->pb_leaf_boxes, c->pb_node_boxes, c->pb_flags, c->pb_n_leaves);
        c->build_launches += 3;
        if (P.pb2d_knn > 0 && (P.techniques & UPBP_PB2D)) {
            // KNN photon radii over the LBVH just built (its boxes hold the points), then refit
            // the boxes to the per-photon spheres
            ensure(c, c->pb_r2, sizeof(float) * nph);
            if (P.knn_exact) {
                launch_photon_knn_r2(c->pb_pos.as<float4>(), nph, c->pb_nodes.as<BNode>(), c->pb_n_leaves, leaf,
                                     P.pb2d_knn, P.radius_pb2d, c->pb_r2.as<float>(), c->knn_status.as<int>(), s);
            } else {
                // the reference's search over the photons in light-vertex order (EmbreeBre::build,
                // Bre.cxx:685-699), queried at every photon of the LBVH
                build_kd_tree(c, c->lv_pos4.as<float4>(), c->ph_lv.as<int32_t>(), nph, c->bbox_ph.as<float>());
                launch_kd_photon_r2(c->kd_tree.as<float4>(), nph, c->pb_pos.as<float4>(), nph, P.pb2d_knn,
                                    P.radius_pb2d, c->pb_r2.as<float>(), s);
            }
            launch_photon_leaf_boxes_r2(c->pb_pos.as<float4>(), c->pb_r2.as<float>(), nph, leaf, 1e-5f,
                                        c->pb_leaf_boxes.as<Box>(), s);
            const int ni = std::max(1, c->pb_n_leaves - 1);
            ck(c, cudaMemsetAsync(c->pb_flags.p, 0, sizeof(int32_t) * ni, s), "memset");
            launch_bottom_up(c->pb_leaf_boxes.as<Box>(), c->pb_n_leaves, c->pb_nodes.as<BNode>(),
                             c->pb_parent_int.as<int32_t>(), c->pb_parent_leaf.as<int32_t>(),
                             c->pb_node_boxes.as<Box>(), c->pb_flags.as<int32_t>(), s);
            c->build_launches += 3;
        }
    }
    // ---- BB1D beams: pieces + LBVH (a replay keeps the piece count of the build it repeats)
    const int replay_pieces = c->n_pieces;
    c->n_pieces = 0;
    c->bm_n_leaves = 0;
    c->gr_valid = false;
    const int64_t nb = c->n_beams;
    if (nb > 0 && (P.techniques & UPBP_BB1D)) {
        const float r = P.radius_bb1d;
        ensure(c, c->bm_thr4, sizeof(float4) * nb);
        ensure(c, c->bm_pdf4, sizeof(float4) * nb);
        ensure(c, c->bm_link, sizeof(int2) * nb);
        ensure(c, c->bm_radius, sizeof(float) * nb);
        launch_pack_beams(c->b_thr_in.as<float>(), c->b_flags_in.as<uint32_t>(), c->b_rsp_in.as<float>(),
                          c->b_rsr_in.as<float>(), c->b_lpw_in.as<float>(), c->b_rsf_in.as<uint32_t>(),
                          c->b_lv_in.as<int32_t>(), c->b_med_in.as<int32_t>(), nb, r, c->bm_thr4.as<float4>(),
                          c->bm_pdf4.as<float4>(), c->bm_link.as<int2>(), c->bm_radius.as<float>(), s);
        const float* rchange = nullptr;
        const float* r2max = nullptr;
        if (P.bb1d_knn > 0) {
            // KNN beam radii from the beam origins
            const int n = (int)nb;
            ensure(c, c->bo_pos, sizeof(float4) * n);
            ensure(c, c->bo_pts, sizeof(float4) * n);
            ensure(c, c->bo_codes, sizeof(uint32_t) * n);
            ensure(c, c->bo_codes_sorted, sizeof(uint32_t) * n);
            ensure(c, c->bo_idx, sizeof(int32_t) * n);
            ensure(c, c->bo_idx_sorted, sizeof(int32_t) * n);
            ensure(c, c->bo_bbox, sizeof(float) * 6);
            ensure(c, c->bm_rchange, sizeof(float) * n);
            ensure(c, c->bm_r2max, sizeof(float) * n);
            ensure(c, c->bbox_partial, sizeof(int32_t) * 8 + sizeof(float) * 6 * 1024);
            launch_beam_origins(c->b_origin.as<float>(), n, c->bo_pos.as<float4>(), s);
            const int ob = std::max(1, std::min(1024, (n + 255) / 256));
            float* part = reinterpret_cast<float*>(c->bbox_partial.as<int32_t>() + 8);
            launch_bbox_partial(c->bo_pos.as<float4>(), nullptr, n, part, ob, s);
            launch_bbox_final(part, ob, c->bo_bbox.as<float>(), s);
            c->build_launches += 3;
            if (!P.knn_exact) {
                // the reference's search over the beam origins in beam order (PhBeams.cxx:80-91)
                build_kd_tree(c, c->bo_pos.as<float4>(), nullptr, n, c->bo_bbox.as<float>());
                // two searches per beam (origin, end point), taken in Morton order of the points
                const int nq = 2 * n;
                ensure(c, c->kd_qpts, sizeof(float4) * nq);
                ensure(c, c->kd_qcodes, sizeof(uint32_t) * nq);
                ensure(c, c->kd_qcodes_sorted, sizeof(uint32_t) * nq);
                ensure(c, c->kd_qidx, sizeof(int32_t) * nq);
                ensure(c, c->kd_qidx_sorted, sizeof(int32_t) * nq);
                ensure(c, c->kd_qd2, sizeof(float) * nq);
                launch_kd_beam_points(c->b_origin.as<float>(), c->b_dir.as<float>(), c->b_len.as<float>(), n,
                                      c->kd_qpts.as<float4>(), s);
                k_iota<<<(nq + 255) / 256, 256, 0, s>>>(c->kd_qidx.as<int32_t>(), nq);
                launch_morton_points(c->kd_qpts.as<float4>(), c->kd_qidx.as<int32_t>(), nq, c->bo_bbox.as<float>(),
                                     c->kd_qcodes.as<uint32_t>(), s);
                sort_pairs(c, c->kd_qcodes.as<uint32_t>(), c->kd_qcodes_sorted.as<uint32_t>(),
                           c->kd_qidx.as<int32_t>(), c->kd_qidx_sorted.as<int32_t>(), nq, 30);
                launch_kd_knn_sorted(c->kd_tree.as<float4>(), n, c->kd_qpts.as<float4>(),
                                     c->kd_qidx_sorted.as<int32_t>(), nq, P.bb1d_knn, c->kd_qd2.as<float>(), s);
                launch_kd_beam_finish(c->kd_qd2.as<float>(), c->b_len.as<float>(), n, r, c->bm_radius.as<float>(),
                                      c->bm_rchange.as<float>(), c->bm_r2max.as<float>(), s);
                c->build_launches += 5;
            } else {  // the exact search: an LBVH over the beam origins, two queries per beam
                k_iota<<<(n + 255) / 256, 256, 0, s>>>(c->bo_idx.as<int32_t>(), n);
                launch_morton_points(c->bo_pos.as<float4>(), c->bo_idx.as<int32_t>(), n, c->bo_bbox.as<float>(),
                                     c->bo_codes.as<uint32_t>(), s);
                sort_pairs(c, c->bo_codes.as<uint32_t>(), c->bo_codes_sorted.as<uint32_t>(), c->bo_idx.as<int32_t>(),
                           c->bo_idx_sorted.as<int32_t>(), n, 30);
                launch_gather_photons(c->bo_idx_sorted.as<int32_t>(), c->bo_pos.as<float4>(), n, c->bo_pts.as<float4>(),
                                      s);
                constexpr int kOriginLeaf = 4;
                ensure(c, c->bo_leaf_boxes, sizeof(Box) * ((n + kOriginLeaf - 1) / kOriginLeaf));
                launch_photon_leaf_boxes(c->bo_pts.as<float4>(), n, kOriginLeaf, 0.f, 1e-6f, c->bo_leaf_boxes.as<Box>(), s);
                build_lbvh(c, c->bo_codes_sorted.as<uint32_t>(), n, kOriginLeaf, c->bo_leaf_codes, c->bo_nodes,
                           c->bo_parent_int, c->bo_parent_leaf, c->bo_leaf_boxes, c->bo_node_boxes, c->bo_flags,
                           c->bo_n_leaves);
                launch_beam_knn(c->b_origin.as<float>(), c->b_dir.as<float>(), c->b_len.as<float>(), n,
                                c->bo_nodes.as<BNode>(), c->bo_n_leaves, c->bo_pts.as<float4>(), kOriginLeaf, P.bb1d_knn,
                                r, c->bm_radius.as<float>(), c->bm_rchange.as<float>(), c->bm_r2max.as<float>(),
                                c->knn_status.as<int>(), s);
                c->build_launches += 9;
            }
            rchange = c->bm_rchange.as<float>();
            r2max = c->bm_r2max.as<float>();
        }
        const float piece_len = std::max(1e-6f, c->piece_len_r * r);
        ensure(c, c->bm_counts, sizeof(int32_t) * (nb + 1));
        ensure(c, c->bm_offsets, sizeof(int32_t) * (nb + 1));
        launch_piece_counts(c->b_len.as<float>(), nb, piece_len, c->bm_counts.as<int32_t>(), s);
        ck(c, cudaMemsetAsync(c->bm_counts.as<int32_t>() + nb, 0, sizeof(int32_t), s), "memset");
        size_t b = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, b, c->bm_counts.as<int32_t>(), c->bm_offsets.as<int32_t>(),
                                      (int)(nb + 1), s);
        ensure(c, c->cub_tmp, b);
        ck(c, cub::DeviceScan::ExclusiveSum(c->cub_tmp.p, b, c->bm_counts.as<int32_t>(), c->bm_offsets.as<int32_t>(),
                                            (int)(nb + 1), s),
           "ExclusiveSum");
        int32_t total = replay_pieces;
        if (!c->replay) {
            ck(c, cudaMemcpyAsync(&total, c->bm_offsets.as<int32_t>() + nb, sizeof(int32_t), cudaMemcpyDeviceToHost,
                                  s),
               "copy pieces");
            ck(c, cudaStreamSynchronize(s), "sync");
        }
        const int np = total;
        c->n_pieces = np;
        ensure(c, c->pc_a2, sizeof(float4) * np);
        ensure(c, c->pc_b2, sizeof(float4) * np);
        ensure(c, c->pc_c2, sizeof(float4) * np);
        ensure(c, c->pc_boxes2, sizeof(Box) * np);
        ensure(c, c->pc_codes, sizeof(uint32_t) * np);
        ensure(c, c->pc_codes_sorted, sizeof(uint32_t) * np);
        ensure(c, c->pc_perm, sizeof(int32_t) * np);
        ensure(c, c->pc_perm_sorted, sizeof(int32_t) * np);
        ensure(c, c->bbox_pc, sizeof(float) * 6);
        // Morton codes of the pieces' midpoints in the box of the beam segments, sorted; the piece
        // records are then written directly in that order
        const int bblocks = (int)std::max<int64_t>(1, std::min<int64_t>(1024, (nb + 255) / 256));
        ensure(c, c->bbox_partial, sizeof(int32_t) * 8 + sizeof(float) * 6 * 1024);
        float* partial = reinterpret_cast<float*>(c->bbox_partial.as<int32_t>() + 8);
        launch_bbox_beams_partial(c->b_origin.as<float>(), c->b_dir.as<float>(), c->b_len.as<float>(), nb, partial,
                                  bblocks, s);
        launch_bbox_final(partial, bblocks, c->bbox_pc.as<float>(), s);
        launch_piece_codes(c->b_origin.as<float>(), c->b_dir.as<float>(), c->b_len.as<float>(), nb,
                           c->bm_offsets.as<int32_t>(), np, c->bbox_pc.as<float>(), c->pc_codes.as<uint32_t>(),
                           c->pc_perm.as<int32_t>(), s);
        sort_pairs(c, c->pc_codes.as<uint32_t>(), c->pc_codes_sorted.as<uint32_t>(), c->pc_perm.as<int32_t>(),
                   c->pc_perm_sorted.as<int32_t>(), np, 30);
        const float eps = bb1d_box_eps(r);
        launch_emit_sorted(c->b_origin.as<float>(), c->b_dir.as<float>(), c->b_len.as<float>(),
                           c->b_med_in.as<int32_t>(), nb, c->bm_offsets.as<int32_t>(), c->pc_perm_sorted.as<int32_t>(),
                           np, r, eps, rchange ? c->bm_radius.as<float>() : nullptr, rchange, r2max,
                           c->pc_a2.as<float4>(), c->pc_b2.as<float4>(), c->pc_c2.as<float4>(), c->pc_boxes2.as<Box>(),
                           s);
        const int leaf = std::max(1, c->bb1d_leaf);
        const int nl = (np + leaf - 1) / leaf;
        ensure(c, c->bm_leaf_boxes, sizeof(Box) * nl);
        launch_box_leaf_boxes(c->pc_boxes2.as<Box>(), np, leaf, c->bm_leaf_boxes.as<Box>(), s);
        build_lbvh(c, c->pc_codes_sorted.as<uint32_t>(), np, leaf, c->bm_leaf_codes, c->bm_nodes, c->bm_parent_int,
                   c->bm_parent_leaf, c->bm_leaf_boxes, c->bm_node_boxes, c->bm_flagsbuf, c->bm_n_leaves);
        c->build_launches += 8;
        if (c->mode != UPBP_MODE_PLAIN) {
            ensure(c, c->pc_pay, sizeof(PiecePayload) * np);
            // without MIS the payload holds the beam's throughput, flags and radius only
            launch_piece_payload(c->pc_c2.as<float4>(), np, c->bm_thr4.as<float4>(), c->bm_pdf4.as<float4>(),
                                 c->bm_link.as<int2>(), c->bm_radius.as<float>(),
                                 mis ? c->lv_info4.as<int4>() : nullptr, mis ? c->lv_mis.as<upbp_mis>() : nullptr,
                                 mis ? c->light_sums.as<LightSum>() : nullptr, c->pc_pay.as<PiecePayload>(), s);
            c->build_launches += 1;
            if (c->bgrid.grid_res > 0) {
                // the grid gather's payload: one per beam (the piece payload's layout)
                ensure(c, c->gr_pay, sizeof(PiecePayload) * nb);
                launch_piece_payload(nullptr, (int)nb, c->bm_thr4.as<float4>(), c->bm_pdf4.as<float4>(),
                                     c->bm_link.as<int2>(), c->bm_radius.as<float>(),
                                     mis ? c->lv_info4.as<int4>() : nullptr, mis ? c->lv_mis.as<upbp_mis>() : nullptr,
                                     mis ? c->light_sums.as<LightSum>() : nullptr, c->gr_pay.as<PiecePayload>(), s);
                c->build_launches += 1;
            }
        }
        if (c->bgrid.grid_res > 0) build_grid(c, s, r, rchange ? c->bm_radius.as<float>() : nullptr, rchange);
    }
    mark(c, 1, s);
    ck(c, cudaGetLastError(), "build launch");
    if (knn && !c->replay) {  // the KNN searches' traversal stacks must not have overflowed
        int h = 0;
        ck(c, cudaMemcpyAsync(&h, c->knn_status.p, sizeof(int), cudaMemcpyDeviceToHost, s), "knn status");
        ck(c, cudaStreamSynchronize(s), "sync");
        if (h) fail(c, UPBP_ERR_CAPACITY, "KNN radius search: traversal stack overflow");
    }
    c->built = true;
    if (!c->replay) c->evaluated = false;
}

GatherConsts make_consts(upbp_ctx* c)
{
    GatherConsts K{};
    K.P = c->P;
    K.n_media = (int)c->media.size();
    for (int i = 0; i < K.n_media; ++i) K.media[i] = c->media[i];
    K.has_bb1d_beams = (c->P.techniques & UPBP_BB1D) && c->n_beams > 0;
    K.eps = 1e-4f;
    K.bb1d_extra = bb1d_reach_extra(c->P.radius_bb1d);
    return K;
}

LightSoA light_soa(upbp_ctx* c)
{
    LightSoA L{};
    L.pos = c->lv_pos4.as<float4>();
    L.dir = c->lv_dir4.as<float4>();
    L.thr = c->lv_thr4.as<float4>();
    L.info = c->lv_info4.as<int4>();
    L.mis = c->lv_mis.as<upbp_mis>();
    L.path_ends = c->path_ends.as<int32_t>();
    L.sums = c->mode != UPBP_MODE_PLAIN ? c->light_sums.as<LightSum>() : nullptr;
    L.n = c->n_lv;
    return L;
}

SegQueriesDev seg_dev(upbp_ctx* c)
{
    SegQueriesDev Q{};
    Q.origin = c->sq_origin.as<float>();
    Q.direction = c->sq_dir.as<float>();
    Q.seg_begin = c->sq_seg_begin.as<int32_t>();
    Q.seg_count = c->sq_seg_count.as<int32_t>();
    Q.flags = c->sq_flags.as<uint32_t>();
    Q.path_length = c->sq_plen.as<int32_t>();
    Q.last_pdf_w_inv = c->sq_lpw.as<float>();
    Q.throughput = c->sq_thr.as<float>();
    Q.pixel = c->sq_pixel.as<int32_t>();
    Q.cam_mis_begin = c->sq_cam_begin.as<int64_t>();
    Q.seg_dist_min = c->seg_dmin.as<float>();
    Q.seg_dist_max = c->seg_dmax.as<float>();
    Q.seg_pdf = c->seg_pdf.as<float>();
    Q.seg_rev_pdf = c->seg_rev.as<float>();
    Q.seg_attenuation = c->seg_att.as<float>();
    Q.seg_medium = c->seg_med.as<int32_t>();
    Q.n = c->n_sq;
    return Q;
}

HashGridDev hash_dev(upbp_ctx* c)
{
    HashGridDev G{};
    G.pos = c->hg_pos.as<float4>();
    G.start = c->hg_start.as<int32_t>();
    G.end = c->hg_end.as<int32_t>();
    for (int k = 0; k < 3; ++k) {
        G.bbox_min[k] = c->hg_bbox[k];
        G.bbox_max[k] = c->hg_bbox[3 + k];
    }
    G.inv_cell = c->hg_inv_cell;
    G.r2 = c->P.radius_pp3d * c->P.radius_pp3d;
    G.cells = std::max(1, c->P.hash_cells);
    G.n = (c->P.techniques & UPBP_PP3D) ? c->n_ph : 0;
    return G;
}

PointQueriesDev point_dev(upbp_ctx* c)
{
    PointQueriesDev Q{};
    Q.position = c->pq_pos.as<float>();
    Q.dir_fix = c->pq_dir.as<float>();
    Q.medium_id = c->pq_med.as<int32_t>();
    Q.path_length = c->pq_plen.as<int32_t>();
    Q.throughput = c->pq_thr.as<float>();
    Q.pixel = c->pq_pixel.as<int32_t>();
    Q.cam_mis_begin = c->pq_cam_begin.as<int64_t>();
    Q.n = c->n_pq;
    return Q;
}

PhotonBVH photon_bvh(upbp_ctx* c)
{
    PhotonBVH B{};
    B.pos = c->pb_pos.as<float4>();
    B.nodes = c->pb_nodes.as<BNode>();
    B.n = (c->P.techniques & UPBP_PB2D) ? c->n_ph : 0;
    B.leaf = std::max(1, c->pb2d_leaf);
    B.n_leaves = c->pb_n_leaves;
    B.r2 = (c->P.pb2d_knn > 0 && (c->P.techniques & UPBP_PB2D) && c->n_ph > 0) ? c->pb_r2.as<float>() : nullptr;
    return B;
}

BeamBVH beam_bvh(upbp_ctx* c)
{
    BeamBVH B{};
    B.pa = c->pc_a2.as<float4>();
    B.pb = c->pc_b2.as<float4>();
    B.pc = c->pc_c2.as<float4>();
    B.nodes = c->bm_nodes.as<BNode>();
    B.n = c->n_pieces;
    B.pay = c->mode != UPBP_MODE_PLAIN ? c->pc_pay.as<PiecePayload>() : nullptr;
    B.leaf = std::max(1, c->bb1d_leaf);
    B.n_leaves = c->bm_n_leaves;
    return B;
}

BeamGrid grid_dev(upbp_ctx* c)
{
    BeamGrid G{};
    G.hdr = c->gr_hdr.as<GridHeader>();
    G.cells = c->gr_cells.as<uint32_t>();
    G.pdf = c->bgrid.max_beams_in_cell > 0 ? c->gr_pdf.as<float>() : nullptr;
    G.ptr = c->gr_ptr.as<int32_t>();
    G.rec_a = c->gr_rec_a.as<float4>();
    G.rec_b = c->gr_rec_b.as<float4>();
    G.medium = c->b_med_in.as<int32_t>();
    G.pay = c->mode != UPBP_MODE_PLAIN ? c->gr_pay.as<PiecePayload>() : nullptr;
    return G;
}

BeamSoA beam_soa(upbp_ctx* c)
{
    BeamSoA S{};
    S.thr = c->bm_thr4.as<float4>();
    S.pdf = c->bm_pdf4.as<float4>();
    S.link = c->bm_link.as<int2>();
    S.radius = c->bm_radius.as<float>();
    S.rchange = (c->P.bb1d_knn > 0 && c->n_beams > 0 && (c->P.techniques & UPBP_BB1D)) ? c->bm_rchange.as<float>()
                                                                                          : nullptr;
    S.radius_const = c->P.radius_bb1d;  // what k_pack_beams stores for every beam without KNN radii
    S.n = c->n_beams;
    return S;
}

// FP64 suffix sums of the camera walks, per segment query and per point query.
void prepare_cam_sums(upbp_ctx* c, cudaStream_t s, const CamSum** cs_seg, const CamSum** cs_pt)
{
    const int64_t nq = c->n_sq, np = c->n_pq;
    const upbp_mis* cam = c->cam_mis.as<upbp_mis>();
    ensure(c, c->cam_sums_seg, sizeof(CamSum) * std::max<int64_t>(nq, 1));
    ensure(c, c->cam_sums_pt, sizeof(CamSum) * std::max<int64_t>(np, 1));
    const uint32_t tq = c->P.query_beam_type | c->P.techniques;
    launch_cam_sums(cam, c->sq_cam_begin.as<int64_t>(), c->sq_plen.as<int32_t>(), nq, tq, c->P.query_beam_type,
                    c->P.photon_beam_type, c->cam_sums_seg.as<CamSum>(), s);
    launch_cam_sums(cam, c->pq_cam_begin.as<int64_t>(), c->pq_plen.as<int32_t>(), np, c->P.techniques,
                    c->P.query_beam_type, c->P.photon_beam_type, c->cam_sums_pt.as<CamSum>(), s);
    *cs_seg = c->cam_sums_seg.as<CamSum>();
    *cs_pt = c->cam_sums_pt.as<CamSum>();
    c->eval_launches += 2;
}

// The generic-precision gathers (FP64 evaluation, adjoint) over the context's structures.
// Order the segment queries along a Morton curve of their midpoints, so that the warps in flight
// traverse neighbouring parts of the LBVHs (L2 reuse).  nullptr: keep the given order.
const int32_t* query_order(upbp_ctx* c, const SegQueriesDev& Q, cudaStream_t s)
{
    const int64_t nq = Q.n;
    const bool have_bbox = c->n_pieces > 0 || c->n_ph > 0;
    if (!c->order_queries || nq <= 1 || !have_bbox) return nullptr;
    ensure(c, c->q_keys, sizeof(uint32_t) * nq);
    ensure(c, c->q_keys_sorted, sizeof(uint32_t) * nq);
    ensure(c, c->q_iota, sizeof(int32_t) * nq);
    ensure(c, c->q_order, sizeof(int32_t) * nq);
    launch_query_keys(Q, c->n_pieces > 0 ? c->bbox_pc.as<float>() : c->bbox_ph.as<float>(), c->query_order,
                      c->P.image_width, c->q_keys.as<uint32_t>(), c->q_iota.as<int32_t>(), s);
    size_t b = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, b, c->q_keys.as<uint32_t>(), c->q_keys_sorted.as<uint32_t>(),
                                    c->q_iota.as<int32_t>(), c->q_order.as<int32_t>(), (int)nq, 0, 30, s);
    ensure(c, c->cub_tmp, b);
    ck(c, cub::DeviceRadixSort::SortPairs(c->cub_tmp.p, b, c->q_keys.as<uint32_t>(), c->q_keys_sorted.as<uint32_t>(),
                                          c->q_iota.as<int32_t>(), c->q_order.as<int32_t>(), (int)nq, 0, 30, s),
       "SortPairs");
    c->eval_launches += 5;
    return c->q_order.as<int32_t>();
}

gen::GenLaunch generic_launch(upbp_ctx* c, const CamSum* cs_seg, const CamSum* cs_pt, int grad_medium)
{
    gen::GenLaunch A{};
    A.K = make_consts(c);
    A.G.n_media = (int)c->media_raw.size();
    for (int i = 0; i < A.G.n_media; ++i) A.G.raw[i] = c->media_raw[i];
    A.G.grad_medium = grad_medium;
    A.L = light_soa(c);
    A.photons = photon_bvh(c);
    A.beams = beam_bvh(c);
    A.bs = beam_soa(c);
    A.hash = hash_dev(c);
    A.sq = seg_dev(c);
    A.pq = point_dev(c);
    A.cam = c->cam_mis.as<upbp_mis>();
    A.cs_seg = cs_seg;
    A.cs_pt = cs_pt;
    if (!c->num_sms) ck(c, cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device), "attr");
    ensure(c, c->work, sizeof(unsigned int) * 4);
    ensure(c, c->status, sizeof(int) * 4);
    ck(c, cudaMemsetAsync(c->work.p, 0, sizeof(unsigned int) * 4, c->stream), "memset");
    ck(c, cudaMemsetAsync(c->status.p, 0, sizeof(int) * 4, c->stream), "memset");
    A.work = c->work.as<unsigned int>();
    A.status = c->status.as<int>();
    A.bb1d_grid = c->num_sms * gen::generic_bb1d_blocks_per_sm(grad_medium >= 0);
    A.pb2d_grid = c->num_sms * gen::generic_pb2d_blocks_per_sm(grad_medium >= 0);
    A.bp2d_grid = c->num_sms * gen::generic_bp2d_blocks_per_sm(grad_medium >= 0);
    A.order = query_order(c, A.sq, c->stream);
    return A;
}

void record_status(upbp_ctx* c, cudaStream_t s)
{
    if (!c->status_host) ck(c, cudaHostAlloc((void**)&c->status_host, sizeof(int), cudaHostAllocDefault),
                            "cudaHostAlloc");
    ck(c, cudaMemcpyAsync(c->status_host, c->status.p, sizeof(int), cudaMemcpyDeviceToHost, s), "status");
    c->status_pending = true;
}

void do_evaluate(upbp_ctx* c)
{
    if (!c->built) fail(c, UPBP_ERR_NOT_BUILT, "upbp_build was not called");
    cudaStream_t s = c->stream;
    c->eval_launches = 0;
    c->status_pending = false;
    const GatherConsts K = make_consts(c);
    const LightSoA L = light_soa(c);
    const int64_t nq = c->n_sq, np = c->n_pq;
    const size_t npix = (size_t)std::max(0, c->P.image_width) * (size_t)std::max(0, c->P.image_height);
    ensure(c, c->image, sizeof(float) * 3 * std::max<size_t>(npix, 1));
    ensure(c, c->out_pb2d, sizeof(float) * 3 * std::max<int64_t>(nq, 1));
    ensure(c, c->out_bb1d, sizeof(float) * 3 * std::max<int64_t>(nq, 1));
    ensure(c, c->out_pp3d, sizeof(float) * 3 * std::max<int64_t>(np, 1));
    ensure(c, c->cnt_pb2d, sizeof(uint32_t) * std::max<int64_t>(nq, 1));
    ensure(c, c->cnt_bb1d, sizeof(uint32_t) * std::max<int64_t>(nq, 1));
    ensure(c, c->cnt_pp3d, sizeof(uint32_t) * std::max<int64_t>(np, 1));
    ensure(c, c->hash_pb2d, sizeof(uint64_t) * std::max<int64_t>(nq, 1));
    ensure(c, c->hash_bb1d, sizeof(uint64_t) * std::max<int64_t>(nq, 1));
    ensure(c, c->hash_pp3d, sizeof(uint64_t) * std::max<int64_t>(np, 1));
    const bool bp2d = (c->P.techniques & UPBP_BP2D) && np > 0 && c->n_pieces > 0;
    if (bp2d) {
        ensure(c, c->out_bp2d, sizeof(float) * 3 * np);
        ensure(c, c->cnt_bp2d, sizeof(uint32_t) * np);
        ensure(c, c->hash_bp2d, sizeof(uint64_t) * np);
    }
    ensure(c, c->tested, sizeof(unsigned long long) * 4);
    ck(c, cudaMemsetAsync(c->tested.p, 0, sizeof(unsigned long long) * 4, s), "memset");
    const upbp_mis* cam = c->cam_mis.as<upbp_mis>();
    float* img = npix ? c->image.as<float>() : nullptr;
    unsigned long long* tested = c->tested.as<unsigned long long>();

    const bool mixed = c->mode == UPBP_MODE_MIXED;
    const bool mis = !(c->P.techniques & UPBP_NO_MIS);
    if (mis && nq > 0 && c->sq_mis_missing)
        fail(c, UPBP_ERR_INVALID_ARG, "segment query %s is NULL (only UPBP_NO_MIS runs without it)", c->sq_mis_missing);
    const CamSum* cs_seg = nullptr;
    const CamSum* cs_pt = nullptr;
    if (c->mode != UPBP_MODE_PLAIN && mis) prepare_cam_sums(c, s, &cs_seg, &cs_pt);
    if (c->mode == UPBP_MODE_FP64) {
        // FP64 oracle on the GPU: the same candidates, FP64 geometry, contributions and MIS
        gen::GenLaunch A = generic_launch(c, cs_seg, cs_pt, -1);
        A.out_pp3d = gen::GenOut{c->out_pp3d.as<float>(), img, c->cnt_pp3d.as<uint32_t>(),
                                 c->hash_pp3d.as<unsigned long long>(), nullptr, nullptr};
        A.out_pb2d = gen::GenOut{c->out_pb2d.as<float>(), img, c->cnt_pb2d.as<uint32_t>(),
                                 c->hash_pb2d.as<unsigned long long>(), nullptr, nullptr};
        A.out_bb1d = gen::GenOut{c->out_bb1d.as<float>(), img, c->cnt_bb1d.as<uint32_t>(),
                                 c->hash_bb1d.as<unsigned long long>(), nullptr, nullptr};
        if (bp2d)
            A.out_bp2d = gen::GenOut{c->out_bp2d.as<float>(), img, c->cnt_bp2d.as<uint32_t>(),
                                     c->hash_bp2d.as<unsigned long long>(), nullptr, nullptr};
        for (int k = 2; k <= 4; ++k) mark(c, k, s);
        gen::launch_generic(A, false, s);
        record_status(c, s);
        c->eval_launches += 3;
        mark(c, 5, s);
        ck(c, cudaGetLastError(), "generic gather launch");
        c->evaluated = true;
        return;
    }
    const bool grid_mode = c->bgrid.grid_res > 0 && c->gr_valid;
    // PB2D and BB1D in the one persistent segment kernel (not with the beam grid)
    const bool fused = c->bb1d_kernel >= 3 && !grid_mode;
    // B-P2D and PB2D are both 2-D kernel gathers; pb2d_kernel selects thread or warp per query for both
    const bool bp2d_warp = bp2d && c->pb2d_kernel == 1 && c->bb1d_kernel >= 1;
    if ((nq > 0 && (c->bb1d_kernel >= 1 || grid_mode)) || bp2d_warp) {
        // persistent warp kernels: work counters (BB1D or the fused kernel: [0], PB2D: [1],
        // B-P2D: [2]) and the traversal status word they share
        if (!c->num_sms) ck(c, cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device), "attr");
        ensure(c, c->work, sizeof(unsigned int) * 4);
        ensure(c, c->status, sizeof(int) * 4);
        ck(c, cudaMemsetAsync(c->work.p, 0, sizeof(unsigned int) * 4, s), "memset");
        ck(c, cudaMemsetAsync(c->status.p, 0, sizeof(int) * 4, s), "memset");
    }
    mark(c, 2, s);
    if (np > 0) {
        const HashGridDev G = hash_dev(c);
        const PointQueriesDev Q = point_dev(c);
        Outputs O{c->out_pp3d.as<float>(), img, c->cnt_pp3d.as<uint32_t>(),
                  c->hash_pp3d.as<unsigned long long>(), tested + 2};
        launch_gather_pp3d(K, L, G, Q, cam, cs_pt, O, c->block, mixed, s);
        c->eval_launches += 1;
        if (bp2d) {
            const Outputs Ob{c->out_bp2d.as<float>(), img, c->cnt_bp2d.as<uint32_t>(),
                             c->hash_bp2d.as<unsigned long long>(), tested + 3};
            if (bp2d_warp)
                launch_bp2d_warp(K, beam_bvh(c), beam_soa(c), Q, Ob, c->num_sms * bp2d_warp_blocks_per_sm(),
                                 c->work.as<unsigned int>() + 2, c->status.as<int>(), s);
            else
                launch_gather_bp2d(K, beam_bvh(c), beam_soa(c), Q, Ob, c->block, s);
            c->eval_launches += 1;
        }
    }
    mark(c, 3, s);
    const SegQueriesDev Q = seg_dev(c);
    const int32_t* order = query_order(c, Q, s);
    if (nq > 0 && !fused) {
        const PhotonBVH B = photon_bvh(c);
        Outputs O{c->out_pb2d.as<float>(), img, c->cnt_pb2d.as<uint32_t>(),
                  c->hash_pb2d.as<unsigned long long>(), tested + 0};
        if (c->pb2d_kernel == 1 && c->bb1d_kernel >= 1) {
            const int grid = c->num_sms * pb2d_warp_blocks_per_sm(mixed);
            launch_pb2d_warp(K, L, B, Q, cam, cs_seg, O, grid, mixed, c->work.as<unsigned int>() + 1,
                             c->status.as<int>(), order, s);
        } else {
            launch_gather_pb2d(K, L, B, Q, cam, cs_seg, O, c->block, mixed, s, order);
        }
        c->eval_launches += 1;
    }
    mark(c, 4, s);
    // The per-query BB1D cost varies by an order of magnitude, and a heavy query drawn late from
    // the work queue keeps a few warps busy after the others have finished.  Its PB2D candidate
    // count predicts it (both grow with the beam and photon density along the ray), so the
    // queries above kHeavyFactor x the mean PB2D count go first.
    const int32_t* bb_order = order;
    if (order && nq > 1 && !fused && c->bb1d_kernel >= 1 && (c->P.techniques & UPBP_PB2D) && c->n_ph > 0) {
        constexpr unsigned kHeavyFactor = 4;
        ensure(c, c->bb_keys, sizeof(uint32_t) * nq);
        ensure(c, c->bb_keys_sorted, sizeof(uint32_t) * nq);
        ensure(c, c->bb_iota, sizeof(int32_t) * nq);
        ensure(c, c->bb_order, sizeof(int32_t) * nq);
        ensure(c, c->bb_sum, sizeof(unsigned long long));
        ck(c, cudaMemsetAsync(c->bb_sum.p, 0, sizeof(unsigned long long), s), "memset");
        launch_heavy_keys(c->cnt_pb2d.as<uint32_t>(), nq, c->bb_sum.as<unsigned long long>(), kHeavyFactor,
                          c->q_keys.as<uint32_t>(), c->bb_keys.as<uint32_t>(), c->bb_iota.as<int32_t>(), s);
        size_t b = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, b, c->bb_keys.as<uint32_t>(), c->bb_keys_sorted.as<uint32_t>(),
                                        c->bb_iota.as<int32_t>(), c->bb_order.as<int32_t>(), (int)nq, 0, 31, s);
        ensure(c, c->cub_tmp, b);
        ck(c, cub::DeviceRadixSort::SortPairs(c->cub_tmp.p, b, c->bb_keys.as<uint32_t>(),
                                              c->bb_keys_sorted.as<uint32_t>(), c->bb_iota.as<int32_t>(),
                                              c->bb_order.as<int32_t>(), (int)nq, 0, 31, s),
           "SortPairs");
        bb_order = c->bb_order.as<int32_t>();
        c->eval_launches += 4;
    }
    if (nq > 0) {
        const BeamBVH B = beam_bvh(c);
        const BeamSoA S = beam_soa(c);
        Outputs O{c->out_bb1d.as<float>(), img, c->cnt_bb1d.as<uint32_t>(),
                  c->hash_bb1d.as<unsigned long long>(), tested + 1};
        if (grid_mode) {
            const int grid = c->num_sms * bb1d_grid_blocks_per_sm(mixed);
            launch_bb1d_grid(K, L, grid_dev(c), S, Q, cam, cs_seg, O, grid, mixed, c->work.as<unsigned int>(),
                             bb_order, s);
        } else if (fused) {
            const Outputs Opb{c->out_pb2d.as<float>(), img, c->cnt_pb2d.as<uint32_t>(),
                              c->hash_pb2d.as<unsigned long long>(), tested + 0};
            const int grid = c->num_sms * segments_warp_blocks_per_sm(mixed, c->bb1d_kernel);
            launch_segments_warp(K, L, photon_bvh(c), B, S, Q, cam, cs_seg, Opb, O, grid, mixed,
                                 c->work.as<unsigned int>(), c->status.as<int>(), order, s, c->bb1d_kernel);
            record_status(c, s);
        } else if (c->bb1d_kernel >= 1) {
            const int grid = c->num_sms * bb1d_warp_blocks_per_sm(mixed, c->bb1d_kernel);
            launch_bb1d_warp(K, L, B, S, Q, cam, cs_seg, O, grid, mixed, c->work.as<unsigned int>(),
                             c->status.as<int>(), bb_order, s, c->bb1d_kernel);
            record_status(c, s);
        } else {
            launch_gather_bb1d(K, L, B, S, Q, cam, cs_seg, O, c->block, mixed, s);
        }
        c->eval_launches += 1;
    }
    if (bp2d_warp && !c->status_pending) record_status(c, s);
    mark(c, 5, s);
    ck(c, cudaGetLastError(), "gather launch");
    c->evaluated = true;
}

template <class F>
int guarded(upbp_ctx* c, F&& f)
{
    if (!c) return UPBP_ERR_INVALID_ARG;
    try {
        ck(c, cudaSetDevice(c->device), "cudaSetDevice");
        f();
        return UPBP_OK;
    } catch (const Error& e) {
        return e.code;
    } catch (const std::bad_alloc&) {
        c->err = "host allocation failed";
        return UPBP_ERR_OUT_OF_MEMORY;
    }
}

}  // namespace

extern "C" {

int upbp_ctx_create(upbp_ctx** out, int device)
{
    if (!out) return UPBP_ERR_INVALID_ARG;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return UPBP_ERR_CUDA;
    }
    upbp_ctx* c = new (std::nothrow) upbp_ctx();
    if (!c) return UPBP_ERR_OUT_OF_MEMORY;
    c->device = device;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        return UPBP_ERR_CUDA;
    }
    c->stream = c->own_stream;
    for (auto& e : c->ev) cudaEventCreate(&e);
    *out = c;
    return UPBP_OK;
}

int upbp_ctx_destroy(upbp_ctx* c)
{
    if (!c) return UPBP_ERR_INVALID_ARG;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    drop_graph(c);
    DBuf* all[] = {&c->lv_pos_in, &c->lv_thr_in, &c->lv_dir_in, &c->lv_cont_in, &c->lv_pidx_in, &c->lv_plen_in,
                   &c->lv_med_in, &c->lv_flags_in, &c->lv_mis, &c->path_ends, &c->b_origin, &c->b_dir, &c->b_len,
                   &c->b_thr_in, &c->b_flags_in, &c->b_rsp_in, &c->b_rsr_in, &c->b_rsf_in, &c->b_lpw_in,
                   &c->b_med_in, &c->b_lv_in, &c->cam_mis, &c->sq_origin, &c->sq_dir, &c->sq_seg_begin,
                   &c->sq_seg_count, &c->sq_flags, &c->sq_plen, &c->sq_lpw, &c->sq_thr, &c->sq_pixel,
                   &c->sq_cam_begin, &c->seg_dmin, &c->seg_dmax, &c->seg_pdf, &c->seg_rev, &c->seg_att, &c->seg_med,
                   &c->pq_pos, &c->pq_dir, &c->pq_med, &c->pq_plen, &c->pq_thr, &c->pq_pixel, &c->pq_cam_begin,
                   &c->lv_pos4, &c->lv_dir4, &c->lv_thr4, &c->lv_info4, &c->lv_inmed, &c->ph_lv, &c->ph_lv_sorted,
                   &c->ph_keys, &c->ph_keys_sorted, &c->bbox_partial, &c->bbox_ph, &c->hg_start, &c->hg_end,
                   &c->hg_pos, &c->pb_pos, &c->pb_leaf_codes, &c->pb_nodes, &c->pb_parent_int, &c->pb_parent_leaf,
                   &c->pb_leaf_boxes, &c->pb_node_boxes, &c->pb_flags, &c->bm_thr4, &c->bm_pdf4, &c->bm_link,
                   &c->bm_radius, &c->bm_counts, &c->bm_offsets,
                   &c->pc_a2, &c->pc_b2, &c->pc_c2, &c->pc_boxes2, &c->pc_codes, &c->pc_codes_sorted, &c->pc_perm,
                   &c->pc_perm_sorted, &c->bbox_pc, &c->bm_leaf_codes, &c->bm_nodes, &c->bm_parent_int,
                   &c->bm_parent_leaf, &c->bm_leaf_boxes, &c->bm_node_boxes, &c->bm_flagsbuf, &c->cub_tmp,
                   &c->out_pb2d, &c->out_bb1d, &c->out_pp3d, &c->image, &c->cnt_pb2d, &c->cnt_bb1d, &c->cnt_pp3d,
                   &c->hash_pb2d, &c->hash_bb1d, &c->hash_pp3d, &c->tested, &c->light_sums, &c->cam_sums_seg,
                   &c->cam_sums_pt, &c->work, &c->status, &c->pc_pay, &c->q_keys, &c->q_keys_sorted, &c->q_iota,
                   &c->q_order, &c->grad_img, &c->grad_acc, &c->out_bp2d, &c->cnt_bp2d, &c->hash_bp2d,
                   &c->pb_r2, &c->bm_rchange, &c->bm_r2max, &c->knn_status, &c->kd_org, &c->kd_tree,
                   &c->kd_boxes, &c->kd_pa, &c->kd_pb, &c->bo_pos, &c->bo_pts, &c->bo_codes,
                   &c->bo_codes_sorted, &c->bo_idx, &c->bo_idx_sorted, &c->bo_bbox, &c->bo_leaf_codes, &c->bo_nodes,
                   &c->bo_parent_int, &c->bo_parent_leaf, &c->bo_leaf_boxes, &c->bo_node_boxes, &c->bo_flags,
                   &c->tr_cnt, &c->tr_off, &c->tr_status, &c->bb_keys, &c->bb_keys_sorted, &c->bb_iota,
                   &c->bb_order, &c->bb_sum, &c->gr_hdr, &c->gr_partial, &c->gr_counts, &c->gr_offsets,
                   &c->gr_keys, &c->gr_keys_sorted, &c->gr_keys_unique, &c->gr_num, &c->gr_cellcount,
                   &c->gr_cells, &c->gr_ptr, &c->gr_pdf, &c->gr_draws, &c->gr_draw_off, &c->gr_rnd,
                   &c->gr_rec_a, &c->gr_rec_b, &c->gr_pay, &c->kd_qpts, &c->kd_qcodes, &c->kd_qcodes_sorted,
                   &c->kd_qidx, &c->kd_qidx_sorted, &c->kd_qd2};
    for (DBuf* b : all) free_buf(*b);
    if (c->status_host) cudaFreeHost(c->status_host);
    for (auto& e : c->ev)
        if (e) cudaEventDestroy(e);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
    return UPBP_OK;
}

const char* upbp_last_error(const upbp_ctx* c) { return c ? c->err.c_str() : "null context"; }

int upbp_set_mode(upbp_ctx* c, int mode)
{
    return guarded(c, [&] {
        drop_graph(c);
        if (mode != UPBP_MODE_PLAIN && mode != UPBP_MODE_MIXED && mode != UPBP_MODE_FP64)
            fail(c, UPBP_ERR_INVALID_ARG, "unknown mode %d", mode);
        if (mode != c->mode) c->built = false;
        c->mode = mode;
    });
}

static bool pow2_in(int v, int lo, int hi) { return v >= lo && v <= hi && (v & (v - 1)) == 0; }

int upbp_set_tuning(upbp_ctx* c, const upbp_tuning* tu)
{
    return guarded(c, [&] {
        drop_graph(c);
        if (!tu) fail(c, UPBP_ERR_INVALID_ARG, "tuning is NULL");
        if (!pow2_in(tu->pb2d_leaf, 1, 64) || !pow2_in(tu->bb1d_leaf, 1, 64))
            fail(c, UPBP_ERR_INVALID_ARG, "leaf sizes must be powers of two in [1, 64]");
        if (tu->block_threads < 32 || tu->block_threads > 256 || (tu->block_threads % 32))
            fail(c, UPBP_ERR_INVALID_ARG, "block_threads must be a multiple of 32 in [32, 256]");
        if (!(tu->beam_piece_radii >= 1.f && tu->beam_piece_radii <= 1024.f))
            fail(c, UPBP_ERR_INVALID_ARG, "beam_piece_radii must be in [1, 1024]");
        if (tu->bb1d_kernel < 0 || tu->bb1d_kernel > 4) fail(c, UPBP_ERR_INVALID_ARG, "bb1d_kernel must be in [0, 4]");
        if (tu->pb2d_kernel < 0 || tu->pb2d_kernel > 1) fail(c, UPBP_ERR_INVALID_ARG, "pb2d_kernel must be 0 or 1");
        if (tu->query_order < 0 || tu->query_order > 2) fail(c, UPBP_ERR_INVALID_ARG, "query_order must be in [0, 2]");
        c->pb2d_leaf = tu->pb2d_leaf;
        c->bb1d_leaf = tu->bb1d_leaf;
        c->block = tu->block_threads;
        c->piece_len_r = tu->beam_piece_radii;
        c->bb1d_kernel = tu->bb1d_kernel;
        c->pb2d_kernel = tu->pb2d_kernel;
        c->query_order = tu->query_order;
        c->built = false;
    });
}

int upbp_set_bb1d_grid(upbp_ctx* c, const upbp_bb1d_grid* g)
{
    return guarded(c, [&] {
        drop_graph(c);
        if (!g) fail(c, UPBP_ERR_INVALID_ARG, "grid is NULL");
        if (g->grid_res > 1024) fail(c, UPBP_ERR_INVALID_ARG, "grid_res must be at most 1024");
        if (g->reduction > 3)
            fail(c, UPBP_ERR_INVALID_ARG, "reduction must be 0 (PRESAMPLE), 1 (OFFSET), 2 (RESAMPLE_FIXED) or 3 (SAMPLED)");
        c->bgrid = *g;
        c->built = false;
    });
}

int upbp_get_tuning(const upbp_ctx* c, upbp_tuning* tu)
{
    if (!c || !tu) return UPBP_ERR_INVALID_ARG;
    tu->pb2d_leaf = c->pb2d_leaf;
    tu->bb1d_leaf = c->bb1d_leaf;
    tu->block_threads = c->block;
    tu->beam_piece_radii = c->piece_len_r;
    tu->bb1d_kernel = c->bb1d_kernel;
    tu->pb2d_kernel = c->pb2d_kernel;
    tu->query_order = c->query_order;
    return UPBP_OK;
}

int upbp_set_stream(upbp_ctx* c, void* stream)
{
    return guarded(c, [&] { drop_graph(c); c->stream = stream ? static_cast<cudaStream_t>(stream) : c->own_stream; });
}

int upbp_set_media(upbp_ctx* c, const upbp_medium* media, int32_t n)
{
    return guarded(c, [&] {
        drop_graph(c);
        if (!media || n <= 0 || n > UPBP_MAX_MEDIA) fail(c, UPBP_ERR_INVALID_ARG, "n_media must be in [1, %d]", UPBP_MAX_MEDIA);
        c->media.clear();
        c->media_raw.assign(media, media + n);
        for (int i = 0; i < n; ++i) c->media.push_back(derive_medium(media[i]));
    });
}

int upbp_set_params(upbp_ctx* c, const upbp_params* p)
{
    return guarded(c, [&] {
        drop_graph(c);
        if (!p) fail(c, UPBP_ERR_INVALID_ARG, "params is NULL");
        if (p->max_path_length + 1 > UPBP_MAX_CAM) fail(c, UPBP_ERR_INVALID_ARG, "max_path_length too large");
        if (!(p->radius_pp3d > 0) || !(p->radius_pb2d > 0) || !(p->radius_bb1d > 0))
            fail(c, UPBP_ERR_INVALID_ARG, "radii must be positive");
        if ((p->query_beam_type != UPBP_SHORT_BEAM && p->query_beam_type != UPBP_LONG_BEAM) ||
            (p->photon_beam_type != UPBP_SHORT_BEAM && p->photon_beam_type != UPBP_LONG_BEAM))
            fail(c, UPBP_ERR_INVALID_ARG, "beam types must be SHORT_BEAM or LONG_BEAM");
        if (p->image_width < 0 || p->image_height < 0) fail(c, UPBP_ERR_INVALID_ARG, "negative image size");
        if (p->pb2d_knn < 0 || p->pb2d_knn > kMaxKnn || p->bb1d_knn < 0 || p->bb1d_knn > kMaxKnn)
            fail(c, UPBP_ERR_INVALID_ARG, "KNN counts must be in [0, %d]", kMaxKnn);
        if ((p->techniques & UPBP_NO_MIS) && (p->techniques & UPBP_PP3D))
            fail(c, UPBP_ERR_INVALID_ARG, "UPBP_NO_MIS with UPBP_PP3D: the reference has no PP3D without MIS");
        c->P = *p;
        c->have_params = true;
        c->built = false;
    });
}

int upbp_set_light_vertices(upbp_ctx* c, const upbp_light_vertices* lv)
{
    return guarded(c, [&] {
        drop_graph(c);
        if (!lv || lv->n < 0 || lv->n > (int64_t)INT32_MAX || lv->n_paths < 0)
            fail(c, UPBP_ERR_INVALID_ARG, "bad light vertex count");
        const int64_t n = lv->n;
        upload(c, c->lv_pos_in, lv->position, 3 * n, "position");
        upload(c, c->lv_thr_in, lv->throughput, 3 * n, "throughput");
        upload(c, c->lv_dir_in, lv->dir_fix, 3 * n, "dir_fix");
        c->lv_mis_missing = nullptr;
        upload_mis(c, c->lv_cont_in, lv->cont_prob, n, "cont_prob", 0, &c->lv_mis_missing);
        upload_mis(c, c->lv_pidx_in, lv->path_idx, n, "path_idx", 0, &c->lv_mis_missing);
        upload(c, c->lv_plen_in, lv->path_length, n, "path_length");
        upload(c, c->lv_med_in, lv->medium_id, n, "medium_id");
        upload(c, c->lv_flags_in, lv->flags, n, "flags");
        upload_mis(c, c->lv_mis, lv->mis, n, "mis", 0, &c->lv_mis_missing);
        upload_mis(c, c->path_ends, lv->path_ends, lv->n_paths, "path_ends", 0, &c->lv_mis_missing);
        if (n > 0 && lv->n_paths == 0 && !c->lv_mis_missing) c->lv_mis_missing = "path_ends";
        c->n_lv = n;
        c->n_paths = lv->n_paths;
        c->built = false;
    });
}

int upbp_set_beams(upbp_ctx* c, const upbp_beams* b)
{
    return guarded(c, [&] {
        drop_graph(c);
        if (!b || b->n < 0 || b->n > (int64_t)(1 << 28)) fail(c, UPBP_ERR_INVALID_ARG, "bad beam count");
        const int64_t n = b->n;
        upload(c, c->b_origin, b->origin, 3 * n, "beam origin");
        upload(c, c->b_dir, b->direction, 3 * n, "beam direction");
        upload(c, c->b_len, b->length, n, "beam length");
        upload(c, c->b_thr_in, b->throughput, 3 * n, "beam throughput");
        upload(c, c->b_flags_in, b->flags, n, "beam flags");
        c->beam_mis_missing = nullptr;
        upload_mis(c, c->b_rsp_in, b->ray_sample_pdf, n, "beam ray_sample_pdf", 0, &c->beam_mis_missing);
        upload_mis(c, c->b_rsr_in, b->ray_sample_rev_pdf, n, "beam ray_sample_rev_pdf", 0, &c->beam_mis_missing);
        upload_mis(c, c->b_rsf_in, b->ray_sampling_flags, n, "beam ray_sampling_flags", 0, &c->beam_mis_missing);
        upload_mis(c, c->b_lpw_in, b->last_pdf_w_inv, n, "beam last_pdf_w_inv", 0, &c->beam_mis_missing);
        upload(c, c->b_med_in, b->medium_id, n, "beam medium_id");
        upload_mis(c, c->b_lv_in, b->light_vertex, n, "beam light_vertex", 0xff, &c->beam_mis_missing);
        c->n_beams = n;
        c->built = false;
    });
}

int upbp_build(upbp_ctx* c)
{
    return guarded(c, [&] { do_build(c); });
}

int upbp_set_camera_mis(upbp_ctx* c, const upbp_mis* rec, int64_t n)
{
    return guarded(c, [&] {
        drop_graph(c);
        if (n < 0) fail(c, UPBP_ERR_INVALID_ARG, "negative camera record count");
        upload(c, c->cam_mis, rec, n, "camera mis");
        c->n_cam = n;
    });
}

int upbp_set_segment_queries(upbp_ctx* c, const upbp_segment_queries* q)
{
    return guarded(c, [&] {
        drop_graph(c);
        if (!q || q->n < 0 || q->n_segments < 0) fail(c, UPBP_ERR_INVALID_ARG, "bad segment query counts");
        const int64_t n = q->n, s = q->n_segments;
        upload(c, c->sq_origin, q->origin, 3 * n, "origin");
        upload(c, c->sq_dir, q->direction, 3 * n, "direction");
        upload(c, c->sq_seg_begin, q->seg_begin, n, "seg_begin");
        upload(c, c->sq_seg_count, q->seg_count, n, "seg_count");
        upload(c, c->sq_flags, q->flags, n, "flags");
        upload(c, c->sq_plen, q->path_length, n, "path_length");
        c->sq_mis_missing = nullptr;
        upload_mis(c, c->sq_lpw, q->last_pdf_w_inv, n, "last_pdf_w_inv", 0, &c->sq_mis_missing);
        upload(c, c->sq_thr, q->throughput, 3 * n, "throughput");
        upload(c, c->sq_pixel, q->pixel, n, "pixel");
        upload_mis(c, c->sq_cam_begin, q->cam_mis_begin, n, "cam_mis_begin", 0, &c->sq_mis_missing);
        upload(c, c->seg_dmin, q->seg_dist_min, s, "seg_dist_min");
        upload(c, c->seg_dmax, q->seg_dist_max, s, "seg_dist_max");
        upload(c, c->seg_pdf, q->seg_pdf, s, "seg_pdf");
        upload(c, c->seg_rev, q->seg_rev_pdf, s, "seg_rev_pdf");
        upload(c, c->seg_att, q->seg_attenuation, 3 * s, "seg_attenuation");
        upload(c, c->seg_med, q->seg_medium, s, "seg_medium");
        c->n_sq = n;
        c->n_seg = s;
    });
}

int upbp_set_point_queries(upbp_ctx* c, const upbp_point_queries* q)
{
    return guarded(c, [&] {
        drop_graph(c);
        if (!q || q->n < 0) fail(c, UPBP_ERR_INVALID_ARG, "bad point query count");
        const int64_t n = q->n;
        upload(c, c->pq_pos, q->position, 3 * n, "position");
        upload(c, c->pq_dir, q->dir_fix, 3 * n, "dir_fix");
        upload(c, c->pq_med, q->medium_id, n, "medium_id");
        upload(c, c->pq_plen, q->path_length, n, "path_length");
        upload(c, c->pq_thr, q->throughput, 3 * n, "throughput");
        upload(c, c->pq_pixel, q->pixel, n, "pixel");
        upload(c, c->pq_cam_begin, q->cam_mis_begin, n, "cam_mis_begin");
        c->n_pq = n;
    });
}

namespace {

// Per-path counts (count pass) -> exclusive offsets -> totals on the host.  `k` arrays of n ints
// live in tr_cnt / tr_off, each followed by a zero so that offset[n] is the total.
void trace_offsets(upbp_ctx* c, int k, int64_t n, int64_t* totals)
{
    cudaStream_t s = c->stream;
    int* cnt = c->tr_cnt.as<int>();
    int* off = c->tr_off.as<int>();
    const size_t tb = trace::scan_temp_bytes((int)(n + 1));
    ensure(c, c->cub_tmp, tb);
    for (int j = 0; j < k; ++j) {
        ck(c, cudaMemsetAsync(cnt + j * (n + 1) + n, 0, sizeof(int), s), "memset");
        trace::exclusive_scan(cnt + j * (n + 1), off + j * (n + 1), (int)(n + 1), c->cub_tmp.p, c->cub_tmp.cap, s);
        ck(c, cudaGetLastError(), "scan");
    }
    std::vector<int> t(k);
    for (int j = 0; j < k; ++j)
        ck(c, cudaMemcpyAsync(&t[j], off + j * (n + 1) + n, sizeof(int), cudaMemcpyDeviceToHost, s), "copy totals");
    ck(c, cudaStreamSynchronize(s), "sync");
    for (int j = 0; j < k; ++j) {
        if (t[j] < 0) fail(c, UPBP_ERR_CAPACITY, "traced record count overflows 32 bits");
        totals[j] = t[j];
    }
}

// After a write pass: every path wrote exactly the records its count pass sized.
void check_trace_status(upbp_ctx* c, const char* pass)
{
    int st = 0;
    ck(c, cudaMemcpyAsync(&st, c->tr_status.as<int>(), sizeof(int), cudaMemcpyDeviceToHost, c->stream), pass);
    ck(c, cudaStreamSynchronize(c->stream), pass);
    if (st) fail(c, UPBP_ERR_CUDA, "%s: a path's write pass differed from its count pass", pass);
}

trace::TraceScene trace_scene(upbp_ctx* c, const upbp_scene* sc, uint32_t iteration)
{
    if (!sc) fail(c, UPBP_ERR_INVALID_ARG, "scene is NULL");
    if (!c->have_params) fail(c, UPBP_ERR_INVALID_ARG, "upbp_set_params must precede the device-side passes");
    trace::TraceScene S;
    if (const char* e = trace::make_scene(*sc, c->P, iteration, &S)) fail(c, UPBP_ERR_INVALID_ARG, "scene: %s", e);
    return S;
}

}  // namespace

int upbp_trace_light_paths(upbp_ctx* c, const upbp_scene* sc, uint32_t iteration)
{
    return guarded(c, [&] {
        drop_graph(c);
        const trace::TraceScene S = trace_scene(c, sc, iteration);
        const int64_t n = S.light_paths;
        // every path holds at most max_path_length vertices and (max_path_length - 1) * 2 n_boxes beams
        if (n * S.max_path_length * (2 * S.n_boxes) >= (int64_t)INT32_MAX)
            fail(c, UPBP_ERR_CAPACITY, "too many light paths for 32-bit record offsets");
        cudaStream_t s = c->stream;
        ensure(c, c->tr_cnt, sizeof(int) * 2 * (n + 1));
        ensure(c, c->tr_off, sizeof(int) * 2 * (n + 1));
        c->lv_mis_missing = c->beam_mis_missing = nullptr;  // the pass writes every record
        trace::LightOut O{};
        O.v_count = c->tr_cnt.as<int>();
        O.b_count = O.v_count + (n + 1);
        trace::launch_light(S, false, O, s);
        ck(c, cudaGetLastError(), "light pass (count)");
        int64_t tot[2];
        trace_offsets(c, 2, n, tot);
        const int64_t nv = tot[0], nb = tot[1];
        ensure(c, c->lv_pos_in, sizeof(float) * 3 * nv);
        ensure(c, c->lv_thr_in, sizeof(float) * 3 * nv);
        ensure(c, c->lv_dir_in, sizeof(float) * 3 * nv);
        ensure(c, c->lv_cont_in, sizeof(float) * nv);
        ensure(c, c->lv_pidx_in, sizeof(int32_t) * nv);
        ensure(c, c->lv_plen_in, sizeof(int32_t) * nv);
        ensure(c, c->lv_med_in, sizeof(int32_t) * nv);
        ensure(c, c->lv_flags_in, sizeof(uint32_t) * nv);
        ensure(c, c->lv_mis, sizeof(upbp_mis) * nv);
        ensure(c, c->path_ends, sizeof(int32_t) * n);
        ensure(c, c->b_origin, sizeof(float) * 3 * nb);
        ensure(c, c->b_dir, sizeof(float) * 3 * nb);
        ensure(c, c->b_len, sizeof(float) * nb);
        ensure(c, c->b_thr_in, sizeof(float) * 3 * nb);
        ensure(c, c->b_flags_in, sizeof(uint32_t) * nb);
        ensure(c, c->b_rsp_in, sizeof(float) * nb);
        ensure(c, c->b_rsr_in, sizeof(float) * nb);
        ensure(c, c->b_rsf_in, sizeof(uint32_t) * nb);
        ensure(c, c->b_lpw_in, sizeof(float) * nb);
        ensure(c, c->b_med_in, sizeof(int32_t) * nb);
        ensure(c, c->b_lv_in, sizeof(int32_t) * nb);
        O.v_off = c->tr_off.as<int>();
        O.b_off = O.v_off + (n + 1);
        O.pos = c->lv_pos_in.as<float>();
        O.thr = c->lv_thr_in.as<float>();
        O.dir = c->lv_dir_in.as<float>();
        O.cont = c->lv_cont_in.as<float>();
        O.pidx = c->lv_pidx_in.as<int>();
        O.plen = c->lv_plen_in.as<int>();
        O.med = c->lv_med_in.as<int>();
        O.flags = c->lv_flags_in.as<uint32_t>();
        O.mis = c->lv_mis.as<upbp_mis>();
        O.path_ends = c->path_ends.as<int>();
        O.b_origin = c->b_origin.as<float>();
        O.b_dir = c->b_dir.as<float>();
        O.b_len = c->b_len.as<float>();
        O.b_thr = c->b_thr_in.as<float>();
        O.b_flags = c->b_flags_in.as<uint32_t>();
        O.b_rsp = c->b_rsp_in.as<float>();
        O.b_rsr = c->b_rsr_in.as<float>();
        O.b_rsf = c->b_rsf_in.as<uint32_t>();
        O.b_lpw = c->b_lpw_in.as<float>();
        O.b_med = c->b_med_in.as<int>();
        O.b_lv = c->b_lv_in.as<int>();
        ensure(c, c->tr_status, sizeof(int));
        ck(c, cudaMemsetAsync(c->tr_status.p, 0, sizeof(int), s), "memset");
        O.status = c->tr_status.as<int>();
        trace::launch_light(S, true, O, s);
        ck(c, cudaGetLastError(), "light pass (write)");
        check_trace_status(c, "light pass");
        c->n_lv = nv;
        c->n_paths = (int32_t)n;
        c->n_beams = nb;
        c->built = false;
    });
}

int upbp_trace_camera_paths(upbp_ctx* c, const upbp_scene* sc, uint32_t iteration)
{
    return guarded(c, [&] {
        drop_graph(c);
        const trace::TraceScene S = trace_scene(c, sc, iteration);
        const int64_t n = (int64_t)S.width * S.height;
        // per pixel at most max_path_length segment queries of 2 n_boxes segments, and camera
        // records sum over L of (2 L + 1)
        const int64_t per_pixel = (int64_t)S.max_path_length * (2 * S.n_boxes + 2 * S.max_path_length + 2);
        if (n * per_pixel >= (int64_t)INT32_MAX)
            fail(c, UPBP_ERR_CAPACITY, "too many pixels for 32-bit record offsets");
        cudaStream_t s = c->stream;
        ensure(c, c->tr_cnt, sizeof(int) * 4 * (n + 1));
        ensure(c, c->tr_off, sizeof(int) * 4 * (n + 1));
        c->sq_mis_missing = nullptr;  // the pass writes every record
        trace::CameraOut O{};
        O.q_count = c->tr_cnt.as<int>();
        O.s_count = O.q_count + (n + 1);
        O.p_count = O.s_count + (n + 1);
        O.c_count = O.p_count + (n + 1);
        trace::launch_camera(S, false, O, s);
        ck(c, cudaGetLastError(), "camera pass (count)");
        int64_t tot[4];
        trace_offsets(c, 4, n, tot);
        const int64_t nq = tot[0], ns = tot[1], np = tot[2], nc = tot[3];
        ensure(c, c->sq_origin, sizeof(float) * 3 * nq);
        ensure(c, c->sq_dir, sizeof(float) * 3 * nq);
        ensure(c, c->sq_seg_begin, sizeof(int32_t) * nq);
        ensure(c, c->sq_seg_count, sizeof(int32_t) * nq);
        ensure(c, c->sq_flags, sizeof(uint32_t) * nq);
        ensure(c, c->sq_plen, sizeof(int32_t) * nq);
        ensure(c, c->sq_lpw, sizeof(float) * nq);
        ensure(c, c->sq_thr, sizeof(float) * 3 * nq);
        ensure(c, c->sq_pixel, sizeof(int32_t) * nq);
        ensure(c, c->sq_cam_begin, sizeof(int64_t) * nq);
        ensure(c, c->seg_dmin, sizeof(float) * ns);
        ensure(c, c->seg_dmax, sizeof(float) * ns);
        ensure(c, c->seg_pdf, sizeof(float) * ns);
        ensure(c, c->seg_rev, sizeof(float) * ns);
        ensure(c, c->seg_att, sizeof(float) * 3 * ns);
        ensure(c, c->seg_med, sizeof(int32_t) * ns);
        ensure(c, c->pq_pos, sizeof(float) * 3 * np);
        ensure(c, c->pq_dir, sizeof(float) * 3 * np);
        ensure(c, c->pq_med, sizeof(int32_t) * np);
        ensure(c, c->pq_plen, sizeof(int32_t) * np);
        ensure(c, c->pq_thr, sizeof(float) * 3 * np);
        ensure(c, c->pq_pixel, sizeof(int32_t) * np);
        ensure(c, c->pq_cam_begin, sizeof(int64_t) * np);
        ensure(c, c->cam_mis, sizeof(upbp_mis) * nc);
        O.q_off = c->tr_off.as<int>();
        O.s_off = O.q_off + (n + 1);
        O.p_off = O.s_off + (n + 1);
        O.c_off = O.p_off + (n + 1);
        O.sq_origin = c->sq_origin.as<float>();
        O.sq_dir = c->sq_dir.as<float>();
        O.sq_seg_begin = c->sq_seg_begin.as<int>();
        O.sq_seg_count = c->sq_seg_count.as<int>();
        O.sq_flags = c->sq_flags.as<uint32_t>();
        O.sq_plen = c->sq_plen.as<int>();
        O.sq_lpw = c->sq_lpw.as<float>();
        O.sq_thr = c->sq_thr.as<float>();
        O.sq_pixel = c->sq_pixel.as<int>();
        O.sq_cam_begin = c->sq_cam_begin.as<int64_t>();
        O.seg_dmin = c->seg_dmin.as<float>();
        O.seg_dmax = c->seg_dmax.as<float>();
        O.seg_pdf = c->seg_pdf.as<float>();
        O.seg_rev = c->seg_rev.as<float>();
        O.seg_att = c->seg_att.as<float>();
        O.seg_med = c->seg_med.as<int>();
        O.pq_pos = c->pq_pos.as<float>();
        O.pq_dir = c->pq_dir.as<float>();
        O.pq_med = c->pq_med.as<int>();
        O.pq_plen = c->pq_plen.as<int>();
        O.pq_thr = c->pq_thr.as<float>();
        O.pq_pixel = c->pq_pixel.as<int>();
        O.pq_cam_begin = c->pq_cam_begin.as<int64_t>();
        O.cam = c->cam_mis.as<upbp_mis>();
        ensure(c, c->tr_status, sizeof(int));
        ck(c, cudaMemsetAsync(c->tr_status.p, 0, sizeof(int), s), "memset");
        O.status = c->tr_status.as<int>();
        trace::launch_camera(S, true, O, s);
        ck(c, cudaGetLastError(), "camera pass (write)");
        check_trace_status(c, "camera pass");
        c->n_sq = nq;
        c->n_seg = ns;
        c->n_pq = np;
        c->n_cam = nc;
    });
}

int upbp_read_input(upbp_ctx* c, const char* name, void* dst, int64_t capacity, int64_t* bytes)
{
    return guarded(c, [&] {
        if (!name) fail(c, UPBP_ERR_INVALID_ARG, "name is NULL");
        struct Entry {
            const char* name;
            DBuf* buf;
            int64_t bytes;
        };
        const int64_t nv = c->n_lv, nb = c->n_beams, nq = c->n_sq, ns = c->n_seg, np = c->n_pq;
        const Entry table[] = {
            {"lv_position", &c->lv_pos_in, 12 * nv}, {"lv_throughput", &c->lv_thr_in, 12 * nv},
            {"lv_dir_fix", &c->lv_dir_in, 12 * nv}, {"lv_cont_prob", &c->lv_cont_in, 4 * nv},
            {"lv_path_idx", &c->lv_pidx_in, 4 * nv}, {"lv_path_length", &c->lv_plen_in, 4 * nv},
            {"lv_medium_id", &c->lv_med_in, 4 * nv}, {"lv_flags", &c->lv_flags_in, 4 * nv},
            {"lv_mis", &c->lv_mis, (int64_t)sizeof(upbp_mis) * nv}, {"lv_path_ends", &c->path_ends, 4 * (int64_t)c->n_paths},
            {"beam_origin", &c->b_origin, 12 * nb}, {"beam_direction", &c->b_dir, 12 * nb},
            {"beam_length", &c->b_len, 4 * nb}, {"beam_throughput", &c->b_thr_in, 12 * nb},
            {"beam_flags", &c->b_flags_in, 4 * nb}, {"beam_ray_sample_pdf", &c->b_rsp_in, 4 * nb},
            {"beam_ray_sample_rev_pdf", &c->b_rsr_in, 4 * nb}, {"beam_ray_sampling_flags", &c->b_rsf_in, 4 * nb},
            {"beam_last_pdf_w_inv", &c->b_lpw_in, 4 * nb}, {"beam_medium_id", &c->b_med_in, 4 * nb},
            {"beam_light_vertex", &c->b_lv_in, 4 * nb}, {"cam_mis", &c->cam_mis, (int64_t)sizeof(upbp_mis) * c->n_cam},
            {"sq_origin", &c->sq_origin, 12 * nq}, {"sq_direction", &c->sq_dir, 12 * nq},
            {"sq_seg_begin", &c->sq_seg_begin, 4 * nq}, {"sq_seg_count", &c->sq_seg_count, 4 * nq},
            {"sq_flags", &c->sq_flags, 4 * nq}, {"sq_path_length", &c->sq_plen, 4 * nq},
            {"sq_last_pdf_w_inv", &c->sq_lpw, 4 * nq}, {"sq_throughput", &c->sq_thr, 12 * nq},
            {"sq_pixel", &c->sq_pixel, 4 * nq}, {"sq_cam_mis_begin", &c->sq_cam_begin, 8 * nq},
            {"seg_dist_min", &c->seg_dmin, 4 * ns}, {"seg_dist_max", &c->seg_dmax, 4 * ns},
            {"seg_pdf", &c->seg_pdf, 4 * ns}, {"seg_rev_pdf", &c->seg_rev, 4 * ns},
            {"seg_attenuation", &c->seg_att, 12 * ns}, {"seg_medium", &c->seg_med, 4 * ns},
            {"pq_position", &c->pq_pos, 12 * np}, {"pq_dir_fix", &c->pq_dir, 12 * np},
            {"pq_medium_id", &c->pq_med, 4 * np}, {"pq_path_length", &c->pq_plen, 4 * np},
            {"pq_throughput", &c->pq_thr, 12 * np}, {"pq_pixel", &c->pq_pixel, 4 * np},
            {"pq_cam_mis_begin", &c->pq_cam_begin, 8 * np},
            // the beam grid of the last build (upbp_set_bb1d_grid): the reference's mCells,
            // mPointers as beam ids, mPdfs
            {"bb1d_grid_cells", &c->gr_cells, c->gr_valid ? 4 * (int64_t)c->gr_host.n_cells : 0},
            {"bb1d_grid_beams", &c->gr_ptr, c->gr_valid ? 4 * c->gr_pairs : 0},
            {"bb1d_grid_pdfs", &c->gr_pdf,
             c->gr_valid && c->bgrid.max_beams_in_cell > 0 ? 4 * ((int64_t)c->gr_host.n_cells - 1) : 0},
        };
        for (const Entry& e : table) {
            if (std::strcmp(e.name, name) != 0) continue;
            if (bytes) *bytes = e.bytes;
            if (!dst || e.bytes == 0) return;
            if (capacity < e.bytes) fail(c, UPBP_ERR_INVALID_ARG, "%s needs %lld bytes", name, (long long)e.bytes);
            ck(c, cudaMemcpyAsync(dst, e.buf->p, (size_t)e.bytes, cudaMemcpyDefault, c->stream), name);
            ck(c, cudaStreamSynchronize(c->stream), "sync");
            return;
        }
        fail(c, UPBP_ERR_INVALID_ARG, "unknown input array %s", name);
    });
}

int upbp_evaluate(upbp_ctx* c)
{
    return guarded(c, [&] { do_evaluate(c); });
}

int upbp_capture_graph(upbp_ctx* c)
{
    return guarded(c, [&] {
        if (!c->built || !c->evaluated)
            fail(c, UPBP_ERR_NOT_BUILT, "capture needs upbp_build and upbp_evaluate of the current inputs first");
        drop_graph(c);
        cudaStream_t s = c->stream;
        if (s == nullptr) fail(c, UPBP_ERR_INVALID_ARG, "graph capture needs a non-default stream");
        const size_t npix = (size_t)std::max(0, c->P.image_width) * (size_t)std::max(0, c->P.image_height);
        ck(c, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        c->replay = true;
        cudaGraph_t g = nullptr;
        try {
            if (npix) ck(c, cudaMemsetAsync(c->image.p, 0, sizeof(float) * 3 * npix, s), "memset image");
            do_build(c);
            do_evaluate(c);
        } catch (...) {
            c->replay = false;
            cudaStreamEndCapture(s, &g);
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            throw;
        }
        c->replay = false;
        ck(c, cudaStreamEndCapture(s, &g), "cudaStreamEndCapture");
        cudaGraphExec_t e = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&e, g, 0);
        cudaGraphDestroy(g);
        ck(c, ie, "cudaGraphInstantiate");
        c->graph_exec = e;
        c->graph_status = c->status_pending;
    });
}

int upbp_launch_graph(upbp_ctx* c)
{
    return guarded(c, [&] {
        if (!c->graph_exec) fail(c, UPBP_ERR_NOT_BUILT, "no graph: inputs changed or upbp_capture_graph not called");
        ck(c, cudaGraphLaunch(c->graph_exec, c->stream), "cudaGraphLaunch");
        c->status_pending = c->graph_status;
    });
}

int upbp_read_segment_results(upbp_ctx* c, float* pb2d, float* bb1d)
{
    return guarded(c, [&] {
        const size_t bytes = sizeof(float) * 3 * (size_t)c->n_sq;
        if (pb2d && bytes) ck(c, cudaMemcpyAsync(pb2d, c->out_pb2d.p, bytes, cudaMemcpyDefault, c->stream), "read");
        if (bb1d && bytes) ck(c, cudaMemcpyAsync(bb1d, c->out_bb1d.p, bytes, cudaMemcpyDefault, c->stream), "read");
        ck(c, cudaStreamSynchronize(c->stream), "sync");
        check_status(c);
    });
}

int upbp_read_point_results(upbp_ctx* c, float* pp3d)
{
    return guarded(c, [&] {
        const size_t bytes = sizeof(float) * 3 * (size_t)c->n_pq;
        if (pp3d && bytes) ck(c, cudaMemcpyAsync(pp3d, c->out_pp3d.p, bytes, cudaMemcpyDefault, c->stream), "read");
        ck(c, cudaStreamSynchronize(c->stream), "sync");
        check_status(c);
    });
}

int upbp_read_query_stats(upbp_ctx* c, const upbp_query_stats* st)
{
    return guarded(c, [&] {
        if (!st) fail(c, UPBP_ERR_INVALID_ARG, "stats is NULL");
        const size_t nq = (size_t)c->n_sq, np = (size_t)c->n_pq;
        auto rd = [&](void* dst, const DBuf& src, size_t bytes) {
            if (dst && bytes) ck(c, cudaMemcpyAsync(dst, src.p, bytes, cudaMemcpyDefault, c->stream), "read stats");
        };
        rd(st->count_pb2d, c->cnt_pb2d, 4 * nq);
        rd(st->hash_pb2d, c->hash_pb2d, 8 * nq);
        rd(st->count_bb1d, c->cnt_bb1d, 4 * nq);
        rd(st->hash_bb1d, c->hash_bb1d, 8 * nq);
        rd(st->count_pp3d, c->cnt_pp3d, 4 * np);
        rd(st->hash_pp3d, c->hash_pp3d, 8 * np);
        ck(c, cudaStreamSynchronize(c->stream), "sync");
        check_status(c);
    });
}

int upbp_adjoint(upbp_ctx* c, const float* grad_image, int32_t medium, double* grad)
{
    return guarded(c, [&] {
        if (!grad_image || !grad) fail(c, UPBP_ERR_INVALID_ARG, "grad_image and grad must not be NULL");
        if (medium < 0 || medium >= (int)c->media_raw.size()) fail(c, UPBP_ERR_INVALID_ARG, "medium out of range");
        if (!c->built) fail(c, UPBP_ERR_NOT_BUILT, "upbp_build was not called");
        if (c->mode == UPBP_MODE_PLAIN)
            fail(c, UPBP_ERR_INVALID_ARG, "the adjoint needs UPBP_MODE_MIXED or UPBP_MODE_FP64 structures");
        if (c->bgrid.grid_res > 0)
            fail(c, UPBP_ERR_INVALID_ARG, "the adjoint evaluates BB1D over the beam pieces, not the beam grid");
        cudaStream_t s = c->stream;
        c->eval_launches = 0;
        c->status_pending = false;
        const size_t npix = (size_t)std::max(0, c->P.image_width) * (size_t)std::max(0, c->P.image_height);
        ensure(c, c->grad_img, sizeof(float) * 3 * std::max<size_t>(npix, 1));
        if (npix)
            ck(c, cudaMemcpyAsync(c->grad_img.p, grad_image, sizeof(float) * 3 * npix, cudaMemcpyDefault, s),
               "grad_image");
        ensure(c, c->grad_acc, sizeof(double) * 8);
        ck(c, cudaMemsetAsync(c->grad_acc.p, 0, sizeof(double) * 8, s), "memset");
        const CamSum* cs_seg = nullptr;
        const CamSum* cs_pt = nullptr;
        if (!(c->P.techniques & UPBP_NO_MIS)) prepare_cam_sums(c, s, &cs_seg, &cs_pt);
        gen::GenLaunch A = generic_launch(c, cs_seg, cs_pt, medium);
        const gen::GenOut O{nullptr, nullptr, nullptr, nullptr, c->grad_img.as<float>(), c->grad_acc.as<double>()};
        A.out_pp3d = A.out_pb2d = A.out_bb1d = A.out_bp2d = O;
        gen::launch_generic(A, true, s);
        c->eval_launches += 3;
        record_status(c, s);
        ck(c, cudaGetLastError(), "adjoint launch");
        double h[8];
        ck(c, cudaMemcpyAsync(h, c->grad_acc.p, sizeof(double) * 8, cudaMemcpyDeviceToHost, s), "read grad");
        ck(c, cudaStreamSynchronize(s), "sync");
        check_status(c);
        for (int i = 0; i < 7; ++i) grad[i] = h[i];
    });
}

int upbp_read_bp2d_results(upbp_ctx* c, float* rgb, uint32_t* count, uint64_t* hash)
{
    return guarded(c, [&] {
        const size_t np = (size_t)c->n_pq;
        if (np == 0) return;
        if (!(c->P.techniques & UPBP_BP2D) || !c->out_bp2d.p || c->out_bp2d.cap < sizeof(float) * 3 * np)
            fail(c, UPBP_ERR_NOT_BUILT, "no B-P2D results: UPBP_BP2D is not in the techniques of the last evaluate");
        auto rd = [&](void* dst, const DBuf& src, size_t bytes) {
            if (dst) ck(c, cudaMemcpyAsync(dst, src.p, bytes, cudaMemcpyDefault, c->stream), "read bp2d");
        };
        rd(rgb, c->out_bp2d, sizeof(float) * 3 * np);
        rd(count, c->cnt_bp2d, sizeof(uint32_t) * np);
        rd(hash, c->hash_bp2d, sizeof(uint64_t) * np);
        ck(c, cudaStreamSynchronize(c->stream), "sync");
        check_status(c);
    });
}

int upbp_device_bytes(const upbp_ctx* c, uint64_t* bytes)
{
    if (!c || !bytes) return UPBP_ERR_INVALID_ARG;
    *bytes = (uint64_t)c->bytes;
    return UPBP_OK;
}

int upbp_read_tested_counts(upbp_ctx* c, uint64_t* tested)
{
    return guarded(c, [&] {
        if (!tested) fail(c, UPBP_ERR_INVALID_ARG, "tested is NULL");
        unsigned long long h[4] = {0, 0, 0, 0};
        if (c->tested.p) {
            ck(c, cudaMemcpyAsync(h, c->tested.p, sizeof(h), cudaMemcpyDeviceToHost, c->stream), "read tested");
            ck(c, cudaStreamSynchronize(c->stream), "sync");
        check_status(c);
        }
        for (int i = 0; i < 3; ++i) tested[i] = (uint64_t)h[i];
    });
}

int upbp_clear_image(upbp_ctx* c)
{
    return guarded(c, [&] {
        const size_t npix = (size_t)std::max(0, c->P.image_width) * (size_t)std::max(0, c->P.image_height);
        ensure(c, c->image, sizeof(float) * 3 * std::max<size_t>(npix, 1));
        ck(c, cudaMemsetAsync(c->image.p, 0, sizeof(float) * 3 * npix, c->stream), "memset image");
        // and the per-query results of the last evaluate (the next evaluate overwrites them)
        for (DBuf* b : {&c->out_pb2d, &c->out_bb1d, &c->out_pp3d, &c->out_bp2d, &c->cnt_pb2d, &c->cnt_bb1d,
                        &c->cnt_pp3d, &c->cnt_bp2d, &c->hash_pb2d, &c->hash_bb1d, &c->hash_pp3d, &c->hash_bp2d})
            if (b->p) ck(c, cudaMemsetAsync(b->p, 0, b->cap, c->stream), "memset results");
    });
}

int upbp_read_image(upbp_ctx* c, float* rgb)
{
    return guarded(c, [&] {
        if (!rgb) fail(c, UPBP_ERR_INVALID_ARG, "rgb is NULL");
        const size_t npix = (size_t)std::max(0, c->P.image_width) * (size_t)std::max(0, c->P.image_height);
        if (npix) ck(c, cudaMemcpyAsync(rgb, c->image.p, sizeof(float) * 3 * npix, cudaMemcpyDefault, c->stream), "read image");
        ck(c, cudaStreamSynchronize(c->stream), "sync");
        check_status(c);
    });
}

int upbp_last_launch_count(const upbp_ctx* c, int* b, int* e)
{
    if (!c) return UPBP_ERR_INVALID_ARG;
    if (b) *b = c->build_launches;
    if (e) *e = c->eval_launches;
    return UPBP_OK;
}

int upbp_last_timings(const upbp_ctx* cc, float* build_ms, float* pp3d_ms, float* pb2d_ms, float* bb1d_ms)
{
    upbp_ctx* c = const_cast<upbp_ctx*>(cc);
    return guarded(c, [&] {
        ck(c, cudaStreamSynchronize(c->stream), "sync");
        check_status(c);
        float v = 0.f;
        if (build_ms) { cudaEventElapsedTime(&v, c->ev[0], c->ev[1]); *build_ms = v; }
        if (pp3d_ms) { cudaEventElapsedTime(&v, c->ev[2], c->ev[3]); *pp3d_ms = v; }
        if (pb2d_ms) { cudaEventElapsedTime(&v, c->ev[3], c->ev[4]); *pb2d_ms = v; }
        if (bb1d_ms) { cudaEventElapsedTime(&v, c->ev[4], c->ev[5]); *bb1d_ms = v; }
        cudaGetLastError();
    });
}

int upbp_destroy_structures(upbp_ctx* c)
{
    return guarded(c, [&] {
        drop_graph(c);
        c->built = false;
        c->n_ph = 0;
        c->pb_n_leaves = 0;
        c->n_pieces = 0;
        c->bm_n_leaves = 0;
    });
}

}  // extern "C"
