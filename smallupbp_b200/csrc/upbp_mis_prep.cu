// Precompute kernels of the FP64 MIS partial sums (see upbp_mis_prep.cuh).
#include "upbp_kernels.cuh"
#include "upbp_mis_prep.cuh"

namespace upbp {

namespace {

// One thread per light path: walk its vertices from the light source outwards.
__global__ void k_light_sums(const upbp_mis* __restrict__ mis, const int32_t* __restrict__ path_ends, int n_paths,
                             uint32_t tech, uint32_t qbt, uint32_t pbt, LightSum* __restrict__ out)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n_paths) return;
    const int start = p == 0 ? 0 : path_ends[p - 1];
    const int end = path_ends[p];
    double G_prev = 0.0;       // G(u-1)
    double H_prev = 0.0;       // M(u-1) + T(u-1) with u-1's own reverse ray pdf
    float revwb_prev = 0.f;    // revWB_{u-1}
    bool spec_prev = false;    // spec(u-1)
    const bool bpt = (tech & UPBP_BPT) != 0;
    for (int u = start; u < end; ++u) {
        const upbp_mis m = load_mis(mis + u);
        const bool spec = (m.flags & UPBP_MIS_IS_SPECULAR) != 0;
        double fix, rc;
        light_merge_terms(m, tech, qbt, pbt, fix, rc);
        // next(u) = u-1 for u > start, u itself at the light source (PathWeight.hxx:177)
        const bool next_spec = u > start ? spec_prev : spec;
        const double B = (bpt && !spec && !next_spec) ? 1.0 : 0.0;
        const double T = (double)m.pdf_a_inv * (B + G_prev);
        const double H = fix + (double)m.ray_sample_rev_pdf_inv * rc + T;
        const double G = m.rev_pdf_a == 0.f ? 0.0 : (double)m.rev_pdf_a * H;
        LightSum s;
        // u as the merged photon (index 0) of a PB2D / PP3D walk
        const bool b0 = bpt && (u > start ? !spec_prev : !spec);
        s.a = b0 ? (double)m.pdf_a_inv : 0.0;
        s.c = (u > start && !(tech & UPBP_PREVIOUS)) ? (double)m.pdf_a_inv * (double)revwb_prev * H_prev : 0.0;
        // u as the beam-origin vertex (index 1) of a BB1D walk
        s.d = fix + T;
        s.e = rc;
        s.bptb = (bpt && !spec) ? 1.f : 0.f;
        s.pad = 0;
        out[u] = s;
        G_prev = G;
        H_prev = H;
        revwb_prev = m.rev_pdf_a_without_bsdf;
        spec_prev = spec;
    }
}

// One thread per query: the camera walk over entries L-2 .. 1 (walk indices >= 2).
__global__ void k_cam_sums(const upbp_mis* __restrict__ cam, const int64_t* __restrict__ begin,
                           const int32_t* __restrict__ path_length, int64_t n, uint32_t tech, uint32_t qbt,
                           uint32_t pbt, CamSum* __restrict__ out)
{
    const int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (q >= n) return;
    const upbp_mis* snap = cam + begin[q];
    const int L = path_length[q];
    double prod = 1.0, s_other = 0.0, s_bb1d = 0.0;
    uint32_t flags = 0;
    if (L >= 3) {
        if (snap[L - 2].flags & UPBP_MIS_IS_SPECULAR) flags |= 2u;
    } else if (L == 2) {
        if (snap[1].flags & UPBP_MIS_IS_SPECULAR) flags |= 2u;
    }
    for (int k = L - 2; k >= 1; --k) {
        const upbp_mis m = load_mis(snap + k);
        const bool spec = (m.flags & UPBP_MIS_IS_SPECULAR) != 0;
        if ((tech & UPBP_BB1D_PREVIOUS) && !spec) {
            s_bb1d = 0.0;
            flags |= 1u;
        }
        prod *= (double)m.rev_pdf_a;
        double o, b;
        cam_merge_terms<double>(m, !spec, m.sin_theta, m.ray_sample_rev_pdf_inv, m.ray_sample_rev_pdfs_ratio, tech, qbt, pbt, o,
                        b);
        s_other += prod * o;
        s_bb1d += prod * b;
        prod *= (double)m.pdf_a_inv;
        const bool next_spec = k > 1 ? (snap[k - 1].flags & UPBP_MIS_IS_SPECULAR) != 0 : spec;
        if ((tech & UPBP_BPT) && !spec && !next_spec) s_other += prod;
    }
    CamSum c;
    c.s_other = s_other;
    c.s_bb1d = s_bb1d;
    c.f_other = (float)s_other;
    c.f_bb1d = (float)s_bb1d;
    c.flags = flags;
    c.pad = 0;
    out[q] = c;
}

}  // namespace

void launch_light_sums(const upbp_mis* mis, const int32_t* path_ends, int n_paths, uint32_t tech, uint32_t qbt,
                       uint32_t pbt, LightSum* out, cudaStream_t s)
{
    if (n_paths > 0) k_light_sums<<<(n_paths + 127) / 128, 128, 0, s>>>(mis, path_ends, n_paths, tech, qbt, pbt, out);
}

void launch_cam_sums(const upbp_mis* cam, const int64_t* begin, const int32_t* path_length, int64_t n, uint32_t tech,
                     uint32_t qbt, uint32_t pbt, CamSum* out, cudaStream_t s)
{
    if (n > 0) k_cam_sums<<<(int)((n + 127) / 128), 128, 0, s>>>(cam, begin, path_length, n, tech, qbt, pbt, out);
}

}  // namespace upbp
