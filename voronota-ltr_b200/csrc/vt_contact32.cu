// vt_contact32.cu -- FP32 bulk contact kernel (one warp per pair).
//
// Works in coordinates relative to ball a (the CSR holds each neighbour's centre minus
// a's centre, rounded once to float, and its radius), so contour geometry keeps ~7
// significant digits of a's neighbourhood rather than of the absolute coordinates.
// Every fuzzy decision is evaluated with an uncertainty band (vt_geom.cuh, Dec<float,
// true>); a pair with any decision inside its band is marked unsure and recomputed by
// the FP64 kernel, as is a pair whose contour outgrew the warp.
#include "vt_contact.cuh"
#include "vt_pipeline.cuh"

namespace vt {

namespace {

#ifndef VT_C32_WARPS
#define VT_C32_WARPS 4
#endif
#ifndef VT_C32_MINB
#define VT_C32_MINB 1
#endif
constexpr int kWarps = VT_C32_WARPS;

#ifdef VT_DEBUG_SITES
__device__ unsigned long long g_debug_sites[32];
#endif

template <bool FULL>
__global__ void __launch_bounds__(kWarps * 32, VT_C32_MINB) k_contact32(DevBufs b, uint32_t P, float band) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t p = blockIdx.x * kWarps + w; p < P; p += gridDim.x * kWarps) {
        const uint32_t a = b.pair_a[p], eb = b.pair_e[p];
        const uint32_t off = b.nb_off[a], cnt = b.nb_cnt[a];
        PairGeom<float> g;
        const float Ra = (float)b.sph[a].w;
        const float4 rb = b.nb_rel[eb];
        g.A = {{0.f, 0.f, 0.f}, Ra};
        g.B = {{rb.x, rb.y, rb.z}, rb.w};
        g.a_id = a;
        g.b_id = b.nb_id[eb];
        g.S = Ra + rb.w;
        g.e0 = band * g.S;
        const float4* rel = b.nb_rel + off;
        const uint32_t* nid = b.nb_id + off;
        auto nbf = [&](int e) {
            Nb<float> r;
            float4 v = rel[e];
            r.s = {{v.x, v.y, v.z}, v.w};
            r.id = nid[e];
            return r;
        };
        WarpContact r = contact_warp<float, true, FULL>(g, (int)cnt, (int)(eb - off), nbf);
#ifdef VT_DEBUG_SITES
        if (lane == 0 && r.unsure) atomicAdd(&g_debug_sites[r.site < 0 ? 31 : r.site], 1ull);
#endif
        if (lane == 0) {
            uint8_t st = (r.valid ? kValid : 0) | (r.unsure ? kUnsure : 0) | (r.overflow ? kOverflow : 0);
            b.p_status[p] = st;
            b.p_area[p] = r.valid ? r.area : 0.0;
            b.p_arc[p] = r.valid ? r.arc : 0.0;
            b.p_central[p] = r.valid && r.central ? 1 : 0;
            b.p_sa_a[p] = r.valid ? r.sa_a : 0.0;
            b.p_sa_b[p] = r.valid ? r.sa_b : 0.0;
            b.p_pv_a[p] = r.valid ? r.pv_a : 0.0;
            b.p_pv_b[p] = r.valid ? r.pv_b : 0.0;
        }
    }
}

}  // namespace

void launch_contact_f32(const DevBufs& b, uint32_t P, int full, cudaStream_t s) {
    size_t g = (P + kWarps - 1) / kWarps;
    if (g < 1) g = 1;
    if (g > 148 * 64) g = 148 * 64;
    if (full)
        k_contact32<true><<<(unsigned)g, kWarps * 32, 0, s>>>(b, P, b.fp32_band);
    else
        k_contact32<false><<<(unsigned)g, kWarps * 32, 0, s>>>(b, P, b.fp32_band);
    count_launch();
}

}  // namespace vt

#ifdef VT_DEBUG_SITES
// Debug builds only: histogram of the first unsure step per flagged pair (read and clear).
extern "C" int vt_debug_flag_sites(unsigned long long* out32) {
    cudaMemcpyFromSymbol(out32, vt::g_debug_sites, 32 * sizeof(unsigned long long));
    unsigned long long z[32] = {0};
    cudaMemcpyToSymbol(vt::g_debug_sites, z, sizeof(z));
    return 0;
}
#endif
