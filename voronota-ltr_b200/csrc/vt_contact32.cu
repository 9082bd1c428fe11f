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

constexpr int kWarps = 4;

template <bool FULL>
__global__ void __launch_bounds__(kWarps * 32) k_contact32(DevBufs b, uint32_t P) {
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
        const float S = Ra + rb.w;
        g.tol = kTolRel * S;
        g.tolsq = kTolRel * S * S;
        g.tol3 = kTolRel * S * S * S;
        g.tola = kTolRel * 8.f;
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
        k_contact32<true><<<(unsigned)g, kWarps * 32, 0, s>>>(b, P);
    else
        k_contact32<false><<<(unsigned)g, kWarps * 32, 0, s>>>(b, P);
    count_launch();
}

}  // namespace vt
