// vt_adjoint.cu -- hand-written adjoint of
//     L = sum_i w_i SAS_i + sum_i v_i V_i + sum_k u_k area_k
// with respect to the centres and radii of the balls (no counterpart in the reference).
//
// The backward pass recomputes every contact's contour (FP64 warp kernel, the same
// clipping as the forward) instead of storing it, and differentiates through the
// geometry of the final region rather than through the clipping steps:
//
// * A contact (a, b) is the region of the radical plane P_ab inside the circle
//   C_ab = S_a n P_ab and on a's side of the radical planes P_ac of the cutting
//   neighbours c.  Its area changes only through its boundary: dA = sum over boundary
//   pieces of the integral of the in-plane outward normal velocity.  With the power
//   functions F_c(x) = |x-p_a|^2 - R_a^2 - |x-p_c|^2 + R_c^2 (zero on P_ac) and
//   G(x) = |x-p_a|^2 - R_a^2, a point on the edge of c moves outward by
//       v = (-dF_c(x) + k_c dF_b(x)) / |n_c - k_c n_b|,   n_c = grad F_c,
//       k_c = n_c.n_b / |n_b|^2,
//   and a point of an arc by v = (-dG(x) + k_G dF_b(x)) / (2 rho), k_G = d_a / D, where dF
//   are the parameter derivatives at fixed x.  These are affine in x, so an edge
//   contributes its length times v at its midpoint, and the arcs contribute through their
//   total length L and first moment X = integral of x ds.
// * SAS_a = R_a^2 |E_a|, E_a the exposed directions of sphere a, whose boundary is made of
//   the arcs of a's contacts.  On sphere a an arc of contact (a, b) moves by
//       nu.dw = ((x-p_b).(dp_a - dp_b) + dR_a (R_a^2+R_b^2-D^2)/(2 R_a) - R_b dR_b)
//               / (D rho)          (per unit length on the unit sphere, times 1/R_a),
//   giving d SAS_a = 2 R_a dR_a |E_a| + R_a^2 d|E_a|; the arcs bound E_b the same way.
//
// * The cell volume is V_a = SAS_a R_a / 3 + sum_b pyr_ab (types.rs:647-649) with the
//   pyramid pyr_ab = |q_ab - p_a| area_ab / 3 signed by the solid angle (contact.rs:
//   374-379).  That sign is negative exactly when the circle centre q_ab lies behind p_a
//   as seen from p_b (contact.rs:839-845), so pyr_ab = t_ab area_ab / 3 with the signed
//   distance t_ab = (D^2 + R_a^2 - R_b^2) / (2 D) from p_a to the radical plane.  Hence
//   v_a V_a adds v_a R_a / 3 to the SAS weight of a, v_a SAS_a / 3 to dL/dR_a, and, per
//   contact, (v_a t_ab + v_b t_ba) / 3 to its area weight plus area/3 times the
//   derivatives of t_ab and t_ba (vt_adjoint.cuh).  Where compute_sas leaves SAS at 0
//   (no arcs, or the full-sphere sanity reset of types.rs:651-657) V is the pyramid sum
//   alone, which the zero SAS weight of such a cell gives; a detached ball (V = 4 pi R^3
//   / 3, SAS = 4 pi R^2) gets dV/dR = SAS the same way.
//
// Periodic images contribute to the ball they image (id mod n); only balls with a cell
// whose SAS is positive receive SAS terms, only balls with a cell volume terms.
// Accumulation uses double atomics.
#include <cmath>

#include "vt_adjoint.cuh"

namespace vt {

namespace {

constexpr int kWarps = 4;

__device__ __forceinline__ Sph<double> sph_of(double4 v) { return {{v.x, v.y, v.z}, v.w}; }

// w_eff: the SAS weight of each ball, w + v R / 3 (the SAS R / 3 part of its volume),
// where the ball has a cell with a positive SAS; v_eff: the volume weight where it has a
// cell (null without volume weights)
__global__ void k_w_eff(uint32_t n, const double* __restrict__ w, const double* __restrict__ v,
                        const uint8_t* __restrict__ cell_flag, const double* __restrict__ cell_sas,
                        const double4* __restrict__ sph, double* __restrict__ w_eff, double* __restrict__ v_eff) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const bool cell = cell_flag[i] != 0;
        const double vi = (v && cell) ? v[i] : 0.0;
        w_eff[i] = (cell && cell_sas[i] > 0.0) ? (w ? w[i] : 0.0) + vi * sph[i].w / 3.0 : 0.0;
        if (v_eff) v_eff[i] = vi;
    }
}
// d SAS_i / d R_i at fixed exposed directions: 2 SAS_i / R_i; and d(SAS_i R_i / 3) / dR_i
// at fixed SAS: SAS_i / 3
__global__ void k_sas_scale(uint32_t n, const double* __restrict__ w_eff, const double* __restrict__ v_eff,
                            const double* __restrict__ cell_sas, const double4* __restrict__ sph,
                            double* __restrict__ grad) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double vi = v_eff ? v_eff[i] : 0.0;
        if (w_eff[i] != 0.0 || (vi != 0.0 && cell_sas[i] > 0.0))
            grad[4 * (size_t)i + 3] += w_eff[i] * 2.0 * cell_sas[i] / sph[i].w + vi * cell_sas[i] / 3.0;
    }
}

// FP64 adjoint: all valid pairs, or (from_list) the pairs the FP32 adjoint listed.  At
// most 128 registers (4 resident blocks), like the FP64 contact kernel.
template <bool VOL>
__global__ void __launch_bounds__(kWarps * 32, 4)
    k_adjoint64(DevBufs b, uint32_t P, int from_list, const double* __restrict__ u_contact,
                const double* __restrict__ w_eff, const double* __restrict__ v_eff, double* __restrict__ grad) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t n = b.n;
    const uint32_t count = from_list ? *b.d_redo_count : P;
    for (uint32_t it = blockIdx.x * kWarps + w; it < count; it += gridDim.x * kWarps) {
        const uint32_t p = from_list ? b.redo_list[it] : it;
        if (!(b.p_status[p] & kValid)) continue;
        const uint32_t a = b.pair_a[p], eb = b.pair_e[p];
        const uint32_t bid = b.nb_id[eb];
        AdjPair G;
        if (!adjoint_weights(b, p, a, bid, u_contact, w_eff, v_eff, G)) continue;
        const uint32_t off = b.nb_off[a], cnt = b.nb_cnt[a];
        PairGeom<double> g;
        g.A = sph_of(b.sph[a]);
        g.B = sph_of(b.sph[b.nb_slot[eb]]);
        g.a_id = a;
        g.b_id = bid;
        g.e0 = 0.0;
        g.S = g.A.r + g.B.r;
        const double4* sph = b.sph;
        const uint32_t* nslot = b.nb_slot + off;
        const uint32_t* nid = b.nb_id + off;
        auto nbf = [&](int e) {
            Nb<double> r;
            r.s = sph_of(sph[nslot[e]]);
            r.id = nid[e];
            return r;
        };
        ContourOut<double> co;
        WarpContact r = contact_warp<double, false, false>(g, (int)cnt, (int)(eb - off), nbf, &co);
        if (!r.valid) {  // a contour beyond the warp's 32 points goes to the serial adjoint
            if (lane == 0 && r.overflow) b.serial_list[atomicAdd(b.d_serial_count, 1u)] = p;
            continue;
        }
        G.pa = g.A.c;
        G.pb = g.B.c;
        G.Ra = g.A.r;
        G.Rb = g.B.r;
        G.q = co.ic.c;
        G.rho = co.ic.r;
        G.axis = co.axis;
        G.a = a;
        G.bid = bid;
        const int len = co.len;
        const int nx = len > 0 ? (lane + 1 < len ? lane + 1 : 0) : 0;
        const Pt<double> nxt = shfl_pt(co.q, nx);
        auto sphere_of = [&](uint32_t c) {
            for (uint32_t e = 0; e < cnt; ++e)
                if (nid[e] == c) return sph[nslot[e]];
            return make_double4(0.0, 0.0, 0.0, 0.0);
        };
        adjoint_pair<VOL>(G, co.full, len, co.q.p, nxt.p, co.q.ang, co.q.rid, nxt.lid, sphere_of, grad, n);
    }
}

int gb(size_t n) { return grid_blocks(n, 256, 148 * 16); }

void launch_adjoint64(const DevBufs& b, uint32_t P, int from_list, const double* u_contact, const double* w_eff,
                      const double* v_eff, double* grad, cudaStream_t s) {
    const int g = grid_blocks(P, kWarps, 148 * 64);
    if (v_eff)
        k_adjoint64<true><<<g, kWarps * 32, 0, s>>>(b, P, from_list, u_contact, w_eff, v_eff, grad);
    else
        k_adjoint64<false><<<g, kWarps * 32, 0, s>>>(b, P, from_list, u_contact, w_eff, v_eff, grad);
}

}  // namespace

void set_hex_table_adjoint() {
    double hs[8], hc[8];
    int n = 0;
    hex_table_values(hs, hc, &n);
    cudaMemcpyToSymbol(c_hex_sin, hs, sizeof(hs));
    cudaMemcpyToSymbol(c_hex_cos, hc, sizeof(hc));
    cudaMemcpyToSymbol(c_hex_n, &n, sizeof(int));
}

void launch_adjoint(const DevBufs& b, uint32_t P, const double* w_sas, const double* v_vol, const double* u_contact,
                    double* w_eff, double* v_eff, double* grad, cudaStream_t s) {
    const uint32_t n = b.n;
    double* ve = v_vol ? v_eff : nullptr;
    cudaMemsetAsync(grad, 0, 4 * sizeof(double) * n, s);
    cudaMemsetAsync(b.d_serial_count, 0, sizeof(uint32_t), s);
    k_w_eff<<<gb(n), 256, 0, s>>>(n, w_sas, v_vol, b.cell_flag, b.cell_sas, b.sph, w_eff, ve); count_launch();
    if (P) {
        if (b.nb_rel) {
            // FP32 contours; pairs with a decision in the band are redone in FP64
            cudaMemsetAsync(b.d_redo_count, 0, sizeof(uint32_t), s);
            launch_adjoint_f32(b, P, u_contact, w_eff, ve, grad, s);
            launch_adjoint64(b, P, 1, u_contact, w_eff, ve, grad, s);
        } else {
            launch_adjoint64(b, P, 0, u_contact, w_eff, ve, grad, s);
        }
        count_launch();
        launch_adjoint_serial(b, u_contact, w_eff, ve, grad, s);
    }
    k_sas_scale<<<gb(n), 256, 0, s>>>(n, w_eff, ve, b.cell_sas, b.sph, grad); count_launch();
}

}  // namespace vt
