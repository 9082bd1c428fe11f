// vt_adjoint.cu -- hand-written adjoint of
//     L = sum_i w_i SAS_i + sum_k u_k area_k
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
// Periodic images contribute to the ball they image (id mod n); only balls with a cell
// whose SAS is positive receive SAS terms.  Accumulation uses double atomics.
#include <cmath>

#include "vt_contact.cuh"
#include "vt_pipeline.cuh"

namespace vt {

namespace {

constexpr int kWarps = 4;
constexpr uint32_t kErrAdjoint = 32u;  // a contour needed the serial kernel: not differentiated

__device__ __forceinline__ Sph<double> sph_of(double4 v) { return {{v.x, v.y, v.z}, v.w}; }

__device__ __forceinline__ double wsum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}
__device__ __forceinline__ V3<double> wsum3(V3<double> v) { return {wsum(v.x), wsum(v.y), wsum(v.z)}; }

__device__ __forceinline__ void add_grad(double* grad, uint32_t id, uint32_t n, V3<double> gp, double gr) {
    const size_t i = 4 * (size_t)(id % n);
    atomicAdd(grad + i, gp.x);
    atomicAdd(grad + i + 1, gp.y);
    atomicAdd(grad + i + 2, gp.z);
    atomicAdd(grad + i + 3, gr);
}

__global__ void k_w_eff(uint32_t n, const double* __restrict__ w, const uint8_t* __restrict__ cell_flag,
                        const double* __restrict__ cell_sas, double* __restrict__ w_eff) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        w_eff[i] = (w && cell_flag[i] && cell_sas[i] > 0.0) ? w[i] : 0.0;
}
// d SAS_i / d R_i at fixed exposed directions: 2 SAS_i / R_i
__global__ void k_sas_scale(uint32_t n, const double* __restrict__ w_eff, const double* __restrict__ cell_sas,
                            const double4* __restrict__ sph, double* __restrict__ grad) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (w_eff[i] != 0.0) grad[4 * (size_t)i + 3] += w_eff[i] * 2.0 * cell_sas[i] / sph[i].w;
}

__global__ void __launch_bounds__(kWarps * 32)
    k_adjoint64(DevBufs b, uint32_t P, const double* __restrict__ u_contact, const double* __restrict__ w_eff,
                double* __restrict__ grad) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t n = b.n;
    for (uint32_t p = blockIdx.x * kWarps + w; p < P; p += gridDim.x * kWarps) {
        if (!(b.p_status[p] & kValid)) continue;
        const uint32_t a = b.pair_a[p], eb = b.pair_e[p];
        const uint32_t bid = b.nb_id[eb];
        const bool kept = b.keep_off[p + 1] != b.keep_off[p];
        const double u = (u_contact && kept) ? u_contact[b.keep_off[p]] : 0.0;
        const double wa = w_eff[a];
        const double wb = bid < n ? w_eff[bid] : 0.0;
        if (u == 0.0 && wa == 0.0 && wb == 0.0) continue;
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
        if (!r.valid) {
            if (lane == 0 && r.overflow) atomicOr(b.err, kErrAdjoint);
            continue;
        }
        const V3<double> pa = g.A.c, pb = g.B.c;
        const double Ra = g.A.r, Rb = g.B.r;
        const V3<double> q = co.ic.c;
        const double rho = co.ic.r;
        const V3<double> dab = pb - pa;
        const double D2 = dot(dab, dab), D = sqrt(D2);
        const int len = co.len;
        // this lane's boundary piece
        V3<double> ga = mk<double>(0, 0, 0), gb = mk<double>(0, 0, 0);
        double gra = 0.0, grb = 0.0, Lk = 0.0;
        V3<double> Xk = mk<double>(0, 0, 0);
        const int nx = len > 0 ? (lane + 1 < len ? lane + 1 : 0) : 0;
        const Pt<double> nxt = shfl_pt(co.q, nx);
        if (!co.full && lane < len) {
            const Pt<double>& pt = co.q;
            if (pt.rid == a && nxt.lid == a) {
                const double al = pt.ang;
                if (al > 0.0) {
                    const V3<double> e1 = normalize(pt.p - q);
                    const double h = 0.5 * al;
                    const V3<double> mm = e1 * cos(h) + cross(co.axis, e1) * sin(h);
                    Lk = rho * al;
                    Xk = q * Lk + mm * (2.0 * rho * rho * sin(h));
                }
            } else if (u != 0.0) {
                // straight edge on the radical plane of a and c = pt.rid
                const uint32_t c = pt.rid;
                uint32_t slot = 0xffffffffu;
                for (uint32_t e = 0; e < cnt; ++e)
                    if (nid[e] == c) {
                        slot = nslot[e];
                        break;
                    }
                if (slot != 0xffffffffu) {
                    const Sph<double> C = sph_of(sph[slot]);
                    const V3<double> dac = C.c - pa;
                    const double kap = dot(dac, dab) / D2;
                    const V3<double> perp = (dac - dab * kap) * 2.0;
                    const double lam = 1.0 / norm(perp);
                    const V3<double> xm = (pt.p + nxt.p) * 0.5;
                    const double coef = u * norm(nxt.p - pt.p) * lam;
                    add_grad(grad, c, n, (xm - C.c) * (-2.0 * coef), -2.0 * C.r * coef);
                    ga = (xm - pa) * (2.0 * coef * (1.0 - kap));
                    gra = 2.0 * Ra * coef * (1.0 - kap);
                    gb = (xm - pb) * (2.0 * coef * kap);
                    grb = 2.0 * Rb * coef * kap;
                }
            }
        }
        double L = wsum(Lk);
        V3<double> X = wsum3(Xk);
        ga = wsum3(ga);
        gb = wsum3(gb);
        gra = wsum(gra);
        grb = wsum(grb);
        if (co.full) {
            L = 2.0 * kPi * rho;
            X = q * L;
        }
        if (lane == 0) {
            if (L > 0.0 && rho > 0.0) {
                const double da = dot(q - pa, dab) / D;
                const double kG = da / D;
                const V3<double> Xa = X - pa * L, Xb = X - pb * L;
                // area through the arcs
                ga = ga + Xa * (u * (1.0 - kG) / rho);
                gra += u * (1.0 - kG) * Ra * L / rho;
                gb = gb + Xb * (u * kG / rho);
                grb += u * kG * Rb * L / rho;
                // SAS of a and of b through the same arcs
                const double s = 1.0 / (D * rho);
                const double cmix = (Ra * Ra + Rb * Rb - D2) * 0.5;
                ga = ga + Xb * (wa * Ra * s) - Xa * (wb * Rb * s);
                gb = gb - Xb * (wa * Ra * s) + Xa * (wb * Rb * s);
                gra += wa * L * cmix * s - wb * Rb * Ra * L * s;
                grb += wb * L * cmix * s - wa * Ra * Rb * L * s;
            }
            add_grad(grad, a, n, ga, gra);
            add_grad(grad, bid, n, gb, grb);
        }
    }
}

int gb(size_t n) { return grid_blocks(n, 256, 148 * 16); }

}  // namespace

void set_hex_table_adjoint() {
    double hs[8], hc[8];
    int n = 0;
    hex_table_values(hs, hc, &n);
    cudaMemcpyToSymbol(c_hex_sin, hs, sizeof(hs));
    cudaMemcpyToSymbol(c_hex_cos, hc, sizeof(hc));
    cudaMemcpyToSymbol(c_hex_n, &n, sizeof(int));
}

void launch_adjoint(const DevBufs& b, uint32_t P, const double* w_sas, const double* u_contact, double* w_eff,
                    double* grad, cudaStream_t s) {
    const uint32_t n = b.n;
    cudaMemsetAsync(grad, 0, 4 * sizeof(double) * n, s);
    k_w_eff<<<gb(n), 256, 0, s>>>(n, w_sas, b.cell_flag, b.cell_sas, w_eff); count_launch();
    if (P) {
        k_adjoint64<<<grid_blocks(P, kWarps, 148 * 64), kWarps * 32, 0, s>>>(b, P, u_contact, w_eff, grad);
        count_launch();
    }
    k_sas_scale<<<gb(n), 256, 0, s>>>(n, w_eff, b.cell_sas, b.sph, grad); count_launch();
}

}  // namespace vt
