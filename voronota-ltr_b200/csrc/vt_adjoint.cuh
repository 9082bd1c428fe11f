// vt_adjoint.cuh -- the adjoint epilogue shared by the FP64 and FP32 adjoint kernels
// (vt_adjoint.cu, vt_contact32.cu): from a contact's final contour, the gradient of
// u * area + w_a * SAS_a + w_b * SAS_b + v_a * pyr_a + v_b * pyr_b with respect to the
// balls' centres and radii (pyr_a = t_ab area / 3, the contact's pyramid volume seen from
// a).  The formulas are derived in vt_adjoint.cu.
#pragma once
#include "vt_contact.cuh"
#include "vt_pipeline.cuh"

namespace vt {

constexpr uint32_t kErrAdjoint = 32u;  // a contour needed the serial kernel: not differentiated

__device__ __forceinline__ double adj_wsum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}
__device__ __forceinline__ V3<double> adj_wsum3(V3<double> v) {
    return {adj_wsum(v.x), adj_wsum(v.y), adj_wsum(v.z)};
}
__device__ __forceinline__ void adj_add_grad(double* grad, uint32_t id, uint32_t n, V3<double> gp, double gr) {
    const size_t i = 4 * (size_t)(id % n);
    atomicAdd(grad + i, gp.x);
    atomicAdd(grad + i + 1, gp.y);
    atomicAdd(grad + i + 2, gp.z);
    atomicAdd(grad + i + 3, gr);
}

// Double geometry of pair (a, b) and its weights.
struct AdjPair {
    V3<double> pa, pb, q, axis;  // centres, circle centre, unit axis a -> b
    double Ra, Rb, rho;
    uint32_t a, bid;
    double u, wa, wb;  // area weight (output contact), SAS weights of a and b
    double va, vb;     // volume weights of a and b (0 without a cell, or b an image)
    double area;       // the forward's area of the contact
};

// The pair's area weight with the pyramid volumes t_ab A / 3 and t_ba A / 3 folded in
// (t_ab = (D^2 + Ra^2 - Rb^2) / (2 D): signed distance from p_a to the radical plane).
template <bool VOL>
__device__ __forceinline__ double adj_area_weight(const AdjPair& G) {
    double u = G.u;
    if constexpr (VOL) {
        const V3<double> dab = G.pb - G.pa;
        const double D = sqrt(dot(dab, dab));
        const double t_ab = 0.5 * D + (G.Ra * G.Ra - G.Rb * G.Rb) / (2.0 * D), t_ba = D - t_ab;
        u += (G.va * t_ab + G.vb * t_ba) / 3.0;
    }
    return u;
}

// One contour point's share: point P, the next point Pn, the arc angle of its segment,
// its rid and the next point's lid.  An arc adds its length and first moment to (Lk, Xk);
// a straight edge (on the radical plane of a and c = rid) adds the area weight u times its
// boundary velocity to the gradients of a and b (ga, gra, gb, grb) and of c (directly).
template <typename SphereOf>
__device__ __forceinline__ void adj_point(const AdjPair& G, double u, V3<double> P, V3<double> Pn, double ang,
                                          uint32_t rid, uint32_t nlid, SphereOf sphere_of, double* grad, uint32_t n,
                                          V3<double>& ga, double& gra, V3<double>& gb, double& grb, double& Lk,
                                          V3<double>& Xk) {
    const V3<double> pa = G.pa, pb = G.pb, q = G.q;
    if (rid == G.a && nlid == G.a) {
        if (ang > 0.0) {
            const V3<double> e1 = normalize(P - q);
            const double h = 0.5 * ang;
            const V3<double> mm = e1 * cos(h) + cross(G.axis, e1) * sin(h);
            const double l = G.rho * ang;
            Lk += l;
            Xk = Xk + q * l + mm * (2.0 * G.rho * G.rho * sin(h));
        }
    } else if (u != 0.0) {
        const double4 C = sphere_of(rid);
        if (C.w > 0.0) {
            const V3<double> dab = pb - pa;
            const double D2 = dot(dab, dab);
            const V3<double> pc = mk<double>(C.x, C.y, C.z);
            const V3<double> dac = pc - pa;
            const double kap = dot(dac, dab) / D2;
            const V3<double> perp = (dac - dab * kap) * 2.0;
            const double lam = 1.0 / norm(perp);
            const V3<double> xm = (P + Pn) * 0.5;
            const double coef = u * norm(Pn - P) * lam;
            adj_add_grad(grad, rid, n, (xm - pc) * (-2.0 * coef), -2.0 * C.w * coef);
            ga = ga + (xm - pa) * (2.0 * coef * (1.0 - kap));
            gra += 2.0 * G.Ra * coef * (1.0 - kap);
            gb = gb + (xm - pb) * (2.0 * coef * kap);
            grb += 2.0 * G.Rb * coef * kap;
        }
    }
}

// The pair's terms through its arcs (total length L, first moment X) and pyramids, added
// to the edge terms (ga, gra, gb, grb) and accumulated into a's and b's gradients.
template <bool VOL>
__device__ __forceinline__ void adj_finish(const AdjPair& G, double u, double L, V3<double> X, V3<double> ga,
                                           double gra, V3<double> gb, double grb, double* grad, uint32_t n) {
    const V3<double> pa = G.pa, pb = G.pb, q = G.q;
    const double Ra = G.Ra, Rb = G.Rb, rho = G.rho, wa = G.wa, wb = G.wb;
    const V3<double> dab = pb - pa;
    const double D2 = dot(dab, dab), D = sqrt(D2);
    if (L > 0.0 && rho > 0.0) {
        const double kG = dot(q - pa, dab) / D2;
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
    if (VOL && (G.va != 0.0 || G.vb != 0.0)) {
        // pyramid volumes through t_ab and t_ba at fixed area:
        // dt_ab/dD = 1/2 - dRR/(2 D^2), dt_ab/dRa = Ra/D, dt_ab/dRb = -Rb/D, t_ba = D - t_ab
        const double c = G.area / 3.0;
        const double k = (Ra * Ra - Rb * Rb) / (2.0 * D2);
        const double gD = c * (G.va * (0.5 - k) + G.vb * (0.5 + k));
        const V3<double> nh = dab / D;
        ga = ga - nh * gD;
        gb = gb + nh * gD;
        gra += c * (G.va - G.vb) * Ra / D;
        grb += c * (G.vb - G.va) * Rb / D;
    }
    adj_add_grad(grad, G.a, n, ga, gra);
    adj_add_grad(grad, G.bid, n, gb, grb);
}

// Warp-collective: every lane calls it.  VOL: the pair carries volume weights (va, vb,
// area); without them the pyramid terms are compiled out.  Lane k < len holds contour
// point P (absolute), the next point Pn, the arc angle of its segment, its rid and the
// next point's lid; full: no cut (the whole circle).  sphere_of(id) returns the double
// sphere of a's neighbour with that reference id (w = 0 if not found).
template <bool VOL, typename SphereOf>
__device__ __forceinline__ void adjoint_pair(const AdjPair& G, bool full, int len, V3<double> P, V3<double> Pn,
                                             double ang, uint32_t rid, uint32_t nlid, SphereOf sphere_of,
                                             double* grad, uint32_t n) {
    const int lane = threadIdx.x & 31;
    const double u = adj_area_weight<VOL>(G);
    V3<double> ga = mk<double>(0, 0, 0), gb = mk<double>(0, 0, 0);
    double gra = 0.0, grb = 0.0, Lk = 0.0;
    V3<double> Xk = mk<double>(0, 0, 0);
    if (!full && lane < len) adj_point(G, u, P, Pn, ang, rid, nlid, sphere_of, grad, n, ga, gra, gb, grb, Lk, Xk);
    double L = adj_wsum(Lk);
    V3<double> X = adj_wsum3(Xk);
    ga = adj_wsum3(ga);
    gb = adj_wsum3(gb);
    gra = adj_wsum(gra);
    grb = adj_wsum(grb);
    if (full) {
        L = 2.0 * kPi * G.rho;
        X = G.q * L;
    }
    if (lane == 0) adj_finish<VOL>(G, u, L, X, ga, gra, gb, grb, grad, n);
}

// FP64 position of an FP32 contour vertex from the planes that define it: the radical
// planes of (a, b), (a, lid), (a, rid), or the circle of (a, b) and one plane where lid
// or rid is a.  y0 is the FP32 point relative to a; returns y0 when the construction is
// ill-conditioned (and then clears *ok when given).  sphere_of(id) gives a neighbour's
// double sphere.
template <typename SphereOf>
__device__ __forceinline__ V3<double> snap_vertex(const AdjPair& G, V3<double> y0, uint32_t lid, uint32_t rid,
                                                  SphereOf sphere_of, bool* ok = nullptr) {
    const V3<double> db = G.pb - G.pa;
    const double hb = 0.5 * (dot(db, db) + G.Ra * G.Ra - G.Rb * G.Rb);
    auto plane = [&](uint32_t c, V3<double>& d, double& h) {
        const double4 C = sphere_of(c);
        if (C.w <= 0.0) return false;
        d = mk<double>(C.x, C.y, C.z) - G.pa;
        h = 0.5 * (dot(d, d) + G.Ra * G.Ra - C.w * C.w);
        return true;
    };
    if (lid != G.a && rid != G.a) {
        V3<double> d1, d2;
        double h1, h2;
        if (!plane(lid, d1, h1) || !plane(rid, d2, h2)) { if (ok) *ok = false; return y0; }
        // Cramer on rows db, d1, d2
        const V3<double> c12 = cross(d1, d2), c2b = cross(d2, db), cb1 = cross(db, d1);
        const double det = dot(db, c12);
        const double scale = norm(db) * norm(d1) * norm(d2);
        if (!(fabs(det) > 1e-6 * scale)) { if (ok) *ok = false; return y0; }
        return (c12 * hb + c2b * h1 + cb1 * h2) / det;
    }
    const uint32_t c = lid == G.a ? rid : lid;
    if (c == G.a) { if (ok) *ok = false; return y0; }
    V3<double> dc;
    double hc;
    if (!plane(c, dc, hc)) { if (ok) *ok = false; return y0; }
    // the line of planes b and c: y = y_line + t * dir, then |y - q_rel| = rho
    const V3<double> dir = cross(db, dc);
    const double dd = dot(dir, dir);
    if (!(dd > 1e-12 * dot(db, db) * dot(dc, dc))) { if (ok) *ok = false; return y0; }
    const V3<double> y_line = (cross(dc, dir) * hb + cross(dir, db) * hc) / dd;
    const V3<double> qr = G.q - G.pa;
    const V3<double> w = y_line - qr;
    const double A = dd, B = 2.0 * dot(w, dir), Cq = dot(w, w) - G.rho * G.rho;
    const double disc = B * B - 4.0 * A * Cq;
    if (!(disc >= 0.0)) { if (ok) *ok = false; return y0; }
    const double sq = sqrt(disc);
    const double t1 = (-B - sq) / (2.0 * A), t2 = (-B + sq) / (2.0 * A);
    const V3<double> y1 = y_line + dir * t1, y2 = y_line + dir * t2;
    return norm2(y1 - y0) <= norm2(y2 - y0) ? y1 : y2;
}

// Weights of pair p's contact: u of its output contact (kept pairs), w and v of both
// ends (a periodic image's cell is its own ball's, reached through that ball's pairs);
// v_eff null: no volume term.
__device__ __forceinline__ bool adjoint_weights(const DevBufs& b, uint32_t p, uint32_t a, uint32_t bid,
                                                const double* u_contact, const double* w_eff,
                                                const double* v_eff, AdjPair& G) {
    const bool kept = b.keep_off[p + 1] != b.keep_off[p];
    G.u = (u_contact && kept) ? u_contact[b.keep_off[p]] : 0.0;
    G.wa = w_eff[a];
    G.wb = bid < b.n ? w_eff[bid] : 0.0;
    G.va = v_eff ? v_eff[a] : 0.0;
    G.vb = (v_eff && bid < b.n) ? v_eff[bid] : 0.0;
    G.area = v_eff ? b.p_area[p] : 0.0;
    return G.u != 0.0 || G.wa != 0.0 || G.wb != 0.0 || G.va != 0.0 || G.vb != 0.0;
}

}  // namespace vt
