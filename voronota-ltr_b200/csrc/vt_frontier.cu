// vt_frontier.cu -- kernels of the updateable tessellation: change detection, the
// dirty-ball frontier (changed balls and their old and new neighbours), neighbour-list
// splice, frontier pair generation, the per-ball contact table splice and per-ball cells.
// FP64 throughout (compiled with --fmad=false like the rest of the pipeline).
#include <cfloat>

#include "vt_frontier.cuh"
#include "vt_geom.cuh"

namespace vt {

namespace {

constexpr int kBlock = 256;
constexpr int kWarps = 8;         // warps per block of the warp-per-ball kernels
constexpr int kRankCap = 512;     // new table entries one ball may receive in one pass
constexpr uint32_t kErrTable = 16u;  // a ball received more new entries than kRankCap

struct PBoxArgF {
    double v[9];
};

__device__ __forceinline__ double wsum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__global__ void k_images_all(double4* __restrict__ sph, uint32_t n, PBoxArgF pb) {
    const size_t total = (size_t)n * 26;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        uint32_t j = (uint32_t)(t % n);
        int g = (int)(t / n);
        int sx, sy, sz;
        neighbor_shift(g, sx, sy, sz);
        sph[(size_t)(g + 1) * n + j] = shift_sphere(sph[j], pb.v, sx, sy, sz);
    }
}

// sphere_equals_sphere (geometry.rs:73-75): |dR|, |dx|, |dy|, |dz| <= 1e-10
__global__ void k_changed_flags(const uint64_t* __restrict__ ids, uint32_t k, const double* __restrict__ src,
                                int src_by_id, uint32_t n, double probe, const double* __restrict__ balls,
                                uint32_t* __restrict__ flags) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < k; t += gridDim.x * blockDim.x) {
        uint64_t id = ids ? ids[t] : t;
        uint32_t f = 0;
        if (id < n) {
            const double* v = src + 4 * (src_by_id ? id : (uint64_t)t);
            const double* o = balls + 4 * id;  // the stored sphere: (x, y, z, r + probe)
            const double R = v[3] + probe, Ro = o[3] + probe;
            bool eq = fabs(R - Ro) <= kEps && fabs(v[0] - o[0]) <= kEps && fabs(v[1] - o[1]) <= kEps &&
                      fabs(v[2] - o[2]) <= kEps;
            f = eq ? 0u : 1u;
        }
        flags[t] = f;
    }
}
__global__ void k_changed_compact(const uint64_t* __restrict__ ids, uint32_t k, const double* __restrict__ src,
                                  int src_by_id, const uint32_t* __restrict__ off, uint32_t* __restrict__ changed,
                                  double4* __restrict__ changed_ball) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < k; t += gridDim.x * blockDim.x) {
        uint32_t o = off[t];
        if (off[t + 1] == o) continue;
        uint64_t id = ids ? ids[t] : t;
        const double* v = src + 4 * (src_by_id ? id : (uint64_t)t);
        changed[o] = (uint32_t)id;
        changed_ball[o] = make_double4(v[0], v[1], v[2], v[3]);
    }
}
__global__ void k_clamp_count(uint32_t* count, uint32_t cap) {
    if (threadIdx.x == 0 && blockIdx.x == 0 && *count > cap) *count = cap;
}
__global__ void k_apply_changed(const uint32_t* __restrict__ changed, const double4* __restrict__ cb,
                                const uint32_t* __restrict__ count, double* __restrict__ balls) {
    const uint32_t m = *count;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
        const uint32_t c = changed[t];
        const double4 v = cb[t];
        balls[4 * (size_t)c] = v.x;
        balls[4 * (size_t)c + 1] = v.y;
        balls[4 * (size_t)c + 2] = v.z;
        balls[4 * (size_t)c + 3] = v.w;
    }
}
__global__ void k_mark_list(const uint32_t* __restrict__ list, const uint32_t* __restrict__ count,
                            uint32_t* __restrict__ mark, uint32_t val, uint32_t* __restrict__ d_new) {
    const uint32_t m = *count;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x)
        if (atomicCAS(&mark[list[t]], 0u, val) == 0u) atomicAdd(d_new, 1u);
}
__global__ void __launch_bounds__(kWarps * 32)
    k_mark_neighbours(const uint32_t* __restrict__ list, const uint32_t* __restrict__ count,
                      const uint32_t* __restrict__ row_of, ListsRef L, uint32_t n, uint32_t* __restrict__ mark,
                      uint32_t val, uint32_t* __restrict__ d_new, uint32_t* __restrict__ append) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t m = *count;
    for (uint32_t t = blockIdx.x * kWarps + w; t < m; t += gridDim.x * kWarps) {
        const uint32_t c = list[t];
        const uint32_t row = row_of ? row_of[c] : c;
        const uint32_t cnt = L.cnt[row], off = L.off[row];
        for (uint32_t e = lane; e < cnt; e += 32) {
            const uint32_t x = L.id[off + e] % n;
            if (atomicCAS(&mark[x], 0u, val) == 0u) {
                uint32_t at = atomicAdd(d_new, 1u);
                if (append) append[at] = x;
            }
        }
    }
}
__global__ void k_mark_table_partners(uint32_t id, TableRef T, uint32_t* __restrict__ mark) {
    const uint32_t s = T.off[id], e = T.off[id + 1];
    if (blockIdx.x == 0 && threadIdx.x == 0) mark[id] = 1u;
    for (uint32_t q = s + threadIdx.x; q < e; q += blockDim.x) {
        const uint32_t o = T.a[q] == id ? T.b[q] : T.a[q];
        mark[o] = 1u;
    }
}
__global__ void k_nonzero(const uint32_t* __restrict__ mark, uint32_t n, uint32_t* __restrict__ flags) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        flags[i] = mark[i] ? 1u : 0u;
}
__global__ void k_compact_index(const uint32_t* __restrict__ off, uint32_t n, uint32_t* __restrict__ list) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (off[i + 1] != off[i]) list[off[i]] = i;
}
__global__ void k_row_of(const uint32_t* __restrict__ list, const uint32_t* __restrict__ count,
                         uint32_t* __restrict__ row_of) {
    const uint32_t m = *count;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) row_of[list[t]] = t;
}
__global__ void k_splice_counts(uint32_t n, const uint32_t* __restrict__ mark, const uint32_t* __restrict__ row_of,
                                const uint32_t* __restrict__ old_cnt, const uint32_t* __restrict__ c1,
                                const uint32_t* __restrict__ c2, uint32_t* __restrict__ cnt) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t m = mark[i];
        cnt[i] = m == 0 ? old_cnt[i] : (m == 1 ? c1[row_of[i]] : c2[row_of[i]]);
    }
}
__global__ void __launch_bounds__(kWarps * 32)
    k_splice_lists(uint32_t n, const uint32_t* __restrict__ mark, const uint32_t* __restrict__ row_of, ListsRef o,
                   ListsRef t1, ListsRef t2, const uint32_t* __restrict__ new_off, uint32_t* __restrict__ id,
                   double* __restrict__ val, float4* __restrict__ rel) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t i = blockIdx.x * kWarps + w; i < n; i += gridDim.x * kWarps) {
        const uint32_t m = mark[i];
        const ListsRef& L = m == 0 ? o : (m == 1 ? t1 : t2);
        const uint32_t row = m == 0 ? i : row_of[i];
        const uint32_t cnt = L.cnt[row], so = L.off[row], d = new_off[i];
        for (uint32_t e = lane; e < cnt; e += 32) {
            id[d + e] = L.id[so + e];
            val[d + e] = L.val[so + e];
            if (rel) rel[d + e] = L.rel[so + e];
        }
    }
}

// collect_collision_pairs (updateable.rs:516-561): a involved and not excluded; b's
// canonical ball involved and not excluded; a < b, or b a periodic image.  need > 0: also
// mark[a] >= need or mark[b's canonical ball] >= need.
template <bool FILL>
__global__ void __launch_bounds__(kWarps * 32)
    k_upd_pairs(const uint32_t* __restrict__ list, const uint32_t* __restrict__ count, uint32_t n, int periodic,
                ListsRef L, const uint8_t* __restrict__ excl, const uint32_t* __restrict__ mark, uint32_t need,
                uint32_t* __restrict__ npair, const uint32_t* __restrict__ pair_off, uint32_t* __restrict__ pair_a,
                uint32_t* __restrict__ pair_e, int32_t* __restrict__ nb_pair) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t m = list ? *count : n;
    for (uint32_t t = blockIdx.x * kWarps + w; t < m; t += gridDim.x * kWarps) {
        const uint32_t a = list ? list[t] : t;
        const bool a_ok = !excl[a];
        const bool a_need = need == 0 || mark[a] >= need;
        const uint32_t cnt = L.cnt[a], off = L.off[a];
        uint32_t rank = FILL ? pair_off[a] : 0u;
        for (uint32_t e0 = 0; e0 < cnt; e0 += 32) {
            const uint32_t e = e0 + lane;
            bool gen = false;
            if (e < cnt && a_ok) {
                const uint32_t bid = L.id[off + e];
                const uint32_t bc = periodic ? bid % n : bid;
                gen = (!mark || mark[bc]) && !excl[bc] && ((periodic && bid >= n) || a < bid) &&
                      (a_need || mark[bc] >= need);
            }
            const unsigned bal = __ballot_sync(0xffffffffu, gen);
            if (FILL && e < cnt) {
                int32_t p = -1;
                if (gen) {
                    p = (int32_t)(rank + __popc(bal & ((1u << lane) - 1u)));
                    pair_a[p] = a;
                    pair_e[p] = off + e;
                }
                nb_pair[off + e] = p;
            }
            rank += __popc(bal);
        }
        if (!FILL && lane == 0) npair[a] = rank;
    }
}

__global__ void k_new_contacts(uint32_t P, const uint32_t* __restrict__ keep_off, DevBufs b, NewContacts nc) {
    const uint32_t n = b.n;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < P; p += gridDim.x * blockDim.x) {
        const uint32_t k = keep_off[p];
        if (keep_off[p + 1] == k) continue;
        // ensure_ids_ordered on the raw ids is a no-op (a < b or b an image); then ids % n
        // and ensure_ids_ordered again (types.rs:408-414)
        uint32_t ia = b.pair_a[p] % n, ib = b.nb_id[b.pair_e[p]] % n;
        const bool swap = ia > ib;
        double sa = b.p_sa_a[p], sb = b.p_sa_b[p], pa = b.p_pv_a[p], pb = b.p_pv_b[p];
        if (swap) {
            uint32_t t = ia;
            ia = ib;
            ib = t;
            double x = sa;
            sa = sb;
            sb = x;
            x = pa;
            pa = pb;
            pb = x;
        }
        nc.a[k] = ia;
        nc.b[k] = ib;
        nc.area[k] = b.p_area[p];
        nc.arc[k] = b.p_arc[p];
        nc.sa_a[k] = sa;
        nc.sa_b[k] = sb;
        nc.pv_a[k] = pa;
        nc.pv_b[k] = pb;
        nc.central[k] = b.p_central[p];
        nc.pair[k] = p;
        if (nc.gaa && b.p_arcm) {
            // the SAS adjoint through this contact's arcs: with X the arcs' first moment
            // about a, L their length, s = 1 / (D rho) and c = (Ra^2 + Rb^2 - D^2) / 2,
            //   dSAS_a/dp_a = Ra s (X - (b-a) L),  dSAS_a/dR_a = L c s,  dSAS_a/dR_b = -Ra Rb L s
            // (and a <-> b), dSAS_a/dp_b = -dSAS_a/dp_a
            const double4 A4 = b.sph[b.pair_a[p]], B4 = b.sph[b.nb_slot[b.pair_e[p]]];
            const V3<double> dab = mk<double>(B4.x - A4.x, B4.y - A4.y, B4.z - A4.z);
            const double Ra = A4.w, Rb = B4.w, D2 = dot(dab, dab), D = sqrt(D2);
            const double L = b.p_arc[p];
            const double* xm = b.p_arcm + 6 * (size_t)p;
            const V3<double> Xa = mk<double>(xm[0], xm[1], xm[2]);
            double4 aa = make_double4(0, 0, 0, 0), ab = aa, ba = aa, bb = aa;
            const double da = D > 0.0 ? (D2 + Ra * Ra - Rb * Rb) / (2.0 * D) : 0.0;
            const double rho = sqrt(fmax(Ra * Ra - da * da, 0.0));
            if (L > 0.0 && rho > 0.0 && D > 0.0) {
                const double s = 1.0 / (D * rho), c = 0.5 * (Ra * Ra + Rb * Rb - D2);
                const V3<double> Xb = Xa - dab * L;
                const V3<double> ga = Xb * (Ra * s), gb = Xa * (Rb * s);
                aa = make_double4(ga.x, ga.y, ga.z, L * c * s);
                ab = make_double4(-ga.x, -ga.y, -ga.z, -Ra * Rb * L * s);
                bb = make_double4(gb.x, gb.y, gb.z, L * c * s);
                ba = make_double4(-gb.x, -gb.y, -gb.z, -Rb * Ra * L * s);
            }
            nc.gaa[k] = swap ? bb : aa;
            nc.gab[k] = swap ? ba : ab;
            nc.gba[k] = swap ? ab : ba;
            nc.gbb[k] = swap ? aa : bb;
            // the volume adjoint through the contact's face (Reynolds' transport theorem:
            // a cell's volume changes by the normal velocity of its boundary).  The face lies
            // on the radical plane, whose point x moves towards b by ((x - a).dp_a -
            // (x - b).dp_b + Ra dRa - Rb dRb) / D; over the face that integrates to the
            // face's area A and first moment M_a = integral of (x - a) (M_b = M_a - A (b - a)):
            //   dV_a/dp_a = M_a / D - A n,  dV_a/dR_a = A Ra / D,   n = (b - a) / D,
            //   dV_b/dp_a = -M_a / D,       dV_b/dR_a = -A Ra / D,
            // and a <-> b with n -> -n.  The -A n term is the exposed sphere's share: the
            // cell's boundary is closed, so the integral of the outward normal over the
            // exposed part of sphere a is minus the sum of A n over a's faces; its radius
            // term (the exposed area) is added per ball by the gather.
            double4 vaa = make_double4(0, 0, 0, 0), vab = vaa, vba = vaa, vbb = vaa;
            const double A = b.p_area[p];
            if (A > 0.0 && D > 0.0) {
                const V3<double> Ma = mk<double>(xm[3], xm[4], xm[5]);
                const V3<double> Mb = Ma - dab * A;
                const V3<double> nh = dab / D;
                const V3<double> ca = Ma / D - nh * A, cb = Mb / D + nh * A;
                vaa = make_double4(ca.x, ca.y, ca.z, A * Ra / D);  // dV_a / d(a)
                vba = make_double4(-Ma.x / D, -Ma.y / D, -Ma.z / D, -A * Ra / D);  // dV_b / d(a)
                vbb = make_double4(cb.x, cb.y, cb.z, A * Rb / D);  // dV_b / d(b)
                vab = make_double4(-Mb.x / D, -Mb.y / D, -Mb.z / D, -A * Rb / D);  // dV_a / d(b)
            }
            nc.vaa[k] = swap ? vbb : vaa;
            nc.vab[k] = swap ? vba : vab;
            nc.vba[k] = swap ? vab : vba;
            nc.vbb[k] = swap ? vaa : vbb;
        }
    }
}

__global__ void k_table_counts(uint32_t n, const uint32_t* __restrict__ mark, TableRef o,
                               uint32_t* __restrict__ keep_cnt) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (!o.off) {
            keep_cnt[i] = 0;
            continue;
        }
        const uint32_t s = o.off[i], e = o.off[i + 1];
        uint32_t k = e - s;
        if (mark[i]) {
            k = 0;
            for (uint32_t q = s; q < e; ++q) {
                const uint32_t other = o.a[q] == i ? o.b[q] : o.a[q];
                if (!mark[other]) ++k;
            }
        }
        keep_cnt[i] = k;
    }
}
__global__ void k_table_new_counts(NewContacts nc, const uint32_t* __restrict__ nc_count,
                                   uint32_t* __restrict__ new_cnt) {
    const uint32_t m = *nc_count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        atomicAdd(&new_cnt[nc.a[k]], 1u);
        if (nc.b[k] != nc.a[k]) atomicAdd(&new_cnt[nc.b[k]], 1u);
    }
}
__global__ void k_add_u32(const uint32_t* __restrict__ x, const uint32_t* __restrict__ y, uint32_t n,
                          uint32_t* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = x[i] + y[i];
}
__device__ __forceinline__ void copy_entry(const TableRef& o, uint32_t q, const TableRef& w, uint32_t d) {
    w.a[d] = o.a[q];
    w.b[d] = o.b[q];
    w.area[d] = o.area[q];
    w.arc[d] = o.arc[q];
    w.sa[d] = o.sa[q];
    w.pv[d] = o.pv[q];
    w.flags[d] = o.flags[q];
    if (w.gA) {
        w.gA[d] = o.gA[q];
        w.gB[d] = o.gB[q];
        w.vA[d] = o.vA[q];
        w.vB[d] = o.vB[q];
    }
}
__global__ void __launch_bounds__(kWarps * 32)
    k_table_copy_kept(uint32_t n, const uint32_t* __restrict__ mark, TableRef o, TableRef w) {
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    for (uint32_t i = blockIdx.x * kWarps + wp; i < n; i += gridDim.x * kWarps) {
        const uint32_t s = o.off[i], e = o.off[i + 1], d0 = w.off[i];
        const bool inv = mark[i] != 0;
        uint32_t d = d0;
        for (uint32_t q0 = s; q0 < e; q0 += 32) {
            const uint32_t q = q0 + lane;
            bool keep = false;
            if (q < e) {
                if (!inv) {
                    keep = true;
                } else {
                    const uint32_t other = o.a[q] == i ? o.b[q] : o.a[q];
                    keep = mark[other] == 0;
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, keep);
            if (keep) copy_entry(o, q, w, d + __popc(bal & ((1u << lane) - 1u)));
            d += __popc(bal);
        }
    }
}
__global__ void k_table_scatter_new(NewContacts nc, const uint32_t* __restrict__ nc_count, TableRef w,
                                    const uint32_t* __restrict__ keep_cnt, uint32_t* __restrict__ cursor,
                                    uint32_t* __restrict__ tmp_k) {
    const uint32_t m = *nc_count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const uint32_t a = nc.a[k], b = nc.b[k];
        tmp_k[w.off[a] + keep_cnt[a] + atomicAdd(&cursor[a], 1u)] = k;
        if (b != a) tmp_k[w.off[b] + keep_cnt[b] + atomicAdd(&cursor[b], 1u)] = k;
    }
}
// The new entries of ball i sit after its kept ones, in the order of their contact index
// (the order the reference pushes them, updateable.rs:503-509).
__global__ void __launch_bounds__(kWarps * 32)
    k_table_write_new(uint32_t n, NewContacts nc, TableRef w, const uint32_t* __restrict__ keep_cnt,
                      const uint32_t* __restrict__ new_cnt, const uint32_t* __restrict__ tmp_k,
                      uint32_t* __restrict__ err) {
    __shared__ uint32_t s_k[kWarps][kRankCap];
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    for (uint32_t i = blockIdx.x * kWarps + wp; i < n; i += gridDim.x * kWarps) {
        const uint32_t m = new_cnt[i];
        if (m == 0) continue;
        if (m > (uint32_t)kRankCap) {
            if (lane == 0) atomicOr(err, kErrTable);
            continue;
        }
        const uint32_t base = w.off[i] + keep_cnt[i];
        for (uint32_t t = lane; t < m; t += 32) s_k[wp][t] = tmp_k[base + t];
        __syncwarp();
        for (uint32_t t = lane; t < m; t += 32) {
            const uint32_t k = s_k[wp][t];
            uint32_t r = 0;
            for (uint32_t u = 0; u < m; ++u) r += s_k[wp][u] < k ? 1u : 0u;
            const uint32_t d = base + r;
            const bool own_a = nc.a[k] == i;
            w.a[d] = nc.a[k];
            w.b[d] = nc.b[k];
            w.area[d] = nc.area[k];
            w.arc[d] = nc.arc[k];
            w.sa[d] = own_a ? nc.sa_a[k] : nc.sa_b[k];
            w.pv[d] = own_a ? nc.pv_a[k] : nc.pv_b[k];
            w.flags[d] = (uint8_t)((nc.central[k] ? 1u : 0u) | (own_a ? 2u : 0u));
            if (w.gA) {
                w.gA[d] = own_a ? nc.gaa[k] : nc.gbb[k];
                w.gB[d] = own_a ? nc.gba[k] : nc.gab[k];
                w.vA[d] = own_a ? nc.vaa[k] : nc.vbb[k];
                w.vB[d] = own_a ? nc.vba[k] : nc.vab[k];
            }
        }
        __syncwarp();
    }
}
__global__ void __launch_bounds__(kWarps * 32)
    k_table_cells(const uint32_t* __restrict__ list, const uint32_t* __restrict__ count, TableRef T,
                  const double4* __restrict__ sph, const uint8_t* __restrict__ excl, uint8_t* __restrict__ cell_flag,
                  double* __restrict__ cell_sas, double* __restrict__ cell_vol, float cell_band,
                  uint8_t* __restrict__ unsure, int keep_empty) {
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    const uint32_t m = *count;
    for (uint32_t t = blockIdx.x * kWarps + wp; t < m; t += gridDim.x * kWarps) {
        const uint32_t i = list[t];
        const uint32_t s = T.off[i], e = T.off[i + 1];
        double arc = 0, spos = 0, sneg = 0, ppos = 0, pneg = 0;
        for (uint32_t q = s + lane; q < e; q += 32) {  // CellContactSummary::add (types.rs:589-609)
            const double sa = T.sa[q], pv = T.pv[q];
            arc += T.arc[q];
            spos += fmax(sa, 0.0);
            sneg -= fmin(sa, 0.0);
            ppos += fmax(pv, 0.0);
            pneg -= fmin(pv, 0.0);
        }
        arc = wsum(arc);
        spos = wsum(spos);
        sneg = wsum(sneg);
        ppos = wsum(ppos);
        pneg = wsum(pneg);
        if (lane == 0 && !(keep_empty && e == s)) {
            const uint32_t cnt = e - s;
            const double r = sph[i].w;
            uint8_t flag = 0;
            double sas = 0.0, vol = 0.0;
            bool uns = false;
            if (cnt > 0) {
                flag = 1;
                cell_from_sums(cnt, arc, spos, sneg, ppos, pneg, r, cell_band, &uns, &sas, &vol);
            } else if (!excl[i]) {  // compute_sas_detached (types.rs:666-675)
                flag = 1;
                sas = 4.0 * kPi * r * r;
                vol = sas * r / 3.0;
            }
            cell_flag[i] = flag;
            cell_sas[i] = sas;
            cell_vol[i] = vol;
            if (unsure) unsure[i] = uns ? 1 : 0;
        }
    }
}
__global__ void k_table_update(NewContacts nc, const uint32_t* __restrict__ nc_count, TableRef T,
                               uint32_t* __restrict__ err) {
    const uint32_t m = *nc_count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const uint32_t a = nc.a[k], b = nc.b[k];
        for (int side = 0; side < (a == b ? 1 : 2); ++side) {
            const uint32_t i = side ? b : a;
            const bool own_a = i == a;
            uint32_t d = T.off[i];
            const uint32_t e = T.off[i + 1];
            while (d < e && !(T.a[d] == a && T.b[d] == b)) ++d;
            if (d == e) {
                atomicOr(err, kErrRefresh);
                continue;
            }
            T.area[d] = nc.area[k];
            T.arc[d] = nc.arc[k];
            T.sa[d] = own_a ? nc.sa_a[k] : nc.sa_b[k];
            T.pv[d] = own_a ? nc.pv_a[k] : nc.pv_b[k];
            T.flags[d] = (uint8_t)((T.flags[d] & ~1u) | (nc.central[k] ? 1u : 0u));
            if (T.gA) {
                T.gA[d] = own_a ? nc.gaa[k] : nc.gbb[k];
                T.gB[d] = own_a ? nc.gba[k] : nc.gab[k];
                T.vA[d] = own_a ? nc.vaa[k] : nc.vbb[k];
                T.vB[d] = own_a ? nc.vba[k] : nc.vab[k];
            }
        }
    }
}
__global__ void k_list_flagged(const uint32_t* __restrict__ list, const uint32_t* __restrict__ count,
                               const uint8_t* __restrict__ flag, uint32_t* __restrict__ out,
                               uint32_t* __restrict__ d_out) {
    const uint32_t m = *count;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < m; t += gridDim.x * blockDim.x) {
        const uint32_t i = list[t];
        if (flag[i]) out[atomicAdd(d_out, 1u)] = i;
    }
}
// w == null: every SAS weight is `w_default` (1 for the total SAS, 0 for no SAS term)
__device__ __forceinline__ double sas_weight(const double* w, double w_default, const uint8_t* cell_flag,
                                             const double* cell_sas, uint32_t i) {
    return (cell_flag[i] && cell_sas[i] > 0.0) ? (w ? w[i] : w_default) : 0.0;
}
__device__ __forceinline__ double vol_weight(const double* v, const uint8_t* cell_flag, uint32_t i) {
    return (v && cell_flag[i]) ? v[i] : 0.0;
}
__global__ void __launch_bounds__(kWarps * 32)
    k_table_grad(uint32_t n, TableRef T, const double* __restrict__ w, double w_default, const double* __restrict__ v,
                 const uint8_t* __restrict__ cell_flag, const double* __restrict__ cell_sas,
                 const double4* __restrict__ sph, double* __restrict__ grad) {
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
    for (uint32_t i = blockIdx.x * kWarps + wp; i < n; i += gridDim.x * kWarps) {
        const double wi = sas_weight(w, w_default, cell_flag, cell_sas, i);
        const double vi = vol_weight(v, cell_flag, i);
        double gx = 0, gy = 0, gz = 0, gr = 0;
        for (uint32_t q = T.off[i] + lane; q < T.off[i + 1]; q += 32) {
            const uint32_t other = T.a[q] == i ? T.b[q] : T.a[q];
            const double wo = sas_weight(w, w_default, cell_flag, cell_sas, other);
            const double4 A = T.gA[q], B = T.gB[q];
            gx += wi * A.x + wo * B.x;
            gy += wi * A.y + wo * B.y;
            gz += wi * A.z + wo * B.z;
            gr += wi * A.w + wo * B.w;
            if (v) {
                const double vo = vol_weight(v, cell_flag, other);
                const double4 VA = T.vA[q], VB = T.vB[q];
                gx += vi * VA.x + vo * VB.x;
                gy += vi * VA.y + vo * VB.y;
                gz += vi * VA.z + vo * VB.z;
                gr += vi * VA.w + vo * VB.w;
            }
        }
        gx = wsum(gx);
        gy = wsum(gy);
        gz = wsum(gz);
        gr = wsum(gr);
        if (lane == 0) {
            // radius scaling of the exposed area: dSAS/dR = 2 SAS / R at fixed directions;
            // the exposed sphere's share of dV/dR is the exposed area itself
            if (wi != 0.0) gr += wi * 2.0 * cell_sas[i] / sph[i].w;
            if (vi != 0.0) gr += vi * cell_sas[i];
            grad[4 * (size_t)i] = gx;
            grad[4 * (size_t)i + 1] = gy;
            grad[4 * (size_t)i + 2] = gz;
            grad[4 * (size_t)i + 3] = gr;
        }
    }
}
__global__ void k_owner_flags(const uint8_t* __restrict__ flags, uint32_t M, uint32_t* __restrict__ out) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x)
        out[q] = (flags[q] & 2u) ? 1u : 0u;
}
__global__ void k_summary_contacts(TableRef T, uint32_t M, const uint32_t* __restrict__ off, uint32_t* __restrict__ a,
                                   uint32_t* __restrict__ b, double* __restrict__ area, double* __restrict__ arc,
                                   uint8_t* __restrict__ central) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < M; q += gridDim.x * blockDim.x) {
        const uint32_t o = off[q];
        if (off[q + 1] == o) continue;
        a[o] = T.a[q];
        b[o] = T.b[q];
        area[o] = T.area[q];
        arc[o] = T.arc[q];
        central[o] = T.flags[q] & 1u;
    }
}
__global__ void k_cell_flags_u32(const uint8_t* __restrict__ flag, uint32_t n, uint32_t* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = flag[i];
}
__global__ void k_summary_cells(const uint32_t* __restrict__ off, uint32_t n, const double* __restrict__ sas,
                                const double* __restrict__ vol, uint32_t* __restrict__ index,
                                double* __restrict__ osas, double* __restrict__ ovol) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t o = off[i];
        if (off[i + 1] == o) continue;
        index[o] = i;
        osas[o] = sas[i];
        ovol[o] = vol[i];
    }
}

int gb(size_t n) { return grid_blocks(n, kBlock, 148 * 16); }
int gw(size_t n) { return grid_blocks(n, kWarps, 148 * 32); }

}  // namespace

void launch_images_all(double4* sph, uint32_t n, const double* pbox9, cudaStream_t s) {
    PBoxArgF pb;
    for (int k = 0; k < 9; ++k) pb.v[k] = pbox9[k];
    k_images_all<<<gb((size_t)n * 26), kBlock, 0, s>>>(sph, n, pb); count_launch();
}
void launch_changed_flags(const uint64_t* ids, uint32_t k, const double* src, int src_by_id, uint32_t n,
                          double probe, const double* balls, uint32_t* flags, cudaStream_t s) {
    k_changed_flags<<<gb(k), kBlock, 0, s>>>(ids, k, src, src_by_id, n, probe, balls, flags); count_launch();
}
void launch_changed_compact(const uint64_t* ids, uint32_t k, const double* src, int src_by_id, const uint32_t* off,
                            uint32_t* changed, double4* changed_ball, cudaStream_t s) {
    k_changed_compact<<<gb(k), kBlock, 0, s>>>(ids, k, src, src_by_id, off, changed, changed_ball); count_launch();
}
void launch_clamp_count(uint32_t* count, uint32_t cap, cudaStream_t s) {
    k_clamp_count<<<1, 32, 0, s>>>(count, cap); count_launch();
}
void launch_apply_changed(const uint32_t* changed, const double4* cb, const uint32_t* count, uint32_t max_count,
                          double* balls, cudaStream_t s) {
    k_apply_changed<<<gb(max_count), kBlock, 0, s>>>(changed, cb, count, balls); count_launch();
}
void launch_mark_list(const uint32_t* list, const uint32_t* count, uint32_t max_count, uint32_t* mark, uint32_t val,
                      uint32_t* d_new, cudaStream_t s) {
    k_mark_list<<<gb(max_count), kBlock, 0, s>>>(list, count, mark, val, d_new); count_launch();
}
void launch_mark_neighbours(const uint32_t* list, const uint32_t* count, uint32_t max_count, const uint32_t* row_of,
                            ListsRef lists, uint32_t n, uint32_t* mark, uint32_t val, uint32_t* d_new,
                            uint32_t* append, cudaStream_t s) {
    k_mark_neighbours<<<gw(max_count), kWarps * 32, 0, s>>>(list, count, row_of, lists, n, mark, val, d_new, append);
    count_launch();
}
void launch_mark_table_partners(uint32_t id, TableRef tab, uint32_t* mark, cudaStream_t s) {
    k_mark_table_partners<<<1, kBlock, 0, s>>>(id, tab, mark); count_launch();
}
void launch_nonzero(const uint32_t* mark, uint32_t n, uint32_t* flags, cudaStream_t s) {
    k_nonzero<<<gb(n), kBlock, 0, s>>>(mark, n, flags); count_launch();
}
void launch_compact_index(const uint32_t* off, uint32_t n, uint32_t* list, cudaStream_t s) {
    k_compact_index<<<gb(n), kBlock, 0, s>>>(off, n, list); count_launch();
}
void launch_row_of(const uint32_t* list, const uint32_t* count, uint32_t max_count, uint32_t* row_of,
                   cudaStream_t s) {
    k_row_of<<<gb(max_count), kBlock, 0, s>>>(list, count, row_of); count_launch();
}
void launch_splice_counts(uint32_t n, const uint32_t* mark, const uint32_t* row_of, const uint32_t* old_cnt,
                          const uint32_t* c1, const uint32_t* c2, uint32_t* cnt, cudaStream_t s) {
    k_splice_counts<<<gb(n), kBlock, 0, s>>>(n, mark, row_of, old_cnt, c1, c2, cnt); count_launch();
}
void launch_splice_lists(uint32_t n, const uint32_t* mark, const uint32_t* row_of, ListsRef old, ListsRef t1,
                         ListsRef t2, const uint32_t* new_off, uint32_t* id, double* val, float4* rel,
                         cudaStream_t s) {
    k_splice_lists<<<gw(n), kWarps * 32, 0, s>>>(n, mark, row_of, old, t1, t2, new_off, id, val, rel);
    count_launch();
}
void launch_upd_pairs(int fill, const uint32_t* list, const uint32_t* count, uint32_t max_count, uint32_t n,
                      int periodic, ListsRef lists, const uint8_t* excl, const uint32_t* mark, uint32_t need,
                      uint32_t* npair, const uint32_t* pair_off, uint32_t* pair_a, uint32_t* pair_e,
                      int32_t* nb_pair, cudaStream_t s) {
    const uint32_t m = list ? max_count : n;
    if (fill)
        k_upd_pairs<true><<<gw(m), kWarps * 32, 0, s>>>(list, count, n, periodic, lists, excl, mark, need, npair,
                                                        pair_off, pair_a, pair_e, nb_pair);
    else
        k_upd_pairs<false><<<gw(m), kWarps * 32, 0, s>>>(list, count, n, periodic, lists, excl, mark, need, npair,
                                                         pair_off, pair_a, pair_e, nb_pair);
    count_launch();
}
void launch_new_contacts(uint32_t P, const uint32_t* keep_off, const DevBufs& b, NewContacts nc, cudaStream_t s) {
    k_new_contacts<<<gb(P), kBlock, 0, s>>>(P, keep_off, b, nc); count_launch();
}
void launch_table_counts(uint32_t n, const uint32_t* mark, TableRef old, uint32_t* keep_cnt, cudaStream_t s) {
    k_table_counts<<<gb(n), kBlock, 0, s>>>(n, mark, old, keep_cnt); count_launch();
}
void launch_table_new_counts(const NewContacts& nc, const uint32_t* nc_count, uint32_t max_nc, uint32_t* new_cnt,
                             cudaStream_t s) {
    k_table_new_counts<<<gb(max_nc), kBlock, 0, s>>>(nc, nc_count, new_cnt); count_launch();
}
void launch_add_u32(const uint32_t* x, const uint32_t* y, uint32_t n, uint32_t* out, cudaStream_t s) {
    k_add_u32<<<gb(n), kBlock, 0, s>>>(x, y, n, out); count_launch();
}
void launch_table_copy_kept(uint32_t n, const uint32_t* mark, TableRef old, TableRef nw, cudaStream_t s) {
    k_table_copy_kept<<<gw(n), kWarps * 32, 0, s>>>(n, mark, old, nw); count_launch();
}
void launch_table_scatter_new(const NewContacts& nc, const uint32_t* nc_count, uint32_t max_nc, TableRef nw,
                              const uint32_t* keep_cnt, uint32_t* cursor, uint32_t* tmp_k, cudaStream_t s) {
    k_table_scatter_new<<<gb(max_nc), kBlock, 0, s>>>(nc, nc_count, nw, keep_cnt, cursor, tmp_k); count_launch();
}
void launch_table_write_new(uint32_t n, const NewContacts& nc, TableRef nw, const uint32_t* keep_cnt,
                            const uint32_t* new_cnt, const uint32_t* tmp_k, uint32_t* err, cudaStream_t s) {
    k_table_write_new<<<gw(n), kWarps * 32, 0, s>>>(n, nc, nw, keep_cnt, new_cnt, tmp_k, err); count_launch();
}
void launch_table_cells(const uint32_t* list, const uint32_t* count, uint32_t max_count, TableRef tab,
                        const double4* sph, const uint8_t* excl, uint8_t* cell_flag, double* cell_sas,
                        double* cell_vol, float cell_band, uint8_t* unsure, cudaStream_t s, int keep_empty) {
    k_table_cells<<<gw(max_count), kWarps * 32, 0, s>>>(list, count, tab, sph, excl, cell_flag, cell_sas, cell_vol,
                                                        cell_band, unsure, keep_empty);
    count_launch();
}
void launch_table_update(const NewContacts& nc, const uint32_t* nc_count, uint32_t max_nc, TableRef tab,
                         uint32_t* err, cudaStream_t s) {
    k_table_update<<<gb(max_nc), kBlock, 0, s>>>(nc, nc_count, tab, err); count_launch();
}
void launch_list_flagged(const uint32_t* list, const uint32_t* count, uint32_t max_count, const uint8_t* flag,
                         uint32_t* out, uint32_t* d_out, cudaStream_t s) {
    k_list_flagged<<<gb(max_count), kBlock, 0, s>>>(list, count, flag, out, d_out); count_launch();
}
void launch_table_grad(uint32_t n, TableRef tab, const double* w, double w_default, const double* v,
                       const uint8_t* cell_flag, const double* cell_sas,
                       const double4* sph, double* grad, cudaStream_t s) {
    k_table_grad<<<gw(n), kWarps * 32, 0, s>>>(n, tab, w, w_default, v, cell_flag, cell_sas, sph, grad);
    count_launch();
}
void launch_owner_flags(const uint8_t* flags, uint32_t M, uint32_t* out, cudaStream_t s) {
    k_owner_flags<<<gb(M), kBlock, 0, s>>>(flags, M, out); count_launch();
}
void launch_summary_contacts(TableRef tab, uint32_t M, const uint32_t* off, uint32_t* a, uint32_t* b, double* area,
                             double* arc, uint8_t* central, cudaStream_t s) {
    k_summary_contacts<<<gb(M), kBlock, 0, s>>>(tab, M, off, a, b, area, arc, central); count_launch();
}
void launch_cell_flags_u32(const uint8_t* flag, uint32_t n, uint32_t* out, cudaStream_t s) {
    k_cell_flags_u32<<<gb(n), kBlock, 0, s>>>(flag, n, out); count_launch();
}
void launch_summary_cells(const uint32_t* off, uint32_t n, const double* sas, const double* vol, uint32_t* index,
                          double* osas, double* ovol, cudaStream_t s) {
    k_summary_cells<<<gb(n), kBlock, 0, s>>>(off, n, sas, vol, index, osas, ovol); count_launch();
}

}  // namespace vt
