// vt_noalloc.cu -- contact descriptors without any device allocation.
//
// Who needs this: callers that must not call cudaMalloc/cudaFree once they are running --
// a custom call inside another framework whose allocator owns the whole device (XLA-style
// runtimes that pre-reserve most of HBM and forbid foreign allocations), real-time loops
// that cannot risk the allocator's synchronisation and latency spikes, and plugin hosts
// that only hand out pre-allocated buffers.  The regular engine grows a cudaMalloc'd
// workspace on demand; this entry point instead runs the serial contour kernel
// (construct_contact_descriptor, one thread per pair) with its contour scratch in a
// file-scope __device__ array that exists for the life of the process on every GPU that
// loads the library.
//
// Limits: 1024 resident threads, each with room for 192 contour points.  The contour
// starts as the 7-point hexagon at the first cutting neighbour and each cut adds at most
// one point (a single outside point becomes two; a run of outside points collapses to
// two), so after the cuts a pair whose `a` lists at most 57 neighbours holds at most
// 7 + 56 = 63 points.  The restriction to the circle keeps the outside points while it
// inserts up to two points per edge, so its peak is 3 x 63 = 189 <= 192 points.  Longer
// neighbour lists are rejected before any work with VT_ERR_CAPACITY; a contour that still
// outgrew its slot would make the call return VT_ERR_CAPACITY as well (error bit 4).
// Malformed input (a pair or neighbour index not below num_spheres, offsets that are not
// ascending, a non-finite coordinate or a negative radius among the spheres a pair
// reads) is rejected with VT_ERR_INVALID before the contact kernel runs, as the regular
// path rejects it.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/voronota_b200.h"
#include "vt_geom.cuh"

namespace vt {
// message for vt_last_error() (defined with the engine in vt_engine.cu)
void set_last_error(const std::string& msg);
}  // namespace vt

namespace {

using namespace vt;

constexpr int kSlots = 1024;  // threads launched, one contour slot each
constexpr int kCap = 192;     // contour points per slot
constexpr int kMaxNeighbors = 57;
static_assert(3 * (7 + kMaxNeighbors - 1) <= kCap, "the peak contour of a 57-neighbour list must fit a slot");
static_assert(kMaxNeighbors == VT_NOALLOC_MAX_NEIGHBORS, "header and kernel disagree");

// bits of the error word (scratch word 0)
constexpr uint32_t kNaCapacity = 1u;  // a listed a has more than kMaxNeighbors neighbours
constexpr uint32_t kNaIndex = 2u;     // a pair / neighbour index or the offsets are malformed
constexpr uint32_t kNaOverflow = 4u;  // a contour outgrew its slot (not expected within the limit)
constexpr uint32_t kNaValue = 8u;     // a non-finite coordinate or a negative radius

struct NP {  // one contour point (contact.rs:36-47)
    double x, y, z, ang;
    uint32_t lid, rid;
    int state;  // 0 inside, 1 outside
    int pad;
};
static_assert(sizeof(NP) == 48, "contour point layout");

constexpr size_t kCtrlBytes = 256;  // word 0: error flag
constexpr size_t kScratchBytes = kCtrlBytes + (size_t)kSlots * kCap * sizeof(NP);
static_assert(kScratchBytes == VT_NOALLOC_SCRATCH_BYTES, "header and kernel disagree");

// The scratch itself (9,437,440 bytes per device).  Host code must not use this name as
// an address: it is a host-side shadow; the device address comes from
// cudaGetSymbolAddress at set-up.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
constexpr int kMaxDevices = 64;
void* g_scratch_ptr[kMaxDevices] = {};

struct In {
    const double* sph;
    const uint32_t* off;
    const uint32_t* nbi;
    const uint32_t* pa;
    const uint32_t* pb;
    uint32_t np, ns;
};

__device__ __forceinline__ Sph<double> sphere(const In& in, uint32_t i) {
    const double* s = in.sph + 4 * (size_t)i;
    return {{s[0], s[1], s[2]}, s[3]};
}

struct Contour {
    NP* v;
    int n;
    bool overflow;
    __device__ void insert(int at, const NP& s) {
        if (n >= kCap) {
            overflow = true;
            return;
        }
        for (int k = n; k > at; --k) v[k] = v[k - 1];
        v[at] = s;
        ++n;
    }
    __device__ void erase(int from, int to) {
        int d = to - from;
        if (d <= 0) return;
        for (int k = from; k + d < n; ++k) v[k] = v[k + d];
        n -= d;
    }
};
__device__ __forceinline__ V3<double> P3(const NP& s) { return {s.x, s.y, s.z}; }
__device__ __forceinline__ NP mkp(V3<double> p, uint32_t l, uint32_t r) {
    NP s;
    s.x = p.x;
    s.y = p.y;
    s.z = p.z;
    s.ang = 0.0;
    s.lid = l;
    s.rid = r;
    s.state = 0;
    s.pad = 0;
    return s;
}

__constant__ double c_ns_sin[8];
__constant__ double c_ns_cos[8];
__constant__ int c_ns_n[1];

// clip_contact (contact.rs:196-341) for pair (a, b) with a's sorted neighbour list.
__device__ bool clip(const In& in, uint32_t a, uint32_t b, Contour& c, Sph<double>& ic, V3<double>& bary,
                     double& sum_arc, double& area) {
    Dec<double, false> d;
    const Sph<double> A = sphere(in, a), B = sphere(in, b);
    if (!sphere_intersects(d, A, B, 0.0) || sphere_contains(d, A, B, 0.0, 0.0) || sphere_contains(d, B, A, 0.0, 0.0))
        return false;
    ic = intersection_circle(A, B);
    V3<double> axis = normalize(B.c - A.c);
    if (ic.r <= 0.0) return false;
    c.n = 0;
    bool init = false;
    for (uint32_t e = in.off[a]; e < in.off[a + 1]; ++e) {
        uint32_t nid = in.nbi[e];
        if (nid == b) continue;
        Sph<double> C = sphere(in, nid);
        if (!sphere_intersects(d, ic, C, 0.0) || !sphere_intersects(d, B, C, 0.0)) continue;
        if (sphere_contains(d, C, A, 0.0, 0.0) || sphere_contains(d, C, B, 0.0, 0.0)) return false;
        V3<double> pc = ic_center(A, C);
        V3<double> pn = normalize(C.c - A.c);
        double cos_val = dot(normalize(ic.c - A.c), normalize(pc - A.c));
        if (fabs(cos_val) >= 1.0) {
            if (halfspace(d, pc, pn, ic.c, 0.0) > 0) return false;
            continue;
        }
        double l = fabs(sd_plane_unit(pc, pn, ic.c));
        double xl = l / sqrt(fma(cos_val, -cos_val, 1.0));
        if (xl >= ic.r) {
            if (halfspace(d, pc, pn, ic.c, 0.0) >= 0) return false;
            continue;
        }
        if (!init) {
            V3<double> first = any_normal(axis) * ic.r * kHexScale;
            c.n = 0;
            c.v[c.n++] = mkp(ic.c + first, a, a);
            for (int k = 1; k < c_ns_n[0]; ++k)
                c.insert(c.n, mkp(ic.c + rotate_around_axis(axis, c_ns_sin[k], c_ns_cos[k], first), a, a));
            init = true;
        } else {
            double thr = norm2(pc - A.c);
            bool any = false;
            for (int k = 0; k < c.n && !any; ++k) any = norm2(P3(c.v[k]) - A.c) >= thr;
            if (!any) continue;
        }
        int outs = 0;
        for (int k = 0; k < c.n; ++k)
            if (halfspace(d, pc, pn, P3(c.v[k]), 0.0) >= 0) {
                c.v[k].lid = c.v[k].rid = nid;
                ++outs;
            }
        if (outs == 0) continue;
        if (outs >= c.n) return false;
        if (c.n < 3) continue;
        auto is_out = [&](int k) { return c.v[k].lid == nid && c.v[k].rid == nid; };
        int start = 0, end = c.n - 1;
        while (start < c.n && !is_out(start)) ++start;
        while (end >= 0 && !is_out(end)) --end;
        if (start == 0 && end == c.n - 1) {
            end = 0;
            while (end + 1 < c.n && is_out(end + 1)) ++end;
            start = c.n - 1;
            while (start > 0 && is_out(start - 1)) --start;
        }
        if (start == end) {
            NP cp = c.v[start];
            c.insert(start, cp);
            end = start + 1;
        } else if (start < end) {
            if (start + 1 < end) c.erase(start + 1, end);
            end = start + 1;
        } else {
            if (start + 1 < c.n) c.erase(start + 1, c.n);
            if (end > 0) c.erase(0, end);
            start = c.n - 1;
            end = 0;
        }
        if (c.overflow) return false;
        int nn = c.n;
        int il = start > 0 ? start - 1 : nn - 1;
        V3<double> lip = plane_segment(d, pc, pn, P3(c.v[start]), P3(c.v[il]), 0.0);
        NP nsp = mkp(lip, c.v[il].rid, c.v[start].lid);
        c.v[start] = nsp;
        int ir = end + 1 < nn ? end + 1 : 0;
        V3<double> rip = plane_segment(d, pc, pn, P3(c.v[end]), P3(c.v[ir]), 0.0);
        NP nep = mkp(rip, c.v[end].rid, c.v[ir].lid);
        c.v[end] = nep;
        if (!(norm2(P3(c.v[end]) - P3(c.v[start])) - kEps > 0.0)) {
            c.v[start].rid = c.v[end].rid;
            c.erase(end, end + 1);
        }
    }
    sum_arc = 0.0;
    area = 0.0;
    if (!init) {
        bary = ic.c;
        sum_arc = kTau;
        area = ic.r * ic.r * kPi;
        c.n = 0;
        return area > 0.0;
    }
    // restrict_contour_to_circle (contact.rs:631-769)
    int outsiders = 0;
    for (int k = 0; k < c.n; ++k) {
        bool inside = norm2(P3(c.v[k]) - ic.c) <= ic.r * ic.r;
        c.v[k].state = inside ? 0 : 1;
        outsiders += inside ? 0 : 1;
    }
    if (outsiders > 0) {
        int insertions = 0;
        int i = 0;
        while (i < c.n) {
            int ni = (i + 1) % c.n;
            int s1 = c.v[i].state, s2 = c.v[ni].state;
            if (s1 == 1 || s2 == 1) {
                V3<double> ip, mp, ip1, ip2;
                if (s1 == 1 && s2 == 1) {
                    if (project_inside_line(d, ic.c, P3(c.v[i]), P3(c.v[ni]), &mp, 0.0, 0.0) &&
                        norm2(mp - ic.c) <= ic.r * ic.r) {
                        bool ok1 = segment_circle(d, ic, mp, P3(c.v[i]), &ip1, 0.0, 0.0);
                        bool ok2 = segment_circle(d, ic, mp, P3(c.v[ni]), &ip2, 0.0, 0.0);
                        if (ok1 && ok2) {
                            uint32_t rid = c.v[i].rid, lid = c.v[ni].lid;
                            c.insert(i + 1, mkp(ip1, a, rid));
                            c.insert(i + 2, mkp(ip2, lid, a));
                            insertions += 2;
                            i += 2;
                        }
                    }
                } else if (s1 == 1) {
                    if (segment_circle(d, ic, P3(c.v[ni]), P3(c.v[i]), &ip, 0.0, 0.0)) {
                        uint32_t rid = c.v[i].rid;
                        c.insert(i + 1, mkp(ip, a, rid));
                        insertions += 1;
                        i += 1;
                    } else {
                        c.v[ni].lid = a;
                        c.v[ni].rid = c.v[i].rid;
                    }
                } else {
                    if (segment_circle(d, ic, P3(c.v[i]), P3(c.v[ni]), &ip, 0.0, 0.0)) {
                        uint32_t lid = c.v[ni].lid;
                        c.insert(i + 1, mkp(ip, lid, a));
                        insertions += 1;
                        i += 1;
                    } else {
                        c.v[i].lid = c.v[ni].lid;
                        c.v[i].rid = a;
                    }
                }
                if (c.overflow) return false;
            }
            i += 1;
        }
        if (insertions == 0) return false;
        int m = 0;
        for (int k = 0; k < c.n; ++k)
            if (c.v[k].state != 1) c.v[m++] = c.v[k];
        c.n = m;
        if (c.n < 2) return false;
        for (int k = 0; k < c.n; ++k) {
            int nk = (k + 1) % c.n;
            if (c.v[k].rid == a && c.v[nk].lid == a) {
                double ang = directed_angle(d, ic.c, P3(c.v[k]), P3(c.v[nk]), ic.c + axis, 0.0);
                c.v[k].ang = ang;
                sum_arc += ang;
            }
        }
        if (sum_arc + kEps > kTau || (c.n > 2 && fabs(sum_arc - kTau) <= kEps)) return false;
    }
    // calculate_contour_area (contact.rs:773-793)
    V3<double> s = mk<double>(0, 0, 0);
    for (int k = 0; k < c.n; ++k) s = s + P3(c.v[k]);
    bary = s / (double)c.n;
    for (int k = 0; k < c.n; ++k) {
        int nk = (k + 1) % c.n;
        area += triangle_area(bary, P3(c.v[k]), P3(c.v[nk]));
        if (c.v[k].ang > 0.0) area += ic.r * ic.r * (c.v[k].ang - sin(c.v[k].ang)) * 0.5;
    }
    return area > 0.0;
}

// calculate_solid_angle (contact.rs:797-848)
__device__ double solid(const Sph<double>& a, const Sph<double>& b, const Sph<double>& ic, const Contour& c) {
    double turn = 0.0;
    if (c.n == 0) {
        turn = kTau * norm(ic.c - a.c) / a.r;
    } else {
        for (int i = 0; i < c.n; ++i) {
            const NP& p0 = c.v[i > 0 ? i - 1 : c.n - 1];
            const NP& p1 = c.v[i];
            const NP& p2 = c.v[(i + 1) % c.n];
            if (p0.ang > 0.0) {
                V3<double> dd = cross(b.c - a.c, P3(p1) - ic.c);
                double dv = dot(dd, P3(p0) - P3(p1));
                if ((p0.ang < kPi && dv < 0.0) || (p0.ang > kPi && dv > 0.0)) dd = -dd;
                turn += kPi - min_dihedral(a.c, P3(p1), P3(p1) + dd, P3(p2));
            } else if (p1.ang > 0.0) {
                V3<double> dd = cross(b.c - a.c, P3(p1) - ic.c);
                double dv = dot(dd, P3(p2) - P3(p1));
                if ((p1.ang < kPi && dv < 0.0) || (p1.ang > kPi && dv > 0.0)) dd = -dd;
                turn += kPi - min_dihedral(a.c, P3(p1), P3(p0), P3(p1) + dd);
                turn += p1.ang * (norm(ic.c - a.c) / a.r);
            } else {
                turn += kPi - min_dihedral(a.c, P3(p1), P3(p0), P3(p2));
            }
        }
    }
    double sa = kTau - turn;
    if (dot(ic.c - a.c, ic.c - b.c) > 0.0 && norm2(a.c - ic.c) < norm2(b.c - ic.c)) sa = -sa;
    return sa;
}

// contour_is_central (contact.rs:411-444)
__device__ bool central(V3<double> center, const Contour& c, V3<double> bary) {
    for (int k = 0; k < c.n; ++k)
        if (c.v[k].ang - 1e-10 > kPi) return true;
    for (int i = 0; i < c.n; ++i) {
        V3<double> pi = P3(c.v[i]), pj = P3(c.v[(i + 1) % c.n]);
        V3<double> edge = pj - pi;
        double len = norm(edge);
        if (len < 1e-10) continue;
        V3<double> u = edge / len;
        V3<double> foot = pi + u * dot(u, bary - pi);
        if (dot(bary - foot, center - pi) < 0.0) return false;
    }
    return true;
}

__device__ __forceinline__ bool sphere_ok(const In& in, uint32_t i) {
    const double* s = in.sph + 4 * (size_t)i;
    return isfinite(s[0]) && isfinite(s[1]) && isfinite(s[2]) && isfinite(s[3]) && s[3] >= 0.0;
}

// Every read the contact kernel will make, checked first: the pair's ids, a's offsets
// (ascending and within the index array, whose length is off[num_spheres]), a's
// neighbour ids, and the spheres of a, b and the neighbours.
__global__ void k_check_lists(In in, unsigned char* scratch) {
    uint32_t* err = reinterpret_cast<uint32_t*>(scratch);
    const uint32_t total = in.off[in.ns];
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < in.np; p += gridDim.x * blockDim.x) {
        const uint32_t a = in.pa[p], b = in.pb[p];
        if (a >= in.ns || b >= in.ns) {
            atomicOr(err, kNaIndex);
            continue;
        }
        const uint32_t lo = in.off[a], hi = in.off[a + 1];
        if (lo > hi || hi > total) {
            atomicOr(err, kNaIndex);
            continue;
        }
        if (hi - lo > (uint32_t)kMaxNeighbors) {
            atomicOr(err, kNaCapacity);
            continue;
        }
        uint32_t bits = 0;
        if (!sphere_ok(in, a) || !sphere_ok(in, b)) bits |= kNaValue;
        for (uint32_t e = lo; e < hi; ++e) {
            const uint32_t c = in.nbi[e];
            if (c >= in.ns) {
                bits |= kNaIndex;
                break;
            }
            if (!sphere_ok(in, c)) bits |= kNaValue;
        }
        if (bits) atomicOr(err, bits);
    }
}

__global__ void __launch_bounds__(128) k_contact_noalloc(In in, unsigned char* scratch, uint8_t* st, double* area,
                                                         double* arc, uint8_t* cen, double* sa, double* sb,
                                                         double* pa, double* pb) {
    const uint32_t slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= (uint32_t)kSlots) return;
    NP* mine = reinterpret_cast<NP*>(scratch + kCtrlBytes) + (size_t)slot * kCap;
    for (uint32_t p = slot; p < in.np; p += kSlots) {
        const uint32_t a = in.pa[p], b = in.pb[p];
        Contour c;
        c.v = mine;
        c.n = 0;
        c.overflow = false;
        Sph<double> ic;
        V3<double> bary;
        double sum_arc = 0.0, ar = 0.0;
        bool ok = clip(in, a, b, c, ic, bary, sum_arc, ar) && !c.overflow;
        if (c.overflow) atomicOr(reinterpret_cast<uint32_t*>(scratch), kNaOverflow);
        st[p] = ok ? 1 : 0;
        area[p] = ok ? ar : 0.0;
        arc[p] = ok ? sum_arc * ic.r : 0.0;
        cen[p] = ok && central(ic.c, c, bary) ? 1 : 0;
        if (sa) {
            double s_a = 0.0, s_b = 0.0, v_a = 0.0, v_b = 0.0;
            if (ok) {
                const Sph<double> A = sphere(in, a), B = sphere(in, b);
                s_a = solid(A, B, ic, c);
                s_b = solid(B, A, ic, c);
                v_a = norm(ic.c - A.c) * ar / 3.0 * (s_a < 0.0 ? -1.0 : 1.0);
                v_b = norm(ic.c - B.c) * ar / 3.0 * (s_b < 0.0 ? -1.0 : 1.0);
            }
            sa[p] = s_a;
            sb[p] = s_b;
            pa[p] = v_a;
            pb[p] = v_b;
        }
    }
}

// Per-device set-up: the scratch's device address and the hexagon rotation table (the
// sin/cos of the reference's accumulated half angles, from the host C library).
int setup_current_device(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        vt::set_last_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        return VT_ERR_NO_DEVICE;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        vt::set_last_error("device index out of range");
        return VT_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr) {
            vt::set_last_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return VT_ERR_CUDA;
        }
        double hs[8] = {0}, hc[8] = {0};
        int k = 1;
        for (double ang = kFracPi3; ang < kTau && k < 8; ang += kFracPi3, ++k) {
            hs[k] = std::sin(ang / 2.0);
            hc[k] = std::cos(ang / 2.0);
        }
        if (cudaMemcpyToSymbol(c_ns_sin, hs, sizeof(hs)) != cudaSuccess ||
            cudaMemcpyToSymbol(c_ns_cos, hc, sizeof(hc)) != cudaSuccess ||
            cudaMemcpyToSymbol(c_ns_n, &k, sizeof(int)) != cudaSuccess) {
            vt::set_last_error("uploading the hexagon table failed");
            return VT_ERR_CUDA;
        }
        g_scratch_ptr[dev] = ptr;
    }
    *out = g_scratch_ptr[dev];
    return VT_OK;
}

}  // namespace

extern "C" int vt_contact_descriptors_noalloc(const double* d_spheres, uint64_t num_spheres,
                                              const uint32_t* d_nb_offsets, const uint32_t* d_nb_index,
                                              const uint32_t* d_pair_a, const uint32_t* d_pair_b,
                                              uint64_t num_pairs, uint8_t* d_status, double* d_area,
                                              double* d_arc_length, uint8_t* d_central, double* d_solid_a,
                                              double* d_solid_b, double* d_pyramid_a, double* d_pyramid_b,
                                              void* stream) {
    if (num_spheres >= 0xffffffffull || num_pairs >= 0xffffffffull) {
        vt::set_last_error("num_spheres and num_pairs must be below 2^32");
        return VT_ERR_INVALID;
    }
    if (num_pairs == 0) return VT_OK;
    if (!d_spheres || !d_nb_offsets || !d_nb_index || !d_pair_a || !d_pair_b || !d_status || !d_area ||
        !d_arc_length || !d_central) {
        vt::set_last_error("null pointer argument");
        return VT_ERR_INVALID;
    }
    const bool full = d_solid_a != nullptr;
    if (full && (!d_solid_b || !d_pyramid_a || !d_pyramid_b)) {
        vt::set_last_error("solid angle / pyramid volume outputs must be all given or all NULL");
        return VT_ERR_INVALID;
    }
    void* ptr = nullptr;
    int st = setup_current_device(&ptr);
    if (st != VT_OK) return st;
    unsigned char* scratch = static_cast<unsigned char*>(ptr);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    In in{d_spheres, d_nb_offsets, d_nb_index, d_pair_a, d_pair_b, (uint32_t)num_pairs, (uint32_t)num_spheres};
    // the error word must start at zero on every call; the contour slots are written
    // before they are read
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(uint32_t), s);
    k_check_lists<<<64, 256, 0, s>>>(in, scratch);
    uint32_t h_err = 0;
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, scratch, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        vt::set_last_error(std::string("CUDA: ") + cudaGetErrorString(e));
        return VT_ERR_CUDA;
    }
    if (h_err & kNaIndex) {
        vt::set_last_error("a pair or neighbour index is not below num_spheres, or the neighbour offsets are not "
                           "ascending within the index array");
        return VT_ERR_INVALID;
    }
    if (h_err & kNaValue) {
        vt::set_last_error("a sphere read by a pair has a non-finite coordinate or a negative radius");
        return VT_ERR_INVALID;
    }
    if (h_err & kNaCapacity) {
        vt::set_last_error("a neighbour list has more than 57 entries; the no-allocation scratch holds 192 contour "
                "points per pair (use vt_compute_tessellation for such inputs)");
        return VT_ERR_CAPACITY;
    }
    k_contact_noalloc<<<kSlots / 128, 128, 0, s>>>(in, scratch, d_status, d_area, d_arc_length, d_central,
                                                   d_solid_a, d_solid_b, d_pyramid_a, d_pyramid_b);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h_err, scratch, sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        vt::set_last_error(std::string("CUDA: ") + cudaGetErrorString(e));
        return VT_ERR_CUDA;
    }
    if (h_err & kNaOverflow) {
        vt::set_last_error("a contour outgrew the 192 points of its scratch slot; its contact is not computed");
        return VT_ERR_CAPACITY;
    }
    return VT_OK;
}

