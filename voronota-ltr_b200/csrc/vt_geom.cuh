// vt_geom.cuh -- device geometry for the radical-tessellation kernels.
//
// Scalar-generic (T = double for the exact path, T = float for the FP32 bulk path).
// The FP64 instantiation follows the reference arithmetic operation by operation
// (src/geometry.rs; `mul_add` -> fma, everything else uncontracted: the FP64
// translation units are compiled with --fmad=false) so that its decisions equal the
// CPU oracle's.  The FP32 instantiation works in coordinates relative to ball `a`,
// uses atan2-based angles (well conditioned near 0 and pi where acos is not) and
// records every fuzzy decision whose margin is inside an error band in `Dec::unsure`;
// such pairs are recomputed by the FP64 kernel.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace vt {

constexpr double kEps = 1e-10;  // geometry.rs:17 EPSILON
constexpr double kPi = 3.14159265358979323846;
constexpr double kTau = 6.28318530717958647692;
constexpr double kFracPi3 = 1.04719755119659774615;
constexpr double kHexScale = 1.19;  // contact.rs:448 HEXAGON_SCALE

template <typename T>
struct V3 {
    T x, y, z;
};
template <typename T>
__device__ __forceinline__ V3<T> mk(T x, T y, T z) {
    return {x, y, z};
}
template <typename T>
__device__ __forceinline__ V3<T> operator+(V3<T> a, V3<T> b) {
    return {a.x + b.x, a.y + b.y, a.z + b.z};
}
template <typename T>
__device__ __forceinline__ V3<T> operator-(V3<T> a, V3<T> b) {
    return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <typename T>
__device__ __forceinline__ V3<T> operator-(V3<T> a) {
    return {-a.x, -a.y, -a.z};
}
template <typename T>
__device__ __forceinline__ V3<T> operator*(V3<T> a, T s) {
    return {a.x * s, a.y * s, a.z * s};
}
template <typename T>
__device__ __forceinline__ V3<T> operator/(V3<T> a, T s) {
    return {a.x / s, a.y / s, a.z / s};
}
// nalgebra Vector3 dot: (x*x' + y*y') + z*z'
template <typename T>
__device__ __forceinline__ T dot(V3<T> a, V3<T> b) {
    return (a.x * b.x + a.y * b.y) + a.z * b.z;
}
template <typename T>
__device__ __forceinline__ T norm2(V3<T> a) {
    return dot(a, a);
}
template <typename T>
__device__ __forceinline__ T norm(V3<T> a) {
    return sqrt(norm2(a));
}
template <typename T>
__device__ __forceinline__ V3<T> normalize(V3<T> a) {
    return a / norm(a);
}
#ifndef VT_FP32_UNIT
// FP64: normalize out of line (one copy).  Inlined at each of its call sites (a square root
// and three divisions, with their slow paths, at about fifteen places) the FP64 contour's
// code outgrew the instruction cache: the FP64 contact kernel stalled on instruction fetch
// (5.6 cycles per issued instruction) and took 16.7 ms at the 100k lattice, 12.0 ms with
// this copy.  The FP32 contact unit, whose double code is on its hot path, keeps it inline.
static __device__ __noinline__ V3<double> normalize(V3<double> a) { return a / norm(a); }
#endif
template <typename T>
__device__ __forceinline__ V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

template <typename T>
struct Sph {
    V3<T> c;
    T r;
};

// ---- fuzzy decisions (geometry.rs:22-54) with an uncertainty band for FP32 ----
// Each test returns the reference's boolean; when FLAG is set and the margin to the
// threshold is within `tol`, the decision is recorded as unsure.
template <typename T, bool FLAG>
struct Dec {
    bool unsure = false;
    __device__ __forceinline__ void band(T margin, T tol) {
        if (FLAG && fabs(margin) <= tol) unsure = true;
    }
    // a + EPS < b
    __device__ __forceinline__ bool lt(T a, T b, T tol) {
        band(b - a, tol);
        return a + (T)kEps < b;
    }
    // a - EPS > b
    __device__ __forceinline__ bool gt(T a, T b, T tol) {
        band(a - b, tol);
        return a - (T)kEps > b;
    }
    // a < b + EPS
    __device__ __forceinline__ bool le(T a, T b, T tol) {
        band(b - a, tol);
        return a < b + (T)kEps;
    }
    // a + EPS > b
    __device__ __forceinline__ bool ge(T a, T b, T tol) {
        band(a - b, tol);
        return a + (T)kEps > b;
    }
    // |a - b| <= EPS
    __device__ __forceinline__ bool eq(T a, T b, T tol) {
        band(fabs(a - b), tol);
        return fabs(a - b) <= (T)kEps;
    }
    // plain comparisons against a threshold, with the band
    __device__ __forceinline__ bool less(T a, T b, T tol) {
        band(b - a, tol);
        return a < b;
    }
    __device__ __forceinline__ bool less_eq(T a, T b, T tol) {
        band(b - a, tol);
        return a <= b;
    }
    __device__ __forceinline__ bool greater(T a, T b, T tol) {
        band(a - b, tol);
        return a > b;
    }
    __device__ __forceinline__ bool greater_eq(T a, T b, T tol) {
        band(a - b, tol);
        return a >= b;
    }
};


// ---- sphere predicates (geometry.rs:66-82) ----
template <typename T, bool F>
__device__ __forceinline__ bool sphere_intersects(Dec<T, F>& d, const Sph<T>& a, const Sph<T>& b, T tolsq) {
    T sum_r = a.r + b.r;
    return d.lt(norm2(b.c - a.c), sum_r * sum_r, tolsq);
}
template <typename T, bool F>
__device__ __forceinline__ bool sphere_contains(Dec<T, F>& d, const Sph<T>& a, const Sph<T>& b, T tol, T tolsq) {
    // ge(a.r, b.r) && le(|b-a|^2, (a.r-b.r)^2), evaluated so that an unsure half does
    // not matter when the other half is surely false.
    T diff_r = a.r - b.r;
    Dec<T, F> d1, d2;
    bool p = d1.ge(a.r, b.r, tol);
    bool q = d2.le(norm2(b.c - a.c), diff_r * diff_r, tolsq);
    if (F) {
        bool p_sure_false = !p && !d1.unsure;
        bool q_sure_false = !q && !d2.unsure;
        if (!(p_sure_false || q_sure_false) && (d1.unsure || d2.unsure)) d.unsure = true;
    }
    return p && q;
}

// signed_distance_to_plane_unit (:96-102)
template <typename T>
__device__ __forceinline__ T sd_plane_unit(V3<T> pp, V3<T> n, V3<T> x) {
    return dot(n, x - pp);
}
// halfspace_of_point_unit (:118-131); returns 1 / -1 / 0
template <typename T, bool F>
__device__ __forceinline__ int halfspace(Dec<T, F>& d, V3<T> pp, V3<T> n, V3<T> x, T tol) {
    T sd = sd_plane_unit(pp, n, x);
    d.band(sd - (T)kEps, tol);
    d.band(sd + (T)kEps, tol);
    if (sd - (T)kEps > (T)0) return 1;
    if (sd + (T)kEps < (T)0) return -1;
    return 0;
}
// intersection_of_plane_and_segment (:134-148); the reference re-normalises the normal
template <typename T, bool F>
__device__ __forceinline__ V3<T> plane_segment(Dec<T, F>& d, V3<T> pp, V3<T> n, V3<T> a, V3<T> b, T tol) {
    V3<T> nn = normalize(n);
    T da = sd_plane_unit(pp, nn, a);
    T db = sd_plane_unit(pp, nn, b);
    if (d.less(fabs(da - db), (T)kEps, tol)) return a;
    T t = da / (da - db);
    return a + (b - a) * t;
}
// triangle_area (:152-154); FP32 with a correctly rounded square root (an output value)
__device__ __forceinline__ double triangle_area(V3<double> a, V3<double> b, V3<double> c) {
    return norm(cross(b - a, c - a)) / 2.0;
}
__device__ __forceinline__ float triangle_area(V3<float> a, V3<float> b, V3<float> c) {
    return 0.5f * __fsqrt_rn(norm2(cross(b - a, c - a)));
}

// angle between two vectors: FP64 follows min_angle (:157-161) exactly (acos of the
// clamped dot of the normalised vectors); FP32 uses atan2(|u x v|, u . v).
__device__ __forceinline__ double vec_angle(V3<double> u, V3<double> v) {
    V3<double> v1 = normalize(u), v2 = normalize(v);
    double c = dot(v1, v2);
    c = c < -1.0 ? -1.0 : (c > 1.0 ? 1.0 : c);
    return acos(c);
}
// FP32 angles are formed in double from the float vectors: products of floats are exact
// in double, so the only error left is the (unbiased) rounding of the float inputs.  A
// biased angle would bias every solid angle and, through SAS = (4 pi - sum) R^2 of a
// buried ball, be amplified in the SAS areas.
__device__ __forceinline__ V3<double> widen(V3<float> v) { return {(double)v.x, (double)v.y, (double)v.z}; }
__device__ __forceinline__ double vec_angle_wide(V3<float> u, V3<float> v) {
    V3<double> a = widen(u), b = widen(v);
    return atan2(norm(cross(a, b)), dot(a, b));
}
__device__ __forceinline__ float vec_angle(V3<float> u, V3<float> v) { return (float)vec_angle_wide(u, v); }
// pi minus the angle between u and v (FP32 turn terms of the solid angle), in double.
__device__ __forceinline__ double vec_supplement(V3<float> u, V3<float> v) {
    V3<double> a = widen(u), b = widen(v);
    return atan2(norm(cross(a, b)), -dot(a, b));
}

// directed_angle (:165-176).  FP32: the angle and its reflex form 2 pi - angle are
// evaluated in double and rounded once.
template <typename T, bool F>
__device__ __forceinline__ T directed_angle(Dec<T, F>& d, V3<T> o, V3<T> a, V3<T> b, V3<T> c, T tol) {
    V3<T> v1 = normalize(a - o), v2 = normalize(b - o);
    V3<T> n = cross(v1, v2);
    bool direct = d.greater_eq(dot(c - o, n), (T)0, tol);
    if constexpr (sizeof(T) == 4) {
        double angle = vec_angle_wide(a - o, b - o);
        return (T)(direct ? angle : kTau - angle);
    } else {
        T angle = vec_angle(a - o, b - o);
        if (direct) return angle;
        return (T)kTau - angle;
    }
}

// any_normal_of_vector (:179-193)
template <typename T>
__device__ __forceinline__ V3<T> any_normal(V3<T> a) {
    const T e = (T)kEps;
    V3<T> b = a;
    bool x0 = fabs(b.x) <= e, y0 = fabs(b.y) <= e, z0 = fabs(b.z) <= e;
    if (!x0 && (!y0 || !z0)) {
        b.x = -b.x;
        return normalize(cross(a, b));
    } else if (!y0 && (!x0 || !z0)) {
        b.y = -b.y;
        return normalize(cross(a, b));
    } else if (!x0) {
        return mk<T>(0, 1, 0);
    }
    return mk<T>(1, 0, 0);
}

// rotate_point_around_axis (:196-203): UnitQuaternion::from_axis_angle then q * p, with
// s = sin(angle / 2) and c = cos(angle / 2) supplied by the caller.
__device__ __forceinline__ V3<double> rotate_around_axis(V3<double> axis, double s, double c, V3<double> p) {
    if (norm2(axis) <= 0.0) return p;
    V3<double> u = normalize(axis);
    V3<double> qv = u * s;
    V3<double> t = cross(qv, p) * 2.0;
    V3<double> cr = cross(qv, t);
    return (t * c + cr) + p;
}

// intersection circle of two spheres (:229-239).  FP64 exactly as the reference; FP32
// uses the product form of r^2 = R_a^2 - h^2, which keeps precision near tangency.
__device__ __forceinline__ Sph<double> intersection_circle(const Sph<double>& a, const Sph<double>& b) {
    V3<double> cv = b.c - a.c;
    double cm = norm(cv);
    if (cm < kEps) return {a.c, 0.0};
    double cos_g = fma(b.r, -b.r, fma(a.r, a.r, cm * cm)) / (2.0 * a.r * cm);
    double sin_g = sqrt(fmax(1.0 - cos_g * cos_g, 0.0));
    V3<double> center = a.c + cv * (a.r * cos_g / cm);
    return {center, a.r * sin_g};
}
// The FP32 circle feeds every output value (areas, arc lengths, solid angles), so it is
// formed with correctly rounded square roots and divisions even where the kernel is
// compiled with approximate ones.
__device__ __forceinline__ float norm_rn(V3<float> v) { return __fsqrt_rn(norm2(v)); }
__device__ __forceinline__ Sph<float> intersection_circle(const Sph<float>& a, const Sph<float>& b) {
    V3<float> cv = b.c - a.c;
    float cm = norm_rn(cv);
    if (cm < (float)kEps) return {a.c, 0.0f};
    float h = __fdiv_rn(a.r * a.r + cm * cm - b.r * b.r, 2.0f * cm);
    float s = a.r + b.r, dr = a.r - b.r;
    float r2 = __fdiv_rn((s - cm) * (s + cm) * (cm - dr) * (cm + dr), 4.0f * cm * cm);
    return {a.c + cv * __fdiv_rn(h, cm), __fsqrt_rn(fmaxf(r2, 0.0f))};
}
// center_of_intersection_circle (:218-226)
__device__ __forceinline__ V3<double> ic_center(const Sph<double>& a, const Sph<double>& b) {
    V3<double> cv = b.c - a.c;
    double cm = norm(cv);
    if (cm < kEps) return a.c;
    double cos_g = fma(b.r, -b.r, fma(a.r, a.r, cm * cm)) / (2.0 * a.r * cm);
    return a.c + cv * (a.r * cos_g / cm);
}
__device__ __forceinline__ V3<float> ic_center(const Sph<float>& a, const Sph<float>& b) {
    V3<float> cv = b.c - a.c;
    float cm2 = norm2(cv);
    if (cm2 < (float)(kEps * kEps)) return a.c;
    // a cutting plane's position fixes the cut points on it: a correctly rounded division
    // (the kernel's approximate one, and a product with a rounded reciprocal, are biased:
    // between two balls of one radius the plane sits at exactly 0.5 of the distance, and
    // those land below it more often than above)
    float h_over_cm = __fdiv_rn(a.r * a.r + cm2 - b.r * b.r, 2.0f * cm2);
    return a.c + cv * h_over_cm;
}
// distance_to_intersection_circle_center (:208-215)
__device__ __forceinline__ double dist_to_ic_center(const Sph<double>& a, const Sph<double>& b) {
    double cm = norm(b.c - a.c);
    if (cm < kEps) return 0.0;
    double cos_g = fma(b.r, -b.r, fma(a.r, a.r, cm * cm)) / (2.0 * a.r * cm);
    return a.r * cos_g;
}

// project_point_inside_line (:243-255)
template <typename T, bool F>
__device__ __forceinline__ bool project_inside_line(Dec<T, F>& d, V3<T> o, V3<T> a, V3<T> b, V3<T>* out, T tol,
                                                    T tolsq) {
    V3<T> v = normalize(b - a);
    T l = dot(v, o - a);
    Dec<T, F> d1, d2;
    bool p = d1.greater(l, (T)0, tol);
    bool q = d2.less_eq(l * l, norm2(b - a), tolsq);
    if (F && (d1.unsure || d2.unsure) && !((!p && !d1.unsure) || (!q && !d2.unsure))) d.unsure = true;
    if (p && q) {
        *out = a + v * l;
        return true;
    }
    return false;
}
// intersect_segment_with_circle (:258-280)
template <typename T, bool F>
__device__ __forceinline__ bool segment_circle(Dec<T, F>& d, const Sph<T>& circle, V3<T> p_in, V3<T> p_out,
                                               V3<T>* out, T tol, T tolsq) {
    T dist = norm(p_in - p_out);
    if (d.less_eq(dist, (T)0, tol)) return false;
    V3<T> v = (p_in - p_out) / dist;
    V3<T> u = circle.c - p_out;
    V3<T> s = p_out + v * dot(v, u);
    T ll = fma(circle.r, circle.r, -norm2(circle.c - s));
    if (d.greater_eq(ll, (T)0, tolsq)) {
        *out = s - v * sqrt(fmax(ll, (T)0));
        return true;
    }
    return false;
}

// min_dihedral_angle (:283-293): angle between the components of b1-o and b2-o
// orthogonal to a-o.
template <typename T>
__device__ __forceinline__ T min_dihedral(V3<T> o, V3<T> a, V3<T> b1, V3<T> b2) {
    V3<T> oa = normalize(a - o);
    V3<T> d1 = b1 - (o + oa * dot(oa, b1 - o));
    V3<T> d2 = b2 - (o + oa * dot(oa, b2 - o));
    return vec_angle(d1, d2);
}
// pi - min_dihedral_angle for the FP32 turn terms of the solid angle, evaluated in double
// from the widened float points: the dihedral at edge o-a between the half-planes
// towards b1 and b2 is the angle between the normals (a-o) x (b1-o) and (a-o) x (b2-o).
// Products of floats are exact in double, so a point b next to a (a vertex beside a short
// contour edge) loses nothing to the cancellation of a float projection; the turn sum is
// then the solid angle of the polygon with the float vertices.
__device__ __forceinline__ double dihedral_supplement(V3<float> o, V3<float> a, V3<float> b1, V3<float> b2) {
    const V3<double> O = widen(o);
    const V3<double> ax = widen(a) - O, u1 = widen(b1) - O, u2 = widen(b2) - O;
    const V3<double> n1 = cross(ax, u1), n2 = cross(ax, u2);
    return atan2(norm(cross(n1, n2)), -dot(n1, n2));
}

}  // namespace vt
