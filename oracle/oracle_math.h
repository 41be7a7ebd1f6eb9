// oracle_math.h — scalar/vector helpers with WGSL semantics, for the CPU oracle.
//
// TEST INFRASTRUCTURE: this directory is the CPU oracle that checks the CUDA engine.
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use it.
//
// Rules that make the restatement reproducible (compile with -ffp-contract=off):
//  * WGSL mix(a,b,t) = a*(1-t) + b*t; clamp(x,lo,hi) = min(max(x,lo),hi);
//    smoothstep(lo,hi,x) = t*t*(3-2t), t = clamp((x-lo)/(hi-lo),0,1);
//    fract(x) = x - floor(x)   (WGSL built-ins, used by shader.rs throughout).
//  * i32(f) truncates toward zero and saturates (WGSL conversion rules); NaN -> 0.
//  * dot/length evaluate ((x*x + y*y) + z*z).
//  * exp() on the J update (shader.rs:1853) is a degree-10 Taylor polynomial in
//    Horner form, |x| <= 0.35, identical in the CUDA engine, so both sides agree
//    bit for bit (the WGSL backend's exp precision is implementation-defined).
#pragma once
#include <cmath>
#include <cstdint>
#include <algorithm>

namespace orc {

template <class R> struct v2 { R x, y; };
template <class R> struct v3 { R x, y, z; };

template <class R> inline v3<R> V3(R x, R y, R z) { return v3<R>{x, y, z}; }
template <class R> inline v3<R> operator+(v3<R> a, v3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline v3<R> operator-(v3<R> a, v3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline v3<R> operator-(v3<R> a) { return {-a.x, -a.y, -a.z}; }
template <class R> inline v3<R> operator*(v3<R> a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline v3<R> operator*(R s, v3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> inline v3<R> operator/(v3<R> a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <class R> inline v3<R>& operator+=(v3<R>& a, v3<R> b) { a = a + b; return a; }
template <class R> inline v3<R>& operator-=(v3<R>& a, v3<R> b) { a = a - b; return a; }
template <class R> inline v3<R>& operator*=(v3<R>& a, R s) { a = a * s; return a; }
template <class R> inline R dot(v3<R> a, v3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline R length(v3<R> a) { return std::sqrt(dot(a, a)); }
template <class R> inline R dot2(v2<R> a, v2<R> b) { return a.x * b.x + a.y * b.y; }
template <class R> inline R length2(v2<R> a) { return std::sqrt(dot2(a, a)); }

template <class R> inline R wmin(R a, R b) { return std::fmin(a, b); }
template <class R> inline R wmax(R a, R b) { return std::fmax(a, b); }
template <class R> inline R wclamp(R x, R lo, R hi) { return wmin(wmax(x, lo), hi); }
template <class R> inline R mix(R a, R b, R t) { return a * (R(1) - t) + b * t; }
template <class R> inline v3<R> mix(v3<R> a, v3<R> b, R t) {
    return {mix(a.x, b.x, t), mix(a.y, b.y, t), mix(a.z, b.z, t)};
}
template <class R> inline R smoothstep(R lo, R hi, R x) {
    R t = wclamp((x - lo) / (hi - lo), R(0), R(1));
    return t * t * (R(3) - R(2) * t);
}
template <class R> inline R wfract(R x) { return x - std::floor(x); }

template <class R> inline int32_t to_i32(R x) {
    if (x != x) return 0;
    if (x >= R(2147483647.0)) return INT32_MAX;
    if (x <= R(-2147483648.0)) return INT32_MIN;
    return (int32_t)x;
}
template <class R> inline int64_t to_i64(R x) {
    if (x != x) return 0;
    if (x >= R(9223372036854775807.0)) return INT64_MAX;
    if (x <= R(-9223372036854775808.0)) return INT64_MIN;
    return (int64_t)x;
}
template <class R> inline uint32_t to_u32(R x) {
    if (x != x || x <= R(0)) return 0u;
    if (x >= R(4294967295.0)) return UINT32_MAX;
    return (uint32_t)x;
}

// exp(x) for |x| <= 0.35: sum_{k=0..10} x^k/k! in Horner form (Taylor series).
inline float exp_small(float x) {
    float p = 2.7557319e-07f;           // 1/10!
    p = p * x + 2.7557319e-06f;         // 1/9!
    p = p * x + 2.4801587e-05f;         // 1/8!
    p = p * x + 1.9841270e-04f;         // 1/7!
    p = p * x + 1.3888889e-03f;         // 1/6!
    p = p * x + 8.3333333e-03f;         // 1/5!
    p = p * x + 4.1666667e-02f;         // 1/4!
    p = p * x + 1.6666667e-01f;         // 1/3!
    p = p * x + 0.5f;
    p = p * x + 1.0f;
    p = p * x + 1.0f;
    return p;
}
inline double exp_small(double x) { return std::exp(x); }

// SplitMix64 (Steele, Lea, Flood 2014): the seeded stream of the scene generators.
struct SplitMix64 {
    uint64_t s;
    explicit SplitMix64(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    // uniform float in [0,1) with 24 random bits
    float uniform() { return (float)(next() >> 40) * (1.0f / 16777216.0f); }
    // uniform double in (0,1]
    double uniform_open() { return ((double)(next() >> 11) + 1.0) * (1.0 / 9007199254740992.0); }
};

}  // namespace orc
