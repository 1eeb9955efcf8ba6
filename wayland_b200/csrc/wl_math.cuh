// wl_math.cuh - vector maths, random streams and transcendental functions shared by the
// kernels (host + device).
//
// Vector operators follow glm 1.0.1's semantics, the arithmetic the reference's device code is
// written in (src/Frontend/Device/*.h): componentwise operators, vector / scalar divides each
// component, dot = (x*x' + y*y') + z*z', normalize(v) = v * (1 / sqrt(dot(v, v))).
//
// Two arithmetic modes select the transcendental functions:
//   WL_STRICT_MATH defined : the project's own sin/cos/log below (IEEE operations only); the
//                            translation unit is compiled with -fmad=false -prec-div=true
//                            -prec-sqrt=true -ftz=false, which makes every result bit-identical
//                            to the CPU oracle.
//   otherwise              : hardware approximations (__sinf, __cosf, __logf) under
//                            --use_fast_math, the reference's own compile mode (Module.h:23-31).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include <cstring>
#include <math.h>

#define WL_HD __host__ __device__ __forceinline__

namespace wl {

WL_HD float as_float(uint32_t u) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(u);
#else
    float f;
    std::memcpy(&f, &u, 4);
    return f;
#endif
}
WL_HD uint32_t as_uint(float f) {
#ifdef __CUDA_ARCH__
    return __float_as_uint(f);
#else
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
#endif
}

struct v3 {
    float x, y, z;
    WL_HD v3() : x(0.f), y(0.f), z(0.f) {}
    WL_HD v3(float a, float b, float c) : x(a), y(b), z(c) {}
    WL_HD explicit v3(float s) : x(s), y(s), z(s) {}
};
WL_HD v3 operator+(v3 a, v3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
WL_HD v3 operator-(v3 a, v3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
WL_HD v3 operator*(v3 a, v3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
WL_HD v3 operator/(v3 a, v3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
WL_HD v3 operator*(v3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
WL_HD v3 operator*(float s, v3 a) { return v3(s * a.x, s * a.y, s * a.z); }
WL_HD v3 operator/(v3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
WL_HD v3 operator+(v3 a, float s) { return v3(a.x + s, a.y + s, a.z + s); }
WL_HD v3 operator-(v3 a) { return v3(-a.x, -a.y, -a.z); }
WL_HD float dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
WL_HD v3 cross(v3 a, v3 b) {
    return v3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
WL_HD float length(v3 a) { return sqrtf(dot(a, a)); }
WL_HD v3 normalize(v3 a) { return a * (1.0f / sqrtf(dot(a, a))); }
// Common.h:72-100: the reference's own clamp / lerp (not glm's)
WL_HD float clampf(float a, float lo, float hi) { return a < lo ? lo : (a > hi ? hi : a); }
WL_HD v3 clampv(v3 v, float lo, float hi) {
    return v3(clampf(v.x, lo, hi), clampf(v.y, lo, hi), clampf(v.z, lo, hi));
}
WL_HD float lerpf(float a, float b, float w) { return a * (1.0f - w) + b * w; }
WL_HD v3 lerpv(v3 a, v3 b, float w) { return v3(lerpf(a.x, b.x, w), lerpf(a.y, b.y, w), lerpf(a.z, b.z, w)); }
WL_HD v3 ld3(const float *p) { return v3(p[0], p[1], p[2]); }
WL_HD v3 f4xyz(float4 a) { return v3(a.x, a.y, a.z); }

// Utils/MathConstants.h:6-10
constexpr float PI = 3.14159265358979323846f;
constexpr float TWO_PI = PI * 2.0f;
constexpr float RECIP_PI = 1.f / PI;

// ---------------------------------------------------------------------------------------
// The project's sin/cos/log (WL_MATH_STRICT). Cody-Waite reduction by pi/2 with a 21-bit head
// (k * head exact for the k that occur), Taylor polynomials of sin to r^9 and cos to r^10 on
// |r| <= pi/4; log by exponent split with m in [sqrt(1/2), sqrt(2)) and
// log m = 2 atanh((m - 1)/(m + 1)) as the odd series to f^9. Coefficients are 1/n! and 1/(2k+1).
WL_HD float own_sin_core(float r, float s) {
    float p = 0x1.71de3ap-19f;
    p = p * s + -0x1.a01a02p-13f;
    p = p * s + 0x1.111112p-7f;
    p = p * s + -0x1.555556p-3f;
    return r + (r * s) * p;
}
WL_HD float own_cos_core(float s) {
    float p = -0x1.27e4fcp-22f;
    p = p * s + 0x1.a01a02p-16f;
    p = p * s + -0x1.6c16c2p-10f;
    p = p * s + 0x1.555556p-5f;
    p = p * s + -0.5f;
    return 1.0f + s * p;
}
WL_HD void own_sincosf(float x, float *sn, float *cs) {
    if (!(fabsf(x) < 1.0e5f)) {
        *sn = as_float(0x7fc00000u);
        *cs = *sn;
        return;
    }
#ifdef __CUDA_ARCH__
    float kf = rintf(x * 0x1.45f306p-1f);
#else
    float kf = nearbyintf(x * 0x1.45f306p-1f);
#endif
    int k = (int)kf;
    float r = (x - kf * 0x1.921fb0p+0f) - kf * 0x1.5110b4p-22f;
    float s = r * r;
    float sr = own_sin_core(r, s), cr = own_cos_core(s);
    switch (k & 3) {
    case 0: *sn = sr; *cs = cr; break;
    case 1: *sn = cr; *cs = -sr; break;
    case 2: *sn = -sr; *cs = -cr; break;
    default: *sn = -cr; *cs = sr; break;
    }
}
WL_HD float own_logf(float x) {
    if (x != x || x < 0.0f) return as_float(0x7fc00000u);
    if (x == 0.0f) return as_float(0xff800000u);
    if (x == as_float(0x7f800000u)) return x;
    uint32_t b = as_uint(x);
    int e = 0;
    if ((b >> 23) == 0) {
        b = as_uint(x * 8388608.0f);
        e = -23;
    }
    e += (int)(b >> 23) - 127;
    float m = as_float((b & 0x7fffffu) | 0x3f800000u);
    if (m > 0x1.6a09e6p+0f) {
        m = m * 0.5f;
        e += 1;
    }
    float f = (m - 1.0f) / (m + 1.0f);
    float s = f * f;
    float p = 0x1.c71c72p-4f;
    p = p * s + 0x1.24924ap-3f;
    p = p * s + 0x1.99999ap-3f;
    p = p * s + 0x1.555556p-2f;
    p = p * s + 1.0f;
    float ef = (float)e;
    return ef * 0x1.62e400p-1f + (ef * 0x1.7f7d1cp-20f + (2.0f * f) * p);
}

#if defined(WL_STRICT_MATH) || !defined(__CUDA_ARCH__)
WL_HD float m_sin(float x) { float s, c; own_sincosf(x, &s, &c); return s; }
WL_HD float m_cos(float x) { float s, c; own_sincosf(x, &s, &c); return c; }
WL_HD float m_log(float x) { return own_logf(x); }
#else
__device__ __forceinline__ float m_sin(float x) { return __sinf(x); }
__device__ __forceinline__ float m_cos(float x) { return __cosf(x); }
__device__ __forceinline__ float m_log(float x) { return __logf(x); }
#endif

// ---------------------------------------------------------------------------------------
// Random streams. TEA_LCG: seed = tea<4>(pixel, frame), then the LCG of Random.h:53-71.
// PCG32: O'Neill 2014, XSH-RR 64/32, increment from the pixel index, state from splitmix64.
WL_HD uint32_t tea4(uint32_t val0, uint32_t val1) {  // Random.h:34-50
    uint32_t v0 = val0, v1 = val1, s0 = 0;
#pragma unroll
    for (int n = 0; n < 4; n++) {
        s0 += 0x9e3779b9u;
        v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
        v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
    }
    return v0;
}
WL_HD uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
constexpr uint64_t PCG_MUL = 6364136223846793005ULL;

struct Rng {
    uint64_t state;
    uint32_t pixel;
    uint32_t mode;
    WL_HD float next() {
        if (mode == 0) {
            uint32_t s = (uint32_t)state;
            s = 1664525u * s + 1013904223u;
            state = s;
            return (float)(s & 0x00FFFFFFu) / (float)0x01000000;
        }
        uint64_t old = state;
        state = old * PCG_MUL + (((uint64_t)pixel << 1) | 1u);
        uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        uint32_t r = (xs >> rot) | (xs << ((32u - rot) & 31u));
        return (float)(r >> 8) * 0x1p-24f;
    }
};
WL_HD Rng make_rng(uint32_t mode, uint64_t seed, uint32_t pixel, uint32_t frame) {
    Rng r;
    r.mode = mode;
    r.pixel = pixel;
    if (mode == 0) {
        r.state = tea4(pixel, frame);  // PathTracing.cu:47
    } else {
        uint64_t inc = ((uint64_t)pixel << 1) | 1u;
        uint64_t init = splitmix64(seed ^ ((uint64_t)frame << 32) ^ (uint64_t)pixel);
        uint64_t s = 0;
        s = s * PCG_MUL + inc;
        s += init;
        s = s * PCG_MUL + inc;
        r.state = s;
    }
    return r;
}

// ---------------------------------------------------------------------------------------
// Exactly rounded single-precision operations that the compiler may not contract or reorder,
// for the arithmetic that defines a hit (identical on host and device).
#ifdef __CUDA_ARCH__
#define XADD(a, b) __fadd_rn((a), (b))
#define XSUB(a, b) __fsub_rn((a), (b))
#define XMUL(a, b) __fmul_rn((a), (b))
#define XDIV(a, b) __fdiv_rn((a), (b))
#else
#define XADD(a, b) ((a) + (b))
#define XSUB(a, b) ((a) - (b))
#define XMUL(a, b) ((a) * (b))
#define XDIV(a, b) ((a) / (b))
#endif

// Watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2(1) 2013): the project's definition
// of a hit. Single precision in exactly this order, double-precision recomputation when an edge
// function evaluates to 0, hit iff tmin < t < tmax with t = T / det. u, v are the barycentric
// weights of vertices 1 and 2.
struct RayPre {
    int kx, ky, kz;
    float sx, sy, sz;
};
WL_HD RayPre ray_pre(float dx, float dy, float dz) {
    float ax = fabsf(dx), ay = fabsf(dy), az = fabsf(dz);
    int kz = (ax > ay) ? ((ax > az) ? 0 : 2) : ((ay > az) ? 1 : 2);
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    float d[3] = {dx, dy, dz};
    if (d[kz] < 0.0f) { int t = kx; kx = ky; ky = t; }
    RayPre p;
    p.kx = kx; p.ky = ky; p.kz = kz;
    p.sx = XDIV(d[kx], d[kz]);
    p.sy = XDIV(d[ky], d[kz]);
    p.sz = XDIV(1.0f, d[kz]);
    return p;
}
WL_HD float sel3(float a, float b, float c, int k) { return k == 0 ? a : (k == 1 ? b : c); }

WL_HD bool tri_hit(const RayPre &p, float ox, float oy, float oz, float4 v0, float4 v1, float4 v2,
                   float tmin, float tmax, float &t_out, float &u_out, float &v_out) {
    float A0 = XSUB(v0.x, ox), A1 = XSUB(v0.y, oy), A2 = XSUB(v0.z, oz);
    float B0 = XSUB(v1.x, ox), B1 = XSUB(v1.y, oy), B2 = XSUB(v1.z, oz);
    float C0 = XSUB(v2.x, ox), C1 = XSUB(v2.y, oy), C2 = XSUB(v2.z, oz);
    float Akx = sel3(A0, A1, A2, p.kx), Aky = sel3(A0, A1, A2, p.ky), Akz = sel3(A0, A1, A2, p.kz);
    float Bkx = sel3(B0, B1, B2, p.kx), Bky = sel3(B0, B1, B2, p.ky), Bkz = sel3(B0, B1, B2, p.kz);
    float Ckx = sel3(C0, C1, C2, p.kx), Cky = sel3(C0, C1, C2, p.ky), Ckz = sel3(C0, C1, C2, p.kz);
    float ax = XSUB(Akx, XMUL(p.sx, Akz)), ay = XSUB(Aky, XMUL(p.sy, Akz));
    float bx = XSUB(Bkx, XMUL(p.sx, Bkz)), by = XSUB(Bky, XMUL(p.sy, Bkz));
    float cx = XSUB(Ckx, XMUL(p.sx, Ckz)), cy = XSUB(Cky, XMUL(p.sy, Ckz));
    float U = XSUB(XMUL(cx, by), XMUL(cy, bx));
    float V = XSUB(XMUL(ax, cy), XMUL(ay, cx));
    float W = XSUB(XMUL(bx, ay), XMUL(by, ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = (float)((double)cx * (double)by - (double)cy * (double)bx);
        V = (float)((double)ax * (double)cy - (double)ay * (double)cx);
        W = (float)((double)bx * (double)ay - (double)by * (double)ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = XADD(XADD(U, V), W);
    if (det == 0.0f) return false;
    float az = XMUL(p.sz, Akz), bz = XMUL(p.sz, Bkz), cz = XMUL(p.sz, Ckz);
    float T = XADD(XADD(XMUL(U, az), XMUL(V, bz)), XMUL(W, cz));
    float t = XDIV(T, det);
    if (!(t > tmin && t < tmax)) return false;
    t_out = t;
    u_out = XDIV(V, det);
    v_out = XDIV(W, det);
    return true;
}

}  // namespace wl
