// wl_oracle.cpp - CPU oracle (test infrastructure only; see wl_oracle.h).
//
// Build: g++ -O2 -std=c++17 -ffp-contract=off -fno-fast-math -fopenmp -shared -fPIC
// (no FMA contraction and IEEE division/sqrt, so single precision results are bit-identical to
// the GPU kernels compiled in WL_MATH_STRICT mode).
//
// Expression order follows the reference line by line (each function cites file:line); glm's
// own operator semantics are restated in struct V3 below (glm 1.0.1: componentwise operators,
// dot = (x*x' + y*y') + z*z', normalize = v * (1 / sqrt(dot(v, v))), length = sqrt(dot(v, v)),
// cross = (y z' - y' z, z x' - z' x, x y' - x' y)).
#include "wl_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <cstdio>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr uint32_t INVALID = 0xFFFFFFFFu;

// ---------------------------------------------------------------------------------------
// glm-like 3-vector (float or double)
template <class T> struct V3 {
    T x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(T a, T b, T c) : x(a), y(b), z(c) {}
    explicit V3(T s) : x(s), y(s), z(s) {}
    T operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
template <class T> V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> V3<T> operator*(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> V3<T> operator/(V3<T> a, V3<T> b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class T> V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> V3<T> operator*(T s, V3<T> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> V3<T> operator+(V3<T> a, T s) { return {a.x + s, a.y + s, a.z + s}; }
template <class T> V3<T> operator-(V3<T> a) { return {-a.x, -a.y, -a.z}; }
template <class T> T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> V3<T> cross(V3<T> a, V3<T> b) {
    return {a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y};
}
template <class T> T length(V3<T> a) { return std::sqrt(dot(a, a)); }
template <class T> V3<T> normalize(V3<T> a) { return a * (T(1) / std::sqrt(dot(a, a))); }

// Common.h:72-100 clamp/lerp (not glm's)
template <class T> T clampf(T a, T lo, T hi) { return a < lo ? lo : (a > hi ? hi : a); }
template <class T> V3<T> clampv(V3<T> v, T lo, T hi) {
    return {clampf(v.x, lo, hi), clampf(v.y, lo, hi), clampf(v.z, lo, hi)};
}
template <class T> T lerp(T a, T b, T w) { return a * (T(1) - w) + b * w; }
template <class T> V3<T> lerp(V3<T> a, V3<T> b, T w) {
    return {lerp(a.x, b.x, w), lerp(a.y, b.y, w), lerp(a.z, b.z, w)};
}

// ---------------------------------------------------------------------------------------
// The project's sin/cos/log for FP32 strict mode (own implementation, not the C library's):
// Cody-Waite reduction by pi/2 with a 21-bit head so k * head is exact, then Taylor
// polynomials of sin (to r^9) and cos (to r^10) on |r| <= pi/4; log by exponent split,
// m in [sqrt(1/2), sqrt(2)), log m = 2 atanh((m-1)/(m+1)) as an odd series to f^9.
float own_sinf_core(float r, float s) {
    float p = 0x1.71de3ap-19f;          // 1/9!
    p = p * s + -0x1.a01a02p-13f;       // -1/7!
    p = p * s + 0x1.111112p-7f;         // 1/5!
    p = p * s + -0x1.555556p-3f;        // -1/3!
    return r + (r * s) * p;
}
float own_cosf_core(float s) {
    float p = -0x1.27e4fcp-22f;         // -1/10!
    p = p * s + 0x1.a01a02p-16f;        // 1/8!
    p = p * s + -0x1.6c16c2p-10f;       // -1/6!
    p = p * s + 0x1.555556p-5f;         // 1/4!
    p = p * s + -0.5f;                  // -1/2!
    return 1.0f + s * p;
}
void own_sincosf(float x, float *sn, float *cs) {
    if (!(std::fabs(x) < 1.0e5f)) {  // outside the range the reduction is built for
        *sn = std::numeric_limits<float>::quiet_NaN();
        *cs = *sn;
        return;
    }
    float kf = std::nearbyint(x * 0x1.45f306p-1f);  // x * 2/pi, round to nearest even
    int k = (int)kf;
    float r = (x - kf * 0x1.921fb0p+0f) - kf * 0x1.5110b4p-22f;
    float s = r * r;
    float sr = own_sinf_core(r, s), cr = own_cosf_core(s);
    switch (k & 3) {
    case 0: *sn = sr; *cs = cr; break;
    case 1: *sn = cr; *cs = -sr; break;
    case 2: *sn = -sr; *cs = -cr; break;
    default: *sn = -cr; *cs = sr; break;
    }
}
float own_logf(float x) {
    if (x != x || x < 0.0f) return std::numeric_limits<float>::quiet_NaN();
    if (x == 0.0f) return -std::numeric_limits<float>::infinity();
    if (std::isinf(x)) return x;
    uint32_t b;
    std::memcpy(&b, &x, 4);
    int e = 0;
    if ((b >> 23) == 0) {  // subnormal: scale by 2^23
        float y = x * 8388608.0f;
        std::memcpy(&b, &y, 4);
        e = -23;
    }
    e += (int)(b >> 23) - 127;
    uint32_t mb = (b & 0x7fffffu) | 0x3f800000u;
    float m;
    std::memcpy(&m, &mb, 4);
    if (m > 0x1.6a09e6p+0f) {  // sqrt(2)
        m = m * 0.5f;
        e += 1;
    }
    float f = (m - 1.0f) / (m + 1.0f);
    float s = f * f;
    float p = 0x1.c71c72p-4f;            // 1/9
    p = p * s + 0x1.24924ap-3f;          // 1/7
    p = p * s + 0x1.99999ap-3f;          // 1/5
    p = p * s + 0x1.555556p-2f;          // 1/3
    p = p * s + 1.0f;
    float ef = (float)e;
    return ef * 0x1.62e400p-1f + (ef * 0x1.7f7d1cp-20f + (2.0f * f) * p);
}

// math dispatch: float -> the project's functions; double -> the C library
inline float m_sin(float x) { float s, c; own_sincosf(x, &s, &c); return s; }
inline float m_cos(float x) { float s, c; own_sincosf(x, &s, &c); return c; }
inline float m_log(float x) { return own_logf(x); }
inline double m_sin(double x) { return std::sin(x); }
inline double m_cos(double x) { return std::cos(x); }
inline double m_log(double x) { return std::log(x); }

// Utils/MathConstants.h:6-10: PI is the float nearest pi; TWO_PI = PI * 2; RECIP_PI = 1 / PI
// (all float). The FP64 oracle uses the double constants instead.
template <class T> struct C;
template <> struct C<float> {
    static float pi() { return 3.14159265358979323846f; }
    static float two_pi() { return 3.14159265358979323846f * 2.0f; }
    static float recip_pi() { return 1.f / 3.14159265358979323846f; }
};
template <> struct C<double> {
    static double pi() { return 3.14159265358979323846; }
    static double two_pi() { return 2.0 * 3.14159265358979323846; }
    static double recip_pi() { return 1.0 / 3.14159265358979323846; }
};
// A literal written as a float in the reference; exact double in the FP64 oracle.
template <class T> inline T kc(float f, double d);
template <> inline float kc<float>(float f, double) { return f; }
template <> inline double kc<double>(float, double d) { return d; }
#define K(x) kc<T>(x##f, x)

// ---------------------------------------------------------------------------------------
// Random.h:34-71
uint32_t tea4(uint32_t val0, uint32_t val1) {
    uint32_t v0 = val0, v1 = val1, s0 = 0;
    for (int n = 0; n < 4; n++) {
        s0 += 0x9e3779b9u;
        v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + s0) ^ ((v1 >> 5) + 0xc8013ea4u);
        v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + s0) ^ ((v0 >> 5) + 0x7e95761eu);
    }
    return v0;
}

// Per-path random stream: the reference's LCG, or PCG32 (O'Neill 2014, XSH-RR 64/32).
struct Rng {
    uint32_t mode;
    uint64_t state;
    uint64_t inc;
    float next() {
        if (mode == WL_RNG_TEA_LCG) {  // lcg + rnd (Random.h:53-71)
            uint32_t s = (uint32_t)state;
            s = 1664525u * s + 1013904223u;
            state = s;
            return (float)(s & 0x00FFFFFFu) / (float)0x01000000;
        }
        uint64_t old = state;
        state = old * 6364136223846793005ULL + inc;
        uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        uint32_t r = (xs >> rot) | (xs << ((32u - rot) & 31u));
        return (float)(r >> 8) * 0x1p-24f;
    }
};
uint64_t splitmix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
Rng make_rng(uint32_t mode, uint64_t seed, uint32_t pixel, uint32_t frame) {
    Rng r;
    r.mode = mode;
    if (mode == WL_RNG_TEA_LCG) {
        r.state = tea4(pixel, frame);  // PathTracing.cu:47
        r.inc = 0;
    } else {
        uint64_t init = splitmix64(seed ^ ((uint64_t)frame << 32) ^ (uint64_t)pixel);
        r.inc = ((uint64_t)pixel << 1) | 1u;
        r.state = 0;
        r.state = r.state * 6364136223846793005ULL + r.inc;
        r.state += init;
        r.state = r.state * 6364136223846793005ULL + r.inc;
    }
    return r;
}

// ---------------------------------------------------------------------------------------
// Material maths, Common.h:102-181
template <class T> void onb(V3<T> n, V3<T> &u, V3<T> &v) {  // Common.h:102-116
    T x = n.x, y = n.y, z = n.z;
    T sign = std::copysign(T(1), z);
    T a = T(-1) / (sign + z);
    T b = x * y * a;
    u = V3<T>(T(1) + sign * x * x * a, sign * b, -sign * x);
    v = V3<T>(b, sign + y * y * a, -y);
}
template <class T> T schlick(T u) {  // Common.h:122-127
    T m = clampf(T(1) - u, T(0), T(1));
    T m2 = m * m;
    return m2 * m2 * m;
}
template <class T> T fresnel(T ci, T ct, T eta) {  // Common.h:129-137
    const T rs = (ci - ct * eta) / (ci + eta * ct);
    const T rp = (ci * eta - ct) / (ci * eta + ct);
    return K(0.5) * (rs * rs + rp * rp);
}
template <class T> T gtr1(T ndh, T a) {  // Common.h:139-146
    if (a >= T(1)) return T(1) / C<T>::pi();
    T a2 = a * a;
    T t = T(1) + (a2 - T(1)) * ndh * ndh;
    return (a2 - T(1)) / (C<T>::pi() * m_log(a2) * t);
}
template <class T> T gtr2(T ndh, T a) {  // Common.h:148-153
    T a2 = a * a;
    T t = T(1) + (a2 - T(1)) * ndh * ndh;
    return a2 / (C<T>::pi() * t * t);
}
template <class T> T smithg(T ndv, T ag) {  // Common.h:155-161
    T a = ag * ag;
    T b = ndv * ndv;
    return T(1) / (ndv + std::sqrt(a + b - a * b));
}
template <class T> T lambda_beckmann(V3<T> w, V3<T> n) {  // Common.h:163-179
    const T alphax = K(0.5);
    T wdn = dot(w, n);
    T abs_tan = std::fabs(length(cross(w, n)) / wdn);
    if (std::isinf(abs_tan)) return T(0);
    T a = T(1) / (alphax * abs_tan);
    if (a >= K(1.6)) return T(0);
    return (T(1) - K(1.259) * a + K(0.396) * a * a) / (K(3.535) * a + K(2.181) * a * a);
}

template <class T> struct Mat {
    V3<T> color;
    T metallic, roughness, specular, specular_tint, eta, trans, subsurface, anisotropic, sheen,
        sheen_tint, clearcoat, clearcoat_gloss;
};
template <class T> Mat<T> to_mat(const wl_disney &d) {
    Mat<T> m;
    m.color = V3<T>(d.color[0], d.color[1], d.color[2]);
    m.metallic = d.metallic; m.roughness = d.roughness; m.specular = d.specular;
    m.specular_tint = d.specular_tint; m.eta = d.eta; m.trans = d.trans;
    m.subsurface = d.subsurface; m.anisotropic = d.anisotropic; m.sheen = d.sheen;
    m.sheen_tint = d.sheen_tint; m.clearcoat = d.clearcoat; m.clearcoat_gloss = d.clearcoat_gloss;
    return m;
}

// Cspec0 as written at Evaluate.h:47-50 and :129-132
template <class T> V3<T> cspec0(const Mat<T> &m, V3<T> cdlin, V3<T> ctint) {
    return lerp(m.specular * K(0.08) * lerp(V3<T>(T(1)), ctint, m.specular_tint), cdlin,
                m.metallic);
}
template <class T> V3<T> ctint_of(V3<T> cdlin, T &cdlum) {
    cdlum = K(0.3) * cdlin.x + K(0.6) * cdlin.y + K(0.1) * cdlin.z;
    return cdlum > T(0) ? cdlin / cdlum : V3<T>(T(1));
}

// EvalDisneyTransmit, Evaluate.h:10-76
template <class T>
V3<T> eval_transmit(const Mat<T> &m, V3<T> Ns, V3<T> /*Ng*/, V3<T> V, V3<T> L, V3<T> tex) {
    V3<T> N = Ns;
    V3<T> cc = tex * m.color;
    T ndl = dot(N, L);
    T ndv = dot(N, V);
    T eta = T(1) / m.eta;
    if (ndl > T(0)) {
        eta = T(1) / eta;
        N = -N;
    }
    if (ndl == T(0) || ndv == T(0)) return V3<T>(T(0));
    T refract = ((T(1) - ndv * ndv) * eta * eta >= T(1)) ? T(1) : T(0);
    T cdlum;
    V3<T> ctint = ctint_of(cc, cdlum);
    V3<T> cs0 = cspec0(m, cc, ctint);
    (void)cs0;
    V3<T> wh = normalize(L + V * eta);
    if (dot(wh, N) < T(0)) wh = -wh;
    if (dot(L, wh) * dot(V, wh) > T(0)) return V3<T>(T(0));
    T sqrt_denom = dot(L, wh) + eta * dot(V, wh);
    T factor = T(1) / eta;
    V3<T> Tc = m.trans * cc;
    T gs = T(1) / (T(1) + lambda_beckmann(V, N) + lambda_beckmann(L, N));
    T a = std::fmax(K(0.001), m.roughness);
    T ds = gtr2(dot(N, wh), a);
    T f = fresnel(std::fabs(dot(V, wh)), std::fabs(dot(L, wh)), eta);
    V3<T> out = (T(1) - refract) * (T(1) - f) * Tc *
                std::fabs(ds * gs * eta * eta * std::fabs(dot(L, wh)) * std::fabs(dot(V, wh)) *
                          factor * factor / (ndl * ndl * sqrt_denom * sqrt_denom));
    return out;
}

// EvalDisneyBSDF, Evaluate.h:78-191 (the clearcoat terms Dr/Fr/Gr are computed there but never
// used in the result; they are omitted here)
template <class T>
V3<T> eval_disney(const Mat<T> &m, V3<T> Ns_, V3<T> Ng, V3<T> V, V3<T> L, V3<T> tex) {
    V3<T> cc = tex * m.color;
    V3<T> Ns = Ns_;
    T ndl = dot(Ns, L);
    T gndl = dot(Ng, L);
    T ndv = dot(Ns, V);
    T gndv = dot(Ng, V);
    T eta = T(1) / m.eta;
    if (m.trans < K(0.1) && (gndl * gndv <= T(0) || ndl * ndv <= T(0))) return V3<T>(T(0));
    if (m.trans > K(0.9) && (gndl * gndv * ndl * ndv <= T(0))) return V3<T>(T(0));
    if (ndl * ndv <= T(0)) return eval_transmit(m, Ns, Ng, V, L, tex);
    if (m.metallic + cc.x + cc.y + cc.z <= T(0)) return V3<T>(T(0));
    if (ndl < T(0) && ndv < T(0)) {
        Ns = -Ns;
        eta = T(1) / eta;
        ndl *= T(-1);
        ndv *= T(-1);
    }
    V3<T> H = normalize(L + V);
    T ndh = dot(Ns, H);
    T ldh = dot(L, H);
    T refract = ((T(1) - ndv * ndv) * eta * eta >= T(1)) ? T(1) : T(0);
    V3<T> cdlin = cc;
    T cdlum;
    V3<T> ctint = ctint_of(cdlin, cdlum);
    V3<T> cs0 = cspec0(m, cdlin, ctint);
    V3<T> csheen = lerp(V3<T>(T(1)), ctint, m.sheen_tint);
    T fl = schlick(ndl), fv = schlick(ndv);
    T fd90 = K(0.5) + K(2.0) * ldh * ldh * m.roughness;
    T fd = lerp(T(1), fd90, fl) * lerp(T(1), fd90, fv);
    T fss90 = ldh * ldh * m.roughness;
    T fss = lerp(T(1), fss90, fl) * lerp(T(1), fss90, fv);
    T ss = K(1.25) * (fss * (T(1) / (ndl + ndv) - K(0.5)) + K(0.5));
    T a = std::fmax(K(0.001), m.roughness);
    T ds = gtr2(ndh, a);
    T fh = schlick(ldh);
    V3<T> fs = lerp(cs0, V3<T>(T(1)), fh);
    T roughg = std::sqrt(m.roughness * K(0.5) + K(0.5));
    T gs = smithg(ndl, roughg) * smithg(ndv, roughg);
    V3<T> fsheen = fh * m.sheen * csheen;
    T trans = m.trans;
    T cos_i = std::fabs(dot(Ns, V));
    T sin2_i = T(1) - cos_i * cos_i;
    T sin2_t = eta * eta * sin2_i;
    T cos_t = T(1);
    if (sin2_t <= T(1)) cos_t = std::sqrt(T(1) - sin2_t);
    T f = fresnel(cos_i, cos_t, eta);
    V3<T> out = ((C<T>::recip_pi() * lerp(fd, ss, m.subsurface) * cdlin + fsheen) *
                 (T(1) - m.metallic)) *
                (T(1) - trans * (T(1) - f) * (T(1) - refract));
    if (trans > T(0))
        out = out + gs * ds * (T(1) - trans * (T(1) - refract) * (T(1) - f));
    else
        out = out + gs * ds * fs;
    return out;
}


// PdfDisneyBSDF, Pdf.h:42-117
template <class T> T pdf_disney(const Mat<T> &m, V3<T> Ns_, V3<T> /*Ng*/, V3<T> V, V3<T> L) {
    T trans_ratio = m.trans;
    V3<T> Ns = Ns_;
    T eta = m.eta;
    if (dot(Ns, V) < T(0)) {
        eta = T(1) / eta;
        Ns = -Ns;
    }
    T pdf = T(0);
    T ndv = std::fabs(dot(V, Ns));
    V3<T> wh = -normalize(V + L * eta);
    T spec_alpha = m.roughness;
    T cc_alpha = lerp(K(0.1), K(0.001), m.clearcoat_gloss);
    T diffuse_ratio = K(0.5) * (T(1) - m.metallic);
    T specular_ratio = T(1) - diffuse_ratio;
    V3<T> half = normalize(L + V);
    T cos_theta = std::fabs(dot(half, Ns));
    T pdf_gtr2 = gtr2(cos_theta, spec_alpha) * cos_theta;
    T pdf_gtr1 = gtr1(cos_theta, cc_alpha) * cos_theta;
    T ratio = T(1) / (T(1) + m.clearcoat);
    T pdf_spec = lerp(pdf_gtr1, pdf_gtr2, ratio) / (K(4.0) * std::fabs(dot(L, half)));
    T pdf_diff = std::fabs(dot(L, Ns)) * C<T>::recip_pi();
    T cos_i = std::fabs(dot(wh, V));
    T sin2_i = T(1) - cos_i * cos_i;
    T sin2_t = T(1) / (eta * eta) * sin2_i;
    T refract_ratio = T(0);
    T temp = (T(1) - ndv * ndv) / (eta * eta);
    if (temp < T(1)) refract_ratio = T(1) - fresnel(ndv, std::sqrt(T(1) - temp), eta);
    pdf = (diffuse_ratio * pdf_diff + specular_ratio * pdf_spec) * (T(1) - trans_ratio * refract_ratio);
    if (sin2_t <= T(1) && dot(L, wh) * dot(V, wh) < T(0)) {
        T sqrt_denom = eta * dot(L, wh) + dot(V, wh);
        T dwh_dwi = std::fabs((eta * eta * dot(L, wh)) / (sqrt_denom * sqrt_denom));
        T a = std::fmax(K(0.001), m.roughness);
        T ds = gtr2(std::fabs(dot(wh, Ns)), a);
        T pdf_trans = ds * std::fabs(dot(Ns, wh)) * dwh_dwi;
        pdf += trans_ratio * pdf_trans * refract_ratio;
    }
    cos_i = std::fabs(dot(half, V));
    sin2_i = T(1) - cos_i * cos_i;
    sin2_t = T(1) / (eta * eta) * sin2_i;
    if (sin2_t > T(1))
        pdf += (diffuse_ratio * pdf_diff + specular_ratio * pdf_spec) * trans_ratio * refract_ratio;
    return pdf;
}

// SampleUniformDisk + SampleCosineHemisphere, Sample.h:24-52
template <class T> V3<T> sample_cosine_hemisphere(V3<T> n, Rng &rng) {
    V3<T> x, y;
    onb(n, x, y);
    T r = std::sqrt(T(rng.next()));
    T theta = T(rng.next()) * C<T>::two_pi();
    T dx = r * m_cos(theta), dy = r * m_sin(theta);
    T z = std::sqrt(T(1) - dx * dx - dy * dy);
    return x * dx + y * dy + n * z;
}

// SampleDisneyBSDF, Sample.h:134-231
template <class T> V3<T> sample_disney(const Mat<T> &m, V3<T> Ns_, V3<T> /*Ng*/, V3<T> V, Rng &rng) {
    T r1 = rng.next(), r2 = rng.next(), r3 = rng.next(), r4 = rng.next();
    V3<T> Ns = Ns_;
    T eta = T(1) / m.eta;
    if (dot(Ns, V) < T(0)) {
        eta = T(1) / eta;
        Ns = -Ns;
    }
    T ndv = std::fabs(dot(Ns, V));
    T trans_ratio = m.trans;
    T transprob = rng.next();
    T refractprob = rng.next();
    T probability = rng.next();
    T diffuse_ratio = K(0.5) * (T(1) - m.metallic);
    if (transprob < trans_ratio) {
        T refract_ratio = T(0);
        T temp = (T(1) - ndv * ndv) * (eta * eta);
        if (temp < T(1)) refract_ratio = T(1) - fresnel(ndv, std::sqrt(T(1) - temp), eta);
        if (refractprob < refract_ratio) {
            V3<T> ox, oy;
            onb(Ns, ox, oy);
            T a = m.roughness;
            T phi = r3 * C<T>::two_pi();
            T cos_t = std::sqrt((T(1) - r4) / (T(1) + (a * a - T(1)) * r4));
            T sin_t = std::sqrt(T(1) - (cos_t * cos_t));
            T sin_p = m_sin(phi);
            T cos_p = m_cos(phi);
            V3<T> h(sin_t * cos_p, sin_t * sin_p, cos_t);
            h = h.x * ox + h.y * oy + h.z * Ns;
            if (dot(V, Ns) == T(0)) return -V;
            T cos_i = dot(h, V);
            T sin2_i = T(1) - cos_i * cos_i;
            T sin2_t = eta * eta * sin2_i;
            if (sin2_t <= T(1)) {
                T cos_tt = std::sqrt(T(1) - sin2_t);
                V3<T> L = normalize(eta * -V + (eta * cos_i - cos_tt) * h);
                if (cos_i < T(0)) {
                    T ldh = dot(L, h);
                    L = L - T(2) * ldh * h;
                }
                return L;
            }
            return h * T(2) * dot(h, V) - V;
        }
    }
    V3<T> ox, oy;
    onb(Ns, ox, oy);
    V3<T> dir;
    if (probability < diffuse_ratio) {
        dir = sample_cosine_hemisphere(Ns, rng);
    } else {
        T a = m.roughness;
        T phi = r1 * C<T>::two_pi();
        T cos_t = std::sqrt((T(1) - r2) / (T(1) + (a * a - T(1)) * r2));
        T sin_t = std::sqrt(T(1) - (cos_t * cos_t));
        T sin_p = m_sin(phi);
        T cos_p = m_cos(phi);
        V3<T> h(sin_t * cos_p, sin_t * sin_p, cos_t);
        h = h.z * Ns + h.x * ox + h.y * oy;
        dir = T(2) * dot(V, h) * h - V;
    }
    return dir;
}

// AceApprox, Tonemap.h:34-43 (glm::clamp keeps NaN)
V3<float> ace(V3<float> rad) {
    rad = rad * 0.6f;
    const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    V3<float> num = rad * (a * rad + b);
    V3<float> den = rad * (c * rad + d) + e;
    V3<float> q = num / den;
    auto gc = [](float v) {  // glm::clamp = min(max(v, lo), hi) with max(x,y) = x<y?y:x
        float t = (v < 0.0f) ? 0.0f : v;
        return (1.0f < t) ? 1.0f : t;
    };
    return {gc(q.x), gc(q.y), gc(q.z)};
}

// ---------------------------------------------------------------------------------------
// Watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2013), the project's definition of a
// hit: single precision, operations in exactly this order, double-precision recomputation of
// an edge function that evaluates to 0, hit when tmin < t < tmax with t = T / det.
struct RayPre {
    int kx, ky, kz;
    float sx, sy, sz;
};
RayPre ray_pre(const float d[3]) {
    float ax = std::fabs(d[0]), ay = std::fabs(d[1]), az = std::fabs(d[2]);
    int kz = (ax > ay) ? ((ax > az) ? 0 : 2) : ((ay > az) ? 1 : 2);
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    if (d[kz] < 0.0f) std::swap(kx, ky);
    RayPre p;
    p.kx = kx; p.ky = ky; p.kz = kz;
    p.sx = d[kx] / d[kz];
    p.sy = d[ky] / d[kz];
    p.sz = 1.0f / d[kz];
    return p;
}
bool tri_hit(const RayPre &p, const float o[3], const float *v0, const float *v1, const float *v2,
             float tmin, float tmax, float &t_out, float &u_out, float &v_out) {
    float A[3] = {v0[0] - o[0], v0[1] - o[1], v0[2] - o[2]};
    float B[3] = {v1[0] - o[0], v1[1] - o[1], v1[2] - o[2]};
    float Cc[3] = {v2[0] - o[0], v2[1] - o[1], v2[2] - o[2]};
    float ax = A[p.kx] - p.sx * A[p.kz], ay = A[p.ky] - p.sy * A[p.kz];
    float bx = B[p.kx] - p.sx * B[p.kz], by = B[p.ky] - p.sy * B[p.kz];
    float cx = Cc[p.kx] - p.sx * Cc[p.kz], cy = Cc[p.ky] - p.sy * Cc[p.kz];
    float U = cx * by - cy * bx;
    float V = ax * cy - ay * cx;
    float W = bx * ay - by * ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = (float)((double)cx * (double)by - (double)cy * (double)bx);
        V = (float)((double)ax * (double)cy - (double)ay * (double)cx);
        W = (float)((double)bx * (double)ay - (double)by * (double)ax);
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    float det = U + V + W;
    if (det == 0.0f) return false;
    float az = p.sz * A[p.kz], bz = p.sz * B[p.kz], cz = p.sz * Cc[p.kz];
    float T = U * az + V * bz + W * cz;
    float t = T / det;
    if (!(t > tmin && t < tmax)) return false;
    t_out = t;
    u_out = V / det;
    v_out = W / det;
    return true;
}

// FP64 version of the same test (cross-check only)
bool tri_hit_f64(const double o[3], const double d[3], const double *v0, const double *v1,
                 const double *v2, double tmin, double tmax, double &t_out) {
    double ax_ = std::fabs(d[0]), ay_ = std::fabs(d[1]), az_ = std::fabs(d[2]);
    int kz = (ax_ > ay_) ? ((ax_ > az_) ? 0 : 2) : ((ay_ > az_) ? 1 : 2);
    int kx = (kz + 1) % 3, ky = (kx + 1) % 3;
    if (d[kz] < 0) std::swap(kx, ky);
    double sx = d[kx] / d[kz], sy = d[ky] / d[kz], sz = 1.0 / d[kz];
    double A[3], B[3], Cc[3];
    for (int i = 0; i < 3; i++) { A[i] = v0[i] - o[i]; B[i] = v1[i] - o[i]; Cc[i] = v2[i] - o[i]; }
    double ax = A[kx] - sx * A[kz], ay = A[ky] - sy * A[kz];
    double bx = B[kx] - sx * B[kz], by = B[ky] - sy * B[kz];
    double cx = Cc[kx] - sx * Cc[kz], cy = Cc[ky] - sy * Cc[kz];
    double U = cx * by - cy * bx, V = ax * cy - ay * cx, W = bx * ay - by * ax;
    if ((U < 0 || V < 0 || W < 0) && (U > 0 || V > 0 || W > 0)) return false;
    double det = U + V + W;
    if (det == 0) return false;
    double T = U * sz * A[kz] + V * sz * B[kz] + W * sz * Cc[kz];
    double t = T / det;
    if (!(t > tmin && t < tmax)) return false;
    t_out = t;
    return true;
}

inline const float *vtx(const float *V, uint32_t i) { return V + 3 * (size_t)i; }

// closest hit = lexicographic minimum of (t, prim) over triangles with tmin < t < tmax
void cast_bf_one(const float *V, const uint32_t *I, uint32_t nT, const wl_ray &r, uint32_t mode,
                 wl_hit &h) {
    RayPre p = ray_pre(r.dir);
    h.t = r.tmax; h.prim = INVALID; h.u = 0; h.v = 0;
    for (uint32_t i = 0; i < nT; i++) {
        float t, u, v;
        if (!tri_hit(p, r.org, vtx(V, I[3 * i]), vtx(V, I[3 * i + 1]), vtx(V, I[3 * i + 2]), r.tmin,
                     r.tmax, t, u, v))
            continue;
        if (mode == WL_CAST_ANY) { h.prim = 0; h.t = t; return; }
        if (t < h.t || (t == h.t && i < h.prim)) { h.t = t; h.prim = i; h.u = u; h.v = v; }
    }
}

// ---------------------------------------------------------------------------------------
// 63-bit Morton codes over triangle-AABB centres (21 bits per axis, x most significant).
uint64_t expand21(uint32_t v) {
    uint64_t x = v & 0x1fffffu;
    x = (x | x << 32) & 0x1f00000000ffffULL;
    x = (x | x << 16) & 0x1f0000ff0000ffULL;
    x = (x | x << 8) & 0x100f00f00f00f00fULL;
    x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}
void centroids(const float *V, const uint32_t *I, uint32_t nT, std::vector<float> &c, float lo[3],
               float hi[3]) {
    c.resize(3 * (size_t)nT);
    for (int a = 0; a < 3; a++) { lo[a] = INFINITY; hi[a] = -INFINITY; }
    for (uint32_t i = 0; i < nT; i++) {
        for (int a = 0; a < 3; a++) {
            float p0 = V[3 * (size_t)I[3 * i] + a], p1 = V[3 * (size_t)I[3 * i + 1] + a],
                  p2 = V[3 * (size_t)I[3 * i + 2] + a];
            float mn = std::fmin(std::fmin(p0, p1), p2), mx = std::fmax(std::fmax(p0, p1), p2);
            float cc = (mn + mx) * 0.5f;
            c[3 * (size_t)i + a] = cc;
            lo[a] = std::fmin(lo[a], cc);
            hi[a] = std::fmax(hi[a], cc);
        }
    }
}
void morton63(const float *V, const uint32_t *I, uint32_t nT, uint64_t *codes) {
    std::vector<float> c;
    float lo[3], hi[3];
    centroids(V, I, nT, c, lo, hi);
    float scale[3];
    for (int a = 0; a < 3; a++) {
        float ext = hi[a] - lo[a];
        scale[a] = ext > 0.0f ? 2097152.0f / ext : 0.0f;
    }
    for (uint32_t i = 0; i < nT; i++) {
        uint32_t q[3];
        for (int a = 0; a < 3; a++) {
            float f = (c[3 * (size_t)i + a] - lo[a]) * scale[a];
            f = std::fmin(std::fmax(f, 0.0f), 2097151.0f);
            q[a] = (uint32_t)f;
        }
        codes[i] = (expand21(q[0]) << 2) | (expand21(q[1]) << 1) | expand21(q[2]);
    }
}

// Karras 2012 ("Maximizing parallelism in the construction of BVHs, octrees and k-d trees"):
// internal nodes 0..n-2, leaves n-1..2n-2; keys made unique by the sorted index.
struct Karras {
    const uint64_t *k;
    int n;
    int delta(int i, int j) const {
        if (j < 0 || j > n - 1) return -1;
        uint64_t a = k[i], b = k[j];
        if (a == b) return 64 + __builtin_clz((uint32_t)(i ^ j));
        return __builtin_clzll(a ^ b);
    }
    void node(int i, int &left, int &right) const {
        int d = (delta(i, i + 1) - delta(i, i - 1)) > 0 ? 1 : -1;
        int dmin = delta(i, i - d);
        int lmax = 2;
        while (delta(i, i + lmax * d) > dmin) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (delta(i, i + (l + t) * d) > dmin) l += t;
        int j = i + l * d;
        int dnode = delta(i, j);
        int s = 0;
        int div = 2;
        int t = (l + div - 1) / div;
        while (true) {
            if (delta(i, i + (s + t) * d) > dnode) s += t;
            if (t <= 1) break;
            div <<= 1;
            t = (l + div - 1) / div;
        }
        int g = i + s * d + (d < 0 ? d : 0);
        int lo = i < j ? i : j, hi = i < j ? j : i;
        left = (lo == g) ? (n - 1 + g) : g;
        right = (hi == g + 1) ? (n - 1 + g + 1) : (g + 1);
    }
};

void lbvh(const float *V, const uint32_t *I, uint32_t nT, uint32_t *sorted_prims, int32_t *left,
          int32_t *right, int32_t *parent, float *bounds) {
    std::vector<uint64_t> codes(nT);
    morton63(V, I, nT, codes.data());
    std::vector<uint32_t> idx(nT);
    for (uint32_t i = 0; i < nT; i++) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) {
        return codes[a] < codes[b] || (codes[a] == codes[b] && a < b);
    });
    std::vector<uint64_t> sk(nT);
    for (uint32_t i = 0; i < nT; i++) { sk[i] = codes[idx[i]]; sorted_prims[i] = idx[i]; }
    int n = (int)nT;
    int total = 2 * n - 1;
    for (int i = 0; i < total; i++) parent[i] = -1;
    Karras kr{sk.data(), n};
    for (int i = 0; i < n - 1; i++) {
        int l, r;
        kr.node(i, l, r);
        left[i] = l; right[i] = r;
        parent[l] = i; parent[r] = i;
    }
    if (!bounds) return;
    // leaf boxes then internal boxes bottom-up (children before parents: process by depth)
    for (int i = 0; i < n; i++) {
        uint32_t pr = idx[i];
        float *b = bounds + 6 * (size_t)(n - 1 + i);
        for (int a = 0; a < 3; a++) {
            float p0 = V[3 * (size_t)I[3 * pr] + a], p1 = V[3 * (size_t)I[3 * pr + 1] + a],
                  p2 = V[3 * (size_t)I[3 * pr + 2] + a];
            b[a] = std::fmin(std::fmin(p0, p1), p2);
            b[3 + a] = std::fmax(std::fmax(p0, p1), p2);
        }
    }
    // post-order via explicit stack from the root (node 0)
    if (n < 2) return;
    std::vector<int> order;
    order.reserve(n);
    std::vector<int> st{0};
    while (!st.empty()) {
        int x = st.back(); st.pop_back();
        order.push_back(x);
        if (left[x] < n - 1) st.push_back(left[x]);
        if (right[x] < n - 1) st.push_back(right[x]);
    }
    for (auto it = order.rbegin(); it != order.rend(); ++it) {
        int x = *it;
        float *b = bounds + 6 * (size_t)x, *bl = bounds + 6 * (size_t)left[x],
              *br = bounds + 6 * (size_t)right[x];
        for (int a = 0; a < 3; a++) {
            b[a] = std::fmin(bl[a], br[a]);
            b[3 + a] = std::fmax(bl[3 + a], br[3 + a]);
        }
    }
}

// ---------------------------------------------------------------------------------------
// CPU BVH for the oracle: binary, binned SAH (16 bins), <= 4 triangles per leaf. Box tests are
// done in double with a relative pad so they never reject a triangle the FP32 test accepts;
// closest-hit results therefore equal the brute-force definition above.
struct OBvh {
    struct Node { float lo[3], hi[3]; int left, count; };  // count>0: leaf at prims[left..]
    std::vector<Node> nodes;
    std::vector<uint32_t> prims;
    const float *V = nullptr;
    const uint32_t *I = nullptr;
    std::vector<float> tv;  // triangle vertices in prim order (9 floats)
};
void tri_box(const float *V, const uint32_t *I, uint32_t t, float lo[3], float hi[3]) {
    for (int a = 0; a < 3; a++) {
        float p0 = V[3 * (size_t)I[3 * t] + a], p1 = V[3 * (size_t)I[3 * t + 1] + a],
              p2 = V[3 * (size_t)I[3 * t + 2] + a];
        lo[a] = std::fmin(std::fmin(p0, p1), p2);
        hi[a] = std::fmax(std::fmax(p0, p1), p2);
    }
}
float half_area(const float lo[3], const float hi[3]) {
    float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    if (dx < 0) return 0;
    return dx * dy + dy * dz + dz * dx;
}
void obvh_build(OBvh &b, const std::vector<float> &tlo, const std::vector<float> &thi,
                const std::vector<float> &tc, uint32_t begin, uint32_t end, int node) {
    auto &nd = b.nodes[node];
    for (int a = 0; a < 3; a++) { nd.lo[a] = INFINITY; nd.hi[a] = -INFINITY; }
    float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = begin; i < end; i++) {
        uint32_t t = b.prims[i];
        for (int a = 0; a < 3; a++) {
            nd.lo[a] = std::fmin(nd.lo[a], tlo[3 * t + a]);
            nd.hi[a] = std::fmax(nd.hi[a], thi[3 * t + a]);
            clo[a] = std::fmin(clo[a], tc[3 * t + a]);
            chi[a] = std::fmax(chi[a], tc[3 * t + a]);
        }
    }
    uint32_t cnt = end - begin;
    if (cnt <= 4) { nd.left = (int)begin; nd.count = (int)cnt; return; }
    const int NB = 16;
    float best = INFINITY; int bax = -1, bsplit = -1;
    for (int a = 0; a < 3; a++) {
        float ext = chi[a] - clo[a];
        if (!(ext > 0)) continue;
        float blo[NB][3], bhi[NB][3]; int bc[NB] = {0};
        for (int k = 0; k < NB; k++) for (int q = 0; q < 3; q++) { blo[k][q] = INFINITY; bhi[k][q] = -INFINITY; }
        for (uint32_t i = begin; i < end; i++) {
            uint32_t t = b.prims[i];
            int k = (int)((tc[3 * t + a] - clo[a]) / ext * NB); if (k >= NB) k = NB - 1;
            bc[k]++;
            for (int q = 0; q < 3; q++) { blo[k][q] = std::fmin(blo[k][q], tlo[3 * t + q]); bhi[k][q] = std::fmax(bhi[k][q], thi[3 * t + q]); }
        }
        float rlo[NB][3], rhi[NB][3]; int rc[NB];
        float alo[3] = {INFINITY, INFINITY, INFINITY}, ahi[3] = {-INFINITY, -INFINITY, -INFINITY}; int ac = 0;
        for (int k = NB - 1; k >= 1; k--) {
            for (int q = 0; q < 3; q++) { alo[q] = std::fmin(alo[q], blo[k][q]); ahi[q] = std::fmax(ahi[q], bhi[k][q]); }
            ac += bc[k];
            for (int q = 0; q < 3; q++) { rlo[k][q] = alo[q]; rhi[k][q] = ahi[q]; }
            rc[k] = ac;
        }
        float llo[3] = {INFINITY, INFINITY, INFINITY}, lhi[3] = {-INFINITY, -INFINITY, -INFINITY}; int lc = 0;
        for (int k = 0; k < NB - 1; k++) {
            for (int q = 0; q < 3; q++) { llo[q] = std::fmin(llo[q], blo[k][q]); lhi[q] = std::fmax(lhi[q], bhi[k][q]); }
            lc += bc[k];
            if (lc == 0 || rc[k + 1] == 0) continue;
            float cost = half_area(llo, lhi) * lc + half_area(rlo[k + 1], rhi[k + 1]) * rc[k + 1];
            if (cost < best) { best = cost; bax = a; bsplit = k; }
        }
    }
    uint32_t mid;
    if (bax < 0) {
        mid = begin + cnt / 2;
    } else {
        float ext = chi[bax] - clo[bax];
        auto it = std::partition(b.prims.begin() + begin, b.prims.begin() + end, [&](uint32_t t) {
            int k = (int)((tc[3 * t + bax] - clo[bax]) / ext * NB); if (k >= NB) k = NB - 1;
            return k <= bsplit;
        });
        mid = (uint32_t)(it - b.prims.begin());
        if (mid == begin || mid == end) mid = begin + cnt / 2;
    }
    int l = (int)b.nodes.size();
    b.nodes.push_back({});
    b.nodes.push_back({});
    b.nodes[node].left = l;
    b.nodes[node].count = 0;
    obvh_build(b, tlo, thi, tc, begin, mid, l);
    obvh_build(b, tlo, thi, tc, mid, end, l + 1);
}
OBvh *obvh_create(const float *V, const uint32_t *I, uint32_t nT) {
    OBvh *b = new OBvh();
    b->V = V; b->I = I;
    if (nT == 0) return b;
    std::vector<float> tlo(3 * (size_t)nT), thi(3 * (size_t)nT), tc(3 * (size_t)nT);
    for (uint32_t t = 0; t < nT; t++) {
        tri_box(V, I, t, &tlo[3 * t], &thi[3 * t]);
        for (int a = 0; a < 3; a++) tc[3 * t + a] = 0.5f * (tlo[3 * t + a] + thi[3 * t + a]);
    }
    b->prims.resize(nT);
    for (uint32_t i = 0; i < nT; i++) b->prims[i] = i;
    b->nodes.reserve(2 * (size_t)nT);
    b->nodes.push_back({});
    obvh_build(*b, tlo, thi, tc, 0, nT, 0);
    b->tv.resize(9 * (size_t)nT);
    for (uint32_t i = 0; i < nT; i++) {
        uint32_t t = b->prims[i];
        for (int k = 0; k < 3; k++)
            for (int a = 0; a < 3; a++) b->tv[9 * (size_t)i + 3 * k + a] = V[3 * (size_t)I[3 * t + k] + a];
    }
    return b;
}
bool box_hit(const OBvh::Node &nd, const double o[3], const double id[3], double tmin, double tmax) {
    double t0 = tmin, t1 = tmax;
    for (int a = 0; a < 3; a++) {
        double pad = 1e-6 * (std::fabs((double)nd.lo[a]) + std::fabs((double)nd.hi[a])) + 1e-30;
        double lo = nd.lo[a] - pad, hi = nd.hi[a] + pad;
        double ta = (lo - o[a]) * id[a], tb = (hi - o[a]) * id[a];
        if (ta != ta) ta = -INFINITY;  // 0 * inf: origin on the slab plane, parallel ray
        if (tb != tb) tb = INFINITY;
        double tn = std::fmin(ta, tb), tf = std::fmax(ta, tb);
        t0 = std::fmax(t0, tn);
        t1 = std::fmin(t1, tf);
    }
    return t0 <= t1 * (1.0 + 1e-9);
}
void obvh_cast_one(const OBvh &b, const wl_ray &r, uint32_t mode, wl_hit &h) {
    h.t = r.tmax; h.prim = INVALID; h.u = 0; h.v = 0;
    if (b.nodes.empty()) return;
    RayPre p = ray_pre(r.dir);
    double o[3] = {r.org[0], r.org[1], r.org[2]};
    double id[3];
    for (int a = 0; a < 3; a++) id[a] = 1.0 / (double)r.dir[a];
    int st[128]; int sp = 0;
    st[sp++] = 0;
    while (sp) {
        const OBvh::Node &nd = b.nodes[st[--sp]];
        if (!box_hit(nd, o, id, (double)r.tmin * 0.999 - 1e-30, (double)h.t * 1.000001 + 1e-30)) continue;
        if (nd.count > 0) {
            for (int i = nd.left; i < nd.left + nd.count; i++) {
                const float *tv = &b.tv[9 * (size_t)i];
                float t, u, v;
                if (!tri_hit(p, r.org, tv, tv + 3, tv + 6, r.tmin, r.tmax, t, u, v)) continue;
                uint32_t prim = b.prims[i];
                if (mode == WL_CAST_ANY) { h.prim = 0; h.t = t; return; }
                if (t < h.t || (t == h.t && prim < h.prim)) { h.t = t; h.prim = prim; h.u = u; h.v = v; }
            }
        } else {
            st[sp++] = nd.left;
            st[sp++] = nd.left + 1;
        }
    }
}

// ---------------------------------------------------------------------------------------
// The path tracer: PathTracing.cu:40-288 restated over the flattened scene.
struct SceneView {
    const or_scene *s;
    std::vector<uint32_t> tri_light;
    const OBvh *bvh;
    // WL_LIGHTS_POWER: emissive triangles in light order, their FP64 CDF and each light's area
    // pdf lum(L) / total (float and double)
    std::vector<uint32_t> emit_tri;
    std::vector<double> emit_cdf;
    std::vector<float> pdf_power;
    std::vector<double> pdf_power64;
};

// The emitter CDF in the device's order (pt_strict.cu, k_emit_*): weights area * luminance(L),
// chunks of 256 summed sequentially, chunk sums sequentially, cdf = (local + offset) / total.
void build_emit_cdf(SceneView &sv) {
    const or_scene *s = sv.s;
    std::vector<uint32_t> emit_light;
    for (uint32_t l = 0; l < s->nLight; l++)
        for (uint32_t t = 0; t < s->lights[l].tri_count; t++) {
            sv.emit_tri.push_back(s->lights[l].first_tri + t);
            emit_light.push_back(l);
        }
    const size_t n = sv.emit_tri.size();
    auto lum = [&](uint32_t l) {
        const float *L = s->lights[l].L;
        return 0.2126 * (double)L[0] + 0.7152 * (double)L[1] + 0.0722 * (double)L[2];
    };
    sv.emit_cdf.assign(n, 0.0);
    const size_t CH = 256, chunks = (n + CH - 1) / CH;
    std::vector<double> chunk(chunks + 1, 0.0);
    for (size_t c = 0; c < chunks; c++) {
        double acc = 0.0;
        for (size_t i = c * CH; i < std::min(n, (c + 1) * CH); i++) {
            const uint32_t *t = s->I + 3 * (size_t)sv.emit_tri[i];
            const float *a = s->V + 3 * (size_t)t[0], *b = s->V + 3 * (size_t)t[1], *cc = s->V + 3 * (size_t)t[2];
            double ax = a[0], ay = a[1], az = a[2];
            double e1x = b[0] - ax, e1y = b[1] - ay, e1z = b[2] - az;
            double e2x = cc[0] - ax, e2y = cc[1] - ay, e2z = cc[2] - az;
            double cx = e1y * e2z - e1z * e2y, cy = e1z * e2x - e1x * e2z, cz = e1x * e2y - e1y * e2x;
            double area = 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
            acc = acc + area * lum(emit_light[i]);
            sv.emit_cdf[i] = acc;
        }
        chunk[c] = acc;
    }
    double off = 0.0;
    for (size_t c = 0; c < chunks; c++) {
        double v = chunk[c];
        chunk[c] = off;
        off = off + v;
    }
    for (size_t i = 0; i < n; i++) sv.emit_cdf[i] = off > 0.0 ? (sv.emit_cdf[i] + chunk[i / CH]) / off : 0.0;
    sv.pdf_power.assign(s->nLight, 0.0f);
    sv.pdf_power64.assign(s->nLight, 0.0);
    for (uint32_t l = 0; l < s->nLight; l++) {
        sv.pdf_power64[l] = off > 0.0 ? lum(l) / off : 0.0;
        sv.pdf_power[l] = (float)sv.pdf_power64[l];
    }
}

template <class T> T power_pdf(const SceneView &sv, uint32_t l);
template <> float power_pdf<float>(const SceneView &sv, uint32_t l) { return sv.pdf_power[l]; }
template <> double power_pdf<double>(const SceneView &sv, uint32_t l) { return sv.pdf_power64[l]; }

template <class T> V3<T> vload(const float *p, uint32_t i) {
    return V3<T>(p[3 * (size_t)i], p[3 * (size_t)i + 1], p[3 * (size_t)i + 2]);
}
inline bool tri_has_normal(const or_scene *s, uint32_t t) {
    if (!s->N) return false;
    return s->tri_flags ? (s->tri_flags[t] & 1u) != 0 : true;
}

template <class T>
T tri_area(const or_scene *s, uint32_t t) {  // GetTriangleArea, Common.h:59-62
    V3<T> a = vload<T>(s->V, s->I[3 * t]), b = vload<T>(s->V, s->I[3 * t + 1]),
          c = vload<T>(s->V, s->I[3 * t + 2]);
    return K(0.5) * length(cross(b - a, c - a));
}

// SampleAreaLightPos, Sample.h:105-132 (uniform light, uniform triangle, uniform area).
// The light-normal interpolation keeps the reference's weights: Barycentric(n0, n1, n2, coord)
// with coord = (1-u-v, u, v) reads coord.x and coord.y (Common.h:40-51).
template <class T>
void sample_light(const SceneView &sv, Rng &rng, V3<T> &pos, V3<T> &N, T &pdf, uint32_t &lid,
                  bool power = false) {
    const or_scene *s = sv.s;
    uint32_t idx, t;
    T p;
    if (power) {
        // an emissive triangle from the FP64 CDF (first entry above the random number)
        const double target = (double)rng.next();
        size_t lo = 0, hi = sv.emit_cdf.size() - 1;
        while (lo < hi) {
            size_t mid = (lo + hi) >> 1;
            if (sv.emit_cdf[mid] > target) hi = mid;
            else lo = mid + 1;
        }
        t = sv.emit_tri[lo];
        idx = sv.tri_light[t];
        p = power_pdf<T>(sv, idx);
    } else {
        idx = (uint32_t)((float)s->nLight * rng.next());
        if (idx >= s->nLight) idx = s->nLight - 1;
        const wl_area_light &lt0 = s->lights[idx];
        p = T(1) / T(s->nLight);
        uint32_t tri = (uint32_t)(rng.next() * (float)lt0.tri_count);
        if (tri >= lt0.tri_count) tri = lt0.tri_count - 1;
        p = p / T(lt0.tri_count);
        t = lt0.first_tri + tri;
    }
    const wl_area_light &lt = s->lights[idx];
    V3<T> v0 = vload<T>(s->V, s->I[3 * t]), v1 = vload<T>(s->V, s->I[3 * t + 1]),
          v2 = vload<T>(s->V, s->I[3 * t + 2]);
    T u = rng.next(), v = rng.next();
    if (u + v > T(1)) { u = T(1) - u; v = T(1) - v; }
    V3<T> coord(T(1) - u - v, u, v);
    pos = v0 + u * (v1 - v0) + v * (v2 - v0);
    if (!power) p = p / tri_area<T>(s, t);
    if (tri_has_normal(s, lt.first_tri)) {
        V3<T> n0 = vload<T>(s->N, s->I[3 * t]), n1 = vload<T>(s->N, s->I[3 * t + 1]),
              n2 = vload<T>(s->N, s->I[3 * t + 2]);
        V3<T> nn = n0 * (T(1) - coord.x - coord.y) + n1 * coord.x + n2 * coord.y;
        N = normalize(nn);
    } else {
        N = normalize(cross(v1 - v0, v2 - v0));
    }
    pdf = p;
    lid = idx;
}

// Texture colour of a hit (PathTracing.cu:262-268): interpolated texture coordinates
// (BarycentricByIndices, Common.h:40-51) and a bilinear, wrapping, normalised RGBA8 read with the
// texture unit's documented arithmetic (coordinates u W - 0.5, weights with 8 fractional bits),
// in FP32 as the GPU's strict mode computes it.
V3<float> tex_color(const or_scene *s, uint32_t prim, float bu, float bv) {
    int32_t t = s->mats[s->tri_material[prim]].texture;
    if (t < 0 || (uint32_t)t >= s->nTex || !s->UV) return V3<float>(1.0f);
    const float *a = s->UV + 2 * (size_t)s->I[3 * prim], *b = s->UV + 2 * (size_t)s->I[3 * prim + 1],
                *c = s->UV + 2 * (size_t)s->I[3 * prim + 2];
    float w0 = 1.0f - bu - bv;
    float tu = a[0] * w0 + b[0] * bu + c[0] * bv;
    float tv = a[1] * w0 + b[1] * bu + c[1] * bv;
    const int W = (int)s->tex_w[t], H = (int)s->tex_h[t];
    const uint32_t *px = s->tex_rgba[t];
    float x = (tu - std::floor(tu)) * (float)W - 0.5f;
    float y = (tv - std::floor(tv)) * (float)H - 0.5f;
    float fx = std::floor(x), fy = std::floor(y);
    float al = (float)(int)((x - fx) * 256.0f + 0.5f) * (1.0f / 256.0f);
    float be = (float)(int)((y - fy) * 256.0f + 0.5f) * (1.0f / 256.0f);
    int i0 = (int)fx, j0 = (int)fy;
    i0 = ((i0 % W) + W) % W;
    j0 = ((j0 % H) + H) % H;
    int i1 = i0 + 1 == W ? 0 : i0 + 1, j1 = j0 + 1 == H ? 0 : j0 + 1;
    uint32_t p00 = px[(size_t)j0 * W + i0], p10 = px[(size_t)j0 * W + i1];
    uint32_t p01 = px[(size_t)j1 * W + i0], p11 = px[(size_t)j1 * W + i1];
    float w00 = (1.0f - al) * (1.0f - be), w10 = al * (1.0f - be), w01 = (1.0f - al) * be, w11 = al * be;
    float o[3];
    for (int k = 0; k < 3; k++) {
        float c00 = (float)((p00 >> (8 * k)) & 0xffu) / 255.0f, c10 = (float)((p10 >> (8 * k)) & 0xffu) / 255.0f;
        float c01 = (float)((p01 >> (8 * k)) & 0xffu) / 255.0f, c11 = (float)((p11 >> (8 * k)) & 0xffu) / 255.0f;
        o[k] = w00 * c00 + w10 * c10 + w01 * c01 + w11 * c11;
    }
    return V3<float>(o[0], o[1], o[2]);
}

template <class T> struct PathOut { V3<T> radiance; uint32_t segments; };

template <class T>
PathOut<T> trace_path(const SceneView &sv, const wl_camera &cam, const wl_render_params &P,
                      uint32_t px, uint32_t py, uint32_t frame) {
    const or_scene *s = sv.s;
    uint32_t pixel = P.width * py + px;
    Rng rng = make_rng(P.rng, P.seed, pixel, frame);
    PathOut<T> out;
    out.segments = 0;
    V3<T> radiance(T(0)), throughput(T(1)), last_term(T(1));
    T last_pdf = T(1);
    V3<T> last_dir, last_ns, last_ng, last_tex(T(1));
    const wl_disney *last_mat = nullptr;
    uint32_t depth = 0;
    // PinholeGenerateRay, Camera.h:28-35
    V3<T> pos(cam.pos[0], cam.pos[1], cam.pos[2]);
    V3<T> lookat(cam.look_at[0], cam.look_at[1], cam.look_at[2]);
    V3<T> right(cam.right[0], cam.right[1], cam.right[2]), up(cam.up[0], cam.up[1], cam.up[2]);
    T cu = T(2) * (T(px) + T(rng.next())) / T(P.width) - T(1);
    T cv = T(2) * (T(py) + T(rng.next())) / T(P.height) - T(1);
    V3<T> dir = normalize(lookat + right * cu + up * cv);
    const T eps = T(P.eps);
    const T env_r = T(P.env[0]), env_g = T(P.env[1]), env_b = T(P.env[2]);
    const bool has_env = P.env[0] != 0.0f || P.env[1] != 0.0f || P.env[2] != 0.0f;
    while (true) {
        // closest hit (PathTracing.cu:72-75); traversal runs in FP32 on the FP32 ray
        wl_ray ray;
        ray.org[0] = (float)pos.x; ray.org[1] = (float)pos.y; ray.org[2] = (float)pos.z;
        ray.dir[0] = (float)dir.x; ray.dir[1] = (float)dir.y; ray.dir[2] = (float)dir.z;
        ray.tmin = P.eps; ray.tmax = 1e30f;
        wl_hit hit;
        obvh_cast_one(*sv.bvh, ray, WL_CAST_CLOSEST, hit);
        out.segments++;
        if (hit.prim == INVALID) {  // __miss__radiance, PathTracing.cu:163-171
            if (has_env) radiance = radiance + throughput * last_term * V3<T>(env_r, env_g, env_b);
            break;
        }
        // __closesthit__radiance, PathTracing.cu:181-288
        depth += 1;
        uint32_t prim = hit.prim;
        V3<T> a = vload<T>(s->V, s->I[3 * prim]), b = vload<T>(s->V, s->I[3 * prim + 1]),
              c = vload<T>(s->V, s->I[3 * prim + 2]);
        V3<T> Ng = normalize(cross(b - a, c - a));
        V3<T> Ns;
        if (tri_has_normal(s, prim)) {
            T bu = T(hit.u), bv = T(hit.v);
            V3<T> n0 = vload<T>(s->N, s->I[3 * prim]), n1 = vload<T>(s->N, s->I[3 * prim + 1]),
                  n2 = vload<T>(s->N, s->I[3 * prim + 2]);
            Ns = normalize(n0 * (T(1) - bu - bv) + n1 * bu + n2 * bv);
        } else {
            Ns = Ng;
        }
        T tt = T(hit.t);
        V3<T> hit_pos = pos + dir * tt;
        uint32_t lid = sv.tri_light[prim];
        if (lid != INVALID) {
            const wl_area_light &lt = s->lights[lid];
            if (depth == 1 || (P.strategy != WL_STRATEGY_NEE && (lt.two_sided || dot(Ns, dir) < T(0)))) {
                T nee_pdf = T(0);
                if (P.strategy != WL_STRATEGY_UPT && depth > 1) {
                    // PdfAreaLightPos, Pdf.h:28-39 (or the power CDF's area pdf)
                    T lp;
                    if (P.lights == WL_LIGHTS_POWER) {
                        lp = power_pdf<T>(sv, lid);
                    } else {
                        lp = T(1) / T(s->nLight);
                        lp /= T(lt.tri_count);
                        lp /= tri_area<T>(s, prim);
                    }
                    nee_pdf = lp * tt * tt / std::fabs(dot(Ns, dir));
                }
                T upt_pdf = last_pdf;
                V3<T> L(lt.L[0], lt.L[1], lt.L[2]);
                radiance = radiance + throughput * L * last_term * (upt_pdf / (upt_pdf + nee_pdf));
            }
            break;
        }
        if (depth >= P.max_depth) break;
        const wl_disney &md = s->mats[s->tri_material[prim]];
        Mat<T> m = to_mat<T>(md);
        if (m.trans < K(0.1)) {
            if (dot(Ng, dir) > T(0)) Ng = -Ng;
            if (dot(Ns, dir) > T(0)) Ns = -Ns;
        }
        V3<T> ndir = sample_disney(m, Ns, Ng, -dir, rng);
        ndir = normalize(ndir);
        T pdf = pdf_disney(m, Ns, Ng, -dir, ndir);
        if (pdf < T(0) || std::isnan(pdf)) break;
        V3<float> tf = tex_color(s, prim, hit.u, hit.v);
        V3<T> tex(T(tf.x), T(tf.y), T(tf.z));
        throughput = throughput * last_term;
        T cosw = dot(ndir, Ns);
        V3<T> bsdf = clampv(eval_disney(m, Ns, Ng, -dir, ndir, tex), T(0), K(1e30));
        last_term = bsdf * std::fabs(cosw) / pdf;
        pos = hit_pos;
        last_dir = dir;
        last_tex = tex;
        dir = ndir;
        last_ns = Ns;
        last_ng = Ng;
        last_pdf = pdf;
        last_mat = &md;
        // next-event estimation (PathTracing.cu:81-129)
        if (P.strategy != WL_STRATEGY_UPT && s->nLight > 0) {
            V3<T> lpos, lN; T lpdf; uint32_t li;
            sample_light(sv, rng, lpos, lN, lpdf, li, P.lights == WL_LIGHTS_POWER);
            V3<T> vis = lpos - pos;
            T dist = length(vis);
            vis = vis / dist;
            wl_ray sr;
            sr.org[0] = (float)pos.x; sr.org[1] = (float)pos.y; sr.org[2] = (float)pos.z;
            sr.dir[0] = (float)vis.x; sr.dir[1] = (float)vis.y; sr.dir[2] = (float)vis.z;
            sr.tmin = P.eps;
            sr.tmax = (float)(dist * (T(1) - eps));
            wl_hit sh;
            obvh_cast_one(*sv.bvh, sr, WL_CAST_ANY, sh);
            if (sh.prim == INVALID) {
                T cos1 = dot(lN, vis);
                T cos2 = dot(last_ns, vis);
                const wl_area_light &lt = s->lights[li];
                if (lt.two_sided || cos1 < T(0)) {
                    T nee_pdf = lpdf * dist * dist / std::fabs(cos1);
                    T upt_pdf = T(0);
                    Mat<T> lm = to_mat<T>(*last_mat);
                    if (P.strategy != WL_STRATEGY_NEE) {
                        upt_pdf = pdf_disney(lm, last_ns, last_ng, -last_dir, vis);
                        if (upt_pdf < T(0) || std::isnan(upt_pdf)) upt_pdf = T(0);
                    }
                    V3<T> bv = clampv(eval_disney(lm, last_ns, last_ng, -last_dir, vis, last_tex), T(0), K(1e30));
                    V3<T> L(lt.L[0], lt.L[1], lt.L[2]);
                    radiance = radiance + throughput * bv * std::fabs(cos2) * L / nee_pdf *
                                              (T(1) - upt_pdf / (upt_pdf + nee_pdf));
                }
            }
        }
        // Russian roulette (PathTracing.cu:130-138)
        if (depth > P.rr_depth) {
            if (T(rng.next()) > T(P.rr_prob)) break;
            throughput = throughput / T(P.rr_prob);
        }
    }
    out.radiance = radiance;
    return out;
}

// Ambient occlusion, AO.cu:21-130: camera_samples camera rays per pixel; at a hit, ao_rays
// cosine-hemisphere rays (SampleCosineHemisphere with pdf, Sample.h:55-66) of length radius;
// each unoccluded ray adds dot(dir, N) / PI / ao_rays / pdf. A camera ray that misses adds 0
// (the reference would trace from the previous sample's hit point).
double ao_frame(const SceneView &sv, const wl_camera &cam, const wl_ao_params &P, uint32_t px,
               uint32_t py, uint32_t frame, uint64_t &rays) {
    const or_scene *s = sv.s;
    uint32_t pixel = P.width * py + px;
    Rng rng = make_rng(P.rng, P.seed, pixel, frame);
    double acc = 0.0;
    V3<float> lookat(cam.look_at[0], cam.look_at[1], cam.look_at[2]);
    V3<float> right(cam.right[0], cam.right[1], cam.right[2]), up(cam.up[0], cam.up[1], cam.up[2]);
    for (uint32_t k = 0; k < P.camera_samples; k++) {
        float rad = 0.0f;
        float cu = 2.f * ((float)px + rng.next()) / (float)P.width - 1.f;
        float cv = 2.f * ((float)py + rng.next()) / (float)P.height - 1.f;
        V3<float> dir = normalize(lookat + right * cu + up * cv);
        wl_ray ray = {{cam.pos[0], cam.pos[1], cam.pos[2]}, P.eps, {dir.x, dir.y, dir.z}, 1e30f};
        wl_hit hit;
        obvh_cast_one(*sv.bvh, ray, WL_CAST_CLOSEST, hit);
        rays++;
        if (hit.prim != INVALID) {
            uint32_t prim = hit.prim;
            V3<float> N;
            if (tri_has_normal(s, prim)) {
                float bu = hit.u, bv = hit.v;
                N = vload<float>(s->N, s->I[3 * prim]) * (1.0f - bu - bv) +
                    vload<float>(s->N, s->I[3 * prim + 1]) * bu + vload<float>(s->N, s->I[3 * prim + 2]) * bv;
            } else {
                V3<float> a = vload<float>(s->V, s->I[3 * prim]), b = vload<float>(s->V, s->I[3 * prim + 1]),
                          c = vload<float>(s->V, s->I[3 * prim + 2]);
                N = cross(b - a, c - a);
            }
            N = normalize(N);
            if (dot(N, dir) > 0.0f) N = -N;
            V3<float> pos = V3<float>(cam.pos[0], cam.pos[1], cam.pos[2]) + dir * hit.t;
            for (uint32_t j = 0; j < P.ao_rays; j++) {
                V3<float> x, y;
                onb(N, x, y);
                float r = std::sqrt(rng.next());
                float theta = rng.next() * C<float>::two_pi();
                float dx = r * m_cos(theta), dy = r * m_sin(theta);
                float z = std::sqrt(1.0f - dx * dx - dy * dy);
                float pdf = z / C<float>::pi();
                V3<float> od = x * dx + y * dy + N * z;
                wl_ray sr = {{pos.x, pos.y, pos.z}, P.eps, {od.x, od.y, od.z}, P.radius};
                wl_hit sh;
                obvh_cast_one(*sv.bvh, sr, WL_CAST_ANY, sh);
                rays++;
                if (sh.prim == INVALID) rad += dot(od, N) / C<float>::pi() / (float)P.ao_rays / pdf;
            }
        } else {
            for (uint32_t j = 0; j < 2 * P.ao_rays; j++) rng.next();
        }
        acc += (double)(rad / (float)P.camera_samples);
    }
    return acc;  // AO.cu keeps the frame value in double (glm::dvec4 thisFrame)
}

// ---------------------------------------------------------------------------------------
// Bidirectional path tracer: Programs/BDPT/BDPT.cu:42-567 restated over the flattened scene.
// A subpath vertex (BDPT.h BDPTVertex without the texture colour, which is 1 for every triangle
// of a flattened scene): the light vertex of the light subpath has mat == nullptr and light >= 0.
template <class T> struct BdVertex {
    V3<T> pos, ns, ng, wi, tput;
    const wl_disney *mat;
    int32_t light;
    T pdf, pdf_inv, pdf_light;
};

// ComputePdfForward (BDPT.cu:42-50): area-measure pdf of reaching `next` from `mid` by BSDF
// sampling with incoming direction wi.
template <class T> T bd_pdf_forward(V3<T> wi, const BdVertex<T> &mid, const BdVertex<T> &next) {
    V3<T> d = next.pos - mid.pos;
    T dist = length(d);
    d = d / dist;
    T p = pdf_disney(to_mat<T>(*mid.mat), mid.ns, mid.ng, wi, d);
    return clampf(p, K(1e-30), K(1e30)) * std::fabs(dot(next.ns, d)) / (dist * dist);
}

// ComputePdfLightDir (BDPT.cu:52-58): cosine emission from light vertex l towards e, area measure.
template <class T> T bd_pdf_light_dir(const BdVertex<T> &l, const BdVertex<T> &e) {
    V3<T> d = e.pos - l.pos;
    T dist = length(d);
    d = d / dist;
    return dot(d, l.ns) * C<T>::recip_pi() * std::fabs(dot(d, e.ns)) / (dist * dist);
}

// MISweight (BDPT.cu:61-217) with the reference's settings: USE_UPT, not PT_MODE, balance
// heuristic. lightEnd == -1 is the eye path that reached a light (E[eyeEnd] is the light
// vertex, Lp points at it).
template <class T>
T bd_mis_weight(const BdVertex<T> *E, const BdVertex<T> *Lp, int eyeEnd, int lightEnd) {
    const int strategies = eyeEnd + lightEnd + 1 + 1;
    T fwd[2 * WL_BDPT_MAX_VERTICES], inv[2 * WL_BDPT_MAX_VERTICES];
    int nf = 0, ni = 0;
    if (lightEnd == -1) {
        for (int i = 1; i <= eyeEnd; ++i) {
            fwd[nf++] = E[i].pdf;
            inv[ni++] = E[i].pdf_inv;
        }
    } else if (eyeEnd == 0 && lightEnd == 0) {
        const BdVertex<T> &e = E[0], &l = Lp[0];
        fwd[nf++] = bd_pdf_forward(e.wi, e, l);
        inv[ni++] = bd_pdf_light_dir(l, e);
    } else if (eyeEnd == 0) {
        const BdVertex<T> &e = E[0], &l = Lp[lightEnd], &ll = Lp[lightEnd - 1];
        V3<T> d = normalize(l.pos - e.pos);
        T p_el = bd_pdf_forward(e.wi, e, l);
        T p_le = bd_pdf_forward(l.wi, l, e);
        T p_ll = bd_pdf_forward(-d, l, ll);
        fwd[nf++] = p_el;
        inv[ni++] = p_le;
        fwd[nf++] = p_ll;
        inv[ni++] = ll.pdf_inv;
        for (int i = lightEnd - 2; i >= 0; --i) {
            fwd[nf++] = Lp[i].pdf;
            inv[ni++] = Lp[i].pdf_inv;
        }
    } else if (lightEnd == 0) {
        const BdVertex<T> &ee = E[eyeEnd - 1], &e = E[eyeEnd], &l = Lp[0];
        V3<T> d = normalize(l.pos - e.pos);
        T p_ee = bd_pdf_forward(d, e, ee);
        T p_el = bd_pdf_forward(e.wi, e, l);
        T p_le = bd_pdf_light_dir(l, e);
        for (int i = 1; i < eyeEnd; ++i) {
            fwd[nf++] = E[i].pdf;
            inv[ni++] = E[i].pdf_inv;
        }
        fwd[nf++] = e.pdf;
        inv[ni++] = p_ee;
        fwd[nf++] = p_el;
        inv[ni++] = p_le;
    } else {
        const BdVertex<T> &ee = E[eyeEnd - 1], &e = E[eyeEnd];
        const BdVertex<T> &l = Lp[lightEnd], &ll = Lp[lightEnd - 1];
        V3<T> d = normalize(l.pos - e.pos);
        T p_ee = bd_pdf_forward(d, e, ee);
        T p_el = bd_pdf_forward(e.wi, e, l);
        T p_le = bd_pdf_forward(l.wi, l, e);
        T p_ll = bd_pdf_forward(-d, l, ll);
        for (int i = 1; i < eyeEnd; ++i) {
            fwd[nf++] = E[i].pdf;
            inv[ni++] = E[i].pdf_inv;
        }
        fwd[nf++] = e.pdf;
        inv[ni++] = p_ee;
        fwd[nf++] = p_el;
        inv[ni++] = p_le;
        fwd[nf++] = p_ll;
        inv[ni++] = ll.pdf_inv;
        for (int i = lightEnd - 2; i >= 0; --i) {
            fwd[nf++] = Lp[i].pdf;
            inv[ni++] = Lp[i].pdf_inv;
        }
    }
    inv[ni++] = Lp[0].pdf_light;
    T den = T(1), tmp = T(1);
    for (int i = eyeEnd - 1; i >= 0; --i) {
        tmp *= inv[i + 1] / fwd[i];
        den += tmp;
    }
    tmp = T(1);
    for (int i = eyeEnd + 1; i < strategies; ++i) {
        tmp *= fwd[i - 1] / inv[i];
        den += tmp;
    }
    T w = T(1) / den;
    if (w < T(0) || std::isnan(w) || std::isinf(w)) return T(0);
    return w;
}

// Surface record of a closest hit (__closesthit__radiance, BDPT.cu:581-640): geometric and
// shading normals, flipped towards the ray unless the triangle is an emitter or transmissive.
template <class T> struct BdHit {
    V3<T> pos, ns, ng;
    int32_t light;
    const wl_disney *mat;
};
template <class T>
BdHit<T> bd_surface(const SceneView &sv, const wl_hit &hit, V3<T> org, V3<T> dir) {
    const or_scene *s = sv.s;
    uint32_t prim = hit.prim;
    V3<T> a = vload<T>(s->V, s->I[3 * prim]), b = vload<T>(s->V, s->I[3 * prim + 1]),
          c = vload<T>(s->V, s->I[3 * prim + 2]);
    BdHit<T> h;
    h.ng = normalize(cross(b - a, c - a));
    if (tri_has_normal(s, prim)) {
        T bu = T(hit.u), bv = T(hit.v);
        h.ns = normalize(vload<T>(s->N, s->I[3 * prim]) * (T(1) - bu - bv) +
                         vload<T>(s->N, s->I[3 * prim + 1]) * bu + vload<T>(s->N, s->I[3 * prim + 2]) * bv);
    } else {
        h.ns = h.ng;
    }
    h.pos = org + dir * T(hit.t);
    uint32_t lid = sv.tri_light[prim];
    h.light = lid == INVALID ? -1 : (int32_t)lid;
    h.mat = &s->mats[s->tri_material[prim]];
    if (h.light < 0 && to_mat<T>(*h.mat).trans < K(0.1)) {
        if (dot(h.ng, dir) > T(0)) h.ng = -h.ng;
        if (dot(h.ns, dir) > T(0)) h.ns = -h.ns;
    }
    return h;
}

template <class T> bool bd_cast(const SceneView &sv, V3<T> o, V3<T> d, float tmin, float tmax,
                                uint32_t mode, wl_hit &hit) {
    wl_ray r;
    r.org[0] = (float)o.x; r.org[1] = (float)o.y; r.org[2] = (float)o.z;
    r.dir[0] = (float)d.x; r.dir[1] = (float)d.y; r.dir[2] = (float)d.z;
    r.tmin = tmin;
    r.tmax = tmax;
    obvh_cast_one(*sv.bvh, r, mode, hit);
    return hit.prim != INVALID;
}

// TraceEyeSubpath (BDPT.cu:219-336). Returns the number of stored eye vertices; `radiance`
// receives the light reached by the eye path itself (MIS-weighted after the first bounce).
template <class T>
uint32_t bd_eye(const SceneView &sv, const wl_camera &cam, const wl_render_params &P, uint32_t px,
                uint32_t py, Rng &rng, BdVertex<T> *E, V3<T> &radiance, uint64_t &rays) {
    const or_scene *s = sv.s;
    V3<T> org(cam.pos[0], cam.pos[1], cam.pos[2]);
    V3<T> lookat(cam.look_at[0], cam.look_at[1], cam.look_at[2]);
    V3<T> right(cam.right[0], cam.right[1], cam.right[2]), up(cam.up[0], cam.up[1], cam.up[2]);
    T cu = T(2) * (T(px) + T(rng.next())) / T(P.width) - T(1);
    T cv = T(2) * (T(py) + T(rng.next())) / T(P.height) - T(1);
    V3<T> dir = normalize(lookat + right * cu + up * cv);
    uint32_t depth = 0;
    bool hit_light = false;
    T rr_k = T(1);
    while (depth < P.max_depth) {
        wl_hit hit;
        rays++;
        if (!bd_cast(sv, org, dir, P.eps, 1e30f, WL_CAST_CLOSEST, hit)) break;
        depth += 1;
        BdHit<T> h = bd_surface(sv, hit, org, dir);
        hit_light = h.light >= 0;
        const uint32_t v = depth - 1;
        BdVertex<T> &e = E[v];
        e.pos = h.pos; e.ns = h.ns; e.ng = h.ng; e.wi = -dir;
        e.mat = h.mat; e.light = h.light;
        e.pdf = T(0); e.pdf_light = T(0); e.pdf_inv = T(0);
        if (v == 0) {
            e.tput = V3<T>(T(1));
            e.pdf = T(1);
        } else {
            const BdVertex<T> &le = E[v - 1];
            Mat<T> lm = to_mat<T>(*le.mat);
            V3<T> f = eval_disney(lm, le.ns, le.ng, le.wi, dir, V3<T>(T(1)));
            T cosw = dot(dir, le.ns);
            T pdf = clampf(pdf_disney(lm, le.ns, le.ng, le.wi, dir), K(1e-30), K(1e30));
            e.tput = le.tput * clampv(f, T(0), K(1e30)) * std::fabs(cosw) / pdf * rr_k;
            V3<T> d = e.pos - le.pos;
            e.pdf = pdf * std::fabs(dot(e.wi, e.ns)) / dot(d, d);
        }
        if (v >= 2) E[v - 1].pdf_inv = bd_pdf_forward(-e.wi, E[v - 1], E[v - 2]);
        if (hit_light) {
            const wl_area_light &lt = s->lights[h.light];
            if (!lt.two_sided && dot(e.ns, dir) > T(0)) break;
            V3<T> L(lt.L[0], lt.L[1], lt.L[2]);
            if (v == 0) {
                radiance = L;
            } else {
                e.pdf_inv = bd_pdf_light_dir(e, E[v - 1]);
                // PdfAreaLightPos (Pdf.h:18-26) of the hit triangle
                T lp = T(1) / T(s->nLight);
                lp /= T(lt.tri_count);
                lp /= tri_area<T>(s, hit.prim);
                e.pdf_light = lp;
                radiance = L * e.tput * bd_mis_weight(E, &e, (int)v, -1);
            }
            break;
        }
        // Russian roulette (BDPT.cu:315-325); never reached with at most 10 vertices
        T rr_rate = clampf(K(1.2) - T(depth) * K(0.5), K(0.1), T(1));
        rr_k = T(1);
        if (depth > 10) {
            if (T(rng.next()) > rr_rate) break;
            rr_k = T(1) / rr_rate;
        }
        dir = normalize(sample_disney(to_mat<T>(*e.mat), e.ns, e.ng, e.wi, rng));
        org = e.pos;
    }
    return hit_light ? depth - 1 : depth;
}

// TraceLightSubpath (BDPT.cu:338-452). Returns the number of light-subpath vertices (the
// light vertex included).
template <class T>
uint32_t bd_light(const SceneView &sv, const wl_render_params &P, Rng &rng, BdVertex<T> *Lp,
                  uint64_t &rays) {
    const or_scene *s = sv.s;
    V3<T> lpos, lN;
    T lpdf;
    uint32_t lid;
    sample_light(sv, rng, lpos, lN, lpdf, lid);
    // SampleCosineHemisphere with pdf (Sample.h:55-66) around the light normal
    V3<T> x, y;
    onb(lN, x, y);
    T r = std::sqrt(T(rng.next()));
    T theta = T(rng.next()) * C<T>::two_pi();
    T dx = r * m_cos(theta), dy = r * m_sin(theta);
    T z = std::sqrt(T(1) - dx * dx - dy * dy);
    T dir_pdf = z / C<T>::pi();
    V3<T> dir = x * dx + y * dy + lN * z;
    BdVertex<T> &l = Lp[0];
    l.pos = lpos; l.ns = lN; l.ng = lN;
    l.mat = nullptr;
    l.pdf = T(0); l.pdf_inv = T(0); l.pdf_light = lpdf;
    l.light = (int32_t)lid;
    l.wi = V3<T>(T(0));
    const wl_area_light &lt = s->lights[lid];
    l.tput = V3<T>(lt.L[0], lt.L[1], lt.L[2]) / lpdf;
    uint32_t depth = 1;
    bool hit_light = false;
    T rr_k = T(1);
    V3<T> org = lpos;
    while (depth < P.max_depth) {
        wl_hit hit;
        rays++;
        if (!bd_cast(sv, org, dir, P.eps, 1e30f, WL_CAST_CLOSEST, hit)) break;
        depth += 1;
        BdHit<T> h = bd_surface(sv, hit, org, dir);
        if (h.light >= 0) {
            hit_light = true;
            break;
        }
        const uint32_t vi = depth - 1;
        BdVertex<T> &v = Lp[vi];
        v.pos = h.pos; v.ns = h.ns; v.ng = h.ng; v.wi = -dir;
        v.mat = h.mat; v.light = -1;
        v.pdf = T(0); v.pdf_light = T(0); v.pdf_inv = T(0);
        BdVertex<T> &lv = Lp[vi - 1];
        if (vi == 1) {
            V3<T> d = v.pos - lv.pos;
            T dist = length(d);
            d = d / dist;
            v.tput = Lp[0].tput * std::fabs(dot(d, lv.ns)) / dir_pdf * rr_k;
            lv.pdf_inv = dir_pdf * std::fabs(dot(dir, v.ns)) / (dist * dist);
        } else {
            Mat<T> lm = to_mat<T>(*lv.mat);
            V3<T> f = eval_disney(lm, lv.ns, lv.ng, lv.wi, dir, V3<T>(T(1)));
            T cosw = dot(dir, lv.ns);
            T pdf = clampf(pdf_disney(lm, lv.ns, lv.ng, lv.wi, dir), K(1e-30), K(1e30));
            v.tput = lv.tput * clampv(f, T(0), K(1e30)) * std::fabs(cosw) / pdf * rr_k;
            V3<T> d = v.pos - lv.pos;
            lv.pdf_inv = pdf * std::fabs(dot(v.wi, v.ns)) / dot(d, d);
            Lp[vi - 2].pdf = bd_pdf_forward(-v.wi, lv, Lp[vi - 2]);
        }
        T rr_rate = clampf(K(1.2) - T(depth) * K(0.5), K(0.1), T(1));
        rr_k = T(1);
        if (depth > 10) {
            if (T(rng.next()) > rr_rate) break;
            rr_k = T(1) / rr_rate;
        }
        dir = normalize(sample_disney(to_mat<T>(*v.mat), v.ns, v.ng, v.wi, rng));
        org = v.pos;
    }
    return hit_light ? depth - 1 : depth;
}

// EvalContri (BDPT.cu:455-489) without its visibility ray, which the caller casts.
template <class T> V3<T> bd_contribution(const SceneView &sv, const BdVertex<T> &e,
                                          const BdVertex<T> &l, V3<T> vis, T dist) {
    if (l.light >= 0 && !sv.s->lights[l.light].two_sided && dot(l.ns, vis) > T(0)) return V3<T>(T(0));
    V3<T> fe = eval_disney(to_mat<T>(*e.mat), e.ns, e.ng, e.wi, vis, V3<T>(T(1)));
    V3<T> c = e.tput * fe * std::fabs(dot(e.ns, vis)) * std::fabs(dot(l.ns, vis)) * l.tput /
              (dist * dist);
    if (l.light < 0) c = c * eval_disney(to_mat<T>(*l.mat), l.ns, l.ng, -vis, l.wi, V3<T>(T(1)));
    return c;
}

// One sample of __raygen__RenderFrame (BDPT.cu:522-560): the value added to the film.
// max_len > 0 restricts the estimator to the paths of at most max_len vertices after the
// camera (eye subpaths of max_len vertices, light subpaths of max_len - 1, connections with
// i + j + 2 <= max_len): the bidirectional part of a render whose radiance cache takes the
// longer paths (wl_render_nrc with WL_STRATEGY_BDPT).
template <class T>
V3<T> bd_sample(const SceneView &sv, const wl_camera &cam, const wl_render_params &P, uint32_t px,
                uint32_t py, uint32_t frame, uint64_t &rays, uint32_t max_len = 0) {
    uint32_t pixel = P.width * py + px;
    Rng rng = make_rng(P.rng, P.seed, pixel, frame);
    BdVertex<T> E[WL_BDPT_MAX_VERTICES], Lp[WL_BDPT_MAX_VERTICES];
    V3<T> radiance(T(0));
    wl_render_params PE = P, PL = P;
    if (max_len) {
        PE.max_depth = max_len;
        PL.max_depth = max_len > 1 ? max_len - 1 : 1;
    }
    uint32_t ne = bd_eye(sv, cam, PE, px, py, rng, E, radiance, rays);
    V3<T> out = V3<T>(T(0)) + radiance;
    if (ne == 0 || sv.s->nLight == 0) return out;
    uint32_t nl = bd_light(sv, PL, rng, Lp, rays);
    V3<T> conn(T(0));
    for (uint32_t i = 0; i < ne; ++i) {
        for (uint32_t j = 0; j < nl; ++j) {
            if (max_len && i + j + 2 > max_len) continue;
            const BdVertex<T> &e = E[i], &l = Lp[j];
            V3<T> vis = l.pos - e.pos;
            T dist = length(vis);
            vis = vis / dist;
            wl_hit sh;
            rays++;
            const float eps = P.eps;
            if (bd_cast(sv, e.pos, vis, eps, (float)(dist * (T(1) - T(eps))), WL_CAST_ANY, sh)) continue;
            V3<T> c = bd_contribution(sv, e, l, vis, dist);
            if (!(c.x + c.y + c.z > K(1e-10))) continue;
            conn = conn + c * bd_mis_weight(E, Lp, (int)i, (int)j);
        }
    }
    return out + conn;
}

}  // namespace

// ========================================================================================
extern "C" {

uint32_t or_tea4(uint32_t v0, uint32_t v1) { return tea4(v0, v1); }

void or_rng_stream(uint32_t rng, uint64_t seed, uint32_t pixel, uint32_t frame, uint32_t count,
                   float *out) {
    Rng r = make_rng(rng, seed, pixel, frame);
    for (uint32_t i = 0; i < count; i++) out[i] = r.next();
}

void or_lcg_stream(uint32_t state, uint32_t count, float *out) {
    Rng r;
    r.mode = WL_RNG_TEA_LCG;
    r.state = state;
    r.inc = 0;
    for (uint32_t i = 0; i < count; i++) out[i] = r.next();
}

float or_sinf(float x) { return m_sin(x); }
float or_cosf(float x) { return m_cos(x); }
float or_logf(float x) { return m_log(x); }

static V3<float> ld3(const float *p, uint32_t i) { return V3<float>(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
static void st3(float *p, uint32_t i, V3<float> v) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }

void or_disney_eval(uint32_t n, const wl_disney *mats, const float *Ns, const float *Ng,
                    const float *V, const float *L, const float *tex, float *out) {
    for (uint32_t i = 0; i < n; i++)
        st3(out, i, eval_disney(to_mat<float>(mats[i]), ld3(Ns, i), ld3(Ng, i), ld3(V, i), ld3(L, i),
                                tex ? ld3(tex, i) : V3<float>(1.f)));
}
void or_disney_pdf(uint32_t n, const wl_disney *mats, const float *Ns, const float *Ng,
                   const float *V, const float *L, float *out) {
    for (uint32_t i = 0; i < n; i++)
        out[i] = pdf_disney(to_mat<float>(mats[i]), ld3(Ns, i), ld3(Ng, i), ld3(V, i), ld3(L, i));
}
void or_disney_sample(uint32_t n, const wl_disney *mats, const float *Ns, const float *Ng,
                      const float *V, uint32_t *seeds, float *out) {
    for (uint32_t i = 0; i < n; i++) {
        Rng r; r.mode = WL_RNG_TEA_LCG; r.state = seeds[i]; r.inc = 0;
        st3(out, i, sample_disney(to_mat<float>(mats[i]), ld3(Ns, i), ld3(Ng, i), ld3(V, i), r));
        seeds[i] = (uint32_t)r.state;
    }
}
void or_camera_ray(const wl_camera *cam, uint32_t W, uint32_t H, uint32_t n, const uint32_t *px,
                   const uint32_t *py, uint32_t *seeds, float *dirs) {
    for (uint32_t i = 0; i < n; i++) {
        Rng r; r.mode = WL_RNG_TEA_LCG; r.state = seeds[i]; r.inc = 0;
        V3<float> lookat(cam->look_at[0], cam->look_at[1], cam->look_at[2]);
        V3<float> right(cam->right[0], cam->right[1], cam->right[2]), up(cam->up[0], cam->up[1], cam->up[2]);
        float u = 2.f * ((float)px[i] + r.next()) / (float)W - 1.f;
        float v = 2.f * ((float)py[i] + r.next()) / (float)H - 1.f;
        st3(dirs, i, normalize(lookat + right * u + up * v));
        seeds[i] = (uint32_t)r.state;
    }
}
void or_ace(uint32_t n, const float *rgb, float *out) {
    for (uint32_t i = 0; i < n; i++) st3(out, i, ace(ld3(rgb, i)));
}

void or_cast_bruteforce(const float *V, const uint32_t *I, uint32_t nT, const wl_ray *rays,
                        uint32_t n, uint32_t mode, wl_hit *hits) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)n; i++) cast_bf_one(V, I, nT, rays[i], mode, hits[i]);
}
void or_cast_bruteforce_f64(const float *V, const uint32_t *I, uint32_t nT, const wl_ray *rays,
                            uint32_t n, double *t_out, uint32_t *prim_out) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < (int64_t)n; i++) {
        double o[3] = {rays[i].org[0], rays[i].org[1], rays[i].org[2]};
        double d[3] = {rays[i].dir[0], rays[i].dir[1], rays[i].dir[2]};
        double best = rays[i].tmax; uint32_t bp = INVALID;
        for (uint32_t t = 0; t < nT; t++) {
            double v[3][3];
            for (int k = 0; k < 3; k++) for (int a = 0; a < 3; a++) v[k][a] = V[3 * (size_t)I[3 * t + k] + a];
            double th;
            if (tri_hit_f64(o, d, v[0], v[1], v[2], rays[i].tmin, rays[i].tmax, th) && th < best) { best = th; bp = t; }
        }
        t_out[i] = best; prim_out[i] = bp;
    }
}
void or_morton63(const float *V, const uint32_t *I, uint32_t nT, uint64_t *codes) {
    morton63(V, I, nT, codes);
}
void or_lbvh(const float *V, const uint32_t *I, uint32_t nT, uint32_t *sorted_prims,
             int32_t *left, int32_t *right, int32_t *parent, float *bounds) {
    lbvh(V, I, nT, sorted_prims, left, right, parent, bounds);
}

void *or_bvh_create(const float *V, const uint32_t *I, uint32_t nT) { return obvh_create(V, I, nT); }
void or_bvh_destroy(void *b) { delete (OBvh *)b; }
void or_cast_bvh(void *b, const wl_ray *rays, uint32_t n, uint32_t mode, wl_hit *hits) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < (int64_t)n; i++) obvh_cast_one(*(OBvh *)b, rays[i], mode, hits[i]);
}

uint64_t or_render(const or_scene *scene, void *bvh, const wl_camera *cam,
                   const wl_render_params *p, int prec, int threads, float *film_rgb,
                   double *film64, uint32_t pixel_begin, uint32_t pixel_end) {
    SceneView sv;
    sv.s = scene;
    sv.bvh = (const OBvh *)bvh;
    sv.tri_light.assign(scene->nT, INVALID);
    for (uint32_t l = 0; l < scene->nLight; l++)
        for (uint32_t t = 0; t < scene->lights[l].tri_count; t++)
            sv.tri_light[scene->lights[l].first_tri + t] = l;
    build_emit_cdf(sv);
    uint32_t npix = p->width * p->height;
    if (pixel_end > npix) pixel_end = npix;
    uint64_t segs = 0;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : segs)
    for (int64_t pix = pixel_begin; pix < (int64_t)pixel_end; pix++) {
        uint32_t px = (uint32_t)(pix % p->width), py = (uint32_t)(pix / p->width);
        float acc[3] = {0, 0, 0};
        double sum[3] = {0, 0, 0};
        if (film_rgb) for (int c = 0; c < 3; c++) acc[c] = film_rgb[3 * pix + c];
        for (uint32_t s = 0; s < p->spp; s++) {
            uint32_t f = p->first_frame + s;
            double r[3];
            if (prec == 0) {
                PathOut<float> o = trace_path<float>(sv, *cam, *p, px, py, f);
                r[0] = o.radiance.x; r[1] = o.radiance.y; r[2] = o.radiance.z;
                segs += o.segments;
            } else {
                PathOut<double> o = trace_path<double>(sv, *cam, *p, px, py, f);
                r[0] = o.radiance.x; r[1] = o.radiance.y; r[2] = o.radiance.z;
                segs += o.segments;
            }
            // a path whose radiance is not finite contributes 0 (the reference would keep a
            // NaN in its running mean for the rest of the run)
            if (!(std::isfinite(r[0]) && std::isfinite(r[1]) && std::isfinite(r[2]))) r[0] = r[1] = r[2] = 0;
            // film running mean in double, stored as float (PathTracing.cu:145-154)
            for (int c = 0; c < 3; c++) {
                float thisf = (float)r[c];
                if (f == 0) acc[c] = thisf;
                else {
                    double w0 = (double)((float)f / ((float)f + 1.0f));
                    double w1 = (double)(1.0f / ((float)f + 1.0f));
                    acc[c] = (float)((double)acc[c] * w0 + (double)thisf * w1);
                }
                sum[c] += r[c];
            }
        }
        if (film_rgb) for (int c = 0; c < 3; c++) film_rgb[3 * pix + c] = acc[c];
        if (film64) for (int c = 0; c < 3; c++) film64[3 * pix + c] = sum[c] / (double)p->spp;
    }
    return segs;
}

uint64_t or_render_ao(const or_scene *scene, void *bvh, const wl_camera *cam,
                      const wl_ao_params *p, int threads, float *film_rgb, double *film64) {
    SceneView sv;
    sv.s = scene;
    sv.bvh = (const OBvh *)bvh;
    uint32_t npix = p->width * p->height;
    uint64_t rays = 0;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : rays)
    for (int64_t pix = 0; pix < (int64_t)npix; pix++) {
        uint32_t px = (uint32_t)(pix % p->width), py = (uint32_t)(pix / p->width);
        float acc = film_rgb[3 * pix];
        double sum = 0.0;
        for (uint32_t s = 0; s < p->spp; s++) {
            uint32_t f = p->first_frame + s;
            double v = ao_frame(sv, *cam, *p, px, py, f, rays);
            if (f == 0) acc = (float)v;
            else acc = (float)((double)acc * (double)((float)f / ((float)f + 1.0f)) +
                               v * (double)(1.0f / ((float)f + 1.0f)));
            sum += v;
        }
        for (int c = 0; c < 3; c++) film_rgb[3 * pix + c] = acc;
        if (film64) for (int c = 0; c < 3; c++) film64[3 * pix + c] = sum / (double)p->spp;
    }
    return rays;
}

uint64_t or_render_bdpt(const or_scene *scene, void *bvh, const wl_camera *cam,
                        const wl_render_params *p, int prec, int threads, float *film_rgb,
                        double *film64) {
    return or_render_bdpt_len(scene, bvh, cam, p, 0, prec, threads, film_rgb, film64);
}

uint64_t or_render_bdpt_len(const or_scene *scene, void *bvh, const wl_camera *cam,
                            const wl_render_params *p, uint32_t max_len, int prec, int threads,
                            float *film_rgb, double *film64) {
    SceneView sv;
    sv.s = scene;
    sv.bvh = (const OBvh *)bvh;
    sv.tri_light.assign(scene->nT, INVALID);
    for (uint32_t l = 0; l < scene->nLight; l++)
        for (uint32_t t = 0; t < scene->lights[l].tri_count; t++)
            sv.tri_light[scene->lights[l].first_tri + t] = l;
    uint32_t npix = p->width * p->height;
    uint64_t rays = 0;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#endif
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : rays)
    for (int64_t pix = 0; pix < (int64_t)npix; pix++) {
        uint32_t px = (uint32_t)(pix % p->width), py = (uint32_t)(pix / p->width);
        float acc[3] = {0, 0, 0};
        double sum[3] = {0, 0, 0};
        if (film_rgb) for (int c = 0; c < 3; c++) acc[c] = film_rgb[3 * pix + c];
        for (uint32_t s = 0; s < p->spp; s++) {
            uint32_t f = p->first_frame + s;
            double r[3];
            if (prec == 0) {
                V3<float> o = bd_sample<float>(sv, *cam, *p, px, py, f, rays, max_len);
                r[0] = o.x; r[1] = o.y; r[2] = o.z;
            } else {
                V3<double> o = bd_sample<double>(sv, *cam, *p, px, py, f, rays, max_len);
                r[0] = o.x; r[1] = o.y; r[2] = o.z;
            }
            // a sample that is not finite contributes 0 (the reference would keep a NaN in its
            // running mean for the rest of the run)
            if (!(std::isfinite(r[0]) && std::isfinite(r[1]) && std::isfinite(r[2]))) r[0] = r[1] = r[2] = 0;
            // FP32 running mean with FP32 weights (BDPT.cu:548-556)
            for (int c = 0; c < 3; c++) {
                float thisf = (float)r[c];
                if (f == 0) acc[c] = thisf;
                else acc[c] = acc[c] * ((float)f / ((float)f + 1.0f)) + thisf * (1.0f / ((float)f + 1.0f));
                sum[c] += r[c];
            }
        }
        if (film_rgb) for (int c = 0; c < 3; c++) film_rgb[3 * pix + c] = acc[c];
        if (film64) for (int c = 0; c < 3; c++) film64[3 * pix + c] = sum[c] / (double)p->spp;
    }
    return rays;
}

double or_relmse(const float *img, const double *ref, uint64_t n, double eps) {
    double acc = 0;
    for (uint64_t i = 0; i < n; i++) {
        double d = (double)img[i] - ref[i];
        acc += d * d / (ref[i] * ref[i] + eps);
    }
    return n ? acc / (double)n : 0.0;
}

}  // extern "C"
