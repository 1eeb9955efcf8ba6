// glm.hpp - project-written subset of glm 1.0.1 (MIT, g-truc/glm), restated for building the
// reference's src/Frontend/Device/*.h as host C++. Test infrastructure only (oracle/_ref).
// Semantics follow glm's published definitions: componentwise operators (vector / scalar
// divides each component), dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z, length = sqrt(dot),
// normalize(v) = v * (1 / sqrt(dot(v, v))), cross as in glm/detail/func_geometric.inl,
// clamp(x, lo, hi) = min(max(x, lo), hi) with max(a, b) = a < b ? b : a, min(a, b) = b < a ? b : a.
// mat4 is column-major (m[c] = column c); mat4 * vec4 = (m[0] v.x + m[1] v.y) + (m[2] v.z +
// m[3] v.w) as glm/detail/type_mat4x4.inl groups it; make_mat4 reads 16 floats column by column
// (glm/gtc/type_ptr.inl); transpose swaps m[i][j] and m[j][i].
#pragma once
#include <cmath>
#include <cstdint>

namespace glm {

template <class T> struct tvec2 {
    T x, y;
    tvec2() : x(0), y(0) {}
    tvec2(T a, T b) : x(a), y(b) {}
    explicit tvec2(T s) : x(s), y(s) {}
};
template <class T> struct tvec4;
template <class T> struct tvec3 {
    T x, y, z;
    tvec3() : x(0), y(0), z(0) {}
    tvec3(T a, T b, T c) : x(a), y(b), z(c) {}
    explicit tvec3(T s) : x(s), y(s), z(s) {}
    template <class U> tvec3(const tvec4<U> &v) : x((T)v.x), y((T)v.y), z((T)v.z) {}
    template <class U> explicit tvec3(const tvec3<U> &v) : x((T)v.x), y((T)v.y), z((T)v.z) {}
    tvec3 &operator+=(const tvec3 &o) { x += o.x; y += o.y; z += o.z; return *this; }
    tvec3 &operator-=(const tvec3 &o) { x -= o.x; y -= o.y; z -= o.z; return *this; }
    tvec3 &operator*=(const tvec3 &o) { x *= o.x; y *= o.y; z *= o.z; return *this; }
    tvec3 &operator*=(T s) { x *= s; y *= s; z *= s; return *this; }
    tvec3 &operator+=(T s) { x += s; y += s; z += s; return *this; }
    tvec3 &operator-=(T s) { x -= s; y -= s; z -= s; return *this; }
    tvec3 &operator/=(T s) { x /= s; y /= s; z /= s; return *this; }
};
template <class T> struct tvec4 {
    T x, y, z, w;
    tvec4() : x(0), y(0), z(0), w(0) {}
    tvec4(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
    explicit tvec4(T s) : x(s), y(s), z(s), w(s) {}
    tvec4(const tvec3<T> &v, T d) : x(v.x), y(v.y), z(v.z), w(d) {}
    template <class U> tvec4(const tvec4<U> &v) : x((T)v.x), y((T)v.y), z((T)v.z), w((T)v.w) {}
    T &operator[](int i) { return (&x)[i]; }
    const T &operator[](int i) const { return (&x)[i]; }
};

template <class T> tvec3<T> operator+(const tvec3<T> &a, const tvec3<T> &b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> tvec3<T> operator-(const tvec3<T> &a, const tvec3<T> &b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> tvec3<T> operator*(const tvec3<T> &a, const tvec3<T> &b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> tvec3<T> operator/(const tvec3<T> &a, const tvec3<T> &b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class T> tvec3<T> operator-(const tvec3<T> &a) { return {-a.x, -a.y, -a.z}; }
// scalar forms; the scalar type is taken from the vector (a double or int literal converts)
template <class T> struct ident { typedef T type; };
template <class T> tvec3<T> operator*(const tvec3<T> &a, typename ident<T>::type s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> tvec3<T> operator*(typename ident<T>::type s, const tvec3<T> &a) { return {s * a.x, s * a.y, s * a.z}; }
template <class T> tvec3<T> operator/(const tvec3<T> &a, typename ident<T>::type s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> tvec3<T> operator/(typename ident<T>::type s, const tvec3<T> &a) { return {s / a.x, s / a.y, s / a.z}; }
template <class T> tvec3<T> operator+(const tvec3<T> &a, typename ident<T>::type s) { return {a.x + s, a.y + s, a.z + s}; }
template <class T> tvec3<T> operator+(typename ident<T>::type s, const tvec3<T> &a) { return {s + a.x, s + a.y, s + a.z}; }
template <class T> tvec3<T> operator-(const tvec3<T> &a, typename ident<T>::type s) { return {a.x - s, a.y - s, a.z - s}; }
template <class T> tvec3<T> operator-(typename ident<T>::type s, const tvec3<T> &a) { return {s - a.x, s - a.y, s - a.z}; }

template <class T> tvec2<T> operator*(const tvec2<T> &a, typename ident<T>::type s) { return {a.x * s, a.y * s}; }
template <class T> tvec2<T> operator+(const tvec2<T> &a, const tvec2<T> &b) { return {a.x + b.x, a.y + b.y}; }
template <class T> tvec4<T> operator*(const tvec4<T> &a, typename ident<T>::type s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
template <class T> tvec4<T> operator+(const tvec4<T> &a, const tvec4<T> &b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }

template <class T> T dot(const tvec3<T> &a, const tvec3<T> &b) {
    tvec3<T> t = a * b;
    return t.x + t.y + t.z;
}
template <class T> tvec3<T> cross(const tvec3<T> &x, const tvec3<T> &y) {
    return {x.y * y.z - y.y * x.z, x.z * y.x - y.z * x.x, x.x * y.y - y.x * x.y};
}
template <class T> T length(const tvec3<T> &v) { return std::sqrt(dot(v, v)); }
template <class T> T inversesqrt(T x) { return static_cast<T>(1) / std::sqrt(x); }
template <class T> tvec3<T> normalize(const tvec3<T> &v) { return v * inversesqrt(dot(v, v)); }
template <class T> T gmax(T a, T b) { return a < b ? b : a; }
template <class T> T gmin(T a, T b) { return b < a ? b : a; }
template <class T> tvec3<T> clamp(const tvec3<T> &v, typename ident<T>::type lo, typename ident<T>::type hi) {
    return {gmin(gmax(v.x, lo), hi), gmin(gmax(v.y, lo), hi), gmin(gmax(v.z, lo), hi)};
}
template <class T> tvec4<T> clamp(const tvec4<T> &v, typename ident<T>::type lo, typename ident<T>::type hi) {
    return {gmin(gmax(v.x, lo), hi), gmin(gmax(v.y, lo), hi), gmin(gmax(v.z, lo), hi), gmin(gmax(v.w, lo), hi)};
}

// ---- the matrix part the reference's frontend uses (SceneManager, Shape, Camera) ----------
template <class T> tvec4<T> operator*(const tvec4<T> &a, const tvec4<T> &b) { return {a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w}; }
template <class T> tvec4<T> operator*(typename ident<T>::type s, const tvec4<T> &a) { return {s * a.x, s * a.y, s * a.z, s * a.w}; }
// dot of 4-vectors as glm's compute_dot: (x + y) + (z + w) of the componentwise product
template <class T> T dot(const tvec4<T> &a, const tvec4<T> &b) {
    tvec4<T> t = a * b;
    return (t.x + t.y) + (t.z + t.w);
}
template <class T> tvec4<T> normalize(const tvec4<T> &v) { return v * inversesqrt(dot(v, v)); }
template <class T> T tan(T x) { return std::tan(x); }
// column-major 4x4: m[c] is column c
template <class T> struct tmat4 {
    tvec4<T> c[4];
    tvec4<T> &operator[](int i) { return c[i]; }
    const tvec4<T> &operator[](int i) const { return c[i]; }
};
// m * v as glm's mat4x4 * vec4: (m0 v.x + m1 v.y) + (m2 v.z + m3 v.w), each product componentwise
template <class T> tvec4<T> operator*(const tmat4<T> &m, const tvec4<T> &v) {
    const tvec4<T> a = m[0] * v.x + m[1] * v.y;
    const tvec4<T> b = m[2] * v.z + m[3] * v.w;
    return a + b;
}
template <class T> tmat4<T> transpose(const tmat4<T> &m) {
    tmat4<T> r;
    for (int i = 0; i < 4; i++) r[i] = tvec4<T>(m[0][i], m[1][i], m[2][i], m[3][i]);
    return r;
}
template <class T> tmat4<T> make_mat4(const T *p) {
    tmat4<T> r;
    for (int i = 0; i < 4; i++) r[i] = tvec4<T>(p[4 * i], p[4 * i + 1], p[4 * i + 2], p[4 * i + 3]);
    return r;
}
template <class T> tvec3<T> make_vec3(const T *p) { return tvec3<T>(p[0], p[1], p[2]); }
template <class T> tvec2<T> make_vec2(const T *p) { return tvec2<T>(p[0], p[1]); }

typedef tvec2<float> vec2;
typedef tvec3<float> vec3;
typedef tvec4<float> vec4;
typedef tvec4<double> dvec4;
typedef tvec2<int> ivec2;
typedef tvec3<int> ivec3;
typedef tvec4<uint8_t> u8vec4;
typedef tmat4<float> mat4;

}  // namespace glm
