// glm.hpp : TEST INFRASTRUCTURE ONLY — a minimal stand-in for the GLM math library, written for
// this repository, so that the reference's sysrap headers (sphoton.h, stran.h, stra.h) compile for
// the CPU build of its qsim path (oracle/ref_cpu_sim.cc).  That path never calls into these types;
// they only need to exist for the headers' other functions.  Column-major 4x4 matrices of column
// vectors, as GLM's.  What the headers' emitted code references is defined below (glm_impl.hpp);
// the rest is declared only (an inline function that nothing calls is never emitted).
#pragma once
#include <cstddef>
#include <string>

namespace glm {

template <typename T> struct tvec4;
template <typename T> struct tvec3;

template <typename T> struct tvec2 {
    T x, y;
    tvec2();
    explicit tvec2(T s);
    tvec2(T a, T b);
    T& operator[](int i);
    const T& operator[](int i) const;
};

template <typename T> struct tvec3 {
    T x, y, z;
    tvec3();
    explicit tvec3(T s);
    tvec3(T a, T b, T c);
    explicit tvec3(const tvec4<T>& v);
    template <typename U> explicit tvec3(const tvec3<U>& v);
    T& operator[](int i);
    const T& operator[](int i) const;
    tvec3& operator+=(const tvec3& o);
    tvec3& operator-=(const tvec3& o);
    tvec3& operator*=(T s);
    tvec3& operator/=(T s);
};

template <typename T> struct tvec4 {
    T x, y, z, w;
    tvec4();
    explicit tvec4(T s);
    tvec4(T a, T b, T c, T d);
    tvec4(const tvec3<T>& v, T d);
    template <typename U> explicit tvec4(const tvec4<U>& v);
    T& operator[](int i);
    const T& operator[](int i) const;
    tvec4& operator+=(const tvec4& o);
    tvec4& operator*=(T s);
};

template <typename T> struct tmat4x4 {
    tvec4<T> c[4];
    tmat4x4();
    explicit tmat4x4(T s);
    tmat4x4(const tvec4<T>& a, const tvec4<T>& b, const tvec4<T>& c2, const tvec4<T>& d);
    template <typename U> tmat4x4(const tmat4x4<U>& m);
    tvec4<T>& operator[](int i);
    const tvec4<T>& operator[](int i) const;
    tmat4x4& operator*=(const tmat4x4& o);
};

template <typename T> struct tmat3x3 {
    tvec3<T> c[3];
    tmat3x3();
    explicit tmat3x3(T s);
    explicit tmat3x3(const tmat4x4<T>& m);
    tvec3<T>& operator[](int i);
    const tvec3<T>& operator[](int i) const;
};

template <typename T> struct tquat {
    T x, y, z, w;
    tquat();
    tquat(T w_, T x_, T y_, T z_);
};

typedef tvec2<float> vec2;
typedef tvec3<float> vec3;
typedef tvec4<float> vec4;
typedef tvec2<double> dvec2;
typedef tvec3<double> dvec3;
typedef tvec4<double> dvec4;
typedef tvec2<int> ivec2;
typedef tvec3<int> ivec3;
typedef tvec4<int> ivec4;
typedef tvec4<unsigned> uvec4;
typedef tmat4x4<float> mat4;
typedef tmat4x4<double> dmat4;
typedef tmat3x3<float> mat3;
typedef tquat<float> quat;
typedef tquat<double> dquat;

template <typename T> tvec2<T> operator+(const tvec2<T>&, const tvec2<T>&);
template <typename T> tvec2<T> operator-(const tvec2<T>&, const tvec2<T>&);
template <typename T> tvec2<T> operator*(const tvec2<T>&, T);
template <typename T> tvec2<T> operator*(T, const tvec2<T>&);
template <typename T> tvec3<T> operator+(const tvec3<T>&, const tvec3<T>&);
template <typename T> tvec3<T> operator-(const tvec3<T>&, const tvec3<T>&);
template <typename T> tvec3<T> operator-(const tvec3<T>&);
template <typename T> tvec3<T> operator*(const tvec3<T>&, const tvec3<T>&);
template <typename T> tvec3<T> operator*(const tvec3<T>&, T);
template <typename T> tvec3<T> operator*(T, const tvec3<T>&);
template <typename T> tvec3<T> operator/(const tvec3<T>&, T);
template <typename T> tvec4<T> operator+(const tvec4<T>&, const tvec4<T>&);
template <typename T> tvec4<T> operator-(const tvec4<T>&, const tvec4<T>&);
template <typename T> tvec4<T> operator*(const tvec4<T>&, T);
template <typename T> tvec4<T> operator*(T, const tvec4<T>&);
template <typename T> tvec4<T> operator/(const tvec4<T>&, T);
template <typename T> tvec4<T> operator*(const tmat4x4<T>&, const tvec4<T>&);
template <typename T> tvec4<T> operator*(const tvec4<T>&, const tmat4x4<T>&);
template <typename T> tmat4x4<T> operator*(const tmat4x4<T>&, const tmat4x4<T>&);
template <typename T> tmat4x4<T> operator*(const tmat4x4<T>&, T);
template <typename T> tmat4x4<T> operator+(const tmat4x4<T>&, const tmat4x4<T>&);
template <typename T> tmat4x4<T> operator-(const tmat4x4<T>&, const tmat4x4<T>&);
template <typename T> tvec3<T> operator*(const tmat3x3<T>&, const tvec3<T>&);
template <typename T> tquat<T> operator*(const tquat<T>&, const tquat<T>&);
template <typename T> tvec3<T> operator*(const tquat<T>&, const tvec3<T>&);
template <typename T> bool operator==(const tvec3<T>&, const tvec3<T>&);
template <typename T> bool operator!=(const tvec3<T>&, const tvec3<T>&);
template <typename T> bool operator==(const tvec4<T>&, const tvec4<T>&);
template <typename T> bool operator==(const tmat4x4<T>&, const tmat4x4<T>&);
template <typename T> bool operator!=(const tmat4x4<T>&, const tmat4x4<T>&);

template <typename V> V normalize(const V&);
template <typename V> auto length(const V&) -> decltype(V().x);
template <typename V> auto dot(const V&, const V&) -> decltype(V().x);
template <typename T> tvec3<T> cross(const tvec3<T>&, const tvec3<T>&);
template <typename M> M inverse(const M&);
template <typename M> M transpose(const M&);
template <typename V> V abs(const V&);
template <typename V> V sin(const V&);
template <typename V> V cos(const V&);
template <typename V> auto compMax(const V&) -> decltype(V().x);
template <typename V> auto compMin(const V&) -> decltype(V().x);
template <typename T> T pi();
template <typename T> T radians(T);
template <typename T> T degrees(T);
template <typename X> auto value_ptr(X& x) -> decltype(&x[0][0]);
template <typename X> auto value_ptr(const X& x) -> decltype(&x[0][0]);
template <typename T> const T* value_ptr(const tvec4<T>&);
template <typename T> T* value_ptr(tvec4<T>&);
template <typename T> const T* value_ptr(const tvec3<T>&);
template <typename T> T* value_ptr(tvec3<T>&);
template <typename T> tmat4x4<T> make_mat4x4(const T*);
template <typename T> tmat4x4<T> make_mat4(const T*);
template <typename T> tvec3<T> make_vec3(const T*);
template <typename T> tvec4<T> make_vec4(const T*);
template <typename T> tmat4x4<T> translate(const tvec3<T>&);
template <typename T> tmat4x4<T> translate(const tmat4x4<T>&, const tvec3<T>&);
template <typename T> tmat4x4<T> scale(const tvec3<T>&);
template <typename T> tmat4x4<T> scale(const tmat4x4<T>&, const tvec3<T>&);
template <typename T> tmat4x4<T> rotate(T, const tvec3<T>&);
template <typename T> tmat4x4<T> rotate(const tmat4x4<T>&, T, const tvec3<T>&);
template <typename T> tmat4x4<T> lookAt(const tvec3<T>&, const tvec3<T>&, const tvec3<T>&);
template <typename T> tmat4x4<T> ortho(T, T, T, T, T, T);
template <typename T> tmat4x4<T> frustum(T, T, T, T, T, T);
template <typename M> M identity();
template <typename T> tquat<T> angleAxis(T, const tvec3<T>&);
template <typename T> tmat4x4<T> mat4_cast(const tquat<T>&);
template <typename T> tquat<T> quat_cast(const tmat4x4<T>&);
template <typename T> tquat<T> conjugate(const tquat<T>&);
template <typename T> tquat<T> slerp(const tquat<T>&, const tquat<T>&, T);
template <typename V, typename S> V catmullRom(const V&, const V&, const V&, const V&, const S&);
template <typename X> std::string to_string(const X&);

}  // namespace glm

#include "glm_impl.hpp"
