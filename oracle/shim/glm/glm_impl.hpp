// glm_impl.hpp : TEST INFRASTRUCTURE ONLY — definitions of the parts of the glm.hpp stand-in that
// the reference headers' emitted functions reference (vector access and arithmetic, the 4x4
// matrix products, transpose, inverse by cofactors, translate/scale/rotate), written for this
// repository.
#pragma once
#include <cmath>

namespace glm {

template <typename T> tvec3<T>::tvec3() : x(0), y(0), z(0) {}
template <typename T> tvec3<T>::tvec3(T s) : x(s), y(s), z(s) {}
template <typename T> tvec3<T>::tvec3(T a, T b, T c) : x(a), y(b), z(c) {}
template <typename T> tvec3<T>::tvec3(const tvec4<T>& v) : x(v.x), y(v.y), z(v.z) {}
template <typename T> T& tvec3<T>::operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
template <typename T> const T& tvec3<T>::operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
template <typename T> tvec4<T>::tvec4() : x(0), y(0), z(0), w(0) {}
template <typename T> tvec4<T>::tvec4(T s) : x(s), y(s), z(s), w(s) {}
template <typename T> tvec4<T>::tvec4(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
template <typename T> tvec4<T>::tvec4(const tvec3<T>& v, T d) : x(v.x), y(v.y), z(v.z), w(d) {}
template <typename T> T& tvec4<T>::operator[](int i) { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }
template <typename T> const T& tvec4<T>::operator[](int i) const { return i == 0 ? x : (i == 1 ? y : (i == 2 ? z : w)); }

template <typename T> tmat4x4<T>::tmat4x4() : tmat4x4(T(1)) {}
template <typename T> tmat4x4<T>::tmat4x4(T s)
{
    for (int i = 0; i < 4; i++) for (int j = 0; j < 4; j++) c[i][j] = i == j ? s : T(0);
}
template <typename T> tmat4x4<T>::tmat4x4(const tvec4<T>& a, const tvec4<T>& b, const tvec4<T>& c2, const tvec4<T>& d)
{
    c[0] = a; c[1] = b; c[2] = c2; c[3] = d;
}
template <typename T> template <typename U> tmat4x4<T>::tmat4x4(const tmat4x4<U>& m)
{
    for (int i = 0; i < 4; i++) for (int j = 0; j < 4; j++) c[i][j] = T(m[i][j]);
}
template <typename T> tvec4<T>& tmat4x4<T>::operator[](int i) { return c[i]; }
template <typename T> const tvec4<T>& tmat4x4<T>::operator[](int i) const { return c[i]; }

template <typename T> tvec3<T> operator-(const tvec3<T>& a, const tvec3<T>& b) { return tvec3<T>(a.x - b.x, a.y - b.y, a.z - b.z); }
template <typename T> tvec3<T> operator-(const tvec3<T>& a) { return tvec3<T>(-a.x, -a.y, -a.z); }
template <typename T> tvec4<T> operator*(const tmat4x4<T>& m, const tvec4<T>& v)
{
    tvec4<T> r(T(0));
    for (int i = 0; i < 4; i++) for (int j = 0; j < 4; j++) r[j] += m[i][j] * v[i];
    return r;
}
template <typename T> tmat4x4<T> operator*(const tmat4x4<T>& a, const tmat4x4<T>& b)
{
    tmat4x4<T> r(T(0));
    for (int i = 0; i < 4; i++) r[i] = a * b[i];
    return r;
}
template <typename T> tmat4x4<T>& tmat4x4<T>::operator*=(const tmat4x4& o) { *this = *this * o; return *this; }

template <typename V> auto dot(const V& a, const V& b) -> decltype(V().x)
{
    decltype(V().x) s = 0;
    for (int i = 0; i < (int)(sizeof(V) / sizeof(a.x)); i++) s += a[i] * b[i];
    return s;
}
template <typename T> tvec3<T> cross(const tvec3<T>& a, const tvec3<T>& b)
{
    return tvec3<T>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <typename V> V normalize(const V& a)
{
    const auto l = std::sqrt(dot(a, a));
    V r = a;
    for (int i = 0; i < (int)(sizeof(V) / sizeof(a.x)); i++) r[i] = a[i] / l;
    return r;
}
template <typename V> V abs(const V& a)
{
    V r = a;
    for (int i = 0; i < (int)(sizeof(V) / sizeof(a.x)); i++) r[i] = std::abs(a[i]);
    return r;
}
template <typename T> T pi() { return T(3.14159265358979323846); }
template <typename M> M transpose(const M& m)
{
    M r;
    for (int i = 0; i < 4; i++) for (int j = 0; j < 4; j++) r[i][j] = m[j][i];
    return r;
}
// inverse of a 4x4 matrix by Gauss-Jordan elimination with partial pivoting (identity if singular)
template <typename M> M inverse(const M& m)
{
    double a[4][8];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) { a[i][j] = (double)m[j][i]; a[i][4 + j] = i == j ? 1.0 : 0.0; }
    for (int col = 0; col < 4; col++) {
        int piv = col;
        for (int r = col + 1; r < 4; r++) if (std::fabs(a[r][col]) > std::fabs(a[piv][col])) piv = r;
        if (a[piv][col] == 0.0) return M();
        if (piv != col) for (int j = 0; j < 8; j++) { const double t = a[col][j]; a[col][j] = a[piv][j]; a[piv][j] = t; }
        const double inv = 1.0 / a[col][col];
        for (int j = 0; j < 8; j++) a[col][j] *= inv;
        for (int r = 0; r < 4; r++) {
            if (r == col) continue;
            const double f = a[r][col];
            for (int j = 0; j < 8; j++) a[r][j] -= f * a[col][j];
        }
    }
    M r;
    for (int i = 0; i < 4; i++) for (int j = 0; j < 4; j++) r[j][i] = a[i][4 + j];
    return r;
}
template <typename X> auto value_ptr(X& x) -> decltype(&x[0][0]) { return &x[0][0]; }
template <typename X> auto value_ptr(const X& x) -> decltype(&x[0][0]) { return &x[0][0]; }
template <typename T> T* value_ptr(tvec4<T>& v) { return &v.x; }
template <typename T> T* value_ptr(tvec3<T>& v) { return &v.x; }
template <typename T> tmat4x4<T> make_mat4x4(const T* p)
{
    tmat4x4<T> r;
    for (int i = 0; i < 4; i++) for (int j = 0; j < 4; j++) r[i][j] = p[4 * i + j];
    return r;
}
template <typename T> tmat4x4<T> translate(const tmat4x4<T>& m, const tvec3<T>& v)
{
    tmat4x4<T> r = m;
    for (int j = 0; j < 4; j++) r[3][j] = m[0][j] * v.x + m[1][j] * v.y + m[2][j] * v.z + m[3][j];
    return r;
}
template <typename T> tmat4x4<T> scale(const tmat4x4<T>& m, const tvec3<T>& v)
{
    tmat4x4<T> r = m;
    for (int j = 0; j < 4; j++) { r[0][j] = m[0][j] * v.x; r[1][j] = m[1][j] * v.y; r[2][j] = m[2][j] * v.z; }
    return r;
}
// rotation by angle a about axis (Rodrigues), applied after m
template <typename T> tmat4x4<T> rotate(const tmat4x4<T>& m, T a, const tvec3<T>& axis)
{
    const tvec3<T> u = normalize(axis);
    const T c = std::cos(a), s = std::sin(a), k = T(1) - c;
    tmat4x4<T> R(T(1));
    R[0][0] = c + k * u.x * u.x;       R[0][1] = k * u.x * u.y + s * u.z; R[0][2] = k * u.x * u.z - s * u.y;
    R[1][0] = k * u.y * u.x - s * u.z; R[1][1] = c + k * u.y * u.y;       R[1][2] = k * u.y * u.z + s * u.x;
    R[2][0] = k * u.z * u.x + s * u.y; R[2][1] = k * u.z * u.y - s * u.x; R[2][2] = c + k * u.z * u.z;
    return m * R;
}

}  // namespace glm
