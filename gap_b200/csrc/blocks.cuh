// 2x2 block and 2-vector arithmetic for the block-sparse Newton Jacobian.
// A block is row-major [a b; c d] = [dP/dtheta dP/d|V|; dQ/dtheta dQ/d|V|].
#pragma once
#include <cuda_runtime.h>

namespace gapk {

template <typename T>
struct Blk {
    T a, b, c, d;
};
template <typename T>
struct Vec2 {
    T x, y;
};

__device__ __forceinline__ Blk<float> ldb(const Blk<float>* p) {
    float4 v = *reinterpret_cast<const float4*>(p);
    return {v.x, v.y, v.z, v.w};
}
__device__ __forceinline__ Blk<double> ldb(const Blk<double>* p) {
    const double2* q = reinterpret_cast<const double2*>(p);
    double2 u = q[0], w = q[1];
    return {u.x, u.y, w.x, w.y};
}
__device__ __forceinline__ void stb(Blk<float>* p, Blk<float> v) {
    *reinterpret_cast<float4*>(p) = make_float4(v.a, v.b, v.c, v.d);
}
__device__ __forceinline__ void stb(Blk<double>* p, Blk<double> v) {
    double2* q = reinterpret_cast<double2*>(p);
    q[0] = make_double2(v.a, v.b);
    q[1] = make_double2(v.c, v.d);
}
__device__ __forceinline__ Vec2<float> ldv(const Vec2<float>* p) {
    float2 v = *reinterpret_cast<const float2*>(p);
    return {v.x, v.y};
}
__device__ __forceinline__ Vec2<double> ldv(const Vec2<double>* p) {
    double2 v = *reinterpret_cast<const double2*>(p);
    return {v.x, v.y};
}
__device__ __forceinline__ void stv(Vec2<float>* p, Vec2<float> v) {
    *reinterpret_cast<float2*>(p) = make_float2(v.x, v.y);
}
__device__ __forceinline__ void stv(Vec2<double>* p, Vec2<double> v) {
    *reinterpret_cast<double2*>(p) = make_double2(v.x, v.y);
}

// acc -= X * Y
template <typename T>
__device__ __forceinline__ void msub(Blk<T>& acc, Blk<T> const& X, Blk<T> const& Y) {
    acc.a = fma(-X.a, Y.a, acc.a);
    acc.a = fma(-X.b, Y.c, acc.a);
    acc.b = fma(-X.a, Y.b, acc.b);
    acc.b = fma(-X.b, Y.d, acc.b);
    acc.c = fma(-X.c, Y.a, acc.c);
    acc.c = fma(-X.d, Y.c, acc.c);
    acc.d = fma(-X.c, Y.b, acc.d);
    acc.d = fma(-X.d, Y.d, acc.d);
}
template <typename T>
__device__ __forceinline__ Blk<T> mul(Blk<T> const& X, Blk<T> const& Y) {
    Blk<T> r;
    r.a = fma(X.a, Y.a, X.b * Y.c);
    r.b = fma(X.a, Y.b, X.b * Y.d);
    r.c = fma(X.c, Y.a, X.d * Y.c);
    r.d = fma(X.c, Y.b, X.d * Y.d);
    return r;
}
// acc -= X * v
template <typename T>
__device__ __forceinline__ void msubv(Vec2<T>& acc, Blk<T> const& X, Vec2<T> const& v) {
    acc.x = fma(-X.a, v.x, acc.x);
    acc.x = fma(-X.b, v.y, acc.x);
    acc.y = fma(-X.c, v.x, acc.y);
    acc.y = fma(-X.d, v.y, acc.y);
}
// acc -= X^T * v
template <typename T>
__device__ __forceinline__ void msubtv(Vec2<T>& acc, Blk<T> const& X, Vec2<T> const& v) {
    acc.x = fma(-X.a, v.x, acc.x);
    acc.x = fma(-X.c, v.y, acc.x);
    acc.y = fma(-X.b, v.x, acc.y);
    acc.y = fma(-X.d, v.y, acc.y);
}
template <typename T>
__device__ __forceinline__ Vec2<T> mulv(Blk<T> const& X, Vec2<T> const& v) {
    return {fma(X.a, v.x, X.b * v.y), fma(X.c, v.x, X.d * v.y)};
}
template <typename T>
__device__ __forceinline__ Vec2<T> multv(Blk<T> const& X, Vec2<T> const& v) {
    return {fma(X.a, v.x, X.c * v.y), fma(X.b, v.x, X.d * v.y)};
}

// 2x2 inverse of a pivot block.  ok=false when partial pivoting inside the block meets a
// pivot below 1e-14 in magnitude (the reference LU's pivot tolerance,
// src/solver/lu/cpu/cpu_lu_solver.cpp:65,112) or a non-finite value; the block is then
// returned unchanged.
template <typename T>
__device__ __forceinline__ Blk<T> inv2(Blk<T> const& X, bool& ok) {
    const T tol = T(1e-14);
    const T fa = fabs(X.a), fc = fabs(X.c);
    const T p1 = fa >= fc ? fa : fc;
    const T schur = fa >= fc ? X.d - X.c * (X.b / X.a) : X.b - X.a * (X.d / X.c);
    const T det = X.a * X.d - X.b * X.c;
    ok = p1 >= tol && fabs(schur) >= tol && isfinite(det) && det != T(0);
    if (!ok) return X;
    const T r = T(1) / det;
    return {X.d * r, -X.b * r, -X.c * r, X.a * r};
}

// NaN-propagating max of non-negative values
__device__ __forceinline__ double nmax(double a, double b) {
    return (a != a || a > b) ? a : b;
}

}  // namespace gapk
