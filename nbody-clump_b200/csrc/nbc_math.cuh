// nbc_math.cuh -- small vector algebra for the engine's kernels.
//
// The operations mirror the helpers the reference's kernels use
// (src/type.h:10-305): Length() returns 0 when the squared length is at or
// below 1e-32, Quat2IvDCM is the body->world rotation of a quaternion stored
// (x, y, z, w) with w the scalar part, Quat2DCM its transpose.
#pragma once
#include <cuda_runtime.h>

namespace nbc {

template <typename R> struct V3 { R x, y, z; };

template <typename R> __host__ __device__ __forceinline__ V3<R> v3(R x, R y, R z) { return {x, y, z}; }
template <typename R> __host__ __device__ __forceinline__ V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <typename R> __host__ __device__ __forceinline__ V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <typename R> __host__ __device__ __forceinline__ V3<R> operator-(V3<R> a) { return {-a.x, -a.y, -a.z}; }
template <typename R> __host__ __device__ __forceinline__ V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <typename R> __host__ __device__ __forceinline__ R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <typename R> __host__ __device__ __forceinline__ V3<R> cross(V3<R> a, V3<R> b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename R> __host__ __device__ __forceinline__ R len_floor(V3<R> a) {
    R t = a.x * a.x + a.y * a.y + a.z * a.z;
    return t > R(1e-32) ? sqrt(t) : R(0);
}
template <typename R, typename S> __host__ __device__ __forceinline__ V3<R> cvt(V3<S> a) {
    return {R(a.x), R(a.y), R(a.z)};
}

// Real4 storage type of each precision
template <typename R> struct Vec4;
template <> struct Vec4<float> { using T = float4; };
template <> struct Vec4<double> { using T = double4; };
template <typename R> using R4 = typename Vec4<R>::T;

template <typename R> __device__ __forceinline__ V3<R> xyz(R4<R> a) { return {a.x, a.y, a.z}; }
__device__ __forceinline__ V3<double> xyzd(double4 a) { return {a.x, a.y, a.z}; }
template <typename R> __device__ __forceinline__ R4<R> pack(V3<R> a, R w) {
    R4<R> o; o.x = a.x; o.y = a.y; o.z = a.z; o.w = w; return o;
}

// body->world rotation (Quat2IvDCM, src/type.h:238-250) applied to u
__host__ __device__ __forceinline__ V3<double> rot_b2w(double4 q, V3<double> u) {
    double m00 = q.x * q.x - q.y * q.y - q.z * q.z + q.w * q.w;
    double m10 = 2.0 * (q.x * q.y + q.z * q.w);
    double m20 = 2.0 * (q.x * q.z - q.y * q.w);
    double m01 = 2.0 * (q.x * q.y - q.z * q.w);
    double m11 = -q.x * q.x + q.y * q.y - q.z * q.z + q.w * q.w;
    double m21 = 2.0 * (q.y * q.z + q.x * q.w);
    double m02 = 2.0 * (q.x * q.z + q.y * q.w);
    double m12 = 2.0 * (q.y * q.z - q.x * q.w);
    double m22 = -q.x * q.x - q.y * q.y + q.z * q.z + q.w * q.w;
    return {m00 * u.x + m01 * u.y + m02 * u.z, m10 * u.x + m11 * u.y + m12 * u.z,
            m20 * u.x + m21 * u.y + m22 * u.z};
}
// world->body rotation (Quat2DCM, src/type.h:223-236) applied to u
__host__ __device__ __forceinline__ V3<double> rot_w2b(double4 q, V3<double> u) {
    double m00 = q.x * q.x - q.y * q.y - q.z * q.z + q.w * q.w;
    double m10 = 2.0 * (q.x * q.y - q.z * q.w);
    double m20 = 2.0 * (q.x * q.z + q.y * q.w);
    double m01 = 2.0 * (q.x * q.y + q.z * q.w);
    double m11 = -q.x * q.x + q.y * q.y - q.z * q.z + q.w * q.w;
    double m21 = 2.0 * (q.y * q.z - q.x * q.w);
    double m02 = 2.0 * (q.x * q.z - q.y * q.w);
    double m12 = 2.0 * (q.y * q.z + q.x * q.w);
    double m22 = -q.x * q.x - q.y * q.y + q.z * q.z + q.w * q.w;
    return {m00 * u.x + m01 * u.y + m02 * u.z, m10 * u.x + m11 * u.y + m12 * u.z,
            m20 * u.x + m21 * u.y + m22 * u.z};
}

}  // namespace nbc
