// Device-side helpers shared by the solid-step kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "errors.h"

#define CVFES_CUDA_TRY(expr)                                                              \
    do {                                                                                  \
        cudaError_t _e = (expr);                                                          \
        if (_e != cudaSuccess)                                                            \
            return cvfes::fail(CVFES_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #expr, \
                               cudaGetErrorString(_e));                                   \
    } while (0)

#define CVFES_LAUNCH_CHECK(what)                                                           \
    do {                                                                                   \
        cudaError_t _e = cudaGetLastError();                                               \
        if (_e != cudaSuccess)                                                             \
            return cvfes::fail(CVFES_ERR_CUDA, "%s launch failed: %s", what,               \
                               cudaGetErrorString(_e));                                    \
    } while (0)

namespace cvfes {

constexpr int kSlabStride = 28;  // 27 stiffness entries per slot, padded to 16 B multiples

// VEC consecutive samples of one dof row, loaded/stored as one 8- or 16-byte access.
template <typename T, int V>
struct alignas(sizeof(T) * V) Vec {
    T v[V];
};

template <typename T, int V>
__device__ __forceinline__ Vec<T, V> ld(const T* p) {
    return *reinterpret_cast<const Vec<T, V>*>(p);
}
template <typename T, int V>
__device__ __forceinline__ Vec<T, V> ldg(const T* p) {
    Vec<T, V> r;
    if constexpr (sizeof(T) * V == 16) {
        float4 q = __ldg(reinterpret_cast<const float4*>(p));
        r = *reinterpret_cast<Vec<T, V>*>(&q);
    } else if constexpr (sizeof(T) * V == 8) {
        float2 q = __ldg(reinterpret_cast<const float2*>(p));
        r = *reinterpret_cast<Vec<T, V>*>(&q);
    } else {
        r.v[0] = __ldg(p);
    }
    return r;
}
// Asynchronous global -> shared copy of BYTES (4, 8 or 16) per thread (LSU path).
template <int BYTES>
__device__ __forceinline__ void cp_async(uint32_t dst, const void* src) {
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(dst), "l"(src), "n"(BYTES)
                     : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_all;" ::: "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// VEC values from shared memory (the caller guarantees VEC*sizeof(T) alignment)
template <typename T, int V>
__device__ __forceinline__ Vec<T, V> lds(const unsigned char* p) {
    return *reinterpret_cast<const Vec<T, V>*>(p);
}
template <typename T, int V>
__device__ __forceinline__ void st(T* p, const Vec<T, V>& x) {
    *reinterpret_cast<Vec<T, V>*>(p) = x;
}
// Streaming store: the new state is not re-read by this launch.
template <typename T, int V>
__device__ __forceinline__ void stcs(T* p, const Vec<T, V>& x) {
    if constexpr (sizeof(T) * V == 16) {
        __stcs(reinterpret_cast<float4*>(p), *reinterpret_cast<const float4*>(&x));
    } else if constexpr (sizeof(T) * V == 8) {
        __stcs(reinterpret_cast<float2*>(p), *reinterpret_cast<const float2*>(&x));
    } else {
        __stcs(p, x.v[0]);
    }
}
// Streaming load for data read once per launch (u_prev, inverse mass).
template <typename T, int V>
__device__ __forceinline__ Vec<T, V> ldcs(const T* p) {
    Vec<T, V> r;
    if constexpr (sizeof(T) * V == 16) {
        float4 q = __ldcs(reinterpret_cast<const float4*>(p));
        r = *reinterpret_cast<Vec<T, V>*>(&q);
    } else if constexpr (sizeof(T) * V == 8) {
        float2 q = __ldcs(reinterpret_cast<const float2*>(p));
        r = *reinterpret_cast<Vec<T, V>*>(&q);
    } else {
        r.v[0] = __ldcs(p);
    }
    return r;
}

// acc += k * x over the VEC lanes; FP32 pairs use the packed sm_100 FMA.
template <typename T, int V>
__device__ __forceinline__ void axpy(Vec<T, V>& acc, T k, const Vec<T, V>& x) {
    if constexpr (std::is_same<T, float>::value && (V % 2) == 0) {
#pragma unroll
        for (int i = 0; i < V; i += 2) {
            float2 r = __ffma2_rn(make_float2(k, k), make_float2(x.v[i], x.v[i + 1]),
                                  make_float2(acc.v[i], acc.v[i + 1]));
            acc.v[i] = r.x;
            acc.v[i + 1] = r.y;
        }
    } else {
#pragma unroll
        for (int i = 0; i < V; ++i) acc.v[i] = fma(k, x.v[i], acc.v[i]);
    }
}
// acc += c * x lane-wise
template <typename T, int V>
__device__ __forceinline__ void vfma(Vec<T, V>& acc, const Vec<T, V>& c, const Vec<T, V>& x) {
    if constexpr (std::is_same<T, float>::value && (V % 2) == 0) {
#pragma unroll
        for (int i = 0; i < V; i += 2) {
            float2 r = __ffma2_rn(make_float2(c.v[i], c.v[i + 1]), make_float2(x.v[i], x.v[i + 1]),
                                  make_float2(acc.v[i], acc.v[i + 1]));
            acc.v[i] = r.x;
            acc.v[i + 1] = r.y;
        }
    } else {
#pragma unroll
        for (int i = 0; i < V; ++i) acc.v[i] = fma(c.v[i], x.v[i], acc.v[i]);
    }
}
template <typename T, int V>
__device__ __forceinline__ Vec<T, V> vsub(const Vec<T, V>& a, const Vec<T, V>& b) {
    Vec<T, V> r;
    if constexpr (std::is_same<T, float>::value && (V % 2) == 0) {
        // a - b as one packed FMA per pair: (-1) * b + a, exact like the subtraction
#pragma unroll
        for (int i = 0; i < V; i += 2) {
            float2 q = __ffma2_rn(make_float2(b.v[i], b.v[i + 1]), make_float2(-1.0f, -1.0f),
                                  make_float2(a.v[i], a.v[i + 1]));
            r.v[i] = q.x;
            r.v[i + 1] = q.y;
        }
    } else {
#pragma unroll
        for (int i = 0; i < V; ++i) r.v[i] = a.v[i] - b.v[i];
    }
    return r;
}
template <typename T, int V>
__device__ __forceinline__ Vec<T, V> vzero() {
    Vec<T, V> r;
#pragma unroll
    for (int i = 0; i < V; ++i) r.v[i] = T(0);
    return r;
}
template <typename T, int V>
__device__ __forceinline__ Vec<T, V> vfill(T x) {
    Vec<T, V> r;
#pragma unroll
    for (int i = 0; i < V; ++i) r.v[i] = x;
    return r;
}

inline unsigned grid_1d(long long work, int block) {
    long long g = (work + block - 1) / block;
    return (unsigned)(g > 0 ? g : 1);
}

}  // namespace cvfes
