// Element stress recovery per sample (OptimizedCalculateStress,
// optimizedSolidAssemble.pyx:1116-1223, called from physicsSolver.py:416-424 at each
// save): on the element frame of the geometry x + u_g, the local displacement
// TT u_e, the five local stresses E * D B lU (membrane xx, yy, xy and transverse
// shear xz, yz; D / (1 - nu^2) with shear factor 5/6), the local tensor
// [[xx, xy, xz], [xy, yy, yz], [xz, yz, 0]] rotated to the global frame (T^T s T),
// and its xx, yy, xy, xz, yz entries.  B annihilates rigid translations, so the
// displacement enters as differences from the element's node 0 (exact in FP32 for
// small relative motion).  One thread per (element, sample), samples fastest.
#include <cuda_runtime.h>

#include "common.cuh"

namespace cvfes {

template <typename T>
__global__ void k_stress(long long n_elems, int S, const double* __restrict__ nodes,
                         const int32_t* __restrict__ elems, const double* __restrict__ young,
                         const T* __restrict__ u, const T* __restrict__ ug, T nu,
                         T* __restrict__ stress) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long e = g / S;
    if (e >= n_elems) return;
    const int s = (int)(g - e * S);
    const int n0 = elems[3 * e], n1 = elems[3 * e + 1], n2 = elems[3 * e + 2];
    const int nid[3] = {n0, n1, n2};
    // positions relative to node 0 and displacement differences
    T P[3][3], du[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const size_t rk = (3 * (size_t)nid[k] + d) * S + s;
            const size_t r0 = (3 * (size_t)n0 + d) * S + s;
            const T x = (T)(nodes[3 * (size_t)nid[k] + d] - nodes[3 * (size_t)n0 + d]);
            P[k][d] = k == 0 ? T(0) : x + (ug ? ug[rk] - ug[r0] : T(0));
            du[k][d] = k == 0 ? T(0) : u[rk] - u[r0];
        }
    T ex[3], ey[3], ez[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) ex[d] = P[2][d] - P[1][d];
    T inv = rsqrt(ex[0] * ex[0] + ex[1] * ex[1] + ex[2] * ex[2]);
#pragma unroll
    for (int d = 0; d < 3; ++d) ex[d] *= inv;
#pragma unroll
    for (int d = 0; d < 3; ++d) ey[d] = P[0][d] - P[2][d];
    const T pr = ex[0] * ey[0] + ex[1] * ey[1] + ex[2] * ey[2];
#pragma unroll
    for (int d = 0; d < 3; ++d) ey[d] -= pr * ex[d];
    inv = rsqrt(ey[0] * ey[0] + ey[1] * ey[1] + ey[2] * ey[2]);
#pragma unroll
    for (int d = 0; d < 3; ++d) ey[d] *= inv;
    ez[0] = ex[1] * ey[2] - ex[2] * ey[1];
    ez[1] = ex[2] * ey[0] - ex[0] * ey[2];
    ez[2] = ex[0] * ey[1] - ex[1] * ey[0];
    T lx[3], ly[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lx[k] = P[k][0] * ex[0] + P[k][1] * ex[1] + P[k][2] * ex[2];
        ly[k] = P[k][0] * ey[0] + P[k][1] * ey[1] + P[k][2] * ey[2];
    }
    const T area = T(0.5) * ((lx[1] * ly[2] - lx[2] * ly[1]) - (lx[0] * ly[2] - lx[2] * ly[0]) +
                             (lx[0] * ly[1] - lx[1] * ly[0]));
    const T b[3] = {ly[1] - ly[2], ly[2] - ly[0], ly[0] - ly[1]};
    const T c[3] = {lx[2] - lx[1], lx[0] - lx[2], lx[1] - lx[0]};
    // local strains B lU (B = [b; c] / (2 area))
    T exx = 0, eyy = 0, gxy = 0, gxz = 0, gyz = 0;
#pragma unroll
    for (int k = 1; k < 3; ++k) {
        const T lu = ex[0] * du[k][0] + ex[1] * du[k][1] + ex[2] * du[k][2];
        const T lv = ey[0] * du[k][0] + ey[1] * du[k][1] + ey[2] * du[k][2];
        const T lw = ez[0] * du[k][0] + ez[1] * du[k][1] + ez[2] * du[k][2];
        exx += b[k] * lu;
        eyy += c[k] * lv;
        gxy += c[k] * lu + b[k] * lv;
        gxz += b[k] * lw;
        gyz += c[k] * lw;
    }
    const T inv2a = T(1) / (T(2) * area);
    const T E = (T)young[(size_t)e * S + s];
    const T f = E / (T(1) - nu * nu) * inv2a;
    const T k56 = T(5) / T(6);
    const T sxx = f * (exx + nu * eyy);
    const T syy = f * (nu * exx + eyy);
    const T sxy = f * T(0.5) * (T(1) - nu) * gxy;
    const T sxz = f * T(0.5) * k56 * (T(1) - nu) * gxz;
    const T syz = f * T(0.5) * k56 * (T(1) - nu) * gyz;
    // global tensor G = T^T L T, L = [[sxx, sxy, sxz], [sxy, syy, syz], [sxz, syz, 0]]
    const T L[3][3] = {{sxx, sxy, sxz}, {sxy, syy, syz}, {sxz, syz, T(0)}};
    const T* R[3] = {ex, ey, ez};
    T G[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            T acc = 0;
#pragma unroll
            for (int p = 0; p < 3; ++p)
#pragma unroll
                for (int q = 0; q < 3; ++q) acc += R[p][i] * L[p][q] * R[q][j];
            G[i][j] = acc;
        }
    T* o = stress + ((size_t)e * S + s) * 5;
    o[0] = G[0][0];
    o[1] = G[1][1];
    o[2] = G[0][1];
    o[3] = G[0][2];
    o[4] = G[1][2];
}

template <typename T>
int launch_stress(long long n_elems, long long S, const double* nodes, const int32_t* elems,
                  const double* young, const T* u, const T* ug, double nu, T* stress,
                  cudaStream_t st) {
    if (n_elems <= 0 || S <= 0 || S > INT32_MAX || !nodes || !elems || !young || !u || !stress)
        return fail(CVFES_ERR_ARG, "cvfes_solid_stress: bad argument");
    k_stress<T><<<grid_1d(n_elems * S, 256), 256, 0, st>>>(n_elems, (int)S, nodes, elems, young,
                                                           u, ug, (T)nu, stress);
    CVFES_LAUNCH_CHECK("k_stress");
    return CVFES_OK;
}

}  // namespace cvfes

using namespace cvfes;

extern "C" int cvfes_solid_stress_f64(int64_t n_elems, int64_t n_samples, const double* nodes,
                                      const int32_t* elems, const double* young, const double* u,
                                      const double* ug, double nu, double* stress, void* stream) {
    return launch_stress<double>(n_elems, n_samples, nodes, elems, young, u, ug, nu, stress,
                                 (cudaStream_t)stream);
}

extern "C" int cvfes_solid_stress_f32(int64_t n_elems, int64_t n_samples, const double* nodes,
                                      const int32_t* elems, const double* young, const float* u,
                                      const float* ug, double nu, float* stress, void* stream) {
    return launch_stress<float>(n_elems, n_samples, nodes, elems, young, u, ug, nu, stress,
                                (cudaStream_t)stream);
}
