// One-time set-up kernels of the membrane solid step, all FP64:
//   * per-element local frame, B, BᵀDB and the unit stiffness Kt_e = TTᵀ(A·BᵀDB)TT,
//     scattered as 3x9 row slabs into the node-centric slot layout;
//   * lumped mass per (node, sample) and the unit-pressure nodal load;
//   * optional block-CSR assembly K[nnzb][S][3][3] in the reference layout.
// Math follows optimizedSolidAssemble.pyx:82-127 (frame), :520-560 (B, BᵀDB),
// :562-583 (stiffness, mass, rotation), :585-590 (traction), :434-454 (lumping).
#include <cuda_runtime.h>

#include "common.cuh"

namespace cvfes {

struct DMat {
    double d[25];
};

__global__ void k_templates(int n_elems, const double* __restrict__ nodes,
                            const int32_t* __restrict__ elems, DMat D,
                            const int32_t* __restrict__ elem_slot,
                            const int32_t* __restrict__ slot_rec, double* __restrict__ slot_k64,
                            float* __restrict__ slot_k32, double* __restrict__ kt_full,
                            double* __restrict__ area_out, double* __restrict__ normal_out) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_elems) return;
    int nid[3];
    double p[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        nid[a] = elems[3 * e + a];
#pragma unroll
        for (int k = 0; k < 3; ++k) p[a][k] = nodes[3 * (size_t)nid[a] + k];
    }
    // Local frame (pyx:82-114): x along n2-n1, y Gram-Schmidt of n0-n2, z = x cross y.
    double e0[3], e1[3], T[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        e0[k] = p[2][k] - p[1][k];
        e1[k] = p[0][k] - p[2][k];
    }
    double nrm = sqrt(e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2]);
#pragma unroll
    for (int k = 0; k < 3; ++k) T[0][k] = e0[k] / nrm;
    double pr = e1[0] * T[0][0] + e1[1] * T[0][1] + e1[2] * T[0][2];
#pragma unroll
    for (int k = 0; k < 3; ++k) T[1][k] = e1[k] - pr * T[0][k];
    nrm = sqrt(T[1][0] * T[1][0] + T[1][1] * T[1][1] + T[1][2] * T[1][2]);
#pragma unroll
    for (int k = 0; k < 3; ++k) T[1][k] = T[1][k] / nrm;
    T[2][0] = T[0][1] * T[1][2] - T[0][2] * T[1][1];
    T[2][1] = T[0][2] * T[1][0] - T[0][0] * T[1][2];
    T[2][2] = T[0][0] * T[1][1] - T[0][1] * T[1][0];

    double lx[3], ly[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        lx[a] = p[a][0] * T[0][0] + p[a][1] * T[0][1] + p[a][2] * T[0][2];
        ly[a] = p[a][0] * T[1][0] + p[a][1] * T[1][1] + p[a][2] * T[1][2];
    }
    const double area = ((lx[1] * ly[2] - lx[2] * ly[1]) - (lx[0] * ly[2] - lx[2] * ly[0]) +
                         (lx[0] * ly[1] - lx[1] * ly[0])) *
                        0.5;
    const double c1 = 2.0 * area;
    const double by[3] = {(ly[1] - ly[2]) / c1, (ly[2] - ly[0]) / c1, (ly[0] - ly[1]) / c1};
    const double bx[3] = {(lx[2] - lx[1]) / c1, (lx[0] - lx[2]) / c1, (lx[1] - lx[0]) / c1};
    // B (5x9), pyx:551-556.
    double B[5][9];
#pragma unroll
    for (int r = 0; r < 5; ++r)
#pragma unroll
        for (int c = 0; c < 9; ++c) B[r][c] = 0.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        B[0][3 * a] = by[a];
        B[2][3 * a + 1] = by[a];
        B[3][3 * a + 2] = by[a];
        B[1][3 * a + 1] = bx[a];
        B[2][3 * a] = bx[a];
        B[4][3 * a + 2] = bx[a];
    }
    // BᵀD (9x5) then BᵀDB (9x9), summed in the reference's index order.
    double btd[9][5];
#pragma unroll
    for (int i = 0; i < 9; ++i)
#pragma unroll
        for (int j = 0; j < 5; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < 5; ++k) s += B[k][i] * D.d[5 * k + j];
            btd[i][j] = s;
        }
    double K[9][9];
#pragma unroll
    for (int i = 0; i < 9; ++i)
#pragma unroll
        for (int j = 0; j < 9; ++j) {
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < 5; ++k) s += btd[i][k] * B[k][j];
            K[i][j] = s * area;
        }
    // gK = TTᵀ K TT with TT = blockdiag(T,T,T); only the non-zero terms of the
    // reference's 9-term sums are formed.
    double tk[9][9];
#pragma unroll
    for (int i = 0; i < 9; ++i)
#pragma unroll
        for (int j = 0; j < 9; ++j) {
            const int bi = (i / 3) * 3, ii = i % 3;
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) s += T[k][ii] * K[bi + k][j];
            tk[i][j] = s;
        }
#pragma unroll
    for (int i = 0; i < 9; ++i)
#pragma unroll
        for (int j = 0; j < 9; ++j) {
            const int bj = (j / 3) * 3, jj = j % 3;
            double s = 0.0;
#pragma unroll
            for (int k = 0; k < 3; ++k) s += tk[i][bj + k] * T[k][jj];
            K[i][j] = s;
        }

    if (kt_full) {
#pragma unroll
        for (int i = 0; i < 81; ++i) kt_full[81 * (size_t)e + i] = K[i / 9][i % 9];
    }
    if (area_out) area_out[e] = area;
    if (normal_out) {
#pragma unroll
        for (int k = 0; k < 3; ++k) normal_out[3 * (size_t)e + k] = T[2][k];
    }
    if (slot_k64 || slot_k32) {
#pragma unroll
        for (int la = 0; la < 3; ++la) {
            const int s = elem_slot[3 * e + la];
            const int b1 = slot_rec[4 * s + 1], b2 = slot_rec[4 * s + 2];
            const int lb[3] = {la, b1 == nid[0] ? 0 : (b1 == nid[1] ? 1 : 2),
                               b2 == nid[0] ? 0 : (b2 == nid[1] ? 1 : 2)};
#pragma unroll
            for (int q = 0; q < 3; ++q)
#pragma unroll
                for (int i = 0; i < 3; ++i)
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        const double val = K[3 * la + i][3 * lb[q] + j];
                        const size_t o = (size_t)kSlabStride * s + 9 * q + 3 * i + j;
                        if (slot_k64) slot_k64[o] = val;
                        if (slot_k32) slot_k32[o] = (float)val;
                    }
            if (slot_k64) slot_k64[(size_t)kSlabStride * s + 27] = 0.0;
            if (slot_k32) slot_k32[(size_t)kSlabStride * s + 27] = 0.0f;
        }
    }
}

struct MW {
    double w[9];  // w[3a + g] = rho * wt_g^2 * N_g(a)
};

// One thread per (node, sample): lumped mass m = sum over incident elements of
// area * sum_g mw[la][g] * h_g; FP64 inverse (0 where m == 0, the reference's
// where=LHS!=0 guard).  Sample 0 also forms the unit-pressure load.
__global__ void k_mass_load(int n_nodes, int S, const int32_t* __restrict__ node_ptr,
                            const int32_t* __restrict__ slot_rec, const double* __restrict__ area,
                            const double* __restrict__ normal, const double* __restrict__ gthick,
                            int n_gauss, MW mw, double* __restrict__ lm, double* __restrict__ invm64,
                            float* __restrict__ invm32, double* __restrict__ fhat64,
                            float* __restrict__ fhat32) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long a = g / S;
    const int s = (int)(g - a * S);
    if (a >= n_nodes) return;
    const int k0 = node_ptr[a], k1 = node_ptr[a + 1];
    double m = 0.0;
    double f[3] = {0.0, 0.0, 0.0};
    for (int k = k0; k < k1; ++k) {
        const int e = slot_rec[4 * k];
        const int la = (slot_rec[4 * k + 3] >> 8) & 3;
        const double A = area[e];
        const double* h = gthick + ((size_t)e * S + s) * n_gauss;
        const double h1 = h[n_gauss > 1 ? 1 : 0], h2 = h[n_gauss > 1 ? 2 : 0];
        m += A * (mw.w[3 * la] * h[0] + mw.w[3 * la + 1] * h1 + mw.w[3 * la + 2] * h2);
        if (s == 0) {
            const double c = (1.0 / 3.0) * A;
#pragma unroll
            for (int d = 0; d < 3; ++d) f[d] += normal[3 * (size_t)e + d] * c;
        }
    }
    const size_t o = (size_t)a * S + s;
    const double inv = (m != 0.0) ? 1.0 / m : 0.0;
    if (lm) lm[o] = m;
    if (invm64) invm64[o] = inv;
    if (invm32) invm32[o] = (float)inv;
    if (s == 0) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            if (fhat64) fhat64[4 * a + d] = f[d];
            if (fhat32) fhat32[4 * a + d] = (float)f[d];
        }
        if (fhat64) fhat64[4 * a + 3] = 0.0;
        if (fhat32) fhat32[4 * a + 3] = 0.0f;
    }
}

// Elements of one colour share no node, so their blocks never collide.
__global__ void k_assemble_bsr(int n_in_color, int S, const int32_t* __restrict__ color_elems,
                               const double* __restrict__ kt_full, const double* __restrict__ coef,
                               const int32_t* __restrict__ block_pos, double* __restrict__ K) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long i = g / S;
    const int s = (int)(g - i * S);
    if (i >= n_in_color) return;
    const int e = color_elems[i];
    const double c = coef[(size_t)e * S + s];
    const double* kt = kt_full + 81 * (size_t)e;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
            const size_t pos = (size_t)block_pos[9 * (size_t)e + 3 * a + b];
            double* dst = K + (pos * S + s) * 9;
#pragma unroll
            for (int ii = 0; ii < 3; ++ii)
#pragma unroll
                for (int jj = 0; jj < 3; ++jj)
                    dst[3 * ii + jj] += kt[9 * (3 * a + ii) + 3 * b + jj] * c;
        }
}

}  // namespace cvfes

using namespace cvfes;

extern "C" int cvfes_solid_templates_f64(int64_t n_nodes, int64_t n_elems, const double* nodes,
                                         const int32_t* elems, const double* dmat,
                                         const int32_t* elem_slot, const int32_t* slot_rec,
                                         double* slot_k64, float* slot_k32, double* kt_full,
                                         double* area, double* normal, void* stream) {
    if (n_nodes <= 0 || n_elems <= 0 || n_elems >= INT32_MAX / 3 || !nodes || !elems || !dmat)
        return fail(CVFES_ERR_ARG, "cvfes_solid_templates_f64: bad argument");
    if ((slot_k64 || slot_k32) && (!elem_slot || !slot_rec))
        return fail(CVFES_ERR_ARG, "cvfes_solid_templates_f64: slabs need elem_slot and slot_rec");
    DMat D;
    for (int i = 0; i < 25; ++i) D.d[i] = dmat[i];
    const int block = 128;
    k_templates<<<grid_1d(n_elems, block), block, 0, (cudaStream_t)stream>>>(
        (int)n_elems, nodes, elems, D, elem_slot, slot_rec, slot_k64, slot_k32, kt_full, area,
        normal);
    CVFES_LAUNCH_CHECK("k_templates");
    return CVFES_OK;
}

extern "C" int cvfes_solid_mass_load_f64(int64_t n_nodes, int64_t n_elems, int64_t n_samples,
                                         const int32_t* node_ptr, const int32_t* slot_rec,
                                         const double* area, const double* normal,
                                         const double* gthick, int32_t n_gauss,
                                         const double* mw_host,
                                         double* lm, double* invm64, float* invm32,
                                         double* fhat64, float* fhat32, void* stream) {
    if (n_nodes <= 0 || n_elems <= 0 || n_samples <= 0 || !node_ptr || !slot_rec || !area ||
        !normal || !gthick || !mw_host || (n_gauss != 1 && n_gauss != 3))
        return fail(CVFES_ERR_ARG, "cvfes_solid_mass_load_f64: bad argument");
    MW mw;
    for (int i = 0; i < 9; ++i) mw.w[i] = mw_host[i];
    const int block = 256;
    k_mass_load<<<grid_1d(n_nodes * n_samples, block), block, 0, (cudaStream_t)stream>>>(
        (int)n_nodes, (int)n_samples, node_ptr, slot_rec, area, normal, gthick, n_gauss, mw, lm,
        invm64,
        invm32, fhat64, fhat32);
    CVFES_LAUNCH_CHECK("k_mass_load");
    return CVFES_OK;
}

extern "C" int cvfes_solid_assemble_bsr_f64(int64_t n_elems, int64_t n_samples,
                                            const double* kt_full, const double* coef,
                                            const int32_t* block_pos, int32_t n_colors,
                                            const int64_t* color_ptr,
                                            const int32_t* color_elems, double* K, void* stream) {
    if (n_elems <= 0 || n_samples <= 0 || !kt_full || !coef || !block_pos || n_colors <= 0 ||
        !color_ptr || !color_elems || !K)
        return fail(CVFES_ERR_ARG, "cvfes_solid_assemble_bsr_f64: bad argument");
    if (color_ptr[0] != 0 || color_ptr[n_colors] != n_elems)
        return fail(CVFES_ERR_ARG, "cvfes_solid_assemble_bsr_f64: colour groups do not cover E");
    const int block = 256;
    for (int c = 0; c < n_colors; ++c) {
        const int64_t n = color_ptr[c + 1] - color_ptr[c];
        if (n <= 0) continue;
        k_assemble_bsr<<<grid_1d(n * n_samples, block), block, 0, (cudaStream_t)stream>>>(
            (int)n, (int)n_samples, color_elems + color_ptr[c], kt_full, coef, block_pos, K);
        CVFES_LAUNCH_CHECK("k_assemble_bsr");
    }
    return CVFES_OK;
}
