// Discrete adjoint of the explicit membrane time step for a displacement-mismatch
// objective, with respect to per-element, per-sample log E and log h.
//
// Forward step n (n = 0 .. T-1), free rows, W = w0 * inverse lumped mass:
//     u_{n+1} = u_n + (1 - eta)(u_n - u_{n-1}) + W (p_n fhat - K(c) u_n),   K(c) = sum_e c_e Khat_e
// clamped rows hold the clamp value, c_e = E_e h_e, and the objective is
//     J_s = sum_{n in O} sum_{i in obs} |u_n(i) - uobs_n(i)|^2,   O = {n : n % obs_every == 0, n > 0}.
// With chi_n = W mu_n (mu the adjoint of u_n, zero on clamped rows) the reverse
// recursion has the form of the forward step:
//     chi_n = chi_{n+1} + (1 - eta)(chi_{n+1} - chi_{n+2}) - W K chi_{n+1} + W dJ/du_n
// and the gradients are
//     dJ/dlogE_e = -c_e Gamma_e,   Gamma_e = sum_n chi_{n+1,e}^T Khat_e u_{n,e}
//     dJ/dlogh_e = -c_e Gamma_e - h_e sum_{a in e} alpha_{e,a} invm_a G_a,   G_a = sum_n chi_{n+1,a} . r_{n,a}
// with r_n = p_n fhat - K u_n and alpha_{e,a} the element's lumped-mass weight of node a
// (m_a = sum_e h_e alpha_{e,a}).  The damping is mass-proportional, so eta does not
// depend on the material.
//
// States u_n are not stored: the reverse sweep runs the forward step backwards,
//     u_{n-1} = u_n - ((u_{n+1} - u_n) - W r_n) / (1 - eta),
// in the same kernel that advances chi, and replaces the reconstructed pair by the
// exact pair (u_m, u_{m+1}) saved by the forward pass at every checkpoint m (every
// ckpt_every steps), so the reconstruction drift never spans more than one segment.
// Both recursions share one pass over the node's slots: the fan-ordered slot rows of
// Khat are applied to u_n and chi_{n+1}, and the slot of each element's local node 0
// (its owner) also evaluates the element's bilinear form from the difference
// vectors (u_b - u_a, chi_b - chi_a), which needs only the blocks K_b1b1, K_b1b2,
// K_b2b2 of that slot's two neighbours (rigid translations are in Khat's null space).
// Every element and node accumulator is written by one thread: no atomics.
#include <cuda_runtime.h>

#include <type_traits>

#include "common.cuh"
#include "step_core.cuh"

namespace cvfes {

constexpr int kObsChunk = 16;   // observation nodes per block of the mismatch kernel
constexpr int kOwnStride = 28;  // K_b1b1 (9), K_b1b2 (9), K_b2b2 (9), pad

struct MassWeights {
    double w[9];  // w[3a + g]: lumped-mass weight of local node a at quadrature point g
};

// Owner-slot neighbour blocks of every element, in the owner slot's (b1, b2) order,
// stored at the owner slot (the slot of the element's local node 0); the entries of the
// other slots are not used.
template <typename T>
__global__ void k_owner_blocks(long long n_elems, const int32_t* __restrict__ elems,
                               const int32_t* __restrict__ elem_slot,
                               const int32_t* __restrict__ slot_rec, const T* __restrict__ slab,
                               T* __restrict__ own) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e >= n_elems) return;
    const int s0 = elem_slot[3 * e];
    const int b1 = slot_rec[4 * s0 + 1], b2 = slot_rec[4 * s0 + 2];
    const int l1 = elems[3 * e + 1] == b1 ? 1 : 2;
    const int s1 = elem_slot[3 * e + l1], s2 = elem_slot[3 * e + 3 - l1];
    const int q = slot_rec[4 * s1 + 1] == b2 ? 1 : 2;  // block of b2 in b1's slot
    T* o = own + (size_t)kOwnStride * s0;
    const T* k1 = slab + (size_t)kSlabStride * s1;
    const T* k2 = slab + (size_t)kSlabStride * s2;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
        o[i] = k1[i];
        o[9 + i] = k1[9 * q + i];
        o[18 + i] = k2[i];
    }
    o[27] = T(0);
}

// coef = E*h and thickness h from the log-material of each element and sample.
__global__ void k_material_log(long long n, const double* __restrict__ logE,
                               const double* __restrict__ logh, double* __restrict__ coef64,
                               float* __restrict__ coef32, double* __restrict__ thick) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double h = exp(logh[i]);
    const double c = exp(logE[i]) * h;
    if (coef64) coef64[i] = c;
    if (coef32) coef32[i] = (float)c;
    if (thick) thick[i] = h;
}

// Observation step k: either record u at the observation nodes, or add the squared
// mismatch of this block's observation nodes into jpart[k][block][s].
template <typename T>
__global__ void k_obs(int n_obs, int S, const int32_t* __restrict__ obs_nodes,
                      const T* __restrict__ u, T* __restrict__ obs_k, double* __restrict__ jpart_k,
                      int record) {
    const int s = blockIdx.y * blockDim.x + threadIdx.x;
    if (s >= S) return;
    const int i0 = blockIdx.x * kObsChunk;
    const int i1 = min(n_obs, i0 + kObsChunk);
    double acc = 0.0;
    for (int i = i0; i < i1; ++i) {
        const size_t a = (size_t)obs_nodes[i];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const T v = u[(3 * a + c) * S + s];
            const size_t o = ((size_t)i * 3 + c) * S + s;
            if (record) {
                obs_k[o] = v;
            } else {
                const double d = (double)v - (double)obs_k[o];
                acc = fma(d, d, acc);
            }
        }
    }
    if (!record) jpart_k[(size_t)blockIdx.x * S + s] = acc;
}

// J[s] = sum over observation steps and node blocks, in a fixed order.
__global__ void k_obs_reduce(long long n_parts, int S, const double* __restrict__ jpart,
                             double* __restrict__ J) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= S) return;
    double acc = 0.0;
    for (long long k = 0; k < n_parts; ++k) acc += jpart[(size_t)k * S + s];
    J[s] = acc;
}

// chi_n += W dJ/du_n = W * 2 (u_n - uobs_n) at the free observation nodes.
template <typename T>
__global__ void k_adj_force(int n_obs, int S, const int32_t* __restrict__ obs_nodes,
                            int n_clamped, const T* __restrict__ invm, T w0,
                            const T* __restrict__ u, const T* __restrict__ obs_k, T* __restrict__ chi) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long i = g / S;
    if (i >= n_obs) return;
    const int s = (int)(g - i * S);
    const size_t a = (size_t)obs_nodes[i];
    if ((long long)a < n_clamped) return;
    const T w = w0 * invm[a * S + s];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const size_t r = (3 * a + c) * S + s;
        const T d = u[r] - obs_k[((size_t)i * 3 + c) * S + s];
        chi[r] += w * T(2) * d;
    }
}

template <typename T>
struct RevArgs {
    const int32_t* node_ptr;
    const int4* rec;
    const T* slab;
    const T* own;
    const T* fhat;
    const T* coef;
    const T* invm;
    const T* u;    // u_n
    T* uo;         // in: u_{n+1}; out: u_{n-1}
    const T* x;    // chi_{n+1}
    T* xo;         // in: chi_{n+2}; out: chi_n (without the observation forcing)
    T* gam;        // (E, S) Gamma accumulator
    T* gm;         // (N, S) G accumulator, or null
    const double* p;  // pressure of forward step n
    long long n_nodes;
    int S;
    int n_clamped;
    T clamp;
    T eta;
    T inv1meta;
    T w0;
    int tpn;
    int npb;
    int nch;        // sample chunks of 32*VEC per node block (fan kernel)
    int cap_slots;  // slot capacity of the shared-memory stage (fan kernel)
    int* status;    // bit 0: a bounded wait gave up; bit 1: stage too small
    int pf_dist = 0;   // fan kernel: nodes ahead whose rows are prefetched into L2 (0: off)
    int pf_parts = 0;  // bit 0: node rows; bit 1: element coefficient and Gamma rows
    int pf_group = 1;  // node blocks covered by one prefetching block
};

// Prefetch into L2 the rows that nodes a0 .. a0 + n - 1 read in a reverse step: u_n,
// chi_{n+1}, u_{n+1}, chi_{n+2}, inverse mass, the G row, and the coefficient and
// Gamma rows of their elements (found through their slot records).
template <typename T, bool GM>
__device__ __forceinline__ void rev_prefetch(const RevArgs<T>& A, long long a0, int n,
                                             int lane) {
    if (a0 >= A.n_nodes) return;
    const long long a1 = (a0 + n < A.n_nodes) ? a0 + n : A.n_nodes;
    const size_t S = (size_t)A.S;
    const size_t nrow = (size_t)(a1 - a0) * S * sizeof(T);
    if (A.pf_parts & 1) {
        if (lane == 0) bulk_prefetch_l2(A.u + (size_t)a0 * 3 * S, 3 * nrow);
        if (lane == 1) bulk_prefetch_l2(A.x + (size_t)a0 * 3 * S, 3 * nrow);
        if (lane == 2) bulk_prefetch_l2(A.uo + (size_t)a0 * 3 * S, 3 * nrow);
        if (lane == 3) bulk_prefetch_l2(A.xo + (size_t)a0 * 3 * S, 3 * nrow);
        if (lane == 4) bulk_prefetch_l2(A.invm + (size_t)a0 * S, nrow);
        if constexpr (GM) {
            if (lane == 5) bulk_prefetch_l2(A.gm + (size_t)a0 * S, nrow);
        }
    }
    if (!(A.pf_parts & 2)) return;
    const int kb = __ldg(A.node_ptr + a0), ke = __ldg(A.node_ptr + a1);
    for (int k = kb + lane; k < ke; k += 32) {
        const size_t e = (size_t)__ldg(&A.rec[k].x);
        bulk_prefetch_l2(A.coef + e * S, S * sizeof(T));
        bulk_prefetch_l2(A.gam + e * S, S * sizeof(T));
    }
}

template <typename T>
__device__ __forceinline__ void load27(const T* K, T (&kk)[27]) {
    if constexpr (std::is_same<T, float>::value) {
#pragma unroll
        for (int q = 0; q < 7; ++q) {
            const float4 t = __ldg(reinterpret_cast<const float4*>(K) + q);
            if (4 * q + 0 < 27) kk[4 * q + 0] = t.x;
            if (4 * q + 1 < 27) kk[4 * q + 1] = t.y;
            if (4 * q + 2 < 27) kk[4 * q + 2] = t.z;
            if (4 * q + 3 < 27) kk[4 * q + 3] = t.w;
        }
    } else {
#pragma unroll
        for (int q = 0; q < 14; ++q) {
            const double2 t = __ldg(reinterpret_cast<const double2*>(K) + q);
            if (2 * q + 0 < 27) kk[2 * q + 0] = t.x;
            if (2 * q + 1 < 27) kk[2 * q + 1] = t.y;
        }
    }
}

// Gamma_e += dchi^T Khat_e du for the element owned by this slot: (u1, u2) and (x1, x2) are
// the first and second neighbour rows of u_n and chi_{n+1}, already differences
// u_b - u_a in the DIFF form, raw rows otherwise.
template <typename T, int V, bool DIFF, bool SMEM_OWN = false>
__device__ __forceinline__ void owner_grad(const RevArgs<T>& A, int e, const T* own, size_t S,
                                           size_t col,
                                           const Vec<T, V> (&u1)[3], const Vec<T, V> (&u2)[3],
                                           const Vec<T, V> (&x1)[3], const Vec<T, V> (&x2)[3],
                                           const Vec<T, V> (&ua)[3], const Vec<T, V> (&ca)[3]) {
    Vec<T, V> du1[3], du2[3], dy1[3], dy2[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if constexpr (DIFF) {
            du1[d] = u1[d];
            du2[d] = u2[d];
            dy1[d] = x1[d];
            dy2[d] = x2[d];
        } else {
            du1[d] = vsub(u1[d], ua[d]);
            du2[d] = vsub(u2[d], ua[d]);
            dy1[d] = vsub(x1[d], ca[d]);
            dy2[d] = vsub(x2[d], ca[d]);
        }
    }
    // own points into global memory (gather kernel) or shared memory (fan kernel, SMEM_OWN):
    // plain generic loads, not the global-only read-only path.  From shared memory they
    // are volatile, so that each of the 27 values is read where it is used instead of all
    // of them being hoisted into registers beside the three rotating neighbour-row sets
    // (the fan kernel spilled at its 128-register cap with them hoisted; it fits without).
    using OwnPtr = typename std::conditional<SMEM_OWN, const volatile T*, const T*>::type;
    const OwnPtr ob = own;
    Vec<T, V> g = vzero<T, V>();
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        Vec<T, V> z1 = vzero<T, V>(), z2 = vzero<T, V>();
#pragma unroll
        for (int jj = 0; jj < 3; ++jj) {
            axpy(z1, ob[3 * i + jj], du1[jj]);       // K_b1b1
            axpy(z1, ob[9 + 3 * i + jj], du2[jj]);   // K_b1b2
            axpy(z2, ob[9 + 3 * jj + i], du1[jj]);   // K_b2b1 = K_b1b2^T
            axpy(z2, ob[18 + 3 * i + jj], du2[jj]);  // K_b2b2
        }
        vfma(g, dy1[i], z1);
        vfma(g, dy2[i], z2);
    }
    T* gp = A.gam + (size_t)e * S + col;
    Vec<T, V> gv = ld<T, V>(gp);
#pragma unroll
    for (int q = 0; q < V; ++q) gv.v[q] += g.v[q];
    st<T, V>(gp, gv);
}

// Node update of one reverse step: u_{n-1} (backward step), chi_n, and G += chi_{n+1} . r_n.
template <typename T, int V, bool GM>
__device__ __forceinline__ void rev_epilogue(const RevArgs<T>& A, long long a, size_t S,
                                             size_t col, size_t row, const Vec<T, V> (&ua)[3],
                                             const Vec<T, V> (&ca)[3],
                                             const Vec<T, V> (&accU)[3],
                                             const Vec<T, V> (&accC)[3]) {
    if (a < A.n_clamped) {
        const Vec<T, V> cl = vfill<T, V>(A.clamp), z = vzero<T, V>();
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            st<T, V>(A.uo + row + d * S, cl);
            st<T, V>(A.xo + row + d * S, z);
        }
        return;
    }
    const T p = (T)A.p[0];
    const Vec<T, V> im = ldg<T, V>(A.invm + (size_t)a * S + col);
    Vec<T, V> gacc = vzero<T, V>();
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const T f = p * __ldg(A.fhat + 4 * a + d);
        const Vec<T, V> u1 = ld<T, V>(A.uo + row + d * S);
        const Vec<T, V> x2o = ld<T, V>(A.xo + row + d * S);
        Vec<T, V> um, xn;
#pragma unroll
        for (int i = 0; i < V; ++i) {
            const bool live = im.v[i] != T(0);
            const T w = A.w0 * im.v[i];
            const T r = f - accU[d].v[i];
            const T dv = ((u1.v[i] - ua[d].v[i]) - w * r) * A.inv1meta;
            um.v[i] = live ? ua[d].v[i] - dv : T(0);
            const T dx = ca[d].v[i] - x2o.v[i];
            xn.v[i] = live ? ca[d].v[i] + fma(-A.eta, dx, dx) - w * accC[d].v[i] : T(0);
            if constexpr (GM) gacc.v[i] = fma(ca[d].v[i], r, gacc.v[i]);
        }
        st<T, V>(A.uo + row + d * S, um);
        st<T, V>(A.xo + row + d * S, xn);
    }
    if constexpr (GM) {
        T* gp = A.gm + (size_t)a * S + col;
        Vec<T, V> gv = ld<T, V>(gp);
#pragma unroll
        for (int q = 0; q < V; ++q) gv.v[q] += gacc.v[q];
        st<T, V>(gp, gv);
    }
}

// One reverse step for (node a, V samples): reconstruct u_{n-1}, advance chi, accumulate
// Gamma over the elements this node owns and G of this node.  Rows are gathered
// through L1; a fan continuation reuses the previous slot's second neighbour.
template <typename T, int V, bool DIFF, bool GM>
__global__ void __launch_bounds__(256) k_reverse(RevArgs<T> A) {
    long long a;
    int vec;
    if (!map_row(A.tpn, A.npb, A.n_nodes, A.S / V, a, vec)) return;
    const size_t S = (size_t)A.S;
    const size_t col = (size_t)vec * V;
    const size_t row = (size_t)a * 3 * S + col;
    Vec<T, V> ua[3], ca[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        ua[d] = ldg<T, V>(A.u + row + d * S);
        ca[d] = ldg<T, V>(A.x + row + d * S);
    }
    Vec<T, V> accU[3], accC[3], cu[3], cc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        accU[d] = vzero<T, V>();
        accC[d] = vzero<T, V>();
        cu[d] = vzero<T, V>();
        cc[d] = vzero<T, V>();
    }
    const int k0 = __ldg(A.node_ptr + a), k1 = __ldg(A.node_ptr + a + 1);
    for (int k = k0; k < k1; ++k) {
        const int4 r = __ldg(A.rec + k);
        Vec<T, V> x1[3], x2[3], y1[3], y2[3];
        if (r.w & 1) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                x1[d] = cu[d];
                y1[d] = cc[d];
            }
        } else {
            const size_t o1 = (size_t)r.y * 3 * S + col;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                x1[d] = ldg<T, V>(A.u + o1 + d * S);
                y1[d] = ldg<T, V>(A.x + o1 + d * S);
                if constexpr (DIFF) {
                    x1[d] = vsub(x1[d], ua[d]);
                    y1[d] = vsub(y1[d], ca[d]);
                }
            }
        }
        const size_t o2 = (size_t)r.z * 3 * S + col;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            x2[d] = ldg<T, V>(A.u + o2 + d * S);
            y2[d] = ldg<T, V>(A.x + o2 + d * S);
            if constexpr (DIFF) {
                x2[d] = vsub(x2[d], ua[d]);
                y2[d] = vsub(y2[d], ca[d]);
            }
        }
        const Vec<T, V> c = ldg<T, V>(A.coef + (size_t)r.x * S + col);
        T kk[27];
        load27<T>(A.slab + (size_t)kSlabStride * k, kk);
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            Vec<T, V> tu = vzero<T, V>(), tc = vzero<T, V>();
            if constexpr (!DIFF) {
#pragma unroll
                for (int jj = 0; jj < 3; ++jj) {
                    axpy(tu, kk[3 * i + jj], ua[jj]);
                    axpy(tc, kk[3 * i + jj], ca[jj]);
                }
            }
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) {
                axpy(tu, kk[9 + 3 * i + jj], x1[jj]);
                axpy(tc, kk[9 + 3 * i + jj], y1[jj]);
            }
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) {
                axpy(tu, kk[18 + 3 * i + jj], x2[jj]);
                axpy(tc, kk[18 + 3 * i + jj], y2[jj]);
            }
            vfma(accU[i], c, tu);
            vfma(accC[i], c, tc);
        }
        if (((r.w >> 8) & 3) == 0)
            owner_grad<T, V, DIFF>(A, r.x, A.own + (size_t)kOwnStride * k, S, col, x1, x2, y1, y2,
                                   ua, ca);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            cu[d] = x2[d];
            cc[d] = y2[d];
        }
    }
    rev_epilogue<T, V, GM>(A, a, S, col, row, ua, ca, accU, accC);
}

// ------------------------------------------------------------ fan-rotation reverse step
// As the forward fan kernel: a warp per node and 32*VEC-sample chunk, the block's slot
// records and stiffness rows bulk-copied (TMA) into shared memory, and the neighbour
// rows of u_n and chi_{n+1} rotating through three register sets so that the loads of
// slot k+1 are in flight while slot k is multiplied.
template <typename T, int V>
__device__ __forceinline__ void load3(Vec<T, V> (&x)[3], const T* __restrict__ base, int node,
                                      size_t S, size_t col) {
    const T* p = base + (size_t)node * 3 * S + col;
#pragma unroll
    for (int d = 0; d < 3; ++d) x[d] = ldg<T, V>(p + d * S);
}
template <typename T, int V, bool DIFF>
__device__ __forceinline__ void diff3(Vec<T, V> (&x)[3], const Vec<T, V> (&ref)[3]) {
    if constexpr (DIFF) {
#pragma unroll
        for (int d = 0; d < 3; ++d) x[d] = vsub(x[d], ref[d]);
    }
}

// Both row products of one slot from one read of its stiffness rows (shared memory).
template <typename T, int V, bool DIFF>
__device__ __forceinline__ void slot_fma2(const T* K, const Vec<T, V>& c,
                                          const Vec<T, V> (&u1)[3], const Vec<T, V> (&u2)[3],
                                          const Vec<T, V> (&x1)[3], const Vec<T, V> (&x2)[3],
                                          const Vec<T, V> (&ua)[3], const Vec<T, V> (&ca)[3],
                                          Vec<T, V> (&accU)[3], Vec<T, V> (&accC)[3]) {
    T kk[28];
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int q = (DIFF ? 2 : 0); q < 7; ++q) {
            const float4 t = reinterpret_cast<const float4*>(K)[q];
            kk[4 * q] = t.x;
            kk[4 * q + 1] = t.y;
            kk[4 * q + 2] = t.z;
            kk[4 * q + 3] = t.w;
        }
    } else {
#pragma unroll
        for (int q = (DIFF ? 4 : 0); q < 14; ++q) {
            const double2 t = reinterpret_cast<const double2*>(K)[q];
            kk[2 * q] = t.x;
            kk[2 * q + 1] = t.y;
        }
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        Vec<T, V> tu = vzero<T, V>(), tc = vzero<T, V>();
        if constexpr (!DIFF) {
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) {
                axpy(tu, kk[3 * i + jj], ua[jj]);
                axpy(tc, kk[3 * i + jj], ca[jj]);
            }
        }
#pragma unroll
        for (int jj = 0; jj < 3; ++jj) {
            axpy(tu, kk[9 + 3 * i + jj], u1[jj]);
            axpy(tc, kk[9 + 3 * i + jj], x1[jj]);
        }
#pragma unroll
        for (int jj = 0; jj < 3; ++jj) {
            axpy(tu, kk[18 + 3 * i + jj], u2[jj]);
            axpy(tc, kk[18 + 3 * i + jj], x2[jj]);
        }
        vfma(accU[i], c, tu);
        vfma(accC[i], c, tc);
    }
}

template <typename T, int V, bool DIFF>
__device__ __forceinline__ void rev_phase(int& k, int k1, const int4* srec, const T* sslab,
                                          const T* sown, const RevArgs<T>& A, size_t S, size_t col,
                                          const Vec<T, V> (&ua)[3], const Vec<T, V> (&ca)[3],
                                          Vec<T, V> (&accU)[3], Vec<T, V> (&accC)[3],
                                          Vec<T, V> (&pu)[3], Vec<T, V> (&px)[3],
                                          Vec<T, V> (&cu)[3], Vec<T, V> (&cx)[3],
                                          const Vec<T, V>& ccur, Vec<T, V> (&nu)[3],
                                          Vec<T, V> (&nx)[3], Vec<T, V>& cnxt) {
    const bool more = k + 1 < k1;
    int4 rn = make_int4(0, 0, 0, 1);
    if (more) {
        rn = srec[k + 1];
        load3<T, V>(nu, A.u, rn.z, S, col);
        load3<T, V>(nx, A.x, rn.z, S, col);
        cnxt = ldg<T, V>(A.coef + (size_t)rn.x * S + col);
    }
    diff3<T, V, DIFF>(cu, ua);
    diff3<T, V, DIFF>(cx, ca);
    const int4 r = srec[k];
    slot_fma2<T, V, DIFF>(sslab + (size_t)kSlabStride * k, ccur, pu, cu, px, cx, ua, ca, accU,
                          accC);
    if (((r.w >> 8) & 3) == 0)
        owner_grad<T, V, DIFF, true>(A, r.x, sown + (size_t)kOwnStride * k, S, col, pu, cu, px, cx, ua,
                               ca);
    if (more && !(rn.w & 1)) {  // fan break: the next slot's first neighbour is new
        load3<T, V>(cu, A.u, rn.y, S, col);
        load3<T, V>(cx, A.x, rn.y, S, col);
        diff3<T, V, DIFF>(cu, ua);
        diff3<T, V, DIFF>(cx, ca);
    }
    ++k;
}

template <typename T, int V, bool DIFF, bool GM, int MINB>
__global__ void __launch_bounds__(256, MINB) k_reverse_fan(RevArgs<T> A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const long long nb = blockIdx.x / A.nch;
    const int chunk = (int)(blockIdx.x - nb * A.nch);
    const long long a0 = nb * A.npb;
    const long long a1 = (a0 + A.npb < A.n_nodes) ? a0 + A.npb : A.n_nodes;
    const int kb = __ldg(A.node_ptr + a0), ke = __ldg(A.node_ptr + a1);
    const int nsl = ke - kb;
    if (nsl > A.cap_slots) {
        if (threadIdx.x == 0 && A.status) atomicOr(A.status, 2);
        return;
    }
    const uint32_t bar = smem_u32(smem);
    int4* srec = reinterpret_cast<int4*>(smem + 16);
    T* sslab = reinterpret_cast<T*>(smem + 16 + (size_t)A.cap_slots * 16);
    T* sown = sslab + (size_t)A.cap_slots * kSlabStride;
    if (threadIdx.x == 0) mbar_init(bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t b_rec = (uint32_t)nsl * 16u;
        const uint32_t b_slab = (uint32_t)nsl * (uint32_t)(kSlabStride * sizeof(T));
        mbar_arrive_expect_tx(bar, b_rec + 2 * b_slab);
        if (nsl > 0) {
            bulk_g2s(smem_u32(srec), A.rec + kb, b_rec, bar);
            bulk_g2s(smem_u32(sslab), A.slab + (size_t)kb * kSlabStride, b_slab, bar);
            bulk_g2s(smem_u32(sown), A.own + (size_t)kb * kOwnStride, b_slab, bar);
        }
    }
    const long long a = a0 + warp;
    const bool active = warp < A.npb && a < a1;
    const size_t S = (size_t)A.S;
    const size_t col = ((size_t)chunk * 32 + lane) * V;
    const size_t row = (size_t)a * 3 * S + col;
    Vec<T, V> ua[3], ca[3];
    if (active) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            ua[d] = ldg<T, V>(A.u + row + d * S);
            ca[d] = ldg<T, V>(A.x + row + d * S);
            prefetch_l2(A.uo + row + d * S);
            prefetch_l2(A.xo + row + d * S);
        }
        prefetch_l2(A.invm + (size_t)a * S + col);
    }
    if (A.pf_dist > 0 && chunk == 0 && nb % A.pf_group == 0 && warp == A.npb - 1)
        rev_prefetch<T, GM>(A, a0 + A.pf_dist, A.npb * A.pf_group, lane);
    if (!mbar_wait_bounded(bar, 0, kMaxPolls)) {
        if (lane == 0 && A.status) atomicOr(A.status, 1);
        return;
    }
    if (!active) return;
    Vec<T, V> accU[3], accC[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        accU[d] = vzero<T, V>();
        accC[d] = vzero<T, V>();
    }
    const int k0 = __ldg(A.node_ptr + a) - kb, k1 = __ldg(A.node_ptr + a + 1) - kb;
    if (k0 < k1) {
        Vec<T, V> U0[3], U1[3], U2[3], X0[3], X1[3], X2[3], c0, c1, c2;
        const int4 r0 = srec[k0];
        load3<T, V>(U0, A.u, r0.y, S, col);
        load3<T, V>(X0, A.x, r0.y, S, col);
        load3<T, V>(U1, A.u, r0.z, S, col);
        load3<T, V>(X1, A.x, r0.z, S, col);
        c1 = ldg<T, V>(A.coef + (size_t)r0.x * S + col);
        diff3<T, V, DIFF>(U0, ua);
        diff3<T, V, DIFF>(X0, ca);
        int k = k0;
        while (true) {
            rev_phase<T, V, DIFF>(k, k1, srec, sslab, sown, A, S, col, ua, ca, accU, accC, U0, X0, U1,
                                  X1, c1, U2, X2, c2);
            if (k >= k1) break;
            rev_phase<T, V, DIFF>(k, k1, srec, sslab, sown, A, S, col, ua, ca, accU, accC, U1, X1, U2,
                                  X2, c2, U0, X0, c0);
            if (k >= k1) break;
            rev_phase<T, V, DIFF>(k, k1, srec, sslab, sown, A, S, col, ua, ca, accU, accC, U2, X2, U0,
                                  X0, c0, U1, X1, c1);
            if (k >= k1) break;
        }
    }
    rev_epilogue<T, V, GM>(A, a, S, col, row, ua, ca, accU, accC);
}

// ------------------------------------------------------------ persistent reverse step
// k_reverse_fan as a persistent grid: each block walks work items (node block, sample
// chunk; chunk fastest) with a stride of the grid and stages the slot records,
// stiffness rows and owner blocks of its NEXT item by TMA into the other of two
// shared-memory stages while its warps run the current one.  Stage s of the block's
// i-th item completes its mbarrier's phase (i / 2) % 2; a block barrier at the end of
// every item frees the stage for reuse.  Same products in the same order: same bits.
template <typename T>
__device__ __forceinline__ void revp_issue(const RevArgs<T>& A, long long w, uint32_t bar,
                                           int4* srec, T* sslab, T* sown) {
    const long long nb = w / A.nch;
    const long long a0 = nb * A.npb;
    const long long a1 = (a0 + A.npb < A.n_nodes) ? a0 + A.npb : A.n_nodes;
    const int kb = __ldg(A.node_ptr + a0), ke = __ldg(A.node_ptr + a1);
    const int nsl = ke - kb;
    if (nsl > A.cap_slots || nsl <= 0) {
        if (nsl > A.cap_slots && A.status) atomicOr(A.status, 2);
        mbar_arrive_expect_tx(bar, 0);
        return;
    }
    const uint32_t b_rec = (uint32_t)nsl * 16u;
    const uint32_t b_slab = (uint32_t)nsl * (uint32_t)(kSlabStride * sizeof(T));
    mbar_arrive_expect_tx(bar, b_rec + 2 * b_slab);
    bulk_g2s(smem_u32(srec), A.rec + kb, b_rec, bar);
    bulk_g2s(smem_u32(sslab), A.slab + (size_t)kb * kSlabStride, b_slab, bar);
    bulk_g2s(smem_u32(sown), A.own + (size_t)kb * kOwnStride, b_slab, bar);
}

template <typename T, int V, bool DIFF, bool GM, int MINB>
__global__ void __launch_bounds__(256, MINB) k_reverse_fanp(RevArgs<T> A, long long n_items) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const size_t cap = (size_t)A.cap_slots;
    const size_t stage_bytes = cap * (16 + 2 * kSlabStride * sizeof(T));
    // stage q: records, stiffness rows, owner blocks at smem + 16 + q * stage_bytes
    const uint32_t bar0 = smem_u32(smem);
    auto srec_of = [&](int q) {
        return reinterpret_cast<int4*>(smem + 16 + q * stage_bytes);
    };
    auto sslab_of = [&](int q) {
        return reinterpret_cast<T*>(smem + 16 + q * stage_bytes + cap * 16);
    };
    auto sown_of = [&](int q) { return sslab_of(q) + cap * kSlabStride; };
    if (threadIdx.x == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
    }
    __syncthreads();
    long long w = blockIdx.x;
    if (threadIdx.x == 0 && w < n_items) revp_issue<T>(A, w, bar0, srec_of(0), sslab_of(0), sown_of(0));
    const size_t S = (size_t)A.S;
    for (int it = 0; w < n_items; w += gridDim.x, ++it) {
        const int sg = it & 1;
        const long long wn = w + gridDim.x;
        if (threadIdx.x == 0 && wn < n_items)
            revp_issue<T>(A, wn, bar0 + 8 * (sg ^ 1), srec_of(sg ^ 1), sslab_of(sg ^ 1),
                          sown_of(sg ^ 1));
        const long long nb = w / A.nch;
        const int chunk = (int)(w - nb * A.nch);
        const long long a0 = nb * A.npb;
        const long long a1 = (a0 + A.npb < A.n_nodes) ? a0 + A.npb : A.n_nodes;
        const long long a = a0 + warp;
        const bool active = warp < A.npb && a < a1;
        const size_t col = ((size_t)chunk * 32 + lane) * V;
        const size_t row = (size_t)a * 3 * S + col;
        Vec<T, V> ua[3], ca[3];
        if (active) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                ua[d] = ldg<T, V>(A.u + row + d * S);
                ca[d] = ldg<T, V>(A.x + row + d * S);
                prefetch_l2(A.uo + row + d * S);
                prefetch_l2(A.xo + row + d * S);
            }
            prefetch_l2(A.invm + (size_t)a * S + col);
        }
        if (A.pf_dist > 0 && chunk == 0 && nb % A.pf_group == 0 && warp == A.npb - 1)
            rev_prefetch<T, GM>(A, a0 + A.pf_dist, A.npb * A.pf_group, lane);
        if (!mbar_wait_bounded(bar0 + 8 * sg, (uint32_t)((it >> 1) & 1), kMaxPolls)) {
            if (lane == 0 && A.status) atomicOr(A.status, 1);
            return;
        }
        if (active) {
            const int4* srec = srec_of(sg);
            const T* sslab = sslab_of(sg);
            const T* sown = sown_of(sg);
            const int kb = __ldg(A.node_ptr + a0);
            Vec<T, V> accU[3], accC[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                accU[d] = vzero<T, V>();
                accC[d] = vzero<T, V>();
            }
            const int k0 = __ldg(A.node_ptr + a) - kb, k1 = __ldg(A.node_ptr + a + 1) - kb;
            if (k0 < k1) {
                Vec<T, V> U0[3], U1[3], U2[3], X0[3], X1[3], X2[3], c0, c1, c2;
                const int4 r0 = srec[k0];
                load3<T, V>(U0, A.u, r0.y, S, col);
                load3<T, V>(X0, A.x, r0.y, S, col);
                load3<T, V>(U1, A.u, r0.z, S, col);
                load3<T, V>(X1, A.x, r0.z, S, col);
                c1 = ldg<T, V>(A.coef + (size_t)r0.x * S + col);
                diff3<T, V, DIFF>(U0, ua);
                diff3<T, V, DIFF>(X0, ca);
                int k = k0;
                while (true) {
                    rev_phase<T, V, DIFF>(k, k1, srec, sslab, sown, A, S, col, ua, ca, accU, accC,
                                          U0, X0, U1, X1, c1, U2, X2, c2);
                    if (k >= k1) break;
                    rev_phase<T, V, DIFF>(k, k1, srec, sslab, sown, A, S, col, ua, ca, accU, accC,
                                          U1, X1, U2, X2, c2, U0, X0, c0);
                    if (k >= k1) break;
                    rev_phase<T, V, DIFF>(k, k1, srec, sslab, sown, A, S, col, ua, ca, accU, accC,
                                          U2, X2, U0, X0, c0, U1, X1, c1);
                    if (k >= k1) break;
                }
            }
            rev_epilogue<T, V, GM>(A, a, S, col, row, ua, ca, accU, accC);
        }
        __syncthreads();
    }
}

// dJ/dlogE = -c Gamma; dJ/dlogh = -c Gamma - h sum_a alpha_{e,a} G_a / m_a.
template <typename T>
__global__ void k_grad_final(long long n_elems, int S, const int32_t* __restrict__ elems,
                             const double* __restrict__ area, MassWeights mw,
                             const double* __restrict__ lm, const double* __restrict__ logE,
                             const double* __restrict__ logh, const T* __restrict__ gam,
                             const T* __restrict__ gm, double* __restrict__ gE,
                             double* __restrict__ gh) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long e = g / S;
    if (e >= n_elems) return;
    const int s = (int)(g - e * S);
    const size_t o = (size_t)e * S + s;
    const double h = exp(logh[o]);
    const double c = exp(logE[o]) * h;
    const double ge = -c * (double)gam[o];
    if (gE) gE[o] = ge;
    if (gh) {
        double m = 0.0;
        if (gm) {
#pragma unroll
            for (int la = 0; la < 3; ++la) {
                const size_t na = (size_t)elems[3 * e + la];
                const double alpha = area[e] * (mw.w[3 * la] + mw.w[3 * la + 1] + mw.w[3 * la + 2]);
                m += alpha * (double)gm[na * S + s] / lm[na * S + s];
            }
        }
        gh[o] = ge - h * m;
    }
}

struct RevTuning {
    int vec;      // samples per thread (upper bound)
    int npb;      // nodes (warps) per block of the fan kernel
    int variant;  // 0: L1-gather kernel; 1: fan-rotation kernel with staged slots;
                  // 2: as 1, persistent, the next item's slots staged under the current
    int minb;     // resident blocks per SM asked of the compiler (fan kernel)
};
// Defaults from sweeps on B200: FP32 on the 256x1024 tube with 128 samples and the
// stenosed 512x2048 tube (reverse 6.25 s per 1000 steps; the persistent variant 7.89 s);
// FP64 on the 64x128 tube with 64 samples (reverse pass of 500 steps: vec 1 with 4 nodes
// per block 29.6 ms, vec 2 with 2 nodes 30.6 ms, persistent 30.2 ms).
static RevTuning g_rev32 = {2, 2, 1, 2};
static RevTuning g_rev64 = {1, 4, 2, 2};
template <typename T>
RevTuning& rev_tuning() {
    return sizeof(T) == 4 ? g_rev32 : g_rev64;
}

constexpr size_t kRevMaxStage = 160 * 1024;

template <typename Kern, typename T>
int launch_rev_fan(Kern kernel, unsigned grid, int threads, size_t smem, cudaStream_t st,
                   const RevArgs<T>& A) {
    if (smem > 48 * 1024) {
        cudaError_t e =
            cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess)
            return fail(CVFES_ERR_CUDA, "k_reverse_fan smem attribute: %s", cudaGetErrorString(e));
    }
    kernel<<<grid, threads, smem, st>>>(A);
    CVFES_LAUNCH_CHECK("k_reverse_fan");
    return CVFES_OK;
}

template <typename T, int V, bool DIFF, bool GM>
int launch_rev_fan_m(int minb, unsigned grid, int threads, size_t smem, cudaStream_t st,
                     const RevArgs<T>& A) {
    switch (minb) {
        case 4: return launch_rev_fan(k_reverse_fan<T, V, DIFF, GM, 4>, grid, threads, smem, st, A);
        case 3: return launch_rev_fan(k_reverse_fan<T, V, DIFF, GM, 3>, grid, threads, smem, st, A);
        case 2: return launch_rev_fan(k_reverse_fan<T, V, DIFF, GM, 2>, grid, threads, smem, st, A);
        default: return launch_rev_fan(k_reverse_fan<T, V, DIFF, GM, 1>, grid, threads, smem, st, A);
    }
}

// The persistent reverse kernel on as many blocks as are resident (at most one per item).
template <typename Kern, typename T>
int launch_rev_fanp(Kern kernel, long long n_items, int threads, size_t smem, cudaStream_t st,
                    const RevArgs<T>& A) {
    int per_sm = 0;
    const int rc =
        fanp_blocks_per_sm(reinterpret_cast<const void*>(kernel), threads, smem, &per_sm);
    if (rc) return rc;
    long long blocks = (long long)per_sm * device_sm_count();
    if (blocks > n_items) blocks = n_items;
    kernel<<<(unsigned)blocks, threads, smem, st>>>(A, n_items);
    CVFES_LAUNCH_CHECK("k_reverse_fanp");
    return CVFES_OK;
}

template <typename T, int V, bool DIFF, bool GM>
int launch_rev_fanp_m(int minb, long long n_items, int threads, size_t smem, cudaStream_t st,
                      const RevArgs<T>& A) {
    switch (minb) {
        case 3:
            return launch_rev_fanp(k_reverse_fanp<T, V, DIFF, GM, 3>, n_items, threads, smem, st,
                                   A);
        case 2:
            return launch_rev_fanp(k_reverse_fanp<T, V, DIFF, GM, 2>, n_items, threads, smem, st,
                                   A);
        default:
            return launch_rev_fanp(k_reverse_fanp<T, V, DIFF, GM, 1>, n_items, threads, smem, st,
                                   A);
    }
}

template <typename T, int V, bool DIFF>
int launch_rev_v(const RevTuning& tu, bool fan, bool gmv, unsigned fan_grid, size_t smem,
                 const RowGrid& rg, cudaStream_t st, const RevArgs<T>& A) {
    if (fan && tu.variant == 2) {
        const int threads = 32 * tu.npb;
        const size_t smem2 = 16 + 2 * (smem - 16);
        return gmv ? launch_rev_fanp_m<T, V, DIFF, true>(tu.minb, fan_grid, threads, smem2, st, A)
                   : launch_rev_fanp_m<T, V, DIFF, false>(tu.minb, fan_grid, threads, smem2, st,
                                                          A);
    }
    if (fan) {
        const int threads = 32 * tu.npb;
        return gmv ? launch_rev_fan_m<T, V, DIFF, true>(tu.minb, fan_grid, threads, smem, st, A)
                   : launch_rev_fan_m<T, V, DIFF, false>(tu.minb, fan_grid, threads, smem, st, A);
    }
    if (gmv) k_reverse<T, V, DIFF, true><<<rg.grid, 256, 0, st>>>(A);
    else k_reverse<T, V, DIFF, false><<<rg.grid, 256, 0, st>>>(A);
    CVFES_LAUNCH_CHECK("k_reverse");
    return CVFES_OK;
}

template <typename T>
int launch_reverse_step(const cvfes_adjoint_desc* d, const T* u, T* uo, const T* x, T* xo,
                        long long n, cudaStream_t st) {
    const cvfes_solid_mesh* m = &d->mesh;
    RevArgs<T> A;
    A.node_ptr = m->node_ptr;
    A.rec = reinterpret_cast<const int4*>(m->slot_rec);
    A.slab = static_cast<const T*>(m->slot_k);
    A.own = static_cast<const T*>(d->owner_blocks);
    A.fhat = static_cast<const T*>(m->fhat);
    A.coef = static_cast<const T*>(d->coef);
    A.invm = static_cast<const T*>(d->invm);
    A.u = u;
    A.uo = uo;
    A.x = x;
    A.xo = xo;
    A.gam = static_cast<T*>(d->gamma);
    A.gm = static_cast<T*>(d->gmass);
    A.p = d->p_sched + n;
    A.n_nodes = m->n_nodes;
    A.S = (int)m->n_samples;
    A.n_clamped = (int)m->n_clamped;
    A.clamp = (T)m->clamp_value;
    A.status = m->status;
    const double g = 0.5 * d->dt * d->damp;
    const double eta = d->dt * d->damp / (1.0 + g);
    A.eta = (T)eta;
    A.inv1meta = (T)(1.0 / (1.0 - eta));
    A.w0 = (T)(d->dt * d->dt / (1.0 + g));
    const RevTuning tu = rev_tuning<T>();
    const Prefetch pf = step_prefetch(sizeof(T) == 4 ? 32 : 64, m->bandwidth);
    A.pf_dist = pf.dist;
    A.pf_parts = pf.parts;
    const void* ptrs[8] = {d->coef, d->invm, u, uo, x, xo, d->gamma, d->gmass};
    int V = (int)(16 / sizeof(T));
    while (V > tu.vec) V /= 2;
    for (; V > 1; V /= 2) {
        bool ok = A.S % V == 0;
        for (int i = 0; i < 8; ++i)
            if (ptrs[i] && reinterpret_cast<uintptr_t>(ptrs[i]) % (V * sizeof(T))) ok = false;
        if (ok) break;
    }
    const RowGrid rg = row_grid(m->n_nodes, A.S / V, 256);
    A.tpn = rg.tpn;
    A.npb = rg.npb;
    A.nch = 1;
    A.cap_slots = 0;
    const long long cap = (long long)tu.npb * m->max_degree;
    const size_t smem = 16 + (size_t)cap * (16 + (kSlabStride + kOwnStride) * sizeof(T));
    const bool fan = (tu.variant == 1 || tu.variant == 2) && m->max_degree > 0 &&
                     (A.S / V) % 32 == 0 && smem <= kRevMaxStage && tu.npb >= 1 && tu.npb <= 8;
    unsigned fan_grid = 0;
    if (fan) {
        A.npb = tu.npb;
        A.tpn = 32;
        A.nch = A.S / V / 32;
        A.pf_group = prefetch_group(A.nch);
        A.pf_parts = prefetch_parts(A.pf_parts, A.nch);
        A.cap_slots = (int)cap;
        fan_grid = (unsigned)(((m->n_nodes + A.npb - 1) / A.npb) * A.nch);
    }
    constexpr bool DIFF = std::is_same<T, float>::value;
    const bool gmv = d->gmass != nullptr;
    if (V == 4) {
        if constexpr (sizeof(T) == 4)
            return launch_rev_v<T, 4, DIFF>(tu, fan, gmv, fan_grid, smem, rg, st, A);
        return fail(CVFES_ERR_UNSUPPORTED, "k_reverse: vec 4 is FP32 only");
    }
    if (V == 2) return launch_rev_v<T, 2, DIFF>(tu, fan, gmv, fan_grid, smem, rg, st, A);
    return launch_rev_v<T, 1, DIFF>(tu, fan, gmv, fan_grid, smem, rg, st, A);
}

int check_adjoint(const cvfes_adjoint_desc* d, const char* who) {
    if (!d) return fail(CVFES_ERR_ARG, "%s: null descriptor", who);
    const cvfes_solid_mesh* m = &d->mesh;
    if (m->n_nodes <= 0 || m->n_samples <= 0 || m->n_samples > INT32_MAX || !m->node_ptr ||
        !m->slot_rec || !m->slot_k || !m->fhat)
        return fail(CVFES_ERR_ARG, "%s: incomplete mesh descriptor", who);
    if (d->precision != 32 && d->precision != 64)
        return fail(CVFES_ERR_ARG, "%s: precision must be 32 or 64", who);
    if (d->n_steps <= 0 || d->ckpt_every <= 0 || d->obs_every <= 0 || d->n_obs < 0)
        return fail(CVFES_ERR_ARG, "%s: steps, checkpoint and observation intervals must be "
                    "positive", who);
    if (!d->coef || !d->invm || !d->owner_blocks || !d->state[0] || !d->state[1] ||
        !d->state[2] || !d->adj[0] || !d->adj[1] || !d->ckpt || !d->p_sched || !d->clock ||
        !d->J || !d->gamma)
        return fail(CVFES_ERR_ARG, "%s: null buffer", who);
    if (d->n_obs > 0 && (!d->obs_nodes || !d->obs || !d->jpart))
        return fail(CVFES_ERR_ARG, "%s: observation buffers missing", who);
    if (!(d->dt > 0.0)) return fail(CVFES_ERR_ARG, "%s: dt must be positive", who);
    return CVFES_OK;
}

template <typename T>
int adjoint_forward(const cvfes_adjoint_desc* d, int* out_cur, int* out_prev, cudaStream_t st) {
    int rc = check_adjoint(d, "cvfes_adjoint_forward");
    if (rc) return rc;
    const cvfes_solid_mesh* m = &d->mesh;
    const long long S = m->n_samples, N = m->n_nodes, T_ = d->n_steps;
    const long long C = d->ckpt_every, K = d->obs_every;
    const size_t state = (size_t)3 * N * S;
    const size_t sbytes = state * sizeof(T);
    T* buf[3] = {static_cast<T*>(d->state[0]), static_cast<T*>(d->state[1]),
                 static_cast<T*>(d->state[2])};
    T* ck = static_cast<T*>(d->ckpt);
    T* obs = static_cast<T*>(d->obs);
    for (int q = 0; q < 3; ++q) CVFES_CUDA_TRY(cudaMemsetAsync(buf[q], 0, sbytes, st));
    CVFES_CUDA_TRY(cudaMemsetAsync(d->clock, 0, sizeof(int64_t), st));
    CVFES_CUDA_TRY(cudaMemsetAsync(d->J, 0, S * sizeof(double), st));
    const int nchunk = (d->n_obs + kObsChunk - 1) / kObsChunk;
    int cur = 0, prev = 1, nxt = 2;
    long long n = 0;
    while (n < T_) {
        long long next = T_;
        const long long no = (n / K + 1) * K;
        if (no < next) next = no;
        long long mc = (n / C) * C + 1;
        if (mc <= n) mc += C;
        if (mc < next) next = mc;
        int ci = 0, pi = 1;
        const int order[3] = {cur, prev, nxt};
        if constexpr (sizeof(T) == 8)
            rc = cvfes_solid_advance_f64(m, static_cast<const double*>(d->coef),
                                         static_cast<const double*>(d->invm), buf[cur], buf[prev],
                                         buf[nxt], d->p_sched, d->clock, next - n, d->dt, d->damp,
                                         &ci, &pi, st);
        else
            rc = cvfes_solid_advance_f32(m, static_cast<const float*>(d->coef),
                                         static_cast<const float*>(d->invm), buf[cur], buf[prev],
                                         buf[nxt], d->p_sched, d->clock, next - n, d->dt, d->damp,
                                         &ci, &pi, st);
        if (rc) return rc;
        cur = order[ci];
        prev = order[pi];
        nxt = 3 - cur - prev;
        n = next;
        if ((n - 1) % C == 0) {
            T* slot = ck + (size_t)((n - 1) / C) * 2 * state;
            CVFES_CUDA_TRY(cudaMemcpyAsync(slot, buf[prev], sbytes, cudaMemcpyDeviceToDevice, st));
            CVFES_CUDA_TRY(
                cudaMemcpyAsync(slot + state, buf[cur], sbytes, cudaMemcpyDeviceToDevice, st));
        }
        if (n % K == 0 && d->n_obs > 0) {
            const long long k = n / K - 1;
            dim3 grid((unsigned)nchunk, (unsigned)((S + 127) / 128));
            k_obs<T><<<grid, 128, 0, st>>>(d->n_obs, (int)S, d->obs_nodes, buf[cur],
                                           obs + (size_t)k * d->n_obs * 3 * S,
                                           d->jpart + (size_t)k * nchunk * S, d->record);
            CVFES_LAUNCH_CHECK("k_obs");
        }
    }
    const long long n_obs_steps = T_ / K;
    if (!d->record && d->n_obs > 0 && n_obs_steps > 0) {
        k_obs_reduce<<<(unsigned)((S + 127) / 128), 128, 0, st>>>(n_obs_steps * nchunk, (int)S,
                                                                 d->jpart, d->J);
        CVFES_LAUNCH_CHECK("k_obs_reduce");
    }
    if (out_cur) *out_cur = cur;
    if (out_prev) *out_prev = prev;
    return CVFES_OK;
}

template <typename T>
int adjoint_force(const cvfes_adjoint_desc* d, const T* u, T* chi, long long k, cudaStream_t st) {
    if (d->n_obs <= 0) return CVFES_OK;
    const long long S = d->mesh.n_samples;
    const double g = 0.5 * d->dt * d->damp;
    const T w0 = (T)(d->dt * d->dt / (1.0 + g));
    k_adj_force<T><<<grid_1d((long long)d->n_obs * S, 256), 256, 0, st>>>(
        d->n_obs, (int)S, d->obs_nodes, (int)d->mesh.n_clamped, static_cast<const T*>(d->invm),
        w0, u, static_cast<const T*>(d->obs) + (size_t)k * d->n_obs * 3 * S, chi);
    CVFES_LAUNCH_CHECK("k_adj_force");
    return CVFES_OK;
}

template <typename T>
int adjoint_reverse(const cvfes_adjoint_desc* d, int cur, int prev, cudaStream_t st) {
    int rc = check_adjoint(d, "cvfes_adjoint_reverse");
    if (rc) return rc;
    if (cur < 0 || cur > 2 || prev < 0 || prev > 2 || cur == prev)
        return fail(CVFES_ERR_ARG, "cvfes_adjoint_reverse: bad final state roles");
    const cvfes_solid_mesh* m = &d->mesh;
    const long long S = m->n_samples, N = m->n_nodes, E = m->n_elems, T_ = d->n_steps;
    const long long C = d->ckpt_every, K = d->obs_every;
    const size_t state = (size_t)3 * N * S;
    const size_t sbytes = state * sizeof(T);
    T* uA = static_cast<T*>(d->state[prev]);  // u_n      (starts at u_{T-1})
    T* uB = static_cast<T*>(d->state[cur]);   // u_{n+1}  (starts at u_T)
    T* xA = static_cast<T*>(d->adj[0]);       // chi_{n+1}
    T* xB = static_cast<T*>(d->adj[1]);       // chi_{n+2}
    const T* ck = static_cast<const T*>(d->ckpt);
    CVFES_CUDA_TRY(cudaMemsetAsync(xA, 0, sbytes, st));
    CVFES_CUDA_TRY(cudaMemsetAsync(xB, 0, sbytes, st));
    CVFES_CUDA_TRY(cudaMemsetAsync(d->gamma, 0, (size_t)E * S * sizeof(T), st));
    if (d->gmass) CVFES_CUDA_TRY(cudaMemsetAsync(d->gmass, 0, (size_t)N * S * sizeof(T), st));
    if (T_ % K == 0) {
        rc = adjoint_force<T>(d, uB, xA, T_ / K - 1, st);
        if (rc) return rc;
    }
    for (long long n = T_ - 1; n >= 0; --n) {
        if (n % C == 0) {
            const T* slot = ck + (size_t)(n / C) * 2 * state;
            CVFES_CUDA_TRY(cudaMemcpyAsync(uA, slot, sbytes, cudaMemcpyDeviceToDevice, st));
            CVFES_CUDA_TRY(
                cudaMemcpyAsync(uB, slot + state, sbytes, cudaMemcpyDeviceToDevice, st));
        }
        rc = launch_reverse_step<T>(d, uA, uB, xA, xB, n, st);
        if (rc) return rc;
        T* t = uA;
        uA = uB;
        uB = t;
        t = xA;
        xA = xB;
        xB = t;
        // now uA = u_{n-1}, uB = u_n, xA = chi_n, xB = chi_{n+1}
        if (n > 0 && n % K == 0) {
            rc = adjoint_force<T>(d, uB, xA, n / K - 1, st);
            if (rc) return rc;
        }
    }
    return CVFES_OK;
}

template <typename F>
int capture(F&& issue, cvfes_graph** out) {
    cudaStream_t cs;
    CVFES_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaStreamDestroy(cs);
        return fail(CVFES_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e));
    }
    const int rc = issue(cs);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(cs, &graph);
    cudaStreamDestroy(cs);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return fail(CVFES_ERR_CUDA, "end capture: %s", cudaGetErrorString(e));
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        return fail(CVFES_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
    }
    *out = new cvfes_graph{graph, exec};
    return CVFES_OK;
}

}  // namespace cvfes

using namespace cvfes;

extern "C" int cvfes_set_adjoint_tuning(int32_t precision, int32_t vec, int32_t npb,
                                        int32_t variant, int32_t minb) {
    if ((precision != 32 && precision != 64) || (vec != 1 && vec != 2 && vec != 4) ||
        (precision == 64 && vec == 4) || npb < 1 || npb > 8 || variant < 0 || variant > 2 ||
        minb < 1 || minb > 4 || (variant == 2 && minb > 3))
        return fail(CVFES_ERR_ARG, "cvfes_set_adjoint_tuning: bad argument");
    RevTuning& t = precision == 32 ? g_rev32 : g_rev64;
    t = RevTuning{vec, npb, variant, minb};
    return CVFES_OK;
}

extern "C" int cvfes_get_adjoint_tuning(int32_t precision, int32_t* vec, int32_t* npb,
                                        int32_t* variant, int32_t* minb) {
    if (precision != 32 && precision != 64)
        return fail(CVFES_ERR_ARG, "cvfes_get_adjoint_tuning: precision must be 32 or 64");
    const RevTuning& t = precision == 32 ? g_rev32 : g_rev64;
    if (vec) *vec = t.vec;
    if (npb) *npb = t.npb;
    if (variant) *variant = t.variant;
    if (minb) *minb = t.minb;
    return CVFES_OK;
}

extern "C" int64_t cvfes_adjoint_ckpt_count(int64_t n_steps, int64_t ckpt_every) {
    if (n_steps <= 0 || ckpt_every <= 0) return 0;
    return (n_steps + ckpt_every - 1) / ckpt_every;
}

extern "C" int64_t cvfes_adjoint_jpart_size(int64_t n_steps, int32_t obs_every, int32_t n_obs,
                                            int64_t n_samples) {
    if (n_steps <= 0 || obs_every <= 0 || n_obs <= 0 || n_samples <= 0) return 0;
    return (n_steps / obs_every) * ((n_obs + kObsChunk - 1) / kObsChunk) * n_samples;
}

extern "C" int cvfes_adjoint_owner_blocks(const cvfes_solid_mesh* mesh, int32_t precision,
                                          const int32_t* elems, const int32_t* elem_slot,
                                          void* out, void* stream) {
    if (!mesh || mesh->n_elems <= 0 || !mesh->slot_rec || !mesh->slot_k || !elems || !elem_slot ||
        !out || (precision != 32 && precision != 64))
        return fail(CVFES_ERR_ARG, "cvfes_adjoint_owner_blocks: bad argument");
    const long long E = mesh->n_elems;
    if (precision == 64)
        k_owner_blocks<double><<<grid_1d(E, 256), 256, 0, (cudaStream_t)stream>>>(
            E, elems, elem_slot, mesh->slot_rec, static_cast<const double*>(mesh->slot_k),
            static_cast<double*>(out));
    else
        k_owner_blocks<float><<<grid_1d(E, 256), 256, 0, (cudaStream_t)stream>>>(
            E, elems, elem_slot, mesh->slot_rec, static_cast<const float*>(mesh->slot_k),
            static_cast<float*>(out));
    CVFES_LAUNCH_CHECK("k_owner_blocks");
    return CVFES_OK;
}

extern "C" int cvfes_adjoint_material(int64_t n_elems, int64_t n_samples, const double* logE,
                                      const double* logh, double* coef64, float* coef32,
                                      double* thick, void* stream) {
    if (n_elems <= 0 || n_samples <= 0 || !logE || !logh || (!coef64 && !coef32 && !thick))
        return fail(CVFES_ERR_ARG, "cvfes_adjoint_material: bad argument");
    const long long n = n_elems * n_samples;
    k_material_log<<<grid_1d(n, 256), 256, 0, (cudaStream_t)stream>>>(n, logE, logh, coef64,
                                                                        coef32, thick);
    CVFES_LAUNCH_CHECK("k_material_log");
    return CVFES_OK;
}

extern "C" int cvfes_adjoint_forward(const cvfes_adjoint_desc* d, int32_t* final_cur,
                                     int32_t* final_prev, void* stream) {
    if (!d) return fail(CVFES_ERR_ARG, "cvfes_adjoint_forward: null descriptor");
    if (d->precision == 64) return adjoint_forward<double>(d, final_cur, final_prev, (cudaStream_t)stream);
    return adjoint_forward<float>(d, final_cur, final_prev, (cudaStream_t)stream);
}

extern "C" int cvfes_adjoint_reverse(const cvfes_adjoint_desc* d, int32_t final_cur,
                                     int32_t final_prev, void* stream) {
    if (!d) return fail(CVFES_ERR_ARG, "cvfes_adjoint_reverse: null descriptor");
    if (d->precision == 64) return adjoint_reverse<double>(d, final_cur, final_prev, (cudaStream_t)stream);
    return adjoint_reverse<float>(d, final_cur, final_prev, (cudaStream_t)stream);
}

extern "C" int cvfes_adjoint_gradients(const cvfes_adjoint_desc* d, const int32_t* elems,
                                       const double* area, const double* mass_weights,
                                       const double* lm, const double* logE, const double* logh,
                                       double* grad_logE, double* grad_logh, void* stream) {
    int rc = check_adjoint(d, "cvfes_adjoint_gradients");
    if (rc) return rc;
    if (!elems || !area || !logE || !logh || (!grad_logE && !grad_logh))
        return fail(CVFES_ERR_ARG, "cvfes_adjoint_gradients: bad argument");
    if (grad_logh && (!d->gmass || !lm || !mass_weights))
        return fail(CVFES_ERR_ARG,
                    "cvfes_adjoint_gradients: the log h gradient needs the G accumulator, the "
                    "lumped mass and the mass weights");
    MassWeights mw{};
    if (mass_weights)
        for (int i = 0; i < 9; ++i) mw.w[i] = mass_weights[i];
    const long long E = d->mesh.n_elems, S = d->mesh.n_samples;
    if (d->precision == 64)
        k_grad_final<double><<<grid_1d(E * S, 256), 256, 0, (cudaStream_t)stream>>>(
            E, (int)S, elems, area, mw, lm, logE, logh, static_cast<const double*>(d->gamma),
            static_cast<const double*>(d->gmass), grad_logE, grad_logh);
    else
        k_grad_final<float><<<grid_1d(E * S, 256), 256, 0, (cudaStream_t)stream>>>(
            E, (int)S, elems, area, mw, lm, logE, logh, static_cast<const float*>(d->gamma),
            static_cast<const float*>(d->gmass), grad_logE, grad_logh);
    CVFES_LAUNCH_CHECK("k_grad_final");
    return CVFES_OK;
}

extern "C" int cvfes_adjoint_capture(const cvfes_adjoint_desc* d, int32_t which, int32_t cur,
                                     int32_t prev, int32_t* final_cur, int32_t* final_prev,
                                     cvfes_graph** out) {
    if (!d || !out || (which != 0 && which != 1))
        return fail(CVFES_ERR_ARG, "cvfes_adjoint_capture: bad argument");
    return capture(
        [&](cudaStream_t cs) -> int {
            if (which == 0) return cvfes_adjoint_forward(d, final_cur, final_prev, cs);
            return cvfes_adjoint_reverse(d, cur, prev, cs);
        },
        out);
}
