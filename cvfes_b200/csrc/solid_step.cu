// Per-step kernels of the ensemble membrane solid time step.
//
// Layout: state u[3N][S] with samples innermost.  One thread owns one node and
// VEC consecutive samples; it walks the node's incident elements in fan order,
// gathers the two other nodes' displacements (16-byte vector loads across
// samples), multiplies by the element's 3x9 stiffness rows (shared by all
// samples) and the element's per-sample coefficient E*h, and accumulates the
// node's row of K_s u_s in registers.  No scatter, no atomics, no colouring:
// every row is owned by exactly one thread.  The explicit damped update
// (physicsSolver.py:272-285, physicsSolverSDampGPUs.cl:416-446) and the
// Dirichlet rows are fused into the same pass, so each step reads u_n, u_{n-1},
// the inverse mass and the coefficients once and writes u_{n+1} once.
//
// The update is evaluated in increment form
//     dv = u_n - u_{n-1};  v = dv - eta*dv + w*(p*fhat - K u_n);  u_{n+1} = u_n + v
//     eta = dt*damp/(1 + dt*damp/2),  w = dt^2/((1 + dt*damp/2) m)
// which is the reference's (dt^2 f + 2 m u - dt^2 K u + (dt/2 c - m) u_prev)/(m + dt/2 c)
// with c = damp*m, rearranged so that the coefficients multiplying u_n carry no
// rounding error (this matters for the FP32 state form).
//
// FP32 form (DIFF): each element row is applied to neighbour differences
// (u_b - u_a); the self block is minus the sum of the two others, so rigid
// translations are exactly in the null space and the FP32 cancellation error
// scales with |u_b - u_a| instead of |u|.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <type_traits>

#include "common.cuh"
#include "step_core.cuh"

namespace cvfes {

template <typename T, int V, bool DIFF>
__global__ void __launch_bounds__(256) k_step(StepArgs<T> A) {
    long long a;
    int vec;
    if (!map_row(A.tpn, A.npb, A.n_nodes, A.S / V, a, vec)) return;
    const size_t S = (size_t)A.S;
    const size_t col = (size_t)vec * V;
    const size_t row = (size_t)a * 3 * S + col;
    if (a < A.n_clamped) {
        clamp_store<T, V>(A, S, row);
        return;
    }
    Vec<T, V> ua[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) ua[d] = ldg<T, V>(A.u + row + d * S);
    T f[3];
    node_load<T>(A, a, step_pressure<T>(A), f);
    Vec<T, V> acc[3];
    ku_row<T, V, DIFF>(A.node_ptr, A.rec, A.slab, A.coef, A.u, S, col, a, ua, acc);
    step_epilogue<T, V>(A, a, S, col, row, ua, acc, f);
}

// ------------------------------------------------------------ TMA-staged step
// Row a of K_s u_s with the node's slot records and stiffness rows read from
// shared memory; the gathers of element k+1 are issued before element k is
// multiplied, so two elements' loads are in flight per warp.
template <typename T, int V, bool DIFF>
__device__ __forceinline__ void ku_row_staged(const int4* srec, const T* sslab, int k0, int k1,
                                              const T* __restrict__ u, const T* __restrict__ coef,
                                              size_t S, size_t col, const Vec<T, V> (&ua)[3],
                                              Vec<T, V> (&acc)[3]) {
#pragma unroll
    for (int d = 0; d < 3; ++d) acc[d] = vzero<T, V>();
    if (k0 >= k1) return;
    int4 r = srec[k0];
    Vec<T, V> x1[3], x2[3], c;
    {
        const T* p1 = u + (size_t)r.y * 3 * S + col;
        const T* p2 = u + (size_t)r.z * 3 * S + col;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            x1[d] = ldg<T, V>(p1 + d * S);
            x2[d] = ldg<T, V>(p2 + d * S);
        }
        c = ldg<T, V>(coef + (size_t)r.x * S + col);
    }
#pragma unroll 1
    for (int k = k0; k < k1; ++k) {
        const bool more = k + 1 < k1;
        int4 rn = r;
        Vec<T, V> x2n[3], cn;
        if (more) {
            rn = srec[k + 1];
            const T* p2 = u + (size_t)rn.z * 3 * S + col;
#pragma unroll
            for (int d = 0; d < 3; ++d) x2n[d] = ldg<T, V>(p2 + d * S);
            cn = ldg<T, V>(coef + (size_t)rn.x * S + col);
        }
        const T* K = sslab + (size_t)kSlabStride * k;
        Vec<T, V> d1[3], d2[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            d1[d] = DIFF ? vsub(x1[d], ua[d]) : x1[d];
            d2[d] = DIFF ? vsub(x2[d], ua[d]) : x2[d];
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            Vec<T, V> t = vzero<T, V>();
            if constexpr (!DIFF) {
#pragma unroll
                for (int jj = 0; jj < 3; ++jj) axpy(t, K[3 * i + jj], ua[jj]);
            }
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) axpy(t, K[9 + 3 * i + jj], d1[jj]);
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) axpy(t, K[18 + 3 * i + jj], d2[jj]);
            vfma(acc[i], c, t);
        }
        if (more) {
            if (rn.w & 1) {
#pragma unroll
                for (int d = 0; d < 3; ++d) x1[d] = x2[d];
            } else {
                const T* p1 = u + (size_t)rn.y * 3 * S + col;
#pragma unroll
                for (int d = 0; d < 3; ++d) x1[d] = ldg<T, V>(p1 + d * S);
            }
#pragma unroll
            for (int d = 0; d < 3; ++d) x2[d] = x2n[d];
            c = cn;
            r = rn;
        }
    }
}

// One warp per node and 32*VEC samples of it; a block holds npb consecutive nodes
// of one sample chunk (blockIdx.y).  Thread 0 stages the block's slot records and
// stiffness rows with two TMA bulk copies while every warp loads its node's own
// displacement and prefetches its epilogue rows into L2.
template <typename T, int V, bool DIFF, int MINB>
__global__ void __launch_bounds__(256, MINB) k_step_staged(StepArgs<T> A) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const long long a0 = (long long)blockIdx.x * A.npb;
    const long long a1 = (a0 + A.npb < A.n_nodes) ? a0 + A.npb : A.n_nodes;
    const int kb = __ldg(A.node_ptr + a0), ke = __ldg(A.node_ptr + a1);
    const int nsl = ke - kb;
    if (nsl > A.cap_slots) {  // cannot happen when cap_slots = npb * max_degree
        if (threadIdx.x == 0 && A.status) atomicOr(A.status, 2);
        return;
    }
    const uint32_t bar = smem_u32(smem);
    int4* srec = reinterpret_cast<int4*>(smem + 16);
    T* sslab = reinterpret_cast<T*>(smem + 16 + (size_t)A.cap_slots * 16);
    const bool probe = A.probe_polls > 0;
    if (threadIdx.x == 0) mbar_init(bar, probe ? 2 : 1);
    __syncthreads();
    if (threadIdx.x == 0 && !probe) {
        const uint32_t b_rec = (uint32_t)nsl * 16u;
        const uint32_t b_slab = (uint32_t)nsl * (uint32_t)(kSlabStride * sizeof(T));
        mbar_arrive_expect_tx(bar, b_rec + b_slab);
        if (nsl > 0) {
            bulk_g2s(smem_u32(srec), A.rec + kb, b_rec, bar);
            bulk_g2s(smem_u32(sslab), A.slab + (size_t)kb * kSlabStride, b_slab, bar);
        }
    }
    const long long a = a0 + warp;
    const bool active = warp < A.npb && a < a1;
    const size_t S = (size_t)A.S;
    const size_t col = ((size_t)blockIdx.y * 32 + lane) * V;
    const size_t row = (size_t)a * 3 * S + col;
    const bool clamped = a < A.n_clamped;
    Vec<T, V> ua[3];
    T f[3];
    if (active && !clamped) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            ua[d] = ldg<T, V>(A.u + row + d * S);
            prefetch_l2(A.up + row + d * S);
        }
        prefetch_l2(A.invm + (size_t)a * S + col);
        node_load<T>(A, a, step_pressure<T>(A), f);
    }
    if (!mbar_wait_bounded(bar, 0, kMaxPolls)) {
        if (lane == 0 && A.status) atomicOr(A.status, 1);
        return;
    }
    if (!active) return;
    if (clamped) {
        clamp_store<T, V>(A, S, row);
        return;
    }
    Vec<T, V> acc[3];
    const int k0 = __ldg(A.node_ptr + a) - kb, k1 = __ldg(A.node_ptr + a + 1) - kb;
    ku_row_staged<T, V, DIFF>(srec, sslab, k0, k1, A.u, A.coef, S, col, ua, acc);
    step_epilogue<T, V>(A, a, S, col, row, ua, acc, f);
}

template <typename T, int V, bool DIFF>
__global__ void __launch_bounds__(256)
    k_kmul(const int32_t* node_ptr, const int4* rec, const T* slab, const T* coef, const T* u,
           T* res, long long n_nodes, int S_, int accumulate, int tpn, int npb) {
    long long a;
    int vec;
    if (!map_row(tpn, npb, n_nodes, S_ / V, a, vec)) return;
    const size_t S = (size_t)S_;
    const size_t col = (size_t)vec * V;
    const size_t row = (size_t)a * 3 * S + col;
    Vec<T, V> ua[3], acc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) ua[d] = ldg<T, V>(u + row + d * S);
    ku_row<T, V, DIFF>(node_ptr, rec, slab, coef, u, S, col, a, ua, acc);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        Vec<T, V> o = acc[d];
        if (accumulate) {
            const Vec<T, V> r = ld<T, V>(res + row + d * S);
#pragma unroll
            for (int i = 0; i < V; ++i) o.v[i] += r.v[i];
        }
        st<T, V>(res + row + d * S, o);
    }
}

// u_prev = u0 - dt du0 + dt^2/2 ddu0, ddu0 = (p0 f - damp m du0 - K u0)/m  (0 where m == 0;
// the launcher passes damp = 0 for damping per dof, whose calc_ddu has no damping term);
// in the velocity-state form (vel) the increment u0 - u_prev = dt du0 - dt^2/2 ddu0 instead.
template <typename T>
__global__ void k_init(const T* fhat, const T* invm, const T* u0, const T* du0, const T* ku,
                       T* u_prev, long long n_nodes, int S, T p0, T dt, T damp, int vel) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long a = g / S;
    if (a >= n_nodes) return;
    const int s = (int)(g - a * S);
    const T im = invm[(size_t)a * S + s];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const size_t o = ((size_t)a * 3 + d) * S + s;
        const T m = im != T(0) ? T(1) / im : T(0);
        const T rhs = p0 * fhat[4 * a + d] - damp * m * du0[o] - ku[o];  // damp = 0: per dof
        const T acc = im != T(0) ? rhs * im : T(0);
        u_prev[o] = vel ? dt * du0[o] - T(0.5) * dt * dt * acc
                        : u0[o] - dt * du0[o] + T(0.5) * dt * dt * acc;
    }
}

// res += K v in the reference layout K[nnzb][S][3][3] (MultiplyByVector).
__global__ void k_bsr_spmv(long long n_nodes, int S, const long long* __restrict__ indptr,
                           const long long* __restrict__ indices, const double* __restrict__ K,
                           const double* __restrict__ v, double* __restrict__ res) {
    const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const long long a = g / S;
    if (a >= n_nodes) return;
    const int s = (int)(g - a * S);
    double r0 = 0.0, r1 = 0.0, r2 = 0.0;
    for (long long ia = indptr[a]; ia < indptr[a + 1]; ++ia) {
        const long long b = indices[ia];
        const double* m = K + ((size_t)ia * S + s) * 9;
        const double v0 = v[(3 * b) * S + s], v1 = v[(3 * b + 1) * S + s],
                     v2 = v[(3 * b + 2) * S + s];
        r0 += m[0] * v0 + m[1] * v1 + m[2] * v2;
        r1 += m[3] * v0 + m[4] * v1 + m[5] * v2;
        r2 += m[6] * v0 + m[7] * v1 + m[8] * v2;
    }
    res[(3 * a) * S + s] += r0;
    res[(3 * a + 1) * S + s] += r1;
    res[(3 * a + 2) * S + s] += r2;
}

__global__ void k_clock_add(long long* clock, long long n) { clock[0] += n; }

// ------------------------------------------------------------ fan-rotation step
// TMA-staged slot rows (as k_step_staged) + the fan-rotation row; 1D grid with the
// sample chunk fastest, so the chunks of one node block share its slot rows in L2.
// With pf_dist > 0 the last warp of the first chunk of every pf_group-th node block
// prefetches the rows of the pf_group node blocks pf_dist nodes ahead.
// AHEAD = 2: each element's rows are requested two elements ahead (ku_row_fan2).
template <typename T, int V, bool DIFF, int MINB, int AHEAD = 1>
__global__ void __launch_bounds__(256, MINB) k_step_fan(StepArgs<T> A) {
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
    const bool probe = A.probe_polls > 0;
    if (threadIdx.x == 0) mbar_init(bar, probe ? 2 : 1);
    __syncthreads();
    if (threadIdx.x == 0 && !probe) {
        const uint32_t b_rec = (uint32_t)nsl * 16u;
        const uint32_t b_slab = (uint32_t)nsl * (uint32_t)(kSlabStride * sizeof(T));
        mbar_arrive_expect_tx(bar, b_rec + b_slab);
        if (nsl > 0) {
            bulk_g2s(smem_u32(srec), A.rec + kb, b_rec, bar);
            bulk_g2s(smem_u32(sslab), A.slab + (size_t)kb * kSlabStride, b_slab, bar);
        }
    }
    const long long a = a0 + warp;
    const bool active = warp < A.npb && a < a1;
    const size_t S = (size_t)A.S;
    const size_t col = ((size_t)chunk * 32 + lane) * V;
    const size_t row = (size_t)a * 3 * S + col;
    const bool clamped = a < A.n_clamped;
    Vec<T, V> ua[3];
    T f[3];
    if (active && !clamped) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            ua[d] = ldg<T, V>(A.u + row + d * S);
            if (A.pf_parts & 4) prefetch_l1(A.up + row + d * S);
            else prefetch_l2(A.up + row + d * S);
        }
        if (A.pf_parts & 4) prefetch_l1(A.invm + (size_t)a * S + col);
        else prefetch_l2(A.invm + (size_t)a * S + col);
        node_load<T>(A, a, step_pressure<T>(A), f);
    }
    if (A.pf_dist > 0 && chunk == 0 && nb % A.pf_group == 0 && warp == A.npb - 1)
        fan_prefetch(A, a0 + A.pf_dist, A.npb * A.pf_group, lane);
    if (!mbar_wait_bounded(bar, 0, probe ? A.probe_polls : kMaxPolls)) {
        if (lane == 0 && A.status) atomicOr(A.status, 1);
        return;
    }
    if (!active) return;
    if (clamped) {
        clamp_store<T, V>(A, S, row);
        return;
    }
    Vec<T, V> acc[3];
    const int k0 = __ldg(A.node_ptr + a) - kb, k1 = __ldg(A.node_ptr + a + 1) - kb;
    if constexpr (AHEAD == 2)
        ku_row_fan2<T, V, DIFF>(srec, sslab, k0, k1, A.u, A.coef, S, col, ua, acc);
    else
        ku_row_fan<T, V, DIFF>(srec, sslab, k0, k1, A.u, A.coef, S, col, ua, acc);
    step_epilogue<T, V>(A, a, S, col, row, ua, acc, f);
}

// ------------------------------------------------------------ persistent fan step
// The fan kernel as a persistent grid: each block walks work items (node block, sample
// chunk; chunk fastest) with a stride of the grid, and stages the slot records and
// stiffness rows of its NEXT item by TMA into the other of two shared-memory stages
// while the warps multiply the current one, so the per-item staging latency is off the
// critical path.  Stage s of the block's i-th item completes its mbarrier's phase
// (i / 2) % 2; a block barrier at the end of every item frees the stage for reuse.
template <typename T>
__device__ __forceinline__ void fanp_issue(const StepArgs<T>& A, long long w, uint32_t bar,
                                           int4* srec, T* sslab) {
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
    mbar_arrive_expect_tx(bar, b_rec + b_slab);
    bulk_g2s(smem_u32(srec), A.rec + kb, b_rec, bar);
    bulk_g2s(smem_u32(sslab), A.slab + (size_t)kb * kSlabStride, b_slab, bar);
}

// With A.norm_part (fused norms, shared-memory mode) the grid is a multiple of nch, so
// block b always has sample chunk b % nch; its per-lane FP64 sums follow the two stages
// in shared memory.  Without norms this is the plain persistent step.
template <typename T, int V, bool DIFF, int MINB>
__global__ void __launch_bounds__(256, MINB) k_step_fanp(StepArgs<T> A, long long n_items) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const size_t stage_bytes = (size_t)A.cap_slots * (16 + kSlabStride * sizeof(T));
    // stage q: barrier at smem + 8q, records then stiffness rows at smem + 16 + q * stage_bytes
    const uint32_t bar0 = smem_u32(smem);
    int4* const srec0 = reinterpret_cast<int4*>(smem + 16);
    T* const sslab0 = reinterpret_cast<T*>(smem + 16 + (size_t)A.cap_slots * 16);
    constexpr int kAcc = 4 * V * 32;  // doubles of one warp's norm accumulators
    double* const nbase = reinterpret_cast<double*>(smem + 16 + 2 * stage_bytes);
    double* const nacc = A.norm_part ? nbase + warp * kAcc + lane : nullptr;
    if (nacc) {
#pragma unroll
        for (int q = 0; q < 4 * V; ++q) nacc[q * 32] = 0.0;
    }
    if (threadIdx.x == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
    }
    __syncthreads();
    long long w = blockIdx.x;
    if (threadIdx.x == 0 && w < n_items) fanp_issue<T>(A, w, bar0, srec0, sslab0);
    const size_t S = (size_t)A.S;
    const T p = step_pressure<T>(A);
    for (int it = 0; w < n_items; w += gridDim.x, ++it) {
        const int sg = it & 1;
        const long long wn = w + gridDim.x;
        if (threadIdx.x == 0 && wn < n_items)
            fanp_issue<T>(A, wn, bar0 + 8 * (sg ^ 1), stage_rec(srec0, stage_bytes, sg ^ 1), stage_slab(sslab0, stage_bytes, sg ^ 1));
        const long long nb = w / A.nch;
        const int chunk = (int)(w - nb * A.nch);
        const long long a0 = nb * A.npb;
        const long long a1 = (a0 + A.npb < A.n_nodes) ? a0 + A.npb : A.n_nodes;
        const long long a = a0 + warp;
        const bool active = warp < A.npb && a < a1;
        const size_t col = ((size_t)chunk * 32 + lane) * V;
        const size_t row = (size_t)a * 3 * S + col;
        const bool clamped = a < A.n_clamped;
        Vec<T, V> ua[3];
        T f[3];
        if (active && !clamped) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                ua[d] = ldg<T, V>(A.u + row + d * S);
                prefetch_l2(A.up + row + d * S);
            }
            prefetch_l2(A.invm + (size_t)a * S + col);
            node_load<T>(A, a, p, f);
        }
        // No L2 prefetch ahead here: the prefetching warp's dependent slot-record loads
        // hold its whole block at the item barrier (measured 2.466 -> 3.579 ms/step on the
        // 256x1024 tube with it; node rows alone 3.06 ms).
        if (!mbar_wait_bounded(bar0 + 8 * sg, (uint32_t)((it >> 1) & 1), kMaxPolls)) {
            if (lane == 0 && A.status) atomicOr(A.status, 1);
            return;
        }
        if (active) {
            if (clamped) {
                clamp_store<T, V>(A, S, row, nacc, a, col);
            } else {
                const int kb = __ldg(A.node_ptr + a0);
                const int k0 = __ldg(A.node_ptr + a) - kb, k1 = __ldg(A.node_ptr + a + 1) - kb;
                Vec<T, V> acc[3];
                ku_row_fan<T, V, DIFF>(stage_rec(srec0, stage_bytes, sg),
                                       stage_slab(sslab0, stage_bytes, sg), k0, k1, A.u, A.coef,
                                       S, col, ua, acc);
                step_epilogue<T, V>(A, a, S, col, row, ua, acc, f, nacc);
            }
        }
        __syncthreads();
    }
    if (A.norm_part) {  // this block's sums over its nodes, warps added in order
        const int chunk = (int)(blockIdx.x % A.nch);
        const long long prow = blockIdx.x / A.nch;
        for (int t = threadIdx.x; t < kAcc; t += blockDim.x) {
            const int q = t / (32 * V), c = t - q * 32 * V;  // c: sample of the chunk
            const int ln = c / V, i = c - ln * V;
            double sum = 0.0;
            for (int w = 0; w < A.npb; ++w) sum += nbase[w * kAcc + (q * V + i) * 32 + ln];
            A.norm_part[((size_t)prow * S + (size_t)chunk * 32 * V + c) * 4 + q] = sum;
        }
    }
}

// The persistent step with the norms fused in (tensor-memory mode, the default): the
// grid is a multiple of nch, so block b always has sample chunk b % nch; each lane adds
// its nodes' terms to FP64 sums in tensor memory (norms_add), and at its end the block
// writes one row of partial sums, its warps added in order.  A kernel of its own: the
// plain step without any tensor-memory instruction is 6% faster (2.30 against 2.44
// ms/step on the 256x1024 tube, and 7.2 against 8.1 ms for 500 steps of the 64x128
// tube).  Every wait is bounded: a wait that gives up sets status bit 0, the block stops
// after the item (all warps leave the loop together), waits with a bound for the copies
// it issued, frees its tensor memory and returns.
template <typename T, int V, bool DIFF, int MINB>
__global__ void __launch_bounds__(256, MINB) k_step_fanp_tm(StepArgs<T> A, long long n_items) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ uint32_t tmem_slot;
    __shared__ int stop;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const size_t stage_bytes = (size_t)A.cap_slots * (16 + kSlabStride * sizeof(T));
    // stage q: barrier at smem + 8q, records then stiffness rows at smem + 16 + q * stage_bytes
    const uint32_t bar0 = smem_u32(smem);
    int4* const srec0 = reinterpret_cast<int4*>(smem + 16);
    T* const sslab0 = reinterpret_cast<T*>(smem + 16 + (size_t)A.cap_slots * 16);
    const uint32_t tcols = blockDim.x > 128 ? 64u : 32u;
    if (warp == 0) {
        tmem_alloc(&tmem_slot, tcols);
        tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
        stop = 0;
    }
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    // this lane's TMEM row: the warp's lane quarter and, above 4 warps, the second 32 columns
    const uint32_t tm =
        tmem_slot + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(warp >> 2) * 32u;
    norms_zero<V>(tm);
    long long w = blockIdx.x;
    if (threadIdx.x == 0 && w < n_items) fanp_issue<T>(A, w, bar0, srec0, sslab0);
    const size_t S = (size_t)A.S;
    const T p = step_pressure<T>(A);
    int stop_it = 0;  // the item at which a wait gave up
    for (int it = 0; w < n_items; w += gridDim.x, ++it) {
        const int sg = it & 1;
        const long long wn = w + gridDim.x;
        if (threadIdx.x == 0 && wn < n_items)
            fanp_issue<T>(A, wn, bar0 + 8 * (sg ^ 1), stage_rec(srec0, stage_bytes, sg ^ 1), stage_slab(sslab0, stage_bytes, sg ^ 1));
        const long long nb = w / A.nch;
        const int chunk = (int)(w - nb * A.nch);
        const long long a0 = nb * A.npb;
        const long long a1 = (a0 + A.npb < A.n_nodes) ? a0 + A.npb : A.n_nodes;
        const long long a = a0 + warp;
        const bool active = warp < A.npb && a < a1;
        const size_t col = ((size_t)chunk * 32 + lane) * V;
        const size_t row = (size_t)a * 3 * S + col;
        const bool clamped = a < A.n_clamped;
        Vec<T, V> ua[3];
        T f[3];
        if (active && !clamped) {
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                ua[d] = ldg<T, V>(A.u + row + d * S);
                prefetch_l2(A.up + row + d * S);
            }
            prefetch_l2(A.invm + (size_t)a * S + col);
            node_load<T>(A, a, p, f);
        }
        // No L2 prefetch ahead here: the prefetching warp's dependent slot-record loads
        // hold its whole block at the item barrier (measured 2.466 -> 3.579 ms/step on the
        // 256x1024 tube with it; node rows alone 3.06 ms).
        // warp-uniform, so that the tensor-memory accesses of the epilogue stay converged;
        // a wait that gives up stops the whole block after this item
        const bool ready = __all_sync(
            0xffffffffu, mbar_wait_bounded(bar0 + 8 * sg, (uint32_t)((it >> 1) & 1), kMaxPolls));
        if (!ready && lane == 0) {
            if (A.status) atomicOr(A.status, 1);
            stop = 1;
        }
        if (ready && active) {
            if (clamped) {
                clamp_store_tm<T, V>(A, S, row, tm, a, col);
            } else {
                const int kb = __ldg(A.node_ptr + a0);
                const int k0 = __ldg(A.node_ptr + a) - kb, k1 = __ldg(A.node_ptr + a + 1) - kb;
                Vec<T, V> acc[3];
                ku_row_fan<T, V, DIFF>(stage_rec(srec0, stage_bytes, sg),
                                       stage_slab(sslab0, stage_bytes, sg), k0, k1, A.u, A.coef,
                                       S, col, ua, acc);
                step_epilogue_tm<T, V>(A, a, S, col, row, ua, acc, f, tm);
            }
        }
        __syncthreads();
        if (*(volatile int*)&stop) {
            stop_it = it;
            break;
        }
    }
    if (*(volatile int*)&stop && threadIdx.x == 0) {
        // the copies still in flight into this block's stages: the timed-out one and the
        // one issued for the next item
        const int sg = stop_it & 1;
        mbar_wait_bounded(bar0 + 8 * sg, (uint32_t)((stop_it >> 1) & 1), kMaxPolls);
        if (w + gridDim.x < n_items)
            mbar_wait_bounded(bar0 + 8 * (sg ^ 1), (uint32_t)(((stop_it + 1) >> 1) & 1),
                              kMaxPolls);
    }
    // this block's sums over its nodes, warps added in order, in the (idle) stage memory
    double* const scr = reinterpret_cast<double*>(smem + 16);
    for (int wv = 0; wv < A.npb; ++wv) {
        if (warp == wv) norms_fold<V>(tm, scr + lane, wv == 0);
        __syncthreads();
    }
    const int chunk = (int)(blockIdx.x % A.nch);
    const long long prow = blockIdx.x / A.nch;
    for (int t = threadIdx.x; t < 4 * V * 32; t += blockDim.x) {
        const int q = t / (32 * V), c = t - q * 32 * V;  // c: sample of the chunk
        const int ln = c / V, i = c - ln * V;
        A.norm_part[((size_t)prow * S + (size_t)chunk * 32 * V + c) * 4 + q] =
            scr[(q * V + i) * 32 + ln];
    }
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    if (warp == 0) tmem_dealloc(tmem_slot, tcols);
}

// ------------------------------------------------------------ burst-gather step
// As k_step_fan (TMA-staged slot rows, a warp per node and sample chunk), but every
// neighbour row of the node and every element coefficient row is requested at once,
// before any product: the node's whole gather (deg + 1 row sets and deg coefficient
// rows, deg <= MAXD) is in flight together, which raises the bytes in flight per SM
// over the fan kernel's one-element lookahead.  Neighbour row j+1 is the second
// neighbour of slot j and the first of slot j+1 (fan order); a fan break past slot 0
// loads its first neighbour when the slot is multiplied.
template <typename T, int V, bool DIFF, int MAXD, int MINB>
__global__ void __launch_bounds__(256, MINB) k_step_burst(StepArgs<T> A) {
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
    const bool probe = A.probe_polls > 0;
    if (threadIdx.x == 0) mbar_init(bar, probe ? 2 : 1);
    __syncthreads();
    if (threadIdx.x == 0 && !probe) {
        const uint32_t b_rec = (uint32_t)nsl * 16u;
        const uint32_t b_slab = (uint32_t)nsl * (uint32_t)(kSlabStride * sizeof(T));
        mbar_arrive_expect_tx(bar, b_rec + b_slab);
        if (nsl > 0) {
            bulk_g2s(smem_u32(srec), A.rec + kb, b_rec, bar);
            bulk_g2s(smem_u32(sslab), A.slab + (size_t)kb * kSlabStride, b_slab, bar);
        }
    }
    const long long a = a0 + warp;
    const bool active = warp < A.npb && a < a1;
    const size_t S = (size_t)A.S;
    const size_t col = ((size_t)chunk * 32 + lane) * V;
    const size_t row = (size_t)a * 3 * S + col;
    const bool clamped = a < A.n_clamped;
    Vec<T, V> ua[3];
    T f[3];
    if (active && !clamped) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            ua[d] = ldg<T, V>(A.u + row + d * S);
            prefetch_l2(A.up + row + d * S);
        }
        prefetch_l2(A.invm + (size_t)a * S + col);
        node_load<T>(A, a, step_pressure<T>(A), f);
    }
    if (!mbar_wait_bounded(bar, 0, kMaxPolls)) {
        if (lane == 0 && A.status) atomicOr(A.status, 1);
        return;
    }
    if (!active) return;
    if (clamped) {
        clamp_store<T, V>(A, S, row);
        return;
    }
    const int k0 = __ldg(A.node_ptr + a) - kb;
    const int deg = __ldg(A.node_ptr + a + 1) - kb - k0;
    Vec<T, V> R[MAXD + 1][3];
    Vec<T, V> C[MAXD];
    if (deg > 0) load_rows<T, V>(R[0], A.u, srec[k0].y, S, col);
#pragma unroll
    for (int j = 0; j < MAXD; ++j) {
        if (j < deg) {
            const int4 r = srec[k0 + j];
            load_rows<T, V>(R[j + 1], A.u, r.z, S, col);
            C[j] = ldg<T, V>(A.coef + (size_t)r.x * S + col);
        }
    }
    Vec<T, V> acc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) acc[d] = vzero<T, V>();
    if (deg > 0) to_diff<T, V, DIFF>(R[0], ua);
#pragma unroll
    for (int j = 0; j < MAXD; ++j) {
        if (j < deg) {
            to_diff<T, V, DIFF>(R[j + 1], ua);
            const int4 r = srec[k0 + j];
            if (j > 0 && !(r.w & 1)) {  // fan break: a first neighbour of its own
                Vec<T, V> b1[3];
                load_rows<T, V>(b1, A.u, r.y, S, col);
                to_diff<T, V, DIFF>(b1, ua);
                slot_fma<T, V, DIFF>(sslab + (size_t)kSlabStride * (k0 + j), C[j], b1, R[j + 1],
                                     ua, acc);
            } else {
                slot_fma<T, V, DIFF>(sslab + (size_t)kSlabStride * (k0 + j), C[j], R[j], R[j + 1],
                                     ua, acc);
            }
        }
    }
    step_epilogue<T, V>(A, a, S, col, row, ua, acc, f);
}

// ------------------------------------------------------------ pipelined persistent step
// Persistent kernel: every warp owns a private STAGES-deep ring of shared-memory
// stages and walks its own sequence of work items (node, 32*VEC-sample chunk;
// chunk fastest; item g = warp id + i * total warps).  For the item STAGES-1
// ahead, each lane issues one TMA bulk copy of one row (its node's u, u_prev and
// inverse-mass rows, every element's second-neighbour rows and coefficient row,
// the slot records and the stiffness rows) into the stage, all completing on the
// stage's mbarrier; meanwhile the warp multiplies the current item entirely out
// of shared memory.  Slot records of the item after that are already in lane
// registers, fetched one iteration earlier.  Warps never wait for each other.
//
// Stage layout: [0, RB*rows) rows of 32*VEC samples, then records, then stiffness
// rows.  Rows: 0-2 u_a, 3-5 u_prev, 6 inverse mass, 7-9 first neighbour of slot 0
// (open fans only), then 4 per slot: second neighbour (3 dofs) and coefficient.
constexpr int kPipeFixedRows = 10;

template <typename T>
struct PipeArgs {
    StepArgs<T> s;
    long long n_items;
    int stage_bytes;
    int rec_off;   // byte offset of the records inside a stage
    int slab_off;  // byte offset of the stiffness rows inside a stage
    int hdr_off;   // byte offset of the header (degree, unit load) inside a stage
    int max_deg;
};

__device__ __forceinline__ void fence_async_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ int4 shfl4(int4 v, int src) {
    return make_int4(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src),
                     __shfl_sync(0xffffffffu, v.z, src), __shfl_sync(0xffffffffu, v.w, src));
}

template <typename T, int V, bool DIFF, int STAGES>
__global__ void __launch_bounds__(256, 1) k_step_pipe(PipeArgs<T> P) {
    extern __shared__ __align__(16) unsigned char smem[];
    const StepArgs<T>& A = P.s;
    constexpr int LB = V * (int)sizeof(T);  // one lane's slice of a row
    constexpr int RB = 32 * LB;             // one row of 32*VEC samples
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int nwarps = blockDim.x >> 5;
    unsigned char* wbase = smem + (size_t)warp * (STAGES * (size_t)P.stage_bytes + 64);
    uint64_t* bars = reinterpret_cast<uint64_t*>(wbase + STAGES * (size_t)P.stage_bytes);
    if (lane < STAGES) mbar_init(smem_u32(bars + lane), 1);
    __syncwarp();
    const long long gw = (long long)blockIdx.x * nwarps + warp;
    const long long GW = (long long)gridDim.x * nwarps;
    const size_t S = (size_t)A.S;
    const int nch = A.nch;

    // Issue the stage of item g with its records in lane registers (lane k = slot k).
    auto issue = [&](int st, long long g, int4 rq, int k0, int deg) {
        unsigned char* sb = wbase + (size_t)st * P.stage_bytes;
        const uint32_t bar = smem_u32(bars + st);
        const long long a = g / nch;
        const int chunk = (int)(g - a * nch);
        const size_t col = (size_t)chunk * 32 * V;
        const bool clamped = a < A.n_clamped;
        const int4 rlast = shfl4(rq, deg > 0 ? deg - 1 : 0);
        const int4 rfirst = shfl4(rq, 0);
        const bool open = deg > 0 && rlast.z != rfirst.y;
        // records and stiffness rows: two TMA bulk copies on the stage's mbarrier
        const uint32_t b_rec = clamped ? 0u : (uint32_t)deg * 16u;
        const uint32_t b_slab =
            clamped ? 0u : (uint32_t)deg * (uint32_t)(kSlabStride * sizeof(T));
        if (lane == 0) {
            mbar_arrive_expect_tx(bar, b_rec + b_slab);
            if (b_rec) {
                bulk_g2s(smem_u32(sb + P.rec_off), A.rec + k0, b_rec, bar);
                bulk_g2s(smem_u32(sb + P.slab_off), A.slab + (size_t)k0 * kSlabStride, b_slab,
                         bar);
            }
        }
        if (clamped) return;
        // header: degree (plain store) and the node's unit load (cp.async)
        if (lane == 0) *reinterpret_cast<int*>(sb + P.hdr_off) = deg;
        if (lane * 16 < 4 * (int)sizeof(T))
            cp_async<16>(smem_u32(sb + P.hdr_off + 16) + lane * 16,
                         reinterpret_cast<const unsigned char*>(A.fhat + 4 * a) + lane * 16);
        // rows: every lane copies its own VEC-sample slice of each row with cp.async
        const uint32_t ls = smem_u32(sb) + lane * LB;
        const size_t cl = col + (size_t)lane * V;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            cp_async<LB>(ls + d * RB, A.u + ((size_t)a * 3 + d) * S + cl);
            cp_async<LB>(ls + (3 + d) * RB, A.up + ((size_t)a * 3 + d) * S + cl);
        }
        cp_async<LB>(ls + 6 * RB, A.invm + (size_t)a * S + cl);
        if (open) {
#pragma unroll
            for (int d = 0; d < 3; ++d)
                cp_async<LB>(ls + (7 + d) * RB, A.u + ((size_t)rfirst.y * 3 + d) * S + cl);
        }
        for (int k = 0; k < deg; ++k) {
            const int4 rs = shfl4(rq, k);
            const uint32_t d0 = ls + (kPipeFixedRows + 4 * k) * RB;
            const T* p2 = A.u + (size_t)rs.z * 3 * S + cl;
#pragma unroll
            for (int d = 0; d < 3; ++d) cp_async<LB>(d0 + d * RB, p2 + d * S);
            cp_async<LB>(d0 + 3 * RB, A.coef + (size_t)rs.x * S + cl);
        }
    };
    // Records and slot range of item g, lane k holding slot k (deg <= 32).
    auto fetch = [&](long long g, int4& rq, int& k0, int& deg) {
        rq = make_int4(0, 0, 0, 0);
        k0 = 0;
        deg = 0;
        if (g >= P.n_items) return;
        const long long a = g / nch;
        k0 = __ldg(A.node_ptr + a);
        deg = __ldg(A.node_ptr + a + 1) - k0;
        if (lane < deg) rq = __ldg(A.rec + k0 + lane);
    };

    const T p = step_pressure<T>(A);
    uint32_t parity = 0;  // bit st: parity of the next completion of stage st
    int4 rq;
    int k0q, degq;
    // prologue: fill STAGES-1 stages; one cp.async group per stage, empty ones included,
    // so that "STAGES-1 groups still pending" always means the oldest one is complete
    long long gi = gw;
    fetch(gi, rq, k0q, degq);
    for (int s = 0; s < STAGES - 1; ++s) {
        const long long g = gw + s * GW;
        if (g < P.n_items) issue(s, g, rq, k0q, degq);
        cp_async_commit();
        fetch(g + GW, rq, k0q, degq);
    }
    int st = 0;
    for (long long g = gw; g < P.n_items; g += GW) {
        // issue the item STAGES-1 ahead into the stage freed last iteration
        const long long gn = g + (long long)(STAGES - 1) * GW;
        const int stn = (st + STAGES - 1) % STAGES;
        if (gn < P.n_items) {
            fence_async_shared();
            issue(stn, gn, rq, k0q, degq);
        }
        cp_async_commit();
        fetch(gn + GW, rq, k0q, degq);
        // wait for the current stage: this lane's rows, then the bulk-copied rows; the
        // header's unit load was copied by lanes 0-1, so the warp syncs before reading it
        cp_async_wait_group<STAGES - 1>();
        __syncwarp();
        const uint32_t bar = smem_u32(bars + st);
        if (!mbar_wait_bounded(bar, (parity >> st) & 1u, kMaxPolls)) {
            if (lane == 0 && A.status) atomicOr(A.status, 1);
            cp_async_wait_all();
            return;
        }
        parity ^= 1u << st;
        const unsigned char* sb = wbase + (size_t)st * P.stage_bytes;
        const long long a = g / nch;
        const int chunk = (int)(g - a * nch);
        const size_t col = ((size_t)chunk * 32 + lane) * V;
        const size_t row = (size_t)a * 3 * S + col;
        if (a < A.n_clamped) {
            clamp_store<T, V>(A, S, row);
        } else {
            const unsigned char* ln = sb + lane * V * sizeof(T);
            const int4* srec = reinterpret_cast<const int4*>(sb + P.rec_off);
            const T* sslab = reinterpret_cast<const T*>(sb + P.slab_off);
            const int deg = *reinterpret_cast<const int*>(sb + P.hdr_off);
            const T* fhs = reinterpret_cast<const T*>(sb + P.hdr_off + 16);
            Vec<T, V> ua[3], acc[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                ua[d] = lds<T, V>(ln + d * RB);
                acc[d] = vzero<T, V>();
            }
            if (deg > 0) {
                const bool open = srec[deg - 1].z != srec[0].y;
                Vec<T, V> d1[3];
                const unsigned char* x1p = open ? ln + 7 * RB : ln + (kPipeFixedRows + 4 * (deg - 1)) * RB;
#pragma unroll
                for (int d = 0; d < 3; ++d) d1[d] = lds<T, V>(x1p + d * RB);
                to_diff<T, V, DIFF>(d1, ua);
                for (int k = 0; k < deg; ++k) {
                    const unsigned char* xp = ln + (kPipeFixedRows + 4 * k) * RB;
                    if (k > 0 && !(srec[k].w & 1)) {  // fan break: first neighbour from global
                        load_rows<T, V>(d1, A.u, srec[k].y, S, col);
                        to_diff<T, V, DIFF>(d1, ua);
                    }
                    Vec<T, V> d2[3];
#pragma unroll
                    for (int d = 0; d < 3; ++d) d2[d] = lds<T, V>(xp + d * RB);
                    to_diff<T, V, DIFF>(d2, ua);
                    const Vec<T, V> c = lds<T, V>(xp + 3 * RB);
                    slot_fma<T, V, DIFF>(sslab + (size_t)kSlabStride * k, c, d1, d2, ua, acc);
#pragma unroll
                    for (int d = 0; d < 3; ++d) d1[d] = d2[d];
                }
            }
            // epilogue out of the stage
            const Vec<T, V> im = lds<T, V>(ln + 6 * RB);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const Vec<T, V> up = lds<T, V>(ln + (3 + d) * RB);
                T load = p * fhs[d];
                if (A.trac) load += __ldg(A.trac + 4 * a + d);
                Vec<T, V> o;
#pragma unroll
                for (int i = 0; i < V; ++i) {
                    const T dv = ua[d].v[i] - up.v[i];
                    const T w = A.w0 * im.v[i];
                    const T v = fma(w, load - acc[d].v[i], fma(-row_eta(A, im.v[i]), dv, dv));
                    o.v[i] = (im.v[i] != T(0)) ? ua[d].v[i] + v : T(0);
                }
                stcs<T, V>(A.un + row + d * S, o);
            }
        }
        __syncwarp();  // every lane is done reading this stage before it is refilled
        st = (st + 1) % STAGES;
    }
    // drain: no copies are left in flight (every issued stage was waited on above)
}

// ------------------------------------------------------------ cp.async gather step
// Same block shape and TMA-staged slot rows as k_step_staged, but each warp then
// issues the whole gather of its node at once: every lane copies its V-sample
// slice of each needed row (first fan neighbour, each element's second neighbour
// and coefficient, the node's u_prev rows and inverse mass) global -> shared with
// cp.async, waits once, and multiplies entirely out of shared memory.  Data in
// flight costs no registers, so all of a node's loads overlap.  Each lane reads
// back only the bytes it copied itself, so no warp barrier is needed.

// rows of the per-warp buffer: 3 (first x1) + 4 per slot (x2 dofs, coef) + 4 (u_prev, invm)
__host__ __device__ constexpr int gather_rows(int max_degree) { return 7 + 4 * max_degree; }

template <typename T, int V, bool DIFF, int MINB>
__global__ void __launch_bounds__(256, MINB) k_step_gather(StepArgs<T> A) {
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr int LB = V * (int)sizeof(T);  // bytes of one lane's slice of a row
    constexpr int RB = 32 * LB;             // bytes of one warp row
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const long long a0 = (long long)blockIdx.x * A.npb;
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
    unsigned char* wbuf = smem + 16 + (size_t)A.cap_slots * (16 + kSlabStride * sizeof(T)) +
                          (size_t)warp * A.gather_rows * RB + lane * LB;
    const uint32_t wsm = smem_u32(wbuf);
    if (threadIdx.x == 0) mbar_init(bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t b_rec = (uint32_t)nsl * 16u;
        const uint32_t b_slab = (uint32_t)nsl * (uint32_t)(kSlabStride * sizeof(T));
        mbar_arrive_expect_tx(bar, b_rec + b_slab);
        if (nsl > 0) {
            bulk_g2s(smem_u32(srec), A.rec + kb, b_rec, bar);
            bulk_g2s(smem_u32(sslab), A.slab + (size_t)kb * kSlabStride, b_slab, bar);
        }
    }
    const long long a = a0 + warp;
    const bool active = warp < A.npb && a < a1;
    const size_t S = (size_t)A.S;
    const size_t col = ((size_t)blockIdx.y * 32 + lane) * V;
    const size_t row = (size_t)a * 3 * S + col;
    const bool clamped = a < A.n_clamped;
    Vec<T, V> ua[3];
    int k0 = 0, k1 = 0;
    if (active && !clamped) {
#pragma unroll
        for (int d = 0; d < 3; ++d) ua[d] = ldg<T, V>(A.u + row + d * S);
        k0 = __ldg(A.node_ptr + a) - kb;
        k1 = __ldg(A.node_ptr + a + 1) - kb;
        // epilogue rows go first: they do not depend on the staged slot records
        const int eb = 3 + 4 * (k1 - k0);
#pragma unroll
        for (int d = 0; d < 3; ++d) cp_async<LB>(wsm + (eb + d) * RB, A.up + row + d * S);
        cp_async<LB>(wsm + (eb + 3) * RB, A.invm + (size_t)a * S + col);
    }
    if (!mbar_wait_bounded(bar, 0, kMaxPolls)) {
        if (lane == 0 && A.status) atomicOr(A.status, 1);
        cp_async_wait_all();
        return;
    }
    if (!active) return;
    if (clamped) {
        clamp_store<T, V>(A, S, row);
        return;
    }
    // issue the whole gather
    if (k1 > k0) {
        const int4 r0 = srec[k0];
        const T* p1 = A.u + (size_t)r0.y * 3 * S + col;
#pragma unroll
        for (int d = 0; d < 3; ++d) cp_async<LB>(wsm + d * RB, p1 + d * S);
    }
    for (int k = k0; k < k1; ++k) {
        const int4 r = srec[k];
        const uint32_t base = wsm + (3 + 4 * (k - k0)) * RB;
        const T* p2 = A.u + (size_t)r.z * 3 * S + col;
#pragma unroll
        for (int d = 0; d < 3; ++d) cp_async<LB>(base + d * RB, p2 + d * S);
        cp_async<LB>(base + 3 * RB, A.coef + (size_t)r.x * S + col);
    }
    cp_async_wait_all();

    Vec<T, V> acc[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) acc[d] = vzero<T, V>();
    for (int k = k0; k < k1; ++k) {
        const int4 r = srec[k];
        const unsigned char* x2p = wbuf + (3 + 4 * (k - k0)) * RB;
        Vec<T, V> d1[3], d2[3];
        if (k == k0 || (r.w & 1)) {
            const unsigned char* x1p = (k == k0) ? wbuf : x2p - 4 * RB;
#pragma unroll
            for (int d = 0; d < 3; ++d) d1[d] = lds<T, V>(x1p + d * RB);
        } else {  // fan break inside the row: fetch the first neighbour directly
            const T* p1 = A.u + (size_t)r.y * 3 * S + col;
#pragma unroll
            for (int d = 0; d < 3; ++d) d1[d] = ldg<T, V>(p1 + d * S);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            d2[d] = lds<T, V>(x2p + d * RB);
            if constexpr (DIFF) {
                d1[d] = vsub(d1[d], ua[d]);
                d2[d] = vsub(d2[d], ua[d]);
            }
        }
        const Vec<T, V> c = lds<T, V>(x2p + 3 * RB);
        const T* K = sslab + (size_t)kSlabStride * k;
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
            Vec<T, V> t = vzero<T, V>();
            if constexpr (!DIFF) {
#pragma unroll
                for (int jj = 0; jj < 3; ++jj) axpy(t, kk[3 * i + jj], ua[jj]);
            }
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) axpy(t, kk[9 + 3 * i + jj], d1[jj]);
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) axpy(t, kk[18 + 3 * i + jj], d2[jj]);
            vfma(acc[i], c, t);
        }
    }
    // epilogue out of shared memory
    const int eb = 3 + 4 * (k1 - k0);
    const double pd = A.p_sched ? A.p_sched[(A.clock ? A.clock[0] : 0LL) + A.j] : A.pressure;
    const T p = (T)pd;
    const Vec<T, V> im = lds<T, V>(wbuf + (eb + 3) * RB);
    const T* fh = A.fhat + 4 * a;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const Vec<T, V> up = lds<T, V>(wbuf + (eb + d) * RB);
        T load = p * __ldg(fh + d);
        if (A.trac) load += __ldg(A.trac + 4 * a + d);
        Vec<T, V> o;
#pragma unroll
        for (int i = 0; i < V; ++i) {
            const T dv = ua[d].v[i] - up.v[i];
            const T w = A.w0 * im.v[i];
            const T v = fma(w, load - acc[d].v[i], fma(-row_eta(A, im.v[i]), dv, dv));
            o.v[i] = (im.v[i] != T(0)) ? ua[d].v[i] + v : T(0);
        }
        stcs<T, V>(A.un + row + d * S, o);
    }
}

// ------------------------------------------------------------------ norms
constexpr int kNormThreads = 128;
inline long long norm_chunks(long long n_nodes) {
    long long c = (n_nodes + 63) / 64;
    return std::max(1LL, std::min(1024LL, c));
}

// VEL: `up` holds the increment v = u_n - u_{n-1} (velocity-state form), else u_{n-1}.
template <typename T, bool VEL>
__global__ void k_norms_partial(long long n_nodes, int S, long long npc, const T* __restrict__ u,
                                const T* __restrict__ up, const T* __restrict__ invm,
                                double* __restrict__ work) {
    const long long chunk = blockIdx.x;
    const int s = blockIdx.y * kNormThreads + threadIdx.x;
    if (s >= S) return;
    const long long a0 = chunk * npc, a1 = (a0 + npc < n_nodes) ? a0 + npc : n_nodes;
    double su = 0.0, sv = 0.0, sm = 0.0;
    long long nf = 0;
    for (long long a = a0; a < a1; ++a) {
        // the node terms in the state's type, in the fused step's order (norms_add)
        const T im = invm[(size_t)a * S + s];
        T su_a = T(0), dv2 = T(0);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const size_t o = ((size_t)a * 3 + d) * S + s;
            const T x = u[o], y = up[o];
            if (!isfinite(x)) ++nf;
            su_a = fma(x, x, su_a);
            const T dv = VEL ? y : x - y;
            dv2 = fma(dv, dv, dv2);
        }
        su += (double)su_a;
        sv += (double)dv2;
        sm += (double)(norm_mass(im) * dv2);
    }
    double* w = work + ((size_t)chunk * S + s) * 4;
    w[0] = su;
    w[1] = sv;
    w[2] = sm;
    w[3] = (double)nf;
}

// Sums of the partial rows per (sample, quantity): a block owns kFinalPairs consecutive
// (sample, quantity) pairs (coalesced across its lanes) and kFinalGroups row groups;
// group g adds rows g, g + kFinalGroups, ... into four accumulators, and the groups'
// sums are added in group order, so the result depends only on the row count.
constexpr int kFinalPairs = 32, kFinalGroups = 8;
__global__ void __launch_bounds__(kFinalPairs * kFinalGroups)
    k_norms_final(long long n_chunks, int S, const double* __restrict__ work,
                  double* __restrict__ out, double* __restrict__ total_nonfinite) {
    __shared__ double part[kFinalGroups][kFinalPairs];
    const int lp = threadIdx.x % kFinalPairs, g = threadIdx.x / kFinalPairs;
    const long long t = (long long)blockIdx.x * kFinalPairs + lp;  // pair s * 4 + q
    const long long P = 4LL * S;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    if (t < P) {
        long long c = g;
        const size_t stride = (size_t)kFinalGroups * P;
        const double* w = work + (size_t)c * P + t;
        for (; c + 3 * kFinalGroups < n_chunks; c += 4 * kFinalGroups, w += 4 * stride) {
            a0 += w[0];
            a1 += w[stride];
            a2 += w[2 * stride];
            a3 += w[3 * stride];
        }
        for (; c < n_chunks; c += kFinalGroups, w += stride) a0 += w[0];
    }
    part[g][lp] = (a0 + a1) + (a2 + a3);
    __syncthreads();
    if (g != 0 || t >= P) return;
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < kFinalGroups; ++k) acc += part[k][lp];
    out[t] = acc;
    if ((t & 3) == 3 && acc != 0.0) atomicAdd(total_nonfinite, acc);
}
inline unsigned final_grid(long long S) { return grid_1d(4 * S, kFinalPairs); }

// ------------------------------------------------------------------ launchers
template <typename T>
int pick_vec(const void* const* ptrs, int n, int S) {
    const int maxv = (int)(16 / sizeof(T));
    for (int v = maxv; v > 1; v /= 2) {
        if (S % v) continue;
        bool ok = true;
        for (int i = 0; i < n; ++i)
            if (ptrs[i] && (reinterpret_cast<uintptr_t>(ptrs[i]) % (v * sizeof(T)))) ok = false;
        if (ok) return v;
    }
    return 1;
}

int check_mesh(const cvfes_solid_mesh* m, const char* who) {
    if (!m || m->n_nodes <= 0 || m->n_samples <= 0 || !m->node_ptr || !m->slot_rec ||
        !m->slot_k || !m->fhat)
        return fail(CVFES_ERR_ARG, "%s: incomplete mesh descriptor", who);
    if (m->n_samples > INT32_MAX || m->n_clamped < 0 || m->n_clamped > m->n_nodes)
        return fail(CVFES_ERR_ARG, "%s: bad sample count or clamped-row count", who);
    if (reinterpret_cast<uintptr_t>(m->slot_k) % 16 || reinterpret_cast<uintptr_t>(m->slot_rec) % 16)
        return fail(CVFES_ERR_ARG, "%s: slot arrays must be 16-byte aligned", who);
    return CVFES_OK;
}

struct StepTuning {
    int vec;
    int npb;
    int staged;
    int minb;  // minimum resident blocks per SM asked of the compiler (register cap)
};
// Defaults from sweeps on the 256x1024 tube with 512 samples (B200), ms/step:
// FP32 (velocity-state form): persistent fan 2.441 (4 nodes per block), 2.445 (2), 2.562
// (3), fan 2.606 (2), 2.598 (4), fan with loads two elements ahead 2.637; FP64: fan 5.750,
// persistent fan 6.088 (2 nodes per block), two ahead 5.981; on another box with the
// final kernels, FP64 persistent fan with 4 nodes per block 5.421 against the fan's 5.821
// (1 sample per thread at 3 blocks' registers: 6.47 to 8.07).  2 blocks per SM worth of
// registers.
static StepTuning g_tune32 = {4, 4, 6, 2};
static StepTuning g_tune64 = {2, 4, 6, 2};
// L2 prefetch of the fan kernels: distance in nodes (-1: the mesh's bandwidth + 128;
// 0: off) and parts (bit 0 node rows, bit 1 element coefficient rows; -1: automatic).
// Sweeps on the 256x1024 tube (bandwidth 257, 512 samples): 256 .. 768 nodes ahead
// are equally good (FP32 -3%, FP64 -3.5% step time with both parts, none with node
// rows alone); 2048 and more overflow what L2 keeps and are slower than none.  On the
// stenosed 512x2048 tube (128 samples) both parts slow the forward step by 4.5% and
// node rows alone speed the reverse step up by 2.4%.
static int g_pf_dist[2] = {-1, -1};
static int g_pf_parts[2] = {-1, -1};
// Polls of the failure-path test of the fan kernel's bounded wait (0: off).
static int g_wait_probe = 0;
Prefetch step_prefetch(int precision, long long bandwidth) {
    const int q = precision == 32 ? 0 : 1;
    Prefetch p{g_pf_dist[q], g_pf_parts[q]};
    if (p.dist < 0) {
        const long long d = bandwidth > 0 ? bandwidth + 128 : 0;
        p.dist = d < (1 << 20) ? (int)d : (1 << 20);
    }
    if (p.parts == 0) p.dist = 0;
    return p;
}
template <typename T>
StepTuning& tuning_of() {
    return sizeof(T) == 4 ? g_tune32 : g_tune64;
}
constexpr size_t kMaxStageBytes = 160 * 1024;

template <typename K, typename A_>
int launch_staged(K kernel, dim3 grid, int threads, size_t smem, cudaStream_t st, const A_& A) {
    if (smem > 48 * 1024) {
        cudaError_t e =
            cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess)
            return fail(CVFES_ERR_CUDA, "k_step_staged smem attribute: %s", cudaGetErrorString(e));
    }
    kernel<<<grid, threads, smem, st>>>(A);
    CVFES_LAUNCH_CHECK("k_step_staged");
    return CVFES_OK;
}

inline int sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 148;
    return n > 0 ? n : 148;
}

// Persistent pipelined step: `warps` warps per block, `stages` stages per warp.
template <typename T, int V, bool DIFF, int STAGES>
int launch_pipe_s(const StepArgs<T>& A, long long max_deg, int warps, cudaStream_t st) {
    constexpr int RB = 32 * V * (int)sizeof(T);
    PipeArgs<T> P;
    P.s = A;
    P.n_items = A.n_nodes * A.nch;
    P.max_deg = (int)max_deg;
    P.rec_off = (kPipeFixedRows + 4 * (int)max_deg) * RB;
    P.slab_off = P.rec_off + (int)max_deg * 16;
    P.hdr_off = ((P.slab_off + (int)max_deg * kSlabStride * (int)sizeof(T)) + 15) / 16 * 16;
    P.stage_bytes = (P.hdr_off + 64 + 127) / 128 * 128;
    const size_t smem = (size_t)warps * ((size_t)STAGES * P.stage_bytes + 64);
    if (smem > 227 * 1024) return CVFES_ERR_UNSUPPORTED;
    auto kernel = k_step_pipe<T, V, DIFF, STAGES>;
    if (smem > 48 * 1024) {
        cudaError_t e =
            cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess)
            return fail(CVFES_ERR_CUDA, "k_step_pipe smem attribute: %s", cudaGetErrorString(e));
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 32 * warps, smem) !=
            cudaSuccess ||
        per_sm < 1)
        return fail(CVFES_ERR_CUDA, "k_step_pipe does not fit on an SM (%zu B smem)", smem);
    long long blocks = (long long)per_sm * sm_count();
    const long long need = (P.n_items + warps - 1) / warps;
    if (blocks > need) blocks = need;
    kernel<<<(unsigned)blocks, 32 * warps, smem, st>>>(P);
    CVFES_LAUNCH_CHECK("k_step_pipe");
    return CVFES_OK;
}

template <typename T, int V, bool DIFF>
int launch_pipe(const StepArgs<T>& A, long long max_deg, int warps, int stages, cudaStream_t st) {
    switch (stages) {
        case 4: return launch_pipe_s<T, V, DIFF, 4>(A, max_deg, warps, st);
        case 3: return launch_pipe_s<T, V, DIFF, 3>(A, max_deg, warps, st);
        default: return launch_pipe_s<T, V, DIFF, 2>(A, max_deg, warps, st);
    }
}

// Resident blocks per SM of a persistent kernel at this block size and shared memory,
// with the shared-memory attribute set when it needs more than 48 KB; looked up once
// per (kernel, device, block, shared memory) and kept, since every step launches it.
int device_sm_count() { return sm_count(); }

int fanp_blocks_per_sm(const void* kernel, int threads, size_t smem, int* per_sm) {
    struct Entry {
        const void* k;
        int dev, threads;
        size_t smem;
        int per_sm;
    };
    static Entry cache[32];
    static int n_cache = 0;
    static std::mutex mu;
    int dev = 0;
    CVFES_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    for (int i = 0; i < n_cache; ++i)
        if (cache[i].k == kernel && cache[i].dev == dev && cache[i].threads == threads &&
            cache[i].smem == smem) {
            *per_sm = cache[i].per_sm;
            return CVFES_OK;
        }
    if (smem > 48 * 1024) {
        cudaError_t e =
            cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess)
            return fail(CVFES_ERR_CUDA, "k_step_fanp smem attribute: %s", cudaGetErrorString(e));
    }
    // From the kernel's registers and shared memory against the SM's budgets.  Not the
    // occupancy calculator: it reports one block per SM for a kernel that contains a
    // tensor-memory allocation, whose blocks here give up their allocation permit at
    // their start and hold 32 or 64 of the SM's 512 columns only when the norms are fused.
    cudaFuncAttributes fa;
    CVFES_CUDA_TRY(cudaFuncGetAttributes(&fa, kernel));
    int regs_sm = 0, smem_sm = 0, reserved = 0, thr_sm = 0, blk_sm = 0;
    CVFES_CUDA_TRY(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev));
    CVFES_CUDA_TRY(
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    CVFES_CUDA_TRY(
        cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
    CVFES_CUDA_TRY(
        cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev));
    CVFES_CUDA_TRY(cudaDeviceGetAttribute(&blk_sm, cudaDevAttrMaxBlocksPerMultiprocessor, dev));
    const int warps = (threads + 31) / 32;
    // registers: allocated per warp in units of 256, from the four sub-partitions' quarters
    const int per_warp = ((fa.numRegs * 32 + 255) / 256) * 256;
    const int by_regs = per_warp > 0 ? 4 * ((regs_sm / 4) / per_warp) / warps : blk_sm;
    const size_t per_block = fa.sharedSizeBytes + smem + (size_t)reserved;
    const int by_smem = (int)((size_t)smem_sm / per_block);
    const int by_thr = thr_sm / (32 * warps);
    const int n = std::min(std::min(by_regs, by_smem), std::min(by_thr, blk_sm));
    if (n <= 0) return fail(CVFES_ERR_CUDA, "k_step_fanp: no resident block fits");
    if (n_cache < 32) cache[n_cache++] = Entry{kernel, dev, threads, smem, n};
    *per_sm = n;
    return CVFES_OK;
}

// Where the fused norms keep their sums: 0 tensor memory (k_step_fanp_tm), 1 shared memory
// (k_step_fanp).  Both give bitwise the same norms.
static std::atomic<int> g_norms_mode{0};

// The persistent fan kernel on as many blocks as are resident (at most one per work
// item).  With fused norms the grid is rounded down to a multiple of the sample chunks
// and capped at max_rows chunks' worth, and *rows gets the partial rows written.
template <typename K, typename T>
int launch_fanp_k(K kernel, long long n_items, int threads, size_t smem, cudaStream_t st,
                  const StepArgs<T>& A, long long max_rows, long long* rows) {
    int per_sm = 0;
    const int rc = fanp_blocks_per_sm(reinterpret_cast<const void*>(kernel), threads, smem,
                                      &per_sm);
    if (rc) return rc;
    // fused norms in tensor memory: each block holds 32 columns (64 above 4 warps), and
    // a block waits in its allocation until the SM's 512 columns have room
    if (A.norm_part && g_norms_mode.load() == 0) {
        const int cap = threads > 128 ? 8 : 16;
        if (per_sm > cap) per_sm = cap;
    }
    long long blocks = (long long)per_sm * sm_count();
    if (blocks > n_items) blocks = n_items;
    if (A.norm_part) {
        if (blocks > max_rows * A.nch) blocks = max_rows * A.nch;
        blocks -= blocks % A.nch;
        if (blocks < A.nch) blocks = A.nch;
        if (rows) *rows = blocks / A.nch;
    }
    kernel<<<(unsigned)blocks, threads, smem, st>>>(A, n_items);
    CVFES_LAUNCH_CHECK("k_step_fanp");
    return CVFES_OK;
}

template <typename T, int V, bool DIFF>
int launch_fanp(int minb, long long n_items, int threads, size_t smem, cudaStream_t st,
                const StepArgs<T>& A, long long max_rows = 0, long long* rows = nullptr) {
#define CVFES_FANP_K(K, MB) launch_fanp_k(K<T, V, DIFF, MB>, n_items, threads, smem, st, A, max_rows, rows)
#define CVFES_FANP(K)                                   \
    switch (minb) {                                     \
        case 4: return CVFES_FANP_K(K, 4);              \
        case 3: return CVFES_FANP_K(K, 3);              \
        case 2: return CVFES_FANP_K(K, 2);              \
        default: return CVFES_FANP_K(K, 1);             \
    }
    if (A.norm_part && g_norms_mode.load() == 0) {
        // the block's sums are added up in the (idle) stage memory at its end
        const size_t scratch = 16 + (size_t)4 * V * 32 * sizeof(double);
        if (smem < scratch) smem = scratch;
        CVFES_FANP(k_step_fanp_tm)
    }
    if (A.norm_part) smem += (size_t)A.npb * 4 * V * 32 * sizeof(double);
    CVFES_FANP(k_step_fanp)
#undef CVFES_FANP
#undef CVFES_FANP_K
}

template <typename T, int V, bool DIFF, int MAXD>
int launch_burst(int minb, dim3 g1, int threads, size_t smem, cudaStream_t st,
                 const StepArgs<T>& A) {
    switch (minb) {
        case 4: return launch_staged(k_step_burst<T, V, DIFF, MAXD, 4>, g1, threads, smem, st, A);
        case 3: return launch_staged(k_step_burst<T, V, DIFF, MAXD, 3>, g1, threads, smem, st, A);
        case 2: return launch_staged(k_step_burst<T, V, DIFF, MAXD, 2>, g1, threads, smem, st, A);
        default: return launch_staged(k_step_burst<T, V, DIFF, MAXD, 1>, g1, threads, smem, st, A);
    }
}

template <typename T, int V, bool DIFF>
int launch_staged_v(int variant, int minb, dim3 grid, int threads, size_t smem, cudaStream_t st,
                    const StepArgs<T>& A, long long max_degree = 0) {
    if (variant == 6) {
        const long long n_items = (long long)grid.x * grid.y;
        const size_t smem2 = 16 + 2 * (smem - 16);
        return launch_fanp<T, V, DIFF>(minb, n_items, threads, smem2, st, A);
    }
    if (variant == 5 && max_degree > 0 && max_degree <= 8) {
        const dim3 g1((unsigned)((long long)grid.x * grid.y));
        if (max_degree <= 6) return launch_burst<T, V, DIFF, 6>(minb, g1, threads, smem, st, A);
        return launch_burst<T, V, DIFF, 8>(minb, g1, threads, smem, st, A);
    }
    if (variant == 8) {
        const dim3 g1((unsigned)((long long)grid.x * grid.y));
        switch (minb) {
            case 3: return launch_staged(k_step_fan<T, V, DIFF, 3, 2>, g1, threads, smem, st, A);
            case 2: return launch_staged(k_step_fan<T, V, DIFF, 2, 2>, g1, threads, smem, st, A);
            default: return launch_staged(k_step_fan<T, V, DIFF, 1, 2>, g1, threads, smem, st, A);
        }
    }
    if (variant == 3 || variant == 5) {
        const dim3 g1((unsigned)((long long)grid.x * grid.y));
        switch (minb) {
            case 4: return launch_staged(k_step_fan<T, V, DIFF, 4>, g1, threads, smem, st, A);
            case 3: return launch_staged(k_step_fan<T, V, DIFF, 3>, g1, threads, smem, st, A);
            case 2: return launch_staged(k_step_fan<T, V, DIFF, 2>, g1, threads, smem, st, A);
            default: return launch_staged(k_step_fan<T, V, DIFF, 1>, g1, threads, smem, st, A);
        }
    }
    if (variant == 2) {
        switch (minb) {
            case 4: return launch_staged(k_step_gather<T, V, DIFF, 4>, grid, threads, smem, st, A);
            case 3: return launch_staged(k_step_gather<T, V, DIFF, 3>, grid, threads, smem, st, A);
            case 2: return launch_staged(k_step_gather<T, V, DIFF, 2>, grid, threads, smem, st, A);
            default: return launch_staged(k_step_gather<T, V, DIFF, 1>, grid, threads, smem, st, A);
        }
    }
    switch (minb) {
        case 4: return launch_staged(k_step_staged<T, V, DIFF, 4>, grid, threads, smem, st, A);
        case 3: return launch_staged(k_step_staged<T, V, DIFF, 3>, grid, threads, smem, st, A);
        case 2: return launch_staged(k_step_staged<T, V, DIFF, 2>, grid, threads, smem, st, A);
        default: return launch_staged(k_step_staged<T, V, DIFF, 1>, grid, threads, smem, st, A);
    }
}

// norm_work (optional): fuse the per-sample norms of the new state into the step (the
// persistent fan kernel); *norm_rows gets the partial rows written to norm_work, or 0
// when the shape has no fused kernel (the caller then runs the separate norms pass).
template <typename T>
int launch_step(const cvfes_solid_mesh* m, const T* coef, const T* invm, const T* u,
                const T* up, T* un, const double* p_sched, const long long* clock, long long j,
                double pressure, const T* trac, double dt, double damp, cudaStream_t st,
                double* norm_work = nullptr, long long* norm_rows = nullptr,
                long long max_rows = 0) {
    if (norm_rows) *norm_rows = 0;
    int rc = check_mesh(m, "cvfes_solid_step");
    if (rc) return rc;
    if (!coef || !invm || !u || !up || !un)
        return fail(CVFES_ERR_ARG, "cvfes_solid_step: null state pointer");
    if (!(dt > 0.0)) return fail(CVFES_ERR_ARG, "cvfes_solid_step: dt must be positive");
    StepArgs<T> A;
    A.node_ptr = m->node_ptr;
    A.rec = reinterpret_cast<const int4*>(m->slot_rec);
    A.slab = static_cast<const T*>(m->slot_k);
    A.fhat = static_cast<const T*>(m->fhat);
    A.coef = coef;
    A.invm = invm;
    A.u = u;
    A.up = up;
    A.un = un;
    A.trac = trac;
    A.p_sched = p_sched;
    A.clock = clock;
    A.j = j;
    A.pressure = pressure;
    A.n_nodes = m->n_nodes;
    A.S = (int)m->n_samples;
    A.n_clamped = (int)m->n_clamped;
    A.clamp = (T)m->clamp_value;
    const double g = 0.5 * dt * damp;
    if (m->damping_form != 0 && m->damping_form != 1)
        return fail(CVFES_ERR_ARG, "cvfes_solid_step: damping_form must be 0 or 1");
    if (m->damping_form == 1) {  // damping force per dof: eta = dt damp / m, no LHS term
        A.damp_per_dof = 1;
        A.eta = (T)(dt * damp);
        A.w0 = (T)(dt * dt);
    } else {
        A.eta = (T)(dt * damp / (1.0 + g));
        A.w0 = (T)(dt * dt / (1.0 + g));
    }
    A.status = m->status;
    A.cap_slots = 0;
    if (m->state_form != 0 && m->state_form != 1)
        return fail(CVFES_ERR_ARG, "cvfes_solid_step: state_form must be 0 or 1");
    if (m->state_form == 1) {
        if (up == u || up == un)
            return fail(CVFES_ERR_ARG, "cvfes_solid_step: the increment buffer must be its own");
        A.vel = const_cast<T*>(up);
    }
    const void* ptrs[6] = {coef, invm, u, up, un, nullptr};
    StepTuning tune = tuning_of<T>();
    // The velocity-state form is fused into the kernels that share step_epilogue; the
    // cp.async-gather (2), pipelined (4) and TMA-tiled (7) variants run the fan kernel.
    if (A.vel && (tune.staged == 2 || tune.staged == 4 || tune.staged == 7)) {
        tune.staged = 3;
        tune.minb = 2;
    }
    const Prefetch pf = step_prefetch(sizeof(T) == 4 ? 32 : 64, m->bandwidth);
    A.pf_dist = pf.dist;
    A.pf_parts = pf.parts;
    A.probe_polls = g_wait_probe;
    if (A.probe_polls > 0) {  // only the fan kernel has the probe; it needs a status word
        if (!A.status)
            return fail(CVFES_ERR_ARG, "cvfes_solid_step: the wait probe needs a status word");
        tune.staged = 3;
        tune.minb = 2;
    }
    int V = pick_vec<T>(ptrs, 5, A.S);
    while (V > tune.vec) V /= 2;
    constexpr bool DIFF = std::is_same<T, float>::value;
    // The warp-per-node kernels need S/V to be a multiple of 32: narrow the sample
    // vector to make it so (S = 64 with 4 per thread -> 2 per thread), else they fall
    // back to the row-gather kernel at the original width.
    const int V_rows = V;
    if (tune.staged != 0 && (A.S / V) % 32 != 0) {
        int v2 = V;
        while (v2 > 1 && (A.S / v2) % 32 != 0) v2 /= 2;
        if ((A.S / v2) % 32 == 0) V = v2;
    }
    if (tune.staged == 7) {  // TMA-tiled strips; the fan kernel where they do not apply
        const int trc = launch_step_tile<T>(m, A, tune.vec, st);
        if (trc <= 0) return trc;
        tune.staged = 3;
        tune.minb = 2;
    }
    // Pipelined persistent kernel (npb = warps per block, minb = stages per warp).
    if (tune.staged == 4 && m->max_degree > 0 && m->max_degree <= 32 && (A.S / V) % 32 == 0) {
        A.nch = A.S / V / 32;
        A.npb = tune.npb;
        A.tpn = 32;
        A.cap_slots = 0;
        A.gather_rows = 0;
        const int stages = tune.minb < 2 ? 2 : (tune.minb > 4 ? 4 : tune.minb);
        int prc = CVFES_ERR_UNSUPPORTED;
        if (V == 4) {
            if constexpr (sizeof(T) == 4)
                prc = launch_pipe<T, 4, DIFF>(A, m->max_degree, tune.npb, stages, st);
        } else if (V == 2) {
            prc = launch_pipe<T, 2, DIFF>(A, m->max_degree, tune.npb, stages, st);
        } else {
            prc = launch_pipe<T, 1, DIFF>(A, m->max_degree, tune.npb, stages, st);
        }
        if (prc != CVFES_ERR_UNSUPPORTED) return prc;  // else fall through to a smaller kernel
    }
    // TMA-staged kernels: a warp per node needs S/V to be a multiple of 32.
    const long long cap = (long long)tune.npb * m->max_degree;
    A.gather_rows = gather_rows((int)m->max_degree);
    size_t smem = 16 + (size_t)cap * (16 + kSlabStride * sizeof(T));
    if (tune.staged == 2) smem += (size_t)tune.npb * A.gather_rows * 32 * V * sizeof(T);
    if (tune.staged && m->max_degree > 0 && (A.S / V) % 32 == 0 && smem <= kMaxStageBytes) {
        A.npb = tune.npb;
        A.tpn = 32;
        A.cap_slots = (int)cap;
        A.nch = A.S / V / 32;
        A.pf_group = prefetch_group(A.nch);
        A.pf_parts = prefetch_parts(A.pf_parts, A.nch);
        const dim3 grid((unsigned)((m->n_nodes + A.npb - 1) / A.npb), (unsigned)(A.S / V / 32));
        const int threads = 32 * A.npb;
        if (norm_work && max_rows > 0 && !A.probe_polls) {  // fused norms: persistent fan
            A.norm_part = norm_work;
            const long long n_items = (long long)grid.x * grid.y;
            const size_t smem2 = 16 + 2 * (smem - 16);
            const int minb = tune.staged == 6 ? tune.minb : 2;
            if (V == 4) {
                if constexpr (sizeof(T) == 4)
                    return launch_fanp<T, 4, DIFF>(minb, n_items, threads, smem2, st, A, max_rows,
                                                   norm_rows);
            } else if (V == 2) {
                return launch_fanp<T, 2, DIFF>(minb, n_items, threads, smem2, st, A, max_rows,
                                               norm_rows);
            }
            return launch_fanp<T, 1, DIFF>(minb, n_items, threads, smem2, st, A, max_rows,
                                           norm_rows);
        }
        if (V == 4) {
            if constexpr (sizeof(T) == 4)
                rc = launch_staged_v<T, 4, DIFF>(tune.staged, tune.minb, grid, threads, smem, st,
                                                 A, m->max_degree);
        } else if (V == 2) {
            rc = launch_staged_v<T, 2, DIFF>(tune.staged, tune.minb, grid, threads, smem, st, A,
                                             m->max_degree);
        } else {
            rc = launch_staged_v<T, 1, DIFF>(tune.staged, tune.minb, grid, threads, smem, st, A,
                                             m->max_degree);
        }
        return rc;
    }
    if (A.probe_polls > 0)
        return fail(CVFES_ERR_UNSUPPORTED,
                    "cvfes_solid_step: the wait probe needs the fan kernel (S / vec a multiple "
                    "of 32 and the mesh's max_degree)");
    V = V_rows;
    const int block = 256;
    const RowGrid rg = row_grid(m->n_nodes, A.S / V, block);
    A.tpn = rg.tpn;
    A.npb = rg.npb;
    if (V == 4) {
        if constexpr (sizeof(T) == 4) k_step<T, 4, DIFF><<<rg.grid, block, 0, st>>>(A);
    } else if (V == 2) {
        k_step<T, 2, DIFF><<<rg.grid, block, 0, st>>>(A);
    } else {
        k_step<T, 1, DIFF><<<rg.grid, block, 0, st>>>(A);
    }
    CVFES_LAUNCH_CHECK("k_step");
    return CVFES_OK;
}

template <typename T>
int launch_kmul(const cvfes_solid_mesh* m, const T* coef, const T* u, T* res, int accumulate,
                cudaStream_t st) {
    int rc = check_mesh(m, "cvfes_solid_kmul");
    if (rc) return rc;
    if (!coef || !u || !res) return fail(CVFES_ERR_ARG, "cvfes_solid_kmul: null pointer");
    const int S = (int)m->n_samples;
    const void* ptrs[3] = {coef, u, res};
    const int V = pick_vec<T>(ptrs, 3, S);
    const int block = 256;
    const RowGrid rg = row_grid(m->n_nodes, S / V, block);
    const dim3 grid = rg.grid;
    constexpr bool DIFF = std::is_same<T, float>::value;
    const int4* rec = reinterpret_cast<const int4*>(m->slot_rec);
    const T* slab = static_cast<const T*>(m->slot_k);
    if (V == 4) {
        if constexpr (sizeof(T) == 4)
            k_kmul<T, 4, DIFF><<<grid, block, 0, st>>>(m->node_ptr, rec, slab, coef, u, res,
                                                       m->n_nodes, S, accumulate, rg.tpn, rg.npb);
    } else if (V == 2) {
        k_kmul<T, 2, DIFF><<<grid, block, 0, st>>>(m->node_ptr, rec, slab, coef, u, res,
                                                   m->n_nodes, S, accumulate, rg.tpn, rg.npb);
    } else {
        k_kmul<T, 1, DIFF><<<grid, block, 0, st>>>(m->node_ptr, rec, slab, coef, u, res,
                                                   m->n_nodes, S, accumulate, rg.tpn, rg.npb);
    }
    CVFES_LAUNCH_CHECK("k_kmul");
    return CVFES_OK;
}

template <typename T>
int launch_advance(const cvfes_solid_mesh* m, const T* coef, const T* invm, T* b0, T* b1, T* b2,
                   const double* p_sched, long long* clock, long long n_steps, double dt,
                   double damp, int* cur_idx, int* prev_idx, cudaStream_t st) {
    if (n_steps < 0) return fail(CVFES_ERR_ARG, "cvfes_solid_advance: negative step count");
    if (!p_sched) return fail(CVFES_ERR_ARG, "cvfes_solid_advance: needs a pressure schedule");
    T* buf[3] = {b0, b1, b2};
    int cur = 0, prev = 1, nxt = 2;
    const bool vel = m && m->state_form == 1;
    for (long long j = 0; j < n_steps; ++j) {
        int rc = launch_step<T>(m, coef, invm, buf[cur], buf[prev], buf[nxt], p_sched, clock, j,
                                0.0, nullptr, dt, damp, st);
        if (rc) return rc;
        if (vel) {  // the increment stays in place; the displacement buffers swap
            const int t = cur;
            cur = nxt;
            nxt = t;
            continue;
        }
        const int old_prev = prev;
        prev = cur;
        cur = nxt;
        nxt = old_prev;
    }
    if (clock && n_steps > 0) {
        k_clock_add<<<1, 1, 0, st>>>(clock, n_steps);
        CVFES_LAUNCH_CHECK("k_clock_add");
    }
    if (cur_idx) *cur_idx = cur;
    if (prev_idx) *prev_idx = prev;
    return CVFES_OK;
}

template <typename T>
int launch_init(const cvfes_solid_mesh* m, const T* coef, const T* invm, const T* u0,
                const T* du0, T* u_prev, T* work, double p0, double dt, double damp,
                cudaStream_t st) {
    if (!u0 || !du0 || !u_prev || !work || !invm)
        return fail(CVFES_ERR_ARG, "cvfes_solid_init: null pointer");
    int rc = launch_kmul<T>(m, coef, u0, work, 0, st);
    if (rc) return rc;
    const int S = (int)m->n_samples;
    const int block = 256;
    k_init<T><<<grid_1d(m->n_nodes * S, block), block, 0, st>>>(
        static_cast<const T*>(m->fhat), invm, u0, du0, work, u_prev, m->n_nodes, S, (T)p0, (T)dt,
        (T)(m->damping_form == 1 ? 0.0 : damp), m->state_form == 1 ? 1 : 0);
    CVFES_LAUNCH_CHECK("k_init");
    return CVFES_OK;
}

template <typename T>
int launch_norms(long long n_nodes, long long S, const T* u, const T* up, const T* invm,
                 double* work, double* out, int check_finite, cudaStream_t st, bool vel = false) {
    if (n_nodes <= 0 || S <= 0 || S > INT32_MAX || !u || !up || !invm || !work || !out)
        return fail(CVFES_ERR_ARG, "cvfes_solid_norms: bad argument");
    const long long nch = norm_chunks(n_nodes);
    const long long npc = (n_nodes + nch - 1) / nch;
    double* total = work + (size_t)nch * S * 4;
    CVFES_CUDA_TRY(cudaMemsetAsync(total, 0, sizeof(double), st));
    dim3 grid((unsigned)nch, (unsigned)((S + kNormThreads - 1) / kNormThreads));
    if (vel)
        k_norms_partial<T, true><<<grid, kNormThreads, 0, st>>>(n_nodes, (int)S, npc, u, up, invm,
                                                                work);
    else
        k_norms_partial<T, false><<<grid, kNormThreads, 0, st>>>(n_nodes, (int)S, npc, u, up, invm,
                                                                 work);
    CVFES_LAUNCH_CHECK("k_norms_partial");
    k_norms_final<<<final_grid(S), kFinalPairs * kFinalGroups, 0, st>>>(nch, (int)S, work, out, total);
    CVFES_LAUNCH_CHECK("k_norms_final");
    if (check_finite) {
        double h = 0.0;
        CVFES_CUDA_TRY(cudaMemcpyAsync(&h, total, sizeof(double), cudaMemcpyDeviceToHost, st));
        CVFES_CUDA_TRY(cudaStreamSynchronize(st));
        if (h != 0.0)
            return fail(CVFES_ERR_NONFINITE, "watchdog: %.0f non-finite state values", h);
    }
    return CVFES_OK;
}

}  // namespace cvfes

using namespace cvfes;

extern "C" int cvfes_solid_kmul_f64(const cvfes_solid_mesh* mesh, const double* coef,
                                    const double* u, double* res, int32_t accumulate,
                                    void* stream) {
    return launch_kmul<double>(mesh, coef, u, res, accumulate, (cudaStream_t)stream);
}
extern "C" int cvfes_solid_kmul_f32(const cvfes_solid_mesh* mesh, const float* coef,
                                    const float* u, float* res, int32_t accumulate,
                                    void* stream) {
    return launch_kmul<float>(mesh, coef, u, res, accumulate, (cudaStream_t)stream);
}

extern "C" int cvfes_solid_step_f64(const cvfes_solid_mesh* mesh, const double* coef,
                                    const double* invm, const double* u, const double* u_prev,
                                    double* u_next, const double* p_sched, const int64_t* clock,
                                    int64_t j, double pressure, const double* trac, double dt,
                                    double damp, void* stream) {
    return launch_step<double>(mesh, coef, invm, u, u_prev, u_next, p_sched,
                               reinterpret_cast<const long long*>(clock), j, pressure, trac, dt,
                               damp, (cudaStream_t)stream);
}
extern "C" int cvfes_solid_step_f32(const cvfes_solid_mesh* mesh, const float* coef,
                                    const float* invm, const float* u, const float* u_prev,
                                    float* u_next, const double* p_sched, const int64_t* clock,
                                    int64_t j, double pressure, const float* trac, double dt,
                                    double damp, void* stream) {
    return launch_step<float>(mesh, coef, invm, u, u_prev, u_next, p_sched,
                              reinterpret_cast<const long long*>(clock), j, pressure, trac, dt,
                              damp, (cudaStream_t)stream);
}

// One step and the FP64 norms of the new state: fused into the persistent fan kernel
// where the shape allows, else the step followed by the separate norms pass.
template <typename T>
int launch_step_norms(const cvfes_solid_mesh* m, const T* coef, const T* invm, const T* u,
                      const T* up, T* un, const double* p_sched, const long long* clock,
                      long long j, double pressure, const T* trac, double dt, double damp,
                      double* work, double* out, double* out_host, int check_finite,
                      cudaStream_t st) {
    int rc = check_mesh(m, "cvfes_solid_step_norms");
    if (rc) return rc;
    if (!work || !out) return fail(CVFES_ERR_ARG, "cvfes_solid_step_norms: null work or out");
    const long long N = m->n_nodes, S = m->n_samples;
    const long long max_rows = norm_chunks(N);  // the rows cvfes_norms_work_size provides
    long long rows = 0;
    rc = launch_step<T>(m, coef, invm, u, up, un, p_sched, clock, j, pressure, trac, dt, damp, st,
                        work, &rows, max_rows);
    if (rc) return rc;
    const bool vel = m->state_form == 1;
    double* total = nullptr;
    if (rows == 0) {  // no fused kernel for this shape: the separate pass over the new state
        rc = launch_norms<T>(N, S, un, vel ? up : u, invm, work, out, out_host ? 0 : check_finite,
                             st, vel);
        if (rc) return rc;
        total = work + (size_t)norm_chunks(N) * S * 4;
    } else {
        total = work + (size_t)rows * S * 4;
        CVFES_CUDA_TRY(cudaMemsetAsync(total, 0, sizeof(double), st));
        k_norms_final<<<final_grid(S), kFinalPairs * kFinalGroups, 0, st>>>(rows, (int)S, work,
                                                                            out, total);
        CVFES_LAUNCH_CHECK("k_norms_final");
    }
    if (!out_host && !check_finite) return CVFES_OK;
    // one synchronisation for everything the host reads: the norms (out_host), the
    // non-finite total and the status word of the bounded waits (read and cleared)
    double h = 0.0;
    int32_t stat = 0;
    if (out_host)
        CVFES_CUDA_TRY(cudaMemcpyAsync(out_host, out, (size_t)S * 4 * sizeof(double),
                                       cudaMemcpyDeviceToHost, st));
    CVFES_CUDA_TRY(cudaMemcpyAsync(&h, total, sizeof(double), cudaMemcpyDeviceToHost, st));
    if (out_host && m->status) {
        CVFES_CUDA_TRY(cudaMemcpyAsync(&stat, m->status, sizeof(stat), cudaMemcpyDeviceToHost, st));
        CVFES_CUDA_TRY(cudaMemsetAsync(m->status, 0, sizeof(int32_t), st));
    }
    CVFES_CUDA_TRY(cudaStreamSynchronize(st));
    if (stat & 1) return fail(CVFES_ERR_TIMEOUT, "a bounded device wait gave up (status %d)", stat);
    if (stat) return fail(CVFES_ERR_ARG, "device status %d: slot stage overflow", stat);
    if (check_finite && h != 0.0)
        return fail(CVFES_ERR_NONFINITE, "watchdog: %.0f non-finite state values", h);
    return CVFES_OK;
}

extern "C" int cvfes_solid_step_norms_f64(const cvfes_solid_mesh* mesh, const double* coef,
                                          const double* invm, const double* u,
                                          const double* u_prev, double* u_next,
                                          const double* p_sched, const int64_t* clock, int64_t j,
                                          double pressure, const double* trac, double dt,
                                          double damp, double* work, double* out,
                                          double* out_host, int32_t check_finite, void* stream) {
    return launch_step_norms<double>(mesh, coef, invm, u, u_prev, u_next, p_sched,
                                     reinterpret_cast<const long long*>(clock), j, pressure, trac,
                                     dt, damp, work, out, out_host, check_finite,
                                     (cudaStream_t)stream);
}
extern "C" int cvfes_solid_step_norms_f32(const cvfes_solid_mesh* mesh, const float* coef,
                                          const float* invm, const float* u, const float* u_prev,
                                          float* u_next, const double* p_sched,
                                          const int64_t* clock, int64_t j, double pressure,
                                          const float* trac, double dt, double damp, double* work,
                                          double* out, double* out_host,
                                          int32_t check_finite, void* stream) {
    return launch_step_norms<float>(mesh, coef, invm, u, u_prev, u_next, p_sched,
                                    reinterpret_cast<const long long*>(clock), j, pressure, trac,
                                    dt, damp, work, out, out_host, check_finite,
                                    (cudaStream_t)stream);
}

extern "C" int cvfes_solid_advance_f64(const cvfes_solid_mesh* mesh, const double* coef,
                                       const double* invm, double* buf0, double* buf1,
                                       double* buf2, const double* p_sched, int64_t* clock,
                                       int64_t n_steps, double dt, double damp, int32_t* cur_idx,
                                       int32_t* prev_idx, void* stream) {
    return launch_advance<double>(mesh, coef, invm, buf0, buf1, buf2, p_sched,
                                  reinterpret_cast<long long*>(clock), n_steps, dt, damp,
                                  cur_idx, prev_idx, (cudaStream_t)stream);
}
extern "C" int cvfes_solid_advance_f32(const cvfes_solid_mesh* mesh, const float* coef,
                                       const float* invm, float* buf0, float* buf1, float* buf2,
                                       const double* p_sched, int64_t* clock, int64_t n_steps,
                                       double dt, double damp, int32_t* cur_idx,
                                       int32_t* prev_idx, void* stream) {
    return launch_advance<float>(mesh, coef, invm, buf0, buf1, buf2, p_sched,
                                 reinterpret_cast<long long*>(clock), n_steps, dt, damp, cur_idx,
                                 prev_idx, (cudaStream_t)stream);
}

extern "C" int cvfes_solid_init_f64(const cvfes_solid_mesh* mesh, const double* coef,
                                    const double* invm, const double* u0, const double* du0,
                                    double* u_prev, double* work, double p0, double dt,
                                    double damp, void* stream) {
    return launch_init<double>(mesh, coef, invm, u0, du0, u_prev, work, p0, dt, damp,
                               (cudaStream_t)stream);
}
extern "C" int cvfes_solid_init_f32(const cvfes_solid_mesh* mesh, const float* coef,
                                    const float* invm, const float* u0, const float* du0,
                                    float* u_prev, float* work, double p0, double dt, double damp,
                                    void* stream) {
    return launch_init<float>(mesh, coef, invm, u0, du0, u_prev, work, p0, dt, damp,
                              (cudaStream_t)stream);
}

extern "C" int cvfes_bsr_spmv_f64(int64_t n_nodes, int64_t n_samples, const int64_t* indptr,
                                  const int64_t* indices, const double* K, const double* v,
                                  double* res, void* stream) {
    if (n_nodes <= 0 || n_samples <= 0 || n_samples > INT32_MAX || !indptr || !indices || !K ||
        !v || !res)
        return fail(CVFES_ERR_ARG, "cvfes_bsr_spmv_f64: bad argument");
    k_bsr_spmv<<<grid_1d(n_nodes * n_samples, 256), 256, 0, (cudaStream_t)stream>>>(
        n_nodes, (int)n_samples, reinterpret_cast<const long long*>(indptr),
        reinterpret_cast<const long long*>(indices), K, v, res);
    CVFES_LAUNCH_CHECK("k_bsr_spmv");
    return CVFES_OK;
}

extern "C" int64_t cvfes_norms_work_size(int64_t n_nodes, int64_t n_samples) {
    if (n_nodes <= 0 || n_samples <= 0) return 0;
    return norm_chunks(n_nodes) * n_samples * 4 + 1;
}

extern "C" int cvfes_solid_norms_f64(int64_t n_nodes, int64_t n_samples, const double* u,
                                     const double* u_prev, const double* invm, double* work,
                                     double* out, int32_t check_finite, void* stream) {
    return launch_norms<double>(n_nodes, n_samples, u, u_prev, invm, work, out, check_finite,
                                (cudaStream_t)stream);
}
extern "C" int cvfes_solid_norms_f32(int64_t n_nodes, int64_t n_samples, const float* u,
                                     const float* u_prev, const float* invm, double* work,
                                     double* out, int32_t check_finite, void* stream) {
    return launch_norms<float>(n_nodes, n_samples, u, u_prev, invm, work, out, check_finite,
                               (cudaStream_t)stream);
}
extern "C" int cvfes_solid_norms_vel_f64(int64_t n_nodes, int64_t n_samples, const double* u,
                                         const double* vel, const double* invm, double* work,
                                         double* out, int32_t check_finite, void* stream) {
    return launch_norms<double>(n_nodes, n_samples, u, vel, invm, work, out, check_finite,
                                (cudaStream_t)stream, true);
}
extern "C" int cvfes_solid_norms_vel_f32(int64_t n_nodes, int64_t n_samples, const float* u,
                                         const float* vel, const float* invm, double* work,
                                         double* out, int32_t check_finite, void* stream) {
    return launch_norms<float>(n_nodes, n_samples, u, vel, invm, work, out, check_finite,
                               (cudaStream_t)stream, true);
}

// ------------------------------------------------------------------ CUDA graphs

extern "C" int cvfes_graph_capture_advance(const cvfes_solid_mesh* mesh, int32_t precision,
                                           const void* coef, const void* invm, void* buf0,
                                           void* buf1, void* buf2, const double* p_sched,
                                           int64_t* clock, int64_t chunk, double dt, double damp,
                                           void* stream, cvfes_graph** out) {
    (void)stream;
    // the buffers must be back in their places after a chunk: a period of 3 steps in the
    // previous-displacement form, 2 in the velocity-state form
    const int period = (mesh && mesh->state_form == 1) ? 2 : 3;
    if (!out || chunk <= 0 || chunk % period != 0 || !clock)
        return fail(CVFES_ERR_ARG,
                    "cvfes_graph_capture_advance: chunk must be a positive multiple of %d and a "
                    "clock is required",
                    period);
    if (precision != 32 && precision != 64)
        return fail(CVFES_ERR_ARG, "cvfes_graph_capture_advance: precision must be 32 or 64");
    cudaStream_t cs;
    CVFES_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaStreamDestroy(cs);
        return fail(CVFES_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e));
    }
    int rc;
    if (precision == 64)
        rc = launch_advance<double>(mesh, (const double*)coef, (const double*)invm, (double*)buf0,
                                    (double*)buf1, (double*)buf2, p_sched,
                                    reinterpret_cast<long long*>(clock), chunk, dt, damp, nullptr,
                                    nullptr, cs);
    else
        rc = launch_advance<float>(mesh, (const float*)coef, (const float*)invm, (float*)buf0,
                                   (float*)buf1, (float*)buf2, p_sched,
                                   reinterpret_cast<long long*>(clock), chunk, dt, damp, nullptr,
                                   nullptr, cs);
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
        return fail(CVFES_ERR_CUDA, "instantiate: %s", cudaGetErrorString(e));
    }
    cvfes_graph* g = new cvfes_graph;
    g->graph = graph;
    g->exec = exec;
    *out = g;
    return CVFES_OK;
}

extern "C" int cvfes_graph_launch(cvfes_graph* g, void* stream) {
    if (!g || !g->exec) return fail(CVFES_ERR_ARG, "cvfes_graph_launch: null graph");
    CVFES_CUDA_TRY(cudaGraphLaunch(g->exec, (cudaStream_t)stream));
    return CVFES_OK;
}

extern "C" int cvfes_graph_destroy(cvfes_graph* g) {
    if (!g) return CVFES_OK;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return CVFES_OK;
}

// ------------------------------------------------------------------ tuning, status
extern "C" int cvfes_set_step_tuning(int32_t precision, int32_t vec, int32_t npb,
                                     int32_t staged, int32_t minb) {
    if (precision != 32 && precision != 64)
        return fail(CVFES_ERR_ARG, "cvfes_set_step_tuning: precision must be 32 or 64");
    const int maxv = precision == 32 ? 4 : 2;
    if (vec < 1 || vec > maxv || (vec & (vec - 1)))
        return fail(CVFES_ERR_ARG, "cvfes_set_step_tuning: vec must be 1, 2%s",
                    maxv == 4 ? " or 4" : "");
    if (npb < 1 || npb > 8)
        return fail(CVFES_ERR_ARG, "cvfes_set_step_tuning: npb must be in 1..8");
    if (minb < 1 || minb > 4)
        return fail(CVFES_ERR_ARG, "cvfes_set_step_tuning: minb must be in 1..4");
    if (staged < 0 || staged > 8)
        return fail(CVFES_ERR_ARG, "cvfes_set_step_tuning: staged must be in 0..8");
    if (staged == 8 && minb > 3)
        return fail(CVFES_ERR_ARG, "cvfes_set_step_tuning: staged 8 takes minb 1..3");
    StepTuning& t = precision == 32 ? g_tune32 : g_tune64;
    t.vec = vec;
    t.npb = npb;
    t.staged = staged;
    t.minb = minb;
    return CVFES_OK;
}

extern "C" int cvfes_get_step_tuning(int32_t precision, int32_t* vec, int32_t* npb,
                                     int32_t* staged, int32_t* minb) {
    if (precision != 32 && precision != 64)
        return fail(CVFES_ERR_ARG, "cvfes_get_step_tuning: precision must be 32 or 64");
    const StepTuning& t = precision == 32 ? g_tune32 : g_tune64;
    if (vec) *vec = t.vec;
    if (npb) *npb = t.npb;
    if (staged) *staged = t.staged;
    if (minb) *minb = t.minb;
    return CVFES_OK;
}

extern "C" int cvfes_set_step_prefetch(int32_t precision, int32_t distance, int32_t parts) {
    if (precision != 32 && precision != 64)
        return fail(CVFES_ERR_ARG, "cvfes_set_step_prefetch: precision must be 32 or 64");
    if (distance < -1 || distance > (1 << 20))
        return fail(CVFES_ERR_ARG, "cvfes_set_step_prefetch: distance must be in -1..2^20");
    if (parts < -1 || parts > 7)
        return fail(CVFES_ERR_ARG, "cvfes_set_step_prefetch: parts must be in -1..7");
    const int q = precision == 32 ? 0 : 1;
    g_pf_dist[q] = distance;
    g_pf_parts[q] = parts;
    return CVFES_OK;
}

extern "C" int cvfes_get_step_prefetch(int32_t precision, int32_t* distance, int32_t* parts) {
    if (precision != 32 && precision != 64)
        return fail(CVFES_ERR_ARG, "cvfes_get_step_prefetch: precision must be 32 or 64");
    const int q = precision == 32 ? 0 : 1;
    if (distance) *distance = g_pf_dist[q];
    if (parts) *parts = g_pf_parts[q];
    return CVFES_OK;
}

extern "C" int cvfes_set_norms_memory(int32_t mode) {
    if (mode != 0 && mode != 1)
        return fail(CVFES_ERR_ARG, "cvfes_set_norms_memory: mode must be 0 (tensor) or 1 (shared)");
    g_norms_mode = mode;
    return CVFES_OK;
}

extern "C" int cvfes_set_wait_probe(int32_t polls) {
    if (polls < 0 || polls > (1 << 20))
        return fail(CVFES_ERR_ARG, "cvfes_set_wait_probe: polls must be 0..2^20");
    g_wait_probe = polls;
    return CVFES_OK;
}

extern "C" int cvfes_status_read(int32_t* status, void* stream) {
    if (!status) return fail(CVFES_ERR_ARG, "cvfes_status_read: null status");
    int32_t h = 0;
    cudaStream_t st = (cudaStream_t)stream;
    CVFES_CUDA_TRY(cudaMemcpyAsync(&h, status, sizeof(h), cudaMemcpyDeviceToHost, st));
    CVFES_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(int32_t), st));
    CVFES_CUDA_TRY(cudaStreamSynchronize(st));
    if (h & 1) return fail(CVFES_ERR_TIMEOUT, "a bounded device wait gave up (status %d)", h);
    if (h) return fail(CVFES_ERR_ARG, "device status %d: slot stage overflow", h);
    return CVFES_OK;
}

// ------------------------------------------------------------ allocation-free norms
// Some callers cannot hand the library a device workspace and must not make it
// allocate one: a watchdog that runs between the steps of a large ensemble whose
// state fills the GPU (a cudaMalloc there can fail, and it synchronises the
// device), or a host framework whose own memory pool owns all device memory.
// For them the FP64 norms reduction keeps its block partials in this fixed
// array instead of a caller workspace.  It is 4 MiB on every GPU that loads the
// library, held until the process exits.
constexpr long long kNormScratchDoubles = 1LL << 19;
static __device__ __align__(256) double g_norm_scratch[kNormScratchDoubles];

// Device address of g_norm_scratch on the current device.  In host code the name
// g_norm_scratch is only a host-side stand-in, so its address must come from
// cudaGetSymbolAddress with that device current.  It is looked up on every call and
// not cached: a cached address would outlive a cudaDeviceReset or a change of the
// current context and point at memory that is no longer the array.  The lookup is a
// query; only the first one on a device may load the library's module, which is why
// the first call on a device must come before any stream capture.
static int norm_scratch_address(double** out) {
    int dev = -1;
    CVFES_CUDA_TRY(cudaGetDevice(&dev));
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_norm_scratch);
    if (e != cudaSuccess || !p)
        return fail(CVFES_ERR_CUDA, "cudaGetSymbolAddress(g_norm_scratch) on device %d: %s", dev,
                    cudaGetErrorString(e));
    *out = static_cast<double*>(p);
    return CVFES_OK;
}

extern "C" int cvfes_solid_norms_noalloc_f32(int64_t n_nodes, int64_t n_samples, const float* u,
                                             const float* u_prev, const float* invm,
                                             double* out, int32_t check_finite, void* stream) {
    if (n_nodes <= 0 || n_samples <= 0 || !u || !u_prev || !invm || !out)
        return fail(CVFES_ERR_ARG, "cvfes_solid_norms_noalloc_f32: bad argument");
    if (4 * n_samples + 1 > kNormScratchDoubles)
        return fail(CVFES_ERR_ARG,
                    "cvfes_solid_norms_noalloc_f32: %lld samples exceed the fixed scratch "
                    "(at most %lld samples)",
                    (long long)n_samples, (kNormScratchDoubles - 1) / 4);
    double* work = nullptr;
    int rc = norm_scratch_address(&work);
    if (rc) return rc;
    const long long S = n_samples;
    long long nch = norm_chunks(n_nodes);
    const long long fit = (kNormScratchDoubles - 1) / (4 * S);
    if (nch > fit) nch = fit;
    const long long npc = (n_nodes + nch - 1) / nch;
    nch = (n_nodes + npc - 1) / npc;
    cudaStream_t st = (cudaStream_t)stream;
    double* total = work + (size_t)nch * S * 4;  // the non-finite counter starts at zero
    CVFES_CUDA_TRY(cudaMemsetAsync(total, 0, sizeof(double), st));
    dim3 grid((unsigned)nch, (unsigned)((S + kNormThreads - 1) / kNormThreads));
    k_norms_partial<float, false><<<grid, kNormThreads, 0, st>>>(n_nodes, (int)S, npc, u, u_prev,
                                                                 invm, work);
    CVFES_LAUNCH_CHECK("k_norms_partial (fixed scratch)");
    k_norms_final<<<final_grid(S), kFinalPairs * kFinalGroups, 0, st>>>(nch, (int)S, work, out, total);
    CVFES_LAUNCH_CHECK("k_norms_final (fixed scratch)");
    if (check_finite) {
        double h = 0.0;
        CVFES_CUDA_TRY(cudaMemcpyAsync(&h, total, sizeof(double), cudaMemcpyDeviceToHost, st));
        CVFES_CUDA_TRY(cudaStreamSynchronize(st));
        if (h != 0.0)
            return fail(CVFES_ERR_NONFINITE, "watchdog: %.0f non-finite state values", h);
    }
    return CVFES_OK;
}
