// Device building blocks of the membrane solid step shared by the single-mesh
// kernels (solid_step.cu) and the batched multi-mesh kernel (solid_batched.cu):
// launch arguments, TMA / mbarrier helpers with bounded waits, the thread ->
// (node, samples) map, the row gather K_s u_s and the fused damped update.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "common.cuh"

namespace cvfes {

template <typename T>
struct StepArgs {
    const int32_t* node_ptr;
    const int4* rec;
    const T* slab;
    const T* fhat;
    const T* coef;
    const T* invm;
    const T* u;
    const T* up;
    T* un;
    const T* trac;
    const double* p_sched;
    const long long* clock;
    long long j;
    double pressure;
    long long n_nodes;
    int S;
    int n_clamped;
    T clamp;
    T eta;
    T w0;
    int tpn;
    int npb;
    int cap_slots;   // slot capacity of the shared-memory stage (staged kernel)
    int gather_rows; // rows of each warp's gather buffer (gather kernel)
    int nch;         // sample chunks per node block (staged kernels; 1D grid, chunk fastest)
    int* status;     // bit 0: a bounded wait gave up
    int pf_dist = 0;  // fan kernel: nodes ahead whose rows are prefetched into L2 (0: off)
    int pf_parts = 0; // bit 0: node rows; bit 1: element coefficient rows
    int pf_group = 1; // node blocks covered by one prefetching block
    // Velocity-state form (null: the second state buffer `up` holds u_{n-1}).  When set
    // it equals `up`, which then holds the increment v_n = u_n - u_{n-1}: the step reads
    // it and writes v_{n+1} back in place (each row is read and written by its owner
    // thread only), and u_{n+1} = u_n + v_{n+1} goes to `un`.  The increment is then
    // never rebuilt from two rounded displacements, so the FP32 rounding of u does not
    // feed back into the velocity.
    T* vel = nullptr;
    // Failure-path test of the bounded waits (0: off).  When > 0 the fan kernel sets
    // its stage barrier up for two arrivals, issues no copy and waits at most this many
    // polls: the wait gives up with nothing in flight, the kernel records bit 0 in
    // `status` and returns without writing the step.
    int probe_polls = 0;
    // Fused per-sample norms (persistent fan kernel only; null: off).  Each block keeps
    // one sample chunk for its whole life and accumulates, per lane and sample, the FP64
    // sums of u_{n+1}^2, du^2, m du^2 and the non-finite count of u_{n+1} over all its
    // nodes in shared memory; at its end it writes them to row blockIdx.x / nch of
    // norm_part [rows][S][4], which k_norms_final then sums in row order.
    double* norm_part = nullptr;
    // Damping per dof (the OpenCL class's calc_u): eta = dt damp / m per row, w = dt^2 / m.
    // Off: mass-proportional damping, one eta for all rows.  Set: A.eta holds dt damp.
    int damp_per_dof = 0;
};

// eta of one row: dt damp / m (damping per dof) or the launch's eta.
template <typename T>
__device__ __forceinline__ T row_eta(const StepArgs<T>& A, T im) {
    return A.damp_per_dof ? A.eta * im : A.eta;
}

// Norm terms of one node (sum of squares of its three new values, of its three
// increments, and the count of non-finite values) are formed in the state's type and
// only the node sums are taken to FP64: with the FP32 state each node term carries
// three FP32 roundings (the mass-weighted one also a reciprocal of at most 1 ulp and a
// product: <= 4e-7 relative; all terms positive, so the sum over nodes keeps the
// bound), and the FP64 sums
// over nodes need three conversions per node instead of seven (a conversion to FP64
// runs at a quarter of the FP64 rate; per value they cost a tenth of the step).  The
// separate norms pass forms the same node terms in the same order.
// FP32: the hardware reciprocal approximation (rcp.approx, at most 1 ulp), one instruction
// where the correctly rounded reciprocal cost 4% of the step as a norm term.
__device__ __forceinline__ float norm_mass(float im) {
    float m;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(m) : "f"(im));
    return im != 0.f ? m : 0.f;
}
__device__ __forceinline__ double norm_mass(double im) { return im != 0.0 ? 1.0 / im : 0.0; }

// ------------------------------------------------------------ tensor-memory accumulators
// The fused norms keep each lane's FP64 sums in tensor memory (TMEM), which the step
// does not otherwise use: no shared memory (the L1 that serves the neighbour-row
// gathers) and no registers between nodes.  Warp w of a block owns TMEM lanes
// 32 (w % 4) .. + 31 and columns from 32 (w / 4); in its lane's row, quantity q (sum u^2,
// sum du^2, sum m du^2) of sample i is the double at columns 2 (q V + i) and + 1, and
// the non-finite count of sample i the integer at column 6 V + i.

__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {  // warp-wide
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"((uint32_t)__cvta_generic_to_shared(slot)), "r"(cols) : "memory");
}
// The block allocates no more tensor memory.  A kernel that contains an allocation gets
// further blocks on an SM only after its resident blocks have said so (measured on the
// persistent fan kernel: one block per SM otherwise), so every block says it, whether it
// allocated or not.
__device__ __forceinline__ void tmem_relinquish() {  // warp-wide
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t cols) {  // warp-wide
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols)
                 : "memory");
}
__device__ __forceinline__ void tmem_fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_wait_st() {
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
// N consecutive 32-bit columns of the lane's row (32x32b shape: one row per lane).
template <int N>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, uint32_t (&r)[N]) {
    static_assert(N == 1 || N == 2 || N == 4 || N == 8, "tmem_ld: 1, 2, 4 or 8 columns");
    if constexpr (N == 1) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];"
                     : "=r"(r[0]) : "r"(taddr) : "memory");
    } else if constexpr (N == 2) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];"
                     : "=r"(r[0]), "=r"(r[1]) : "r"(taddr) : "memory");
    } else if constexpr (N == 4) {
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(taddr) : "memory");
    } else {
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
              "=r"(r[7])
            : "r"(taddr)
            : "memory");
    }
}
template <int N>
__device__ __forceinline__ void tmem_st(uint32_t taddr, const uint32_t (&r)[N]) {
    static_assert(N == 1 || N == 2 || N == 4 || N == 8, "tmem_st: 1, 2, 4 or 8 columns");
    if constexpr (N == 1) {
        asm volatile("tcgen05.st.sync.aligned.32x32b.x1.b32 [%0], {%1};" ::"r"(taddr), "r"(r[0])
                     : "memory");
    } else if constexpr (N == 2) {
        asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(taddr),
                     "r"(r[0]), "r"(r[1])
                     : "memory");
    } else if constexpr (N == 4) {
        asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr),
                     "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3])
                     : "memory");
    } else {
        asm volatile(
            "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(
                taddr),
            "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7])
            : "memory");
    }
}
__device__ __forceinline__ void add_to_words(uint32_t& lo, uint32_t& hi, double x) {
    const double v = __hiloint2double((int)hi, (int)lo) + x;
    lo = (uint32_t)__double2loint(v);
    hi = (uint32_t)__double2hiint(v);
}

// Zero the lane's accumulators (every thread of the warp calls it).
template <int V>
__device__ __forceinline__ void norms_zero(uint32_t tm) {
    uint32_t z[2 * V], zn[V];
#pragma unroll
    for (int i = 0; i < 2 * V; ++i) z[i] = 0u;
#pragma unroll
    for (int i = 0; i < V; ++i) zn[i] = 0u;
#pragma unroll
    for (int q = 0; q < 3; ++q) tmem_st<2 * V>(tm + (uint32_t)(q * 2 * V), z);
    tmem_st<V>(tm + (uint32_t)(6 * V), zn);
    tmem_wait_st();
}

// Add one node's terms to the lane's accumulators (every thread of the warp calls it).
template <typename T, int V>
__device__ __forceinline__ void norms_add(uint32_t tm, const Vec<T, V>& im, const T (&su)[V],
                                          const T (&sv)[V], const int (&nf)[V]) {
    uint32_t r[3][2 * V];
    tmem_wait_st();  // the previous node's stores to these columns
#pragma unroll
    for (int q = 0; q < 3; ++q) tmem_ld<2 * V>(tm + (uint32_t)(q * 2 * V), r[q]);
    tmem_wait_ld();
#pragma unroll
    for (int q = 0; q < 3; ++q) {
#pragma unroll
        for (int i = 0; i < V; ++i) {
            const T x = q == 0 ? su[i] : (q == 1 ? sv[i] : norm_mass(im.v[i]) * sv[i]);
            add_to_words(r[q][2 * i], r[q][2 * i + 1], (double)x);
        }
        tmem_st<2 * V>(tm + (uint32_t)(q * 2 * V), r[q]);
    }
    int any = 0;
#pragma unroll
    for (int i = 0; i < V; ++i) any |= nf[i];
    if (__any_sync(0xffffffffu, any != 0)) {  // rare: a non-finite value in the warp's node
        uint32_t rn[V];
        tmem_ld<V>(tm + (uint32_t)(6 * V), rn);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < V; ++i) rn[i] += (uint32_t)nf[i];
        tmem_st<V>(tm + (uint32_t)(6 * V), rn);
    }
}

// Add the lane's sums to dst[(q V + i) * 32] (quantity q of sample i; q = 3 the non-finite
// count), or store them there when first; one quantity at a time (every thread of the
// warp calls it).
template <int V>
__device__ __forceinline__ void norms_fold(uint32_t tm, double* dst, bool first) {
    tmem_wait_st();
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        uint32_t r[2 * V];
        tmem_ld<2 * V>(tm + (uint32_t)(q * 2 * V), r);
        tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < V; ++i) {
            double* c = dst + (q * V + i) * 32;
            const double x = __hiloint2double((int)r[2 * i + 1], (int)r[2 * i]);
            *c = first ? x : *c + x;
        }
    }
    uint32_t rn[V];
    tmem_ld<V>(tm + (uint32_t)(6 * V), rn);
    tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < V; ++i) {
        double* c = dst + (3 * V + i) * 32;
        *c = first ? (double)rn[i] : *c + (double)rn[i];
    }
}

// Per-lane accumulator of the fused norms: quantity q of sample i of the lane's vector
// at nacc[(q * V + i) * 32] (lanes innermost: no shared-memory bank conflicts).
template <typename T, int V>
__device__ __forceinline__ void norms_add_smem(double* nacc, const Vec<T, V>& im, const T (&su)[V],
                                          const T (&sv)[V], const int (&nf)[V]) {
#pragma unroll
    for (int i = 0; i < V; ++i) {
        nacc[(0 * V + i) * 32] += (double)su[i];
        nacc[(1 * V + i) * 32] += (double)sv[i];
        nacc[(2 * V + i) * 32] += (double)(norm_mass(im.v[i]) * sv[i]);
        if (nf[i]) nacc[(3 * V + i) * 32] += (double)nf[i];
    }
}

// ------------------------------------------------------------ TMA / mbarrier helpers
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}
// One-dimensional TMA bulk copy global -> this CTA's shared memory (no multicast).
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes,
                                         uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.b32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(phase)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after max_polls try_wait rounds (each round suspends the
// thread for a bounded, hardware-chosen time), so a lost transfer cannot hang the GPU.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t phase, int max_polls) {
    for (int i = 0; i < max_polls; ++i)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}
__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}
// L2 prefetch of a byte range by the bulk-copy unit (no registers, no L1 line).  The
// range is shrunk to 16-byte boundaries, so nothing outside [p, p + bytes) is touched.
__device__ __forceinline__ void bulk_prefetch_l2(const void* p, size_t bytes) {
    uintptr_t b = (reinterpret_cast<uintptr_t>(p) + 15) & ~uintptr_t(15);
    const uintptr_t e = (reinterpret_cast<uintptr_t>(p) + bytes) & ~uintptr_t(15);
    while (b < e) {
        const uint32_t n = (uint32_t)((e - b) < 32768 ? (e - b) : 32768);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(b), "r"(n) : "memory");
        b += n;
    }
}
constexpr int kMaxPolls = 1 << 22;

// Record and stiffness-row pointers of stage q of a two-stage shared-memory ring.
template <typename P>
__device__ __forceinline__ P* stage_ptr(P* base0, size_t stage_bytes, int q) {
    return reinterpret_cast<P*>(reinterpret_cast<unsigned char*>(base0) + q * stage_bytes);
}
__device__ __forceinline__ int4* stage_rec(int4* base0, size_t stage_bytes, int q) {
    return stage_ptr(base0, stage_bytes, q);
}
template <typename T>
__device__ __forceinline__ T* stage_slab(T* base0, size_t stage_bytes, int q) {
    return stage_ptr(base0, stage_bytes, q);
}

// Prefetch into L2 the rows that nodes a0 .. a0 + n - 1 will read: their displacement
// rows (which lower-numbered neighbours touch first), previous displacement, inverse
// mass and the coefficient rows of their elements.  One lane per contiguous range; the
// coefficient rows are found through the nodes' slot records.
template <typename T>
__device__ __forceinline__ void fan_prefetch(const StepArgs<T>& A, long long a0, int n,
                                             int lane) {
    if (a0 >= A.n_nodes) return;
    const long long a1 = (a0 + n < A.n_nodes) ? a0 + n : A.n_nodes;
    const size_t S = (size_t)A.S;
    const size_t nrow = (size_t)(a1 - a0) * S * sizeof(T);
    if (A.pf_parts & 1) {
        if (lane == 0) bulk_prefetch_l2(A.u + (size_t)a0 * 3 * S, 3 * nrow);
        if (lane == 1) bulk_prefetch_l2(A.up + (size_t)a0 * 3 * S, 3 * nrow);
        if (lane == 2) bulk_prefetch_l2(A.invm + (size_t)a0 * S, nrow);
    }
    if (!(A.pf_parts & 2)) return;
    const int kb = __ldg(A.node_ptr + a0), ke = __ldg(A.node_ptr + a1);
    for (int k = kb + lane; k < ke; k += 32)
        bulk_prefetch_l2(A.coef + (size_t)__ldg(&A.rec[k].x) * S, S * sizeof(T));
}

// Thread -> (node, sample vector).  A block holds `npb` consecutive nodes and
// `tpn` consecutive sample vectors of each (tpn = min(S/VEC, 32)); blockIdx.y
// picks the sample chunk, the last one partly filled when S/VEC is not a
// multiple of 32.  The warps of one block therefore gather overlapping
// neighbour rows and element coefficients of one sample chunk.
__device__ __forceinline__ bool map_row(int tpn, int npb, long long n_nodes, int sv,
                                        long long& a, int& vec) {
    const int t = threadIdx.x / tpn;
    if (t >= npb) return false;
    a = (long long)blockIdx.x * npb + t;
    vec = blockIdx.y * tpn + (threadIdx.x - t * tpn);
    return a < n_nodes && vec < sv;
}

// L2 prefetch of the fan kernels for a mesh of this bandwidth under the current setting
// of cvfes_set_step_prefetch: distance in nodes (0: off) and the parts prefetched (bit 0
// node rows, bit 1 element coefficient rows; -1: by prefetch_parts at launch).
struct Prefetch {
    int dist, parts;
};
// A prefetching block covers enough node blocks for kPrefetchChunks sample chunks of
// work (the first chunk of every node block when there are that many chunks), so the
// per-block cost of issuing the prefetches is spread the same way at any sample count.
constexpr int kPrefetchChunks = 4;
inline int prefetch_group(int chunks) {
    return chunks >= kPrefetchChunks ? 1 : (kPrefetchChunks + chunks - 1) / chunks;
}
// Automatic parts (-1): node rows and coefficient rows with at least kPrefetchChunks
// sample chunks per node block, node rows only below (the coefficient rows' dependent
// slot-record loads then cost more than they save).
inline int prefetch_parts(int parts, int chunks) {
    return parts >= 0 ? parts : (chunks >= kPrefetchChunks ? 3 : 1);
}
Prefetch step_prefetch(int precision, long long bandwidth);

struct RowGrid {
    dim3 grid;
    int tpn, npb;
};

inline RowGrid row_grid(long long n_nodes, int sv, int block) {
    RowGrid g;
    g.tpn = sv < 32 ? sv : 32;
    g.npb = block / g.tpn;
    g.grid = dim3((unsigned)((n_nodes + g.npb - 1) / g.npb), (unsigned)((sv + g.tpn - 1) / g.tpn));
    return g;
}

// Row a of K_s u_s for VEC samples starting at column col.
template <typename T, int V, bool DIFF>
__device__ __forceinline__ void ku_row(const int32_t* __restrict__ node_ptr,
                                       const int4* __restrict__ rec, const T* __restrict__ slab,
                                       const T* __restrict__ coef, const T* __restrict__ u,
                                       size_t S, size_t col, long long a, const Vec<T, V> (&ua)[3],
                                       Vec<T, V> (&acc)[3]) {
    const int k0 = __ldg(node_ptr + a), k1 = __ldg(node_ptr + a + 1);
#pragma unroll
    for (int d = 0; d < 3; ++d) acc[d] = vzero<T, V>();
    Vec<T, V> carry[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) carry[d] = vzero<T, V>();
#pragma unroll 2
    for (int k = k0; k < k1; ++k) {
        const int4 r = __ldg(rec + k);
        Vec<T, V> x1[3], x2[3];
        if (r.w & 1) {
#pragma unroll
            for (int d = 0; d < 3; ++d) x1[d] = carry[d];
        } else {
            const T* p1 = u + (size_t)r.y * 3 * S + col;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                x1[d] = ldg<T, V>(p1 + d * S);
                if constexpr (DIFF) x1[d] = vsub(x1[d], ua[d]);
            }
        }
        const T* p2 = u + (size_t)r.z * 3 * S + col;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            x2[d] = ldg<T, V>(p2 + d * S);
            if constexpr (DIFF) x2[d] = vsub(x2[d], ua[d]);
        }
        const Vec<T, V> c = ldg<T, V>(coef + (size_t)r.x * S + col);
        const T* K = slab + (size_t)kSlabStride * k;
        T kk[27];
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
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            Vec<T, V> t = vzero<T, V>();
            if constexpr (!DIFF) {
#pragma unroll
                for (int jj = 0; jj < 3; ++jj) axpy(t, kk[3 * i + jj], ua[jj]);
            }
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) axpy(t, kk[9 + 3 * i + jj], x1[jj]);
#pragma unroll
            for (int jj = 0; jj < 3; ++jj) axpy(t, kk[18 + 3 * i + jj], x2[jj]);
            vfma(acc[i], c, t);
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) carry[d] = x2[d];
    }
}

// The step's pressure: one value per launch, so it is read once at kernel entry
// (a schedule entry indexed by the device clock, or the value passed by the host).
template <typename T>
__device__ __forceinline__ T step_pressure(const StepArgs<T>& A) {
    return (T)(A.p_sched ? A.p_sched[(A.clock ? A.clock[0] : 0LL) + A.j] : A.pressure);
}

// Nodal external load p*fhat (+ traction) of node a, read early by the caller.
template <typename T>
__device__ __forceinline__ void node_load(const StepArgs<T>& A, long long a, T p, T (&f)[3]) {
    const float4* q = nullptr;
#pragma unroll
    for (int d = 0; d < 3; ++d) f[d] = p * __ldg(A.fhat + 4 * a + d);
    if (A.trac) {
#pragma unroll
        for (int d = 0; d < 3; ++d) f[d] += __ldg(A.trac + 4 * a + d);
    }
    (void)q;
}

// Fused update of one node row (increment form, see the file header) and its store,
// from the row's u_{n-1} and inverse mass already in registers.
template <typename T, int V>
__device__ __forceinline__ void step_update(const StepArgs<T>& A, size_t S, size_t row,
                                            const Vec<T, V> (&ua)[3], const Vec<T, V> (&acc)[3],
                                            const T (&f)[3], const Vec<T, V> (&ups)[3],
                                            const Vec<T, V>& im) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const Vec<T, V>& up = ups[d];
        const T load = f[d];
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

// Dirichlet row: u_{n+1} = clamp; in the velocity-state form also v_{n+1} = clamp - u_n.
// With nacc (fused norms) the row's contributions are added there.
template <typename T, int V>
__device__ __forceinline__ void clamp_store(const StepArgs<T>& A, size_t S, size_t row,
                                            double* nacc = nullptr, long long a = 0,
                                            size_t col = 0) {
    const Vec<T, V> cl = vfill<T, V>(A.clamp);
    T su[V], sv[V];
    int nf[V];
#pragma unroll
    for (int i = 0; i < V; ++i) {
        su[i] = sv[i] = T(0);
        nf[i] = 0;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        if (A.vel || nacc) {
            const Vec<T, V> dv = vsub(cl, ldg<T, V>(A.u + row + d * S));
            if (A.vel) stcs<T, V>(A.vel + row + d * S, dv);
            if (nacc) {
#pragma unroll
                for (int i = 0; i < V; ++i) {
                    su[i] = fma(cl.v[i], cl.v[i], su[i]);
                    sv[i] = fma(dv.v[i], dv.v[i], sv[i]);
                    nf[i] += isfinite(cl.v[i]) ? 0 : 1;
                }
            }
        }
        stcs<T, V>(A.un + row + d * S, cl);
    }
    if (nacc) norms_add_smem<T, V>(nacc, ldcs<T, V>(A.invm + (size_t)a * S + col), su, sv, nf);
}

// As step_update, reading the row's u_{n-1} (or v_n) and inverse mass here.
// With nacc (fused norms) the row's contributions to the per-sample sums of u_{n+1}^2,
// du^2 (v_{n+1}^2, or u_{n+1} - u_n) and m du^2 are added there (node terms as norms_add).
template <typename T, int V>
__device__ __forceinline__ void step_epilogue(const StepArgs<T>& A, long long a, size_t S,
                                              size_t col, size_t row, const Vec<T, V> (&ua)[3],
                                              const Vec<T, V> (&acc)[3], const T (&f)[3],
                                              double* nacc = nullptr) {
    const Vec<T, V> im = ldcs<T, V>(A.invm + (size_t)a * S + col);
    T su[V], sv[V];
    int nf[V];
#pragma unroll
    for (int i = 0; i < V; ++i) {
        su[i] = sv[i] = T(0);
        nf[i] = 0;
    }
    if (A.vel) {
        // velocity-state form: v_{n+1} = v_n (1 - eta) + w (p f - K u_n), u_{n+1} = u_n + v_{n+1};
        // a row without mass (u_{n+1} = 0) keeps v_{n+1} = -u_n, the exact increment.
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const Vec<T, V> vo = ldcs<T, V>(A.up + row + d * S);
            const T load = f[d];
            Vec<T, V> o, vn;
#pragma unroll
            for (int i = 0; i < V; ++i) {
                const T w = A.w0 * im.v[i];
                const T v = fma(w, load - acc[d].v[i], fma(-row_eta(A, im.v[i]), vo.v[i], vo.v[i]));
                const bool live = im.v[i] != T(0);
                o.v[i] = live ? ua[d].v[i] + v : T(0);
                vn.v[i] = live ? v : -ua[d].v[i];
                if (nacc) {
                    su[i] = fma(o.v[i], o.v[i], su[i]);
                    sv[i] = fma(vn.v[i], vn.v[i], sv[i]);
                    nf[i] += isfinite(o.v[i]) ? 0 : 1;
                }
            }
            stcs<T, V>(A.un + row + d * S, o);
            stcs<T, V>(A.vel + row + d * S, vn);
        }
        if (nacc) norms_add_smem<T, V>(nacc, im, su, sv, nf);
        return;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const Vec<T, V> up = ldcs<T, V>(A.up + row + d * S);
        const T load = f[d];
        Vec<T, V> o;
#pragma unroll
        for (int i = 0; i < V; ++i) {
            const T dv = ua[d].v[i] - up.v[i];
            const T w = A.w0 * im.v[i];
            const T v = fma(w, load - acc[d].v[i], fma(-row_eta(A, im.v[i]), dv, dv));
            o.v[i] = (im.v[i] != T(0)) ? ua[d].v[i] + v : T(0);
            if (nacc) {
                const T du = o.v[i] - ua[d].v[i];
                su[i] = fma(o.v[i], o.v[i], su[i]);
                sv[i] = fma(du, du, sv[i]);
                nf[i] += isfinite(o.v[i]) ? 0 : 1;
            }
        }
        stcs<T, V>(A.un + row + d * S, o);
    }
    if (nacc) norms_add_smem<T, V>(nacc, im, su, sv, nf);
}

// clamp_store and step_epilogue with the norms' sums in tensor memory at tm (norms_add),
// for the persistent step with the norms fused in.  Copies, not one template over both
// sinks: with one template the plain persistent step compiled to a schedule 3.5% slower
// (2.376 against 2.295 ms/step on the 256x1024 tube, same box), although its norm code
// never runs.
template <typename T, int V>
__device__ __forceinline__ void clamp_store_tm(const StepArgs<T>& A, size_t S, size_t row,
                                               uint32_t tm, long long a, size_t col) {
    const Vec<T, V> cl = vfill<T, V>(A.clamp);
    T su[V], sv[V];
    int nf[V];
#pragma unroll
    for (int i = 0; i < V; ++i) {
        su[i] = sv[i] = T(0);
        nf[i] = 0;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const Vec<T, V> dv = vsub(cl, ldg<T, V>(A.u + row + d * S));
        if (A.vel) stcs<T, V>(A.vel + row + d * S, dv);
#pragma unroll
        for (int i = 0; i < V; ++i) {
            su[i] = fma(cl.v[i], cl.v[i], su[i]);
            sv[i] = fma(dv.v[i], dv.v[i], sv[i]);
            nf[i] += isfinite(cl.v[i]) ? 0 : 1;
        }
        stcs<T, V>(A.un + row + d * S, cl);
    }
    norms_add<T, V>(tm, ldcs<T, V>(A.invm + (size_t)a * S + col), su, sv, nf);
}

// As step_update, reading the row's u_{n-1} (or v_n) and inverse mass here.
template <typename T, int V>
__device__ __forceinline__ void step_epilogue_tm(const StepArgs<T>& A, long long a, size_t S,
                                                 size_t col, size_t row, const Vec<T, V> (&ua)[3],
                                                 const Vec<T, V> (&acc)[3], const T (&f)[3],
                                                 uint32_t tm) {
    const Vec<T, V> im = ldcs<T, V>(A.invm + (size_t)a * S + col);
    T su[V], sv[V];
    int nf[V];
#pragma unroll
    for (int i = 0; i < V; ++i) {
        su[i] = sv[i] = T(0);
        nf[i] = 0;
    }
    if (A.vel) {
        // velocity-state form: v_{n+1} = v_n (1 - eta) + w (p f - K u_n), u_{n+1} = u_n + v_{n+1};
        // a row without mass (u_{n+1} = 0) keeps v_{n+1} = -u_n, the exact increment.
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const Vec<T, V> vo = ldcs<T, V>(A.up + row + d * S);
            const T load = f[d];
            Vec<T, V> o, vn;
#pragma unroll
            for (int i = 0; i < V; ++i) {
                const T w = A.w0 * im.v[i];
                const T v = fma(w, load - acc[d].v[i], fma(-row_eta(A, im.v[i]), vo.v[i], vo.v[i]));
                const bool live = im.v[i] != T(0);
                o.v[i] = live ? ua[d].v[i] + v : T(0);
                vn.v[i] = live ? v : -ua[d].v[i];
                su[i] = fma(o.v[i], o.v[i], su[i]);
                sv[i] = fma(vn.v[i], vn.v[i], sv[i]);
                nf[i] += isfinite(o.v[i]) ? 0 : 1;
            }
            stcs<T, V>(A.un + row + d * S, o);
            stcs<T, V>(A.vel + row + d * S, vn);
        }
        norms_add<T, V>(tm, im, su, sv, nf);
        return;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const Vec<T, V> up = ldcs<T, V>(A.up + row + d * S);
        const T load = f[d];
        Vec<T, V> o;
#pragma unroll
        for (int i = 0; i < V; ++i) {
            const T dv = ua[d].v[i] - up.v[i];
            const T w = A.w0 * im.v[i];
            const T v = fma(w, load - acc[d].v[i], fma(-row_eta(A, im.v[i]), dv, dv));
            o.v[i] = (im.v[i] != T(0)) ? ua[d].v[i] + v : T(0);
            const T du = o.v[i] - ua[d].v[i];
            su[i] = fma(o.v[i], o.v[i], su[i]);
            sv[i] = fma(du, du, sv[i]);
            nf[i] += isfinite(o.v[i]) ? 0 : 1;
        }
        stcs<T, V>(A.un + row + d * S, o);
    }
    norms_add<T, V>(tm, im, su, sv, nf);
}

// ------------------------------------------------------------ fan-rotation row
// The fan order makes the first neighbour of element k the second neighbour of
// element k-1, so element k needs only one new neighbour row set.  Three register
// buffers rotate through the roles (previous = first neighbour, current = second
// neighbour, next = in flight); the slot loop is unrolled three times so the
// rotation is a renaming, not a copy.  Neighbour rows are turned into differences
// u_b - u_a once (FP32 form) and reused by the following element.
template <typename T, int V>
__device__ __forceinline__ void load_rows(Vec<T, V> (&x)[3], const T* __restrict__ u, int node,
                                          size_t S, size_t col) {
    const T* p = u + (size_t)node * 3 * S + col;
#pragma unroll
    for (int d = 0; d < 3; ++d) x[d] = ldg<T, V>(p + d * S);
}
template <typename T, int V, bool DIFF>
__device__ __forceinline__ void to_diff(Vec<T, V> (&x)[3], const Vec<T, V> (&ua)[3]) {
    if constexpr (DIFF) {
#pragma unroll
        for (int d = 0; d < 3; ++d) x[d] = vsub(x[d], ua[d]);
    }
}
template <typename T, int V, bool DIFF>
__device__ __forceinline__ void slot_fma(const T* K, const Vec<T, V>& c, const Vec<T, V> (&d1)[3],
                                         const Vec<T, V> (&d2)[3], const Vec<T, V> (&ua)[3],
                                         Vec<T, V> (&acc)[3]) {
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

// One element of the fan: prev holds the first neighbour (difference), cur the
// second one as loaded; the next element's row set is issued into nxt first.
template <typename T, int V, bool DIFF>
__device__ __forceinline__ void fan_phase(int& k, int k1, const int4* srec, const T* sslab,
                                          const T* __restrict__ u, const T* __restrict__ coef,
                                          size_t S, size_t col, const Vec<T, V> (&ua)[3],
                                          Vec<T, V> (&acc)[3], Vec<T, V> (&prev)[3],
                                          Vec<T, V> (&cur)[3], const Vec<T, V>& ccur,
                                          Vec<T, V> (&nxt)[3], Vec<T, V>& cnxt) {
    const bool more = k + 1 < k1;
    int4 rn = make_int4(0, 0, 0, 1);
    if (more) {
        rn = srec[k + 1];
        load_rows<T, V>(nxt, u, rn.z, S, col);
        cnxt = ldg<T, V>(coef + (size_t)rn.x * S + col);
    }
    to_diff<T, V, DIFF>(cur, ua);
    slot_fma<T, V, DIFF>(sslab + (size_t)kSlabStride * k, ccur, prev, cur, ua, acc);
    if (more && !(rn.w & 1)) {  // fan break: the next element's first neighbour is new
        load_rows<T, V>(cur, u, rn.y, S, col);
        to_diff<T, V, DIFF>(cur, ua);
    }
    ++k;
}

template <typename T, int V, bool DIFF>
__device__ __forceinline__ void ku_row_fan(const int4* srec, const T* sslab, int k0, int k1,
                                           const T* __restrict__ u, const T* __restrict__ coef,
                                           size_t S, size_t col, const Vec<T, V> (&ua)[3],
                                           Vec<T, V> (&acc)[3]) {
#pragma unroll
    for (int d = 0; d < 3; ++d) acc[d] = vzero<T, V>();
    if (k0 >= k1) return;
    Vec<T, V> B0[3], B1[3], B2[3], c0, c1, c2;
    const int4 r0 = srec[k0];
    load_rows<T, V>(B0, u, r0.y, S, col);
    load_rows<T, V>(B1, u, r0.z, S, col);
    c1 = ldg<T, V>(coef + (size_t)r0.x * S + col);
    to_diff<T, V, DIFF>(B0, ua);
    int k = k0;
    while (true) {
        fan_phase<T, V, DIFF>(k, k1, srec, sslab, u, coef, S, col, ua, acc, B0, B1, c1, B2, c2);
        if (k >= k1) break;
        fan_phase<T, V, DIFF>(k, k1, srec, sslab, u, coef, S, col, ua, acc, B1, B2, c2, B0, c0);
        if (k >= k1) break;
        fan_phase<T, V, DIFF>(k, k1, srec, sslab, u, coef, S, col, ua, acc, B2, B0, c0, B1, c1);
        if (k >= k1) break;
    }
}

// ------------------------------------------------------------ fan row, two ahead
// As ku_row_fan, with each element's new neighbour row and coefficient row requested
// two elements ahead: four register buffers rotate (first neighbour, second neighbour,
// and the next two elements' rows in flight), the slot loop unrolled four times.  The
// products and their order are those of ku_row_fan, so the bits are the same.
template <typename T, int V, bool DIFF>
__device__ __forceinline__ void fan2_phase(int& k, int k1, const int4* srec, const T* sslab,
                                           const T* __restrict__ u, const T* __restrict__ coef,
                                           size_t S, size_t col, const Vec<T, V> (&ua)[3],
                                           Vec<T, V> (&acc)[3], Vec<T, V> (&prev)[3],
                                           Vec<T, V> (&cur)[3], const Vec<T, V>& ccur,
                                           Vec<T, V> (&n2)[3], Vec<T, V>& c2) {
    if (k + 2 < k1) {
        const int4 r2 = srec[k + 2];
        load_rows<T, V>(n2, u, r2.z, S, col);
        c2 = ldg<T, V>(coef + (size_t)r2.x * S + col);
    }
    to_diff<T, V, DIFF>(cur, ua);
    slot_fma<T, V, DIFF>(sslab + (size_t)kSlabStride * k, ccur, prev, cur, ua, acc);
    if (k + 1 < k1) {
        const int4 r1 = srec[k + 1];
        if (!(r1.w & 1)) {  // fan break: the next element's first neighbour is new
            load_rows<T, V>(cur, u, r1.y, S, col);
            to_diff<T, V, DIFF>(cur, ua);
        }
    }
    ++k;
}

template <typename T, int V, bool DIFF>
__device__ __forceinline__ void ku_row_fan2(const int4* srec, const T* sslab, int k0, int k1,
                                            const T* __restrict__ u, const T* __restrict__ coef,
                                            size_t S, size_t col, const Vec<T, V> (&ua)[3],
                                            Vec<T, V> (&acc)[3]) {
#pragma unroll
    for (int d = 0; d < 3; ++d) acc[d] = vzero<T, V>();
    if (k0 >= k1) return;
    Vec<T, V> B0[3], B1[3], B2[3], B3[3], c0, c1, c2, c3;
    const int4 r0 = srec[k0];
    load_rows<T, V>(B0, u, r0.y, S, col);
    load_rows<T, V>(B1, u, r0.z, S, col);
    c0 = ldg<T, V>(coef + (size_t)r0.x * S + col);
    if (k0 + 1 < k1) {
        const int4 r1 = srec[k0 + 1];
        load_rows<T, V>(B2, u, r1.z, S, col);
        c1 = ldg<T, V>(coef + (size_t)r1.x * S + col);
    }
    to_diff<T, V, DIFF>(B0, ua);
    int k = k0;
    while (true) {
        fan2_phase<T, V, DIFF>(k, k1, srec, sslab, u, coef, S, col, ua, acc, B0, B1, c0, B3, c2);
        if (k >= k1) break;
        fan2_phase<T, V, DIFF>(k, k1, srec, sslab, u, coef, S, col, ua, acc, B1, B2, c1, B0, c3);
        if (k >= k1) break;
        fan2_phase<T, V, DIFF>(k, k1, srec, sslab, u, coef, S, col, ua, acc, B2, B3, c2, B1, c0);
        if (k >= k1) break;
        fan2_phase<T, V, DIFF>(k, k1, srec, sslab, u, coef, S, col, ua, acc, B3, B0, c3, B2, c1);
        if (k >= k1) break;
    }
}

// L1 prefetch of one address (the line lands in L1 and L2; no register is written).
__device__ __forceinline__ void prefetch_l1(const void* p) {
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
}

// Resident blocks per SM of a persistent kernel (solid_step.cu; cached per kernel,
// device, block size and shared memory) and the device's SM count.
int fanp_blocks_per_sm(const void* kernel, int threads, size_t smem, int* per_sm);
int device_sm_count();

// TMA-tiled step (solid_tile.cu): returns 1 without launching when the mesh has no
// tiling or the shape does not fit the tiled kernel.
template <typename T>
int launch_step_tile(const cvfes_solid_mesh* m, const StepArgs<T>& A, int vec_max,
                     cudaStream_t st);

}  // namespace cvfes

// Executable CUDA graph handed out through the C ABI (cvfes_graph_* entry points).
struct cvfes_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};
