// Batched multi-mesh solid step: many independent tube meshes with their own node
// counts, sample counts, time steps and pressure schedules advance together in one
// persistent launch per step.
//
// The caller packs one descriptor per mesh into a device table (cvfes_batch_pack).
// Work item w of the batch is (mesh m, node block, sample chunk) with the chunk
// fastest; item offsets per mesh are prefix sums, so a block finds its mesh by a
// binary search.  Blocks loop over items with a grid stride (persistent), and each
// thread runs the same row gather K_s u_s and fused damped update as the
// single-mesh L1 kernel, so a mesh advanced in a batch is bitwise identical to the
// same mesh advanced alone.  All meshes rotate their three state buffers in lock
// step (the rotation phase is the step count mod 6, which fixes the roles of both
// state forms); the phase and the step's offset into the pressure schedules are
// launch arguments (a device clock supplies the base offset inside CUDA graphs).
//
// Two kernels walk the items.  The gather kernel (variant 0) runs the single-mesh L1
// row gather per thread.  The fan kernel (variant 1) gives each item to a block of
// kBatchWarps warps: the item's slot records and stiffness rows are staged by TMA
// into one of two shared-memory stages while the previous item is multiplied, and
// each thread walks its node's fan with the three-buffer rotation of the single-mesh
// fan kernel (a warp holds 32 / min(32, S/VEC) nodes when a mesh has few samples).
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"
#include "step_core.cuh"

namespace cvfes {

// One mesh of the batch as the kernels see it (type-agnostic pointers).
struct BatchMesh {
    const int32_t* node_ptr;
    const int4* rec;
    const void* slab;
    const void* fhat;
    const void* coef;
    const void* invm;
    void* buf[3];
    const double* p_sched;
    long long n_nodes;
    long long item_off;  // first work item of this mesh
    int S;
    int n_clamped;
    double clamp;
    double eta;
    double w0;
    int tpn;     // threads per node chunk
    int npb;     // nodes per block
    int chunks;  // sample chunks per node block (the last one may be partial)
    int form;    // 1: velocity-state form (buf[1] holds the increment), 0: u_{n-1} in buf
    int damp_dof;  // 1: damping per dof (eta = dt damp / m per row), 0: mass-proportional
    // fan kernel layout: items of kBatchWarps warps, f_npw nodes per warp
    long long f_off;  // first fan item of this mesh
    int f_tpn;        // lanes per node (min(32, S/VEC))
    int f_npw;        // nodes per warp (32 / f_tpn)
    int f_chunks;     // sample chunks per node block
    int max_deg;      // slots of the busiest node
    int* status;      // this mesh's device status word (bit 0: a bounded wait gave up)
};

constexpr int kBatchWarps = 2;

// Buffer roles of a mesh at rotation phase rot = (steps taken) % 6.  Previous-
// displacement form: u_n = buf[(3 - rot % 3) % 3], u_{n-1} the next one, u_{n+1} the
// one after.  Velocity-state form: the increment stays in buf[1] and u_n alternates
// between buf[0] (even phases) and buf[2] (odd phases).
__device__ __forceinline__ void batch_roles(const BatchMesh& M, int rot, int& cur, int& prev,
                                            int& nxt) {
    if (M.form) {
        cur = (rot & 1) ? 2 : 0;
        prev = 1;
        nxt = 2 - cur;
    } else {
        cur = (3 - rot % 3) % 3;
        prev = (cur + 1) % 3;
        nxt = (cur + 2) % 3;
    }
}

__device__ __forceinline__ int batch_mesh_of(const BatchMesh* __restrict__ tab, int n_meshes,
                                             long long w, bool fan) {
    int lo = 0, hi = n_meshes - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const long long off = fan ? __ldg(&tab[mid].f_off) : __ldg(&tab[mid].item_off);
        if (off <= w) lo = mid; else hi = mid - 1;
    }
    return lo;
}

template <typename T, int V, bool DIFF>
__global__ void __launch_bounds__(256) k_step_batched(const BatchMesh* __restrict__ tab,
                                                     int n_meshes, long long total, int rot,
                                                     const long long* clock, long long j) {
    const long long base = clock ? clock[0] : 0LL;
    for (long long w = blockIdx.x; w < total; w += gridDim.x) {
        const BatchMesh& M = tab[batch_mesh_of(tab, n_meshes, w, false)];
        int cur, prev, nxt;
        batch_roles(M, rot, cur, prev, nxt);
        const long long local = w - M.item_off;
        const long long nb = local / M.chunks;
        const int chunk = (int)(local - nb * M.chunks);
        const int t = threadIdx.x / M.tpn;
        if (t >= M.npb) continue;
        const long long a = nb * M.npb + t;
        if (a >= M.n_nodes) continue;
        const int vec = chunk * M.tpn + (threadIdx.x - t * M.tpn);
        if (vec * V >= M.S) continue;  // last chunk of S/V not a multiple of 32
        StepArgs<T> A;
        A.node_ptr = M.node_ptr;
        A.rec = M.rec;
        A.slab = static_cast<const T*>(M.slab);
        A.fhat = static_cast<const T*>(M.fhat);
        A.coef = static_cast<const T*>(M.coef);
        A.invm = static_cast<const T*>(M.invm);
        A.u = static_cast<const T*>(M.buf[cur]);
        A.up = static_cast<const T*>(M.buf[prev]);
        A.un = static_cast<T*>(M.buf[nxt]);
        A.vel = M.form ? static_cast<T*>(M.buf[prev]) : nullptr;
        A.trac = nullptr;
        A.p_sched = M.p_sched;
        A.clock = nullptr;
        A.j = base + j;
        A.pressure = 0.0;
        A.n_nodes = M.n_nodes;
        A.S = M.S;
        A.n_clamped = M.n_clamped;
        A.clamp = (T)M.clamp;
        A.eta = (T)M.eta;
        A.w0 = (T)M.w0;
        A.damp_per_dof = M.damp_dof;
        const size_t S = (size_t)M.S;
        const size_t col = (size_t)vec * V;
        const size_t row = (size_t)a * 3 * S + col;
        if (a < M.n_clamped) {
            clamp_store<T, V>(A, S, row);
            continue;
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
}


// Stage the slot records and stiffness rows of fan item w into (srec, sslab); returns the
// item's mesh.
template <typename T>
__device__ __forceinline__ int batch_fan_issue(const BatchMesh* __restrict__ tab, int n_meshes,
                                               long long w, int cap, uint32_t bar, int4* srec,
                                               T* sslab) {
    const int m = batch_mesh_of(tab, n_meshes, w, true);
    const BatchMesh& M = tab[m];
    const long long nb = (w - M.f_off) / M.f_chunks;
    const long long a0 = nb * (long long)(kBatchWarps * M.f_npw);
    long long a1 = a0 + kBatchWarps * M.f_npw;
    if (a1 > M.n_nodes) a1 = M.n_nodes;
    const int kb = __ldg(M.node_ptr + a0), ke = __ldg(M.node_ptr + a1);
    const int nsl = ke - kb;
    if (nsl <= 0 || nsl > cap) {
        mbar_arrive_expect_tx(bar, 0);
        return m;
    }
    const uint32_t b_rec = (uint32_t)nsl * 16u;
    const uint32_t b_slab = (uint32_t)nsl * (uint32_t)(kSlabStride * sizeof(T));
    mbar_arrive_expect_tx(bar, b_rec + b_slab);
    bulk_g2s(smem_u32(srec), M.rec + kb, b_rec, bar);
    bulk_g2s(smem_u32(sslab), static_cast<const T*>(M.slab) + (size_t)kb * kSlabStride, b_slab,
             bar);
    return m;
}

template <typename T, int V, bool DIFF, int MINB>
__global__ void __launch_bounds__(32 * kBatchWarps, MINB)
    k_batch_fan(const BatchMesh* __restrict__ tab, int n_meshes, long long total, int cap,
                int rot, const long long* clock, long long j) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const long long base = clock ? clock[0] : 0LL;
    const size_t stage_bytes = (size_t)cap * (16 + kSlabStride * sizeof(T));
    // stage q: barrier at smem + 8q, records then stiffness rows at smem + 16 + q * stage_bytes
    const uint32_t bar0 = smem_u32(smem);
    int4* const srec0 = reinterpret_cast<int4*>(smem + 16);
    T* const sslab0 = reinterpret_cast<T*>(smem + 16 + (size_t)cap * 16);
    // the mesh of the item in each stage, found by thread 0 when it issues the item's copies
    // (one binary search per item instead of one per thread)
    __shared__ int smesh[2];
    if (threadIdx.x == 0) {
        mbar_init(bar0, 1);
        mbar_init(bar0 + 8, 1);
    }
    __syncthreads();
    long long w = blockIdx.x;
    if (threadIdx.x == 0 && w < total)
        smesh[0] = batch_fan_issue<T>(tab, n_meshes, w, cap, bar0, srec0, sslab0);
    __syncthreads();
    for (int it = 0; w < total; w += gridDim.x, ++it) {
        const int sg = it & 1;
        const long long wn = w + gridDim.x;
        if (threadIdx.x == 0 && wn < total)
            smesh[sg ^ 1] = batch_fan_issue<T>(tab, n_meshes, wn, cap, bar0 + 8 * (sg ^ 1), stage_rec(srec0, stage_bytes, sg ^ 1), stage_slab(sslab0, stage_bytes, sg ^ 1));
        const BatchMesh& M = tab[smesh[sg]];
        int cur, prev, nxt;
        batch_roles(M, rot, cur, prev, nxt);
        const long long local = w - M.f_off;
        const long long nb = local / M.f_chunks;
        const int chunk = (int)(local - nb * M.f_chunks);
        const long long a0 = nb * (long long)(kBatchWarps * M.f_npw);
        const int sub = lane / M.f_tpn, l = lane - sub * M.f_tpn;
        const long long a = a0 + (long long)warp * M.f_npw + sub;
        const int vec = chunk * M.f_tpn + l;
        const bool active = sub < M.f_npw && a < M.n_nodes && vec * V < M.S;
        StepArgs<T> A;
        A.node_ptr = M.node_ptr;
        A.rec = M.rec;
        A.slab = static_cast<const T*>(M.slab);
        A.fhat = static_cast<const T*>(M.fhat);
        A.coef = static_cast<const T*>(M.coef);
        A.invm = static_cast<const T*>(M.invm);
        A.u = static_cast<const T*>(M.buf[cur]);
        A.up = static_cast<const T*>(M.buf[prev]);
        A.un = static_cast<T*>(M.buf[nxt]);
        A.vel = M.form ? static_cast<T*>(M.buf[prev]) : nullptr;
        A.trac = nullptr;
        A.p_sched = M.p_sched;
        A.clock = nullptr;
        A.j = base + j;
        A.pressure = 0.0;
        A.n_nodes = M.n_nodes;
        A.S = M.S;
        A.n_clamped = M.n_clamped;
        A.clamp = (T)M.clamp;
        A.eta = (T)M.eta;
        A.w0 = (T)M.w0;
        A.damp_per_dof = M.damp_dof;
        const size_t S = (size_t)M.S;
        const size_t col = (size_t)vec * V;
        const size_t row = (size_t)a * 3 * S + col;
        const bool clamped = a < M.n_clamped;
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
        if (!mbar_wait_bounded(bar0 + 8 * sg, (uint32_t)((it >> 1) & 1), kMaxPolls)) {
            if (lane == 0 && M.status) atomicOr(M.status, 1);
            return;
        }
        if (active) {
            if (clamped) {
                clamp_store<T, V>(A, S, row);
            } else {
                const int kb = __ldg(M.node_ptr + a0);
                const int k0 = __ldg(M.node_ptr + a) - kb, k1 = __ldg(M.node_ptr + a + 1) - kb;
                Vec<T, V> acc[3];
                ku_row_fan<T, V, DIFF>(stage_rec(srec0, stage_bytes, sg),
                                       stage_slab(sslab0, stage_bytes, sg), k0, k1, A.u, A.coef,
                                       S, col, ua, acc);
                step_epilogue<T, V>(A, a, S, col, row, ua, acc, f);
            }
        }
        __syncthreads();
    }
}

__global__ void k_batch_clock_add(long long* clock, long long n) { clock[0] += n; }

template <typename T>
int launch_batched(const BatchMesh* tab, int n_meshes, long long total, int vec, int rot,
                   const long long* clock, long long j, int grid, cudaStream_t st) {
    constexpr bool DIFF = std::is_same<T, float>::value;
    if (total <= 0) return CVFES_OK;
    if (grid <= 0 || grid > total) grid = (int)(total < (1LL << 30) ? total : (1 << 30));
    if (vec == 4) {
        if constexpr (sizeof(T) == 4)
            k_step_batched<T, 4, DIFF><<<grid, 256, 0, st>>>(tab, n_meshes, total, rot, clock, j);
    } else if (vec == 2) {
        k_step_batched<T, 2, DIFF><<<grid, 256, 0, st>>>(tab, n_meshes, total, rot, clock, j);
    } else {
        k_step_batched<T, 1, DIFF><<<grid, 256, 0, st>>>(tab, n_meshes, total, rot, clock, j);
    }
    CVFES_LAUNCH_CHECK("k_step_batched");
    return CVFES_OK;
}

inline int batch_sm_count() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 148;
    return n > 0 ? n : 148;
}

template <typename K>
int launch_batch_fan_k(K kernel, const BatchMesh* tab, int n_meshes, long long total, int cap,
                       int rot, const long long* clock, long long j, int grid, size_t smem,
                       cudaStream_t st) {
    if (smem > 48 * 1024) {
        cudaError_t e =
            cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess)
            return fail(CVFES_ERR_CUDA, "k_batch_fan smem attribute: %s", cudaGetErrorString(e));
    }
    if (grid <= 0) {
        int per_sm = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 32 * kBatchWarps, smem) !=
                cudaSuccess ||
            per_sm <= 0)
            return fail(CVFES_ERR_CUDA, "k_batch_fan: no resident block fits");
        grid = per_sm * batch_sm_count();
    }
    if (grid > total) grid = (int)total;
    kernel<<<grid, 32 * kBatchWarps, smem, st>>>(tab, n_meshes, total, cap, rot, clock, j);
    CVFES_LAUNCH_CHECK("k_batch_fan");
    return CVFES_OK;
}

template <typename T>
int launch_batch_fan(const BatchMesh* tab, int n_meshes, long long total, int cap, int vec,
                     int rot, const long long* clock, long long j, int grid, cudaStream_t st) {
    constexpr bool DIFF = std::is_same<T, float>::value;
    if (total <= 0) return CVFES_OK;
    const size_t smem = 16 + 2 * (size_t)cap * (16 + kSlabStride * sizeof(T));
    if (cap <= 0 || smem > 200 * 1024)
        return fail(CVFES_ERR_UNSUPPORTED, "cvfes_batch_step: fan stage of %d slots does not fit",
                    cap);
    if (vec == 4) {
        if constexpr (sizeof(T) == 4)
            return launch_batch_fan_k(k_batch_fan<T, 4, DIFF, 8>, tab, n_meshes, total, cap, rot,
                                      clock, j, grid, smem, st);
        return fail(CVFES_ERR_ARG, "cvfes_batch_step: vec 4 is FP32 only");
    }
    if (vec == 2)
        return launch_batch_fan_k(k_batch_fan<T, 2, DIFF, 8>, tab, n_meshes, total, cap, rot, clock,
                                  j, grid, smem, st);
    return launch_batch_fan_k(k_batch_fan<T, 1, DIFF, 8>, tab, n_meshes, total, cap, rot, clock, j,
                              grid, smem, st);
}

}  // namespace cvfes

using namespace cvfes;

extern "C" int64_t cvfes_batch_table_bytes(int32_t n_meshes) {
    return n_meshes > 0 ? (int64_t)n_meshes * (int64_t)sizeof(BatchMesh) : 0;
}

extern "C" int cvfes_batch_pack(const cvfes_batch_item* items, int32_t n_meshes,
                                int32_t precision, int32_t vec, void* table_dev,
                                int64_t* totals) {
    if (!items || n_meshes <= 0 || !table_dev || !totals)
        return fail(CVFES_ERR_ARG, "cvfes_batch_pack: bad argument");
    if (precision != 32 && precision != 64)
        return fail(CVFES_ERR_ARG, "cvfes_batch_pack: precision must be 32 or 64");
    const int maxv = precision == 32 ? 4 : 2;
    if (vec < 1 || vec > maxv || (vec & (vec - 1)))
        return fail(CVFES_ERR_ARG, "cvfes_batch_pack: vec %d not allowed", vec);
    const size_t tsz = precision == 32 ? 4 : 8;
    std::vector<BatchMesh> h(n_meshes);
    long long off = 0, f_off = 0, cap = 0;
    for (int m = 0; m < n_meshes; ++m) {
        const cvfes_batch_item& it = items[m];
        const cvfes_solid_mesh& ms = it.mesh;
        if (ms.n_nodes <= 0 || ms.n_samples <= 0 || ms.n_samples > INT32_MAX || !ms.node_ptr ||
            !ms.slot_rec || !ms.slot_k || !ms.fhat || !it.coef || !it.invm || !it.buf[0] ||
            !it.buf[1] || !it.buf[2])
            return fail(CVFES_ERR_ARG, "cvfes_batch_pack: incomplete mesh %d", m);
        if (ms.n_clamped < 0 || ms.n_clamped > ms.n_nodes)
            return fail(CVFES_ERR_ARG, "cvfes_batch_pack: mesh %d clamped rows", m);
        if (ms.n_samples % vec)
            return fail(CVFES_ERR_ARG,
                        "cvfes_batch_pack: mesh %d has %lld samples, not a multiple of vec %d", m,
                        (long long)ms.n_samples, vec);
        if (!(it.dt > 0.0)) return fail(CVFES_ERR_ARG, "cvfes_batch_pack: mesh %d dt <= 0", m);
        const void* ptrs[5] = {it.coef, it.invm, it.buf[0], it.buf[1], it.buf[2]};
        for (int q = 0; q < 5; ++q)
            if (reinterpret_cast<uintptr_t>(ptrs[q]) % (vec * tsz))
                return fail(CVFES_ERR_ARG, "cvfes_batch_pack: mesh %d buffer %d misaligned", m,
                            q);
        BatchMesh& b = h[m];
        b.node_ptr = ms.node_ptr;
        b.rec = reinterpret_cast<const int4*>(ms.slot_rec);
        b.slab = ms.slot_k;
        b.fhat = ms.fhat;
        b.coef = it.coef;
        b.invm = it.invm;
        for (int q = 0; q < 3; ++q) b.buf[q] = it.buf[q];
        b.p_sched = it.p_sched;
        b.n_nodes = ms.n_nodes;
        b.S = (int)ms.n_samples;
        b.n_clamped = (int)ms.n_clamped;
        b.clamp = ms.clamp_value;
        const double g = 0.5 * it.dt * it.damp;
        if (ms.damping_form != 0 && ms.damping_form != 1)
            return fail(CVFES_ERR_ARG, "cvfes_batch_pack: mesh %d damping_form", m);
        b.damp_dof = ms.damping_form;
        b.eta = b.damp_dof ? it.dt * it.damp : it.dt * it.damp / (1.0 + g);
        b.w0 = b.damp_dof ? it.dt * it.dt : it.dt * it.dt / (1.0 + g);
        const int sv = (int)(ms.n_samples / vec);
        b.tpn = sv < 32 ? sv : 32;
        b.npb = 256 / b.tpn;
        b.chunks = (sv + b.tpn - 1) / b.tpn;
        if (ms.state_form != 0 && ms.state_form != 1)
            return fail(CVFES_ERR_ARG, "cvfes_batch_pack: mesh %d state_form", m);
        b.form = ms.state_form;
        b.item_off = off;
        off += ((ms.n_nodes + b.npb - 1) / b.npb) * b.chunks;
        b.f_tpn = sv < 32 ? sv : 32;
        b.f_npw = 32 / b.f_tpn;
        b.f_chunks = (sv + b.f_tpn - 1) / b.f_tpn;
        b.max_deg = (int)ms.max_degree;
        b.status = ms.status;
        b.f_off = f_off;
        const long long nodes_per_item = (long long)kBatchWarps * b.f_npw;
        f_off += ((ms.n_nodes + nodes_per_item - 1) / nodes_per_item) * b.f_chunks;
        const long long c = ms.max_degree > 0 ? nodes_per_item * ms.max_degree : -1;
        if (c < 0 || cap < 0) cap = -1;
        else if (c > cap) cap = c;
    }
    totals[0] = off;
    totals[1] = f_off;
    totals[2] = cap;
    CVFES_CUDA_TRY(cudaMemcpy(table_dev, h.data(), h.size() * sizeof(BatchMesh),
                              cudaMemcpyHostToDevice));
    return CVFES_OK;
}

extern "C" int cvfes_batch_step(const void* table_dev, int32_t n_meshes, const int64_t* totals,
                                int32_t precision, int32_t vec, int32_t variant, int32_t rot,
                                const int64_t* clock, int64_t j, int32_t grid, void* stream) {
    if (!table_dev || n_meshes <= 0 || !totals || rot < 0 || rot > 5 ||
        (precision != 32 && precision != 64) || (vec != 1 && vec != 2 && vec != 4) ||
        (precision == 64 && vec == 4) || (variant != 0 && variant != 1))
        return fail(CVFES_ERR_ARG, "cvfes_batch_step: bad argument");
    const auto* tab = static_cast<const BatchMesh*>(table_dev);
    const auto* clk = reinterpret_cast<const long long*>(clock);
    if (variant == 1) {
        if (totals[2] <= 0 || totals[2] > INT32_MAX)
            return fail(CVFES_ERR_UNSUPPORTED,
                        "cvfes_batch_step: the fan kernel needs every mesh's max_degree");
        if (precision == 32)
            return launch_batch_fan<float>(tab, n_meshes, totals[1], (int)totals[2], vec, rot, clk,
                                           j, grid, (cudaStream_t)stream);
        return launch_batch_fan<double>(tab, n_meshes, totals[1], (int)totals[2], vec, rot, clk, j,
                                        grid, (cudaStream_t)stream);
    }
    if (precision == 32)
        return launch_batched<float>(tab, n_meshes, totals[0], vec, rot, clk, j, grid,
                                     (cudaStream_t)stream);
    return launch_batched<double>(tab, n_meshes, totals[0], vec, rot, clk, j, grid,
                                  (cudaStream_t)stream);
}

extern "C" int cvfes_batch_advance(const void* table_dev, int32_t n_meshes,
                                   const int64_t* totals, int32_t precision, int32_t vec,
                                   int32_t variant, int32_t rot0, int64_t* clock, int64_t n_steps,
                                   int32_t grid, int32_t* rot_out, void* stream) {
    if (n_steps < 0 || rot0 < 0 || rot0 > 5)
        return fail(CVFES_ERR_ARG, "cvfes_batch_advance: bad argument");
    int rot = rot0;
    for (long long k = 0; k < n_steps; ++k) {
        int rc = cvfes_batch_step(table_dev, n_meshes, totals, precision, vec, variant, rot,
                                  clock, k, grid, stream);
        if (rc) return rc;
        rot = (rot + 1) % 6;
    }
    if (clock && n_steps > 0) {
        k_batch_clock_add<<<1, 1, 0, (cudaStream_t)stream>>>(reinterpret_cast<long long*>(clock),
                                                             n_steps);
        CVFES_LAUNCH_CHECK("k_batch_clock_add");
    }
    if (rot_out) *rot_out = rot;
    return CVFES_OK;
}

extern "C" int cvfes_batch_graph_capture(const void* table_dev, int32_t n_meshes,
                                         const int64_t* totals, int32_t precision, int32_t vec,
                                         int32_t variant, int64_t* clock, int64_t chunk,
                                         int32_t grid, cvfes_graph** out) {
    if (!out || chunk <= 0 || chunk % 6 || !clock)
        return fail(CVFES_ERR_ARG,
                    "cvfes_batch_graph_capture: chunk must be a positive multiple of 6 and a "
                    "clock is required");
    cudaStream_t cs;
    CVFES_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) {
        cudaStreamDestroy(cs);
        return fail(CVFES_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e));
    }
    int rot_end = 0;
    const int rc = cvfes_batch_advance(table_dev, n_meshes, totals, precision, vec, variant, 0,
                                       clock, chunk, grid, &rot_end, cs);
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
    *out = new cvfes_graph{graph, exec};
    return CVFES_OK;
}
