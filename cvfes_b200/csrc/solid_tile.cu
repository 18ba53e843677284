// TMA-tiled membrane solid step (step tuning variant 7).
//
// The row-gather kernels are latency-bound: every element of a node issues its own
// global loads of neighbour rows and of the element's coefficient row.  Here a block
// owns one strip of P consecutive nodes (one warp per node) and one chunk of 32*VEC
// samples, and before multiplying it stages, with one 2D TMA tensor copy each, the few
// windows of consecutive node ids that hold every neighbour of the strip (3 dof rows
// per node) and the windows of element ids that hold the strip's coefficient rows,
// plus the strip's slot records and stiffness rows (1D bulk copies).  The windows come
// from the host tiling (cvfes_mesh_tiles): node numbering runs ring by ring on a tube,
// so a strip's neighbours fall in about three windows of P + 2 ids.  The products then
// read shared memory; the rare ids outside the windows read global memory.  Blocks
// are persistent and keep a ring of STAGES shared-memory stages, so the copies of the
// next items are in flight while the current one is multiplied; warps release each
// stage on their own (no block barrier).  The arithmetic is the
// fan kernel's, element by element in the same order, so the results are bitwise the
// same.
#include <cuda.h>  // CUtensorMap types; the encoder is taken from the runtime's driver entry point
#include <cuda_runtime.h>

#include <mutex>
#include <type_traits>

#include "common.cuh"
#include "step_core.cuh"

namespace cvfes {

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
    static std::once_flag once;
    static EncodeTiledFn fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// Tensor map of a row-major [rows][cols] array of T, copied in boxes of
// box_rows x box_cols; rows past the end read as zeros.
template <typename T>
bool make_map(CUtensorMap* map, const void* base, long long rows, long long cols, int box_cols,
              int box_rows) {
    EncodeTiledFn fn = encode_tiled();
    if (!fn) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)cols * sizeof(T)};
    const cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
    const cuuint32_t es[2] = {1, 1};
    const CUtensorMapDataType dt =
        sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
    return fn(map, dt, 2, const_cast<void*>(base), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// 2D tiled TMA load global -> this CTA's shared memory (no multicast).
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

struct TileArgs {
    const int32_t* win;       // [n_tiles][W + WE] window starts
    const int4* trec;         // [n_slots] shared-memory rows of each slot
    const int32_t* node_loc;  // [n_nodes]
    long long n_items;        // tiles * sample chunks
    int P, H, W, EH, WE, nch, cap;
    int coef_off, rec_off, slab_off, stage_bytes;
};

template <typename T, int C>
__device__ __forceinline__ void tile_issue(const StepArgs<T>& A, const TileArgs& TA,
                                           const CUtensorMap* mu, const CUtensorMap* mc,
                                           long long w, uint32_t bar, unsigned char* stage) {
    const long long t = w / TA.nch;
    const int x = (int)(w - t * TA.nch) * C;
    const int nw = TA.W + TA.WE;
    const int32_t* win = TA.win + t * nw;
    const long long a0 = t * TA.P;
    const long long a1 = (a0 + TA.P < A.n_nodes) ? a0 + TA.P : A.n_nodes;
    const int kb = __ldg(A.node_ptr + a0), ke = __ldg(A.node_ptr + a1);
    int nsl = ke - kb;
    if (nsl > TA.cap) {
        if (A.status) atomicOr(A.status, 2);
        nsl = 0;
    }
    const uint32_t ubox = (uint32_t)(3 * TA.H * C * sizeof(T));
    const uint32_t cbox = (uint32_t)(TA.EH * C * sizeof(T));
    uint32_t bytes = (uint32_t)nsl * (16u + (uint32_t)(kSlabStride * sizeof(T)));
    for (int k = 0; k < TA.W; ++k)
        if (__ldg(win + k) >= 0) bytes += ubox;
    for (int k = 0; k < TA.WE; ++k)
        if (__ldg(win + TA.W + k) >= 0) bytes += cbox;
    mbar_arrive_expect_tx(bar, bytes);
    const uint32_t s0 = smem_u32(stage);
    for (int k = 0; k < TA.W; ++k) {
        const int s = __ldg(win + k);
        if (s >= 0) tma_load_2d(s0 + k * ubox, mu, x, 3 * s, bar);
    }
    for (int k = 0; k < TA.WE; ++k) {
        const int s = __ldg(win + TA.W + k);
        if (s >= 0) tma_load_2d(s0 + TA.coef_off + k * cbox, mc, x, s, bar);
    }
    if (nsl > 0) {
        bulk_g2s(s0 + TA.rec_off, TA.trec + kb, (uint32_t)nsl * 16u, bar);
        bulk_g2s(s0 + TA.slab_off, A.slab + (size_t)kb * kSlabStride,
                 (uint32_t)nsl * (uint32_t)(kSlabStride * sizeof(T)), bar);
    }
}

template <typename T, int V>
__device__ __forceinline__ Vec<T, V> lds_row(const T* p) {
    return *reinterpret_cast<const Vec<T, V>*>(p);
}

// Rows of node `loc` (a shared-memory row when >= 0, else global node -1 - loc).
template <typename T, int V, int C>
__device__ __forceinline__ void tile_node(Vec<T, V> (&x)[3], const T* su, int loc,
                                          const T* __restrict__ u, size_t S, size_t col, int lv) {
    if (loc >= 0) {
#pragma unroll
        for (int d = 0; d < 3; ++d) x[d] = lds_row<T, V>(su + (size_t)(3 * loc + d) * C + lv);
    } else {
        const T* p = u + (size_t)(-1 - loc) * 3 * S + col;
#pragma unroll
        for (int d = 0; d < 3; ++d) x[d] = ldg<T, V>(p + d * S);
    }
}

// u_{n-1} rows, inverse mass and nodal load of this warp's node in work item w
// (zeros when the warp has no unclamped node there).
template <typename T, int V, int C>
__device__ __forceinline__ void tile_epi_load(const StepArgs<T>& A, const TileArgs& TA,
                                              long long w, int warp, int lv, T p,
                                              Vec<T, V> (&up)[3], Vec<T, V>& im, T (&f)[3]) {
    const long long t = w / TA.nch;
    const long long a = t * TA.P + warp;
    if (w < TA.n_items && warp < TA.P && a < A.n_nodes && a >= A.n_clamped) {
        const size_t S = (size_t)A.S;
        const size_t col = (size_t)(w - t * TA.nch) * C + lv;
        const size_t row = (size_t)a * 3 * S + col;
#pragma unroll
        for (int d = 0; d < 3; ++d) up[d] = ldcs<T, V>(A.up + row + d * S);
        im = ldcs<T, V>(A.invm + (size_t)a * S + col);
        node_load<T>(A, a, p, f);
    } else {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            up[d] = vzero<T, V>();
            f[d] = T(0);
        }
        im = vzero<T, V>();
    }
}

// Warps 0..P-1 each own one node of the strip.  Thread 0 also stages: at item i it
// refills the stage of item i-1 with item i+STAGES-1 (a block barrier ends every item).
// A variant where warps released stages one by one through "empty" barriers, and one
// with a separate staging warp, both measured slower on the 256x1024 tube.
template <typename T, int V, int STAGES>
__global__ void __launch_bounds__(512, 1)
    k_step_tile(StepArgs<T> A, TileArgs TA, const __grid_constant__ CUtensorMap mu,
                const __grid_constant__ CUtensorMap mc) {
    constexpr int C = 32 * V;
    constexpr bool DIFF = std::is_same<T, float>::value;
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const uint32_t full0 = smem_u32(smem);
    unsigned char* const st0 = smem + 128;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < STAGES; ++q) mbar_init(full0 + 8 * q, 1);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
        for (int q = 0; q < STAGES - 1; ++q) {
            const long long wq = blockIdx.x + (long long)q * gridDim.x;
            if (wq < TA.n_items)
                tile_issue<T, C>(A, TA, &mu, &mc, wq, full0 + 8 * q, st0 + q * TA.stage_bytes);
        }
    }
    const size_t S = (size_t)A.S;
    const T p = step_pressure<T>(A);
    const int lv = lane * V;
    long long w = blockIdx.x;
    // Epilogue operands (u_{n-1} rows, inverse mass, nodal load) of the item after the
    // current one are requested a whole item ahead, so their latency is hidden.
    Vec<T, V> upc[3], imc;
    T fc[3];
    tile_epi_load<T, V, C>(A, TA, w, warp, lv, p, upc, imc, fc);
    for (int it = 0; w < TA.n_items; w += gridDim.x, ++it) {
        const int sg = it % STAGES;
        if (threadIdx.x == 0) {
            const long long wn = w + (long long)(STAGES - 1) * gridDim.x;
            if (wn < TA.n_items) {
                const int q = (it + STAGES - 1) % STAGES;  // the stage of item it - 1
                tile_issue<T, C>(A, TA, &mu, &mc, wn, full0 + 8 * q, st0 + q * TA.stage_bytes);
            }
        }
        const long long t = w / TA.nch;
        const int chunk = (int)(w - t * TA.nch);
        const long long a0 = t * TA.P;
        const long long a = a0 + warp;
        const bool active = a < A.n_nodes;
        const size_t col = (size_t)chunk * C + lv;
        const size_t row = (size_t)a * 3 * S + col;
        const bool clamped = a < A.n_clamped;
        Vec<T, V> upn[3], imn;
        T fn[3];
        tile_epi_load<T, V, C>(A, TA, w + gridDim.x, warp, lv, p, upn, imn, fn);
        if (!mbar_wait_bounded(full0 + 8 * sg, (uint32_t)((it / STAGES) & 1), kMaxPolls)) {
            if (lane == 0 && A.status) atomicOr(A.status, 1);
            return;
        }
        if (active) {
            if (clamped) {
                const Vec<T, V> cl = vfill<T, V>(A.clamp);
#pragma unroll
                for (int d = 0; d < 3; ++d) stcs<T, V>(A.un + row + d * S, cl);
            } else {
                const unsigned char* sb = st0 + sg * TA.stage_bytes;
                const T* su = reinterpret_cast<const T*>(sb);
                const T* sc = reinterpret_cast<const T*>(sb + TA.coef_off);
                const int4* srec = reinterpret_cast<const int4*>(sb + TA.rec_off);
                const T* sslab = reinterpret_cast<const T*>(sb + TA.slab_off);
                Vec<T, V> ua[3];
                tile_node<T, V, C>(ua, su, __ldg(TA.node_loc + a), A.u, S, col, lv);
                const int kb = __ldg(A.node_ptr + a0);
                const int k0 = __ldg(A.node_ptr + a) - kb, k1 = __ldg(A.node_ptr + a + 1) - kb;
                Vec<T, V> acc[3];
#pragma unroll
                for (int d = 0; d < 3; ++d) acc[d] = vzero<T, V>();
                for (int k = k0; k < k1; ++k) {
                    const int4 r = srec[k];
                    Vec<T, V> d1[3], d2[3];
                    tile_node<T, V, C>(d1, su, r.y, A.u, S, col, lv);
                    tile_node<T, V, C>(d2, su, r.z, A.u, S, col, lv);
                    const Vec<T, V> c = r.x >= 0
                                            ? lds_row<T, V>(sc + (size_t)r.x * C + lv)
                                            : ldg<T, V>(A.coef + (size_t)(-1 - r.x) * S + col);
                    to_diff<T, V, DIFF>(d1, ua);
                    to_diff<T, V, DIFF>(d2, ua);
                    slot_fma<T, V, DIFF>(sslab + (size_t)kSlabStride * k, c, d1, d2, ua, acc);
                }
                step_update<T, V>(A, S, row, ua, acc, fc, upc, imc);
            }
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            upc[d] = upn[d];
            fc[d] = fn[d];
        }
        imc = imn;
        __syncthreads();  // every warp is done with this stage
    }
}

inline int align128(long long x) { return (int)((x + 127) / 128 * 128); }

template <typename T, int V, int STAGES>
int launch_tile_k(const StepArgs<T>& A, const TileArgs& TA, const CUtensorMap& mu,
                  const CUtensorMap& mc, size_t smem, cudaStream_t st) {
    auto kernel = k_step_tile<T, V, STAGES>;
    cudaError_t e =
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return fail(CVFES_ERR_CUDA, "k_step_tile smem attribute: %s", cudaGetErrorString(e));
    const int threads = 32 * TA.P;
    int per_sm = 0, dev = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) !=
            cudaSuccess ||
        per_sm <= 0)
        return fail(CVFES_ERR_CUDA, "k_step_tile: no resident block fits");
    CVFES_CUDA_TRY(cudaGetDevice(&dev));
    CVFES_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    long long blocks = (long long)per_sm * sms;
    if (blocks > TA.n_items) blocks = TA.n_items;
    kernel<<<(unsigned)blocks, threads, smem, st>>>(A, TA, mu, mc);
    CVFES_LAUNCH_CHECK("k_step_tile");
    return CVFES_OK;
}

constexpr size_t kTileMaxSmem = 227 * 1024;

template <typename T>
int launch_step_tile(const cvfes_solid_mesh* m, const StepArgs<T>& A, int vec_max,
                     cudaStream_t st) {
    // Not applicable (returns 1, no error recorded): no tiling, unsupported shape.
    if (!m->tile_win || !m->tile_rec || !m->node_loc || m->max_degree <= 0) return 1;
    const int P = m->tile_p, H = m->tile_h, W = m->tile_w, EH = m->tile_eh, WE = m->tile_we;
    if (P < 1 || P > 16 || W < 1 || W > 4 || WE < 1 || WE > 3 || 3 * H > 256 || EH > 256 ||
        H < P)
        return 1;
    int V = sizeof(T) == 4 ? 4 : 2;
    while (V > vec_max) V /= 2;
    const int C = 32 * V;
    if (A.S % C != 0 || (A.S * sizeof(T)) % 16 != 0) return 1;
    const void* ptrs[5] = {A.u, A.coef, A.up, A.invm, A.un};
    for (int i = 0; i < 5; ++i)
        if (reinterpret_cast<uintptr_t>(ptrs[i]) % 16) return 1;
    TileArgs TA;
    TA.win = m->tile_win;
    TA.trec = reinterpret_cast<const int4*>(m->tile_rec);
    TA.node_loc = m->node_loc;
    TA.P = P;
    TA.H = H;
    TA.W = W;
    TA.EH = EH;
    TA.WE = WE;
    TA.nch = A.S / C;
    TA.cap = (int)(P * m->max_degree);
    const long long n_tiles = (m->n_nodes + P - 1) / P;
    TA.n_items = n_tiles * TA.nch;
    const long long ubytes = (long long)W * 3 * H * C * sizeof(T);
    const long long cbytes = (long long)WE * EH * C * sizeof(T);
    TA.coef_off = align128(ubytes);
    TA.rec_off = TA.coef_off + align128(cbytes);
    TA.slab_off = TA.rec_off + align128((long long)TA.cap * 16);
    TA.stage_bytes = TA.slab_off + align128((long long)TA.cap * kSlabStride * sizeof(T));
    const int stages = (128 + 3 * (size_t)TA.stage_bytes <= kTileMaxSmem) ? 3 : 2;
    const size_t smem = 128 + (size_t)stages * TA.stage_bytes;
    if (smem > kTileMaxSmem) return 1;  // not even two stages fit: the fan kernel
    CUtensorMap mu, mc;
    if (!make_map<T>(&mu, A.u, 3 * m->n_nodes, A.S, C, 3 * H) ||
        !make_map<T>(&mc, A.coef, m->n_elems, A.S, C, EH))
        return 1;
    if (V == 4) {
        if constexpr (sizeof(T) == 4) {
            if (stages == 3) return launch_tile_k<T, 4, 3>(A, TA, mu, mc, smem, st);
            return launch_tile_k<T, 4, 2>(A, TA, mu, mc, smem, st);
        }
        return 1;
    }
    if (V == 2) {
        if (stages == 3) return launch_tile_k<T, 2, 3>(A, TA, mu, mc, smem, st);
        return launch_tile_k<T, 2, 2>(A, TA, mu, mc, smem, st);
    }
    if (stages == 3) return launch_tile_k<T, 1, 3>(A, TA, mu, mc, smem, st);
    return launch_tile_k<T, 1, 2>(A, TA, mu, mc, smem, st);
}

template int launch_step_tile<float>(const cvfes_solid_mesh*, const StepArgs<float>&, int,
                                     cudaStream_t);
template int launch_step_tile<double>(const cvfes_solid_mesh*, const StepArgs<double>&, int,
                                      cudaStream_t);

}  // namespace cvfes
