// Geometric-update ("updated coordinates") form of the membrane solid step.
//
// The stiffness and the follower pressure load of every element are taken on the
// deformed geometry x + u_g of each sample, as the reference's GPU kernel
// assemble_K_P does every step (physicsSolverSDampGPUs.cl:232-393) and its CPU path
// does every `stiffness_update_interval` steps (OptimizedSolidAssembleUpdate,
// optimizedSolidAssemble.pyx:710-819, triggered at physicsSolver.py:296-324):
//   K(x + u_g) u_n   and   p_n * sum_e (A_e / 3) n_e     over the deformed triangles.
// Nothing per sample is stored: the row of node a is formed matrix-free from the
// slot's reference edge vectors X_b - X_a (exact, precomputed) plus the neighbour
// displacement differences, so the FP32 form never subtracts large coordinates.
// Per slot and sample: the local frame (x along edge 1->2, y the Gram-Schmidt of
// edge 2->0, z = x cross y; unit vectors by rsqrt), the in-plane coordinates, the
// area, the 3x3 local blocks
// of B^T D B (membrane + transverse shear, D / (1 - nu^2)) of row a against its two
// neighbours applied to the neighbours' displacement differences in the local frame,
// and the result rotated back; rigid translations are in the null space, so the row
// only needs u_b - u_a.  The update of the state is the linear form's.
#include <cuda_runtime.h>

#include <type_traits>

#include "common.cuh"
#include "step_core.cuh"

namespace cvfes {

constexpr int kGeoStride = 8;  // X_b1 - X_a (3), X_b2 - X_a (3), pad (2)

// Reference edge vectors of every slot (a = the slot's own node).
__global__ void k_slot_geometry(long long n_slots, const double* __restrict__ nodes,
                                const int32_t* __restrict__ elems,
                                const int32_t* __restrict__ slot_rec, double* __restrict__ geo64,
                                float* __restrict__ geo32) {
    const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (s >= n_slots) return;
    const int e = slot_rec[4 * s], b1 = slot_rec[4 * s + 1], b2 = slot_rec[4 * s + 2];
    const int la = (slot_rec[4 * s + 3] >> 8) & 3;
    const int a = elems[3 * (size_t)e + la];
    double g[kGeoStride];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        g[d] = nodes[3 * (size_t)b1 + d] - nodes[3 * (size_t)a + d];
        g[3 + d] = nodes[3 * (size_t)b2 + d] - nodes[3 * (size_t)a + d];
    }
    g[6] = g[7] = 0.0;
#pragma unroll
    for (int q = 0; q < kGeoStride; ++q) {
        if (geo64) geo64[(size_t)kGeoStride * s + q] = g[q];
        if (geo32) geo32[(size_t)kGeoStride * s + q] = (float)g[q];
    }
}

template <typename T>
struct GeoConst {
    T pe0;  // nu
    T pe1;  // (1 - nu) / 2
    T pe2;  // k (1 - nu) / 2
    T pe3;  // 1 - nu^2
    T inv4pe3;  // 1 / (4 (1 - nu^2))
};

template <typename T>
__device__ __forceinline__ T sel3(int i, T x0, T x1, T x2) {
    return i == 0 ? x0 : (i == 1 ? x1 : x2);
}

// Row of node a (local index la) of c_e K_e(x + u_g) applied to the displacement
// differences (d1, d2) of its neighbours b1 = local (la+1)%3, b2 = local (la+2)%3,
// for one sample; q1, q2 are the deformed edge vectors from a.  Adds the row to acc
// and (A/3) n to load.
template <typename T>
__device__ __forceinline__ void geo_row(int la, const T (&q1)[3], const T (&q2)[3],
                                        const T (&d1)[3], const T (&d2)[3], T c,
                                        const GeoConst<T>& K, T (&acc)[3], T (&load)[3]) {
    // positions of the element's nodes 0, 1, 2 relative to a
    const int l1 = la == 2 ? 0 : la + 1;  // local index of b1
    T P[3][3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const T z = T(0);
        // node k is a (la), b1 (l1) or b2 (the remaining one)
        P[0][d] = la == 0 ? z : (l1 == 0 ? q1[d] : q2[d]);
        P[1][d] = la == 1 ? z : (l1 == 1 ? q1[d] : q2[d]);
        P[2][d] = la == 2 ? z : (l1 == 2 ? q1[d] : q2[d]);
    }
    // frame: x along P2 - P1, y Gram-Schmidt of P0 - P2, z = x cross y
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
    // in-plane coordinates, area and the strain-displacement coefficients
    T lx[3], ly[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        lx[k] = P[k][0] * ex[0] + P[k][1] * ex[1] + P[k][2] * ex[2];
        ly[k] = P[k][0] * ey[0] + P[k][1] * ey[1] + P[k][2] * ey[2];
    }
    const T area = T(0.5) * ((lx[1] * ly[2] - lx[2] * ly[1]) - (lx[0] * ly[2] - lx[2] * ly[0]) +
                             (lx[0] * ly[1] - lx[1] * ly[0]));
    const T b0 = ly[1] - ly[2], b1 = ly[2] - ly[0], b2 = ly[0] - ly[1];
    const T c0 = lx[2] - lx[1], c1 = lx[0] - lx[2], c2 = lx[1] - lx[0];
    const int l2 = 3 - la - l1;
    const T bi = sel3(la, b0, b1, b2), ci = sel3(la, c0, c1, c2);
    const T bj1 = sel3(l1, b0, b1, b2), cj1 = sel3(l1, c0, c1, c2);
    const T bj2 = sel3(l2, b0, b1, b2), cj2 = sel3(l2, c0, c1, c2);
    // neighbour differences in the local frame
    T w1[3], w2[3];
    w1[0] = ex[0] * d1[0] + ex[1] * d1[1] + ex[2] * d1[2];
    w1[1] = ey[0] * d1[0] + ey[1] * d1[1] + ey[2] * d1[2];
    w1[2] = ez[0] * d1[0] + ez[1] * d1[1] + ez[2] * d1[2];
    w2[0] = ex[0] * d2[0] + ex[1] * d2[1] + ex[2] * d2[2];
    w2[1] = ey[0] * d2[0] + ey[1] * d2[1] + ey[2] * d2[2];
    w2[2] = ez[0] * d2[0] + ez[1] * d2[1] + ez[2] * d2[2];
    // local blocks (i = a, j = b1 / b2) applied: 2x2 membrane part + transverse shear
    T r[3];
    {
        const T bb = bi * bj1, bc = bi * cj1, cb = ci * bj1, cc = ci * cj1;
        r[0] = (bb + cc * K.pe1) * w1[0] + (bc * K.pe0 + cb * K.pe1) * w1[1];
        r[1] = (cb * K.pe0 + bc * K.pe1) * w1[0] + (cc + bb * K.pe1) * w1[1];
        r[2] = (bb + cc) * K.pe2 * w1[2];
    }
    {
        const T bb = bi * bj2, bc = bi * cj2, cb = ci * bj2, cc = ci * cj2;
        r[0] += (bb + cc * K.pe1) * w2[0] + (bc * K.pe0 + cb * K.pe1) * w2[1];
        r[1] += (cb * K.pe0 + bc * K.pe1) * w2[0] + (cc + bb * K.pe1) * w2[1];
        r[2] += (bb + cc) * K.pe2 * w2[2];
    }
    const T scale = c * K.inv4pe3 / area;
    const T a3 = area * T(1.0 / 3.0);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        acc[d] += scale * (r[0] * ex[d] + r[1] * ey[d] + r[2] * ez[d]);
        load[d] += a3 * ez[d];
    }
}

template <typename T>
struct GeoArgs {
    const T* geo;  // [kGeoStride * n_slots] reference edge vectors
    const T* ug;   // geometry displacement (== the step's u when the geometry is current)
    GeoConst<T> K;
};

// Everything one slot needs: neighbour differences of u_n (and of u_g when it is a
// different state), the coefficient row, the reference edge vectors, a's local index.
template <typename T, int V, bool SAME>
struct GeoSlot {
    Vec<T, V> x1[3], x2[3];
    Vec<T, V> g1[SAME ? 1 : 3], g2[SAME ? 1 : 3];
    Vec<T, V> c;
    T e1[3], e2[3];
    int la;
};

template <typename T, int V, bool SAME>
__device__ __forceinline__ void geo_slot_load(GeoSlot<T, V, SAME>& g, const StepArgs<T>& A,
                                              const GeoArgs<T>& G, int k, size_t S, size_t col,
                                              const Vec<T, V> (&ua)[3], const Vec<T, V> (&ga)[3]) {
    const int4 r = __ldg(A.rec + k);
    g.la = (r.w >> 8) & 3;
    const size_t o1 = (size_t)r.y * 3 * S + col, o2 = (size_t)r.z * 3 * S + col;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        g.x1[d] = vsub(ldg<T, V>(A.u + o1 + d * S), ua[d]);
        g.x2[d] = vsub(ldg<T, V>(A.u + o2 + d * S), ua[d]);
        if constexpr (!SAME) {
            g.g1[d] = vsub(ldg<T, V>(G.ug + o1 + d * S), ga[d]);
            g.g2[d] = vsub(ldg<T, V>(G.ug + o2 + d * S), ga[d]);
        }
    }
    g.c = ldg<T, V>(A.coef + (size_t)r.x * S + col);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        g.e1[d] = __ldg(G.geo + (size_t)kGeoStride * k + d);
        g.e2[d] = __ldg(G.geo + (size_t)kGeoStride * k + 3 + d);
    }
}

// One step, rows through L1: per slot the neighbour rows of u_n (and of u_g when it
// is a different state), the coefficient row and the slot's edge vectors.
template <typename T, int V, bool SAME>
__global__ void __launch_bounds__(256) k_step_geo(StepArgs<T> A, GeoArgs<T> G) {
    long long a;
    int vec;
    if (!map_row(A.tpn, A.npb, A.n_nodes, A.S / V, a, vec)) return;
    const size_t S = (size_t)A.S;
    const size_t col = (size_t)vec * V;
    const size_t row = (size_t)a * 3 * S + col;
    if (a < A.n_clamped) {
        const Vec<T, V> cl = vfill<T, V>(A.clamp);
#pragma unroll
        for (int d = 0; d < 3; ++d) stcs<T, V>(A.un + row + d * S, cl);
        return;
    }
    Vec<T, V> ua[3], ga[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        ua[d] = ldg<T, V>(A.u + row + d * S);
        if constexpr (!SAME) ga[d] = ldg<T, V>(G.ug + row + d * S);
    }
    const T p = step_pressure<T>(A);
    T acc[V][3], load[V][3];
#pragma unroll
    for (int i = 0; i < V; ++i)
#pragma unroll
        for (int d = 0; d < 3; ++d) acc[i][d] = load[i][d] = T(0);
    const int k0 = __ldg(A.node_ptr + a), k1 = __ldg(A.node_ptr + a + 1);
    // The rows, coefficient and edge vectors of slot k+1 are requested before slot k is
    // formed (one slot of lookahead; the per-slot geometry hides their latency).
    GeoSlot<T, V, SAME> nx;
    if (k0 < k1) geo_slot_load<T, V, SAME>(nx, A, G, k0, S, col, ua, ga);
    for (int k = k0; k < k1; ++k) {
        const GeoSlot<T, V, SAME> cu = nx;
        if (k + 1 < k1) geo_slot_load<T, V, SAME>(nx, A, G, k + 1, S, col, ua, ga);
#pragma unroll
        for (int i = 0; i < V; ++i) {
            T q1[3], q2[3], d1[3], d2[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const T g1 = SAME ? cu.x1[d].v[i] : cu.g1[d].v[i];
                const T g2 = SAME ? cu.x2[d].v[i] : cu.g2[d].v[i];
                q1[d] = cu.e1[d] + g1;
                q2[d] = cu.e2[d] + g2;
                d1[d] = cu.x1[d].v[i];
                d2[d] = cu.x2[d].v[i];
            }
            geo_row<T>(cu.la, q1, q2, d1, d2, cu.c.v[i], G.K, acc[i], load[i]);
        }
    }
    const Vec<T, V> im = ldcs<T, V>(A.invm + (size_t)a * S + col);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const Vec<T, V> up = ldcs<T, V>(A.up + row + d * S);
        // nodal traction (calc_u_appTrac, physicsSolverSDampGPUs.cl:436-446), one per node
        const T tr = A.trac ? __ldg(A.trac + 4 * a + d) : T(0);
        Vec<T, V> o;
#pragma unroll
        for (int i = 0; i < V; ++i) {
            const T dv = ua[d].v[i] - up.v[i];
            const T w = A.w0 * im.v[i];
            T f = p * load[i][d];
            if (A.trac) f += tr;
            const T v = fma(w, f - acc[i][d], fma(-row_eta(A, im.v[i]), dv, dv));
            o.v[i] = (im.v[i] != T(0)) ? ua[d].v[i] + v : T(0);
        }
        stcs<T, V>(A.un + row + d * S, o);
    }
}

struct GeoTuning {
    int vec;    // samples per thread (upper bound)
    int block;  // threads per block (64, 128 or 256)
};
// Defaults from sweeps on the 256x1024 tube, 512 samples (B200).
static GeoTuning g_geo32 = {4, 128};
static GeoTuning g_geo64 = {1, 128};

template <typename T>
int launch_step_geo(const cvfes_solid_mesh* m, const T* coef, const T* invm, const T* geo,
                    const T* u, const T* up, T* un, const T* ug, const double* p_sched,
                    const long long* clock, long long j, double pressure, const T* trac,
                    double nu, double dt, double damp, cudaStream_t st) {
    if (!m || m->n_nodes <= 0 || m->n_samples <= 0 || m->n_samples > INT32_MAX || !m->node_ptr ||
        !m->slot_rec || m->n_clamped < 0 || m->n_clamped > m->n_nodes)
        return fail(CVFES_ERR_ARG, "cvfes_solid_step_geo: incomplete mesh descriptor");
    if (!coef || !invm || !geo || !u || !up || !un)
        return fail(CVFES_ERR_ARG, "cvfes_solid_step_geo: null pointer");
    if (!(dt > 0.0) || !(nu > -1.0 && nu < 0.5))
        return fail(CVFES_ERR_ARG, "cvfes_solid_step_geo: dt must be positive and nu in (-1, 0.5)");
    StepArgs<T> A{};
    A.node_ptr = m->node_ptr;
    A.rec = reinterpret_cast<const int4*>(m->slot_rec);
    A.coef = coef;
    A.invm = invm;
    A.u = u;
    A.up = up;
    A.un = un;
    A.p_sched = p_sched;
    A.clock = clock;
    A.j = j;
    A.pressure = pressure;
    A.trac = trac;
    A.n_nodes = m->n_nodes;
    A.S = (int)m->n_samples;
    A.n_clamped = (int)m->n_clamped;
    A.clamp = (T)m->clamp_value;
    const double g = 0.5 * dt * damp;
    if (m->damping_form == 1) {  // damping force per dof: eta = dt damp / m, no LHS term
        A.damp_per_dof = 1;
        A.eta = (T)(dt * damp);
        A.w0 = (T)(dt * dt);
    } else {
        A.eta = (T)(dt * damp / (1.0 + g));
        A.w0 = (T)(dt * dt / (1.0 + g));
    }
    A.status = m->status;
    GeoArgs<T> G;
    G.geo = geo;
    G.ug = ug ? ug : u;
    const double shear_k = 5.0 / 6.0;
    G.K.pe0 = (T)nu;
    G.K.pe1 = (T)(0.5 * (1.0 - nu));
    G.K.pe2 = (T)(0.5 * shear_k * (1.0 - nu));
    G.K.pe3 = (T)(1.0 - nu * nu);
    G.K.inv4pe3 = (T)(0.25 / (1.0 - nu * nu));
    const bool same = G.ug == u;
    const void* ptrs[6] = {coef, invm, u, up, un, G.ug};
    const GeoTuning& tu = sizeof(T) == 4 ? g_geo32 : g_geo64;
    int V = (int)(16 / sizeof(T));
    while (V > tu.vec) V /= 2;
    for (; V > 1; V /= 2) {
        bool ok = A.S % V == 0;
        for (int i = 0; i < 6; ++i)
            if (reinterpret_cast<uintptr_t>(ptrs[i]) % (V * sizeof(T))) ok = false;
        if (ok) break;
    }
    const int block = tu.block;
    const RowGrid rg = row_grid(m->n_nodes, A.S / V, block);
    A.tpn = rg.tpn;
    A.npb = rg.npb;
    if (V == 4) {
        if constexpr (sizeof(T) == 4) {
            if (same) k_step_geo<T, 4, true><<<rg.grid, block, 0, st>>>(A, G);
            else k_step_geo<T, 4, false><<<rg.grid, block, 0, st>>>(A, G);
        }
    } else if (V == 2) {
        if (same) k_step_geo<T, 2, true><<<rg.grid, block, 0, st>>>(A, G);
        else k_step_geo<T, 2, false><<<rg.grid, block, 0, st>>>(A, G);
    } else {
        if (same) k_step_geo<T, 1, true><<<rg.grid, block, 0, st>>>(A, G);
        else k_step_geo<T, 1, false><<<rg.grid, block, 0, st>>>(A, G);
    }
    CVFES_LAUNCH_CHECK("k_step_geo");
    return CVFES_OK;
}

__global__ void k_geo_clock_add(long long* clock, long long n) { clock[0] += n; }

// n_steps geometric steps with the reference's update counter: before each step, if
// counter >= interval the geometry becomes the current state (copied into ugeo, or
// read straight from u_n when interval == 1) and counter = 1, else counter += 1.
template <typename T>
int launch_advance_geo(const cvfes_solid_mesh* m, const T* coef, const T* invm, const T* geo,
                       T* b0, T* b1, T* b2, T* ugeo, const double* p_sched, long long* clock,
                       long long n_steps, long long interval, long long* counter, int geo_live,
                       double nu, double dt, double damp, int* cur_idx, int* prev_idx,
                       int* geo_live_out, cudaStream_t st) {
    if (n_steps < 0 || interval < 1 || !counter || !p_sched || !ugeo)
        return fail(CVFES_ERR_ARG, "cvfes_solid_advance_geo: bad argument");
    T* buf[3] = {b0, b1, b2};
    int cur = 0, prev = 1, nxt = 2;
    const size_t bytes = (size_t)3 * m->n_nodes * m->n_samples * sizeof(T);
    long long c = *counter;
    bool live = geo_live != 0;  // geometry is the current state (interval 1 after an update)
    for (long long j = 0; j < n_steps; ++j) {
        if (c >= interval) {
            if (interval == 1) {
                live = true;
            } else {
                CVFES_CUDA_TRY(cudaMemcpyAsync(ugeo, buf[cur], bytes, cudaMemcpyDeviceToDevice, st));
            }
            c = 1;
        } else {
            c += 1;
        }
        const T* ug = live ? buf[cur] : ugeo;
        int rc = launch_step_geo<T>(m, coef, invm, geo, buf[cur], buf[prev], buf[nxt], ug, p_sched,
                                    clock, j, 0.0, nullptr, nu, dt, damp, st);
        if (rc) return rc;
        const int old_prev = prev;
        prev = cur;
        cur = nxt;
        nxt = old_prev;
    }
    if (clock && n_steps > 0) {
        k_geo_clock_add<<<1, 1, 0, st>>>(clock, n_steps);
        CVFES_LAUNCH_CHECK("k_geo_clock_add");
    }
    *counter = c;
    if (cur_idx) *cur_idx = cur;
    if (prev_idx) *prev_idx = prev;
    if (geo_live_out) *geo_live_out = live ? 1 : 0;
    return CVFES_OK;
}

}  // namespace cvfes

using namespace cvfes;

extern "C" int cvfes_set_geo_tuning(int32_t precision, int32_t vec, int32_t block) {
    if ((precision != 32 && precision != 64) || (vec != 1 && vec != 2 && vec != 4) ||
        (precision == 64 && vec == 4) || (block != 64 && block != 128 && block != 256))
        return fail(CVFES_ERR_ARG, "cvfes_set_geo_tuning: bad argument");
    GeoTuning& t = precision == 32 ? g_geo32 : g_geo64;
    t = GeoTuning{vec, block};
    return CVFES_OK;
}

extern "C" int cvfes_get_geo_tuning(int32_t precision, int32_t* vec, int32_t* block) {
    if (precision != 32 && precision != 64)
        return fail(CVFES_ERR_ARG, "cvfes_get_geo_tuning: precision must be 32 or 64");
    const GeoTuning& t = precision == 32 ? g_geo32 : g_geo64;
    if (vec) *vec = t.vec;
    if (block) *block = t.block;
    return CVFES_OK;
}

extern "C" int cvfes_solid_slot_geometry_f64(int64_t n_elems, const double* nodes,
                                             const int32_t* elems, const int32_t* slot_rec,
                                             double* geo64, float* geo32, void* stream) {
    if (n_elems <= 0 || !nodes || !elems || !slot_rec || (!geo64 && !geo32))
        return fail(CVFES_ERR_ARG, "cvfes_solid_slot_geometry_f64: bad argument");
    const long long ns = 3 * n_elems;
    k_slot_geometry<<<grid_1d(ns, 256), 256, 0, (cudaStream_t)stream>>>(ns, nodes, elems, slot_rec,
                                                                         geo64, geo32);
    CVFES_LAUNCH_CHECK("k_slot_geometry");
    return CVFES_OK;
}

extern "C" int cvfes_solid_step_geo_f64(const cvfes_solid_mesh* mesh, const double* coef,
                                        const double* invm, const double* slot_geo,
                                        const double* u, const double* up, double* un,
                                        const double* ug, const double* p_sched,
                                        const int64_t* clock, int64_t j, double pressure,
                                        const double* trac, double nu, double dt, double damp,
                                        void* stream) {
    return launch_step_geo<double>(mesh, coef, invm, slot_geo, u, up, un, ug, p_sched,
                                   reinterpret_cast<const long long*>(clock), j, pressure, trac,
                                   nu, dt, damp, (cudaStream_t)stream);
}

extern "C" int cvfes_solid_step_geo_f32(const cvfes_solid_mesh* mesh, const float* coef,
                                        const float* invm, const float* slot_geo, const float* u,
                                        const float* up, float* un, const float* ug,
                                        const double* p_sched, const int64_t* clock, int64_t j,
                                        double pressure, const float* trac, double nu, double dt,
                                        double damp, void* stream) {
    return launch_step_geo<float>(mesh, coef, invm, slot_geo, u, up, un, ug, p_sched,
                                  reinterpret_cast<const long long*>(clock), j, pressure, trac,
                                  nu, dt, damp, (cudaStream_t)stream);
}

extern "C" int cvfes_solid_advance_geo_f64(const cvfes_solid_mesh* mesh, const double* coef,
                                           const double* invm, const double* slot_geo,
                                           double* buf0, double* buf1, double* buf2, double* ugeo,
                                           const double* p_sched, int64_t* clock, int64_t n_steps,
                                           int64_t interval, int64_t* counter, int32_t geo_live,
                                           double nu, double dt, double damp, int32_t* cur_idx,
                                           int32_t* prev_idx, int32_t* geo_live_out,
                                           void* stream) {
    long long c = counter ? *counter : 0;
    const int rc = launch_advance_geo<double>(
        mesh, coef, invm, slot_geo, buf0, buf1, buf2, ugeo, p_sched,
        reinterpret_cast<long long*>(clock), n_steps, interval, counter ? &c : nullptr, geo_live,
        nu, dt, damp, cur_idx, prev_idx, geo_live_out, (cudaStream_t)stream);
    if (!rc && counter) *counter = c;
    return rc;
}

extern "C" int cvfes_solid_advance_geo_f32(const cvfes_solid_mesh* mesh, const float* coef,
                                           const float* invm, const float* slot_geo, float* buf0,
                                           float* buf1, float* buf2, float* ugeo,
                                           const double* p_sched, int64_t* clock, int64_t n_steps,
                                           int64_t interval, int64_t* counter, int32_t geo_live,
                                           double nu, double dt, double damp, int32_t* cur_idx,
                                           int32_t* prev_idx, int32_t* geo_live_out,
                                           void* stream) {
    long long c = counter ? *counter : 0;
    const int rc = launch_advance_geo<float>(
        mesh, coef, invm, slot_geo, buf0, buf1, buf2, ugeo, p_sched,
        reinterpret_cast<long long*>(clock), n_steps, interval, counter ? &c : nullptr, geo_live,
        nu, dt, damp, cur_idx, prev_idx, geo_live_out, (cudaStream_t)stream);
    if (!rc && counter) *counter = c;
    return rc;
}
