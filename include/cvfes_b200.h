/*
 * cvfes_b200 — C ABI of the B200 ensemble membrane solid time step.
 *
 * Plain pointers, sizes and a cudaStream_t passed as void*.  Every pointer
 * documented as "device" must be device memory owned by the caller (the
 * Python host layer passes torch tensors); the library never allocates state.
 * Every function returns a status code (CVFES_OK == 0, negative on error) and
 * records a message readable through cvfes_last_error().
 *
 * Layout conventions (identical to the reference's GPU buffers, which are
 * (lclNDof, nSmp) C-order, sample innermost — physicsSolverSDampGPUs.py:188-269):
 *   state / load vectors   T[3*N][S]   (dof-major, sample innermost)
 *   per-element fields     T[E][S]
 *   per-node fields        T[N][S]
 *   Dirichlet rows         local nodes [0, n_clamped)   (boundary-first
 *                          numbering, meshPartition.py:240-254)
 *
 * Each entry point cites the reference interface it replaces.
 */
#ifndef CVFES_B200_H
#define CVFES_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CVFES_OK               0
#define CVFES_ERR_ARG         -1   /* invalid argument (size, null, layout)       */
#define CVFES_ERR_CUDA        -2   /* CUDA runtime error                          */
#define CVFES_ERR_NONFINITE   -3   /* watchdog saw NaN/Inf in the state           */
#define CVFES_ERR_TIMEOUT     -4   /* a bounded device wait gave up               */
#define CVFES_ERR_UNSUPPORTED -5   /* configuration not supported by this build   */
#define CVFES_ERR_MESH        -6   /* mesh preprocessing failed (e.g. colours)    */

/* Node-centric view of a membrane mesh, all arrays device-resident.
 * Slot k in [node_ptr[a], node_ptr[a+1]) is one element incident to node a.
 *   slot_rec[4k+0] element id e
 *   slot_rec[4k+1] first other node of e  (column block 1 of the slot rows)
 *   slot_rec[4k+2] second other node of e (column block 2)
 *   slot_rec[4k+3] bit0: block 1 equals block 2 of slot k-1 (fan order)
 *                  bits 8..9: local index of a inside e
 *   slot_k   [28k + 9q + 3i + j] = Kt_e[3*la+i][3*lb_q+j], q = 0 (a), 1, 2
 *                                  (unit-coefficient element stiffness rows)
 *   fhat     [4a + d]            unit-pressure nodal load, d < 3 (pad at 3)
 */
typedef struct cvfes_solid_mesh {
    int64_t        n_nodes;
    int64_t        n_elems;
    int64_t        n_samples;
    int64_t        n_clamped;
    double         clamp_value;   /* bdyU of ApplyBoundaryCondition */
    const int32_t* node_ptr;      /* [n_nodes + 1]    */
    const int32_t* slot_rec;      /* [4 * n_slots]    */
    const void*    slot_k;        /* [28 * n_slots] T */
    const void*    fhat;          /* [4 * n_nodes]  T */
    int64_t        max_degree;    /* max slots of one node (0: unknown -> no smem staging) */
    int32_t*       status;        /* device int32 or NULL: bit 0 set when a bounded
                                     device wait gave up (read by cvfes_status_read) */
    /* Strip tiling of the TMA-tiled step (staged = 7), from cvfes_mesh_tiles, device
     * arrays; tile_win NULL: no tiling (the tiled variant falls back to the fan).   */
    const int32_t* tile_win;      /* [n_tiles][tile_w + tile_we] window starts      */
    const int32_t* tile_rec;      /* [4 * n_slots] shared-memory rows of each slot  */
    const int32_t* node_loc;      /* [n_nodes] shared-memory row of each node       */
    int32_t        tile_p;        /* nodes per tile                                 */
    int32_t        tile_h;        /* node ids per node window                       */
    int32_t        tile_w;        /* node windows per tile (at most 4)              */
    int32_t        tile_eh;       /* element ids per element window                 */
    int32_t        tile_we;       /* element windows per tile (at most 3)           */
    int32_t        tile_pad;
    int64_t        bandwidth;     /* max |a - b| over the element edges between
                                     unclamped nodes (0: unknown; sets the automatic
                                     L2 prefetch distance of the fan step kernels) */
    int32_t        state_form;    /* what the second state buffer of the template step
                                     holds: 0 = u_{n-1} (the reference's pair of
                                     displacements), 1 = the increment v_n = u_n - u_{n-1},
                                     updated in place by each step (velocity-state form) */
    int32_t        damping_form;  /* 0 = mass-proportional damping LC = damp * LM and the
                                     left-hand side LM + dt/2 LC (SolidSolver,
                                     physicsSolver.py:263-292); 1 = damping force
                                     -damp (u - u_prev) / dt per dof and the left-hand
                                     side LM, with no damping in the start-up
                                     acceleration (the OpenCL class's calc_u and
                                     calc_ddu, physicsSolverSDampGPUs.cl:398-429) */
} cvfes_solid_mesh;

/* Step-kernel tuning (the autotuner sets these; defaults: variant 6 with 4 nodes per
 * block, vec 4 for FP32 and 2 for FP64; minb 2).
 *   precision 32 | 64;  vec: samples per thread (FP32 1|2|4, FP64 1|2);
 *   npb: nodes per block when a warp owns one node (1..8, one warp each);
 *   staged: 0 = slot records, stiffness rows and gathers read through L1;
 *           1 = slot records and stiffness rows staged in shared memory by a
 *               TMA bulk copy, gathers through registers (2 elements in flight);
 *           2 = as 1, and each warp copies its node's whole gather into shared
 *               memory with cp.async before multiplying;
 *           3 = as 1, with the fan's shared neighbour carried between elements
 *               (three-buffer rotation) and the sample chunk fastest in the grid;
 *           4 = persistent pipelined kernel: each warp streams its own work
 *               items through a ring of `minb` (2..4) shared-memory stages
 *               (rows by cp.async, slot rows by TMA); npb = warps per block;
 *           5 = as 1, with the node's whole gather (every neighbour row and
 *               coefficient row) requested before the first product (meshes of
 *               node degree <= 8; otherwise as 3);
 *           6 = as 3, persistent, the next work item's slot rows staged while the
 *               current one is multiplied (two shared-memory stages);
 *           7 = TMA-tiled: a block owns a strip of tile_p nodes and one sample chunk
 *               (64 FP32 / 32 FP64 samples); 2D TMA tensor copies stage the strip's
 *               node windows (all neighbour rows) and element windows (coefficient
 *               rows), with its slot rows, into a ring of shared-memory stages; the
 *               products read shared memory (ids outside the windows read global
 *               memory).  Needs the mesh's tiling (cvfes_mesh_tiles) and S a multiple
 *               of the chunk; otherwise as 3.  vec caps the chunk (vec 1: 32 samples);
 *           8 = as 3, with each element's rows requested two elements ahead (four
 *               register buffers rotate instead of three; minb 1..3);
 *   minb: resident blocks per SM the register allocation must allow (1..4).
 * Applies to launches made after the call (graphs keep what they captured). */
int cvfes_set_step_tuning(int32_t precision, int32_t vec, int32_t npb, int32_t staged,
                          int32_t minb);
int cvfes_get_step_tuning(int32_t precision, int32_t* vec, int32_t* npb, int32_t* staged,
                          int32_t* minb);

/* L2 prefetch of the fan step kernels (staged 3 and 8) and the fan reverse step:
 * each node block's first sample chunk prefetches into L2, by bulk prefetches, rows
 * that the nodes `distance` ahead of it will read.
 *   distance: in nodes; -1 (default) = the mesh's bandwidth + 128 (off when the
 *             descriptor's bandwidth is 0); 0 = off; else 1..2^20;
 *   parts:    bit 0 = the nodes' state, inverse-mass (and adjoint) rows (contiguous
 *             ranges); bit 1 = the coefficient (and Gamma) rows of their elements,
 *             found through their slot records; bit 2 = each warp's own second state
 *             row and inverse-mass row, read at the end of its node, are prefetched
 *             into L1 (instead of L2) when the node starts (fan kernels 3 and 8);
 *             -1 (default) = bits 0 and 1 with at least 4 sample chunks per node
 *             block, bit 0 alone below.
 * With fewer than 4 sample chunks per node block only every k-th node block
 * prefetches, for k node blocks (k = ceil(4 / chunks)).
 * Results are unchanged; only where the loads hit changes.  Applies to launches
 * made after the call (graphs keep what they captured).                        */
int cvfes_set_step_prefetch(int32_t precision, int32_t distance, int32_t parts);
int cvfes_get_step_prefetch(int32_t precision, int32_t* distance, int32_t* parts);

/* Failure-path test of the bounded device waits; no counterpart in the reference.
 * With polls > 0, template steps made after the call run the fan kernel with its
 * shared-memory stage barrier set up for two arrivals and no copy issued, waiting at
 * most `polls` polls: every block's wait gives up with nothing in flight, sets bit 0
 * of the mesh's status word (which must be non-NULL) and returns without writing
 * u_next.  cvfes_status_read then reports CVFES_ERR_TIMEOUT.  0 (the default) turns
 * it off.  Applies to launches made after the call (graphs keep what they captured). */
int cvfes_set_wait_probe(int32_t polls);

/* Where a step with the norms fused in (cvfes_solid_step_norms_*) keeps each lane's sums:
 * 0 (default) tensor memory, in a kernel of its own; 1 shared memory, in the plain
 * persistent kernel (16 KB more per block at 4 nodes per block and 4 samples per
 * thread, taken from the L1 of the neighbour-row gathers).  Both give bitwise the
 * same norms.                                                                       */
int cvfes_set_norms_memory(int32_t mode);

/* Read and clear the device status word of a mesh descriptor (synchronises the
 * stream).  Returns CVFES_ERR_TIMEOUT if a bounded device wait gave up since
 * the last read, else CVFES_OK.                                               */
int cvfes_status_read(int32_t* status, void* stream);

/* ---------------------------------------------------------------- errors */
const char* cvfes_last_error(void);
int         cvfes_version(void);

/* ------------------------------------------------- host preprocessing (CPU)
 * Node -> incident-element slots in fan order.  Replaces the node/element
 * neighbour search of meshColoring.py:25-36 and gives the kernels their
 * gather order.  elems is host int64 [E][3]; outputs host int32.
 * node_ptr [N+1]; slot_rec [4*3E]; elem_slot [3E] (slot of (e, local node)). */
int cvfes_mesh_incidence(int64_t n_nodes, int64_t n_elems, const int64_t* elems,
                         int32_t* node_ptr, int32_t* slot_rec, int32_t* elem_slot);

/* Strip tiling for the TMA-tiled step: tile t holds nodes [t*P, (t+1)*P).  For the
 * unclamped nodes of each tile, windows of H consecutive node ids covering the nodes
 * and all their neighbours (at most W, greedily from the smallest uncovered id) and
 * windows of EH element ids covering their elements (at most WE).  Outputs (host):
 *   tile_win int32 [n_tiles][W+WE]: node window starts, then element window starts
 *            (-1: unused);
 *   tile_rec int32 [4*3E]: per slot, the shared-memory row of its element, first
 *            and second neighbour within the tile's windows (window k, offset i ->
 *            k*H + i, elements k*EH + i), or -1 - id when no window holds it; then the
 *            slot's flags;
 *   node_loc int32 [N]: the row of the node itself, or -1 - id;
 *   stats int64 [4]: tiles, neighbour references outside the windows, element
 *            references outside the windows, most windows a tile would need.     */
int cvfes_mesh_tiles(int64_t n_nodes, int64_t n_elems, const int32_t* node_ptr,
                     const int32_t* slot_rec, int64_t n_clamped, int32_t P, int32_t H, int32_t W,
                     int32_t EH, int32_t WE, int32_t* tile_win, int32_t* tile_rec,
                     int32_t* node_loc, int64_t* stats);

/* Greedy element colouring over the node-sharing graph, smallest free colour
 * in element order (meshColoring.py:7-63).  colors: host int32 [E].
 * Returns the number of colours (>0) or CVFES_ERR_MESH if max_colors is too few. */
int cvfes_mesh_color_greedy(int64_t n_nodes, int64_t n_elems, const int64_t* elems,
                            int32_t max_colors, int32_t* colors);

/* Diagonal of Q^{-1} from a sparse factor Q = L D Lᵀ (selected inversion), for
 * the exact unit-marginal rescaling of the GMRF material samples (the reference
 * rescales by the empirical std across samples, GMRF.py:326-328).  L: host CSC,
 * unit lower triangular, sorted rows (int64 colptr [n+1], rowind, f64 values);
 * d host f64 [n]; out_diag host f64 [n].                                       */
int cvfes_gmrf_selected_inverse_diag(int64_t n, const int64_t* colptr, const int64_t* rowind,
                                     const double* lval, const double* d, double* out_diag);

/* Solve Lᵀ X = B in place (L unit lower triangular, host CSC as above; B host
 * f64 [n][nrhs], samples innermost): the X = L⁻ᵀ Z draw of GMRF.py:310, for
 * many samples at once, OpenMP over sample columns.                           */
int cvfes_gmrf_solve_lt(int64_t n, const int64_t* colptr, const int64_t* rowind,
                        const double* lval, int64_t nrhs, double* b);

/* --------------------------------------------------- one-time device set-up
 * Element frames and unit stiffness templates in FP64 (replaces the per-element
 * part of OptimizedSolidAssembleWithDamping, optimizedSolidAssemble.pyx:520-583,
 * and the initial pass of assemble_K_M_P, physicsSolverSDampGPUs.cl:28-223).
 *   nodes      device f64 [N][3]     elems device int32 [E][3]
 *   dmat       host   f64 [5][5]     (D of physicsSolver.py:184-188, no E)
 *   elem_slot  device int32 [3E]     slot_rec device int32 [4*3E]
 * Outputs (device, any may be NULL): slot_k64 f64 [28*3E], slot_k32 f32 [28*3E],
 *   kt_full f64 [E][81] (full 9x9), area f64 [E], normal f64 [E][3].        */
int cvfes_solid_templates_f64(int64_t n_nodes, int64_t n_elems, const double* nodes,
                              const int32_t* elems, const double* dmat,
                              const int32_t* elem_slot, const int32_t* slot_rec,
                              double* slot_k64, float* slot_k32, double* kt_full,
                              double* area, double* normal, void* stream);

/* Lumped mass and unit pressure load, FP64 (replaces lumpingWithDamping,
 * optimizedSolidAssemble.pyx:434-454, and the traction part, pyx:585-590).
 *   gthick  device f64 [E][S][n_gauss] thickness at the quadrature points;
 *           n_gauss = 3 (one per mid-edge point) or 1 (same thickness at all 3)
 *   mw      host f64 [3][3] row-sum weights mw[a][g] = rho * w_g^2 * N_g(a)
 * Outputs: lm f64 [N][S] (lumped mass, same for x/y/z), invm64 f64 [N][S],
 *   invm32 f32 [N][S] (1/lm, 0 where lm == 0), fhat64 f64 [N][4], fhat32 f32 [N][4]. */
int cvfes_solid_mass_load_f64(int64_t n_nodes, int64_t n_elems, int64_t n_samples,
                              const int32_t* node_ptr, const int32_t* slot_rec,
                              const double* area, const double* normal,
                              const double* gthick, int32_t n_gauss, const double* mw,
                              double* lm, double* invm64, float* invm32,
                              double* fhat64, float* fhat32, void* stream);

/* Block-CSR assembly of K_s = sum_e coef[e,s] Kt_e into the reference layout
 * K[nnzb][S][3][3] (the K output of OptimizedSolidAssembleWithDamping,
 * optimizedSolidAssemble.pyx:365-431).  Deterministic: one launch per colour.
 *   kt_full device f64 [E][81]; coef device f64 [E][S];
 *   block_pos device int32 [E][9] (CSR slot of block (a,b) of element e);
 *   color_ptr host int64 [n_colors+1], color_elems device int32 [E].
 * K must be zeroed by the caller (it accumulates, like the reference).        */
int cvfes_solid_assemble_bsr_f64(int64_t n_elems, int64_t n_samples, const double* kt_full,
                                 const double* coef, const int32_t* block_pos,
                                 int32_t n_colors, const int64_t* color_ptr,
                                 const int32_t* color_elems, double* K, void* stream);

/* ------------------------------------------------------------ the hot path
 * res += K v for the reference block-CSR layout (MultiplyByVector,
 * optimizedSolidAssemble.pyx:1250-1274): indptr/indices device int64,
 * K f64 [nnzb][S][3][3], v and res f64 [3N][S].                               */
int cvfes_bsr_spmv_f64(int64_t n_nodes, int64_t n_samples, const int64_t* indptr,
                       const int64_t* indices, const double* K, const double* v,
                       double* res, void* stream);

/* res = K_s u_s  (+ res if accumulate) from the element templates, all samples
 * (the per-step Ku of assemble_K_P, physicsSolverSDampGPUs.cl:232-393, and
 * MultiplyByVector on the assembled matrix, in template form).                */
int cvfes_solid_kmul_f64(const cvfes_solid_mesh* mesh, const double* coef,
                         const double* u, double* res, int32_t accumulate, void* stream);
int cvfes_solid_kmul_f32(const cvfes_solid_mesh* mesh, const float* coef,
                         const float* u, float* res, int32_t accumulate, void* stream);

/* One explicit damped step for all samples (replaces assemble_K_P + calc_u +
 * host Dirichlet + calc_u_appTrac, physicsSolverSDampGPUs.py:325-399, and
 * SolidSolver.Solve, physicsSolver.py:263-292):
 *   u_next = ( dt^2 (p*fhat - K u) + 2 m u + (dt/2*damp*m - m) u_prev ) / (m (1 + dt/2*damp))
 *   Dirichlet rows of u_next = clamp_value; rows with m == 0 give 0.
 * Pressure is p_sched[clock[0] + j] (device f64 schedule, device int64 clock)
 * or, when p_sched is NULL, the value `pressure`.  trac (device T [N][4] or
 * NULL) adds an external nodal traction dt^2 * trac / (m (1+dt/2 damp))
 * (calc_u_appTrac, physicsSolverSDampGPUs.cl:436-446).
 * With mesh->state_form == 1 (velocity-state form) `u_prev` holds the increment
 * v_n = u_n - u_{n-1} instead and is overwritten in place with v_{n+1}
 * (u_next = u + v_{n+1}); it must not alias u or u_next.  The same update, with
 * the increment carried in its own buffer rather than rebuilt from two rounded
 * displacements.                                                                */
int cvfes_solid_step_f64(const cvfes_solid_mesh* mesh, const double* coef, const double* invm,
                         const double* u, const double* u_prev, double* u_next,
                         const double* p_sched, const int64_t* clock, int64_t j,
                         double pressure, const double* trac, double dt, double damp,
                         void* stream);
int cvfes_solid_step_f32(const cvfes_solid_mesh* mesh, const float* coef, const float* invm,
                         const float* u, const float* u_prev, float* u_next,
                         const double* p_sched, const int64_t* clock, int64_t j,
                         double pressure, const float* trac, double dt, double damp,
                         void* stream);

/* One step as cvfes_solid_step_* and, in the same pass, the FP64 per-sample norms of the
 * new state (out f64 [S][4] as cvfes_solid_norms_*: sum u_next^2, sum du^2, sum m du^2,
 * non-finite count, du = u_next - u, or the new increment in the velocity-state form).
 * The persistent fan kernel accumulates each lane's sums in tensor memory (32 or 64
 * columns per block, freed at its end) while it writes the state, so the state is not
 * read a second time; shapes without it (S / vec not a multiple of 32, no max_degree)
 * run the step and the separate norms pass.
 * work: cvfes_norms_work_size(N, S) doubles.  check_finite: as cvfes_solid_norms_*.
 * out_host (NULL, or S*4 doubles of pinned host memory): when given, the call also copies
 * out to out_host, reads and clears mesh->status (CVFES_ERR_TIMEOUT if a bounded wait
 * gave up) and returns after one stream synchronisation with the norms on the host.
 * Replaces the reference's per-step host round trip of the state
 * (physicsSolverSDampGPUs.py:363-390) with one small read-back of per-sample sums.   */
int cvfes_solid_step_norms_f64(const cvfes_solid_mesh* mesh, const double* coef,
                               const double* invm, const double* u, const double* u_prev,
                               double* u_next, const double* p_sched, const int64_t* clock,
                               int64_t j, double pressure, const double* trac, double dt,
                               double damp, double* work, double* out, double* out_host,
                               int32_t check_finite, void* stream);
int cvfes_solid_step_norms_f32(const cvfes_solid_mesh* mesh, const float* coef,
                               const float* invm, const float* u, const float* u_prev,
                               float* u_next, const double* p_sched, const int64_t* clock,
                               int64_t j, double pressure, const float* trac, double dt,
                               double damp, double* work, double* out, double* out_host,
                               int32_t check_finite, void* stream);

/* n_steps steps with the buffer rotation (u_next, u, u_prev) <- (u_prev, u_next, u)
 * of physicsSolverSDampGPUs.py:398-399.  bufs[0] = u_n, bufs[1] = u_{n-1},
 * bufs[2] = free on entry; on return *rot tells which: u_n is bufs[(rot+0)%3]...
 * precisely, after k steps u_n is bufs[(3 - k % 3) % 3] — returned as *cur_idx,
 * u_{n-1} as *prev_idx.  In the velocity-state form bufs[1] holds the increment for
 * good and u_n alternates between bufs[0] and bufs[2] (*prev_idx stays 1).  After the
 * steps the clock (if given) advances by n_steps.                                  */
int cvfes_solid_advance_f64(const cvfes_solid_mesh* mesh, const double* coef, const double* invm,
                            double* buf0, double* buf1, double* buf2,
                            const double* p_sched, int64_t* clock, int64_t n_steps,
                            double dt, double damp, int32_t* cur_idx, int32_t* prev_idx,
                            void* stream);
int cvfes_solid_advance_f32(const cvfes_solid_mesh* mesh, const float* coef, const float* invm,
                            float* buf0, float* buf1, float* buf2,
                            const double* p_sched, int64_t* clock, int64_t n_steps,
                            double dt, double damp, int32_t* cur_idx, int32_t* prev_idx,
                            void* stream);

/* Initial state u_{-1} = u0 - dt du0 + dt^2/2 ddu0 with ddu0 = (p0 fhat - damp m du0 - K u0)/m
 * (LocalInitialize, physicsSolver.py:209-230; calc_ddu, physicsSolverSDampGPUs.cl:398-409).
 * u0, du0 device T [3N][S]; writes u_prev (in the velocity-state form the increment
 * u0 - u_{-1} = dt du0 - dt^2/2 ddu0).  Uses `work` T [3N][S] for K u0.         */
int cvfes_solid_init_f64(const cvfes_solid_mesh* mesh, const double* coef, const double* invm,
                         const double* u0, const double* du0, double* u_prev, double* work,
                         double p0, double dt, double damp, void* stream);
int cvfes_solid_init_f32(const cvfes_solid_mesh* mesh, const float* coef, const float* invm,
                         const float* u0, const float* du0, float* u_prev, float* work,
                         double p0, double dt, double damp, void* stream);

/* FP64 per-sample norms and the NaN/Inf watchdog (no reference counterpart;
 * the reference only prints wall-clock timers, solver.py:112-131).
 *   out f64 [S][4]: sum u^2, sum (u-u_prev)^2, sum m (u-u_prev)^2 (m from invm),
 *                   count of non-finite values.
 * Sums over nodes are FP64; each node's term (its three values) is formed in the
 * state's type: FP32 terms carry three FP32 roundings (<= 1.8e-7 relative; the
 * mass-weighted term also a reciprocal of at most 1 ulp and a product, <= 4e-7), FP64
 * terms FP64 ones.
 *   work f64, at least cvfes_norms_work_size(N, S) doubles (block partials).
 * Returns CVFES_ERR_NONFINITE (after writing out) when any value is NaN/Inf
 * and check_finite != 0 (this synchronises the stream).                       */
int64_t cvfes_norms_work_size(int64_t n_nodes, int64_t n_samples);
int cvfes_solid_norms_f64(int64_t n_nodes, int64_t n_samples, const double* u,
                          const double* u_prev, const double* invm, double* work,
                          double* out, int32_t check_finite, void* stream);
int cvfes_solid_norms_f32(int64_t n_nodes, int64_t n_samples, const float* u,
                          const float* u_prev, const float* invm, double* work,
                          double* out, int32_t check_finite, void* stream);
/* The same norms for the velocity-state form: `vel` holds the increment v = u_n - u_{n-1},
 * so out[s][1] = sum v^2 and out[s][2] = sum m v^2.                             */
int cvfes_solid_norms_vel_f64(int64_t n_nodes, int64_t n_samples, const double* u,
                              const double* vel, const double* invm, double* work,
                              double* out, int32_t check_finite, void* stream);
int cvfes_solid_norms_vel_f32(int64_t n_nodes, int64_t n_samples, const float* u,
                              const float* vel, const float* invm, double* work,
                              double* out, int32_t check_finite, void* stream);

/* The FP32-state norms of cvfes_solid_norms_f32 without a workspace argument and
 * without allocating anything; no counterpart in the reference.  For callers that
 * hold no device workspace and must not allocate one while the ensemble runs (a
 * between-steps watchdog on a GPU whose memory the state fills, or a framework
 * whose own pool owns all device memory).  The block partials live in a fixed
 * 4 MiB device array compiled into the library (held on every GPU that loads it
 * until exit), so n_samples may be at most 131071; larger requests fail with
 * CVFES_ERR_ARG.  Every call looks up that array's device address on the current
 * device (cudaGetSymbolAddress; nothing is cached, so the address is right after a
 * device reset too); the first lookup on a device may load the library's module, so
 * make the first call before any stream capture.  All calls share the array: calls
 * that overlap on the GPU (e.g. on two streams) race.                          */
int cvfes_solid_norms_noalloc_f32(int64_t n_nodes, int64_t n_samples, const float* u,
                                  const float* u_prev, const float* invm, double* out,
                                  int32_t check_finite, void* stream);

/* ------------------------------------------------------------ CUDA graphs
 * Capture `chunk` steps of cvfes_solid_advance (chunk a multiple of 3 so the
 * buffer roles repeat; of 2 in the velocity-state form) plus the clock increment
 * into one executable graph.
 * Each cvfes_graph_launch advances `chunk` steps.  precision: 32 or 64.       */
typedef struct cvfes_graph cvfes_graph;
int cvfes_graph_capture_advance(const cvfes_solid_mesh* mesh, int32_t precision,
                                const void* coef, const void* invm,
                                void* buf0, void* buf1, void* buf2,
                                const double* p_sched, int64_t* clock, int64_t chunk,
                                double dt, double damp, void* stream, cvfes_graph** out);
int cvfes_graph_launch(cvfes_graph* g, void* stream);
int cvfes_graph_destroy(cvfes_graph* g);

/* ------------------------------------------------------------ batched meshes
 * Many independent meshes (own node and sample counts, time step, damping,
 * pressure schedule) advanced together, one persistent launch per step (the
 * batched form of the per-step solid path; the reference runs one mesh per MPI
 * rank, physicsSolverSDampGPUs.py:325-399).  The caller allocates a device table of
 * cvfes_batch_table_bytes(n) bytes; cvfes_batch_pack fills it (synchronous copy)
 * and writes totals[3]: [0] work items of the gather kernel (variant 0), [1] work
 * items of the fan kernel (variant 1: blocks of 2 warps, slot rows staged by TMA
 * into two shared-memory stages, fan-rotation gathers), [2] the fan kernel's stage
 * capacity in slots (-1 when a mesh has no max_degree).  All meshes rotate their
 * buffers in lock step: with rot = (steps taken) % 6, u_n = buf[(3-rot%3)%3],
 * u_{n-1} = buf[(4-rot%3)%3]; a mesh whose descriptor has state_form 1 keeps its
 * increment in buf[1] and u_n in buf[0] (rot even) or buf[2] (rot odd).  vec: samples per thread (FP32 1|2|4, FP64 1|2), must
 * divide every mesh's S.  grid: blocks of the persistent launch (<= 0: one block per
 * work item for variant 0, as many as fit for variant 1).  Both variants give the
 * same bits as the single-mesh kernels.                                          */
typedef struct cvfes_batch_item {
    cvfes_solid_mesh mesh;       /* descriptor of this mesh (device arrays)     */
    const void*      coef;       /* [E][S] T                                    */
    const void*      invm;       /* [N][S] T                                    */
    void*            buf[3];     /* rotating state buffers [3N][S] T            */
    const double*    p_sched;    /* device pressure schedule or NULL (p = 0)    */
    double           dt;         /* this mesh's time step                       */
    double           damp;       /* mass-proportional damping                   */
} cvfes_batch_item;

int64_t cvfes_batch_table_bytes(int32_t n_meshes);
int cvfes_batch_pack(const cvfes_batch_item* items, int32_t n_meshes, int32_t precision,
                     int32_t vec, void* table_dev, int64_t* totals);
int cvfes_batch_step(const void* table_dev, int32_t n_meshes, const int64_t* totals,
                     int32_t precision, int32_t vec, int32_t variant, int32_t rot,
                     const int64_t* clock, int64_t j, int32_t grid, void* stream);
int cvfes_batch_advance(const void* table_dev, int32_t n_meshes, const int64_t* totals,
                        int32_t precision, int32_t vec, int32_t variant, int32_t rot0,
                        int64_t* clock, int64_t n_steps, int32_t grid, int32_t* rot_out,
                        void* stream);
/* `chunk` batched steps (multiple of 6) and the clock increment as one graph. */
int cvfes_batch_graph_capture(const void* table_dev, int32_t n_meshes, const int64_t* totals,
                              int32_t precision, int32_t vec, int32_t variant, int64_t* clock,
                              int64_t chunk, int32_t grid, cvfes_graph** out);

/* ------------------------------------------------------------ geometric update
 * Stiffness and follower pressure on the deformed geometry x + u_g of each sample:
 * the matrix-free K(x+u_g) u and p * sum_e (A_e/3) n_e of assemble_K_P
 * (physicsSolverSDampGPUs.cl:232-393, every step) and of OptimizedSolidAssembleUpdate
 * (optimizedSolidAssemble.pyx:710-819, every stiffness_update_interval steps,
 * physicsSolver.py:296-324).  The update of the state is cvfes_solid_step's.
 * slot_geo: [8 * 3E] per slot X_b1 - X_a, X_b2 - X_a (reference coordinates), from
 * cvfes_solid_slot_geometry_f64 (nodes device f64 [N][3], elems device int32 [E][3]).
 * ug: geometry displacement [3N][S] (NULL or == u: the current state).
 * trac: NULL or the nodal traction [4N] T (x, y, z, pad; local order, clamped rows
 *       zero), added to the force of every sample as calc_u_appTrac does
 *       (physicsSolverSDampGPUs.cl:436-446) -- as cvfes_solid_step's trac.
 * nu: Poisson ratio of D (physicsSolver.py:184-188, shear factor 5/6).          */
/* Geometric-step kernel choice per precision: samples per thread (1|2|4, FP64 1|2) and
 * threads per block (64|128|256); every choice gives bitwise the same results. */
int cvfes_set_geo_tuning(int32_t precision, int32_t vec, int32_t block);
int cvfes_get_geo_tuning(int32_t precision, int32_t* vec, int32_t* block);
int cvfes_solid_slot_geometry_f64(int64_t n_elems, const double* nodes, const int32_t* elems,
                                  const int32_t* slot_rec, double* geo64, float* geo32,
                                  void* stream);
int cvfes_solid_step_geo_f64(const cvfes_solid_mesh* mesh, const double* coef, const double* invm,
                             const double* slot_geo, const double* u, const double* up,
                             double* un, const double* ug, const double* p_sched,
                             const int64_t* clock, int64_t j, double pressure,
                             const double* trac, double nu, double dt, double damp,
                             void* stream);
int cvfes_solid_step_geo_f32(const cvfes_solid_mesh* mesh, const float* coef, const float* invm,
                             const float* slot_geo, const float* u, const float* up, float* un,
                             const float* ug, const double* p_sched, const int64_t* clock,
                             int64_t j, double pressure, const float* trac, double nu,
                             double dt, double damp, void* stream);
/* n_steps geometric steps with the reference's update counter (physicsSolver.py:299-324):
 * before each step, if *counter >= interval the geometry becomes the current state and
 * *counter = 1, else *counter += 1.  interval 1 reads the geometry straight from u_n
 * (geo_live tells whether that was already so before the call); larger intervals copy
 * u_n into ugeo (caller-owned [3N][S], zeros = undeformed at the start).  Buffers
 * rotate as in cvfes_solid_advance; *counter and *geo_live_out carry the state on. */
int cvfes_solid_advance_geo_f64(const cvfes_solid_mesh* mesh, const double* coef,
                                const double* invm, const double* slot_geo, double* buf0,
                                double* buf1, double* buf2, double* ugeo, const double* p_sched,
                                int64_t* clock, int64_t n_steps, int64_t interval,
                                int64_t* counter, int32_t geo_live, double nu, double dt,
                                double damp, int32_t* cur_idx, int32_t* prev_idx,
                                int32_t* geo_live_out, void* stream);
int cvfes_solid_advance_geo_f32(const cvfes_solid_mesh* mesh, const float* coef,
                                const float* invm, const float* slot_geo, float* buf0,
                                float* buf1, float* buf2, float* ugeo, const double* p_sched,
                                int64_t* clock, int64_t n_steps, int64_t interval,
                                int64_t* counter, int32_t geo_live, double nu, double dt,
                                double damp, int32_t* cur_idx, int32_t* prev_idx,
                                int32_t* geo_live_out, void* stream);

/* ------------------------------------------------------------ stress recovery
 * Element stresses per sample (OptimizedCalculateStress, optimizedSolidAssemble.pyx:
 * 1116-1223; physicsSolver.py:416-424 at each save): global xx, yy, xy, xz, yz of
 * T^T (E D B TT u_e) T on the geometry x + u_g.
 *   nodes device f64 [N][3], elems device int32 [E][3] (the state's node numbering),
 *   young device f64 [E][S] (mean of E over the quadrature points), u [3N][S],
 *   ug [3N][S] geometry displacement or NULL (undeformed), stress out [E][S][5].   */
int cvfes_solid_stress_f64(int64_t n_elems, int64_t n_samples, const double* nodes,
                           const int32_t* elems, const double* young, const double* u,
                           const double* ug, double nu, double* stress, void* stream);
int cvfes_solid_stress_f32(int64_t n_elems, int64_t n_samples, const double* nodes,
                           const int32_t* elems, const double* young, const float* u,
                           const float* ug, double nu, float* stress, void* stream);

/* ------------------------------------------------------------ adjoint
 * Gradient of the displacement-mismatch objective
 *     J_s = sum_{n % obs_every == 0, 0 < n <= T} sum_{i in obs} |u_n(i) - uobs_n(i)|^2
 * with respect to per-element, per-sample log E and log h (inverse wall-stiffness
 * estimation).  No counterpart in the reference, which has no differentiation.
 * The run starts from rest (u_0 = u_{-1} = 0: zero initial displacement and
 * velocity and zero pressure at t = 0, the reference's default start).
 * The forward pass runs T steps, adds up J and saves the pair (u_m, u_{m+1}) at
 * m = 0, C, 2C, ... (C = ckpt_every); the reverse pass runs the adjoint recursion
 * and the forward step backwards from u_T, restarting from each saved pair, and
 * accumulates Gamma (E x S) and optionally G (N x S); cvfes_adjoint_gradients turns
 * them into dJ/dlogE and dJ/dlogh.  All buffers are device memory at the problem's
 * precision T unless typed.                                                       */
typedef struct cvfes_adjoint_desc {
    cvfes_solid_mesh mesh;        /* templates and records at this precision         */
    int32_t      precision;       /* 32 or 64                                        */
    int32_t      record;          /* 1: the forward stores u at the observation nodes
                                     into obs instead of adding up J                 */
    const void*  coef;            /* [E][S] E*h                                      */
    const void*  invm;            /* [N][S] inverse lumped mass                      */
    const void*  owner_blocks;    /* [3E][28] from cvfes_adjoint_owner_blocks        */
    void*        state[3];        /* [3N][S] forward ring; final roles are returned  */
    void*        adj[2];          /* [3N][S] adjoint pair                            */
    void*        ckpt;            /* [ckpt_count][2][3N][S]                          */
    const double* p_sched;        /* [T] pressure of forward step n                  */
    int64_t*     clock;           /* device step counter of the forward steps        */
    int64_t      n_steps;         /* T                                               */
    int64_t      ckpt_every;      /* C                                               */
    int32_t      n_obs;           /* observation nodes (0: J = 0)                    */
    int32_t      obs_every;       /* observation interval in steps                   */
    const int32_t* obs_nodes;     /* [n_obs] distinct node ids                       */
    void*        obs;             /* [T/obs_every][n_obs][3][S] observed u           */
    double*      jpart;           /* [cvfes_adjoint_jpart_size] scratch              */
    double*      J;               /* [S] objective                                   */
    void*        gamma;           /* [E][S] sum_n chi_{n+1}^T Khat_e u_n             */
    void*        gmass;           /* [N][S] sum_n chi_{n+1} . (p_n fhat - K u_n), or
                                     NULL when no log h gradient is wanted           */
    double       dt;
    double       damp;
} cvfes_adjoint_desc;

/* Reverse-step kernel choice per precision: samples per thread (1|2|4, FP64 1|2),
 * nodes per block (1..8), variant (0: L1 gather, 1: fan rotation with TMA-staged
 * slot rows, needing S/vec a multiple of 32; 2: as 1, persistent, each block staging
 * its next work item's slot rows while it runs the current one, minb 1..3), minimum
 * blocks per SM (1..4, a register cap).  Every choice gives bitwise the same results. */
int cvfes_set_adjoint_tuning(int32_t precision, int32_t vec, int32_t npb, int32_t variant,
                             int32_t minb);
int cvfes_get_adjoint_tuning(int32_t precision, int32_t* vec, int32_t* npb, int32_t* variant,
                             int32_t* minb);
int64_t cvfes_adjoint_ckpt_count(int64_t n_steps, int64_t ckpt_every);
int64_t cvfes_adjoint_jpart_size(int64_t n_steps, int32_t obs_every, int32_t n_obs,
                                 int64_t n_samples);
/* Per element, the blocks K_b1b1, K_b1b2, K_b2b2 of the unit stiffness in the order of
 * the slot of its local node 0, stored at that slot: out [3E][28] (the other slots'
 * entries are not written; elems [E][3] int32, elem_slot [E][3] int32). */
int cvfes_adjoint_owner_blocks(const cvfes_solid_mesh* mesh, int32_t precision,
                               const int32_t* elems, const int32_t* elem_slot, void* out,
                               void* stream);
/* coef = exp(logE) exp(logh) (FP64 and/or FP32 copy) and thick = exp(logh), [E][S]. */
int cvfes_adjoint_material(int64_t n_elems, int64_t n_samples, const double* logE,
                           const double* logh, double* coef64, float* coef32, double* thick,
                           void* stream);
int cvfes_adjoint_forward(const cvfes_adjoint_desc* d, int32_t* final_cur, int32_t* final_prev,
                          void* stream);
int cvfes_adjoint_reverse(const cvfes_adjoint_desc* d, int32_t final_cur, int32_t final_prev,
                          void* stream);
/* grad_logE = -c Gamma; grad_logh = grad_logE - h sum_a alpha_{e,a} G_a / m_a, [E][S] FP64.
 * mass_weights: the 9 lumped-mass weights w[3a+g] of cvfes_solid_mass_load_f64;
 * area [E] and lm [N][S] FP64 as produced there. */
int cvfes_adjoint_gradients(const cvfes_adjoint_desc* d, const int32_t* elems,
                            const double* area, const double* mass_weights, const double* lm,
                            const double* logE, const double* logh, double* grad_logE,
                            double* grad_logh, void* stream);
/* which = 0: the forward pass (returns the final roles); 1: the reverse pass from
 * roles (cur, prev).  The graph replays against the descriptor's buffers. */
int cvfes_adjoint_capture(const cvfes_adjoint_desc* d, int32_t which, int32_t cur, int32_t prev,
                          int32_t* final_cur, int32_t* final_prev, cvfes_graph** out);

#ifdef __cplusplus
}
#endif

#endif /* CVFES_B200_H */
