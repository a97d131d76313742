/*
 * vbd_b200.h -- C ABI of the B200 (sm_100a) Vertex Block Descent solver for tetrahedral
 * Neo-Hookean elastodynamics.
 *
 * This is the drop-in boundary for the reference's VBD path (extinguish7/VBD_TetMesh).  Every
 * entry point below names the reference interface it replaces (file:line in that project).
 * Signatures use plain pointers and sizes only.  Layout conventions match the reference's own
 * buffers:
 *   - positions / velocities / inertia: float[3*N], xyz interleaved per vertex (the memory of an
 *     Eigen 3xN column-major matrix, TetMesh::mVertPos.data(); VBD_GPU_Wrapper.cu:257);
 *   - tets: int32[4*T], vertex ids per tet in the reference's local order (TetMesh::tets);
 *   - Dm^-1: float[9*T], row-major per tet (VBD_GPU_Wrapper.cu:277-280);
 *   - colour groups: CSR form of std::vector<std::vector<int>> -- offsets[C+1] and the
 *     concatenated vertex ids (VBD_GPU_Wrapper.h:15).
 * Any pointer argument for bulk data may be host memory (pageable or pinned) or device memory
 * of the solver's device: copies use unified addressing.
 *
 * Error convention: every function returns a vbd_status; VBD_OK is 0.  vbd_last_error() returns
 * the message of the last failing call on the calling thread.  A solver handle is not
 * thread-safe: use one handle per host thread.
 */
#ifndef VBD_B200_H
#define VBD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum vbd_status {
    VBD_OK = 0,
    VBD_ERR_INVALID_ARG = 1,   /* bad pointer, size, index or inconsistent input       */
    VBD_ERR_CUDA = 2,          /* a CUDA runtime call failed                           */
    VBD_ERR_STATE = 3,         /* call not valid in the handle's current state          */
    VBD_ERR_NONFINITE = 4,     /* a NaN / Inf position was produced by the sweep        */
    VBD_ERR_NO_DEVICE = 5,     /* no CUDA device, or the device is not sm_100           */
    VBD_ERR_TIMEOUT = 6,       /* a bounded device-side wait gave up                   */
    VBD_ERR_ALLOC = 7          /* device or host allocation failed                     */
} vbd_status;

typedef struct vbd_solver vbd_solver; /* opaque; owns all device memory of one mesh (or batch) */

/* Library version, as 10000*major + 100*minor + patch (no reference counterpart). */
int vbd_version(void);

/* Message of the last failing call on this thread ("" if none).  No reference counterpart: the
 * reference's calls return void and leave CUDA errors unchecked; every call here returns a
 * vbd_status. */
const char* vbd_last_error(void);

/* ------------------------------------------------------------------------------------------
 * Host-side mesh set-up (no GPU needed).
 * ------------------------------------------------------------------------------------------ */

/* Greedy vertex colouring, bit-exact with GraphColoring::colorVertices (GraphColoring.cpp:28-66,
 * neighbours from GraphColoring::getNeighbors :7-26): vertices in id order take the smallest
 * colour unused by already-coloured vertices sharing a tet.  Writes colour_of[N] and the colour
 * count.  If group_offsets (C+1 entries) and group_vertices (N entries) are non-null, also writes
 * the colour groups in CSR form, each group in ascending vertex id (the reference's
 * std::vector<std::vector<IdType>>).  Pass max_colours = capacity of group_offsets minus one. */
int vbd_color_vertices(int32_t num_verts, int32_t num_tets, const int32_t* tets, int32_t* colour_of,
                       int32_t* num_colours, int32_t max_colours, int32_t* group_offsets,
                       int32_t* group_vertices);

/* Rest volume and lumped mass, as TetMesh::initialize (TetMesh.h:249-265) and
 * TetMesh::computeRestVolume (TetMesh.h:291-298): V_t = |e0.(e1 x e2)|/6, m_i += rho V_t / 4.
 * Either output may be null. */
int vbd_mesh_mass(int32_t num_verts, int32_t num_tets, const float* rest_xyz, const int32_t* tets,
                  float density, float* vertex_mass, float* tet_rest_vol);

/* Dm^-1 (row-major) and V0 = |d3.(d1 x d2)|/6 of each tet's rest shape, as
 * VBDsolver::precomputeTetData (VBD.cpp:36-58) with ElasticEnergy::compute_Dm/compute_Volume
 * (Energy.cpp:6-32). */
int vbd_precompute_tets(int32_t num_verts, int32_t num_tets, const float* rest_xyz, const int32_t* tets,
                        float* dm_inv, float* rest_vol);

/* Accuracy of the factored element records on a mesh (no reference counterpart; host only): the
 * largest relative error, over every tet and local vertex, of the FP32 det M that record layout 3
 * stores and that layout 4 derives as s.w / |q_n|^2, against FP64 (M = the other three rows of
 * Ps Dm^-1, dm_inv float[9T] row-major as for vbd_solver_init); and layout4_loss_fraction, the
 * fraction of incidences on which layout 4's error is above both 1e-5 and 4 x layout 3's error
 * there, leaving out tets that are degenerate in FP32 (layout 3's error above 1e-3), where no FP32
 * form of the element is accurate (above 1e-3: vbd_solver_init's automatic choice takes layout 3).
 * Any output may be null. */
int vbd_factored_record_error(int32_t num_tets, const float* dm_inv, double* err_layout3, double* err_layout4,
                              double* layout4_loss_fraction);

/* ------------------------------------------------------------------------------------------
 * TetGen input and pinning (the reference driver's loadTetgenModel / readNodeFile and its
 * boundary rule, main.cpp:14-168).  Host only.
 * ------------------------------------------------------------------------------------------ */

/* Reads a TetGen .node file.  With positions == NULL only *num_nodes is set (the header count);
 * otherwise `capacity` >= *num_nodes positions are written xyz-interleaved and *first_index (if
 * not NULL) receives the first node's index: 0 means the mesh's ids are 0-based, else 1-based
 * (main.cpp:37-38).  Blank lines and '#' comment lines are skipped. */
int vbd_tetgen_read_node(const char* path, int32_t* num_nodes, int32_t* first_index, float* positions,
                         int32_t capacity);

/* Reads a TetGen .ele file (four vertex ids per element; index_base 0 or 1 is subtracted,
 * main.cpp:113-115).  With tets == NULL only *num_tets is set.  Ids must lie in [0, num_nodes)
 * when num_nodes >= 0. */
int vbd_tetgen_read_ele(const char* path, int32_t index_base, int32_t num_nodes, int32_t* num_tets, int32_t* tets,
                        int32_t capacity);

/* Sets fixed[i] = 1 for every vertex whose coordinate `axis` (0 = x, 1 = y, 2 = z) is at most
 * min + (max - min) * fraction over all vertices, in float arithmetic (main.cpp:127-163 with
 * fraction 0.05 on y); entries already set stay set. */
int vbd_pin_low_fraction(int32_t num_verts, const float* positions, int32_t axis, float fraction, uint8_t* fixed);

/* ------------------------------------------------------------------------------------------
 * Solver handle (one GPU).  Replaces VBD::VBD_GPU_Solver (VBD_GPU_Wrapper.h:7-45) and the
 * step loop of VBD::VBDsolver (VBD.cpp:60-112).
 * ------------------------------------------------------------------------------------------ */

/* Replaces the VBD_GPU_Solver constructor (VBD_GPU_Wrapper.h:9-11).
 * Creates a handle on CUDA device `device`.  `cuda_stream` is a cudaStream_t (may be null: the
 * handle then creates its own non-blocking stream).  Fails with VBD_ERR_NO_DEVICE if the device
 * is absent or is not compute capability 10.0. */
int vbd_solver_create(vbd_solver** out, int device, void* cuda_stream);

/* Frees all device memory of the handle (VBD_GPU_Solver::~VBD_GPU_Solver,
 * VBD_GPU_Wrapper.cu:373-382).  Null is accepted. */
int vbd_solver_destroy(vbd_solver* s);

/* Uploads one mesh (VBD_GPU_Solver::initFromCPU, VBD_GPU_Wrapper.cu:246-315).
 *   positions[3N]       current positions x (TetMesh::mVertPos)
 *   velocities[3N]      may be null (zero)           (TetMesh::mVelocity)
 *   inertia[3N]         may be null (set to x)       (TetMesh::mInertia)
 *   vertex_mass[N]      lumped masses                (TetMesh::vertexMass)
 *   fixed[N]            1 = pinned                   (TetMesh::isFixed)
 *   tets[4T]            vertex ids                   (TetMesh::tets)
 *   num_colours, group_offsets[C+1], group_vertices[N]: colour groups (VBDsolver::vertexColors)
 *   dm_inv[9T], rest_vol[T]                          (VBDsolver::tetDmInv / tetRestVolume)
 *   tet_mu[T], tet_lambda[T]: per-tet Lame parameters (TetMesh::tetMu / tetLambda)
 * Colour groups must partition the vertices and must be independent sets (no tet holds two
 * vertices of one colour); tets must hold four distinct, in-range ids.  Calling it again
 * replaces the previous mesh. */
int vbd_solver_init(vbd_solver* s, int32_t num_verts, int32_t num_tets, const float* positions,
                    const float* velocities, const float* inertia, const float* vertex_mass,
                    const uint8_t* fixed, const int32_t* tets, int32_t num_colours,
                    const int32_t* group_offsets, const int32_t* group_vertices, const float* dm_inv,
                    const float* rest_vol, const float* tet_mu, const float* tet_lambda);

/* Uploads a batch of independent meshes as one solver problem (no reference counterpart: the
 * reference handles one mesh per VBD_GPU_Solver).  Arrays are the meshes' arrays concatenated;
 * vert_offsets[M+1] / tet_offsets[M+1] delimit mesh m, and tets_local holds each mesh's own vertex
 * ids (0-based within the mesh).  Each mesh is coloured with the greedy colouring of
 * GraphColoring::colorVertices on its own; colour c of every mesh is swept by one launch.  Positions,
 * velocities and inertia are then addressed in the concatenated numbering by every other call. */
int vbd_solver_init_batch(vbd_solver* s, int32_t num_meshes, const int32_t* vert_offsets, const int32_t* tet_offsets,
                          const float* positions, const float* velocities, const float* vertex_mass,
                          const uint8_t* fixed, const int32_t* tets_local, const float* dm_inv, const float* rest_vol,
                          const float* tet_mu, const float* tet_lambda);

/* Per-tet materials (TetMesh::tetMu / tetLambda, TetMesh.h:31-32); either pointer may be
 * null to keep the current values. */
int vbd_solver_set_materials(vbd_solver* s, const float* tet_mu, const float* tet_lambda);

/* One (mu, lambda) for every tet: the reference's scalar VBDParams::mu / lambda
 * (VBD.h:22-23, used at VBD.cpp:214-215) and the mu / lambda arguments of
 * VBD_GPU_Solver::solveIteration / solveVBD (VBD_GPU_Wrapper.h:19,28). */
int vbd_solver_set_uniform_material(vbd_solver* s, float mu, float lambda);

/* State transfer.  set_inertia replaces VBD_GPU_Solver::updateInertiaFromCPU
 * (VBD_GPU_Wrapper.cu:369-371); get_positions replaces copyPositionsToCPU (:364-366).  All
 * arrays are float[3N] in the caller's vertex numbering.  Getters complete before returning. */
int vbd_solver_set_positions(vbd_solver* s, const float* xyz);
int vbd_solver_get_positions(vbd_solver* s, float* xyz);
int vbd_solver_set_velocities(vbd_solver* s, const float* xyz);
int vbd_solver_get_velocities(vbd_solver* s, float* xyz);
int vbd_solver_set_inertia(vbd_solver* s, const float* xyz);
int vbd_solver_get_inertia(vbd_solver* s, float* xyz);

/* Initial guess of vbd_solver_solve. */
typedef enum vbd_init_mode {
    VBD_INIT_FROM_POSITIONS = 0, /* iterate from the current x (VBDsolver::step, VBD.cpp:76)   */
    VBD_INIT_FROM_INERTIA = 1    /* iterate from x = y (VBD_GPU_Solver::solveVBD, :334)        */
} vbd_init_mode;

/* `iterations` Gauss-Seidel sweeps over the colour groups with the Chebyshev blend
 * (VBD_GPU_Solver::solveVBD, VBD_GPU_Wrapper.cu:332-362; VBDsolver step loop VBD.cpp:75-96,
 * getAcceleratorOmega :302-311).  Uses the inertia y already on the device.  Asynchronous. */
int vbd_solver_solve(vbd_solver* s, int32_t iterations, float dt_sqr_reciprocal, int32_t use_acceleration,
                     float rho, int32_t init_mode);

/* One sweep without acceleration (VBD_GPU_Solver::solveIteration, VBD_GPU_Wrapper.cu:317-329).
 * Asynchronous. */
int vbd_solver_solve_iteration(vbd_solver* s, float dt_sqr_reciprocal);

/* One time step on the GPU: for each of `substeps` sub-steps of h = dt/substeps, the inertial
 * predictor (VBDsolver::forwardStep VBD.cpp:103-112: x_prev = x, v += h g, y = x + h v; y = x
 * for pinned vertices), `iterations` sweeps with Chebyshev (VBD.cpp:75-96), and the velocity
 * update v = (x - x_prev)/h * 0.999 (TetMesh::updateVelocity, TetMesh.h:305-311).  Replaces
 * VBDsolver::step (VBD.cpp:60-101).  gravity is float[3].  Asynchronous. */
int vbd_solver_step(vbd_solver* s, float dt, int32_t substeps, int32_t iterations, const float* gravity,
                    int32_t use_acceleration, float rho);

/* ---- Adjoint (no reference counterpart) --------------------------------------------------------
 * Gradients of a loss of the final state through a sequence of steps, each step implicitly
 * differentiated as converged: (M/h^2 + H) lam = G is solved with the forward's coloured block
 * Gauss-Seidel over per-vertex 3x3 blocks (off-diagonal blocks applied through per-tet products),
 * then dL/dy = M/h^2 lam, dL/d(mu_t, lambda_t) -= lam . V (F - C) q_n and lam . V (J - 1) C q_n
 * summed over the tet's vertices, and the adjoint flows through y = x + h v + h^2 g and
 * v' = 0.999 (x' - x)/h to the previous step. */

/* Starts recording the steps taken from now on (checkpoint_every > 0): the current positions and
 * velocities, and those after every checkpoint_every-th sub-step, are kept on the device; steps in
 * between are recomputed during the backward pass.  checkpoint_every = 0 stops recording.  The
 * state must change only through vbd_solver_step while recording. */
int vbd_solver_record(vbd_solver* s, int32_t checkpoint_every);

/* Backward pass over every recorded sub-step: dl_dx / dl_dv (float[3N]; dl_dv may be null) are the
 * loss gradient w.r.t. the final positions / velocities; writes dL/dx0, dL/dv0 (float[3N], at
 * recording start) and dL/dmu, dL/dlambda (float[T], accumulated over all steps); any output may
 * be null.  adjoint_iterations = Gauss-Seidel sweeps per step (warm-started from the previous
 * step's lam), accelerated by the forward's Chebyshev weights for spectral-radius estimate
 * adjoint_rho (0 = plain Gauss-Seidel).  The solver's own state is left as it was.  Completes
 * before returning. */
int vbd_solver_backward(vbd_solver* s, const float* dl_dx, const float* dl_dv, int32_t adjoint_iterations,
                        float adjoint_rho, float* dl_dx0, float* dl_dv0, float* dl_dmu, float* dl_dlambda);

/* Waits for all work queued on the handle's stream and reports sticky device errors, and
 * VBD_ERR_TIMEOUT if a grid barrier of the persistent kernel gave up since the last sync.  No
 * reference counterpart: the reference's calls are synchronous. */
int vbd_solver_sync(vbd_solver* s);

/* Failure-detection self-test (no reference counterpart): launches the persistent kernel with one barrier arrival missing and
 * a poll limit of spin_limit, so its first grid barrier can never complete.  Every block gives up
 * after spin_limit polls and exits; *timed_out receives 1 if the device recorded the timeout. */
int vbd_solver_barrier_selftest(vbd_solver* s, int64_t spin_limit, int32_t* timed_out);

/* The energy history of VBD_OPT_ENERGY_EVERY (VBDsolver::energyHistory, VBD.h:70; filled at
 * VBD.cpp:93-95): writes up to `capacity` values, oldest first, and sets *count to the number of
 * values appended since the last reset (a count above capacity means the rest were not copied).
 * reset != 0 empties the history.  Completes the queued work first. */
int vbd_solver_energy_history(vbd_solver* s, double* energies, int32_t capacity, int32_t* count, int32_t reset);

/* Energies (FP64 accumulation over the FP32 state).  Completes before returning.
 *   VBD_ENERGY_IP:      incremental potential sum_i m_i/(2h^2)|x_i - y_i|^2 + sum_t V_t psi(F_t),
 *                       psi = mu/2(|F|^2-3) - mu(J-1) + lambda/2 (J-1)^2 (the energy whose gradient
 *                       the reference's force uses, Energy.cpp:97); h from `h`.
 *   VBD_ENERGY_ELASTIC_LOGJ: VBDsolver::computeTotalEnergy (VBD.cpp:258-288 with
 *                       NeoHookean::compute_Energy NeoHookean.cpp:6-20), J = |det F|; h ignored.
 *   VBD_ENERGY_RESIDUAL: || m_i/h^2 (x_i - y_i) + dE/dx_i ||_2 over free vertices. */
typedef enum vbd_energy_kind {
    VBD_ENERGY_IP = 0,
    VBD_ENERGY_ELASTIC_LOGJ = 1,
    VBD_ENERGY_RESIDUAL = 2
} vbd_energy_kind;
int vbd_solver_energy(vbd_solver* s, int32_t kind, float h, double* out);

/* Device-side counters since the last call with reset != 0: vertices whose 3x3 system failed
 * the |det H| > 1e-8 guard and were left in place (VBD.cpp:141-156; the reference's GPU kernel
 * printed a warning instead, VBD_GPU_Wrapper.cu:232), and whether a non-finite position was
 * produced. */
int vbd_solver_status(vbd_solver* s, int64_t* singular_skips, int32_t* nonfinite, int32_t reset);

/* Tuning knobs (all have measured defaults).
 *   VBD_OPT_LANES:       threads cooperating on one vertex: 1, 2, 4, 8, 16 or 32.  Until it is
 *                        set, vbd_solver_init picks 8 when the free vertices average at least 21
 *                        incident tets, else 4, then doubles it (up to 16) while the largest colour
 *                        times the lanes stays within half of the GPU's resident threads
 *   VBD_OPT_LAYOUT:      0 = tet records gathered through a per-vertex tet list,
 *                        1 = 64 B tet records copied into incidence order and streamed,
 *                        2 = compact 56 B incidence records streamed (other three vertex ids, their
 *                            rows of Ps Dm^-1, V0 mu, V0 lambda)
 *                        3 = factored 48 B incidence records streamed (other three vertex ids,
 *                            s = M q_n, w = cof(M) q_n, det M for M = their rows of Ps Dm^-1, and the
 *                            material products): the element block without forming F or cof(F)
 *                        4 = packed factored 40 B incidence records (the three ids in 21 bits
 *                            each, s, w and the material products; det M = s.w / |q_n|^2 derived):
 *                            meshes of at most 2^21 vertices only (VBD_ERR_INVALID_ARG otherwise)
 *                        Until it is set, vbd_solver_init picks layout 4 when the mesh has at most
 *                        2^21 vertices and layout 4's FP32 det M loses accuracy on at most 0.1% of
 *                        the incidences (vbd_factored_record_error; systematically anisotropic
 *                        meshes exceed it), else layout 3.
 *                        Defaults: 64-thread blocks, PDL, graphs; lanes, layout and prefetch
 *                        chosen by vbd_solver_init.
 *   VBD_OPT_GRAPH:       1 = replay a captured CUDA graph per step, 0 = direct launches
 *   VBD_OPT_KERNEL_TIMING: 1 = launch directly and bracket every colour-sweep kernel with a CUDA
 *                        event pair on the handle's stream (read with vbd_solver_kernel_time)
 *   VBD_OPT_PREFETCH:    0 = load each element record where it is used, 1 = load the next record
 *                        while evaluating the current one, 2 = load a lane's first three records
 *                        before the sweep's dependency wait, 3 = its first two, in a kernel held to
 *                        56 registers (2 and 3: layouts 3 and 4; others run 1).  Until it is set: 2
 *                        with layout 4 when no lane holds more than three records (most incident
 *                        tets of a free vertex / lanes), else 1.  All give the same bits
 *   VBD_OPT_PDL:         1 = launch colour sweeps with programmatic dependent launch, so a sweep
 *                        loads its element data while the previous sweep drains
 *   VBD_OPT_BLOCK:       threads per block of the sweep kernel: 64, 128 or 256
 *   VBD_OPT_PERSISTENT:  1 = run each step / solve as one cooperative launch that walks the colours
 *                        with a grid barrier after each one (bounded wait: a barrier that gives up
 *                        makes the next vbd_solver_sync return VBD_ERR_TIMEOUT);
 *                        2 = run each sub-step / solve as ONE thread-block cluster that keeps both
 *                        position buffers of the mesh (and the pre-sweep positions) in every CTA's
 *                        shared memory, exchanges updated positions through distributed shared
 *                        memory and separates the colours with the cluster's hardware barrier.  For
 *                        meshes whose positions fit (48 B per vertex within the device's per-CTA
 *                        shared memory: about 4,800 vertices on B200) with the factored records (VBD_OPT_LAYOUT 3 or
 *                        4); VBD_ERR_INVALID_ARG otherwise.  Same results as the captured graph at the
 *                        same lane count.  Both persistent forms use VBD_OPT_LANES for every colour
 *                        (at least 4) and evaluate no energy history
 *   VBD_OPT_CLUSTER_CTAS: CTAs of the cluster walk, 1-16; 0 (default) = enough 256-thread
 *                        CTAs to sweep the largest colour in one round, at most 16.  Reading it
 *                        back gives the set count, or the automatic count for the current lanes
 *   VBD_OPT_CLUSTER_RESIDENT: 1 (default) = the cluster walk copies, once per sub-step, the element
 *                        records, inertial targets and incidence spans of the vertices each CTA
 *                        sweeps into that CTA's shared memory when they fit beside the positions,
 *                        so no colour waits on L2 for them; 0 = they are read from L2 each colour.
 *                        Same results either way
 *   VBD_OPT_ADJOINT_ALTERNATE: 1 = adjoint sweeps alternate the colour order (a forward and a
 *                        backward sweep form one symmetric Gauss-Seidel pair)
 *   VBD_OPT_SEMANTICS:   0 = the CPU solver's (VBDsolver, VBD.cpp:114-256): Neo-Hookean element,
 *                        Chebyshev weights with double literals (the default);
 *                        1 = the reference's GPU wrapper's (VBD_GPU_Solver, VBD_GPU_Wrapper.cu:114-362,
 *                        VBD_DeviceMath.cuh:127-198): corotated element (5 Higham polar steps,
 *                        P = 2 mu (F - R) + lambda tr(R^T F - I) R, Hessian 2 mu |q|^2 I +
 *                        lambda (R q)(R q)^T), inertia diagonal x 1.000001, solve3x3 guard, float
 *                        Chebyshev weights, 16 lanes per vertex with the wrapper's summation order,
 *                        tet records read through the per-vertex tet list (any layout), and
 *                        vbd_solver_step starting each sub-step from x = y as main.cpp's GPU loop
 *                        does.  Not with VBD_OPT_PERSISTENT, vbd_solver_record or the adjoint;
 *                        energies and residuals stay the Neo-Hookean ones
 *   VBD_OPT_L2_PREFETCH: 1 = with the compact or factored layout, each colour sweep prefetches the
 *                        records of the colour swept next into L2 (one bulk prefetch per block);
 *                        off by default (slower on the measured meshes)
 *   VBD_OPT_RECORD_CACHE: 1 = the factored records (layouts 3 and 4) are loaded past L1 with an L2
 *                        evict-first policy, so that the stream does not push the vertex state out of
 *                        L2 (the default); 0 = plain read-only loads.  Same results
 *   VBD_OPT_RECORD_PERSIST_MB: with VBD_OPT_RECORD_CACHE, the first this-many megabytes of the record
 *                        stream are loaded with an L2 evict-last policy instead, so that they stay in
 *                        L2 from one sweep to the next (0 = none).  Until it is set, vbd_solver_init
 *                        picks 32 when the vertex state (64 B per vertex) fits in 32 MB, else 0
 *   VBD_OPT_ENERGY_EVERY: k > 0 = vbd_solver_step also evaluates VBDsolver::computeTotalEnergy (the
 *                        VBD_ENERGY_ELASTIC_LOGJ energy, FP64 sums) of the positions after iterations
 *                        0, k, 2k, ... of every sub-step, as VBDsolver::step does with k = 10
 *                        (VBD.cpp:93-95), into a device-side history read by
 *                        vbd_solver_energy_history; 0 = off (the default).  Positions are unchanged.
 *                        With VBD_OPT_PERSISTENT the steps then run as separate launches */
typedef enum vbd_option {
    VBD_OPT_LANES = 0,
    VBD_OPT_LAYOUT = 1,
    VBD_OPT_GRAPH = 2,
    VBD_OPT_KERNEL_TIMING = 3,
    VBD_OPT_PREFETCH = 4,
    VBD_OPT_PDL = 5,
    VBD_OPT_BLOCK = 6,
    VBD_OPT_PERSISTENT = 7,
    VBD_OPT_ADJOINT_ALTERNATE = 8,
    VBD_OPT_SEMANTICS = 9,
    VBD_OPT_L2_PREFETCH = 10,
    VBD_OPT_RECORD_CACHE = 11,
    VBD_OPT_RECORD_PERSIST_MB = 12,
    VBD_OPT_ENERGY_EVERY = 13,
    VBD_OPT_CLUSTER_CTAS = 14,
    VBD_OPT_CLUSTER_RESIDENT = 15
} vbd_option;
int vbd_solver_set_option(vbd_solver* s, int32_t option, int32_t value);
int vbd_solver_get_option(vbd_solver* s, int32_t option, int32_t* value);

/* Per-colour launch shape (no reference counterpart; the reference's kernel runs 16 threads per
 * vertex for every colour, VBD_GPU_Wrapper.cu:320-321): colour c of the sweep runs lanes[c]
 * threads per vertex (1, 2, 4, 8, 16 or 32), and its record prefetch follows the lane count as
 * VBD_OPT_PREFETCH describes.  lanes = NULL goes back to VBD_OPT_LANES for every colour.  Same results as the
 * uniform shape up to the order of the per-vertex sums.  A new mesh (vbd_solver_init) clears it.
 * get_colour_lanes writes the lane count each colour runs. */
int vbd_solver_set_colour_lanes(vbd_solver* s, int32_t num_colours, const int32_t* lanes);
int vbd_solver_get_colour_lanes(vbd_solver* s, int32_t num_colours, int32_t* lanes);

/* Autotuner (no reference counterpart: the reference launches one 16-thread block per vertex,
 * VBD_GPU_Wrapper.cu:320-321): times `repeats` steps of `iterations` sweeps (dt, no gravity,
 * Chebyshev 0.9) for each launch configuration it tries and keeps the fastest, then restores the
 * simulation state (positions, velocities, inertia, counters) it started from.  In order:
 *   1. uniform launch shapes from a fixed list -- threads per vertex, record layout, prefetch,
 *      programmatic dependent launch, block size;
 *   2. the factored records' L2 policy (VBD_OPT_RECORD_CACHE with VBD_OPT_RECORD_PERSIST_MB 0, 32
 *      and 64);
 *   3. per-colour threads per vertex (vbd_solver_set_colour_lanes): greedy over the colours, lane
 *      counts 2, 4, 8 and 16, two passes, restarted under each prefetch depth of the factored
 *      layouts; each candidate is timed alternately with the incumbent (twice each, 2 x repeats
 *      steps) against drift;
 *   4. the persistent colour-walking kernel (VBD_OPT_PERSISTENT 1) against the captured graph,
 *      then, where the mesh fits, the cluster walk (VBD_OPT_PERSISTENT 2) at 4, 8, 16 and 32
 *      threads per vertex with record layouts 3 and 4, and, when it wins, its CTA count
 *      (VBD_OPT_CLUSTER_CTAS) at about 1/2, 3/4 and 3/2 of the automatic count and at 16.
 * Phases 2-4 replace the choice only when faster by more than 1%.  chosen (may be null) receives 5
 * ints: lanes, layout, prefetch, pdl, block; the rest of the choice is read back with
 * vbd_solver_get_option (VBD_OPT_RECORD_CACHE, VBD_OPT_PERSISTENT, VBD_OPT_CLUSTER_CTAS) and
 * vbd_solver_get_colour_lanes. */
int vbd_solver_autotune(vbd_solver* s, float dt, int32_t iterations, int32_t repeats, int32_t* chosen);

/* Allocation-free incremental potential.  No counterpart in the reference: it exists for callers
 * that cannot let a library allocate device memory -- code embedded in a framework that owns the
 * device memory (a PyTorch caching-allocator pool, an engine's fixed arena) or in a fixed-latency
 * loop, where cudaMalloc / cudaFree would synchronise the device or fail once the pool holds the
 * free memory.  It computes the same quantity as vbd_solver_energy(VBD_ENERGY_IP) from caller-owned
 * DEVICE arrays in the reference layouts (positions / inertia float[3N], vertex_mass[N], tets
 * int32[4T], dm_inv float[9T] row-major, rest_vol / tet_mu / tet_lambda float[T]) and writes the
 * FP64 sum to the device pointer `out`.  It allocates nothing: its scratch (block partials and an
 * error flag) is a fixed 32 KiB __device__ array that every GPU loading the library holds until
 * exit, so num_verts + num_tets is limited to 16,777,216 (larger sizes return
 * VBD_ERR_INVALID_ARG).  The first call on each device looks up the scratch address and must come
 * before any stream capture on that device; later calls look it up again, so a cudaDeviceReset
 * between calls is harmless.  Calls share the scratch: calls that overlap on the GPU race.  Runs
 * on `cuda_stream` (null = default stream) and blocks the calling thread until it completes: it
 * reads its error flag back and synchronises the stream, so a call cannot be captured into a CUDA
 * graph.  Tets with ids outside [0, N) are skipped and reported as VBD_ERR_INVALID_ARG. */
int vbd_ip_energy_noalloc(int32_t num_verts, int32_t num_tets, const float* positions, const float* inertia,
                          const float* vertex_mass, const int32_t* tets, const float* dm_inv, const float* rest_vol,
                          const float* tet_mu, const float* tet_lambda, float h, double* out, void* cuda_stream);

/* Sizes of the uploaded mesh: vertices, tets, colours (no reference counterpart). */
int vbd_solver_info(vbd_solver* s, int32_t* num_verts, int32_t* num_tets, int32_t* num_colours);

/* Number of kernels this handle launched since creation (graph replays count their nodes; no
 * reference counterpart). */
int vbd_solver_kernel_launches(vbd_solver* s, int64_t* launches);

/* With VBD_OPT_KERNEL_TIMING on (no reference counterpart): summed device time (ms) of the colour-sweep kernels timed since
 * the last reset, their count, and the algorithmic bytes they moved (per free vertex swept:
 * 60 B per incident tet -- tet id, 4 vertex ids, Dm^-1, V0 -- plus 96 B of vertex state).
 * Completes the timed work first. */
int vbd_solver_kernel_time(vbd_solver* s, double* sweep_ms, int64_t* sweep_launches, double* sweep_bytes,
                           int32_t reset);

#ifdef __cplusplus
}
#endif

#endif /* VBD_B200_H */
