// Solver handle of libvbd_b200: device state, launch sequencing, CUDA-graph replay and the
// solver half of the C ABI declared in include/vbd_b200.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "vbd_b200.h"
#include "vbd_internal.h"
#include "vbd_cluster.cuh"
#include "vbd_kernels.cuh"

namespace vbd {

#define CUDA_TRY(call)                                                                                 \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess)                                                                         \
            VBD_FAIL(VBD_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

#define VBD_TRY(expr)            \
    do {                         \
        int rc_ = (expr);        \
        if (rc_) return rc_;     \
    } while (0)

template <class T> struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    int alloc(size_t count) {
        release();
        if (count == 0) return VBD_OK;
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T));
        if (e != cudaSuccess) {
            p = nullptr;
            VBD_FAIL(VBD_ERR_ALLOC, "cudaMalloc of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
        }
        n = count;
        return VBD_OK;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~DBuf() { release(); }
};

static inline unsigned nblk(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

// getAcceleratorOmega (VBD.cpp:302-311): double literals, float result.
static float omega_of(int order, float rho, float prev) {
    if (order == 1) return 1.0f;
    if (order == 2) return (float)(2.0 / (2.0 - (double)(rho * rho)));
    return (float)(4.0 / (4.0 - (double)(rho * rho * prev)));
}

// getAcceleratorOmega of the GPU wrapper (VBD_GPU_Wrapper.cu:240-244): float arithmetic.
static float omega_of_wrapper(int order, float rho, float prev) {
    if (order == 1) return 1.0f;
    if (order == 2) return 2.0f / (2.0f - (rho * rho));
    return 4.0f / (4.0f - (rho * rho) * prev);
}

using SweepFn = void (*)(SweepParams);

// prefetch 0 / 1 / 2 / 3 = k_sweep's PREFETCH 0 / 1 / 3 and k_sweep_capped's PREFETCH 2 (the deep
// forms for the factored layouts only; the others run PREFETCH 1 for options 2 and 3).  The
// factored layouts' PREFETCH 1 runs as k_sweep_capped (56 registers).  `cache` selects the
// record loads with an L2 policy (factored layouts; k_sweep's CACHE).
template <int L, int LAYOUT, bool CACHE> static SweepFn pick_depth(int prefetch) {
    if (prefetch == 0) return &k_sweep<L, LAYOUT, 0, CACHE>;
    if constexpr (LAYOUT >= 3 && L > 1) {
        if (prefetch == 1) return &k_sweep_capped<L, LAYOUT, 1, CACHE>;
        if (prefetch == 3) return &k_sweep_capped<L, LAYOUT, 2, CACHE>;
        return &k_sweep<L, LAYOUT, 3, CACHE>;
    } else if constexpr (LAYOUT >= 3) {
        return prefetch == 1 ? &k_sweep<L, LAYOUT, 1, CACHE> : &k_sweep<L, LAYOUT, 3, CACHE>;
    } else {
        return &k_sweep<L, LAYOUT, 1, CACHE>;
    }
}

template <int L> static SweepFn pick_sweep(int layout, int prefetch, bool cache) {
    switch (layout) {
        case 0: return pick_depth<L, 0, false>(prefetch);
        case 1: return pick_depth<L, 1, false>(prefetch);
        case 2: return pick_depth<L, 2, false>(prefetch);
        case 3: return cache ? pick_depth<L, 3, true>(prefetch) : pick_depth<L, 3, false>(prefetch);
        default: return cache ? pick_depth<L, 4, true>(prefetch) : pick_depth<L, 4, false>(prefetch);
    }
}

static SweepFn pick_sweep(int lanes, int layout, int prefetch, bool cache) {
    switch (lanes) {
        case 1: return pick_sweep<1>(layout, prefetch, cache);
        case 2: return pick_sweep<2>(layout, prefetch, cache);
        case 4: return pick_sweep<4>(layout, prefetch, cache);
        case 8: return pick_sweep<8>(layout, prefetch, cache);
        case 16: return pick_sweep<16>(layout, prefetch, cache);
        default: return pick_sweep<32>(layout, prefetch, cache);
    }
}

// The cluster walk reads the factored records (layouts 3 and 4), from L2 or resident in shared memory.
template <int L> static void (*pick_cluster(int layout, bool resident))(PersistParams) {
    if (resident) return layout == 3 ? &k_cluster_walk_srec<L, 3> : &k_cluster_walk_srec<L, 4>;
    return layout == 3 ? &k_cluster_walk<L, 3> : &k_cluster_walk<L, 4>;
}

template <int L> static void (*pick_cluster_adjoint(int layout))(AdjWalkParams) {
    return layout == 3 ? &k_cluster_adjoint<L, 3> : &k_cluster_adjoint<L, 4>;
}

template <int L> static void (*pick_persistent(int layout))(PersistParams) {
    switch (layout) {
        case 0: return &k_persistent<L, 0>;
        case 1: return &k_persistent<L, 1>;
        case 2: return &k_persistent<L, 2>;
        case 3: return &k_persistent<L, 3>;
        default: return &k_persistent<L, 4>;
    }
}

// The adjoint reads tet records (layouts 0 and 1) or the forward's streamed incidence records.
template <int L> static void (*pick_adj_sweep(int layout))(AdjParams) {
    switch (layout) {
        case 2: return &k_adj_sweep<L, 2>;
        case 3: return &k_adj_sweep<L, 3>;
        case 4: return &k_adj_sweep<L, 4>;
        default: return &k_adj_sweep<L, 0>;
    }
}

// Key of a captured step / solve graph: everything baked into its kernel parameters.
struct GraphKey {
    int kind;  // 0 = step, 1 = solve, 2 = single sweep
    int iters, accel, init, lanes, layout, prefetch, pdl, block, semantics, l2_prefetch, src;
    int record_cache, persist_mb, energy_every, walk;  // walk: 2 = the adjoint sweeps as a cluster walk
    unsigned long long colour_shape;  // hash of the per-colour lanes (0 = uniform) and the mesh
    float h, dtsr, hg[3], rho;
    bool operator==(const GraphKey& o) const { return std::memcmp(this, &o, sizeof(GraphKey)) == 0; }
};

struct GraphEntry {
    GraphKey key;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    size_t nodes = 0;
};

}  // namespace vbd

struct vbd_solver {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int N = 0, T = 0, C = 0, nfree = 0;
    long long ninc = 0;
    bool ready = false, have_materials = false;
    std::vector<int> cstart;  // colour c = internal ids [cstart[c], cstart[c+1])
    std::vector<int32_t> h_inc_off;  // incidence offsets of the internal vertices (host copy)
    vbd::DBuf<float4> x0, x1, pp, y, v, xprev;
    vbd::DBuf<int> perm, inc_off, inc_tet;
    vbd::DBuf<vbd::TetRec> rec, irec;
    vbd::DBuf<int4> crec;                           // compact (layout 2) or factored (layout 3) records
    vbd::DBuf<float2> cmat;
    vbd::DBuf<int> inc_vertex;                      // internal vertex of each incidence
    vbd::DBuf<float> stage, mat_stage;
    vbd::DBuf<unsigned long long> status;
    vbd::DBuf<double> partials, scalar;
    // defaults: 64-thread blocks, programmatic dependent launch and graphs; lanes, layout and
    // record prefetch are chosen at init from the mesh (below) until their options are set
    int lanes = 8, layout = 3, use_graph = 1, timing = 0, prefetch = 1, pdl = 1, block = 64;
    // Until VBD_OPT_LANES is set, init picks the lane count: 8 lanes when the free vertices average
    // at least 21 incident tets (the 64^3 cube: 22.9, 5.04 vs 5.49 ms/step with 4), else 4 (the
    // 512-block batch: 19.5, 9.06 vs 10.2 ms/step with 8); then doubled, up to 16, while the
    // largest colour would still fill less than half of the GPU's resident threads (taken as 1024
    // per SM, the sweep's occupancy at 60-64 registers): a small mesh leaves SMs idle, and more lanes per vertex shorten
    // each vertex's dependent chain (the 2,673-vertex beam: 24.7 / 19.3 / 17.2 ms per 30 steps
    // with 4 / 8 / 16 lanes).
    bool lanes_auto = true;
    bool layout_auto = true;  // layout 4 when the ids fit its 21-bit fields, else 3 (at init)
    bool prefetch_auto = true;  // see eff_prefetch
    int max_valence = 0;        // most incident tets of any free vertex
    // VBD_OPT_L2_PREFETCH: each colour sweep prefetches the next colour's streamed records into L2.
    // Off by default: on the 64^3 cube it measured 5.48 against 4.78 ms/step (the extra DRAM
    // traffic competes with the running colour's own stream).
    int l2_prefetch = 0;
    // VBD_OPT_RECORD_CACHE: the factored records are loaded with an L2 policy, evict-first except
    // the first persist_mb megabytes of the record stream (VBD_OPT_RECORD_PERSIST_MB), which are
    // loaded evict-last so that they stay in L2 from one sweep to the next.
    // Until they are set, vbd_solver_init turns the evict-first stream on (64^3 cube: 4.12 against
    // 4.46 ms/step) with a 32 MB evict-last prefix when the vertex state (four float4 arrays) fits
    // in 32 MB (cube: 4.08 ms; 64 MB: 4.21, 96 MB: 4.45 -- the prefix then competes with the state).
    int record_cache = 1, persist_mb = 32;
    bool record_cache_auto = true, persist_auto = true;
    // Per-colour threads per vertex (vbd_solver_set_colour_lanes); empty = `lanes` for every colour.
    // Graph keys carry a hash of the per-colour lanes and of the mesh generation (shape_gen, bumped
    // by every vbd_solver_init), so a shape set again reuses its captured graph.
    std::vector<int> colour_lanes;
    std::vector<int> colour_maxval;     // most incident tets of a free vertex, per colour
    int shape_gen = 0;
    // VBD_OPT_ENERGY_EVERY: vbd_solver_step appends VBDsolver::computeTotalEnergy after iterations
    // 0, k, 2k, ... of every sub-step (VBD.cpp:93-95 with k = 10) to a device-side history, read by
    // vbd_solver_energy_history.  ehist_queued counts the values enqueued since the last reset.
    int energy_every = 0;
    vbd::DBuf<double> ehist;
    vbd::DBuf<int> ecount;
    long long ehist_queued = 0;
    std::vector<long long> colour_inc;  // first incidence of each colour (C + 1 entries)
    // VBD_OPT_SEMANTICS: 0 = VBDsolver (VBD.cpp), 1 = VBD_GPU_Solver (VBD_GPU_Wrapper.cu)
    int semantics = 0;
    float omega_next(int k, float rho, float prev) const {
        return semantics ? vbd::omega_of_wrapper(k, rho, prev) : vbd::omega_of(k, rho, prev);
    }
    // whole step in one launch: 1 = cooperative kernel with grid barriers, 2 = one thread-block
    // cluster holding the positions in shared memory (meshes of up to about 7,000 vertices)
    int persistent = 0;
    int cluster_ctas_opt = 0;                       // CTAs of the cluster walk (0 = from the colour sizes)
    int cluster_resident = 1;  // the walk keeps each CTA's element records in shared memory where they fit
    // the resident walk's plan for the mesh, kernel and CTA count it was made for
    int sr_gen = -1, sr_ctas = 0, sr_records = 0, sr_owned = 0, sr_slices = 0;
    const void* sr_fn = nullptr;
    unsigned long long sr_smem = 0;
    bool sr_ok = false;
    // launch shape resolved for the mesh, the kernel and the requested CTAs (the kernel's shared-memory
    // and cluster-size attributes are set per kernel)
    int cl_ctas = 0, cl_block = 0, cl_gen = -1, cl_req = 0;
    const void* cl_fn = nullptr;
    int ca_ctas = 0, ca_gen = -1, ca_req = 0;  // the same for the adjoint walk
    const void* ca_fn = nullptr;
    vbd::DBuf<float> d_adj_omega;
    std::vector<float> adj_omega_cache;
    long long spin_limit = 1LL << 22;               // barrier polls before a persistent launch gives up
    vbd::DBuf<int> d_cstart;
    vbd::DBuf<float> d_omega;
    vbd::DBuf<vbd::GridBarrier> barrier;
    std::vector<float> omega_cache;
    int adj_alternate = 0;  // adjoint sweeps alternate the colour order (symmetric Gauss-Seidel pairs)
    // adjoint tape: sub-steps taken since vbd_solver_record, (x, v) every ckpt_every sub-steps
    struct TapeStep {
        float h, dtsr, hg[3], rho;
        int iters, accel;
    };
    std::vector<TapeStep> tape;
    int ckpt_every = 0;
    std::vector<std::unique_ptr<vbd::DBuf<float4>>> ckpts;  // 2N each: x then v
    vbd::DBuf<float4> adj_lam, adj_lam2, adj_lpp, adj_G, adj_ax, adj_av, adj_seg, adj_save;
    // converged positions of the recorded sub-steps of the newest segment, kept as the forward runs
    // so that the backward starts without recomputing that segment
    vbd::DBuf<float4> live_seg;
    vbd::DBuf<float> adj_gmu, adj_glam;
    int adj_cur = 0;  // which of adj_lam / adj_lam2 holds lam
    long long launches = 0;
    std::vector<vbd::GraphEntry> graphs;
    std::vector<double> colour_bytes;               // algorithmic bytes of one sweep of colour c
    std::vector<cudaEvent_t> ev_pool;               // event pairs of timed sweeps
    std::vector<double> ev_bytes;                   // bytes of each timed sweep
    size_t ev_used = 0;                             // pairs in use
    double timed_ms = 0.0, timed_bytes = 0.0;
    long long timed_launches = 0;

    ~vbd_solver() {
        drop_graphs();
        for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }

    // Folds the recorded event pairs into the running totals (synchronises on the last one).
    int collect_timing() {
        if (ev_used == 0) return VBD_OK;
        CUDA_TRY(cudaEventSynchronize(ev_pool[2 * ev_used - 1]));
        for (size_t k = 0; k < ev_used; ++k) {
            float ms = 0.f;
            CUDA_TRY(cudaEventElapsedTime(&ms, ev_pool[2 * k], ev_pool[2 * k + 1]));
            timed_ms += ms;
            timed_bytes += ev_bytes[k];
        }
        timed_launches += (long long)ev_used;
        ev_used = 0;
        ev_bytes.clear();
        return VBD_OK;
    }

    int timing_event(cudaEvent_t* out) {
        if (ev_pool.size() < 2 * (ev_used + 1)) {
            if (ev_used >= 4096) VBD_TRY(collect_timing());
            while (ev_pool.size() < 2 * (ev_used + 1)) {
                cudaEvent_t e;
                CUDA_TRY(cudaEventCreate(&e));
                ev_pool.push_back(e);
            }
        }
        out[0] = ev_pool[2 * ev_used];
        out[1] = ev_pool[2 * ev_used + 1];
        return VBD_OK;
    }

    void drop_graphs() {
        for (auto& g : graphs) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            if (g.graph) cudaGraphDestroy(g.graph);
        }
        graphs.clear();
    }

    // The record prefetch the sweeps run.  Until VBD_OPT_PREFETCH is set: 2 (the lane's first three
    // records before the dependency wait) with the packed records when no lane holds more than
    // three records, else 1.  Measured on the 64^3 cube (8 lanes, at most 3 records a lane): 4.46
    // against 4.55 ms/step; on the 512-mesh batch (4 lanes, up to 6): 7.72 against 7.44 (both
    // before PREFETCH 1 was held to 56 registers, which brought the cube to 4.48 and the batch to
    // 7.10).
    int eff_prefetch() const { return prefetch_for(lanes, max_valence); }
    int prefetch_for(int L, int maxval) const {
        if (!prefetch_auto) return prefetch;
        return (layout == 4 && L > 0 && (maxval + L - 1) / L <= 3) ? 2 : 1;
    }
    int lanes_of(int c) const { return colour_lanes.empty() ? lanes : colour_lanes[c]; }
    int prefetch_of(int c) const {
        return colour_lanes.empty() ? eff_prefetch() : prefetch_for(colour_lanes[c], colour_maxval[c]);
    }
    // First incidence whose record is loaded evict-first (records before it evict-last).
    int persist_end() const {
        if (!record_cache || persist_mb <= 0) return 0;
        const double rec_bytes = layout == 4 ? 40.0 : 48.0;
        const double n = (double)persist_mb * 1048576.0 / rec_bytes;
        return (int)std::min<double>(n, (double)ninc);
    }
    // The launch-shape fields of a graph key.
    void shape_key(vbd::GraphKey& key) const {
        key.lanes = lanes;
        key.layout = layout;
        key.prefetch = eff_prefetch();
        key.pdl = pdl;
        key.block = block;
        key.semantics = semantics;
        key.l2_prefetch = l2_prefetch;
        key.record_cache = record_cache;
        key.persist_mb = persist_mb;
        unsigned long long h = 1469598103934665603ull ^ (unsigned long long)shape_gen;  // FNV-1a
        for (int L : colour_lanes) h = (h ^ (unsigned long long)L) * 1099511628211ull;
        key.colour_shape = colour_lanes.empty() ? (unsigned long long)shape_gen : h;
        key.energy_every = energy_every;
    }

    // Energies a step of `substeps` x `iters` appends to the history.
    long long energies_per_step(int substeps, int iters) const {
        if (energy_every <= 0 || iters <= 0) return 0;
        return (long long)substeps * ((iters + energy_every - 1) / energy_every);
    }

    // Room in the history for `more` values after those already queued; a larger buffer keeps the
    // queued values (captured graphs bake the buffer's address, so they are dropped).
    int reserve_energies(long long more) {
        if (!ecount.p) {
            VBD_TRY(ecount.alloc(1));
            CUDA_TRY(cudaMemsetAsync(ecount.p, 0, sizeof(int), stream));
        }
        const long long need = ehist_queued + more;
        if (need <= (long long)ehist.n) return VBD_OK;
        if (need > 0x7fffffffLL) VBD_FAIL(VBD_ERR_INVALID_ARG, "energy history is full: read it with reset");
        vbd::DBuf<double> bigger;
        VBD_TRY(bigger.alloc((size_t)std::max<long long>(2 * need, 64)));
        if (ehist_queued > 0 && ehist.p)
            CUDA_TRY(cudaMemcpyAsync(bigger.p, ehist.p, sizeof(double) * (size_t)std::min<long long>(ehist_queued, ehist.n),
                                     cudaMemcpyDeviceToDevice, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        drop_graphs();
        std::swap(ehist.p, bigger.p);
        std::swap(ehist.n, bigger.n);
        return VBD_OK;
    }

    // VBDsolver::computeTotalEnergy (log-J elastic energy, FP64 sums) of positions X, appended to
    // the history.
    int emit_energy_append(const float4* X) {
        const unsigned blocks = std::max(1u, std::min<unsigned>(vbd::nblk(T, 256), 4096u));
        vbd::k_energy<<<blocks, 256, 0, stream>>>(X, y.p, rec.p, 0, T, 1, 0.0, partials.p);
        VBD_TRY(check_launch());
        vbd::k_sum_partials_append<<<1, 1024, 0, stream>>>(partials.p, (int)blocks, ehist.p, ecount.p, (int)ehist.n);
        return check_launch();
    }

    int check_launch() {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) VBD_FAIL(VBD_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
        ++launches;
        return VBD_OK;
    }

    int launch_sweep(int c, float4* xr, float4* xn, bool accel, bool keep_pp, float dtsr, float omega) {
        const int vb = cstart[c], ve = cstart[c + 1];
        if (ve <= vb) return VBD_OK;
        vbd::SweepParams p{xr,     xn,     pp.p,     y.p, inc_off.p, inc_tet.p, rec.p,          irec.p,
                           crec.p, cmat.p, status.p, vb,  ve,        dtsr,      omega, accel ? 1 : 0,
                           keep_pp ? 1 : 0, persist_end(), 0};
        if (l2_prefetch && layout >= 2 && crec.p && C > 0) {
            // the colour swept after this one (colour 0 of the next iteration after the last)
            const int cn = (c + 1) % C;
            const long long j0 = colour_inc[cn], j1 = colour_inc[cn + 1];
            const int words = layout == 4 ? 2 : 3;  // int4 per incidence in crec
            p.l2_next = reinterpret_cast<const char*>(crec.p + words * j0);
            p.l2_bytes = (unsigned long long)(j1 - j0) * 16ull * words;
        }
        const int L = lanes_of(c);
        long long threads = (long long)(ve - vb) * L;
        vbd::SweepFn fn = vbd::pick_sweep(L, layout, prefetch_of(c), record_cache != 0);
        int threads_per_block = block;
        if (semantics) threads = (long long)(ve - vb) * vbd::kWrapperLanes;
        cudaEvent_t ev[2] = {nullptr, nullptr};
        if (timing) {
            VBD_TRY(timing_event(ev));
            CUDA_TRY(cudaEventRecord(ev[0], stream));
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(vbd::nblk(threads, threads_per_block));
        cfg.blockDim = dim3(threads_per_block);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = (pdl && !timing) ? 1 : 0;
        if (semantics) {
            const vbd::WrapperParams w{p.x,    p.xnext,  p.pp,    p.y,    p.inc_off, p.inc_tet, p.rec,   p.irec,  p.crec,
                                       p.cmat, p.status, p.v_begin, p.v_end, p.dtsr, p.omega, p.accel, p.keep_pp, nullptr};
            cfg.gridDim = dim3(vbd::nblk(threads, vbd::kWrapperBlock));
            cfg.blockDim = dim3(vbd::kWrapperBlock);
            CUDA_TRY(cudaLaunchKernelEx(&cfg, &vbd::k_sweep_wrapper, w));
        } else {
            CUDA_TRY(cudaLaunchKernelEx(&cfg, fn, p));
        }
        VBD_TRY(check_launch());
        if (timing) {
            CUDA_TRY(cudaEventRecord(ev[1], stream));
            ev_bytes.push_back(colour_bytes[c]);
            ++ev_used;
        }
        return VBD_OK;
    }

    // `iters` sweeps with the Chebyshev schedule; `cur` tracks which buffer holds x.  With
    // record_energy, the log-J energy of the blended positions is appended after iterations 0, k,
    // 2k, ... (k = energy_every), where VBDsolver::step evaluates it (VBD.cpp:93-95).
    int emit_iterations(int iters, float dtsr, bool accel, float rho, int& cur, bool record_energy = false) {
        float omega = 1.0f;
        for (int k = 1; k <= iters; ++k) {
            bool blend = false;
            if (accel) {
                omega = omega_next(k, rho, omega);
                blend = omega > 1.0f;
            }
            float4* xr = cur ? x1.p : x0.p;
            float4* xo = cur ? x0.p : x1.p;
            for (int c = 0; c < C; ++c) VBD_TRY(launch_sweep(c, xr, xo, blend, accel, dtsr, omega));
            if (blend) cur ^= 1;
            if (record_energy && energy_every > 0 && (k - 1) % energy_every == 0)
                VBD_TRY(emit_energy_append(cur ? x1.p : x0.p));
        }
        return VBD_OK;
    }

    int emit_substep(float h, float dtsr, const float* hg, int iters, bool accel, float rho,
                     bool record_energy = false) {
        vbd::k_predict<<<vbd::nblk(N, 256), 256, 0, stream>>>(x0.p, v.p, xprev.p, y.p, nfree, N, h, hg[0], hg[1],
                                                              hg[2]);
        VBD_TRY(check_launch());
        if (semantics) {
            // main.cpp's GPU loop: solveVBD starts every substep from the inertial target
            // (VBD_GPU_Wrapper.cu:334)
            vbd::k_copy_xyz<<<vbd::nblk(N, 256), 256, 0, stream>>>(y.p, x0.p, x1.p, N);
            VBD_TRY(check_launch());
        }
        int cur = 0;
        VBD_TRY(emit_iterations(iters, dtsr, accel, rho, cur, record_energy));
        if (nfree > 0) {
            vbd::k_finish<<<vbd::nblk(nfree, 256), 256, 0, stream>>>(cur ? x1.p : x0.p, x0.p, xprev.p, v.p, nfree, h,
                                                                     cur, 1);
            VBD_TRY(check_launch());
        }
        return VBD_OK;
    }

    int emit_solve(int iters, float dtsr, bool accel, float rho, int init) {
        if (init == VBD_INIT_FROM_INERTIA) {
            vbd::k_copy_xyz<<<vbd::nblk(N, 256), 256, 0, stream>>>(y.p, x0.p, x1.p, N);
            VBD_TRY(check_launch());
        }
        int cur = 0;
        VBD_TRY(emit_iterations(iters, dtsr, accel, rho, cur));
        if (cur && nfree > 0) {
            vbd::k_finish<<<vbd::nblk(nfree, 256), 256, 0, stream>>>(x1.p, x0.p, nullptr, nullptr, nfree, 1.0f, 1, 0);
            VBD_TRY(check_launch());
        }
        return VBD_OK;
    }

    // Chebyshev weights of `iters` iterations (1 where no blend happens).
    std::vector<float> omega_schedule(int iters, bool accel, float rho) const {
        std::vector<float> w(std::max(iters, 1), 1.0f);
        float omega = 1.0f;
        for (int k = 1; k <= iters; ++k) {
            if (accel) omega = omega_next(k, rho, omega);
            w[k - 1] = accel ? omega : 1.0f;
        }
        return w;
    }

    // The colour starts and the Chebyshev schedule on the device, for the single-launch walks.
    int upload_schedule(int iters, bool accel, float rho) {
        if (d_cstart.n != cstart.size()) {
            VBD_TRY(d_cstart.alloc(cstart.size()));
            CUDA_TRY(cudaMemcpy(d_cstart.p, cstart.data(), sizeof(int) * cstart.size(), cudaMemcpyHostToDevice));
        }
        std::vector<float> w = omega_schedule(iters, accel, rho);
        if (w != omega_cache) {
            if (d_omega.n < w.size()) VBD_TRY(d_omega.alloc(w.size()));
            CUDA_TRY(cudaMemcpyAsync(d_omega.p, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice, stream));
            CUDA_TRY(cudaStreamSynchronize(stream));
            omega_cache = w;
        }
        return VBD_OK;
    }

    // The parameters of a single-launch walk (the persistent kernel or the cluster walk).
    vbd::PersistParams walk_params(int iters, float dtsr, bool accel, bool predict, bool finish, bool from_inertia,
                                   float h, const float* hg) const {
        vbd::PersistParams w{};
        w.sw = vbd::SweepParams{x0.p, x1.p, pp.p, y.p,  inc_off.p, inc_tet.p, rec.p, irec.p, crec.p, cmat.p,
                                status.p, 0,  0,    dtsr, 1.0f,      0,         accel ? 1 : 0, 0, 0};
        w.xa = x0.p;
        w.xb = x1.p;
        w.v = v.p;
        w.xprev = xprev.p;
        w.cstart = d_cstart.p;
        w.omega = d_omega.p;
        w.ncol = C;
        w.iters = iters;
        w.nfree = nfree;
        w.n = N;
        w.predict = predict ? 1 : 0;
        w.finish = finish ? 1 : 0;
        w.init_from_inertia = from_inertia ? 1 : 0;
        w.h = h;
        w.hgx = hg ? hg[0] : 0.f;
        w.hgy = hg ? hg[1] : 0.f;
        w.hgz = hg ? hg[2] : 0.f;
        return w;
    }

    int launch_persistent(int iters, float dtsr, bool accel, float rho, bool predict, bool finish, bool from_inertia,
                          float h, const float* hg, int expected_extra = 0) {
        if (!barrier.p) VBD_TRY(barrier.alloc(1));
        VBD_TRY(upload_schedule(iters, accel, rho));
        const int L = lanes < 4 ? 4 : lanes;
        const int threads = 256;
        void (*fn)(vbd::PersistParams) = nullptr;
        switch (L) {
            case 4: fn = vbd::pick_persistent<4>(layout); break;
            case 8: fn = vbd::pick_persistent<8>(layout); break;
            case 16: fn = vbd::pick_persistent<16>(layout); break;
            default: fn = vbd::pick_persistent<32>(layout); break;
        }
        int per_sm = 0, sms = 0;
        CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, 0));
        CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        if (per_sm < 1) VBD_FAIL(VBD_ERR_CUDA, "persistent kernel cannot be resident");
        const int grid = per_sm * sms;
        vbd::PersistParams pp_ = walk_params(iters, dtsr, accel, predict, finish, from_inertia, h, hg);
        pp_.bar = barrier.p;
        pp_.spin_limit = spin_limit;
        pp_.expected_blocks = grid + expected_extra;
        CUDA_TRY(cudaMemsetAsync(barrier.p, 0, sizeof(vbd::GridBarrier), stream));
        void* args[] = {&pp_};
        CUDA_TRY(cudaLaunchCooperativeKernel(reinterpret_cast<void*>(fn), dim3(grid), dim3(threads), args, 0, stream));
        return check_launch();
    }

    // The cluster walk holds both position buffers of the mesh and the pre-sweep positions in each
    // CTA's shared memory.
    size_t cluster_smem() const { return 3 * sizeof(float4) * (size_t)N; }
    bool cluster_fit(const char** why) const {
        if (semantics) {
            *why = "the cluster walk runs the VBDsolver semantics only";
            return false;
        }
        if (layout != 3 && layout != 4) {
            *why = "the cluster walk reads the factored records (VBD_OPT_LAYOUT 3 or 4)";
            return false;
        }
        int optin = 0;
        if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) != cudaSuccess ||
            cluster_smem() + 64 > (size_t)optin) {  // + the walk's two mbarriers
            *why = "the mesh's positions (48 B per vertex) do not fit in one CTA's shared memory";
            return false;
        }
        return true;
    }

    // CTAs of the cluster walk: enough 256-thread CTAs for the largest colour in one round, at most
    // 16, fewer when the device cannot hold a cluster of that size.
    // Enough CTAs of the cluster walk to sweep the largest colour at L lanes in one round, at most 16.
    int cluster_auto_ctas(int L) const {
        int maxcol = 1;
        for (int c = 0; c < C; ++c) maxcol = std::max(maxcol, cstart[c + 1] - cstart[c]);
        const long long need = (long long)maxcol * L;
        const int block = vbd::kClusterMaxBlock;
        return (int)std::max<long long>(1, std::min<long long>(16, (need + block - 1) / block));
    }

    template <class Params>
    int cluster_ctas_for(void (*fn)(Params), int L, size_t smem, int* out) {
        const int block = vbd::kClusterMaxBlock;
        int ctas = cluster_ctas_opt > 0 ? cluster_ctas_opt : cluster_auto_ctas(L);
        CUDA_TRY(cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)smem));
        CUDA_TRY(cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributeNonPortableClusterSizeAllowed,
                                      1));
        for (; ctas >= 1; --ctas) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(ctas);
            cfg.blockDim = dim3(block);
            cfg.dynamicSmemBytes = smem;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = ctas;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            int clusters = 0;
            const cudaError_t e = cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg);
            if (e == cudaSuccess && clusters >= 1) break;
            (void)cudaGetLastError();
            if (cluster_ctas_opt > 0) VBD_FAIL(VBD_ERR_INVALID_ARG, "a cluster of %d CTAs cannot be resident", ctas);
        }
        if (ctas < 1) VBD_FAIL(VBD_ERR_CUDA, "the cluster walk cannot be resident");
        *out = ctas;
        return VBD_OK;
    }

    int resolve_cluster(void (*fn)(vbd::PersistParams), int L) {
        const void* f = reinterpret_cast<const void*>(fn);
        if (cl_gen == shape_gen && cl_fn == f && cl_req == cluster_ctas_opt && cl_ctas > 0) return VBD_OK;
        cl_ctas = 0;
        VBD_TRY(cluster_ctas_for(fn, L, cluster_smem(), &cl_ctas));
        cl_block = vbd::kClusterMaxBlock;
        cl_fn = f;
        cl_gen = shape_gen;
        cl_req = cluster_ctas_opt;
        return VBD_OK;
    }

    // The adjoint walk holds X, both adjoint buffers and the pre-sweep adjoint: 64 B per vertex.
    size_t cluster_adj_smem() const { return 4 * sizeof(float4) * (size_t)N; }
    bool cluster_adj_fit() const {
        int optin = 0;
        return semantics == 0 && (layout == 3 || layout == 4) &&
               cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) == cudaSuccess &&
               cluster_adj_smem() + 64 <= (size_t)optin;
    }
    // With the cluster walk selected, the adjoint sweeps of a sub-step run as one cluster launch
    // too where the mesh fits.
    bool adj_walk() const { return persistent == 2 && !timing && cluster_adj_fit(); }

    // Set-up of the adjoint walk outside any graph capture: the sweep schedule on the device and
    // the cluster shape.
    int prepare_adj_walk(int sweeps, float rho, void (**fn_out)(vbd::AdjWalkParams)) {
        std::vector<float> w(std::max(sweeps, 1), 1.0f);
        float omega = 1.0f;
        for (int it = 1; it <= sweeps; ++it) {
            if (rho > 0.0f) omega = vbd::omega_of(it, rho, omega);
            w[it - 1] = rho > 0.0f ? omega : 1.0f;
        }
        if (w != adj_omega_cache) {
            if (d_adj_omega.n < w.size()) VBD_TRY(d_adj_omega.alloc(w.size()));
            CUDA_TRY(cudaMemcpyAsync(d_adj_omega.p, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice, stream));
            CUDA_TRY(cudaStreamSynchronize(stream));
            adj_omega_cache = w;
        }
        if (d_cstart.n != cstart.size()) {
            VBD_TRY(d_cstart.alloc(cstart.size()));
            CUDA_TRY(cudaMemcpy(d_cstart.p, cstart.data(), sizeof(int) * cstart.size(), cudaMemcpyHostToDevice));
        }
        const int L = lanes < 4 ? 4 : lanes;
        void (*fn)(vbd::AdjWalkParams) = nullptr;
        switch (L) {
            case 4: fn = vbd::pick_cluster_adjoint<4>(layout); break;
            case 8: fn = vbd::pick_cluster_adjoint<8>(layout); break;
            case 16: fn = vbd::pick_cluster_adjoint<16>(layout); break;
            default: fn = vbd::pick_cluster_adjoint<32>(layout); break;
        }
        const void* f = reinterpret_cast<const void*>(fn);
        if (!(ca_gen == shape_gen && ca_fn == f && ca_req == cluster_ctas_opt && ca_ctas > 0)) {
            ca_ctas = 0;
            VBD_TRY(cluster_ctas_for(fn, L, cluster_adj_smem(), &ca_ctas));
            ca_fn = f;
            ca_gen = shape_gen;
            ca_req = cluster_ctas_opt;
        }
        *fn_out = fn;
        return VBD_OK;
    }

    // The adjoint sweeps of one sub-step as one cluster launch, from the live buffer adj_cur.
    int launch_cluster_adjoint(void (*fn)(vbd::AdjWalkParams), const TapeStep& t, const float4* X, int sweeps,
                               float rho) {
        vbd::AdjWalkParams w{};
        w.a = vbd::AdjParams{X,      nullptr, adj_G.p, y.p,  inc_off.p, inc_tet.p, rec.p,
                             crec.p, cmat.p,  t.dtsr,  0,    0,         nullptr,   nullptr,
                             1.0f,   0,       0};
        w.lam0 = adj_cur ? adj_lam2.p : adj_lam.p;
        w.lam1 = adj_cur ? adj_lam.p : adj_lam2.p;
        w.cstart = d_cstart.p;
        w.omega = d_adj_omega.p;
        w.status = status.p;
        w.ncol = C;
        w.sweeps = sweeps;
        w.n = N;
        w.nfree = nfree;
        w.keep_pp = rho > 0.0f ? 1 : 0;
        w.alternate = adj_alternate;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(ca_ctas);
        cfg.blockDim = dim3(vbd::kClusterMaxBlock);
        cfg.dynamicSmemBytes = cluster_adj_smem();
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = ca_ctas;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CUDA_TRY(cudaLaunchKernelEx(&cfg, fn, w));
        return check_launch();
    }

    // Per-CTA sizes of the resident walk for L lanes and `ctas` CTAs of kClusterMaxBlock threads: the
    // (colour, round) slices, and the most records and vertices any CTA sweeps (the kernel derives
    // the same plan, k_cluster_walk_srec).
    void srec_plan(int L, int ctas, int* records, int* owned, int* slices) const {
        const int gpc = vbd::kClusterMaxBlock / L, G = ctas * gpc;
        int S = 0, rec_max = 0, own_max = 0;
        for (int c = 0; c < C; ++c) S += (cstart[c + 1] - cstart[c] + G - 1) / G;
        for (int k = 0; k < ctas; ++k) {
            long long rec = 0, own = 0;
            for (int c = 0; c < C; ++c) {
                const int vb = cstart[c], ve = cstart[c + 1];
                for (int r = 0; r * G < ve - vb; ++r) {
                    const int vf = vb + r * G + k * gpc;
                    const int cnt = std::max(0, std::min(vf + gpc, ve) - vf);
                    own += cnt;
                    if (cnt) rec += h_inc_off[vf + cnt] - h_inc_off[vf];
                }
            }
            rec_max = (int)std::max<long long>(rec_max, rec);
            own_max = (int)std::max<long long>(own_max, own);
        }
        *records = rec_max;
        *owned = own_max;
        *slices = S;
    }

    // A sub-step (predict and finish) or a solve as one cluster launch: vbd::k_cluster_walk_srec where
    // the CTAs' element data fits in shared memory (and VBD_OPT_CLUSTER_RESIDENT allows it), else
    // vbd::k_cluster_walk.
    int launch_cluster(int iters, float dtsr, bool accel, float rho, bool predict, bool finish, bool from_inertia,
                       float h, const float* hg) {
        const char* why = nullptr;
        if (!cluster_fit(&why)) VBD_FAIL(VBD_ERR_INVALID_ARG, "%s", why);
        VBD_TRY(upload_schedule(iters, accel, rho));
        const int L = lanes < 4 ? 4 : lanes;
        void (*fn)(vbd::PersistParams) = nullptr;
        void (*fn_res)(vbd::PersistParams) = nullptr;
        switch (L) {
            case 4: fn = vbd::pick_cluster<4>(layout, false); fn_res = vbd::pick_cluster<4>(layout, true); break;
            case 8: fn = vbd::pick_cluster<8>(layout, false); fn_res = vbd::pick_cluster<8>(layout, true); break;
            case 16: fn = vbd::pick_cluster<16>(layout, false); fn_res = vbd::pick_cluster<16>(layout, true); break;
            default: fn = vbd::pick_cluster<32>(layout, false); fn_res = vbd::pick_cluster<32>(layout, true); break;
        }
        VBD_TRY(resolve_cluster(fn, L));
        vbd::PersistParams w = walk_params(iters, dtsr, accel, predict, finish, from_inertia, h, hg);
        size_t smem = cluster_smem();
        if (cluster_resident) {
            const void* f = reinterpret_cast<const void*>(fn_res);
            if (!(sr_gen == shape_gen && sr_fn == f && sr_ctas == cl_ctas)) {
                sr_gen = shape_gen;
                sr_fn = f;
                sr_ctas = cl_ctas;
                sr_ok = false;
                srec_plan(L, cl_ctas, &sr_records, &sr_owned, &sr_slices);
                sr_smem = vbd::srec_layout(N, sr_records, sr_owned, sr_slices, C, layout).total;
                int optin = 0;
                CUDA_TRY(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
                if (sr_smem + 64 <= (unsigned long long)optin) {
                    CUDA_TRY(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sr_smem));
                    CUDA_TRY(cudaFuncSetAttribute(f, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
                    cudaLaunchConfig_t q = {};
                    q.gridDim = dim3(cl_ctas);
                    q.blockDim = dim3(cl_block);
                    q.dynamicSmemBytes = (size_t)sr_smem;
                    cudaLaunchAttribute qa[1];
                    qa[0].id = cudaLaunchAttributeClusterDimension;
                    qa[0].val.clusterDim.x = cl_ctas;
                    qa[0].val.clusterDim.y = 1;
                    qa[0].val.clusterDim.z = 1;
                    q.attrs = qa;
                    q.numAttrs = 1;
                    int clusters = 0;
                    sr_ok = cudaOccupancyMaxActiveClusters(&clusters, fn_res, &q) == cudaSuccess && clusters >= 1;
                    (void)cudaGetLastError();
                }
            }
            if (sr_ok) {
                fn = fn_res;
                smem = (size_t)sr_smem;
                w.srec_records = sr_records;
                w.srec_owned = sr_owned;
                w.srec_slices = sr_slices;
            }
        }
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(cl_ctas);
        cfg.blockDim = dim3(cl_block);
        cfg.dynamicSmemBytes = smem;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = cl_ctas;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        CUDA_TRY(cudaLaunchKernelEx(&cfg, fn, w));
        return check_launch();
    }

    // A sub-step or solve through the single-launch walk VBD_OPT_PERSISTENT selects.
    int launch_walk(int iters, float dtsr, bool accel, float rho, bool predict, bool finish, bool from_inertia,
                    float h, const float* hg) {
        if (persistent == 2) return launch_cluster(iters, dtsr, accel, rho, predict, finish, from_inertia, h, hg);
        return launch_persistent(iters, dtsr, accel, rho, predict, finish, from_inertia, h, hg);
    }

    int snapshot(vbd::DBuf<float4>& dst) {
        const size_t b4 = sizeof(float4) * (size_t)N;
        CUDA_TRY(cudaMemcpyAsync(dst.p, x0.p, b4, cudaMemcpyDeviceToDevice, stream));
        CUDA_TRY(cudaMemcpyAsync(dst.p + N, v.p, b4, cudaMemcpyDeviceToDevice, stream));
        return VBD_OK;
    }

    int record_substep(float h, float dtsr, const float* hg, int iters, bool accel, float rho) {
        if (!ckpt_every) return VBD_OK;
        TapeStep t{h, dtsr, {hg[0], hg[1], hg[2]}, rho, iters, accel ? 1 : 0};
        tape.push_back(t);
        const size_t slot = (tape.size() - 1) % (size_t)ckpt_every;
        CUDA_TRY(cudaMemcpyAsync(live_seg.p + slot * (size_t)N, x0.p, sizeof(float4) * (size_t)N,
                                 cudaMemcpyDeviceToDevice, stream));
        if (tape.size() % (size_t)ckpt_every == 0) {
            ckpts.emplace_back(new vbd::DBuf<float4>());
            VBD_TRY(ckpts.back()->alloc(2 * (size_t)N));
            VBD_TRY(snapshot(*ckpts.back()));
        }
        return VBD_OK;
    }

    // One recorded sub-step again, exactly as it ran (same launch sequence, hence same bits).
    int replay_substep(const TapeStep& t) {
        vbd::GraphKey key{};
        key.kind = 0;
        key.iters = t.iters;
        key.accel = t.accel;
        shape_key(key);
        key.energy_every = 0;  // the recompute appends no energies (the sweeps, hence the bits, are the same)
        key.h = t.h;
        key.dtsr = t.dtsr;
        key.hg[0] = t.hg[0];
        key.hg[1] = t.hg[1];
        key.hg[2] = t.hg[2];
        key.rho = t.rho;
        if (persistent && !timing)
            return launch_walk(t.iters, t.dtsr, t.accel != 0, t.rho, true, true, false, t.h, t.hg);
        return run(key, [&] { return emit_substep(t.h, t.dtsr, t.hg, t.iters, t.accel != 0, t.rho); });
    }

    // Adjoint of one recorded sub-step whose converged positions are X: `sweeps` Gauss-Seidel
    // sweeps on (M/h^2 + H) lam = x~ + c v~ with the Chebyshev blend of weight schedule
    // getAcceleratorOmega(k, rho) (rho = 0: plain Gauss-Seidel), then the parameter gradients, the
    // pinned-vertex coupling and the step's adjoint update.
    int emit_adjoint_substep(const TapeStep& t, const float4* X, int sweeps, float rho,
                             void (*walk)(vbd::AdjWalkParams) = nullptr) {
        const float c = 0.999f / t.h;
        const int L = lanes < 4 ? 4 : lanes;
        vbd::k_adj_rhs<<<vbd::nblk(std::max(nfree, 1), 256), 256, 0, stream>>>(adj_ax.p, adj_av.p, adj_G.p, c, nfree);
        VBD_TRY(check_launch());
        int cur = adj_cur;
        float omega = 1.0f;
        const bool accel = rho > 0.0f;
        if (walk) {
            // all sweeps in one cluster launch; the live buffer afterwards follows the same flips
            VBD_TRY(launch_cluster_adjoint(walk, t, X, sweeps, rho));
            for (int it = 1; it <= sweeps && accel; ++it) {
                omega = vbd::omega_of(it, rho, omega);
                if (omega > 1.0f) cur ^= 1;
            }
        }
        for (int it = 1; it <= sweeps && !walk; ++it) {
            bool blend = false;
            if (accel) {
                omega = vbd::omega_of(it, rho, omega);
                blend = omega > 1.0f;
            }
            float4* lr = cur ? adj_lam2.p : adj_lam.p;
            float4* lo = cur ? adj_lam.p : adj_lam2.p;
            vbd::AdjParams ap{X,         lr,      adj_G.p, y.p,   inc_off.p,     inc_tet.p,     rec.p,
                              crec.p,    cmat.p,  t.dtsr,  0,     0,             lo,            adj_lpp.p,
                              omega,     blend ? 1 : 0,    accel ? 1 : 0};
            const int alay = layout >= 2 ? layout : 0;
            for (int k = 0; k < C; ++k) {
                const int col = (adj_alternate && (it % 2 == 0)) ? C - 1 - k : k;
                ap.v_begin = cstart[col];
                ap.v_end = cstart[col + 1];
                if (ap.v_end <= ap.v_begin) continue;
                void (*fn)(vbd::AdjParams) = nullptr;
                switch (L) {
                    case 4: fn = vbd::pick_adj_sweep<4>(alay); break;
                    case 8: fn = vbd::pick_adj_sweep<8>(alay); break;
                    case 16: fn = vbd::pick_adj_sweep<16>(alay); break;
                    default: fn = vbd::pick_adj_sweep<32>(alay); break;
                }
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3(vbd::nblk((long long)(ap.v_end - ap.v_begin) * L, 128));
                cfg.blockDim = dim3(128);
                cfg.stream = stream;
                cudaLaunchAttribute attr[1];
                attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
                attr[0].val.programmaticStreamSerializationAllowed = 1;
                cfg.attrs = attr;
                cfg.numAttrs = pdl ? 1 : 0;
                CUDA_TRY(cudaLaunchKernelEx(&cfg, fn, ap));
                VBD_TRY(check_launch());
            }
            if (blend) cur ^= 1;
        }
        float4* lam = cur ? adj_lam2.p : adj_lam.p;
        if (T > 0) {
            vbd::k_adj_params<<<vbd::nblk(T, 256), 256, 0, stream>>>(rec.p, X, lam, adj_gmu.p, adj_glam.p, T);
            VBD_TRY(check_launch());
        }
        if (N > nfree) {
            vbd::AdjParams ap{X,      lam,     adj_G.p, y.p,  inc_off.p, inc_tet.p, rec.p,
                              crec.p, cmat.p,  t.dtsr,  nfree, N,        nullptr,   nullptr,
                              1.0f,   0,       0};
            const unsigned grid = vbd::nblk((long long)(N - nfree) * 8, 256);
            vbd::k_adj_pinned<8><<<grid, 256, 0, stream>>>(ap, adj_ax.p);
            VBD_TRY(check_launch());
        }
        if (nfree > 0) {
            vbd::k_adj_update<<<vbd::nblk(nfree, 256), 256, 0, stream>>>(lam, y.p, adj_ax.p, adj_av.p, t.dtsr, c, t.h,
                                                                      nfree);
            VBD_TRY(check_launch());
        }
        return VBD_OK;
    }

    // The adjoint sequence of a sub-step is replayed as a graph keyed by its parameters, the
    // positions slot it reads and which adjoint buffer is live.
    // `src` tells the state buffers apart (0 = recomputed segment, 1 = kept newest segment): the
    // captured graph bakes X's address.
    int adjoint_substep(const TapeStep& t, int slot, const float4* X, int sweeps, float rho, int src) {
        vbd::GraphKey key{};
        key.kind = 3 + slot;
        key.src = src;
        key.iters = sweeps;
        key.init = adj_cur;
        key.lanes = lanes;
        key.layout = layout;
        key.pdl = pdl;
        key.accel = adj_alternate;
        key.h = t.h;
        key.dtsr = t.dtsr;
        key.rho = rho;
        void (*walk)(vbd::AdjWalkParams) = nullptr;
        if (adj_walk()) {
            VBD_TRY(prepare_adj_walk(sweeps, rho, &walk));
            key.walk = 2;
            key.block = ca_ctas;
        }
        VBD_TRY(run(key, [&] { return emit_adjoint_substep(t, X, sweeps, rho, walk); }));
        float omega = 1.0f;
        for (int it = 1; it <= sweeps && rho > 0.0f; ++it) {
            omega = vbd::omega_of(it, rho, omega);
            if (omega > 1.0f) adj_cur ^= 1;
        }
        return VBD_OK;
    }

    template <class Emit> int run(const vbd::GraphKey& key, Emit emit) {
        if (!use_graph || timing) return emit();
        vbd::GraphEntry* hit = nullptr;
        for (auto& g : graphs)
            if (g.key == key) hit = &g;
        if (!hit) {
            vbd::GraphEntry e;
            e.key = key;
            const long long saved = launches;
            CUDA_TRY(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            int rc = emit();
            cudaGraph_t g = nullptr;
            cudaError_t ce = cudaStreamEndCapture(stream, &g);
            launches = saved;
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            if (ce != cudaSuccess) VBD_FAIL(VBD_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
            e.graph = g;
            CUDA_TRY(cudaGraphGetNodes(g, nullptr, &e.nodes));
            cudaError_t ie = cudaGraphInstantiate(&e.exec, g, 0);
            if (ie != cudaSuccess) {
                cudaGraphDestroy(g);
                VBD_FAIL(VBD_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(ie));
            }
            if (graphs.size() >= 64) {
                cudaGraphExecDestroy(graphs.front().exec);
                cudaGraphDestroy(graphs.front().graph);
                graphs.erase(graphs.begin());
            }
            graphs.push_back(e);
            hit = &graphs.back();
        }
        CUDA_TRY(cudaGraphLaunch(hit->exec, stream));
        launches += (long long)hit->nodes;
        return VBD_OK;
    }

    int upload3(const float* src, float4* d0, float4* d1) {
        CUDA_TRY(cudaMemcpyAsync(stage.p, src, sizeof(float) * 3 * (size_t)N, cudaMemcpyDefault, stream));
        vbd::k_scatter3<<<vbd::nblk(N, 256), 256, 0, stream>>>(stage.p, perm.p, d0, d1, N);
        VBD_TRY(check_launch());
        CUDA_TRY(cudaStreamSynchronize(stream));
        return VBD_OK;
    }

    int download3(const float4* src, float* dst) {
        vbd::k_gather3<<<vbd::nblk(N, 256), 256, 0, stream>>>(src, perm.p, stage.p, N);
        VBD_TRY(check_launch());
        CUDA_TRY(cudaMemcpyAsync(dst, stage.p, sizeof(float) * 3 * (size_t)N, cudaMemcpyDefault, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return VBD_OK;
    }

    // Captured graphs bake in buffer addresses: every (re)allocation or release of the streamed
    // record copies invalidates them.
    int repack_stream() {
        if (layout != 1 && irec.p) {
            drop_graphs();
            irec.release();
        }
        if (layout != 2 && layout != 4 && cmat.p) {
            drop_graphs();
            cmat.release();
        }
        if (layout < 2 && crec.p) {
            drop_graphs();
            crec.release();
        }
        if (layout == 1) {
            if (irec.n != (size_t)ninc) {
                drop_graphs();
                VBD_TRY(irec.alloc(ninc));
            }
            if (ninc > 0) {
                vbd::k_pack_stream<<<vbd::nblk(ninc, 256), 256, 0, stream>>>(rec.p, inc_tet.p, irec.p, (int)ninc);
                VBD_TRY(check_launch());
            }
        } else if (layout >= 2) {
            const size_t words = layout == 4 ? 2 : 3;
            if (crec.n != words * (size_t)ninc) {
                drop_graphs();
                VBD_TRY(crec.alloc(words * (size_t)ninc));
            }
            if (layout != 3 && cmat.n != (size_t)ninc) {
                drop_graphs();
                VBD_TRY(cmat.alloc(ninc));
            }
            if (ninc > 0 && layout == 2) {
                vbd::k_pack_compact<<<vbd::nblk(ninc, 256), 256, 0, stream>>>(rec.p, inc_tet.p, inc_vertex.p, crec.p,
                                                                             cmat.p, (int)ninc);
                VBD_TRY(check_launch());
            } else if (ninc > 0 && layout == 3) {
                vbd::k_pack_factored<false><<<vbd::nblk(ninc, 256), 256, 0, stream>>>(
                    rec.p, inc_tet.p, inc_vertex.p, crec.p, nullptr, (int)ninc);
                VBD_TRY(check_launch());
            } else if (ninc > 0) {
                vbd::k_pack_factored<true><<<vbd::nblk(ninc, 256), 256, 0, stream>>>(
                    rec.p, inc_tet.p, inc_vertex.p, crec.p, cmat.p, (int)ninc);
                VBD_TRY(check_launch());
            }
        }
        return VBD_OK;
    }

    int reduce_scalar(unsigned blocks, double* out) {
        vbd::k_sum_partials<<<1, 1024, 0, stream>>>(partials.p, (int)blocks, scalar.p);
        VBD_TRY(check_launch());
        CUDA_TRY(cudaMemcpyAsync(out, scalar.p, sizeof(double), cudaMemcpyDeviceToHost, stream));
        CUDA_TRY(cudaStreamSynchronize(stream));
        return VBD_OK;
    }
};

namespace {

struct DeviceScope {
    int prev = -1;
    explicit DeviceScope(int d) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != d) cudaSetDevice(d);
    }
    ~DeviceScope() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

int need_ready(vbd_solver* s) {
    if (!s) VBD_FAIL(VBD_ERR_INVALID_ARG, "null solver handle");
    if (!s->ready) VBD_FAIL(VBD_ERR_STATE, "solver has no mesh: call vbd_solver_init first");
    return VBD_OK;
}

}  // namespace

extern "C" {

int vbd_solver_create(vbd_solver** out, int device, void* cuda_stream) {
    vbd::clear_error();
    if (!out) VBD_FAIL(VBD_ERR_INVALID_ARG, "out is null");
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        VBD_FAIL(VBD_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= count) VBD_FAIL(VBD_ERR_NO_DEVICE, "device %d out of range (%d devices)", device, count);
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10 || prop.minor != 0)
        VBD_FAIL(VBD_ERR_NO_DEVICE, "device %d is sm_%d%d; this library is built for sm_100a only", device,
                 prop.major, prop.minor);
    DeviceScope scope(device);
    std::unique_ptr<vbd_solver> s(new vbd_solver());
    s->device = device;
    if (cuda_stream) {
        s->stream = static_cast<cudaStream_t>(cuda_stream);
    } else {
        CUDA_TRY(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        s->own_stream = true;
    }
    VBD_TRY(s->status.alloc(vbd::ST_SLOTS));
    CUDA_TRY(cudaMemset(s->status.p, 0, sizeof(unsigned long long) * vbd::ST_SLOTS));
    VBD_TRY(s->scalar.alloc(1));
    *out = s.release();
    return VBD_OK;
}

int vbd_solver_destroy(vbd_solver* s) {
    vbd::clear_error();
    if (!s) return VBD_OK;
    DeviceScope scope(s->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    delete s;
    return VBD_OK;
}

int vbd_solver_init(vbd_solver* s, int32_t N, int32_t T, const float* positions, const float* velocities,
                    const float* inertia, const float* vertex_mass, const uint8_t* fixed, const int32_t* tets,
                    int32_t num_colours, const int32_t* group_offsets, const int32_t* group_vertices,
                    const float* dm_inv, const float* rest_vol, const float* tet_mu, const float* tet_lambda) {
    vbd::clear_error();
    if (!s) VBD_FAIL(VBD_ERR_INVALID_ARG, "null solver handle");
    if (N <= 0) VBD_FAIL(VBD_ERR_INVALID_ARG, "num_verts must be positive (got %d)", N);
    if (T < 0) VBD_FAIL(VBD_ERR_INVALID_ARG, "num_tets is negative");
    if (!positions || !vertex_mass || !fixed) VBD_FAIL(VBD_ERR_INVALID_ARG, "positions, vertex_mass, fixed are required");
    if (T > 0 && (!dm_inv || !rest_vol)) VBD_FAIL(VBD_ERR_INVALID_ARG, "dm_inv and rest_vol are required");
    if (num_colours < 0 || (num_colours > 0 && (!group_offsets || !group_vertices)))
        VBD_FAIL(VBD_ERR_INVALID_ARG, "colour groups missing");
    if ((tet_mu == nullptr) != (tet_lambda == nullptr))
        VBD_FAIL(VBD_ERR_INVALID_ARG, "give both tet_mu and tet_lambda, or neither");
    if ((long long)T * 4 > 0x7fffffffLL) VBD_FAIL(VBD_ERR_INVALID_ARG, "too many tets for 32-bit incidence ids");
    if (!s->layout_auto && s->layout == 4 && N > vbd::kPackedMaxVertices)
        VBD_FAIL(VBD_ERR_INVALID_ARG, "layout 4 holds vertex ids below 2^21; this mesh has %d vertices", N);
    VBD_TRY(vbd::check_tets(N, T, tets));
    // colour groups: a partition of the vertices into independent sets
    if (num_colours == 0 || group_offsets[0] != 0 || group_offsets[num_colours] != N)
        VBD_FAIL(VBD_ERR_INVALID_ARG, "colour groups must cover all %d vertices", N);
    std::vector<int32_t> colour(N, -1);
    for (int c = 0; c < num_colours; ++c) {
        if (group_offsets[c + 1] < group_offsets[c]) VBD_FAIL(VBD_ERR_INVALID_ARG, "colour offsets decrease at %d", c);
        for (int k = group_offsets[c]; k < group_offsets[c + 1]; ++k) {
            int vtx = group_vertices[k];
            if (vtx < 0 || vtx >= N) VBD_FAIL(VBD_ERR_INVALID_ARG, "colour group %d holds vertex %d out of range", c, vtx);
            if (colour[vtx] != -1) VBD_FAIL(VBD_ERR_INVALID_ARG, "vertex %d appears in two colour groups", vtx);
            colour[vtx] = c;
        }
    }
    for (int t = 0; t < T; ++t) {
        const int32_t* q = tets + 4LL * t;
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < a; ++b)
                if (colour[q[a]] == colour[q[b]])
                    VBD_FAIL(VBD_ERR_INVALID_ARG,
                             "colour groups are not independent: vertices %d and %d of tet %d share colour %d", q[a],
                             q[b], t, colour[q[a]]);
    }
    for (int i = 0; i < N; ++i)
        if (!(vertex_mass[i] >= 0.0f) || !std::isfinite(vertex_mass[i]))
            VBD_FAIL(VBD_ERR_INVALID_ARG, "vertex_mass[%d] is negative or not finite", i);

    DeviceScope scope(s->device);
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->ready = false;
    s->drop_graphs();
    s->irec.release();
    s->crec.release();
    s->cmat.release();

    // Internal order: free vertices colour by colour (group order), then the pinned ones.
    std::vector<int32_t> perm;
    perm.reserve(N);
    std::vector<int> cstart(num_colours + 1, 0);
    for (int c = 0; c < num_colours; ++c) {
        cstart[c] = (int)perm.size();
        for (int k = group_offsets[c]; k < group_offsets[c + 1]; ++k)
            if (!fixed[group_vertices[k]]) perm.push_back(group_vertices[k]);
    }
    cstart[num_colours] = (int)perm.size();
    const int nfree = (int)perm.size();
    for (int i = 0; i < N; ++i)
        if (fixed[i]) perm.push_back(i);
    std::vector<int32_t> iperm(N);
    for (int i = 0; i < N; ++i) iperm[perm[i]] = i;

    // Incident tets of each free vertex, ascending tet id (TetMesh::vertAdjacentTets).
    std::vector<int32_t> voff(N + 1), vtets(4LL * T);
    vbd::build_vertex_tets(N, T, tets, voff.data(), vtets.data());
    // Incident tets of every vertex (free ones first, so the sweeps' incidences are [0, ninc); the
    // pinned vertices' lists serve the adjoint's coupling term).
    std::vector<int32_t> inc_off(N + 1, 0);
    for (int i = 0; i < N; ++i) inc_off[i + 1] = inc_off[i] + (voff[perm[i] + 1] - voff[perm[i]]);
    const long long ninc = inc_off[nfree];
    const long long ninc_all = inc_off[N];
    std::vector<int32_t> inc_tet(std::max<long long>(ninc_all, 1)), inc_vertex(std::max<long long>(ninc_all, 1));
    for (int i = 0; i < N; ++i) {
        std::copy(vtets.begin() + voff[perm[i]], vtets.begin() + voff[perm[i] + 1], inc_tet.begin() + inc_off[i]);
        std::fill(inc_vertex.begin() + inc_off[i], inc_vertex.begin() + inc_off[i + 1], i);
    }

    std::vector<vbd::TetRec> rec(std::max(T, 1));
    for (int t = 0; t < T; ++t) {
        const int32_t* q = tets + 4LL * t;
        const float* d = dm_inv + 9LL * t;
        vbd::TetRec& r = rec[t];
        r.ids = make_int4(iperm[q[0]], iperm[q[1]], iperm[q[2]], iperm[q[3]]);
        r.a = make_float4(d[0], d[1], d[2], d[3]);
        r.b = make_float4(d[4], d[5], d[6], d[7]);
        r.c = make_float4(d[8], rest_vol[t], tet_mu ? tet_mu[t] : 0.0f, tet_lambda ? tet_lambda[t] : 0.0f);
    }

    std::vector<float4> hx(N), hv(N), hy(N);
    for (int i = 0; i < N; ++i) {
        const int o = perm[i];
        hx[i] = make_float4(positions[3LL * o], positions[3LL * o + 1], positions[3LL * o + 2], 0.0f);
        hv[i] = velocities ? make_float4(velocities[3LL * o], velocities[3LL * o + 1], velocities[3LL * o + 2], 0.0f)
                           : make_float4(0.f, 0.f, 0.f, 0.f);
        const float* yy = inertia ? inertia + 3LL * o : positions + 3LL * o;
        hy[i] = make_float4(yy[0], yy[1], yy[2], vertex_mass[o]);
    }

    VBD_TRY(s->x0.alloc(N));
    VBD_TRY(s->x1.alloc(N));
    VBD_TRY(s->pp.alloc(N));
    VBD_TRY(s->y.alloc(N));
    VBD_TRY(s->v.alloc(N));
    VBD_TRY(s->xprev.alloc(N));
    VBD_TRY(s->perm.alloc(N));
    VBD_TRY(s->inc_off.alloc(N + 1));
    VBD_TRY(s->inc_tet.alloc(inc_tet.size()));
    VBD_TRY(s->inc_vertex.alloc(inc_vertex.size()));
    VBD_TRY(s->rec.alloc(rec.size()));
    VBD_TRY(s->stage.alloc(3LL * N));
    VBD_TRY(s->mat_stage.alloc(2LL * std::max(T, 1)));
    const long long max_blocks = std::max<long long>(4096, vbd::nblk((long long)N * 32, 256));
    VBD_TRY(s->partials.alloc(max_blocks));
    const size_t b4 = sizeof(float4) * (size_t)N;
    CUDA_TRY(cudaMemcpy(s->x0.p, hx.data(), b4, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(s->x1.p, hx.data(), b4, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(s->xprev.p, hx.data(), b4, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(s->pp.p, hx.data(), b4, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(s->v.p, hv.data(), b4, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(s->y.p, hy.data(), b4, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(s->perm.p, perm.data(), sizeof(int) * N, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(s->inc_off.p, inc_off.data(), sizeof(int) * (N + 1), cudaMemcpyHostToDevice));
    s->h_inc_off = inc_off;  // the cluster walk's resident-record plan reads it on the host
    CUDA_TRY(cudaMemcpy(s->inc_tet.p, inc_tet.data(), sizeof(int) * inc_tet.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(s->inc_vertex.p, inc_vertex.data(), sizeof(int) * inc_vertex.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(s->rec.p, rec.data(), sizeof(vbd::TetRec) * rec.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemset(s->status.p, 0, sizeof(unsigned long long) * vbd::ST_SLOTS));
    // the energy history belongs to the previous mesh
    s->ehist_queued = 0;
    if (s->ecount.p) CUDA_TRY(cudaMemset(s->ecount.p, 0, sizeof(int)));

    if (s->lanes_auto) {
        int L = (nfree > 0 && (double)ninc >= 21.0 * nfree) ? 8 : 4;
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
        long long largest = 0;
        for (int c = 0; c < num_colours; ++c) largest = std::max<long long>(largest, cstart[c + 1] - cstart[c]);
        while (L < 16 && largest * L * 2 <= (long long)sms * 1024) L *= 2;
        s->lanes = L;
    }
    if (s->layout_auto) {
        // Layout 4 derives det M from s and w, which cancels on anisotropic tets (a vertex whose row
        // of Ps Dm^-1 is small next to the others); layout 3 stores det M.  On sliver tets both carry
        // the FP32 conditioning error of Dm^-1 itself, which the reference's own F = Ds Dm^-1 shares.
        // So layout 4 is kept unless it loses accuracy on more than a small fraction of the
        // incidences.
        double e3 = 0.0, e4 = 0.0, f4 = 0.0;
        vbd::factored_detm_error(T, dm_inv, &e3, &e4, &f4);
        s->layout = (N <= vbd::kPackedMaxVertices && f4 <= vbd::kFactoredLossFraction) ? 4 : 3;
    }
    if (s->record_cache_auto) s->record_cache = 1;
    if (s->persist_auto) s->persist_mb = 64.0 * N <= 32.0 * 1048576.0 ? 32 : 0;
    s->max_valence = 0;
    for (int i = 0; i < nfree; ++i) s->max_valence = std::max(s->max_valence, inc_off[i + 1] - inc_off[i]);
    s->colour_maxval.assign(num_colours, 0);
    for (int c = 0; c < num_colours; ++c)
        for (int i = cstart[c]; i < cstart[c + 1]; ++i)
            s->colour_maxval[c] = std::max(s->colour_maxval[c], inc_off[i + 1] - inc_off[i]);
    // a per-colour launch shape belongs to the previous mesh's colours
    s->colour_lanes.clear();
    ++s->shape_gen;
    s->colour_inc.assign(num_colours + 1, 0);
    for (int c = 0; c <= num_colours; ++c) s->colour_inc[c] = inc_off[cstart[c]];
    s->colour_bytes.assign(num_colours, 0.0);
    for (int c = 0; c < num_colours; ++c)
        for (int i = cstart[c]; i < cstart[c + 1]; ++i)
            s->colour_bytes[c] += 60.0 * (inc_off[i + 1] - inc_off[i]) + 96.0;
    s->N = N;
    s->T = T;
    s->C = num_colours;
    s->nfree = nfree;
    s->ninc = ninc;
    s->cstart = cstart;
    s->d_cstart.release();
    s->have_materials = tet_mu != nullptr;
    VBD_TRY(s->repack_stream());
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->ready = true;
    return VBD_OK;
}

int vbd_solver_init_batch(vbd_solver* s, int32_t M, const int32_t* voff, const int32_t* toff, const float* positions,
                          const float* velocities, const float* vertex_mass, const uint8_t* fixed,
                          const int32_t* tets_local, const float* dm_inv, const float* rest_vol, const float* tet_mu,
                          const float* tet_lambda) {
    vbd::clear_error();
    if (!s) VBD_FAIL(VBD_ERR_INVALID_ARG, "null solver handle");
    if (M <= 0 || !voff || !toff) VBD_FAIL(VBD_ERR_INVALID_ARG, "need num_meshes > 0 and the offset arrays");
    if (voff[0] != 0 || toff[0] != 0) VBD_FAIL(VBD_ERR_INVALID_ARG, "offsets must start at 0");
    for (int m = 0; m < M; ++m)
        if (voff[m + 1] < voff[m] || toff[m + 1] < toff[m])
            VBD_FAIL(VBD_ERR_INVALID_ARG, "offsets of mesh %d decrease", m);
    const int32_t N = voff[M], T = toff[M];
    if (T > 0 && !tets_local) VBD_FAIL(VBD_ERR_INVALID_ARG, "tets_local is null");
    // global ids; each mesh's ids must stay inside its own vertex range
    std::vector<int32_t> tets(4LL * T);
    for (int m = 0; m < M; ++m) {
        const int32_t nv = voff[m + 1] - voff[m];
        for (int64_t k = 4LL * toff[m]; k < 4LL * toff[m + 1]; ++k) {
            const int32_t id = tets_local[k];
            if (id < 0 || id >= nv)
                VBD_FAIL(VBD_ERR_INVALID_ARG, "mesh %d: tet %lld holds local vertex id %d outside [0, %d)", m,
                         (long long)(k / 4), id, nv);
            tets[k] = id + voff[m];
        }
    }
    // Greedy colouring of the union: a vertex's neighbours all lie in its own mesh, so every mesh
    // receives exactly its own GraphColoring::colorVertices assignment.
    std::vector<int32_t> colour_of(N);
    int32_t nc = 0;
    VBD_TRY(vbd_color_vertices(N, T, tets.data(), colour_of.data(), &nc, 0, nullptr, nullptr));
    std::vector<int32_t> offs(nc + 1), verts(N);
    VBD_TRY(vbd_color_vertices(N, T, tets.data(), colour_of.data(), &nc, nc, offs.data(), verts.data()));
    return vbd_solver_init(s, N, T, positions, velocities, nullptr, vertex_mass, fixed, tets.data(), nc, offs.data(),
                           verts.data(), dm_inv, rest_vol, tet_mu, tet_lambda);
}

int vbd_solver_set_materials(vbd_solver* s, const float* tet_mu, const float* tet_lambda) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (!tet_mu && !tet_lambda) return VBD_OK;
    if (!s->have_materials && !(tet_mu && tet_lambda))
        VBD_FAIL(VBD_ERR_STATE, "materials were never set: give both tet_mu and tet_lambda");
    DeviceScope scope(s->device);
    if (s->T == 0) {
        s->have_materials = true;
        return VBD_OK;
    }
    float* dmu = nullptr;
    float* dlam = nullptr;
    if (tet_mu) {
        dmu = s->mat_stage.p;
        CUDA_TRY(cudaMemcpyAsync(dmu, tet_mu, sizeof(float) * s->T, cudaMemcpyDefault, s->stream));
    }
    if (tet_lambda) {
        dlam = s->mat_stage.p + s->T;
        CUDA_TRY(cudaMemcpyAsync(dlam, tet_lambda, sizeof(float) * s->T, cudaMemcpyDefault, s->stream));
    }
    vbd::k_set_materials<<<vbd::nblk(s->T, 256), 256, 0, s->stream>>>(s->rec.p, dmu, dlam, -1.f, -1.f, s->T);
    VBD_TRY(s->check_launch());
    VBD_TRY(s->repack_stream());
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    s->have_materials = true;
    return VBD_OK;
}

int vbd_solver_set_uniform_material(vbd_solver* s, float mu, float lambda) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (!(mu >= 0.f) || !(lambda >= 0.f) || !std::isfinite(mu) || !std::isfinite(lambda))
        VBD_FAIL(VBD_ERR_INVALID_ARG, "mu and lambda must be finite and non-negative");
    DeviceScope scope(s->device);
    if (s->T > 0) {
        vbd::k_set_materials<<<vbd::nblk(s->T, 256), 256, 0, s->stream>>>(s->rec.p, nullptr, nullptr, mu, lambda,
                                                                          s->T);
        VBD_TRY(s->check_launch());
        VBD_TRY(s->repack_stream());
        CUDA_TRY(cudaStreamSynchronize(s->stream));
    }
    s->have_materials = true;
    return VBD_OK;
}

int vbd_solver_set_positions(vbd_solver* s, const float* xyz) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (!xyz) VBD_FAIL(VBD_ERR_INVALID_ARG, "xyz is null");
    DeviceScope scope(s->device);
    return s->upload3(xyz, s->x0.p, s->x1.p);
}

int vbd_solver_get_positions(vbd_solver* s, float* xyz) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (!xyz) VBD_FAIL(VBD_ERR_INVALID_ARG, "xyz is null");
    DeviceScope scope(s->device);
    return s->download3(s->x0.p, xyz);
}

int vbd_solver_set_velocities(vbd_solver* s, const float* xyz) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (!xyz) VBD_FAIL(VBD_ERR_INVALID_ARG, "xyz is null");
    DeviceScope scope(s->device);
    return s->upload3(xyz, s->v.p, nullptr);
}

int vbd_solver_get_velocities(vbd_solver* s, float* xyz) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (!xyz) VBD_FAIL(VBD_ERR_INVALID_ARG, "xyz is null");
    DeviceScope scope(s->device);
    return s->download3(s->v.p, xyz);
}

int vbd_solver_set_inertia(vbd_solver* s, const float* xyz) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (!xyz) VBD_FAIL(VBD_ERR_INVALID_ARG, "xyz is null");
    DeviceScope scope(s->device);
    return s->upload3(xyz, s->y.p, nullptr);
}

int vbd_solver_get_inertia(vbd_solver* s, float* xyz) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (!xyz) VBD_FAIL(VBD_ERR_INVALID_ARG, "xyz is null");
    DeviceScope scope(s->device);
    return s->download3(s->y.p, xyz);
}

int vbd_solver_solve(vbd_solver* s, int32_t iterations, float dt_sqr_reciprocal, int32_t use_acceleration, float rho,
                     int32_t init_mode) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (!s->have_materials) VBD_FAIL(VBD_ERR_STATE, "materials not set");
    if (iterations < 0) VBD_FAIL(VBD_ERR_INVALID_ARG, "iterations must be >= 0");
    if (!(dt_sqr_reciprocal > 0.f) || !std::isfinite(dt_sqr_reciprocal))
        VBD_FAIL(VBD_ERR_INVALID_ARG, "dt_sqr_reciprocal must be positive and finite");
    if (init_mode != VBD_INIT_FROM_POSITIONS && init_mode != VBD_INIT_FROM_INERTIA)
        VBD_FAIL(VBD_ERR_INVALID_ARG, "unknown init_mode %d", init_mode);
    DeviceScope scope(s->device);
    vbd::GraphKey key{};
    key.kind = 1;
    key.iters = iterations;
    key.accel = use_acceleration ? 1 : 0;
    key.init = init_mode;
    s->shape_key(key);
    key.dtsr = dt_sqr_reciprocal;
    key.rho = rho;
    if (s->persistent && !s->timing)
        return s->launch_walk(iterations, dt_sqr_reciprocal, use_acceleration != 0, rho, false, false,
                              init_mode == VBD_INIT_FROM_INERTIA, 1.0f, nullptr);
    return s->run(key, [&] { return s->emit_solve(iterations, dt_sqr_reciprocal, use_acceleration != 0, rho, init_mode); });
}

int vbd_solver_solve_iteration(vbd_solver* s, float dt_sqr_reciprocal) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (!s->have_materials) VBD_FAIL(VBD_ERR_STATE, "materials not set");
    if (!(dt_sqr_reciprocal > 0.f) || !std::isfinite(dt_sqr_reciprocal))
        VBD_FAIL(VBD_ERR_INVALID_ARG, "dt_sqr_reciprocal must be positive and finite");
    DeviceScope scope(s->device);
    int cur = 0;
    return s->emit_iterations(1, dt_sqr_reciprocal, false, 0.f, cur);
}

int vbd_solver_step(vbd_solver* s, float dt, int32_t substeps, int32_t iterations, const float* gravity,
                    int32_t use_acceleration, float rho) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (!s->have_materials) VBD_FAIL(VBD_ERR_STATE, "materials not set");
    if (!(dt > 0.f) || !std::isfinite(dt)) VBD_FAIL(VBD_ERR_INVALID_ARG, "dt must be positive and finite");
    if (substeps < 1) VBD_FAIL(VBD_ERR_INVALID_ARG, "substeps must be >= 1");
    if (iterations < 0) VBD_FAIL(VBD_ERR_INVALID_ARG, "iterations must be >= 0");
    if (!gravity) VBD_FAIL(VBD_ERR_INVALID_ARG, "gravity is null");
    DeviceScope scope(s->device);
    const float h = dt / (float)substeps;
    // 1/h^2: VBD.cpp computes it through double, main.cpp's GPU loop in float (main.cpp:211)
    const float dtsr = s->semantics ? 1.0f / (h * h) : (float)(1.0 / (double)(h * h));
    const float hg[3] = {h * gravity[0], h * gravity[1], h * gravity[2]};
    vbd::GraphKey key{};
    key.kind = 0;
    key.iters = iterations;
    key.accel = use_acceleration ? 1 : 0;
    s->shape_key(key);
    key.h = h;
    key.dtsr = dtsr;
    key.hg[0] = hg[0];
    key.hg[1] = hg[1];
    key.hg[2] = hg[2];
    key.rho = rho;
    const long long nenergy = s->energies_per_step(substeps, iterations);
    if (nenergy > 0) VBD_TRY(s->reserve_energies(nenergy));
    for (int k = 0; k < substeps; ++k) {
        // the persistent kernel evaluates no energies: with an energy history the step runs as
        // separate launches
        if (s->persistent && !s->timing && nenergy == 0)
            VBD_TRY(s->launch_walk(iterations, dtsr, use_acceleration != 0, rho, true, true, false, h, hg));
        else
            VBD_TRY(s->run(key, [&] {
                return s->emit_substep(h, dtsr, hg, iterations, use_acceleration != 0, rho, nenergy > 0);
            }));
        VBD_TRY(s->record_substep(h, dtsr, hg, iterations, use_acceleration != 0, rho));
    }
    s->ehist_queued += nenergy;
    return VBD_OK;
}

int vbd_solver_energy_history(vbd_solver* s, double* energies, int32_t capacity, int32_t* count, int32_t reset) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (!count) VBD_FAIL(VBD_ERR_INVALID_ARG, "count is null");
    if (capacity < 0 || (capacity > 0 && !energies)) VBD_FAIL(VBD_ERR_INVALID_ARG, "need energies[capacity]");
    DeviceScope scope(s->device);
    int n = 0;
    if (s->ecount.p) {
        CUDA_TRY(cudaMemcpyAsync(&n, s->ecount.p, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
        CUDA_TRY(cudaStreamSynchronize(s->stream));
    }
    const int avail = (int)std::min<long long>(n, (long long)s->ehist.n);
    const int copy = std::min(avail, capacity);
    if (copy > 0) {
        CUDA_TRY(cudaMemcpyAsync(energies, s->ehist.p, sizeof(double) * copy, cudaMemcpyDefault, s->stream));
        CUDA_TRY(cudaStreamSynchronize(s->stream));
    }
    *count = n;
    if (reset && s->ecount.p) {
        CUDA_TRY(cudaMemsetAsync(s->ecount.p, 0, sizeof(int), s->stream));
        CUDA_TRY(cudaStreamSynchronize(s->stream));
        s->ehist_queued = 0;
    }
    return VBD_OK;
}

int vbd_solver_record(vbd_solver* s, int32_t checkpoint_every) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (checkpoint_every < 0) VBD_FAIL(VBD_ERR_INVALID_ARG, "checkpoint_every must be >= 0");
    if (checkpoint_every > 0 && s->semantics)
        VBD_FAIL(VBD_ERR_STATE, "the adjoint differentiates the VBDsolver semantics; set VBD_OPT_SEMANTICS to 0");
    DeviceScope scope(s->device);
    s->tape.clear();
    s->ckpts.clear();
    s->ckpt_every = checkpoint_every;
    if (checkpoint_every > 0) {
        if (s->live_seg.n != (size_t)checkpoint_every * s->N) {
            s->drop_graphs();
            VBD_TRY(s->live_seg.alloc((size_t)checkpoint_every * s->N));
        }
        s->ckpts.emplace_back(new vbd::DBuf<float4>());
        VBD_TRY(s->ckpts.back()->alloc(2 * (size_t)s->N));
        VBD_TRY(s->snapshot(*s->ckpts.back()));
        CUDA_TRY(cudaStreamSynchronize(s->stream));
    }
    return VBD_OK;
}

int vbd_solver_backward(vbd_solver* s, const float* dl_dx, const float* dl_dv, int32_t adjoint_iterations,
                        float adjoint_rho, float* dl_dx0, float* dl_dv0, float* dl_dmu, float* dl_dlambda) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (s->ckpt_every <= 0 || s->ckpts.empty()) VBD_FAIL(VBD_ERR_STATE, "nothing recorded: call vbd_solver_record first");
    if (!dl_dx) VBD_FAIL(VBD_ERR_INVALID_ARG, "dl_dx is null");
    if (adjoint_iterations < 1) VBD_FAIL(VBD_ERR_INVALID_ARG, "adjoint_iterations must be >= 1");
    if (!(adjoint_rho >= 0.0f) || !(adjoint_rho < 1.0f)) VBD_FAIL(VBD_ERR_INVALID_ARG, "adjoint_rho must be in [0, 1)");
    DeviceScope scope(s->device);
    const int N = s->N, T = s->T, K = s->ckpt_every;
    const size_t b4 = sizeof(float4) * (size_t)N;
    // adjoint buffers; captured graphs bake their addresses, so any reallocation drops them
    for (auto* b : {&s->adj_lam, &s->adj_lam2, &s->adj_lpp, &s->adj_G, &s->adj_ax, &s->adj_av})
        if (b->n != (size_t)N) {
            s->drop_graphs();
            VBD_TRY(b->alloc(N));
        }
    if (s->adj_seg.n != (size_t)K * N) {
        s->drop_graphs();
        VBD_TRY(s->adj_seg.alloc((size_t)K * N));
    }
    if (s->adj_save.n != 6 * (size_t)N) VBD_TRY(s->adj_save.alloc(6 * (size_t)N));
    if (s->adj_gmu.n != (size_t)std::max(T, 1)) {
        s->drop_graphs();
        VBD_TRY(s->adj_gmu.alloc(std::max(T, 1)));
        VBD_TRY(s->adj_glam.alloc(std::max(T, 1)));
    }
    // keep the caller's state; the recompute overwrites it
    float4* live[6] = {s->x0.p, s->x1.p, s->pp.p, s->y.p, s->v.p, s->xprev.p};
    for (int k = 0; k < 6; ++k)
        CUDA_TRY(cudaMemcpyAsync(s->adj_save.p + (size_t)k * N, live[k], b4, cudaMemcpyDeviceToDevice, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->adj_lam.p, 0, b4, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->adj_lam2.p, 0, b4, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->adj_lpp.p, 0, b4, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->adj_gmu.p, 0, sizeof(float) * s->adj_gmu.n, s->stream));
    CUDA_TRY(cudaMemsetAsync(s->adj_glam.p, 0, sizeof(float) * s->adj_glam.n, s->stream));
    s->adj_cur = 0;
    VBD_TRY(s->upload3(dl_dx, s->adj_ax.p, nullptr));
    if (dl_dv)
        VBD_TRY(s->upload3(dl_dv, s->adj_av.p, nullptr));
    else
        CUDA_TRY(cudaMemsetAsync(s->adj_av.p, 0, b4, s->stream));
    const int nsteps = (int)s->tape.size();
    const int nseg = (nsteps + K - 1) / K;
    int rc = VBD_OK;
    for (int seg = nseg - 1; seg >= 0 && !rc; --seg) {
        const int t0 = seg * K, t1 = std::min(nsteps, t0 + K);
        // the newest segment's converged states were kept during the forward; older segments are
        // recomputed from their checkpoint (same graphs, hence the same bits)
        const bool live = seg == nseg - 1;
        float4* states = live ? s->live_seg.p : s->adj_seg.p;
        if (!live) {
            vbd::DBuf<float4>& ck = *s->ckpts[seg];
            CUDA_TRY(cudaMemcpyAsync(s->x0.p, ck.p, b4, cudaMemcpyDeviceToDevice, s->stream));
            CUDA_TRY(cudaMemcpyAsync(s->x1.p, ck.p, b4, cudaMemcpyDeviceToDevice, s->stream));
            CUDA_TRY(cudaMemcpyAsync(s->v.p, ck.p + N, b4, cudaMemcpyDeviceToDevice, s->stream));
            for (int t = t0; t < t1 && !rc; ++t) {
                rc = s->replay_substep(s->tape[t]);
                if (!rc && cudaMemcpyAsync(s->adj_seg.p + (size_t)(t - t0) * N, s->x0.p, b4,
                                           cudaMemcpyDeviceToDevice, s->stream) != cudaSuccess)
                    VBD_FAIL(VBD_ERR_CUDA, "segment copy failed");
            }
        }
        for (int t = t1 - 1; t >= t0 && !rc; --t)
            rc = s->adjoint_substep(s->tape[t], t - t0, states + (size_t)(t - t0) * N, adjoint_iterations,
                                    adjoint_rho, live ? 1 : 0);
    }
    if (!rc) {
        if (dl_dx0) rc = s->download3(s->adj_ax.p, dl_dx0);
        if (!rc && dl_dv0) rc = s->download3(s->adj_av.p, dl_dv0);
        if (!rc && dl_dmu && T > 0 &&
            cudaMemcpyAsync(dl_dmu, s->adj_gmu.p, sizeof(float) * T, cudaMemcpyDefault, s->stream) != cudaSuccess)
            rc = VBD_ERR_CUDA;
        if (!rc && dl_dlambda && T > 0 &&
            cudaMemcpyAsync(dl_dlambda, s->adj_glam.p, sizeof(float) * T, cudaMemcpyDefault, s->stream) != cudaSuccess)
            rc = VBD_ERR_CUDA;
    }
    for (int k = 0; k < 6; ++k)
        CUDA_TRY(cudaMemcpyAsync(live[k], s->adj_save.p + (size_t)k * N, b4, cudaMemcpyDeviceToDevice, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    return rc;
}

int vbd_solver_sync(vbd_solver* s) {
    vbd::clear_error();
    if (!s) VBD_FAIL(VBD_ERR_INVALID_ARG, "null solver handle");
    DeviceScope scope(s->device);
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (s->status.p) {
        unsigned long long t[2] = {0, 0};  // ST_TIMEOUT, ST_WALK_TIMEOUT
        CUDA_TRY(cudaMemcpy(t, s->status.p + vbd::ST_TIMEOUT, sizeof(t), cudaMemcpyDeviceToHost));
        if (t[0] || t[1]) {
            CUDA_TRY(cudaMemset(s->status.p + vbd::ST_TIMEOUT, 0, sizeof(t)));
            if (t[0]) VBD_FAIL(VBD_ERR_TIMEOUT, "a grid barrier of the persistent kernel gave up waiting");
            VBD_FAIL(VBD_ERR_TIMEOUT, "an mbarrier wait of the cluster walk gave up");
        }
    }
    return VBD_OK;
}

int vbd_solver_barrier_selftest(vbd_solver* s, int64_t spin_limit, int32_t* timed_out) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (!timed_out || spin_limit < 1) VBD_FAIL(VBD_ERR_INVALID_ARG, "need timed_out and spin_limit >= 1");
    DeviceScope scope(s->device);
    const long long saved = s->spin_limit;
    s->spin_limit = spin_limit;
    // one arrival more than the grid has: the first barrier can never complete
    int rc = s->launch_persistent(0, 1.0f, false, 0.0f, false, false, false, 1.0f, nullptr, 1);
    s->spin_limit = saved;
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    unsigned long long t = 0;
    CUDA_TRY(cudaMemcpy(&t, s->status.p + vbd::ST_TIMEOUT, sizeof(t), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemset(s->status.p + vbd::ST_TIMEOUT, 0, sizeof(t)));
    *timed_out = t ? 1 : 0;
    return VBD_OK;
}

int vbd_solver_energy(vbd_solver* s, int32_t kind, float h, double* out) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (!out) VBD_FAIL(VBD_ERR_INVALID_ARG, "out is null");
    if (kind < 0 || kind > 2) VBD_FAIL(VBD_ERR_INVALID_ARG, "unknown energy kind %d", kind);
    if (kind != VBD_ENERGY_ELASTIC_LOGJ && (!(h > 0.f) || !std::isfinite(h)))
        VBD_FAIL(VBD_ERR_INVALID_ARG, "h must be positive and finite");
    DeviceScope scope(s->device);
    if (kind == VBD_ENERGY_RESIDUAL) {
        if (s->nfree == 0) {
            *out = 0.0;
            return VBD_OK;
        }
        vbd::SweepParams p{s->x0.p,     nullptr, s->pp.p,    s->y.p, s->inc_off.p, s->inc_tet.p,
                           s->rec.p,    s->irec.p, s->crec.p, s->cmat.p, s->status.p, 0,
                           s->nfree,    (float)(1.0 / ((double)h * h)), 1.0f, 0, 0, 0, 0};
        const int L = std::max(4, s->lanes);
        const unsigned blocks = vbd::nblk((long long)s->nfree * L, 256);
        switch (L) {
            case 4: vbd::k_residual<4><<<blocks, 256, 0, s->stream>>>(p, s->partials.p); break;
            case 8: vbd::k_residual<8><<<blocks, 256, 0, s->stream>>>(p, s->partials.p); break;
            case 16: vbd::k_residual<16><<<blocks, 256, 0, s->stream>>>(p, s->partials.p); break;
            default: vbd::k_residual<32><<<blocks, 256, 0, s->stream>>>(p, s->partials.p); break;
        }
        VBD_TRY(s->check_launch());
        double r2 = 0.0;
        VBD_TRY(s->reduce_scalar(blocks, &r2));
        *out = std::sqrt(r2);
        return VBD_OK;
    }
    const long long work = std::max<long long>(kind == VBD_ENERGY_IP ? s->N : 0, s->T);
    const unsigned blocks = std::max(1u, std::min<unsigned>(vbd::nblk(work, 256), 4096u));
    const double inv_h2 = kind == VBD_ENERGY_IP ? 1.0 / ((double)h * h) : 0.0;
    vbd::k_energy<<<blocks, 256, 0, s->stream>>>(s->x0.p, s->y.p, s->rec.p, kind == VBD_ENERGY_IP ? s->N : 0, s->T,
                                                 kind, inv_h2, s->partials.p);
    VBD_TRY(s->check_launch());
    return s->reduce_scalar(blocks, out);
}

int vbd_solver_status(vbd_solver* s, int64_t* singular_skips, int32_t* nonfinite, int32_t reset) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    DeviceScope scope(s->device);
    unsigned long long h[vbd::ST_SLOTS];
    CUDA_TRY(cudaMemcpyAsync(h, s->status.p, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (singular_skips) *singular_skips = (int64_t)h[vbd::ST_SINGULAR];
    if (nonfinite) *nonfinite = h[vbd::ST_NONFINITE] ? 1 : 0;
    if (reset) {
        CUDA_TRY(cudaMemsetAsync(s->status.p, 0, sizeof(h), s->stream));
        CUDA_TRY(cudaStreamSynchronize(s->stream));
    }
    return VBD_OK;
}

int vbd_solver_set_option(vbd_solver* s, int32_t option, int32_t value) {
    vbd::clear_error();
    if (!s) VBD_FAIL(VBD_ERR_INVALID_ARG, "null solver handle");
    DeviceScope scope(s->device);
    switch (option) {
        case VBD_OPT_LANES:
            if (value != 1 && value != 2 && value != 4 && value != 8 && value != 16 && value != 32)
                VBD_FAIL(VBD_ERR_INVALID_ARG, "lanes must be 1, 2, 4, 8, 16 or 32");
            s->lanes = value;
            s->lanes_auto = false;
            return VBD_OK;
        case VBD_OPT_PREFETCH:
            if (value < 0 || value > 3) VBD_FAIL(VBD_ERR_INVALID_ARG, "prefetch must be 0, 1, 2 or 3");
            s->prefetch = value;
            s->prefetch_auto = false;
            return VBD_OK;
        case VBD_OPT_RECORD_CACHE:
            s->record_cache = value ? 1 : 0;
            s->record_cache_auto = false;
            return VBD_OK;
        case VBD_OPT_RECORD_PERSIST_MB:
            if (value < 0) VBD_FAIL(VBD_ERR_INVALID_ARG, "persist megabytes must be >= 0");
            s->persist_mb = value;
            s->persist_auto = false;
            return VBD_OK;
        case VBD_OPT_ENERGY_EVERY:
            if (value < 0) VBD_FAIL(VBD_ERR_INVALID_ARG, "energy interval must be >= 0");
            s->energy_every = value;
            return VBD_OK;
        case VBD_OPT_PDL:
            s->pdl = value ? 1 : 0;
            return VBD_OK;
        case VBD_OPT_PERSISTENT:
            if (value < 0 || value > 2) VBD_FAIL(VBD_ERR_INVALID_ARG, "persistent must be 0, 1 or 2");
            if (value && s->semantics)
                VBD_FAIL(VBD_ERR_INVALID_ARG, "the persistent kernel runs the VBDsolver semantics only");
            if (value == 2 && s->ready) {
                const char* why = nullptr;
                if (!s->cluster_fit(&why)) VBD_FAIL(VBD_ERR_INVALID_ARG, "%s", why);
            }
            s->persistent = value;
            return VBD_OK;
        case VBD_OPT_CLUSTER_CTAS:
            if (value < 0 || value > 16) VBD_FAIL(VBD_ERR_INVALID_ARG, "cluster CTAs must be 0 (automatic) to 16");
            s->cluster_ctas_opt = value;
            return VBD_OK;
        case VBD_OPT_CLUSTER_RESIDENT:
            s->cluster_resident = value ? 1 : 0;
            return VBD_OK;
        case VBD_OPT_L2_PREFETCH:
            s->l2_prefetch = value ? 1 : 0;
            return VBD_OK;
        case VBD_OPT_SEMANTICS:
            if (value != 0 && value != 1) VBD_FAIL(VBD_ERR_INVALID_ARG, "semantics must be 0 (VBDsolver) or 1 (VBD_GPU_Solver)");
            if (value && s->persistent)
                VBD_FAIL(VBD_ERR_INVALID_ARG, "the persistent kernel runs the VBDsolver semantics only");
            if (value && s->ckpt_every > 0)
                VBD_FAIL(VBD_ERR_STATE, "recording for the adjoint is on; the adjoint needs the VBDsolver semantics");
            s->semantics = value;
            return VBD_OK;
        case VBD_OPT_ADJOINT_ALTERNATE:
            s->adj_alternate = value ? 1 : 0;
            return VBD_OK;
        case VBD_OPT_BLOCK:
            if (value != 64 && value != 128 && value != 256)
                VBD_FAIL(VBD_ERR_INVALID_ARG, "block must be 64, 128 or 256");
            s->block = value;
            return VBD_OK;
        case VBD_OPT_LAYOUT:
            if (value < 0 || value > 4) VBD_FAIL(VBD_ERR_INVALID_ARG, "layout must be 0, 1, 2, 3 or 4");
            if (value == 4 && s->ready && s->N > vbd::kPackedMaxVertices)
                VBD_FAIL(VBD_ERR_INVALID_ARG, "layout 4 holds vertex ids below 2^21; this mesh has %d vertices", s->N);
            s->layout = value;
            s->layout_auto = false;
            if (s->ready) {
                VBD_TRY(s->repack_stream());
                CUDA_TRY(cudaStreamSynchronize(s->stream));
            }
            return VBD_OK;
        case VBD_OPT_GRAPH:
            s->use_graph = value ? 1 : 0;
            return VBD_OK;
        case VBD_OPT_KERNEL_TIMING:
            s->timing = value ? 1 : 0;
            return VBD_OK;
        default:
            VBD_FAIL(VBD_ERR_INVALID_ARG, "unknown option %d", option);
    }
}

int vbd_solver_get_option(vbd_solver* s, int32_t option, int32_t* value) {
    vbd::clear_error();
    if (!s || !value) VBD_FAIL(VBD_ERR_INVALID_ARG, "null argument");
    switch (option) {
        case VBD_OPT_LANES: *value = s->lanes; return VBD_OK;
        case VBD_OPT_LAYOUT: *value = s->layout; return VBD_OK;
        case VBD_OPT_GRAPH: *value = s->use_graph; return VBD_OK;
        case VBD_OPT_KERNEL_TIMING: *value = s->timing; return VBD_OK;
        case VBD_OPT_PREFETCH: *value = s->eff_prefetch(); return VBD_OK;
        case VBD_OPT_PDL: *value = s->pdl; return VBD_OK;
        case VBD_OPT_BLOCK: *value = s->block; return VBD_OK;
        case VBD_OPT_PERSISTENT: *value = s->persistent; return VBD_OK;
        case VBD_OPT_CLUSTER_RESIDENT: *value = s->cluster_resident; return VBD_OK;
        case VBD_OPT_CLUSTER_CTAS:
            *value = s->cluster_ctas_opt > 0 || !s->ready ? s->cluster_ctas_opt
                                                           : s->cluster_auto_ctas(s->lanes < 4 ? 4 : s->lanes);
            return VBD_OK;
        case VBD_OPT_SEMANTICS: *value = s->semantics; return VBD_OK;
        case VBD_OPT_L2_PREFETCH: *value = s->l2_prefetch; return VBD_OK;
        case VBD_OPT_ADJOINT_ALTERNATE: *value = s->adj_alternate; return VBD_OK;
        case VBD_OPT_RECORD_CACHE: *value = s->record_cache; return VBD_OK;
        case VBD_OPT_RECORD_PERSIST_MB: *value = s->persist_mb; return VBD_OK;
        case VBD_OPT_ENERGY_EVERY: *value = s->energy_every; return VBD_OK;
        default: VBD_FAIL(VBD_ERR_INVALID_ARG, "unknown option %d", option);
    }
}

int vbd_solver_set_colour_lanes(vbd_solver* s, int32_t num_colours, const int32_t* lanes) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (!lanes) {
        s->colour_lanes.clear();
        return VBD_OK;
    }
    if (num_colours != s->C) VBD_FAIL(VBD_ERR_INVALID_ARG, "need one lane count per colour (%d), got %d", s->C, num_colours);
    for (int c = 0; c < num_colours; ++c) {
        const int v = lanes[c];
        if (v != 1 && v != 2 && v != 4 && v != 8 && v != 16 && v != 32)
            VBD_FAIL(VBD_ERR_INVALID_ARG, "colour %d: lanes must be 1, 2, 4, 8, 16 or 32 (got %d)", c, v);
    }
    s->colour_lanes.assign(lanes, lanes + num_colours);
    return VBD_OK;
}

int vbd_solver_get_colour_lanes(vbd_solver* s, int32_t num_colours, int32_t* lanes) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (!lanes || num_colours != s->C)
        VBD_FAIL(VBD_ERR_INVALID_ARG, "need an array of one entry per colour (%d)", s->C);
    for (int c = 0; c < num_colours; ++c) lanes[c] = s->lanes_of(c);
    return VBD_OK;
}

int vbd_solver_info(vbd_solver* s, int32_t* num_verts, int32_t* num_tets, int32_t* num_colours) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (num_verts) *num_verts = s->N;
    if (num_tets) *num_tets = s->T;
    if (num_colours) *num_colours = s->C;
    return VBD_OK;
}

int vbd_solver_kernel_time(vbd_solver* s, double* sweep_ms, int64_t* sweep_launches, double* sweep_bytes,
                           int32_t reset) {
    vbd::clear_error();
    if (!s) VBD_FAIL(VBD_ERR_INVALID_ARG, "null solver handle");
    DeviceScope scope(s->device);
    VBD_TRY(s->collect_timing());
    if (sweep_ms) *sweep_ms = s->timed_ms;
    if (sweep_launches) *sweep_launches = s->timed_launches;
    if (sweep_bytes) *sweep_bytes = s->timed_bytes;
    if (reset) {
        s->timed_ms = 0.0;
        s->timed_bytes = 0.0;
        s->timed_launches = 0;
    }
    return VBD_OK;
}

int vbd_solver_autotune(vbd_solver* s, float dt, int32_t iterations, int32_t repeats, int32_t* chosen) {
    vbd::clear_error();
    VBD_TRY(need_ready(s));
    if (!s->have_materials) VBD_FAIL(VBD_ERR_STATE, "materials not set");
    if (!(dt > 0.f) || iterations < 1 || repeats < 1) VBD_FAIL(VBD_ERR_INVALID_ARG, "need dt > 0, iterations >= 1, repeats >= 1");
    DeviceScope scope(s->device);
    // Save the state the candidate steps overwrite.
    const size_t b4 = sizeof(float4) * (size_t)s->N;
    vbd::DBuf<float4> save;
    VBD_TRY(save.alloc(6 * (size_t)s->N));
    float4* bufs[6] = {s->x0.p, s->x1.p, s->pp.p, s->y.p, s->v.p, s->xprev.p};
    for (int k = 0; k < 6; ++k)
        CUDA_TRY(cudaMemcpyAsync(save.p + (size_t)k * s->N, bufs[k], b4, cudaMemcpyDeviceToDevice, s->stream));
    unsigned long long st[vbd::ST_SLOTS];
    CUDA_TRY(cudaMemcpyAsync(st, s->status.p, sizeof(st), cudaMemcpyDeviceToHost, s->stream));
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    const int saved_timing = s->timing;
    const int saved_energy = s->energy_every;
    s->timing = 0;
    s->energy_every = 0;  // the candidate steps append no energies
    // The whole launch configuration a candidate sets.
    struct Cand {
        int lanes, layout, prefetch, pdl, block, persistent, cache, persist;
        std::vector<int> colour_lanes;  // empty = `lanes` for every colour
        int ctas = 0;                   // CTAs of the cluster walk (0 = automatic)
    };
    const float g[3] = {0.f, 0.f, 0.f};
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    auto apply = [&](const Cand& c) -> int {
        s->lanes = c.lanes;
        s->prefetch = c.prefetch;
        s->pdl = c.pdl;
        s->block = c.block;
        s->persistent = c.persistent;
        s->record_cache = c.cache;
        s->persist_mb = c.persist;
        s->colour_lanes = c.colour_lanes;
        s->cluster_ctas_opt = c.ctas;
        if (s->layout != c.layout) {
            s->layout = c.layout;
            return s->repack_stream();
        }
        return VBD_OK;
    };
    // device time of `repeats` steps after one warm-up step (which captures the graph); the
    // simulation state is restored afterwards
    int reps = repeats;  // timed steps per candidate
    auto time_of = [&](const Cand& c, float* ms) -> int {
        VBD_TRY(apply(c));
        VBD_TRY(vbd_solver_step(s, dt, 1, iterations, g, 1, 0.9f));
        CUDA_TRY(cudaEventRecord(e0, s->stream));
        for (int r = 0; r < reps; ++r) VBD_TRY(vbd_solver_step(s, dt, 1, iterations, g, 1, 0.9f));
        CUDA_TRY(cudaEventRecord(e1, s->stream));
        CUDA_TRY(cudaEventSynchronize(e1));
        VBD_TRY(vbd_solver_sync(s));  // a persistent barrier that gave up makes the candidate fail
        CUDA_TRY(cudaEventElapsedTime(ms, e0, e1));
        for (int k = 0; k < 6; ++k)
            CUDA_TRY(cudaMemcpyAsync(bufs[k], save.p + (size_t)k * s->N, b4, cudaMemcpyDeviceToDevice, s->stream));
        return VBD_OK;
    };
    // Phase 1: uniform launch shapes (threads per vertex, record layout, prefetch, PDL, block).
    static const int uniform[][5] = {
        {8, 4, 2, 1, 64}, {8, 4, 3, 1, 64}, {8, 4, 1, 1, 64}, {8, 4, 1, 1, 128}, {4, 4, 1, 1, 128},
        {16, 4, 2, 1, 64}, {16, 4, 1, 1, 64}, {8, 4, 0, 1, 64},
        {8, 3, 1, 1, 64}, {8, 3, 1, 1, 128}, {4, 3, 1, 1, 128}, {16, 3, 1, 1, 64}, {8, 3, 0, 1, 64},
        {8, 3, 1, 0, 64}, {4, 2, 1, 1, 128}, {8, 2, 1, 1, 64},  {2, 2, 1, 1, 128}, {8, 1, 1, 1, 128},
        {8, 0, 1, 1, 128}, {4, 0, 1, 1, 128},
    };
    Cand best{s->lanes,      s->layout,       s->eff_prefetch(), s->pdl,          s->block,
              s->persistent, s->record_cache, s->persist_mb,     s->colour_lanes, s->cluster_ctas_opt};
    float best_ms = 1e30f;
    const int init_persist = s->persist_mb;  // the init-time record policy, for the factored candidates
    s->prefetch_auto = false;
    int rc = VBD_OK;
    for (const auto& u : uniform) {
        if (u[1] == 4 && s->N > vbd::kPackedMaxVertices) continue;
        Cand c{u[0], u[1], u[2], u[3], u[4], 0, u[1] >= 3 ? 1 : 0, u[1] >= 3 ? init_persist : 0, {}};
        float ms = 0.f;
        if ((rc = time_of(c, &ms))) break;
        if (ms < best_ms) {
            best_ms = ms;
            best = c;
        }
    }
    // A later phase replaces the choice only when it is faster by more than 1% (timing noise).
    auto try_cand = [&](const Cand& c) -> int {
        float ms = 0.f;
        VBD_TRY(time_of(c, &ms));
        if (ms < 0.99f * best_ms) {
            best_ms = ms;
            best = c;
        }
        return VBD_OK;
    };
    // Phase 2: the factored records' L2 policy: plain loads, or the evict-first stream with an
    // evict-last prefix of 0, 32 or 64 MB.  (The 64^3 cube is fastest with the stream and 32 MB;
    // the 512-mesh batch, whose vertex state alone outgrows L2, with plain loads.)
    if (!rc && best.layout >= 3) {
        const Cand base = best;
        for (int pm : {-1, 0, 32, 64}) {
            Cand c = base;
            c.cache = pm < 0 ? 0 : 1;
            c.persist = pm < 0 ? 0 : pm;
            if (c.cache == base.cache && c.persist == base.persist) continue;
            if ((rc = try_cand(c))) break;
        }
    }
    // Phase 3: per-colour threads per vertex.  A colour's lane count moves the step by 1-3%, about
    // as much as the drift between timings taken a few seconds apart, so each candidate is timed
    // alternately with the incumbent, twice each over 2 x repeats steps, and replaces it when the
    // sums differ by more than 1%.  Greedy over the colours (lane counts 2, 4, 8, 16), two passes,
    // restarted from uniform lanes under each factored prefetch depth (which interacts with the
    // lane count: the 64^3 cube is fastest with the three-deep prefetch and lanes 4,8,4,8,4,4,8,8).
    auto beats = [&](const Cand& c, const Cand& inc, bool* better) -> int {
        float a = 0.f, b = 0.f, t = 0.f;
        for (int r = 0; r < 2; ++r) {
            VBD_TRY(time_of(inc, &t));
            a += t;
            VBD_TRY(time_of(c, &t));
            b += t;
        }
        *better = b < 0.99f * a;
        return VBD_OK;
    };
    if (!rc && s->semantics == 0 && s->C > 1) {
        reps = 2 * repeats;
        std::vector<int> depths{best.prefetch};
        if (best.layout >= 3)
            for (int pf : {1, 2, 3})
                if (pf != best.prefetch) depths.push_back(pf);
        Cand overall = best;
        float overall_ms = 1e30f;
        for (size_t d = 0; d < depths.size() && !rc; ++d) {
            Cand inc = best;
            inc.prefetch = depths[d];
            inc.colour_lanes.assign(s->C, inc.lanes);
            for (int pass = 0; pass < 2 && !rc; ++pass)
                for (int col = 0; col < s->C && !rc; ++col)
                    for (int L : {2, 4, 8, 16}) {
                        if (L == inc.colour_lanes[col]) continue;
                        Cand c = inc;
                        c.colour_lanes[col] = L;
                        bool better = false;
                        if ((rc = beats(c, inc, &better))) break;
                        if (better) inc = c;
                    }
            float ms = 0.f;
            if (!rc && !(rc = time_of(inc, &ms)) && ms < overall_ms) {
                overall_ms = ms;
                overall = inc;
            }
        }
        if (!rc) {
            bool better = false;
            if (!(rc = beats(overall, best, &better)) && better) best = overall;
        }
        if (!rc) rc = time_of(best, &best_ms);  // the incumbent at this phase's length, for phase 4
    }
    // Phase 4: the whole step as one persistent colour-walking launch (uniform lanes, no per-colour
    // shape) against the captured graph.
    if (!rc && s->semantics == 0) {
        const Cand base = best;
        Cand c = base;
        c.persistent = 1;
        c.colour_lanes.clear();
        rc = try_cand(c);
        // the cluster walk, for a mesh whose positions fit in one CTA's shared memory: each lane count
        // with either factored layout (the stored det M of layout 3 saves a division per record,
        // which counts where the records stay in L2)
        const char* why = nullptr;
        if (!rc && base.layout >= 3 && s->cluster_fit(&why)) {
            for (int lay : {3, 4}) {
                if (lay == 4 && s->N > vbd::kPackedMaxVertices) continue;
                for (int L : {4, 8, 16, 32}) {
                    Cand k = base;
                    k.persistent = 2;
                    k.lanes = L;
                    k.layout = lay;
                    k.colour_lanes.clear();
                    if ((rc = try_cand(k))) break;
                }
                if (rc) break;
            }
            // the chosen walk's CTA count around the automatic one (fewer CTAs send fewer copies of
            // each update; more take fewer rounds)
            if (!rc && best.persistent == 2 && best.ctas == 0) {
                const int a = s->cluster_auto_ctas(best.lanes < 4 ? 4 : best.lanes);
                const Cand walk = best;
                for (int n : {a / 2, (3 * a) / 4, a + (a + 1) / 2, 16}) {
                    n = std::min(16, std::max(1, n));
                    if (n == a) continue;
                    Cand k = walk;
                    k.ctas = n;
                    if ((rc = try_cand(k))) break;
                }
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (int k = 0; k < 6; ++k)
        CUDA_TRY(cudaMemcpyAsync(bufs[k], save.p + (size_t)k * s->N, b4, cudaMemcpyDeviceToDevice, s->stream));
    CUDA_TRY(cudaMemcpyAsync(s->status.p, st, sizeof(st), cudaMemcpyHostToDevice, s->stream));
    s->timing = saved_timing;
    s->energy_every = saved_energy;
    s->record_cache_auto = s->persist_auto = false;  // the tuned policy stays for this mesh
    const int arc = apply(best);
    CUDA_TRY(cudaStreamSynchronize(s->stream));
    if (rc) return rc;
    if (arc) return arc;
    if (chosen) {
        chosen[0] = best.lanes;
        chosen[1] = best.layout;
        chosen[2] = best.prefetch;
        chosen[3] = best.pdl;
        chosen[4] = best.block;
    }
    return VBD_OK;
}

int vbd_solver_kernel_launches(vbd_solver* s, int64_t* launches) {
    vbd::clear_error();
    if (!s || !launches) VBD_FAIL(VBD_ERR_INVALID_ARG, "null argument");
    *launches = s->launches;
    return VBD_OK;
}

}  // extern "C"
