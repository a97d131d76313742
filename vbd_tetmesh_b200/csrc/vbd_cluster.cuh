// The cluster-resident colour walk: a whole sub-step of a mesh whose positions fit in one CTA's
// shared memory, run by ONE thread-block cluster.
//
// The per-colour launches of the graph path cost about 2.4 us each however small the colour; a
// mesh of a few thousand vertices (the differentiated beam: 2,673 vertices, 8 colours of about
// 330) gives each launch well under a microsecond of work.  Here no kernel boundary separates the
// colours, and neighbour positions come from shared memory instead of L2:
//   * every CTA of the cluster holds both position buffers of the whole mesh (2 x N float4 in
//     dynamic shared memory), and the pre-sweep positions of the vertices it sweeps;
//   * a vertex's group of LANES threads gathers from its own CTA's copy; after the block solve the
//     group's lanes send x~ (and the Chebyshev-blended position) to every CTA of the cluster with
//     st.async, a remote shared-memory store that completes its bytes on the receiving CTA's
//     mbarrier;
//   * each CTA knows how many bytes colour c brings (16 B per vertex of the colour, 32 B when the
//     iteration blends) and waits on its own mbarrier for them, then sweeps colour c + 1.  No
//     cluster-wide barrier or memory fence sits between colours.  Two mbarriers alternate by
//     colour, because a CTA that has all of colour c may send colour c + 1 before a slower CTA
//     has finished waiting for colour c, and each colour's bytes are announced on the receiving
//     CTA before any CTA can send them (see k_cluster_walk);
//   * while waiting, each thread loads the next colour's element records, inertial target and
//     pre-sweep position, so their latency overlaps the wait.
// Why the in-place sweep stays exact: a CTA sends its colour-c results only after it has read
// every position its colour-c vertices need, so a CTA that holds all of colour c knows that every
// CTA has finished reading for colour c, and may overwrite colour c + 1 positions anywhere.
// The arithmetic is the graph path's (Elem<LAYOUT>::contrib, group_reduce, block_solve,
// cheb_blend, predict_vertex, damped_velocity) with the same lane-to-record assignment, so the
// positions and velocities equal the graph path's at the same lane count.
#pragma once

#include "vbd_kernels.cuh"

namespace vbd {

constexpr int kClusterMaxBlock = 256;  // threads per CTA of the cluster walk
constexpr int kClusterAhead = 3;       // element records per lane loaded while waiting for a colour

__device__ __forceinline__ unsigned cluster_rank() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ unsigned cluster_size() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}

// Cluster-wide barrier (taken once before the first colour and once before the walk ends), split so
// that independent loads can be issued between the two halves.  The release / acquire pair orders
// every shared (local and distributed) and global memory access before the arrive against those
// after the wait, across the cluster.  Every thread of the cluster takes it, each warp reconverged
// first, so the warp-aligned forms apply.
__device__ __forceinline__ void cluster_arrive() {
    __syncwarp();
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }

// The shared-memory address in CTA `rank` of the cluster that corresponds to this CTA's `local`.
__device__ __forceinline__ unsigned cluster_map(unsigned local, unsigned rank) {
    unsigned r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
    return r;
}

// mbarrier with one expected arrival per phase (this CTA's expect_tx) plus transaction bytes.
__device__ __forceinline__ void mbar_init(unsigned bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect(unsigned bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// 16 bytes into shared memory of a CTA of the cluster (addr from cluster_map), completing 16
// transaction bytes on that CTA's mbarrier rbar (also from cluster_map).
__device__ __forceinline__ void st_async(unsigned addr, float4 v, unsigned rbar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.f32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(addr),
                 "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "r"(rbar)
                 : "memory");
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the mbarrier phase of `parity`.  Bounded: after kClusterWaitNs, or once any thread of
// the launch has given up (status[ST_WALK_TIMEOUT], checked every 256 polls), it sets that flag and
// returns false.  The decision is made warp-wide so the warp's shuffles stay converged.
constexpr unsigned long long kClusterWaitNs = 1000000000ull;  // 1 s
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, unsigned long long* status) {
    bool done = mbar_try(bar, parity);
    if (!done) {
        const unsigned long long t0 = global_ns();
        for (unsigned i = 1; !done; ++i) {
            done = mbar_try(bar, parity);
            if (!done && (i & 255u) == 0u &&
                (global_ns() - t0 > kClusterWaitNs ||
                 *reinterpret_cast<volatile unsigned long long*>(status + ST_WALK_TIMEOUT) != 0ull))
                break;
        }
    }
    done = __all_sync(0xffffffffu, done);
    if (!done) atomicOr(reinterpret_cast<unsigned int*>(status + ST_WALK_TIMEOUT), 1u);
    return done;
}

// What a vertex group needs before it can sweep its vertex, loaded while the previous colour is
// still arriving: the lane's first kClusterAhead element records, and (first lane) the inertial target and the
// position before the previous sweep.  Element data and y do not change during the sweeps; the
// pre-sweep position is kept in this CTA's shared memory (pp, indexed by vertex) and written only
// by this same thread.
template <int LAYOUT> struct Ahead {
    typename Elem<LAYOUT>::Rec buf[kClusterAhead];
    float4 y, q;
    int j0, j1;
};

// with_y = false leaves a.y unset: before the walk's first barrier the predictor's y may not yet
// be visible.
template <int LANES, int LAYOUT>
__device__ __forceinline__ void load_ahead(const PersistParams& p, const float4* pp, int v, bool active, int lane,
                                           Ahead<LAYOUT>& a, bool with_y = true) {
    a.j0 = 0;
    a.j1 = 0;
    if (active) {
        a.j0 = __ldg(p.sw.inc_off + v);
        a.j1 = __ldg(p.sw.inc_off + v + 1);
    }
    const int j = a.j0 + lane;
#pragma unroll
    for (int k = 0; k < kClusterAhead; ++k)
        if (j + k * LANES < a.j1) a.buf[k] = Elem<LAYOUT>::fetch(p.sw, j + k * LANES);
    if (active && lane == 0) {
        if (with_y) a.y = __ldcg(p.sw.y + v);  // written by the predictor in other CTAs: read from L2
        a.q = pp[v];
    }
}

// One vertex of a colour sweep from the CTA's copy of the positions `xs`; x~ and the blended
// position are then sent to every CTA's `xs` / `xb` copy, completing on each CTA's mbarrier `bar`.
// All lanes of the warp call it.
template <int LANES, int LAYOUT>
__device__ __forceinline__ void cluster_vertex(const PersistParams& p, const float4* xs, const float4* xb, float4* pp,
                                               unsigned bar, int v, bool active, int lane, int lane_w, unsigned csize,
                                               bool blend, float omega, const Ahead<LAYOUT>& a) {
    const float4 xi = active ? xs[v] : make_float4(0.f, 0.f, 0.f, 0.f);
    Acc acc;
    acc.zero();
    const int j = a.j0 + lane;
#pragma unroll
    for (int k = 0; k < kClusterAhead; ++k)
        if (j + k * LANES < a.j1) Elem<LAYOUT>::template contrib<true>(a.buf[k], v, xi, xs, acc);
    for (int jj = j + kClusterAhead * LANES; jj < a.j1; jj += LANES)
        Elem<LAYOUT>::template contrib<true>(Elem<LAYOUT>::fetch(p.sw, jj), v, xi, xs, acc);
    group_reduce<LANES>(acc);
    float4 xn = xi, xa = xi;
    if (active && lane == 0) {
        xn = block_solve(acc, xi, a.y, p.sw.dtsr, p.sw.status);
        if (blend) xa = cheb_blend(xn, a.q, omega);
        if (p.sw.keep_pp) pp[v] = xi;
    }
    // the group's first lane holds the results; every lane of the group then sends them to CTAs
    // lane, lane + LANES, ... of the cluster
    const int leader = lane_w & ~(LANES - 1);
    xn.x = __shfl_sync(0xffffffffu, xn.x, leader);
    xn.y = __shfl_sync(0xffffffffu, xn.y, leader);
    xn.z = __shfl_sync(0xffffffffu, xn.z, leader);
    xn.w = __shfl_sync(0xffffffffu, xn.w, leader);
    if (blend) {
        xa.x = __shfl_sync(0xffffffffu, xa.x, leader);
        xa.y = __shfl_sync(0xffffffffu, xa.y, leader);
        xa.z = __shfl_sync(0xffffffffu, xa.z, leader);
        xa.w = __shfl_sync(0xffffffffu, xa.w, leader);
    }
    if (!active) return;
    const unsigned sn = (unsigned)__cvta_generic_to_shared(xs + v);
    const unsigned sa = (unsigned)__cvta_generic_to_shared(xb + v);
    for (unsigned r = (unsigned)lane; r < csize; r += LANES) {
        const unsigned rb = cluster_map(bar, r);
        st_async(cluster_map(sn, r), xn, rb);
        if (blend) st_async(cluster_map(sa, r), xa, rb);
    }
}

// Bytes colour g (counted over all iterations) brings to every CTA: 16 per vertex of the colour,
// 32 when its iteration blends.
__device__ __forceinline__ unsigned walk_bytes(const PersistParams& p, unsigned g) {
    const int k = (int)(g / (unsigned)p.ncol), c = (int)(g % (unsigned)p.ncol);
    const int size = __ldg(p.cstart + c + 1) - __ldg(p.cstart + c);
    return (unsigned)size * (__ldg(p.omega + k) > 1.0f ? 32u : 16u);
}

// A whole sub-step (or solve) of one mesh in one cluster: the predictor (or the x = y start),
// `iters` Gauss-Seidel iterations over the colours with the Chebyshev schedule, the velocity
// update.  Launched as one cluster of gridDim.x CTAs with 3 * n float4 of dynamic shared memory.
// The position before the previous sweep (pp) lives in shared memory only: each sub-step writes it
// at its first iteration, whose Chebyshev weight is 1 (no blend), before any blend reads it, so
// the global pp array is not used.
// Vertex groups are numbered across the cluster; group g sweeps vertices vb + g, vb + g + groups,
// ... of each colour [vb, ve).
template <int LANES, int LAYOUT>
__global__ void __launch_bounds__(kClusterMaxBlock, 1) k_cluster_walk(PersistParams p) {
    extern __shared__ float4 sx[];  // [0, n): buffer 0 (xa), [n, 2n): buffer 1 (xb), [2n, 3n): pp
    __shared__ __align__(8) unsigned long long mbar[2];  // colour c completes on mbar[c & 1]
    const int n = p.n;
    float4* spp = sx + 2 * n;  // entries of the vertices this CTA's groups own
    const unsigned csize = cluster_size();
    const int tid = threadIdx.x;
    const int gt = (int)cluster_rank() * (int)blockDim.x + tid;
    const int nthreads = (int)csize * (int)blockDim.x;
    const int lane_w = tid & 31;
    const int lane = LANES == 1 ? 0 : (lane_w & (LANES - 1));
    const int grp = gt / LANES;
    const int ngroups = nthreads / LANES;
    float4* y = const_cast<float4*>(p.sw.y);
    const unsigned bar0 = (unsigned)__cvta_generic_to_shared(&mbar[0]);
    // Colour g completes on mbar[g & 1].  Its bytes are announced (expect_tx) before any CTA can
    // send them: colours 0 and 1 here, before the cluster barrier below; colour g + 2 by this CTA
    // once colour g is complete here and before this CTA sends anything of colour g + 1 (the
    // __syncthreads_and after each wait orders the two), while other CTAs send colour g + 2 only
    // after they hold all of colour g + 1.
    const unsigned total = (unsigned)max(p.iters, 0) * (unsigned)p.ncol;
    if (tid == 0) {
        mbar_init(bar0);
        mbar_init(bar0 + 8);
        if (total > 0) mbar_expect(bar0, walk_bytes(p, 0));
        if (total > 1) mbar_expect(bar0 + 8, walk_bytes(p, 1));
        fence_mbar_init();
    }

    if (p.predict)
        for (int i = gt; i < n; i += nthreads)
            predict_vertex(i, p.xa, p.v, p.xprev, y, p.nfree, p.h, p.hgx, p.hgy, p.hgz);
    if (p.init_from_inertia)  // x = y in both global buffers (k_copy_xyz); the host never sets predict too
        for (int i = gt; i < n; i += nthreads) {
            const float4 yi = y[i];
            float4 a = p.xa[i], b = p.xb[i];
            a.x = b.x = yi.x;
            a.y = b.y = yi.y;
            a.z = b.z = yi.z;
            p.xa[i] = a;
            p.xb[i] = b;
        }
    // this CTA's copy of both buffers (the predictor leaves x unchanged)
    for (int i = tid; i < n; i += blockDim.x) {
        float4 a = p.xa[i];
        float4 b = p.xb[i];
        if (p.init_from_inertia) {
            const float4 yi = y[i];
            a.x = b.x = yi.x;
            a.y = b.y = yi.y;
            a.z = b.z = yi.z;
        }
        sx[i] = a;
        sx[n + i] = b;
    }
    // every CTA's mbarriers and copies are ready before any CTA sends, and the predictor's y is
    // visible after the wait
    cluster_arrive();
    Ahead<LAYOUT> ah;
    const int v0 = __ldg(p.cstart) + grp;
    const bool act0 = p.iters > 0 && p.ncol > 0 && v0 < __ldg(p.cstart + 1);
    if (p.iters > 0 && p.ncol > 0) load_ahead<LANES, LAYOUT>(p, spp, v0, act0, lane, ah, false);
    cluster_wait();
    if (act0 && lane == 0) ah.y = __ldcg(p.sw.y + v0);

    int cur = 0;
    unsigned gc = 0;  // colours swept so far
    bool alive = true;
    for (int k = 0; k < p.iters && alive; ++k) {
        const float om = __ldg(p.omega + k);
        const bool blend = om > 1.0f;
        const float4* xs = sx + (cur ? n : 0);
        const float4* xb = sx + (cur ? 0 : n);
        for (int c = 0; c < p.ncol; ++c, ++gc) {
            const int vb = __ldg(p.cstart + c), ve = __ldg(p.cstart + c + 1);
            const unsigned bar = bar0 + 8u * (gc & 1u);
            const int rounds = (ve - vb + ngroups - 1) / ngroups;
            for (int r = 0; r < rounds; ++r) {
                const int v = vb + r * ngroups + grp;
                const bool active = v < ve;
                if (r == 0) {
                    cluster_vertex<LANES, LAYOUT>(p, xs, xb, spp, bar, v, active, lane, lane_w, csize, blend, om, ah);
                } else {
                    Ahead<LAYOUT> a;
                    load_ahead<LANES, LAYOUT>(p, spp, v, active, lane, a);
                    cluster_vertex<LANES, LAYOUT>(p, xs, xb, spp, bar, v, active, lane, lane_w, csize, blend, om, a);
                }
            }
            // the first round of the colour swept next (colour 0 of the next iteration after the last)
            const bool last = (k == p.iters - 1) && (c == p.ncol - 1);
            if (!last) {
                const int cn = c + 1 < p.ncol ? c + 1 : 0;
                const int v = __ldg(p.cstart + cn) + grp;
                load_ahead<LANES, LAYOUT>(p, spp, v, v < __ldg(p.cstart + cn + 1), lane, ah);
            }
            const bool ok = mbar_wait(bar, (gc >> 1) & 1u, p.sw.status);
            if (tid == 0 && ok && gc + 2 < total) mbar_expect(bar, walk_bytes(p, gc + 2));
            alive = __syncthreads_and(ok) != 0;
            if (!alive) break;
        }
        if (blend) cur ^= 1;
    }
    // no CTA leaves while another may still send to it
    cluster_arrive();
    cluster_wait();
    if (!alive) return;

    // every CTA holds the final positions; free vertices go back to buffer 0 (and the velocity)
    const float4* xf = sx + (cur ? n : 0);
    for (int i = gt; i < p.nfree; i += nthreads) {
        const float4 xi = xf[i];
        p.xa[i] = xi;
        if (p.finish) p.v[i] = damped_velocity(xi, p.xprev[i], p.v[i], p.h);
    }
}

// ---- The cluster walk with resident element data ------------------------------------------------
//
// In the walk above, the CTA that finishes a colour last has no wait in which its next colour's
// element records (from L2) could arrive, so their latency sits on the critical path every colour
// (long-scoreboard stalls lead its profile).  Where they fit, each CTA instead copies, once per
// sub-step, the records, inertial targets and incidence spans of exactly the vertices its groups
// sweep into shared memory.  Group g of CTA k sweeps, in round r of colour c, vertex
// vb_c + r * groups + k * gpc + (g - k * gpc): the CTA's vertices of one (colour, round) slice are
// one contiguous run, and so are their incidences, so a slice is one contiguous copy.  Same
// arithmetic and record order as the walk above, hence the same bits.

// Byte offsets of the regions of the resident walk's dynamic shared memory (16-byte aligned).
struct SrecLayout {
    unsigned long long x, rec, mat, y, pp, span, tab, rows, total;
};
__host__ __device__ inline unsigned long long srec_align(unsigned long long b) { return (b + 15ull) & ~15ull; }
__host__ __device__ inline SrecLayout srec_layout(int n, int records, int owned, int slices, int ncol, int layout) {
    SrecLayout L;
    const unsigned long long words = layout == 4 ? 2 : 3;  // int4 per record in the record stream
    L.x = 0;
    L.rec = srec_align(L.x + 32ull * (unsigned long long)n);
    L.mat = srec_align(L.rec + 16ull * words * (unsigned long long)records);
    L.y = srec_align(L.mat + (layout == 4 ? 8ull * (unsigned long long)records : 0ull));
    L.pp = srec_align(L.y + 16ull * (unsigned long long)owned);
    L.span = srec_align(L.pp + 16ull * (unsigned long long)owned);
    L.tab = srec_align(L.span + 8ull * (unsigned long long)owned);
    L.rows = srec_align(L.tab + 16ull * (unsigned long long)slices);
    L.total = srec_align(L.rows + 4ull * (unsigned long long)(ncol + 1));
    return L;
}

// A record from shared memory, in the layouts' raw form.
template <int LAYOUT> struct SRec;
template <> struct SRec<4> {
    __device__ __forceinline__ static FactRaw4 get(const int4* cs, const float2* cm, int j) {
        FactRaw4 r;
        r.w0 = cs[2 * j];
        r.w1 = reinterpret_cast<const float4*>(cs)[2 * j + 1];
        r.m = cm[j];
        return r;
    }
};
template <> struct SRec<3> {
    __device__ __forceinline__ static FactRaw3 get(const int4* cs, const float2*, int j) {
        FactRaw3 r;
        r.w0 = cs[3 * j];
        r.w1 = reinterpret_cast<const float4*>(cs)[3 * j + 1];
        r.w2 = reinterpret_cast<const float4*>(cs)[3 * j + 2];
        return r;
    }
};

// One vertex of a colour sweep with its CTA-local data at slot lv (records [span.x, span.y) of the
// CTA's resident records).  All lanes of the warp call it.
template <int LANES, int LAYOUT>
__device__ __forceinline__ void cluster_vertex_srec(const PersistParams& p, const float4* xs, const float4* xb,
                                                    const int4* cs, const float2* cm, const float4* ys, float4* pps,
                                                    const int2* spans, unsigned bar, int v, int lv, bool active,
                                                    int lane, int lane_w, unsigned csize, bool blend, float omega) {
    const float4 xi = active ? xs[v] : make_float4(0.f, 0.f, 0.f, 0.f);
    const int2 sp = active ? spans[lv] : make_int2(0, 0);
    Acc acc;
    acc.zero();
    for (int j = sp.x + lane; j < sp.y; j += LANES)
        Elem<LAYOUT>::template contrib<true>(SRec<LAYOUT>::get(cs, cm, j), v, xi, xs, acc);
    group_reduce<LANES>(acc);
    float4 xn = xi, xa = xi;
    if (active && lane == 0) {
        xn = block_solve(acc, xi, ys[lv], p.sw.dtsr, p.sw.status);
        if (blend) xa = cheb_blend(xn, pps[lv], omega);
        if (p.sw.keep_pp) pps[lv] = xi;
    }
    const int leader = lane_w & ~(LANES - 1);
    xn.x = __shfl_sync(0xffffffffu, xn.x, leader);
    xn.y = __shfl_sync(0xffffffffu, xn.y, leader);
    xn.z = __shfl_sync(0xffffffffu, xn.z, leader);
    xn.w = __shfl_sync(0xffffffffu, xn.w, leader);
    if (blend) {
        xa.x = __shfl_sync(0xffffffffu, xa.x, leader);
        xa.y = __shfl_sync(0xffffffffu, xa.y, leader);
        xa.z = __shfl_sync(0xffffffffu, xa.z, leader);
        xa.w = __shfl_sync(0xffffffffu, xa.w, leader);
    }
    if (!active) return;
    const unsigned sn = (unsigned)__cvta_generic_to_shared(xs + v);
    const unsigned sa = (unsigned)__cvta_generic_to_shared(xb + v);
    for (unsigned r = (unsigned)lane; r < csize; r += LANES) {
        const unsigned rb = cluster_map(bar, r);
        st_async(cluster_map(sn, r), xn, rb);
        if (blend) st_async(cluster_map(sa, r), xa, rb);
    }
}

// The walk above with each CTA's element records, inertial targets and pre-sweep positions resident
// in its shared memory (layout srec_layout; the host sizes it from the same slice plan).
template <int LANES, int LAYOUT>
__global__ void __launch_bounds__(kClusterMaxBlock, 1) k_cluster_walk_srec(PersistParams p) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ __align__(8) unsigned long long mbar[2];
    __shared__ int plan_ok;
    const int n = p.n;
    const SrecLayout Ly = srec_layout(n, p.srec_records, p.srec_owned, p.srec_slices, p.ncol, LAYOUT);
    float4* sx = reinterpret_cast<float4*>(smem + Ly.x);
    int4* cs = reinterpret_cast<int4*>(smem + Ly.rec);
    float2* cm = reinterpret_cast<float2*>(smem + Ly.mat);
    float4* ys = reinterpret_cast<float4*>(smem + Ly.y);
    float4* pps = reinterpret_cast<float4*>(smem + Ly.pp);
    int2* spans = reinterpret_cast<int2*>(smem + Ly.span);
    int4* tab = reinterpret_cast<int4*>(smem + Ly.tab);  // per slice: first vertex, count, vertex slot, record slot
    int* rows = reinterpret_cast<int*>(smem + Ly.rows);  // first slice of each colour
    const unsigned csize = cluster_size();
    const unsigned crank = cluster_rank();
    const int tid = threadIdx.x;
    const int gt = (int)crank * (int)blockDim.x + tid;
    const int nthreads = (int)csize * (int)blockDim.x;
    const int lane_w = tid & 31;
    const int lane = LANES == 1 ? 0 : (lane_w & (LANES - 1));
    const int grp = gt / LANES;
    const int ngroups = nthreads / LANES;
    const int gpc = (int)blockDim.x / LANES;  // groups per CTA
    const int lg = tid / LANES;               // this thread's group within the CTA
    float4* y = const_cast<float4*>(p.sw.y);
    const unsigned bar0 = (unsigned)__cvta_generic_to_shared(&mbar[0]);
    const unsigned total = (unsigned)max(p.iters, 0) * (unsigned)p.ncol;
    if (tid == 0) {  // as in k_cluster_walk: colours 0 and 1 announced before the first barrier
        mbar_init(bar0);
        mbar_init(bar0 + 8);
        if (total > 0) mbar_expect(bar0, walk_bytes(p, 0));
        if (total > 1) mbar_expect(bar0 + 8, walk_bytes(p, 1));
        fence_mbar_init();
        // this CTA's (colour, round) slices
        int sl = 0, vbase = 0, rbase = 0;
        for (int c = 0; c < p.ncol; ++c) {
            rows[c] = sl;
            const int vb = __ldg(p.cstart + c), ve = __ldg(p.cstart + c + 1);
            const int rounds = (ve - vb + ngroups - 1) / ngroups;
            for (int r = 0; r < rounds; ++r, ++sl) {
                const int vf = vb + r * ngroups + (int)crank * gpc;
                const int cnt = max(0, min(vf + gpc, ve) - vf);
                if (sl < p.srec_slices) tab[sl] = make_int4(vf, cnt, vbase, rbase);
                vbase += cnt;
                if (cnt) rbase += __ldg(p.sw.inc_off + vf + cnt) - __ldg(p.sw.inc_off + vf);
            }
        }
        rows[p.ncol] = sl;
        // the host sized the regions from the same plan; refuse rather than overrun them
        plan_ok = sl == p.srec_slices && vbase <= p.srec_owned && rbase <= p.srec_records;
        if (!plan_ok) atomicOr(reinterpret_cast<unsigned int*>(p.sw.status + ST_WALK_TIMEOUT), 1u);
    }

    if (p.predict)
        for (int i = gt; i < n; i += nthreads)
            predict_vertex(i, p.xa, p.v, p.xprev, y, p.nfree, p.h, p.hgx, p.hgy, p.hgz);
    if (p.init_from_inertia)
        for (int i = gt; i < n; i += nthreads) {
            const float4 yi = y[i];
            float4 a = p.xa[i], b = p.xb[i];
            a.x = b.x = yi.x;
            a.y = b.y = yi.y;
            a.z = b.z = yi.z;
            p.xa[i] = a;
            p.xb[i] = b;
        }
    for (int i = tid; i < n; i += blockDim.x) {
        float4 a = p.xa[i];
        float4 b = p.xb[i];
        if (p.init_from_inertia) {
            const float4 yi = y[i];
            a.x = b.x = yi.x;
            a.y = b.y = yi.y;
            a.z = b.z = yi.z;
        }
        sx[i] = a;
        sx[n + i] = b;
    }
    __syncthreads();
    const bool ok_plan = plan_ok != 0;
    constexpr int words = LAYOUT == 4 ? 2 : 3;
    if (ok_plan)  // the CTA's records and incidence spans, one contiguous run per slice
        for (int sl = 0; sl < p.srec_slices; ++sl) {
            const int4 t = tab[sl];
            if (t.y == 0) continue;
            const int jb = __ldg(p.sw.inc_off + t.x);
            const int cnt = __ldg(p.sw.inc_off + t.x + t.y) - jb;
            for (int w = tid; w < cnt * words; w += blockDim.x) cs[t.w * words + w] = __ldg(p.sw.crec + jb * words + w);
            if constexpr (LAYOUT == 4)
                for (int i = tid; i < cnt; i += blockDim.x) cm[t.w + i] = __ldg(p.sw.cmat + jb + i);
            for (int i = tid; i < t.y; i += blockDim.x)
                spans[t.z + i] = make_int2(t.w + __ldg(p.sw.inc_off + t.x + i) - jb,
                                           t.w + __ldg(p.sw.inc_off + t.x + i + 1) - jb);
        }
    cluster_arrive();
    cluster_wait();
    if (ok_plan)  // inertial targets: the predictor's writes are visible after the barrier
        for (int sl = 0; sl < p.srec_slices; ++sl) {
            const int4 t = tab[sl];
            for (int i = tid; i < t.y; i += blockDim.x) ys[t.z + i] = __ldcg(p.sw.y + t.x + i);
        }
    __syncthreads();

    int cur = 0;
    unsigned gc = 0;
    bool alive = ok_plan;
    for (int k = 0; k < p.iters && alive; ++k) {
        const float om = __ldg(p.omega + k);
        const bool blend = om > 1.0f;
        const float4* xs = sx + (cur ? n : 0);
        const float4* xb = sx + (cur ? 0 : n);
        for (int c = 0; c < p.ncol; ++c, ++gc) {
            const int vb = __ldg(p.cstart + c), ve = __ldg(p.cstart + c + 1);
            const unsigned bar = bar0 + 8u * (gc & 1u);
            const int rounds = (ve - vb + ngroups - 1) / ngroups;
            for (int r = 0; r < rounds; ++r) {
                const int v = vb + r * ngroups + grp;
                const int lv = tab[rows[c] + r].z + lg;
                cluster_vertex_srec<LANES, LAYOUT>(p, xs, xb, cs, cm, ys, pps, spans, bar, v, lv, v < ve, lane, lane_w,
                                                   csize, blend, om);
            }
            const bool ok = mbar_wait(bar, (gc >> 1) & 1u, p.sw.status);
            if (tid == 0 && ok && gc + 2 < total) mbar_expect(bar, walk_bytes(p, gc + 2));
            alive = __syncthreads_and(ok) != 0;
            if (!alive) break;
        }
        if (blend) cur ^= 1;
    }
    cluster_arrive();
    cluster_wait();
    if (!alive) return;
    const float4* xf = sx + (cur ? n : 0);
    for (int i = gt; i < p.nfree; i += nthreads) {
        const float4 xi = xf[i];
        p.xa[i] = xi;
        if (p.finish) p.v[i] = damped_velocity(xi, p.xprev[i], p.v[i], p.h);
    }
}

// ---- The adjoint sweeps of one sub-step as a cluster walk ----------------------------------------
//
// The same exchange for the adjoint's coloured Gauss-Seidel on (M/h^2 + H) lam = G: every CTA holds
// the converged positions X and both adjoint buffers of the whole mesh, plus the pre-sweep adjoint
// of the vertices it sweeps (64 B per vertex); a vertex group reads X and lam from its own copy and
// sends lam~ (and the blended adjoint) to every CTA with st.async.  Arithmetic as k_adj_sweep
// (fact_adjoint, group_reduce, adj_block_solve, adj_blend), so lam equals the launch-per-colour
// path's bit for bit.
struct AdjWalkParams {
    AdjParams a;           // X, G, y (mass), element records, dtsr; lam / lam_next / lam_pp unused
    float4* lam0;          // the adjoint at entry (the walk starts from it)
    float4* lam1;          // the other buffer; the result lands in lam0 or lam1 as the blends flip
    const int* cstart;
    const float* omega;    // Chebyshev weight of each sweep (1 = no blend)
    unsigned long long* status;
    int ncol, sweeps, n, nfree;
    int keep_pp;           // Chebyshev on: keep the pre-sweep adjoint
    int alternate;         // even sweeps take the colours in reverse order
};

template <int LAYOUT> struct AdjAhead {
    typename AdjElem<LAYOUT>::Rec buf[kClusterAhead];
    float4 g, q;  // right-hand side and pre-sweep adjoint of the group's vertex (first lane)
    float m;      // its mass
    int j0, j1;
};

template <int LANES, int LAYOUT>
__device__ __forceinline__ void load_adj_ahead(const AdjWalkParams& p, const float4* pp, int v, bool active, int lane,
                                               AdjAhead<LAYOUT>& a) {
    a.j0 = 0;
    a.j1 = 0;
    if (active) {
        a.j0 = __ldg(p.a.inc_off + v);
        a.j1 = __ldg(p.a.inc_off + v + 1);
    }
    const int j = a.j0 + lane;
#pragma unroll
    for (int k = 0; k < kClusterAhead; ++k)
        if (j + k * LANES < a.j1) a.buf[k] = AdjElem<LAYOUT>::fetch(p.a, j + k * LANES);
    if (active && lane == 0) {
        a.g = __ldg(p.a.G + v);
        a.m = __ldg(&p.a.y[v].w);
        a.q = pp[v];
    }
}

template <int LANES, int LAYOUT>
__device__ __forceinline__ void cluster_adj_vertex(const AdjWalkParams& p, const float4* sX, const float4* lr,
                                                   const float4* lo, float4* pp, unsigned bar, int v, bool active,
                                                   int lane, int lane_w, unsigned csize, bool blend, float omega,
                                                   const AdjAhead<LAYOUT>& a) {
    const float4 xi = active ? sX[v] : make_float4(0.f, 0.f, 0.f, 0.f);
    Acc acc;  // h.. = diagonal block, g. = off-diagonal product
    acc.zero();
    const int j = a.j0 + lane;
#pragma unroll
    for (int k = 0; k < kClusterAhead; ++k)
        if (j + k * LANES < a.j1) fact_adjoint(decode_fact(a.buf[k]), xi, sX, lr, acc);
    for (int jj = j + kClusterAhead * LANES; jj < a.j1; jj += LANES)
        fact_adjoint(decode_fact(AdjElem<LAYOUT>::fetch(p.a, jj)), xi, sX, lr, acc);
    group_reduce<LANES>(acc);
    float4 l = make_float4(0.f, 0.f, 0.f, 0.f), la = l;
    if (active && lane == 0) {
        l = adj_block_solve(acc, a.m, p.a.dtsr, a.g);
        const float4 lold = lr[v];
        if (blend) la = adj_blend(l, a.q, omega);
        if (p.keep_pp) pp[v] = lold;
    }
    const int leader = lane_w & ~(LANES - 1);
    l.x = __shfl_sync(0xffffffffu, l.x, leader);
    l.y = __shfl_sync(0xffffffffu, l.y, leader);
    l.z = __shfl_sync(0xffffffffu, l.z, leader);
    l.w = __shfl_sync(0xffffffffu, l.w, leader);
    if (blend) {
        la.x = __shfl_sync(0xffffffffu, la.x, leader);
        la.y = __shfl_sync(0xffffffffu, la.y, leader);
        la.z = __shfl_sync(0xffffffffu, la.z, leader);
        la.w = __shfl_sync(0xffffffffu, la.w, leader);
    }
    if (!active) return;
    const unsigned sn = (unsigned)__cvta_generic_to_shared(lr + v);
    const unsigned sa = (unsigned)__cvta_generic_to_shared(lo + v);
    for (unsigned r = (unsigned)lane; r < csize; r += LANES) {
        const unsigned rb = cluster_map(bar, r);
        st_async(cluster_map(sn, r), l, rb);
        if (blend) st_async(cluster_map(sa, r), la, rb);
    }
}

// The colour swept k-th in sweep `it` (1-based): reversed on even sweeps when alternating.
__device__ __forceinline__ int adj_colour(const AdjWalkParams& p, int it, int k) {
    return (p.alternate && (it % 2 == 0)) ? p.ncol - 1 - k : k;
}

// Bytes the g-th colour swept (over all sweeps) brings to every CTA.
__device__ __forceinline__ unsigned adj_walk_bytes(const AdjWalkParams& p, unsigned g) {
    const int it = (int)(g / (unsigned)p.ncol) + 1;
    const int col = adj_colour(p, it, (int)(g % (unsigned)p.ncol));
    const int size = __ldg(p.cstart + col + 1) - __ldg(p.cstart + col);
    return (unsigned)size * (__ldg(p.omega + it - 1) > 1.0f ? 32u : 16u);
}

template <int LANES, int LAYOUT>
__global__ void __launch_bounds__(kClusterMaxBlock, 1) k_cluster_adjoint(AdjWalkParams p) {
    extern __shared__ float4 sx[];  // [0, n): X, [n, 2n) and [2n, 3n): lam buffers, [3n, 4n): lam_pp
    __shared__ __align__(8) unsigned long long mbar[2];
    const int n = p.n;
    const float4* sX = sx;
    float4* sL = sx + n;
    float4* spp = sx + 3 * n;
    const unsigned csize = cluster_size();
    const int tid = threadIdx.x;
    const int gt = (int)cluster_rank() * (int)blockDim.x + tid;
    const int nthreads = (int)csize * (int)blockDim.x;
    const int lane_w = tid & 31;
    const int lane = LANES == 1 ? 0 : (lane_w & (LANES - 1));
    const int grp = gt / LANES;
    const int ngroups = nthreads / LANES;
    const unsigned bar0 = (unsigned)__cvta_generic_to_shared(&mbar[0]);
    // the byte announcements follow the forward walk's order (k_cluster_walk)
    const unsigned total = (unsigned)max(p.sweeps, 0) * (unsigned)p.ncol;
    if (tid == 0) {
        mbar_init(bar0);
        mbar_init(bar0 + 8);
        if (total > 0) mbar_expect(bar0, adj_walk_bytes(p, 0));
        if (total > 1) mbar_expect(bar0 + 8, adj_walk_bytes(p, 1));
        fence_mbar_init();
    }
    // both buffers start from the entry adjoint (pinned entries are 0 and stay 0)
    for (int i = tid; i < n; i += blockDim.x) {
        sx[i] = __ldg(p.a.X + i);
        const float4 l = p.lam0[i];
        sL[i] = l;
        sL[n + i] = l;
    }
    cluster_arrive();
    AdjAhead<LAYOUT> ah;
    if (p.sweeps > 0 && p.ncol > 0) {
        const int c0 = adj_colour(p, 1, 0);
        const int v = __ldg(p.cstart + c0) + grp;
        load_adj_ahead<LANES, LAYOUT>(p, spp, v, v < __ldg(p.cstart + c0 + 1), lane, ah);
    }
    cluster_wait();

    int cur = 0;
    unsigned gc = 0;
    bool alive = true;
    for (int it = 1; it <= p.sweeps && alive; ++it) {
        const float om = __ldg(p.omega + it - 1);
        const bool blend = om > 1.0f;
        const float4* lr = sL + (cur ? n : 0);
        const float4* lo = sL + (cur ? 0 : n);
        for (int k = 0; k < p.ncol; ++k, ++gc) {
            const int col = adj_colour(p, it, k);
            const int vb = __ldg(p.cstart + col), ve = __ldg(p.cstart + col + 1);
            const unsigned bar = bar0 + 8u * (gc & 1u);
            const int rounds = (ve - vb + ngroups - 1) / ngroups;
            for (int r = 0; r < rounds; ++r) {
                const int v = vb + r * ngroups + grp;
                const bool active = v < ve;
                if (r == 0) {
                    cluster_adj_vertex<LANES, LAYOUT>(p, sX, lr, lo, spp, bar, v, active, lane, lane_w, csize, blend,
                                                      om, ah);
                } else {
                    AdjAhead<LAYOUT> a;
                    load_adj_ahead<LANES, LAYOUT>(p, spp, v, active, lane, a);
                    cluster_adj_vertex<LANES, LAYOUT>(p, sX, lr, lo, spp, bar, v, active, lane, lane_w, csize, blend,
                                                      om, a);
                }
            }
            // the first round of the colour swept next
            const bool last = (it == p.sweeps) && (k == p.ncol - 1);
            if (!last) {
                const int cn = k + 1 < p.ncol ? adj_colour(p, it, k + 1) : adj_colour(p, it + 1, 0);
                const int v = __ldg(p.cstart + cn) + grp;
                load_adj_ahead<LANES, LAYOUT>(p, spp, v, v < __ldg(p.cstart + cn + 1), lane, ah);
            }
            const bool ok = mbar_wait(bar, (gc >> 1) & 1u, p.status);
            if (tid == 0 && ok && gc + 2 < total) mbar_expect(bar, adj_walk_bytes(p, gc + 2));
            alive = __syncthreads_and(ok) != 0;
            if (!alive) break;
        }
        if (blend) cur ^= 1;
    }
    cluster_arrive();
    cluster_wait();
    if (!alive) return;
    // the adjoint of the free vertices back to the buffer the launch-per-colour path leaves it in
    const float4* lf = sL + (cur ? n : 0);
    float4* out = cur ? p.lam1 : p.lam0;
    for (int i = gt; i < p.nfree; i += nthreads) out[i] = lf[i];
}

}  // namespace vbd
