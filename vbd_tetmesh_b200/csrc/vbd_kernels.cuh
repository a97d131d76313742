// Device code of the VBD solver: data layout, per-incidence element math and the kernels.
//
// Layout in HBM (one mesh, or a batch of meshes concatenated):
//   Vertices are renumbered "internally": the free vertices of colour 0, then of colour 1, ...,
//   then every pinned vertex.  Each colour is therefore one contiguous id range and a sweep
//   kernel reads and writes its own vertices' state fully coalesced.
//   float4 x[2][N]   positions, ping-pong pair (w unused)      -- Chebyshev needs x~ and x^(k)
//   float4 pp[N]     position before the previous sweep       -- VBDsolver::prevPrevPos
//   float4 y[N]      inertial target, w = lumped mass         -- TetMesh::mInertia / vertexMass
//   float4 v[N], xprev[N]                                       -- TetMesh::mVelocity / mVertPrevPos
//   TetRec rec[T]    64 B per tet, in the caller's tet order:  four internal vertex ids, Dm^-1
//                    row-major, V0, mu, lambda
//   int inc_off[N+1], inc_tet[4T]: per free vertex, its incident tets in ascending tet id
//                    (TetMesh::vertAdjacentTets); pinned vertices own none.
//   TetRec irec[4T]  (optional "streamed" layout) rec[inc_tet[j]] copied in incidence order, so a
//                    sweep reads its element data as one sequential stream.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace vbd {

struct __align__(16) TetRec {
    int4 ids;   // internal vertex ids in the tet's local order
    float4 a;   // Dm^-1: (0,0) (0,1) (0,2) (1,0)
    float4 b;   //        (1,1) (1,2) (2,0) (2,1)
    float4 c;   //        (2,2), V0, mu, lambda
};
static_assert(sizeof(TetRec) == 64, "TetRec must be 64 bytes");

// ST_TIMEOUT: a grid barrier of the persistent kernel gave up; ST_WALK_TIMEOUT: an mbarrier wait
// of a cluster walk gave up.
enum StatusSlot { ST_SINGULAR = 0, ST_NONFINITE = 1, ST_TIMEOUT = 2, ST_WALK_TIMEOUT = 3, ST_SLOTS = 4 };

struct SweepParams {
    float4* x;                 // positions being swept in place (Gauss-Seidel)
    float4* xnext;             // receives the Chebyshev-blended position (when accel)
    float4* pp;                // position before the previous sweep
    const float4* y;           // inertial target, w = mass
    const int* inc_off;
    const int* inc_tet;
    const TetRec* rec;
    const TetRec* irec;
    const int4* crec;          // streamed incidence records: 3 x int4 (layouts 2, 3) or 2 x int4 (layout 4)
    const float2* cmat;        // (V0 mu, V0 lambda) per incidence (layouts 2, 4)
    unsigned long long* status;
    int v_begin, v_end;
    float dtsr;                // 1/h^2
    float omega;
    int accel;                 // write x^(k) = omega (x~ - pp) + pp to xnext (VBD.cpp:290-300)
    int keep_pp;               // store the pre-sweep position into pp (VBD.cpp:78,89)
    // Streamed records of incidences below persist_end are read with the L2 evict-last policy, the
    // rest evict-first (kernels built with a record cache policy only).  The two ints also keep
    // this block above 128 bytes: on the 64^3 cube the step measured 4.61 ms at 136 bytes (and the
    // same at 152 to 264), 4.81 ms at 128 and 5.05 ms at 120 (A/B on one B200, kernel arithmetic
    // unchanged); the cause is not known.
    int persist_end;
    int reserved_;
    const char* l2_next;       // element records of the colour swept next (16 B aligned), prefetched
    unsigned long long l2_bytes;  // into L2 while this colour runs; 0 = none
};

// Programmatic dependent launch: let the next kernel in the stream start its prologue now, and
// wait until every kernel before this one has finished and its writes are visible.  Both are
// no-ops for a kernel launched without the programmatic-serialization attribute.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ TetRec load_rec(const TetRec* p) {
    TetRec r;
    const int4* q = reinterpret_cast<const int4*>(p);
    r.ids = __ldg(q);
    int4 t;
    t = __ldg(q + 1);
    r.a = make_float4(__int_as_float(t.x), __int_as_float(t.y), __int_as_float(t.z), __int_as_float(t.w));
    t = __ldg(q + 2);
    r.b = make_float4(__int_as_float(t.x), __int_as_float(t.y), __int_as_float(t.z), __int_as_float(t.w));
    t = __ldg(q + 3);
    r.c = make_float4(__int_as_float(t.x), __int_as_float(t.y), __int_as_float(t.z), __int_as_float(t.w));
    return r;
}

// Accumulators of one vertex's elastic terms: the symmetric 3x3 Hessian block (6 entries) and
// the gradient (3 entries).
struct Acc {
    float h00, h01, h02, h11, h12, h22, g0, g1, g2;
    __device__ __forceinline__ void zero() { h00 = h01 = h02 = h11 = h12 = h22 = g0 = g1 = g2 = 0.f; }
};

// Element contribution of tet `r` to vertex `v` (internal id), whose position is `xi`.
// Neighbour positions are gathered from X, which this kernel never writes at those ids (they are
// of another colour).  Follows ElasticEnergy::compute_Hessian_and_Gradient (Energy.cpp:90-158)
// as used by VBDsolver::computeTetContribution (VBD.cpp:205-256):
//   Ds = [x1-x0, x2-x0, x3-x0], F = Ds Dm^-1, J = det F, C = cof F,
//   P = mu (F - C) + lambda (J - 1) C, q = row n of Ps Dm^-1,
//   gradient  g_n  = V P q,
//   Hessian   H_nn = V (mu |q|^2 I + lambda (C q)(C q)^T)   -- the (n,n) block of the literal
//   12x12 assembly; the cofactor-derivative terms vanish in that block because dC_ij/dF_kl is
//   antisymmetric in (j,l) and is contracted with the symmetric q q^T.
// Position loads: the read-only path when positions cannot change while the kernel runs (one
// colour per launch), plain coherent loads inside the persistent kernel, where other blocks
// rewrite them between grid barriers.
template <bool COHERENT> __device__ __forceinline__ float4 load_pos(const float4* X, int i) {
    if (COHERENT) return X[i];
    return __ldg(X + i);
}

template <bool WANT_H, bool COHERENT = false>
__device__ __forceinline__ void tet_contrib(const TetRec& r, int v, float4 xi, const float4* __restrict__ X,
                                            Acc& acc) {
    const int i0 = r.ids.x, i1 = r.ids.y, i2 = r.ids.z, i3 = r.ids.w;
    const float4 p0 = (i0 == v) ? xi : load_pos<COHERENT>(X, i0);
    const float4 p1 = (i1 == v) ? xi : load_pos<COHERENT>(X, i1);
    const float4 p2 = (i2 == v) ? xi : load_pos<COHERENT>(X, i2);
    const float4 p3 = (i3 == v) ? xi : load_pos<COHERENT>(X, i3);
    const int n = (i0 == v) ? 0 : (i1 == v) ? 1 : (i2 == v) ? 2 : 3;

    const float D00 = r.a.x, D01 = r.a.y, D02 = r.a.z, D10 = r.a.w;
    const float D11 = r.b.x, D12 = r.b.y, D20 = r.b.z, D21 = r.b.w;
    const float D22 = r.c.x, V0 = r.c.y, mu = r.c.z, lam = r.c.w;

    const float e1x = p1.x - p0.x, e1y = p1.y - p0.y, e1z = p1.z - p0.z;
    const float e2x = p2.x - p0.x, e2y = p2.y - p0.y, e2z = p2.z - p0.z;
    const float e3x = p3.x - p0.x, e3y = p3.y - p0.y, e3z = p3.z - p0.z;

    // F = Ds * Dm^-1
    const float F00 = e1x * D00 + e2x * D10 + e3x * D20;
    const float F01 = e1x * D01 + e2x * D11 + e3x * D21;
    const float F02 = e1x * D02 + e2x * D12 + e3x * D22;
    const float F10 = e1y * D00 + e2y * D10 + e3y * D20;
    const float F11 = e1y * D01 + e2y * D11 + e3y * D21;
    const float F12 = e1y * D02 + e2y * D12 + e3y * D22;
    const float F20 = e1z * D00 + e2z * D10 + e3z * D20;
    const float F21 = e1z * D01 + e2z * D11 + e3z * D21;
    const float F22 = e1z * D02 + e2z * D12 + e3z * D22;

    // cofactor matrix
    const float C00 = F11 * F22 - F12 * F21;
    const float C01 = F12 * F20 - F10 * F22;
    const float C02 = F10 * F21 - F11 * F20;
    const float C10 = F21 * F02 - F22 * F01;
    const float C11 = F22 * F00 - F20 * F02;
    const float C12 = F20 * F01 - F21 * F00;
    const float C20 = F01 * F12 - F02 * F11;
    const float C21 = F02 * F10 - F00 * F12;
    const float C22 = F00 * F11 - F01 * F10;
    const float J = F00 * C00 + F01 * C01 + F02 * C02;
    const float s = lam * (J - 1.0f);

    // q = row n of Ps * Dm^-1
    float qx, qy, qz;
    if (n == 0) {
        qx = -D00 - D10 - D20;
        qy = -D01 - D11 - D21;
        qz = -D02 - D12 - D22;
    } else if (n == 1) {
        qx = D00; qy = D01; qz = D02;
    } else if (n == 2) {
        qx = D10; qy = D11; qz = D12;
    } else {
        qx = D20; qy = D21; qz = D22;
    }

    const float Fq0 = F00 * qx + F01 * qy + F02 * qz;
    const float Fq1 = F10 * qx + F11 * qy + F12 * qz;
    const float Fq2 = F20 * qx + F21 * qy + F22 * qz;
    const float Cq0 = C00 * qx + C01 * qy + C02 * qz;
    const float Cq1 = C10 * qx + C11 * qy + C12 * qz;
    const float Cq2 = C20 * qx + C21 * qy + C22 * qz;

    acc.g0 += V0 * (mu * (Fq0 - Cq0) + s * Cq0);
    acc.g1 += V0 * (mu * (Fq1 - Cq1) + s * Cq1);
    acc.g2 += V0 * (mu * (Fq2 - Cq2) + s * Cq2);
    if (WANT_H) {
        const float a = V0 * mu * (qx * qx + qy * qy + qz * qz);
        const float b = V0 * lam;
        const float b0 = b * Cq0, b1 = b * Cq1, b2 = b * Cq2;
        acc.h00 += a + b0 * Cq0;
        acc.h01 += b0 * Cq1;
        acc.h02 += b0 * Cq2;
        acc.h11 += a + b1 * Cq1;
        acc.h12 += b1 * Cq2;
        acc.h22 += a + b2 * Cq2;
    }
}

// Compact incidence record (layout 2), 48 B + 8 B per (vertex, tet) incidence:
//   int4  {nb0 | n << 30, nb1, nb2, q0.x}   the tet's other three vertices in local order, the
//   float4{q0.y, q0.z, q1.x, q1.y}           vertex's own local index n, and rows q_k of
//   float4{q1.z, q2.x, q2.y, q2.z}           Q = Ps Dm^-1 for those three vertices
//   float2{V0 mu, V0 lambda}                 (separate stream)
// Because the rows of Q sum to zero, F = Ds Dm^-1 = sum_k (x_k - x_n) q_k^T over the three other
// vertices, and the vertex's own row is q_n = -(q0 + q1 + q2).
struct CompactRec {
    int nb0, nb1, nb2;
    float q[9];
    float a, b;  // V0 mu, V0 lambda
};

constexpr int kCompactIdMask = 0x3fffffff;

__device__ __forceinline__ CompactRec load_compact(const int4* __restrict__ crec, const float2* __restrict__ cmat,
                                                   int j) {
    const int4 w0 = __ldg(crec + 3 * j);
    const int4 w1 = __ldg(crec + 3 * j + 1);
    const int4 w2 = __ldg(crec + 3 * j + 2);
    const float2 m = __ldg(cmat + j);
    CompactRec r;
    r.nb0 = w0.x & kCompactIdMask;
    r.nb1 = w0.y;
    r.nb2 = w0.z;
    r.q[0] = __int_as_float(w0.w);
    r.q[1] = __int_as_float(w1.x);
    r.q[2] = __int_as_float(w1.y);
    r.q[3] = __int_as_float(w1.z);
    r.q[4] = __int_as_float(w1.w);
    r.q[5] = __int_as_float(w2.x);
    r.q[6] = __int_as_float(w2.y);
    r.q[7] = __int_as_float(w2.z);
    r.q[8] = __int_as_float(w2.w);
    r.a = m.x;
    r.b = m.y;
    return r;
}

// Same element block as tet_contrib, from a compact record: g_n = V P q_n,
// H_nn = V (mu |q_n|^2 I + lambda (C q_n)(C q_n)^T), with V mu and V lambda premultiplied.
template <bool WANT_H, bool COHERENT = false>
__device__ __forceinline__ void compact_contrib(const CompactRec& r, float4 xi, const float4* __restrict__ X,
                                                Acc& acc) {
    const float4 p0 = load_pos<COHERENT>(X, r.nb0);
    const float4 p1 = load_pos<COHERENT>(X, r.nb1);
    const float4 p2 = load_pos<COHERENT>(X, r.nb2);
    const float d0x = p0.x - xi.x, d0y = p0.y - xi.y, d0z = p0.z - xi.z;
    const float d1x = p1.x - xi.x, d1y = p1.y - xi.y, d1z = p1.z - xi.z;
    const float d2x = p2.x - xi.x, d2y = p2.y - xi.y, d2z = p2.z - xi.z;
    const float* q = r.q;
    const float F00 = d0x * q[0] + d1x * q[3] + d2x * q[6];
    const float F01 = d0x * q[1] + d1x * q[4] + d2x * q[7];
    const float F02 = d0x * q[2] + d1x * q[5] + d2x * q[8];
    const float F10 = d0y * q[0] + d1y * q[3] + d2y * q[6];
    const float F11 = d0y * q[1] + d1y * q[4] + d2y * q[7];
    const float F12 = d0y * q[2] + d1y * q[5] + d2y * q[8];
    const float F20 = d0z * q[0] + d1z * q[3] + d2z * q[6];
    const float F21 = d0z * q[1] + d1z * q[4] + d2z * q[7];
    const float F22 = d0z * q[2] + d1z * q[5] + d2z * q[8];
    const float C00 = F11 * F22 - F12 * F21;
    const float C01 = F12 * F20 - F10 * F22;
    const float C02 = F10 * F21 - F11 * F20;
    const float C10 = F21 * F02 - F22 * F01;
    const float C11 = F22 * F00 - F20 * F02;
    const float C12 = F20 * F01 - F21 * F00;
    const float C20 = F01 * F12 - F02 * F11;
    const float C21 = F02 * F10 - F00 * F12;
    const float C22 = F00 * F11 - F01 * F10;
    const float J = F00 * C00 + F01 * C01 + F02 * C02;
    const float qx = -(q[0] + q[3] + q[6]);
    const float qy = -(q[1] + q[4] + q[7]);
    const float qz = -(q[2] + q[5] + q[8]);
    const float Fq0 = F00 * qx + F01 * qy + F02 * qz;
    const float Fq1 = F10 * qx + F11 * qy + F12 * qz;
    const float Fq2 = F20 * qx + F21 * qy + F22 * qz;
    const float Cq0 = C00 * qx + C01 * qy + C02 * qz;
    const float Cq1 = C10 * qx + C11 * qy + C12 * qz;
    const float Cq2 = C20 * qx + C21 * qy + C22 * qz;
    const float bj = r.b * (J - 1.0f);
    acc.g0 += r.a * (Fq0 - Cq0) + bj * Cq0;
    acc.g1 += r.a * (Fq1 - Cq1) + bj * Cq1;
    acc.g2 += r.a * (Fq2 - Cq2) + bj * Cq2;
    if (WANT_H) {
        const float am = r.a * (qx * qx + qy * qy + qz * qz);
        const float b0 = r.b * Cq0, b1 = r.b * Cq1, b2 = r.b * Cq2;
        acc.h00 += am + b0 * Cq0;
        acc.h01 += b0 * Cq1;
        acc.h02 += b0 * Cq2;
        acc.h11 += am + b1 * Cq1;
        acc.h12 += b1 * Cq2;
        acc.h22 += am + b2 * Cq2;
    }
}

// Factored incidence record (layout 3), 48 B per (vertex, tet) incidence.  With M the 3x3
// matrix whose rows are q_k of the three other vertices (the compact record's q) and q_n their
// negated sum, F = D M for D = [d_0 d_1 d_2], d_k = x_k - x_n.  Hence
//   F q_n = D s,          s = M q_n
//   C q_n = cof(D) w,     w = cof(M) q_n       (cof(D M) = cof(D) cof(M))
//   J     = det(D) det(M)
// and cof(D) has the columns d_1 x d_2, d_2 x d_0, d_0 x d_1.  The per-incidence constants s, w,
// det M are packed once, so a sweep never forms F or cof(F): about 70 floating-point operations
// per incidence instead of about 115.  Same element block as tet_contrib up to rounding.
//   int4  {nb0 | n << 30, nb1, nb2, s0}
//   float4{s1, s2, w0, w1}
//   float4{w2, det M, V0 mu, V0 lambda}
// |q_n|^2 (for the Hessian's V0 mu |q_n|^2 I term) is -(s0 + s1 + s2), since the rows of Q sum to
// zero; it is not stored (a 4 B stream per incidence cost 0.17 ms of the cube's 4.78 ms step).
struct FactRec {
    int nb0, nb1, nb2;
    float s0, s1, s2, w0, w1, w2, detm, a, b, am;
};

// The raw words of a factored record.  A fetch only loads them; they are decoded where the record
// is used, so no instruction waits on a prefetched record before the next prefetch is issued.
struct FactRaw3 {
    int4 w0;
    float4 w1, w2;
};

__device__ __forceinline__ FactRaw3 load_fact(const int4* __restrict__ crec, int j) {
    FactRaw3 r;
    r.w0 = __ldg(crec + 3 * j);
    r.w1 = __ldg(reinterpret_cast<const float4*>(crec) + 3 * j + 1);
    r.w2 = __ldg(reinterpret_cast<const float4*>(crec) + 3 * j + 2);
    return r;
}

__device__ __forceinline__ FactRec decode_fact(const FactRaw3& w) {
    FactRec r;
    r.nb0 = w.w0.x & kCompactIdMask;
    r.nb1 = w.w0.y;
    r.nb2 = w.w0.z;
    r.s0 = __int_as_float(w.w0.w);
    r.s1 = w.w1.x;
    r.s2 = w.w1.y;
    r.w0 = w.w1.z;
    r.w1 = w.w1.w;
    r.w2 = w.w2.x;
    r.detm = w.w2.y;
    r.a = w.w2.z;
    r.b = w.w2.w;
    // V0 mu |q_n|^2: the rows of Q sum to zero, so sum_k s_k = sum_k q_k . q_n = -|q_n|^2.  Rounded
    // on its own (no fused multiply-add into the Hessian sums), so every launch shape computes it
    // identically.
    r.am = __fmul_rn(r.a, -(r.s0 + r.s1 + r.s2));
    return r;
}

// Packed factored record (layout 4), 40 B per incidence in two streams:
//   int4  {ids.lo, ids.hi, s0, s1}    the other three vertices, 21 bits each in 64 bits
//   float4{s2, w0, w1, w2}
//   float2{V0 mu, V0 lambda}          (separate stream, as for layout 2)
// det M is not stored: M^T cof(M) = det(M) I gives s . w = q_n^T M^T cof(M) q_n = det(M) |q_n|^2,
// with |q_n|^2 = -(s0 + s1 + s2) as above.  The local index n is not needed by the factored form.
// Ids must be below 2^21; the host keeps layout 3 for larger meshes.
constexpr int kPackedIdBits = 21;
constexpr int kPackedIdMask = (1 << kPackedIdBits) - 1;
constexpr long long kPackedMaxVertices = 1LL << kPackedIdBits;

struct FactRaw4 {
    int4 w0;
    float4 w1;
    float2 m;
};

__device__ __forceinline__ FactRaw4 load_fact_packed(const int4* __restrict__ crec, const float2* __restrict__ cmat,
                                                     int j) {
    FactRaw4 r;
    r.w0 = __ldg(crec + 2 * j);
    r.w1 = __ldg(reinterpret_cast<const float4*>(crec) + 2 * j + 1);
    r.m = __ldg(cmat + j);
    return r;
}

// L2 eviction policy of a streamed record load (createpolicy): evict-first for records that are
// read once per sweep, so that they do not push the vertex state out of L2; evict-last for the
// share of the stream that is kept resident across sweeps.
__device__ __forceinline__ unsigned long long record_policy(bool keep) {
    unsigned long long first, last;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(first));
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(last));
    return keep ? last : first;
}

// Read-only record loads with an L2 policy; the records bypass L1, which keeps its capacity for
// the neighbour positions.
__device__ __forceinline__ int4 ld_rec(const int4* p, unsigned long long pol) {
    int4 r;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%4], %5;"
        : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
        : "l"(p), "l"(pol));
    return r;
}

__device__ __forceinline__ float4 ld_rec(const float4* p, unsigned long long pol) {
    float4 r;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
        : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
        : "l"(p), "l"(pol));
    return r;
}

__device__ __forceinline__ float2 ld_rec(const float2* p, unsigned long long pol) {
    float2 r;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f32 {%0,%1}, [%2], %3;"
        : "=f"(r.x), "=f"(r.y)
        : "l"(p), "l"(pol));
    return r;
}

__device__ __forceinline__ FactRaw4 load_fact_packed(const int4* __restrict__ crec, const float2* __restrict__ cmat,
                                                     int j, unsigned long long pol) {
    FactRaw4 r;
    r.w0 = ld_rec(crec + 2 * j, pol);
    r.w1 = ld_rec(reinterpret_cast<const float4*>(crec) + 2 * j + 1, pol);
    r.m = ld_rec(cmat + j, pol);
    return r;
}

__device__ __forceinline__ FactRaw3 load_fact(const int4* __restrict__ crec, int j, unsigned long long pol) {
    FactRaw3 r;
    r.w0 = ld_rec(crec + 3 * j, pol);
    r.w1 = ld_rec(reinterpret_cast<const float4*>(crec) + 3 * j + 1, pol);
    r.w2 = ld_rec(reinterpret_cast<const float4*>(crec) + 3 * j + 2, pol);
    return r;
}

__device__ __forceinline__ FactRec decode_fact(const FactRaw4& w) {
    const unsigned lo = (unsigned)w.w0.x, hi = (unsigned)w.w0.y;
    FactRec r;
    r.nb0 = (int)(lo & kPackedIdMask);
    r.nb1 = (int)(__funnelshift_r(lo, hi, kPackedIdBits) & kPackedIdMask);
    r.nb2 = (int)((hi >> (2 * kPackedIdBits - 32)) & kPackedIdMask);
    r.s0 = __int_as_float(w.w0.z);
    r.s1 = __int_as_float(w.w0.w);
    r.s2 = w.w1.x;
    r.w0 = w.w1.y;
    r.w1 = w.w1.z;
    r.w2 = w.w1.w;
    r.a = w.m.x;
    r.b = w.m.y;
    // Explicit roundings, so every launch shape derives the same det M and V0 mu |q_n|^2.
    const float qq = -(r.s0 + r.s1 + r.s2);
    const float sw = __fmaf_rn(r.s2, r.w2, __fmaf_rn(r.s1, r.w1, __fmul_rn(r.s0, r.w0)));
    r.detm = __fdiv_rn(sw, qq);
    r.am = __fmul_rn(r.a, qq);
    return r;
}

template <bool WANT_H, bool COHERENT = false>
__device__ __forceinline__ void fact_contrib(const FactRec& r, float4 xi, const float4* __restrict__ X, Acc& acc) {
    const float4 p0 = load_pos<COHERENT>(X, r.nb0);
    const float4 p1 = load_pos<COHERENT>(X, r.nb1);
    const float4 p2 = load_pos<COHERENT>(X, r.nb2);
    const float d0x = p0.x - xi.x, d0y = p0.y - xi.y, d0z = p0.z - xi.z;
    const float d1x = p1.x - xi.x, d1y = p1.y - xi.y, d1z = p1.z - xi.z;
    const float d2x = p2.x - xi.x, d2y = p2.y - xi.y, d2z = p2.z - xi.z;
    // columns of cof(D)
    const float c0x = d1y * d2z - d1z * d2y, c0y = d1z * d2x - d1x * d2z, c0z = d1x * d2y - d1y * d2x;
    const float c1x = d2y * d0z - d2z * d0y, c1y = d2z * d0x - d2x * d0z, c1z = d2x * d0y - d2y * d0x;
    const float c2x = d0y * d1z - d0z * d1y, c2y = d0z * d1x - d0x * d1z, c2z = d0x * d1y - d0y * d1x;
    const float J = (d0x * c0x + d0y * c0y + d0z * c0z) * r.detm;
    const float Fq0 = d0x * r.s0 + d1x * r.s1 + d2x * r.s2;
    const float Fq1 = d0y * r.s0 + d1y * r.s1 + d2y * r.s2;
    const float Fq2 = d0z * r.s0 + d1z * r.s1 + d2z * r.s2;
    const float Cq0 = c0x * r.w0 + c1x * r.w1 + c2x * r.w2;
    const float Cq1 = c0y * r.w0 + c1y * r.w1 + c2y * r.w2;
    const float Cq2 = c0z * r.w0 + c1z * r.w1 + c2z * r.w2;
    const float bj = r.b * (J - 1.0f);
    acc.g0 += r.a * (Fq0 - Cq0) + bj * Cq0;
    acc.g1 += r.a * (Fq1 - Cq1) + bj * Cq1;
    acc.g2 += r.a * (Fq2 - Cq2) + bj * Cq2;
    if (WANT_H) {
        const float b0 = r.b * Cq0, b1 = r.b * Cq1, b2 = r.b * Cq2;
        acc.h00 += r.am + b0 * Cq0;
        acc.h01 += b0 * Cq1;
        acc.h02 += b0 * Cq2;
        acc.h11 += r.am + b1 * Cq1;
        acc.h12 += b1 * Cq2;
        acc.h22 += r.am + b2 * Cq2;
    }
}

template <int LANES>
__device__ __forceinline__ void group_reduce(Acc& a) {
#pragma unroll
    for (int o = LANES / 2; o > 0; o >>= 1) {
        a.h00 += __shfl_xor_sync(0xffffffffu, a.h00, o);
        a.h01 += __shfl_xor_sync(0xffffffffu, a.h01, o);
        a.h02 += __shfl_xor_sync(0xffffffffu, a.h02, o);
        a.h11 += __shfl_xor_sync(0xffffffffu, a.h11, o);
        a.h12 += __shfl_xor_sync(0xffffffffu, a.h12, o);
        a.h22 += __shfl_xor_sync(0xffffffffu, a.h22, o);
        a.g0 += __shfl_xor_sync(0xffffffffu, a.g0, o);
        a.g1 += __shfl_xor_sync(0xffffffffu, a.g1, o);
        a.g2 += __shfl_xor_sync(0xffffffffu, a.g2, o);
    }
}

// Element data of incidence j under each record layout:
//   0 = tet record gathered through inc_tet, 1 = tet record streamed in incidence order,
//   2 = compact streamed record, 3 = factored streamed record, 4 = packed factored record.
// fetch_hint loads the factored records with an L2 policy (record_policy); the other layouts
// ignore the policy.
template <int LAYOUT> struct Elem;
template <> struct Elem<0> {
    using Rec = TetRec;
    __device__ __forceinline__ static Rec fetch(const SweepParams& p, int j) {
        return load_rec(p.rec + __ldg(p.inc_tet + j));
    }
    __device__ __forceinline__ static Rec fetch_hint(const SweepParams& p, int j, unsigned long long) {
        return fetch(p, j);
    }
    template <bool COHERENT>
    __device__ __forceinline__ static void contrib(const Rec& r, int v, float4 xi, const float4* X, Acc& acc) {
        tet_contrib<true, COHERENT>(r, v, xi, X, acc);
    }
};
template <> struct Elem<1> {
    using Rec = TetRec;
    __device__ __forceinline__ static Rec fetch(const SweepParams& p, int j) { return load_rec(p.irec + j); }
    __device__ __forceinline__ static Rec fetch_hint(const SweepParams& p, int j, unsigned long long) {
        return fetch(p, j);
    }
    template <bool COHERENT>
    __device__ __forceinline__ static void contrib(const Rec& r, int v, float4 xi, const float4* X, Acc& acc) {
        tet_contrib<true, COHERENT>(r, v, xi, X, acc);
    }
};
template <> struct Elem<2> {
    using Rec = CompactRec;
    __device__ __forceinline__ static Rec fetch(const SweepParams& p, int j) { return load_compact(p.crec, p.cmat, j); }
    __device__ __forceinline__ static Rec fetch_hint(const SweepParams& p, int j, unsigned long long) {
        return fetch(p, j);
    }
    template <bool COHERENT>
    __device__ __forceinline__ static void contrib(const Rec& r, int, float4 xi, const float4* X, Acc& acc) {
        compact_contrib<true, COHERENT>(r, xi, X, acc);
    }
};
template <> struct Elem<3> {
    using Rec = FactRaw3;
    __device__ __forceinline__ static Rec fetch(const SweepParams& p, int j) { return load_fact(p.crec, j); }
    __device__ __forceinline__ static Rec fetch_hint(const SweepParams& p, int j, unsigned long long pol) {
        return load_fact(p.crec, j, pol);
    }
    template <bool COHERENT>
    __device__ __forceinline__ static void contrib(const Rec& r, int, float4 xi, const float4* X, Acc& acc) {
        fact_contrib<true, COHERENT>(decode_fact(r), xi, X, acc);
    }
};

template <> struct Elem<4> {
    using Rec = FactRaw4;
    __device__ __forceinline__ static Rec fetch(const SweepParams& p, int j) {
        return load_fact_packed(p.crec, p.cmat, j);
    }
    __device__ __forceinline__ static Rec fetch_hint(const SweepParams& p, int j, unsigned long long pol) {
        return load_fact_packed(p.crec, p.cmat, j, pol);
    }
    template <bool COHERENT>
    __device__ __forceinline__ static void contrib(const Rec& r, int, float4 xi, const float4* X, Acc& acc) {
        fact_contrib<true, COHERENT>(decode_fact(r), xi, X, acc);
    }
};

// The vertex block update of VBDsolver::solveVertex + solve (VBD.cpp:124-203) for vertex v:
// LANES threads split its incident tets, reduce with warp shuffles, and the group's first lane
// solves (m/h^2 I + sum H_nn) dx = m/h^2 (y - x) - sum g_n with the adjugate formula behind the
// |det| > 1e-8 guard (VBD.cpp:141-152, Types.h:85-112), then writes x~, the Chebyshev blend
// x^(k) = omega (x~ - pp) + pp (VBD.cpp:290-300) and the pre-sweep position into pp.
// Every lane of the warp must call it (shuffles); `active` marks lanes with a real vertex.
//   LAYOUT   : element record layout (Elem<0..4>)
//   PREFETCH : the next element record is loaded while the current one is evaluated
//   COHERENT : positions read with coherent loads (persistent kernel)
// `nxt` holds the lane's first record if PREFETCH (fetched by the caller).
template <int LANES>
__device__ __forceinline__ void vertex_solve(const SweepParams& p, int v, int lane, bool active, float4 xi, Acc& acc);

// Record j of a sweep: plain read-only loads, or (CACHE) loads with the L2 policy `pol`.
template <int LAYOUT, bool CACHE>
__device__ __forceinline__ typename Elem<LAYOUT>::Rec fetch_rec(const SweepParams& p, int j, unsigned long long pol) {
    if constexpr (CACHE) return Elem<LAYOUT>::fetch_hint(p, j, pol);
    else return Elem<LAYOUT>::fetch(p, j);
}

template <int LANES, int LAYOUT, bool PREFETCH, bool COHERENT, bool CACHE = false>
__device__ __forceinline__ void vertex_update(const SweepParams& p, int v, int lane, bool active, int j, int j1,
                                              typename Elem<LAYOUT>::Rec nxt, unsigned long long pol = 0) {
    const float4 xi = active ? p.x[v] : make_float4(0.f, 0.f, 0.f, 0.f);
    Acc acc;
    acc.zero();
    for (; j < j1; j += LANES) {
        typename Elem<LAYOUT>::Rec r;
        if (PREFETCH) {
            r = nxt;
            if (j + LANES < j1) nxt = fetch_rec<LAYOUT, CACHE>(p, j + LANES, pol);
        } else {
            r = fetch_rec<LAYOUT, CACHE>(p, j, pol);
        }
        Elem<LAYOUT>::template contrib<COHERENT>(r, v, xi, p.x, acc);
    }
    vertex_solve<LANES>(p, v, lane, active, xi, acc);
}

// The group's reduction and the first lane's block solve, Chebyshev blend and stores (the second
// half of vertex_update).
// The block solve of one vertex from its reduced sums (VBD.cpp:141-152, Types.h:85-112): returns
// the new position, or xi where |det H| <= 1e-8 (counted in status); flags a non-finite result.
__device__ __forceinline__ float4 block_solve(const Acc& acc, float4 xi, float4 yi, float dtsr,
                                              unsigned long long* status) {
    const float cm = yi.w * dtsr;
    const float H00 = cm + acc.h00, H01 = acc.h01, H02 = acc.h02;
    const float H11 = cm + acc.h11, H12 = acc.h12, H22 = cm + acc.h22;
    const float f0 = (yi.w * (yi.x - xi.x)) * dtsr - acc.g0;
    const float f1 = (yi.w * (yi.y - xi.y)) * dtsr - acc.g1;
    const float f2 = (yi.w * (yi.z - xi.z)) * dtsr - acc.g2;
    // adjugate of the symmetric H
    const float A00 = H11 * H22 - H12 * H12;
    const float A01 = H02 * H12 - H01 * H22;
    const float A02 = H01 * H12 - H02 * H11;
    const float A11 = H00 * H22 - H02 * H02;
    const float A12 = H02 * H01 - H00 * H12;
    const float A22 = H00 * H11 - H01 * H01;
    const float det = H00 * A00 + H01 * A01 + H02 * A02;
    float4 xn = xi;
    if (fabsf(det) > 1e-8f) {
        const float inv = 1.0f / det;
        xn.x = xi.x + inv * (A00 * f0 + A01 * f1 + A02 * f2);
        xn.y = xi.y + inv * (A01 * f0 + A11 * f1 + A12 * f2);
        xn.z = xi.z + inv * (A02 * f0 + A12 * f1 + A22 * f2);
    } else {
        atomicAdd(status + ST_SINGULAR, 1ull);
    }
    if (!(isfinite(xn.x) && isfinite(xn.y) && isfinite(xn.z))) status[ST_NONFINITE] = 1ull;
    return xn;
}

// The Chebyshev blend x^(k) = omega (x~ - pp) + pp (VBD.cpp:290-300).
__device__ __forceinline__ float4 cheb_blend(float4 xn, float4 q, float omega) {
    float4 xa;
    xa.x = omega * (xn.x - q.x) + q.x;
    xa.y = omega * (xn.y - q.y) + q.y;
    xa.z = omega * (xn.z - q.z) + q.z;
    xa.w = xn.w;
    return xa;
}

template <int LANES>
__device__ __forceinline__ void vertex_solve(const SweepParams& p, int v, int lane, bool active, float4 xi, Acc& acc) {
    group_reduce<LANES>(acc);
    if (!active || lane != 0) return;
    const float4 xn = block_solve(acc, xi, p.y[v], p.dtsr, p.status);
    p.x[v] = xn;
    if (p.accel) p.xnext[v] = cheb_blend(xn, p.pp[v], p.omega);
    if (p.keep_pp) p.pp[v] = xi;
}

// This block's share of [base, base + bytes) prefetched into L2 with one bulk prefetch
// (cp.async.bulk.prefetch: no shared memory, no completion to wait for).  The share is a
// 16-byte-aligned slice that stays inside the range; bytes is a multiple of 16 and base is
// 16-byte aligned.
__device__ __forceinline__ void l2_prefetch_share(const char* base, unsigned long long bytes) {
    const unsigned long long units = bytes >> 4;
    const unsigned long long per = (units + gridDim.x - 1) / gridDim.x;
    const unsigned long long first = per * blockIdx.x;
    if (first >= units) return;
    unsigned long long n = units - first < per ? units - first : per;
    const char* ptr = base + (first << 4);
    while (n) {
        const unsigned chunk = n > (1ull << 20) ? (1u << 20) : (unsigned)n;  // 16 MiB per instruction
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(ptr), "r"(chunk << 4) : "memory");
        ptr += (unsigned long long)chunk << 4;
        n -= chunk;
    }
}

// The vertex's inertial target and pre-sweep position, read by the group's first lane only after
// the element loop (vertex_solve), are prefetched into L1 right after the dependency wait, so their
// latency overlaps the loop instead of following it; no registers are held.  After the wait every
// earlier kernel's writes are visible, so the lines are current.  (Measured on the 64^3 cube: 4.26
// against 4.45 ms/step; an L2 prefetch measured the same.)
__device__ __forceinline__ void prefetch_state(const SweepParams& p, int v, int lane, bool active) {
    if (active && lane == 0) {
        asm volatile("prefetch.global.L1 [%0];" ::"l"(p.y + v));
        asm volatile("prefetch.global.L1 [%0];" ::"l"(p.pp + v));
    }
}

// One colour of one Gauss-Seidel sweep per launch (VBDsolver::solve, VBD.cpp:114-158).  Element
// data never changes during a sweep, so records are fetched before the dependency wait; positions
// are read only after it.
//   PREFETCH 0: records are loaded where they are used
//   PREFETCH 1: the lane's first record before the wait, then one record ahead
//   PREFETCH k >= 2: the lane's first k records before the wait, any further ones where used, so a
//            lane with at most k records pays no DRAM round trip after the wait; same summation
//            order, so the same bits as PREFETCH 1.  (Keeping k records in flight past the first k,
//            as a ring, took 70-80 registers and ran slower.)
//   CACHE:   records loaded with an L2 policy: evict-last for incidences below p.persist_end, else
//            evict-first (the factored layouts; the others ignore it).  Same bits either way.
template <int LANES, int LAYOUT, int PREFETCH, bool CACHE = false>
__device__ __forceinline__ void sweep_body(const SweepParams& p) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = LANES == 1 ? 0 : (threadIdx.x & (LANES - 1));
    const int v = p.v_begin + t / LANES;
    const bool active = v < p.v_end;
    int j0 = 0, j1 = 0;
    if (active) {
        j0 = __ldg(p.inc_off + v);
        j1 = __ldg(p.inc_off + v + 1);
    }
    const int j = j0 + lane;
    const unsigned long long pol = CACHE ? record_policy(j0 < p.persist_end) : 0ull;
    if constexpr (PREFETCH >= 2) {
        typename Elem<LAYOUT>::Rec buf[PREFETCH];
#pragma unroll
        for (int k = 0; k < PREFETCH; ++k)
            if (j + k * LANES < j1) buf[k] = fetch_rec<LAYOUT, CACHE>(p, j + k * LANES, pol);
        if (p.l2_bytes && threadIdx.x == 0) l2_prefetch_share(p.l2_next, p.l2_bytes);
        pdl_trigger();
        pdl_wait();
        prefetch_state(p, v, lane, active);
        const float4 xi = active ? p.x[v] : make_float4(0.f, 0.f, 0.f, 0.f);
        Acc acc;
        acc.zero();
#pragma unroll
        for (int k = 0; k < PREFETCH; ++k)
            if (j + k * LANES < j1) Elem<LAYOUT>::template contrib<false>(buf[k], v, xi, p.x, acc);
        for (int jj = j + PREFETCH * LANES; jj < j1; jj += LANES)
            Elem<LAYOUT>::template contrib<false>(fetch_rec<LAYOUT, CACHE>(p, jj, pol), v, xi, p.x, acc);
        vertex_solve<LANES>(p, v, lane, active, xi, acc);
    } else {
        typename Elem<LAYOUT>::Rec nxt;
        if (PREFETCH && j < j1) nxt = fetch_rec<LAYOUT, CACHE>(p, j, pol);
        if (p.l2_bytes && threadIdx.x == 0) l2_prefetch_share(p.l2_next, p.l2_bytes);
        pdl_trigger();
        pdl_wait();
        prefetch_state(p, v, lane, active);
        vertex_update<LANES, LAYOUT, PREFETCH != 0, false, CACHE>(p, v, lane, active, j, j1, nxt, pol);
    }
}

template <int LANES, int LAYOUT, int PREFETCH, bool CACHE = false>
__global__ void __launch_bounds__(256) k_sweep(SweepParams p) {
    sweep_body<LANES, LAYOUT, PREFETCH, CACHE>(p);
}

// The factored layouts with one record ahead, held to 56 registers: they fit without spilling (62-63
// uncapped), which raises occupancy from 16 to 18 blocks of 64 threads per SM.  Same body, same
// bits.  Measured on one box: 7.10 against 7.48 ms per step on the 512-mesh batch, 4.48 against 4.58
// ms on the 64^3 cube.  The deep prefetch spills at 56 and runs slower, so it keeps k_sweep.
template <int LANES, int LAYOUT, int PREFETCH = 1, bool CACHE = false>
__global__ void __maxnreg__(56) k_sweep_capped(SweepParams p) {
    sweep_body<LANES, LAYOUT, PREFETCH, CACHE>(p);
}

// ---- VBD_GPU_Solver semantics (the reference's GPU wrapper) ------------------------------------
//
// The element and vertex update of vbd_solve_color_kernel (VBD_GPU_Wrapper.cu:114-235) with
// computeTetContributionLocalCorotated (VBD_DeviceMath.cuh:127-198), in that code's arithmetic:
//   F = Ds Dm^-1 (Ds columns x_k - x_0), R by 5 Higham steps R <- (R + cof(R)/det R)/2 that stop
//   when |det R| < 1e-8, tr = R:F - 3, P = 2 mu (F - R) + lambda tr R, g = V P q_n,
//   H = V (2 mu |q_n|^2 I + lambda (R q_n)(R q_n)^T);
// 16 lanes per vertex, lane t summing tets t, t + 16, ... (H += H_e, f -= g_e), then the 16
// partial sums added in lane order onto H = m/h^2 * 1.000001 I, f = m/h^2 (y - x), and the 3x3
// solve of solve3x3 (VBD_DeviceMath.cuh:47-64: row-0 determinant, skip when |det| < 1e-8).
// The Chebyshev blend is the reference's post-sweep kernel (VBD_GPU_Wrapper.cu:8-20) folded into
// the sweep exactly as for the default semantics.

__device__ __forceinline__ float det3_row0(const float A[3][3]) {
    return A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
           A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
}

__device__ __forceinline__ void cofactor3(const float F[3][3], float C[3][3]) {
    C[0][0] = F[1][1] * F[2][2] - F[1][2] * F[2][1];
    C[0][1] = F[1][2] * F[2][0] - F[1][0] * F[2][2];
    C[0][2] = F[1][0] * F[2][1] - F[1][1] * F[2][0];
    C[1][0] = F[2][1] * F[0][2] - F[2][2] * F[0][1];
    C[1][1] = F[2][2] * F[0][0] - F[2][0] * F[0][2];
    C[1][2] = F[2][0] * F[0][1] - F[2][1] * F[0][0];
    C[2][0] = F[0][1] * F[1][2] - F[0][2] * F[1][1];
    C[2][1] = F[0][2] * F[1][0] - F[0][0] * F[1][2];
    C[2][2] = F[0][0] * F[1][1] - F[0][1] * F[1][0];
}

// Corotated block of tet r at vertex v (internal id); false when v is not one of its vertices.
__device__ __forceinline__ bool corot_block(const TetRec& r, int v, float4 xi, const float4* __restrict__ X,
                                            float H[9], float g[3]) {
    const int ids[4] = {r.ids.x, r.ids.y, r.ids.z, r.ids.w};
    const int n = (ids[0] == v) ? 0 : (ids[1] == v) ? 1 : (ids[2] == v) ? 2 : (ids[3] == v) ? 3 : -1;
    if (n < 0) return false;
    float4 pos[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) pos[k] = (ids[k] == v) ? xi : X[ids[k]];
    const float Di[3][3] = {{r.a.x, r.a.y, r.a.z}, {r.a.w, r.b.x, r.b.y}, {r.b.z, r.b.w, r.c.x}};
    const float Ds[3][3] = {{pos[1].x - pos[0].x, pos[2].x - pos[0].x, pos[3].x - pos[0].x},
                            {pos[1].y - pos[0].y, pos[2].y - pos[0].y, pos[3].y - pos[0].y},
                            {pos[1].z - pos[0].z, pos[2].z - pos[0].z, pos[3].z - pos[0].z}};
    float F[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) F[a][b] = Ds[a][0] * Di[0][b] + Ds[a][1] * Di[1][b] + Ds[a][2] * Di[2][b];
    float R[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) R[a][b] = F[a][b];
    for (int it = 0; it < 5; ++it) {
        const float det = det3_row0(R);
        if (fabsf(det) < 1e-8f) break;
        float C[3][3];
        cofactor3(R, C);
        const float inv = 1.0f / det;
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b) R[a][b] = 0.5f * (R[a][b] + C[a][b] * inv);
    }
    float tr = 0.0f;
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) tr += R[a][b] * F[a][b];
    tr -= 3.0f;
    const float mu = r.c.z, lam = r.c.w, vol = r.c.y;
    float P[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) P[a][b] = 2.0f * mu * (F[a][b] - R[a][b]) + lam * tr * R[a][b];
    float q[3];
    if (n == 0) {
        q[0] = -Di[0][0] - Di[1][0] - Di[2][0];
        q[1] = -Di[0][1] - Di[1][1] - Di[2][1];
        q[2] = -Di[0][2] - Di[1][2] - Di[2][2];
    } else {
        q[0] = Di[n - 1][0];
        q[1] = Di[n - 1][1];
        q[2] = Di[n - 1][2];
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) g[a] = vol * (P[a][0] * q[0] + P[a][1] * q[1] + P[a][2] * q[2]);
    const float qsq = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
    float RQ[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) RQ[a] = R[a][0] * q[0] + R[a][1] * q[1] + R[a][2] * q[2];
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int b = 0; b < 3; ++b) H[3 * a + b] = vol * ((a == b ? 2.0f * mu * qsq : 0.0f) + lam * RQ[a] * RQ[b]);
    return true;
}

constexpr int kWrapperLanes = 16;

// Tet records are read through the per-vertex tet list whatever the layout option, as the
// reference's kernel reads them; this one code path is the one checked bit for bit against it.
// Records are loaded where they are used (no prefetch) and the kernel is held to 64 registers (4
// blocks of 256 per SM, a few bytes of spill): 15.2 ms for a 50-iteration solve on the 64^3 cube
// with the shuffle reduction of that time (13.8 ms now), against 20.4 ms with prefetch at 99
// registers and 16.5 ms at 79.  Tighter caps spill heavily,
// run slower, and change ptxas's fused multiply-add choices (no longer bit-identical).
constexpr int kWrapperBlock = 256;

// Its parameter block is its own (the fields it reads, in SweepParams's order): the kernel's
// compiled arithmetic was checked bit for bit with this block, and a different block layout has
// been seen to change nvcc's fused multiply-add choices in it.
struct WrapperParams {
    float4* x;
    float4* xnext;
    float4* pp;
    const float4* y;
    const int* inc_off;
    const int* inc_tet;
    const TetRec* rec;
    const TetRec* irec;
    const int4* crec;
    const float2* cmat;
    unsigned long long* status;
    int v_begin, v_end;
    float dtsr;
    float omega;
    int accel;
    int keep_pp;
    const float* cam;
};

__global__ void __launch_bounds__(kWrapperBlock, 4) k_sweep_wrapper(WrapperParams p) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & (kWrapperLanes - 1);
    const int v = p.v_begin + t / kWrapperLanes;
    const bool active = v < p.v_end;
    int j0 = 0, j1 = 0;
    if (active) {
        j0 = __ldg(p.inc_off + v);
        j1 = __ldg(p.inc_off + v + 1);
    }
    int j = j0 + lane;
    pdl_trigger();
    pdl_wait();
    const float4 xi = active ? p.x[v] : make_float4(0.f, 0.f, 0.f, 0.f);
    float hs[9], fs[3];
#pragma unroll
    for (int k = 0; k < 9; ++k) hs[k] = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; ++k) fs[k] = 0.0f;
    for (; j < j1; j += kWrapperLanes) {
        const TetRec r = load_rec(p.rec + __ldg(p.inc_tet + j));
        float H[9], g[3];
        if (corot_block(r, v, xi, p.x, H, g)) {
#pragma unroll
            for (int k = 0; k < 9; ++k) hs[k] += H[k];
#pragma unroll
            for (int k = 0; k < 3; ++k) fs[k] -= g[k];
        }
    }
    // partial sums added in lane order by the group's first lane
    float Hf[9], ff[3];
    if (lane == 0 && active) {
        const float4 yi = p.y[v];
        const float coeff = yi.w * p.dtsr;
        const float reg = coeff * 1.000001f;
#pragma unroll
        for (int k = 0; k < 9; ++k) Hf[k] = (k % 4 == 0) ? reg : 0.0f;
        ff[0] = coeff * (yi.x - xi.x);
        ff[1] = coeff * (yi.y - xi.y);
        ff[2] = coeff * (yi.z - xi.z);
    }
    // The 16 lanes' partial sums reach the first lane through shared memory (12 floats per thread,
    // 12 KB per block) rather than 192 warp shuffles per pair of vertices; the additions and their
    // order are unchanged.  Measured on the 64^3 cube: 13.8 against 15.2 ms per solve, still
    // bit-identical to the reference's kernels.  (Spreading the additions over four lanes was
    // faster still, 13.4 ms, but changed results in the last bit.)
    __shared__ float red[kWrapperBlock * 12];
    {
        float* mine = red + 12 * threadIdx.x;
#pragma unroll
        for (int k = 0; k < 9; ++k) mine[k] = hs[k];
#pragma unroll
        for (int k = 0; k < 3; ++k) mine[9 + k] = fs[k];
    }
    __syncwarp();
    if (lane == 0 && active) {
        const float* grp = red + 12 * threadIdx.x;
        for (int src = 0; src < kWrapperLanes; ++src) {
#pragma unroll
            for (int k = 0; k < 9; ++k) Hf[k] += grp[12 * src + k];
#pragma unroll
            for (int k = 0; k < 3; ++k) ff[k] += grp[12 * src + 9 + k];
        }
    }
    if (!active || lane != 0) return;
    const float A[3][3] = {{Hf[0], Hf[1], Hf[2]}, {Hf[3], Hf[4], Hf[5]}, {Hf[6], Hf[7], Hf[8]}};
    const float det = det3_row0(A);
    float4 xn = xi;
    if (fabsf(det) < 1.0e-8f) {
        atomicAdd(p.status + ST_SINGULAR, 1ull);
    } else {
        float adj[3][3];
        cofactor3(A, adj);
        const float inv = 1.0f / det;
        xn.x = xi.x + inv * (adj[0][0] * ff[0] + adj[1][0] * ff[1] + adj[2][0] * ff[2]);
        xn.y = xi.y + inv * (adj[0][1] * ff[0] + adj[1][1] * ff[1] + adj[2][1] * ff[2]);
        xn.z = xi.z + inv * (adj[0][2] * ff[0] + adj[1][2] * ff[1] + adj[2][2] * ff[2]);
    }
    if (!(isfinite(xn.x) && isfinite(xn.y) && isfinite(xn.z))) p.status[ST_NONFINITE] = 1ull;
    p.x[v] = xn;
    if (p.accel) {
        const float4 q = p.pp[v];
        float4 xa;
        xa.x = p.omega * (xn.x - q.x) + q.x;
        xa.y = p.omega * (xn.y - q.y) + q.y;
        xa.z = p.omega * (xn.z - q.z) + q.z;
        xa.w = xn.w;
        p.xnext[v] = xa;
    }
    if (p.keep_pp) p.pp[v] = xi;
}

// ---- persistent colour-walking kernel -------------------------------------------------------

struct GridBarrier {
    unsigned int count;
    unsigned int gen;
};

struct PersistParams {
    SweepParams sw;           // dtsr, y, element data, status; x / xnext / accel / omega set per sweep
    float4* xa;               // position buffers (positions start and end in xa)
    float4* xb;
    float4* v;
    float4* xprev;
    const int* cstart;        // colour c = internal ids [cstart[c], cstart[c+1])
    const float* omega;       // Chebyshev weight of each iteration (1 = no blend)
    GridBarrier* bar;
    long long spin_limit;     // polls of the barrier flag before giving up
    int ncol, iters, nfree, n;
    int predict;              // run the inertial predictor first
    int finish;               // run the velocity update last
    int init_from_inertia;    // start from x = y
    int expected_blocks;      // arrivals the barrier waits for (gridDim.x in normal use)
    float h, hgx, hgy, hgz;
    // the cluster walk with resident element data: per CTA at most srec_records records and
    // srec_owned vertices, srec_slices (colour, round) slices
    int srec_records, srec_owned, srec_slices;
};

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid-wide barrier of a cooperative launch with a bounded wait: after spin_limit polls the
// waiting block records ST_TIMEOUT and the call returns false (the caller then exits), so a
// barrier that can never complete ends the kernel instead of hanging it.
__device__ __forceinline__ bool grid_barrier(GridBarrier* bar, int expected, long long spin_limit,
                                             unsigned long long* status) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned gen = ld_acquire_gpu(&bar->gen);
        __threadfence();
        const unsigned arrived = atomicAdd(&bar->count, 1u);
        if (arrived == (unsigned)expected - 1u) {
            bar->count = 0u;
            __threadfence();
            st_release_gpu(&bar->gen, gen + 1u);
        } else {
            long long polls = 0;
            while (ld_acquire_gpu(&bar->gen) == gen) {
                if (++polls > spin_limit) {
                    ok = 0;
                    atomicOr(reinterpret_cast<unsigned int*>(status + ST_TIMEOUT), 1u);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Whole step (or solve) in one cooperative launch: predictor, `iters` sweeps over the colours
// with a grid barrier after each colour, velocity update.  Same arithmetic as k_predict /
// k_sweep / k_finish, so results are bit-identical to the multi-launch path.
template <int LANES, int LAYOUT>
__global__ void __launch_bounds__(256, 4) k_persistent(PersistParams p) {
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nthreads = gridDim.x * blockDim.x;
    if (p.predict) {
        for (int i = gtid; i < p.n; i += nthreads) {
            const float4 xi = p.xa[i];
            p.xprev[i] = xi;
            float4 yi = p.sw.y[i];
            if (i < p.nfree) {
                float4 vi = p.v[i];
                vi.x += p.hgx;
                vi.y += p.hgy;
                vi.z += p.hgz;
                p.v[i] = vi;
                yi.x = __fadd_rn(xi.x, __fmul_rn(p.h, vi.x));
                yi.y = __fadd_rn(xi.y, __fmul_rn(p.h, vi.y));
                yi.z = __fadd_rn(xi.z, __fmul_rn(p.h, vi.z));
            } else {
                yi.x = xi.x;
                yi.y = xi.y;
                yi.z = xi.z;
            }
            const_cast<float4*>(p.sw.y)[i] = yi;
        }
    }
    if (p.init_from_inertia) {
        for (int i = gtid; i < p.n; i += nthreads) {
            const float4 yi = p.sw.y[i];
            float4 a = p.xa[i], b = p.xb[i];
            a.x = b.x = yi.x;
            a.y = b.y = yi.y;
            a.z = b.z = yi.z;
            p.xa[i] = a;
            p.xb[i] = b;
        }
    }
    if (!grid_barrier(p.bar, p.expected_blocks, p.spin_limit, p.sw.status)) return;

    const int lane_w = threadIdx.x & 31;
    const int lane = LANES == 1 ? 0 : (lane_w & (LANES - 1));
    const int groups_per_warp = 32 / LANES;
    const int warp = gtid >> 5;
    const int nwarps = nthreads >> 5;
    int cur = 0;
    SweepParams sp = p.sw;
    for (int k = 0; k < p.iters; ++k) {
        const float om = p.omega[k];
        const bool blend = om > 1.0f;
        sp.x = cur ? p.xb : p.xa;
        sp.xnext = cur ? p.xa : p.xb;
        sp.omega = om;
        sp.accel = blend ? 1 : 0;
        for (int c = 0; c < p.ncol; ++c) {
            const int vb = p.cstart[c], ve = p.cstart[c + 1];
            for (int base = vb + warp * groups_per_warp; base < ve; base += nwarps * groups_per_warp) {
                const int v = base + lane_w / LANES;
                const bool active = v < ve;
                int j0 = 0, j1 = 0;
                if (active) {
                    j0 = __ldg(sp.inc_off + v);
                    j1 = __ldg(sp.inc_off + v + 1);
                }
                const int j = j0 + lane;
                typename Elem<LAYOUT>::Rec nxt;
                if (j < j1) nxt = Elem<LAYOUT>::fetch(sp, j);
                vertex_update<LANES, LAYOUT, true, true>(sp, v, lane, active, j, j1, nxt);
            }
            if (!grid_barrier(p.bar, p.expected_blocks, p.spin_limit, p.sw.status)) return;
        }
        if (blend) cur ^= 1;
    }
    for (int i = gtid; i < p.nfree; i += nthreads) {
        const float4 xf = cur ? p.xb[i] : p.xa[i];
        if (cur) p.xa[i] = xf;
        if (p.finish) {
            const float4 xp = p.xprev[i];
            float4 vi = p.v[i];
            vi.x = ((xf.x - xp.x) / p.h) * 0.999f;
            vi.y = ((xf.y - xp.y) / p.h) * 0.999f;
            vi.z = ((xf.z - xp.z) / p.h) * 0.999f;
            p.v[i] = vi;
        }
    }
}

// Inertial predictor (VBDsolver::forwardStep, VBD.cpp:103-112; TetMesh::applyGravity /
// computeInertia / savePreviousPosition, TetMesh.h:319-348).  Free vertices are [0, nfree).
// y = x + h v is rounded after the product and after the sum (no fused multiply-add), as the
// reference's host code computes it.
__device__ __forceinline__ void predict_vertex(int i, const float4* __restrict__ x, float4* __restrict__ v,
                                               float4* __restrict__ xprev, float4* __restrict__ y, int nfree, float h,
                                               float hgx, float hgy, float hgz) {
    const float4 xi = x[i];
    xprev[i] = xi;
    float4 yi = y[i];
    if (i < nfree) {
        float4 vi = v[i];
        vi.x += hgx;
        vi.y += hgy;
        vi.z += hgz;
        v[i] = vi;
        yi.x = __fadd_rn(xi.x, __fmul_rn(h, vi.x));
        yi.y = __fadd_rn(xi.y, __fmul_rn(h, vi.y));
        yi.z = __fadd_rn(xi.z, __fmul_rn(h, vi.z));
    } else {
        yi.x = xi.x;
        yi.y = xi.y;
        yi.z = xi.z;
    }
    y[i] = yi;
}

__global__ void k_predict(const float4* __restrict__ x, float4* __restrict__ v, float4* __restrict__ xprev,
                          float4* __restrict__ y, int nfree, int n, float h, float hgx, float hgy, float hgz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) predict_vertex(i, x, v, xprev, y, nfree, h, hgx, hgy, hgz);
}

// Velocity update v = (x - x_prev)/h * 0.999 (TetMesh::updateVelocity, TetMesh.h:305-311) and,
// when the final positions sit in the second buffer, their copy back into the first.
__device__ __forceinline__ float4 damped_velocity(float4 xi, float4 xp, float4 vi, float h) {
    vi.x = ((xi.x - xp.x) / h) * 0.999f;
    vi.y = ((xi.y - xp.y) / h) * 0.999f;
    vi.z = ((xi.z - xp.z) / h) * 0.999f;
    return vi;
}

__global__ void k_finish(const float4* __restrict__ xf, float4* __restrict__ x0, const float4* __restrict__ xprev,
                         float4* __restrict__ v, int nfree, float h, int copy_back, int update_v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nfree) return;
    const float4 xi = xf[i];
    if (copy_back) x0[i] = xi;
    if (update_v) v[i] = damped_velocity(xi, xprev[i], v[i], h);
}

// dst.xyz = src.xyz over [0, n), keeping dst.w (x = y start, VBD_GPU_Wrapper.cu:334).
__global__ void k_copy_xyz(const float4* __restrict__ src, float4* __restrict__ d0, float4* __restrict__ d1, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 s = src[i];
    float4 a = d0[i];
    a.x = s.x; a.y = s.y; a.z = s.z;
    d0[i] = a;
    if (d1) {
        float4 b = d1[i];
        b.x = s.x; b.y = s.y; b.z = s.z;
        d1[i] = b;
    }
}

// Caller-order float[3N] <-> internal float4 (perm[i] = caller id of internal vertex i).
__global__ void k_scatter3(const float* __restrict__ stage, const int* __restrict__ perm, float4* d0, float4* d1,
                           int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int o = perm[i];
    const float sx = stage[3 * o], sy = stage[3 * o + 1], sz = stage[3 * o + 2];
    float4 a = d0[i];
    a.x = sx; a.y = sy; a.z = sz;
    d0[i] = a;
    if (d1) {
        float4 b = d1[i];
        b.x = sx; b.y = sy; b.z = sz;
        d1[i] = b;
    }
}

__global__ void k_gather3(const float4* __restrict__ src, const int* __restrict__ perm, float* __restrict__ stage,
                          int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int o = perm[i];
    const float4 s = src[i];
    stage[3 * o] = s.x;
    stage[3 * o + 1] = s.y;
    stage[3 * o + 2] = s.z;
}

// rec[t].c.zw = (mu, lambda); either array may be null.
__global__ void k_set_materials(TetRec* rec, const float* __restrict__ mu, const float* __restrict__ lam, float mu0,
                                float lam0, int ntet) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntet) return;
    float4 c = rec[t].c;
    c.z = mu ? mu[t] : (mu0 >= 0.f ? mu0 : c.z);
    c.w = lam ? lam[t] : (lam0 >= 0.f ? lam0 : c.w);
    rec[t].c = c;
}

// irec[j] = rec[inc_tet[j]]: the incidence-ordered copy.
__global__ void k_pack_stream(const TetRec* __restrict__ rec, const int* __restrict__ inc_tet, TetRec* __restrict__ irec,
                              int ninc) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ninc) return;
    irec[j] = rec[inc_tet[j]];
}

// Compact incidence records from the tet records (layout 2): for incidence j of vertex v (internal
// id, inc_vertex[j]) in tet inc_tet[j], the other three vertices in local order with their rows
// of Q = Ps Dm^-1, the vertex's local index, and (V0 mu, V0 lambda).
__global__ void k_pack_compact(const TetRec* __restrict__ rec, const int* __restrict__ inc_tet,
                               const int* __restrict__ inc_vertex, int4* __restrict__ crec, float2* __restrict__ cmat,
                               int ninc) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ninc) return;
    const TetRec r = rec[inc_tet[j]];
    const int v = inc_vertex[j];
    const int ids[4] = {r.ids.x, r.ids.y, r.ids.z, r.ids.w};
    const float D[3][3] = {{r.a.x, r.a.y, r.a.z}, {r.a.w, r.b.x, r.b.y}, {r.b.z, r.b.w, r.c.x}};
    float Q[4][3];
    for (int c = 0; c < 3; ++c) {
        Q[0][c] = -D[0][c] - D[1][c] - D[2][c];
        for (int k = 1; k < 4; ++k) Q[k][c] = D[k - 1][c];
    }
    int n = 3;
    for (int k = 0; k < 4; ++k)
        if (ids[k] == v) {
            n = k;
            break;
        }
    int nb[3];
    float q[9];
    int m = 0;
    for (int k = 0; k < 4; ++k) {
        if (k == n) continue;
        nb[m] = ids[k];
        for (int c = 0; c < 3; ++c) q[3 * m + c] = Q[k][c];
        ++m;
    }
    crec[3 * j] = make_int4(nb[0] | (n << 30), nb[1], nb[2], __float_as_int(q[0]));
    crec[3 * j + 1] = make_int4(__float_as_int(q[1]), __float_as_int(q[2]), __float_as_int(q[3]), __float_as_int(q[4]));
    crec[3 * j + 2] = make_int4(__float_as_int(q[5]), __float_as_int(q[6]), __float_as_int(q[7]), __float_as_int(q[8]));
    cmat[j] = make_float2(r.c.y * r.c.z, r.c.y * r.c.w);
}

// Factored records from the tet records: M's rows in the compact record's order, then
// s = M q_n, w = cof(M) q_n, det M and the material products.  PACKED writes layout 4 (ids in
// 21 bits each, no det M, materials into cmat), otherwise layout 3.
template <bool PACKED>
__global__ void k_pack_factored(const TetRec* __restrict__ rec, const int* __restrict__ inc_tet,
                                const int* __restrict__ inc_vertex, int4* __restrict__ crec,
                                float2* __restrict__ cmat, int ninc) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ninc) return;
    const TetRec r = rec[inc_tet[j]];
    const int v = inc_vertex[j];
    const int ids[4] = {r.ids.x, r.ids.y, r.ids.z, r.ids.w};
    const float D[3][3] = {{r.a.x, r.a.y, r.a.z}, {r.a.w, r.b.x, r.b.y}, {r.b.z, r.b.w, r.c.x}};
    float Q[4][3];
    for (int c = 0; c < 3; ++c) {
        Q[0][c] = -D[0][c] - D[1][c] - D[2][c];
        for (int k = 1; k < 4; ++k) Q[k][c] = D[k - 1][c];
    }
    int n = 3;
    for (int k = 0; k < 4; ++k)
        if (ids[k] == v) {
            n = k;
            break;
        }
    int nb[3];
    float M[3][3];
    int m = 0;
    for (int k = 0; k < 4; ++k) {
        if (k == n) continue;
        nb[m] = ids[k];
        for (int c = 0; c < 3; ++c) M[m][c] = Q[k][c];
        ++m;
    }
    const float q[3] = {-(M[0][0] + M[1][0] + M[2][0]), -(M[0][1] + M[1][1] + M[2][1]), -(M[0][2] + M[1][2] + M[2][2])};
    float cof[3][3];
    cof[0][0] = M[1][1] * M[2][2] - M[1][2] * M[2][1];
    cof[0][1] = M[1][2] * M[2][0] - M[1][0] * M[2][2];
    cof[0][2] = M[1][0] * M[2][1] - M[1][1] * M[2][0];
    cof[1][0] = M[2][1] * M[0][2] - M[2][2] * M[0][1];
    cof[1][1] = M[2][2] * M[0][0] - M[2][0] * M[0][2];
    cof[1][2] = M[2][0] * M[0][1] - M[2][1] * M[0][0];
    cof[2][0] = M[0][1] * M[1][2] - M[0][2] * M[1][1];
    cof[2][1] = M[0][2] * M[1][0] - M[0][0] * M[1][2];
    cof[2][2] = M[0][0] * M[1][1] - M[0][1] * M[1][0];
    float sv[3], wv[3];
    for (int i = 0; i < 3; ++i) {
        sv[i] = M[i][0] * q[0] + M[i][1] * q[1] + M[i][2] * q[2];
        wv[i] = cof[i][0] * q[0] + cof[i][1] * q[1] + cof[i][2] * q[2];
    }
    const float detm = M[0][0] * cof[0][0] + M[0][1] * cof[0][1] + M[0][2] * cof[0][2];
    const float a = r.c.y * r.c.z, b = r.c.y * r.c.w;
    if (PACKED) {
        const unsigned lo = (unsigned)nb[0] | ((unsigned)nb[1] << kPackedIdBits);
        const unsigned hi = ((unsigned)nb[1] >> (32 - kPackedIdBits)) | ((unsigned)nb[2] << (2 * kPackedIdBits - 32));
        crec[2 * j] = make_int4((int)lo, (int)hi, __float_as_int(sv[0]), __float_as_int(sv[1]));
        crec[2 * j + 1] = make_int4(__float_as_int(sv[2]), __float_as_int(wv[0]), __float_as_int(wv[1]), __float_as_int(wv[2]));
        cmat[j] = make_float2(a, b);
        return;
    }
    crec[3 * j] = make_int4(nb[0] | (n << 30), nb[1], nb[2], __float_as_int(sv[0]));
    crec[3 * j + 1] = make_int4(__float_as_int(sv[1]), __float_as_int(sv[2]), __float_as_int(wv[0]), __float_as_int(wv[1]));
    crec[3 * j + 2] = make_int4(__float_as_int(wv[2]), __float_as_int(detm), __float_as_int(a), __float_as_int(b));
}

// ---- implicit adjoint of a converged step --------------------------------------------------
//
// A step's positions x' solve M/h^2 (x' - y) + dPsi/dx(x') = 0 on free vertices.  Its adjoint
// solves (M/h^2 + H(x')) lam = G by the same coloured block Gauss-Seidel as the forward: vertex i
// sets lam_i = A_ii^-1 (G_i - sum_{j != i} A_ij lam_j), where the off-diagonal sum is applied per
// tet as V dP(dF') q_i with dF' = sum_{k != i} lam_k q_k^T, dP = dP/dF[dF'] = mu (dF' - dC) +
// lambda (C : dF') C + lambda (J - 1) dC, dC the directional derivative of cof F; A_ii is the
// forward's exact diagonal block m/h^2 I + sum V (mu |q|^2 I + lambda (C q)(C q)^T).

// The element seen from vertex v: the other three vertices, their rows q_k of Q = Ps Dm^-1, the
// vertex's own row q_n, and (V mu, V lambda).
struct ElemView {
    int nb[3];
    float q[3][3];
    float qn[3];
    float a, b;
};

__device__ __forceinline__ ElemView view_of(const TetRec& r, int v) {
    const int ids[4] = {r.ids.x, r.ids.y, r.ids.z, r.ids.w};
    const float D[3][3] = {{r.a.x, r.a.y, r.a.z}, {r.a.w, r.b.x, r.b.y}, {r.b.z, r.b.w, r.c.x}};
    const int n = (ids[0] == v) ? 0 : (ids[1] == v) ? 1 : (ids[2] == v) ? 2 : 3;
    ElemView e;
    float Q[4][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        Q[0][c] = -D[0][c] - D[1][c] - D[2][c];
        Q[1][c] = D[0][c];
        Q[2][c] = D[1][c];
        Q[3][c] = D[2][c];
    }
    int m = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (k == n) {
#pragma unroll
            for (int c = 0; c < 3; ++c) e.qn[c] = Q[k][c];
        } else {
            e.nb[m] = ids[k];
#pragma unroll
            for (int c = 0; c < 3; ++c) e.q[m][c] = Q[k][c];
            ++m;
        }
    }
    e.a = r.c.y * r.c.z;
    e.b = r.c.y * r.c.w;
    return e;
}

__device__ __forceinline__ ElemView view_of(const CompactRec& r, int) {
    ElemView e;
    e.nb[0] = r.nb0;
    e.nb[1] = r.nb1;
    e.nb[2] = r.nb2;
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int c = 0; c < 3; ++c) e.q[k][c] = r.q[3 * k + c];
#pragma unroll
    for (int c = 0; c < 3; ++c) e.qn[c] = -(r.q[c] + r.q[3 + c] + r.q[6 + c]);
    e.a = r.a;
    e.b = r.b;
    return e;
}

__device__ __forceinline__ void cof3(const float F[3][3], float C[3][3]) {
    C[0][0] = F[1][1] * F[2][2] - F[1][2] * F[2][1];
    C[0][1] = F[1][2] * F[2][0] - F[1][0] * F[2][2];
    C[0][2] = F[1][0] * F[2][1] - F[1][1] * F[2][0];
    C[1][0] = F[2][1] * F[0][2] - F[2][2] * F[0][1];
    C[1][1] = F[2][2] * F[0][0] - F[2][0] * F[0][2];
    C[1][2] = F[2][0] * F[0][1] - F[2][1] * F[0][0];
    C[2][0] = F[0][1] * F[1][2] - F[0][2] * F[1][1];
    C[2][1] = F[0][2] * F[1][0] - F[0][0] * F[1][2];
    C[2][2] = F[0][0] * F[1][1] - F[0][1] * F[1][0];
}

// Directional derivative of the cofactor matrix: d/dt cof(F + t D) at t = 0.
__device__ __forceinline__ void dcof3(const float F[3][3], const float D[3][3], float dC[3][3]) {
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            dC[i][j] = D[i1][j1] * F[i2][j2] + F[i1][j1] * D[i2][j2] - D[i1][j2] * F[i2][j1] - F[i1][j2] * D[i2][j1];
        }
}

// F, C, J of the element at positions X, seen from vertex v at xi.
__device__ __forceinline__ void elem_F(const ElemView& e, float4 xi, const float4* __restrict__ X, float F[3][3],
                                       float C[3][3], float& J) {
    float d[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float4 p = X[e.nb[k]];
        d[k][0] = p.x - xi.x;
        d[k][1] = p.y - xi.y;
        d[k][2] = p.z - xi.z;
    }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) F[r][c] = d[0][r] * e.q[0][c] + d[1][r] * e.q[1][c] + d[2][r] * e.q[2][c];
    cof3(F, C);
    J = F[0][0] * C[0][0] + F[0][1] * C[0][1] + F[0][2] * C[0][2];
}

// Off-diagonal product of the element at vertex v: V dP(sum_{k != v} lam_k q_k^T) q_v.
__device__ __forceinline__ void elem_offdiag(const ElemView& e, const float F[3][3], const float C[3][3], float J,
                                             const float4* __restrict__ L, float out[3]) {
    float dF[3][3];
    float l[3][3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float4 p = L[e.nb[k]];
        l[k][0] = p.x;
        l[k][1] = p.y;
        l[k][2] = p.z;
    }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) dF[r][c] = l[0][r] * e.q[0][c] + l[1][r] * e.q[1][c] + l[2][r] * e.q[2][c];
    float dC[3][3];
    dcof3(F, dF, dC);
    float dJ = 0.f;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) dJ += C[r][c] * dF[r][c];
    const float jm1 = J - 1.0f;
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        float acc = 0.f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float dP = e.a * (dF[r][c] - dC[r][c]) + e.b * (dJ * C[r][c] + jm1 * dC[r][c]);
            acc += dP * e.qn[c];
        }
        out[r] = acc;
    }
}

struct AdjParams {
    const float4* X;          // converged positions of the step
    float4* lam;              // adjoint, updated in place (pinned entries stay 0)
    const float4* G;          // right-hand side
    const float4* y;          // w = mass
    const int* inc_off;
    const int* inc_tet;
    const TetRec* rec;
    const int4* crec;         // compact incidence records (when the forward uses them)
    const float2* cmat;
    float dtsr;
    int v_begin, v_end;
    float4* lam_next;         // Chebyshev: receives omega (lam~ - lam_pp) + lam_pp
    float4* lam_pp;           // Chebyshev: adjoint before the previous sweep
    float omega;
    int accel;                // write lam_next
    int keep_pp;              // store the pre-sweep adjoint into lam_pp
};

template <int LAYOUT> struct AdjElem;
template <> struct AdjElem<0> {
    using Rec = TetRec;
    __device__ __forceinline__ static Rec fetch(const AdjParams& p, int j) { return load_rec(p.rec + __ldg(p.inc_tet + j)); }
};
template <> struct AdjElem<2> {
    using Rec = CompactRec;
    __device__ __forceinline__ static Rec fetch(const AdjParams& p, int j) { return load_compact(p.crec, p.cmat, j); }
};
template <> struct AdjElem<3> {
    using Rec = FactRaw3;
    __device__ __forceinline__ static Rec fetch(const AdjParams& p, int j) { return load_fact(p.crec, j); }
};
template <> struct AdjElem<4> {
    using Rec = FactRaw4;
    __device__ __forceinline__ static Rec fetch(const AdjParams& p, int j) { return load_fact_packed(p.crec, p.cmat, j); }
};

// Adjoint element terms from a factored record (F = D M, dF = L M with L = [lam_0 lam_1 lam_2]):
//   dF q_n = L s,   dC q_n = dcof(D)[L] w,   dJ = C : dF = det M sum_k c_k . lam_k
// with c_k the columns of cof(D) and dcof(D)[L] the columns lam_1 x d_2 + d_1 x lam_2 (and
// cyclic); off-diagonal product V dP(dF) q_n = a (dF q_n - dC q_n) + b (dJ C q_n + (J - 1) dC q_n),
// diagonal block am I + b (C q_n)(C q_n)^T.
__device__ __forceinline__ void fact_adjoint(const FactRec& r, float4 xi, const float4* __restrict__ X,
                                             const float4* __restrict__ L, Acc& acc) {
    const float4 p0 = X[r.nb0], p1 = X[r.nb1], p2 = X[r.nb2];
    const float4 l0 = L[r.nb0], l1 = L[r.nb1], l2 = L[r.nb2];
    const float d0[3] = {p0.x - xi.x, p0.y - xi.y, p0.z - xi.z};
    const float d1[3] = {p1.x - xi.x, p1.y - xi.y, p1.z - xi.z};
    const float d2[3] = {p2.x - xi.x, p2.y - xi.y, p2.z - xi.z};
    const float m0[3] = {l0.x, l0.y, l0.z}, m1[3] = {l1.x, l1.y, l1.z}, m2[3] = {l2.x, l2.y, l2.z};
    float c0[3], c1[3], c2[3], e0[3], e1[3], e2[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const int i1 = (i + 1) % 3, i2 = (i + 2) % 3;
        c0[i] = d1[i1] * d2[i2] - d1[i2] * d2[i1];
        c1[i] = d2[i1] * d0[i2] - d2[i2] * d0[i1];
        c2[i] = d0[i1] * d1[i2] - d0[i2] * d1[i1];
        e0[i] = (m1[i1] * d2[i2] - m1[i2] * d2[i1]) + (d1[i1] * m2[i2] - d1[i2] * m2[i1]);
        e1[i] = (m2[i1] * d0[i2] - m2[i2] * d0[i1]) + (d2[i1] * m0[i2] - d2[i2] * m0[i1]);
        e2[i] = (m0[i1] * d1[i2] - m0[i2] * d1[i1]) + (d0[i1] * m1[i2] - d0[i2] * m1[i1]);
    }
    const float J = (d0[0] * c0[0] + d0[1] * c0[1] + d0[2] * c0[2]) * r.detm;
    const float dJ = r.detm * ((c0[0] * m0[0] + c0[1] * m0[1] + c0[2] * m0[2]) +
                               (c1[0] * m1[0] + c1[1] * m1[1] + c1[2] * m1[2]) +
                               (c2[0] * m2[0] + c2[1] * m2[1] + c2[2] * m2[2]));
    const float jm1 = J - 1.0f;
    float o[3], Cq[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        Cq[i] = c0[i] * r.w0 + c1[i] * r.w1 + c2[i] * r.w2;
        const float dFq = m0[i] * r.s0 + m1[i] * r.s1 + m2[i] * r.s2;
        const float dCq = e0[i] * r.w0 + e1[i] * r.w1 + e2[i] * r.w2;
        o[i] = r.a * (dFq - dCq) + r.b * (dJ * Cq[i] + jm1 * dCq);
    }
    acc.g0 += o[0];
    acc.g1 += o[1];
    acc.g2 += o[2];
    acc.h00 += r.am + r.b * Cq[0] * Cq[0];
    acc.h01 += r.b * Cq[0] * Cq[1];
    acc.h02 += r.b * Cq[0] * Cq[2];
    acc.h11 += r.am + r.b * Cq[1] * Cq[1];
    acc.h12 += r.b * Cq[1] * Cq[2];
    acc.h22 += r.am + r.b * Cq[2] * Cq[2];
}

// The adjoint block solve of one vertex of mass m: (m/h^2 I + H_vv) lam = g - (the off-diagonal
// products summed in acc.g), with the diagonal block in acc.h; lam = 0 where |det| <= 1e-30.
__device__ __forceinline__ float4 adj_block_solve(const Acc& acc, float m, float dtsr, float4 g) {
    const float cm = m * dtsr;
    const float H00 = cm + acc.h00, H01 = acc.h01, H02 = acc.h02, H11 = cm + acc.h11, H12 = acc.h12, H22 = cm + acc.h22;
    const float f0 = g.x - acc.g0, f1 = g.y - acc.g1, f2 = g.z - acc.g2;
    const float A00 = H11 * H22 - H12 * H12, A01 = H02 * H12 - H01 * H22, A02 = H01 * H12 - H02 * H11;
    const float A11 = H00 * H22 - H02 * H02, A12 = H02 * H01 - H00 * H12, A22 = H00 * H11 - H01 * H01;
    const float det = H00 * A00 + H01 * A01 + H02 * A02;
    float4 l = make_float4(0.f, 0.f, 0.f, 0.f);
    if (fabsf(det) > 1e-30f) {
        const float inv = 1.0f / det;
        l.x = inv * (A00 * f0 + A01 * f1 + A02 * f2);
        l.y = inv * (A01 * f0 + A11 * f1 + A12 * f2);
        l.z = inv * (A02 * f0 + A12 * f1 + A22 * f2);
    }
    return l;
}

// The adjoint's Chebyshev blend omega (lam~ - lam_pp) + lam_pp.
__device__ __forceinline__ float4 adj_blend(float4 l, float4 q, float omega) {
    return make_float4(omega * (l.x - q.x) + q.x, omega * (l.y - q.y) + q.y, omega * (l.z - q.z) + q.z, 0.f);
}

// One colour of one adjoint Gauss-Seidel sweep.  LAYOUT 0 reads tet records through inc_tet,
// LAYOUT 2 the forward's compact incidence records; the lane's first record is fetched before the
// programmatic-launch dependency wait, the next one while the current is evaluated.
template <int LANES, int LAYOUT>
__global__ void __launch_bounds__(256) k_adj_sweep(AdjParams p) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & (LANES - 1);
    const int v = p.v_begin + t / LANES;
    const bool active = v < p.v_end;
    int j0 = 0, j1 = 0;
    if (active) {
        j0 = __ldg(p.inc_off + v);
        j1 = __ldg(p.inc_off + v + 1);
    }
    int j = j0 + lane;
    typename AdjElem<LAYOUT>::Rec nxt;
    if (j < j1) nxt = AdjElem<LAYOUT>::fetch(p, j);
    pdl_trigger();
    pdl_wait();
    const float4 xi = active ? p.X[v] : make_float4(0.f, 0.f, 0.f, 0.f);
    Acc acc;  // h.. = diagonal block, g. = off-diagonal product
    acc.zero();
    for (; j < j1; j += LANES) {
        const typename AdjElem<LAYOUT>::Rec r = nxt;
        if (j + LANES < j1) nxt = AdjElem<LAYOUT>::fetch(p, j + LANES);
        if constexpr (LAYOUT >= 3) {
            fact_adjoint(decode_fact(r), xi, p.X, p.lam, acc);
            continue;
        } else {
        const ElemView e = view_of(r, v);
        float F[3][3], C[3][3], J;
        elem_F(e, xi, p.X, F, C, J);
        float o[3];
        elem_offdiag(e, F, C, J, p.lam, o);
        acc.g0 += o[0];
        acc.g1 += o[1];
        acc.g2 += o[2];
        float Cq[3];
#pragma unroll
        for (int r2 = 0; r2 < 3; ++r2) Cq[r2] = C[r2][0] * e.qn[0] + C[r2][1] * e.qn[1] + C[r2][2] * e.qn[2];
        const float am = e.a * (e.qn[0] * e.qn[0] + e.qn[1] * e.qn[1] + e.qn[2] * e.qn[2]);
        acc.h00 += am + e.b * Cq[0] * Cq[0];
        acc.h01 += e.b * Cq[0] * Cq[1];
        acc.h02 += e.b * Cq[0] * Cq[2];
        acc.h11 += am + e.b * Cq[1] * Cq[1];
        acc.h12 += e.b * Cq[1] * Cq[2];
        acc.h22 += am + e.b * Cq[2] * Cq[2];
        }
    }
    group_reduce<LANES>(acc);
    if (!active || lane != 0) return;
    const float4 l = adj_block_solve(acc, p.y[v].w, p.dtsr, p.G[v]);
    const float4 lold = p.lam[v];
    p.lam[v] = l;
    if (p.accel) p.lam_next[v] = adj_blend(l, p.lam_pp[v], p.omega);
    if (p.keep_pp) p.lam_pp[v] = lold;
}

// G = x~ + c v~ on free vertices [0, nfree).
__global__ void k_adj_rhs(const float4* __restrict__ ax, const float4* __restrict__ av, float4* __restrict__ G, float c,
                          int nfree) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nfree) return;
    const float4 a = ax[i], b = av[i];
    G[i] = make_float4(a.x + c * b.x, a.y + c * b.y, a.z + c * b.z, 0.f);
}

// Pinned vertices [v_begin, v_end): x~_p -= sum_e V dP(sum_{k != p} lam_k q_k^T) q_p (their coupling
// to the free vertices through the converged positions); v~_p unchanged.
template <int LANES>
__global__ void __launch_bounds__(256) k_adj_pinned(AdjParams p, float4* __restrict__ ax) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & (LANES - 1);
    const int v = p.v_begin + t / LANES;
    const bool active = v < p.v_end;
    int j0 = 0, j1 = 0;
    float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
    if (active) {
        j0 = p.inc_off[v];
        j1 = p.inc_off[v + 1];
        xi = p.X[v];
    }
    Acc acc;
    acc.zero();
    for (int j = j0 + lane; j < j1; j += LANES) {
        const TetRec r = load_rec(p.rec + p.inc_tet[j]);
        const ElemView e = view_of(r, v);
        float F[3][3], C[3][3], J;
        elem_F(e, xi, p.X, F, C, J);
        float o[3];
        elem_offdiag(e, F, C, J, p.lam, o);
        acc.g0 += o[0];
        acc.g1 += o[1];
        acc.g2 += o[2];
    }
    group_reduce<LANES>(acc);
    if (!active || lane != 0) return;
    float4 a = ax[v];
    a.x -= acc.g0;
    a.y -= acc.g1;
    a.z -= acc.g2;
    ax[v] = a;
}

// Free vertices: y~ = m/h^2 lam, x~ = y~ - c v~, v~ = h y~.
__global__ void k_adj_update(const float4* __restrict__ lam, const float4* __restrict__ y, float4* __restrict__ ax,
                             float4* __restrict__ av, float dtsr, float c, float h, int nfree) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nfree) return;
    const float4 l = lam[i];
    const float cm = y[i].w * dtsr;
    const float4 b = av[i];
    const float yx = cm * l.x, yy = cm * l.y, yz = cm * l.z;
    ax[i] = make_float4(yx - c * b.x, yy - c * b.y, yz - c * b.z, 0.f);
    av[i] = make_float4(h * yx, h * yy, h * yz, 0.f);
}

// Per tet: dL/dmu -= sum_n lam_n . V (F - C) q_n, dL/dlambda -= sum_n lam_n . V (J - 1) C q_n
// (accumulated over steps; lam of pinned vertices is 0).
__global__ void k_adj_params(const TetRec* __restrict__ rec, const float4* __restrict__ X,
                             const float4* __restrict__ lam, float* __restrict__ gmu, float* __restrict__ glam, int ntet) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntet) return;
    const TetRec r = load_rec(rec + t);
    const int ids[4] = {r.ids.x, r.ids.y, r.ids.z, r.ids.w};
    const float D[3][3] = {{r.a.x, r.a.y, r.a.z}, {r.a.w, r.b.x, r.b.y}, {r.b.z, r.b.w, r.c.x}};
    float Q[4][3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        Q[0][c] = -D[0][c] - D[1][c] - D[2][c];
        Q[1][c] = D[0][c];
        Q[2][c] = D[1][c];
        Q[3][c] = D[2][c];
    }
    float4 P[4], Lm[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        P[k] = X[ids[k]];
        Lm[k] = lam[ids[k]];
    }
    float F[3][3];
#pragma unroll
    for (int rr = 0; rr < 3; ++rr) {
        const float o = rr == 0 ? P[0].x : rr == 1 ? P[0].y : P[0].z;
        const float e1 = (rr == 0 ? P[1].x : rr == 1 ? P[1].y : P[1].z) - o;
        const float e2 = (rr == 0 ? P[2].x : rr == 1 ? P[2].y : P[2].z) - o;
        const float e3 = (rr == 0 ? P[3].x : rr == 1 ? P[3].y : P[3].z) - o;
#pragma unroll
        for (int c = 0; c < 3; ++c) F[rr][c] = e1 * D[0][c] + e2 * D[1][c] + e3 * D[2][c];
    }
    float C[3][3];
    cof3(F, C);
    const float J = F[0][0] * C[0][0] + F[0][1] * C[0][1] + F[0][2] * C[0][2];
    float sm = 0.f, sl = 0.f;
#pragma unroll
    for (int n = 0; n < 4; ++n) {
        const float l[3] = {Lm[n].x, Lm[n].y, Lm[n].z};
#pragma unroll
        for (int rr = 0; rr < 3; ++rr) {
            float fq = 0.f, cq = 0.f;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                fq += (F[rr][c] - C[rr][c]) * Q[n][c];
                cq += C[rr][c] * Q[n][c];
            }
            sm += l[rr] * fq;
            sl += l[rr] * cq;
        }
    }
    const float V = r.c.y;
    gmu[t] -= V * sm;
    glam[t] -= V * (J - 1.0f) * sl;
}

// ---- FP64 reductions (energies, residual) ---------------------------------------------------

template <int BS>
__device__ __forceinline__ void block_sum_store(double val, double* partials) {
    __shared__ double red[BS / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) val += __shfl_xor_sync(0xffffffffu, val, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = val;
    __syncthreads();
    if (threadIdx.x < 32) {
        double w = threadIdx.x < BS / 32 ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        if (threadIdx.x == 0) partials[blockIdx.x] = w;
    }
}

// Sums partials[0..n) in a fixed order (deterministic) into out[0].
__global__ void k_sum_partials(const double* __restrict__ partials, int n, double* __restrict__ out) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += partials[i];
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double w = threadIdx.x < (int)(blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        if (threadIdx.x == 0) out[0] = w;
    }
}

// Sums partials[0..n) as k_sum_partials does and appends the sum to a history: hist[*count] when
// *count < capacity; *count always advances, so a reader sees how many sums were produced.  One
// block, so the append needs no atomics.
__global__ void k_sum_partials_append(const double* __restrict__ partials, int n, double* __restrict__ hist,
                                      int* __restrict__ count, int capacity) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += partials[i];
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double w = threadIdx.x < (int)(blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        if (threadIdx.x == 0) {
            const int k = *count;
            if (k < capacity) hist[k] = w;
            *count = k + 1;
        }
    }
}

__device__ __forceinline__ void tet_F_double(const TetRec& r, const float4* __restrict__ X, double F[3][3]) {
    const float4 p0 = X[r.ids.x], p1 = X[r.ids.y], p2 = X[r.ids.z], p3 = X[r.ids.w];
    const double e[3][3] = {{(double)p1.x - p0.x, (double)p2.x - p0.x, (double)p3.x - p0.x},
                            {(double)p1.y - p0.y, (double)p2.y - p0.y, (double)p3.y - p0.y},
                            {(double)p1.z - p0.z, (double)p2.z - p0.z, (double)p3.z - p0.z}};
    const double D[3][3] = {{r.a.x, r.a.y, r.a.z}, {r.a.w, r.b.x, r.b.y}, {r.b.z, r.b.w, r.c.x}};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) F[i][j] = e[i][0] * D[0][j] + e[i][1] * D[1][j] + e[i][2] * D[2][j];
}

__device__ __forceinline__ double det3d(const double F[3][3]) {
    return F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) - F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
           F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
}

// kind 0: incremental potential (inertia over vertices [0, nvert) + J-1 Neo-Hookean over tets)
// kind 1: log-J Neo-Hookean elastic energy only (VBDsolver::computeTotalEnergy)
__global__ void __launch_bounds__(256) k_energy(const float4* __restrict__ X, const float4* __restrict__ Y,
                                                const TetRec* __restrict__ rec, int nvert, int ntet, int kind,
                                                double inv_h2, double* __restrict__ partials) {
    double acc = 0.0;
    const int stride = gridDim.x * blockDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (kind == 0) {
        for (int i = t0; i < nvert; i += stride) {
            const float4 x = X[i], y = Y[i];
            const double dx = (double)x.x - y.x, dy = (double)x.y - y.y, dz = (double)x.z - y.z;
            acc += 0.5 * (double)y.w * inv_h2 * (dx * dx + dy * dy + dz * dz);
        }
    }
    for (int t = t0; t < ntet; t += stride) {
        const TetRec r = load_rec(rec + t);
        double F[3][3];
        tet_F_double(r, X, F);
        double tr = 0.0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) tr += F[i][j] * F[i][j];
        const double J = det3d(F);
        const double mu = r.c.z, lam = r.c.w, V0 = r.c.y;
        double psi;
        if (kind == 0) {
            psi = 0.5 * mu * (tr - 3.0) - mu * (J - 1.0) + 0.5 * lam * (J - 1.0) * (J - 1.0);
        } else {
            const double lj = log(fabs(J));
            psi = 0.5 * mu * (tr - 3.0) - mu * lj + 0.5 * lam * lj * lj;
        }
        acc += V0 * psi;
    }
    block_sum_store<256>(acc, partials);
}

// |m/h^2 (x - y) + dE/dx|^2 summed over the free vertices [v_begin, v_end): one LANES-thread
// group per vertex as in k_sweep, one FP64 partial per block.
template <int LANES>
__global__ void __launch_bounds__(256) k_residual(SweepParams p, double* __restrict__ partials) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & (LANES - 1);
    const int v = p.v_begin + t / LANES;
    const bool active = v < p.v_end;
    float4 xi = make_float4(0.f, 0.f, 0.f, 0.f);
    int j0 = 0, j1 = 0;
    if (active) {
        xi = p.x[v];
        j0 = p.inc_off[v];
        j1 = p.inc_off[v + 1];
    }
    Acc a;
    a.zero();
    for (int j = j0 + lane; j < j1; j += LANES) {
        const TetRec r = load_rec(p.rec + p.inc_tet[j]);
        tet_contrib<false>(r, v, xi, p.x, a);
    }
    group_reduce<LANES>(a);
    double r2 = 0.0;
    if (active && lane == 0) {
        const float4 yi = p.y[v];
        const double cm = (double)yi.w * p.dtsr;
        const double r0 = cm * ((double)xi.x - yi.x) + a.g0;
        const double r1 = cm * ((double)xi.y - yi.y) + a.g1;
        const double rz = cm * ((double)xi.z - yi.z) + a.g2;
        r2 = r0 * r0 + r1 * r1 + rz * rz;
    }
    block_sum_store<256>(r2, partials);
}

}  // namespace vbd
