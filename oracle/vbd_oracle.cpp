// VBD oracle -- TEST INFRASTRUCTURE ONLY.
//
// A plain-C++ (no Eigen) restatement of the reference's CPU Vertex Block Descent path
// (extinguish7/VBD_TetMesh), templated on float / double.  Only tests/, the smoke check in
// __graft_entry__.py and the CPU-baseline leg of bench.py may load this library, and only as
// the checker or as the timed CPU baseline -- never on the product path.
//
// Parity status: the reference needs Eigen 3, which is absent from this image, so it cannot
// be built with its real dependency.  This restatement is pinned against the reference's own
// sources (TetMesh.h, VBD.cpp, Energy.cpp, GraphColoring.cpp, NeoHookean.cpp) compiled
// unchanged against this project's Eigen-API subset header (see oracle/Makefile, target
// `ref`, and tests/test_oracle_pin.py).  Eigen's own arithmetic (product summation order,
// inverse, JacobiSVD) is NOT pinned: Eigen expressions are evaluated here eagerly, in source
// order, with inner products accumulated left to right.
//
// What it follows (file:line in the reference):
//   TetMesh::initialize            TetMesh.h:213-275 (mass = rho*V/4, adjacency in tet order)
//   TetMesh::computeRestVolume     TetMesh.h:291-298
//   GraphColoring::colorVertices   GraphColoring.cpp:7-66 (greedy, vertex-id order)
//   VBDsolver::precomputeTetData   VBD.cpp:36-58, Energy.cpp:6-32 (Dm, Dm^-1, V0)
//   VBDsolver::step                VBD.cpp:60-101 (serial colour order = numThreads 1)
//   VBDsolver::forwardStep         VBD.cpp:103-112, TetMesh.h:319-348
//   VBDsolver::solve/solveVertex   VBD.cpp:114-203, Types.h:85-112 (det guard 1e-8)
//   computeTetContribution         VBD.cpp:205-256, Energy.cpp:90-158 (literal 12x12 form)
//   computeTotalEnergy             VBD.cpp:258-288, NeoHookean.cpp:6-20 (log-J NH, J = |det F|)
//   Chebyshev                      VBD.cpp:290-311
//   TetMesh::updateVelocity        TetMesh.h:305-311 (x0.999)
// The reference parallelises the colour loop with OpenMP (VBD.cpp:120), which races between
// adjacent colours; this oracle runs colours serially (the numThreads=1 semantics).  Within one
// colour the vertex updates are independent, so the optional threaded mode (within-colour
// parallel) returns bit-identical results.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

template <class T> struct M3 {
    T m[3][3];
};

template <class T> static inline T dot3(const T* a, const T* b) {
    T s = a[0] * b[0];
    s += a[1] * b[1];
    s += a[2] * b[2];
    return s;
}

// Eigen cross product (component formulas of the standard 3-vector cross product).
template <class T> static inline void cross3(const T* a, const T* b, T* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// Cofactor-expansion determinant along row 0 (Types.h:87-89; the same formula serves
// Matrix3::determinant() in VBD.cpp:141).
template <class T> static inline T det3(const M3<T>& A) {
    const auto& a = A.m;
    return a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
           a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
           a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
}

// Cofactor matrix, Energy.cpp:61-73.
template <class T> static inline M3<T> cofactor(const M3<T>& Fm) {
    const auto& F = Fm.m;
    M3<T> C;
    C.m[0][0] = F[1][1] * F[2][2] - F[1][2] * F[2][1];
    C.m[0][1] = F[1][2] * F[2][0] - F[1][0] * F[2][2];
    C.m[0][2] = F[1][0] * F[2][1] - F[1][1] * F[2][0];
    C.m[1][0] = F[2][1] * F[0][2] - F[2][2] * F[0][1];
    C.m[1][1] = F[2][2] * F[0][0] - F[2][0] * F[0][2];
    C.m[1][2] = F[2][0] * F[0][1] - F[2][1] * F[0][0];
    C.m[2][0] = F[0][1] * F[1][2] - F[0][2] * F[1][1];
    C.m[2][1] = F[0][2] * F[1][0] - F[0][0] * F[1][2];
    C.m[2][2] = F[0][0] * F[1][1] - F[0][1] * F[1][0];
    return C;
}

// Directional derivative of the cofactor matrix, Energy.cpp:76-88.
template <class T> static inline M3<T> cofactor_deriv(const M3<T>& Fm, const M3<T>& dFm) {
    const auto& F = Fm.m;
    const auto& d = dFm.m;
    M3<T> o;
    o.m[0][0] = d[1][1] * F[2][2] + F[1][1] * d[2][2] - d[1][2] * F[2][1] - F[1][2] * d[2][1];
    o.m[0][1] = d[1][2] * F[2][0] + F[1][2] * d[2][0] - d[1][0] * F[2][2] - F[1][0] * d[2][2];
    o.m[0][2] = d[1][0] * F[2][1] + F[1][0] * d[2][1] - d[1][1] * F[2][0] - F[1][1] * d[2][0];
    o.m[1][0] = d[2][1] * F[0][2] + F[2][1] * d[0][2] - d[2][2] * F[0][1] - F[2][2] * d[0][1];
    o.m[1][1] = d[2][2] * F[0][0] + F[2][2] * d[0][0] - d[2][0] * F[0][2] - F[2][0] * d[0][2];
    o.m[1][2] = d[2][0] * F[0][1] + F[2][0] * d[0][1] - d[2][1] * F[0][0] - F[2][1] * d[0][0];
    o.m[2][0] = d[0][1] * F[1][2] + F[0][1] * d[1][2] - d[0][2] * F[1][1] - F[0][2] * d[1][1];
    o.m[2][1] = d[0][2] * F[1][0] + F[0][2] * d[1][0] - d[0][0] * F[1][2] - F[0][0] * d[1][2];
    o.m[2][2] = d[0][0] * F[1][1] + F[0][0] * d[1][1] - d[0][1] * F[1][0] - F[0][1] * d[1][0];
    return o;
}

template <class T> static inline M3<T> matmul(const M3<T>& A, const M3<T>& B) {
    M3<T> C;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            T s = A.m[i][0] * B.m[0][j];
            s += A.m[i][1] * B.m[1][j];
            s += A.m[i][2] * B.m[2][j];
            C.m[i][j] = s;
        }
    return C;
}

// Inverse by transposed cofactors over the determinant (Dm.inverse() in VBD.cpp:49; the
// standard adjugate formula, cofactors taken cyclically, det expanded along column 0).
template <class T> static inline M3<T> inverse3(const M3<T>& A) {
    auto cof = [&](int i, int j) {
        int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
        return A.m[i1][j1] * A.m[i2][j2] - A.m[i1][j2] * A.m[i2][j1];
    };
    T c00 = cof(0, 0), c10 = cof(1, 0), c20 = cof(2, 0);
    T det = c00 * A.m[0][0];
    det += c10 * A.m[1][0];
    det += c20 * A.m[2][0];
    T inv = T(1) / det;
    M3<T> R;
    R.m[0][0] = c00 * inv;
    R.m[0][1] = c10 * inv;
    R.m[0][2] = c20 * inv;
    for (int r = 1; r < 3; ++r)
        for (int c = 0; c < 3; ++c) R.m[r][c] = cof(c, r) * inv;
    return R;
}

// Ds / Dm: columns x1-x0, x2-x0, x3-x0 (Energy.cpp:6-14).
template <class T> static inline M3<T> edge_matrix(const T* x, const int32_t* tet) {
    M3<T> D;
    for (int c = 0; c < 3; ++c) {
        const T* a = x + 3 * tet[c + 1];
        const T* o = x + 3 * tet[0];
        for (int r = 0; r < 3; ++r) D.m[r][c] = a[r] - o[r];
    }
    return D;
}

// compute_Volume, Energy.cpp:24-32: |d3 . (d1 x d2)| / 6.
template <class T> static inline T edge_volume(const M3<T>& Ds) {
    T d1[3] = {Ds.m[0][0], Ds.m[1][0], Ds.m[2][0]};
    T d2[3] = {Ds.m[0][1], Ds.m[1][1], Ds.m[2][1]};
    T d3[3] = {Ds.m[0][2], Ds.m[1][2], Ds.m[2][2]};
    T c[3];
    cross3(d1, d2, c);
    return std::abs(dot3(d3, c)) / T(6);
}

// TetMesh::computeRestVolume, TetMesh.h:291-298: |e0 . (e1 x e2)| / 6.
template <class T> static inline T rest_volume(const T* rest, const int32_t* tet) {
    T e[3][3];
    for (int k = 0; k < 3; ++k)
        for (int r = 0; r < 3; ++r) e[k][r] = rest[3 * tet[k + 1] + r] - rest[3 * tet[0] + r];
    T c[3];
    cross3(e[1], e[2], c);
    return std::abs(dot3(e[0], c)) / T(6);
}

// (T)(lambda * (J - 1.0)): the reference mixes a double literal into a float expression
// (Energy.cpp:97,127); the scalar is formed in double and then used as a float factor.
template <class T> static inline T lam_jm1(T lambda, T J) {
    return T(double(lambda) * (double(J) - 1.0));
}

// Q = Ps * DmInv (Energy.cpp:101-106): row 0 = -(sum of DmInv rows), row k = DmInv row k-1.
template <class T> static inline void q_rows(const M3<T>& Di, T Q[4][3]) {
    for (int c = 0; c < 3; ++c) {
        T s = -Di.m[0][c];
        s += -Di.m[1][c];
        s += -Di.m[2][c];
        Q[0][c] = s;
        for (int k = 1; k < 4; ++k) Q[k][c] = Di.m[k - 1][c];
    }
}

// Literal restatement of ElasticEnergy::compute_Hessian_and_Gradient (Energy.cpp:90-158)
// restricted to what VBDsolver::computeTetContribution keeps (VBD.cpp:250-255): gradient
// segment n and Hessian block (n,n).  With full12 set, every 3x3 block of the 12x12 element
// Hessian is formed (the reference's cost) and block (n,n) is returned.
template <class T>
static void tet_block_literal(const M3<T>& DmInv, const M3<T>& F, T lambda, T mu, T volume, int n,
                              T Hn[3][3], T gn[3], bool full12) {
    T J = det3(F);
    M3<T> C = cofactor(F);
    T s = lam_jm1(lambda, J);
    M3<T> P;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            T a = mu * (F.m[i][j] - C.m[i][j]);
            T b = s * C.m[i][j];
            P.m[i][j] = a + b;
        }
    T Q[4][3];
    q_rows(DmInv, Q);
    // g_nodes = (volume * P) * Q^T
    for (int i = 0; i < 3; ++i) {
        T vp0 = volume * P.m[i][0], vp1 = volume * P.m[i][1], vp2 = volume * P.m[i][2];
        T g = vp0 * Q[n][0];
        g += vp1 * Q[n][1];
        g += vp2 * Q[n][2];
        gn[i] = g;
    }
    // HF(vi + 3 vj, i + 3 j) = dP(vi, vj) for dF = e_i e_j^T (Energy.cpp:115-136)
    T HF[9][9];
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) {
            int col = i + 3 * j;
            M3<T> dF{};
            dF.m[i][j] = T(1);
            T dJ = C.m[i][j];
            M3<T> dC = cofactor_deriv(F, dF);
            T ldJ = lambda * dJ;
            for (int vj = 0; vj < 3; ++vj)
                for (int vi = 0; vi < 3; ++vi) {
                    T a = mu * (dF.m[vi][vj] - dC.m[vi][vj]);
                    T b = ldJ * C.m[vi][vj];
                    T c = s * dC.m[vi][vj];
                    HF[vi + 3 * vj][col] = (a + b) + c;
                }
        }
    // 12x12 assembly (Energy.cpp:139-154)
    auto block = [&](int bn, int bm, T out[3][3]) {
        for (int c = 0; c < 3; ++c)
            for (int cp = 0; cp < 3; ++cp) {
                T val = T(0);
                for (int b = 0; b < 3; ++b)
                    for (int d = 0; d < 3; ++d) val += HF[c + 3 * b][cp + 3 * d] * Q[bn][b] * Q[bm][d];
                out[c][cp] = volume * val;
            }
    };
    if (full12) {
        T tmp[3][3];
        for (int bn = 0; bn < 4; ++bn)
            for (int bm = 0; bm < 4; ++bm) {
                block(bn, bm, tmp);
                if (bn == n && bm == n) std::memcpy(Hn, tmp, sizeof(tmp));
            }
    } else {
        block(n, n, Hn);
    }
}

// Closed form of the same block: H_nn = V (mu |q|^2 I + lambda (C q)(C q)^T), g_n = V P q.
// The cofactor-derivative terms of the literal form contract to zero against q q^T because
// dC_ij/dF_kl is antisymmetric in (j, l).
template <class T>
static void tet_block_closed(const M3<T>& DmInv, const M3<T>& F, T lambda, T mu, T volume, int n,
                             T Hn[3][3], T gn[3]) {
    T J = det3(F);
    M3<T> C = cofactor(F);
    T s = lam_jm1(lambda, J);
    T Q[4][3];
    q_rows(DmInv, Q);
    const T* q = Q[n];
    T Cq[3];
    for (int i = 0; i < 3; ++i) {
        T g = T(0), cq = T(0);
        for (int k = 0; k < 3; ++k) {
            T p = mu * (F.m[i][k] - C.m[i][k]) + s * C.m[i][k];
            g += (volume * p) * q[k];
            cq += C.m[i][k] * q[k];
        }
        gn[i] = g;
        Cq[i] = cq;
    }
    T qq = dot3(q, q);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            Hn[i][j] = volume * ((i == j ? mu * qq : T(0)) + lambda * Cq[i] * Cq[j]);
}

// WRAPPER: the semantics of the reference's GPU wrapper (VBD_GPU_Solver) instead of VBDsolver's.
enum Mode { LITERAL = 0, LITERAL_FULL12 = 1, CLOSED = 2, WRAPPER = 3 };

// ---- VBD_GPU_Solver semantics (VBD_GPU_Wrapper.cu:114-235, 332-362; VBD_DeviceMath.cuh) ----------

// det3x3 of VBD_DeviceMath.cuh:11-15 (expansion along row 0).
template <class T> static inline T det3_row0(const T A[3][3]) {
    return A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) - A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
           A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
}

template <class T> static inline void cof3(const T F[3][3], T C[3][3]) {
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

// computeTetContributionLocalCorotated (VBD_DeviceMath.cuh:127-198): polar factor R of F by five
// Higham steps R <- (R + cof(R)/det R)/2 (stopping when |det R| < 1e-8), tr = R:F - 3,
// P = 2 mu (F - R) + lambda tr R, g = V P q_n, H = V (2 mu |q_n|^2 I + lambda (R q_n)(R q_n)^T).
template <class T>
static void corot_block(const M3<T>& Di, const M3<T>& Fm, T mu, T lambda, T volume, int n, T H[9], T g[3]) {
    T F[3][3], R[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) R[a][b] = F[a][b] = Fm.m[a][b];
    for (int it = 0; it < 5; ++it) {
        T det = det3_row0(R);
        if (std::abs(double(det)) < 1e-8) break;
        T C[3][3];
        cof3(R, C);
        T inv = T(1) / det;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) R[a][b] = T(0.5) * (R[a][b] + C[a][b] * inv);
    }
    T tr = T(0);
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) tr += R[a][b] * F[a][b];
    tr -= T(3);
    T P[3][3];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) P[a][b] = T(2) * mu * (F[a][b] - R[a][b]) + lambda * tr * R[a][b];
    T q[3];
    if (n == 0) {
        for (int c = 0; c < 3; ++c) q[c] = -Di.m[0][c] - Di.m[1][c] - Di.m[2][c];
    } else {
        for (int c = 0; c < 3; ++c) q[c] = Di.m[n - 1][c];
    }
    for (int a = 0; a < 3; ++a) g[a] = volume * (P[a][0] * q[0] + P[a][1] * q[1] + P[a][2] * q[2]);
    T qsq = q[0] * q[0] + q[1] * q[1] + q[2] * q[2];
    T RQ[3];
    for (int a = 0; a < 3; ++a) RQ[a] = R[a][0] * q[0] + R[a][1] * q[1] + R[a][2] * q[2];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) H[3 * a + b] = volume * ((a == b ? T(2) * mu * qsq : T(0)) + lambda * RQ[a] * RQ[b]);
}

template <class T> struct Sim {
    int N = 0, NT = 0;
    std::vector<T> rest, x, xprev, v, y, pp, mass, tetRestVol, V0, mu, lam;
    std::vector<M3<T>> DmInv;
    std::vector<int32_t> tets;
    std::vector<uint8_t> fixed;
    std::vector<int32_t> adj_off, adj;  // vertAdjacentTets as CSR, ascending tet id
    std::vector<std::vector<int32_t>> colors;
    int mode = LITERAL;
    int threads = 1;

    void setup(int n, int nt, const double* rest_, const double* x_, const double* v_, const int32_t* tets_,
               const uint8_t* fixed_, const double* mu_, const double* lam_, double density) {
        N = n;
        NT = nt;
        rest.assign(rest_, rest_ + 3 * n);
        x.assign(x_, x_ + 3 * n);
        xprev = x;
        v.assign(3 * n, T(0));
        if (v_)
            for (int i = 0; i < 3 * n; ++i) v[i] = T(v_[i]);
        y.assign(3 * n, T(0));
        pp.assign(3 * n, T(0));
        tets.assign(tets_, tets_ + 4 * nt);
        fixed.assign(fixed_, fixed_ + n);
        mu.resize(nt);
        lam.resize(nt);
        for (int t = 0; t < nt; ++t) {
            mu[t] = T(mu_[t]);
            lam[t] = T(lam_[t]);
        }
        // TetMesh::initialize (TetMesh.h:249-265)
        mass.assign(n, T(0));
        tetRestVol.resize(nt);
        std::vector<int32_t> cnt(n + 1, 0);
        T rho = T(density);
        for (int t = 0; t < nt; ++t) {
            T vol = rest_volume(rest.data(), &tets[4 * t]);
            tetRestVol[t] = vol;
            T tetMass = vol * rho;
            for (int j = 0; j < 4; ++j) {
                cnt[tets[4 * t + j] + 1]++;
                mass[tets[4 * t + j]] += tetMass / T(4);
            }
        }
        adj_off.assign(n + 1, 0);
        for (int i = 0; i < n; ++i) adj_off[i + 1] = adj_off[i] + cnt[i + 1];
        adj.assign(adj_off[n], 0);
        std::vector<int32_t> fill(adj_off.begin(), adj_off.end() - 1);
        for (int t = 0; t < nt; ++t)
            for (int j = 0; j < 4; ++j) adj[fill[tets[4 * t + j]]++] = t;
        // VBDsolver::precomputeTetData (VBD.cpp:36-58)
        DmInv.resize(nt);
        V0.resize(nt);
        for (int t = 0; t < nt; ++t) {
            M3<T> Dm = edge_matrix(rest.data(), &tets[4 * t]);
            DmInv[t] = inverse3(Dm);
            V0[t] = edge_volume(Dm);
        }
    }

    // GraphColoring::colorVertices (GraphColoring.cpp:28-66) with getNeighbors (:7-26).
    void color() {
        std::vector<int32_t> col(N, -1);
        std::vector<int32_t> stamp;  // stamp[c] == v+1 <=> colour c used by a neighbour of v
        colors.clear();
        for (int vtx = 0; vtx < N; ++vtx) {
            for (int a = adj_off[vtx]; a < adj_off[vtx + 1]; ++a) {
                const int32_t* tet = &tets[4 * adj[a]];
                for (int i = 0; i < 4; ++i) {
                    int nb = tet[i];
                    if (nb != vtx && col[nb] != -1) {
                        if ((int)stamp.size() <= col[nb]) stamp.resize(col[nb] + 1, 0);
                        stamp[col[nb]] = vtx + 1;
                    }
                }
            }
            int c = 0;
            while (c < (int)stamp.size() && stamp[c] == vtx + 1) ++c;
            col[vtx] = c;
            if ((int)colors.size() <= c) colors.resize(c + 1);
            colors[c].push_back(vtx);
        }
    }

    // VBDsolver::solveVertex + the update in VBDsolver::solve (VBD.cpp:124-156, 160-203).
    // vbd_solve_color_kernel (VBD_GPU_Wrapper.cu:114-235) for one vertex: 16 partial sums (thread t
    // of the block takes incident tets t, t + 16, ...), added in thread order onto
    // H = m/h^2 * 1.000001 I and f = m/h^2 (y - x); solve3x3 (VBD_DeviceMath.cuh:47-64).
    void solve_vertex_wrapper(int vid, T dtSqrRecip) {
        constexpr int kThreads = 16;
        T hs[kThreads][9] = {}, fs[kThreads][3] = {};
        for (int a = adj_off[vid]; a < adj_off[vid + 1]; ++a) {
            const int lane = (a - adj_off[vid]) % kThreads;
            int t = adj[a];
            const int32_t* tet = &tets[4 * t];
            int n = -1;
            for (int i = 0; i < 4; ++i)
                if (tet[i] == vid) {
                    n = i;
                    break;
                }
            if (n < 0) continue;
            M3<T> Ds = edge_matrix(x.data(), tet);
            M3<T> F = matmul(Ds, DmInv[t]);
            T Hl[9], gl[3];
            corot_block(DmInv[t], F, mu[t], lam[t], V0[t], n, Hl, gl);
            for (int k = 0; k < 9; ++k) hs[lane][k] += Hl[k];
            for (int k = 0; k < 3; ++k) fs[lane][k] -= gl[k];
        }
        T coeff = mass[vid] * dtSqrRecip;
        T reg = coeff * T(1.000001f);
        T H[3][3] = {{reg, T(0), T(0)}, {T(0), reg, T(0)}, {T(0), T(0), reg}};
        T f[3];
        for (int c = 0; c < 3; ++c) f[c] = coeff * (y[3 * vid + c] - x[3 * vid + c]);
        for (int l = 0; l < kThreads; ++l) {
            for (int k = 0; k < 9; ++k) H[k / 3][k % 3] += hs[l][k];
            for (int k = 0; k < 3; ++k) f[k] += fs[l][k];
        }
        T det = det3_row0(H);
        if (std::abs(double(det)) < 1e-8) return;
        T adjm[3][3];
        cof3(H, adjm);
        T inv = T(1) / det;
        for (int i = 0; i < 3; ++i) x[3 * vid + i] += inv * (adjm[0][i] * f[0] + adjm[1][i] * f[1] + adjm[2][i] * f[2]);
    }

    void solve_vertex(int vid, T dtSqrRecip) {
        if (mode == WRAPPER) {
            solve_vertex_wrapper(vid, dtSqrRecip);
            return;
        }
        T H[3][3] = {};
        T f[3];
        T m = mass[vid];
        T md = m * dtSqrRecip;
        for (int i = 0; i < 3; ++i) H[i][i] += md;
        for (int i = 0; i < 3; ++i) {
            T d = y[3 * vid + i] - x[3 * vid + i];
            f[i] = (m * d) * dtSqrRecip;
        }
        for (int a = adj_off[vid]; a < adj_off[vid + 1]; ++a) {
            int t = adj[a];
            const int32_t* tet = &tets[4 * t];
            int n = -1;
            for (int i = 0; i < 4; ++i)
                if (tet[i] == vid) {
                    n = i;
                    break;
                }
            if (n < 0) continue;
            M3<T> Ds = edge_matrix(x.data(), tet);
            M3<T> F = matmul(Ds, DmInv[t]);
            T Hl[3][3], gl[3];
            if (mode == CLOSED)
                tet_block_closed(DmInv[t], F, lam[t], mu[t], V0[t], n, Hl, gl);
            else
                tet_block_literal(DmInv[t], F, lam[t], mu[t], V0[t], n, Hl, gl, mode == LITERAL_FULL12);
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) H[i][j] += Hl[i][j];
            for (int i = 0; i < 3; ++i) f[i] -= gl[i];
        }
        M3<T> A;
        std::memcpy(A.m, H, sizeof(H));
        T det = det3(A);
        if (std::abs(double(det)) > 1e-8) {
            // AnalyticSolver3x3::solve (Types.h:85-112)
            if (std::abs(double(det)) < 1e-8) return;
            T invDet = T(1) / det;
            T adjm[3][3];
            adjm[0][0] = H[1][1] * H[2][2] - H[1][2] * H[2][1];
            adjm[0][1] = H[0][2] * H[2][1] - H[0][1] * H[2][2];
            adjm[0][2] = H[0][1] * H[1][2] - H[0][2] * H[1][1];
            adjm[1][0] = H[1][2] * H[2][0] - H[1][0] * H[2][2];
            adjm[1][1] = H[0][0] * H[2][2] - H[0][2] * H[2][0];
            adjm[1][2] = H[0][2] * H[1][0] - H[0][0] * H[1][2];
            adjm[2][0] = H[1][0] * H[2][1] - H[1][1] * H[2][0];
            adjm[2][1] = H[0][1] * H[2][0] - H[0][0] * H[2][1];
            adjm[2][2] = H[0][0] * H[1][1] - H[0][1] * H[1][0];
            for (int i = 0; i < 3; ++i) {
                T p = adjm[i][0] * f[0];
                p += adjm[i][1] * f[1];
                p += adjm[i][2] * f[2];
                x[3 * vid + i] += invDet * p;
            }
        }
    }

    // One Gauss-Seidel sweep, colour by colour (VBD.cpp:114-158).
    void sweep(T dtSqrRecip) {
        for (const auto& grp : colors) {
            int ng = (int)grp.size();
#ifdef _OPENMP
#pragma omp parallel for num_threads(threads) schedule(static) if (threads > 1)
#endif
            for (int k = 0; k < ng; ++k) {
                int vid = grp[k];
                if (fixed[vid]) continue;
                solve_vertex(vid, dtSqrRecip);
            }
        }
    }

    // getAcceleratorOmega of the GPU wrapper (VBD_GPU_Wrapper.cu:240-244): arithmetic in T.
    static T omega_of_wrapper(int order, T rho, T prev) {
        if (order == 1) return T(1);
        if (order == 2) return T(2) / (T(2) - (rho * rho));
        return T(4) / (T(4) - (rho * rho) * prev);
    }

    // getAcceleratorOmega (VBD.cpp:302-311), with the reference's double literals.
    static T omega_of(int order, T rho, T prev) {
        if (order == 1) return T(1);
        if (order == 2) return T(2.0 / (2.0 - double(rho * rho)));
        return T(4.0 / (4.0 - double(rho * rho * prev)));
    }

    // VBDsolver::computeTotalEnergy (VBD.cpp:258-288) with NeoHookean::compute_Energy
    // (NeoHookean.cpp:6-20); the singular-value product is |det F|.
    T total_energy_ref() const {
        T total = T(0);
        for (int t = 0; t < NT; ++t) {
            M3<T> Ds = edge_matrix(x.data(), &tets[4 * t]);
            M3<T> F = matmul(Ds, DmInv[t]);
            T J = std::abs(det3(F));
            // (F^T F).trace(): diagonal entries of the product, each a column's inner product
            T tr = T(0);
            for (int i = 0; i < 3; ++i) {
                T d = F.m[0][i] * F.m[0][i];
                d += F.m[1][i] * F.m[1][i];
                d += F.m[2][i] * F.m[2][i];
                tr += d;
            }
            T lj = std::log(J);
            T E = T(double(mu[t]) * 0.5 * double(tr - T(3)) - double(mu[t] * lj) +
                    0.5 * double(lam[t]) * std::pow(double(lj), 2.0));
            total += E * V0[t];
        }
        return total;
    }

    // The iteration loop of VBDsolver::step (VBD.cpp:75-96): sweeps with the Chebyshev blend.
    void solve_loop(T dtSqrRecip, int iters, bool accel, T rho, std::vector<double>* ehist) {
        T omega = T(1);
        for (int it = 0; it < iters; ++it) {
            std::vector<T> cur = x;
            sweep(dtSqrRecip);
            if (accel) {
                omega = mode == WRAPPER ? omega_of_wrapper(it + 1, rho, omega) : omega_of(it + 1, rho, omega);
                if (omega > T(1)) {
                    for (int i = 0; i < N; ++i) {
                        if (fixed[i]) continue;
                        for (int c = 0; c < 3; ++c) {
                            T d = x[3 * i + c] - pp[3 * i + c];
                            x[3 * i + c] = omega * d + pp[3 * i + c];
                        }
                    }
                }
                pp.swap(cur);
            }
            if (ehist && it % 10 == 0) ehist->push_back(double(total_energy_ref()));
        }
    }

    void step(T dt, int substeps, int iters, const T g[3], bool accel, T rho, std::vector<double>* ehist) {
        T subDt = dt / T(substeps);
        for (int s = 0; s < substeps; ++s) {
            // forwardStep (VBD.cpp:103-112)
            xprev = x;
            for (int i = 0; i < N; ++i) {
                if (fixed[i]) continue;
                for (int c = 0; c < 3; ++c) v[3 * i + c] += subDt * g[c];
            }
            for (int i = 0; i < N; ++i)
                for (int c = 0; c < 3; ++c)
                    y[3 * i + c] = fixed[i] ? x[3 * i + c] : x[3 * i + c] + subDt * v[3 * i + c];
            T dtSqrRecip = T(1.0 / double(subDt * subDt));
            // main.cpp's GPU loop: solveVBD starts from x = y and takes 1/subDt^2 in float
            // (main.cpp:211-225, VBD_GPU_Wrapper.cu:334)
            if (mode == WRAPPER) {
                x = y;
                dtSqrRecip = T(1) / (subDt * subDt);
            }
            solve_loop(dtSqrRecip, iters, accel, rho, ehist);
            // updateVelocity (TetMesh.h:305-311)
            for (int i = 0; i < N; ++i) {
                if (fixed[i]) continue;
                for (int c = 0; c < 3; ++c) {
                    T d = x[3 * i + c] - xprev[3 * i + c];
                    v[3 * i + c] = (d / subDt) * T(0.999);
                }
            }
        }
    }

    // || m_i/h^2 (x_i - y_i) + dE/dx_i ||_2 over free vertices (closed-form gradient, double sums).
    double residual_norm(T dtSqrRecip) const {
        double r2 = 0.0;
        for (int vid = 0; vid < N; ++vid) {
            if (fixed[vid]) continue;
            double r[3];
            for (int c = 0; c < 3; ++c)
                r[c] = double(mass[vid]) * double(dtSqrRecip) * (double(x[3 * vid + c]) - double(y[3 * vid + c]));
            for (int a = adj_off[vid]; a < adj_off[vid + 1]; ++a) {
                int t = adj[a];
                const int32_t* tet = &tets[4 * t];
                int n = 0;
                while (tet[n] != vid) ++n;
                M3<T> Ds = edge_matrix(x.data(), tet);
                M3<T> F = matmul(Ds, DmInv[t]);
                T Hl[3][3], gl[3];
                tet_block_closed(DmInv[t], F, lam[t], mu[t], V0[t], n, Hl, gl);
                for (int c = 0; c < 3; ++c) r[c] += double(gl[c]);
            }
            r2 += r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        }
        return std::sqrt(r2);
    }

    // Incremental potential sum_i m_i/(2h^2)|x_i - y_i|^2 + sum_t V_t psi(F_t) with the
    // force-consistent energy psi = mu/2 (|F|^2 - 3) - mu (J - 1) + lambda/2 (J - 1)^2,
    // accumulated in double.
    double ip_energy(double h) const {
        double e = 0.0;
        double ih2 = 1.0 / (h * h);
        for (int i = 0; i < N; ++i) {
            double d2 = 0;
            for (int c = 0; c < 3; ++c) {
                double d = double(x[3 * i + c]) - double(y[3 * i + c]);
                d2 += d * d;
            }
            e += 0.5 * double(mass[i]) * ih2 * d2;
        }
        for (int t = 0; t < NT; ++t) e += elastic_psi(t) * double(V0[t]);
        return e;
    }

    double elastic_psi(int t) const {
        M3<double> Ds, Di;
        const int32_t* tet = &tets[4 * t];
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r) Ds.m[r][c] = double(x[3 * tet[c + 1] + r]) - double(x[3 * tet[0] + r]);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) Di.m[r][c] = double(DmInv[t].m[r][c]);
        M3<double> F = matmul(Ds, Di);
        double J = det3(F), tr = 0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) tr += F.m[i][j] * F.m[i][j];
        double m = double(mu[t]), l = double(lam[t]);
        return 0.5 * m * (tr - 3.0) - m * (J - 1.0) + 0.5 * l * (J - 1.0) * (J - 1.0);
    }
};

// ---- FP64 implicit adjoint of the step sequence (the reference gradient) -----------------------
//
// Each step is treated as converged: M/h^2 (x' - y) + dPsi/dx(x'; mu, lambda) = 0 on free vertices,
// y = x + h v + h^2 g, v' = 0.999 (x' - x) / h, pinned vertices fixed.  Backward per step, with
// X~, V~ the adjoints of (x', v'):
//   G = X~ + c V~ (c = 0.999/h),  A_ff lam = G_f with A = M/h^2 + Hessian of Psi at x',
//   y~ = M/h^2 lam,  x~ = y~ - c V~, v~ = h y~ (free),  x~_p = X~_p - (A_pf lam)_p, v~_p = V~_p,
//   dL/dmu_e -= sum_n lam_n . V (F - C) q_n,  dL/dlambda_e -= sum_n lam_n . V (J - 1) C q_n.
// A_ff lam = G is solved by conjugate gradients on the assembled block matrix (element Hessians
// from the literal 12x12 form of Energy.cpp:115-154).
struct AdjointF64 {
    Sim<double> sim;
    std::vector<std::vector<double>> xs, vs;  // positions / velocities at the start of each step, and the final state
    // neighbour structure: for vertex i, sorted neighbour list including i, and block storage
    std::vector<int32_t> nb_off, nb;
    std::vector<double> blocks;  // 9 per (i, j) entry

    int find(int i, int j) const {
        const int32_t* b = nb.data() + nb_off[i];
        const int n = nb_off[i + 1] - nb_off[i];
        return nb_off[i] + int(std::lower_bound(b, b + n, j) - b);
    }

    void build_pattern() {
        std::vector<std::vector<int32_t>> adj(sim.N);
        for (int t = 0; t < sim.NT; ++t)
            for (int a = 0; a < 4; ++a)
                for (int b = 0; b < 4; ++b) adj[sim.tets[4 * t + a]].push_back(sim.tets[4 * t + b]);
        nb_off.assign(sim.N + 1, 0);
        nb.clear();
        for (int i = 0; i < sim.N; ++i) {
            adj[i].push_back(i);
            std::sort(adj[i].begin(), adj[i].end());
            adj[i].erase(std::unique(adj[i].begin(), adj[i].end()), adj[i].end());
            nb.insert(nb.end(), adj[i].begin(), adj[i].end());
            nb_off[i + 1] = (int)nb.size();
        }
    }

    // full 12x12 element Hessian (as 16 3x3 blocks) and gradient, double
    static void element(const M3<double>& Di, const M3<double>& F, double lam, double mu, double V, double H[4][4][3][3]) {
        double J = det3(F);
        M3<double> C = cofactor(F);
        double Q[4][3];
        q_rows(Di, Q);
        double HF[9][9];
        for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i) {
                M3<double> dF{};
                dF.m[i][j] = 1.0;
                M3<double> dC = cofactor_deriv(F, dF);
                for (int vj = 0; vj < 3; ++vj)
                    for (int vi = 0; vi < 3; ++vi)
                        HF[vi + 3 * vj][i + 3 * j] = mu * (dF.m[vi][vj] - dC.m[vi][vj]) + lam * C.m[i][j] * C.m[vi][vj] +
                                                      lam * (J - 1.0) * dC.m[vi][vj];
            }
        for (int n = 0; n < 4; ++n)
            for (int m = 0; m < 4; ++m)
                for (int c = 0; c < 3; ++c)
                    for (int cp = 0; cp < 3; ++cp) {
                        double val = 0.0;
                        for (int b = 0; b < 3; ++b)
                            for (int d = 0; d < 3; ++d) val += HF[c + 3 * b][cp + 3 * d] * Q[n][b] * Q[m][d];
                        H[n][m][c][cp] = V * val;
                    }
    }

    M3<double> F_of(const std::vector<double>& x, int t) const {
        M3<double> Ds = edge_matrix(x.data(), &sim.tets[4 * t]);
        return matmul(Ds, sim.DmInv[t]);
    }

    void assemble(const std::vector<double>& x, double ih2) {
        blocks.assign(nb.size() * 9, 0.0);
        for (int i = 0; i < sim.N; ++i) {
            const int k = find(i, i);
            for (int c = 0; c < 3; ++c) blocks[9 * k + 4 * c] += sim.mass[i] * ih2;
        }
        double H[4][4][3][3];
        for (int t = 0; t < sim.NT; ++t) {
            element(sim.DmInv[t], F_of(x, t), sim.lam[t], sim.mu[t], sim.V0[t], H);
            const int32_t* q = &sim.tets[4 * t];
            for (int n = 0; n < 4; ++n)
                for (int m = 0; m < 4; ++m) {
                    const int k = find(q[n], q[m]);
                    for (int c = 0; c < 3; ++c)
                        for (int cp = 0; cp < 3; ++cp) blocks[9 * k + 3 * c + cp] += H[n][m][c][cp];
                }
        }
    }

    // y = A x restricted to rows/cols of the given mask (1 = included)
    void matvec(const std::vector<double>& x, std::vector<double>& y, const std::vector<uint8_t>& row_mask,
                const std::vector<uint8_t>& col_mask) const {
        y.assign(3 * sim.N, 0.0);
        for (int i = 0; i < sim.N; ++i) {
            if (!row_mask[i]) continue;
            for (int k = nb_off[i]; k < nb_off[i + 1]; ++k) {
                const int j = nb[k];
                if (!col_mask[j]) continue;
                for (int c = 0; c < 3; ++c)
                    for (int cp = 0; cp < 3; ++cp) y[3 * i + c] += blocks[9 * k + 3 * c + cp] * x[3 * j + cp];
            }
        }
    }

    int cg(const std::vector<double>& b, std::vector<double>& x, const std::vector<uint8_t>& mask, int maxit,
           double tol) const {
        x.assign(3 * sim.N, 0.0);
        std::vector<double> r = b, p, Ap;
        for (int i = 0; i < sim.N; ++i)
            if (!mask[i]) r[3 * i] = r[3 * i + 1] = r[3 * i + 2] = 0.0;
        p = r;
        double rr = 0.0, bb = 0.0;
        for (double v : r) rr += v * v;
        bb = rr;
        if (bb == 0.0) return 0;
        int it = 0;
        for (; it < maxit && rr > tol * tol * bb; ++it) {
            matvec(p, Ap, mask, mask);
            double pAp = 0.0;
            for (size_t k = 0; k < p.size(); ++k) pAp += p[k] * Ap[k];
            const double alpha = rr / pAp;
            for (size_t k = 0; k < p.size(); ++k) {
                x[k] += alpha * p[k];
                r[k] -= alpha * Ap[k];
            }
            double rr2 = 0.0;
            for (double v : r) rr2 += v * v;
            const double beta = rr2 / rr;
            rr = rr2;
            for (size_t k = 0; k < p.size(); ++k) p[k] = r[k] + beta * p[k];
        }
        return it;
    }

    void forward(int steps, double dt, int iters, const double* g, bool accel, double rho) {
        xs.clear();
        vs.clear();
        double gg[3] = {g[0], g[1], g[2]};
        for (int k = 0; k < steps; ++k) {
            xs.push_back(sim.x);
            vs.push_back(sim.v);
            sim.step(dt, 1, iters, gg, accel, rho, nullptr);
        }
        xs.push_back(sim.x);
        vs.push_back(sim.v);
    }

    // Backward through all recorded steps.
    int backward(double dt, const double* dLdx, const double* dLdv, double* gx0, double* gv0, double* gmu, double* glam,
                 double* max_rel_residual) {
        const int N = sim.N;
        const double h = dt, ih2 = 1.0 / (h * h), c = 0.999 / h;
        std::vector<double> ax(dLdx, dLdx + 3 * N), av(3 * N, 0.0);
        if (dLdv) av.assign(dLdv, dLdv + 3 * N);
        std::vector<double> gm(sim.NT, 0.0), gl(sim.NT, 0.0);
        std::vector<uint8_t> freem(N), pinm(N);
        for (int i = 0; i < N; ++i) {
            freem[i] = sim.fixed[i] ? 0 : 1;
            pinm[i] = sim.fixed[i] ? 1 : 0;
        }
        double worst = 0.0;
        int total_it = 0;
        const int steps = (int)xs.size() - 1;
        for (int t = steps - 1; t >= 0; --t) {
            const std::vector<double>& xn = xs[t + 1];
            assemble(xn, ih2);
            std::vector<double> G(3 * N, 0.0), lamv, Ap;
            for (int i = 0; i < N; ++i)
                for (int k = 0; k < 3; ++k) G[3 * i + k] = freem[i] ? ax[3 * i + k] + c * av[3 * i + k] : 0.0;
            total_it += cg(G, lamv, freem, 20000, 1e-13);
            // residual check
            matvec(lamv, Ap, freem, freem);
            double rn = 0.0, gn = 0.0;
            for (int k = 0; k < 3 * N; ++k) {
                rn += (Ap[k] - G[k]) * (Ap[k] - G[k]);
                gn += G[k] * G[k];
            }
            if (gn > 0) worst = std::max(worst, std::sqrt(rn / gn));
            // parameter gradients
            for (int e = 0; e < sim.NT; ++e) {
                const int32_t* q = &sim.tets[4 * e];
                M3<double> F = F_of(xn, e);
                M3<double> C = cofactor(F);
                const double J = det3(F);
                double Q[4][3];
                q_rows(sim.DmInv[e], Q);
                for (int n = 0; n < 4; ++n) {
                    const int vi = q[n];
                    if (!freem[vi]) continue;
                    for (int r = 0; r < 3; ++r) {
                        double fq = 0, cq = 0;
                        for (int k = 0; k < 3; ++k) {
                            fq += (F.m[r][k] - C.m[r][k]) * Q[n][k];
                            cq += C.m[r][k] * Q[n][k];
                        }
                        gm[e] -= lamv[3 * vi + r] * sim.V0[e] * fq;
                        gl[e] -= lamv[3 * vi + r] * sim.V0[e] * (J - 1.0) * cq;
                    }
                }
            }
            // pinned: x~_p = X~_p - (A_pf lam)_p
            std::vector<double> Apf;
            matvec(lamv, Apf, pinm, freem);
            for (int i = 0; i < N; ++i)
                for (int k = 0; k < 3; ++k) {
                    const int d = 3 * i + k;
                    if (freem[i]) {
                        const double yb = sim.mass[i] * ih2 * lamv[d];
                        ax[d] = yb - c * av[d];
                        av[d] = h * yb;
                    } else {
                        ax[d] = ax[d] - Apf[d];
                    }
                }
        }
        for (int k = 0; k < 3 * N; ++k) {
            gx0[k] = ax[k];
            gv0[k] = av[k];
        }
        for (int e = 0; e < sim.NT; ++e) {
            gmu[e] = gm[e];
            glam[e] = gl[e];
        }
        if (max_rel_residual) *max_rel_residual = worst;
        return total_it;
    }
};

template <class T> static void to_T(const double* in, std::vector<T>& out, int n) {
    out.resize(n);
    for (int i = 0; i < n; ++i) out[i] = T(in[i]);
}

template <class T>
static int simulate(int mode, int threads, int N, int NT, const double* rest, const double* x0, const double* v0,
                    const int32_t* tets, const uint8_t* fixed, const double* tmu, const double* tlam, double density,
                    double dt, int substeps, int iters, const double* g, int accel, double rho, int nsteps,
                    double* x_out, double* v_out, double* ip_out, double* ehist_out, int* ncolors_out) {
    std::vector<T> r, x, v;
    to_T(rest, r, 3 * N);
    to_T(x0, x, 3 * N);
    if (v0) to_T(v0, v, 3 * N);
    std::vector<double> rd(r.begin(), r.end()), xd(x.begin(), x.end()), vd(v.begin(), v.end());
    Sim<T> s;
    s.mode = mode;
    s.threads = threads;
    s.setup(N, NT, rd.data(), xd.data(), v0 ? vd.data() : nullptr, tets, fixed, tmu, tlam, density);
    s.color();
    if (ncolors_out) *ncolors_out = (int)s.colors.size();
    T gg[3] = {T(g[0]), T(g[1]), T(g[2])};
    std::vector<double> eh;
    for (int st = 0; st < nsteps; ++st) {
        s.step(T(dt), substeps, iters, gg, accel != 0, T(rho), ehist_out ? &eh : nullptr);
        if (ip_out) ip_out[st] = s.ip_energy(double(T(dt) / T(substeps)));
    }
    for (int i = 0; i < 3 * N; ++i) {
        x_out[i] = double(s.x[i]);
        if (v_out) v_out[i] = double(s.v[i]);
    }
    if (ehist_out)
        for (size_t i = 0; i < eh.size(); ++i) ehist_out[i] = eh[i];
    return 0;
}

}  // namespace orc

extern "C" {

// Greedy colouring; returns the colour count, writes colour_of[N].
int orc_color_vertices(int N, int NT, const int32_t* tets, int32_t* colour_of) {
    orc::Sim<float> s;
    s.N = N;
    s.NT = NT;
    s.tets.assign(tets, tets + 4 * NT);
    std::vector<int32_t> cnt(N + 1, 0);
    for (int t = 0; t < NT; ++t)
        for (int j = 0; j < 4; ++j) cnt[tets[4 * t + j] + 1]++;
    s.adj_off.assign(N + 1, 0);
    for (int i = 0; i < N; ++i) s.adj_off[i + 1] = s.adj_off[i] + cnt[i + 1];
    s.adj.assign(s.adj_off[N], 0);
    std::vector<int32_t> fill(s.adj_off.begin(), s.adj_off.end() - 1);
    for (int t = 0; t < NT; ++t)
        for (int j = 0; j < 4; ++j) s.adj[fill[tets[4 * t + j]]++] = t;
    s.color();
    for (size_t c = 0; c < s.colors.size(); ++c)
        for (int vtx : s.colors[c]) colour_of[vtx] = (int32_t)c;
    return (int)s.colors.size();
}

// Mass (TetMesh::initialize), Dm^-1 row-major and V0 (precomputeTetData); precision 32 or 64.
void orc_mesh_setup(int precision, int N, int NT, const double* rest, const int32_t* tets, double density,
                    double* mass, double* tet_rest_vol, double* dminv, double* v0) {
    std::vector<double> zero(3 * N, 0.0);
    std::vector<uint8_t> fx(N, 0);
    std::vector<double> one(NT, 1.0);
    auto run = [&](auto s) {
        using T = typename std::remove_reference_t<decltype(s.mass)>::value_type;
        std::vector<T> r;
        orc::to_T(rest, r, 3 * N);
        std::vector<double> rd(r.begin(), r.end());
        s.setup(N, NT, rd.data(), rd.data(), nullptr, tets, fx.data(), one.data(), one.data(), density);
        for (int i = 0; i < N; ++i) mass[i] = double(s.mass[i]);
        for (int t = 0; t < NT; ++t) {
            tet_rest_vol[t] = double(s.tetRestVol[t]);
            v0[t] = double(s.V0[t]);
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) dminv[9 * t + 3 * a + b] = double(s.DmInv[t].m[a][b]);
        }
    };
    if (precision == 64)
        run(orc::Sim<double>());
    else
        run(orc::Sim<float>());
}

// Runs nsteps of VBDsolver::step.  mode: 0 literal block, 1 literal full 12x12, 2 closed form,
// 3 the GPU wrapper's semantics (corotated element; each substep as main.cpp's GPU loop runs it).
// ip_out[nsteps] (nullable): incremental potential after each step; ehist_out (nullable):
// computeTotalEnergy every 10 iterations, nsteps*substeps*ceil(iters/10) values.
int orc_simulate(int precision, int mode, int threads, int N, int NT, const double* rest, const double* x0,
                 const double* v0, const int32_t* tets, const uint8_t* fixed, const double* tet_mu,
                 const double* tet_lambda, double density, double dt, int substeps, int iters, const double* gravity,
                 int use_accel, double rho, int nsteps, double* x_out, double* v_out, double* ip_out,
                 double* ehist_out, int* ncolors_out) {
    if (precision == 64)
        return orc::simulate<double>(mode, threads, N, NT, rest, x0, v0, tets, fixed, tet_mu, tet_lambda, density,
                                     dt, substeps, iters, gravity, use_accel, rho, nsteps, x_out, v_out, ip_out,
                                     ehist_out, ncolors_out);
    return orc::simulate<float>(mode, threads, N, NT, rest, x0, v0, tets, fixed, tet_mu, tet_lambda, density, dt,
                                substeps, iters, gravity, use_accel, rho, nsteps, x_out, v_out, ip_out, ehist_out,
                                ncolors_out);
}

// The solve loop alone (VBD_GPU_Solver::solveVBD semantics, VBD_GPU_Wrapper.cu:332-362, with the
// CPU path's Neo-Hookean element): positions x0, inertia y0, `iters` sweeps from x0
// (init_from_inertia = 0) or from y0 (1).  Writes the final positions.
int orc_solve(int precision, int mode, int threads, int N, int NT, const double* rest, const double* x0,
              const double* y0, const int32_t* tets, const uint8_t* fixed, const double* tet_mu,
              const double* tet_lambda, double density, double dt_sqr_reciprocal, int iters, int use_accel,
              double rho, int init_from_inertia, double* x_out) {
    auto run = [&](auto zero) {
        using T = decltype(zero);
        std::vector<T> r, x, y;
        orc::to_T(rest, r, 3 * N);
        orc::to_T(x0, x, 3 * N);
        orc::to_T(y0, y, 3 * N);
        std::vector<double> rd(r.begin(), r.end()), xd(x.begin(), x.end());
        orc::Sim<T> s;
        s.mode = mode;
        s.threads = threads;
        s.setup(N, NT, rd.data(), xd.data(), nullptr, tets, fixed, tet_mu, tet_lambda, density);
        s.color();
        s.y = y;
        if (init_from_inertia) s.x = y;
        s.solve_loop(T(dt_sqr_reciprocal), iters, use_accel != 0, T(rho), nullptr);
        for (int i = 0; i < 3 * N; ++i) x_out[i] = double(s.x[i]);
    };
    if (precision == 64)
        run(double(0));
    else
        run(float(0));
    return 0;
}

// Residual norm of a state (double): || m_i/h^2 (x_i - y_i) + dE/dx_i || over free vertices.
double orc_residual(int N, int NT, const double* rest, const double* x, const double* y, const int32_t* tets,
                    const uint8_t* fixed, const double* tet_mu, const double* tet_lambda, double density,
                    double dt_sqr_reciprocal) {
    orc::Sim<double> s;
    s.setup(N, NT, rest, x, nullptr, tets, fixed, tet_mu, tet_lambda, density);
    s.y.assign(y, y + 3 * N);
    return s.residual_norm(dt_sqr_reciprocal);
}

// One element's block for vertex n: literal (mode 0/1) or closed form (mode 2).
void orc_tet_block(int precision, int mode, const double* F9, const double* dminv9, double mu, double lambda,
                   double vol, int n, double* H9, double* g3) {
    auto run = [&](auto zero) {
        using T = decltype(zero);
        orc::M3<T> F, D;
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) {
                F.m[a][b] = T(F9[3 * a + b]);
                D.m[a][b] = T(dminv9[3 * a + b]);
            }
        T H[3][3], g[3];
        if (mode == orc::WRAPPER) {
            T Hf[9];
            orc::corot_block(D, F, T(mu), T(lambda), T(vol), n, Hf, g);
            for (int k = 0; k < 9; ++k) H[k / 3][k % 3] = Hf[k];
        } else if (mode == orc::CLOSED)
            orc::tet_block_closed(D, F, T(lambda), T(mu), T(vol), n, H, g);
        else
            orc::tet_block_literal(D, F, T(lambda), T(mu), T(vol), n, H, g, mode == orc::LITERAL_FULL12);
        for (int a = 0; a < 3; ++a) {
            g3[a] = double(g[a]);
            for (int b = 0; b < 3; ++b) H9[3 * a + b] = double(H[a][b]);
        }
    };
    if (precision == 64)
        run(double(0));
    else
        run(float(0));
}

// Incremental potential (double) of a state given y, masses and per-tet data (row-major Dm^-1).
double orc_ip_energy(int N, int NT, const double* x, const double* y, const double* mass, const int32_t* tets,
                     const double* dminv, const double* v0, const double* tet_mu, const double* tet_lambda,
                     double h) {
    orc::Sim<double> s;
    s.N = N;
    s.NT = NT;
    s.x.assign(x, x + 3 * N);
    s.y.assign(y, y + 3 * N);
    s.mass.assign(mass, mass + N);
    s.tets.assign(tets, tets + 4 * NT);
    s.V0.assign(v0, v0 + NT);
    s.mu.assign(tet_mu, tet_mu + NT);
    s.lam.assign(tet_lambda, tet_lambda + NT);
    s.DmInv.resize(NT);
    for (int t = 0; t < NT; ++t)
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b < 3; ++b) s.DmInv[t].m[a][b] = dminv[9 * t + 3 * a + b];
    return s.ip_energy(h);
}

// Persistent FP32 simulation handle for timing the CPU baseline without its one-off set-up.
void* orc_handle_create(int mode, int threads, int N, int NT, const double* rest, const double* x0, const double* v0,
                        const int32_t* tets, const uint8_t* fixed, const double* tet_mu, const double* tet_lambda,
                        double density) {
    auto* s = new orc::Sim<float>();
    s->mode = mode;
    s->threads = threads;
    std::vector<float> r, x, v;
    orc::to_T(rest, r, 3 * N);
    orc::to_T(x0, x, 3 * N);
    orc::to_T(v0, v, 3 * N);
    std::vector<double> rd(r.begin(), r.end()), xd(x.begin(), x.end()), vd(v.begin(), v.end());
    s->setup(N, NT, rd.data(), xd.data(), vd.data(), tets, fixed, tet_mu, tet_lambda, density);
    s->color();
    return s;
}

// `steps` calls of VBDsolver::step; with_energy evaluates computeTotalEnergy every 10 iterations.
void orc_handle_step(void* h, int steps, double dt, int substeps, int iters, const double* g, int use_accel, double rho,
                     int with_energy) {
    auto* s = static_cast<orc::Sim<float>*>(h);
    float gg[3] = {float(g[0]), float(g[1]), float(g[2])};
    std::vector<double> eh;
    for (int k = 0; k < steps; ++k)
        s->step(float(dt), substeps, iters, gg, use_accel != 0, float(rho), with_energy ? &eh : nullptr);
}

void orc_handle_positions(void* h, double* x_out) {
    auto* s = static_cast<orc::Sim<float>*>(h);
    for (int i = 0; i < 3 * s->N; ++i) x_out[i] = double(s->x[i]);
}

void orc_handle_destroy(void* h) { delete static_cast<orc::Sim<float>*>(h); }

// FP64 forward of `steps` steps (substeps 1) from (x0, v0) and the implicit adjoint of the final-state
// loss gradient (dLdx, dLdv nullable): writes final positions, dL/dx0, dL/dv0, dL/dmu, dL/dlambda.
int orc_adjoint_f64(int N, int NT, const double* rest, const double* x0, const double* v0, const int32_t* tets,
                    const uint8_t* fixed, const double* tet_mu, const double* tet_lambda, double density, double dt,
                    int iters, const double* g, int use_accel, double rho, int steps, const double* dLdx,
                    const double* dLdv, double* x_final, double* gx0, double* gv0, double* gmu, double* glam,
                    double* max_rel_residual) {
    orc::AdjointF64 a;
    a.sim.mode = orc::CLOSED;
#ifdef _OPENMP
    a.sim.threads = omp_get_max_threads();
#endif
    a.sim.setup(N, NT, rest, x0, v0, tets, fixed, tet_mu, tet_lambda, density);
    a.sim.color();
    a.build_pattern();
    a.forward(steps, dt, iters, g, use_accel != 0, rho);
    for (int k = 0; k < 3 * N; ++k) x_final[k] = a.sim.x[k];
    if (!dLdx) return 0;
    return a.backward(dt, dLdx, dLdv, gx0, gv0, gmu, glam, max_rel_residual);
}

int orc_num_threads_max(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
}
