// Drives the reference's own VBD sources through their public C++ API -- TEST INFRASTRUCTURE ONLY.
//
// Built by `make -C oracle ref` into oracle/_ref/libvbdref.so from the reference's TetMesh.h,
// VBD.cpp, Energy.cpp, GraphColoring.cpp and NeoHookean.cpp, compiled unchanged against this
// project's Eigen-API subset (include/vbd/eigen_lite.h; the reference's own dependency, Eigen 3,
// is absent from this image).  Used for two things only:
//   * pinning the oracle restatement (tests/test_oracle_pin.py and the fixtures it checks), and
//   * the CPU baseline of bench.py (the reference's own code timed on the host cores).
// Nothing here restates the algorithm: every step calls a reference member function.
#include <cstdint>
#include <vector>

#include "GraphColoring.h"
#include "TetMesh.h"
#include "VBD.h"

using namespace VBD;

namespace {

struct RefSim {
    TetMesh mesh;
    VBDsolver solver;
    int iter_in_step = 0;  // position inside the step's iteration loop (for ref_iterations)
    Real omega = 1.0f;
};

}  // namespace

extern "C" {

// TetMesh::initialize + VBDsolver::setParams / initializeColoring / precomputeTetData.
void* ref_create(int N, int T, const float* rest, const float* x0, const float* v0, const int32_t* tets,
                 const uint8_t* fixed, float density, float mu, float lambda, float dt, int substeps, int iters,
                 const float* g, int use_accel, float rho, int threads) {
    auto* r = new RefSim();
    std::vector<Vec3> rp(N), cp(N);
    for (int i = 0; i < N; ++i) {
        rp[i] = Vec3(rest[3 * i], rest[3 * i + 1], rest[3 * i + 2]);
        cp[i] = Vec3(x0[3 * i], x0[3 * i + 1], x0[3 * i + 2]);
    }
    std::vector<TetVIdsArr> tv(T);
    for (int t = 0; t < T; ++t)
        for (int a = 0; a < 4; ++a) tv[t][a] = tets[4 * t + a];
    std::vector<IdType> fx;
    for (int i = 0; i < N; ++i)
        if (fixed[i]) fx.push_back(i);
    r->mesh.initialize(rp, cp, density, tv, mu, lambda, fx);
    if (v0)
        for (int i = 0; i < N; ++i) r->mesh.mVelocity.col(i) = Vec3(v0[3 * i], v0[3 * i + 1], v0[3 * i + 2]);
    VBDParams p;
    p.dt = dt;
    p.numIterations = iters;
    p.substeps = substeps;
    p.gravity = Vec3(g[0], g[1], g[2]);
    p.useAcceleration = use_accel != 0;
    p.accelerationRho = rho;
    p.numThreads = threads;
    p.mu = mu;
    p.lambda = lambda;
    p.density = density;
    r->solver.setParams(p);
    r->solver.initializeColoring(r->mesh);
    r->solver.precomputeTetData(r->mesh);
    return r;
}

// `steps` calls of VBDsolver::step.
void ref_step(void* h, int steps) {
    auto* r = static_cast<RefSim*>(h);
    for (int k = 0; k < steps; ++k) r->solver.step(r->mesh);
}

// `n` iterations of VBDsolver::step's loop, one at a time, through the solver's public members
// (forwardStep, solve, getAcceleratorOmega, applyAcceleration, computeTotalEnergy,
// TetMesh::updateVelocity), in the order VBD.cpp:70-100 calls them; a step's predictor runs
// before its first iteration and its velocity update after its last.  Used to time bounded
// samples of a step.
void ref_iterations(void* h, int n) {
    auto* r = static_cast<RefSim*>(h);
    VBDsolver& s = r->solver;
    const VBDParams& p = s.params;
    const Real subDt = p.dt / p.substeps;
    for (int k = 0; k < n; ++k) {
        const int it = r->iter_in_step;
        if (it == 0) {
            s.forwardStep(r->mesh);
            r->omega = 1.0;
        }
        TVerticesMat currentPos = r->mesh.mVertPos;
        s.solve(r->mesh);
        if (p.useAcceleration) {
            r->omega = s.getAcceleratorOmega(it + 1, p.accelerationRho, r->omega);
            if (r->omega > 1.0) s.applyAcceleration(r->mesh, r->omega);
            s.prevPrevPos = currentPos;
        }
        if (it % 10 == 0) s.energyHistory.push_back(s.computeTotalEnergy(r->mesh));
        r->iter_in_step = it + 1;
        if (r->iter_in_step == p.numIterations) {
            r->mesh.updateVelocity(subDt);
            r->iter_in_step = 0;
        }
    }
}

void ref_state(void* h, float* x, float* v) {
    auto* r = static_cast<RefSim*>(h);
    const int N = (int)r->mesh.numVerts;
    for (int i = 0; i < 3 * N; ++i) {
        if (x) x[i] = r->mesh.mVertPos.data()[i];
        if (v) v[i] = r->mesh.mVelocity.data()[i];
    }
}

// Set-up products: colour of each vertex, lumped mass, TetMesh::tetRestVol, Dm^-1 (row-major),
// VBDsolver::tetRestVolume.  Any pointer may be null.
int ref_setup(void* h, int32_t* colour_of, float* mass, float* tet_rest_vol, float* dminv, float* v0) {
    auto* r = static_cast<RefSim*>(h);
    const auto& groups = r->solver.getVertexColors();
    if (colour_of)
        for (size_t c = 0; c < groups.size(); ++c)
            for (IdType vtx : groups[c]) colour_of[vtx] = (int32_t)c;
    const int N = (int)r->mesh.numVerts, T = (int)r->mesh.numTets;
    if (mass)
        for (int i = 0; i < N; ++i) mass[i] = r->mesh.vertexMass(i);
    if (tet_rest_vol)
        for (int t = 0; t < T; ++t) tet_rest_vol[t] = r->mesh.tetRestVol[t];
    const auto& dm = r->solver.getTetDmInv();
    if (dminv)
        for (int t = 0; t < T; ++t)
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) dminv[9 * t + 3 * a + b] = dm[t](a, b);
    if (v0)
        for (int t = 0; t < T; ++t) v0[t] = r->solver.getTetRestVol()[t];
    return (int)groups.size();
}

// VBDsolver::energyHistory (computeTotalEnergy every 10 iterations); returns its length.
int ref_energy_history(void* h, double* out, int cap) {
    auto* r = static_cast<RefSim*>(h);
    const auto& e = r->solver.energyHistory;
    for (int i = 0; i < (int)e.size() && i < cap; ++i) out[i] = e[i];
    return (int)e.size();
}

void ref_destroy(void* h) { delete static_cast<RefSim*>(h); }
}
