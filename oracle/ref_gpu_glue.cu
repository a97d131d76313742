// Drives the reference's own GPU path (VBD::VBD_GPU_Solver, VBD_GPU_Wrapper.cu) through its public
// C++ API -- TEST INFRASTRUCTURE ONLY.
//
// Built by `make -C oracle refgpu` into oracle/_ref/libvbdref_gpu.so from the reference's
// VBD_GPU_Wrapper.cu (+ VBD_DeviceMath.cuh) and its CPU sources, compiled unchanged against this
// project's Eigen-API subset.  It runs the reference's kernels (vbd_solve_color_kernel, 16 threads
// per vertex; vbd_apply_chebyshev_kernel) on the GPU for two purposes only:
//   * pinning the wrapper-semantics restatement (oracle mode 3) and the GPU wrapper mode against
//     the reference's own outputs (tests/test_gpu_wrapper_mode.py), and
//   * timing the reference's GPU kernels beside this project's on the same B200 (bench.py).
// Nothing here restates the algorithm: every step calls a reference member function.  Read for
// safety before use: fixed-size launches (one 16-thread block per vertex of a colour, shared
// arrays sized for 32 threads), in-bounds CSR reads for a valid mesh, no waits.
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "GraphColoring.h"
#include "TetMesh.h"
#include "VBD.h"
#include "VBD_GPU_Wrapper.h"

using namespace VBD;

namespace {

struct RefGpu {
    TetMesh mesh;
    VBDsolver cpu;
    VBD_GPU_Solver gpu;
    VBDParams params;
};

int last_cuda() { return cudaGetLastError() == cudaSuccess ? 0 : 1; }

}  // namespace

extern "C" {

// TetMesh::initialize, VBDsolver colouring / precompute, VBD_GPU_Solver::initFromCPU (main.cpp:200-208).
void* refgpu_create(int N, int T, const float* rest, const float* x0, const int32_t* tets, const uint8_t* fixed,
                    float density, float mu, float lambda, float dt, int substeps, int iters, const float* g,
                    int use_accel, float rho) {
    auto* r = new RefGpu();
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
    VBDParams p;
    p.dt = dt;
    p.numIterations = iters;
    p.substeps = substeps;
    p.gravity = Vec3(g[0], g[1], g[2]);
    p.useAcceleration = use_accel != 0;
    p.accelerationRho = rho;
    p.numThreads = 1;
    p.mu = mu;
    p.lambda = lambda;
    p.density = density;
    r->params = p;
    r->cpu.setParams(p);
    r->cpu.initializeColoring(r->mesh);
    r->cpu.precomputeTetData(r->mesh);
    r->gpu.initFromCPU(r->mesh, r->cpu.getVertexColors(), r->cpu.getTetDmInv(), r->cpu.getTetRestVol());
    if (cudaDeviceSynchronize() != cudaSuccess) {
        delete r;
        return nullptr;
    }
    return r;
}

// mesh.mInertia = y, then VBD_GPU_Solver::updateInertiaFromCPU.
int refgpu_set_inertia(void* h, const float* y) {
    auto* r = static_cast<RefGpu*>(h);
    for (size_t i = 0; i < r->mesh.numVerts; ++i)
        r->mesh.mInertia.col((Eigen::Index)i) = Vec3(y[3 * i], y[3 * i + 1], y[3 * i + 2]);
    r->gpu.updateInertiaFromCPU(r->mesh);
    return last_cuda();
}

// VBD_GPU_Solver::solveVBD bracketed by CUDA events on the legacy default stream (the stream the
// reference launches on); *ms receives the elapsed device time.
int refgpu_solve(void* h, int iters, float dtsr, float mu, float lambda, int use_accel, float rho, float* ms) {
    auto* r = static_cast<RefGpu*>(h);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, 0);
    r->gpu.solveVBD(iters, dtsr, mu, lambda, use_accel != 0, rho);
    cudaEventRecord(e1, 0);
    cudaEventSynchronize(e1);
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    if (ms) *ms = t;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return last_cuda();
}

// One frame of main.cpp's GPU loop (main.cpp:214-229): per substep forwardStep on the CPU,
// updateInertiaFromCPU, solveVBD, copyPositionsToCPU, updateVelocity.
int refgpu_frame(void* h, float mu, float lambda) {
    auto* r = static_cast<RefGpu*>(h);
    const VBDParams& p = r->params;
    const Real subDt = p.dt / p.substeps;
    const Real dtsr = 1.0f / (subDt * subDt);
    for (int s = 0; s < p.substeps; ++s) {
        r->cpu.forwardStep(r->mesh);
        r->gpu.updateInertiaFromCPU(r->mesh);
        r->gpu.solveVBD(p.numIterations, dtsr, mu, lambda, p.useAcceleration, p.accelerationRho);
        r->gpu.copyPositionsToCPU(r->mesh);
        r->mesh.updateVelocity(subDt);
    }
    return last_cuda();
}

// Positions after VBD_GPU_Solver::copyPositionsToCPU, xyz-interleaved.
int refgpu_positions(void* h, float* out) {
    auto* r = static_cast<RefGpu*>(h);
    r->gpu.copyPositionsToCPU(r->mesh);
    for (size_t i = 0; i < r->mesh.numVerts; ++i)
        for (int c = 0; c < 3; ++c) out[3 * i + c] = r->mesh.mVertPos(c, (Eigen::Index)i);
    return last_cuda();
}

// Velocities of the host mesh (after refgpu_frame), xyz-interleaved.
void refgpu_velocities(void* h, float* out) {
    auto* r = static_cast<RefGpu*>(h);
    for (size_t i = 0; i < r->mesh.numVerts; ++i)
        for (int c = 0; c < 3; ++c) out[3 * i + c] = r->mesh.mVelocity(c, (Eigen::Index)i);
}

void refgpu_destroy(void* h) { delete static_cast<RefGpu*>(h); }

}  // extern "C"
