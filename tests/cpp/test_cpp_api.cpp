// Exercises the C++ drop-in surface (include/vbd/*.h) the way the reference's callers do:
//   flow 1: VBDsolver::step(mesh) (VBD.cpp:60-101), all on the GPU;
//   flow 2: the reference driver's GPU loop (main.cpp:215-232): host forwardStep,
//           VBD_GPU_Solver::updateInertiaFromCPU / solveVBD / copyPositionsToCPU, host updateVelocity;
//   flow 3: VBDsolver::step with VBDParams::usePerTetMaterials: tet t starts with
//           mu (1 + t%5 / 8), lambda (1 + t%3 / 4), and after steps / 2 steps mu of every even tet is
//           multiplied by 1.5 (the solver must pick the change up).
// Usage: test_cpp_api <input.bin> <output.bin> <obj path>
// input:  int32 N, T, iterations, steps; float32 density, mu, lambda, dt, rho; rest[3N] f32,
//         tets[4T] i32, fixed[N] u8
// output: flow-1 positions[3N], velocities[3N], flow-2 positions[3N] (f32), flow-1 energy (f32),
//         number of surface triangles (int32), colour count (int32), flow-3 positions[3N] (f32)
#include <cstdio>
#include <fstream>
#include <iostream>
#include <vector>

#include "VBD.h"
#include "VBD_GPU_Wrapper.h"

using namespace VBD;

template <class T> static void rd(std::ifstream& in, T* p, size_t n) { in.read(reinterpret_cast<char*>(p), sizeof(T) * n); }
template <class T> static void wr(std::ofstream& out, const T* p, size_t n) {
    out.write(reinterpret_cast<const char*>(p), sizeof(T) * n);
}

int main(int argc, char** argv) {
    if (argc < 4) {
        std::cerr << "usage: test_cpp_api <input.bin> <output.bin> <obj path>\n";
        return 2;
    }
    std::ifstream in(argv[1], std::ios::binary);
    int32_t hdr[4];
    float prm[5];
    rd(in, hdr, 4);
    rd(in, prm, 5);
    const int N = hdr[0], T = hdr[1], iters = hdr[2], steps = hdr[3];
    const float density = prm[0], mu = prm[1], lambda = prm[2], dt = prm[3], rho = prm[4];
    std::vector<float> rest(3 * (size_t)N);
    std::vector<int32_t> tv(4 * (size_t)T);
    std::vector<uint8_t> fx(N);
    rd(in, rest.data(), rest.size());
    rd(in, tv.data(), tv.size());
    rd(in, fx.data(), fx.size());

    std::vector<Vec3> pos(N);
    for (int i = 0; i < N; ++i) pos[i] = Vec3(rest[3 * i], rest[3 * i + 1], rest[3 * i + 2]);
    std::vector<TetVIdsArr> tets(T);
    for (int t = 0; t < T; ++t)
        for (int a = 0; a < 4; ++a) tets[t][a] = tv[4 * t + a];
    std::vector<IdType> fixedList;
    for (int i = 0; i < N; ++i)
        if (fx[i]) fixedList.push_back(i);

    VBDParams params;
    params.dt = dt;
    params.numIterations = iters;
    params.substeps = 1;
    params.gravity << 0.0f, -9.8f, 0.0f;
    params.useAcceleration = true;
    params.accelerationRho = rho;
    params.mu = mu;
    params.lambda = lambda;
    params.density = density;

    // flow 1
    TetMesh mesh;
    mesh.initialize(pos, pos, density, tets, mu, lambda, fixedList);
    VBDsolver solver;
    solver.setParams(params);
    for (int s = 0; s < steps; ++s) solver.step(mesh);
    const float energy = solver.computeTotalEnergy(mesh);
    const int ncol = (int)solver.getVertexColors().size();

    // flow 2
    TetMesh mesh2;
    mesh2.initialize(pos, pos, density, tets, mu, lambda, fixedList);
    VBDsolver cpu;
    cpu.setParams(params);
    cpu.initializeColoring(mesh2);
    cpu.precomputeTetData(mesh2);
    VBD_GPU_Solver gpu;
    gpu.initFromCPU(mesh2, cpu.getVertexColors(), cpu.getTetDmInv(), cpu.getTetRestVol());
    const Real subDt = params.dt / params.substeps;
    const Real dtSqrReciprocal = 1.0f / (subDt * subDt);
    for (int s = 0; s < steps; ++s) {
        cpu.forwardStep(mesh2);
        gpu.updateInertiaFromCPU(mesh2);
        gpu.solveVBD(params.numIterations, dtSqrReciprocal, params.mu, params.lambda, params.useAcceleration,
                     params.accelerationRho);
        gpu.copyPositionsToCPU(mesh2);
        mesh2.updateVelocity(subDt);
    }

    // flow 3
    TetMesh mesh3;
    mesh3.initialize(pos, pos, density, tets, mu, lambda, fixedList);
    for (int t = 0; t < T; ++t) {
        mesh3.tetMu[t] = mu * (1.0f + 0.125f * (float)(t % 5));
        mesh3.tetLambda[t] = lambda * (1.0f + 0.25f * (float)(t % 3));
    }
    VBDParams p3 = params;
    p3.usePerTetMaterials = true;
    VBDsolver solver3;
    solver3.setParams(p3);
    for (int s = 0; s < steps; ++s) {
        if (s == steps / 2)
            for (int t = 0; t < T; t += 2) mesh3.tetMu[t] *= 1.5f;
        solver3.step(mesh3);
    }

    const bool objOk = mesh.exportToObj(argv[3]);
    const int32_t nsurf = (int32_t)mesh.extractSurfaceFaces().size();
    std::ofstream out(argv[2], std::ios::binary);
    wr(out, mesh.mVertPos.data(), 3 * (size_t)N);
    wr(out, mesh.mVelocity.data(), 3 * (size_t)N);
    wr(out, mesh2.mVertPos.data(), 3 * (size_t)N);
    wr(out, &energy, 1);
    wr(out, &nsurf, 1);
    const int32_t nc = ncol;
    wr(out, &nc, 1);
    wr(out, mesh3.mVertPos.data(), 3 * (size_t)N);
    return objOk ? 0 : 1;
}
