// Drives VBDsolver::simulate (VBD.cpp:313-330) through the C++ drop-in surface (include/vbd/VBD.h)
// with a per-frame callback, as a caller of the reference would, and writes what a caller sees:
// the final state, what the callback observed, and energyHistory.
// Usage: test_simulate <input.bin> <output.bin> [resident]   (resident: VBDParams::deviceResident)
// input:  int32 N, T, iterations, frames, substeps, use_acceleration; float32 density, mu, lambda,
//         dt, rho; rest[3N] f32, x0[3N] f32, v0[3N] f32, tets[4T] i32, fixed[N] u8
// output: positions[3N], velocities[3N] (f32); int32 callbacks, int32 frames_in_order,
//         int32 positions_match (every callback saw the mesh the frame's step left);
//         int32 history length; float32 energyHistory[...]
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "VBD.h"

using namespace VBD;

template <class T> static void rd(std::ifstream& in, T* p, size_t n) { in.read(reinterpret_cast<char*>(p), sizeof(T) * n); }
template <class T> static void wr(std::ofstream& out, const T* p, size_t n) {
    out.write(reinterpret_cast<const char*>(p), sizeof(T) * n);
}

int main(int argc, char** argv) {
    if (argc < 3) {
        std::cerr << "usage: test_simulate <input.bin> <output.bin>\n";
        return 2;
    }
    std::ifstream in(argv[1], std::ios::binary);
    int32_t hdr[6];
    float prm[5];
    rd(in, hdr, 6);
    rd(in, prm, 5);
    const int N = hdr[0], T = hdr[1], iters = hdr[2], frames = hdr[3], substeps = hdr[4], accel = hdr[5];
    std::vector<float> rest(3 * (size_t)N), x0(3 * (size_t)N), v0(3 * (size_t)N);
    std::vector<int32_t> tv(4 * (size_t)T);
    std::vector<uint8_t> fx(N);
    rd(in, rest.data(), rest.size());
    rd(in, x0.data(), x0.size());
    rd(in, v0.data(), v0.size());
    rd(in, tv.data(), tv.size());
    rd(in, fx.data(), fx.size());

    std::vector<Vec3> rp(N), cp(N);
    for (int i = 0; i < N; ++i) {
        rp[i] = Vec3(rest[3 * i], rest[3 * i + 1], rest[3 * i + 2]);
        cp[i] = Vec3(x0[3 * i], x0[3 * i + 1], x0[3 * i + 2]);
    }
    std::vector<TetVIdsArr> tets(T);
    for (int t = 0; t < T; ++t)
        for (int a = 0; a < 4; ++a) tets[t][a] = tv[4 * t + a];
    std::vector<IdType> fixedList;
    for (int i = 0; i < N; ++i)
        if (fx[i]) fixedList.push_back(i);

    TetMesh mesh;
    mesh.initialize(rp, cp, prm[0], tets, prm[1], prm[2], fixedList);
    for (int i = 0; i < N; ++i) mesh.mVelocity.col(i) = Vec3(v0[3 * i], v0[3 * i + 1], v0[3 * i + 2]);

    VBDParams params;
    params.dt = prm[3];
    params.numIterations = iters;
    params.substeps = substeps;
    params.gravity << 0.0f, -9.8f, 0.0f;
    params.useAcceleration = accel != 0;
    params.accelerationRho = prm[4];
    params.mu = prm[1];
    params.lambda = prm[2];
    params.density = prm[0];
    params.deviceResident = argc > 3 && std::string(argv[3]) == "resident";

    VBDsolver solver;
    solver.setParams(params);
    // energyHistory is cleared by simulate: a stale entry must not survive
    solver.energyHistory.push_back(-1.0f);
    int32_t callbacks = 0, inOrder = 1, positionsMatch = 1;
    TVerticesMat last;
    solver.simulate(mesh, frames, [&](int frame, TetMesh& m) {
        if (frame != callbacks) inOrder = 0;
        ++callbacks;
        // the callback sees the positions the frame's step produced: the next frame starts from them
        if (callbacks > 1 && last.cols() == m.mVertPos.cols()) {
            bool moved = false;
            for (Eigen::Index k = 0; k < m.mVertPos.cols() && !moved; ++k)
                for (int c = 0; c < 3; ++c)
                    if (m.mVertPos(c, k) != last(c, k)) moved = true;
            if (!moved && frames > 1) positionsMatch = 0;
        }
        last = m.mVertPos;
    });
    // the mesh after simulate is the mesh the last callback saw
    for (Eigen::Index k = 0; k < mesh.mVertPos.cols(); ++k)
        for (int c = 0; c < 3; ++c)
            if (mesh.mVertPos(c, k) != last(c, k)) positionsMatch = 0;

    std::ofstream out(argv[2], std::ios::binary);
    wr(out, mesh.mVertPos.data(), 3 * (size_t)N);
    wr(out, mesh.mVelocity.data(), 3 * (size_t)N);
    wr(out, &callbacks, 1);
    wr(out, &inOrder, 1);
    wr(out, &positionsMatch, 1);
    const int32_t nh = (int32_t)solver.energyHistory.size();
    wr(out, &nh, 1);
    wr(out, solver.energyHistory.data(), solver.energyHistory.size());
    return 0;
}
