// Runs the reference driver's own TetGen loader (loadTetgenModel / readNodeFile, main.cpp:14-168)
// on given files and dumps the resulting TetMesh -- TEST INFRASTRUCTURE ONLY.
//
// Built by `make -C oracle reftetgen` into oracle/_ref/ref_tetgen from the reference's main.cpp
// (its main() renamed by the preprocessor and never called) with its CPU sources, against this
// project's Eigen-API subset.  The GPU wrapper members main.cpp's driver references are defined
// here as empty stubs: the loader does not use them and nothing calls them.
//
// Usage: ref_tetgen <rest.node> <current.node or ""> <mesh.ele> <density> <mu> <lambda> <out.bin> [mesh.obj]
// out.bin: int32 N, T; float32 rest[3N], current[3N]; int32 tets[4T]; uint8 fixed[N]; float32 mass[N]
#define main reference_driver_main
#include "main.cpp"
#undef main

#include <cstdio>
#include <cstdlib>

namespace VBD {
void VBD_GPU_Solver::initFromCPU(const TetMesh&, const std::vector<std::vector<int>>&, const std::vector<Matrix3r>&,
                                 const std::vector<Real>&) {}
void VBD_GPU_Solver::solveIteration(Real, Real, Real) {}
void VBD_GPU_Solver::copyPositionsToCPU(TetMesh&) {}
void VBD_GPU_Solver::updateInertiaFromCPU(const TetMesh&) {}
void VBD_GPU_Solver::solveVBD(int, Real, Real, Real, bool, Real) {}
VBD_GPU_Solver::~VBD_GPU_Solver() {}
}  // namespace VBD

int main(int argc, char** argv) {
    if (argc < 8) {
        std::fprintf(stderr, "usage: ref_tetgen rest.node current.node mesh.ele density mu lambda out.bin\n");
        return 2;
    }
    VBD::TetMesh mesh;
    loadTetgenModel(argv[1], argv[2], argv[3], mesh, (Real)std::atof(argv[4]), (Real)std::atof(argv[5]),
                    (Real)std::atof(argv[6]));
    FILE* f = std::fopen(argv[7], "wb");
    if (!f) return 1;
    const int32_t hdr[2] = {(int32_t)mesh.numVerts, (int32_t)mesh.numTets};
    std::fwrite(hdr, sizeof(int32_t), 2, f);
    std::fwrite(mesh.mRestPos.data(), sizeof(float), 3 * mesh.numVerts, f);
    std::fwrite(mesh.mVertPos.data(), sizeof(float), 3 * mesh.numVerts, f);
    for (size_t t = 0; t < mesh.numTets; ++t)
        for (int a = 0; a < 4; ++a) {
            const int32_t v = mesh.tets[t][a];
            std::fwrite(&v, sizeof(int32_t), 1, f);
        }
    for (size_t i = 0; i < mesh.numVerts; ++i) {
        const uint8_t b = mesh.isFixed[i] ? 1 : 0;
        std::fwrite(&b, 1, 1, f);
    }
    for (size_t i = 0; i < mesh.numVerts; ++i) {
        const float m = mesh.vertexMass((Eigen::Index)i);
        std::fwrite(&m, sizeof(float), 1, f);
    }
    std::fclose(f);
    if (argc > 8) mesh.exportToObj(argv[8]);
    return 0;
}
