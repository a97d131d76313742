// Loads a TetGen mesh with include/vbd/TetGenIO.h (this project's loader) and dumps the TetMesh in
// the format of oracle/ref_tetgen_harness.cpp, for tests/test_tetgen.py.
// Usage: test_tetgen <rest.node> <current.node or ""> <mesh.ele> <density> <mu> <lambda> <out.bin> [mesh.obj]
#include <cstdio>
#include <cstdlib>

#include "TetGenIO.h"

int main(int argc, char** argv) {
    if (argc < 8) {
        std::fprintf(stderr, "usage: test_tetgen rest.node current.node mesh.ele density mu lambda out.bin\n");
        return 2;
    }
    VBD::TetMesh mesh;
    if (!VBD::loadTetgenModel(argv[1], argv[2], argv[3], mesh, (Real)std::atof(argv[4]), (Real)std::atof(argv[5]),
                              (Real)std::atof(argv[6])))
        return 3;
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
