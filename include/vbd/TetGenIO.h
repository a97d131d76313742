// TetGenIO.h -- the reference driver's TetGen input (readNodeFile / loadTetgenModel, main.cpp:14-168)
// as library functions over libvbd_b200's host readers (vbd_tetgen_read_node / _ele,
// vbd_pin_low_fraction), so C++ and Python callers read files identically.
//
// Same inputs and rules as main.cpp: a rest .node file, an optional current .node file (missing or
// empty: the rest positions are used), an .ele file; ids 0-based when the first rest node's index
// is 0, else 1-based; vertices within 5% of the extent above the minimum y of the current
// positions pinned (TetgenPinning selects the axes and the fraction).  Unlike main.cpp, failures
// are reported by the return value (false, the mesh untouched) instead of only printed, and blank
// and '#' comment lines are skipped.
#pragma once

#include <iostream>
#include <string>
#include <vector>

#include "TetMesh.h"
#include "Types.h"

namespace VBD {

struct TetgenPinning {
    bool fixX = false;  // main.cpp:127 (off there)
    bool fixY = true;   // main.cpp:128
    bool fixZ = false;
    Real fraction = 0.05f;
};

// Positions of a .node file (empty on failure, with a message on stderr); start_from_0 is set when
// the first node's index is 0 (main.cpp:14-45).
inline std::vector<Vec3> readNodeFile(const std::string& nodeFilename, bool& start_from_0) {
    std::vector<Vec3> positions;
    int32_t n = 0, first = 0;
    if (vbd_tetgen_read_node(nodeFilename.c_str(), &n, nullptr, nullptr, 0) != VBD_OK) {
        std::cerr << vbd_last_error() << std::endl;
        return positions;
    }
    std::vector<float> flat(3 * (size_t)n);
    if (vbd_tetgen_read_node(nodeFilename.c_str(), &n, &first, flat.data(), n) != VBD_OK) {
        std::cerr << vbd_last_error() << std::endl;
        return positions;
    }
    if (n > 0 && first == 0) start_from_0 = true;
    positions.resize((size_t)n);
    for (int32_t i = 0; i < n; ++i) positions[(size_t)i] = Vec3(flat[3 * i], flat[3 * i + 1], flat[3 * i + 2]);
    return positions;
}

// loadTetgenModel of main.cpp:48-168: reads the files, pins, and calls TetMesh::initialize.
inline bool loadTetgenModel(const std::string& restNodeFilename, const std::string& currentNodeFilename,
                            const std::string& eleFilename, TetMesh& mesh, Real density, Real mu, Real lambda,
                            const TetgenPinning& pin = TetgenPinning()) {
    bool start_from_0 = false;
    std::vector<Vec3> rest = readNodeFile(restNodeFilename, start_from_0);
    if (rest.empty()) return false;
    bool unused = false;
    std::vector<Vec3> current;
    if (!currentNodeFilename.empty()) current = readNodeFile(currentNodeFilename, unused);
    if (current.empty()) current = rest;
    if (current.size() != rest.size()) {
        std::cerr << "rest nodes and current nodes count mismatch" << std::endl;
        return false;
    }
    const int32_t n = (int32_t)rest.size();
    int32_t nt = 0;
    if (vbd_tetgen_read_ele(eleFilename.c_str(), start_from_0 ? 0 : 1, n, &nt, nullptr, 0) != VBD_OK) {
        std::cerr << vbd_last_error() << std::endl;
        return false;
    }
    std::vector<int32_t> flat(4 * (size_t)nt);
    if (vbd_tetgen_read_ele(eleFilename.c_str(), start_from_0 ? 0 : 1, n, &nt, flat.data(), nt) != VBD_OK) {
        std::cerr << vbd_last_error() << std::endl;
        return false;
    }
    std::vector<TetVIdsArr> tets((size_t)nt);
    for (int32_t t = 0; t < nt; ++t)
        for (int a = 0; a < 4; ++a) tets[(size_t)t][a] = flat[4 * (size_t)t + a];
    std::vector<float> cur(3 * (size_t)n);
    for (int32_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) cur[3 * (size_t)i + c] = current[(size_t)i][c];
    std::vector<uint8_t> fixed((size_t)n, 0);
    const bool axes[3] = {pin.fixX, pin.fixY, pin.fixZ};
    for (int a = 0; a < 3; ++a)
        if (axes[a]) vbdCheck(vbd_pin_low_fraction(n, cur.data(), a, pin.fraction, fixed.data()), "vbd_pin_low_fraction");
    std::vector<IdType> fixedVerts;
    for (int32_t i = 0; i < n; ++i)
        if (fixed[(size_t)i]) fixedVerts.push_back(i);
    mesh.initialize(rest, current, density, tets, mu, lambda, fixedVerts);
    return true;
}

}  // namespace VBD
