// TetGen mesh input (.node / .ele) and the fraction-of-extent pinning rule of the reference's
// driver (main.cpp:14-168), behind the C ABI so the C++ header (include/vbd/TetGenIO.h) and the
// Python package read files identically.
//
// Parsing follows main.cpp's readNodeFile / loadTetgenModel: the first line's first number is the
// record count; each record line starts with its index followed by x y z (node) or four vertex ids
// (element), further columns ignored; numbers are read with the C++ stream extraction operators.
// Indices are 0-based when the first node's index is 0, else 1-based and shifted down by one.
// Additionally, blank lines and lines whose first non-blank character is '#' are skipped (TetGen
// writes such comment lines); files the reference driver reads are read the same way.
#include <cstdint>
#include <fstream>
#include <limits>
#include <sstream>
#include <string>
#include <vector>

#include "vbd_b200.h"
#include "vbd_internal.h"

namespace {

bool next_record(std::ifstream& in, std::string& line) {
    while (std::getline(in, line)) {
        size_t p = line.find_first_not_of(" \t\r");
        if (p == std::string::npos || line[p] == '#') continue;
        return true;
    }
    return false;
}

int read_header(std::ifstream& in, const char* path, long long& count) {
    std::string line;
    if (!next_record(in, line)) VBD_FAIL(VBD_ERR_INVALID_ARG, "'%s': no header line", path);
    std::istringstream ss(line);
    if (!(ss >> count) || count < 0 || count > std::numeric_limits<int32_t>::max())
        VBD_FAIL(VBD_ERR_INVALID_ARG, "'%s': bad record count in header", path);
    return VBD_OK;
}

}  // namespace

extern "C" {

int vbd_tetgen_read_node(const char* path, int32_t* num_nodes, int32_t* first_index, float* positions,
                         int32_t capacity) {
    vbd::clear_error();
    if (!path || !num_nodes) VBD_FAIL(VBD_ERR_INVALID_ARG, "path and num_nodes are required");
    std::ifstream in(path);
    if (!in) VBD_FAIL(VBD_ERR_INVALID_ARG, "'%s' file not found", path);
    long long count = 0;
    if (int rc = read_header(in, path, count)) return rc;
    *num_nodes = (int32_t)count;
    if (!positions) return VBD_OK;
    if (capacity < count) VBD_FAIL(VBD_ERR_INVALID_ARG, "positions hold %d nodes, the file has %lld", capacity, count);
    std::string line;
    for (long long i = 0; i < count; ++i) {
        if (!next_record(in, line)) VBD_FAIL(VBD_ERR_INVALID_ARG, "'%s': %lld of %lld node lines", path, i, count);
        std::istringstream ss(line);
        long long idx;
        float x, y, z;
        if (!(ss >> idx >> x >> y >> z)) VBD_FAIL(VBD_ERR_INVALID_ARG, "'%s': bad node line %lld", path, i + 1);
        if (i == 0 && first_index) *first_index = (int32_t)idx;
        positions[3 * i] = x;
        positions[3 * i + 1] = y;
        positions[3 * i + 2] = z;
    }
    return VBD_OK;
}

int vbd_tetgen_read_ele(const char* path, int32_t index_base, int32_t num_nodes, int32_t* num_tets, int32_t* tets,
                        int32_t capacity) {
    vbd::clear_error();
    if (!path || !num_tets) VBD_FAIL(VBD_ERR_INVALID_ARG, "path and num_tets are required");
    if (index_base != 0 && index_base != 1) VBD_FAIL(VBD_ERR_INVALID_ARG, "index_base must be 0 or 1");
    std::ifstream in(path);
    if (!in) VBD_FAIL(VBD_ERR_INVALID_ARG, "'%s' file not found", path);
    long long count = 0;
    if (int rc = read_header(in, path, count)) return rc;
    *num_tets = (int32_t)count;
    if (!tets) return VBD_OK;
    if (capacity < count) VBD_FAIL(VBD_ERR_INVALID_ARG, "tets hold %d elements, the file has %lld", capacity, count);
    std::string line;
    for (long long t = 0; t < count; ++t) {
        if (!next_record(in, line)) VBD_FAIL(VBD_ERR_INVALID_ARG, "'%s': %lld of %lld element lines", path, t, count);
        std::istringstream ss(line);
        long long idx, v[4];
        if (!(ss >> idx >> v[0] >> v[1] >> v[2] >> v[3]))
            VBD_FAIL(VBD_ERR_INVALID_ARG, "'%s': bad element line %lld", path, t + 1);
        for (int a = 0; a < 4; ++a) {
            long long id = v[a] - index_base;
            if (id < 0 || (num_nodes >= 0 && id >= num_nodes))
                VBD_FAIL(VBD_ERR_INVALID_ARG, "'%s': element %lld names node %lld, outside the %d nodes", path, t,
                         v[a], num_nodes);
            tets[4 * t + a] = (int32_t)id;
        }
    }
    return VBD_OK;
}

int vbd_pin_low_fraction(int32_t num_verts, const float* positions, int32_t axis, float fraction, uint8_t* fixed) {
    vbd::clear_error();
    if (num_verts < 0 || (num_verts > 0 && (!positions || !fixed)))
        VBD_FAIL(VBD_ERR_INVALID_ARG, "positions and fixed are required");
    if (axis < 0 || axis > 2) VBD_FAIL(VBD_ERR_INVALID_ARG, "axis must be 0, 1 or 2");
    float lo = std::numeric_limits<float>::max(), hi = std::numeric_limits<float>::lowest();
    for (int32_t i = 0; i < num_verts; ++i) {
        const float c = positions[3LL * i + axis];
        if (c < lo) lo = c;
        if (c > hi) hi = c;
    }
    const float threshold = lo + (hi - lo) * fraction;
    for (int32_t i = 0; i < num_verts; ++i)
        if (positions[3LL * i + axis] <= threshold) fixed[i] = 1;
    return VBD_OK;
}

}  // extern "C"
