// Internal helpers shared by the host and device translation units of libvbd_b200.
#pragma once

#include <cstdarg>
#include <cstdint>
#include <string>

namespace vbd {

// Records the message of the last failing call on this thread (read by vbd_last_error()).
void set_error(const char* fmt, ...);
void clear_error();
const char* last_error();

// Shared validation of the topology arrays: ids in range and four distinct ids per tet.
int check_tets(int32_t num_verts, int32_t num_tets, const int32_t* tets);

// Vertex -> incident tets in ascending tet id (TetMesh::vertAdjacentTets, TetMesh.h:262).
void build_vertex_tets(int32_t num_verts, int32_t num_tets, const int32_t* tets, int32_t* offsets /*N+1*/,
                       int32_t* tet_ids /*4T*/);

// Worst relative FP32 error of det M in the factored record layouts 3 and 4, and layout 4's worst
// error over what an incidence allows it (vbd_factored_record_error).
void factored_detm_error(int32_t num_tets, const float* dm_inv, double* err3, double* err4, double* excess4);

// Layout 4's det M may be off by this much relative, or by this many times layout 3's error on the
// same incidence (the conditioning of Dm^-1, which every FP32 form of the element shares).
constexpr double kFactoredDetmTol = 1e-5;
constexpr double kFactoredDetmRatio = 4.0;
// An incidence whose stored det M is off by more than this is degenerate in FP32.
constexpr double kFactoredDegenerate = 1e-3;

}  // namespace vbd

#define VBD_FAIL(code, ...)            \
    do {                               \
        ::vbd::set_error(__VA_ARGS__); \
        return (code);                 \
    } while (0)
