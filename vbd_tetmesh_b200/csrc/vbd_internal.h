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

// Worst relative FP32 error of det M in the factored record layouts 3 and 4, and the fraction of
// incidences on which layout 4 loses accuracy (vbd_factored_record_error).
void factored_detm_error(int32_t num_tets, const float* dm_inv, double* err3, double* err4, double* frac4);

// Layout 4 loses accuracy on an incidence when its det M is off by more than this relative and by
// more than this many times layout 3's error there (the conditioning of Dm^-1, which every FP32 form
// of the element shares).
constexpr double kFactoredDetmTol = 1e-5;
constexpr double kFactoredDetmRatio = 4.0;
// An incidence whose stored det M is off by more than this is degenerate in FP32.
constexpr double kFactoredDegenerate = 1e-3;
// The automatic layout choice takes layout 3 when layout 4 loses accuracy on more than this
// fraction of the incidences (systematic anisotropy); a few isolated thin tets do not move the
// positions measurably (the 512-mesh batch: 4.08e-6 against 4.15e-6 of the diagonal from FP64).
constexpr double kFactoredLossFraction = 1e-3;

}  // namespace vbd

#define VBD_FAIL(code, ...)            \
    do {                               \
        ::vbd::set_error(__VA_ARGS__); \
        return (code);                 \
    } while (0)
