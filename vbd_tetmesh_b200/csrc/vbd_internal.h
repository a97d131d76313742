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

}  // namespace vbd

#define VBD_FAIL(code, ...)            \
    do {                               \
        ::vbd::set_error(__VA_ARGS__); \
        return (code);                 \
    } while (0)
