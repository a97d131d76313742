// GraphColoring.h -- greedy vertex colouring (reference GraphColoring.h:15-47 / GraphColoring.cpp:28-66),
// computed by libvbd_b200 (vbd_color_vertices) bit for bit.
#pragma once

#include <array>
#include <vector>

#include "Types.h"

namespace VBD {

class GraphColoring {
  public:
    // Colour groups in ascending vertex id; vertAdjacentTets is accepted for signature
    // compatibility (the adjacency is rebuilt from the tets in ascending tet order).
    static std::vector<std::vector<IdType>> colorVertices(const std::vector<std::vector<IdType>>& /*vertAdjacentTets*/,
                                                          const std::vector<TetVIdsArr>& tets, size_t numVerts) {
        std::vector<int32_t> flat(4 * tets.size());
        for (size_t t = 0; t < tets.size(); ++t)
            for (int a = 0; a < 4; ++a) flat[4 * t + a] = tets[t][a];
        std::vector<int32_t> colour((size_t)numVerts);
        int32_t nc = 0;
        vbdCheck(vbd_color_vertices((int32_t)numVerts, (int32_t)tets.size(), flat.data(), colour.data(), &nc, 0,
                                    nullptr, nullptr),
                 "vbd_color_vertices");
        std::vector<std::vector<IdType>> groups((size_t)nc);
        for (size_t v = 0; v < numVerts; ++v) groups[(size_t)colour[v]].push_back((IdType)v);
        return groups;
    }
    static size_t getNumColors(const std::vector<std::vector<IdType>>& colors) { return colors.size(); }
};

}  // namespace VBD
