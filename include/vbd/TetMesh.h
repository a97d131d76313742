// TetMesh.h -- the reference's tetrahedral mesh state (TetMesh.h:19-349) with the same public fields
// and methods.  Set-up arithmetic (rest volumes, lumped masses) comes from libvbd_b200 so that it is
// bit-identical with the reference; the per-vertex update helpers run on the host as in the reference.
#pragma once

#include <algorithm>
#include <fstream>
#include <iostream>
#include <limits>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "Types.h"

namespace VBD {

struct TetMesh {
    TVerticesMat mRestPos;      // rest positions (3 x N)
    TVerticesMat mVertPos;      // current positions
    TVerticesMat mVertPrevPos;  // positions at the start of the last step
    TVerticesMat mVelocity;
    TVerticesMat mInertia;      // inertial target y
    VecDynamic vertexMass;

    std::vector<TetVIdsArr> tets;
    std::vector<FloatingType> tetRestVol;
    std::vector<FloatingType> tetMu;
    std::vector<FloatingType> tetLambda;
    std::vector<std::vector<IdType>> vertAdjacentTets;  // ascending tet id
    size_t numVerts = 0;
    size_t numTets = 0;
    std::vector<bool> isFixed;

    // A triangle with its vertex ids sorted (face identity), and one with its original order.
    struct TriangleFace {
        IdType v[3];
        TriangleFace() { v[0] = v[1] = v[2] = -1; }
        TriangleFace(IdType a, IdType b, IdType c) {
            v[0] = a;
            v[1] = b;
            v[2] = c;
            std::sort(v, v + 3);
        }
        bool operator==(const TriangleFace& o) const { return v[0] == o.v[0] && v[1] == o.v[1] && v[2] == o.v[2]; }
        bool operator<(const TriangleFace& o) const {
            if (v[0] != o.v[0]) return v[0] < o.v[0];
            if (v[1] != o.v[1]) return v[1] < o.v[1];
            return v[2] < o.v[2];
        }
    };
    struct OrientedTriangle {
        IdType v0, v1, v2;
        OrientedTriangle() : v0(-1), v1(-1), v2(-1) {}
        OrientedTriangle(IdType a, IdType b, IdType c) : v0(a), v1(b), v2(c) {}
    };

    // Boundary triangles: faces of exactly one tet, oriented as first met, in sorted-face order
    // (TetMesh.h:80-141).
    std::vector<Vec3I> extractSurfaceFaces() const {
        std::map<TriangleFace, std::pair<int, OrientedTriangle>> faces;
        for (size_t t = 0; t < numTets; ++t) {
            const auto& q = tets[t];
            const OrientedTriangle f[4] = {OrientedTriangle(q[0], q[2], q[1]), OrientedTriangle(q[0], q[1], q[3]),
                                           OrientedTriangle(q[0], q[3], q[2]), OrientedTriangle(q[1], q[2], q[3])};
            for (const auto& tri : f) {
                auto it = faces.find(TriangleFace(tri.v0, tri.v1, tri.v2));
                if (it == faces.end())
                    faces.emplace(TriangleFace(tri.v0, tri.v1, tri.v2), std::make_pair(1, tri));
                else
                    ++it->second.first;
            }
        }
        std::vector<Vec3I> out;
        for (const auto& kv : faces)
            if (kv.second.first == 1) out.push_back(Vec3I(kv.second.second.v0, kv.second.second.v1, kv.second.second.v2));
        return out;
    }

    // Vertices and boundary triangles as a Wavefront OBJ file (TetMesh.h:147-186).
    bool exportToObj(const std::string& filepath) const {
        std::ofstream out(filepath.c_str());
        if (!out.is_open()) {
            std::cerr << "Error: Cannot open file for writing: " << filepath << std::endl;
            return false;
        }
        out << "# TetMesh OBJ Export\n# Vertices: " << numVerts << "\n# Tetrahedra: " << numTets << "\n\n";
        for (size_t i = 0; i < numVerts; ++i)
            out << "v " << mVertPos(0, (Eigen::Index)i) << " " << mVertPos(1, (Eigen::Index)i) << " "
                << mVertPos(2, (Eigen::Index)i) << "\n";
        out << "\n";
        const std::vector<Vec3I> faces = extractSurfaceFaces();
        out << "# Surface Triangles: " << faces.size() << "\n";
        for (const auto& f : faces) out << "f " << (f[0] + 1) << " " << (f[1] + 1) << " " << (f[2] + 1) << "\n";
        return true;
    }

    Eigen::Block<TVerticesMat, 3, 1> vertex(IdType i) { return mVertPos.block<3, 1>(0, i); }
    const Eigen::Block<const TVerticesMat, 3, 1> vertex(IdType i) const { return mVertPos.block<3, 1>(0, i); }

    // Rest / current positions, lumped masses rho V / 4, adjacency, pinned vertices
    // (TetMesh::initialize, TetMesh.h:213-275).
    void initialize(const std::vector<Vec3>& rest_positions, const std::vector<Vec3>& current_positions,
                    FloatingType density, const std::vector<TetVIdsArr>& tetIndices, FloatingType mu, FloatingType lambda,
                    const std::vector<IdType>& fixedVerts = {}) {
        numVerts = rest_positions.size();
        numTets = tetIndices.size();
        const Eigen::Index n = (Eigen::Index)numVerts;
        mRestPos.resize(3, n);
        mVertPos.resize(3, n);
        mVertPrevPos.resize(3, n);
        mVelocity.resize(3, n);
        mInertia.resize(3, n);
        vertexMass.resize(n);
        mRestPos.setZero();
        mVertPos.setZero();
        mVertPrevPos.setZero();
        mVelocity.setZero();
        mInertia.setZero();
        for (Eigen::Index i = 0; i < n; ++i) {
            mRestPos.col(i) = rest_positions[(size_t)i];
            mVertPos.col(i) = current_positions[(size_t)i];
            mVertPrevPos.col(i) = current_positions[(size_t)i];
        }
        tets = tetIndices;
        tetMu.assign(numTets, mu);
        tetLambda.assign(numTets, lambda);
        tetRestVol.assign(numTets, 0.0f);
        std::vector<int32_t> flat(4 * numTets);
        for (size_t t = 0; t < numTets; ++t)
            for (int a = 0; a < 4; ++a) flat[4 * t + a] = tets[t][a];
        std::vector<float> mass(numVerts);
        vbdCheck(vbd_mesh_mass((int32_t)numVerts, (int32_t)numTets, mRestPos.data(), flat.data(), density, mass.data(),
                               tetRestVol.data()),
                 "vbd_mesh_mass");
        for (Eigen::Index i = 0; i < n; ++i) vertexMass(i) = mass[(size_t)i];
        vertAdjacentTets.assign(numVerts, {});
        for (size_t t = 0; t < numTets; ++t)
            for (int a = 0; a < 4; ++a) vertAdjacentTets[(size_t)tets[t][a]].push_back((IdType)t);
        isFixed.assign(numVerts, false);
        for (IdType vid : fixedVerts)
            if (vid >= 0 && vid < (IdType)numVerts) isFixed[(size_t)vid] = true;
    }

    FloatingType computeTetVolume(IdType tetId) const { return volumeOf(mVertPos, tetId); }
    FloatingType computeRestVolume(IdType tetId) const { return volumeOf(mRestPos, tetId); }

    // v = (x - x_prev)/dt * 0.999 on free vertices (TetMesh.h:305-311)
    void updateVelocity(FloatingType dt) {
        for (size_t i = 0; i < numVerts; ++i)
            if (!isFixed[i])
                for (int c = 0; c < 3; ++c) {
                    const Eigen::Index k = (Eigen::Index)i;
                    mVelocity(c, k) = ((mVertPos(c, k) - mVertPrevPos(c, k)) / dt) * 0.999f;
                }
    }
    // v += dt g on free vertices (TetMesh.h:319-325)
    void applyGravity(const Vec3& gravity, FloatingType dt) {
        for (size_t i = 0; i < numVerts; ++i)
            if (!isFixed[i])
                for (int c = 0; c < 3; ++c) mVelocity(c, (Eigen::Index)i) += dt * gravity[c];
    }
    // y = x + dt v (free), y = x (pinned) (TetMesh.h:332-341)
    void computeInertia(FloatingType dt) {
        for (size_t i = 0; i < numVerts; ++i)
            for (int c = 0; c < 3; ++c) {
                const Eigen::Index k = (Eigen::Index)i;
                mInertia(c, k) = isFixed[i] ? mVertPos(c, k) : mVertPos(c, k) + dt * mVelocity(c, k);
            }
    }
    void savePreviousPosition() { mVertPrevPos = mVertPos; }

  private:
    FloatingType volumeOf(const TVerticesMat& X, IdType tetId) const {
        const auto& v = tets[(size_t)tetId];
        Real e[3][3];
        for (int k = 0; k < 3; ++k)
            for (int r = 0; r < 3; ++r) e[k][r] = X(r, v[k + 1]) - X(r, v[0]);
        const Real c0 = e[1][1] * e[2][2] - e[1][2] * e[2][1];
        const Real c1 = e[1][2] * e[2][0] - e[1][0] * e[2][2];
        const Real c2 = e[1][0] * e[2][1] - e[1][1] * e[2][0];
        Real d = e[0][0] * c0;
        d += e[0][1] * c1;
        d += e[0][2] * c2;
        return std::abs(d) / 6.0f;
    }
};

}  // namespace VBD
