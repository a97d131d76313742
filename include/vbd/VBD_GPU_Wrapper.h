// VBD_GPU_Wrapper.h -- VBD_GPU_Solver with the reference's API (VBD_GPU_Wrapper.h:7-45) over
// libvbd_b200.  Move-only RAII owner of one vbd_solver handle.
//
// The handle runs the wrapper's own semantics (VBD_OPT_SEMANTICS = 1): the corotated element of
// computeTetContributionLocalCorotated (VBD_DeviceMath.cuh:127-198), the 1.000001 inertia diagonal,
// solve3x3's guard, float Chebyshev weights, and solveVBD's x = y initial guess
// (VBD_GPU_Wrapper.cu:332-362).  setSemantics(0) switches to the CPU solver's Neo-Hookean update
// (Energy.cpp:90-158) instead.  Failures throw std::runtime_error with the library's message.
#pragma once

#include <utility>
#include <vector>

#include "TetMesh.h"
#include "Types.h"

namespace VBD {

class VBD_GPU_Solver {
  public:
    VBD_GPU_Solver() = default;
    ~VBD_GPU_Solver() {
        if (s_) vbd_solver_destroy(s_);
    }
    VBD_GPU_Solver(const VBD_GPU_Solver&) = delete;
    VBD_GPU_Solver& operator=(const VBD_GPU_Solver&) = delete;
    VBD_GPU_Solver(VBD_GPU_Solver&& o) noexcept { swap(o); }
    VBD_GPU_Solver& operator=(VBD_GPU_Solver&& o) noexcept {
        swap(o);
        return *this;
    }

    // Uploads the mesh (VBD_GPU_Wrapper.cu:246-315).  Calling it again replaces the mesh.
    void initFromCPU(const TetMesh& mesh, const std::vector<std::vector<int>>& vertexColors,
                     const std::vector<Matrix3r>& tetDmInv, const std::vector<Real>& tetRestVol) {
        if (!s_) vbdCheck(vbd_solver_create(&s_, 0, nullptr), "vbd_solver_create");
        std::vector<int32_t> flat(4 * mesh.numTets);
        for (size_t t = 0; t < mesh.numTets; ++t)
            for (int a = 0; a < 4; ++a) flat[4 * t + a] = mesh.tets[t][a];
        std::vector<uint8_t> fixed(mesh.numVerts);
        for (size_t i = 0; i < mesh.numVerts; ++i) fixed[i] = mesh.isFixed[i] ? 1 : 0;
        std::vector<int32_t> offs(1, 0), verts;
        for (const auto& g : vertexColors) {
            verts.insert(verts.end(), g.begin(), g.end());
            offs.push_back((int32_t)verts.size());
        }
        std::vector<float> dm(9 * tetDmInv.size());
        for (size_t t = 0; t < tetDmInv.size(); ++t)
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) dm[9 * t + 3 * a + b] = tetDmInv[t](a, b);
        std::vector<float> mass(mesh.numVerts);
        for (size_t i = 0; i < mesh.numVerts; ++i) mass[i] = mesh.vertexMass((Eigen::Index)i);
        vbdCheck(vbd_solver_init(s_, (int32_t)mesh.numVerts, (int32_t)mesh.numTets, mesh.mVertPos.data(),
                                 mesh.mVelocity.data(), mesh.mInertia.data(), mass.data(), fixed.data(), flat.data(),
                                 (int32_t)vertexColors.size(), offs.data(), verts.data(), dm.data(), tetRestVol.data(),
                                 nullptr, nullptr),
                 "vbd_solver_init");
        vbdCheck(vbd_solver_set_option(s_, VBD_OPT_SEMANTICS, semantics_), "vbd_solver_set_option");
        mu_ = lambda_ = -1.0f;
    }

    // 1 (default) = the reference GPU wrapper's semantics, 0 = VBDsolver's (not in the reference API).
    void setSemantics(int semantics) {
        semantics_ = semantics;
        if (s_) vbdCheck(vbd_solver_set_option(s_, VBD_OPT_SEMANTICS, semantics_), "vbd_solver_set_option");
    }

    // One sweep over all colours (VBD_GPU_Wrapper.cu:317-329).
    void solveIteration(Real dtSqrReciprocal, Real mu, Real lambda) {
        material(mu, lambda);
        vbdCheck(vbd_solver_solve_iteration(s_, dtSqrReciprocal), "vbd_solver_solve_iteration");
    }

    // x = y, then numIterations sweeps with the Chebyshev blend (VBD_GPU_Wrapper.cu:332-362).
    void solveVBD(int numIterations, Real dtSqrReciprocal, Real mu, Real lambda, bool useAcceleration = true,
                  Real rho = 0.99f) {
        material(mu, lambda);
        vbdCheck(vbd_solver_solve(s_, numIterations, dtSqrReciprocal, useAcceleration ? 1 : 0, rho,
                                  VBD_INIT_FROM_INERTIA),
                 "vbd_solver_solve");
    }

    void copyPositionsToCPU(TetMesh& mesh) {
        vbdCheck(vbd_solver_get_positions(s_, mesh.mVertPos.data()), "vbd_solver_get_positions");
    }

    void updateInertiaFromCPU(const TetMesh& mesh) {
        vbdCheck(vbd_solver_set_inertia(s_, mesh.mInertia.data()), "vbd_solver_set_inertia");
    }

    vbd_solver* handle() const { return s_; }

  private:
    void material(Real mu, Real lambda) {
        if (mu != mu_ || lambda != lambda_) {
            vbdCheck(vbd_solver_set_uniform_material(s_, mu, lambda), "vbd_solver_set_uniform_material");
            mu_ = mu;
            lambda_ = lambda;
        }
    }
    void swap(VBD_GPU_Solver& o) noexcept {
        std::swap(s_, o.s_);
        std::swap(mu_, o.mu_);
        std::swap(lambda_, o.lambda_);
        std::swap(semantics_, o.semantics_);
    }
    vbd_solver* s_ = nullptr;
    Real mu_ = -1.0f, lambda_ = -1.0f;
    int semantics_ = 1;
};

}  // namespace VBD
