// VBD.h -- VBDParams and VBDsolver with the reference's API (VBD.h:14-140), running on the GPU.
//
// step() / simulate() keep the reference's semantics (VBDsolver::step, VBD.cpp:60-101: predictor,
// numIterations Gauss-Seidel colour sweeps with the Chebyshev blend, velocity update x 0.999) but
// execute through libvbd_b200: the TetMesh's positions and velocities are uploaded, one
// vbd_solver_step runs on the device, and positions, velocities and the inertial target are read
// back (or, with the VBDParams::deviceResident extension, stay on the device until syncToHost).  Colouring and Dm^-1 / V0 are computed by the library bit-exactly with the reference.
// energyHistory is filled as the reference fills it: computeTotalEnergy after iterations 0, 10,
// 20, ... of every sub-step (VBD.cpp:93-95), evaluated on the device inside the step (FP64 sums)
// and read back once per step; simulate() clears it first and evaluates the energy once more after
// every frame, which the reference only prints in VBD_DEBUG builds (VBD.cpp:313-330).
// Differences from the reference, by design:
//   * numThreads is ignored (the GPU sweeps each colour in parallel; results equal the reference's
//     single-thread run up to summation order, without its colour-loop race, VBD.cpp:120);
//   * solveVertex / computeTetContribution (per-vertex CPU helpers) are not provided.
#pragma once

#include <algorithm>
#include <cstddef>
#include <functional>
#include <vector>

#include "GraphColoring.h"
#include "TetMesh.h"
#include "Types.h"

namespace VBD {

struct VBDParams {
    Real dt = 0.01666666f;
    int numIterations = 50;
    int substeps = 1;
    Vec3 gravity{0, -9.8f, 0};
    bool useAcceleration = false;
    Real accelerationRho = 0.75f;
    int numThreads = 4;  // accepted for compatibility; the sweep runs on the GPU
    Real mu = 1e6f;
    Real lambda = 1e6f;
    Real density = 1000.0f;
    // extensions
    bool usePerTetMaterials = false;   // use TetMesh::tetMu / tetLambda instead of mu / lambda
    int device = 0;                    // CUDA device of the solver
    // Keep the state on the GPU between steps: step() uploads the mesh's positions and velocities
    // only at the first step and after markHostChanged(), and reads nothing back; syncToHost(mesh)
    // brings positions, velocities, the inertial target and the steps' energyHistory entries back
    // (simulate() does so before each callback).  mVertPrevPos is not maintained in this mode.
    // Default: the reference's behaviour, every step reads the state from and writes it back to the
    // TetMesh.
    bool deviceResident = false;
};

class VBDsolver {
  public:
    VBDsolver() = default;
    ~VBDsolver() { release(); }
    VBDsolver(const VBDsolver&) = delete;
    VBDsolver& operator=(const VBDsolver&) = delete;

    void setParams(const VBDParams& p) { params = p; }

    void initializeColoring(const TetMesh& mesh) {
        vertexColors = GraphColoring::colorVertices(mesh.vertAdjacentTets, mesh.tets, mesh.numVerts);
        prevPrevPos.resize(3, (Eigen::Index)mesh.numVerts);
        prevPrevPos.setZero();
    }

    void precomputeTetData(const TetMesh& mesh) {
        const std::vector<int32_t> flat = flatTets(mesh);
        std::vector<float> dm(9 * mesh.numTets);
        tetRestVolume.assign(mesh.numTets, 0.0f);
        vbdCheck(vbd_precompute_tets((int32_t)mesh.numVerts, (int32_t)mesh.numTets, mesh.mRestPos.data(), flat.data(),
                                     dm.data(), tetRestVolume.data()),
                 "vbd_precompute_tets");
        tetDmInv.assign(mesh.numTets, Matrix3r());
        for (size_t t = 0; t < mesh.numTets; ++t)
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) tetDmInv[t](a, b) = dm[9 * t + 3 * a + b];
    }

    void step(TetMesh& mesh) {
        if (vertexColors.empty()) {
            initializeColoring(mesh);
            precomputeTetData(mesh);
        }
        ensureDevice(mesh);
        if (!params.deviceResident || deviceStale_) {
            vbdCheck(vbd_solver_set_positions(gpu_, mesh.mVertPos.data()), "vbd_solver_set_positions");
            vbdCheck(vbd_solver_set_velocities(gpu_, mesh.mVelocity.data()), "vbd_solver_set_velocities");
            deviceStale_ = false;
        }
        if (!params.deviceResident) mesh.savePreviousPosition();
        const float g[3] = {params.gravity[0], params.gravity[1], params.gravity[2]};
        vbdCheck(vbd_solver_step(gpu_, params.dt, params.substeps, params.numIterations, g,
                                 params.useAcceleration ? 1 : 0, params.accelerationRho),
                 "vbd_solver_step");
        hostStale_ = true;
        if (!params.deviceResident) syncToHost(mesh);
    }

    void simulate(TetMesh& mesh, int numFrames, std::function<void(int, TetMesh&)> callback = nullptr) {
        syncToHost(mesh);  // earlier resident steps' state and energies first
        energyHistory.clear();
        for (int frame = 0; frame < numFrames; ++frame) {
            step(mesh);
            syncToHost(mesh);  // the callback and the caller see the frame's state
            // the frame's energy (VBD.cpp:318-319), from the state the step left on the device
            const Real energy = deviceEnergy();
            VBD_LOG("Frame " << frame << " completed, Energy: " << energy);
            (void)energy;
            if (callback) callback(frame, mesh);
        }
    }

    // Elastic log-J Neo-Hookean energy of the mesh's current positions (VBD.cpp:258-288), summed
    // in FP64 on the device.  With deviceResident the GPU's positions are the current ones unless
    // the host copy was marked changed.
    Real computeTotalEnergy(const TetMesh& mesh) const {
        ensureDevice(mesh);
        if (!params.deviceResident || deviceStale_) {
            vbdCheck(vbd_solver_set_positions(gpu_, mesh.mVertPos.data()), "vbd_solver_set_positions");
            if (params.deviceResident) vbdCheck(vbd_solver_set_velocities(gpu_, mesh.mVelocity.data()),
                                                "vbd_solver_set_velocities");
            deviceStale_ = false;
        }
        return deviceEnergy();
    }

    // deviceResident: positions, velocities and the inertial target back into the mesh, if a step
    // has run since the last sync.  (Without deviceResident every step already does this.)
    // The energies the steps since the last sync evaluated after iterations 0, 10, 20, ...
    // (VBD.cpp:93-95) are appended to energyHistory here too.
    void syncToHost(TetMesh& mesh) {
        if (!gpu_ || !hostStale_) return;
        vbdCheck(vbd_solver_get_positions(gpu_, mesh.mVertPos.data()), "vbd_solver_get_positions");
        vbdCheck(vbd_solver_get_velocities(gpu_, mesh.mVelocity.data()), "vbd_solver_get_velocities");
        vbdCheck(vbd_solver_get_inertia(gpu_, mesh.mInertia.data()), "vbd_solver_get_inertia");
        int32_t n = 0;
        vbdCheck(vbd_solver_energy_history(gpu_, nullptr, 0, &n, 0), "vbd_solver_energy_history");
        std::vector<double> e((size_t)n);
        vbdCheck(vbd_solver_energy_history(gpu_, e.data(), n, &n, 1), "vbd_solver_energy_history");
        for (double v : e) energyHistory.push_back((Real)v);
        hostStale_ = false;
    }

    // deviceResident: the caller changed the mesh's positions or velocities; the next step (or
    // computeTotalEnergy) uploads them.
    void markHostChanged() { deviceStale_ = true; }

    const std::vector<std::vector<IdType>>& getVertexColors() const { return vertexColors; }
    const std::vector<Matrix3r>& getTetDmInv() const { return tetDmInv; }
    const std::vector<Real>& getTetRestVol() const { return tetRestVolume; }

    VBDParams params;
    std::vector<std::vector<IdType>> vertexColors;
    TVerticesMat prevPrevPos;
    std::vector<Real> energyHistory;
    std::vector<Matrix3r> tetDmInv;
    std::vector<Real> tetRestVolume;

    // Predictor on the host, as the reference (VBD.cpp:103-112).
    void forwardStep(TetMesh& mesh) {
        mesh.savePreviousPosition();
        mesh.applyGravity(params.gravity, params.dt / params.substeps);
        mesh.computeInertia(params.dt / params.substeps);
    }

    // One Gauss-Seidel sweep over all colours from mesh.mVertPos towards mesh.mInertia
    // (VBD.cpp:114-158), on the device.
    void solve(TetMesh& mesh) {
        if (vertexColors.empty()) {
            initializeColoring(mesh);
            precomputeTetData(mesh);
        }
        ensureDevice(mesh);
        syncToHost(mesh);  // deviceResident: the mesh first catches up with the device's state
        const Real dt = params.dt / params.substeps;
        const Real dtsr = (Real)(1.0 / (dt * dt));
        vbdCheck(vbd_solver_set_positions(gpu_, mesh.mVertPos.data()), "vbd_solver_set_positions");
        vbdCheck(vbd_solver_set_inertia(gpu_, mesh.mInertia.data()), "vbd_solver_set_inertia");
        vbdCheck(vbd_solver_solve_iteration(gpu_, dtsr), "vbd_solver_solve_iteration");
        vbdCheck(vbd_solver_get_positions(gpu_, mesh.mVertPos.data()), "vbd_solver_get_positions");
    }

    // x = omega (x - x_pp) + x_pp on free vertices (VBD.cpp:290-300), on the host.
    void applyAcceleration(TetMesh& mesh, Real omega) {
        if (omega <= 1.0) return;
        for (size_t i = 0; i < mesh.numVerts; ++i)
            if (!mesh.isFixed[i])
                for (int c = 0; c < 3; ++c) {
                    const Eigen::Index k = (Eigen::Index)i;
                    mesh.mVertPos(c, k) = omega * (mesh.mVertPos(c, k) - prevPrevPos(c, k)) + prevPrevPos(c, k);
                }
    }

    // Chebyshev weights (VBD.cpp:302-311).
    Real getAcceleratorOmega(int order, Real rho, Real prevOmega) {
        if (order == 1) return 1.0f;
        if (order == 2) return (Real)(2.0 / (2.0 - (double)(rho * rho)));
        return (Real)(4.0 / (4.0 - (double)(rho * rho * prevOmega)));
    }

    // The C-ABI handle (null before the first step); for callers mixing both APIs.
    vbd_solver* deviceHandle() const { return gpu_; }

  private:
    static std::vector<int32_t> flatTets(const TetMesh& mesh) {
        std::vector<int32_t> flat(4 * mesh.numTets);
        for (size_t t = 0; t < mesh.numTets; ++t)
            for (int a = 0; a < 4; ++a) flat[4 * t + a] = mesh.tets[t][a];
        return flat;
    }

    // computeTotalEnergy of the positions on the device (no upload).
    Real deviceEnergy() const {
        double e = 0.0;
        vbdCheck(vbd_solver_energy(gpu_, VBD_ENERGY_ELASTIC_LOGJ, 1.0f, &e), "vbd_solver_energy");
        return (Real)e;
    }

    void ensureDevice(const TetMesh& mesh) const {
        if (gpu_ && devVerts_ == mesh.numVerts && devTets_ == mesh.numTets) {
            syncMaterials(mesh);
            return;
        }
        if (!gpu_) {
            vbdCheck(vbd_solver_create(&gpu_, params.device, nullptr), "vbd_solver_create");
            // VBDsolver::step evaluates computeTotalEnergy every 10th iteration (VBD.cpp:93-95)
            vbdCheck(vbd_solver_set_option(gpu_, VBD_OPT_ENERGY_EVERY, 10), "vbd_solver_set_option");
        }
        const std::vector<int32_t> flat = flatTets(mesh);
        std::vector<uint8_t> fixed(mesh.numVerts);
        for (size_t i = 0; i < mesh.numVerts; ++i) fixed[i] = mesh.isFixed[i] ? 1 : 0;
        std::vector<int32_t> offs(1, 0), verts;
        for (const auto& g : vertexColors) {
            verts.insert(verts.end(), g.begin(), g.end());
            offs.push_back((int32_t)verts.size());
        }
        std::vector<float> dm(9 * mesh.numTets);
        for (size_t t = 0; t < mesh.numTets; ++t)
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) dm[9 * t + 3 * a + b] = tetDmInv[t](a, b);
        std::vector<float> mass(mesh.numVerts);
        for (size_t i = 0; i < mesh.numVerts; ++i) mass[i] = mesh.vertexMass((Eigen::Index)i);
        vbdCheck(vbd_solver_init(gpu_, (int32_t)mesh.numVerts, (int32_t)mesh.numTets, mesh.mVertPos.data(),
                                 mesh.mVelocity.data(), mesh.mInertia.data(), mass.data(), fixed.data(), flat.data(),
                                 (int32_t)vertexColors.size(), offs.data(), verts.data(), dm.data(),
                                 tetRestVolume.data(), nullptr, nullptr),
                 "vbd_solver_init");
        devVerts_ = mesh.numVerts;
        devTets_ = mesh.numTets;
        matKey_.clear();
        syncMaterials(mesh);
        deviceStale_ = hostStale_ = false;  // the device now holds the mesh's state
    }

    // Materials as the reference uses them: params.mu / lambda for every tet (VBD.cpp:214-215), or
    // the mesh's per-tet values when usePerTetMaterials is set.
    // The values last uploaded are kept in matKey_ (mu then lambda, per tet or uniform) and compared
    // in place, so an unchanged per-tet material costs one read of the two arrays per step.
    void syncMaterials(const TetMesh& mesh) const {
        if (params.usePerTetMaterials) {
            const size_t T = mesh.tetMu.size();
            if (matPerTet_ && matKey_.size() == 2 * T && mesh.tetLambda.size() == T &&
                std::equal(mesh.tetMu.begin(), mesh.tetMu.end(), matKey_.begin()) &&
                std::equal(mesh.tetLambda.begin(), mesh.tetLambda.end(), matKey_.begin() + (std::ptrdiff_t)T))
                return;
            vbdCheck(vbd_solver_set_materials(gpu_, mesh.tetMu.data(), mesh.tetLambda.data()), "vbd_solver_set_materials");
            matKey_.assign(mesh.tetMu.begin(), mesh.tetMu.end());
            matKey_.insert(matKey_.end(), mesh.tetLambda.begin(), mesh.tetLambda.end());
        } else {
            if (!matPerTet_ && matKey_.size() == 2 && matKey_[0] == params.mu && matKey_[1] == params.lambda) return;
            vbdCheck(vbd_solver_set_uniform_material(gpu_, params.mu, params.lambda), "vbd_solver_set_uniform_material");
            matKey_ = {params.mu, params.lambda};
        }
        matPerTet_ = params.usePerTetMaterials;
    }

    void release() {
        if (gpu_) vbd_solver_destroy(gpu_);
        gpu_ = nullptr;
    }

    mutable vbd_solver* gpu_ = nullptr;
    mutable size_t devVerts_ = 0, devTets_ = 0;
    mutable bool hostStale_ = false;   // the device holds a newer state than the mesh
    mutable bool deviceStale_ = true;  // the mesh holds a newer state than the device
    mutable std::vector<float> matKey_;
    mutable bool matPerTet_ = false;  // matKey_ holds per-tet values
};

}  // namespace VBD
