// Types.h -- scalar, id and Eigen-typed aliases of the VBD C++ surface (same names as the
// reference's Types.h:18-64), the 3x3 analytic solver contract (Types.h:83-120) and the checked-call
// helper used by the header-only C++ layer over libvbd_b200's C ABI.
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <functional>
#ifdef VBD_DEBUG
#include <iostream>
#endif
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef VBD_USE_REAL_EIGEN
#include <Eigen/Core>
#include <Eigen/Dense>
#else
#include "eigen_lite.h"
#endif

#include "vbd_b200.h"

using FloatingType = float;
using Real = FloatingType;

namespace VBD {

using IdType = int32_t;

using Vec2 = Eigen::Matrix<Real, 2, 1>;
using Vec3 = Eigen::Matrix<Real, 3, 1>;
using Vec4 = Eigen::Matrix<Real, 4, 1>;
using Vec6 = Eigen::Matrix<Real, 6, 1>;
using Vec9 = Eigen::Matrix<Real, 9, 1>;
using Vec12 = Eigen::Matrix<Real, 12, 1>;
using VectorXr = Eigen::Matrix<Real, Eigen::Dynamic, 1>;
using Vec2I = Eigen::Matrix<IdType, 2, 1>;
using Vec3I = Eigen::Matrix<IdType, 3, 1>;
using Vec4I = Eigen::Matrix<IdType, 4, 1>;
using Mat2 = Eigen::Matrix<Real, 2, 2>;
using Mat3 = Eigen::Matrix<Real, 3, 3>;
using Mat4 = Eigen::Matrix<Real, 4, 4>;
using Mat3x4 = Eigen::Matrix<Real, 3, 4>;
using MatrixXr = Eigen::Matrix<Real, Eigen::Dynamic, Eigen::Dynamic>;
using Matrix3r = Mat3;
using TVerticesMat = Eigen::Matrix<Real, 3, Eigen::Dynamic>;  // 3 x N, xyz interleaved in data()
using VecDynamic = Eigen::Matrix<Real, Eigen::Dynamic, 1>;
using VecDynamicI = Eigen::Matrix<IdType, Eigen::Dynamic, 1>;
using TetVIdsArr = std::array<IdType, 4>;
using TTetVIdsArr = TetVIdsArr;

#ifndef EPSILON
#define EPSILON 1e-8
#endif

// Debug output, as the reference's Types.h:72-77: printed in VBD_DEBUG builds only.
#ifndef VBD_LOG
#ifdef VBD_DEBUG
#define VBD_LOG(msg) std::cout << "[VBD] " << msg << std::endl
#else
#define VBD_LOG(msg)
#endif
#endif

// Throws std::runtime_error with vbd_last_error() when a C-ABI call fails.
inline void vbdCheck(int status, const char* what) {
    if (status != VBD_OK) throw std::runtime_error(std::string(what) + ": " + vbd_last_error());
}

// 3x3 solve by the adjugate, returning false (and x = 0) when |det A| < 1e-8 -- the contract of the
// reference's AnalyticSolver3x3::solve (Types.h:85-112).
class AnalyticSolver3x3 {
  public:
    static inline bool solve(const Mat3& A, const Vec3& b, Vec3& x) {
        const Real det = A(0, 0) * (A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1)) -
                         A(0, 1) * (A(1, 0) * A(2, 2) - A(1, 2) * A(2, 0)) +
                         A(0, 2) * (A(1, 0) * A(2, 1) - A(1, 1) * A(2, 0));
        if (std::abs(det) < EPSILON) {
            x = Vec3(0, 0, 0);
            return false;
        }
        Mat3 adj;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const int r1 = (j + 1) % 3, r2 = (j + 2) % 3, c1 = (i + 1) % 3, c2 = (i + 2) % 3;
                adj(i, j) = A(r1, c1) * A(r2, c2) - A(r1, c2) * A(r2, c1);
            }
        const Real inv = Real(1) / det;
        x = inv * (adj * b);
        return true;
    }
    static inline bool solveWithRegularization(const Mat3& A, const Vec3& b, Vec3& x, FloatingType reg = 1e-6f) {
        Mat3 Ar = A;
        Ar(0, 0) += reg;
        Ar(1, 1) += reg;
        Ar(2, 2) += reg;
        return solve(Ar, b, x);
    }
};

}  // namespace VBD
