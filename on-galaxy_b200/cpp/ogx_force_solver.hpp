// ogx_force_solver.hpp -- galaxy3d::ForceSolver3D implementations backed by the
// B200 library (libogx.so, C ABI declared in include/ogx.h).
//
// Drop-in replacements for the reference's solvers:
//   OgxAdaptiveFMM3D  for AdaptiveFMM3D(KernelParams3D, int p, int threshold)
//                     (src3d/AdaptiveFMM3D.hpp:20-27)
//   OgxDirect3D       for DirectSolver3D(KernelParams3D)
//                     (src3d/DirectSolver3D.hpp:11-15)
// Both implement the interface of src3d/ForceSolver3D.hpp:20-28 and so run under
// VelocityVerlet3D (src3d/Integrator3D.hpp:17-40) and the reference harnesses
// unchanged.  Include this header with the reference's ForceSolver3D.hpp and
// Kernel3D.hpp on the include path; link with -logx.
//
// Semantics kept from the reference:
//   * computeAccelerations takes the caller's FP64 SoA bodies by const reference
//     and returns one Vec3 per body in the original body order;
//   * softening applies to the near field only (AdaptiveFMM3D.hpp:18);
//   * const methods with mutable diagnostics (lastNumBoxes, lastMaxLeafOcc,
//     AdaptiveFMM3D.hpp:26-27), so one object serves one thread at a time.
// Differences: errors come back as std::runtime_error instead of exit() (the
// reference GPU path calls exit(1)/exit(2), AdaptiveFMM3DGPU.cu:23-26,328); the
// precision form is a constructor argument (FP64 by default, which matches
// AdaptiveFMM3D to 1e-12 relative); potentials are available through
// computePotentials, which the reference solvers do not offer.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "ForceSolver3D.hpp"
#include "Kernel3D.hpp"
#include "ogx.h"

namespace ogx_b200 {

class OgxSolver3D : public galaxy3d::ForceSolver3D {
public:
    OgxSolver3D(const OgxSolver3D&) = delete;
    OgxSolver3D& operator=(const OgxSolver3D&) = delete;
    ~OgxSolver3D() override {
        if (h_) ogx_destroy(h_);
    }

    galaxy3d::Accelerations3D computeAccelerations(const galaxy3d::Bodies3D& bodies) const override {
        galaxy3d::Accelerations3D acc(bodies.size());
        eval(bodies, acc, nullptr);
        return acc;
    }

    // Accelerations and per-body potentials pot_i = -G sum_j m_j / sqrt(r_ij^2 + eps^2)
    // (the spline kernel's potential with OGX_SOFT_SPLINE).
    galaxy3d::Accelerations3D computePotentials(const galaxy3d::Bodies3D& bodies, std::vector<double>& pot) const {
        galaxy3d::Accelerations3D acc(bodies.size());
        pot.assign(bodies.size(), 0.0);
        eval(bodies, acc, pot.data());
        return acc;
    }

    const char* name() const override { return ogx_name(h_); }

    // diagnostics of the last evaluation (AdaptiveFMM3D::lastNumBoxes / lastMaxLeafOcc)
    int lastNumBoxes() const { return stats_.num_boxes; }
    int lastMaxLeafOcc() const { return stats_.max_leaf_occupancy; }
    const ogx_stats& lastStats() const { return stats_; }

protected:
    OgxSolver3D(const galaxy3d::KernelParams3D& k, int solver, int p, int threshold, int precision, int device,
                int softening = OGX_SOFT_PLUMMER) {
        ogx_params prm;
        ogx_params_default(&prm);
        prm.G = k.G;
        prm.eps = k.eps;
        prm.p = p;
        prm.leaf_capacity = threshold;
        prm.solver = solver;
        prm.precision = precision;
        prm.device = device;
        prm.softening = softening;
        check(ogx_create(&prm, &h_), "ogx_create");
    }

private:
    static_assert(sizeof(galaxy3d::Vec3) == 3 * sizeof(double), "Vec3 must be three packed doubles");

    static void check(int rc, const char* what) {
        if (rc != OGX_OK)
            throw std::runtime_error(std::string(what) + ": " + ogx_strerror(rc) + " (" + ogx_last_error_message() + ")");
    }

    void eval(const galaxy3d::Bodies3D& bodies, galaxy3d::Accelerations3D& acc, double* pot) const {
        const int64_t n = (int64_t)bodies.size();
        if (bodies.pos.size() != bodies.mass.size()) throw std::invalid_argument("Bodies3D: pos and mass sizes differ");
        const double* pos = n ? reinterpret_cast<const double*>(bodies.pos.data()) : nullptr;
        double* out = n ? reinterpret_cast<double*>(acc.data()) : nullptr;
        check(ogx_eval(h_, n, pos, n ? bodies.mass.data() : nullptr, out, pot), "ogx_eval");
        check(ogx_last_stats(h_, &stats_), "ogx_last_stats");
    }

    void* h_ = nullptr;
    mutable ogx_stats stats_{};
};

// AdaptiveFMM3D(KernelParams3D kp, int p, int threshold = 64)
class OgxAdaptiveFMM3D : public OgxSolver3D {
public:
    // softening = OGX_SOFT_SPLINE: compact spline kernel with the far field corrected
    // within its support (an extension; the default is the reference's Plummer kernel)
    OgxAdaptiveFMM3D(const galaxy3d::KernelParams3D& k, int p, int threshold = 64, int precision = OGX_PREC_FP64,
                     int device = 0, int softening = OGX_SOFT_PLUMMER)
        : OgxSolver3D(k, OGX_SOLVER_ADAPTIVE_FMM, p, threshold, precision, device, softening) {}
};

// DirectSolver3D(KernelParams3D kp)
class OgxDirect3D : public OgxSolver3D {
public:
    explicit OgxDirect3D(const galaxy3d::KernelParams3D& k, int device = 0, int softening = OGX_SOFT_PLUMMER)
        : OgxSolver3D(k, OGX_SOLVER_DIRECT, 8, 64, OGX_PREC_FP64, device, softening) {}
};

}  // namespace ogx_b200
