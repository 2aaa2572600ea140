// dropin_check.cpp -- checks the C++ drop-in boundary: the B200 solvers plugged
// into the reference's own ForceSolver3D seam (src3d/ForceSolver3D.hpp:20-28)
// next to the reference solvers, on the reference's own Plummer bodies
// (makePlummerSphere, src3d/InitialConditions3D.hpp:100-152).
//
// Test infrastructure: compiled from the reference headers into oracle/_ref/
// by oracle/Makefile, never shipped.  Prints one JSON line:
//   fmm_max_rel      OgxAdaptiveFMM3D (FP64 form) vs AdaptiveFMM3D, same p / threshold
//   direct_max_rel   OgxDirect3D vs DirectSolver3D
//   verlet_max_rel   positions after `steps` VelocityVerlet3D steps driven by each
//                    FMM solver through `const ForceSolver3D&`
//   mixed_rms_rel    OgxAdaptiveFMM3D (mixed form) vs AdaptiveFMM3D
//   boxes_ref / boxes_ogx, maxocc_ref / maxocc_ogx   tree diagnostics
// Exit status: 0 when the run completed, 3 when a solver constructor or call
// threw (the message is printed as "error"), e.g. with no usable CUDA device.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <vector>

#include "AdaptiveFMM3D.hpp"
#include "DirectSolver3D.hpp"
#include "InitialConditions3D.hpp"
#include "Integrator3D.hpp"
#include "ogx_force_solver.hpp"

using namespace galaxy3d;

static double max_rel(const std::vector<Vec3>& a, const std::vector<Vec3>& ref) {
    double m = 0.0;
    for (size_t i = 0; i < a.size(); ++i) {
        const double d = std::sqrt(norm2(a[i] - ref[i])), r = std::sqrt(norm2(ref[i]));
        m = std::fmax(m, r > 0 ? d / r : d);
    }
    return m;
}

static double rms_rel(const std::vector<Vec3>& a, const std::vector<Vec3>& ref) {
    double s = 0.0;
    for (size_t i = 0; i < a.size(); ++i) {
        const double d = std::sqrt(norm2(a[i] - ref[i])), r = std::sqrt(norm2(ref[i]));
        const double e = r > 0 ? d / r : d;
        s += e * e;
    }
    return a.empty() ? 0.0 : std::sqrt(s / (double)a.size());
}

static std::vector<Vec3> run_verlet(const ForceSolver3D& solver, Bodies3D bodies, int steps, double dt) {
    VelocityVerlet3D vv(solver);
    vv.initialize(bodies);
    for (int s = 0; s < steps; ++s) vv.step(bodies, dt);
    return bodies.pos;
}

int main(int argc, char** argv) {
    const size_t n = argc > 1 ? (size_t)std::atol(argv[1]) : 4096;
    const int p = argc > 2 ? std::atoi(argv[2]) : 6;
    const int thr = argc > 3 ? std::atoi(argv[3]) : 32;
    const int steps = 3;
    const double dt = 0.01;
    KernelParams3D kp;
    kp.G = 1.0;
    kp.eps = 0.01;
    PlummerConfig pc;
    pc.N = n;
    pc.seed = 11;
    const Bodies3D bodies = makePlummerSphere(pc);
    try {
        const AdaptiveFMM3D ref_fmm(kp, p, thr);
        const DirectSolver3D ref_direct(kp);
        const ogx_b200::OgxAdaptiveFMM3D ogx_fmm(kp, p, thr);
        const ogx_b200::OgxAdaptiveFMM3D ogx_mixed(kp, p, thr, OGX_PREC_MIXED);
        const ogx_b200::OgxDirect3D ogx_direct(kp);
        const ForceSolver3D& a = ref_fmm;
        const ForceSolver3D& b = ogx_fmm;
        const Accelerations3D acc_ref = a.computeAccelerations(bodies);
        const Accelerations3D acc_ogx = b.computeAccelerations(bodies);
        const Accelerations3D acc_mix = static_cast<const ForceSolver3D&>(ogx_mixed).computeAccelerations(bodies);
        const Accelerations3D dir_ref = static_cast<const ForceSolver3D&>(ref_direct).computeAccelerations(bodies);
        const Accelerations3D dir_ogx = static_cast<const ForceSolver3D&>(ogx_direct).computeAccelerations(bodies);
        const std::vector<Vec3> pos_ref = run_verlet(a, bodies, steps, dt);
        const std::vector<Vec3> pos_ogx = run_verlet(b, bodies, steps, dt);
        std::printf("{\"n\": %zu, \"p\": %d, \"threshold\": %d, \"ref_name\": \"%s\", \"ogx_name\": \"%s\", "
                    "\"fmm_max_rel\": %.3e, \"direct_max_rel\": %.3e, \"verlet_steps\": %d, \"verlet_max_rel\": %.3e, "
                    "\"mixed_rms_rel\": %.3e, \"boxes_ref\": %d, \"boxes_ogx\": %d, \"maxocc_ref\": %d, "
                    "\"maxocc_ogx\": %d}\n",
                    n, p, thr, a.name(), b.name(), max_rel(acc_ogx, acc_ref), max_rel(dir_ogx, dir_ref), steps,
                    max_rel(pos_ogx, pos_ref), rms_rel(acc_mix, acc_ref), ref_fmm.lastNumBoxes, ogx_fmm.lastNumBoxes(),
                    ref_fmm.lastMaxLeafOcc, ogx_fmm.lastMaxLeafOcc());
    } catch (const std::exception& e) {
        std::printf("{\"error\": \"%s\"}\n", e.what());
        return 3;
    }
    return 0;
}
