// ref_gpu_driver.cu -- times the reference's own GPU adaptive FMM on given bodies.
//
// MEASUREMENT INFRASTRUCTURE ONLY (never shipped, never on the product path).  Built by
// oracle/Makefile into oracle/_ref/ref_gpu_fmm, linked with the reference's untouched
// src3d/gpu/AdaptiveFMM3DGPU.cu compiled where it lies.  The call timed is
//   galaxy3d::gpu::adaptiveFmm3dGpu<real>(bodies, G, eps, p, threshold, &timing)
// (src3d/gpu/AdaptiveFMM3DGPU.cu:316-334): the CPU AdaptiveOctree build and lists, the
// host-to-device copies, then the GPU passes; GpuTiming (src3d/gpu/FMM3DGPU.cuh:15-22)
// reports the three parts separately.  p must be 2, 4, 6 or 8 (the reference's own limit).
//
// usage: ref_gpu_fmm BODIES P THRESHOLD fp64|fp32 REPS [ACC_OUT]
//   BODIES : int64 n, then n x 3 doubles (positions), then n doubles (masses)
//   ACC_OUT: the accelerations of the last repetition, n x 3 doubles
// Prints one JSON line with the best-of-REPS times (seconds) of each part.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "gpu/AdaptiveFMM3DGPU.cuh"

using namespace galaxy3d;

int main(int argc, char** argv) {
    if (argc < 6) {
        std::fprintf(stderr, "usage: ref_gpu_fmm BODIES P THRESHOLD fp64|fp32 REPS [ACC_OUT]\n");
        return 2;
    }
    FILE* f = std::fopen(argv[1], "rb");
    if (!f) {
        std::fprintf(stderr, "cannot open %s\n", argv[1]);
        return 2;
    }
    int64_t n = 0;
    if (std::fread(&n, sizeof n, 1, f) != 1 || n <= 0) return 2;
    std::vector<double> pos(3 * n), mass(n);
    if (std::fread(pos.data(), 8, pos.size(), f) != pos.size() || std::fread(mass.data(), 8, mass.size(), f) != mass.size())
        return 2;
    std::fclose(f);
    const int p = std::atoi(argv[2]), thr = std::atoi(argv[3]), reps = std::max(1, std::atoi(argv[5]));
    const bool fp64 = std::string(argv[4]) == "fp64";
    if (p != 2 && p != 4 && p != 6 && p != 8) {
        std::fprintf(stderr, "the reference GPU FMM supports p = 2, 4, 6, 8 only\n");
        return 2;
    }
    Bodies3D b;
    b.resize((std::size_t)n);
    for (int64_t i = 0; i < n; ++i) {
        b.pos[i] = Vec3{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
        b.mass[i] = mass[i];
    }
    double best_tree = 1e300, best_up = 1e300, best_comp = 1e300, best_total = 1e300;
    int nboxes = 0, occ = 0;
    Accelerations3D acc;
    for (int r = 0; r < reps; ++r) {
        gpu::GpuTiming t{};
        acc = fp64 ? gpu::adaptiveFmm3dGpu<double>(b, 1.0, 0.0, p, thr, &t) : gpu::adaptiveFmm3dGpu<float>(b, 1.0, 0.0, p, thr, &t);
        best_tree = std::min(best_tree, t.treeBuildSec);
        best_up = std::min(best_up, t.uploadSec);
        best_comp = std::min(best_comp, t.computeSec);
        best_total = std::min(best_total, t.treeBuildSec + t.uploadSec + t.computeSec);
        nboxes = t.nBoxes;
        occ = t.maxLeafOcc;
    }
    if (argc > 6) {
        FILE* o = std::fopen(argv[6], "wb");
        if (o) {
            for (const Vec3& a : acc) {
                const double v[3] = {a.x, a.y, a.z};
                std::fwrite(v, 8, 3, o);
            }
            std::fclose(o);
        }
    }
    std::printf("{\"n\": %lld, \"p\": %d, \"threshold\": %d, \"precision\": \"%s\", \"reps\": %d, \"tree_build_s\": %.6f, "
                "\"upload_s\": %.6f, \"gpu_compute_s\": %.6f, \"total_s\": %.6f, \"num_boxes\": %d, \"max_leaf_occ\": %d}\n",
                (long long)n, p, thr, fp64 ? "fp64" : "fp32", reps, best_tree, best_up, best_comp, best_total, nboxes, occ);
    return 0;
}
