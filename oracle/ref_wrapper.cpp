// ref_wrapper.cpp -- C entry points around the UNMODIFIED reference headers.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile against the
// reference's src3d/ headers (header-only C++17) into oracle/_ref/libogx_ref.so.
// It is used to (1) pin the C restatement in ogx_oracle.c, (2) generate the
// golden fixtures under tests/golden/, and (3) time the reference's own CPU
// AdaptiveFMM3D as the benchmark's reference arm.  Nothing here is shipped.
//
// Wrapped reference entry points:
//   galaxy3d::DirectSolver3D::computeAccelerations   src3d/DirectSolver3D.hpp:15
//   galaxy3d::AdaptiveFMM3D::computeAccelerations    src3d/AdaptiveFMM3D.hpp:29
//   galaxy3d::AdaptiveOctree::build / buildLists     src3d/AdaptiveOctree.hpp:65,137
//   galaxy3d::makePlummerSphere                      src3d/InitialConditions3D.hpp:100
//   galaxy3d::makeDisk                               src3d/gpu/GalaxyIC.hpp:43
//   galaxy3d::fmm::{computeY,P2M,M2M,M2L,L2L,...}    src3d/FmmExpansions3D.hpp
// plus the seeded geometry of the reference's operator unit tests
// (src3d/fmm3d_tests.cpp:85-109, 196-288) and of adaptive_tests.cpp:27-37,
// re-expressed here with the same std:: distributions and call order so the
// generated points are bit-identical to the ones those tests use.
#include <cstdint>
#include <cstring>
#include <random>
#include <thread>
#include <vector>

#include "AdaptiveFMM3D.hpp"
#include "AdaptiveOctree.hpp"
#include "DirectSolver3D.hpp"
#include "FmmExpansions3D.hpp"
#include "InitialConditions3D.hpp"
#include "gpu/GalaxyIC.hpp"

using namespace galaxy3d;

namespace {
Bodies3D toBodies(long n, const double* pos, const double* mass) {
    Bodies3D b;
    b.resize((std::size_t)n);
    for (long i = 0; i < n; ++i) {
        b.pos[i] = Vec3{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
        b.mass[i] = mass ? mass[i] : 0.0;
    }
    return b;
}
void fromAcc(const Accelerations3D& a, double* out) {
    for (std::size_t i = 0; i < a.size(); ++i) { out[3 * i] = a[i].x; out[3 * i + 1] = a[i].y; out[3 * i + 2] = a[i].z; }
}
void fromBodies(const Bodies3D& b, double* pos, double* vel, double* mass) {
    for (std::size_t i = 0; i < b.size(); ++i) {
        if (pos) { pos[3 * i] = b.pos[i].x; pos[3 * i + 1] = b.pos[i].y; pos[3 * i + 2] = b.pos[i].z; }
        if (vel) { vel[3 * i] = b.vel[i].x; vel[3 * i + 1] = b.vel[i].y; vel[3 * i + 2] = b.vel[i].z; }
        if (mass) mass[i] = b.mass[i];
    }
}
Vec3 randDir(std::mt19937& rng) {  // geometry helper of fmm3d_tests.cpp:85-90
    std::uniform_real_distribution<double> u(0, 1);
    const double TAU = 2.0 * std::acos(-1.0);
    const double cz = 2 * u(rng) - 1, sz = std::sqrt(std::max(0.0, 1 - cz * cz)), ph = TAU * u(rng);
    return Vec3{sz * std::cos(ph), sz * std::sin(ph), cz};
}
}  // namespace

extern "C" {

int ref_direct(long n, const double* pos, const double* mass, double G, double eps, double* acc) {
    const Bodies3D b = toBodies(n, pos, mass);
    fromAcc(DirectSolver3D(KernelParams3D{G, eps}).computeAccelerations(b), acc);
    return 0;
}

int ref_adaptive_fmm(long n, const double* pos, const double* mass, double G, double eps, int p, int thr,
                     double* acc, int* stats /* [maxLeafOcc, numBoxes] or NULL */) {
    const Bodies3D b = toBodies(n, pos, mass);
    AdaptiveFMM3D f(KernelParams3D{G, eps}, p, thr);
    fromAcc(f.computeAccelerations(b), acc);
    if (stats) { stats[0] = f.lastMaxLeafOcc; stats[1] = f.lastNumBoxes; }
    return 0;
}

// Ensemble throughput of the reference CPU solver: `nsys` independent systems
// (each n bodies, concatenated) evaluated by `threads` worker threads, one
// AdaptiveFMM3D per system.  fmm::logFact's lazily built static table is
// initialised on the calling thread first so the workers only read it.
int ref_adaptive_fmm_batch(int nsys, long n, const double* pos, const double* mass, double G, double eps,
                           int p, int thr, int threads, double* acc) {
    (void)fmm::logFact(1);
    std::vector<std::thread> ws;
    for (int w = 0; w < threads; ++w)
        ws.emplace_back([=]() {
            for (int s = w; s < nsys; s += threads) {
                const Bodies3D b = toBodies(n, pos + 3 * n * (long)s, mass + n * (long)s);
                AdaptiveFMM3D f(KernelParams3D{G, eps}, p, thr);
                fromAcc(f.computeAccelerations(b), acc + 3 * n * (long)s);
            }
        });
    for (auto& t : ws) t.join();
    return 0;
}

int ref_plummer(long n, unsigned seed, double a, double* pos, double* vel, double* mass) {
    PlummerConfig pc;
    pc.N = (std::size_t)n; pc.a = a; pc.total_mass = 1.0; pc.G = 1.0; pc.seed = seed;
    fromBodies(makePlummerSphere(pc), pos, vel, mass);
    return 0;
}

// adaptive_tests.cpp:27-33 generator (uniform cube, masses U(0.5,1.5))
int ref_uniform_cube(long n, unsigned seed, double* pos, double* mass) {
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> u(-1.0, 1.0), um(0.5, 1.5);
    for (long i = 0; i < n; ++i) {
        const double x = u(rng), y = u(rng), z = u(rng);  // brace-init order: x, y, z
        pos[3 * i] = x; pos[3 * i + 1] = y; pos[3 * i + 2] = z;
        mass[i] = um(rng);
    }
    return 0;
}

int ref_disk(long n, unsigned seed, double* pos, double* mass) {
    DiskParams dp; dp.N = (std::size_t)n; dp.seed = seed;
    fromBodies(makeDisk(dp), pos, nullptr, mass);
    return 0;
}

// fmm3d_tests.cpp:91-109 point sets: kind 0 = ball(c, rad, n, seed) -> pos+q,
// kind 1 = shell(c, rmin=rad, rmax=rad2, n, seed) -> pos only.
int ref_test_points(int kind, const double* c, double rad, double rad2, int n, unsigned seed,
                    double* pos, double* q) {
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> u(0, 1);
    const Vec3 cc{c[0], c[1], c[2]};
    for (int i = 0; i < n; ++i) {
        // Same expressions as the test file so the compiler sequences the
        // RNG calls inside them identically.
        Vec3 v;
        if (kind == 0) {
            v = cc + (rad * std::cbrt(u(rng))) * randDir(rng);
            const double qq = 0.5 + u(rng);
            if (q) q[i] = qq;
        } else {
            v = cc + (rad + (rad2 - rad) * u(rng)) * randDir(rng);
        }
        pos[3 * i] = v.x; pos[3 * i + 1] = v.y; pos[3 * i + 2] = v.z;
    }
    return 0;
}

int ref_harmonics(double x, double y, double z, int L, double* Y) {
    std::vector<fmm::Complex> v;
    fmm::computeY(Vec3{x, y, z}, L, v);
    for (std::size_t i = 0; i < v.size(); ++i) { Y[2 * i] = v[i].real(); Y[2 * i + 1] = v[i].imag(); }
    return 0;
}

int ref_p2m(int p, const double* c, int n, const double* pos, const double* q, double* M) {
    std::vector<Vec3> ps(n); std::vector<double> qs(q, q + n);
    for (int i = 0; i < n; ++i) ps[i] = Vec3{pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    const fmm::Multipole mp = fmm::P2M(Vec3{c[0], c[1], c[2]}, ps, qs, p);
    for (std::size_t i = 0; i < mp.M.size(); ++i) { M[2 * i] = mp.M[i].real(); M[2 * i + 1] = mp.M[i].imag(); }
    return 0;
}

int ref_translate(int kind, int p, const double* cf, const double* ct, const double* in, double* out) {
    const int S = (p + 1) * (p + 1);
    if (kind == 0 || kind == 1) {
        fmm::Multipole m(Vec3{cf[0], cf[1], cf[2]}, p);
        for (int i = 0; i < S; ++i) m.M[i] = fmm::Complex{in[2 * i], in[2 * i + 1]};
        if (kind == 0) {
            const fmm::Multipole o = fmm::M2M(m, Vec3{ct[0], ct[1], ct[2]});
            for (int i = 0; i < S; ++i) { out[2 * i] = o.M[i].real(); out[2 * i + 1] = o.M[i].imag(); }
        } else {
            const fmm::Local o = fmm::M2L(m, Vec3{ct[0], ct[1], ct[2]});
            for (int i = 0; i < S; ++i) { out[2 * i] = o.L[i].real(); out[2 * i + 1] = o.L[i].imag(); }
        }
    } else {
        fmm::Local l(Vec3{cf[0], cf[1], cf[2]}, p);
        for (int i = 0; i < S; ++i) l.L[i] = fmm::Complex{in[2 * i], in[2 * i + 1]};
        const fmm::Local o = fmm::L2L(l, Vec3{ct[0], ct[1], ct[2]});
        for (int i = 0; i < S; ++i) { out[2 * i] = o.L[i].real(); out[2 * i + 1] = o.L[i].imag(); }
    }
    return 0;
}

int ref_eval(int kind, int p, const double* c, const double* coef, int nt, const double* tpos, double* out4) {
    const int S = (p + 1) * (p + 1);
    for (int t = 0; t < nt; ++t) {
        const Vec3 tt{tpos[3 * t], tpos[3 * t + 1], tpos[3 * t + 2]};
        fmm::Complex ph; Vec3 g;
        if (kind == 0) {
            fmm::Multipole m(Vec3{c[0], c[1], c[2]}, p);
            for (int i = 0; i < S; ++i) m.M[i] = fmm::Complex{coef[2 * i], coef[2 * i + 1]};
            ph = fmm::multipolePotential(m, tt); g = fmm::multipoleField(m, tt);
        } else {
            fmm::Local l(Vec3{c[0], c[1], c[2]}, p);
            for (int i = 0; i < S; ++i) l.L[i] = fmm::Complex{coef[2 * i], coef[2 * i + 1]};
            ph = fmm::localPotential(l, tt); g = fmm::localField(l, tt);
        }
        out4[4 * t] = ph.real(); out4[4 * t + 1] = g.x; out4[4 * t + 2] = g.y; out4[4 * t + 3] = g.z;
    }
    return 0;
}

// ---- tree + lists export --------------------------------------------------
struct RefTree {
    AdaptiveOctree t;
    std::vector<int> ix, iy, iz;
};

void* ref_tree_create(long n, const double* pos, int thr, double epsFloor) {
    RefTree* r = new RefTree;
    const Bodies3D b = toBodies(n, pos, nullptr);
    r->t.build(b, thr, epsFloor);
    r->t.buildLists();
    const int nb = (int)r->t.box.size();
    r->ix.assign(nb, 0); r->iy.assign(nb, 0); r->iz.assign(nb, 0);
    for (int p = 0; p < nb; ++p)  // parents precede children in box order
        for (int o = 0; o < 8; ++o) {
            const int c = r->t.box[p].child[o];
            if (c < 0) continue;
            r->ix[c] = 2 * r->ix[p] + (o & 1);
            r->iy[c] = 2 * r->iy[p] + ((o >> 1) & 1);
            r->iz[c] = 2 * r->iz[p] + ((o >> 2) & 1);
        }
    return r;
}
void ref_tree_destroy(void* h) { delete (RefTree*)h; }
void ref_tree_sizes(void* h, long* s) {
    RefTree* r = (RefTree*)h;
    const AdaptiveOctree& t = r->t;
    s[0] = (long)t.box.size(); s[1] = (long)t.leaves.size();
    const std::vector<std::vector<int>>* ls[5] = {&t.colleague, &t.U, &t.V, &t.W, &t.X};
    for (int k = 0; k < 5; ++k) { long z = 0; for (auto& v : *ls[k]) z += (long)v.size(); s[2 + k] = z; }
}
void ref_tree_boxes(void* h, int* boxes, double* centers, int* perm) {
    RefTree* r = (RefTree*)h;
    const AdaptiveOctree& t = r->t;
    for (std::size_t b = 0; b < t.box.size(); ++b) {
        const ABox& x = t.box[b];
        int* o = boxes + 8 * b;
        o[0] = x.level; o[1] = r->ix[b]; o[2] = r->iy[b]; o[3] = r->iz[b];
        o[4] = x.parent; o[5] = x.leaf ? 1 : 0; o[6] = x.pfirst; o[7] = x.pcount;
        if (centers) { centers[4 * b] = x.cx; centers[4 * b + 1] = x.cy; centers[4 * b + 2] = x.cz; centers[4 * b + 3] = x.half; }
    }
    if (perm) for (std::size_t k = 0; k < t.origIndex.size(); ++k) perm[k] = t.origIndex[k];
}
void ref_tree_list(void* h, int which, long* off, int* idx) {
    RefTree* r = (RefTree*)h;
    const AdaptiveOctree& t = r->t;
    const std::vector<std::vector<int>>* ls[5] = {&t.colleague, &t.U, &t.V, &t.W, &t.X};
    const auto& L = *ls[which];
    long e = 0;
    for (std::size_t b = 0; b < L.size(); ++b) {
        off[b] = e;
        for (int c : L[b]) idx[e++] = c;
    }
    off[L.size()] = e;
}

}  // extern "C"
