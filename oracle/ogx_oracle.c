/*
 * ogx_oracle.c -- CPU restatement of on-galaxy's 3D adaptive-FMM force path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the B200
 * library: only the test suite, the smoke check and the CPU-baseline leg of
 * the benchmark load it.  The product library never links or calls it.
 *
 * Every routine restates the reference algorithm (adam1sm/on-galaxy, src3d/)
 * in plain C99 with the same operation order where that matters:
 *   - DirectSolver3D::computeAccelerations      src3d/DirectSolver3D.hpp:15-34
 *   - pairAcceleration / pairPotential          src3d/Kernel3D.hpp:31-42
 *   - fmm::logFact/Acoef/jpow/idx               src3d/FmmExpansions3D.hpp:46-70
 *   - fmm::computeY                             src3d/FmmExpansions3D.hpp:75-107
 *   - gradient coefficients cz_R..dm_S          src3d/FmmExpansions3D.hpp:111-129
 *   - fmm::P2M                                  src3d/FmmExpansions3D.hpp:148-163
 *   - multipolePotential / multipoleField       src3d/FmmExpansions3D.hpp:166-200
 *   - localPotential / localField               src3d/FmmExpansions3D.hpp:203-235
 *   - fmm::M2M / M2L / L2L                      src3d/FmmExpansions3D.hpp:242-330
 *   - AdaptiveOctree::build/subdivide           src3d/AdaptiveOctree.hpp:65-134
 *   - AdaptiveOctree::adjacent                  src3d/AdaptiveOctree.hpp:58-62
 *   - AdaptiveOctree::buildLists (+helpers)     src3d/AdaptiveOctree.hpp:137-189
 *   - AdaptiveFMM3D::computeAccelerations       src3d/AdaptiveFMM3D.hpp:29-110
 *   - AdaptiveFMM3D::p2lAccum                   src3d/AdaptiveFMM3D.hpp:117-128
 *
 * Additions the reference does not have (stated, not pinned by it):
 *   - per-body potentials pot_i = -G * Phi_i (Phi = +sum q/r, the reference's
 *     sign convention in FmmExpansions3D.hpp:28-33); the FMM potential is
 *     assembled from localPotential + multipolePotential (W) + softened
 *     direct sum (U), the same decomposition the accelerations use.
 *   - integer box coordinates (ix,iy,iz) at each box's level, used to compare
 *     trees with different box numberings as canonical sets.
 *   - OpenMP over independent boxes / bodies.  Per-box arithmetic order is
 *     unchanged: levels are processed in dependency order (children before
 *     parents on the way up, parents before children on the way down).
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef double complex zc;

#define ORC_MAXDEPTH 24

/* ------------------------------------------------------------------------ */
/* constants: FmmExpansions3D.hpp:46-70                                      */
/* ------------------------------------------------------------------------ */
static double g_logfact[256];
static int g_logfact_ready = 0;

static void orc_init_tables(void) {
    if (g_logfact_ready) return;
    g_logfact[0] = 0.0;
    for (int i = 1; i < 256; ++i) g_logfact[i] = g_logfact[i - 1] + log((double)i);
    g_logfact_ready = 1;
}
static double orc_logfact(int k) { return k < 0 ? 0.0 : g_logfact[k]; }

/* A_n^m = (-1)^n / sqrt((n-m)! (n+m)!) */
static double orc_A(int n, int m) {
    const double s = (n & 1) ? -1.0 : 1.0;
    return s * exp(-0.5 * (orc_logfact(n - m) + orc_logfact(n + m)));
}
/* i^e for even e */
static double orc_ipow_even(int e) {
    long h = e / 2;
    long hm = ((h % 2) + 2) % 2;
    return hm == 0 ? 1.0 : -1.0;
}
static inline int orc_idx(int n, int m) { return n * n + n + m; }
static inline int orc_iabs(int a) { return a < 0 ? -a : a; }

/* ------------------------------------------------------------------------ */
/* spherical harmonics: FmmExpansions3D.hpp:75-107                           */
/* Y has (L+1)^2 entries; Q is caller scratch of (L+1)^2 doubles.            */
/* ------------------------------------------------------------------------ */
static double orc_harmonics(double vx, double vy, double vz, int L, zc* Y, double* Q) {
    const double r = sqrt(vx * vx + vy * vy + vz * vz);
    const int S = (L + 1) * (L + 1);
    for (int i = 0; i < S; ++i) { Y[i] = 0.0; Q[i] = 0.0; }
    const double cz = (r > 0) ? vz / r : 1.0;
    const double rxy2 = vx * vx + vy * vy;
    const double sxy = sqrt(rxy2 > 0.0 ? rxy2 : 0.0);
    const double sth = (r > 0) ? sxy / r : 0.0;
    const double phi = atan2(vy, vx);
#define QQ(n, m) Q[(n) * (L + 1) + (m)]
    QQ(0, 0) = 1.0;
    for (int m = 1; m <= L; ++m) QQ(m, m) = sth * sqrt((2.0 * m - 1.0) / (2.0 * m)) * QQ(m - 1, m - 1);
    for (int m = 0; m <= L; ++m) {
        if (m + 1 <= L) QQ(m + 1, m) = cz * sqrt(2.0 * m + 1.0) * QQ(m, m);
        for (int n = m + 2; n <= L; ++n)
            QQ(n, m) = (cz * (2.0 * n - 1.0) * QQ(n - 1, m) -
                        sqrt((double)((n - 1) * (n - 1) - m * m)) * QQ(n - 2, m)) /
                       sqrt((double)(n * n - m * m));
    }
    for (int n = 0; n <= L; ++n)
        for (int m = 0; m <= n; ++m) {
            const zc e = cos(m * phi) + I * sin(m * phi);
            const double qq = QQ(n, m);
            Y[orc_idx(n, m)] = qq * e;
            if (m > 0) Y[orc_idx(n, -m)] = qq * conj(e);
        }
#undef QQ
    return r;
}

/* derivative coefficients: FmmExpansions3D.hpp:111-129 */
static double cz_R(int n, int m) { return sqrt((double)(n * n - m * m)); }
static double cp_R(int n, int m) { const double s = (m >= 0) ? -1.0 : 1.0; return s * sqrt((double)((n - m) * (n - m - 1))); }
static double cm_R(int n, int m) { const double s = (m > 0) ? 1.0 : -1.0; return s * sqrt((double)((n + m) * (n + m - 1))); }
static double dz_S(int n, int m) { return -sqrt((double)((n + 1) * (n + 1) - m * m)); }
static double dp_S(int n, int m) { const double s = (m >= 0) ? -1.0 : 1.0; return s * sqrt((double)((n + m + 1) * (n + m + 2))); }
static double dm_S(int n, int m) { const double s = (m > 0) ? 1.0 : -1.0; return s * sqrt((double)((n - m + 1) * (n - m + 2))); }

/* scratch big enough for degree 2*ORC_PMAX */
#define ORC_PMAX 16
#define ORC_SMAX ((2 * ORC_PMAX + 2) * (2 * ORC_PMAX + 2))
typedef struct { zc Y[ORC_SMAX]; double Q[ORC_SMAX]; double rp[2 * ORC_PMAX + 4]; } orc_scratch;

/* ------------------------------------------------------------------------ */
/* operators on full complex coefficient arrays, size (p+1)^2                */
/* ------------------------------------------------------------------------ */

/* P2M accumulate: FmmExpansions3D.hpp:148-163 (body loop body) */
static void orc_p2m_add(zc* M, int p, double cx, double cy, double cz,
                        double x, double y, double z, double q, orc_scratch* s) {
    const double rho = orc_harmonics(x - cx, y - cy, z - cz, p, s->Y, s->Q);
    double rp = 1.0;
    for (int n = 0; n <= p; ++n) {
        for (int m = -n; m <= n; ++m) M[orc_idx(n, m)] += q * rp * s->Y[orc_idx(n, -m)];
        rp *= rho;
    }
}

/* multipole potential: FmmExpansions3D.hpp:166-177 */
static zc orc_mpole_pot(const zc* M, int p, double cx, double cy, double cz,
                        double tx, double ty, double tz, orc_scratch* s) {
    const double r = orc_harmonics(tx - cx, ty - cy, tz - cz, p, s->Y, s->Q);
    zc phi = 0.0;
    const double invr = 1.0 / r;
    double invrn1 = invr;
    for (int n = 0; n <= p; ++n) {
        for (int m = -n; m <= n; ++m) phi += M[orc_idx(n, m)] * s->Y[orc_idx(n, m)] * invrn1;
        invrn1 *= invr;
    }
    return phi;
}

/* multipole gradient (M2P): FmmExpansions3D.hpp:180-200 */
static void orc_mpole_field(const zc* M, int p, double cx, double cy, double cz,
                            double tx, double ty, double tz, double g[3], orc_scratch* s) {
    const double r = orc_harmonics(tx - cx, ty - cy, tz - cz, p + 1, s->Y, s->Q);
    double* invr = s->rp;
    invr[0] = 1.0;
    for (int k = 1; k < p + 3; ++k) invr[k] = invr[k - 1] / r;
#define SS(N, MM) (((N) < 0 || orc_iabs(MM) > (N)) ? (zc)0.0 : s->Y[orc_idx((N), (MM))] * invr[(N) + 1])
    zc gx = 0.0, gy = 0.0, gz = 0.0;
    for (int n = 0; n <= p; ++n)
        for (int m = -n; m <= n; ++m) {
            const zc c = M[orc_idx(n, m)];
            const zc sp = SS(n + 1, m + 1), sm = SS(n + 1, m - 1), s0 = SS(n + 1, m);
            gx += c * 0.5 * (dp_S(n, m) * sp + dm_S(n, m) * sm);
            gy += c * (-0.5 * I) * (dp_S(n, m) * sp - dm_S(n, m) * sm);
            gz += c * dz_S(n, m) * s0;
        }
#undef SS
    g[0] = creal(gx); g[1] = creal(gy); g[2] = creal(gz);
}

/* local potential: FmmExpansions3D.hpp:203-213 */
static zc orc_local_pot(const zc* L, int p, double cx, double cy, double cz,
                        double tx, double ty, double tz, orc_scratch* s) {
    const double r = orc_harmonics(tx - cx, ty - cy, tz - cz, p, s->Y, s->Q);
    zc phi = 0.0;
    double rn = 1.0;
    for (int n = 0; n <= p; ++n) {
        for (int m = -n; m <= n; ++m) phi += L[orc_idx(n, m)] * s->Y[orc_idx(n, m)] * rn;
        rn *= r;
    }
    return phi;
}

/* local gradient (L2P): FmmExpansions3D.hpp:215-235 */
static void orc_local_field(const zc* L, int p, double cx, double cy, double cz,
                            double tx, double ty, double tz, double g[3], orc_scratch* s) {
    const double r = orc_harmonics(tx - cx, ty - cy, tz - cz, p, s->Y, s->Q);
    double* rp = s->rp;
    rp[0] = 1.0;
    for (int k = 1; k < p + 2; ++k) rp[k] = rp[k - 1] * r;
#define RR(N, MM) (((N) < 0 || orc_iabs(MM) > (N)) ? (zc)0.0 : s->Y[orc_idx((N), (MM))] * rp[(N)])
    zc gx = 0.0, gy = 0.0, gz = 0.0;
    for (int n = 0; n <= p; ++n)
        for (int m = -n; m <= n; ++m) {
            const zc c = L[orc_idx(n, m)];
            const zc rpp = RR(n - 1, m + 1), rmm = RR(n - 1, m - 1), r0 = RR(n - 1, m);
            gx += c * 0.5 * (cp_R(n, m) * rpp + cm_R(n, m) * rmm);
            gy += c * (-0.5 * I) * (cp_R(n, m) * rpp - cm_R(n, m) * rmm);
            gz += c * cz_R(n, m) * r0;
        }
#undef RR
    g[0] = creal(gx); g[1] = creal(gy); g[2] = creal(gz);
}

/* M2M (returns shifted expansion into out, zeroed first): FmmExpansions3D.hpp:242-265 */
static void orc_m2m(const zc* in, int p, double ocx, double ocy, double ocz,
                    double ncx, double ncy, double ncz, zc* out, orc_scratch* s) {
    const double rho = orc_harmonics(ocx - ncx, ocy - ncy, ocz - ncz, p, s->Y, s->Q);
    double* rp = s->rp;
    rp[0] = 1.0;
    for (int n = 1; n <= p; ++n) rp[n] = rp[n - 1] * rho;
    for (int j = 0; j <= p; ++j)
        for (int k = -j; k <= j; ++k) {
            zc acc = 0.0;
            for (int n = 0; n <= j; ++n)
                for (int m = -n; m <= n; ++m) {
                    const int jj = j - n, kk = k - m;
                    if (orc_iabs(kk) > jj) continue;
                    const double J = orc_ipow_even(orc_iabs(k) - orc_iabs(m) - orc_iabs(k - m));
                    acc += in[orc_idx(jj, kk)] * J * orc_A(n, m) * orc_A(jj, kk) * rp[n] * s->Y[orc_idx(n, -m)];
                }
            out[orc_idx(j, k)] = acc / orc_A(j, k);
        }
}

/* M2L: FmmExpansions3D.hpp:273-299.  out receives the translated local. */
static void orc_m2l(const zc* in, int p, double scx, double scy, double scz,
                    double lcx, double lcy, double lcz, zc* out, orc_scratch* s) {
    const double rho = orc_harmonics(lcx - scx, lcy - scy, lcz - scz, 2 * p, s->Y, s->Q);
    double* rp = s->rp;
    rp[0] = 1.0;
    for (int n = 1; n < 2 * p + 2; ++n) rp[n] = rp[n - 1] * rho;
    for (int j = 0; j <= p; ++j)
        for (int k = -j; k <= j; ++k) {
            zc acc = 0.0;
            for (int n = 0; n <= p; ++n)
                for (int m = -n; m <= n; ++m) {
                    const int deg = j + n, ord = m - k;
                    if (orc_iabs(ord) > deg) continue;
                    const double J = orc_ipow_even(orc_iabs(k - m) - orc_iabs(k) - orc_iabs(m));
                    acc += in[orc_idx(n, m)] * J * orc_A(n, m) * orc_A(j, k) * s->Y[orc_idx(deg, ord)] /
                           (orc_A(deg, ord) * rp[deg + 1]);
                }
            out[orc_idx(j, k)] = ((j & 1) ? -1.0 : 1.0) * acc;
        }
}

/* L2L: FmmExpansions3D.hpp:307-330 */
static void orc_l2l(const zc* in, int p, double ocx, double ocy, double ocz,
                    double ncx, double ncy, double ncz, zc* out, orc_scratch* s) {
    const double rho = orc_harmonics(ncx - ocx, ncy - ocy, ncz - ocz, p, s->Y, s->Q);
    double* rp = s->rp;
    rp[0] = 1.0;
    for (int n = 1; n <= p; ++n) rp[n] = rp[n - 1] * rho;
    for (int j = 0; j <= p; ++j)
        for (int k = -j; k <= j; ++k) {
            zc acc = 0.0;
            for (int n = j; n <= p; ++n)
                for (int m = -n; m <= n; ++m) {
                    const int nn = n - j, kk = m - k;
                    if (orc_iabs(kk) > nn) continue;
                    const double J = orc_ipow_even(orc_iabs(m) - orc_iabs(m - k) - orc_iabs(k));
                    acc += in[orc_idx(n, m)] * J * orc_A(nn, kk) * orc_A(j, k) * s->Y[orc_idx(nn, kk)] * rp[nn] /
                           orc_A(n, m);
                }
            out[orc_idx(j, k)] = acc;
        }
}

/* P2L accumulate of one source: AdaptiveFMM3D.hpp:117-128 (inner body) */
static void orc_p2l_add(zc* L, int p, double cx, double cy, double cz,
                        double x, double y, double z, double q, orc_scratch* s) {
    const double rho = orc_harmonics(x - cx, y - cy, z - cz, p, s->Y, s->Q);
    double inv = 1.0 / rho;
    for (int n = 0; n <= p; ++n) {
        for (int m = -n; m <= n; ++m) L[orc_idx(n, m)] += q * s->Y[orc_idx(n, -m)] * inv;
        inv /= rho;
    }
}

/* ------------------------------------------------------------------------ */
/* exported single-operator entry points (used by the operator pin tests)    */
/* coefficient arrays are interleaved (re, im) doubles, (p+1)^2 complex.     */
/* ------------------------------------------------------------------------ */
int orc_op_p2m(int p, const double* c, int n, const double* pos, const double* q, double* M_out) {
    if (p < 0 || p > ORC_PMAX) return 1;
    orc_init_tables();
    const int S = (p + 1) * (p + 1);
    zc* M = (zc*)calloc(S, sizeof(zc));
    orc_scratch sc;
    for (int i = 0; i < n; ++i) orc_p2m_add(M, p, c[0], c[1], c[2], pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], q[i], &sc);
    for (int i = 0; i < S; ++i) { M_out[2 * i] = creal(M[i]); M_out[2 * i + 1] = cimag(M[i]); }
    free(M);
    return 0;
}

static void unpack(int S, const double* a, zc* z) { for (int i = 0; i < S; ++i) z[i] = a[2 * i] + I * a[2 * i + 1]; }
static void pack(int S, const zc* z, double* a) { for (int i = 0; i < S; ++i) { a[2 * i] = creal(z[i]); a[2 * i + 1] = cimag(z[i]); } }

/* kind: 0=M2M(c_from -> c_to), 1=M2L(source c_from -> local c_to), 2=L2L(c_from -> c_to) */
int orc_op_translate(int kind, int p, const double* c_from, const double* c_to, const double* in, double* out) {
    if (p < 0 || p > ORC_PMAX) return 1;
    orc_init_tables();
    const int S = (p + 1) * (p + 1);
    zc* zi = (zc*)malloc(S * sizeof(zc));
    zc* zo = (zc*)calloc(S, sizeof(zc));
    orc_scratch sc;
    unpack(S, in, zi);
    if (kind == 0) orc_m2m(zi, p, c_from[0], c_from[1], c_from[2], c_to[0], c_to[1], c_to[2], zo, &sc);
    else if (kind == 1) orc_m2l(zi, p, c_from[0], c_from[1], c_from[2], c_to[0], c_to[1], c_to[2], zo, &sc);
    else orc_l2l(zi, p, c_from[0], c_from[1], c_from[2], c_to[0], c_to[1], c_to[2], zo, &sc);
    pack(S, zo, out);
    free(zi); free(zo);
    return 0;
}

/* kind: 0=multipole (pot, grad), 1=local (pot, grad).  out4 = (Re pot, gx, gy, gz) per target */
int orc_op_eval(int kind, int p, const double* c, const double* coef, int nt, const double* tpos, double* out4) {
    if (p < 0 || p > ORC_PMAX) return 1;
    orc_init_tables();
    const int S = (p + 1) * (p + 1);
    zc* z = (zc*)malloc(S * sizeof(zc));
    unpack(S, coef, z);
    orc_scratch sc;
    for (int t = 0; t < nt; ++t) {
        double g[3];
        zc ph;
        if (kind == 0) {
            ph = orc_mpole_pot(z, p, c[0], c[1], c[2], tpos[3 * t], tpos[3 * t + 1], tpos[3 * t + 2], &sc);
            orc_mpole_field(z, p, c[0], c[1], c[2], tpos[3 * t], tpos[3 * t + 1], tpos[3 * t + 2], g, &sc);
        } else {
            ph = orc_local_pot(z, p, c[0], c[1], c[2], tpos[3 * t], tpos[3 * t + 1], tpos[3 * t + 2], &sc);
            orc_local_field(z, p, c[0], c[1], c[2], tpos[3 * t], tpos[3 * t + 1], tpos[3 * t + 2], g, &sc);
        }
        out4[4 * t] = creal(ph); out4[4 * t + 1] = g[0]; out4[4 * t + 2] = g[1]; out4[4 * t + 3] = g[2];
    }
    free(z);
    return 0;
}

/* source-to-local (P2L) of a point set about c: the test helper of fmm3d_tests.cpp:51-64 */
int orc_op_p2l(int p, const double* c, int n, const double* pos, const double* q, double* L_out) {
    if (p < 0 || p > ORC_PMAX) return 1;
    orc_init_tables();
    const int S = (p + 1) * (p + 1);
    zc* L = (zc*)calloc(S, sizeof(zc));
    orc_scratch sc;
    for (int i = 0; i < n; ++i) orc_p2l_add(L, p, c[0], c[1], c[2], pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], q[i], &sc);
    pack(S, L, L_out);
    free(L);
    return 0;
}

/* harmonics export (pin against closed forms, fmm3d_tests.cpp:134-157) */
int orc_op_harmonics(double x, double y, double z, int L, double* Y_out) {
    if (L < 0 || 2 * L > 2 * ORC_PMAX + 1) return 1;
    orc_scratch sc;
    orc_harmonics(x, y, z, L, sc.Y, sc.Q);
    pack((L + 1) * (L + 1), sc.Y, Y_out);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* direct all-pairs: DirectSolver3D.hpp:15-34 + Kernel3D.hpp:39-42           */
/* pos: n x 3 AoS (the Vec3 layout), acc: n x 3, pot: n or NULL              */
/* ------------------------------------------------------------------------ */
int orc_direct(long n, const double* pos, const double* mass, double G, double eps,
               double* acc, double* pot) {
    const double eps2 = eps * eps;
    for (long i = 0; i < 3 * n; ++i) acc[i] = 0.0;
    if (pot) for (long i = 0; i < n; ++i) pot[i] = 0.0;
    for (long i = 0; i < n; ++i) {
        for (long j = i + 1; j < n; ++j) {
            const double dx = pos[3 * j] - pos[3 * i], dy = pos[3 * j + 1] - pos[3 * i + 1],
                         dz = pos[3 * j + 2] - pos[3 * i + 2];
            const double r2 = (dx * dx + dy * dy + dz * dz) + eps2;
            const double inv = 1.0 / (r2 * sqrt(r2));
            const double gi = G * inv;
            const double bx = gi * dx, by = gi * dy, bz = gi * dz;
            acc[3 * i] += mass[j] * bx; acc[3 * i + 1] += mass[j] * by; acc[3 * i + 2] += mass[j] * bz;
            acc[3 * j] -= mass[i] * bx; acc[3 * j + 1] -= mass[i] * by; acc[3 * j + 2] -= mass[i] * bz;
            if (pot) {
                const double ir = 1.0 / sqrt(r2);
                pot[i] -= G * mass[j] * ir;
                pot[j] -= G * mass[i] * ir;
            }
        }
    }
    return 0;
}

/* direct for a subset of targets (spot checks at large N); per-target sum over j != i */
int orc_direct_targets(long n, const double* pos, const double* mass, double G, double eps,
                       long nt, const long* targets, double* acc, double* pot) {
    const double eps2 = eps * eps;
#pragma omp parallel for schedule(dynamic, 4)
    for (long t = 0; t < nt; ++t) {
        const long i = targets[t];
        double ax = 0, ay = 0, az = 0, ph = 0;
        for (long j = 0; j < n; ++j) {
            if (j == i) continue;
            const double dx = pos[3 * j] - pos[3 * i], dy = pos[3 * j + 1] - pos[3 * i + 1],
                         dz = pos[3 * j + 2] - pos[3 * i + 2];
            const double r2 = (dx * dx + dy * dy + dz * dz) + eps2;
            const double inv = 1.0 / (r2 * sqrt(r2));
            ax += mass[j] * inv * dx; ay += mass[j] * inv * dy; az += mass[j] * inv * dz;
            ph += mass[j] / sqrt(r2);
        }
        acc[3 * t] = G * ax; acc[3 * t + 1] = G * ay; acc[3 * t + 2] = G * az;
        if (pot) pot[t] = -G * ph;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* adaptive octree: AdaptiveOctree.hpp:31-196                                */
/* ------------------------------------------------------------------------ */
typedef struct { int* a; int n, cap; } ivec;
static void iv_push(ivec* v, int x) {
    if (v->n == v->cap) { v->cap = v->cap ? 2 * v->cap : 8; v->a = (int*)realloc(v->a, v->cap * sizeof(int)); }
    v->a[v->n++] = x;
}

typedef struct {
    int nbox, capbox;
    int* parent; int* child; int* level; int* pfirst; int* pcount; char* leaf;
    int* ix; int* iy; int* iz;
    double* cx; double* cy; double* cz; double* half;
    long n;
    int* perm;            /* reordered position -> original index */
    double* px; double* py; double* pz; double* m;
    double tol, epsFloor;
    int threshold, maxDepth;
    ivec leaves;
    ivec *col, *U, *V, *W, *X;
} orc_tree;

static int tree_new_box(orc_tree* t) {
    if (t->nbox == t->capbox) {
        int c = t->capbox ? 2 * t->capbox : 64;
        t->parent = realloc(t->parent, c * sizeof(int)); t->child = realloc(t->child, 8 * c * sizeof(int));
        t->level = realloc(t->level, c * sizeof(int)); t->pfirst = realloc(t->pfirst, c * sizeof(int));
        t->pcount = realloc(t->pcount, c * sizeof(int)); t->leaf = realloc(t->leaf, c);
        t->ix = realloc(t->ix, c * sizeof(int)); t->iy = realloc(t->iy, c * sizeof(int)); t->iz = realloc(t->iz, c * sizeof(int));
        t->cx = realloc(t->cx, c * sizeof(double)); t->cy = realloc(t->cy, c * sizeof(double));
        t->cz = realloc(t->cz, c * sizeof(double)); t->half = realloc(t->half, c * sizeof(double));
        t->capbox = c;
    }
    const int b = t->nbox++;
    t->parent[b] = -1;
    for (int o = 0; o < 8; ++o) t->child[8 * b + o] = -1;
    t->level[b] = 0; t->pfirst[b] = 0; t->pcount[b] = 0; t->leaf[b] = 1;
    t->ix[b] = t->iy[b] = t->iz[b] = 0;
    t->cx[b] = t->cy[b] = t->cz[b] = t->half[b] = 0.0;
    return b;
}

/* AdaptiveOctree::adjacent, :58-62 */
static int tree_adjacent(const orc_tree* t, int a, int b) {
    const double s = t->half[a] + t->half[b] + t->tol;
    return fabs(t->cx[a] - t->cx[b]) <= s && fabs(t->cy[a] - t->cy[b]) <= s && fabs(t->cz[a] - t->cz[b]) <= s;
}

/* AdaptiveOctree::subdivide, :99-134 (stable counting sort into octants) */
static void tree_subdivide(orc_tree* t, int bi, const double* pos, int* idx, int* tmp) {
    if (t->pcount[bi] <= t->threshold || 2.0 * t->half[bi] <= t->epsFloor || t->level[bi] >= t->maxDepth) return;
    const double ccx = t->cx[bi], ccy = t->cy[bi], ccz = t->cz[bi], chalf = t->half[bi];
    const int lo = t->pfirst[bi], hi = t->pfirst[bi] + t->pcount[bi];
    const double h2 = 0.5 * chalf;
#define OCT(j) ((pos[3 * (j)] >= ccx ? 1 : 0) | (pos[3 * (j) + 1] >= ccy ? 2 : 0) | (pos[3 * (j) + 2] >= ccz ? 4 : 0))
    int cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = lo; k < hi; ++k) ++cnt[OCT(idx[k])];
    int start[8], off[8], acc = lo;
    for (int o = 0; o < 8; ++o) { start[o] = acc; off[o] = acc; acc += cnt[o]; }
    memcpy(tmp + lo, idx + lo, (size_t)(hi - lo) * sizeof(int));
    for (int k = lo; k < hi; ++k) { const int j = tmp[k]; idx[off[OCT(j)]++] = j; }
#undef OCT
    t->leaf[bi] = 0;
    const int clevel = t->level[bi];
    const int cix = t->ix[bi], ciy = t->iy[bi], ciz = t->iz[bi];
    for (int o = 0; o < 8; ++o) {
        if (cnt[o] == 0) continue;
        const int ch = tree_new_box(t);
        t->parent[ch] = bi; t->level[ch] = clevel + 1; t->half[ch] = h2;
        t->cx[ch] = ccx + ((o & 1) ? h2 : -h2);
        t->cy[ch] = ccy + ((o & 2) ? h2 : -h2);
        t->cz[ch] = ccz + ((o & 4) ? h2 : -h2);
        t->pfirst[ch] = start[o]; t->pcount[ch] = cnt[o];
        t->ix[ch] = 2 * cix + (o & 1); t->iy[ch] = 2 * ciy + ((o >> 1) & 1); t->iz[ch] = 2 * ciz + ((o >> 2) & 1);
        t->child[8 * bi + o] = ch;
    }
    for (int o = 0; o < 8; ++o) {
        const int ch = t->child[8 * bi + o];
        if (ch >= 0) tree_subdivide(t, ch, pos, idx, tmp);
    }
}

/* AdaptiveOctree::build, :65-97 */
static void tree_build(orc_tree* t, long n, const double* pos, const double* mass, int threshold, double epsFloor) {
    memset(t, 0, sizeof(*t));
    t->threshold = threshold; t->epsFloor = epsFloor; t->maxDepth = ORC_MAXDEPTH; t->n = n;
    int* idx = (int*)malloc((n > 0 ? n : 1) * sizeof(int));
    int* tmp = (int*)malloc((n > 0 ? n : 1) * sizeof(int));
    for (long i = 0; i < n; ++i) idx[i] = (int)i;
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (long i = 0; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            const double v = pos[3 * i + a];
            lo[a] = (v < lo[a]) ? v : lo[a];     /* std::min(lo, v) */
            hi[a] = (hi[a] < v) ? v : hi[a];     /* std::max(hi, v) */
        }
    const double cx = 0.5 * (lo[0] + hi[0]), cy = 0.5 * (lo[1] + hi[1]), cz = 0.5 * (lo[2] + hi[2]);
    double ext = hi[0] - lo[0];
    if (ext < hi[1] - lo[1]) ext = hi[1] - lo[1];
    if (ext < hi[2] - lo[2]) ext = hi[2] - lo[2];
    double half = 0.5 * ext;
    if (!(half > 0)) half = 1.0;
    half *= 1.0 + 1e-9;
    t->tol = 1e-9 * half;
    const int root = tree_new_box(t);
    t->cx[root] = cx; t->cy[root] = cy; t->cz[root] = cz; t->half[root] = half;
    t->pfirst[root] = 0; t->pcount[root] = (int)n;
    tree_subdivide(t, root, pos, idx, tmp);
    t->perm = idx;
    t->px = malloc((n > 0 ? n : 1) * sizeof(double)); t->py = malloc((n > 0 ? n : 1) * sizeof(double));
    t->pz = malloc((n > 0 ? n : 1) * sizeof(double)); t->m = malloc((n > 0 ? n : 1) * sizeof(double));
    for (long k = 0; k < n; ++k) {
        const int j = idx[k];
        t->px[k] = pos[3 * j]; t->py[k] = pos[3 * j + 1]; t->pz[k] = pos[3 * j + 2]; t->m[k] = mass ? mass[j] : 0.0;
    }
    free(tmp);
    for (int b = 0; b < t->nbox; ++b) if (t->leaf[b] && t->pcount[b] > 0) iv_push(&t->leaves, b);
}

/* collectAdjLeaves, :176-180 */
static void tree_collect_adj_leaves(const orc_tree* t, int node, int b, ivec* out) {
    if (!tree_adjacent(t, node, b)) return;
    if (t->leaf[node]) { if (t->pcount[node] > 0) iv_push(out, node); return; }
    for (int o = 0; o < 8; ++o) if (t->child[8 * node + o] >= 0) tree_collect_adj_leaves(t, t->child[8 * node + o], b, out);
}
/* descendW, :181-189 */
static void tree_descend_w(orc_tree* t, int node, int b) {
    for (int o = 0; o < 8; ++o) {
        const int ch = t->child[8 * node + o];
        if (ch < 0) continue;
        if (!tree_adjacent(t, ch, b)) iv_push(&t->W[b], ch);
        else if (!t->leaf[ch]) tree_descend_w(t, ch, b);
    }
}

/* buildLists, :137-174 */
static void tree_lists(orc_tree* t) {
    const int nb = t->nbox;
    t->col = calloc(nb, sizeof(ivec)); t->U = calloc(nb, sizeof(ivec)); t->V = calloc(nb, sizeof(ivec));
    t->W = calloc(nb, sizeof(ivec)); t->X = calloc(nb, sizeof(ivec));
    iv_push(&t->col[0], 0);
    for (int b = 1; b < nb; ++b) {
        const int par = t->parent[b];
        for (int q = 0; q < t->col[par].n; ++q) {
            const int pc = t->col[par].a[q];
            for (int o = 0; o < 8; ++o) {
                const int c = t->child[8 * pc + o];
                if (c >= 0 && tree_adjacent(t, b, c)) iv_push(&t->col[b], c);
            }
        }
    }
    for (int b = 1; b < nb; ++b) {
        const int par = t->parent[b];
        for (int q = 0; q < t->col[par].n; ++q) {
            const int pc = t->col[par].a[q];
            for (int o = 0; o < 8; ++o) {
                const int c = t->child[8 * pc + o];
                if (c >= 0 && !tree_adjacent(t, b, c)) iv_push(&t->V[b], c);
            }
        }
    }
    for (int l = 0; l < t->leaves.n; ++l) { const int b = t->leaves.a[l]; tree_collect_adj_leaves(t, 0, b, &t->U[b]); }
    for (int l = 0; l < t->leaves.n; ++l) {
        const int b = t->leaves.a[l];
        for (int q = 0; q < t->col[b].n; ++q) {
            const int c = t->col[b].a[q];
            if (c != b && !t->leaf[c]) tree_descend_w(t, c, b);
        }
    }
    for (int l = 0; l < t->leaves.n; ++l) {
        const int c = t->leaves.a[l];
        for (int q = 0; q < t->W[c].n; ++q) iv_push(&t->X[t->W[c].a[q]], c);
    }
}

static void tree_free(orc_tree* t) {
    free(t->parent); free(t->child); free(t->level); free(t->pfirst); free(t->pcount); free(t->leaf);
    free(t->ix); free(t->iy); free(t->iz); free(t->cx); free(t->cy); free(t->cz); free(t->half);
    free(t->perm); free(t->px); free(t->py); free(t->pz); free(t->m); free(t->leaves.a);
    ivec* ls[5] = {t->col, t->U, t->V, t->W, t->X};
    for (int k = 0; k < 5; ++k) {
        if (!ls[k]) continue;
        for (int b = 0; b < t->nbox; ++b) free(ls[k][b].a);
        free(ls[k]);
    }
    memset(t, 0, sizeof(*t));
}

/* ---- exported tree handle (for list parity tests) ---------------------- */
void* orc_tree_create(long n, const double* pos, int threshold, double epsFloor) {
    orc_tree* t = (orc_tree*)malloc(sizeof(orc_tree));
    tree_build(t, n, pos, NULL, threshold, epsFloor);
    tree_lists(t);
    return t;
}
void orc_tree_destroy(void* h) { if (h) { tree_free((orc_tree*)h); free(h); } }

/* sizes[0]=nbox, [1]=nleaf, [2..6]=total |colleague|,|U|,|V|,|W|,|X| */
void orc_tree_sizes(void* h, long* sizes) {
    orc_tree* t = (orc_tree*)h;
    sizes[0] = t->nbox; sizes[1] = t->leaves.n;
    ivec* ls[5] = {t->col, t->U, t->V, t->W, t->X};
    for (int k = 0; k < 5; ++k) { long s = 0; for (int b = 0; b < t->nbox; ++b) s += ls[k][b].n; sizes[2 + k] = s; }
}
/* boxes: int32 rows of (level, ix, iy, iz, parent, leaf, pfirst, pcount) -> nbox x 8;
   centers: nbox x 4 doubles (cx, cy, cz, half); perm: n ints.
   which: 0..4 = colleague, U, V, W, X; off: nbox+1, idx: total */
void orc_tree_boxes(void* h, int* boxes, double* centers, int* perm) {
    orc_tree* t = (orc_tree*)h;
    for (int b = 0; b < t->nbox; ++b) {
        int* r = boxes + 8 * b;
        r[0] = t->level[b]; r[1] = t->ix[b]; r[2] = t->iy[b]; r[3] = t->iz[b];
        r[4] = t->parent[b]; r[5] = t->leaf[b]; r[6] = t->pfirst[b]; r[7] = t->pcount[b];
        if (centers) { centers[4 * b] = t->cx[b]; centers[4 * b + 1] = t->cy[b]; centers[4 * b + 2] = t->cz[b]; centers[4 * b + 3] = t->half[b]; }
    }
    if (perm) for (long k = 0; k < t->n; ++k) perm[k] = t->perm[k];
}
void orc_tree_list(void* h, int which, long* off, int* idx) {
    orc_tree* t = (orc_tree*)h;
    ivec* ls[5] = {t->col, t->U, t->V, t->W, t->X};
    ivec* L = ls[which];
    long e = 0;
    for (int b = 0; b < t->nbox; ++b) {
        off[b] = e;
        for (int q = 0; q < L[b].n; ++q) idx[e++] = L[b].a[q];
    }
    off[t->nbox] = e;
}

/* ------------------------------------------------------------------------ */
/* adaptive FMM: AdaptiveFMM3D.hpp:29-110 (+ potentials)                     */
/* ------------------------------------------------------------------------ */
int orc_adaptive_fmm(long n, const double* pos, const double* mass, double G, double eps,
                     int p, int threshold, double* acc, double* pot) {
    if (p < 1 || p > ORC_PMAX || threshold < 1) return 1;
    orc_init_tables();
    for (long i = 0; i < 3 * n; ++i) acc[i] = 0.0;
    if (pot) for (long i = 0; i < n; ++i) pot[i] = 0.0;
    if (n == 0) return 0;
    orc_tree t;
    tree_build(&t, n, pos, mass, threshold, eps);
    tree_lists(&t);
    const int nb = t.nbox;
    const int S = (p + 1) * (p + 1);
    zc* M = (zc*)calloc((size_t)nb * S, sizeof(zc));
    zc* L = (zc*)calloc((size_t)nb * S, sizeof(zc));
    int maxlev = 0;
    for (int b = 0; b < nb; ++b) if (t.level[b] > maxlev) maxlev = t.level[b];
    /* boxes grouped per level, each group in index order */
    int* lvcnt = (int*)calloc(maxlev + 2, sizeof(int));
    for (int b = 0; b < nb; ++b) lvcnt[t.level[b] + 1]++;
    for (int l = 0; l <= maxlev; ++l) lvcnt[l + 1] += lvcnt[l];
    int* lvbox = (int*)malloc(nb * sizeof(int));
    {
        int* cur = (int*)malloc((maxlev + 1) * sizeof(int));
        for (int l = 0; l <= maxlev; ++l) cur[l] = lvcnt[l];
        for (int b = 0; b < nb; ++b) lvbox[cur[t.level[b]]++] = b;
        free(cur);
    }

    /* upward: P2M per leaf (:53-61) */
#pragma omp parallel for schedule(dynamic, 16)
    for (int l = 0; l < t.leaves.n; ++l) {
        orc_scratch sc;
        const int b = t.leaves.a[l];
        for (int k = t.pfirst[b]; k < t.pfirst[b] + t.pcount[b]; ++k)
            orc_p2m_add(M + (size_t)b * S, p, t.cx[b], t.cy[b], t.cz[b], t.px[k], t.py[k], t.pz[k], t.m[k], &sc);
    }
    /* M2M bottom-up (:62-71); reference order is reverse index, per box children o=0..7 */
    for (int lev = maxlev; lev >= 0; --lev) {
#pragma omp parallel for schedule(dynamic, 8)
        for (int q = lvcnt[lev]; q < lvcnt[lev + 1]; ++q) {
            const int b = lvbox[q];
            if (t.leaf[b]) continue;
            orc_scratch sc;
            zc sh[(ORC_PMAX + 1) * (ORC_PMAX + 1)];
            for (int o = 0; o < 8; ++o) {
                const int ch = t.child[8 * b + o];
                if (ch < 0) continue;
                orc_m2m(M + (size_t)ch * S, p, t.cx[ch], t.cy[ch], t.cz[ch], t.cx[b], t.cy[b], t.cz[b], sh, &sc);
                for (int s = 0; s < S; ++s) M[(size_t)b * S + s] += sh[s];
            }
        }
    }
    /* downward (:74-85): L2L from parent, V -> M2L, X -> P2L */
    for (int lev = 0; lev <= maxlev; ++lev) {
#pragma omp parallel for schedule(dynamic, 8)
        for (int q = lvcnt[lev]; q < lvcnt[lev + 1]; ++q) {
            const int b = lvbox[q];
            orc_scratch sc;
            zc tmp[(ORC_PMAX + 1) * (ORC_PMAX + 1)];
            zc* Lb = L + (size_t)b * S;
            if (t.parent[b] >= 0) {
                const int pa = t.parent[b];
                orc_l2l(L + (size_t)pa * S, p, t.cx[pa], t.cy[pa], t.cz[pa], t.cx[b], t.cy[b], t.cz[b], tmp, &sc);
                for (int s = 0; s < S; ++s) Lb[s] += tmp[s];
            }
            for (int v = 0; v < t.V[b].n; ++v) {
                const int c = t.V[b].a[v];
                orc_m2l(M + (size_t)c * S, p, t.cx[c], t.cy[c], t.cz[c], t.cx[b], t.cy[b], t.cz[b], tmp, &sc);
                for (int s = 0; s < S; ++s) Lb[s] += tmp[s];
            }
            for (int x = 0; x < t.X[b].n; ++x) {
                const int c = t.X[b].a[x];
                for (int k = t.pfirst[c]; k < t.pfirst[c] + t.pcount[c]; ++k)
                    orc_p2l_add(Lb, p, t.cx[b], t.cy[b], t.cz[b], t.px[k], t.py[k], t.pz[k], t.m[k], &sc);
            }
        }
    }
    /* leaves (:89-108): L2P + W -> M2P + U -> P2P (softened), acc[orig] = G (far + near) */
    const double eps2 = eps * eps;
#pragma omp parallel for schedule(dynamic, 4)
    for (int l = 0; l < t.leaves.n; ++l) {
        orc_scratch sc;
        const int b = t.leaves.a[l];
        for (int ti = t.pfirst[b]; ti < t.pfirst[b] + t.pcount[b]; ++ti) {
            const double zx = t.px[ti], zy = t.py[ti], zz = t.pz[ti];
            double f[3], g[3];
            orc_local_field(L + (size_t)b * S, p, t.cx[b], t.cy[b], t.cz[b], zx, zy, zz, f, &sc);
            double phi = 0.0;
            if (pot) phi = creal(orc_local_pot(L + (size_t)b * S, p, t.cx[b], t.cy[b], t.cz[b], zx, zy, zz, &sc));
            for (int w = 0; w < t.W[b].n; ++w) {
                const int c = t.W[b].a[w];
                orc_mpole_field(M + (size_t)c * S, p, t.cx[c], t.cy[c], t.cz[c], zx, zy, zz, g, &sc);
                f[0] += g[0]; f[1] += g[1]; f[2] += g[2];
                if (pot) phi += creal(orc_mpole_pot(M + (size_t)c * S, p, t.cx[c], t.cy[c], t.cz[c], zx, zy, zz, &sc));
            }
            double nx = 0, ny = 0, nz = 0, nphi = 0;
            for (int u = 0; u < t.U[b].n; ++u) {
                const int uc = t.U[b].a[u];
                for (int j = t.pfirst[uc]; j < t.pfirst[uc] + t.pcount[uc]; ++j) {
                    if (j == ti) continue;
                    const double dx = t.px[j] - zx, dy = t.py[j] - zy, dz = t.pz[j] - zz;
                    const double r2 = (dx * dx + dy * dy + dz * dz) + eps2;
                    const double w = t.m[j] / (r2 * sqrt(r2));
                    nx += w * dx; ny += w * dy; nz += w * dz;
                    if (pot) nphi += t.m[j] / sqrt(r2);
                }
            }
            const int oi = t.perm[ti];
            acc[3 * oi] = G * (f[0] + nx); acc[3 * oi + 1] = G * (f[1] + ny); acc[3 * oi + 2] = G * (f[2] + nz);
            if (pot) pot[oi] = -G * (phi + nphi);
        }
    }
    free(lvcnt); free(lvbox); free(M); free(L);
    tree_free(&t);
    return 0;
}

/* error metric of adaptive_tests.cpp:40-50: out[0]=max_rel, out[1]=rms_rel */
void orc_rel_err(long n, const double* ref, const double* got, double* out) {
    double amax = 0;
    for (long i = 0; i < n; ++i) {
        const double a = sqrt(ref[3 * i] * ref[3 * i] + ref[3 * i + 1] * ref[3 * i + 1] + ref[3 * i + 2] * ref[3 * i + 2]);
        if (a > amax) amax = a;
    }
    const double fl = 1e-30 + 1e-6 * amax;
    double mx = 0, num = 0, den = 0;
    for (long i = 0; i < n; ++i) {
        const double dx = got[3 * i] - ref[3 * i], dy = got[3 * i + 1] - ref[3 * i + 1], dz = got[3 * i + 2] - ref[3 * i + 2];
        const double e = sqrt(dx * dx + dy * dy + dz * dz);
        const double a = sqrt(ref[3 * i] * ref[3 * i] + ref[3 * i + 1] * ref[3 * i + 1] + ref[3 * i + 2] * ref[3 * i + 2]);
        const double r = e / (a > fl ? a : fl);
        if (r > mx) mx = r;
        num += e * e;
        den += a * a;
    }
    out[0] = mx;
    out[1] = den > 0 ? sqrt(num / den) : 0.0;
}
