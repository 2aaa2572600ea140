// ogx_tables.cpp -- level-independent translation matrices, built on the host.
//
// The reference translates expansions with the naive O(p^4) GR1997 formulas
// (src3d/FmmExpansions3D.hpp:242-330), recomputing spherical harmonics for
// every box pair.  Here every translation is precomputed ONCE per order p as
// a real K x K matrix (K = (p+1)^2) acting on scaled coefficients
//     M'_n = M_n / side^n,   L'_n = L_n * side^n,
// which makes each operator independent of the tree level:
//   M2M (child octant s):  M'_parent = MM_s  M'_child         (FmmExpansions3D.hpp:242)
//   L2L (child octant s):  L'_child  = LL_s  L'_parent        (FmmExpansions3D.hpp:307)
//   M2L (offset o):        L'_target += (1/side) T_o M'_source (FmmExpansions3D.hpp:273)
// o = (source centre - target centre) / side is an integer vector in
// [-3,3]^3 \ [-1,1]^3 for every V-list pair (children of the parent's
// colleagues that are not adjacent, src3d/AdaptiveOctree.hpp:153-161).
// Coefficients are evaluated in long double from the same harmonics (no
// Condon-Shortley phase, FmmExpansions3D.hpp:16-21) and A_n^m constants.
#include <cmath>
#include <complex>
#include <vector>

#include "ogx_internal.cuh"

namespace ogx {
namespace {

using ld = long double;
using zl = std::complex<long double>;

inline int cidx(int n, int m) { return n * n + n + m; }
inline int iabs(int a) { return a < 0 ? -a : a; }

ld fact(int k) {
    ld f = 1.0L;
    for (int i = 2; i <= k; ++i) f *= (ld)i;
    return f;
}
// A_n^m = (-1)^n / sqrt((n-m)!(n+m)!)   (FmmExpansions3D.hpp:56-60)
ld Acoef(int n, int m) {
    const ld s = (n & 1) ? -1.0L : 1.0L;
    return s / std::sqrt(fact(n - m) * fact(n + m));
}
// i^e for even e   (FmmExpansions3D.hpp:62-67)
ld jpow(int e) {
    const int h = e / 2;
    return (((h % 2) + 2) % 2 == 0) ? 1.0L : -1.0L;
}

// Y_n^m(direction of v), n <= L, full m range; returns |v|  (FmmExpansions3D.hpp:75-107)
ld harmonics(ld x, ld y, ld z, int L, std::vector<zl>& Y) {
    const ld r = std::sqrt(x * x + y * y + z * z);
    Y.assign((L + 1) * (L + 1), zl(0, 0));
    const ld cz = (r > 0) ? z / r : 1.0L;
    const ld sth = (r > 0) ? std::sqrt(std::max((ld)0, x * x + y * y)) / r : 0.0L;
    const ld phi = std::atan2(y, x);
    std::vector<ld> Q((L + 1) * (L + 1), 0.0L);
    auto q = [&](int n, int m) -> ld& { return Q[n * (L + 1) + m]; };
    q(0, 0) = 1.0L;
    for (int m = 1; m <= L; ++m) q(m, m) = sth * std::sqrt((2.0L * m - 1.0L) / (2.0L * m)) * q(m - 1, m - 1);
    for (int m = 0; m <= L; ++m) {
        if (m + 1 <= L) q(m + 1, m) = cz * std::sqrt(2.0L * m + 1.0L) * q(m, m);
        for (int n = m + 2; n <= L; ++n)
            q(n, m) = (cz * (2.0L * n - 1.0L) * q(n - 1, m) - std::sqrt((ld)((n - 1) * (n - 1) - m * m)) * q(n - 2, m)) /
                      std::sqrt((ld)(n * n - m * m));
    }
    for (int n = 0; n <= L; ++n)
        for (int m = 0; m <= n; ++m) {
            const zl e(std::cos(m * phi), std::sin(m * phi));
            Y[cidx(n, m)] = q(n, m) * e;
            if (m > 0) Y[cidx(n, -m)] = q(n, m) * std::conj(e);
        }
    return r;
}

// real dof index for (n, m >= 0, part): part 0 = re, 1 = im
inline int rdof(int n, int m, int part) { return m == 0 ? n * n : n * n + 2 * m - 1 + part; }

// Assemble the real K x K matrix of a complex-linear map given on the full
// (n, m) index range, using M_n^{-m} = conj(M_n^m) on the input side and
// storing only k >= 0 on the output side.
template <class F>
void realify(int p, F coef, double* out) {
    const int K = num_dofs(p);
    for (int i = 0; i < K * K; ++i) out[i] = 0.0;
    for (int j = 0; j <= p; ++j)
        for (int k = 0; k <= j; ++k)
            for (int n = 0; n <= p; ++n)
                for (int m = 0; m <= n; ++m) {
                    const int rre = rdof(j, k, 0), rim = rdof(j, k, 1);
                    if (m == 0) {
                        const zl c = coef(j, k, n, 0);
                        out[rre * K + rdof(n, 0, 0)] = (double)c.real();
                        if (k > 0) out[rim * K + rdof(n, 0, 0)] = (double)c.imag();
                    } else {
                        const zl c1 = coef(j, k, n, m), c2 = coef(j, k, n, -m);
                        const zl s = c1 + c2, d = c1 - c2;
                        out[rre * K + rdof(n, m, 0)] = (double)s.real();
                        out[rre * K + rdof(n, m, 1)] = (double)(-d.imag());
                        if (k > 0) {
                            out[rim * K + rdof(n, m, 0)] = (double)s.imag();
                            out[rim * K + rdof(n, m, 1)] = (double)d.real();
                        }
                    }
                }
}

}  // namespace

void build_operator(int kind, int p, int index, double* out) {
    std::vector<zl> Y;
    if (kind == 0 || kind == 1) {
        const ld dx = (index & 1) ? 0.5L : -0.5L, dy = (index & 2) ? 0.5L : -0.5L, dz = (index & 4) ? 0.5L : -0.5L;
        if (kind == 0) {
            // M2M, t = old(child) - new(parent) centre = delta (child side units)
            const ld rho = harmonics(dx, dy, dz, p, Y);
            realify(p, [&](int j, int k, int nin, int min) -> zl {
                const int n = j - nin, m = k - min;
                if (n < 0 || iabs(m) > n || iabs(min) > nin) return zl(0, 0);
                const ld J = jpow(iabs(k) - iabs(m) - iabs(k - m));
                const ld sc = std::pow(0.5L, (ld)j);
                return sc * J * Acoef(n, m) * Acoef(nin, min) * std::pow(rho, (ld)n) * Y[cidx(n, -m)] / Acoef(j, k);
            }, out);
        } else {
            // L2L, t = new(child) - old(parent) centre = delta (child side units)
            const ld rho = harmonics(dx, dy, dz, p, Y);
            realify(p, [&](int j, int k, int n, int m) -> zl {
                if (n < j) return zl(0, 0);
                const int nn = n - j, kk = m - k;
                if (iabs(kk) > nn) return zl(0, 0);
                const ld J = jpow(iabs(m) - iabs(m - k) - iabs(k));
                const ld sc = std::pow(0.5L, (ld)n);
                return sc * J * Acoef(nn, kk) * Acoef(j, k) * Y[cidx(nn, kk)] * std::pow(rho, (ld)nn) / Acoef(n, m);
            }, out);
        }
        return;
    }
    // M2L: index -> offset o = source - target (box-side units); t = target - source = -o
    const int ox = index % 7 - 3, oy = (index / 7) % 7 - 3, oz = index / 49 - 3;
    const int K = num_dofs(p);
    if (std::max(iabs(ox), std::max(iabs(oy), iabs(oz))) <= 1) {
        for (int i = 0; i < K * K; ++i) out[i] = 0.0;
        return;
    }
    build_m2l_offset(p, (ld)ox, (ld)oy, (ld)oz, out);
}

// M2L matrix for any offset o = source - target (box-side units), |o| well separated
void build_m2l_offset(int p, long double ox, long double oy, long double oz, double* out) {
    std::vector<zl> Y;
    const ld rho = harmonics(-ox, -oy, -oz, 2 * p, Y);
    realify(p, [&](int j, int k, int n, int m) -> zl {
        const int deg = j + n, ord = m - k;
        if (iabs(ord) > deg) return zl(0, 0);
        const ld J = jpow(iabs(k - m) - iabs(k) - iabs(m));
        const ld sgn = (j & 1) ? -1.0L : 1.0L;
        return sgn * J * Acoef(n, m) * Acoef(j, k) * Y[cidx(deg, ord)] / (Acoef(deg, ord) * std::pow(rho, (ld)(deg + 1)));
    }, out);
}

// ---- rotation-based M2L (the third form) ----------------------------------------
// T_o = Q_o^-1 Z_|o| Q_o, where Q_o rotates expansion coefficients by a rotation R
// that takes o to |o| z (Q_o v(x) = v(R x), v(x) = the coefficient vector of a unit
// source on the unit sphere, which is the same for multipoles and locals: both are
// Y_n^-m(x) there, so one Q serves both sides), and Z_|o| is the M2L along the z axis,
// which couples only equal orders m (and the same re / im part, with the same
// matrix).  Q_o is block diagonal by degree; its blocks are solved from the action
// of R on sampled unit vectors (least squares in long double, 2(2n+1) samples).
// Cost per V pair: 2 sum_n (2n+1)^2 + sum_m (p+1-m)^2 FMAs (2,223 at p = 8) instead
// of K^2 (6,561).
namespace {

// Gauss-Jordan with partial pivoting: a (n x n, row-major) <- a^-1
bool invert_ld(std::vector<ld>& a, int n) {
    std::vector<ld> inv((size_t)n * n, 0.0L);
    for (int i = 0; i < n; ++i) inv[(size_t)i * n + i] = 1.0L;
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(a[(size_t)r * n + c]) > std::fabs(a[(size_t)piv * n + c])) piv = r;
        if (std::fabs(a[(size_t)piv * n + c]) < 1e-30L) return false;
        if (piv != c)
            for (int k = 0; k < n; ++k) {
                std::swap(a[(size_t)c * n + k], a[(size_t)piv * n + k]);
                std::swap(inv[(size_t)c * n + k], inv[(size_t)piv * n + k]);
            }
        const ld d = a[(size_t)c * n + c];
        for (int k = 0; k < n; ++k) {
            a[(size_t)c * n + k] /= d;
            inv[(size_t)c * n + k] /= d;
        }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const ld f = a[(size_t)r * n + c];
            if (f == 0.0L) continue;
            for (int k = 0; k < n; ++k) {
                a[(size_t)r * n + k] -= f * a[(size_t)c * n + k];
                inv[(size_t)r * n + k] -= f * inv[(size_t)c * n + k];
            }
        }
    }
    a.swap(inv);
    return true;
}

// degree-n block of the real coefficient vector of a unit source at unit vector u:
// (Re Y_n^0, Re Y_n^1, -Im Y_n^1, ...), Y_n^-m = conj(Y_n^m)
void unit_vector_block(ld x, ld y, ld z, int n, std::vector<ld>& out) {
    std::vector<zl> Y;
    harmonics(x, y, z, n, Y);
    out.assign(2 * n + 1, 0.0L);
    out[0] = Y[cidx(n, 0)].real();
    for (int m = 1; m <= n; ++m) {
        out[2 * m - 1] = Y[cidx(n, m)].real();
        out[2 * m] = -Y[cidx(n, m)].imag();
    }
}

}  // namespace

int rot_pack_size(int p) {
    int q = 0, z = 0;
    for (int n = 0; n <= p; ++n) q += (2 * n + 1) * (2 * n + 1);
    for (int m = 0; m <= p; ++m) z += (p + 1 - m) * (p + 1 - m);
    return 2 * q + z;
}

// Pack for V offset `index` (as build_operator kind 2): [Q blocks | Q^-1 blocks | Z
// blocks], each Q block (2n+1)^2 row-major in degree order, each Z block m the
// (p+1-m)^2 matrix Z[j-m][n-m] for degrees j, n >= m.  Returns false for offsets
// that are not in a V list (all zero then).
bool build_rot_pack(int p, int index, double* out) {
    const int ox = index % 7 - 3, oy = (index / 7) % 7 - 3, oz = index / 49 - 3;
    const int total = rot_pack_size(p);
    for (int i = 0; i < total; ++i) out[i] = 0.0;
    if (std::max(iabs(ox), std::max(iabs(oy), iabs(oz))) <= 1) return false;
    // rotation R with R o = |o| z (Rodrigues about o x z)
    const ld ol = std::sqrt((ld)(ox * ox + oy * oy + oz * oz));
    const ld u[3] = {ox / ol, oy / ol, oz / ol};
    ld Rm[3][3];
    {
        const ld ax0 = u[1], ax1 = -u[0];   // u x z
        const ld sn = std::sqrt(ax0 * ax0 + ax1 * ax1), cs = u[2];
        if (sn < 1e-18L) {
            const ld sg = cs > 0 ? 1.0L : -1.0L;   // o along +z: identity; along -z: turn about x
            const ld I[3][3] = {{1, 0, 0}, {0, sg, 0}, {0, 0, sg}};
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) Rm[i][j] = I[i][j];
        } else {
            const ld k0 = ax0 / sn, k1 = ax1 / sn, k2 = 0.0L;
            const ld Kx[3][3] = {{0, -k2, k1}, {k2, 0, -k0}, {-k1, k0, 0}};
            for (int i = 0; i < 3; ++i)
                for (int j = 0; j < 3; ++j) {
                    ld kk = 0;
                    for (int l = 0; l < 3; ++l) kk += Kx[i][l] * Kx[l][j];
                    Rm[i][j] = (i == j ? 1.0L : 0.0L) + sn * Kx[i][j] + (1.0L - cs) * kk;
                }
        }
    }
    double* Qo = out;
    int qsz = 0;
    for (int n = 0; n <= p; ++n) qsz += (2 * n + 1) * (2 * n + 1);
    double* Qi = out + qsz;
    double* Zo = out + 2 * qsz;
    int off = 0;
    for (int n = 0; n <= p; ++n) {
        const int w = 2 * n + 1, ns = 2 * w;
        // fixed, well spread sample directions (spherical Fibonacci)
        std::vector<ld> A((size_t)w * ns), B((size_t)w * ns), v;
        for (int i = 0; i < ns; ++i) {
            const ld zc = 1.0L - (2.0L * i + 1.0L) / ns;
            const ld rr = std::sqrt(std::max((ld)0, 1.0L - zc * zc));
            const ld ph = 2.399963229728653322L * i + 0.3L;
            const ld x = rr * std::cos(ph), y = rr * std::sin(ph);
            unit_vector_block(x, y, zc, n, v);
            for (int r = 0; r < w; ++r) A[(size_t)r * ns + i] = v[r];
            const ld X = Rm[0][0] * x + Rm[0][1] * y + Rm[0][2] * zc;
            const ld Yy = Rm[1][0] * x + Rm[1][1] * y + Rm[1][2] * zc;
            const ld Zz = Rm[2][0] * x + Rm[2][1] * y + Rm[2][2] * zc;
            unit_vector_block(X, Yy, Zz, n, v);
            for (int r = 0; r < w; ++r) B[(size_t)r * ns + i] = v[r];
        }
        // Q_n = B A^T (A A^T)^-1
        std::vector<ld> AAt((size_t)w * w, 0.0L), BAt((size_t)w * w, 0.0L);
        for (int r = 0; r < w; ++r)
            for (int c = 0; c < w; ++c)
                for (int i = 0; i < ns; ++i) {
                    AAt[(size_t)r * w + c] += A[(size_t)r * ns + i] * A[(size_t)c * ns + i];
                    BAt[(size_t)r * w + c] += B[(size_t)r * ns + i] * A[(size_t)c * ns + i];
                }
        if (!invert_ld(AAt, w)) return false;
        std::vector<ld> Qn((size_t)w * w, 0.0L);
        for (int r = 0; r < w; ++r)
            for (int c = 0; c < w; ++c)
                for (int k = 0; k < w; ++k) Qn[(size_t)r * w + c] += BAt[(size_t)r * w + k] * AAt[(size_t)k * w + c];
        std::vector<ld> Qinv = Qn;
        if (!invert_ld(Qinv, w)) return false;
        for (int i = 0; i < w * w; ++i) {
            Qo[off + i] = (double)Qn[i];
            Qi[off + i] = (double)Qinv[i];
        }
        off += w * w;
    }
    // Z: the M2L along +z at distance |o|, restricted to equal orders (re parts)
    const int K = num_dofs(p);
    std::vector<double> T((size_t)K * K);
    build_m2l_offset(p, 0.0L, 0.0L, ol, T.data());
    int zo = 0;
    for (int m = 0; m <= p; ++m) {
        const int w = p + 1 - m;
        for (int j = m; j <= p; ++j)
            for (int n = m; n <= p; ++n) Zo[zo + (j - m) * w + (n - m)] = T[(size_t)rdof(j, m, 0) * K + rdof(n, m, 0)];
        zo += w * w;
    }
    return true;
}

}  // namespace ogx

extern "C" int ogx_operator_matrix(int kind, int p, int index, double* out) {
    if (!out || p < 1 || p > ogx::kPMax) return OGX_ERR_INVALID;
    if ((kind == 0 || kind == 1) && (index < 0 || index > 7)) return OGX_ERR_INVALID;
    if ((kind == 2 || kind == 3) && (index < 0 || index >= 343)) return OGX_ERR_INVALID;
    if (kind < 0 || kind > 3) return OGX_ERR_INVALID;
    if (kind <= 2) {
        ogx::build_operator(kind, p, index, out);
        return OGX_OK;
    }
    // kind 3: the rotation factors of M2L offset `index` multiplied back out,
    // Q^-1 Z Q as a dense K x K matrix (equal to kind 2 up to rounding)
    const int K = ogx::num_dofs(p);
    std::vector<double> pk((size_t)ogx::rot_pack_size(p));
    for (int i = 0; i < K * K; ++i) out[i] = 0.0;
    if (!ogx::build_rot_pack(p, index, pk.data())) return OGX_OK;
    int qsz = 0;
    for (int n = 0; n <= p; ++n) qsz += (2 * n + 1) * (2 * n + 1);
    const double* Q = pk.data();
    const double* Qi = Q + qsz;
    const double* Z = Q + 2 * qsz;
    // dense Q and Q^-1
    std::vector<double> Qd((size_t)K * K, 0.0), Qid((size_t)K * K, 0.0), Zd((size_t)K * K, 0.0);
    int off = 0;
    for (int n = 0; n <= p; ++n) {
        const int w = 2 * n + 1;
        for (int r = 0; r < w; ++r)
            for (int c = 0; c < w; ++c) {
                Qd[(size_t)(n * n + r) * K + n * n + c] = Q[off + r * w + c];
                Qid[(size_t)(n * n + r) * K + n * n + c] = Qi[off + r * w + c];
            }
        off += w * w;
    }
    int zo = 0;
    for (int m = 0; m <= p; ++m) {
        const int w = p + 1 - m;
        for (int j = m; j <= p; ++j)
            for (int n = m; n <= p; ++n) {
                const double v = Z[zo + (j - m) * w + (n - m)];
                const int jr = m == 0 ? j * j : j * j + 2 * m - 1, nr = m == 0 ? n * n : n * n + 2 * m - 1;
                Zd[(size_t)jr * K + nr] = v;
                if (m > 0) Zd[(size_t)(jr + 1) * K + nr + 1] = v;
            }
        zo += w * w;
    }
    std::vector<double> ZQ((size_t)K * K, 0.0);
    for (int i = 0; i < K; ++i)
        for (int k = 0; k < K; ++k) {
            const double a = Zd[(size_t)i * K + k];
            if (a == 0.0) continue;
            for (int j = 0; j < K; ++j) ZQ[(size_t)i * K + j] += a * Qd[(size_t)k * K + j];
        }
    for (int i = 0; i < K; ++i)
        for (int k = 0; k < K; ++k) {
            const double a = Qid[(size_t)i * K + k];
            if (a == 0.0) continue;
            for (int j = 0; j < K; ++j) out[(size_t)i * K + j] += a * ZQ[(size_t)k * K + j];
        }
    return OGX_OK;
}
