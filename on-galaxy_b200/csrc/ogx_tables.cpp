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
    const ld rho = harmonics((ld)-ox, (ld)-oy, (ld)-oz, 2 * p, Y);
    realify(p, [&](int j, int k, int n, int m) -> zl {
        const int deg = j + n, ord = m - k;
        if (iabs(ord) > deg) return zl(0, 0);
        const ld J = jpow(iabs(k - m) - iabs(k) - iabs(m));
        const ld sgn = (j & 1) ? -1.0L : 1.0L;
        return sgn * J * Acoef(n, m) * Acoef(j, k) * Y[cidx(deg, ord)] / (Acoef(deg, ord) * std::pow(rho, (ld)(deg + 1)));
    }, out);
}

}  // namespace ogx

extern "C" int ogx_operator_matrix(int kind, int p, int index, double* out) {
    if (!out || p < 1 || p > ogx::kPMax) return OGX_ERR_INVALID;
    if ((kind == 0 || kind == 1) && (index < 0 || index > 7)) return OGX_ERR_INVALID;
    if (kind == 2 && (index < 0 || index >= 343)) return OGX_ERR_INVALID;
    if (kind < 0 || kind > 2) return OGX_ERR_INVALID;
    ogx::build_operator(kind, p, index, out);
    return OGX_OK;
}
