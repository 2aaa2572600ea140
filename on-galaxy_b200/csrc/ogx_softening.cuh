// ogx_softening.cuh -- the compact-support softening kernel (OGX_SOFT_SPLINE).
//
// Cubic spline of Monaghan & Lattanzio (1985) as GADGET-2 uses it (Springel 2005,
// MNRAS 364, 1105, eq. 4), support h = 2.8 eps.  With u = r / h the potential of a unit
// mass is -W(u) / h,
//   W(u) = 16/3 u^2 - 48/5 u^4 + 32/5 u^5 - 14/5                          0 <= u < 1/2
//   W(u) = 1/(15 u) + 32/3 u^2 - 16 u^3 + 48/5 u^4 - 32/15 u^5 - 16/5    1/2 <= u < 1
//   W(u) = -1/u                                                            u >= 1
// and the acceleration it exerts is g(r) (r_j - r_i) with g = W'(u) / (h^3 u).  Here
// k = -W(u) / h (so pot = -G sum m k, k = 1/r beyond h) and g are returned; both are
// continuous with their first derivatives at u = 1/2 and u = 1, k(0) = 1 / eps.
#pragma once

namespace ogx {

template <class T>
__device__ __forceinline__ void spline_gk(T r2, T h, T hinv, T& g, T& k) {
    if (r2 >= h * h) {
        T y;
        if constexpr (sizeof(T) == 4) y = rsqrtf(r2); else y = rsqrt(r2);
        g = y * y * y;
        k = y;
        return;
    }
    T r;
    if constexpr (sizeof(T) == 4) r = sqrtf(r2); else r = sqrt(r2);
    const T u = r * hinv;
    const T u2 = u * u;
    const T hinv3 = hinv * hinv * hinv;
    if (u < T(0.5)) {
        g = hinv3 * (T(32.0 / 3.0) + u2 * (T(32.0) * u - T(38.4)));
        k = hinv * (T(2.8) - u2 * (T(16.0 / 3.0) + u2 * (T(6.4) * u - T(9.6))));
    } else {
        const T iu = T(1) / u;
        g = hinv3 * (T(64.0 / 3.0) - T(48.0) * u + T(38.4) * u2 - T(32.0 / 3.0) * u2 * u - T(1.0 / 15.0) * iu * iu * iu);
        k = hinv * (T(3.2) - T(1.0 / 15.0) * iu - u2 * (T(32.0 / 3.0) + u * (T(-16.0) + u * (T(9.6) - T(32.0 / 15.0) * u))));
    }
}

// the spline's support for a softening length eps
inline double spline_support(double eps) { return 2.8 * eps; }

}  // namespace ogx
