// ogx_harmonics.cuh -- solid harmonics and expansion-coefficient helpers.
//
// The reference evaluates Y_n^m through cos/sin/atan2 and the seminormalised
// Legendre recurrence (src3d/FmmExpansions3D.hpp:75-107) and multiplies by
// rho^n or rho^-(n+1) afterwards.  Here the same functions are generated
// directly as solid harmonics in Cartesian form, column by column in m, so a
// thread never holds more than the current column:
//   R_n^m = rho^n Y_n^m:           R_m^m = (x+iy) a_m R_{m-1}^{m-1}
//                                  R_{m+1}^m = z b_m R_m^m
//                                  R_n^m = z A_nm R_{n-1}^m - r^2 B_nm R_{n-2}^m
//   S_n^m = Y_n^m / rho^{n+1}:     same recurrences with a factor 1/r^2 per step
// with a_m = sqrt((2m-1)/2m), b_m = sqrt(2m+1), A_nm = (2n-1)/sqrt(n^2-m^2),
// B_nm = sqrt((n-1)^2-m^2)/sqrt(n^2-m^2): the reference's Q recurrence
// multiplied through by rho^n e^{i m phi} (no trigonometric calls).
//
// Real coefficient layout (K = (p+1)^2 doubles): dof(n,0) = n^2,
// dof(n,m>0) = n^2 + 2m - 1 (real part), n^2 + 2m (imaginary part).
// Negative orders follow from c_n^{-m} = conj(c_n^m) for real sources.
#pragma once

#include <cmath>
#include <mutex>

#include "ogx_internal.cuh"

namespace ogx {

constexpr int kTab = kDegMax + 2;

struct HarmTables {
    double a[kTab];
    double b[kTab];
    double A[kTab][kTab];
    double B[kTab][kTab];
    // gradient-coefficient constants (derivative recurrences of FmmExpansions3D.hpp:111-129)
    double gz[kTab][kTab], gp[kTab][kTab], gm[kTab][kTab];  // local  -> degree n (from degree n+1)
    double hz[kTab][kTab], hp[kTab][kTab], hm[kTab][kTab];  // mpole  -> degree n (from degree n-1)
    // FP32 copies of the recurrence constants for the FP32 kernels (no conversion per use)
    float fa[kTab], fb[kTab], fA[kTab][kTab], fB[kTab][kTab];
};

// the reference's derivative coefficients (FmmExpansions3D.hpp:111-129)
inline double ref_cz_R(int n, int m) { return std::sqrt(double(n * n - m * m)); }
inline double ref_cp_R(int n, int m) { return ((m >= 0) ? -1.0 : 1.0) * std::sqrt(double((n - m) * (n - m - 1))); }
inline double ref_cm_R(int n, int m) { return ((m > 0) ? 1.0 : -1.0) * std::sqrt(double((n + m) * (n + m - 1))); }
inline double ref_dz_S(int n, int m) { return -std::sqrt(double((n + 1) * (n + 1) - m * m)); }
inline double ref_dp_S(int n, int m) { return ((m >= 0) ? -1.0 : 1.0) * std::sqrt(double((n + m + 1) * (n + m + 2))); }
inline double ref_dm_S(int n, int m) { return ((m > 0) ? 1.0 : -1.0) * std::sqrt(double((n - m + 1) * (n - m + 2))); }

// One copy per translation unit (whole-program compilation, no device linking);
// every unit that launches harmonic kernels calls harm_tables_ready() first.
static __constant__ HarmTables c_harm;
// the same tables in global memory, for kernels whose lanes index them divergently
// (the constant cache serialises lanes that read different addresses)
static __device__ HarmTables g_harm;

static inline void fill_harm_tables(HarmTables& t) {
    t = HarmTables{};
    for (int m = 0; m < kTab; ++m) {
        t.a[m] = m > 0 ? std::sqrt((2.0 * m - 1.0) / (2.0 * m)) : 1.0;
        t.b[m] = std::sqrt(2.0 * m + 1.0);
    }
    for (int m = 0; m < kTab; ++m) {
        t.fa[m] = (float)t.a[m];
        t.fb[m] = (float)t.b[m];
    }
    for (int n = 0; n < kTab; ++n)
        for (int m = 0; m < kTab; ++m) {
            if (n >= m + 2) {
                const double d = std::sqrt((double)(n * n - m * m));
                t.A[n][m] = (2.0 * n - 1.0) / d;
                t.B[n][m] = std::sqrt((double)((n - 1) * (n - 1) - m * m)) / d;
                t.fA[n][m] = (float)t.A[n][m];
                t.fB[n][m] = (float)t.B[n][m];
            }
            if (m <= n) {
                // G_n^m from L_{n+1}^{m}, L_{n+1}^{m-1}, L_{n+1}^{m+1}
                t.gz[n][m] = ref_cz_R(n + 1, m);
                t.gp[n][m] = ref_cp_R(n + 1, m - 1);
                t.gm[n][m] = ref_cm_R(n + 1, m + 1);
                // H_n^m from M_{n-1}^{m}, M_{n-1}^{m-1}, M_{n-1}^{m+1} (zero where the source order is absent)
                if (n >= 1) {
                    t.hz[n][m] = (m <= n - 1) ? ref_dz_S(n - 1, m) : 0.0;
                    t.hp[n][m] = (std::abs(m - 1) <= n - 1) ? ref_dp_S(n - 1, m - 1) : 0.0;
                    t.hm[n][m] = (m + 1 <= n - 1) ? ref_dm_S(n - 1, m + 1) : 0.0;
                }
            }
        }
}

static inline int harm_tables_ready(int device) {
    static std::mutex mu;
    static bool done[64] = {};
    std::lock_guard<std::mutex> lk(mu);
    if (device < 0 || device >= 64) return OGX_ERR_INVALID;
    if (done[device]) return OGX_OK;
    HarmTables t;
    fill_harm_tables(t);
    cudaError_t e = cudaMemcpyToSymbol(c_harm, &t, sizeof(t));
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_harm, &t, sizeof(t));
    // the copies from the pageable t may still be in flight on the legacy stream,
    // which the library's non-blocking streams do not wait for
    if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
    if (e != cudaSuccess) {
        set_last_error(OGX_ERR_CUDA, std::string("harmonic tables: ") + cudaGetErrorString(e));
        return OGX_ERR_CUDA;
    }
    done[device] = true;
    return OGX_OK;
}

__host__ __device__ __forceinline__ constexpr int dof_re(int n, int m) { return m == 0 ? n * n : n * n + 2 * m - 1; }

// Visit R_n^m(x,y,z), n <= P (m >= 0), calling f(n, m, re, im) column by column.
// recurrence constants in the arithmetic type (FP32 kernels read the FP32 copies)
template <class T> __device__ __forceinline__ T harm_a(int m) {
    if constexpr (sizeof(T) == 4) return c_harm.fa[m]; else return (T)c_harm.a[m];
}
template <class T> __device__ __forceinline__ T harm_b(int m) {
    if constexpr (sizeof(T) == 4) return c_harm.fb[m]; else return (T)c_harm.b[m];
}
template <class T> __device__ __forceinline__ T harm_A(int n, int m) {
    if constexpr (sizeof(T) == 4) return c_harm.fA[n][m]; else return (T)c_harm.A[n][m];
}
template <class T> __device__ __forceinline__ T harm_B(int n, int m) {
    if constexpr (sizeof(T) == 4) return c_harm.fB[n][m]; else return (T)c_harm.B[n][m];
}

template <int P, class T, class F>
__device__ __forceinline__ void for_regular(T x, T y, T z, F&& f) {
    const T r2 = x * x + y * y + z * z;
    T dr = 1, di = 0;  // R_m^m
#pragma unroll
    for (int m = 0; m <= P; ++m) {
        if (m > 0) {
            const T a = harm_a<T>(m);
            const T nr = a * (x * dr - y * di), ni = a * (x * di + y * dr);
            dr = nr;
            di = ni;
        }
        f(m, m, dr, di);
        if (m + 1 <= P) {
            const T bz = harm_b<T>(m) * z;
            T pr = dr, pi = di;              // R_{n-2}
            T cr = bz * dr, ci = bz * di;    // R_{n-1}
            f(m + 1, m, cr, ci);
#pragma unroll
            for (int n = m + 2; n <= P; ++n) {
                const T A = harm_A<T>(n, m) * z, B = harm_B<T>(n, m) * r2;
                const T qr = A * cr - B * pr, qi = A * ci - B * pi;
                pr = cr; pi = ci; cr = qr; ci = qi;
                f(n, m, cr, ci);
            }
        }
    }
}

// Visit S_n^m(x,y,z), n <= P (m >= 0).  The origin is excluded by construction
// (sources and targets of M2P/P2L are in well-separated boxes).
template <int P, class T, class F>
__device__ __forceinline__ void for_singular(T x, T y, T z, F&& f) {
    const T r2 = x * x + y * y + z * z;
    T ir2, dr, di = 0;         // dr = S_0^0 = 1/rho
    if constexpr (sizeof(T) == 4) {
        dr = rsqrtf(r2);       // FP32 path: one rsqrt instead of a division and a square root
        ir2 = dr * dr;
    } else {
        ir2 = T(1) / r2;
        dr = sqrt(ir2);
    }
    const T zr = z * ir2;      // FP32 path: one product per visit instead of two
#pragma unroll
    for (int m = 0; m <= P; ++m) {
        if (m > 0) {
            const T a = harm_a<T>(m) * ir2;
            const T nr = a * (x * dr - y * di), ni = a * (x * di + y * dr);
            dr = nr;
            di = ni;
        }
        f(m, m, dr, di);
        if (m + 1 <= P) {
            const T bz = (sizeof(T) == 4) ? harm_b<T>(m) * zr : harm_b<T>(m) * z * ir2;
            T pr = dr, pi = di;
            T cr = bz * dr, ci = bz * di;
            f(m + 1, m, cr, ci);
#pragma unroll
            for (int n = m + 2; n <= P; ++n) {
                const T A = (sizeof(T) == 4) ? harm_A<T>(n, m) * zr : harm_A<T>(n, m) * z * ir2;
                const T B = harm_B<T>(n, m) * ir2;
                const T qr = A * cr - B * pr, qi = A * ci - B * pi;
                pr = cr; pi = ci; cr = qr; ci = qi;
                f(n, m, cr, ci);
            }
        }
    }
}

// complex coefficient c_n^m from a real layout (m may be negative)
template <class T>
__device__ __forceinline__ void coef_get(const T* c, int n, int m, T& re, T& im) {
    if (m < -n || m > n || n < 0) { re = 0; im = 0; return; }
    if (m == 0) { re = c[n * n]; im = 0; return; }
    const int am = m < 0 ? -m : m;
    re = c[n * n + 2 * am - 1];
    im = c[n * n + 2 * am];
    if (m < 0) im = -im;
}

__device__ __forceinline__ void dof_decode(int d, int& n, int& m, int& part) {
    n = (int)floorf(sqrtf((float)d) + 1e-4f);
    const int r = d - n * n;
    m = (r + 1) >> 1;
    part = (r == 0) ? 0 : ((r - 1) & 1);
}

// Gradient coefficients of a local expansion (degree P -> P-1), in the real
// layout, for the three axes.  From the derivative recurrences of
// FmmExpansions3D.hpp:111-119 as used by localField (:215-235):
//   Gz_n^m = cz_R(n+1,m) L_{n+1}^m
//   Gx_n^m = (cp_R(n+1,m-1) L_{n+1}^{m-1} + cm_R(n+1,m+1) L_{n+1}^{m+1}) / 2
//   Gy_n^m = -i (cp_R(n+1,m-1) L_{n+1}^{m-1} - cm_R(n+1,m+1) L_{n+1}^{m+1}) / 2
// Every returned value is for one real dof index `d` of degree <= P-1.
template <class Tin, class T>
__device__ __forceinline__ void local_grad_dof(const Tin* L, int d, T g[3]) {
    int n, m, part;
    dof_decode(d, n, m, part);
    const int N = n + 1;
    Tin lr, li, pr, pi, mr, mi;
    coef_get(L, N, m, lr, li);
    coef_get(L, N, m - 1, mr, mi);
    coef_get(L, N, m + 1, pr, pi);
    const double czr = c_harm.gz[n][m], cpr = c_harm.gp[n][m], cmr = c_harm.gm[n][m];
    const double xr = 0.5 * (cpr * mr + cmr * pr), xi = 0.5 * (cpr * mi + cmr * pi);
    const double dr = cpr * mr - cmr * pr, di = cpr * mi - cmr * pi;  // -i/2 (a - b)
    if (part == 0) { g[0] = (T)xr; g[1] = (T)(0.5 * di); g[2] = (T)(czr * lr); }
    else { g[0] = (T)xi; g[1] = (T)(-0.5 * dr); g[2] = (T)(czr * li); }
}

// Gradient coefficients of a multipole expansion (degree P -> P+1), from
// dz_S/dp_S/dm_S (FmmExpansions3D.hpp:121-129) as used by multipoleField (:180-200):
//   Hz_n^m = dz_S(n-1,m) M_{n-1}^m
//   Hx_n^m = (dp_S(n-1,m-1) M_{n-1}^{m-1} + dm_S(n-1,m+1) M_{n-1}^{m+1}) / 2
//   Hy_n^m = -i (dp_S(n-1,m-1) M_{n-1}^{m-1} - dm_S(n-1,m+1) M_{n-1}^{m+1}) / 2
template <class Tin, class T>
__device__ __forceinline__ void mpole_grad_dof(const Tin* M, int d, T g[3]) {
    int n, m, part;
    dof_decode(d, n, m, part);
    if (n == 0) { g[0] = g[1] = g[2] = 0; return; }
    const int N = n - 1;
    Tin lr, li, pr, pi, mr, mi;
    coef_get(M, N, m, lr, li);
    coef_get(M, N, m - 1, mr, mi);
    coef_get(M, N, m + 1, pr, pi);
    const double dzs = c_harm.hz[n][m], dps = c_harm.hp[n][m], dms = c_harm.hm[n][m];
    const double xr = 0.5 * (dps * mr + dms * pr), xi = 0.5 * (dps * mi + dms * pi);
    const double dr = dps * mr - dms * pr, di = dps * mi - dms * pi;
    if (part == 0) { g[0] = (T)xr; g[1] = (T)(0.5 * di); g[2] = (T)(dzs * lr); }
    else { g[0] = (T)xi; g[1] = (T)(-0.5 * dr); g[2] = (T)(dzs * li); }
}

}  // namespace ogx
