// ogx_expansion_kernels.cuh -- particle <-> expansion kernels, templated on the
// arithmetic type T (double for the plain form, float for the mixed form).
// Global-to-box-centre shifts (x - c) are always taken in FP64 and only the
// scaled box-relative coordinate u = (x - c) / side is rounded to T.
#pragma once

#include "ogx_harmonics.cuh"

namespace ogx {

// ---- P2M / P2L: particle -> expansion --------------------------------------------
// MODE 0: P2M for leaf t (fmm::P2M, src3d/FmmExpansions3D.hpp:148-163): store
//         M'_n^m = sum q conj(R_n^m(u)),  u = (x - c)/side.
// MODE 1: P2L for box t over X(t) (AdaptiveFMM3D::p2lAccum, src3d/AdaptiveFMM3D.hpp:117-128):
//         L'_n^m += sum (q/side) conj(S_n^m(u)).
// Warp per target: lanes build the harmonics of 32 sources into shared memory
// (one row each), then every lane sums a few coefficient columns.
template <int P, int MODE, class T>
__global__ void __launch_bounds__(128) k_p2x(TreeView tv, int ntargets, double* out) {
    constexpr int K = (P + 1) * (P + 1);
    constexpr int LD = K | 1;
    extern __shared__ __align__(16) unsigned char s_raw[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int t = blockIdx.x * 4 + wid;
    if (t >= ntargets || t >= (MODE == 0 ? tv_nleaf(tv) : tv_nb(tv)) || tv_over(tv)) return;
    T* buf = reinterpret_cast<T*>(s_raw) + (size_t)wid * 32 * LD;
    const int b = (MODE == 0) ? tv.leafbox[t] : t;
    int64_t e0, e1;
    if (MODE == 0) { e0 = 0; e1 = 1; }
    else { e0 = tv.x_off[b]; e1 = tv.x_off[b + 1]; if (e0 == e1) return; }
    const double cx = tv.center[4 * b], cy = tv.center[4 * b + 1], cz = tv.center[4 * b + 2];
    const double side = 2.0 * tv.center[4 * b + 3], inv = 1.0 / side;
    constexpr int NPL = (K + 31) / 32;
    double acc[NPL];
#pragma unroll
    for (int q = 0; q < NPL; ++q) acc[q] = 0.0;
    for (int64_t e = e0; e < e1; ++e) {
        const int src = (MODE == 0) ? b : tv.x_idx[e];
        const int f0 = tv.pfirst[src], cnt = tv.pcount[src];
        for (int j0 = 0; j0 < cnt; j0 += 32) {
            const int j = j0 + lane;
            T* row = buf + (size_t)lane * LD;
            if (j < cnt) {
                const int i = f0 + j;
                const T q = (T)tv.pm[i];
                const T ux = (T)((tv.px[i] - cx) * inv), uy = (T)((tv.py[i] - cy) * inv), uz = (T)((tv.pz[i] - cz) * inv);
                auto put = [&](int n, int m, T re, T im) {
                    if (m == 0) row[n * n] = q * re;
                    else { row[n * n + 2 * m - 1] = q * re; row[n * n + 2 * m] = -q * im; }
                };
                if (MODE == 0) for_regular<P>(ux, uy, uz, put);
                else for_singular<P>(ux, uy, uz, put);
            } else {
                for (int d = 0; d < K; ++d) row[d] = T(0);
            }
            __syncwarp();
#pragma unroll
            for (int q = 0; q < NPL; ++q) {
                const int d = lane + 32 * q;
                if (d < K) {
                    T s = 0;
#pragma unroll 8
                    for (int r = 0; r < 32; ++r) s += buf[(size_t)r * LD + d];
                    acc[q] += (double)s;
                }
            }
            __syncwarp();
        }
    }
#pragma unroll
    for (int q = 0; q < NPL; ++q) {
        const int d = lane + 32 * q;
        if (d < K) {
            if (MODE == 0) out[(size_t)b * K + d] = acc[q];
            else out[(size_t)b * K + d] += acc[q] * inv;
        }
    }
}

template <int P, class T>
constexpr size_t p2x_smem_bytes() {
    return (size_t)4 * 32 * ((P + 1) * (P + 1) | 1) * sizeof(T);
}

// ---- evaluation coefficient sets ---------------------------------------------------
// Per box (MODE 0): multipole gradient set H (3 x (P+2)^2, degree P+1) and the
// multipole itself (K), for every box that is a member of some W list (X list
// non-empty).  Per leaf (MODE 1): local gradient set G (3 x P^2, degree P-1) and
// the local itself.  Stored in T, one contiguous record per box / leaf:
//   record = [x-set | y-set | z-set | coefficients]
template <int P>
struct EvalLayout {
    static constexpr int K = (P + 1) * (P + 1);
    static constexpr int KG = P * P;
    static constexpr int KH = (P + 2) * (P + 2);
    static constexpr int HREC = 3 * KH + K;
    static constexpr int GREC = 3 * KG + K;
};

template <int P, int MODE, class T>
__global__ void __launch_bounds__(128) k_eval_coeffs(TreeView tv, int count, const double* __restrict__ coef, T* __restrict__ rec) {
    using Lo = EvalLayout<P>;
    const int lane = threadIdx.x & 31;
    const int k = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (k >= count || k >= (MODE == 0 ? tv_nb(tv) : tv_nleaf(tv)) || tv_over(tv)) return;
    const int b = (MODE == 0) ? k : tv.leafbox[k];
    if (MODE == 0 && tv.x_off[b] == tv.x_off[b + 1]) return;
    const double* c = coef + (size_t)b * Lo::K;
    if (MODE == 0) {
        T* o = rec + (size_t)k * Lo::HREC;
        for (int d = lane; d < Lo::KH; d += 32) {
            T g[3];
            mpole_grad_dof(c, d, g);
            o[d] = g[0]; o[Lo::KH + d] = g[1]; o[2 * Lo::KH + d] = g[2];
        }
        for (int d = lane; d < Lo::K; d += 32) o[3 * Lo::KH + d] = (T)c[d];
    } else {
        T* o = rec + (size_t)k * Lo::GREC;
        for (int d = lane; d < Lo::KG; d += 32) {
            T g[3];
            local_grad_dof(c, d, g);
            o[d] = g[0]; o[Lo::KG + d] = g[1]; o[2 * Lo::KG + d] = g[2];
        }
        for (int d = lane; d < Lo::K; d += 32) o[3 * Lo::KG + d] = (T)c[d];
    }
}

// sum over (n, m>=0) of w_m Re(c_nm z_nm) for one dof visit
template <class T>
__device__ __forceinline__ T re_term(const T* c, int dr, int m, T re, T im) {
    return m == 0 ? c[dr] * re : T(2) * (c[dr] * re - c[dr + 1] * im);
}

// ---- leaf far field: L2P + W-list M2P -----------------------------------------------
// Warp per leaf, lanes over its bodies.  L2P (fmm::localField, :215-235) and M2P
// (fmm::multipoleField, :180-200) are evaluated as sum_nm Re(G_nm R_nm(u)) and
// sum_nm Re(H_nm S_nm(u)) with the precomputed coefficient records staged in
// shared memory once per (leaf, box); the harmonics are generated column by
// column so no body holds more than one column.
template <int P, bool POT, class T>
__global__ void __launch_bounds__(128) k_leaf_far(TreeView tv, const T* __restrict__ hrec, const T* __restrict__ grec,
                                                  double* __restrict__ far) {
    using Lo = EvalLayout<P>;
    constexpr int K = Lo::K, KG = Lo::KG, KH = Lo::KH;
    __shared__ T s_rec[4][Lo::HREC > Lo::GREC ? Lo::HREC : Lo::GREC];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int lf = blockIdx.x * 4 + wid;
    if (lf >= tv.nleaf || lf >= tv_nleaf(tv) || tv_over(tv)) return;
    T* sr = s_rec[wid];
    const int b = tv.leafbox[lf];
    const int f0 = tv.pfirst[b], cnt = tv.pcount[b];
    const double cx = tv.center[4 * b], cy = tv.center[4 * b + 1], cz = tv.center[4 * b + 2];
    const double side = 2.0 * tv.center[4 * b + 3], inv = 1.0 / side;
    const int64_t w0 = tv.w_off[lf], w1 = tv.w_off[lf + 1];
    for (int j0 = 0; j0 < cnt; j0 += 32) {
        const int j = j0 + lane;
        const bool act = j < cnt;
        const int i = f0 + (act ? j : 0);
        const double x = tv.px[i], y = tv.py[i], z = tv.pz[i];
        double gx, gy, gz, phi = 0.0;
        {
            const T* g = grec + (size_t)lf * Lo::GREC;
            for (int d = lane; d < (POT ? Lo::GREC : 3 * KG); d += 32) sr[d] = g[d];
            __syncwarp();
            const T ux = (T)((x - cx) * inv), uy = (T)((y - cy) * inv), uz = (T)((z - cz) * inv);
            T ax = 0, ay = 0, az = 0, ph = 0;
            for_regular<P>(ux, uy, uz, [&](int n, int m, T re, T im) {
                const int dr = dof_re(n, m);
                if (POT) ph += re_term(sr + 3 * KG, dr, m, re, im);
                if (n < P) {
                    ax += re_term(sr, dr, m, re, im);
                    ay += re_term(sr + KG, dr, m, re, im);
                    az += re_term(sr + 2 * KG, dr, m, re, im);
                }
            });
            gx = (double)ax * inv; gy = (double)ay * inv; gz = (double)az * inv;
            if (POT) phi = (double)ph;
            __syncwarp();
        }
        for (int64_t e = w0; e < w1; ++e) {
            const int c = tv.w_idx[e];
            const T* h = hrec + (size_t)c * Lo::HREC;
            for (int d = lane; d < (POT ? Lo::HREC : 3 * KH); d += 32) sr[d] = h[d];
            __syncwarp();
            const double winv = 1.0 / (2.0 * tv.center[4 * c + 3]);
            const T ux = (T)((x - tv.center[4 * c]) * winv), uy = (T)((y - tv.center[4 * c + 1]) * winv),
                    uz = (T)((z - tv.center[4 * c + 2]) * winv);
            T ax = 0, ay = 0, az = 0, ph = 0;
            for_singular<P + 1>(ux, uy, uz, [&](int n, int m, T re, T im) {
                const int dr = dof_re(n, m);
                if (POT && n <= P) ph += re_term(sr + 3 * KH, dr, m, re, im);
                ax += re_term(sr, dr, m, re, im);
                ay += re_term(sr + KH, dr, m, re, im);
                az += re_term(sr + 2 * KH, dr, m, re, im);
            });
            gx += (double)ax * winv * winv; gy += (double)ay * winv * winv; gz += (double)az * winv * winv;
            if (POT) phi += (double)ph * winv;
            __syncwarp();
        }
        if (act) {
            far[4 * (size_t)i] = gx; far[4 * (size_t)i + 1] = gy; far[4 * (size_t)i + 2] = gz; far[4 * (size_t)i + 3] = phi;
        }
    }
}

}  // namespace ogx
