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
    if (t >= ntargets) return;
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

// ---- leaf far field: L2P + W-list M2P -----------------------------------------------
// Warp per leaf, lanes over its bodies.  L2P (fmm::localField, :215-235) and M2P
// (fmm::multipoleField, :180-200) are evaluated as sum_nm Re(G_nm R_nm(u)) and
// sum_nm Re(H_nm S_nm(u)) with the gradient coefficient sets G (degree P-1) and
// H (degree P+1) formed once per (leaf, box) in shared memory; the harmonics are
// generated column by column so no body holds more than one column.
template <int P, bool POT, class T>
__global__ void __launch_bounds__(128) k_leaf_far(TreeView tv, const double* mpole, const double* local, double* far) {
    constexpr int K = (P + 1) * (P + 1);
    constexpr int KG = P * P;
    constexpr int KH = (P + 2) * (P + 2);
    __shared__ T s_c[4][K];
    __shared__ T s_g[4][3][KH];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int lf = blockIdx.x * 4 + wid;
    if (lf >= tv.nleaf) return;
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
            for (int d = lane; d < K; d += 32) s_c[wid][d] = (T)local[(size_t)b * K + d];
            for (int d = lane; d < KG; d += 32) {
                T g[3];
                local_grad_dof(local + (size_t)b * K, d, g);
                s_g[wid][0][d] = g[0]; s_g[wid][1][d] = g[1]; s_g[wid][2][d] = g[2];
            }
            __syncwarp();
            const T ux = (T)((x - cx) * inv), uy = (T)((y - cy) * inv), uz = (T)((z - cz) * inv);
            T ax = 0, ay = 0, az = 0, ph = 0;
            for_regular<P>(ux, uy, uz, [&](int n, int m, T re, T im) {
                const T w = (m == 0) ? T(1) : T(2);
                const int dr = dof_re(n, m);
                if (POT) ph += w * (s_c[wid][dr] * re - (m ? s_c[wid][dr + 1] * im : T(0)));
                if (n < P) {
                    ax += w * (s_g[wid][0][dr] * re - (m ? s_g[wid][0][dr + 1] * im : T(0)));
                    ay += w * (s_g[wid][1][dr] * re - (m ? s_g[wid][1][dr + 1] * im : T(0)));
                    az += w * (s_g[wid][2][dr] * re - (m ? s_g[wid][2][dr + 1] * im : T(0)));
                }
            });
            gx = (double)ax * inv; gy = (double)ay * inv; gz = (double)az * inv;
            if (POT) phi = (double)ph;
            __syncwarp();
        }
        for (int64_t e = w0; e < w1; ++e) {
            const int c = tv.w_idx[e];
            if (POT)
                for (int d = lane; d < K; d += 32) s_c[wid][d] = (T)mpole[(size_t)c * K + d];
            for (int d = lane; d < KH; d += 32) {
                T g[3];
                mpole_grad_dof(mpole + (size_t)c * K, d, g);
                s_g[wid][0][d] = g[0]; s_g[wid][1][d] = g[1]; s_g[wid][2][d] = g[2];
            }
            __syncwarp();
            const double winv = 1.0 / (2.0 * tv.center[4 * c + 3]);
            const T ux = (T)((x - tv.center[4 * c]) * winv), uy = (T)((y - tv.center[4 * c + 1]) * winv),
                    uz = (T)((z - tv.center[4 * c + 2]) * winv);
            T ax = 0, ay = 0, az = 0, ph = 0;
            for_singular<P + 1>(ux, uy, uz, [&](int n, int m, T re, T im) {
                const T w = (m == 0) ? T(1) : T(2);
                const int dr = dof_re(n, m);
                if (POT && n <= P) ph += w * (s_c[wid][dr] * re - (m ? s_c[wid][dr + 1] * im : T(0)));
                ax += w * (s_g[wid][0][dr] * re - (m ? s_g[wid][0][dr + 1] * im : T(0)));
                ay += w * (s_g[wid][1][dr] * re - (m ? s_g[wid][1][dr + 1] * im : T(0)));
                az += w * (s_g[wid][2][dr] * re - (m ? s_g[wid][2][dr + 1] * im : T(0)));
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
