// ogx_direct.cu -- all-pairs direct summation on the GPU (the FP64 oracle path).
//
// Replaces DirectSolver3D::computeAccelerations (src3d/DirectSolver3D.hpp:15-34):
//   a_i = G sum_{j != i} m_j (r_j - r_i) / (|r_j - r_i|^2 + eps^2)^{3/2}
// The reference walks unique pairs i<j and applies Newton's third law; on the
// GPU every target sums its own row (no write conflicts), sources stream
// through shared memory in tiles of 256 bodies packed as (x, y, z, m).
// (|d|^2+eps^2)^{-3/2} is formed from the double-precision rsqrt cubed.
// The optional potential is pot_i = -G sum_{j != i} m_j / sqrt(|d|^2 + eps^2)
// (Kernel3D.hpp:39-42 per body, without the m_i factor).
// With OGX_SOFT_SPLINE every pair takes the spline kernel (ogx_softening.cuh) instead.
#include "ogx_internal.cuh"
#include "ogx_softening.cuh"

namespace ogx {
namespace {

constexpr int DT = 256;

// SOFT: the spline kernel of support hs (ogx_softening.cuh) instead of Plummer's eps2
template <class T, bool POT, bool SOFT = false>
__global__ void __launch_bounds__(DT) k_direct(const double* __restrict__ pos, const double* __restrict__ mass, int64_t n, T G,
                                               T eps2, double* __restrict__ acc, double* __restrict__ pot, T hs = 0,
                                               T hinv = 0) {
    __shared__ T s[DT][4];
    const int64_t i = blockIdx.x * (int64_t)DT + threadIdx.x;
    const bool act = i < n;
    const T xi = act ? (T)pos[3 * i] : T(0), yi = act ? (T)pos[3 * i + 1] : T(0), zi = act ? (T)pos[3 * i + 2] : T(0);
    T ax = 0, ay = 0, az = 0, ph = 0;
    for (int64_t t0 = 0; t0 < n; t0 += DT) {
        const int64_t j = t0 + threadIdx.x;
        __syncthreads();
        if (j < n) {
            s[threadIdx.x][0] = (T)pos[3 * j];
            s[threadIdx.x][1] = (T)pos[3 * j + 1];
            s[threadIdx.x][2] = (T)pos[3 * j + 2];
            s[threadIdx.x][3] = (T)mass[j];
        } else {
            s[threadIdx.x][0] = s[threadIdx.x][1] = s[threadIdx.x][2] = s[threadIdx.x][3] = T(0);
        }
        __syncthreads();
        const int lim = (int)min((int64_t)DT, n - t0);
        if (i >= t0 && i < t0 + lim) {
            // tile holding the target itself: skip j == i
            for (int k = 0; k < lim; ++k) {
                if (t0 + k == i) continue;
                const T dx = s[k][0] - xi, dy = s[k][1] - yi, dz = s[k][2] - zi;
                if constexpr (SOFT) {
                    T g, kk;
                    spline_gk<T>(dx * dx + dy * dy + dz * dz, hs, hinv, g, kk);
                    const T w = s[k][3] * g;
                    ax += w * dx; ay += w * dy; az += w * dz;
                    if (POT) ph += s[k][3] * kk;
                } else {
                    const T r2 = dx * dx + dy * dy + dz * dz + eps2;
                    const T ir = rsqrt(r2);
                    const T w = s[k][3] * ir * ir * ir;
                    ax += w * dx; ay += w * dy; az += w * dz;
                    if (POT) ph += s[k][3] * ir;
                }
            }
        } else {
#pragma unroll 4
            for (int k = 0; k < lim; ++k) {
                const T dx = s[k][0] - xi, dy = s[k][1] - yi, dz = s[k][2] - zi;
                if constexpr (SOFT) {
                    T g, kk;
                    spline_gk<T>(dx * dx + dy * dy + dz * dz, hs, hinv, g, kk);
                    const T w = s[k][3] * g;
                    ax += w * dx; ay += w * dy; az += w * dz;
                    if (POT) ph += s[k][3] * kk;
                } else {
                    const T r2 = dx * dx + dy * dy + dz * dz + eps2;
                    const T ir = rsqrt(r2);
                    const T w = s[k][3] * ir * ir * ir;
                    ax += w * dx; ay += w * dy; az += w * dz;
                    if (POT) ph += s[k][3] * ir;
                }
            }
        }
    }
    if (act) {
        acc[3 * i] = (double)(G * ax);
        acc[3 * i + 1] = (double)(G * ay);
        acc[3 * i + 2] = (double)(G * az);
        if (POT) pot[i] = -(double)(G * ph);
    }
}

}  // namespace

// FP64 direct sum on caller-provided device buffers and stream (no handle)
int direct_launch(const double* d_pos, const double* d_mass, int64_t n, double G, double eps2, double* d_acc, double* d_pot,
                  cudaStream_t st) {
    if (n == 0) return OGX_OK;
    const int grid = (int)((n + DT - 1) / DT);
    if (d_pot) k_direct<double, true><<<grid, DT, 0, st>>>(d_pos, d_mass, n, G, eps2, d_acc, d_pot);
    else k_direct<double, false><<<grid, DT, 0, st>>>(d_pos, d_mass, n, G, eps2, d_acc, nullptr);
    OGX_CUDA(cudaGetLastError());
    return OGX_OK;
}

int direct_eval(Handle& h, const double* d_pos, const double* d_mass, int64_t n, double* d_acc, double* d_pot, bool fp32) {
    if (n == 0) return OGX_OK;
    const int grid = (int)((n + DT - 1) / DT);
    const double eps2 = h.prm.eps * h.prm.eps;
    if (h.prm.softening == OGX_SOFT_SPLINE && !fp32) {
        const double hs = spline_support(h.prm.eps), hinv = hs > 0.0 ? 1.0 / hs : 0.0;
        if (d_pot) k_direct<double, true, true><<<grid, DT, 0, h.stream>>>(d_pos, d_mass, n, h.prm.G, eps2, d_acc, d_pot, hs, hinv);
        else k_direct<double, false, true><<<grid, DT, 0, h.stream>>>(d_pos, d_mass, n, h.prm.G, eps2, d_acc, nullptr, hs, hinv);
        ++h.launches;
        OGX_CUDA(cudaGetLastError());
        return OGX_OK;
    }
    if (fp32) {
        if (d_pot) { k_direct<float, true><<<grid, DT, 0, h.stream>>>(d_pos, d_mass, n, (float)h.prm.G, (float)eps2, d_acc, d_pot); ++h.launches; }
        else { k_direct<float, false><<<grid, DT, 0, h.stream>>>(d_pos, d_mass, n, (float)h.prm.G, (float)eps2, d_acc, nullptr); ++h.launches; }
    } else {
        if (d_pot) { k_direct<double, true><<<grid, DT, 0, h.stream>>>(d_pos, d_mass, n, h.prm.G, eps2, d_acc, d_pot); ++h.launches; }
        else { k_direct<double, false><<<grid, DT, 0, h.stream>>>(d_pos, d_mass, n, h.prm.G, eps2, d_acc, nullptr); ++h.launches; }
    }
    OGX_CUDA(cudaGetLastError());
    return OGX_OK;
}

}  // namespace ogx
