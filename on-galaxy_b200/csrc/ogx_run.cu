// ogx_run.cu -- device-side support for running a simulation: the two-galaxy
// merger initial conditions, FP64 energy / momentum diagnostics, species tags
// and float32 position frames.
//
// Replaces the host loops of the reference's driver:
//   makeDisk / setCircularVelocities / placeGalaxy / concat   src3d/gpu/GalaxyIC.hpp:43-125
//   the merger set-up of galaxy_sim                           src3d/gpu/galaxy_sim.cu:113-137
//   computeDiagnostics (O(N^2) pair sum)                      src3d/Diagnostics3D.hpp:20-38
//   comSep (centre-of-mass separation of the two galaxies)    src3d/gpu/galaxy_sim.cu:209-216
//   dumpFrame (float32 positions, original order)             src3d/gpu/galaxy_sim.cu:186-193
// The initial conditions follow the benchmark workload's profiles (80% exponential
// sech^2 disk, 20% Hernquist bulge, velocities v_c^2 = -a_R R from the FP64 field
// plus dispersion), drawn on the device from a counter-based Philox4x32-10
// generator (Salmon, Moraes, Dror, Shaw, SC'11), so a body's draws depend only on
// (seed, galaxy, body index).
#include <cmath>

#include "ogx_internal.cuh"

namespace ogx {
namespace {

// ---- Philox4x32-10: 10 rounds of the 4x32 Philox bijection, keyed per stream -----
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}

// two doubles in [0, 1) with 53 random bits each
__device__ __forceinline__ void uniform2(uint4 r, double& a, double& b) {
    a = ((double)(r.x >> 5) * 67108864.0 + (double)(r.y >> 6)) * (1.0 / 9007199254740992.0);
    b = ((double)(r.z >> 5) * 67108864.0 + (double)(r.w >> 6)) * (1.0 / 9007199254740992.0);
}

// draw block `blk` of body i: 4 uniforms
__device__ __forceinline__ void draw4(uint64_t seed, int g, int64_t i, uint32_t blk, double u[4]) {
    const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32) ^ (0x51ED2701u * (uint32_t)(g + 1)));
    const uint4 ctr = make_uint4((uint32_t)i, (uint32_t)((uint64_t)i >> 32), blk, 0u);
    uint4 r0 = philox4x32_10(ctr, key);
    uint4 r1 = philox4x32_10(make_uint4(ctr.x, ctr.y, ctr.z, 1u), key);
    uniform2(r0, u[0], u[1]);
    uniform2(r1, u[2], u[3]);
}

// Gamma(2) CDF on x >= 0 and its inverse by bisection (monotone, 60 halvings)
__device__ __forceinline__ double gamma2_cdf(double x) { return 1.0 - (1.0 + x) * exp(-x); }
__device__ double gamma2_inv(double u, double xmax) {
    double lo = 0.0, hi = xmax;
    for (int it = 0; it < 60; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (gamma2_cdf(mid) < u) lo = mid; else hi = mid;
    }
    return 0.5 * (lo + hi);
}

struct GalaxyProfile {
    double Rd, z0, Md, ab, Mb;
    int64_t nd, nb;
};

// body i of one galaxy, galaxy frame: disk bodies 0..nd-1, bulge nd..nd+nb-1
__global__ void k_ic_galaxy(GalaxyProfile gp, uint64_t seed, int g, double* __restrict__ pos, double* __restrict__ mass) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t n = gp.nd + gp.nb;
    if (i >= n) return;
    double u[4];
    draw4(seed, g, i, 0u, u);
    double x, y, z, m;
    if (i < gp.nd) {
        // exponential surface density ~ exp(-R/Rd): R/Rd ~ Gamma(2), cut at 10 Rd
        const double R = gp.Rd * gamma2_inv(u[0] * gamma2_cdf(10.0), 10.0);
        const double ph = 2.0 * M_PI * u[1];
        // sech^2(z/z0): CDF (1 + tanh(z/z0)) / 2, cut at |z| <= 10 z0
        z = gp.z0 * atanh((2.0 * u[2] - 1.0) * tanh(10.0));
        x = R * cos(ph);
        y = R * sin(ph);
        m = gp.Md / (double)max(gp.nd, (int64_t)1);
    } else {
        // Hernquist: M(<r)/Mb = r^2 / (r + a)^2 -> r = a s / (1 - s), s = sqrt(u), cut at 50 a
        const double s = sqrt(u[0] * (50.0 / 51.0) * (50.0 / 51.0));
        const double r = gp.ab * s / (1.0 - s);
        const double cz = 2.0 * u[1] - 1.0, sz = sqrt(fmax(0.0, 1.0 - cz * cz)), ph = 2.0 * M_PI * u[2];
        x = r * sz * cos(ph);
        y = r * sz * sin(ph);
        z = r * cz;
        m = gp.Mb / (double)max(gp.nb, (int64_t)1);
    }
    pos[3 * i] = x;
    pos[3 * i + 1] = y;
    pos[3 * i + 2] = z;
    mass[i] = m;
}

// circular velocity from the measured FP64 field, v_c^2 = -a_R R, tangential in
// the disk plane, plus an isotropic Gaussian dispersion disp * v_c (Box-Muller)
__global__ void k_ic_velocities(int64_t n, uint64_t seed, int g, double disp, const double* __restrict__ pos,
                                const double* __restrict__ acc, double* __restrict__ vel) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = pos[3 * i], y = pos[3 * i + 1];
    const double R = sqrt(x * x + y * y);
    double vx = 0.0, vy = 0.0, vc = 0.0;
    if (R > 1e-6) {
        const double ar = (acc[3 * i] * x + acc[3 * i + 1] * y) / R;
        vc = sqrt(fmax(-ar * R, 0.0));
        vx = -vc * y / R;
        vy = vc * x / R;
    }
    double u[4];
    draw4(seed, g, i, 1u, u);
    const double r1 = sqrt(-2.0 * log(fmax(u[0], 1e-300))), r2 = sqrt(-2.0 * log(fmax(u[2], 1e-300)));
    const double sig = disp * vc;
    vel[3 * i] = vx + sig * r1 * cos(2.0 * M_PI * u[1]);
    vel[3 * i + 1] = vy + sig * r1 * sin(2.0 * M_PI * u[1]);
    vel[3 * i + 2] = sig * r2 * cos(2.0 * M_PI * u[3]);
}

// placeGalaxy: rotate by `incl` about x, then shift by centre / bulk velocity
__global__ void k_ic_place(int64_t n, double c, double s, double cx, double vx, double* pos, double* vel,
                           int8_t* species, int8_t tag) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double py = pos[3 * i + 1], pz = pos[3 * i + 2];
    pos[3 * i] += cx;
    pos[3 * i + 1] = c * py - s * pz;
    pos[3 * i + 2] = s * py + c * pz;
    const double wy = vel[3 * i + 1], wz = vel[3 * i + 2];
    vel[3 * i] += vx;
    vel[3 * i + 1] = c * wy - s * wz;
    vel[3 * i + 2] = s * wy + c * wz;
    species[i] = tag;
}

// ---- diagnostics: fixed-order FP64 reductions (deterministic) -------------------------
// per body: 0 kinetic 1/2 m v^2, 1 potential 1/2 m pot, 2-4 momentum m v, 5-7 angular
// momentum m r x v, 8-11 species-0 mass and m r, 12-15 the same for the other species
constexpr int DIAG_Q = 16;
constexpr int DIAG_BLOCKS = 256;
constexpr int DIAG_THREADS = 256;

__global__ void __launch_bounds__(DIAG_THREADS) k_diag_partial(int64_t n, const double* __restrict__ pos,
                                                               const double* __restrict__ vel,
                                                               const double* __restrict__ mass,
                                                               const double* __restrict__ pot,
                                                               const int8_t* __restrict__ species, double* part) {
    __shared__ double s[DIAG_Q][DIAG_THREADS];
    double a[DIAG_Q];
#pragma unroll
    for (int q = 0; q < DIAG_Q; ++q) a[q] = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)DIAG_THREADS + threadIdx.x; i < n; i += (int64_t)DIAG_BLOCKS * DIAG_THREADS) {
        const double m = mass[i];
        const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
        const double vx = vel[3 * i], vy = vel[3 * i + 1], vz = vel[3 * i + 2];
        a[0] += 0.5 * m * (vx * vx + vy * vy + vz * vz);
        a[1] += 0.5 * m * pot[i];
        a[2] += m * vx; a[3] += m * vy; a[4] += m * vz;
        a[5] += m * (y * vz - z * vy); a[6] += m * (z * vx - x * vz); a[7] += m * (x * vy - y * vx);
        const int o = (species && species[i] != 0) ? 12 : 8;
        a[o] += m; a[o + 1] += m * x; a[o + 2] += m * y; a[o + 3] += m * z;
    }
#pragma unroll
    for (int q = 0; q < DIAG_Q; ++q) s[q][threadIdx.x] = a[q];
    __syncthreads();
    for (int w = DIAG_THREADS / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int q = 0; q < DIAG_Q; ++q) s[q][threadIdx.x] += s[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < DIAG_Q) part[(size_t)blockIdx.x * DIAG_Q + threadIdx.x] = s[threadIdx.x][0];
}

__global__ void k_diag_final(const double* __restrict__ part, double* out) {
    const int q = threadIdx.x;
    if (q >= DIAG_Q) return;
    double v = 0.0;
    for (int b = 0; b < DIAG_BLOCKS; ++b) v += part[(size_t)b * DIAG_Q + q];
    out[q] = v;
}

__global__ void k_to_f32(int64_t n3, const double* __restrict__ src, float* __restrict__ dst) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n3) dst[i] = (float)src[i];
}

struct DevScope {
    int prev = -1;
    explicit DevScope(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DevScope() {
        int cur;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

inline int blocks_for(int64_t n, int b) { return (int)((n + b - 1) / b); }

}  // namespace
}  // namespace ogx

using namespace ogx;

extern "C" {

int ogx_merger_params_default(ogx_merger_params* mp) {
    if (!mp) return OGX_ERR_INVALID;
    mp->n_per = 500000;
    mp->seed = 1;
    mp->sep = 5.0;
    mp->vrel = 0.5;
    mp->tilt_deg = 30.0;
    mp->disp_frac = 0.1;
    mp->Rd = 1.0;
    mp->z0 = 0.1;
    mp->Md = 1.0;
    mp->ab = 0.2;
    mp->Mb = 0.25;
    mp->bulge_frac = 0.2;
    return OGX_OK;
}

int ogx_ic_merger(void* handle, const ogx_merger_params* mp, int8_t* species_out) {
    if (!handle || !mp || mp->n_per < 2 || mp->n_per > (int64_t)INT32_MAX / 4 || !(mp->bulge_frac >= 0.0) ||
        !(mp->bulge_frac <= 1.0) || !(mp->Rd > 0) || !(mp->z0 > 0) || !(mp->ab > 0))
        return OGX_ERR_INVALID;
    Handle& h = *static_cast<Handle*>(handle);
    DevScope ds(h.device);
    drop_step_graph(h);   // a new system: new sizes and capacities
    const int64_t np = mp->n_per, n = 2 * np;
    double *dp, *dv, *dm, *da, *dacc;
    int8_t* dsp;
    OGX_TRY(arena_get(h.ws, S_POS, 3 * n, &dp));
    OGX_TRY(arena_get(h.ws, S_VEL, 3 * n, &dv));
    OGX_TRY(arena_get(h.ws, S_MASS, n, &dm));
    OGX_TRY(arena_get(h.ws, S_ACC, 3 * n, &da));
    OGX_TRY(arena_get(h.ws, S_IC_ACC, 3 * np, &dacc));
    OGX_TRY(arena_get(h.ws, S_SPECIES, n, &dsp));
    GalaxyProfile gp;
    gp.Rd = mp->Rd; gp.z0 = mp->z0; gp.Md = mp->Md; gp.ab = mp->ab; gp.Mb = mp->Mb;
    gp.nb = (int64_t)llround(mp->bulge_frac * (double)np);
    gp.nd = np - gp.nb;
    const int saved_prec = h.prm.precision;
    h.prm.precision = OGX_PREC_FP64;  // the circular-velocity field is the FP64 solve
    int rc = OGX_OK;
    for (int g = 0; g < 2 && rc == OGX_OK; ++g) {
        double* pg = dp + 3 * g * np;
        double* vg = dv + 3 * g * np;
        double* mg = dm + g * np;
        k_ic_galaxy<<<blocks_for(np, 256), 256, 0, h.stream>>>(gp, mp->seed, g, pg, mg);
        rc = eval_device_shared(h, np, pg, mg, dacc, nullptr);
        if (rc != OGX_OK) break;
        k_ic_velocities<<<blocks_for(np, 256), 256, 0, h.stream>>>(np, mp->seed, g, mp->disp_frac, pg, dacc, vg);
        const double incl = (g == 0 ? 0.0 : mp->tilt_deg) * M_PI / 180.0;
        k_ic_place<<<blocks_for(np, 256), 256, 0, h.stream>>>(np, cos(incl), sin(incl), g == 0 ? -mp->sep : mp->sep,
                                                              g == 0 ? 0.5 * mp->vrel : -0.5 * mp->vrel, pg, vg,
                                                              dsp + g * np, (int8_t)g);
        h.launches += 3;
    }
    h.prm.precision = saved_prec;
    OGX_TRY(rc);
    OGX_CUDA(cudaGetLastError());
    // VelocityVerlet3D::initialize with the handle's own form
    OGX_TRY(eval_device_shared(h, n, dp, dm, da, nullptr));
    finish_stats_shared(h);
    h.resident = true;
    h.n = n;
    h.species_set = true;
    if (species_out) {
        OGX_CUDA(cudaMemcpyAsync(species_out, dsp, n, cudaMemcpyDeviceToHost, h.stream));
        OGX_CUDA(cudaStreamSynchronize(h.stream));
    }
    return OGX_OK;
}

int ogx_set_species(void* handle, const int8_t* species) {
    if (!handle || !species) return OGX_ERR_INVALID;
    Handle& h = *static_cast<Handle*>(handle);
    if (!h.resident) return OGX_ERR_STATE;
    DevScope ds(h.device);
    int8_t* dsp;
    OGX_TRY(arena_get(h.ws, S_SPECIES, h.n, &dsp));
    OGX_CUDA(cudaMemcpyAsync(dsp, species, h.n, cudaMemcpyHostToDevice, h.stream));
    OGX_CUDA(cudaStreamSynchronize(h.stream));
    h.species_set = true;
    return OGX_OK;
}

int ogx_diagnostics(void* handle, double* out) {
    if (!handle || !out) return OGX_ERR_INVALID;
    Handle& h = *static_cast<Handle*>(handle);
    if (!h.resident) return OGX_ERR_STATE;
    DevScope ds(h.device);
    const int64_t n = h.n;
    double *dp, *dv, *dm, *dpot, *dacc, *part;
    int8_t* dsp = nullptr;
    OGX_TRY(arena_get(h.ws, S_POS, 3 * n, &dp));
    OGX_TRY(arena_get(h.ws, S_VEL, 3 * n, &dv));
    OGX_TRY(arena_get(h.ws, S_MASS, n, &dm));
    OGX_TRY(arena_get(h.ws, S_DIAG_POT, n, &dpot));
    OGX_TRY(arena_get(h.ws, S_DIAG_ACC, 3 * n, &dacc));
    OGX_TRY(arena_get(h.ws, S_DIAG_PART, DIAG_BLOCKS * DIAG_Q + DIAG_Q, &part));
    if (h.species_set) OGX_TRY(arena_get(h.ws, S_SPECIES, n, &dsp));
    // potentials at the current positions (the handle's form)
    OGX_TRY(eval_device_shared(h, n, dp, dm, dacc, dpot));
    k_diag_partial<<<DIAG_BLOCKS, DIAG_THREADS, 0, h.stream>>>(n, dp, dv, dm, dpot, dsp, part);
    k_diag_final<<<1, 32, 0, h.stream>>>(part, part + DIAG_BLOCKS * DIAG_Q);
    h.launches += 2;
    double r[DIAG_Q];
    OGX_CUDA(cudaMemcpyAsync(r, part + DIAG_BLOCKS * DIAG_Q, sizeof(r), cudaMemcpyDeviceToHost, h.stream));
    OGX_CUDA(cudaStreamSynchronize(h.stream));
    out[0] = r[0];
    out[1] = r[1];
    out[2] = r[0] + r[1];
    for (int k = 0; k < 6; ++k) out[3 + k] = r[2 + k];
    double c0[3] = {0, 0, 0}, c1[3] = {0, 0, 0};
    for (int k = 0; k < 3; ++k) {
        c0[k] = r[8] > 0 ? r[9 + k] / r[8] : 0.0;
        c1[k] = r[12] > 0 ? r[13 + k] / r[12] : 0.0;
        out[9 + k] = c0[k];
        out[12 + k] = c1[k];
    }
    out[15] = (r[8] > 0 && r[12] > 0) ? std::sqrt((c0[0] - c1[0]) * (c0[0] - c1[0]) + (c0[1] - c1[1]) * (c0[1] - c1[1]) +
                                                  (c0[2] - c1[2]) * (c0[2] - c1[2]))
                                      : 0.0;
    return OGX_OK;
}

int ogx_download_frame(void* handle, float* pos_f32) {
    if (!handle || !pos_f32) return OGX_ERR_INVALID;
    Handle& h = *static_cast<Handle*>(handle);
    if (!h.resident) return OGX_ERR_STATE;
    DevScope ds(h.device);
    const int64_t n3 = 3 * h.n;
    double* dp;
    float* fr;
    OGX_TRY(arena_get(h.ws, S_POS, n3, &dp));
    OGX_TRY(arena_get(h.ws, S_FRAME, n3, &fr));
    k_to_f32<<<blocks_for(n3, 256), 256, 0, h.stream>>>(n3, dp, fr);
    ++h.launches;
    OGX_CUDA(cudaMemcpyAsync(pos_f32, fr, n3 * sizeof(float), cudaMemcpyDeviceToHost, h.stream));
    OGX_CUDA(cudaStreamSynchronize(h.stream));
    return OGX_OK;
}

}  // extern "C"
