// ogx_noalloc.cu -- FP64 direct summation that allocates no device memory.
//
// ogx_eval on the direct solver stages the caller's host buffers in device
// memory the handle allocates.  Some callers cannot let a library allocate:
// cudaMalloc / cudaFree may synchronise the whole device and so stall every
// other stream of a latency-bound process, and processes that reserve their
// device memory up front under a fixed budget cannot have a library take more
// behind their back.  ogx_direct_eval_noalloc serves them: it stages bodies and
// results in one fixed array that the library image reserves on every GPU it is
// loaded on (kNoAllocMaxBodies bodies, 4 MiB, held until the process exits) and
// runs the same direct-sum kernel as the direct solver.
#include <mutex>

#include "ogx_internal.cuh"

namespace ogx {
namespace {

constexpr int64_t kNoAllocMaxBodies = 65536;
// staging layout, N = kNoAllocMaxBodies doubles each: pos (3N) | mass (N) | acc (3N) | pot (N)
static __device__ __align__(256) double g_noalloc_scratch[8 * kNoAllocMaxBodies];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_base[kMaxDevices] = {};

// Device address of the staging array on the current device, looked up once per
// device (with that device current).  Host code never uses the array's name as
// a device pointer: on the host it only identifies the symbol.
int noalloc_scratch(double** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) {
        set_last_error(OGX_ERR_NO_DEVICE, "no CUDA device");
        return OGX_ERR_NO_DEVICE;
    }
    if (dev >= kMaxDevices) {
        set_last_error(OGX_ERR_UNSUPPORTED, "device ordinal beyond the no-alloc table");
        return OGX_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_base[dev]) {
        double* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_last_error(OGX_ERR_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e));
            return OGX_ERR_CUDA;
        }
        g_noalloc_base[dev] = p;
    }
    *out = g_noalloc_base[dev];
    return OGX_OK;
}

}  // namespace
}  // namespace ogx

using namespace ogx;

extern "C" int ogx_direct_eval_noalloc(int64_t n, const double* pos, const double* mass, double G, double eps, double* acc,
                                       double* pot, void* stream) {
    if (n < 0 || (n > 0 && (!pos || !mass || !acc))) {
        set_last_error(OGX_ERR_INVALID, "ogx_direct_eval_noalloc: bad n or null buffer");
        return OGX_ERR_INVALID;
    }
    if (n > kNoAllocMaxBodies) {
        set_last_error(OGX_ERR_INVALID, "ogx_direct_eval_noalloc: n = " + std::to_string(n) +
                                            " exceeds the no-alloc maximum of " + std::to_string(kNoAllocMaxBodies) +
                                            " bodies");
        return OGX_ERR_INVALID;
    }
    const cudaStream_t st = (cudaStream_t)stream;
    if (st) {
        // the staging array is looked up for the current device: a stream of another
        // device would pair that device's work with this device's array
        int sdev = -1, cur = -1;
        OGX_CUDA(cudaStreamGetDevice(st, &sdev));
        OGX_CUDA(cudaGetDevice(&cur));
        if (sdev != cur) {
            set_last_error(OGX_ERR_INVALID, "ogx_direct_eval_noalloc: the stream belongs to device " +
                                                std::to_string(sdev) + ", the current device is " + std::to_string(cur));
            return OGX_ERR_INVALID;
        }
    }
    double* base = nullptr;
    OGX_TRY(noalloc_scratch(&base));
    if (n == 0) return OGX_OK;
    const int64_t N = kNoAllocMaxBodies;
    double* d_pos = base;
    double* d_mass = base + 3 * N;
    double* d_acc = base + 4 * N;
    double* d_pot = base + 7 * N;
    // every staged input is overwritten in full and the kernel writes every output
    // it is asked for, so no part of the array has to start at zero
    OGX_CUDA(cudaMemcpyAsync(d_pos, pos, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, st));
    OGX_CUDA(cudaMemcpyAsync(d_mass, mass, sizeof(double) * n, cudaMemcpyHostToDevice, st));
    OGX_TRY(direct_launch(d_pos, d_mass, n, G, eps * eps, d_acc, pot ? d_pot : nullptr, st));
    OGX_CUDA(cudaMemcpyAsync(acc, d_acc, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, st));
    if (pot) OGX_CUDA(cudaMemcpyAsync(pot, d_pot, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    OGX_CUDA(cudaStreamSynchronize(st));
    return OGX_OK;
}
