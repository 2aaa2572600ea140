// ogx_sort.cu -- stable LSD radix sort and exclusive scans.
//
// The tree build needs two stable sorts (the reference gets the same order
// from its recursive stable counting sort, src3d/AdaptiveOctree.hpp:114-118):
//   1. bodies by their 72-bit octant path (9 passes of 8 bits),
//   2. bodies by leaf id, starting from the original order, so that inside a
//      leaf the bodies keep their original index order (2-3 passes).
// Each pass: per-tile digit histogram -> one exclusive scan over
// (digit, tile) -> stable scatter.  The scatter ranks keys inside a warp with
// __match_any_sync, keeps per-warp digit counters in shared memory and
// orders warps by their contiguous sub-tiles, so the pass is stable.
#include "ogx_internal.cuh"

namespace ogx {
namespace {

constexpr int RS_THREADS = 256;
constexpr int RS_IPT = 16;
constexpr int RS_TILE = RS_THREADS * RS_IPT;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr unsigned FULL = 0xffffffffu;

struct Key32 {
    uint32_t* k;
    using T = uint32_t;
    __device__ __forceinline__ T load(int64_t i) const { return k[i]; }
    __device__ __forceinline__ void store(int64_t i, T v) const { k[i] = v; }
    __device__ __forceinline__ static uint32_t digit(T v, int pass) { return (v >> (8 * pass)) & 0xFFu; }
};

struct K72 {
    uint64_t hi;
    uint32_t lo;
};
struct Key72 {
    uint64_t* hi;
    uint32_t* lo;
    using T = K72;
    __device__ __forceinline__ T load(int64_t i) const { return K72{hi[i], lo[i]}; }
    __device__ __forceinline__ void store(int64_t i, T v) const { hi[i] = v.hi; lo[i] = v.lo; }
    // digit `pass` of the 72-bit value (hi << 9) | lo
    __device__ __forceinline__ static uint32_t digit(T v, int pass) {
        if (pass == 0) return v.lo & 0xFFu;
        if (pass == 1) return ((v.lo >> 8) & 1u) | (uint32_t)((v.hi & 0x7Full) << 1);
        return (uint32_t)((v.hi >> (8 * pass - 9)) & 0xFFull);
    }
};

template <class KO>
__global__ void __launch_bounds__(RS_THREADS) rs_hist(KO keys, int64_t n, int pass, uint32_t* hist, int nblocks) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int64_t start = (int64_t)blockIdx.x * RS_TILE;
    for (int k = threadIdx.x; k < RS_TILE; k += RS_THREADS) {
        const int64_t i = start + k;
        const bool valid = i < n;
        const uint32_t d = valid ? KO::digit(keys.load(i), pass) : 0xFFFFFFFFu;
        const unsigned peers = __match_any_sync(FULL, d);
        if (valid && lane == __ffs(peers) - 1) atomicAdd(&h[d], (uint32_t)__popc(peers));
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Digit-major histogram hist[d * nblocks + b] -> exclusive offsets within each digit
// (one CTA per digit, coalesced over the tiles), digit totals into tot[d].
__global__ void __launch_bounds__(1024) rs_scan_digit(uint32_t* hist, int nblocks, uint32_t* tot) {
    __shared__ uint32_t warp_sum[32];
    __shared__ uint32_t carry;
    uint32_t* a = hist + (size_t)blockIdx.x * nblocks;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    if (t == 0) carry = 0;
    __syncthreads();
    for (int b0 = 0; b0 < nblocks; b0 += 1024) {
        const int i = b0 + t;
        const uint32_t v = (i < nblocks) ? a[i] : 0u;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(FULL, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sum[w] = x;
        __syncthreads();
        if (w == 0) {
            uint32_t s = warp_sum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(FULL, s, o);
                if (lane >= o) s += y;
            }
            warp_sum[lane] = s;
        }
        __syncthreads();
        const uint32_t ex = carry + (w > 0 ? warp_sum[w - 1] : 0u) + x - v;
        if (i < nblocks) a[i] = ex;
        __syncthreads();
        if (t == 0) carry += warp_sum[31];
        __syncthreads();
    }
    if (t == 0) tot[blockIdx.x] = carry;
}

// exclusive scan of the 256 digit totals (in place)
__global__ void __launch_bounds__(256) rs_scan_totals(uint32_t* tot) {
    __shared__ uint32_t s[256];
    const int t = threadIdx.x;
    const uint32_t v = tot[t];
    s[t] = v;
    __syncthreads();
    for (int o = 1; o < 256; o <<= 1) {
        const uint32_t y = (t >= o) ? s[t - o] : 0u;
        __syncthreads();
        s[t] += y;
        __syncthreads();
    }
    tot[t] = s[t] - v;
}

template <class KO>
__global__ void __launch_bounds__(RS_THREADS) rs_scatter(KO kin, KO kout, const uint32_t* vin, uint32_t* vout, int64_t n,
                                                         int pass, const uint32_t* scanned, int nblocks, const uint32_t* digit_base) {
    __shared__ uint32_t wcnt[RS_WARPS][256];
    __shared__ uint32_t gbase[256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < RS_WARPS * 256; i += RS_THREADS) (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    const int64_t base = (int64_t)blockIdx.x * RS_TILE + (int64_t)w * 32 * RS_IPT;
    typename KO::T key[RS_IPT];
    uint32_t val[RS_IPT], loc[RS_IPT], dig[RS_IPT];
#pragma unroll
    for (int r = 0; r < RS_IPT; ++r) {
        const int64_t i = base + r * 32 + lane;
        const bool valid = i < n;
        uint32_t d = 0xFFFFFFFFu;
        if (valid) {
            key[r] = kin.load(i);
            val[r] = vin[i];
            d = KO::digit(key[r], pass);
        }
        const unsigned peers = __match_any_sync(FULL, d);
        uint32_t l = 0;
        if (valid) l = wcnt[w][d] + __popc(peers & lt);
        __syncwarp();
        if (valid && lane == __ffs(peers) - 1) wcnt[w][d] += __popc(peers);
        __syncwarp();
        loc[r] = l;
        dig[r] = d;
    }
    __syncthreads();
    {
        const int d = threadIdx.x;  // RS_THREADS == 256 bins
        uint32_t run = 0;
#pragma unroll
        for (int ww = 0; ww < RS_WARPS; ++ww) {
            const uint32_t c = wcnt[ww][d];
            wcnt[ww][d] = run;
            run += c;
        }
        gbase[d] = digit_base[d] + scanned[(int64_t)d * nblocks + blockIdx.x];
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_IPT; ++r) {
        const int64_t i = base + r * 32 + lane;
        if (i < n) {
            const uint32_t d = dig[r];
            const int64_t pos = (int64_t)gbase[d] + wcnt[w][d] + loc[r];
            kout.store(pos, key[r]);
            vout[pos] = val[r];
        }
    }
}

// ---- generic exclusive scan int32 -> int64 (out has n+1 entries) --------------
constexpr int SC_THREADS = 1024;
constexpr int SC_IPT = 4;
constexpr int SC_TILE = SC_THREADS * SC_IPT;

__device__ __forceinline__ int64_t block_excl_scan_i64(int64_t v, int64_t* sh, int64_t* total) {
    // sh: 32 int64 scratch
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int64_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[w] = x;
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        int64_t s = (lane < nw) ? sh[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(FULL, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) sh[lane] = s;
    }
    __syncthreads();
    const int64_t wpre = (w > 0) ? sh[w - 1] : 0;
    if (total) *total = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return wpre + x - v;
}

__global__ void __launch_bounds__(SC_THREADS) sc_partials(const int* in, int64_t n, int64_t* part) {
    __shared__ int64_t sh[32];
    const int64_t b = (int64_t)blockIdx.x * SC_TILE + (int64_t)threadIdx.x * SC_IPT;
    int64_t s = 0;
#pragma unroll
    for (int k = 0; k < SC_IPT; ++k)
        if (b + k < n) s += in[b + k];
    int64_t tot;
    block_excl_scan_i64(s, sh, &tot);
    if (threadIdx.x == 0) part[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SC_THREADS) sc_scan_partials(int64_t* part, int64_t m) {
    __shared__ int64_t sh[32];
    __shared__ int64_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int64_t b = 0; b < m; b += SC_THREADS) {
        const int64_t i = b + threadIdx.x;
        const int64_t v = (i < m) ? part[i] : 0;
        int64_t tot;
        const int64_t ex = block_excl_scan_i64(v, sh, &tot);
        if (i < m) part[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) part[m] = carry;
}

__global__ void __launch_bounds__(SC_THREADS) sc_finish(const int* in, int64_t n, const int64_t* part, int64_t* out, int nparts) {
    __shared__ int64_t sh[32];
    const int64_t b = (int64_t)blockIdx.x * SC_TILE + (int64_t)threadIdx.x * SC_IPT;
    int64_t v[SC_IPT];
    int64_t s = 0;
#pragma unroll
    for (int k = 0; k < SC_IPT; ++k) {
        v[k] = (b + k < n) ? in[b + k] : 0;
        s += v[k];
    }
    int64_t run = part[blockIdx.x] + block_excl_scan_i64(s, sh, nullptr);
#pragma unroll
    for (int k = 0; k < SC_IPT; ++k) {
        if (b + k < n) out[b + k] = run;
        run += v[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = part[nparts];
}

}  // namespace

int scan_i32_to_i64(Handle& h, const int* in, int64_t* out, int64_t n) {
    const int nparts = (int)((n + SC_TILE - 1) / SC_TILE);
    int64_t* part;
    OGX_TRY(arena_get(h.ws, S_SCAN_TMP, (size_t)nparts + 1, &part));
    if (n == 0) {
        OGX_CUDA(cudaMemsetAsync(out, 0, sizeof(int64_t), h.stream));
        return OGX_OK;
    }
    sc_partials<<<nparts, SC_THREADS, 0, h.stream>>>(in, n, part); ++h.launches;
    sc_scan_partials<<<1, SC_THREADS, 0, h.stream>>>(part, nparts); ++h.launches;
    sc_finish<<<nparts, SC_THREADS, 0, h.stream>>>(in, n, part, out, nparts); ++h.launches;
    OGX_CUDA(cudaGetLastError());
    return OGX_OK;
}

template <class KO>
static int radix_passes(Handle& h, KO a, KO b, uint32_t* va, uint32_t* vb, int64_t n, int npasses, int* which,
                        int first_pass = 0) {
    const int nblocks = (int)((n + RS_TILE - 1) / RS_TILE);
    uint32_t* hist;
    OGX_TRY(arena_get(h.ws, S_RS_HIST, (size_t)256 * nblocks + 256, &hist));
    uint32_t* tot = hist + (size_t)256 * nblocks;
    KO src = a, dst = b;
    uint32_t *vs = va, *vd = vb;
    for (int pass = first_pass; pass < npasses; ++pass) {
        rs_hist<KO><<<nblocks, RS_THREADS, 0, h.stream>>>(src, n, pass, hist, nblocks); ++h.launches;
        rs_scan_digit<<<256, 1024, 0, h.stream>>>(hist, nblocks, tot); ++h.launches;
        rs_scan_totals<<<1, 256, 0, h.stream>>>(tot); ++h.launches;
        rs_scatter<KO><<<nblocks, RS_THREADS, 0, h.stream>>>(src, dst, vs, vd, n, pass, hist, nblocks, tot); ++h.launches;
        std::swap(src, dst);
        std::swap(vs, vd);
    }
    OGX_CUDA(cudaGetLastError());
    *which = (npasses - first_pass) & 1;  // 0: result in a, 1: result in b
    return OGX_OK;
}

int radix_sort_u32(Handle& h, Slot kin, Slot vin, Slot kalt, Slot valt, int64_t n, int bits, uint32_t** kout,
                   uint32_t** vout) {
    uint32_t *k0, *v0, *k1, *v1;
    OGX_TRY(arena_get(h.ws, kin, n, &k0));
    OGX_TRY(arena_get(h.ws, vin, n, &v0));
    OGX_TRY(arena_get(h.ws, kalt, n, &k1));
    OGX_TRY(arena_get(h.ws, valt, n, &v1));
    int npasses = (bits + 7) / 8;
    if (npasses < 1) npasses = 1;
    int which = 0;
    if (n > 0) OGX_TRY(radix_passes(h, Key32{k0}, Key32{k1}, v0, v1, n, npasses, &which));
    *kout = which ? k1 : k0;
    *vout = which ? v1 : v0;
    return OGX_OK;
}

int radix_sort_key72(Handle& h, int64_t n, int first_pass, uint64_t** khi, uint32_t** klo, uint32_t** idx) {
    uint64_t *h0, *h1;
    uint32_t *l0, *l1, *i0, *i1;
    OGX_TRY(arena_get(h.ws, S_KHI, n, &h0));
    OGX_TRY(arena_get(h.ws, S_KLO, n, &l0));
    OGX_TRY(arena_get(h.ws, S_IDX, n, &i0));
    OGX_TRY(arena_get(h.ws, S_KHI2, n, &h1));
    OGX_TRY(arena_get(h.ws, S_KLO2, n, &l1));
    OGX_TRY(arena_get(h.ws, S_IDX2, n, &i1));
    int which = 0;
    if (n > 0) OGX_TRY(radix_passes(h, Key72{h0, l0}, Key72{h1, l1}, i0, i1, n, 9, &which, first_pass));
    *khi = which ? h1 : h0;
    *klo = which ? l1 : l0;
    *idx = which ? i1 : i0;
    return OGX_OK;
}

}  // namespace ogx
