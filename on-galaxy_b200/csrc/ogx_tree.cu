// ogx_tree.cu -- adaptive octree and CGR interaction lists on the GPU.
//
// Replaces AdaptiveOctree::build/subdivide/buildLists
// (src3d/AdaptiveOctree.hpp:65-189), which the reference runs recursively on
// one CPU core.  The boxes, body order and U/V/W/X lists produced here are
// the reference's as sets (box numbering differs: level-major, Morton order
// within a level).
//
// Tree, without recursion:
//  1. root cube from a min/max reduction, same FP64 arithmetic as :71-81;
//  2. per body the 24-level octant path, replaying the reference's FP64
//     comparisons against the recursively shifted centres (:109-127), packed
//     as a 72-bit key; stable radix sort by key;
//  3. a box at level l with count > thr splits (with the eps floor and depth
//     cap of :102-103).  Count > thr at level l for the box holding sorted
//     position i  <=>  some window [j, j+thr] containing i has common key
//     prefix >= l.  A sliding-window max of cpl(j, j+thr) gives every body's
//     leaf level in O(n) with no level-by-level recursion;
//  4. box records (level, first position) are emitted per position and
//     stably sorted by level -> level-major box ids; parents by binary search;
//  5. bodies are stably re-sorted by leaf id from the original order, which
//     reproduces the reference's within-leaf order (original index order).
// Lists:
//  - colleagues: level-synchronous from the parent's colleagues' children,
//    stored in 27 offset slots (:143-151);
//  - V is implicit: children of the parent's colleagues at integer offset
//    max|o| >= 2 (:154-161); the FP64 adjacency predicate is re-evaluated on
//    every candidate and disagreements are counted (expected 0);
//  - U/W per leaf (:164-169,176-189): same-level and coarser adjacent leaves
//    come from the colleague slots of the leaf and its ancestors, finer ones
//    from a bounded explicit-stack descent of non-leaf colleagues;
//  - X = transpose of W via a stable sort (:171-173).
#include "ogx_tree_common.cuh"

namespace ogx {
namespace {

constexpr unsigned FULL = 0xffffffffu;

// ---- 1. root cube -----------------------------------------------------------
__global__ void k_bbox_partial(const double* pos, int64_t n, double* part) {
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double v = pos[3 * i + a];
            lo[a] = fmin(lo[a], v);
            hi[a] = fmax(hi[a], v);
        }
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = fmin(lo[a], __shfl_xor_sync(FULL, lo[a], o));
            hi[a] = fmax(hi[a], __shfl_xor_sync(FULL, hi[a], o));
        }
    __shared__ double sh[32][6];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
        for (int a = 0; a < 3; ++a) { sh[w][a] = lo[a]; sh[w][3 + a] = hi[a]; }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int ww = 1; ww < (int)(blockDim.x >> 5); ++ww)
            for (int a = 0; a < 3; ++a) { sh[0][a] = fmin(sh[0][a], sh[ww][a]); sh[0][3 + a] = fmax(sh[0][3 + a], sh[ww][3 + a]); }
        for (int a = 0; a < 6; ++a) part[6 * blockIdx.x + a] = sh[0][a];
    }
}

// AdaptiveOctree::build :71-81; eps-floor level from subdivide :102
__global__ void __launch_bounds__(256) k_bbox_final(const double* part, int nparts, double eps_floor, RootInfo* root) {
    __shared__ double sh[8][6];
    double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
    for (int b = threadIdx.x; b < nparts; b += blockDim.x)
        for (int a = 0; a < 3; ++a) { lo[a] = fmin(lo[a], part[6 * b + a]); hi[a] = fmax(hi[a], part[6 * b + 3 + a]); }
#pragma unroll
    for (int a = 0; a < 3; ++a)
        for (int o = 16; o > 0; o >>= 1) {
            lo[a] = fmin(lo[a], __shfl_xor_sync(FULL, lo[a], o));
            hi[a] = fmax(hi[a], __shfl_xor_sync(FULL, hi[a], o));
        }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
        for (int a = 0; a < 3; ++a) { sh[w][a] = lo[a]; sh[w][3 + a] = hi[a]; }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int ww = 1; ww < (int)(blockDim.x >> 5); ++ww)
        for (int a = 0; a < 3; ++a) { lo[a] = fmin(lo[a], sh[ww][a]); hi[a] = fmax(hi[a], sh[ww][3 + a]); }
    for (int a = 0; a < 3; ++a) { lo[a] = fmin(lo[a], sh[0][a]); hi[a] = fmax(hi[a], sh[0][3 + a]); }
    RootInfo r;
    for (int a = 0; a < 3; ++a) r.c[a] = __dmul_rn(0.5, __dadd_rn(lo[a], hi[a]));
    double ext = __dsub_rn(hi[0], lo[0]);
    const double e1 = __dsub_rn(hi[1], lo[1]), e2 = __dsub_rn(hi[2], lo[2]);
    if (ext < e1) ext = e1;
    if (ext < e2) ext = e2;
    double half = __dmul_rn(0.5, ext);
    if (!(half > 0)) half = 1.0;
    half = __dmul_rn(half, 1.0 + 1e-9);
    r.half = half;
    r.tol = __dmul_rn(1e-9, half);
    int leps = kMaxDepth + 1;
    double h = half;
    for (int l = 0; l <= kMaxDepth; ++l) {
        if (__dmul_rn(2.0, h) <= eps_floor) { leps = l; break; }
        h = __dmul_rn(0.5, h);
    }
    r.leps = leps;
    r.pad = 0;
    *root = r;
}

// ---- 2. octant keys -----------------------------------------------------------
__global__ void k_keys(const double* pos, int64_t n, const RootInfo* root, uint64_t* khi, uint32_t* klo, uint32_t* idx) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = pos[3 * i], y = pos[3 * i + 1], z = pos[3 * i + 2];
    double cx = root->c[0], cy = root->c[1], cz = root->c[2], h = root->half;
    uint64_t hi = 0;
    uint32_t lo = 0;
#pragma unroll 1
    for (int l = 1; l <= kMaxDepth; ++l) {
        const int bx = x >= cx, by = y >= cy, bz = z >= cz;
        const uint32_t o = (uint32_t)(bx | (by << 1) | (bz << 2));
        const double h2 = __dmul_rn(0.5, h);
        cx = __dadd_rn(cx, bx ? h2 : -h2);
        cy = __dadd_rn(cy, by ? h2 : -h2);
        cz = __dadd_rn(cz, bz ? h2 : -h2);
        h = h2;
        if (l <= kHiLevels) hi = (hi << 3) | o;
        else lo = (lo << 3) | o;
    }
    khi[i] = hi;
    klo[i] = lo;
    idx[i] = (uint32_t)i;
}

__device__ __forceinline__ int cpl72(uint64_t ha, uint32_t la, uint64_t hb, uint32_t lb) {
    const uint64_t x = ha ^ hb;
    if (x) return (__clzll((long long)x) - 1) / 3;
    const uint32_t y = la ^ lb;
    if (y) return kHiLevels + (__clz((int)y) - 23) / 3;
    return kMaxDepth;
}
__device__ __forceinline__ int key_digit(uint64_t hi, uint32_t lo, int level) {
    return level <= kHiLevels ? (int)((hi >> (3 * (kHiLevels - level))) & 7ull) : (int)((lo >> (3 * (kMaxDepth - level))) & 7u);
}

// ---- 3. topology per sorted position ------------------------------------------
__global__ void k_topo_pairs(const uint64_t* khi, const uint32_t* klo, int64_t n, int thr, int* dfirst, signed char* cplthr) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t hi = khi[i];
    const uint32_t lo = klo[i];
    dfirst[i] = (i == 0) ? 0 : cpl72(khi[i - 1], klo[i - 1], hi, lo) + 1;
    cplthr[i] = (i + thr < n) ? (signed char)cpl72(hi, lo, khi[i + thr], klo[i + thr]) : (signed char)-1;
}

constexpr int WM_BLOCK = 1024;
// leaf level L(i) = min(W(i)+1, leps, maxDepth), W = window max of cplthr over [i-thr, i].
// Also box-start count c_i, leaf-start flag, level histogram (difference form).
__global__ void __launch_bounds__(WM_BLOCK) k_topo_levels(const signed char* cplthr, const int* dfirst, int64_t n, int thr,
                                                          const RootInfo* root, int* leaflev, int* cnt, int* leafflag,
                                                          DevCounts* counts) {
    extern __shared__ signed char s_cpl[];
    __shared__ int s_hist[kMaxDepth + 2];
    const int64_t b0 = (int64_t)blockIdx.x * WM_BLOCK;
    const int win = thr + 1;
    const int span = WM_BLOCK + win - 1;
    for (int k = threadIdx.x; k < span; k += WM_BLOCK) {
        const int64_t j = b0 - (win - 1) + k;
        s_cpl[k] = (j >= 0 && j < n) ? cplthr[j] : (signed char)-1;
    }
    if (threadIdx.x < kMaxDepth + 2) s_hist[threadIdx.x] = 0;
    __syncthreads();
    const int64_t i = b0 + threadIdx.x;
    if (i < n) {
        int w = -1;
        for (int k = 0; k < win; ++k) w = max(w, (int)s_cpl[threadIdx.x + k]);
        int L = w + 1;
        L = min(L, root->leps);
        L = min(L, kMaxDepth);
        const int d = dfirst[i];
        const int from = (i == 0) ? 0 : d;
        const int c = max(0, L - from + 1);
        leaflev[i] = L;
        cnt[i] = c;
        leafflag[i] = (i == 0 || d <= L) ? 1 : 0;
        if (c > 0) {
            atomicAdd(&s_hist[from], 1);
            atomicAdd(&s_hist[L + 1], -1);
        }
    }
    __syncthreads();
    if (threadIdx.x < kMaxDepth + 2 && s_hist[threadIdx.x] != 0) atomicAdd(&counts->level_hist[threadIdx.x], s_hist[threadIdx.x]);
}

__global__ void k_counts_finalize(DevCounts* counts, const int64_t* recoff, const int64_t* leafscan, int64_t n, int* level_off_dev) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    counts->num_boxes = recoff[n];
    counts->num_leaves = leafscan[n];
    counts->nb32 = (int32_t)recoff[n];
    counts->nleaf32 = (int32_t)leafscan[n];
    int run = 0, maxl = 0;
    int cum = 0;
    level_off_dev[0] = 0;
    for (int l = 0; l <= kMaxDepth; ++l) {
        run += counts->level_hist[l];   // boxes at level l
        counts->level_hist[l] = run;
        if (run > 0) maxl = l;
        cum += run;
        level_off_dev[l + 1] = cum;
    }
    counts->level_hist[kMaxDepth + 1] = 0;
    counts->max_level = maxl;
}

__global__ void k_emit_records(const int* cnt, const int* dfirst, const int* leaflev, const int64_t* recoff, int64_t n,
                               uint32_t* reckey, uint32_t* recpos, const int* leafflag, const int64_t* leafscan,
                               int* leafstart, const DevCounts* counts) {
    if (counts->overflow) return;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i > n) return;
    if (i == n) { leafstart[leafscan[n]] = (int)n; return; }
    const int c = cnt[i];
    if (c > 0) {
        const int from = (i == 0) ? 0 : dfirst[i];
        const int64_t o = recoff[i];
        for (int k = 0; k < c; ++k) {
            reckey[o + k] = (uint32_t)(from + k);
            recpos[o + k] = (uint32_t)i;
        }
    }
    if (leafflag[i]) leafstart[leafscan[i]] = (int)i;
}

// ---- 4. boxes -------------------------------------------------------------------
// k < nb_cap; records k >= the device box count are capacity padding: null boxes
__global__ void k_boxes(int nb_cap, const uint32_t* reclev, const uint32_t* recpos, const int* level_off, const uint64_t* khi,
                        const uint32_t* klo, const int* leaflev, const int64_t* leafscan, const int* leafstart,
                        const RootInfo* root, int* level, int* coord, double* center, int* parent, int* child, int* leafid,
                        int* pfirst, int* pcount, int* leafbox, const DevCounts* counts) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nb_cap || counts->overflow) return;
    if (k >= counts->nb32) {
        level[k] = -1;
        coord[3 * k] = coord[3 * k + 1] = coord[3 * k + 2] = 0;
        center[4 * k] = center[4 * k + 1] = center[4 * k + 2] = center[4 * k + 3] = 0.0;
        parent[k] = -1;
        leafid[k] = -1;
        pfirst[k] = 0;
        pcount[k] = 0;
        return;
    }
    const int l = (int)reclev[k];
    const int s = (int)recpos[k];
    const uint64_t hi = khi[s];
    const uint32_t lo = klo[s];
    double cx = root->c[0], cy = root->c[1], cz = root->c[2], h = root->half;
    int ix = 0, iy = 0, iz = 0;
    for (int lv = 1; lv <= l; ++lv) {
        const int o = key_digit(hi, lo, lv);
        const int bx = o & 1, by = (o >> 1) & 1, bz = (o >> 2) & 1;
        const double h2 = __dmul_rn(0.5, h);
        cx = __dadd_rn(cx, bx ? h2 : -h2);
        cy = __dadd_rn(cy, by ? h2 : -h2);
        cz = __dadd_rn(cz, bz ? h2 : -h2);
        h = h2;
        ix = 2 * ix + bx;
        iy = 2 * iy + by;
        iz = 2 * iz + bz;
    }
    level[k] = l;
    coord[3 * k] = ix; coord[3 * k + 1] = iy; coord[3 * k + 2] = iz;
    center[4 * k] = cx; center[4 * k + 1] = cy; center[4 * k + 2] = cz; center[4 * k + 3] = h;
    pfirst[k] = s;
    const bool isleaf = leaflev[s] == l;
    if (isleaf) {
        const int lf = (int)leafscan[s];
        leafid[k] = lf;
        leafbox[lf] = k;
        pcount[k] = leafstart[lf + 1] - s;
    } else {
        leafid[k] = -1;
    }
    if (l == 0) { parent[k] = -1; return; }
    // parent: last box of level l-1 whose first position <= s
    int lo_i = level_off[l - 1], hi_i = level_off[l] - 1;
    while (lo_i < hi_i) {
        const int mid = (lo_i + hi_i + 1) >> 1;
        if ((int)recpos[mid] <= s) lo_i = mid; else hi_i = mid - 1;
    }
    parent[k] = lo_i;
    child[8 * lo_i + key_digit(hi, lo, l)] = k;
}

__global__ void k_leaf_occupancy(int nleaf_cap, const int* leafbox, const int* pcount, DevCounts* counts) {
    if (counts->overflow) return;
    const int lf = blockIdx.x * blockDim.x + threadIdx.x;
    int c = (lf < nleaf_cap && lf < counts->nleaf32) ? pcount[leafbox[lf]] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c = max(c, __shfl_xor_sync(FULL, c, o));
    if ((threadIdx.x & 31) == 0 && c > 0) atomicMax(&counts->max_leaf_occ, c);
}

// ---- 5. final body order ----------------------------------------------------------
__global__ void k_leafkey(const uint32_t* perm_key, const int64_t* leafscan, int64_t n, uint32_t* leafkey, uint32_t* ident) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    leafkey[perm_key[i]] = (uint32_t)(leafscan[i + 1] - 1);  // leaf id containing sorted position i
    ident[i] = (uint32_t)i;
}
__global__ void k_gather_bodies(const uint32_t* perm, const double* pos, const double* mass, int64_t n, int* perm_out,
                                double* px, double* py, double* pz, double* pm) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t j = perm[i];
    perm_out[i] = (int)j;
    px[i] = pos[3 * j]; py[i] = pos[3 * j + 1]; pz[i] = pos[3 * j + 2];
    pm[i] = mass[j];
}

}  // namespace

static // flag the non-leaf boxes and count them per level
__global__ void k_nonleaf_flags(int nb_cap, const int* __restrict__ leafid, const int* __restrict__ level, int* flag,
                                DevCounts* counts) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb_cap) return;
    const int f = !counts->overflow && b < counts->nb32 && leafid[b] < 0;
    flag[b] = f;
    if (f) atomicAdd(&counts->nonleaf_level[level[b]], 1);
}

__global__ void k_nonleaf_emit(int nb, const int* __restrict__ flag, const int64_t* __restrict__ off, int* out) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b < nb && flag[b]) out[off[b]] = b;
}

// nl_off[l] = first non-leaf box of level l in the compacted list (exclusive scan of
// the per-level counts; the list is level-major)
__global__ void k_nonleaf_offsets(const DevCounts* counts, int* nl_off) {
    if (threadIdx.x != 0) return;
    int c = 0;
    for (int l = 0; l <= kMaxDepth; ++l) {
        nl_off[l] = c;
        c += counts->nonleaf_level[l];
    }
    nl_off[kMaxDepth + 1] = c;
}

// After a sort by levels 1..16 only (digit passes 3..8): flags a level-16 box that
// holds more than thr bodies, i.e. bodies whose leaf may lie deeper, for which the
// order of the lower digits matters.  Keys of one box are contiguous, so such a box
// has two keys thr apart with the same 48-bit prefix (bits 15..62 of the high word).
__global__ void k_deep_check(const uint64_t* __restrict__ khi, int64_t n, int thr, DevCounts* counts) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i + thr < n && (khi[i] >> 15) == (khi[i + thr] >> 15)) counts->deep_flag = 1;
}

inline int grid_for(int64_t n, int b) { return (int)((n + b - 1) / b); }
static inline int bits_for(int64_t v) {
    int b = 1;
    while ((1ll << b) <= v) ++b;
    return b;
}

// Capacity mode: flags an evaluation whose tree does not fit the capacities it was
// launched with (or that needs the full 24-level key sort it was not launched with).
__global__ void k_check_tree(DevCounts* counts, int nb_cap, int nleaf_cap, int levels_cap, int full_sort) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (counts->num_boxes > nb_cap || counts->num_leaves > nleaf_cap || counts->max_level + 1 > levels_cap ||
        (counts->deep_flag && !full_sort))
        counts->overflow = 1;
}

// a[k] = v for start <= k < cap, start read on the device (padding behind a device count)
__global__ void k_fill_tail_u32(uint32_t* a, const int32_t* start, int64_t cap, uint32_t v) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < cap && k >= *start) a[k] = v;
}

int tree_build(Handle& h, const double* d_pos, const double* d_mass, int64_t n) {
    const cudaStream_t st = h.stream;
    const int thr = h.prm.leaf_capacity;
    DevCounts* dc;
    RootInfo* root;
    double* part;
    OGX_TRY(arena_get(h.ws, S_COUNTS, 1, &dc));
    h.d_err = &dc->kernel_error;
    OGX_TRY(arena_get(h.ws, S_ROOT, 1, &root));
    const int nparts = 296;
    OGX_TRY(arena_get(h.ws, S_BBOX, 6 * nparts, &part));
    OGX_CUDA(cudaMemsetAsync(dc, 0, sizeof(DevCounts), st));

    k_bbox_partial<<<nparts, 256, 0, st>>>(d_pos, n, part); ++h.launches;
    k_bbox_final<<<1, 256, 0, st>>>(part, nparts, h.prm.eps, root); ++h.launches;

    uint64_t* khi;
    uint32_t *klo, *kidx;
    uint64_t* khi_in;
    uint32_t *klo_in, *kidx_in;
    OGX_TRY(arena_get(h.ws, S_KHI, n, &khi_in));
    OGX_TRY(arena_get(h.ws, S_KLO, n, &klo_in));
    OGX_TRY(arena_get(h.ws, S_IDX, n, &kidx_in));

    int *dfirst, *leaflev, *cnt, *leafflag, *leafstart, *level_off_dev;
    signed char* cplthr;
    int64_t *recoff, *leafscan;
    OGX_TRY(arena_get(h.ws, S_TOPO_D, n, &dfirst));
    OGX_TRY(arena_get(h.ws, S_TOPO_CPL, n, &cplthr));
    OGX_TRY(arena_get(h.ws, S_TOPO_L, n, &leaflev));
    OGX_TRY(arena_get(h.ws, S_TOPO_CNT, 2 * n + 64, &cnt));
    leafflag = cnt + n + 32;
    OGX_TRY(arena_get(h.ws, S_TOPO_COFF, 2 * (n + 1), &recoff));
    leafscan = recoff + (n + 1);
    OGX_TRY(arena_get(h.ws, S_LEAFSTART, n + 2 + kMaxDepth + 2, &leafstart));
    level_off_dev = leafstart + n + 2;
    const size_t wm_smem = WM_BLOCK + thr + 16;
    if (wm_smem > 48 * 1024) {
        OGX_CUDA(smem_optin((const void*)k_topo_levels, (int)wm_smem));
    }

    // Leaves need the key order only down to their own level.  First attempt: sort
    // by levels 1..16 (6 of the 9 digit passes); if some level-16 box holds more than
    // thr bodies (deep clusters) the counts read at sync point 1 say so and the build
    // is repeated with the full 72-bit sort.  In capacity mode there is no read-back:
    // the sort depth is the one the capacities were taken with, and a tree that needs
    // more sets the overflow flag.
    int nb = 0, nleaf = 0;
    for (int attempt = 0;; ++attempt) {
        const bool full = (attempt > 0) || (h.cap_mode && h.cap.full_sort);
        const int first_pass = full ? 0 : 3;
        if (attempt > 0) OGX_CUDA(cudaMemsetAsync(dc, 0, sizeof(DevCounts), st));
        k_keys<<<grid_for(n, 256), 256, 0, st>>>(d_pos, n, root, khi_in, klo_in, kidx_in); ++h.launches;
        OGX_TRY(radix_sort_key72(h, n, first_pass, &khi, &klo, &kidx));
        if (first_pass > 0 && n > thr) { k_deep_check<<<grid_for(n, 256), 256, 0, st>>>(khi, n, thr, dc); ++h.launches; }
        k_topo_pairs<<<grid_for(n, 256), 256, 0, st>>>(khi, klo, n, thr, dfirst, cplthr); ++h.launches;
        k_topo_levels<<<grid_for(n, WM_BLOCK), WM_BLOCK, wm_smem, st>>>(cplthr, dfirst, n, thr, root, leaflev, cnt, leafflag, dc); ++h.launches;
        OGX_TRY(scan_i32_to_i64(h, cnt, recoff, n));
        OGX_TRY(scan_i32_to_i64(h, leafflag, leafscan, n));
        k_counts_finalize<<<1, 32, 0, st>>>(dc, recoff, leafscan, n, level_off_dev); ++h.launches;
        if (h.cap_mode) {
            nb = h.cap.nb;
            nleaf = h.cap.nleaf;
            k_check_tree<<<1, 32, 0, st>>>(dc, nb, nleaf, h.cap.levels, full ? 1 : 0); ++h.launches;
            h.max_level = h.cap.levels - 1;
            h.full_sort_used = full;
            break;
        }
        // sync point 1: box / leaf / level counts
        OGX_CUDA(cudaMemcpyAsync(h.h_counts, dc, sizeof(DevCounts), cudaMemcpyDeviceToHost, st));
        OGX_CUDA(cudaStreamSynchronize(st));
        if (!h.h_counts->deep_flag || first_pass == 0) {
            h.full_sort_used = full;
            break;
        }
    }
    if (!h.cap_mode) {
        nb = (int)h.h_counts->num_boxes;
        nleaf = (int)h.h_counts->num_leaves;
        h.max_level = h.h_counts->max_level;
        h.level_off.assign(h.max_level + 2, 0);
        for (int l = 0; l <= h.max_level; ++l) h.level_off[l + 1] = h.level_off[l] + h.h_counts->level_hist[l];
    }
    h.d_counts = dc;
    h.d_level_off = level_off_dev;

    // box records (level, first sorted body): capacity padding behind the device count
    // gets level 31 and so sorts after every real record
    uint32_t *reckey, *recpos;
    OGX_TRY(arena_get(h.ws, S_REC_KEY, nb, &reckey));
    OGX_TRY(arena_get(h.ws, S_REC_POS, nb, &recpos));
    k_emit_records<<<grid_for(n + 1, 256), 256, 0, st>>>(cnt, dfirst, leaflev, recoff, n, reckey, recpos, leafflag, leafscan,
                                                          leafstart, dc); ++h.launches;
    if (h.cap_mode) { k_fill_tail_u32<<<grid_for(nb, 256), 256, 0, st>>>(reckey, &dc->nb32, nb, 31u); ++h.launches; }
    uint32_t *reclev, *recpos_s;
    OGX_TRY(radix_sort_u32(h, S_REC_KEY, S_REC_POS, S_REC_KEY2, S_REC_POS2, nb, 5, &reclev, &recpos_s));

    int *level, *coord, *parent, *child, *leafid, *pfirst, *pcount, *leafbox;
    double* center;
    OGX_TRY(arena_get(h.ws, S_BOX_LEVEL, nb, &level));
    OGX_TRY(arena_get(h.ws, S_BOX_COORD, 3 * (size_t)nb, &coord));
    OGX_TRY(arena_get(h.ws, S_BOX_CENTER, 4 * (size_t)nb, &center));
    OGX_TRY(arena_get(h.ws, S_BOX_PARENT, nb, &parent));
    OGX_TRY(arena_get(h.ws, S_BOX_CHILD, 8 * (size_t)nb, &child));
    OGX_TRY(arena_get(h.ws, S_BOX_LEAFID, nb, &leafid));
    OGX_TRY(arena_get(h.ws, S_BOX_PFIRST, nb, &pfirst));
    OGX_TRY(arena_get(h.ws, S_BOX_PCOUNT, nb, &pcount));
    OGX_TRY(arena_get(h.ws, S_LEAF_BOX, nleaf, &leafbox));
    OGX_CUDA(cudaMemsetAsync(child, 0xFF, 8 * sizeof(int) * (size_t)nb, st));
    OGX_CUDA(cudaMemsetAsync(pcount, 0, sizeof(int) * (size_t)nb, st));
    k_boxes<<<grid_for(nb, 128), 128, 0, st>>>(nb, reclev, recpos_s, level_off_dev, khi, klo, leaflev, leafscan, leafstart, root,
                                                level, coord, center, parent, child, leafid, pfirst, pcount, leafbox, dc); ++h.launches;
    k_leaf_occupancy<<<grid_for(nleaf, 128), 128, 0, st>>>(nleaf, leafbox, pcount, dc); ++h.launches;

    // non-leaf boxes in box order (level-major, so each level's parents are contiguous)
    int *nl_flag, *nonleaf;
    int64_t* nl_off;
    OGX_TRY(arena_get(h.ws, S_NONLEAF_FLAG, nb, &nl_flag));
    OGX_TRY(arena_get(h.ws, S_NONLEAF_OFF, nb + 1, &nl_off));
    OGX_TRY(arena_get(h.ws, S_NONLEAF, nb, &nonleaf));
    k_nonleaf_flags<<<grid_for(nb, 256), 256, 0, st>>>(nb, leafid, level, nl_flag, dc); ++h.launches;
    OGX_TRY(scan_i32_to_i64(h, nl_flag, nl_off, nb));
    k_nonleaf_emit<<<grid_for(nb, 256), 256, 0, st>>>(nb, nl_flag, nl_off, nonleaf); ++h.launches;
    int* nl_loff;
    OGX_TRY(arena_get(h.ws, S_NONLEAF_LOFF, kMaxDepth + 2, &nl_loff));
    k_nonleaf_offsets<<<1, 32, 0, st>>>(dc, nl_loff); ++h.launches;
    h.d_nonleaf = nonleaf;
    h.d_nonleaf_off = nl_loff;

    // final body order: stable by leaf id from the original order
    uint32_t *lk, *ident;
    OGX_TRY(arena_get(h.ws, S_LEAFKEY, n, &lk));
    OGX_TRY(arena_get(h.ws, S_PERM, n, &ident));
    k_leafkey<<<grid_for(n, 256), 256, 0, st>>>(kidx, leafscan, n, lk, ident); ++h.launches;
    uint32_t *lk_s, *perm_s;
    OGX_TRY(radix_sort_u32(h, S_LEAFKEY, S_PERM, S_LEAFKEY2, S_PERM2, n, bits_for(nleaf), &lk_s, &perm_s));
    int* perm;
    double *px, *py, *pz, *pm;
    OGX_TRY(arena_get(h.ws, S_PERM_FINAL, n, &perm));
    OGX_TRY(arena_get(h.ws, S_PX, n, &px));
    OGX_TRY(arena_get(h.ws, S_PY, n, &py));
    OGX_TRY(arena_get(h.ws, S_PZ, n, &pz));
    OGX_TRY(arena_get(h.ws, S_PM, n, &pm));
    if (h.mass_pending) {   // the masses' host copy (ogx_eval) ran beside the steps above
        OGX_CUDA(cudaStreamWaitEvent(st, h.ev_mass, 0));
        h.mass_pending = false;
    }
    k_gather_bodies<<<grid_for(n, 256), 256, 0, st>>>(perm_s, d_pos, d_mass, n, perm, px, py, pz, pm); ++h.launches;
    OGX_CUDA(cudaGetLastError());

    TreeView& tv = h.tv;
    tv.n = (int)n; tv.nb = nb; tv.nleaf = nleaf; tv.root = root; tv.cnt = dc;
    tv.px = px; tv.py = py; tv.pz = pz; tv.pm = pm; tv.perm = perm;
    tv.level = level; tv.coord = coord; tv.center = center; tv.parent = parent; tv.child = child;
    tv.leafid = leafid; tv.pfirst = pfirst; tv.pcount = pcount; tv.leafbox = leafbox;
    return OGX_OK;
}

}  // namespace ogx
