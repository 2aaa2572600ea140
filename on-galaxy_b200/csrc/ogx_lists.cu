// ogx_lists.cu -- Carrier-Greengard-Rokhlin interaction lists on the GPU.
//
// Replaces AdaptiveOctree::buildLists (src3d/AdaptiveOctree.hpp:137-189):
//  - colleagues: same-level adjacent boxes, the children of the parent's
//    colleagues that pass `adjacent` (:143-151).  Box centres are exact binary
//    fractions of the root box, so for same-level boxes that test holds exactly
//    for integer offsets in [-1,1]^3: every (box, slot) finds its colleague in
//    one launch by a binary search of the level's boxes (Morton order) for the
//    offset coordinates.  A second launch replays the reference's recursion over
//    the children of each parent's colleagues with the FP64 predicate and counts
//    every disagreement with the search (expected 0);
//  - V is implicit: children of the parent's colleagues at integer offset
//    max|o| >= 2 (:154-161); every candidate is also classified with the
//    reference's FP64 predicate and disagreements are counted (expected 0);
//  - U/W per leaf (:164-169 with collectAdjLeaves :176-180 and descendW
//    :181-189): warp per leaf, lane d owns colleague slot d: the slot's leaf
//    (same level), the slot of every ancestor (coarser adjacent leaves) and a
//    bounded explicit-stack descent of the slot's non-leaf colleague (finer U
//    members and the W boxes).  A count pass sizes the CSR, a fill pass writes
//    each lane's items at its warp-scan offset, so the order is deterministic;
//  - X = transpose of W through a stable sort by W member (:171-173).
#include <algorithm>

#include "ogx_tree_common.cuh"
#include "ogx_softening.cuh"

namespace ogx {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int UW_STACK = 192;

// p's highest set bit is below q's
__device__ __forceinline__ bool msb_less(unsigned p, unsigned q) { return p < q && p < (p ^ q); }

// Morton order of two boxes of one level from their integer coordinates: the
// dimension whose coordinates first differ at the highest bit decides; at equal
// bits z ranks above y above x (octant digit = x | y << 1 | z << 2)
__device__ __forceinline__ bool morton_less(int ax, int ay, int az, int bx, int by, int bz) {
    const unsigned x = (unsigned)(ax ^ bx), y = (unsigned)(ay ^ by), z = (unsigned)(az ^ bz);
    int d = 2;
    unsigned m = z;
    if (msb_less(m, y)) { d = 1; m = y; }
    if (msb_less(m, x)) d = 0;
    return d == 0 ? ax < bx : (d == 1 ? ay < by : az < bz);
}

// colleague slot d of box b: the box of b's level at integer offset (d % 3 - 1, ...);
// level_off[l] = first box of level l (device)
__global__ void k_colleagues_bs(int nb_cap, const int* __restrict__ level_off, const int* __restrict__ level,
                                const int* __restrict__ coord, int* __restrict__ col, const DevCounts* counts) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= 27 * (int64_t)nb_cap || counts->overflow) return;
    const int b = (int)(t / 27), d = (int)(t - 27 * (int64_t)b);
    if (b >= counts->nb32) { col[t] = -1; return; }
    if (d == 13) { col[t] = b; return; }
    const int l = level[b];
    const int side = 1 << l;
    const int nx = coord[3 * b] + d % 3 - 1, ny = coord[3 * b + 1] + (d / 3) % 3 - 1, nz = coord[3 * b + 2] + d / 9 - 1;
    int found = -1;
    if (l > 0 && nx >= 0 && ny >= 0 && nz >= 0 && nx < side && ny < side && nz < side) {
        int lo = level_off[l], hi = level_off[l + 1] - 1;
        while (lo <= hi) {
            const int mid = (lo + hi) >> 1;
            const int mx = coord[3 * mid], my = coord[3 * mid + 1], mz = coord[3 * mid + 2];
            if (mx == nx && my == ny && mz == nz) { found = mid; break; }
            if (morton_less(mx, my, mz, nx, ny, nz)) lo = mid + 1;
            else hi = mid - 1;
        }
    }
    col[t] = found;
}

// the reference's recursion (children of the parent's colleagues, FP64 `adjacent`)
// checked against the searched colleagues; also counts the V-list pairs
__global__ void __launch_bounds__(128) k_colleagues_check(int first, int count, const int* __restrict__ leafid,
                                                          const int* __restrict__ child, const double* __restrict__ ctr,
                                                          const RootInfo* root, const int* __restrict__ col,
                                                          DevCounts* counts) {
    __shared__ double s_kc[4][8][4];   // centres (x, y, z, half) of each warp's parent's children
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int k = blockIdx.x * 4 + wid;
    if (k >= count || first + k >= counts->nb32 || counts->overflow) return;
    const int P = first + k;
    if (leafid[P] >= 0) return;
    int kids[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) kids[t] = child[8 * P + t];
    if (lane < 32) {
        const int t = lane >> 2, q = lane & 3;
        s_kc[wid][t][q] = (kids[t] >= 0) ? ctr[4 * kids[t] + q] : 0.0;
    }
    __syncwarp();
    const double tol = root->tol;
    int mism = 0, nv = 0;
    if (lane < 27) {
        const int D = lane;
        const int Q = col[27 * P + D];
        if (Q >= 0) {
            const int Dx = D % 3 - 1, Dy = (D / 3) % 3 - 1, Dz = D / 9 - 1;
            for (int s = 0; s < 8; ++s) {
                const int c = child[8 * Q + s];
                if (c < 0) continue;
                const double cx = ctr[4 * c], cy = ctr[4 * c + 1], cz = ctr[4 * c + 2], ch = ctr[4 * c + 3];
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    const int b = kids[t];
                    if (b < 0) continue;
                    const int ox = 2 * Dx + (s & 1) - (t & 1), oy = 2 * Dy + ((s >> 1) & 1) - ((t >> 1) & 1),
                              oz = 2 * Dz + ((s >> 2) & 1) - ((t >> 2) & 1);
                    const bool adj_i = max(abs(ox), max(abs(oy), abs(oz))) <= 1;
                    // adjacent64(ctr, b, c, tol) with both centres already in hand
                    const double* kb = s_kc[wid][t];
                    const double lim = __dadd_rn(__dadd_rn(kb[3], ch), tol);
                    const bool adj_f = fabs(__dsub_rn(kb[0], cx)) <= lim && fabs(__dsub_rn(kb[1], cy)) <= lim &&
                                       fabs(__dsub_rn(kb[2], cz)) <= lim;
                    if (adj_i != adj_f) ++mism;
                    if (adj_i) { if (col[27 * b + colleague_slot(ox, oy, oz)] != c) ++mism; }
                    else ++nv;
                }
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mism += __shfl_xor_sync(FULL, mism, o);
        nv += __shfl_xor_sync(FULL, nv, o);
    }
    if (lane == 0) {
        if (mism) atomicAdd((unsigned long long*)&counts->adj_mismatch, (unsigned long long)mism);
        if (nv) atomicAdd((unsigned long long*)&counts->v_total, (unsigned long long)nv);
    }
}

__device__ __forceinline__ int warp_excl_scan(int v, int lane) {
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(FULL, x, o);
        if (lane >= o) x += y;
    }
    return x - v;
}

template <bool FILL>
__global__ void __launch_bounds__(128) k_uw_warp(int nleaf, const int* __restrict__ leafbox, const int* __restrict__ parent,
                                                 const int* __restrict__ child, const int* __restrict__ leafid,
                                                 const int* __restrict__ col, const double* __restrict__ ctr,
                                                 const int* __restrict__ pcount, const RootInfo* root, int* lane_u, int* lane_w,
                                                 int* ucnt, int* wcnt, const int64_t* uoff, const int64_t* woff, int* uidx,
                                                 int* widx, DevCounts* counts) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int lf = blockIdx.x * 4 + wid;
    if (lf >= nleaf || lf >= counts->nleaf32 || counts->overflow) return;
    const int b = leafbox[lf];
    const double tol = root->tol;
    // adjacent64(ctr, a, b, tol) with b's centre held in registers
    const double bx = ctr[4 * b], by = ctr[4 * b + 1], bz = ctr[4 * b + 2], bh = ctr[4 * b + 3];
    auto adj_b = [&](int a) {
        const double lim = __dadd_rn(__dadd_rn(ctr[4 * a + 3], bh), tol);
        return fabs(__dsub_rn(ctr[4 * a], bx)) <= lim && fabs(__dsub_rn(ctr[4 * a + 1], by)) <= lim &&
               fabs(__dsub_rn(ctr[4 * a + 2], bz)) <= lim;
    };
    int nu = 0, nw = 0;
    int64_t upairs = 0, ub = 0, wb = 0;
    bool overflow = false;
    if (FILL) {
        ub = uoff[lf] + warp_excl_scan(lane_u[32 * lf + lane], lane);
        wb = woff[lf] + warp_excl_scan(lane_w[32 * lf + lane], lane);
    }
    auto addU = [&](int c) {
        if (FILL) uidx[ub + nu] = c;
        else upairs += pcount[c];
        ++nu;
    };
    if (lane < 27) {
        const int d = lane;
        const int c = col[27 * b + d];
        if (c >= 0 && leafid[c] >= 0) addU(c);  // same-level adjacent leaves (b itself in slot 13)
        for (int A = parent[b]; A >= 0; A = parent[A]) {  // coarser adjacent leaves
            const int a2 = col[27 * A + d];
            if (a2 >= 0 && leafid[a2] >= 0 && adj_b(a2)) addU(a2);
        }
        if (c >= 0 && c != b && leafid[c] < 0) {  // finer: descend the non-leaf colleague
            int stk[UW_STACK];
            int sp = 0;
            stk[sp++] = c;
            while (sp > 0) {
                const int node = stk[--sp];
                for (int s = 0; s < 8; ++s) {
                    const int ch = child[8 * node + s];
                    if (ch < 0) continue;
                    if (!adj_b(ch)) {
                        if (FILL) widx[wb + nw] = ch;
                        ++nw;
                    } else if (leafid[ch] >= 0) {
                        addU(ch);
                    } else if (sp < UW_STACK) {
                        stk[sp++] = ch;
                    } else {
                        overflow = true;
                    }
                }
            }
        }
    }
    if (!FILL) {
        lane_u[32 * lf + lane] = nu;
        lane_w[32 * lf + lane] = nw;
        int tu = nu, tw = nw;
        int64_t tp = upairs;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            tu += __shfl_xor_sync(FULL, tu, o);
            tw += __shfl_xor_sync(FULL, tw, o);
            tp += __shfl_xor_sync(FULL, tp, o);
        }
        const bool any_over = __any_sync(FULL, overflow);
        if (lane == 0) {
            ucnt[lf] = tu;
            wcnt[lf] = tw;
            const int64_t pb = pcount[b];
            atomicAdd((unsigned long long*)&counts->p2p_pairs, (unsigned long long)(pb * tp - pb));
            atomicAdd((unsigned long long*)&counts->m2p_evals, (unsigned long long)(pb * tw));
            atomicAdd((unsigned long long*)&counts->p2l_evals, (unsigned long long)(pb * tw));
            if (any_over) atomicAdd((unsigned long long*)&counts->adj_mismatch, 1ull << 40);
        }
    }
}

// X = transpose of W: emit (w, leaf box) in leaf order, count members per box
__global__ void k_x_emit(int nleaf, const int* leafbox, const int64_t* woff, const int* widx, uint32_t* xkey, uint32_t* xval,
                         int* xcnt, const DevCounts* counts) {
    const int lf = blockIdx.x * blockDim.x + threadIdx.x;
    if (lf >= nleaf || lf >= counts->nleaf32 || counts->overflow) return;
    const int b = leafbox[lf];
    for (int64_t e = woff[lf]; e < woff[lf + 1]; ++e) {
        xkey[e] = (uint32_t)widx[e];
        xval[e] = (uint32_t)b;
        atomicAdd(&xcnt[widx[e]], 1);
    }
}

// M2L targets: boxes of level >= 2 keyed by their child octant
// Sort key of an M2L target: its octant t inside the parent (bits 27-29; a tensor-core
// tile holds targets of one octant) and, below it, which of the parent's 27 colleague
// slots D give the target any V-list source (bit 26 - D).  Targets with the same slot
// pattern then share tiles, so a tile runs fewer (colleague, child) combinations and
// fewer of its operand rows are empty (on the 1M merger: 17% fewer combinations).  The
// order of a tile's targets does not change any target's result.
// Launched over the capacity of boxes: the targets are boxes level_off[2] .. nb - 1
// (device counts); slots behind them get key 1 << 30 and sort after every target.
__global__ void k_tgt_keys(int cap, const int* __restrict__ level_off, const int* __restrict__ coord,
                           const int* __restrict__ parent, const int* __restrict__ col, const int* __restrict__ child,
                           uint32_t* key, uint32_t* val, DevCounts* counts) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= cap || counts->overflow) return;
    const int first = level_off[2], ntgt = counts->nb32 - first;
    if (k == 0) counts->ntgt32 = ntgt;
    if (k >= ntgt) {
        key[k] = 1u << 30;
        val[k] = 0xFFFFFFFFu;
        return;
    }
    const int b = first + k;
    const int tx = coord[3 * b] & 1, ty = coord[3 * b + 1] & 1, tz = coord[3 * b + 2] & 1;
    const int par = parent[b];
    uint32_t mask = 0;
    for (int D = 0; D < 27; ++D) {
        const int Q = col[27 * par + D];
        if (Q < 0) continue;
        const int Dx = D % 3 - 1, Dy = (D / 3) % 3 - 1, Dz = D / 9 - 1;
        for (int s = 0; s < 8; ++s) {
            const int ox = 2 * Dx + (s & 1) - tx, oy = 2 * Dy + ((s >> 1) & 1) - ty, oz = 2 * Dz + ((s >> 2) & 1) - tz;
            if (max(abs(ox), max(abs(oy), abs(oz))) > 1 && child[8 * Q + s] >= 0) {
                mask |= 1u << (26 - D);
                break;
            }
        }
    }
    key[k] = ((uint32_t)(tx | (ty << 1) | (tz << 2)) << 27) | mask;
    val[k] = (uint32_t)b;
}

// padded per-octant layout of the M2L targets (sorted by k_tgt_keys' key, octant in
// bits 27-29): every octant group starts on a multiple of `tile`, so a tile never
// mixes octants.  gs[0..8] = group starts,
// gs[9..17] = padded group starts.
__global__ void k_target_groups(const uint32_t* key, const DevCounts* counts, int tile, int fill, int* gs) {
    __shared__ int lo_s[9];
    const int g = threadIdx.x;
    const int ntgt = counts->overflow ? 0 : counts->ntgt32;
    if (g <= 8) {
        int lo = 0, hi = ntgt;  // first index with key >= g
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if ((int)(key[mid] >> 27) < g) lo = mid + 1; else hi = mid;
        }
        lo_s[g] = lo;
        gs[g] = lo;
    }
    __syncthreads();
    if (g == 0) {
        int pad = 0;
        for (int q = 0; q <= 8; ++q) {
            gs[9 + q] = pad;
            if (q < 8) pad += ((lo_s[q + 1] - lo_s[q] + fill - 1) / fill) * tile;
        }
    }
}
// slot q of a padded group holds target (q - start) / tile * fill + (q - start) % tile
// when that slot index is below `fill` (the batch width) and the target exists
__global__ void k_target_pad(const uint32_t* box, const int* gs, int npad, int tile, int fill, uint32_t* pkey,
                             uint32_t* pbox) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= npad) return;
    uint32_t k = 0xFFFFFFFFu, b = 0xFFFFFFFFu;
    for (int g = 0; g < 8; ++g) {
        const int ps = gs[9 + g], pe = gs[9 + g + 1];
        if (q >= ps && q < pe) {
            const int slot = (q - ps) % tile;
            const int local = (q - ps) / tile * fill + slot;
            if (slot < fill && local < gs[g + 1] - gs[g]) { k = (uint32_t)g; b = box[gs[g] + local]; }
            break;
        }
    }
    pkey[q] = k;
    pbox[q] = b;
}


// list totals (the last entry of each exclusive scan over the leaf capacity, whose
// padding counts are zero), checked against the capacities of the index arrays
__global__ void k_check_lists(DevCounts* counts, const int64_t* utot, const int64_t* wtot, int64_t cap_u, int64_t cap_w) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    counts->u_total = *utot;
    counts->w_total = *wtot;
    if (*utot > cap_u || *wtot > cap_w) counts->overflow = 1;
}

// X-list keys behind the W total (device) get `v` and sort last
__global__ void k_fill_tail_x(uint32_t* a, const DevCounts* counts, int64_t cap, uint32_t v) {
    const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (k < cap && k >= counts->w_total) a[k] = v;
}

inline int grid_for(int64_t n, int b) { return (int)((n + b - 1) / b); }
inline int bits_for(int64_t v) {
    int b = 1;
    while ((1ll << b) <= v) ++b;
    return b;
}

// OGX_SOFT_SPLINE: for each leaf b, the leaves c that are not adjacent to b (the far
// field takes their pairs) and whose box lies within the spline's support `hs` of b's
// box, found by a depth-first walk from the root that skips every box farther than hs.
// Adjacency is the U-list predicate (AdaptiveOctree::adjacent, same FP64 operations), so
// every leaf pair is either in b's U list or a candidate here.  Thread per leaf; pass 1
// counts, pass 2 writes in the same order.
constexpr int kSoftStack = 8 * (kMaxDepth + 2);   // > 7 per level + 8: the walk never overflows it
template <bool EMIT>
__global__ void __launch_bounds__(128) k_soft_lists(int nleaf, const int* __restrict__ leafbox, const int* __restrict__ child,
                                                    const int* __restrict__ leafid, const double* __restrict__ ctr,
                                                    const RootInfo* __restrict__ root, double hs, int* cnt,
                                                    const int64_t* __restrict__ off, int* idx, const DevCounts* counts) {
    const int lf = blockIdx.x * blockDim.x + threadIdx.x;
    if (lf >= nleaf) return;
    if (lf >= counts->nleaf32 || counts->overflow) {
        if (!EMIT) cnt[lf] = 0;
        return;
    }
    const int b = leafbox[lf];
    const double tol = root->tol;
    const double bx = ctr[4 * b], by = ctr[4 * b + 1], bz = ctr[4 * b + 2], bh = ctr[4 * b + 3];
    const double hs2 = hs * hs;
    int stack[kSoftStack];
    int sp = 0, n = 0;
    const int64_t o = EMIT ? off[lf] : 0;
    stack[sp++] = 0;   // the root
    while (sp > 0) {
        const int c = stack[--sp];
        const double ch = ctr[4 * c + 3];
        // gap between the two boxes along each axis (0 where they overlap)
        const double gx = fmax(0.0, fabs(ctr[4 * c] - bx) - (ch + bh));
        const double gy = fmax(0.0, fabs(ctr[4 * c + 1] - by) - (ch + bh));
        const double gz = fmax(0.0, fabs(ctr[4 * c + 2] - bz) - (ch + bh));
        if (gx * gx + gy * gy + gz * gz >= hs2) continue;
        if (leafid[c] >= 0) {
            const double lim = __dadd_rn(__dadd_rn(ch, bh), tol);
            const bool adj = fabs(__dsub_rn(ctr[4 * c], bx)) <= lim && fabs(__dsub_rn(ctr[4 * c + 1], by)) <= lim &&
                             fabs(__dsub_rn(ctr[4 * c + 2], bz)) <= lim;
            if (!adj) {
                if (EMIT) idx[o + n] = c;
                ++n;
            }
        } else {
            for (int s = 7; s >= 0; --s) {
                const int k = child[8 * c + s];
                if (k >= 0 && sp < kSoftStack) stack[sp++] = k;
            }
        }
    }
    if (!EMIT) cnt[lf] = n;
}

}  // namespace

// Built after the U/W/X lists of an eager evaluation (one more count read-back).
int soft_lists_build(Handle& h) {
    const cudaStream_t st = h.stream;
    TreeView& tv = h.tv;
    const int nleaf = tv.nleaf;
    int* cnt;
    int64_t* off;
    OGX_TRY(arena_get(h.ws, S_SOFT_CNT, nleaf, &cnt));
    OGX_TRY(arena_get(h.ws, S_SOFT_OFF, nleaf + 1, &off));
    const double hs = spline_support(h.prm.eps);
    k_soft_lists<false><<<grid_for(nleaf, 128), 128, 0, st>>>(nleaf, tv.leafbox, tv.child, tv.leafid, tv.center, tv.root, hs,
                                                              cnt, nullptr, nullptr, h.d_counts); ++h.launches;
    OGX_TRY(scan_i32_to_i64(h, cnt, off, nleaf));
    int64_t ns = 0;
    OGX_CUDA(cudaMemcpyAsync(&ns, off + nleaf, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
    OGX_CUDA(cudaStreamSynchronize(st));
    int* idx;
    OGX_TRY(arena_get(h.ws, S_SOFT_IDX, ns + 1, &idx));
    k_soft_lists<true><<<grid_for(nleaf, 128), 128, 0, st>>>(nleaf, tv.leafbox, tv.child, tv.leafid, tv.center, tv.root, hs,
                                                             nullptr, off, idx, h.d_counts); ++h.launches;
    tv.s_off = off;
    tv.s_idx = idx;
    h.soft_pairs = ns;
    OGX_CUDA(cudaGetLastError());
    return OGX_OK;
}

int lists_build(Handle& h) {
    OGX_TRY(lists_build_targets(h));
    return lists_build_uwx(h);
}

int lists_build_targets(Handle& h) {
    const cudaStream_t st = h.stream;
    TreeView& tv = h.tv;
    const int nb = tv.nb;   // launch size (the capacity in capacity mode)
    DevCounts* dc = h.d_counts;
    int* col;
    OGX_TRY(arena_get(h.ws, S_BOX_COL, 27 * (size_t)nb, &col));
    k_colleagues_bs<<<grid_for(27 * (int64_t)nb, 256), 256, 0, st>>>(nb, h.d_level_off, tv.level, tv.coord, col, dc); ++h.launches;
    k_colleagues_check<<<grid_for(nb, 4), 128, 0, st>>>(0, nb, tv.leafid, tv.child, tv.center, tv.root, col, dc); ++h.launches;
    tv.col = col;

    // M2L targets (levels >= 2) grouped by child octant, then by the slot pattern of
    // their V lists; launched over the box capacity, the padding sorts last.  They need
    // only the colleagues, so they are built on the aux stream beside the U/W passes
    // (which use the scan scratch, not the radix-sort scratch); the main stream joins
    // before the X-list sort, which uses the radix-sort scratch again.
    OGX_CUDA(cudaEventRecord(h.ev_col, st));
    OGX_CUDA(cudaStreamWaitEvent(h.aux, h.ev_col, 0));
    h.stream = h.aux;   // radix_sort_u32 issues on h.stream
    const int tcap = std::max(nb, 1);
    uint32_t *tk, *tb;
    OGX_TRY(arena_get(h.ws, S_TGT_KEY, tcap + 1, &tk));
    OGX_TRY(arena_get(h.ws, S_TGT_BOX, tcap + 1, &tb));
    k_tgt_keys<<<grid_for(tcap, 256), 256, 0, h.aux>>>(tcap, h.d_level_off, tv.coord, tv.parent, col, tv.child, tk, tb, dc); ++h.launches;
    uint32_t *tk_s, *tb_s;
    const int rc_t = radix_sort_u32(h, S_TGT_KEY, S_TGT_BOX, S_TGT_KEY2, S_TGT_BOX2, tcap, 31, &tk_s, &tb_s);
    h.stream = st;
    OGX_TRY(rc_t);
    h.tgt_key = tk_s;
    h.tgt_box = tb_s;
    const int tile = 128;  // tensor-core M2L tile; a multiple of the FP64 kernel's 64
    const int fill = h.tile_fill;   // targets per tile (the M2L batch width)
    const int ntgt_bound = h.cap_mode ? tcap : std::max(0, nb - (h.max_level >= 2 ? h.level_off[2] : nb));
    const int npad = ((ntgt_bound + fill - 1) / fill + 8) * tile;
    int* gs;
    uint32_t *pk, *pb;
    OGX_TRY(arena_get(h.ws, S_TGT_TILE, 32, &gs));
    OGX_TRY(arena_get(h.ws, S_TGT_PKEY, npad, &pk));
    OGX_TRY(arena_get(h.ws, S_TGT_PBOX, npad, &pb));
    k_target_groups<<<1, 32, 0, h.aux>>>(tk_s, dc, tile, fill, gs); ++h.launches;
    k_target_pad<<<grid_for(npad, 256), 256, 0, h.aux>>>(tb_s, gs, npad, tile, fill, pk, pb); ++h.launches;
    h.tgt_tile_key = pk;
    h.tgt_tile_box = pb;
    h.ntgt_pad = npad;
    h.ntgt = ntgt_bound;
    OGX_CUDA(cudaEventRecord(h.ev_tgt, h.aux));
    OGX_CUDA(cudaGetLastError());
    return OGX_OK;
}

int lists_build_uwx(Handle& h) {
    const cudaStream_t st = h.stream;
    TreeView& tv = h.tv;
    const int nb = tv.nb, nleaf = tv.nleaf;   // launch sizes (capacities in capacity mode)
    DevCounts* dc = h.d_counts;
    const int* col = tv.col;
    int *ucnt, *wcnt, *lane_uw;
    int64_t *uoff, *woff;
    OGX_TRY(arena_get(h.ws, S_U_CNT, nleaf, &ucnt));
    OGX_TRY(arena_get(h.ws, S_W_CNT, nleaf, &wcnt));
    OGX_TRY(arena_get(h.ws, S_UW_LANE, 64 * (size_t)nleaf, &lane_uw));
    OGX_TRY(arena_get(h.ws, S_U_OFF, nleaf + 1, &uoff));
    OGX_TRY(arena_get(h.ws, S_W_OFF, nleaf + 1, &woff));
    if (h.cap_mode) {   // padding leaves count nothing
        OGX_CUDA(cudaMemsetAsync(ucnt, 0, sizeof(int) * (size_t)nleaf, st));
        OGX_CUDA(cudaMemsetAsync(wcnt, 0, sizeof(int) * (size_t)nleaf, st));
    }
    int* lane_u = lane_uw;
    int* lane_w = lane_uw + 32 * (size_t)nleaf;
    k_uw_warp<false><<<grid_for(nleaf, 4), 128, 0, st>>>(nleaf, tv.leafbox, tv.parent, tv.child, tv.leafid, col, tv.center,
                                                         tv.pcount, tv.root, lane_u, lane_w, ucnt, wcnt, nullptr, nullptr,
                                                         nullptr, nullptr, dc); ++h.launches;
    OGX_TRY(scan_i32_to_i64(h, ucnt, uoff, nleaf));
    OGX_TRY(scan_i32_to_i64(h, wcnt, woff, nleaf));
    int64_t nu, nw;
    if (h.cap_mode) {
        nu = h.cap.u;
        nw = h.cap.w;
        k_check_lists<<<1, 32, 0, st>>>(dc, uoff + nleaf, woff + nleaf, nu, nw); ++h.launches;
    } else {
        // sync point 2: list sizes
        k_check_lists<<<1, 32, 0, st>>>(dc, uoff + nleaf, woff + nleaf, INT64_MAX, INT64_MAX); ++h.launches;
        OGX_CUDA(cudaMemcpyAsync(h.h_counts, dc, sizeof(DevCounts), cudaMemcpyDeviceToHost, st));
        OGX_CUDA(cudaStreamSynchronize(st));
        nu = h.h_counts->u_total;
        nw = h.h_counts->w_total;
    }
    int *uidx, *widx;
    OGX_TRY(arena_get(h.ws, S_U_IDX, nu + 1, &uidx));
    OGX_TRY(arena_get(h.ws, S_W_IDX, nw + 1, &widx));
    k_uw_warp<true><<<grid_for(nleaf, 4), 128, 0, st>>>(nleaf, tv.leafbox, tv.parent, tv.child, tv.leafid, col, tv.center,
                                                        tv.pcount, tv.root, lane_u, lane_w, nullptr, nullptr, uoff, woff, uidx,
                                                        widx, dc); ++h.launches;
    tv.u_off = uoff; tv.w_off = woff; tv.u_idx = uidx; tv.w_idx = widx;

    OGX_CUDA(cudaStreamWaitEvent(st, h.ev_tgt, 0));   // target sort done with the radix scratch
    // X lists: W transposed by a stable sort on the W member; keys behind the W total
    // (capacity padding) sort last and are never referenced by x_off
    const int xbits = bits_for(nb);
    uint32_t *xk, *xv;
    int* xcnt;
    int64_t* xoff;
    OGX_TRY(arena_get(h.ws, S_X_KEY, nw + 1, &xk));
    OGX_TRY(arena_get(h.ws, S_X_VAL, nw + 1, &xv));
    OGX_TRY(arena_get(h.ws, S_X_CNT, nb, &xcnt));
    OGX_TRY(arena_get(h.ws, S_X_OFF, nb + 1, &xoff));
    OGX_CUDA(cudaMemsetAsync(xcnt, 0, sizeof(int) * (size_t)nb, st));
    k_x_emit<<<grid_for(nleaf, 128), 128, 0, st>>>(nleaf, tv.leafbox, woff, widx, xk, xv, xcnt, dc); ++h.launches;
    if (h.cap_mode) { k_fill_tail_x<<<grid_for(nw, 256), 256, 0, st>>>(xk, dc, nw, (1u << xbits) - 1u); ++h.launches; }
    uint32_t *xk_s, *xv_s;
    OGX_TRY(radix_sort_u32(h, S_X_KEY, S_X_VAL, S_X_KEY2, S_X_VAL2, nw, xbits, &xk_s, &xv_s));
    OGX_TRY(scan_i32_to_i64(h, xcnt, xoff, nb));
    tv.x_off = xoff;
    tv.x_idx = (const int*)xv_s;

    OGX_CUDA(cudaGetLastError());
    return OGX_OK;
}

}  // namespace ogx
