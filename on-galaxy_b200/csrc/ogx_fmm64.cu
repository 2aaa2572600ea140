// ogx_fmm64.cu -- the plain FP64 form of the adaptive FMM evaluation.
//
// Same passes as AdaptiveFMM3D::computeAccelerations (src3d/AdaptiveFMM3D.hpp:29-110)
// but organised for the GPU:
//   P2M           warp per leaf: lanes build harmonics of 32 bodies into shared
//                 memory, then reduce columns (:53-61, FmmExpansions3D.hpp:148-163)
//   M2M           bottom-up in one launch (groups of parents taken level by level,
//                 each waiting for its children), warp per child octant,
//                 level-independent matrices MM_s (:62-71)
//   M2L           all levels in one launch: targets grouped by their octant in
//                 the parent, 64 per CTA; for each of the 189 (colleague slot,
//                 child) combinations the sources of all 64 targets are gathered
//                 into shared memory and multiplied by the offset's matrix T_o
//                 (:78-81; V list implicit in the colleague slots)
//   P2L           warp per box over its X list (:82, :117-128)
//   L2L           top-down in one launch, the same way (:75-77)
//   leaf far      warp per leaf: L2P through gradient coefficients of L, M2P
//                 over the W list through gradient coefficients of M (:92-93)
//   leaf near     warp per leaf: softened P2P over the U list, j != i (:95-103),
//                 then acc[orig] = G (far + near) (:104)
// Potentials (pot = -G Phi) are produced alongside when requested.
#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "ogx_harmonics.cuh"
#include "ogx_expansion_kernels.cuh"
#include "ogx_mixed_kernels.cuh"

namespace ogx {

namespace {

constexpr unsigned FULL = 0xffffffffu;

// ---- leaf far field: coefficient records, then L2P + M2P -------------------------
template <int P, class T>
int launch_far(Handle& h, const double* M, const double* L, double* far, bool pot) {
    using Lo = EvalLayout<P>;
    const cudaStream_t st = h.stream;
    TreeView& tv = h.tv;
    T *hrec, *grec;
    OGX_TRY(arena_get(h.ws, S_EVAL_H, (size_t)tv.nb * Lo::HREC, &hrec));
    OGX_TRY(arena_get(h.ws, S_EVAL_G, (size_t)tv.nleaf * Lo::GREC, &grec));
    k_eval_coeffs<P, 0, T><<<(tv.nb + 3) / 4, 128, 0, st>>>(tv, tv.nb, M, hrec); ++h.launches;
    k_eval_coeffs<P, 1, T><<<(tv.nleaf + 3) / 4, 128, 0, st>>>(tv, tv.nleaf, L, grec); ++h.launches;
    if (pot) { k_leaf_far<P, true, T><<<(tv.nleaf + 3) / 4, 128, 0, st>>>(tv, hrec, grec, far); ++h.launches; }
    else { k_leaf_far<P, false, T><<<(tv.nleaf + 3) / 4, 128, 0, st>>>(tv, hrec, grec, far); ++h.launches; }
    return OGX_OK;
}

// mixed form: FP32 records with folded weights, flat (body, W box) M2P tasks.  The M2P
// part needs only the multipoles, so it runs on the side stream beside the M2L and the
// downward pass (into far_m); the L2P part runs after the downward pass (into far).
template <int P>
int launch_far32_m2p(Handle& h, const double* M, double* far_m, bool pot, cudaStream_t st) {
    using R = mixed::FarRec32<P>;
    TreeView& tv = h.tv;
    float4* hrec;
    OGX_TRY(arena_get(h.ws, S_EVAL_H, (size_t)tv.nb * 2 * R::NEH, &hrec));
    mixed::k_far_rec32<P, 0><<<(tv.nb + 3) / 4, 128, 0, st>>>(tv, tv.nb, M, hrec); ++h.launches;
    // heavy leaves: list, then one CTA of FAR_HW warps per leaf
    int* heavy;
    OGX_TRY(arena_get(h.ws, S_FAR_HEAVY, (size_t)tv.nleaf + 2, &heavy));
    int* ctr = heavy + tv.nleaf;
    OGX_CUDA(cudaMemsetAsync(ctr, 0, 2 * sizeof(int), st));
    mixed::k_far_heavy_list<<<(tv.nleaf + 255) / 256, 256, 0, st>>>(tv, heavy, ctr); ++h.launches;
    const size_t hsmem = mixed::far_heavy_smem_bytes<P>();
    const size_t smem = mixed::far_smem_bytes<P>();
    const int lgrid = (tv.nleaf + mixed::FAR_WARPS - 1) / mixed::FAR_WARPS, lblock = 32 * mixed::FAR_WARPS;
    auto heavyk = pot ? mixed::k_leaf_far32_heavy<P, true, false> : mixed::k_leaf_far32_heavy<P, false, false>;
    auto lightk = pot ? mixed::k_leaf_far32<P, true, false, true> : mixed::k_leaf_far32<P, false, false, true>;
    OGX_CUDA(smem_optin((const void*)heavyk, (int)hsmem));
    OGX_CUDA(smem_optin((const void*)lightk, (int)smem));
    heavyk<<<2 * h.num_sms, 32 * mixed::FAR_HW, hsmem, st>>>(tv, hrec, nullptr, far_m, heavy, ctr); ++h.launches;
    lightk<<<lgrid, lblock, smem, st>>>(tv, hrec, nullptr, far_m); ++h.launches;
    return OGX_OK;
}

template <int P>
int launch_far32_l2p(Handle& h, const double* L, double* far, bool pot) {
    using R = mixed::FarRec32<P>;
    const cudaStream_t st = h.stream;
    TreeView& tv = h.tv;
    float4* grec;
    OGX_TRY(arena_get(h.ws, S_EVAL_G, (size_t)tv.nleaf * 2 * R::NEG, &grec));
    mixed::k_far_rec32<P, 1><<<(tv.nleaf + 3) / 4, 128, 0, st>>>(tv, tv.nleaf, L, grec); ++h.launches;
    const size_t smem = mixed::far_smem_bytes<P>();
    const int lgrid = (tv.nleaf + mixed::FAR_WARPS - 1) / mixed::FAR_WARPS, lblock = 32 * mixed::FAR_WARPS;
    auto l2pk = pot ? mixed::k_leaf_far32<P, true, true, false> : mixed::k_leaf_far32<P, false, true, false>;
    OGX_CUDA(smem_optin((const void*)l2pk, (int)smem));
    l2pk<<<lgrid, lblock, smem, st>>>(tv, nullptr, grec, far); ++h.launches;
    return OGX_OK;
}

// ---- M2M (MODE 0) / L2L (MODE 1): one launch per pass ---------------------------------
// CTA = tr_pb<P>() parents x 8 warps, warp s = child octant s.  Warp s applies the
// operator MM_s / LL_s (transposed, k-major, L2-resident) to its TR_PB parents,
// lanes over output dofs.
//   M2M: M'_P = sum_s MM_s M'_{child s}                (src3d/AdaptiveFMM3D.hpp:62-71)
//        the eight partial products are summed in octant order through shared memory
//   L2L: L'_{child s} = L'own_{child s} + LL_s L'_P     (src3d/AdaptiveFMM3D.hpp:75-77)
// The reference walks the levels one after another (its GPU form launches once per
// level, src3d/gpu/AdaptiveFMM3DGPU.cu:274-289).  Here one launch covers every level.
// The CTAs take groups of TR_PB parents of one level by ticket (an atomic counter) in
// level order: root level first for L2L, deepest level first for M2M.  A group waits
// until its inputs are final: for L2L each parent's local, written by the group that
// holds the parent's parent; for M2M each non-leaf child's multipole.  Those groups hold
// earlier tickets, taken by CTAs that are already running, so every wait ends; each is
// bounded all the same (one that runs out sets *err).  A group publishes its boxes with
// a fence and a release store of ready[box]; data written in this launch is read
// through L2 (ld.global.cg).  The arithmetic per box is the same in any order.
// parents per CTA: each warp applies its operator to TR_PB parents per load of an
// operator row (4 where the shared staging fits the 48 KB static limit)
template <int P>
constexpr int tr_pb() { return (P + 1) * (P + 1) <= 81 ? 4 : 2; }
// operator rows in flight per warp (at most ~128 registers, two CTAs per SM)
template <int P>
constexpr int tr_kb() { return (P + 1) * (P + 1) <= 96 ? 12 : 6; }

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(int* p, int v) {
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// bounded wait until *flag != 0; false when it ran out (*err is then set) or when
// another wait already gave up
__device__ bool wait_ready(const int* flag, int* err, uint32_t limit = sm100::kSpinLimit) {
    for (uint32_t it = 0; it < limit; ++it) {
        if (ld_acquire_gpu(flag)) return true;
        if (*(volatile int*)err) return false;
        if (it > 16) __nanosleep(64);
    }
    atomicExch(err, 1);
    return false;
}

template <int P, int MODE>
__global__ void __launch_bounds__(256) k_translate_flow(TreeView tv, const int* __restrict__ nonleaf,
                                                        const int* __restrict__ nl_off, int nlev, int ibeg, int iend,
                                                        const double* __restrict__ opsT, double* mpole, double* local,
                                                        const double* __restrict__ lown, int* ready, int* ticket,
                                                        int* err) {
    constexpr int K = (P + 1) * (P + 1);
    constexpr int NPL = (K + 31) / 32;
    constexpr int TR_PB = tr_pb<P>();
    __shared__ double s_in[MODE == 0 ? 8 : 1][TR_PB][K];
    __shared__ double s_part[MODE == 0 ? 8 : 1][TR_PB][MODE == 0 ? K : 1];
    __shared__ int s_gend[kMaxDepth + 2];   // groups of the pass's first i+1 levels
    __shared__ int s_t;
    const int lane = threadIdx.x & 31, s = threadIdx.x >> 5;
    if (tv_over(tv) || nlev <= 0 || ibeg >= iend) return;
    if (threadIdx.x == 0) {
        int c = 0;
        for (int i = 0; i < iend; ++i) {
            const int l = MODE == 1 ? i : nlev - 1 - i;
            c += (nl_off[l + 1] - nl_off[l] + TR_PB - 1) / TR_PB;
            s_gend[i] = c;
        }
    }
    for (;;) {
        __syncthreads();   // s_gend is written; the previous group's shared data was read
        // this launch's levels are pass-order indices [ibeg, iend): its tickets count from
        // the first group of level ibeg
        if (threadIdx.x == 0) s_t = atomicAdd(ticket, 1) + (ibeg > 0 ? s_gend[ibeg - 1] : 0);
        __syncthreads();
        const int t = s_t;
        if (t >= s_gend[iend - 1]) break;
        int i = 0;
        while (t >= s_gend[i]) ++i;
        const int l = MODE == 1 ? i : nlev - 1 - i;
        const int p0 = (t - (i > 0 ? s_gend[i - 1] : 0)) * TR_PB;
        const int first = nl_off[l], count = nl_off[l + 1] - first;
        int bx[TR_PB], ch[TR_PB];
        bool any = false;
#pragma unroll
        for (int a = 0; a < TR_PB; ++a) {
            bx[a] = (p0 + a < count) ? nonleaf[first + p0 + a] : -1;
            ch[a] = (bx[a] >= 0) ? tv.child[8 * bx[a] + s] : -1;
            any |= ch[a] >= 0;
        }
        // wait for this group's inputs
        if (MODE == 1) {
            if (l > 0 && threadIdx.x < TR_PB) {
                int b = -1;
#pragma unroll
                for (int a = 0; a < TR_PB; ++a) b = (a == (int)threadIdx.x) ? bx[a] : b;
                if (b >= 0) wait_ready(ready + b, err);   // published by the group of b's parent
            }
        } else if (lane < TR_PB) {
            int c = -1;
#pragma unroll
            for (int a = 0; a < TR_PB; ++a) c = (a == lane) ? ch[a] : c;
            if (c >= 0 && tv.leafid[c] < 0) wait_ready(ready + c, err);
        }
        __syncthreads();
        if (MODE == 0) {
#pragma unroll
            for (int a = 0; a < TR_PB; ++a)
                for (int d = lane; d < K; d += 32) s_in[s][a][d] = (ch[a] >= 0) ? __ldcg(mpole + (size_t)ch[a] * K + d) : 0.0;
            __syncwarp();
        } else {
#pragma unroll
            for (int a = 0; a < TR_PB; ++a)
                for (int d = threadIdx.x; d < K; d += blockDim.x) s_in[0][a][d] = (bx[a] >= 0) ? __ldcg(local + (size_t)bx[a] * K + d) : 0.0;
            __syncthreads();
        }
        double acc[TR_PB][NPL];
#pragma unroll
        for (int a = 0; a < TR_PB; ++a)
#pragma unroll
            for (int q = 0; q < NPL; ++q) acc[a][q] = 0.0;
        if (any) {  // warp-uniform
            const double* T = opsT + (size_t)s * K * K;
            const int si = MODE == 0 ? s : 0;
            // operator rows in batches of TR_KB, all loads of a batch issued before its
            // FMAs (the pass is bound by the chain of L2 round trips); kk order unchanged
            constexpr int TR_KB = tr_kb<P>();
            for (int k0 = 0; k0 < K; k0 += TR_KB) {
                double tq[TR_KB][NPL];
#pragma unroll
                for (int u = 0; u < TR_KB; ++u)
#pragma unroll
                    for (int q = 0; q < NPL; ++q) {
                        const int j = lane + 32 * q;
                        tq[u][q] = (k0 + u < K && j < K) ? __ldg(T + (size_t)(k0 + u) * K + j) : 0.0;
                    }
#pragma unroll
                for (int u = 0; u < TR_KB; ++u) {
                    if (k0 + u >= K) break;
#pragma unroll
                    for (int a = 0; a < TR_PB; ++a) {
                        const double v = s_in[si][a][k0 + u];
#pragma unroll
                        for (int q = 0; q < NPL; ++q) acc[a][q] = fma(tq[u][q], v, acc[a][q]);
                    }
                }
            }
        }
        if (MODE == 1) {
#pragma unroll
            for (int a = 0; a < TR_PB; ++a) {
                if (ch[a] < 0) continue;
#pragma unroll
                for (int q = 0; q < NPL; ++q) {
                    const int j = lane + 32 * q;
                    if (j < K) local[(size_t)ch[a] * K + j] = lown[(size_t)ch[a] * K + j] + acc[a][q];
                }
            }
            __threadfence();
            __syncthreads();
            if (lane < TR_PB) {
                int c = -1;
#pragma unroll
                for (int a = 0; a < TR_PB; ++a) c = (a == lane) ? ch[a] : c;
                if (c >= 0) st_release_gpu(ready + c, 1);
            }
        } else {
#pragma unroll
            for (int a = 0; a < TR_PB; ++a)
#pragma unroll
                for (int q = 0; q < NPL; ++q) {
                    const int j = lane + 32 * q;
                    if (j < K) s_part[s][a][j] = acc[a][q];
                }
            __syncthreads();
#pragma unroll
            for (int a = 0; a < TR_PB; ++a) {
                if (bx[a] < 0) continue;
                for (int d = threadIdx.x; d < K; d += blockDim.x) {
                    double v = 0.0;
#pragma unroll
                    for (int o = 0; o < 8; ++o) v += s_part[o][a][d];
                    mpole[(size_t)bx[a] * K + d] = v;
                }
            }
            __threadfence();
            __syncthreads();
            if (threadIdx.x < TR_PB) {
                int b = -1;
#pragma unroll
                for (int a = 0; a < TR_PB; ++a) b = (a == (int)threadIdx.x) ? bx[a] : b;
                if (b >= 0) st_release_gpu(ready + b, 1);
            }
        }
    }
}

// Groups of one level's translation: enough for the level's boxes (eager: the level
// size is known on the host; capacity mode: the level's capacity)
template <int P>
int translate_groups(const Handle& h, int l) {
    if (h.cap_mode) return (h.cap.level_boxes[l] + tr_pb<P>() - 1) / tr_pb<P>();
    const int nbl = h.level_off[l + 1] - h.level_off[l];   // bound on the level's parents
    return (nbl + tr_pb<P>() - 1) / tr_pb<P>();
}

// A translation pass.  A tree of at least kFlowBoxes boxes takes one launch over every
// level: CTAs for every SM (as many as fit), at most one per group.  A smaller tree (a
// system that shares the GPU with others, typically) takes one launch per level, each
// with its level's groups only: its level chain would otherwise keep waiting CTAs on
// most SMs while its few groups per level run.  Same kernel, same arithmetic per box.
// The ready flags and the ticket counters (one per launch) are cleared first.
constexpr int kFlowBoxes = 32768;
template <int P, int MODE>
int launch_translate(Handle& h, Slot slot, double* M, double* L, const double* Lown) {
    const int nlev = h.max_level;   // parent levels 0 .. max_level-1
    if (nlev <= 0) return OGX_OK;
    int groups = 0;
    for (int l = 0; l < nlev; ++l) groups += translate_groups<P>(h, l);
    if (groups <= 0) return OGX_OK;
    static const int per_sm = [] {
        int b = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_translate_flow<P, MODE>, 256, 0) != cudaSuccess) {
            cudaGetLastError();
            b = 1;
        }
        return std::max(1, b);
    }();
    int* ready;
    const size_t nready = (size_t)h.tv.nb + kMaxDepth + 2;
    OGX_TRY(arena_get(h.ws, slot, nready, &ready));
    OGX_CUDA(cudaMemsetAsync(ready, 0, sizeof(int) * nready, h.stream));
    int* tickets = ready + h.tv.nb;
    const double* ops = MODE == 0 ? h.d_m2m : h.d_l2l;
    if (h.tv.nb >= kFlowBoxes) {
        const int grid = std::min(groups, per_sm * h.num_sms);
        k_translate_flow<P, MODE><<<grid, 256, 0, h.stream>>>(h.tv, h.d_nonleaf, h.d_nonleaf_off, nlev, 0, nlev, ops, M, L,
                                                              Lown, ready, tickets, h.d_err);
        ++h.launches;
    } else {
        for (int i = 0; i < nlev; ++i) {
            const int g = translate_groups<P>(h, MODE == 1 ? i : nlev - 1 - i);
            if (g <= 0) continue;
            k_translate_flow<P, MODE><<<std::min(g, per_sm * h.num_sms), 256, 0, h.stream>>>(
                h.tv, h.d_nonleaf, h.d_nonleaf_off, nlev, i, i + 1, ops, M, L, Lown, ready, tickets + i, h.d_err);
            ++h.launches;
        }
    }
    OGX_CUDA(cudaGetLastError());
    return OGX_OK;
}

template <int P>
int launch_m2m(Handle& h, double* M) {
    return launch_translate<P, 0>(h, S_TR_READY_M, M, nullptr, nullptr);
}

template <int P>
int launch_l2l(Handle& h, double* L, const double* Lown) {
    constexpr int K = (P + 1) * (P + 1);
    // root (no parent): its local is its own M2L/P2L part
    OGX_CUDA(cudaMemcpyAsync(L, Lown, sizeof(double) * K, cudaMemcpyDeviceToDevice, h.stream));   // box 0 is the root
    return launch_translate<P, 1>(h, S_TR_READY_L, nullptr, L, Lown);
}

// ---- M2L (structured, FP64) -----------------------------------------------------------
constexpr int M2L_TGT = 64;
constexpr int M2L_THREADS = 256;

// One CTA = up to 64 targets that share their octant t inside the parent.
template <int P>
__global__ void __launch_bounds__(M2L_THREADS) k_m2l_fp64(TreeView tv, const uint32_t* tgt_key, const uint32_t* tgt_box,
                                                         const double* opsT, const double* mpole, double* lown) {
    constexpr int K = (P + 1) * (P + 1);
    constexpr int LD = K | 1;
    constexpr int NR = (K + 15) / 16;
    extern __shared__ double s_m[];                      // [64][LD]
    __shared__ int s_pcol[M2L_TGT][27];
    __shared__ int s_src[M2L_TGT];
    __shared__ int s_tgt[M2L_TGT];
    __shared__ int s_t;
    const int tid = threadIdx.x;
    const int base = blockIdx.x * M2L_TGT;
    if (tv_over(tv)) return;
    // the padded target layout never mixes octants inside a tile
    if (tid == 0) s_t = (tgt_key[base] == 0xFFFFFFFFu) ? -1 : (int)tgt_key[base];
    __syncthreads();
    const int t = s_t;
    if (t < 0) return;
    if (tid < M2L_TGT) {
        const int i = base + tid;
        const int b = ((int)tgt_key[i] == t) ? (int)tgt_box[i] : -1;
        s_tgt[tid] = b;
        const int P_ = (b >= 0) ? tv.parent[b] : -1;
        for (int d = 0; d < 27; ++d) s_pcol[tid][d] = (P_ >= 0) ? tv.col[27 * P_ + d] : -1;
    }
    __syncthreads();
    const int tx = t & 1, ty = (t >> 1) & 1, tz = (t >> 2) & 1;
    const int tg = tid & 15, rg = tid >> 4;
    double acc[4][NR];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int i = 0; i < NR; ++i) acc[a][i] = 0.0;
    for (int D = 0; D < 27; ++D) {
        const int Dx = D % 3 - 1, Dy = (D / 3) % 3 - 1, Dz = D / 9 - 1;
        for (int s = 0; s < 8; ++s) {
            const int ox = 2 * Dx + (s & 1) - tx, oy = 2 * Dy + ((s >> 1) & 1) - ty, oz = 2 * Dz + ((s >> 2) & 1) - tz;
            if (max(abs(ox), max(abs(oy), abs(oz))) <= 1) continue;  // adjacent: not in V
            int mysrc = -1;
            if (tid < M2L_TGT) {
                const int Q = s_pcol[tid][D];
                mysrc = (Q >= 0) ? tv.child[8 * Q + s] : -1;
                s_src[tid] = mysrc;
            }
            if (!__syncthreads_or(mysrc >= 0)) continue;
            for (int idx = tid; idx < M2L_TGT * K; idx += M2L_THREADS) {
                const int r = idx / K, kk = idx - r * K;
                const int src = s_src[r];
                s_m[r * LD + kk] = (src >= 0) ? mpole[(size_t)src * K + kk] : 0.0;
            }
            __syncthreads();
            const double* T = opsT + (size_t)((ox + 3) + 7 * (oy + 3) + 49 * (oz + 3)) * K * K;
            for (int kk = 0; kk < K; ++kk) {
                double mv[4];
#pragma unroll
                for (int a = 0; a < 4; ++a) mv[a] = s_m[(tg + 16 * a) * LD + kk];
#pragma unroll
                for (int i = 0; i < NR; ++i) {
                    const int j = rg + 16 * i;
                    const double tv_ = (j < K) ? __ldg(T + (size_t)kk * K + j) : 0.0;
#pragma unroll
                    for (int a = 0; a < 4; ++a) acc[a][i] = fma(tv_, mv[a], acc[a][i]);
                }
            }
            __syncthreads();
        }
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int b = s_tgt[tg + 16 * a];
        if (b < 0) continue;
        const double inv = 1.0 / (2.0 * tv.center[4 * b + 3]);
#pragma unroll
        for (int i = 0; i < NR; ++i) {
            const int j = rg + 16 * i;
            if (j < K) lown[(size_t)b * K + j] += acc[a][i] * inv;
        }
    }
}

// ---- leaf near field (P2P over U) + final combine ----------------------------------------
// the leaf and first target of near-field work item w (leaf, chunk of 32 targets):
// chunk_off[lf] <= w < chunk_off[lf + 1]; false past the last item
__device__ __forceinline__ bool near_item(const TreeView& tv, const int64_t* chunk_off, int64_t w, int& lf, int& j0) {
    if (w >= chunk_off[tv.nleaf]) return false;
    int lo = 0, hi = tv.nleaf;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (chunk_off[mid] <= w) lo = mid;
        else hi = mid;
    }
    lf = lo;
    j0 = 32 * (int)(w - chunk_off[lo]);
    return true;
}

// Warp per work item (leaf, chunk of 32 targets), so a leaf held large by the eps floor
// spreads over many warps.
template <bool POT, bool SOFT = false>
__global__ void __launch_bounds__(128) k_leaf_near(TreeView tv, const int64_t* __restrict__ chunk_off, double G, double eps2,
                                                   const double* far, double* acc, double* pot, double hs = 0.0,
                                                   double hinv = 0.0) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int lf, j0;
    if (tv_over(tv) || !near_item(tv, chunk_off, blockIdx.x * 4 + wid, lf, j0)) return;
    const int b = tv.leafbox[lf];
    const int f0 = tv.pfirst[b], cnt = tv.pcount[b];
    {
        const int jj = j0 + lane;
        const bool act = jj < cnt;
        const int i = f0 + (act ? jj : 0);
        const double x = tv.px[i], y = tv.py[i], z = tv.pz[i];
        double ax = 0, ay = 0, az = 0, ph = 0;
        for (int64_t e = tv.u_off[lf]; e < tv.u_off[lf + 1]; ++e) {
            const int c = tv.u_idx[e];
            const int s0 = tv.pfirst[c], sc = tv.pcount[c];
            for (int j = s0; j < s0 + sc; ++j) {
                const double dx = __ldg(tv.px + j) - x, dy = __ldg(tv.py + j) - y, dz = __ldg(tv.pz + j) - z;
                const double mj = (j == i) ? 0.0 : __ldg(tv.pm + j);
                if constexpr (SOFT) {
                    const double r2 = dx * dx + dy * dy + dz * dz;
                    double g, k;
                    spline_gk<double>(j == i ? 1.0 : r2, hs, hinv, g, k);
                    const double w = mj * g;
                    if (j != i) {
                        ax = fma(w, dx, ax); ay = fma(w, dy, ay); az = fma(w, dz, az);
                        if (POT) ph = fma(mj, k, ph);
                    }
                } else {
                    const double r2 = (dx * dx + dy * dy + dz * dz) + eps2;
                    const double ir = rsqrt(r2);
                    const double w = mj * ir * ir * ir;
                    if (j != i) {
                        ax = fma(w, dx, ax); ay = fma(w, dy, ay); az = fma(w, dz, az);
                        if (POT) ph = fma(mj, ir, ph);
                    }
                }
            }
        }
        if (act) {
            const int o = tv.perm[i];
            acc[3 * (size_t)o] = G * (far[4 * (size_t)i] + ax);
            acc[3 * (size_t)o + 1] = G * (far[4 * (size_t)i + 1] + ay);
            acc[3 * (size_t)o + 2] = G * (far[4 * (size_t)i + 2] + az);
            if (POT) pot[o] = -G * (far[4 * (size_t)i + 3] + ph);
        }
    }
}

// ---- OGX_SOFT_SPLINE: the far field's pairs within the support ------------------------
// For each leaf b and each leaf c of its S list (not adjacent to b, within the support hs),
// out[4 i] += sum_j m_j (g(r) - r^-3) (r_j - r_i) and, for potentials, m_j (k(r) - 1/r),
// over the pairs closer than hs (the difference is zero beyond).  The far field took these
// pairs with the Newtonian kernel; with this sum they carry the spline kernel's force.
// Warp per leaf, lanes over the leaf's bodies, FP64 (the plain form; the mixed form runs
// the FP32 near-field kernel over the same lists, mixed::k_leaf_near32<.., 2>).
template <bool POT>
__global__ void __launch_bounds__(128) k_soft_correct(TreeView tv, const int64_t* __restrict__ chunk_off, double hs, double hinv,
                                                      double* out) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int lf, j0;
    if (tv_over(tv) || !near_item(tv, chunk_off, blockIdx.x * 4 + wid, lf, j0)) return;
    const int64_t e0 = tv.s_off[lf], e1 = tv.s_off[lf + 1];
    if (e0 == e1) return;
    const int b = tv.leafbox[lf];
    const int f0 = tv.pfirst[b], cnt = tv.pcount[b];
    const double hs2 = hs * hs;
    {
        const int jj = j0 + lane;
        const bool act = jj < cnt;
        const int i = f0 + (act ? jj : 0);
        const double x = tv.px[i], y = tv.py[i], z = tv.pz[i];
        double ax = 0, ay = 0, az = 0, ph = 0;
        for (int64_t e = e0; e < e1; ++e) {
            const int c = tv.s_idx[e];
            const int s0 = tv.pfirst[c], sc = tv.pcount[c];
            for (int j = s0; j < s0 + sc; ++j) {
                const double dx = __ldg(tv.px + j) - x, dy = __ldg(tv.py + j) - y, dz = __ldg(tv.pz + j) - z;
                const double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 < hs2 && r2 > 0.0) {
                    double g, k;
                    spline_gk<double>(r2, hs, hinv, g, k);
                    const double ir = rsqrt(r2);
                    const double mj = __ldg(tv.pm + j);
                    const double w = mj * (g - ir * ir * ir);
                    ax = fma(w, dx, ax); ay = fma(w, dy, ay); az = fma(w, dz, az);
                    if (POT) ph = fma(mj, k - ir, ph);
                }
            }
        }
        if (act) {
            out[4 * (size_t)i] += ax;
            out[4 * (size_t)i + 1] += ay;
            out[4 * (size_t)i + 2] += az;
            if (POT) out[4 * (size_t)i + 3] += ph;
        }
    }
}

}  // namespace

// One thread runs the translation passes' bounded flag wait, with a limit of `polls`, on
// a flag that nothing sets: the wait runs out and sets *err as in the passes.
__global__ void k_flag_wait_probe(const int* flag, int* err, uint32_t polls) {
    if (threadIdx.x == 0) wait_ready(flag, err, polls);
}

int flag_wait_probe(Handle& h, uint32_t polls, const int* flag, int* err) {
    k_flag_wait_probe<<<1, 32, 0, h.stream>>>(flag, err, polls);
    ++h.launches;
    OGX_CUDA(cudaGetLastError());
    return OGX_OK;
}

// work items of the near field (leaf, chunk of 32 targets), on h.stream; the grid of a
// warp-per-item kernel needs at most nleaf + n / 32 warps
int near_items(Handle& h, int64_t** chunk_off) {
    TreeView& tv = h.tv;
    int* nchunk;
    OGX_TRY(arena_get(h.ws, S_NEAR_CHUNK, (size_t)tv.nleaf, &nchunk));
    OGX_TRY(arena_get(h.ws, S_NEAR_CHUNK_OFF, (size_t)tv.nleaf + 1, chunk_off));
    mixed::k_near_chunks<<<(tv.nleaf + 255) / 256, 256, 0, h.stream>>>(tv, nchunk); ++h.launches;
    return scan_i32_to_i64(h, nchunk, *chunk_off, tv.nleaf);
}

int soft_correct_launch(Handle& h, const int64_t* chunk_off, double* out, bool pot, cudaStream_t st) {
    const TreeView& tv = h.tv;
    if (h.soft_pairs == 0 || tv.nleaf == 0) return OGX_OK;
    const double hs = spline_support(h.prm.eps), hinv = 1.0 / hs;
    const int grid = (tv.nleaf + (tv.n + 31) / 32 + 3) / 4;
    if (pot) k_soft_correct<true><<<grid, 128, 0, st>>>(tv, chunk_off, hs, hinv, out);
    else k_soft_correct<false><<<grid, 128, 0, st>>>(tv, chunk_off, hs, hinv, out);
    ++h.launches;
    OGX_CUDA(cudaGetLastError());
    return OGX_OK;
}

namespace {

// ---- dispatch --------------------------------------------------------------------------
template <int P>
int run_fp64(Handle& h, double* d_acc, double* d_pot) {
    constexpr int K = (P + 1) * (P + 1);
    constexpr int LD = K | 1;
    const cudaStream_t st = h.stream;
    TreeView& tv = h.tv;
    OGX_TRY(harm_tables_ready(h.device));
    double *M, *L, *Lown, *far;
    OGX_TRY(arena_get(h.ws, S_MPOLE, (size_t)tv.nb * K, &M));
    OGX_TRY(arena_get(h.ws, S_LOCAL, (size_t)tv.nb * K, &L));
    OGX_TRY(arena_get(h.ws, S_LOWN, (size_t)tv.nb * K, &Lown));
    OGX_TRY(arena_get(h.ws, S_FAR, 4 * (size_t)tv.n, &far));
    OGX_CUDA(timing_record(h, h.ev[2], st));
    // upward
    const size_t p2x_smem = p2x_smem_bytes<P, double>();
    OGX_CUDA(smem_optin((const void*)k_p2x<P, 0, double>, (int)p2x_smem));
    OGX_CUDA(smem_optin((const void*)k_p2x<P, 1, double>, (int)p2x_smem));
    k_p2x<P, 0, double><<<(tv.nleaf + 3) / 4, 128, p2x_smem, st>>>(tv, tv.nleaf, M); ++h.launches;
    OGX_TRY(launch_m2m<P>(h, M));
    OGX_CUDA(timing_record(h, h.ev[3], st));
    // M2L
    OGX_CUDA(cudaMemsetAsync(Lown, 0, sizeof(double) * (size_t)tv.nb * K, st));
    if (h.ntgt > 0 && h.prm.precision == OGX_PREC_FP64_ROT) {
        // third form: the same V pairs through the rotation-factored operators (ogx_m2l_rot.cu)
        OGX_TRY(m2l_rot_launch(h, M, Lown));
    } else if (h.ntgt > 0) {
        const size_t m2l_smem = (size_t)M2L_TGT * LD * sizeof(double);
        OGX_CUDA(smem_optin((const void*)k_m2l_fp64<P>, (int)m2l_smem));
        const int ntiles = h.ntgt_pad / M2L_TGT;
        k_m2l_fp64<P><<<ntiles, M2L_THREADS, m2l_smem, st>>>(tv, h.tgt_tile_key, h.tgt_tile_box, h.d_m2l, M, Lown); ++h.launches;
    }
    OGX_CUDA(timing_record(h, h.ev[4], st));
    // P2L
    k_p2x<P, 1, double><<<(tv.nb + 3) / 4, 128, p2x_smem, st>>>(tv, tv.nb, Lown); ++h.launches;
    OGX_CUDA(timing_record(h, h.ev[5], st));
    // L2L top-down
    OGX_TRY(launch_l2l<P>(h, L, Lown));
    OGX_CUDA(timing_record(h, h.ev[6], st));
    // leaves
    const bool pot = d_pot != nullptr;
    OGX_TRY((launch_far<P, double>(h, M, L, far, pot)));
    const double G = h.prm.G, eps2 = h.prm.eps * h.prm.eps;
    int64_t* chunk_off;
    OGX_TRY(near_items(h, &chunk_off));
    const int ngrid = (tv.nleaf + (tv.n + 31) / 32 + 3) / 4;   // a warp per work item
    if (h.prm.softening == OGX_SOFT_SPLINE) {
        // the far field's pairs within the support, then the spline kernel in the near field
        OGX_TRY(soft_correct_launch(h, chunk_off, far, pot, st));
        const double hs = spline_support(h.prm.eps), hinv = hs > 0.0 ? 1.0 / hs : 0.0;
        if (pot) k_leaf_near<true, true><<<ngrid, 128, 0, st>>>(tv, chunk_off, G, eps2, far, d_acc, d_pot, hs, hinv);
        else k_leaf_near<false, true><<<ngrid, 128, 0, st>>>(tv, chunk_off, G, eps2, far, d_acc, nullptr, hs, hinv);
        ++h.launches;
    } else if (pot) { k_leaf_near<true><<<ngrid, 128, 0, st>>>(tv, chunk_off, G, eps2, far, d_acc, d_pot); ++h.launches; }
    else { k_leaf_near<false><<<ngrid, 128, 0, st>>>(tv, chunk_off, G, eps2, far, d_acc, nullptr); ++h.launches; }
    OGX_CUDA(timing_record(h, h.ev[7], st));
    OGX_CUDA(cudaGetLastError());
    return OGX_OK;
}

// ---- mixed form ---------------------------------------------------------------------

// Operator images for the tensor-core M2L, per offset o, column slice z, K-chunk c
// and part (hi, lo): rows = the slice's output dofs (all of 1..K-1 when there is one
// slice), K-major in the 128-byte-swizzle layout, exactly the bytes one pipeline
// stage holds, so one bulk copy moves a chunk.
// Also row 0 of every T_o (for the degree-0 local coefficient of potentials).
struct MixedImages {
    std::vector<uint8_t> img;
    std::vector<double> row0;
    std::vector<float> ounscale;
};

// built once per order in this process and shared by every handle
template <int P>
std::shared_ptr<const MixedImages> mixed_images() {
    using C = mixed::TcCfg<P>;
    static std::mutex mu;
    static std::shared_ptr<const MixedImages> cached;
    std::lock_guard<std::mutex> lk(mu);
    if (cached) return cached;
    const int K = C::K;
    std::vector<double> T((size_t)K * K);
    auto mi = std::make_shared<MixedImages>();
    std::vector<uint8_t>& img = mi->img;
    std::vector<double>& row0 = mi->row0;
    std::vector<float>& ounscale = mi->ounscale;
    img.assign((size_t)343 * C::NSPLIT * C::NCH * 2 * C::B_BYTES, 0);
    row0.assign((size_t)343 * K, 0.0);
    ounscale.assign(343, 0.f);
    for (int o = 0; o < 343; ++o) {
        const int ox = o % 7 - 3, oy = (o / 7) % 7 - 3, oz = o / 49 - 3;
        if (std::max(std::abs(ox), std::max(std::abs(oy), std::abs(oz))) <= 1) continue;
        build_operator(2, P, o, T.data());
        for (int k = 0; k < K; ++k) row0[(size_t)o * K + k] = T[k];
        // FP16 images of T_o * 2^-e, largest used entry in [0.5, 1); 2^e undoes it
        double mx = 0.0;
        for (int jr = 0; jr < C::NFULL; ++jr)
            for (int k = 0; k < K; ++k) mx = std::max(mx, std::fabs(T[(size_t)(jr + 1) * K + k]));
        int e = 0;
        if (mx > 0.0) std::frexp(mx, &e);
        const double scale = std::ldexp(1.0, -e);
        ounscale[o] = std::ldexp(1.0f, e);
        // slice z, row jr holds output dof 1 + z N + jr
        for (int z = 0; z < C::NSPLIT; ++z)
        for (int c = 0; c < C::NCH; ++c) {
            uint8_t* hi = img.data() + ((size_t)((o * C::NSPLIT + z) * C::NCH + c) * 2) * C::B_BYTES;
            uint8_t* lo = hi + C::B_BYTES;
            for (int jr = 0; jr < C::N; ++jr)
                for (int kk = 0; kk < C::CH * 16; ++kk) {
                    const int k = c * C::CH * 16 + kk, dof = 1 + z * C::N + jr;
                    if (k >= K || dof >= K) continue;
                    const double x = T[(size_t)dof * K + k] * scale;
                    const __half vh = __double2half(x);
                    const __half vl = __double2half(x - (double)__half2float(vh));
                    const int off = mixed::tile_off(jr, kk);
                    std::memcpy(hi + off, &vh, 2);
                    std::memcpy(lo + off, &vl, 2);
                }
        }
    }
    cached = mi;
    return cached;
}

template <int P>
int ensure_mixed_tables(Handle& h) {
    if (h.mix_ready_p == P) return OGX_OK;
    const auto mi = mixed_images<P>();
    const std::vector<uint8_t>& img = mi->img;
    const std::vector<double>& row0 = mi->row0;
    const std::vector<float>& ounscale = mi->ounscale;
    uint8_t* d_img;
    double* d_row0;
    float* d_ous;
    OGX_TRY(arena_get(h.ws, S_MIX_TOPS, img.size(), &d_img));
    OGX_TRY(arena_get(h.ws, S_MIX_ROW0, row0.size(), &d_row0));
    OGX_TRY(arena_get(h.ws, S_MIX_OUNSCALE, ounscale.size(), &d_ous));
    OGX_CUDA(upload_now(d_img, img.data(), img.size()));
    OGX_CUDA(upload_now(d_row0, row0.data(), row0.size() * sizeof(double)));
    OGX_CUDA(upload_now(d_ous, ounscale.data(), ounscale.size() * sizeof(float)));
    h.d_tc_img = d_img;
    h.d_tc_row0 = d_row0;
    h.d_tc_ounscale = d_ous;
    h.mix_ready_p = P;
    return OGX_OK;
}

// Mixed-form upward pass (P2M, M2M, FP16 hi/lo split of the multipoles) on h.up, forked
// from the main stream right after the tree build; the main stream joins it
// (h.ev_up) before the M2L.
template <int P>
int run_mixed_upward(Handle& h) {
    using C = mixed::TcCfg<P>;
    constexpr int K = (P + 1) * (P + 1);
    TreeView& tv = h.tv;
    OGX_TRY(harm_tables_ready(h.device));
    if constexpr (C::SUPPORTED) OGX_TRY(ensure_mixed_tables<P>(h));
    double* M;
    __half *mhi, *mlo;
    float* mus;
    OGX_TRY(arena_get(h.ws, S_MPOLE, (size_t)tv.nb * K, &M));
    OGX_TRY(arena_get(h.ws, S_MIX_MHI, (size_t)tv.nb * C::KPAD, &mhi));
    OGX_TRY(arena_get(h.ws, S_MIX_MLO, (size_t)tv.nb * C::KPAD, &mlo));
    OGX_TRY(arena_get(h.ws, S_MIX_MUNSCALE, (size_t)tv.nb, &mus));
    const size_t p2x_smem = p2x_smem_bytes<P, float>();
    OGX_CUDA(smem_optin((const void*)k_p2x<P, 0, float>, (int)p2x_smem));
    OGX_CUDA(cudaEventRecord(h.ev_tree, h.stream));
    const cudaStream_t main_st = h.stream, su = h.up;
    OGX_CUDA(cudaStreamWaitEvent(su, h.ev_tree, 0));
    h.stream = su;   // launch_m2m issues on h.stream
    OGX_CUDA(timing_record(h, h.ev[2], su));
    k_p2x<P, 0, float><<<(tv.nleaf + 3) / 4, 128, p2x_smem, su>>>(tv, tv.nleaf, M); ++h.launches;
    const int rc = launch_m2m<P>(h, M);
    h.stream = main_st;
    OGX_TRY(rc);
    if constexpr (C::SUPPORTED) {
        mixed::k_split_mpole<P><<<(tv.nb + 3) / 4, 128, 0, su>>>(M, tv.nb, mhi, mlo, mus, tv.cnt); ++h.launches;
    }
    OGX_CUDA(timing_record(h, h.ev_up_end, su));
    OGX_CUDA(cudaEventRecord(h.ev_up, su));
    return OGX_OK;
}

// Mixed-form M2L on the tensor cores, on h.m2l: it waits for the FP16 split of the
// multipoles (h.ev_up) and the target tiles (h.ev_tgt) and runs beside the U/W/X list
// build; run_mixed joins it (h.ev_m2l) before the P2L, which adds into the same locals.
template <int P>
int run_mixed_m2l(Handle& h, bool pot) {
    using C = mixed::TcCfg<P>;
    constexpr int K = (P + 1) * (P + 1);
    constexpr int LD = K | 1;
    const cudaStream_t sm = h.m2l;
    TreeView& tv = h.tv;
    double *M, *Lown;
    __half *mhi, *mlo;
    float* mus;
    OGX_TRY(arena_get(h.ws, S_MPOLE, (size_t)tv.nb * K, &M));
    OGX_TRY(arena_get(h.ws, S_LOWN, (size_t)tv.nb * K, &Lown));
    OGX_TRY(arena_get(h.ws, S_MIX_MHI, (size_t)tv.nb * C::KPAD, &mhi));
    OGX_TRY(arena_get(h.ws, S_MIX_MLO, (size_t)tv.nb * C::KPAD, &mlo));
    OGX_TRY(arena_get(h.ws, S_MIX_MUNSCALE, (size_t)tv.nb, &mus));
    OGX_CUDA(cudaStreamWaitEvent(sm, h.ev_up, 0));
    OGX_CUDA(cudaStreamWaitEvent(sm, h.ev_tgt, 0));
    OGX_CUDA(timing_record(h, h.ev[3], sm));
    OGX_CUDA(cudaMemsetAsync(Lown, 0, sizeof(double) * (size_t)tv.nb * K, sm));
    if (h.ntgt > 0) {
        if constexpr (C::SUPPORTED) {
            OGX_CUDA(smem_optin((const void*)mixed::k_m2l_tc<P>, C::SMEM));
            mixed::k_m2l_tc<P><<<dim3(h.ntgt_pad / 128, C::NSPLIT), C::THREADS, C::SMEM, sm>>>(
                tv, h.tgt_tile_key, h.tgt_tile_box, mhi, mlo, mus, h.d_tc_img, h.d_tc_ounscale, Lown, h.d_err); ++h.launches;
            if (pot) {
                mixed::k_m2l_dof0<P><<<(h.ntgt_pad + 127) / 128, 128, 0, sm>>>(tv, h.ntgt_pad, h.tgt_tile_key, h.tgt_tile_box,
                                                                             h.d_tc_row0, M, Lown); ++h.launches;
            }
        } else {
            // an order whose operand would not fit TMEM even in slices: the FP64 M2L serves it
            const size_t m2l_smem = (size_t)M2L_TGT * LD * sizeof(double);
            OGX_CUDA(smem_optin((const void*)k_m2l_fp64<P>, (int)m2l_smem));
            k_m2l_fp64<P><<<h.ntgt_pad / M2L_TGT, M2L_THREADS, m2l_smem, sm>>>(tv, h.tgt_tile_key, h.tgt_tile_box, h.d_m2l, M,
                                                                           Lown); ++h.launches;
        }
    }
    OGX_CUDA(timing_record(h, h.ev[4], sm));
    OGX_CUDA(cudaEventRecord(h.ev_m2l, sm));
    OGX_CUDA(cudaGetLastError());
    return OGX_OK;
}

template <int P>
int run_mixed(Handle& h, double* d_acc, double* d_pot) {
    constexpr int K = (P + 1) * (P + 1);
    const cudaStream_t st = h.stream;
    TreeView& tv = h.tv;
    double *M, *L, *Lown, *far;
    OGX_TRY(arena_get(h.ws, S_MPOLE, (size_t)tv.nb * K, &M));
    OGX_TRY(arena_get(h.ws, S_LOCAL, (size_t)tv.nb * K, &L));
    OGX_TRY(arena_get(h.ws, S_LOWN, (size_t)tv.nb * K, &Lown));
    OGX_TRY(arena_get(h.ws, S_FAR, 4 * (size_t)tv.n, &far));
    double *nearb, *far_m;
    OGX_TRY(arena_get(h.ws, S_NEAR32, 4 * (size_t)tv.n, &nearb));
    OGX_TRY(arena_get(h.ws, S_FAR_M, 4 * (size_t)tv.n, &far_m));
    const size_t p2x_smem = p2x_smem_bytes<P, float>();
    OGX_CUDA(smem_optin((const void*)k_p2x<P, 1, float>, (int)p2x_smem));
    // near-field work items (leaf, chunk of 32 targets)
    int64_t* chunk_off;
    OGX_TRY(near_items(h, &chunk_off));
    // join the upward pass (the side stream's M2P reads the multipoles)
    OGX_CUDA(cudaStreamWaitEvent(st, h.ev_up, 0));
    // the far field's M2P part and the near field need the tree, the multipoles and the
    // lists: they start here, beside the M2L (launched on h.m2l before the U/W/X lists)
    OGX_CUDA(cudaEventRecord(h.ev_fork, st));
    // near field on the low-priority side stream, issued after the M2L (which takes
    // whole SMs first): its one-warp blocks fill what the M2L's tiles leave free, the
    // SMs its last wave leaves idle, and then what P2L, L2L and the far field leave idle
    {
        const float eps2 = (float)(h.prm.eps * h.prm.eps);
        float4* rel;
        OGX_TRY(arena_get(h.ws, S_MIX_POS4, 2 * (size_t)tv.n, &rel));
        OGX_CUDA(cudaStreamWaitEvent(h.side, h.ev_fork, 0));
        // the far field's M2P part (multipoles only) first, then the near field
        OGX_TRY(launch_far32_m2p<P>(h, M, far_m, d_pot != nullptr, h.side));
        mixed::k_near_prep<<<(tv.n + 255) / 256, 256, 0, h.side>>>(tv, rel, rel + tv.n); ++h.launches;
        // one block per work item: the leaves' chunks number at most nleaf + n / 32 (a
        // bounded grid left the far chain waiting)
        const int ngrid = tv.nleaf + (tv.n + 31) / 32;
        if (h.prm.softening == OGX_SOFT_SPLINE) {
            // spline kernel in the near field; the far field's pairs within the support are
            // corrected in FP32 into the M2P part (written above on this stream)
            const double hs = spline_support(h.prm.eps);
            const float hsf = (float)hs, hinvf = hs > 0.0 ? (float)(1.0 / hs) : 0.f;
            auto near = d_pot ? (h.near_units == 32 ? mixed::k_leaf_near32<true, 32, 1> : mixed::k_leaf_near32<true, 64, 1>)
                              : (h.near_units == 32 ? mixed::k_leaf_near32<false, 32, 1> : mixed::k_leaf_near32<false, 64, 1>);
            near<<<ngrid, 32, 0, h.side>>>(tv, chunk_off, rel, rel + tv.n, eps2, nearb, hsf, hinvf); ++h.launches;
            if (h.soft_pairs > 0) {
                // the same staging over the S lists, the kernel difference added into far_m
                auto corr = d_pot ? (h.near_units == 32 ? mixed::k_leaf_near32<true, 32, 2> : mixed::k_leaf_near32<true, 64, 2>)
                                  : (h.near_units == 32 ? mixed::k_leaf_near32<false, 32, 2> : mixed::k_leaf_near32<false, 64, 2>);
                corr<<<ngrid, 32, 0, h.side>>>(tv, chunk_off, rel, rel + tv.n, eps2, far_m, hsf, hinvf); ++h.launches;
            }
        } else {
            auto near = d_pot ? (h.near_units == 32 ? mixed::k_leaf_near32<true, 32> : mixed::k_leaf_near32<true, 64>)
                              : (h.near_units == 32 ? mixed::k_leaf_near32<false, 32> : mixed::k_leaf_near32<false, 64>);
            near<<<ngrid, 32, 0, h.side>>>(tv, chunk_off, rel, rel + tv.n, eps2, nearb, 0.f, 0.f); ++h.launches;
        }
        OGX_CUDA(cudaEventRecord(h.ev_join, h.side));
    }
    // join the M2L (its end is timing event 4, recorded on h.m2l)
    OGX_CUDA(cudaStreamWaitEvent(st, h.ev_m2l, 0));
    if constexpr (mixed::P2L32<P>::OK) { mixed::k_p2l32<P><<<tv.nb, 32, 0, st>>>(tv, Lown); ++h.launches; }
    else { k_p2x<P, 1, float><<<(tv.nb + 3) / 4, 128, p2x_smem, st>>>(tv, tv.nb, Lown); ++h.launches; }
    OGX_CUDA(timing_record(h, h.ev[5], st));
    OGX_TRY(launch_l2l<P>(h, L, Lown));
    OGX_CUDA(timing_record(h, h.ev[6], st));
    const bool pot = d_pot != nullptr;
    OGX_TRY(launch_far32_l2p<P>(h, L, far, pot));
    // join the side stream (M2P, near field), then acc = G (far + near) in the caller's order
    OGX_CUDA(cudaStreamWaitEvent(st, h.ev_join, 0));
    const double G = h.prm.G;
    if (pot) { mixed::k_combine<true><<<(tv.n + 255) / 256, 256, 0, st>>>(tv.n, tv.perm, G, far, far_m, nearb, d_acc, d_pot, tv.cnt); ++h.launches; }
    else { mixed::k_combine<false><<<(tv.n + 255) / 256, 256, 0, st>>>(tv.n, tv.perm, G, far, far_m, nearb, d_acc, nullptr, tv.cnt); ++h.launches; }
    OGX_CUDA(timing_record(h, h.ev[7], st));
    OGX_CUDA(cudaGetLastError());
    return OGX_OK;
}

}  // namespace

int fmm_mixed_upward(Handle& h) {
    switch (h.prm.p) {
        case 1: return run_mixed_upward<1>(h);
        case 2: return run_mixed_upward<2>(h);
        case 3: return run_mixed_upward<3>(h);
        case 4: return run_mixed_upward<4>(h);
        case 5: return run_mixed_upward<5>(h);
        case 6: return run_mixed_upward<6>(h);
        case 7: return run_mixed_upward<7>(h);
        case 8: return run_mixed_upward<8>(h);
        case 9: return run_mixed_upward<9>(h);
        case 10: return run_mixed_upward<10>(h);
        case 11: return run_mixed_upward<11>(h);
        case 12: return run_mixed_upward<12>(h);
        default: return OGX_ERR_INVALID;
    }
}

int fmm_mixed_m2l(Handle& h, bool pot) {
    switch (h.prm.p) {
        case 1: return run_mixed_m2l<1>(h, pot);
        case 2: return run_mixed_m2l<2>(h, pot);
        case 3: return run_mixed_m2l<3>(h, pot);
        case 4: return run_mixed_m2l<4>(h, pot);
        case 5: return run_mixed_m2l<5>(h, pot);
        case 6: return run_mixed_m2l<6>(h, pot);
        case 7: return run_mixed_m2l<7>(h, pot);
        case 8: return run_mixed_m2l<8>(h, pot);
        case 9: return run_mixed_m2l<9>(h, pot);
        case 10: return run_mixed_m2l<10>(h, pot);
        case 11: return run_mixed_m2l<11>(h, pot);
        case 12: return run_mixed_m2l<12>(h, pot);
        default: return OGX_ERR_INVALID;
    }
}

int fmm_mixed(Handle& h, double* d_acc, double* d_pot) {
    switch (h.prm.p) {
        case 1: return run_mixed<1>(h, d_acc, d_pot);
        case 2: return run_mixed<2>(h, d_acc, d_pot);
        case 3: return run_mixed<3>(h, d_acc, d_pot);
        case 4: return run_mixed<4>(h, d_acc, d_pot);
        case 5: return run_mixed<5>(h, d_acc, d_pot);
        case 6: return run_mixed<6>(h, d_acc, d_pot);
        case 7: return run_mixed<7>(h, d_acc, d_pot);
        case 8: return run_mixed<8>(h, d_acc, d_pot);
        case 9: return run_mixed<9>(h, d_acc, d_pot);
        case 10: return run_mixed<10>(h, d_acc, d_pot);
        case 11: return run_mixed<11>(h, d_acc, d_pot);
        case 12: return run_mixed<12>(h, d_acc, d_pot);
        default: return OGX_ERR_INVALID;
    }
}

int fmm_fp64(Handle& h, double* d_acc, double* d_pot) {
    switch (h.prm.p) {
        case 1: return run_fp64<1>(h, d_acc, d_pot);
        case 2: return run_fp64<2>(h, d_acc, d_pot);
        case 3: return run_fp64<3>(h, d_acc, d_pot);
        case 4: return run_fp64<4>(h, d_acc, d_pot);
        case 5: return run_fp64<5>(h, d_acc, d_pot);
        case 6: return run_fp64<6>(h, d_acc, d_pot);
        case 7: return run_fp64<7>(h, d_acc, d_pot);
        case 8: return run_fp64<8>(h, d_acc, d_pot);
        case 9: return run_fp64<9>(h, d_acc, d_pot);
        case 10: return run_fp64<10>(h, d_acc, d_pot);
        case 11: return run_fp64<11>(h, d_acc, d_pot);
        case 12: return run_fp64<12>(h, d_acc, d_pot);
        default: return OGX_ERR_INVALID;
    }
}

}  // namespace ogx
