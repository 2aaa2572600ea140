// ogx_mixed_kernels.cuh -- kernels of the mixed-precision form.
//
// M2L on the 5th-generation tensor cores (tcgen05, kind::f16, TMEM accumulators).
// The reference applies fmm::M2L pair by pair (src3d/FmmExpansions3D.hpp:273-299,
// called per V-list entry in src3d/AdaptiveFMM3D.hpp:78-81).  Here:
//   * a CTA owns 128 targets that share their octant t inside their parents
//     (any level: the scaled operator is level independent);
//   * the V list of every such target is the children s of its parent's
//     colleague slots D with offset o = 2(D-1) + s - t, max|o| >= 2 (189
//     combinations for a given t); for one combination every target has at
//     most one source, so the sources of the 128 targets form the rows of a
//     dense operand A (128 x K, zero rows where absent) and the translation is
//     D[128 x N] = A . T_o^T with one operator matrix T_o for the whole tile;
//   * split precision: multipoles and operators are split into FP16 hi + lo
//     parts (11 + 11 significant bits) and D accumulates A_hi B_hi + A_hi B_lo +
//     A_lo B_hi in FP32 (the dropped lo x lo term is ~2^-22 relative).  FP16
//     has the significand of TF32 at half the bytes, and the tensor cores' operand
//     reads (shared memory) bound this kernel; its narrow exponent range is met by
//     scaling every multipole row and every operator by a power of two that puts
//     its largest entry in [0.5, 1), undone exactly per row and combination when
//     the result is drained;
//   * accumulation: FP32 accumulation over all ~6000 MMA steps of a tile loses
//     ~1e-5 of the (strongly cancelling) far field, so every combination gets a
//     fresh FP32 accumulator (a ring of buffers in TMEM) that the epilogue warps
//     drain while the MMA warp proceeds with the next combination.  The drain
//     unscales each combination's result, sums the (at most eight) combinations
//     of one colleague slot D in FP32 registers, and folds each slot's sum into
//     an FP64 accumulator (registers for p <= 8, TMEM otherwise);
//   * operands: K is cut into chunks of 64 fp16 (one 128-byte line per row) in
//     the K-major 128-byte-swizzle layout; A rows are gathered with cp.async,
//     each T_o chunk is a pre-laid-out image copied by the TMA bulk engine
//     (cp.async.bulk, no multicast); up to 4 stages pipeline through mbarriers.
//     A producer thread hands its rows of a stage over with an asynchronous
//     mbarrier arrival that fires when its copies have landed, so it never waits
//     for its own copies and every stage of the ring can be in flight;
//   * warp specialisation: four warps gather the A rows (the colleague table
//     of the tile is staged in shared memory and the next combination's source
//     index is fetched one combination ahead), one lane issues the MMAs, and
//     eight drain warps fold each combination into FP64 and write the result.
// Output degree 0 (L_0^0, only needed for potentials) is excluded from N.
// An MMA of N <= ~160 columns costs about the same time, so for p <= 8 the
// operator's hi and lo images form one N = 2 N operand: A_hi x [B_hi | B_lo] and
// A_lo x B_hi are two MMAs per K step (three otherwise).  TMEM holds two FP32
// buffers (2 x 2N or 2 x N columns) + 2 x N FP64-halves columns, which fits
// N <= 128 (p <= 10).  For p = 11 and 12 the output columns are cut into NSPLIT
// slices (2 x 72 and 3 x 56 dofs), each handled by its own CTA (grid y) in the
// paired form with one 64- or 80-column operand; the A rows are gathered once per
// slice.
//
// Near field in FP32 on leaf-centred double-float coordinates (hi + lo FP32
// relative to the target leaf centre, shift in FP64), r^-1 from rsqrt, every
// U-list entry's partial sum folded into a compensated (Kahan) accumulator.
#pragma once

#include <cuda_fp16.h>

#include "ogx_harmonics.cuh"
#include "ogx_sm100.cuh"
#include "ogx_softening.cuh"

namespace ogx {
namespace mixed {

// column slices of the M2L output: 1 while the unsplit operand fits TMEM (4 NPAD
// <= 512), else the fewest slices whose width allows the paired form (6 NPAD <= 512)
constexpr int tc_round16(int v) { return (v + 15) / 16 * 16; }
constexpr int tc_nsplit(int nfull) {
    if (4 * tc_round16(nfull) <= 512) return 1;
    int s = 2;
    while (6 * tc_round16((nfull + s - 1) / s) > 512) ++s;
    return s;
}

template <int P>
struct TcCfg {
    static constexpr int K = (P + 1) * (P + 1);
    static constexpr int KPAD = (K + 15) / 16 * 16;
    static constexpr int NKS = KPAD / 16;     // K-steps of the MMA (16 fp16 each)
    static constexpr int CH = 4;              // K-steps per pipeline chunk (64 fp16 = one 128-byte line)
    static constexpr int NCH = (NKS + CH - 1) / CH;
    static constexpr int NFULL = K - 1;       // output dofs 1..K-1
    static constexpr int NSPLIT = tc_nsplit(NFULL);
    static constexpr int N = (NFULL + NSPLIT - 1) / NSPLIT;   // dofs of one slice: 1 + z N .. z N + N
    static constexpr int NPAD = (N + 15) / 16 * 16;
    static constexpr int M = 128;
    static constexpr int SBO = 1024;          // bytes between 8-row groups (one swizzle atom)
    static constexpr int A_BYTES = (M / 8) * SBO;
    static constexpr int B_BYTES = (NPAD / 8) * SBO;
    static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
    static constexpr int STAGES = (220 * 1024 / STAGE_BYTES) >= 4 ? 4 : (220 * 1024 / STAGE_BYTES);
    static constexpr int SMEM = STAGES * STAGE_BYTES + 1024;
    // Paired form (p <= 8): B_hi and B_lo are adjacent rows of one N = 2 NPAD operand,
    // so A_hi x [B_hi | B_lo] is one MMA and A_lo x B_hi a second one (two MMAs per
    // K-step instead of three; an MMA costs about the same time up to N ~ 160).
    // A combination buffer then holds [hh + lh | hl], summed when drained.
    static constexpr bool PAIR = 6 * NPAD <= 512;
    static constexpr int DBUF = PAIR ? 2 * NPAD : NPAD;  // TMEM columns of one FP32 buffer
    // REGACC (p <= 8): one group of four drain warps per 16-column slice of the
    // output, each lane keeping its 16 FP64 sums in registers (a combination costs a
    // drain warp one TMEM load round trip); TMEM then holds only FP32 buffers, NBUF
    // of them in a ring, so the MMA runs NBUF - 1 combinations ahead of the drain.
    // Otherwise two column slices, FP64 sums in TMEM at column ACC64, two buffers.
    static constexpr bool REGACC = PAIR;
    static constexpr int NGRP = REGACC ? NPAD / 16 : 2;  // column slices
    static constexpr int MAXG = (NPAD / 16 + NGRP - 1) / NGRP;
    static constexpr int DRAIN_WARPS = 4 * NGRP;
    static constexpr int THREADS = 128 + 32 + 32 * DRAIN_WARPS;   // producers, MMA warp, drain warps
    static constexpr int NBUF = REGACC ? 512 / DBUF : 2;
    static constexpr int ACC64 = 2 * DBUF;    // first column of the FP64 accumulator (TMEM form)
    static constexpr int TMEM_COLS = 512;
    static constexpr bool SUPPORTED = 4 * NPAD <= 512 && STAGES >= 2;
    static_assert(CH * 16 * 2 == 128, "a chunk row must fill exactly one 128-byte swizzle line");
};

// Byte offset of fp16 element (row, kk), kk < 64, inside one operand of a stage,
// in the K-major 128-byte-swizzle layout: each row's 64 fp16 of the chunk fill
// one 128-byte line, 8 rows form a 1024-byte atom, and 16-byte piece j of row r
// sits at piece position j ^ (r mod 8) so the tensor core reads the 8 rows of an
// atom from different banks.  Operand bases are 1024-byte aligned.
__host__ __device__ __forceinline__ int tile_off(int row, int kk) {
    return (row >> 3) * 1024 + (row & 7) * 128 + ((((kk >> 3) ^ row) & 7) << 4) + (kk & 7) * 2;
}

// Warp roles: warps 0-3 gather the A rows (thread r owns target row r), warp 4
// issues the MMAs (one lane), warps 5..5+TcCfg::DRAIN_WARPS-1 fold every
// combination's FP32 result into the FP64 accumulator and write the tile's result.
// A warp may only touch the TMEM lane quarter (warp index mod 4), so the drain warps
// come in groups of four, each group owning a slice of the output columns.
constexpr int TC_PRODUCERS = 128;

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]),
        "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}
__device__ __forceinline__ void tmem_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Add the FP32 combination result in D buffer `a` (16-column groups g0..g1-1) to
// the FP64 accumulator of this warp's 32 lanes; `first` initialises it instead.
// PAIR: the buffer holds two partial products NPAD columns apart.  `unscale`
// (a power of two) undoes the row's source scale and the operator's scale.
template <int NPAD, int DBUF, int ACC64, bool PAIR>
__device__ __forceinline__ void drain_combo(uint32_t tmem_lane, int a, bool first, int g0, int g1, float unscale) {
#pragma unroll 1
    for (int c16 = g0; c16 < g1; ++c16) {
        uint32_t v[16], w[16], lo[16], hi[16];
        sm100::tmem_ld16(tmem_lane + a * DBUF + c16 * 16, v);
        if (PAIR) sm100::tmem_ld16(tmem_lane + a * DBUF + NPAD + c16 * 16, w);
        if (!first) {
            sm100::tmem_ld16(tmem_lane + ACC64 + c16 * 32, lo);
            sm100::tmem_ld16(tmem_lane + ACC64 + c16 * 32 + 16, hi);
        }
        sm100::tmem_ld_wait();
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            double s = (double)(__uint_as_float(v[k]) * unscale);
            if (PAIR) s += (double)(__uint_as_float(w[k]) * unscale);
            if (!first) s += __hiloint2double((int)hi[k], (int)lo[k]);
            lo[k] = (uint32_t)__double2loint(s);
            hi[k] = (uint32_t)__double2hiint(s);
        }
        tmem_st16(tmem_lane + ACC64 + c16 * 32, lo);
        tmem_st16(tmem_lane + ACC64 + c16 * 32 + 16, hi);
    }
    tmem_st_wait();
}

template <int P>
__global__ void __launch_bounds__(TcCfg<P>::THREADS, 1)
    k_m2l_tc(TreeView tv, const uint32_t* __restrict__ tgt_key, const uint32_t* __restrict__ tgt_box,
             const __half* __restrict__ mhi, const __half* __restrict__ mlo, const float* __restrict__ munscale,
             const uint8_t* __restrict__ btab, const float* __restrict__ ounscale, double* __restrict__ lown, int* err) {
    using C = TcCfg<P>;
    static_assert(C::SUPPORTED, "tensor-core M2L: operand does not fit");
    const int zs = blockIdx.y;                    // output column slice
    constexpr int NG = C::NPAD / 16;
    constexpr int NGRP = C::NGRP;
    constexpr int NBUF = C::NBUF;
    static_assert(NBUF * C::DBUF + (C::REGACC ? 0 : 2 * C::NPAD) <= C::TMEM_COLS, "TMEM budget");
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    __shared__ uint64_t afull[C::STAGES], bfull[C::STAGES], empty[C::STAGES], dfull[C::NBUF], dempty[C::NBUF], fin;
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_abort;
    __shared__ int s_t, s_ncombo;
    __shared__ int s_box[128];
    __shared__ int s_Q[27][128];      // colleague slot D of each target's parent
    __shared__ int s_par[128];
    __shared__ uint32_t s_mask[7];    // bit D * 8 + s: some target of the tile has that V source
    __shared__ int s_wcnt[7];
    __shared__ int s_combo[189];      // present combinations: D | s << 5 | o << 8
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int base = blockIdx.x * 128;
    if (tv_over(tv)) return;
    if (tid == 0) {
        s_t = (tgt_key[base] == 0xFFFFFFFFu) ? -1 : (int)tgt_key[base];
        s_abort = 0;
        for (int s = 0; s < C::STAGES; ++s) {
            sm100::mbar_init(&afull[s], TC_PRODUCERS);
            sm100::mbar_init(&bfull[s], 1);
            sm100::mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < C::NBUF; ++a) {
            sm100::mbar_init(&dfull[a], 1);
            sm100::mbar_init(&dempty[a], 32 * C::DRAIN_WARPS);
        }
        sm100::mbar_init(&fin, 1);
        sm100::fence_mbar_init();
    }
    if (tid < 7) s_mask[tid] = 0;
    __syncthreads();
    const int t = s_t;
    if (t < 0) return;
    // the A operands of every stage start at zero (rows without a source are not copied)
    for (int i = tid; i < C::STAGES * 2 * C::A_BYTES / 16; i += blockDim.x) {
        const int sg = i / (2 * C::A_BYTES / 16), off = i - sg * (2 * C::A_BYTES / 16);
        reinterpret_cast<uint4*>(smem + (size_t)sg * C::STAGE_BYTES)[off] = make_uint4(0u, 0u, 0u, 0u);
    }
    sm100::fence_proxy_async();
    const int tx = t & 1, ty = (t >> 1) & 1, tz = (t >> 2) & 1;
    if (warp == 4) sm100::tmem_alloc(&s_tmem, C::TMEM_COLS);
    if (tid < 128) {
        const uint32_t key = tgt_key[base + tid];
        const int myb = (key == (uint32_t)t) ? (int)tgt_box[base + tid] : -1;
        s_box[tid] = myb;
        s_par[tid] = (myb >= 0) ? tv.parent[myb] : -1;
    }
    __syncthreads();
    // Colleague slots and the children they offer, spread over the whole CTA: thread
    // (group g, row r) takes slots D = g, g + NGS, ... of target r, with all its loads
    // in flight together.  A warp holds one g and 32 targets, so one OR over the warp
    // gives the presence bits of its slots.
    {
        constexpr int NGS = C::THREADS / 128;
        constexpr int DPT = (27 + NGS - 1) / NGS;
        constexpr int NW = (DPT * 8 + 31) / 32;
        const int r = tid & 127, g = tid >> 7;
        if (g < NGS) {
            const int par = s_par[r];
            int Qv[DPT];
#pragma unroll
            for (int i = 0; i < DPT; ++i) {
                const int D = g + i * NGS;
                Qv[i] = (D < 27 && par >= 0) ? __ldg(tv.col + 27 * (size_t)par + D) : -1;
            }
            int4 cr[DPT][2];
#pragma unroll
            for (int i = 0; i < DPT; ++i) {
                const int D = g + i * NGS;
                if (D < 27) s_Q[D][r] = Qv[i];
                if (Qv[i] >= 0) {
                    cr[i][0] = __ldg(reinterpret_cast<const int4*>(tv.child + 8 * (size_t)Qv[i]));
                    cr[i][1] = __ldg(reinterpret_cast<const int4*>(tv.child + 8 * (size_t)Qv[i]) + 1);
                } else {
                    cr[i][0] = cr[i][1] = make_int4(-1, -1, -1, -1);
                }
            }
            uint32_t bw[NW];
#pragma unroll
            for (int w = 0; w < NW; ++w) bw[w] = 0;
#pragma unroll
            for (int i = 0; i < DPT; ++i) {
                const int D = g + i * NGS;
                const int Dx = D % 3 - 1, Dy = (D / 3) % 3 - 1, Dz = D / 9 - 1;
                const int ch[8] = {cr[i][0].x, cr[i][0].y, cr[i][0].z, cr[i][0].w,
                                   cr[i][1].x, cr[i][1].y, cr[i][1].z, cr[i][1].w};
#pragma unroll
                for (int s = 0; s < 8; ++s) {
                    const int ox = 2 * Dx + (s & 1) - tx, oy = 2 * Dy + ((s >> 1) & 1) - ty, oz = 2 * Dz + ((s >> 2) & 1) - tz;
                    if (D < 27 && max(abs(ox), max(abs(oy), abs(oz))) > 1 && ch[s] >= 0) bw[i >> 2] |= 1u << (8 * (i & 3) + s);
                }
            }
#pragma unroll
            for (int w = 0; w < NW; ++w) bw[w] = __reduce_or_sync(0xffffffffu, bw[w]);
            if (lane == 0) {
#pragma unroll
                for (int i = 0; i < DPT; ++i) {
                    const int D = g + i * NGS;
                    const uint32_t byte = (bw[i >> 2] >> (8 * (i & 3))) & 0xFFu;
                    if (D < 27 && byte) atomicOr(&s_mask[D >> 2], byte << (8 * (D & 3)));
                }
            }
        }
    }
    __syncthreads();
    // the present combinations in (D, s) order, placed by a ballot prefix over 7 warps
    {
        bool pres = false;
        int code = 0;
        unsigned bal = 0;
        if (tid < 224) {
            const int c = tid, D = c >> 3, s = c & 7;
            if (c < 216 && ((s_mask[c >> 5] >> (c & 31)) & 1u)) {
                const int Dx = D % 3 - 1, Dy = (D / 3) % 3 - 1, Dz = D / 9 - 1;
                const int ox = 2 * Dx + (s & 1) - tx, oy = 2 * Dy + ((s >> 1) & 1) - ty, oz = 2 * Dz + ((s >> 2) & 1) - tz;
                pres = true;
                code = D | (s << 5) | (((ox + 3) + 7 * (oy + 3) + 49 * (oz + 3)) << 8);
            }
            bal = __ballot_sync(0xffffffffu, pres);
            if (lane == 0) s_wcnt[warp] = __popc(bal);
        }
        __syncthreads();
        if (pres) {
            int pos = __popc(bal & ((1u << lane) - 1u));
            for (int w = 0; w < warp; ++w) pos += s_wcnt[w];
            s_combo[pos] = code;
        }
        if (tid == 0) {
            int n = 0;
            for (int w = 0; w < 7; ++w) n += s_wcnt[w];
            s_ncombo = n;
        }
    }
    sm100::tc_fence_before();
    __syncthreads();
    sm100::tc_fence_after();
    const uint32_t tmem = s_tmem;
    const int nco = s_ncombo;

    if (warp == 4) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            constexpr uint32_t idesc = sm100::idesc_f16(C::M, C::NPAD);
            constexpr uint32_t idesc2 = sm100::idesc_f16(C::M, 2 * C::NPAD);
            // descriptors differ only in their 14-bit start-address field (bytes >> 4):
            // build stage 0's once and add the stage / K-step / operand offsets
            const uint64_t desc0 = sm100::smem_desc_sw128(sm100::smem_u32(smem), C::SBO);
            constexpr uint32_t D_LO = C::A_BYTES >> 4, D_BHI = (2 * C::A_BYTES) >> 4,
                               D_BLO = (2 * C::A_BYTES + C::B_BYTES) >> 4, D_STAGE = C::STAGE_BYTES >> 4;
            int u = 0;
            for (int k = 0; k < nco && !s_abort; ++k) {
                const int a = k % NBUF;
                if (k >= NBUF) {
                    if (!sm100::mbar_wait(&dempty[a], ((k / NBUF) - 1) & 1, &s_abort)) {
                        s_abort = 1;
                        atomicExch(err, 1);
                        break;
                    }
                    sm100::tc_fence_after();
                }
                const uint32_t dcol = tmem + a * C::DBUF;
                uint32_t accum = 0;
                for (int c = 0; c < C::NCH && !s_abort; ++c, ++u) {
                    const int s = u % C::STAGES;
                    const uint32_t ph = (u / C::STAGES) & 1;
                    if (!sm100::mbar_wait(&afull[s], ph, &s_abort) || !sm100::mbar_wait(&bfull[s], ph, &s_abort)) {
                        s_abort = 1;
                        atomicExch(err, 1);
                        break;
                    }
                    // the A rows were written by cp.async (generic proxy); the MMA reads
                    // them through the async proxy
                    sm100::fence_proxy_async();
                    sm100::tc_fence_after();
                    const uint64_t ds = desc0 + (uint64_t)(s * D_STAGE);
                    const int nks = min(C::CH, C::NKS - c * C::CH);
#pragma unroll
                    for (int ks = 0; ks < C::CH; ++ks) {
                        if (ks < nks) {
                            const uint64_t dk = ds + (uint64_t)(ks * 2);    // 32 bytes per K-step inside the line
                            if constexpr (C::PAIR) {
                                sm100::mma_f16(dcol, dk, dk + D_BHI, idesc2, accum);      // A_hi x [B_hi | B_lo]
                                accum = 1;
                                sm100::mma_f16(dcol, dk + D_LO, dk + D_BHI, idesc, 1);    // A_lo x B_hi
                            } else {
                                sm100::mma_f16(dcol, dk, dk + D_BHI, idesc, accum);
                                accum = 1;
                                sm100::mma_f16(dcol, dk, dk + D_BLO, idesc, 1);
                                sm100::mma_f16(dcol, dk + D_LO, dk + D_BHI, idesc, 1);
                            }
                        }
                    }
                    sm100::mma_commit(&empty[s]);
                }
                sm100::mma_commit(&dfull[a]);
            }
            // completion of every MMA this thread issued (normal end and abort alike)
            sm100::mma_commit(&fin);
            if (!sm100::mbar_wait(&fin, 0, nullptr)) atomicExch(err, 1);
        }
        __syncwarp();
    } else if (warp < 4) {
        // ---------------- producers: thread r gathers target row r ----------------
        const int r = tid;
        int u = 0;
        bool bulk_pending[C::STAGES];
        uint32_t bulk_phase[C::STAGES];
        for (int s = 0; s < C::STAGES; ++s) bulk_pending[s] = false, bulk_phase[s] = 0;
        // source box of the next combination, fetched one combination ahead
        int src_next = -1;
        if (nco > 0) {
            const int c0 = s_combo[0];
            const int Q = s_Q[c0 & 31][r];
            src_next = (Q >= 0) ? __ldg(tv.child + 8 * (size_t)Q + ((c0 >> 5) & 7)) : -1;
        }
        // exits are warp-uniform: the row copies below shuffle across the warp
        for (int k = 0; k < nco && !__any_sync(0xffffffffu, s_abort != 0); ++k) {
            const int code = s_combo[k];
            const int src = src_next;
            if (k + 1 < nco) {
                const int c1 = s_combo[k + 1];
                const int Q = s_Q[c1 & 31][r];
                src_next = (Q >= 0) ? __ldg(tv.child + 8 * (size_t)Q + ((c1 >> 5) & 7)) : -1;
            }
            const int o = code >> 8;
            for (int c = 0; c < C::NCH; ++c, ++u) {
                const int s = u % C::STAGES;
                if (u >= C::STAGES) {
                    const bool ok = sm100::mbar_wait(&empty[s], ((u / C::STAGES) - 1) & 1, &s_abort);
                    if (!__all_sync(0xffffffffu, ok)) {
                        s_abort = 1;
                        atomicExch(err, 1);
                        break;
                    }
                    bulk_pending[s] = false;
                }
                uint8_t* st = smem + (size_t)s * C::STAGE_BYTES;
                if (r == 0) {
                    const uint8_t* bsrc = btab + ((size_t)((o * C::NSPLIT + zs) * C::NCH + c) * 2) * C::B_BYTES;
                    sm100::mbar_arrive_expect_tx(&bfull[s], 2 * C::B_BYTES);
                    sm100::bulk_g2s(st + 2 * C::A_BYTES, bsrc, C::B_BYTES, &bfull[s]);
                    sm100::bulk_g2s(st + 2 * C::A_BYTES + C::B_BYTES, bsrc + C::B_BYTES, C::B_BYTES, &bfull[s]);
                    bulk_pending[s] = true;
                    bulk_phase[s] = (u / C::STAGES) & 1;
                }
                // the warp copies its 32 rows cooperatively: one instruction moves
                // 16-byte pieces q0..q0+3 of 8 rows, so each source row is read in
                // whole 64-byte runs and a quarter-warp fills 8 consecutive slots
                const int k0 = c * C::CH * 16;
                const int nq = min(8, (C::KPAD - k0) / 8);
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int rl = 8 * (i >> 2) + (lane & 7);         // row within the warp
                    const int part = (i >> 1) & 1;                    // 0: hi, 1: lo
                    const int q = (i & 1) * 4 + (lane >> 3);          // 16-byte piece (8 fp16) of the chunk
                    const int rs = __shfl_sync(0xffffffffu, src, rl);
                    if (q < nq) {
                        // an absent source leaves the row's previous contents (finite
                        // values of an earlier row, or the zeros written at start): the
                        // drain multiplies that row's result by an unscale of 0
                        if (rs >= 0)
                            sm100::cp_async16(st + part * C::A_BYTES + tile_off(32 * warp + rl, 8 * q),
                                              (part ? mlo : mhi) + (size_t)rs * C::KPAD + k0 + 8 * q);
                    }
                }
                // the stage's A barrier counts one arrival per producer thread, made
                // when that thread's copies have landed: the producer moves on at once,
                // so every stage of the ring can have its gathers in flight
                sm100::cp_async_mbar_arrive_noinc(&afull[s]);
            }
        }
        sm100::cp_async_wait_all();
        if (s_abort && r == 0) {
            // let this thread's bulk copies land before the CTA exits
            for (int s = 0; s < C::STAGES; ++s)
                if (bulk_pending[s]) sm100::mbar_wait(&bfull[s], bulk_phase[s], nullptr);
        }
    } else {
        // ---------------- drain warps: FP32 combination -> FP64 accumulator -> L_own ----------------
        const int quarter = warp & 3;                 // the TMEM lane quarter this warp may access
        const int grp = (warp - 5) >> 2;              // column slice of this warp
        const int g0 = grp * NG / NGRP, g1 = (grp + 1) * NG / NGRP;
        const uint32_t tmem_lane = tmem + ((uint32_t)(quarter * 32) << 16);
        const int row = quarter * 32 + lane;
        double racc[C::REGACC ? C::MAXG : 1][16];
        float part[C::REGACC ? C::MAXG : 1][16];
#pragma unroll
        for (int g = 0; g < (C::REGACC ? C::MAXG : 1); ++g)
#pragma unroll
            for (int i = 0; i < 16; ++i) racc[g][i] = 0.0, part[g][i] = 0.f;
        for (int k = 0; k < nco && !s_abort; ++k) {
            const int a = k % NBUF;
            // this row's source for combination k and the scales its operands carry
            const int code = s_combo[k];
            // combinations come grouped by colleague slot D (the eight children of one
            // colleague, at similar distances): their FP32 results are summed in FP32 and
            // the slot's sum is folded into FP64 once, after its last combination
            const bool fold = (k + 1 == nco) || ((s_combo[k + 1] & 31) != (code & 31));
            const int Q = s_Q[code & 31][row];
            const int srcb = (Q >= 0) ? __ldg(tv.child + 8 * (size_t)Q + ((code >> 5) & 7)) : -1;
            const float unscale = (srcb >= 0) ? __ldg(munscale + srcb) * __ldg(ounscale + (code >> 8)) : 0.f;
            if (!sm100::mbar_wait(&dfull[a], (k / NBUF) & 1, &s_abort)) {
                s_abort = 1;
                atomicExch(err, 1);
                break;
            }
            sm100::tc_fence_after();
            if constexpr (C::REGACC) {
#pragma unroll
                for (int g = 0; g < C::MAXG; ++g) {
                    const int c16 = g0 + g;
                    if (c16 < g1) {
                        // two halves of 8 columns keep the drain's registers within the
                        // launch's budget; the two partial products meet in FP32 (w is
                        // ~2^-11 of v)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                            uint32_t v[8], w[8];
                            sm100::tmem_ld8(tmem_lane + a * C::DBUF + c16 * 16 + 8 * h, v);
                            sm100::tmem_ld8(tmem_lane + a * C::DBUF + C::NPAD + c16 * 16 + 8 * h, w);
                            sm100::tmem_ld_wait();
#pragma unroll
                            for (int i = 0; i < 8; ++i)
                                part[g][8 * h + i] = fmaf(__uint_as_float(v[i]) + __uint_as_float(w[i]), unscale, part[g][8 * h + i]);
                        }
                        if (fold) {
#pragma unroll
                            for (int i = 0; i < 16; ++i) {
                                racc[g][i] += (double)part[g][i];
                                part[g][i] = 0.f;
                            }
                        }
                    }
                }
            } else {
                drain_combo<C::NPAD, C::DBUF, C::ACC64, C::PAIR>(tmem_lane, a, k == 0, g0, g1, unscale);
            }
            sm100::tc_fence_before();
            sm100::mbar_arrive(&dempty[a]);
        }
        if (nco >= 1 && !s_abort) {
            const int myb = s_box[quarter * 32 + lane];
            const double inv = (myb >= 0) ? 1.0 / (2.0 * tv.center[4 * myb + 3]) : 0.0;
            if constexpr (C::REGACC) {
                if (myb >= 0) {
#pragma unroll
                    for (int g = 0; g < C::MAXG; ++g) {
                        const int c16 = g0 + g;
                        if (c16 < g1) {
#pragma unroll
                            for (int i = 0; i < 16; ++i) {
                                const int col = c16 * 16 + i, dof = 1 + zs * C::N + col;
                                if (col < C::N && dof < C::K) lown[(size_t)myb * C::K + dof] += racc[g][i] * inv;
                            }
                        }
                    }
                }
            } else {
                sm100::tc_fence_after();
#pragma unroll 1
                for (int c16 = g0; c16 < g1; ++c16) {
                    uint32_t lo[16], hi[16];
                    sm100::tmem_ld16(tmem_lane + C::ACC64 + c16 * 32, lo);
                    sm100::tmem_ld16(tmem_lane + C::ACC64 + c16 * 32 + 16, hi);
                    sm100::tmem_ld_wait();
                    if (myb >= 0) {
#pragma unroll
                        for (int k = 0; k < 16; ++k) {
                            const int col = c16 * 16 + k, dof = 1 + zs * C::N + col;
                            if (col < C::N && dof < C::K)
                                lown[(size_t)myb * C::K + dof] += __hiloint2double((int)hi[k], (int)lo[k]) * inv;
                        }
                    }
                }
            }
        }
    }
    sm100::tc_fence_before();
    __syncthreads();
    if (warp == 4) {
        // the MMA lane waited on `fin` above, so no MMA still writes TMEM here
        sm100::tc_fence_after();
        sm100::tmem_dealloc(tmem, C::TMEM_COLS);
    }
}

// FP64 multipoles -> scaled FP16 hi/lo pairs, rows padded to KPAD with zeros.  Warp
// per box: the row is scaled by a power of two 2^-e so that its largest entry lies
// in [0.5, 1) (FP16 keeps 11 significant bits like TF32 but has a narrow exponent
// range); hi = fp16(x), lo = fp16(x - hi); munscale[b] = 2^e undoes the scaling
// exactly when the M2L result is drained.
template <int P>
__global__ void __launch_bounds__(128) k_split_mpole(const double* __restrict__ M, int nb, __half* __restrict__ hi,
                                                     __half* __restrict__ lo, float* __restrict__ munscale,
                                                     const DevCounts* counts) {
    using C = TcCfg<P>;
    const int lane = threadIdx.x & 31;
    const int b = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (b >= nb || b >= counts->nb32 || counts->overflow) return;
    const double* row = M + (size_t)b * C::K;
    double mx = 0.0;
    for (int k = lane; k < C::K; k += 32) mx = fmax(mx, fabs(row[k]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    int e = 0;
    if (mx > 0.0) frexp(mx, &e);
    const double scale = ldexp(1.0, -e);
    for (int k = lane; k < C::KPAD; k += 32) {
        const double x = (k < C::K) ? row[k] * scale : 0.0;
        const __half h = __double2half(x);
        hi[(size_t)b * C::KPAD + k] = h;
        lo[(size_t)b * C::KPAD + k] = __double2half(x - (double)__half2float(h));
    }
    if (lane == 0) munscale[b] = ldexpf(1.0f, e);
}

// L_0^0 of the M2L (needed only for potentials): FP64 row 0 of every T_o
template <int P>
__global__ void __launch_bounds__(128) k_m2l_dof0(TreeView tv, int ntgt_pad, const uint32_t* tgt_key, const uint32_t* tgt_box,
                                                  const double* row0 /* 343 x K */, const double* M, double* lown) {
    constexpr int K = (P + 1) * (P + 1);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntgt_pad || tv_over(tv) || tgt_key[i] == 0xFFFFFFFFu) return;
    const int b = (int)tgt_box[i], t = (int)tgt_key[i];
    const int par = tv.parent[b];
    const int tx = t & 1, ty = (t >> 1) & 1, tz = (t >> 2) & 1;
    double acc = 0.0;
    for (int D = 0; D < 27; ++D) {
        const int Q = tv.col[27 * par + D];
        if (Q < 0) continue;
        const int Dx = D % 3 - 1, Dy = (D / 3) % 3 - 1, Dz = D / 9 - 1;
        for (int s = 0; s < 8; ++s) {
            const int ox = 2 * Dx + (s & 1) - tx, oy = 2 * Dy + ((s >> 1) & 1) - ty, oz = 2 * Dz + ((s >> 2) & 1) - tz;
            if (max(abs(ox), max(abs(oy), abs(oz))) <= 1) continue;
            const int c = tv.child[8 * Q + s];
            if (c < 0) continue;
            const double* r0 = row0 + (size_t)((ox + 3) + 7 * (oy + 3) + 49 * (oz + 3)) * K;
            for (int k = 0; k < K; ++k) acc = fma(r0[k], M[(size_t)c * K + k], acc);
        }
    }
    lown[(size_t)b * K] += acc / (2.0 * tv.center[4 * b + 3]);
}

// ---- FP32 near field ------------------------------------------------------------
// Double-float coordinates: every sorted body's position relative to the root centre
// is held as hi + lo FP32 (hi = fp32(x - c), lo = fp32((x - c) - hi), the difference
// taken in FP64; k_near_prep, once per evaluation).  For a close pair the two hi parts
// lie within a factor of two of each other, so s_hi - t_hi is exact (Sterbenz) and
// d = (s_hi - t_hi) + (s_lo - t_lo) carries the FP32 relative accuracy of |d| itself
// (absolute error ~2^-48 of the root box), however small |d| is.  No per-leaf shift
// is needed, so the sources of many U-list entries are staged together.
__device__ __forceinline__ void kahan_add(float& s, float& c, float v) {
    const float y = v - c;
    const float t = s + y;
    c = (t - s) - y;
    s = t;
}

constexpr int NEAR_CAP = 128;    // source bodies staged per round (several U-list entries)

// work items of the near field: ceil(bodies / 32) per leaf (none for capacity padding)
__global__ void k_near_chunks(TreeView tv, int* __restrict__ cnt) {
    const int lf = blockIdx.x * blockDim.x + threadIdx.x;
    if (lf >= tv.nleaf) return;
    cnt[lf] = (lf < tv_nleaf(tv) && !tv_over(tv)) ? (tv.pcount[tv.leafbox[lf]] + 31) / 32 : 0;
}

__global__ void __launch_bounds__(256) k_near_prep(TreeView tv, float4* __restrict__ rhi, float4* __restrict__ rlo) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= tv.n || tv_over(tv)) return;
    const double ex = tv.px[i] - tv.root->c[0], ey = tv.py[i] - tv.root->c[1], ez = tv.pz[i] - tv.root->c[2];
    const float hx = (float)ex, hy = (float)ey, hz = (float)ez;
    rhi[i] = make_float4(hx, hy, hz, (float)tv.pm[i]);
    rlo[i] = make_float4((float)(ex - (double)hx), (float)(ey - (double)hy), (float)(ez - (double)hz), 0.f);
}

// softened pair sum of one target over staged sources q = q0, q0 + dq, ... < n;
// SELF: the source at staged position self_q is the target itself and is skipped.
// KM (kernel): 0 Plummer's (eps2); 1 the spline of support hs (ogx_softening.cuh);
// 2 the spline minus the Newtonian kernel, zero from hs on (the far field's pairs
// inside the support, OGX_SOFT_SPLINE)
template <bool SELF, bool POT, int KM = 0>
__device__ __forceinline__ void p2p_part(const float4* __restrict__ shi, const float4* __restrict__ slo, int q0, int dq, int n,
                                         int self_q, const float (&th)[3], const float (&tl)[3], float eps2, float (&a)[4],
                                         float hs = 0.f, float hinv = 0.f) {
#pragma unroll 4
    for (int q = q0; q < n; q += dq) {
        const float4 h = shi[q];
        const float4 l = slo[q];
        const float dx = (h.x - th[0]) + (l.x - tl[0]);
        const float dy = (h.y - th[1]) + (l.y - tl[1]);
        const float dz = (h.z - th[2]) + (l.z - tl[2]);
        const bool self = SELF && (q == self_q);
        if constexpr (KM == 1) {
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            float g, k;
            spline_gk<float>(self ? 1.0f : r2, hs, hinv, g, k);
            const float m = self ? 0.0f : h.w;
            const float w = m * g;
            a[0] = fmaf(w, dx, a[0]);
            a[1] = fmaf(w, dy, a[1]);
            a[2] = fmaf(w, dz, a[2]);
            if (POT) a[3] = fmaf(m, k, a[3]);
        } else if constexpr (KM == 2) {
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            if (r2 < hs * hs && r2 > 0.0f) {
                float g, k;
                spline_gk<float>(r2, hs, hinv, g, k);
                const float y = rsqrtf(r2);
                const float w = h.w * (g - y * y * y);
                a[0] = fmaf(w, dx, a[0]);
                a[1] = fmaf(w, dy, a[1]);
                a[2] = fmaf(w, dz, a[2]);
                if (POT) a[3] = fmaf(h.w, k - y, a[3]);
            }
        } else {
            const float r2 = fmaf(dx, dx, fmaf(dy, dy, fmaf(dz, dz, eps2)));
            // rsqrtf alone (within 2 ulp): its error, ~1e-7 per pair in random directions,
            // stays far below the form's budget
            const float y = rsqrtf(self ? 1.0f : r2);
            const float my = (self ? 0.0f : h.w) * y;
            const float w = my * y * y;
            a[0] = fmaf(w, dx, a[0]);
            a[1] = fmaf(w, dy, a[1]);
            a[2] = fmaf(w, dz, a[2]);
            if (POT) a[3] += my;
        }
    }
}

// Number of source parts G for a chunk of T targets: units (target, part) = T G,
// at most NU, are spread over the 32 lanes in R = ceil(T G / 32) rounds; G maximises
// the busy fraction T G / (32 R) (ties: the smaller G).  With NU = 64 a 17-body leaf
// gets G = 3 (80% busy; one target per lane would leave 47% of the lanes idle), a
// 5-body leaf G = 6 (94%).
template <int NU>
__device__ __forceinline__ int near_parts(int T) {
    int best = 1, bu = 0;
    for (int G = 1; G <= 32 && T * G <= NU; ++G) {
        const int U = T * G;
        const int u = (U << 10) / (32 * ((U + 31) >> 5));   // busy fraction, fixed point
        if (u > bu) { bu = u; best = G; }
    }
    return best;
}

// Warp per target leaf (one warp per block, so a block's resources return as soon as
// its leaf is done).  The leaf's bodies go in chunks of up to 32 targets; in a chunk
// of T targets, unit u = lane + 32 r (r < NU / 32) is target u mod T with source part
// u / T, which takes every G-th source of each staged round.  The leaf itself is one
// round (with the self pair skipped); the bodies of all other U-list entries are
// concatenated and staged NEAR_CAP at a time.  Each unit folds every round's partial
// sum into a compensated (Kahan) accumulator; at the end the G parts of each target
// are added in part order in FP64 through shared memory (deterministic).  Output:
// near[4 i] = (sum m d / r^3 xyz, sum m / r) of sorted body i, FP64.  The kernel needs
// only the tree and the lists, so it runs beside the far-field chain.
// KM = 1: the spline kernel (OGX_SOFT_SPLINE).  KM = 2: the far field's pairs inside the
// spline's support instead: the leaf's S list in place of its U list (no self round),
// the kernel difference, and the result added to near[] rather than stored.
// Work items are (leaf, chunk of 32 targets): chunk_off[lf] is the first item of leaf lf
// (k_near_chunks + an exclusive scan), so a leaf of many bodies (the eps floor stops
// splitting in dense cores) spreads over as many blocks as it has chunks.
template <bool POT, int NU, int KM = 0>
__global__ void __launch_bounds__(32, 32) k_leaf_near32(TreeView tv, const int64_t* __restrict__ chunk_off,
                                                        const float4* __restrict__ rhi, const float4* __restrict__ rlo,
                                                        float eps2, double* __restrict__ near, float hs = 0.f,
                                                        float hinv = 0.f) {
    constexpr int R = NU / 32;
    static_assert(R * 32 == NU && R >= 1 && R <= 2, "near-field units: 32 or 64");
    __shared__ float4 s_hi[NEAR_CAP], s_lo[NEAR_CAP];
    __shared__ double s_red[NU][4];
    const int lane = threadIdx.x & 31;
    if (tv_over(tv)) return;
    const int64_t items = chunk_off[tv.nleaf];
    for (int64_t w = blockIdx.x; w < items; w += gridDim.x) {
        // the leaf of item w: chunk_off[lf] <= w < chunk_off[lf + 1] (warp-uniform search)
        int lo = 0, hi = tv.nleaf;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (chunk_off[mid] <= w) lo = mid;
            else hi = mid;
        }
        const int lf = lo;
        const int b = tv.leafbox[lf];
        const int f0 = tv.pfirst[b], cnt = tv.pcount[b];
        const int64_t u0 = KM == 2 ? tv.s_off[lf] : tv.u_off[lf], u1 = KM == 2 ? tv.s_off[lf + 1] : tv.u_off[lf + 1];
        if (KM == 2 && u0 == u1) continue;
        {
            const int j0 = 32 * (int)(w - chunk_off[lf]);
            const int T = min(32, cnt - j0);
            const int G = near_parts<NU>(T);
            const int U = T * G;
            // the lane's units: target tt[r] (index in the leaf), source part pp[r]
            int tt[R], pp[R];
            bool act[R];
            float th[R][3], tl[R][3];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int u = lane + 32 * r;
                act[r] = u < U;
                tt[r] = act[r] ? u % T : 0;
                pp[r] = act[r] ? u / T : 0;
                const float4 h = rhi[f0 + j0 + tt[r]], l = rlo[f0 + j0 + tt[r]];
                th[r][0] = h.x; th[r][1] = h.y; th[r][2] = h.z;
                tl[r][0] = l.x; tl[r][1] = l.y; tl[r][2] = l.z;
            }
            float ks[R][4], kc[R][4];
#pragma unroll
            for (int r = 0; r < R; ++r)
#pragma unroll
                for (int k = 0; k < 4; ++k) ks[r][k] = kc[r][k] = 0.f;
            // round 0: the leaf itself
            for (int k0 = 0; k0 < (KM == 2 ? 0 : cnt); k0 += NEAR_CAP) {
                const int n = min(NEAR_CAP, cnt - k0);
                __syncwarp();
                for (int q = lane; q < n; q += 32) {
                    s_hi[q] = rhi[f0 + k0 + q];
                    s_lo[q] = rlo[f0 + k0 + q];
                }
                __syncwarp();
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (!act[r]) continue;
                    float a[4] = {0.f, 0.f, 0.f, 0.f};
                    p2p_part<true, POT, KM>(s_hi, s_lo, pp[r], G, n, j0 + tt[r] - k0, th[r], tl[r], eps2, a, hs, hinv);
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (k < 3 || POT) kahan_add(ks[r][k], kc[r][k], a[k]);
                }
            }
            // the other U-list entries, 32 at a time: lane e holds entry e's first body and
            // count; an inclusive scan of the counts maps a flat source position to its entry
            for (int64_t eb = u0; eb < u1; eb += 32) {
                const int64_t e = eb + lane;
                int pf = 0, pc = 0;
                if (e < u1) {
                    const int c = KM == 2 ? tv.s_idx[e] : tv.u_idx[e];
                    if (c != b) { pf = tv.pfirst[c]; pc = tv.pcount[c]; }
                }
                int pre = pc;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(0xffffffffu, pre, o);
                    if (lane >= o) pre += v;
                }
                const int total = __shfl_sync(0xffffffffu, pre, 31);
                for (int base = 0; base < total; base += NEAR_CAP) {
                    const int n = min(NEAR_CAP, total - base);
                    __syncwarp();
                    // warp-uniform trip count: every lane takes part in every shuffle
                    for (int q0 = 0; q0 < n; q0 += 32) {
                        const int q = q0 + lane;
                        const int f = base + q;
                        // entry of flat position f: the number of entries whose inclusive
                        // prefix is <= f (five halving steps over the 32 prefixes)
                        int pos = 0;
#pragma unroll
                        for (int step = 16; step > 0; step >>= 1)
                            if (__shfl_sync(0xffffffffu, pre, pos + step - 1) <= f) pos += step;
                        const int ep = __shfl_sync(0xffffffffu, pre, pos), ec = __shfl_sync(0xffffffffu, pc, pos);
                        const int j = __shfl_sync(0xffffffffu, pf, pos) + f - (ep - ec);
                        if (q < n) {
                            s_hi[q] = rhi[j];
                            s_lo[q] = rlo[j];
                        }
                    }
                    __syncwarp();
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        if (!act[r]) continue;
                        float a[4] = {0.f, 0.f, 0.f, 0.f};
                        p2p_part<false, POT, KM>(s_hi, s_lo, pp[r], G, n, -1, th[r], tl[r], eps2, a, hs, hinv);
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            if (k < 3 || POT) kahan_add(ks[r][k], kc[r][k], a[k]);
                    }
                }
            }
            // the parts of every target, in part order, in FP64
            __syncwarp();
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (act[r])
#pragma unroll
                    for (int k = 0; k < 4; ++k) s_red[lane + 32 * r][k] = (double)ks[r][k] - (double)kc[r][k];
            __syncwarp();
            if (lane < T) {
                double v[4] = {0.0, 0.0, 0.0, 0.0};
                for (int p = 0; p < G; ++p)
#pragma unroll
                    for (int k = 0; k < 4; ++k) v[k] += s_red[p * T + lane][k];
                double2* o = reinterpret_cast<double2*>(near + 4 * (size_t)(f0 + j0 + lane));
                if (KM == 2) {
                    const double2 o0 = o[0], o1 = o[1];
                    o[0] = make_double2(o0.x + v[0], o0.y + v[1]);
                    o[1] = make_double2(o1.x + v[2], o1.y + (POT ? v[3] : 0.0));
                } else {
                    o[0] = make_double2(v[0], v[1]);
                    o[1] = make_double2(v[2], POT ? v[3] : 0.0);
                }
            }
        }
        __syncwarp();
    }
}

// acc[orig] = G (far + near), pot[orig] = -G (far + near) (AdaptiveFMM3D.hpp:104)
// far = far_l (L2P) + far_m (M2P) when the two parts ran apart (far_m non-null)
template <bool POT>
__global__ void k_combine(int n, const int* __restrict__ perm, double G, const double* __restrict__ far,
                          const double* __restrict__ far_m, const double* __restrict__ near, double* __restrict__ acc,
                          double* __restrict__ pot, const DevCounts* counts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || counts->overflow) return;
    const int o = perm[i];
    double2 f0 = reinterpret_cast<const double2*>(far)[2 * (size_t)i];
    double2 f1 = reinterpret_cast<const double2*>(far)[2 * (size_t)i + 1];
    if (far_m) {
        const double2 m0 = reinterpret_cast<const double2*>(far_m)[2 * (size_t)i];
        const double2 m1 = reinterpret_cast<const double2*>(far_m)[2 * (size_t)i + 1];
        f0.x += m0.x; f0.y += m0.y; f1.x += m1.x; f1.y += m1.y;
    }
    const double2 n0 = reinterpret_cast<const double2*>(near)[2 * (size_t)i];
    const double2 n1 = reinterpret_cast<const double2*>(near)[2 * (size_t)i + 1];
    acc[3 * (size_t)o] = G * (f0.x + n0.x);
    acc[3 * (size_t)o + 1] = G * (f0.y + n0.y);
    acc[3 * (size_t)o + 2] = G * (f1.x + n1.x);
    if (POT) pot[o] = -G * (f1.y + n1.y);
}

// ---- leaf far field in FP32 (L2P + W-list M2P) ----------------------------------------
// Coefficient records, one 8-float entry per (n, m >= 0), entry index n(n+1)/2 + m:
//   {gx.re', gx.im', gy.re', gy.im', gz.re', gz.im', phi.re', phi.im'}
// where the real-part weights are folded in (m = 0: (c.re, 0); m > 0: (2 c.re,
// -2 c.im)) so that sum_nm Re(c_nm z_nm) = sum_e re' z.re + im' z.im, two 16-byte
// loads feeding eight FMAs per harmonic.  The gradient coefficient sets are those
// of fmm::localField / fmm::multipoleField (src3d/FmmExpansions3D.hpp:180-235):
//   MODE 0, M2P source box: grad of degree P+1, phi of degree P (from M')
//   MODE 1, L2P leaf:       grad of degree P-1, phi of degree P (from L')
template <int P>
struct FarRec32 {
    static constexpr int NEH = (P + 2) * (P + 3) / 2;   // entries of an M2P record
    static constexpr int NEG = (P + 1) * (P + 2) / 2;   // entries of an L2P record
};

// Both parts (re, im) of entry (n, m) of a gradient coefficient set, the values
// mpole_grad_dof / local_grad_dof give for dofs dof_re(n, m) and dof_re(n, m) + 1,
// with the constants read from global memory (lanes hold different (n, m)).
//   MODE 0: multipole set H from M_{n-1} (dz_S / dp_S / dm_S, FmmExpansions3D.hpp:121-129)
//   MODE 1: local set G from L_{n+1}    (cz_R / cp_R / cm_R, FmmExpansions3D.hpp:111-119)
template <int MODE>
__device__ __forceinline__ void grad_entry(const double* c, int n, int m, float gr[3], float gi[3]) {
    if (MODE == 0 && n == 0) return;
    const int N = MODE == 0 ? n - 1 : n + 1;
    double lr, li, pr, pi, mr, mi;
    coef_get(c, N, m, lr, li);
    coef_get(c, N, m - 1, mr, mi);
    coef_get(c, N, m + 1, pr, pi);
    const double cz = __ldg(MODE == 0 ? &g_harm.hz[n][m] : &g_harm.gz[n][m]);
    const double cp = __ldg(MODE == 0 ? &g_harm.hp[n][m] : &g_harm.gp[n][m]);
    const double cm = __ldg(MODE == 0 ? &g_harm.hm[n][m] : &g_harm.gm[n][m]);
    const double xr = 0.5 * (cp * mr + cm * pr), xi = 0.5 * (cp * mi + cm * pi);
    const double dr = cp * mr - cm * pr, di = cp * mi - cm * pi;
    gr[0] = (float)xr; gr[1] = (float)(0.5 * di); gr[2] = (float)(cz * lr);
    if (m > 0) { gi[0] = (float)xi; gi[1] = (float)(-0.5 * dr); gi[2] = (float)(cz * li); }
}

template <int P, int MODE>
__global__ void __launch_bounds__(128) k_far_rec32(TreeView tv, int count, const double* __restrict__ coef,
                                                   float4* __restrict__ rec) {
    constexpr int K = (P + 1) * (P + 1);
    constexpr int NE = MODE == 0 ? FarRec32<P>::NEH : FarRec32<P>::NEG;
    const int lane = threadIdx.x & 31;
    const int k = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (k >= count || k >= (MODE == 0 ? tv_nb(tv) : tv_nleaf(tv)) || tv_over(tv)) return;
    const int b = (MODE == 0) ? k : tv.leafbox[k];
    if (MODE == 0 && tv.x_off[b] == tv.x_off[b + 1]) return;   // never an M2P source
    const double* c = coef + (size_t)b * K;
    float4* o = rec + (size_t)k * 2 * NE;
    for (int e = lane; e < NE; e += 32) {
        int n = 0;
        while ((n + 1) * (n + 2) / 2 <= e) ++n;
        const int m = e - n * (n + 1) / 2;
        const int dr = dof_re(n, m);
        float gr[3] = {0.f, 0.f, 0.f}, gi[3] = {0.f, 0.f, 0.f};
        float pr = 0.f, pi = 0.f;
        if (MODE == 0 || n < P) grad_entry<MODE>(c, n, m, gr, gi);
        if (n <= P) {
            pr = (float)c[dr];
            if (m > 0) pi = (float)c[dr + 1];
        }
        const float wr = m == 0 ? 1.f : 2.f, wi = m == 0 ? 0.f : -2.f;
        o[2 * e] = make_float4(wr * gr[0], wi * gi[0], wr * gr[1], wi * gi[1]);
        o[2 * e + 1] = make_float4(wr * gr[2], wi * gi[2], wr * pr, wi * pi);
    }
}

__device__ __forceinline__ void far_term(const float4* r, int e, float re, float im, float& ax, float& ay, float& az,
                                         float& ph) {
    const float4 c0 = r[2 * e], c1 = r[2 * e + 1];
    ax = fmaf(c0.x, re, fmaf(c0.y, im, ax));
    ay = fmaf(c0.z, re, fmaf(c0.w, im, ay));
    az = fmaf(c1.x, re, fmaf(c1.y, im, az));
    ph = fmaf(c1.z, re, fmaf(c1.w, im, ph));
}

// shared-memory records per warp: up to FAR_R M2P records (or the leaf's L2P record)
constexpr int FAR_R = 4;
// one warp per block: a block's resources return as soon as its leaf is done,
// so leaves of very different cost do not hold idle warps resident
constexpr int FAR_WARPS = 1;
template <int P>
constexpr int far_warp_f4() { return FAR_R * 2 * FarRec32<P>::NEH; }
template <int P>
constexpr size_t far_smem_bytes() { return FAR_WARPS * sizeof(float4) * (size_t)far_warp_f4<P>(); }

// Leaves with more M2P tasks (bodies x W boxes) than this are handled by a CTA
// of FAR_HW warps instead of a single warp (k_leaf_far32_heavy), so one leaf
// with a long W list does not decide the kernel's length.
constexpr int FAR_HEAVY = 1024;
constexpr int FAR_HW = 8;

// end of the M2P round that starts at task b0: at most 32 tasks spanning at most
// R W boxes (the records one warp stages)
__device__ __forceinline__ int far_round_end(int b0, int nbk, int total, int R) {
    return min(total, min(b0 + 32, (b0 / nbk + R) * nbk));
}

// L2P of body block (nbk bodies staged in sx/sy/sz relative to the leaf centre):
// lane owns bodies lane and lane + 32
template <int P>
__device__ __forceinline__ void far_l2p(const float4* __restrict__ g, int nbk, const double* sx, const double* sy,
                                        const double* sz, double inv, float4* srec, int lane, double (&acc)[2][4]) {
    constexpr int NEG = FarRec32<P>::NEG;
    __syncwarp();
    for (int i = lane; i < 2 * NEG; i += 32) srec[i] = __ldg(g + i);
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int j = lane + 32 * q;
        if (j < nbk) {
            const float ux = (float)(sx[j] * inv), uy = (float)(sy[j] * inv), uz = (float)(sz[j] * inv);
            float ax = 0.f, ay = 0.f, az = 0.f, ph = 0.f;
            for_regular<P>(ux, uy, uz, [&](int n, int m, float re, float im) {
                far_term(srec, n * (n + 1) / 2 + m, re, im, ax, ay, az, ph);
            });
            acc[q][0] += (double)ax * inv;
            acc[q][1] += (double)ay * inv;
            acc[q][2] += (double)az * inv;
            acc[q][3] += (double)ph;
        }
    }
}

// One M2P round, tasks [b0, end) of the body block: the W records the round
// needs go to shared memory first (coalesced 16-byte loads), then lane t of the
// round evaluates task b0 + t; every body sums its own task results in task
// order into acc (FP64).
template <int P, bool POT>
__device__ __forceinline__ void far_m2p_round(const TreeView& tv, const float4* __restrict__ hrec, int64_t w0, int nbk,
                                              int b0, int end, const double* sx, const double* sy, const double* sz,
                                              double cx, double cy, double cz, float4* srec, float4* sres, int lane,
                                              double (&acc)[2][4]) {
    constexpr int NEH = FarRec32<P>::NEH;
    const int wa = b0 / nbk;
    const int nrec = (end - 1) / nbk - wa + 1;
    __syncwarp();
    for (int i = lane; i < nrec * 2 * NEH; i += 32) {
        const int r = i / (2 * NEH), off = i - r * (2 * NEH);
        srec[i] = __ldg(hrec + (size_t)tv.w_idx[w0 + wa + r] * 2 * NEH + off);
    }
    __syncwarp();
    const int t = b0 + lane;
    float4 res = make_float4(0.f, 0.f, 0.f, 0.f);
    if (t < end) {
        const int w = t / nbk, j = t - w * nbk;
        const int c = tv.w_idx[w0 + w];
        const double2 c01 = __ldg(reinterpret_cast<const double2*>(tv.center) + 2 * c);
        const double2 c23 = __ldg(reinterpret_cast<const double2*>(tv.center) + 2 * c + 1);
        const float winv = 1.0f / (2.0f * (float)c23.y);
        const float ux = (float)(sx[j] + (cx - c01.x)) * winv;
        const float uy = (float)(sy[j] + (cy - c01.y)) * winv;
        const float uz = (float)(sz[j] + (cz - c23.x)) * winv;
        const float4* hr = srec + (w - wa) * 2 * NEH;
        float ax = 0.f, ay = 0.f, az = 0.f, ph = 0.f;
        for_singular<P + 1>(ux, uy, uz, [&](int n, int m, float re, float im) {
            far_term(hr, n * (n + 1) / 2 + m, re, im, ax, ay, az, ph);
        });
        const float w2 = winv * winv;
        res = make_float4(ax * w2, ay * w2, az * w2, POT ? ph * winv : 0.f);
    }
    sres[lane] = res;
    __syncwarp();
    const int bm = b0 % nbk;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int j = lane + 32 * q;
        if (j < nbk) {
            int k = j - bm;
            if (k < 0) k += nbk;
            for (; b0 + k < end; k += nbk) {
                const float4 v = sres[k];
                acc[q][0] += v.x; acc[q][1] += v.y; acc[q][2] += v.z; acc[q][3] += v.w;
            }
        }
    }
}

// Warp per leaf (one warp per block, so a block's resources return as soon as
// its leaf is done), bodies in blocks of 64 with positions relative to the leaf
// centre staged in FP64 shared memory.  L2P: lanes over bodies.  M2P: the
// (body, W box) pairs of the block form a flat W-major task list taken 32 at a
// time (far_m2p_round), so a leaf of 17 bodies and 9 W boxes keeps every lane
// busy.  The mixed form runs the two parts apart: M2P (DO_M2P, multipoles only) beside
// the M2L and the downward pass, L2P (DO_L2P) after the downward pass.  With DO_M2P,
// leaves with more than FAR_HEAVY tasks are left to k_leaf_far32_heavy.
template <int P, bool POT, bool DO_L2P, bool DO_M2P>
__global__ void __launch_bounds__(32 * FAR_WARPS, 32 / FAR_WARPS) k_leaf_far32(TreeView tv, const float4* __restrict__ hrec,
                                                                             const float4* __restrict__ grec,
                                                                             double* __restrict__ far) {
    constexpr int NEG = FarRec32<P>::NEG;
    extern __shared__ float4 s_far_dyn[];
    __shared__ double s_pos[FAR_WARPS][3][64];
    __shared__ float4 s_res[FAR_WARPS][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int lf = blockIdx.x * FAR_WARPS + wid;
    if (lf >= tv.nleaf || lf >= tv_nleaf(tv) || tv_over(tv)) return;
    const int b = tv.leafbox[lf];
    const int f0 = tv.pfirst[b], cnt = tv.pcount[b];
    const int64_t w0 = tv.w_off[lf];
    const int nw = DO_M2P ? (int)(tv.w_off[lf + 1] - w0) : 0;
    if (DO_M2P && (int64_t)cnt * nw > FAR_HEAVY) return;
    float4* srec = s_far_dyn + (size_t)wid * far_warp_f4<P>();
    const double cx = tv.center[4 * b], cy = tv.center[4 * b + 1], cz = tv.center[4 * b + 2];
    const double inv = 1.0 / (2.0 * tv.center[4 * b + 3]);
    const float4* g = DO_L2P ? grec + (size_t)lf * 2 * NEG : nullptr;
    double* sx = s_pos[wid][0];
    double* sy = s_pos[wid][1];
    double* sz = s_pos[wid][2];
    for (int jb = 0; jb < cnt; jb += 64) {
        const int nbk = min(64, cnt - jb);
        __syncwarp();
        for (int j = lane; j < nbk; j += 32) {
            const int i = f0 + jb + j;
            sx[j] = tv.px[i] - cx;
            sy[j] = tv.py[i] - cy;
            sz[j] = tv.pz[i] - cz;
        }
        double acc[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
        if (DO_L2P) far_l2p<P>(g, nbk, sx, sy, sz, inv, srec, lane, acc);
        const int total = nbk * nw;
        for (int b0 = 0; b0 < total;) {
            const int end = far_round_end(b0, nbk, total, FAR_R);
            far_m2p_round<P, POT>(tv, hrec, w0, nbk, b0, end, sx, sy, sz, cx, cy, cz, srec, s_res[wid], lane, acc);
            b0 = end;
        }
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int j = lane + 32 * q;
            if (j < nbk) {
                double2* o = reinterpret_cast<double2*>(far + 4 * (size_t)(f0 + jb + j));
                o[0] = make_double2(acc[q][0], acc[q][1]);
                o[1] = make_double2(acc[q][2], acc[q][3]);
            }
        }
    }
}

// Heavy leaves have many bodies, so a round of 32 tasks rarely spans more than two W
// boxes: two records per warp halve the CTA's shared memory (three CTAs per SM fit)
constexpr int FAR_RH = 2;
template <int P>
constexpr int far_heavy_warp_f4() { return FAR_RH * 2 * FarRec32<P>::NEH; }
template <int P>
constexpr size_t far_heavy_smem_bytes() { return FAR_HW * sizeof(float4) * (size_t)far_heavy_warp_f4<P>(); }

// list of the leaves with more than FAR_HEAVY M2P tasks (order irrelevant:
// every leaf's result is computed independently); *count zero before the launch
__global__ void k_far_heavy_list(TreeView tv, int* __restrict__ list, int* count) {
    const int lf = blockIdx.x * blockDim.x + threadIdx.x;
    if (lf >= tv.nleaf || lf >= tv_nleaf(tv) || tv_over(tv)) return;
    if ((int64_t)tv.pcount[tv.leafbox[lf]] * (tv.w_off[lf + 1] - tv.w_off[lf]) > FAR_HEAVY) list[atomicAdd(count, 1)] = lf;
}

// Leaves with more than FAR_HEAVY M2P tasks: a CTA of FAR_HW warps per leaf,
// leaves taken from the heavy list through a shared counter (`ctr[1]`, zero
// before the launch; ctr[0] = list length) so the CTAs balance themselves.  Warp w runs the M2P rounds r = w, w + FAR_HW, ...;
// warp 0 also the L2P; the warps' per-body partial sums are added in warp order
// through shared memory (deterministic).
template <int P, bool POT, bool DO_L2P>
__global__ void __launch_bounds__(32 * FAR_HW, 3) k_leaf_far32_heavy(TreeView tv, const float4* __restrict__ hrec,
                                                                 const float4* __restrict__ grec, double* __restrict__ far,
                                                                 const int* __restrict__ list, int* ctr) {
    constexpr int NEG = FarRec32<P>::NEG;
    extern __shared__ float4 s_far_dyn[];
    __shared__ double s_pos[3][64];
    __shared__ float4 s_res[FAR_HW][32];
    __shared__ double s_part[FAR_HW][64][4];
    __shared__ int s_lf;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    float4* srec = s_far_dyn + (size_t)wid * far_heavy_warp_f4<P>();
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            const int k = atomicAdd(&ctr[1], 1);
            s_lf = (k < ctr[0]) ? list[k] : -1;
        }
        __syncthreads();
        const int lf = s_lf;
        if (lf < 0) return;
        const int b = tv.leafbox[lf];
        const int f0 = tv.pfirst[b], cnt = tv.pcount[b];
        const int64_t w0 = tv.w_off[lf];
        const int nw = (int)(tv.w_off[lf + 1] - w0);
        const double cx = tv.center[4 * b], cy = tv.center[4 * b + 1], cz = tv.center[4 * b + 2];
        const double inv = 1.0 / (2.0 * tv.center[4 * b + 3]);
        for (int jb = 0; jb < cnt; jb += 64) {
            const int nbk = min(64, cnt - jb);
            __syncthreads();
            for (int j = threadIdx.x; j < nbk; j += blockDim.x) {
                const int i = f0 + jb + j;
                s_pos[0][j] = tv.px[i] - cx;
                s_pos[1][j] = tv.py[i] - cy;
                s_pos[2][j] = tv.pz[i] - cz;
            }
            __syncthreads();
            double acc[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
            if (DO_L2P && wid == 0) far_l2p<P>(grec + (size_t)lf * 2 * NEG, nbk, s_pos[0], s_pos[1], s_pos[2], inv, srec, lane, acc);
            const int total = nbk * nw;
            int r = 0;
            for (int b0 = 0; b0 < total; ++r) {
                const int end = far_round_end(b0, nbk, total, FAR_RH);
                if (r % FAR_HW == wid)
                    far_m2p_round<P, POT>(tv, hrec, w0, nbk, b0, end, s_pos[0], s_pos[1], s_pos[2], cx, cy, cz, srec,
                                          s_res[wid], lane, acc);
                b0 = end;
            }
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int j = lane + 32 * q;
                if (j < nbk) {
                    s_part[wid][j][0] = acc[q][0]; s_part[wid][j][1] = acc[q][1];
                    s_part[wid][j][2] = acc[q][2]; s_part[wid][j][3] = acc[q][3];
                }
            }
            __syncthreads();
            for (int t = threadIdx.x; t < 4 * nbk; t += blockDim.x) {
                const int j = t >> 2, comp = t & 3;
                double v = 0.0;
#pragma unroll
                for (int w = 0; w < FAR_HW; ++w) v += s_part[w][j][comp];
                far[4 * (size_t)(f0 + jb + j) + comp] = v;
            }
        }
    }
}

// ---- P2L over X lists in FP32 (p <= 9) ------------------------------------------------
// L_b += sum over the X-list leaves c of b, bodies j of c: q_j S_n^m(x_j - c_b)
// (AdaptiveFMM3D::p2lAccum, src3d/AdaptiveFMM3D.hpp:117-128, scaled by side^n).
// Warp per box (one warp per block).  The bodies of all X-list leaves form one
// flat sequence; lane l takes positions l, l + 32, ... walking the entries on its
// own, so every lane evaluates a body each round however the leaves are sized.
// Each lane sums its K coefficients in registers (FP32); the 32 lane sums are
// added once per box through shared memory in FP64.
template <int P>
struct P2L32 {
    static constexpr int K = (P + 1) * (P + 1);
    static constexpr bool OK = K <= 100;   // register budget of the per-lane sums
};

template <int P>
__global__ void __launch_bounds__(32, 16) k_p2l32(TreeView tv, double* __restrict__ lown) {
    constexpr int K = (P + 1) * (P + 1);
    constexpr int LD = K | 1;
    constexpr int NPL = (K + 31) / 32;
    __shared__ float s_red[32 * LD];
    const int lane = threadIdx.x;
    const int b = blockIdx.x;
    if (b >= tv_nb(tv) || tv_over(tv)) return;
    const int64_t e0 = tv.x_off[b], e1 = tv.x_off[b + 1];
    if (e0 == e1) return;
    const double cx = tv.center[4 * b], cy = tv.center[4 * b + 1], cz = tv.center[4 * b + 2];
    const double inv = 1.0 / (2.0 * tv.center[4 * b + 3]);
    float acc[K];
#pragma unroll
    for (int d = 0; d < K; ++d) acc[d] = 0.f;
    int64_t e = e0;
    int c = tv.x_idx[e];
    int f0 = tv.pfirst[c], cnt = tv.pcount[c];
    int j = lane;
    for (;;) {
        while (e < e1 && j >= cnt) {
            j -= cnt;
            if (++e < e1) {
                c = tv.x_idx[e];
                f0 = tv.pfirst[c];
                cnt = tv.pcount[c];
            }
        }
        const bool act = e < e1;
        if (!__any_sync(0xffffffffu, act)) break;
        if (act) {
            const int i = f0 + j;
            const float q = (float)tv.pm[i];
            const float ux = (float)((tv.px[i] - cx) * inv), uy = (float)((tv.py[i] - cy) * inv),
                        uz = (float)((tv.pz[i] - cz) * inv);
            for_singular<P>(ux, uy, uz, [&](int n, int m, float re, float im) {
                const int dr = dof_re(n, m);
                acc[dr] = fmaf(q, re, acc[dr]);
                if (m > 0) acc[dr + 1] = fmaf(-q, im, acc[dr + 1]);
            });
        }
        j += 32;
    }
#pragma unroll
    for (int d = 0; d < K; ++d) s_red[lane * LD + d] = acc[d];
    __syncwarp();
#pragma unroll
    for (int q = 0; q < NPL; ++q) {
        const int d = lane + 32 * q;
        if (d < K) {
            double sum = 0.0;
#pragma unroll 8
            for (int r = 0; r < 32; ++r) sum += (double)s_red[r * LD + d];
            lown[(size_t)b * K + d] += sum * inv;
        }
    }
}

}  // namespace mixed
}  // namespace ogx
