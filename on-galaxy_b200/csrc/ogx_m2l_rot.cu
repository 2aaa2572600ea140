// ogx_m2l_rot.cu -- the third form's M2L: every operator factored into rotations.
//
// The reference applies each M2L with the dense O(p^4) formulas (fmm::M2L,
// src3d/FmmExpansions3D.hpp:273-300) and defers an O(p^3) rotation scheme (its
// README.md:75).  Here T_o = Q_o^-1 Z_|o| Q_o (factors from build_rot_pack in
// ogx_tables.cpp), applied tile by tile over the same target tiles and (colleague
// slot, child) combinations as the plain form's k_m2l_fp64.  Kept in a file of its
// own: the fully unrolled blocks of twelve orders take minutes to compile, and the
// build then runs it beside the other units.
#include <memory>
#include <mutex>
#include <utility>
#include <vector>

#include "ogx_internal.cuh"

namespace ogx {
namespace {

// targets per CTA; the target tiles are padded to multiples of 128, so 64 divides them
constexpr int ROT_TGT = 64;

// ---- M2L by rotations (the third form) ------------------------------------------------
// T_o = Q_o^-1 Z_|o| Q_o (build_rot_pack): per tile of ROT_TGT targets sharing octant t
// and per present (D, s) combination (offset o) the 64 source multipoles are staged,
// then y = Q_o m (degree blocks) -> z = Z_|o| y (order blocks) -> acc += Q_o^-1 z
// (degree blocks), the last sums kept in registers over all combinations.
// Thread (g, a) = (tid / 64, tid % 64) owns source / target row a and, in each stage, a
// fixed set of blocks: the four groups g take the blocks in snake order of size
// (largest to g = 0, 1, 2, 3, 3, 2, 1, 0, 0, ...), so they carry about equal work.  A
// block runs fully unrolled: its inputs sit in registers and its outputs are
// independent FMA chains, so a thread keeps up to 2p + 1 of them in flight.  The
// factors are read with warp-uniform addresses (every lane of a warp is in the same
// block).  FP64 throughout.
template <int P>
struct RotCfg {
    static constexpr int K = (P + 1) * (P + 1);
    static constexpr int LD = K | 1;
    static constexpr int QSZ = (P + 1) * (2 * P + 1) * (2 * P + 3) / 3;   // sum_n (2n+1)^2
    static constexpr int ZSZ = (P + 1) * (P + 2) * (2 * P + 3) / 6;       // sum_m (P+1-m)^2
    static constexpr int PACK = 2 * QSZ + ZSZ;
    static constexpr size_t SMEM = (size_t)2 * ROT_TGT * LD * sizeof(double);
    // rows per thread: each factor entry loaded feeds RB FMAs (2 where the registers allow)
    static constexpr int RB = P <= 10 ? 2 : 1;
    static constexpr int ROWS = ROT_TGT / RB;          // threads of one block group
    static constexpr int THREADS = 4 * ROWS;
    static constexpr int snake(int i) { return ((i / 4) % 2 == 0) ? i % 4 : 3 - i % 4; }
    // degree blocks: block n has 2n+1 rows; the i-th largest is n = P - i
    static constexpr int deg_group(int n) { return snake(P - n); }
    // position of block n's rows in its group's accumulators (blocks taken largest first)
    static constexpr int deg_pos(int n) {
        int pos = 0;
        for (int q = P; q > n; --q)
            if (deg_group(q) == deg_group(n)) pos += 2 * q + 1;
        return pos;
    }
    static constexpr int group_rows(int g) {
        int r = 0;
        for (int n = 0; n <= P; ++n)
            if (deg_group(n) == g) r += 2 * n + 1;
        return r;
    }
    static constexpr int NACC = group_rows(0) > group_rows(1) ? (group_rows(0) > group_rows(2) ? (group_rows(0) > group_rows(3) ? group_rows(0) : group_rows(3)) : (group_rows(2) > group_rows(3) ? group_rows(2) : group_rows(3)))
                                                               : (group_rows(1) > group_rows(2) ? (group_rows(1) > group_rows(3) ? group_rows(1) : group_rows(3)) : (group_rows(2) > group_rows(3) ? group_rows(2) : group_rows(3)));
    // order blocks: block m has (P+1-m)^2 entries, applied to 1 (m = 0) or 2 (re, im) parts
    static constexpr int ord_work(int m) { return (P + 1 - m) * (P + 1 - m) * (m == 0 ? 1 : 2); }
    static constexpr int ord_group(int m) {
        int rank = 0;
        for (int q = 0; q <= P; ++q)
            if (ord_work(q) > ord_work(m) || (ord_work(q) == ord_work(m) && q < m)) ++rank;
        return snake(rank);
    }
};

// stage A (FWD) or C (!FWD) for degree block N: rows N^2 .. N^2 + 2N of source a
template <int P, int N, bool FWD>
__device__ __forceinline__ void rot_deg_block(const double* __restrict__ F, const double* x_in, double* y_out,
                                              double (&acc)[RotCfg<P>::RB][RotCfg<P>::NACC]) {
    constexpr int w = 2 * N + 1, off = N * (2 * N - 1) * (2 * N + 1) / 3, pos = RotCfg<P>::deg_pos(N);
    constexpr int RB = RotCfg<P>::RB, RS = RotCfg<P>::ROWS * RotCfg<P>::LD;   // row stride of the RB rows
    double x[RB][w];
#pragma unroll
    for (int q = 0; q < RB; ++q)
#pragma unroll
        for (int c = 0; c < w; ++c) x[q][c] = x_in[q * RS + N * N + c];
#pragma unroll
    for (int r = 0; r < w; ++r) {
        double v[RB];
#pragma unroll
        for (int q = 0; q < RB; ++q) v[q] = FWD ? 0.0 : acc[q][pos + r];
#pragma unroll
        for (int c = 0; c < w; ++c) {
            const double f = __ldg(F + off + r * w + c);
#pragma unroll
            for (int q = 0; q < RB; ++q) v[q] = fma(f, x[q][c], v[q]);
        }
#pragma unroll
        for (int q = 0; q < RB; ++q) {
            if (FWD) y_out[q * RS + N * N + r] = v[q];
            else acc[q][pos + r] = v[q];
        }
    }
}

// stage B for order block M: z = Z_M y over degrees M..P, re and im parts
template <int P, int M>
__device__ __forceinline__ void rot_ord_block(const double* __restrict__ Z, const double* y_in, double* z_out) {
    constexpr int L = P + 1 - M;
    constexpr int zoff = RotCfg<P>::ZSZ - L * (L + 1) * (2 * L + 1) / 6;
    constexpr int NP = M == 0 ? 1 : 2;                      // parts re, im: same block
    constexpr int RB = RotCfg<P>::RB, RS = RotCfg<P>::ROWS * RotCfg<P>::LD;
    double yv[RB * NP][L];
#pragma unroll
    for (int q = 0; q < RB * NP; ++q)
#pragma unroll
        for (int d = 0; d < L; ++d) {
            const int n = M + d, part = q % NP;
            yv[q][d] = y_in[(q / NP) * RS + (M == 0 ? n * n : n * n + 2 * M - 1 + part)];
        }
#pragma unroll
    for (int jr = 0; jr < L; ++jr) {
        double v[RB * NP];
#pragma unroll
        for (int q = 0; q < RB * NP; ++q) v[q] = 0.0;
#pragma unroll
        for (int d = 0; d < L; ++d) {
            const double f = __ldg(Z + zoff + jr * L + d);
#pragma unroll
            for (int q = 0; q < RB * NP; ++q) v[q] = fma(f, yv[q][d], v[q]);
        }
        const int j = M + jr;
#pragma unroll
        for (int q = 0; q < RB * NP; ++q)
            z_out[(q / NP) * RS + (M == 0 ? j * j : j * j + 2 * M - 1 + q % NP)] = v[q];
    }
}

template <int P, bool FWD, int... Ns>
__device__ __forceinline__ void rot_deg_stage(std::integer_sequence<int, Ns...>, int g, const double* F, const double* x_in,
                                              double* y_out, double (&acc)[RotCfg<P>::RB][RotCfg<P>::NACC]) {
    // largest blocks first, matching deg_pos
    ((RotCfg<P>::deg_group(P - Ns) == g ? rot_deg_block<P, P - Ns, FWD>(F, x_in, y_out, acc) : void()), ...);
}
template <int P, int... Ms>
__device__ __forceinline__ void rot_ord_stage(std::integer_sequence<int, Ms...>, int g, const double* Z, const double* y_in,
                                              double* z_out) {
    ((RotCfg<P>::ord_group(Ms) == g ? rot_ord_block<P, Ms>(Z, y_in, z_out) : void()), ...);
}

template <int P>
__global__ void __launch_bounds__(RotCfg<P>::THREADS) k_m2l_rot(TreeView tv, const uint32_t* tgt_key, const uint32_t* tgt_box,
                                                        const double* __restrict__ pack, const double* __restrict__ mpole,
                                                        double* lown) {
    using R = RotCfg<P>;
    constexpr int K = R::K, LD = R::LD, RB = R::RB, TH = R::THREADS;
    extern __shared__ double s_rot[];
    double* s_m = s_rot;                    // [64][LD] sources, later z
    double* s_y = s_rot + ROT_TGT * LD;     // [64][LD] y = Q m
    __shared__ int s_pcol[ROT_TGT][27];
    __shared__ int s_src[ROT_TGT];
    __shared__ int s_tgt[ROT_TGT];
    __shared__ int s_t;
    const int tid = threadIdx.x;
    const int ga = tid / R::ROWS, ra = tid % R::ROWS;   // block group; rows ra, ra + ROWS, ...
    const int base = blockIdx.x * ROT_TGT;
    if (tv_over(tv)) return;
    if (tid == 0) s_t = (tgt_key[base] == 0xFFFFFFFFu) ? -1 : (int)tgt_key[base];
    __syncthreads();
    const int t = s_t;
    if (t < 0) return;
    if (tid < ROT_TGT) {
        const int i = base + tid;
        const int b = ((int)tgt_key[i] == t) ? (int)tgt_box[i] : -1;
        s_tgt[tid] = b;
        const int P_ = (b >= 0) ? tv.parent[b] : -1;
        for (int d = 0; d < 27; ++d) s_pcol[tid][d] = (P_ >= 0) ? tv.col[27 * P_ + d] : -1;
    }
    __syncthreads();
    const int tx = t & 1, ty = (t >> 1) & 1, tz = (t >> 2) & 1;
    double acc[RB][R::NACC];
#pragma unroll
    for (int q = 0; q < RB; ++q)
#pragma unroll
        for (int i = 0; i < R::NACC; ++i) acc[q][i] = 0.0;
    using Seq = std::make_integer_sequence<int, P + 1>;
    for (int D = 0; D < 27; ++D) {
        const int Dx = D % 3 - 1, Dy = (D / 3) % 3 - 1, Dz = D / 9 - 1;
        for (int s = 0; s < 8; ++s) {
            const int ox = 2 * Dx + (s & 1) - tx, oy = 2 * Dy + ((s >> 1) & 1) - ty, oz = 2 * Dz + ((s >> 2) & 1) - tz;
            if (max(abs(ox), max(abs(oy), abs(oz))) <= 1) continue;  // adjacent: not in V
            int mysrc = -1;
            if (tid < ROT_TGT) {
                const int Q = s_pcol[tid][D];
                mysrc = (Q >= 0) ? tv.child[8 * Q + s] : -1;
                s_src[tid] = mysrc;
            }
            if (!__syncthreads_or(mysrc >= 0)) continue;
            for (int idx = tid; idx < ROT_TGT * K; idx += TH) {
                const int r = idx / K, kk = idx - r * K;
                const int src = s_src[r];
                s_m[r * LD + kk] = (src >= 0) ? mpole[(size_t)src * K + kk] : 0.0;
            }
            __syncthreads();
            const double* pk = pack + (size_t)((ox + 3) + 7 * (oy + 3) + 49 * (oz + 3)) * R::PACK;
            rot_deg_stage<P, true>(Seq{}, ga, pk, s_m + ra * LD, s_y + ra * LD, acc);              // y = Q m
            __syncthreads();
            rot_ord_stage<P>(Seq{}, ga, pk + 2 * R::QSZ, s_y + ra * LD, s_m + ra * LD);            // z = Z y
            __syncthreads();
            rot_deg_stage<P, false>(Seq{}, ga, pk + R::QSZ, s_m + ra * LD, nullptr, acc);          // acc += Q^-1 z
            __syncthreads();
        }
    }
#pragma unroll
    for (int q = 0; q < RB; ++q) {
        const int b = s_tgt[ra + q * R::ROWS];
        if (b < 0) continue;
        const double inv = 1.0 / (2.0 * tv.center[4 * b + 3]);
#pragma unroll
        for (int n = 0; n <= P; ++n) {
            if (R::deg_group(n) != ga) continue;
            const int pos = R::deg_pos(n);
#pragma unroll
            for (int r = 0; r < 2 * n + 1; ++r) lown[(size_t)b * K + n * n + r] += acc[q][pos + r] * inv;
        }
    }
}

// the 343 rotation packs of order P, built once per order in this process
template <int P>
std::shared_ptr<const std::vector<double>> rot_packs() {
    static std::mutex mu;
    static std::shared_ptr<const std::vector<double>> cached;
    std::lock_guard<std::mutex> lk(mu);
    if (cached) return cached;
    auto v = std::make_shared<std::vector<double>>((size_t)343 * RotCfg<P>::PACK, 0.0);
    for (int o = 0; o < 343; ++o) build_rot_pack(P, o, v->data() + (size_t)o * RotCfg<P>::PACK);
    cached = v;
    return cached;
}

template <int P>
int ensure_rot_tables(Handle& h) {
    if (h.rot_ready_p == P) return OGX_OK;
    static_assert(RotCfg<P>::PACK > 0, "pack");
    const auto pk = rot_packs<P>();
    double* d;
    OGX_TRY(arena_get(h.ws, S_ROT_PACK, pk->size(), &d));
    OGX_CUDA(upload_now(d, pk->data(), pk->size() * sizeof(double)));
    h.d_rot = d;
    h.rot_ready_p = P;
    return OGX_OK;
}

template <int P>
int launch_rot(Handle& h, const double* M, double* Lown) {
    OGX_TRY(ensure_rot_tables<P>(h));
    constexpr size_t rsm = RotCfg<P>::SMEM;
    OGX_CUDA(smem_optin((const void*)k_m2l_rot<P>, (int)rsm));
    k_m2l_rot<P><<<h.ntgt_pad / ROT_TGT, RotCfg<P>::THREADS, rsm, h.stream>>>(h.tv, h.tgt_tile_key, h.tgt_tile_box,
                                                                               h.d_rot, M, Lown);
    ++h.launches;
    OGX_CUDA(cudaGetLastError());
    return OGX_OK;
}

}  // namespace

int m2l_rot_launch(Handle& h, const double* M, double* Lown) {
    switch (h.prm.p) {
        case 1: return launch_rot<1>(h, M, Lown);
        case 2: return launch_rot<2>(h, M, Lown);
        case 3: return launch_rot<3>(h, M, Lown);
        case 4: return launch_rot<4>(h, M, Lown);
        case 5: return launch_rot<5>(h, M, Lown);
        case 6: return launch_rot<6>(h, M, Lown);
        case 7: return launch_rot<7>(h, M, Lown);
        case 8: return launch_rot<8>(h, M, Lown);
        case 9: return launch_rot<9>(h, M, Lown);
        case 10: return launch_rot<10>(h, M, Lown);
        case 11: return launch_rot<11>(h, M, Lown);
        case 12: return launch_rot<12>(h, M, Lown);
        default: return OGX_ERR_INVALID;
    }
}

}  // namespace ogx
