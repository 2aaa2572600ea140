// ogx_internal.cuh -- shared declarations of the B200 adaptive-FMM library.
//
// Data layout in HBM (one handle, one system):
//   bodies   : original order pos (n x 3 f64, caller's Vec3 AoS), mass (n f64)
//              sorted order px/py/pz/m (SoA f64), perm (sorted -> original)
//   keys     : 72-bit octant path (24 levels x 3 bits) as (hi u64: levels 1..21,
//              lo u32: levels 22..24), the exact octant tests of
//              AdaptiveOctree::subdivide (src3d/AdaptiveOctree.hpp:109-127)
//   boxes    : level-major, Morton order within a level; per box level, int
//              coords, FP64 centre/half (same arithmetic as the reference),
//              parent, child[8], leaf id, pfirst/pcount, colleague[27] by
//              relative offset slot (dx+1)+3(dy+1)+9(dz+1)
//   lists    : U, W per leaf and X per box as CSR; V is implicit in the
//              colleague slots (children of the parent's colleagues)
//   expansions: scaled real coefficients, K = (p+1)^2 doubles per box:
//              dof(n,0)=n^2, dof(n,m>0)=n^2+2m-1 (re), n^2+2m (im);
//              M'_n = M_n / side^n, L'_n = L_n * side^n, so every translation
//              operator is a level-independent K x K matrix.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ogx.h"

namespace ogx {

constexpr int kMaxDepth = 24;     // AdaptiveOctree::maxDepth (src3d/AdaptiveOctree.hpp:49)
constexpr int kHiLevels = 21;     // levels packed in the 64-bit key word
constexpr int kPMax = 12;         // largest supported expansion order
constexpr int kDegMax = kPMax + 2;

inline int num_dofs(int p) { return (p + 1) * (p + 1); }

// ---- error plumbing ------------------------------------------------------
struct Error {
    int code;
    std::string msg;
};

#define OGX_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t e__ = (call);                                                        \
        if (e__ != cudaSuccess) {                                                        \
            ::ogx::set_last_error(OGX_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e__)); \
            return (e__ == cudaErrorMemoryAllocation) ? OGX_ERR_OOM : OGX_ERR_CUDA;      \
        }                                                                                \
    } while (0)

#define OGX_TRY(expr)                \
    do {                             \
        int s__ = (expr);            \
        if (s__ != OGX_OK) return s__; \
    } while (0)

void set_last_error(int code, const std::string& msg);

// ---- device buffer arena: grow-only named slots -----------------------------
enum Slot {
    S_POS, S_MASS, S_ACC, S_POT, S_VEL, S_ACC_OLD,
    S_BBOX, S_ROOT, S_KHI, S_KLO, S_IDX, S_KHI2, S_KLO2, S_IDX2,
    S_RS_HIST, S_TOPO_D, S_TOPO_CPL, S_TOPO_L, S_TOPO_CNT, S_TOPO_COFF, S_TOPO_LEAFSCAN,
    S_LEAFSTART, S_REC_KEY, S_REC_POS, S_REC_KEY2, S_REC_POS2, S_COUNTS,
    S_LEAFKEY, S_LEAFKEY2, S_PERM, S_PERM2,
    S_PX, S_PY, S_PZ, S_PM,
    S_BOX_LEVEL, S_BOX_POS, S_BOX_COORD, S_BOX_CENTER, S_BOX_PARENT, S_BOX_CHILD, S_BOX_LEAFID,
    S_BOX_PFIRST, S_BOX_PCOUNT, S_BOX_COL, S_LEAF_BOX,
    S_U_CNT, S_W_CNT, S_U_OFF, S_W_OFF, S_U_IDX, S_W_IDX,
    S_X_KEY, S_X_VAL, S_X_KEY2, S_X_VAL2, S_X_OFF, S_X_IDX, S_X_CNT, S_PERM_FINAL,
    S_TGT_KEY, S_TGT_BOX, S_TGT_KEY2, S_TGT_BOX2, S_TGT_TILE, S_TGT_PKEY, S_TGT_PBOX,
    S_MPOLE, S_LOCAL, S_LOWN, S_FAR, S_FAR_M, S_NEAR, S_SCAN_TMP,
    S_OPS_M2L, S_OPS_M2M, S_OPS_L2L,
    S_MIX_POS4, S_MIX_MHI, S_MIX_MLO, S_MIX_MUNSCALE, S_MIX_OUNSCALE, S_MIX_TOPS, S_MIX_LOWN, S_MIX_ROW0, S_ERR, S_EVAL_H, S_EVAL_G, S_UW_LANE,
    S_NONLEAF_FLAG, S_NONLEAF_OFF, S_NONLEAF, S_NONLEAF_LOFF, S_FAR_HEAVY,
    S_NEAR32, S_SPECIES, S_DIAG_POT, S_DIAG_ACC, S_DIAG_PART, S_FRAME, S_IC_POS, S_IC_MASS, S_IC_ACC,
    S_ROT_PACK, S_TR_READY_M, S_TR_READY_L, S_SOFT_CNT, S_SOFT_OFF, S_SOFT_IDX, S_NEAR_CHUNK, S_NEAR_CHUNK_OFF,
    S_NUM_SLOTS
};

struct Arena {
    void* ptr[S_NUM_SLOTS] = {};
    size_t cap[S_NUM_SLOTS] = {};
    size_t total = 0;
    uint64_t generation = 0;   // bumped by every (re)allocation: a captured step's buffers moved
    bool frozen = false;       // while a step is captured: growing a slot is an error
    int get(Slot s, size_t bytes, void** out);
    void release();
};

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) once per (kernel, device) and size
// in this process, not before every launch: the call costs host time, and a loop of
// short launches (one per tree level) then waits on the host.
inline cudaError_t smem_optin(const void* func, int bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    int& cur = done[{func, dev}];
    if (cur >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) cur = bytes;
    return e;
}

// Host-to-device copy of set-up data (operator tables) that has landed when this
// returns.  cudaMemcpy from pageable host memory returns once the data is staged,
// with the DMA still queued on the legacy stream, and the library's kernels run on
// non-blocking streams that are not ordered after it; the synchronize closes that
// window (it showed when several handles shared the copy engines).
inline cudaError_t upload_now(void* dst, const void* src, size_t bytes) {
    cudaError_t e = cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
    return e;
}

template <class T>
inline int arena_get(Arena& a, Slot s, size_t count, T** out) {
    void* p = nullptr;
    int rc = a.get(s, count * sizeof(T) + 16, &p);
    *out = (T*)p;
    return rc;
}

// ---- root box of the octree (AdaptiveOctree::build, src3d/AdaptiveOctree.hpp:71-81)
struct RootInfo {
    double c[3];
    double half;
    double tol;
    int leps;   // first level whose box edge 2*half <= eps floor (kMaxDepth+1 if none)
    int pad;
};

// Counts produced on the device.  An eager evaluation reads them back at two host sync
// points (box count, list sizes) to size what follows; an evaluation in capacity mode
// (no read-back, so a step can be captured as a CUDA graph) sizes its launches and
// buffers from capacities instead, and every kernel takes its bounds from these device
// counts.  `overflow` is set when a count exceeds its capacity: every later kernel of the
// evaluation then does nothing and the host redoes the evaluation eagerly.
struct DevCounts {
    int64_t num_boxes;
    int64_t num_leaves;
    int32_t level_hist[kMaxDepth + 2];  // boxes per level (difference form before finalise)
    int32_t max_level;
    int32_t max_leaf_occ;
    int64_t u_total, w_total;
    int64_t p2p_pairs, m2p_evals, p2l_evals;
    int64_t adj_mismatch;
    int64_t v_total;
    int32_t kernel_error;  // set by kernels whose bounded waits ran out
    int32_t pad_err;       // zero: the bounded-wait probe's flag that nothing sets
    int32_t nonleaf_level[kMaxDepth + 2];
    int32_t deep_flag;   // some level-16 box holds more than leaf_capacity bodies
    int32_t overflow;    // capacity mode: a count above its capacity (see above)
    int32_t nb32, nleaf32;   // num_boxes, num_leaves
    int32_t ntgt32;          // M2L targets (boxes of level >= 2)
    int32_t pad_cnt;
};

// device view of the tree handed to kernels.  nb and nleaf size the launches (the exact
// counts in an eager evaluation, the capacities in capacity mode); kernels bound their
// work by the device counts in `cnt` (tv_nb, tv_nleaf), which are always exact.
struct TreeView {
    int n, nb, nleaf;
    const DevCounts* cnt;
    const RootInfo* root;
    const double *px, *py, *pz, *pm;   // sorted bodies
    const int* perm;                   // sorted -> original
    const int* level;                  // per box
    const int* coord;                  // per box: ix, iy, iz (3 ints)
    const double* center;              // per box: cx, cy, cz, half
    const int* parent;
    const int* child;                  // 8 per box
    const int* leafid;                 // per box, -1 if not leaf
    const int* pfirst;
    const int* pcount;
    const int* col;                    // 27 per box
    const int* leafbox;                // per leaf
    const int64_t *u_off, *w_off;      // per leaf (nleaf+1)
    const int *u_idx, *w_idx;
    const int64_t* x_off;              // per box (nb+1)
    const int* x_idx;
    // OGX_SOFT_SPLINE: per leaf, the leaves that are not adjacent to it (so the far field
    // takes their pairs) but lie within the spline's support of it (nleaf+1 offsets)
    const int64_t* s_off;
    const int* s_idx;
};

#ifdef __CUDACC__
__device__ __forceinline__ int tv_nb(const TreeView& tv) { return tv.cnt->nb32; }
__device__ __forceinline__ int tv_nleaf(const TreeView& tv) { return tv.cnt->nleaf32; }
__device__ __forceinline__ bool tv_over(const TreeView& tv) { return tv.cnt->overflow != 0; }
#endif

// launch sizes of an evaluation in capacity mode, from an earlier eager evaluation
struct Capacity {
    int nb = 0, nleaf = 0;
    int levels = 0;          // tree levels 0 .. levels-1 are walked by the translations
    int level_boxes[kMaxDepth + 2] = {};   // boxes per level (sizes the translations' grids)
    int64_t u = 0, w = 0;    // U- and W-list entries
    bool full_sort = false;  // sort all 24 key levels (the tree had a deep cluster)
    bool valid = false;
};

struct Handle {
    ogx_params prm{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int device = 0;
    int num_sms = 148;
    Arena ws;
    DevCounts* h_counts = nullptr;  // pinned
    int64_t n_cap_host = 0;
    double* h_stage = nullptr;      // pinned staging for host-buffer calls
    size_t h_stage_cap = 0;
    ogx_stats stats{};
    int64_t launches = 0;            // kernels launched by this handle (running total)
    std::vector<int32_t> level_off;  // host copy of level offsets (num levels + 1)
    int max_level = 0;
    int64_t n = 0;
    // operator tables for prm.p (host built, device resident)
    int ops_p = -1;
    double* d_m2l = nullptr;  // 343 x K x K
    double* d_m2m = nullptr;  // 8 x K x K
    double* d_l2l = nullptr;  // 8 x K x K
    // device-resident integrator state
    bool resident = false;
    bool species_set = false;       // species tags uploaded (or made by ogx_ic_merger)
    cudaEvent_t ev[14] = {};
    // side stream for work that overlaps the main chain (joined back before returning)
    // internal streams: the evaluation runs on `main` (highest priority), forked
    // from and joined back to the caller's stream; overlapping work goes to `side`
    // (lowest priority) so it only fills SMs the main chain leaves idle
    cudaStream_t main = nullptr, side = nullptr, up = nullptr;
    cudaStream_t aux = nullptr;                  // M2L target tiles, beside the U/W list passes
    // mixed form: the tensor-core M2L (middle priority), launched once the multipoles and
    // target tiles are ready, beside the rest of the list build
    cudaStream_t m2l = nullptr;
    cudaEvent_t ev_col = nullptr, ev_tgt = nullptr, ev_m2l = nullptr;
    // host-buffer evaluation: the masses' copy runs on `aux` beside the start of the tree
    // build, which waits for it (ev_mass) before the sorted-body gather
    cudaEvent_t ev_mass = nullptr, ev_pos = nullptr;
    bool mass_pending = false;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_in = nullptr, ev_out = nullptr, ev_tree = nullptr, ev_up = nullptr;
    cudaEvent_t ev_up_end = nullptr;   // timing: end of an upward pass that ran on `up`
    bool upward_split = false;         // the last evaluation ran its upward pass on `up`
    int64_t soft_pairs = 0;            // OGX_SOFT_SPLINE: S-list entries of the last evaluation
    TreeView tv{};
    bool tree_valid = false;
    // mixed-precision tables
    int mix_ready_p = -1;
    int rot_ready_p = -1;          // order of the rotation-M2L factors in d_rot
    double* d_rot = nullptr;       // rotation-M2L factors, 343 packs (build_rot_pack)
    uint8_t* d_tc_img = nullptr;   // tensor-core M2L operator images (hi/lo)
    double* d_tc_row0 = nullptr;   // row 0 of every M2L operator
    float* d_tc_ounscale = nullptr; // per M2L operator: 2^e undoing the scaling of its FP16 images
    int* d_err = nullptr;          // device error word of the bounded waits
    int* h_err = nullptr;          // pinned copy
    // capacity mode and the captured step (ogx_step with step capture on)
    bool cap_mode = false;        // this evaluation sizes its launches from `cap`
    bool full_sort_used = false;  // the last tree build sorted all 24 key levels
    Capacity cap;
    bool capture_steps = false;   // ogx_set_tuning: replay each step as a CUDA graph
    bool capturing = false;       // a capture is being recorded on h.stream
    int cap_warm = 0;             // capacity-mode steps run since `cap` was set
    cudaGraph_t step_graph = nullptr;
    cudaGraphExec_t step_exec = nullptr;
    int64_t step_launches = 0;    // kernels in one captured step
    uint64_t step_gen = 0;        // arena generation the captured step was recorded with
    int64_t overflow_redos = 0;   // steps redone eagerly after an overflow
    int64_t graph_steps = 0;      // steps replayed from the captured graph
    // the captured host-buffer evaluation (ogx_eval with step capture on and page-locked
    // buffers): copies in, evaluation, copies out, for the buffers it was captured with
    struct EvalKey {
        int64_t n = -1;
        const void *pos = nullptr, *mass = nullptr;
        void *acc = nullptr, *pot = nullptr;
        bool operator==(const EvalKey& o) const {
            return n == o.n && pos == o.pos && mass == o.mass && acc == o.acc && pot == o.pot;
        }
    };
    cudaGraph_t eval_graph = nullptr;
    cudaGraphExec_t eval_exec = nullptr;
    EvalKey eval_key;
    uint64_t eval_gen = 0;
    int eval_warm = 0;
    int64_t eval_launches = 0;
    int64_t graph_evals = 0;      // host-buffer evaluations replayed from the captured graph
    DevCounts* d_counts = nullptr;   // the counts of the last evaluation (device)
    int* d_level_off = nullptr;      // first box of every level (device, kMaxDepth + 2)
    // launch-shape knobs (ogx_set_tuning)
    int tile_fill = 128;    // targets per 128-row M2L tile
    int near_units = 64;    // (target, source part) units per near-field chunk
    // M2L targets (levels >= 2) sorted by child octant
    int ntgt = 0;
    const uint32_t* tgt_key = nullptr;
    const uint32_t* tgt_box = nullptr;
    int ntgt_pad = 0;                     // padded per-octant layout, 64 per tile
    const uint32_t* tgt_tile_key = nullptr;
    const uint32_t* tgt_tile_box = nullptr;
    // non-leaf boxes, level-major (M2M / L2L parents); nonleaf_off[l] = first of level l
    const int* d_nonleaf = nullptr;
    const int* d_nonleaf_off = nullptr;   // device, kMaxDepth + 2 entries
};

// A timing event of the evaluation.  While a step is being captured as a CUDA graph
// the record must become an event-record node of the graph (cudaEventRecordExternal);
// a plain record on a capturing stream would only mark a capture dependency.
inline cudaError_t timing_record(const Handle& h, cudaEvent_t e, cudaStream_t st) {
    return cudaEventRecordWithFlags(e, st, h.capturing ? cudaEventRecordExternal : cudaEventRecordDefault);
}

// ---- host-side operator tables (ogx_tables.cpp) -----------------------------
// kind 0: M2M for child octant index (0..7), maps child M' -> parent M'
// kind 1: L2L for child octant index (0..7), maps parent L' -> child L'
// kind 2: M2L for offset index (ox+3)+7(oy+3)+49(oz+3), source minus target in
//         units of the box side; maps source M' -> target L' * side
void build_operator(int kind, int p, int index, double* out /* K*K row-major */);
void build_m2l_offset(int p, long double ox, long double oy, long double oz, double* out /* K*K */);
// rotation-based M2L factors of V offset `index` (ogx_tables.cpp)
int rot_pack_size(int p);
bool build_rot_pack(int p, int index, double* out /* rot_pack_size(p) */);

// ---- phases (defined in the .cu files) -------------------------------------
int tree_build(Handle& h, const double* d_pos, const double* d_mass, int64_t n);
int lists_build(Handle& h);           // both parts below, in order
int lists_build_targets(Handle& h);   // colleagues; M2L target tiles on `aux`
int lists_build_uwx(Handle& h);       // U, W and X lists
int soft_lists_build(Handle& h);      // OGX_SOFT_SPLINE: the leaf pairs the far field takes within the support
int soft_correct_launch(Handle& h, const int64_t* chunk_off, double* out, bool pot, cudaStream_t st);   // FP64: adds the kernel difference over them
int fmm_fp64(Handle& h, double* d_acc, double* d_pot);
int fmm_mixed(Handle& h, double* d_acc, double* d_pot);
int m2l_rot_launch(Handle& h, const double* M, double* Lown);   // third form's M2L, on h.stream
int fmm_mixed_upward(Handle& h);   // upward pass on h.up, right after the tree (before the lists)
int fmm_mixed_m2l(Handle& h, bool pot);   // tensor-core M2L on h.m2l, after the target tiles
int flag_wait_probe(Handle& h, uint32_t polls, const int* flag, int* err);   // translation passes' wait, run out
int direct_eval(Handle& h, const double* d_pos, const double* d_mass, int64_t n, double* d_acc,
                double* d_pot, bool fp32);
int ensure_operator_tables(Handle& h);
void drop_step_graph(Handle& h);   // ogx_api.cu
int eval_device_shared(Handle& h, int64_t n, const double* d_pos, const double* d_mass, double* d_acc, double* d_pot);
void finish_stats_shared(Handle& h);
int direct_launch(const double* d_pos, const double* d_mass, int64_t n, double G, double eps2, double* d_acc, double* d_pot,
                  cudaStream_t st);

// generic radix sort helpers (ogx_sort.cu)
int radix_sort_u32(Handle& h, Slot kin, Slot vin, Slot kalt, Slot valt, int64_t n, int bits,
                   uint32_t** kout, uint32_t** vout);
// stable LSD sort of the 72-bit keys over digit passes first_pass..8 (first_pass 3 orders
// by levels 1..16 only)
int radix_sort_key72(Handle& h, int64_t n, int first_pass, uint64_t** khi, uint32_t** klo, uint32_t** idx);
int scan_i32_to_i64(Handle& h, const int* in, int64_t* out, int64_t n);  // exclusive, out[n] = total

}  // namespace ogx
