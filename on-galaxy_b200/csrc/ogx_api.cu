// ogx_api.cu -- the C ABI (include/ogx.h) and the host runtime behind it.
//
// One handle = one solver instance on one device and stream, the C-level
// equivalent of constructing AdaptiveFMM3D / DirectSolver3D
// (src3d/AdaptiveFMM3D.hpp:22-23, src3d/DirectSolver3D.hpp:13).  The handle
// owns a grow-only arena of device buffers (reused across evaluations, so a
// steady-state step allocates nothing), pinned host buffers for the two
// per-evaluation read-backs of tree sizes, the level-independent operator
// matrices of its expansion order, and the device-resident integrator state.
// Errors are status codes; nothing throws or exits across the boundary
// (the reference exit()s on CUDA errors, src3d/gpu/AdaptiveFMM3DGPU.cu:23-26).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

#include "ogx_harmonics.cuh"
#include "ogx_sm100.cuh"

namespace ogx {

static thread_local std::string g_last_error;
void set_last_error(int, const std::string& msg) { g_last_error = msg; }

int Arena::get(Slot s, size_t bytes, void** out) {
    if (cap[s] < bytes) {
        if (frozen) {
            set_last_error(OGX_ERR_STATE, "a device buffer would grow while a step is captured");
            return OGX_ERR_STATE;
        }
        ++generation;
        if (ptr[s]) {
            cudaFree(ptr[s]);
            total -= cap[s];
            ptr[s] = nullptr;
            cap[s] = 0;
        }
        size_t nb = bytes + bytes / 4;
        nb = (nb + 255) & ~(size_t)255;
        const cudaError_t e = cudaMalloc(&ptr[s], nb);
        if (e != cudaSuccess) {
            cudaGetLastError();
            ptr[s] = nullptr;
            set_last_error(OGX_ERR_OOM, "device allocation failed");
            return OGX_ERR_OOM;
        }
        cap[s] = nb;
        total += nb;
    }
    *out = ptr[s];
    return OGX_OK;
}

void Arena::release() {
    for (int s = 0; s < S_NUM_SLOTS; ++s) {
        if (ptr[s]) cudaFree(ptr[s]);
        ptr[s] = nullptr;
        cap[s] = 0;
    }
    total = 0;
}

// ---- operator tables: built once per order in this process, transposed k-major ----
struct HostOps {
    std::vector<double> m2l, m2m, l2l;
};
static std::mutex g_ops_mu;
static std::map<int, std::shared_ptr<HostOps>> g_ops;

static std::shared_ptr<HostOps> host_ops(int p) {
    std::lock_guard<std::mutex> lk(g_ops_mu);
    auto it = g_ops.find(p);
    if (it != g_ops.end()) return it->second;
    const int K = num_dofs(p);
    auto ops = std::make_shared<HostOps>();
    std::vector<double> tmp((size_t)K * K);
    auto put = [&](std::vector<double>& dst, int count, int kind) {
        dst.assign((size_t)count * K * K, 0.0);
        for (int idx = 0; idx < count; ++idx) {
            build_operator(kind, p, idx, tmp.data());
            double* o = dst.data() + (size_t)idx * K * K;
            for (int j = 0; j < K; ++j)
                for (int k = 0; k < K; ++k) o[(size_t)k * K + j] = tmp[(size_t)j * K + k];
        }
    };
    put(ops->m2m, 8, 0);
    put(ops->l2l, 8, 1);
    put(ops->m2l, 343, 2);
    g_ops[p] = ops;
    return ops;
}

int ensure_operator_tables(Handle& h) {
    if (h.ops_p == h.prm.p) return OGX_OK;
    auto ops = host_ops(h.prm.p);
    OGX_TRY(arena_get(h.ws, S_OPS_M2L, ops->m2l.size(), &h.d_m2l));
    OGX_TRY(arena_get(h.ws, S_OPS_M2M, ops->m2m.size(), &h.d_m2m));
    OGX_TRY(arena_get(h.ws, S_OPS_L2L, ops->l2l.size(), &h.d_l2l));
    OGX_CUDA(upload_now(h.d_m2l, ops->m2l.data(), ops->m2l.size() * sizeof(double)));
    OGX_CUDA(upload_now(h.d_m2m, ops->m2m.data(), ops->m2m.size() * sizeof(double)));
    OGX_CUDA(upload_now(h.d_l2l, ops->l2l.data(), ops->l2l.size() * sizeof(double)));
    h.ops_p = h.prm.p;
    return OGX_OK;
}

static std::mutex g_dev_mu;
static std::vector<int> g_dev_ready;

static int device_init(int dev) {
    std::lock_guard<std::mutex> lk(g_dev_mu);
    if ((int)g_dev_ready.size() <= dev) g_dev_ready.resize(dev + 1, 0);
    if (g_dev_ready[dev]) return OGX_OK;
    g_dev_ready[dev] = 1;
    return OGX_OK;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

static float ev_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
        cudaGetLastError();
        return 0.f;
    }
    return ms;
}

// ---- drift / kick of VelocityVerlet3D (src3d/Integrator3D.hpp:23-40) --------------------
__global__ void k_drift(double* pos, const double* vel, const double* acc, int64_t n3, double dt, double half_dt2) {
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n3) pos[i] += vel[i] * dt + acc[i] * half_dt2;
}
// v += (a_old + a_new) dt / 2, then a_old = a_new.  `counts` (capacity mode): a step
// whose evaluation overflowed its capacities leaves v and a_old untouched, so the host
// can redo the evaluation and the kick.
__global__ void k_kick(double* vel, double* acc_old, const double* acc_new, int64_t n3, double half_dt,
                       const DevCounts* counts) {
    if (counts && counts->overflow) return;
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < n3) {
        vel[i] += (acc_old[i] + acc_new[i]) * half_dt;
        acc_old[i] = acc_new[i];
    }
}

static int device_error(Handle& h);

static int eval_device_on(Handle& h, int64_t n, const double* d_pos, const double* d_mass, double* d_acc, double* d_pot);
static void counts_to_stats(Handle& h);

// Capacities for capacity mode from the counts an eager evaluation read back (box and
// leaf counts at sync point 1, list sizes at sync point 2): an eighth more, plus slack,
// so the small changes of a step's tree fit; one more tree level; the sort depth used.
static void update_capacity(Handle& h) {
    const DevCounts& c = *h.h_counts;
    Capacity& k = h.cap;
    const Capacity old = k;
    k.nb = (int)(c.num_boxes + c.num_boxes / 8 + 128);
    k.nleaf = (int)(c.num_leaves + c.num_leaves / 8 + 128);
    k.levels = std::min(kMaxDepth + 1, c.max_level + 2);
    for (int l = 0; l < kMaxDepth + 2; ++l) {
        const int b = (l <= c.max_level) ? c.level_hist[l] : (c.max_level >= 0 ? c.level_hist[c.max_level] : 0);
        k.level_boxes[l] = b + b / 8 + 8;
    }
    k.u = c.u_total + c.u_total / 8 + 4096;
    k.w = c.w_total + c.w_total / 8 + 4096;
    k.full_sort = h.full_sort_used;
    k.valid = true;
    // a captured step keeps the capacities it was captured with while its counts fit
    if (old.valid && h.step_exec && c.num_boxes <= old.nb && c.num_leaves <= old.nleaf && c.max_level + 1 <= old.levels &&
        c.u_total <= old.u && c.w_total <= old.w && (old.full_sort || !h.full_sort_used))
        k = old;
}

// Every evaluation runs on the handle's internal high-priority stream: ordered
// after the caller's stream's earlier work and before its later work.
static int eval_device(Handle& h, int64_t n, const double* d_pos, const double* d_mass, double* d_acc, double* d_pot) {
    const cudaStream_t user = h.stream;
    OGX_CUDA(cudaEventRecord(h.ev_in, user));
    OGX_CUDA(cudaStreamWaitEvent(h.main, h.ev_in, 0));
    h.stream = h.main;
    const int rc = eval_device_on(h, n, d_pos, d_mass, d_acc, d_pot);
    h.stream = user;
    OGX_CUDA(cudaEventRecord(h.ev_out, h.main));
    OGX_CUDA(cudaStreamWaitEvent(user, h.ev_out, 0));
    return rc;
}

static int eval_device_on(Handle& h, int64_t n, const double* d_pos, const double* d_mass, double* d_acc, double* d_pot) {
    h.n = n;
    h.tree_valid = false;
    std::memset(&h.stats, 0, sizeof(h.stats));
    h.stats.n = n;
    if (n == 0) return OGX_OK;
    const int64_t l0 = h.launches;
    OGX_TRY(device_error(h));
    const cudaStream_t st = h.stream;
    OGX_CUDA(timing_record(h, h.ev[0], st));
    if (h.prm.solver == OGX_SOLVER_DIRECT) {
        OGX_TRY(direct_eval(h, d_pos, d_mass, n, d_acc, d_pot, false));
        OGX_CUDA(timing_record(h, h.ev[8], st));
        h.stats.launches = h.launches - l0;
        return OGX_OK;
    }
    OGX_TRY(ensure_operator_tables(h));
    OGX_TRY(tree_build(h, d_pos, d_mass, n));
    OGX_CUDA(timing_record(h, h.ev[1], st));
    // mixed form: the upward pass needs only the tree, so it runs on its own stream
    // while the lists are built
    h.upward_split = (h.prm.precision == OGX_PREC_MIXED);
    if (h.upward_split) OGX_TRY(fmm_mixed_upward(h));
    OGX_TRY(lists_build_targets(h));
    // mixed form: the M2L needs the multipoles and the target tiles only, so it starts
    // beside the U/W/X list build
    if (h.prm.precision == OGX_PREC_MIXED) OGX_TRY(fmm_mixed_m2l(h, d_pot != nullptr));
    OGX_TRY(lists_build_uwx(h));
    h.soft_pairs = 0;
    if (h.prm.softening == OGX_SOFT_SPLINE && h.prm.eps > 0.0) {
        OGX_TRY(soft_lists_build(h));
        h.stats.list_s = h.soft_pairs;
    }
    OGX_CUDA(timing_record(h, h.ev[9], st));
    h.tree_valid = true;
    // an eager evaluation has read its counts back by now: capacities for capacity mode
    if (!h.cap_mode) update_capacity(h);
    if (h.prm.precision == OGX_PREC_MIXED) OGX_TRY(fmm_mixed(h, d_acc, d_pot));
    else OGX_TRY(fmm_fp64(h, d_acc, d_pot));   // the plain form, or with rotation-based M2L
    // every count of this evaluation (the overflow flag included) reaches the host with it,
    // and so does the error word of its bounded waits (tensor-core M2L, translation passes)
    OGX_CUDA(cudaMemcpyAsync(h.h_counts, h.d_counts, sizeof(DevCounts), cudaMemcpyDeviceToHost, st));
    OGX_CUDA(cudaMemcpyAsync(h.h_err, h.d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    OGX_CUDA(timing_record(h, h.ev[8], st));
    h.stats.launches = h.launches - l0;
    return OGX_OK;
}

// counts of the last evaluation (host copy, valid after a synchronize) into the stats
static void counts_to_stats(Handle& h) {
    const DevCounts& c = *h.h_counts;
    h.stats.num_boxes = (int32_t)c.num_boxes;
    h.stats.num_leaves = (int32_t)c.num_leaves;
    h.stats.max_leaf_occupancy = c.max_leaf_occ;
    h.stats.max_level = c.max_level;
    h.stats.list_u = c.u_total;
    h.stats.list_w = c.w_total;
    h.stats.list_x = c.w_total;
    h.stats.p2p_pairs = c.p2p_pairs;
    h.stats.m2p_evals = c.m2p_evals;
    h.stats.p2l_evals = c.p2l_evals;
    h.stats.adjacency_mismatch = c.adj_mismatch;
    h.stats.list_v = c.v_total;
}

// a bounded device wait that ran out in the previous evaluation (read after a sync)
static int device_error(Handle& h) {
    if (h.h_err && *h.h_err) {
        *h.h_err = 0;
        set_last_error(OGX_ERR_TIMEOUT, "a bounded device wait ran out (tensor-core M2L pipeline or a translation pass)");
        return OGX_ERR_TIMEOUT;
    }
    return OGX_OK;
}

// One thread waits, with the tensor-core pipeline's bounded wait and a limit of
// `polls`, for phase 0 of an mbarrier that expects one arrival that never comes:
// no copy and no MMA is outstanding, so the wait runs out and the error word is
// set exactly as the M2L kernel sets it.
__global__ void k_wait_probe(uint32_t polls, int* err) {
    __shared__ uint64_t bar;
    if (threadIdx.x != 0) return;
    sm100::mbar_init(&bar, 1);
    sm100::fence_mbar_init();
    if (!sm100::mbar_wait(&bar, 0, nullptr, polls)) atomicExch(err, 1);
}

static void finish_stats(Handle& h) {
    if (h.n == 0) return;
    if (cudaEventSynchronize(h.ev[8]) != cudaSuccess) { cudaGetLastError(); return; }
    ogx_stats& s = h.stats;
    s.ms_total = ev_ms(h.ev[0], h.ev[8]);
    if (h.prm.solver == OGX_SOLVER_DIRECT) return;
    counts_to_stats(h);
    s.ms_tree = ev_ms(h.ev[0], h.ev[1]);
    s.ms_lists = ev_ms(h.ev[1], h.ev[9]);
    s.ms_upward = ev_ms(h.ev[2], h.upward_split ? h.ev_up_end : h.ev[3]);
    s.ms_m2l = ev_ms(h.ev[3], h.ev[4]);
    s.ms_p2l = ev_ms(h.ev[4], h.ev[5]);
    s.ms_downward = ev_ms(h.ev[5], h.ev[6]);
    s.ms_leaf = ev_ms(h.ev[6], h.ev[7]);
}

// One leapfrog step (VelocityVerlet3D::step, src3d/Integrator3D.hpp:23-40) on h.stream:
// drift, evaluation (eager, or sized by the capacities in capacity mode), kick.
static int step_once(Handle& h, double* dp, double* dv, const double* dm, double* da, double* dn, double dt) {
    const int64_t n3 = 3 * h.n;
    const int grid = (int)((n3 + 255) / 256);
    k_drift<<<grid, 256, 0, h.stream>>>(dp, dv, da, n3, dt, 0.5 * dt * dt); ++h.launches;
    OGX_TRY(eval_device(h, h.n, dp, dm, dn, nullptr));
    k_kick<<<grid, 256, 0, h.stream>>>(dv, da, dn, n3, 0.5 * dt, h.cap_mode ? h.d_counts : nullptr); ++h.launches;
    OGX_CUDA(cudaGetLastError());
    return OGX_OK;
}

// Release the captured step (its buffers moved, its launch shapes changed, or a later
// step did not fit its capacities).
void drop_step_graph(Handle& h) {
    if (h.step_exec) cudaGraphExecDestroy(h.step_exec);
    if (h.step_graph) cudaGraphDestroy(h.step_graph);
    h.step_exec = nullptr;
    h.step_graph = nullptr;
    h.cap_warm = 0;
    // the captured host-buffer evaluation is released on the same occasions
    if (h.eval_exec) cudaGraphExecDestroy(h.eval_exec);
    if (h.eval_graph) cudaGraphDestroy(h.eval_graph);
    h.eval_exec = nullptr;
    h.eval_graph = nullptr;
    h.eval_warm = 0;
}

// Record one step in capacity mode as a CUDA graph (nothing is launched).
static int capture_step(Handle& h, double* dp, double* dv, const double* dm, double* da, double* dn, double dt) {
    const int64_t l0 = h.launches;
    OGX_CUDA(cudaStreamBeginCapture(h.stream, cudaStreamCaptureModeRelaxed));
    h.capturing = true;
    h.cap_mode = true;
    h.ws.frozen = true;
    const int rc = step_once(h, dp, dv, dm, da, dn, dt);
    h.ws.frozen = false;
    h.cap_mode = false;
    h.capturing = false;
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(h.stream, &g);
    if (rc != OGX_OK || ec != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        if (rc != OGX_OK) return rc;
        set_last_error(OGX_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(ec));
        return OGX_ERR_CUDA;
    }
    // node priorities as captured: the near field keeps the low priority of its stream, so
    // it fills what the main chain leaves idle, as in an eager step
    const cudaError_t ei = cudaGraphInstantiateWithFlags(&h.step_exec, g, cudaGraphInstantiateFlagUseNodePriority);
    if (ei != cudaSuccess) {
        cudaGraphDestroy(g);
        h.step_exec = nullptr;
        set_last_error(OGX_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ei));
        return OGX_ERR_CUDA;
    }
    h.step_graph = g;
    h.step_launches = h.launches - l0;
    h.step_gen = h.ws.generation;
    return OGX_OK;
}

// One step of a resident system (VelocityVerlet3D::step): eager, or with step capture
// on (ogx_set_tuning) the first step after the capacities were set runs uncaptured in
// capacity mode (every buffer grows to its capacity there), the next one is recorded as
// a graph and later steps replay it.  Each step of a capturing handle copies its counts
// to the host; a step whose tree or lists overflowed did nothing after its drift and is
// redone eagerly here, which also sets new capacities.
static int redo_overflowed(Handle& h, double dt) {
    const int64_t n = h.n, n3 = 3 * n;
    double *dp, *dv, *dm, *da, *dn;
    OGX_TRY(arena_get(h.ws, S_POS, n3, &dp));
    OGX_TRY(arena_get(h.ws, S_VEL, n3, &dv));
    OGX_TRY(arena_get(h.ws, S_MASS, n, &dm));
    OGX_TRY(arena_get(h.ws, S_ACC, n3, &da));
    OGX_TRY(arena_get(h.ws, S_ACC_OLD, n3, &dn));
    drop_step_graph(h);
    h.cap_mode = false;
    const int grid = (int)((n3 + 255) / 256);
    OGX_TRY(eval_device(h, n, dp, dm, dn, nullptr));
    k_kick<<<grid, 256, 0, h.stream>>>(dv, da, dn, n3, 0.5 * dt, nullptr); ++h.launches;
    OGX_CUDA(cudaGetLastError());
    ++h.overflow_redos;
    h.stats.launches += 1;
    return OGX_OK;
}

int step_member(Handle& h, double dt) {
    const int64_t n = h.n, n3 = 3 * n;
    double *dp, *dv, *dm, *da, *dn;
    OGX_TRY(arena_get(h.ws, S_POS, n3, &dp));
    OGX_TRY(arena_get(h.ws, S_VEL, n3, &dv));
    OGX_TRY(arena_get(h.ws, S_MASS, n, &dm));
    OGX_TRY(arena_get(h.ws, S_ACC, n3, &da));
    OGX_TRY(arena_get(h.ws, S_ACC_OLD, n3, &dn));
    // a step on the legacy or per-thread default stream cannot be captured: such a handle
    // steps eagerly
    const bool capturable = h.stream != nullptr && h.stream != cudaStreamLegacy && h.stream != cudaStreamPerThread;
    // (the spline kernel's S lists are sized by a count read back in the middle of the
    // evaluation, so such steps stay eager)
    const bool graphed = h.capture_steps && capturable && h.prm.solver == OGX_SOLVER_ADAPTIVE_FMM && h.cap.valid &&
                         h.prm.softening == OGX_SOFT_PLUMMER;
    if (!graphed) {
        h.cap_mode = false;
        OGX_TRY(step_once(h, dp, dv, dm, da, dn, dt));
        h.stats.launches += 2;  // drift + kick around the evaluation
        return OGX_OK;
    }
    if (h.step_exec && h.step_gen != h.ws.generation) drop_step_graph(h);
    int64_t launched = 0;
    if (h.step_exec) {
        OGX_CUDA(cudaGraphLaunch(h.step_exec, h.stream));
        h.launches += h.step_launches;
        launched = h.step_launches;
        ++h.graph_steps;
    } else if (h.cap_warm == 0) {
        const int64_t l0 = h.launches;
        h.cap_mode = true;
        const int rc = step_once(h, dp, dv, dm, da, dn, dt);
        h.cap_mode = false;
        OGX_TRY(rc);
        h.cap_warm = 1;
        launched = h.launches - l0;
    } else {
        OGX_TRY(capture_step(h, dp, dv, dm, da, dn, dt));
        OGX_CUDA(cudaGraphLaunch(h.step_exec, h.stream));
        launched = h.step_launches;
        ++h.graph_steps;
    }
    OGX_CUDA(cudaStreamSynchronize(h.stream));
    OGX_TRY(device_error(h));
    if (h.h_counts->overflow) {
        OGX_TRY(redo_overflowed(h, dt));
    } else {
        finish_stats(h);   // times and counts of the step that just ran
        h.stats.launches = launched;
    }
    return OGX_OK;
}

// Members of an ensemble advance together: one CUDA graph whose child graphs are the
// members' captured steps, launched once per ensemble step.
struct Ensemble {
    std::vector<Handle*> members;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<cudaGraphExec_t> built_from;   // each member's step graph when `exec` was built
    int64_t graph_steps = 0;    // ensemble steps taken by one launch of `exec`
    int64_t member_steps = 0;   // ensemble steps taken member by member (warm-up, capture)
    int64_t redos = 0;          // member steps redone eagerly after an overflow
    int64_t rebuilds = 0;       // times `exec` was built
};

void drop_ensemble_graph(Ensemble& e) {
    if (e.exec) cudaGraphExecDestroy(e.exec);
    if (e.graph) cudaGraphDestroy(e.graph);
    e.exec = nullptr;
    e.graph = nullptr;
    e.built_from.clear();
}

static bool ensemble_current(const Ensemble& e) {
    if (!e.exec) return false;
    for (size_t i = 0; i < e.members.size(); ++i) {
        const Handle& h = *e.members[i];
        if (!h.step_exec || h.step_exec != e.built_from[i] || h.step_gen != h.ws.generation) return false;
    }
    return true;
}

static int build_ensemble_graph(Ensemble& e) {
    drop_ensemble_graph(e);
    cudaGraph_t g = nullptr;
    OGX_CUDA(cudaGraphCreate(&g, 0));
    for (Handle* h : e.members) {
        cudaGraphNode_t node;
        const cudaError_t ec = cudaGraphAddChildGraphNode(&node, g, nullptr, 0, h->step_graph);
        if (ec != cudaSuccess) {
            cudaGraphDestroy(g);
            set_last_error(OGX_ERR_CUDA, std::string("cudaGraphAddChildGraphNode: ") + cudaGetErrorString(ec));
            return OGX_ERR_CUDA;
        }
        e.built_from.push_back(h->step_exec);
    }
    const cudaError_t ei = cudaGraphInstantiateWithFlags(&e.exec, g, cudaGraphInstantiateFlagUseNodePriority);
    if (ei != cudaSuccess) {
        cudaGraphDestroy(g);
        e.exec = nullptr;
        e.built_from.clear();
        set_last_error(OGX_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ei));
        return OGX_ERR_CUDA;
    }
    e.graph = g;
    ++e.rebuilds;
    return OGX_OK;
}

// One step of every member.  While some member has no current step graph (its first
// steps, or after an overflow) the members step one by one; otherwise one launch runs
// all of them, then each member's counts are checked and an overflowed member's step
// is redone eagerly (so the ensemble graph is rebuilt at the next step).
int ensemble_step(Ensemble& e, double dt) {
    if (!ensemble_current(e)) {
        drop_ensemble_graph(e);
        // the members' own steps (uncaptured warm-up, then capture) are independent, so a
        // few host threads take them; each handle is driven by one thread at a time
        const int nm = (int)e.members.size();
        const int nt = std::min(nm, 8);
        std::atomic<int> next{0};
        std::mutex mu;
        int rc_first = OGX_OK;
        std::string msg;
        auto work = [&]() {
            for (;;) {
                const int i = next.fetch_add(1);
                if (i >= nm) return;
                Handle& m = *e.members[i];
                DeviceGuard g(m.device);
                const int rc = step_member(m, dt);
                if (rc != OGX_OK) {
                    std::lock_guard<std::mutex> lk(mu);
                    if (rc_first == OGX_OK) {
                        rc_first = rc;
                        msg = g_last_error;
                    }
                }
            }
        };
        std::vector<std::thread> pool;
        for (int t = 1; t < nt; ++t) pool.emplace_back(work);
        work();
        for (std::thread& t : pool) t.join();
        if (rc_first != OGX_OK) {
            set_last_error(rc_first, msg);
            return rc_first;
        }
        ++e.member_steps;
        bool ready = true;
        for (Handle* h : e.members) ready = ready && h->step_exec && h->step_gen == h->ws.generation;
        if (ready) OGX_TRY(build_ensemble_graph(e));
        return OGX_OK;
    }
    OGX_CUDA(cudaGraphLaunch(e.exec, e.stream));
    OGX_CUDA(cudaStreamSynchronize(e.stream));
    ++e.graph_steps;
    for (Handle* h : e.members) {
        h->launches += h->step_launches;
        ++h->graph_steps;
        OGX_TRY(device_error(*h));
        if (h->h_counts->overflow) {
            OGX_TRY(redo_overflowed(*h, dt));
            ++e.redos;
        } else {
            finish_stats(*h);
            h->stats.launches = h->step_launches;
        }
    }
    for (Handle* h : e.members) OGX_CUDA(cudaStreamSynchronize(h->stream));
    return OGX_OK;
}

}  // namespace ogx

using namespace ogx;

#define HANDLE(hv) Handle& h = *static_cast<Handle*>(hv)

extern "C" {

int ogx_params_default(ogx_params* prm) {
    if (!prm) return OGX_ERR_INVALID;
    std::memset(prm, 0, sizeof(*prm));
    prm->G = 1.0;
    prm->eps = 0.0;
    prm->p = 8;
    prm->leaf_capacity = 64;
    prm->solver = OGX_SOLVER_ADAPTIVE_FMM;
    prm->precision = OGX_PREC_FP64;
    prm->device = 0;
    prm->stream = nullptr;
    return OGX_OK;
}

const char* ogx_strerror(int status) {
    switch (status) {
        case OGX_OK: return "ok";
        case OGX_ERR_INVALID: return "invalid argument";
        case OGX_ERR_CUDA: return "CUDA error";
        case OGX_ERR_NO_DEVICE: return "no CUDA device";
        case OGX_ERR_OOM: return "out of device memory";
        case OGX_ERR_UNSUPPORTED: return "unsupported request";
        case OGX_ERR_TIMEOUT: return "device wait timed out";
        case OGX_ERR_STATE: return "call out of sequence";
        default: return "unknown status";
    }
}

const char* ogx_last_error_message(void) { return g_last_error.c_str(); }

int ogx_create(const ogx_params* prm, void** handle) {
    if (!prm || !handle) return OGX_ERR_INVALID;
    *handle = nullptr;
    if (!(std::isfinite(prm->G)) || !(prm->eps >= 0.0) || !std::isfinite(prm->eps)) return OGX_ERR_INVALID;
    if (prm->solver != OGX_SOLVER_ADAPTIVE_FMM && prm->solver != OGX_SOLVER_DIRECT) return OGX_ERR_INVALID;
    if (prm->precision != OGX_PREC_FP64 && prm->precision != OGX_PREC_MIXED && prm->precision != OGX_PREC_FP64_ROT)
        return OGX_ERR_INVALID;
    if (prm->softening != OGX_SOFT_PLUMMER && prm->softening != OGX_SOFT_SPLINE) return OGX_ERR_INVALID;
    if (prm->solver == OGX_SOLVER_ADAPTIVE_FMM) {
        if (prm->p < 1 || prm->p > kPMax) return OGX_ERR_INVALID;
        if (prm->leaf_capacity < 1 || prm->leaf_capacity > 4096) return OGX_ERR_INVALID;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        set_last_error(OGX_ERR_NO_DEVICE, "no CUDA device");
        return OGX_ERR_NO_DEVICE;
    }
    if (prm->device < 0 || prm->device >= ndev) return OGX_ERR_INVALID;
    DeviceGuard g(prm->device);
    OGX_TRY(device_init(prm->device));
    std::unique_ptr<Handle> h(new Handle);
    h->prm = *prm;
    h->device = prm->device;
    cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, prm->device);
    if (prm->stream) {
        h->stream = (cudaStream_t)prm->stream;
    } else {
        OGX_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        h->own_stream = true;
    }
    OGX_CUDA(cudaMallocHost(&h->h_counts, sizeof(DevCounts)));
    OGX_CUDA(cudaMallocHost(&h->h_err, sizeof(int)));
    *h->h_err = 0;
    std::memset(h->h_counts, 0, sizeof(DevCounts));
    for (auto& e : h->ev) OGX_CUDA(cudaEventCreate(&e));
    int prio_low = 0, prio_high = 0;
    OGX_CUDA(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    OGX_CUDA(cudaStreamCreateWithPriority(&h->main, cudaStreamNonBlocking, prio_high));
    OGX_CUDA(cudaStreamCreateWithPriority(&h->side, cudaStreamNonBlocking, prio_low));
    OGX_CUDA(cudaStreamCreateWithPriority(&h->up, cudaStreamNonBlocking, prio_high));
    OGX_CUDA(cudaStreamCreateWithPriority(&h->aux, cudaStreamNonBlocking, prio_high));
    // the M2L between the list build (high) and the side stream (low), where the
    // device has a level between them
    const int prio_mid = (prio_high - prio_low <= -2 || prio_high - prio_low >= 2) ? (prio_low + prio_high) / 2 : prio_high;
    OGX_CUDA(cudaStreamCreateWithPriority(&h->m2l, cudaStreamNonBlocking, prio_mid));
    OGX_CUDA(cudaEventCreateWithFlags(&h->ev_col, cudaEventDisableTiming));
    OGX_CUDA(cudaEventCreateWithFlags(&h->ev_tgt, cudaEventDisableTiming));
    OGX_CUDA(cudaEventCreateWithFlags(&h->ev_m2l, cudaEventDisableTiming));
    OGX_CUDA(cudaEventCreateWithFlags(&h->ev_mass, cudaEventDisableTiming));
    OGX_CUDA(cudaEventCreateWithFlags(&h->ev_pos, cudaEventDisableTiming));
    for (cudaEvent_t* e : {&h->ev_fork, &h->ev_join, &h->ev_in, &h->ev_out, &h->ev_tree, &h->ev_up})
        OGX_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    OGX_CUDA(cudaEventCreate(&h->ev_up_end));
    *handle = h.release();
    return OGX_OK;
}

int ogx_destroy(void* handle) {
    if (!handle) return OGX_ERR_INVALID;
    Handle* h = static_cast<Handle*>(handle);
    {
        DeviceGuard g(h->device);
        cudaStreamSynchronize(h->stream);
        drop_step_graph(*h);
        h->ws.release();
        if (h->h_counts) cudaFreeHost(h->h_counts);
        if (h->h_err) cudaFreeHost(h->h_err);
        if (h->h_stage) cudaFreeHost(h->h_stage);
        for (auto& e : h->ev)
            if (e) cudaEventDestroy(e);
        for (cudaEvent_t e : {h->ev_col, h->ev_tgt, h->ev_m2l, h->ev_mass, h->ev_pos})
            if (e) cudaEventDestroy(e);
        for (cudaStream_t sx : {h->main, h->side, h->up, h->aux, h->m2l})
            if (sx) {
                cudaStreamSynchronize(sx);
                cudaStreamDestroy(sx);
            }
        for (cudaEvent_t e : {h->ev_fork, h->ev_join, h->ev_in, h->ev_out, h->ev_tree, h->ev_up, h->ev_up_end})
            if (e) cudaEventDestroy(e);
        if (h->own_stream) cudaStreamDestroy(h->stream);
    }
    delete h;
    return OGX_OK;
}

const char* ogx_name(void* handle) {
    if (!handle) return "ogx";
    HANDLE(handle);
    if (h.prm.solver == OGX_SOLVER_DIRECT) return "OgxDirect3D(B200, O(N^2) FP64)";
    return h.prm.precision == OGX_PREC_FP64       ? "OgxAdaptiveFMM3D(B200, FP64)"
           : h.prm.precision == OGX_PREC_FP64_ROT ? "OgxAdaptiveFMM3D(B200, FP64, rotation M2L)"
                                                  : "OgxAdaptiveFMM3D(B200, mixed)";
}

int ogx_eval_device(void* handle, int64_t n, const double* d_pos, const double* d_mass, double* d_acc, double* d_pot) {
    if (!handle || n < 0 || n > (int64_t)INT32_MAX / 2) return OGX_ERR_INVALID;
    if (n > 0 && (!d_pos || !d_mass || !d_acc)) return OGX_ERR_INVALID;
    HANDLE(handle);
    DeviceGuard g(h.device);
    return eval_device(h, n, d_pos, d_mass, d_acc, d_pot);
}

int ogx_synchronize(void* handle) {
    if (!handle) return OGX_ERR_INVALID;
    HANDLE(handle);
    DeviceGuard g(h.device);
    OGX_CUDA(cudaStreamSynchronize(h.stream));
    OGX_TRY(device_error(h));
    return OGX_OK;
}

// Copies in, evaluation, copies out of one host-buffer evaluation, issued on h.stream
// (eagerly, in capacity mode, or into a capture); timing events: h2d ev[10]..ev[11],
// d2h ev[12]..ev[13].
static int eval_host_issue(Handle& h, int64_t n, const double* pos, const double* mass, double* acc, double* pot,
                           double* dp, double* dm, double* da, double* dpot) {
    OGX_CUDA(timing_record(h, h.ev[10], h.stream));
    OGX_CUDA(cudaMemcpyAsync(dp, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h.stream));
    // the masses are first read at the end of the tree build (the sorted-body gather), so
    // their copy runs on the aux stream beside the bounding box, keys and sort
    const bool fmm = h.prm.solver == OGX_SOLVER_ADAPTIVE_FMM;
    if (fmm) {
        // after the positions (the two copies would otherwise share the link and the
        // positions, which the tree build needs first, would arrive no earlier)
        OGX_CUDA(cudaEventRecord(h.ev_pos, h.stream));
        OGX_CUDA(cudaStreamWaitEvent(h.aux, h.ev_pos, 0));
        OGX_CUDA(cudaMemcpyAsync(dm, mass, n * sizeof(double), cudaMemcpyHostToDevice, h.aux));
        OGX_CUDA(cudaEventRecord(h.ev_mass, h.aux));
        OGX_CUDA(timing_record(h, h.ev[11], h.aux));
        h.mass_pending = true;
    } else {
        OGX_CUDA(cudaMemcpyAsync(dm, mass, n * sizeof(double), cudaMemcpyHostToDevice, h.stream));
        OGX_CUDA(timing_record(h, h.ev[11], h.stream));
    }
    const int rc_eval = eval_device(h, n, dp, dm, da, dpot);
    if (h.mass_pending) {   // an evaluation that stopped before the gather still orders the copy
        cudaStreamWaitEvent(h.stream, h.ev_mass, 0);
        h.mass_pending = false;
    }
    OGX_TRY(rc_eval);
    OGX_CUDA(timing_record(h, h.ev[12], h.stream));
    OGX_CUDA(cudaMemcpyAsync(acc, da, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, h.stream));
    if (pot) OGX_CUDA(cudaMemcpyAsync(pot, dpot, n * sizeof(double), cudaMemcpyDeviceToHost, h.stream));
    OGX_CUDA(timing_record(h, h.ev[13], h.stream));
    return OGX_OK;
}

static bool page_locked(const void* p) {
    if (!p) return true;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Record one host-buffer evaluation in capacity mode as a CUDA graph (nothing runs).
static int capture_eval(Handle& h, int64_t n, const double* pos, const double* mass, double* acc, double* pot, double* dp,
                        double* dm, double* da, double* dpot) {
    const int64_t l0 = h.launches;
    OGX_CUDA(cudaStreamBeginCapture(h.stream, cudaStreamCaptureModeRelaxed));
    h.capturing = true;
    h.cap_mode = true;
    h.ws.frozen = true;
    const int rc = eval_host_issue(h, n, pos, mass, acc, pot, dp, dm, da, dpot);
    h.ws.frozen = false;
    h.cap_mode = false;
    h.capturing = false;
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(h.stream, &g);
    if (rc != OGX_OK || ec != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        if (rc != OGX_OK) return rc;
        set_last_error(OGX_ERR_CUDA, std::string("cudaStreamEndCapture: ") + cudaGetErrorString(ec));
        return OGX_ERR_CUDA;
    }
    const cudaError_t ei = cudaGraphInstantiateWithFlags(&h.eval_exec, g, cudaGraphInstantiateFlagUseNodePriority);
    if (ei != cudaSuccess) {
        cudaGraphDestroy(g);
        h.eval_exec = nullptr;
        set_last_error(OGX_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ei));
        return OGX_ERR_CUDA;
    }
    h.eval_graph = g;
    h.eval_launches = h.launches - l0;
    h.eval_gen = h.ws.generation;
    return OGX_OK;
}

// ForceSolver3D::computeAccelerations on host buffers.  Eager by default.  With step
// capture on (ogx_set_tuning), page-locked buffers and an adaptive-FMM handle with
// Plummer softening, the first call after the capacities were set runs uncaptured in
// capacity mode, the next is recorded as a CUDA graph (copies in, evaluation, copies
// out) and later calls with the same n and buffers replay it; a call that outgrew its
// capacities is redone eagerly, which sets new ones.  Results equal eager calls.
int ogx_eval(void* handle, int64_t n, const double* pos, const double* mass, double* acc, double* pot) {
    if (!handle || n < 0 || n > (int64_t)INT32_MAX / 2) return OGX_ERR_INVALID;
    if (n > 0 && (!pos || !mass || !acc)) return OGX_ERR_INVALID;
    HANDLE(handle);
    DeviceGuard g(h.device);
    if (n == 0) {
        eval_device(h, 0, nullptr, nullptr, nullptr, nullptr);
        return OGX_OK;
    }
    double *dp, *dm, *da, *dpot = nullptr;
    OGX_TRY(arena_get(h.ws, S_POS, 3 * n, &dp));
    OGX_TRY(arena_get(h.ws, S_MASS, n, &dm));
    OGX_TRY(arena_get(h.ws, S_ACC, 3 * n, &da));
    if (pot) OGX_TRY(arena_get(h.ws, S_POT, n, &dpot));
    const bool capturable = h.stream != nullptr && h.stream != cudaStreamLegacy && h.stream != cudaStreamPerThread;
    const bool graphed = h.capture_steps && capturable && h.prm.solver == OGX_SOLVER_ADAPTIVE_FMM && h.cap.valid &&
                         h.prm.softening == OGX_SOFT_PLUMMER && page_locked(pos) && page_locked(mass) &&
                         page_locked(acc) && page_locked(pot);
    int64_t launched = 0;
    if (!graphed) {
        h.cap_mode = false;
        OGX_TRY(eval_host_issue(h, n, pos, mass, acc, pot, dp, dm, da, dpot));
    } else {
        Handle::EvalKey key;
        key.n = n; key.pos = pos; key.mass = mass; key.acc = acc; key.pot = pot;
        if (h.eval_exec && (!(key == h.eval_key) || h.eval_gen != h.ws.generation)) {
            if (h.eval_exec) cudaGraphExecDestroy(h.eval_exec);
            if (h.eval_graph) cudaGraphDestroy(h.eval_graph);
            h.eval_exec = nullptr;
            h.eval_graph = nullptr;
            h.eval_warm = 0;
        }
        if (h.eval_exec) {
            OGX_CUDA(cudaGraphLaunch(h.eval_exec, h.stream));
            h.launches += h.eval_launches;
            launched = h.eval_launches;
            ++h.graph_evals;
        } else if (h.eval_warm == 0 || !(key == h.eval_key)) {
            const int64_t l0 = h.launches;
            h.cap_mode = true;
            const int rc = eval_host_issue(h, n, pos, mass, acc, pot, dp, dm, da, dpot);
            h.cap_mode = false;
            OGX_TRY(rc);
            h.eval_warm = 1;
            h.eval_key = key;
            launched = h.launches - l0;
        } else {
            OGX_TRY(capture_eval(h, n, pos, mass, acc, pot, dp, dm, da, dpot));
            OGX_CUDA(cudaGraphLaunch(h.eval_exec, h.stream));
            launched = h.eval_launches;
            ++h.graph_evals;
        }
    }
    OGX_CUDA(cudaStreamSynchronize(h.stream));
    OGX_TRY(device_error(h));
    if (graphed && h.h_counts->overflow) {
        // the tree or the lists outgrew the capacities: redo eagerly (new capacities)
        drop_step_graph(h);
        h.cap_mode = false;
        OGX_TRY(eval_host_issue(h, n, pos, mass, acc, pot, dp, dm, da, dpot));
        OGX_CUDA(cudaStreamSynchronize(h.stream));
        OGX_TRY(device_error(h));
        ++h.overflow_redos;
        launched = 0;
    }
    finish_stats(h);
    if (launched) h.stats.launches = launched;
    h.stats.ms_h2d = ev_ms(h.ev[10], h.ev[11]);
    h.stats.ms_d2h = ev_ms(h.ev[12], h.ev[13]);
    return OGX_OK;
}

int ogx_last_stats(void* handle, ogx_stats* out) {
    if (!handle || !out) return OGX_ERR_INVALID;
    HANDLE(handle);
    DeviceGuard g(h.device);
    if (h.stats.ms_total == 0.0) finish_stats(h);
    h.stats.graph_steps = h.graph_steps;
    h.stats.step_redos = h.overflow_redos;
    h.stats.graph_evals = h.graph_evals;
    *out = h.stats;
    return OGX_OK;
}

// ---- device-resident leapfrog -------------------------------------------------------
int ogx_upload(void* handle, int64_t n, const double* pos, const double* vel, const double* mass) {
    if (!handle || n <= 0 || !pos || !vel || !mass || n > (int64_t)INT32_MAX / 2) return OGX_ERR_INVALID;
    HANDLE(handle);
    DeviceGuard g(h.device);
    drop_step_graph(h);   // a new system: new sizes and capacities
    double *dp, *dv, *dm, *da;
    OGX_TRY(arena_get(h.ws, S_POS, 3 * n, &dp));
    OGX_TRY(arena_get(h.ws, S_VEL, 3 * n, &dv));
    OGX_TRY(arena_get(h.ws, S_MASS, n, &dm));
    OGX_TRY(arena_get(h.ws, S_ACC, 3 * n, &da));
    OGX_CUDA(cudaMemcpyAsync(dp, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h.stream));
    OGX_CUDA(cudaMemcpyAsync(dv, vel, 3 * n * sizeof(double), cudaMemcpyHostToDevice, h.stream));
    OGX_CUDA(cudaMemcpyAsync(dm, mass, n * sizeof(double), cudaMemcpyHostToDevice, h.stream));
    OGX_TRY(eval_device(h, n, dp, dm, da, nullptr));  // VelocityVerlet3D::initialize
    finish_stats(h);
    h.resident = true;
    h.n = n;
    return OGX_OK;
}

int ogx_step(void* handle, double dt, int nsteps) {
    if (!handle || nsteps < 0 || !std::isfinite(dt)) return OGX_ERR_INVALID;
    HANDLE(handle);
    if (!h.resident) return OGX_ERR_STATE;
    DeviceGuard g(h.device);
    for (int s = 0; s < nsteps; ++s) OGX_TRY(step_member(h, dt));
    OGX_CUDA(cudaGetLastError());
    return OGX_OK;
}

// ---- ensembles: every member's step in one graph launch --------------------------------
int ogx_ensemble_create(void* const* handles, int count, void** out) {
    if (!handles || count < 1 || !out) return OGX_ERR_INVALID;
    *out = nullptr;
    std::unique_ptr<Ensemble> e(new Ensemble);
    for (int i = 0; i < count; ++i) {
        if (!handles[i]) return OGX_ERR_INVALID;
        Handle* h = static_cast<Handle*>(handles[i]);
        if (!h->resident || h->prm.solver != OGX_SOLVER_ADAPTIVE_FMM) return OGX_ERR_STATE;
        if (i > 0 && h->device != e->members[0]->device) return OGX_ERR_INVALID;
        for (Handle* o : e->members)
            if (o == h) return OGX_ERR_INVALID;
        e->members.push_back(h);
    }
    DeviceGuard g(e->members[0]->device);
    OGX_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    for (Handle* h : e->members) h->capture_steps = true;
    *out = e.release();
    return OGX_OK;
}

int ogx_ensemble_step(void* ens, double dt, int nsteps) {
    if (!ens || nsteps < 0 || !std::isfinite(dt)) return OGX_ERR_INVALID;
    Ensemble& e = *static_cast<Ensemble*>(ens);
    DeviceGuard g(e.members[0]->device);
    for (int s = 0; s < nsteps; ++s) OGX_TRY(ensemble_step(e, dt));
    return OGX_OK;
}

int ogx_ensemble_stats(void* ens, int64_t* out) {
    if (!ens || !out) return OGX_ERR_INVALID;
    const Ensemble& e = *static_cast<const Ensemble*>(ens);
    out[0] = e.graph_steps;
    out[1] = e.member_steps;
    out[2] = e.redos;
    out[3] = e.rebuilds;
    return OGX_OK;
}

int ogx_ensemble_destroy(void* ens) {
    if (!ens) return OGX_ERR_INVALID;
    Ensemble* e = static_cast<Ensemble*>(ens);
    {
        DeviceGuard g(e->members[0]->device);
        if (e->stream) cudaStreamSynchronize(e->stream);
        drop_ensemble_graph(*e);
        if (e->stream) cudaStreamDestroy(e->stream);
    }
    delete e;
    return OGX_OK;
}

int ogx_download(void* handle, double* pos, double* vel, double* acc) {
    if (!handle) return OGX_ERR_INVALID;
    HANDLE(handle);
    if (!h.resident) return OGX_ERR_STATE;
    DeviceGuard g(h.device);
    const int64_t n3 = 3 * h.n;
    double *dp, *dv, *da;
    OGX_TRY(arena_get(h.ws, S_POS, n3, &dp));
    OGX_TRY(arena_get(h.ws, S_VEL, n3, &dv));
    OGX_TRY(arena_get(h.ws, S_ACC, n3, &da));
    if (pos) OGX_CUDA(cudaMemcpyAsync(pos, dp, n3 * sizeof(double), cudaMemcpyDeviceToHost, h.stream));
    if (vel) OGX_CUDA(cudaMemcpyAsync(vel, dv, n3 * sizeof(double), cudaMemcpyDeviceToHost, h.stream));
    if (acc) OGX_CUDA(cudaMemcpyAsync(acc, da, n3 * sizeof(double), cudaMemcpyDeviceToHost, h.stream));
    OGX_CUDA(cudaStreamSynchronize(h.stream));
    return OGX_OK;
}

// ---- tree export ----------------------------------------------------------------------
int ogx_tree_sizes(void* handle, int64_t* sizes) {
    if (!handle || !sizes) return OGX_ERR_INVALID;
    HANDLE(handle);
    if (!h.tree_valid) return OGX_ERR_STATE;
    DeviceGuard g(h.device);
    OGX_CUDA(cudaStreamSynchronize(h.stream));
    const TreeView& tv = h.tv;
    // exact sizes (a step in capacity mode launched with capacities)
    const int exact_nb = h.h_counts->nb32, exact_nl = h.h_counts->nleaf32;
    std::vector<int> col((size_t)27 * exact_nb), child((size_t)8 * exact_nb), parent(exact_nb);
    OGX_CUDA(cudaMemcpy(col.data(), tv.col, col.size() * sizeof(int), cudaMemcpyDeviceToHost));
    OGX_CUDA(cudaMemcpy(child.data(), tv.child, child.size() * sizeof(int), cudaMemcpyDeviceToHost));
    OGX_CUDA(cudaMemcpy(parent.data(), tv.parent, parent.size() * sizeof(int), cudaMemcpyDeviceToHost));
    std::vector<int> coord((size_t)3 * exact_nb);
    OGX_CUDA(cudaMemcpy(coord.data(), tv.coord, coord.size() * sizeof(int), cudaMemcpyDeviceToHost));
    int64_t ncol = 0, nv = 0;
    for (int b = 0; b < exact_nb; ++b) {
        for (int d = 0; d < 27; ++d) ncol += col[27 * (size_t)b + d] >= 0;
        if (parent[b] < 0) continue;
        const int P = parent[b];
        const int tx = coord[3 * b] & 1, ty = coord[3 * b + 1] & 1, tz = coord[3 * b + 2] & 1;
        for (int D = 0; D < 27; ++D) {
            const int Q = col[27 * (size_t)P + D];
            if (Q < 0) continue;
            for (int s = 0; s < 8; ++s) {
                if (child[8 * (size_t)Q + s] < 0) continue;
                const int ox = 2 * (D % 3 - 1) + (s & 1) - tx, oy = 2 * ((D / 3) % 3 - 1) + ((s >> 1) & 1) - ty,
                          oz = 2 * (D / 9 - 1) + ((s >> 2) & 1) - tz;
                if (std::max(std::abs(ox), std::max(std::abs(oy), std::abs(oz))) >= 2) ++nv;
            }
        }
    }
    sizes[0] = exact_nb;
    sizes[1] = exact_nl;
    sizes[2] = ncol;
    sizes[3] = h.h_counts->u_total;
    sizes[4] = nv;
    sizes[5] = h.h_counts->w_total;
    sizes[6] = h.h_counts->w_total;
    return OGX_OK;
}

int ogx_tree_boxes(void* handle, int32_t* boxes, double* centers, int32_t* perm) {
    if (!handle || !boxes) return OGX_ERR_INVALID;
    HANDLE(handle);
    if (!h.tree_valid) return OGX_ERR_STATE;
    DeviceGuard g(h.device);
    OGX_CUDA(cudaStreamSynchronize(h.stream));
    const TreeView& tv = h.tv;
    // exact sizes (a step in capacity mode launched with capacities)
    const int exact_nb = h.h_counts->nb32, exact_nl = h.h_counts->nleaf32;
    const size_t nb = exact_nb;
    std::vector<int> level(nb), coord(3 * nb), parent(nb), leafid(nb), pfirst(nb), pcount(nb);
    OGX_CUDA(cudaMemcpy(level.data(), tv.level, nb * sizeof(int), cudaMemcpyDeviceToHost));
    OGX_CUDA(cudaMemcpy(coord.data(), tv.coord, 3 * nb * sizeof(int), cudaMemcpyDeviceToHost));
    OGX_CUDA(cudaMemcpy(parent.data(), tv.parent, nb * sizeof(int), cudaMemcpyDeviceToHost));
    OGX_CUDA(cudaMemcpy(leafid.data(), tv.leafid, nb * sizeof(int), cudaMemcpyDeviceToHost));
    OGX_CUDA(cudaMemcpy(pfirst.data(), tv.pfirst, nb * sizeof(int), cudaMemcpyDeviceToHost));
    OGX_CUDA(cudaMemcpy(pcount.data(), tv.pcount, nb * sizeof(int), cudaMemcpyDeviceToHost));
    // non-leaf occupancy = sum over children (boxes are level-major: children follow parents)
    for (size_t b = nb; b-- > 1;)
        if (parent[b] >= 0) pcount[parent[b]] += pcount[b];
    for (size_t b = 0; b < nb; ++b) {
        int32_t* r = boxes + 8 * b;
        r[0] = level[b]; r[1] = coord[3 * b]; r[2] = coord[3 * b + 1]; r[3] = coord[3 * b + 2];
        r[4] = parent[b]; r[5] = leafid[b] >= 0 ? 1 : 0; r[6] = pfirst[b]; r[7] = pcount[b];
    }
    if (centers) OGX_CUDA(cudaMemcpy(centers, tv.center, 4 * nb * sizeof(double), cudaMemcpyDeviceToHost));
    if (perm) OGX_CUDA(cudaMemcpy(perm, tv.perm, (size_t)tv.n * sizeof(int), cudaMemcpyDeviceToHost));
    return OGX_OK;
}

int ogx_tree_list(void* handle, int which, int64_t* off, int32_t* idx) {
    if (!handle || !off || !idx || which < 0 || which > 4) return OGX_ERR_INVALID;
    HANDLE(handle);
    if (!h.tree_valid) return OGX_ERR_STATE;
    DeviceGuard g(h.device);
    OGX_CUDA(cudaStreamSynchronize(h.stream));
    const TreeView& tv = h.tv;
    // exact sizes (a step in capacity mode launched with capacities)
    const int exact_nb = h.h_counts->nb32, exact_nl = h.h_counts->nleaf32;
    const size_t nb = exact_nb, nl = exact_nl;
    if (which == 0 || which == 2) {
        std::vector<int> col(27 * nb), child(8 * nb), parent(nb), coord(3 * nb);
        OGX_CUDA(cudaMemcpy(col.data(), tv.col, col.size() * sizeof(int), cudaMemcpyDeviceToHost));
        OGX_CUDA(cudaMemcpy(child.data(), tv.child, child.size() * sizeof(int), cudaMemcpyDeviceToHost));
        OGX_CUDA(cudaMemcpy(parent.data(), tv.parent, nb * sizeof(int), cudaMemcpyDeviceToHost));
        OGX_CUDA(cudaMemcpy(coord.data(), tv.coord, 3 * nb * sizeof(int), cudaMemcpyDeviceToHost));
        int64_t e = 0;
        for (size_t b = 0; b < nb; ++b) {
            off[b] = e;
            if (which == 0) {
                for (int d = 0; d < 27; ++d)
                    if (col[27 * b + d] >= 0) idx[e++] = col[27 * b + d];
                continue;
            }
            if (parent[b] < 0) continue;
            const int P = parent[b];
            const int tx = coord[3 * b] & 1, ty = coord[3 * b + 1] & 1, tz = coord[3 * b + 2] & 1;
            for (int D = 0; D < 27; ++D) {
                const int Q = col[27 * (size_t)P + D];
                if (Q < 0) continue;
                for (int s = 0; s < 8; ++s) {
                    const int c = child[8 * (size_t)Q + s];
                    if (c < 0) continue;
                    const int ox = 2 * (D % 3 - 1) + (s & 1) - tx, oy = 2 * ((D / 3) % 3 - 1) + ((s >> 1) & 1) - ty,
                              oz = 2 * (D / 9 - 1) + ((s >> 2) & 1) - tz;
                    if (std::max(std::abs(ox), std::max(std::abs(oy), std::abs(oz))) >= 2) idx[e++] = c;
                }
            }
        }
        off[nb] = e;
        return OGX_OK;
    }
    if (which == 4) {
        const int64_t nx = h.h_counts->w_total;
        std::vector<int64_t> xo(nb + 1);
        OGX_CUDA(cudaMemcpy(xo.data(), tv.x_off, (nb + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost));
        std::memcpy(off, xo.data(), (nb + 1) * sizeof(int64_t));
        if (nx) OGX_CUDA(cudaMemcpy(idx, tv.x_idx, nx * sizeof(int), cudaMemcpyDeviceToHost));
        return OGX_OK;
    }
    // U (1) or W (3): per leaf CSR -> per box CSR
    std::vector<int64_t> lo(nl + 1);
    std::vector<int> leafbox(nl), leafid(nb);
    const int64_t tot = (which == 1) ? h.h_counts->u_total : h.h_counts->w_total;
    std::vector<int> li(tot > 0 ? tot : 1);
    OGX_CUDA(cudaMemcpy(lo.data(), which == 1 ? tv.u_off : tv.w_off, (nl + 1) * sizeof(int64_t), cudaMemcpyDeviceToHost));
    if (tot) OGX_CUDA(cudaMemcpy(li.data(), which == 1 ? tv.u_idx : tv.w_idx, tot * sizeof(int), cudaMemcpyDeviceToHost));
    OGX_CUDA(cudaMemcpy(leafid.data(), tv.leafid, nb * sizeof(int), cudaMemcpyDeviceToHost));
    int64_t e = 0;
    for (size_t b = 0; b < nb; ++b) {
        off[b] = e;
        const int lf = leafid[b];
        if (lf < 0) continue;
        for (int64_t q = lo[lf]; q < lo[lf + 1]; ++q) idx[e++] = li[q];
    }
    off[nb] = e;
    return OGX_OK;
}

int ogx_set_tuning(void* handle, const ogx_tuning* t) {
    if (!handle || !t) return OGX_ERR_INVALID;
    HANDLE(handle);
    const int fill = t->m2l_tile_targets ? t->m2l_tile_targets : 128;
    const int units = t->near_units ? t->near_units : 64;
    if ((fill != 32 && fill != 64 && fill != 96 && fill != 128) || (units != 32 && units != 64)) {
        set_last_error(OGX_ERR_INVALID, "ogx_set_tuning: m2l_tile_targets must be 32, 64, 96 or 128 and near_units 32 or 64");
        return OGX_ERR_INVALID;
    }
    if (fill != h.tile_fill || units != h.near_units || (t->capture_steps != 0) != h.capture_steps) drop_step_graph(h);
    h.tile_fill = fill;
    h.near_units = units;
    h.capture_steps = t->capture_steps != 0;
    return OGX_OK;
}

int ogx_get_tuning(void* handle, ogx_tuning* out) {
    if (!handle || !out) return OGX_ERR_INVALID;
    HANDLE(handle);
    out->m2l_tile_targets = h.tile_fill;
    out->near_units = h.near_units;
    out->capture_steps = h.capture_steps ? 1 : 0;
    return OGX_OK;
}

int ogx_check_bounded_wait(void* handle, uint32_t polls) {
    if (!handle || polls == 0) return OGX_ERR_INVALID;
    HANDLE(handle);
    DeviceGuard g(h.device);
    DevCounts* dc;
    OGX_TRY(arena_get(h.ws, S_COUNTS, 1, &dc));
    h.d_err = &dc->kernel_error;
    int ran_out[2] = {0, 0};
    for (int k = 0; k < 2; ++k) {
        // the error word and, for the flag wait, a flag nothing sets (the word beside it)
        OGX_CUDA(cudaMemsetAsync(h.d_err, 0, 2 * sizeof(int), h.stream));
        if (k == 0) {   // the tensor-core pipeline's mbarrier wait
            k_wait_probe<<<1, 32, 0, h.stream>>>(polls, h.d_err);
            ++h.launches;
            OGX_CUDA(cudaGetLastError());
        } else {        // the translation passes' wait on a box's ready flag
            OGX_TRY(flag_wait_probe(h, polls, &dc->pad_err, h.d_err));
        }
        OGX_CUDA(cudaMemcpyAsync(h.h_err, h.d_err, sizeof(int), cudaMemcpyDeviceToHost, h.stream));
        OGX_CUDA(cudaStreamSynchronize(h.stream));
        ran_out[k] = *h.h_err;
        *h.h_err = 0;
    }
    OGX_CUDA(cudaMemsetAsync(h.d_err, 0, 2 * sizeof(int), h.stream));
    OGX_CUDA(cudaStreamSynchronize(h.stream));
    if (ran_out[0] && ran_out[1]) {
        set_last_error(OGX_ERR_TIMEOUT, "both bounded device waits ran out (mbarrier and ready flag)");
        return OGX_ERR_TIMEOUT;
    }
    set_last_error(OGX_ERR_STATE, "a bounded device wait given nothing to wait for did not run out");
    return OGX_ERR_STATE;
}

}  // extern "C"

namespace ogx {
int fmm_mixed(Handle& h, double* d_acc, double* d_pot);
}

namespace ogx {
// entry points for the other C-ABI files (run support in ogx_run.cu)
int eval_device_shared(Handle& h, int64_t n, const double* d_pos, const double* d_mass, double* d_acc, double* d_pot) {
    return eval_device(h, n, d_pos, d_mass, d_acc, d_pot);
}
void finish_stats_shared(Handle& h) { finish_stats(h); }
}  // namespace ogx
