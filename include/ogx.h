/*
 * ogx.h -- C ABI of the B200 adaptive-FMM force library (libogx.so).
 *
 * Drop-in boundary for on-galaxy's galaxy3d::ForceSolver3D
 * (src3d/ForceSolver3D.hpp:20-28):
 *     virtual Accelerations3D computeAccelerations(const Bodies3D&) const = 0;
 *     virtual const char* name() const = 0;
 * A std::vector<Vec3> is contiguous x,y,z doubles, so Bodies3D::pos.data()
 * and Bodies3D::mass.data() pass straight through as `pos` / `mass` below,
 * and the returned accelerations land in a std::vector<Vec3> the same way.
 *
 * Conventions shared by every entry point:
 *   - return value: OGX_OK (0) or an ogx_status error code; no exceptions,
 *     no exit() across the ABI; ogx_strerror() names the code.
 *   - positions/accelerations: n x 3 doubles (x,y,z per body), original order.
 *   - potentials: n doubles, pot_i = -G * sum_{j!=i} m_j / sqrt(r_ij^2 + eps^2)
 *     (direct) or its FMM approximation (the spline kernel's potential with
 *     OGX_SOFT_SPLINE); NULL skips the potential.
 *   - a handle is not thread-safe: one handle per host thread / stream.
 *   - all device work is issued on the handle's stream.
 */
#ifndef OGX_H
#define OGX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    OGX_OK = 0,
    OGX_ERR_INVALID = 1,      /* bad argument (n, p, leaf capacity, pointers) */
    OGX_ERR_CUDA = 2,         /* a CUDA runtime call failed */
    OGX_ERR_NO_DEVICE = 3,    /* no usable CUDA device */
    OGX_ERR_OOM = 4,          /* device allocation failed or over budget */
    OGX_ERR_UNSUPPORTED = 5,  /* valid request this build cannot serve */
    OGX_ERR_TIMEOUT = 6,      /* a bounded device wait ran out */
    OGX_ERR_STATE = 7         /* call out of sequence (e.g. step before upload) */
} ogx_status;

typedef enum {
    OGX_SOLVER_ADAPTIVE_FMM = 0, /* replaces AdaptiveFMM3D (src3d/AdaptiveFMM3D.hpp:20) */
    OGX_SOLVER_DIRECT = 1        /* replaces DirectSolver3D (src3d/DirectSolver3D.hpp:11) */
} ogx_solver;

typedef enum {
    OGX_PREC_FP64 = 0,  /* plain form: FP64 end to end, matches AdaptiveFMM3D to <=1e-12 */
    OGX_PREC_MIXED = 1, /* FP32 P2P + split-precision tensor-core M2L, FP64 upper translations */
    OGX_PREC_FP64_ROT = 2 /* third form, beyond the reference: FP64 end to end with the M2L factored into
                           * rotation, z-axis translation and inverse rotation (O(p^3) per pair instead of
                           * O(p^4)); equal to the plain form up to rounding, not to the reference's operation
                           * order (README.md:75 of the reference defers this operator) */
} ogx_precision;

/* Softening kernel.  The reference softens with Plummer's kernel in the P2P part only and
 * evaluates the far field unsoftened (src3d/AdaptiveFMM3D.hpp:18, :97-105), so every pair the
 * expansions take at a distance comparable to eps sees a different force than it would in the
 * near field; its README names that seam as the cause of its energy drift (README.md:73-75).
 * OGX_SOFT_SPLINE, beyond the reference: the cubic-spline kernel of Monaghan & Lattanzio (1985)
 * in the form GADGET-2 uses (Springel 2005), with support h = 2.8 eps (the potential at r = 0
 * equals Plummer's, -G m / eps).  It is exactly Newtonian for r >= h, so the unsoftened
 * expansions are exact for it there; every pair closer than h that the far field takes (leaves
 * that are not adjacent but lie within h of each other) is corrected by a direct pass with the
 * difference of the two kernels.  The result is the spline-softened force up to the truncation
 * error of the expansions, with no seam.  Steps of such a handle are never captured. */
typedef enum {
    OGX_SOFT_PLUMMER = 0, /* the reference's kernel: m / (r^2 + eps^2)^{3/2} (Kernel3D.hpp:24-42) */
    OGX_SOFT_SPLINE = 1   /* compact cubic spline, h = 2.8 eps, with the far field corrected within h */
} ogx_softening;

typedef struct {
    double G;            /* gravitational constant (KernelParams3D::G) */
    double eps;          /* softening length (KernelParams3D::eps); also the leaf-edge floor */
    int p;               /* expansion order, 1..12 (AdaptiveFMM3D p) */
    int leaf_capacity;   /* split threshold (AdaptiveFMM3D threshold), >= 1 */
    int solver;          /* ogx_solver */
    int precision;       /* ogx_precision */
    int device;          /* CUDA device ordinal */
    void* stream;        /* cudaStream_t to issue on; NULL = a stream owned by the handle */
    int softening;       /* an ogx_softening value; default OGX_SOFT_PLUMMER, the reference's kernel */
} ogx_params;

typedef struct {
    int64_t n;                 /* bodies in the last evaluation */
    int32_t num_boxes;         /* AdaptiveFMM3D::lastNumBoxes */
    int32_t num_leaves;
    int32_t max_leaf_occupancy;/* AdaptiveFMM3D::lastMaxLeafOcc */
    int32_t max_level;
    int64_t list_u, list_v, list_w, list_x; /* interaction-list sizes (pairs of boxes) */
    int64_t p2p_pairs;         /* body-body interactions of the U lists (incl. none for self) */
    int64_t m2p_evals;         /* body x W-box evaluations */
    int64_t p2l_evals;         /* source-body x X-box evaluations */
    int64_t adjacency_mismatch;/* integer vs FP64 adjacency disagreements (0 expected) */
    double ms_tree, ms_lists, ms_upward, ms_m2l, ms_p2l, ms_downward, ms_leaf, ms_total;
    double ms_h2d, ms_d2h;     /* host-buffer calls only */
    int64_t launches;          /* kernels launched by the last evaluation (+ drift/kick in ogx_step) */
    int64_t graph_steps;       /* ogx_step calls' steps replayed from a captured graph (running total) */
    int64_t step_redos;        /* steps redone eagerly after a capacity overflow (running total) */
    int64_t list_s;            /* OGX_SOFT_SPLINE: (leaf, leaf) pairs the far field takes within the support */
    int64_t graph_evals;       /* ogx_eval calls replayed from a captured graph (running total) */
} ogx_stats;

/* Fill *prm with defaults: G=1, eps=0, p=8, leaf_capacity=64, adaptive FMM, FP64, device 0,
 * Plummer softening. */
int ogx_params_default(ogx_params* prm);

/* Constructor: AdaptiveFMM3D(KernelParams3D, int p, int threshold) (src3d/AdaptiveFMM3D.hpp:22-23)
 * or DirectSolver3D(KernelParams3D) (src3d/DirectSolver3D.hpp:13). */
int ogx_create(const ogx_params* prm, void** handle);
int ogx_destroy(void* handle);

/* ForceSolver3D::computeAccelerations (src3d/ForceSolver3D.hpp:24) with HOST buffers:
 * copies in, evaluates, copies out, synchronises.  pot may be NULL. */
int ogx_eval(void* handle, int64_t n, const double* pos, const double* mass, double* acc, double* pot);

/* Same evaluation on DEVICE buffers (pos n*3, mass n, acc n*3, pot n or NULL), issued on the
 * handle's stream.  Returns after the work is enqueued; the tree sizes are read back once per
 * call so the host knows the launch shapes.  Call ogx_synchronize() before reading acc. */
int ogx_eval_device(void* handle, int64_t n, const double* d_pos, const double* d_mass, double* d_acc,
                    double* d_pot);
int ogx_synchronize(void* handle);

/* FP64 direct summation that allocates no device memory (no counterpart in the reference;
 * results equal those of ogx_eval on an OGX_SOLVER_DIRECT handle).  For callers that cannot
 * let a library allocate: cudaMalloc/cudaFree may synchronise the whole device and stall the
 * caller's other streams, and processes that reserve their device memory up front under a
 * fixed budget cannot have a library take more.  No handle is needed.
 * Host buffers: pos n*3 (Vec3 layout), mass n; out acc n*3, pot n or NULL; G and eps as in
 * KernelParams3D; stream is a cudaStream_t of the current device (NULL = the legacy default
 * stream; a stream of another device returns OGX_ERR_INVALID).  Bodies and
 * results are staged in one fixed array that the library reserves on every GPU it is loaded
 * on: at most 65536 bodies (4 MiB, held until the process exits); larger n returns
 * OGX_ERR_INVALID.  The call returns when acc/pot hold the results.
 * The first call on a device looks up that array's device address (once per device, with
 * that device current); make that first call before any stream capture.  All calls on a
 * device share the array: calls that overlap on the GPU (several host threads, or streams
 * that run at the same time) race, so serialise them.  Nothing in the array has to start at
 * zero: each call overwrites the inputs it stages and the kernel writes every output. */
int ogx_direct_eval_noalloc(int64_t n, const double* pos, const double* mass, double G, double eps, double* acc,
                            double* pot, void* stream);

/* ForceSolver3D::name (src3d/ForceSolver3D.hpp:26). */
const char* ogx_name(void* handle);
int ogx_last_stats(void* handle, ogx_stats* out);
const char* ogx_strerror(int status);
/* Launch-shape knobs of the mixed form (no counterpart in the reference, whose only knob is
 * the leaf capacity, AdaptiveFMM3D(KernelParams3D, int p, int threshold),
 * src3d/AdaptiveFMM3D.hpp:22-23).  Neither changes what is computed:
 *   m2l_tile_targets : M2L batch width, the targets placed in one 128-row tensor-core tile
 *                      (32, 64, 96 or 128; default 128).  Narrower batches give small
 *                      systems more tiles to spread over the SMs.  A target's M2L result
 *                      does not depend on it.
 *   near_units       : P2P tile shape, the (target, source part) units a warp spreads over
 *                      its 32 lanes per chunk of up to 32 targets (32 or 64; default 64).
 *                      64 lets a small leaf split its sources into more parts; it changes
 *                      the FP32 summation order of the near field only.
 *   capture_steps    : 1 = ogx_step records a step as a CUDA graph and replays it (default 0).
 *                      Such steps read no counts back in the middle: their launches and
 *                      buffers are sized from capacities set by the last eager evaluation
 *                      (counts plus an eighth).  The first step after the capacities were
 *                      set runs without capture and sizes the buffers, the next is
 *                      recorded, later ones replay it.  A step whose tree or lists exceed
 *                      the capacities does nothing after its drift and is redone eagerly
 *                      inside the same ogx_step call (new capacities, new capture), so the
 *                      results are those of eager steps.  Each step ends with a host sync.
 *                      A handle whose stream is the legacy or per-thread default stream
 *                      steps eagerly (capture is not possible there).
 *                      ogx_eval on page-locked host buffers works the same way: the call
 *                      after the capacities were set runs uncaptured, the next records
 *                      copies in, evaluation and copies out as one graph, and later calls
 *                      with the same n and buffers replay it (other buffers start over).
 *                      Steps and such evaluations of OGX_SOFT_SPLINE handles stay eager.
 * ogx_set_tuning applies from the next evaluation on; 0 in a size field keeps its default. */
typedef struct {
    int m2l_tile_targets;
    int near_units;
    int capture_steps;
} ogx_tuning;
int ogx_set_tuning(void* handle, const ogx_tuning* t);
int ogx_get_tuning(void* handle, ogx_tuning* out);
/* Diagnostic with no counterpart in the reference: runs the library's two kinds of bounded
 * device wait, each giving up after a poll limit and setting the handle's device error word,
 * on something that never happens, with `polls` (>= 1) as the limit: the tensor-core M2L
 * pipeline's mbarrier wait on a barrier nothing arrives on, and the translation passes' wait
 * on a box's ready flag that nothing sets.  Returns OGX_ERR_TIMEOUT when both ran out, as an
 * evaluation whose wait ran out does, and leaves the handle usable: the error word is
 * cleared when it is reported. */
int ogx_check_bounded_wait(void* handle, uint32_t polls);
/* Text of the last error raised on the calling host thread (CUDA message etc.). */
const char* ogx_last_error_message(void);
/* Host-only helper (no GPU needed): the level-independent translation matrix used by the
 * kernels, K x K row-major with K=(p+1)^2 over the real coefficient layout
 * dof(n,0)=n^2, dof(n,m>0)=n^2+2m-1 (re) / n^2+2m (im), scaled M'=M/side^n, L'=L*side^n.
 * kind 0: M2M child octant index (0..7); 1: L2L child octant index (0..7);
 * 2: M2L source-minus-target offset index (ox+3)+7(oy+3)+49(oz+3) (0..342).
 * Replaces the per-pair operators fmm::M2M / fmm::L2L / fmm::M2L
 * (src3d/FmmExpansions3D.hpp:242-330). */
int ogx_operator_matrix(int kind, int p, int index, double* out);

/* ---- device-resident leapfrog: VelocityVerlet3D (src3d/Integrator3D.hpp:15-47) ----
 * upload = bodies onto the device + initialize() (one force evaluation);
 * step   = drift x += v dt + a dt^2/2, evaluate, kick v += (a_old + a_new) dt/2;
 * download copies pos/vel/acc (any may be NULL) back to the host. */
int ogx_upload(void* handle, int64_t n, const double* pos, const double* vel, const double* mass);
int ogx_step(void* handle, double dt, int nsteps);
int ogx_download(void* handle, double* pos, double* vel, double* acc);

/* ---- ensembles: many resident systems advanced by one launch per step ----
 * No counterpart in the reference (its integrator steps one system, Integrator3D.hpp:23-40).
 * ogx_ensemble_create groups resident adaptive-FMM handles of one device (each keeps its own
 * bodies, tree and expansions) and turns step capture on for them.  ogx_ensemble_step then
 * takes `nsteps` leapfrog steps of every member: once every member has a captured step
 * (see ogx_tuning.capture_steps; the first steps after creation or after a member's
 * overflow are taken member by member), a step is one cudaGraphLaunch of a graph whose child
 * graphs are the members' captured steps, so systems of any mix of N advance together with
 * no host work between their kernels.  Each member's result equals its own eager steps.
 * The members must not be used otherwise while an ensemble step runs, and they must outlive
 * the ensemble; they keep step capture on after it is destroyed.  ogx_ensemble_stats:
 * out[0] steps taken by one launch, out[1] steps taken member by member, out[2] member steps
 * redone after an overflow, out[3] times the ensemble graph was built.  Destroying the
 * ensemble leaves the handles alive. */
int ogx_ensemble_create(void* const* handles, int count, void** ensemble);
int ogx_ensemble_step(void* ensemble, double dt, int nsteps);
int ogx_ensemble_stats(void* ensemble, int64_t* out /* 4 */);
int ogx_ensemble_destroy(void* ensemble);

/* ---- tree export of the last adaptive evaluation (parity tests) ----
 * sizes[0]=boxes [1]=leaves [2..6]=|colleague|,|U|,|V|,|W|,|X| (AdaptiveOctree::buildLists,
 * src3d/AdaptiveOctree.hpp:137-189).
 * boxes: num_boxes x 8 int32 (level, ix, iy, iz, parent, leaf, pfirst, pcount),
 * centers: num_boxes x 4 doubles (cx, cy, cz, half), perm: sorted position -> original index.
 * which: 0=colleague 1=U 2=V 3=W 4=X; off has num_boxes+1 entries. */
int ogx_tree_sizes(void* handle, int64_t* sizes);
int ogx_tree_boxes(void* handle, int32_t* boxes, double* centers, int32_t* perm);
int ogx_tree_list(void* handle, int which, int64_t* off, int32_t* idx);

/* ---- running a simulation on the device ---------------------------------------------- */

/* Two-galaxy merger initial conditions.  Replaces makeDisk / setCircularVelocities /
 * placeGalaxy / concat (src3d/gpu/GalaxyIC.hpp:43-125) and the merger set-up of galaxy_sim
 * (src3d/gpu/galaxy_sim.cu:113-137).  Each galaxy: (1 - bulge_frac) of the bodies in an
 * exponential sech^2 disk (Rd, z0, mass Md; cut at 10 Rd and 10 z0), bulge_frac in a
 * Hernquist bulge (ab, Mb; cut at 50 ab).  Velocities: v_c^2 = -a_R R from the FP64 field of
 * the galaxy alone, plus Gaussian dispersion disp_frac * v_c.  Galaxy 0 sits at x = -sep with
 * bulk velocity +vrel/2, galaxy 1 at x = +sep with -vrel/2, tilted by tilt_deg about x. */
typedef struct {
    int64_t n_per;       /* bodies per galaxy */
    uint64_t seed;
    double sep, vrel, tilt_deg, disp_frac;
    double Rd, z0, Md, ab, Mb, bulge_frac;
} ogx_merger_params;

/* Defaults of the 1M benchmark merger: n_per 500000, seed 1, sep 5, vrel 0.5, tilt 30,
 * dispersion 0.1, Rd 1, z0 0.1, Md 1, ab 0.2, Mb 0.25, bulge 20%. */
int ogx_merger_params_default(ogx_merger_params* mp);

/* Generate the merger on the device straight into the handle's resident state (as
 * ogx_upload, including VelocityVerlet3D::initialize), bodies in galaxy order; the species
 * tag of a body is its galaxy (0 or 1), as galaxy_sim tags them.  species_out: NULL or n int8. */
int ogx_ic_merger(void* handle, const ogx_merger_params* mp, int8_t* species_out);

/* Species tags of the resident bodies (n int8, host), used by ogx_diagnostics. */
int ogx_set_species(void* handle, const int8_t* species);

/* Diagnostics of the resident state.  Replaces computeDiagnostics (src3d/Diagnostics3D.hpp:20-38)
 * and comSep (src3d/gpu/galaxy_sim.cu:209-216).  FP64 sums in a fixed order; the potential
 * energy is 1/2 sum m_i pot_i from a force evaluation with potentials at the current
 * positions (the reference sums -G m_i m_j / sqrt(r^2 + eps^2) over pairs; with this
 * library's solvers the far field is unsoftened, as in AdaptiveFMM3D).
 * out[16]: kinetic, potential, total, momentum xyz, angular momentum xyz, centre of mass of
 * species 0 xyz, of the other species xyz, their separation. */
int ogx_diagnostics(void* handle, double* out);

/* Resident positions as float32, n*3 in original body order: one frame of the reference's
 * frames.bin (src3d/gpu/galaxy_sim.cu:186-193). */
int ogx_download_frame(void* handle, float* pos_f32);

#ifdef __cplusplus
}
#endif
#endif /* OGX_H */
