// ogx_serve.cpp -- a serving loop for integration jobs on one GPU, through the C ABI.
//
// Jobs (a seeded stream): Poisson arrivals at --rate jobs/s, N log-uniform in
// [--nmin, --nmax], p drawn from --orders, --smin..--smax leapfrog steps with dt 0.01,
// half Plummer spheres, half two-galaxy disk+bulge systems.  A job is admitted when it
// has arrived and its estimated device footprint fits the --hbm-gb budget next to the
// jobs already resident; it then keeps its own handle (own streams) with bodies, tree
// and expansions on the device until it finishes and frees its memory.  A pool of
// --workers host threads (default 8) runs the resident jobs' steps from one FIFO
// queue, a job re-queued after each of its steps, so every resident job advances
// while at most W steps are in flight on the GPU (continuous batching at step
// granularity, not a queue drained one job at a time).  Before the clock starts, one
// small job per order and initial-condition kind warms the server up.
// --solo runs the same jobs one after another with nothing else on the GPU.
//
// --ensemble --steps S: the batched-ensemble workload instead.  All systems are
// resident together and advance in lockstep (every system finishes step s before any
// starts step s + 1), their steps spread over the same worker pool; the line then also
// carries the lockstep step time (p50 / p99).
//
// --eps E --softening plummer|spline: every job's softening (default: eps 0, Plummer's
// kernel as the reference; spline = compact kernel with the far field corrected inside
// its support, whose steps stay eager);
// --capture: every job's steps replay a CUDA graph of its step (ogx_tuning.capture_steps);
// the results are bit-identical to eager steps.
// --graph (with --ensemble): the systems advance through ogx_ensemble_step, every lockstep
// step one CUDA graph launch whose child graphs are the systems' captured steps (the first
// two steps are taken system by system while each captures its step).
//
// --autotune picks three knobs per job before it runs, by timing steps of dt = 0 of
// that job alone (a coordinate search): the leaf capacity from {32, 48, 64, 96, 128}
// (--thr fixes it instead, default 64), then the M2L batch width (targets per
// tensor-core tile) from {32, 64, 96, 128}, then the P2P tile shape (near-field units
// per warp) from {32, 64}.  The two launch-shape knobs change no physics: a candidate
// is only accepted when its accelerations agree with those of the default shape to a
// relative RMS of 1e-6.  --tune-cache FILE keeps the choices per (initial-condition
// kind, N rounded to a power of two, p, precision) as JSON: read before the run, the
// entries found skip the search, and the file is rewritten with every choice after it.
//
// Prints one JSON line: per-step latency p50 / p99 (the time from a step call until its
// result is on the device, ogx_step + ogx_synchronize), job turnaround p50 / p99 (from
// arrival to the final state on the host), aggregate bodies*steps/s over the wall time,
// the peak number of resident jobs, and per job an FNV-1a digest of its final positions
// and velocities (bit-exact), which the tests compare between --solo and the other modes.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "ogx.h"

namespace {

struct Job {
    int id = 0;
    double arrival = 0.0;  // seconds after start
    int64_t n = 0;
    int p = 8;
    int steps = 10;
    int kind = 0;  // 0 Plummer, 1 two-galaxy disk+bulge
    int thr = 64;  // leaf capacity
    int fill = 128;   // M2L batch width (targets per tensor-core tile)
    int units = 64;   // near-field units per warp
    bool tuned_from_cache = false;
    uint64_t seed = 0;
    // results
    uint64_t digest = 0;
    std::vector<float> step_ms;
    int status = OGX_OK;
    bool rejected = false;   // footprint above the whole budget: never admitted
    double need_bytes = 0.0;  // admission estimate
    double peak_bytes = 0.0;  // device memory above the idle level while it ran (--solo only)
    double t_done = 0.0;      // seconds after start when it finished
    void* h = nullptr;        // its handle while resident
};

// Plummer sphere (a = 1, M = 1, G = 1) drawn on the host: enclosed-mass inverse for
// r (cut at 20 a), isotropic directions, speed fraction by rejection from
// q^2 (1 - q^2)^(7/2), centre of mass and momentum removed
void plummer(int64_t n, uint64_t seed, std::vector<double>& pos, std::vector<double>& vel, std::vector<double>& mass) {
    std::mt19937_64 rng(seed);
    auto uni = [&]() { return (double)(rng() >> 11) * (1.0 / 9007199254740992.0); };
    pos.assign(3 * n, 0.0);
    vel.assign(3 * n, 0.0);
    mass.assign(n, 1.0 / (double)n);
    const double umax = std::pow(20.0, 3) / std::pow(20.0 * 20.0 + 1.0, 1.5);
    double cp[3] = {0, 0, 0}, cv[3] = {0, 0, 0};
    for (int64_t i = 0; i < n; ++i) {
        const double u = std::max(uni() * umax, 1e-12);
        const double r = 1.0 / std::sqrt(std::pow(u, -2.0 / 3.0) - 1.0);
        double q, g;
        do {
            q = uni();
            g = 0.1 * uni();
        } while (g > q * q * std::pow(1.0 - q * q, 3.5));
        const double v = q * std::sqrt(2.0) * std::pow(r * r + 1.0, -0.25);
        for (int pass = 0; pass < 2; ++pass) {
            const double cz = 2.0 * uni() - 1.0, sz = std::sqrt(std::max(0.0, 1.0 - cz * cz)), ph = 2.0 * M_PI * uni();
            const double len = pass == 0 ? r : v;
            double* o = (pass == 0 ? pos.data() : vel.data()) + 3 * i;
            o[0] = len * sz * std::cos(ph);
            o[1] = len * sz * std::sin(ph);
            o[2] = len * cz;
        }
        for (int k = 0; k < 3; ++k) {
            cp[k] += pos[3 * i + k] / (double)n;
            cv[k] += vel[3 * i + k] / (double)n;
        }
    }
    for (int64_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) {
            pos[3 * i + k] -= cp[k];
            vel[3 * i + k] -= cv[k];
        }
}

uint64_t fnv1a(const void* data, size_t bytes, uint64_t h = 1469598103934665603ull) {
    const unsigned char* c = (const unsigned char*)data;
    for (size_t i = 0; i < bytes; ++i) {
        h ^= c[i];
        h *= 1099511628211ull;
    }
    return h;
}

// admission estimate of a job's device footprint: the per-order operator tables
// (343 M2L matrices of K^2 doubles and the mixed form's padded FP16 hi/lo images,
// 20 bytes per matrix entry together, with slack) and per body its coordinates,
// keys, tree, lists and expansions; measured peaks sit below it by 20-50% from
// 16k to 200k bodies at p = 6, 8 and 12
double footprint_bytes(int64_t n, int p) {
    const double K = (double)(p + 1) * (p + 1);
    return 48e6 + 343.0 * K * K * 20.0 + (double)n * (1300.0 + 1.5 * K);
}

bool g_capture = false;   // --capture: every job replays its captured step (ogx_tuning.capture_steps)
double g_eps = 0.0;       // --eps: softening length of every job
int g_softening = OGX_SOFT_PLUMMER;   // --softening plummer|spline

// create the job's handle and its initial conditions on the device
void* open_job(Job& job, int precision) {
    ogx_params prm;
    ogx_params_default(&prm);
    prm.p = job.p;
    prm.leaf_capacity = job.thr;
    prm.precision = precision;
    prm.eps = g_eps;
    prm.softening = g_softening;
    void* h = nullptr;
    if ((job.status = ogx_create(&prm, &h)) != OGX_OK) return nullptr;
    ogx_tuning tu{job.fill, job.units, g_capture ? 1 : 0};
    if ((job.status = ogx_set_tuning(h, &tu)) != OGX_OK) {
        ogx_destroy(h);
        return nullptr;
    }
    if (job.kind == 0) {
        std::vector<double> pos, vel, mass;
        plummer(job.n, job.seed, pos, vel, mass);
        job.status = ogx_upload(h, job.n, pos.data(), vel.data(), mass.data());
    } else {
        ogx_merger_params mp;
        ogx_merger_params_default(&mp);
        mp.n_per = job.n / 2;
        mp.seed = job.seed;
        job.status = ogx_ic_merger(h, &mp, nullptr);
    }
    if (job.status != OGX_OK) {
        ogx_destroy(h);
        return nullptr;
    }
    return h;
}

// one leapfrog step, timed from the call until its result is on the device
void step_job(Job& job, void* h) {
    const auto t0 = std::chrono::steady_clock::now();
    job.status = ogx_step(h, 0.01, 1);
    if (job.status == OGX_OK) job.status = ogx_synchronize(h);
    job.step_ms.push_back((float)std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
}

// digest of the final positions and velocities, then release the handle
void close_job(Job& job, void* h) {
    const int64_t n = (job.kind == 0) ? job.n : 2 * (job.n / 2);
    std::vector<double> pos(3 * n), vel(3 * n);
    if (job.status == OGX_OK) job.status = ogx_download(h, pos.data(), vel.data(), nullptr);
    job.digest = fnv1a(vel.data(), vel.size() * 8, fnv1a(pos.data(), pos.size() * 8));
    ogx_destroy(h);
}

void run_job(Job& job, int precision) {
    void* h = open_job(job, precision);
    if (!h) return;
    for (int s = 0; s < job.steps && job.status == OGX_OK; ++s) step_job(job, h);
    close_job(job, h);
}

// fastest of the second and third of three steps of dt = 0 (the state is unchanged)
float time_steps(Job& job, void* h) {
    float ms = 1e30f;
    for (int r = 0; r < 3 && job.status == OGX_OK; ++r) {
        const auto t0 = std::chrono::steady_clock::now();
        job.status = ogx_step(h, 0.0, 1);
        if (job.status == OGX_OK) job.status = ogx_synchronize(h);
        if (r > 0) ms = std::min(ms, (float)std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    }
    return job.status == OGX_OK ? ms : 1e30f;
}

double rms_rel(const std::vector<double>& ref, const std::vector<double>& got) {
    double num = 0.0, den = 0.0;
    for (size_t i = 0; i < ref.size(); ++i) {
        num += (got[i] - ref[i]) * (got[i] - ref[i]);
        den += ref[i] * ref[i];
    }
    return den > 0.0 ? std::sqrt(num / den) : 0.0;
}

struct TuneChoice {
    int thr = 64, fill = 128, units = 64;
    float ms = 0.f;
};

// the knobs of one job, by coordinate search (see the file comment)
TuneChoice tune_job(Job job, int precision) {
    static const int thrs[] = {32, 48, 64, 96, 128};
    static const int fills[] = {32, 64, 96, 128};
    static const int unitss[] = {32, 64};
    TuneChoice best;
    best.thr = job.thr;
    float best_ms = 1e30f;
    job.fill = 128;
    job.units = 64;
    for (int thr : thrs) {
        job.thr = thr;
        job.status = OGX_OK;
        void* h = open_job(job, precision);
        if (!h) continue;
        const float ms = time_steps(job, h);
        ogx_destroy(h);
        if (ms < best_ms) {
            best_ms = ms;
            best.thr = thr;
        }
    }
    best.ms = best_ms;
    if (precision != OGX_PREC_MIXED) return best;   // the launch-shape knobs serve the mixed form
    job.thr = best.thr;
    job.status = OGX_OK;
    void* h = open_job(job, precision);
    if (!h) return best;
    const int64_t n = (job.kind == 0) ? job.n : 2 * (job.n / 2);
    std::vector<double> ref(3 * n), acc(3 * n);
    // accelerations of the default shape, then each candidate shape on the same state
    if (ogx_step(h, 0.0, 1) != OGX_OK || ogx_download(h, nullptr, nullptr, ref.data()) != OGX_OK) {
        ogx_destroy(h);
        return best;
    }
    auto trial = [&](int fill, int units) -> float {
        ogx_tuning tu{fill, units};
        if (ogx_set_tuning(h, &tu) != OGX_OK) return 1e30f;
        const float ms = time_steps(job, h);
        if (ms >= 1e30f || ogx_download(h, nullptr, nullptr, acc.data()) != OGX_OK) return 1e30f;
        return rms_rel(ref, acc) <= 1e-6 ? ms : 1e30f;   // accuracy gate
    };
    float cur = trial(128, 64);
    for (int fill : fills) {
        if (fill == 128) continue;
        const float ms = trial(fill, best.units);
        if (ms < cur) {
            cur = ms;
            best.fill = fill;
        }
    }
    for (int units : unitss) {
        if (units == best.units) continue;
        const float ms = trial(best.fill, units);
        if (ms < cur) {
            cur = ms;
            best.units = units;
        }
    }
    best.ms = std::min(best_ms, cur);
    ogx_destroy(h);
    return best;
}

// --tune-cache: {"<kind>:n<log2 N>:p<p>:<precision>": {"leaf_capacity": .., "m2l_tile_targets": ..,
// "near_units": .., "ms": ..}, ...}, one entry per line (this program writes and reads it)
std::string tune_key(const Job& jb, int precision) {
    const int lg = (int)std::lround(std::log2((double)std::max<int64_t>(jb.n, 1)));
    return std::string(jb.kind ? "merger" : "plummer") + ":n" + std::to_string(lg) + ":p" + std::to_string(jb.p) + ":" +
           (precision == OGX_PREC_FP64 ? "fp64" : precision == OGX_PREC_FP64_ROT ? "fp64rot" : "mixed");
}

std::map<std::string, TuneChoice> read_tune_cache(const std::string& path) {
    std::map<std::string, TuneChoice> m;
    FILE* f = path.empty() ? nullptr : std::fopen(path.c_str(), "r");
    if (!f) return m;
    char line[512];
    while (std::fgets(line, sizeof line, f)) {
        char key[256];
        TuneChoice c;
        if (std::sscanf(line, " \"%255[^\"]\": {\"leaf_capacity\": %d, \"m2l_tile_targets\": %d, \"near_units\": %d, \"ms\": %f",
                        key, &c.thr, &c.fill, &c.units, &c.ms) == 5)
            m[key] = c;
    }
    std::fclose(f);
    return m;
}

void write_tune_cache(const std::string& path, const std::map<std::string, TuneChoice>& m) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return;
    std::fprintf(f, "{\n");
    size_t k = 0;
    for (const auto& kv : m)
        std::fprintf(f, "\"%s\": {\"leaf_capacity\": %d, \"m2l_tile_targets\": %d, \"near_units\": %d, \"ms\": %.4f}%s\n",
                     kv.first.c_str(), kv.second.thr, kv.second.fill, kv.second.units, kv.second.ms,
                     ++k < m.size() ? "," : "");
    std::fprintf(f, "}\n");
    std::fclose(f);
}

// samples the device's used memory every millisecond while armed (solo runs)
struct MemSampler {
    std::atomic<bool> stop{false}, armed{false};
    std::atomic<double> peak{0.0};
    std::thread th;
    void start() {
        th = std::thread([this]() {
            cudaSetDevice(0);
            while (!stop.load()) {
                size_t fr = 0, tot = 0;
                if (armed.load() && cudaMemGetInfo(&fr, &tot) == cudaSuccess) {
                    const double used = (double)(tot - fr);
                    double cur = peak.load();
                    while (used > cur && !peak.compare_exchange_weak(cur, used)) {
                    }
                }
                std::this_thread::sleep_for(std::chrono::milliseconds(1));
            }
        });
    }
    void finish() {
        stop = true;
        if (th.joinable()) th.join();
    }
};

double device_used() {
    size_t fr = 0, tot = 0;
    return cudaMemGetInfo(&fr, &tot) == cudaSuccess ? (double)(tot - fr) : 0.0;
}

double percentile(std::vector<float> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * (double)(v.size() - 1);
    const size_t lo = (size_t)pos;
    const size_t hi = std::min(lo + 1, v.size() - 1);
    return v[lo] + (pos - (double)lo) * (v[hi] - v[lo]);
}

}  // namespace

int main(int argc, char** argv) {
    int njobs = 24, smin = 10, smax = 200;
    double rate = 20.0, hbm_gb = 150.0;
    int64_t nmin = 16384, nmax = 1 << 20;
    uint64_t seed = 1;
    bool solo = false, ensemble = false, autotune = false, graph = false;
    std::string tune_cache;
    int precision = OGX_PREC_MIXED, thr = 64, workers = 8;
    std::vector<int> orders = {6, 8, 12};
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        auto next = [&]() -> std::string { return (i + 1 < argc) ? argv[++i] : ""; };
        if (a == "--jobs") njobs = std::atoi(next().c_str());
        else if (a == "--rate") rate = std::atof(next().c_str());
        else if (a == "--nmin") nmin = std::atoll(next().c_str());
        else if (a == "--nmax") nmax = std::atoll(next().c_str());
        else if (a == "--smin") smin = std::atoi(next().c_str());
        else if (a == "--smax") smax = std::atoi(next().c_str());
        else if (a == "--hbm-gb") hbm_gb = std::atof(next().c_str());
        else if (a == "--seed") seed = std::strtoull(next().c_str(), nullptr, 10);
        else if (a == "--solo") solo = true;
        else if (a == "--ensemble") ensemble = true;
        else if (a == "--autotune") autotune = true;
        else if (a == "--graph") graph = true;
        else if (a == "--capture") g_capture = true;
        else if (a == "--eps") g_eps = std::atof(next().c_str());
        else if (a == "--softening") {
            const std::string v = next();
            if (v == "plummer") g_softening = OGX_SOFT_PLUMMER;
            else if (v == "spline") g_softening = OGX_SOFT_SPLINE;
            else {
                std::fprintf(stderr, "unknown softening '%s' (expected plummer or spline)\n", v.c_str());
                return 2;
            }
        }
        else if (a == "--tune-cache") tune_cache = next();
        else if (a == "--thr") thr = std::atoi(next().c_str());
        else if (a == "--workers") workers = std::atoi(next().c_str());
        else if (a == "--steps") smin = smax = std::atoi(next().c_str());
        else if (a == "--precision") {
            const std::string v = next();
            if (v == "fp64") precision = OGX_PREC_FP64;
            else if (v == "fp64rot") precision = OGX_PREC_FP64_ROT;
            else if (v == "mixed") precision = OGX_PREC_MIXED;
            else {
                std::fprintf(stderr, "unknown precision '%s' (expected fp64, fp64rot or mixed)\n", v.c_str());
                return 2;
            }
        }
        else if (a == "--orders") {
            orders.clear();
            std::string v = next();
            for (size_t s = 0; s < v.size();) {
                const size_t e = v.find(',', s);
                orders.push_back(std::atoi(v.substr(s, e == std::string::npos ? std::string::npos : e - s).c_str()));
                if (e == std::string::npos) break;
                s = e + 1;
            }
        } else {
            std::fprintf(stderr, "unknown option %s\n", a.c_str());
            return 2;
        }
    }
    if (njobs < 1 || nmin < 2 || nmax < nmin || smin < 1 || smax < smin || orders.empty() || rate <= 0 || thr < 1 || workers < 1 ||
        (ensemble && smin != smax)) {
        std::fprintf(stderr, "bad arguments\n");
        return 2;
    }
    // the seeded job stream
    std::mt19937_64 rng(seed);
    auto uni = [&]() { return (double)(rng() >> 11) * (1.0 / 9007199254740992.0); };
    std::map<std::string, TuneChoice> tcache = read_tune_cache(tune_cache);
    std::vector<Job> jobs(njobs);
    double t = 0.0;
    for (int j = 0; j < njobs; ++j) {
        t += -std::log(1.0 - uni()) / rate;
        Job& jb = jobs[j];
        jb.id = j;
        jb.arrival = t;
        jb.n = (int64_t)std::llround(std::exp(std::log((double)nmin) + uni() * (std::log((double)nmax) - std::log((double)nmin))));
        jb.p = orders[(size_t)(uni() * orders.size()) % orders.size()];
        jb.steps = smin + (int)(uni() * (smax - smin + 1)) % (smax - smin + 1);
        jb.kind = j & 1;
        jb.seed = seed * 1000003ull + (uint64_t)j;
        jb.thr = thr;
        if (ensemble) jb.arrival = 0.0;   // the whole ensemble starts together
    }
    {
        // a device must be there before any job is admitted
        ogx_params prm;
        ogx_params_default(&prm);
        void* probe = nullptr;
        const int rc = ogx_create(&prm, &probe);
        if (rc != OGX_OK) {
            std::printf("{\"error\": \"%s\"}\n", ogx_strerror(rc));
            return 3;
        }
        ogx_destroy(probe);
    }
    // server start-up, before the clock: one small job per order and initial-condition
    // kind loads every kernel module and builds the per-order operator tables, which
    // a running server has done long before its jobs arrive
    const auto w0 = std::chrono::steady_clock::now();
    for (int p : orders)
        for (int kind = 0; kind < 2; ++kind) {
            Job w;
            w.n = 4096;
            w.p = p;
            w.steps = 2;
            w.kind = kind;
            w.thr = thr;
            w.seed = 12345;
            run_job(w, precision);
            if (w.status != OGX_OK) {
                std::printf("{\"error\": \"warm-up job failed: %s\"}\n", ogx_strerror(w.status));
                return 3;
            }
        }
    const double warmup_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
    const double budget = hbm_gb * 1e9;
    MemSampler sampler;
    if (solo) sampler.start();
    const double idle = device_used();
    const auto start = std::chrono::steady_clock::now();
    auto now_s = [&]() { return std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count(); };

    // ---- the worker pool (served and ensemble modes) ----
    // W host threads run the jobs' tasks: open (handle + initial conditions), step,
    // close.  A job's next task is queued only when its previous one has finished,
    // so no handle is used by two threads at once; the FIFO queue interleaves the
    // steps of all resident jobs (continuous batching at step granularity) and W
    // bounds the steps in flight on the GPU.
    enum TaskKind { T_OPEN, T_STEP, T_CLOSE };
    struct Task {
        Job* job;
        TaskKind kind;
    };
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Task> queue;
    bool quit = false, lockstep = false;
    int finished = 0, step_done = 0, running = 0, peak = 0, rejected = 0;
    double in_use = 0.0;
    auto push = [&](Job* j, TaskKind k) {
        {
            std::lock_guard<std::mutex> g(mu);
            queue.push_back({j, k});
        }
        cv_work.notify_one();
    };
    auto worker = [&]() {
        for (;;) {
            Task t;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&]() { return quit || !queue.empty(); });
                if (queue.empty()) return;
                t = queue.front();
                queue.pop_front();
            }
            Job& jb = *t.job;
            if (t.kind == T_OPEN) {
                jb.h = open_job(jb, precision);
                if (lockstep) {
                    std::lock_guard<std::mutex> g(mu);
                    ++step_done;
                    cv_done.notify_all();
                } else {
                    push(&jb, (jb.h && jb.steps > 0) ? T_STEP : T_CLOSE);
                }
            } else if (t.kind == T_STEP) {
                if (jb.h && jb.status == OGX_OK) step_job(jb, jb.h);
                if (lockstep) {
                    std::lock_guard<std::mutex> g(mu);
                    ++step_done;
                    cv_done.notify_all();
                } else {
                    push(&jb, (jb.status == OGX_OK && (int)jb.step_ms.size() < jb.steps) ? T_STEP : T_CLOSE);
                }
            } else {
                if (jb.h) close_job(jb, jb.h);
                jb.h = nullptr;
                jb.t_done = now_s();
                std::lock_guard<std::mutex> g(mu);
                in_use -= jb.need_bytes;
                --running;
                ++finished;
                cv_done.notify_all();
            }
        }
    };
    std::vector<std::thread> pool;
    auto start_pool = [&]() {
        for (int w = 0; w < workers; ++w) pool.emplace_back(worker);
    };
    auto stop_pool = [&]() {
        {
            std::lock_guard<std::mutex> g(mu);
            quit = true;
        }
        cv_work.notify_all();
        for (auto& th : pool) th.join();
        pool.clear();
    };

    if (ensemble && !solo) {
        // lockstep ensemble: every system takes step s before any takes step s + 1
        std::vector<Job*> live;
        for (Job& jb : jobs) {
            jb.need_bytes = footprint_bytes(jb.n, jb.p);
            if (in_use + jb.need_bytes > budget) {
                jb.rejected = true;
                jb.status = OGX_ERR_INVALID;
                ++rejected;
                continue;
            }
            in_use += jb.need_bytes;
            if (autotune) {
                const std::string key = tune_key(jb, precision);
                auto it = tcache.find(key);
                if (it == tcache.end()) it = tcache.emplace(key, tune_job(jb, precision)).first;
                else jb.tuned_from_cache = true;
                jb.thr = it->second.thr;
                jb.fill = it->second.fill;
                jb.units = it->second.units;
            }
            live.push_back(&jb);
        }
        const int L = (int)live.size();
        lockstep = true;
        start_pool();
        auto round = [&](TaskKind k) {
            {
                std::lock_guard<std::mutex> g(mu);
                step_done = 0;
            }
            for (Job* j : live) push(j, k);
            std::unique_lock<std::mutex> lk(mu);
            cv_done.wait(lk, [&]() { return step_done == L; });
        };
        round(T_OPEN);
        std::vector<float> ens_ms;
        const int S = smin;
        int64_t gstats[4] = {0, 0, 0, 0};
        void* ens = nullptr;
        if (graph) {
            std::vector<void*> hs;
            for (Job* j : live)
                if (j->h && j->status == OGX_OK) hs.push_back(j->h);
            const int rc = hs.empty() ? OGX_ERR_STATE : ogx_ensemble_create(hs.data(), (int)hs.size(), &ens);
            if (rc != OGX_OK) {
                std::printf("{\"error\": \"ogx_ensemble_create: %s\"}\n", ogx_strerror(rc));
                return 1;
            }
        }
        const auto e0 = std::chrono::steady_clock::now();
        for (int st = 0; st < S; ++st) {
            const auto t0 = std::chrono::steady_clock::now();
            if (graph) {
                // every member's step in one launch (taken member by member until each
                // member has a captured step)
                const int rc = ogx_ensemble_step(ens, 0.01, 1);
                const float ms = (float)std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
                for (Job* j : live) {
                    if (j->h && j->status == OGX_OK) {
                        if (rc != OGX_OK) j->status = rc;
                        else j->step_ms.push_back(ms);
                    }
                }
            } else {
                round(T_STEP);
            }
            ens_ms.push_back((float)std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
        }
        const double ens_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - e0).count();
        if (ens) {
            ogx_ensemble_stats(ens, gstats);
            ogx_ensemble_destroy(ens);
        }
        lockstep = false;
        running = L;
        for (Job* j : live) push(j, T_CLOSE);
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_done.wait(lk, [&]() { return finished == L; });
        }
        stop_pool();
        sampler.finish();
        double bodysteps = 0.0, bodies = 0.0;
        int failed = 0;
        std::vector<float> all;
        for (const Job& jb : jobs) {
            all.insert(all.end(), jb.step_ms.begin(), jb.step_ms.end());
            bodysteps += (double)jb.n * (double)jb.step_ms.size();
            if (jb.status != OGX_OK && !jb.rejected) ++failed;
            if (jb.status == OGX_OK && !jb.rejected) bodies += (double)jb.n;
        }
        // steady state: all resident bodies over the median lockstep step (the first steps of
        // the one-launch mode step member by member while each member's step is captured)
        const double p50_ens = percentile(ens_ms, 0.5);
        const double steady = p50_ens > 0.0 ? bodies / (p50_ens * 1e-3) : 0.0;
        std::printf("{\"mode\": \"ensemble\", \"precision\": \"%s\", \"jobs\": %d, \"failed\": %d, \"rejected\": %d, "
                    "\"steps\": %zu, \"lockstep_steps\": %d, \"workers\": %d, \"wall_s\": %.3f, \"bodies_steps_per_s\": %.6e, "
                    "\"steady_bodies_steps_per_s\": %.6e, "
                    "\"ensemble_step_ms_p50\": %.3f, \"ensemble_step_ms_p99\": %.3f, \"p50_step_ms\": %.3f, "
                    "\"p99_step_ms\": %.3f, \"peak_concurrent\": %d, \"autotune\": %s, \"warmup_s\": %.3f, "
                    "\"capture\": %s, \"graph\": %s, \"graph_launch_steps\": %lld, \"member_by_member_steps\": %lld, \"member_redos\": %lld, "
                    "\"jobs_detail\": [",
                    precision == OGX_PREC_FP64 ? "fp64" : precision == OGX_PREC_FP64_ROT ? "fp64rot" : "mixed", njobs, failed, rejected, all.size(), S, workers, ens_s,
                    bodysteps / ens_s, steady, p50_ens, percentile(ens_ms, 0.99), percentile(all, 0.5),
                    percentile(all, 0.99), L, autotune ? "true" : "false", warmup_s, g_capture ? "true" : "false", graph ? "true" : "false",
                    (long long)gstats[0], (long long)gstats[1], (long long)gstats[2]);
        for (size_t j = 0; j < jobs.size(); ++j) {
            const Job& jb = jobs[j];
            std::printf("%s{\"id\": %d, \"n\": %lld, \"p\": %d, \"thr\": %d, \"m2l_tile_targets\": %d, \"near_units\": %d, "
                        "\"tuned_from_cache\": %s, \"kind\": \"%s\", \"status\": %d, "
                        "\"rejected\": %s, \"step_ms_p50\": %.3f, \"digest\": \"%016llx\"}",
                        j ? ", " : "", jb.id, (long long)jb.n, jb.p, jb.thr, jb.fill, jb.units,
                        jb.tuned_from_cache ? "true" : "false", jb.kind ? "disk+bulge merger" : "plummer",
                        jb.status, jb.rejected ? "true" : "false", percentile(jb.step_ms, 0.5),
                        (unsigned long long)jb.digest);
        }
        std::printf("]}\n");
        if (autotune && !tune_cache.empty()) write_tune_cache(tune_cache, tcache);
        return failed ? 1 : 0;
    }

    if (!solo) start_pool();
    int admitted = 0;
    for (Job& jb : jobs) {
        jb.need_bytes = footprint_bytes(jb.n, jb.p);
        if (jb.need_bytes > budget) {
            // could never fit, even alone: refused at admission, the loop goes on
            jb.rejected = true;
            jb.status = OGX_ERR_INVALID;
            ++rejected;
            continue;
        }
        if (autotune) {
            const std::string key = tune_key(jb, precision);
            auto it = tcache.find(key);
            if (it == tcache.end()) it = tcache.emplace(key, tune_job(jb, precision)).first;
            else jb.tuned_from_cache = true;
            jb.thr = it->second.thr;
            jb.fill = it->second.fill;
            jb.units = it->second.units;
        }
        if (solo) {
            sampler.peak = 0.0;
            sampler.armed = true;
            run_job(jb, precision);
            sampler.armed = false;
            jb.peak_bytes = std::max(0.0, sampler.peak.load() - idle);
            jb.t_done = now_s();
            continue;
        }
        // wait for the arrival time, then for room under the budget
        const double wait = jb.arrival - now_s();
        if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(wait));
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_done.wait(lk, [&]() { return running == 0 || in_use + jb.need_bytes <= budget; });
            in_use += jb.need_bytes;
            peak = std::max(peak, ++running);
        }
        ++admitted;
        push(&jb, T_OPEN);
    }
    if (!solo) {
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_done.wait(lk, [&]() { return finished == admitted; });
        }
        stop_pool();
    }
    sampler.finish();
    const double wall = now_s();
    std::vector<float> all, turnaround;
    double bodysteps = 0.0, step_s = 0.0;
    int failed = 0;
    for (const Job& jb : jobs) {
        all.insert(all.end(), jb.step_ms.begin(), jb.step_ms.end());
        bodysteps += (double)jb.n * (double)jb.step_ms.size();
        for (float ms : jb.step_ms) step_s += ms * 1e-3;
        if (jb.status != OGX_OK && !jb.rejected) ++failed;
        if (!jb.rejected && !solo) turnaround.push_back((float)(jb.t_done - jb.arrival));
    }
    // wall_s runs from the first arrival to the last job's end and includes every
    // job's set-up (initial conditions, first force evaluation) and, in served mode,
    // the gaps between arrivals; the stepping-only figure divides by the summed step
    // times instead (meaningful alone, where steps do not overlap)
    std::printf("{\"mode\": \"%s\", \"precision\": \"%s\", \"jobs\": %d, \"failed\": %d, \"rejected\": %d, "
                "\"steps\": %zu, \"workers\": %d, \"wall_s\": %.3f, \"warmup_s\": %.3f, \"bodies_steps_per_s\": %.6e, "
                "\"stepping_only_bodies_steps_per_s\": %s, \"p50_step_ms\": %.3f, \"p99_step_ms\": %.3f, "
                "\"job_turnaround_s_p50\": %s, \"job_turnaround_s_p99\": %s, "
                "\"peak_concurrent\": %d, \"hbm_budget_gb\": %.1f, \"capture\": %s, \"jobs_detail\": [",
                solo ? "solo" : "served", precision == OGX_PREC_FP64 ? "fp64" : precision == OGX_PREC_FP64_ROT ? "fp64rot" : "mixed", njobs, failed, rejected,
                all.size(), solo ? 1 : workers, wall, warmup_s, bodysteps / wall,
                solo ? std::to_string(step_s > 0 ? bodysteps / step_s : 0.0).c_str() : "null", percentile(all, 0.5),
                percentile(all, 0.99), solo ? "null" : std::to_string(percentile(turnaround, 0.5)).c_str(),
                solo ? "null" : std::to_string(percentile(turnaround, 0.99)).c_str(), solo ? 1 : peak, hbm_gb,
                g_capture ? "true" : "false");
    for (size_t j = 0; j < jobs.size(); ++j) {
        const Job& jb = jobs[j];
        std::printf("%s{\"id\": %d, \"n\": %lld, \"p\": %d, \"thr\": %d, \"m2l_tile_targets\": %d, \"near_units\": %d, "
                    "\"tuned_from_cache\": %s, \"steps\": %d, \"kind\": \"%s\", "
                    "\"status\": %d, \"rejected\": %s, \"need_mb\": %.1f, \"peak_mb\": %.1f, \"step_ms_p50\": %.3f, "
                    "\"digest\": \"%016llx\"}",
                    j ? ", " : "", jb.id, (long long)jb.n, jb.p, jb.thr, jb.fill, jb.units,
                    jb.tuned_from_cache ? "true" : "false", jb.steps,
                    jb.kind ? "disk+bulge merger" : "plummer", jb.status, jb.rejected ? "true" : "false",
                    jb.need_bytes / 1e6, jb.peak_bytes / 1e6, percentile(jb.step_ms, 0.5),
                    (unsigned long long)jb.digest);
    }
    std::printf("]}\n");
    if (autotune && !tune_cache.empty()) write_tune_cache(tune_cache, tcache);
    return failed ? 1 : 0;
}
