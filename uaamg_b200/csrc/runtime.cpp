// Batched solves and the serving loop of the C-ABI (include/uaamg.h,
// uaamg_solve_batch and uaamg_server_*).  Both run many independent engines on
// one GPU at once: every problem owns an engine (hierarchy + CG state), device
// staging buffers and a stream, and one host thread advances all of them through
// the engine's staged solve (solve_begin / solve_step / solve_poll / solve_end),
// so the problems' two-iteration CUDA graphs overlap on the device.
//
// There is no counterpart in the reference: its solvers run one problem at a time
// on the legacy default stream (src/solver/cuda/cuda_pcg_solver.cu:21-63).  Each
// problem's kernels, launch order and reductions are the ones uaamg_solve issues,
// so a problem's result does not depend on what runs beside it.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "handle.h"

namespace uaamg {
namespace {

using Clock = std::chrono::steady_clock;

double ms_since(Clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

size_t padded_cells(int dim, int nx, int ny, int nz) {
    return (size_t)(nx + 2) * (ny + 2) * (dim == 3 ? (size_t)(nz + 2) : 1);
}

// Device problem: an engine with its mask, FP64 right-hand side and pressure
// staging buffers (reference layout) and a stream.
struct DevProblem {
    Engine* eng = nullptr;
    int prec = -1, dim = 0, nx = 0, ny = 0, nz = 0, dirichlet = 0;
    double dx = 0, dy = 0, dz = 0;
    size_t n = 0;
    uint8_t* d_solid = nullptr;
    double* d_rhs = nullptr;
    double* d_p = nullptr;
    cudaStream_t stream = nullptr;
    bool built = false;
    std::vector<uint8_t> mask;  // host copy of the mask the hierarchy was built for

    size_t bytes() const { return (eng ? eng->device_bytes() : 0) + n * (1 + 16); }

    void release() {
        if (stream) cudaStreamSynchronize(stream);
        delete eng;
        eng = nullptr;
        cudaFree(d_solid);
        cudaFree(d_rhs);
        cudaFree(d_p);
        d_solid = nullptr;
        d_rhs = d_p = nullptr;
        if (stream) cudaStreamDestroy(stream);
        stream = nullptr;
        built = false;
        mask.clear();
        n = 0;
        prec = -1;
    }

    bool same_shape(int p, int d, int x, int y, int z, double hx, double hy, double hz,
                    int dir) const {
        return eng && prec == p && dim == d && nx == x && ny == y && (d == 2 || nz == z) &&
               dx == hx && dy == hy && (d == 2 || dz == hz) && dirichlet == dir;
    }

    // Allocates for the shape (keeps what matches).  Returns an engine error code.
    int prepare(int p, int d, int x, int y, int z, double hx, double hy, double hz, int dir) {
        if (same_shape(p, d, x, y, z, hx, hy, hz, dir)) return E_OK;
        release();
        prec = p; dim = d; nx = x; ny = y; nz = d == 3 ? z : 0;
        dx = hx; dy = hy; dz = d == 3 ? hz : 1.0; dirichlet = dir;
        n = padded_cells(d, x, y, z);
        if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess) {
            cudaGetLastError();
            stream = nullptr;
            return E_CUDA;
        }
        if (cudaMalloc(&d_solid, n) != cudaSuccess || cudaMalloc(&d_rhs, n * 8) != cudaSuccess ||
            cudaMalloc(&d_p, n * 8) != cudaSuccess) {
            cudaGetLastError();
            return E_OOM;
        }
        eng = p == PREC_FP64 ? create_engine_f64() : create_engine_f32(p == PREC_MIXED);
        if (!eng) return E_OOM;
        eng->set_stream(stream);
        return E_OK;
    }

    // Mask upload + hierarchy (blocking on the problem's stream); kept, with the
    // engine's captured CUDA graph, while the mask does not change (as the
    // reference's GPU adapter re-uploads its mask only on a resize,
    // cuda_pcg_solver.cu:45-49).
    int build(const uint8_t* solid_host) {
        if (built && mask.size() == n && std::memcmp(mask.data(), solid_host, n) == 0) return E_OK;
        if (cudaMemcpyAsync(d_solid, solid_host, n, cudaMemcpyHostToDevice, stream) != cudaSuccess)
            return E_CUDA;
        built = false;
        int e = eng->set_problem(dim, nx, ny, nz, dx, dy, dz, d_solid, dirichlet);
        if (e == E_OK) {
            built = true;
            mask.assign(solid_host, solid_host + n);
        }
        return e;
    }

    SolveArgs args(const uaamg_options& o) const {
        SolveArgs a;
        a.rhs = d_rhs;
        a.x = d_p;
        a.max_iter = o.max_iter;
        a.tol = o.tol;
        a.tol_mode = o.tol_mode;
        a.warm = o.warm_start;
        a.replace_every = o.replace_every;
        a.project_mean = o.project_mean;
        a.precond = o.preconditioner;
        a.hist = nullptr;
        a.ref_solid = d_solid;
        return a;
    }
};

// Smoothing schedule of a batch problem chosen by the autotuner: the fastest of
// V(1,1) (the reference's), V(1,1) on the finest level with V(2,2) below, and
// V(2,2), timed as a full solve of the problem itself (the second of two, after the
// graph capture), among those that converge; cached per GPU, precision, shape and
// solid fraction (to 0.05).  The problem's right-hand side must be on the device.
std::vector<int> tune_schedule(DevProblem& d, const uaamg_problem& p, const uaamg_options& o) {
    size_t solid = 0, inner = 0;
    for (int k = (p.dim == 3 ? 1 : 0); k <= (p.dim == 3 ? p.nz : 0); ++k)
        for (int j = 1; j <= p.ny; ++j)
            for (int i = 1; i <= p.nx; ++i) {
                solid += p.solid[i + (size_t)(p.nx + 2) * (j + (size_t)(p.ny + 2) * k)] != 0;
                ++inner;
            }
    const int bucket = (int)(20.0 * (double)solid / (double)(inner ? inner : 1) + 0.5);
    const std::string key = "nu|" + tune_gpu_id() + "|" +
                            (o.precision == PREC_MIXED ? "mixed" : "f32") + "|" + std::to_string(p.dim) +
                            "|" + std::to_string(p.nx) + "x" + std::to_string(p.ny) + "x" +
                            std::to_string(p.dim == 3 ? p.nz : 0) + "|s" + std::to_string(bucket);
    std::vector<int> best;
    if (tune_lookup(key, &best) && best.size() == 2) return best;
    const int cand[3][2] = {{1, 1}, {1, 2}, {2, 2}};
    double best_ms = 1e300;
    best = {1, 1};
    for (const auto& c : cand) {
        d.eng->set_smoothing(c[0], c[1]);
        double ms = 0.0;
        bool ok = true;
        for (int rep = 0; rep < 2 && ok; ++rep) {
            cudaMemsetAsync(d.d_p, 0, d.n * sizeof(double), d.stream);
            cudaStreamSynchronize(d.stream);
            const auto t0 = Clock::now();
            SolveResult r;
            std::memset(&r, 0, sizeof(r));
            ok = d.eng->solve(d.args(o), &r) == E_OK && r.status == CG_CONVERGED;
            ms = ms_since(t0);
        }
        if (ok && ms < best_ms) {
            best_ms = ms;
            best = {c[0], c[1]};
        }
    }
    tune_store(key, best);
    return best;
}

// The small problems of a batch replayed as ONE CUDA graph per step
// (uaamg_set_batch_group): the graph forks to every member's stream, queues its two
// PCG iterations and the copy of its 'done' flag, and joins; two such graphs (one
// per flag buffer) keep two steps in flight.  Finished members' kernels return at
// once, so the graph keeps issuing them until every member has stopped.
struct GroupGraph {
    std::vector<int> members;
    cudaStream_t master = nullptr;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> joins;
    int* flags = nullptr;  // pinned, 2 x members
    int launched = 0, seen = 0, max_steps = 0;
    bool done = false;

    void release() {
        if (master) cudaStreamSynchronize(master);
        for (auto& x : exec) if (x) { cudaGraphExecDestroy(x); x = nullptr; }
        for (auto& e : ev) if (e) { cudaEventDestroy(e); e = nullptr; }
        if (fork) { cudaEventDestroy(fork); fork = nullptr; }
        for (auto& e : joins) if (e) cudaEventDestroy(e);
        joins.clear();
        if (flags) { cudaFreeHost(flags); flags = nullptr; }
        if (master) { cudaStreamDestroy(master); master = nullptr; }
        members.clear();
    }

    // After every member's solve_begin.  Returns false if the graph could not be
    // made (the members then run on their own graphs).
    bool build(std::vector<DevProblem>& slots, const std::vector<int>& m, int max_iter) {
        members = m;
        const int G = (int)m.size();
        max_steps = (max_iter + 1) / 2 + 1;
        if (cudaStreamCreateWithFlags(&master, cudaStreamNonBlocking) != cudaSuccess ||
            cudaHostAlloc(&flags, 2 * G * sizeof(int), cudaHostAllocDefault) != cudaSuccess ||
            cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        std::memset(flags, 0, 2 * G * sizeof(int));
        joins.assign(G, nullptr);
        for (auto& e : joins)
            if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return false;
        // the first launch follows every member's set-up work
        for (int k = 0; k < G; ++k) {
            cudaEventRecord(joins[k], slots[m[k]].stream);
            cudaStreamWaitEvent(master, joins[k], 0);
        }
        for (int slot = 0; slot < 2; ++slot) {
            cudaGraph_t g = nullptr;
            if (cudaStreamBeginCapture(master, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return false;
            cudaEventRecord(fork, master);
            for (int k = 0; k < G; ++k) {
                DevProblem& d = slots[m[k]];
                cudaStreamWaitEvent(d.stream, fork, 0);
                d.eng->enqueue_step(d.stream, &flags[slot * G + k]);
                cudaEventRecord(joins[k], d.stream);
                cudaStreamWaitEvent(master, joins[k], 0);
            }
            if (cudaStreamEndCapture(master, &g) != cudaSuccess || !g) {
                cudaGetLastError();
                return false;
            }
            const cudaError_t ce = cudaGraphInstantiate(&exec[slot], g, 0);
            cudaGraphDestroy(g);
            if (ce != cudaSuccess) {
                cudaGetLastError();
                exec[slot] = nullptr;
                return false;
            }
        }
        return true;
    }

    // Non-blocking: keeps two steps in flight and reads the flags of the oldest one.
    int advance() {
        const int G = (int)members.size();
        while (!done && launched - seen < 2 && launched < max_steps) {
            const int s = launched & 1;
            if (cudaGraphLaunch(exec[s], master) != cudaSuccess) return E_CUDA;
            cudaEventRecord(ev[s], master);
            ++launched;
        }
        if (seen < launched) {
            const cudaError_t q = cudaEventQuery(ev[seen & 1]);
            if (q == cudaErrorNotReady) return E_OK;
            if (q != cudaSuccess) return E_CUDA;
            bool all = true;
            for (int k = 0; k < G; ++k) all = all && flags[(seen & 1) * G + k] != 0;
            ++seen;
            if (all || seen >= max_steps) done = true;
        }
        return E_OK;
    }

    // Once done: every member's stream follows the last step launched.
    void join(std::vector<DevProblem>& slots) {
        cudaEventRecord(fork, master);
        for (int i : members) cudaStreamWaitEvent(slots[i].stream, fork, 0);
    }
};

}  // namespace
}  // namespace uaamg

// Per-problem slots of uaamg_solve_batch, kept on the handle between calls.
struct BatchPool {
    std::vector<uaamg::DevProblem> slots;
};

namespace uaamg {
namespace api {

void free_batch(uaamg_handle* h) {
    if (!h || !h->batch) return;
    for (auto& s : h->batch->slots) s.release();
    delete h->batch;
    h->batch = nullptr;
}

}  // namespace api
}  // namespace uaamg

extern "C" {

uaamg_status uaamg_solve_batch(uaamg_handle* h, int n, const uaamg_problem* probs,
                               const uaamg_options* o, uaamg_stats* stats) {
    using namespace uaamg;
    using api::fail;
    if (!h) return UAAMG_INVALID_ARG;
    if (n < 0 || (n > 0 && !probs)) return fail(h, UAAMG_INVALID_ARG, "batch: bad problem list");
    uaamg_options opts;
    uaamg_default_options(&opts);
    if (o) opts = *o;
    if (opts.max_iter < 0 || !(opts.tol >= 0) || opts.tol_mode < 0 || opts.tol_mode > 1 ||
        opts.precision < 0 || opts.precision > 2)
        return fail(h, UAAMG_INVALID_ARG, "batch: bad options");
    for (int i = 0; i < n; ++i) {
        const uaamg_problem& p = probs[i];
        const int nz = p.dim == 3 ? p.nz : 2;
        if ((p.dim != 2 && p.dim != 3) || p.nx < 2 || p.ny < 2 || nz < 2 || !p.solid || !p.rhs ||
            !p.p || !(p.dx > 0) || !(p.dy > 0) || (p.dim == 3 && !(p.dz > 0)) ||
            padded_cells(p.dim, p.nx, p.ny, p.nz) >= ((size_t)1 << 31))
            return fail(h, UAAMG_INVALID_ARG, "batch: problem " + std::to_string(i) + " is invalid");
    }
    cudaSetDevice(h->device);
    if (!h->batch) h->batch = new (std::nothrow) BatchPool();
    if (!h->batch) return fail(h, UAAMG_OOM, "batch: pool allocation failed");
    auto& slots = h->batch->slots;
    if ((int)slots.size() < n) slots.resize(n);
    const auto t0 = Clock::now();
    // set-up: buffers, mask, hierarchy, right-hand side and the first stage
    for (int i = 0; i < n; ++i) {
        const uaamg_problem& p = probs[i];
        DevProblem& d = slots[i];
        int e = d.prepare(opts.precision, p.dim, p.nx, p.ny, p.nz, p.dx, p.dy, p.dz, h->dirichlet);
        if (e == E_OK) {
            uaamg::api::apply_vcycle_mode(d.eng, h->sweeps);
            d.eng->set_autotune(h->autotune != 0);
            e = d.build(p.solid);
        }
        if (e != E_OK) {
            const uaamg_status s =
                api::map_engine(h, e, ("batch: problem " + std::to_string(i) + " set-up").c_str(), d.eng);
            d.release();
            return s;
        }
        cudaMemcpyAsync(d.d_rhs, p.rhs, d.n * 8, cudaMemcpyHostToDevice, d.stream);
        if (h->autotune && opts.precision != PREC_FP64) {
            const std::vector<int> nu = tune_schedule(d, p, opts);
            d.eng->set_smoothing(nu[0], nu[1]);
        } else {
            d.eng->set_smoothing(h->nu_fine, h->nu_coarse);
        }
        // as uaamg_solve: the result is accumulated into the caller's p
        cudaMemcpyAsync(d.d_p, p.p, d.n * 8, cudaMemcpyHostToDevice, d.stream);
        if ((e = d.eng->solve_begin(d.args(opts))) != E_OK)
            return api::map_engine(h, e, "batch: solve", d.eng);
    }
    // optional: the problems of at most batch_group_cells padded cells share one graph
    GroupGraph grp;
    std::vector<char> grouped(n, 0);
    if (h->batch_group_cells > 0) {
        std::vector<int> m;
        for (int i = 0; i < n; ++i)
            if ((long long)slots[i].n <= h->batch_group_cells) m.push_back(i);
        if (m.size() >= 2 && grp.build(slots, m, opts.max_iter)) {
            for (int i : m) grouped[i] = 1;
        } else {
            grp.release();
        }
    }
    // advance every unfinished problem: keep two steps queued, collect finished ones
    std::vector<char> open(n, 1);
    int left = n;
    uaamg_status first_bad = UAAMG_OK;
    bool group_joined = false;
    while (left > 0) {
        bool progressed = false;
        if (!grp.members.empty() && !grp.done) {
            const int seen = grp.seen;
            if (grp.advance() != E_OK) {
                grp.release();
                return api::fail(h, UAAMG_CUDA_ERROR, "batch: grouped graph launch");
            }
            progressed = grp.seen != seen;
        }
        if (grp.done && !group_joined) {
            grp.join(slots);
            group_joined = true;
        }
        for (int i = 0; i < n; ++i) {
            if (!open[i]) continue;
            DevProblem& d = slots[i];
            bool stopped = false;
            int e = E_OK;
            if (grouped[i]) {
                stopped = group_joined;
            } else {
                e = d.eng->solve_step();
                if (e == E_OK) e = d.eng->solve_poll(false, &stopped);
            }
            if (e != E_OK) return api::map_engine(h, e, "batch: solve", d.eng);
            if (!stopped) continue;
            SolveResult r;
            std::memset(&r, 0, sizeof(r));
            if ((e = d.eng->solve_end(&r)) != E_OK) return api::map_engine(h, e, "batch: solve", d.eng);
            if (d.eng->timed_out())
                return fail(h, UAAMG_TIMEOUT, "batch: a kernel gave up waiting for its tile loads");
            cudaError_t ce = cudaMemcpyAsync(probs[i].p, d.d_p, d.n * 8, cudaMemcpyDeviceToHost, d.stream);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(d.stream);
            if (ce != cudaSuccess) return api::cuda_fail(h, ce, "batch: download");
            uaamg_stats st_local;
            const uaamg_status s = api::fill_stats(d.eng, r, &st_local);
            st_local.solve_ms = ms_since(t0);
            if (stats) stats[i] = st_local;
            if (s != UAAMG_OK && first_bad == UAAMG_OK) first_bad = s;
            open[i] = 0;
            --left;
            progressed = true;
        }
        if (!progressed) std::this_thread::yield();
    }
    grp.release();
    return first_bad;
}

uaamg_status uaamg_set_batch_group(uaamg_handle* h, long long max_cells) {
    if (!h || max_cells < 0) return UAAMG_INVALID_ARG;
    h->batch_group_cells = max_cells;
    return UAAMG_OK;
}

uaamg_status uaamg_set_autotune(uaamg_handle* h, int on) {
    if (!h) return UAAMG_INVALID_ARG;
    h->autotune = on ? 1 : 0;
    for (auto* e : h->eng)
        if (e) e->set_autotune(on != 0);
    for (int q = 0; q < 3; ++q) h->ready[q] = false;  // re-tune at the next set-up
    return UAAMG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Serving loop.

namespace uaamg {
namespace {

// One simulation id resident on the device: its engine and mask, and in d_p the
// FP64 pressure of its last request (the next request's warm start).
struct SimState {
    DevProblem dp;
    std::vector<uint8_t> mask;
    bool has_p = false;
    bool busy = false;
    uint64_t last_used = 0;
    size_t bytes = 0;
};

struct Ticket {
    long long id = 0;
    uaamg_request req{};
    std::vector<uint8_t> solid;
    std::vector<double> rhs;
    Clock::time_point t_submit, t_admit;
    uaamg_result res{};
    bool done = false;
    int slot = -1;
    SimState* sim = nullptr;
    bool ending = false;     // exit work queued; waiting for the slot's event
    int status = UAAMG_OK;   // result status once collected (the pressure copy may follow)
    const double* rhs_ptr = nullptr;  // the right-hand side: rhs.data(), or the caller's
    bool borrow = false;              // UAAMG_REQUEST_BORROW: rhs and p_out are the caller's
};

// Pinned host staging of one concurrent solve, and the event recorded behind its
// exit work and pressure copy.
struct StageBuf {
    double* h = nullptr;
    size_t cap = 0;
    bool used = false;
    cudaEvent_t ev = nullptr;
    bool ensure(size_t n) {
        if (!ev && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            ev = nullptr;
            return false;
        }
        if (n <= cap) return true;
        if (h) cudaFreeHost(h);
        h = nullptr;
        cap = 0;
        if (cudaHostAlloc(&h, n * sizeof(double), cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        cap = n;
        return true;
    }
};

// Device bytes a new id of this shape is expected to hold (engine + staging),
// used for admission before its hierarchy exists.
size_t estimate_bytes(int prec, int dim, int nx, int ny, int nz) {
    const size_t n = padded_cells(dim, nx, ny, nz);
    return n * (prec == PREC_FP64 ? 200 : 120);
}

}  // namespace
}  // namespace uaamg

struct uaamg_server {
    uaamg_server_config cfg{};
    std::thread worker;
    std::mutex mu;
    std::condition_variable cv;
    bool stopping = false;
    long long next_ticket = 1;
    long long outstanding = 0;  // submitted, not finished
    long long completed = 0;
    std::deque<uaamg::Ticket*> pending;
    std::unordered_map<long long, uaamg::Ticket*> tickets;
    // worker-owned (the counters below are also updated under mu for info)
    std::unordered_map<long long, uaamg::SimState*> sims;
    std::vector<uaamg::Ticket*> active;
    std::vector<uaamg::StageBuf> stage;
    // results whose pressure is copied into the caller's p_out by the completion
    // thread (from the pinned staging), so the worker never waits on a host copy
    std::thread completer;
    std::condition_variable cv_copy;
    std::deque<uaamg::Ticket*> to_copy;  // under mu
    std::deque<uaamg::Ticket*> copied;   // under mu; the worker finishes them
    int copying = 0;                     // under mu: handed over, not yet finished
    bool stop_copier = false;
    size_t resident_bytes = 0;
    int resident = 0;
    uint64_t tick = 0;
};

namespace uaamg {
namespace {

void release_sim(uaamg_server* s, SimState* sim) {
    sim->dp.release();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->resident_bytes -= sim->bytes;
        s->resident -= 1;
    }
    delete sim;
}

// Evicts idle ids, least recently used first, until `need` more bytes fit in the
// budget.  False when the idle ids are not enough.
bool make_room(uaamg_server* s, size_t need) {
    while (s->resident_bytes + need > s->cfg.hbm_budget_bytes) {
        auto victim = s->sims.end();
        for (auto it = s->sims.begin(); it != s->sims.end(); ++it)
            if (!it->second->busy &&
                (victim == s->sims.end() || it->second->last_used < victim->second->last_used))
                victim = it;
        if (victim == s->sims.end()) return false;
        SimState* sim = victim->second;
        s->sims.erase(victim);
        release_sim(s, sim);
    }
    return true;
}

void finish(uaamg_server* s, Ticket* t, int status) {
    t->res.ticket = t->id;
    t->res.sim_id = t->req.sim_id;
    t->res.status = status;
    t->res.latency_ms = ms_since(t->t_submit);
    if (t->slot >= 0) s->stage[t->slot].used = false;
    t->slot = -1;
    if (t->sim) {
        t->sim->busy = false;
        t->sim->last_used = ++s->tick;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    t->done = true;
    s->outstanding -= 1;
    s->completed += 1;
    s->cv.notify_all();
}

// Starts an admitted request: its id's hierarchy (reused when the shape and mask
// match), the right-hand side upload and the first solve stage.  Returns false if
// it must wait (no device room yet).
bool start_request(uaamg_server* s, Ticket* t) {
    const uaamg_request& q = t->req;
    const uaamg_server_config& c = s->cfg;
    int slot = -1;
    for (int i = 0; i < (int)s->stage.size(); ++i)
        if (!s->stage[i].used) { slot = i; break; }
    if (slot < 0) return false;  // every staging slot busy: wait for a finishing request
    SimState* sim = nullptr;
    auto it = s->sims.find(q.sim_id);
    if (it != s->sims.end()) {
        sim = it->second;
        if (!sim->dp.same_shape(c.precision, q.dim, q.nx, q.ny, q.nz, q.dx, q.dy, q.dz, 0) ||
            sim->mask != t->solid) {
            s->sims.erase(it);
            release_sim(s, sim);
            sim = nullptr;
        }
    }
    bool warm = false;
    if (!sim) {
        const size_t need = estimate_bytes(c.precision, q.dim, q.nx, q.ny, q.nz);
        if (!make_room(s, need) && !s->active.empty()) return false;
        sim = new (std::nothrow) SimState();
        if (!sim) { finish(s, t, UAAMG_OOM); return true; }
        int e = sim->dp.prepare(c.precision, q.dim, q.nx, q.ny, q.nz, q.dx, q.dy, q.dz, 0);
        if (e == E_OK) e = sim->dp.build(t->solid.data());
        if (e != E_OK) {
            sim->dp.release();
            delete sim;
            finish(s, t, e == E_OOM ? UAAMG_OOM : UAAMG_CUDA_ERROR);
            return true;
        }
        sim->mask = t->solid;
        sim->bytes = sim->dp.bytes();
        s->sims[q.sim_id] = sim;
        std::lock_guard<std::mutex> lk(s->mu);
        s->resident_bytes += sim->bytes;
        s->resident += 1;
    } else {
        warm = c.warm_start && sim->has_p;
    }
    if (!s->stage[slot].ensure(sim->dp.n)) { finish(s, t, UAAMG_OOM); return true; }
    StageBuf& b = s->stage[slot];
    b.used = true;
    t->slot = slot;
    t->sim = sim;
    sim->busy = true;
    DevProblem& d = sim->dp;
    if (t->borrow) {  // straight from the caller's buffer
        cudaMemcpyAsync(d.d_rhs, t->rhs_ptr, d.n * sizeof(double), cudaMemcpyHostToDevice, d.stream);
    } else {
        std::memcpy(b.h, t->rhs_ptr, d.n * sizeof(double));
        cudaMemcpyAsync(d.d_rhs, b.h, d.n * sizeof(double), cudaMemcpyHostToDevice, d.stream);
    }
    if (!warm) cudaMemsetAsync(d.d_p, 0, d.n * sizeof(double), d.stream);
    uaamg_options o;
    uaamg_default_options(&o);
    o.precision = c.precision;
    o.tol = c.tol;
    o.tol_mode = UAAMG_TOL_REL;
    o.max_iter = c.max_iter;
    o.replace_every = c.replace_every;
    o.warm_start = warm ? 1 : 0;
    t->res.warm = warm ? 1 : 0;
    t->t_admit = Clock::now();
    t->res.wait_ms = std::chrono::duration<double, std::milli>(t->t_admit - t->t_submit).count();
    if (d.eng->solve_begin(d.args(o)) != E_OK) {
        sim->has_p = false;
        finish(s, t, UAAMG_CUDA_ERROR);
        return true;
    }
    s->active.push_back(t);
    return true;
}

// Advances one running request without blocking; true when it leaves the active
// list (finished, or handed to the completion thread for its pressure copy).  A
// stopped solve first queues its exit work and the pressure's device-to-host copy
// into the slot's pinned staging, with the slot's event behind them; the result
// is collected on a later pass, once the event reports done.
bool advance(uaamg_server* s, Ticket* t) {
    DevProblem& d = t->sim->dp;
    StageBuf& b = s->stage[t->slot];
    if (!t->ending) {
        bool stopped = false;
        int e = d.eng->solve_step();
        if (e == E_OK) e = d.eng->solve_poll(false, &stopped);
        if (e == E_OK && !stopped) return false;
        if (e == E_OK) e = d.eng->solve_end_enqueue();
        cudaError_t ce = cudaSuccess;
        if (e == E_OK && t->req.p_out)
            ce = cudaMemcpyAsync(t->borrow ? t->req.p_out : b.h, d.d_p, d.n * sizeof(double),
                                 cudaMemcpyDeviceToHost, d.stream);
        if (e == E_OK && ce == cudaSuccess) ce = cudaEventRecord(b.ev, d.stream);
        if (e != E_OK || ce != cudaSuccess) {
            t->sim->has_p = false;
            finish(s, t, UAAMG_CUDA_ERROR);
            return true;
        }
        t->ending = true;
        return false;
    }
    const cudaError_t q = cudaEventQuery(b.ev);
    if (q == cudaErrorNotReady) return false;
    SolveResult r;
    std::memset(&r, 0, sizeof(r));
    int e = q == cudaSuccess ? d.eng->solve_end_collect(&r) : E_CUDA;
    if (e != E_OK || d.eng->timed_out()) {
        t->sim->has_p = false;
        finish(s, t, e == E_OK ? UAAMG_TIMEOUT : UAAMG_CUDA_ERROR);
        return true;
    }
    uaamg_stats st;
    t->status = api::fill_stats(d.eng, r, &st);
    t->res.iterations = st.iterations;
    t->res.rel_residual = st.rel_residual;
    t->sim->has_p = true;
    if (!t->req.p_out || t->borrow) {  // nothing to copy on the host
        finish(s, t, t->status);
        return true;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->to_copy.push_back(t);
    s->copying += 1;
    s->cv_copy.notify_one();
    return true;
}

// Completion thread: copies finished pressures from the pinned staging into the
// callers' p_out; the worker then finishes those tickets (slot and id released).
void copier_main(uaamg_server* s) {
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_copy.wait(lk, [&] { return s->stop_copier || !s->to_copy.empty(); });
        if (s->to_copy.empty()) return;  // stop_copier and nothing left
        Ticket* t = s->to_copy.front();
        s->to_copy.pop_front();
        lk.unlock();
        std::memcpy(t->req.p_out, s->stage[t->slot].h, t->sim->dp.n * sizeof(double));
        lk.lock();
        s->copied.push_back(t);
        s->cv.notify_all();
    }
}

void worker_main(uaamg_server* s) {
    cudaSetDevice(s->cfg.device);
    for (;;) {
        // results whose pressure copy the completion thread has finished
        std::deque<Ticket*> done_copies;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            done_copies.swap(s->copied);
            s->copying -= (int)done_copies.size();
        }
        for (Ticket* t : done_copies) finish(s, t, t->status);
        // admission: FIFO over the queue; a request waits while its id is busy
        std::vector<Ticket*> admit;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (s->pending.empty() && s->active.empty()) {
                if (s->stopping && s->copying == 0) break;
                s->cv.wait(lk, [&] {
                    return (s->stopping && s->copying == 0) || !s->pending.empty() ||
                           !s->copied.empty();
                });
                continue;
            }
            // a result waiting for its host copy still holds its staging slot
            int room = s->cfg.max_active - (int)s->active.size() - s->copying;
            std::vector<long long> blocked;
            for (auto it = s->pending.begin(); it != s->pending.end() && room > 0;) {
                Ticket* t = *it;
                const long long id = t->req.sim_id;
                auto sim = s->sims.find(id);
                bool busy = sim != s->sims.end() && sim->second->busy;
                for (long long b : blocked) busy = busy || b == id;
                for (Ticket* a : admit) busy = busy || a->req.sim_id == id;
                if (busy) {
                    blocked.push_back(id);
                    ++it;
                    continue;
                }
                admit.push_back(t);
                it = s->pending.erase(it);
                --room;
            }
        }
        for (size_t i = 0; i < admit.size(); ++i) {
            if (!start_request(s, admit[i])) {
                // no device room until a running solve finishes: back to the queue front
                std::lock_guard<std::mutex> lk(s->mu);
                for (size_t j = admit.size(); j > i; --j) s->pending.push_front(admit[j - 1]);
                break;
            }
        }
        bool progressed = !admit.empty();
        for (size_t i = 0; i < s->active.size();) {
            if (advance(s, s->active[i])) {
                s->active.erase(s->active.begin() + (long)i);
                progressed = true;
            } else {
                ++i;
            }
        }
        if (!progressed) std::this_thread::yield();
    }
}

}  // namespace
}  // namespace uaamg

extern "C" {

void uaamg_server_default_config(uaamg_server_config* c) {
    if (!c) return;
    c->device = 0;
    c->precision = UAAMG_MIXED;
    c->tol = 1e-6;
    c->max_iter = 500;
    c->replace_every = 10;
    c->warm_start = 1;
    c->max_active = 16;
    c->hbm_budget_bytes = (size_t)150 << 30;
}

uaamg_status uaamg_server_start(uaamg_server** out, const uaamg_server_config* cfg) {
    if (!out) return UAAMG_INVALID_ARG;
    *out = nullptr;
    uaamg_server_config c;
    uaamg_server_default_config(&c);
    if (cfg) c = *cfg;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || c.device < 0 || c.device >= count) {
        cudaGetLastError();
        return UAAMG_INVALID_ARG;
    }
    if (c.precision < 0 || c.precision > 2 || c.max_active < 1 || c.max_iter < 0 || !(c.tol >= 0) ||
        c.hbm_budget_bytes == 0)
        return UAAMG_INVALID_ARG;
    uaamg_server* s = new (std::nothrow) uaamg_server();
    if (!s) return UAAMG_OOM;
    s->cfg = c;
    s->stage.resize(c.max_active);
    s->completer = std::thread(uaamg::copier_main, s);
    s->worker = std::thread(uaamg::worker_main, s);
    *out = s;
    return UAAMG_OK;
}

uaamg_status uaamg_server_submit(uaamg_server* s, const uaamg_request* q, long long* ticket) {
    if (!s || !q || !ticket) return UAAMG_INVALID_ARG;
    const int nz = q->dim == 3 ? q->nz : 2;
    if ((q->dim != 2 && q->dim != 3) || q->nx < 2 || q->ny < 2 || nz < 2 || !q->solid || !q->rhs ||
        !(q->dx > 0) || !(q->dy > 0) || (q->dim == 3 && !(q->dz > 0)))
        return UAAMG_INVALID_ARG;
    const size_t n = uaamg::padded_cells(q->dim, q->nx, q->ny, q->nz);
    if (n >= ((size_t)1 << 31)) return UAAMG_INVALID_ARG;
    uaamg::Ticket* t = new (std::nothrow) uaamg::Ticket();
    if (!t) return UAAMG_OOM;
    t->req = *q;
    if (q->dim == 2) { t->req.nz = 0; t->req.dz = 1.0; }
    t->solid.assign(q->solid, q->solid + n);
    t->borrow = (q->flags & UAAMG_REQUEST_BORROW) != 0;
    if (t->borrow) {
        t->rhs_ptr = q->rhs;
    } else {
        t->rhs.assign(q->rhs, q->rhs + n);
        t->rhs_ptr = t->rhs.data();
    }
    t->req.solid = nullptr;
    t->req.rhs = nullptr;
    t->t_submit = uaamg::Clock::now();
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) { delete t; return UAAMG_INVALID_ARG; }
    t->id = s->next_ticket++;
    s->tickets[t->id] = t;
    s->pending.push_back(t);
    s->outstanding += 1;
    *ticket = t->id;
    s->cv.notify_all();
    return UAAMG_OK;
}

uaamg_status uaamg_server_poll(uaamg_server* s, long long ticket, uaamg_result* res, int* done) {
    if (!s || !done) return UAAMG_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return UAAMG_INVALID_ARG;
    uaamg::Ticket* t = it->second;
    *done = t->done ? 1 : 0;
    if (!t->done) return UAAMG_OK;
    if (res) *res = t->res;
    s->tickets.erase(it);
    delete t;
    return UAAMG_OK;
}

uaamg_status uaamg_server_drain(uaamg_server* s) {
    if (!s) return UAAMG_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv.wait(lk, [&] { return s->outstanding == 0; });
    return UAAMG_OK;
}

uaamg_status uaamg_server_info(uaamg_server* s, size_t* bytes, int* resident, long long* completed) {
    if (!s) return UAAMG_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (bytes) *bytes = s->resident_bytes;
    if (resident) *resident = s->resident;
    if (completed) *completed = s->completed;
    return UAAMG_OK;
}

uaamg_status uaamg_server_stop(uaamg_server* s) {
    if (!s) return UAAMG_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        s->cv.notify_all();
    }
    if (s->worker.joinable()) s->worker.join();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop_copier = true;
        s->cv_copy.notify_all();
    }
    if (s->completer.joinable()) s->completer.join();
    cudaSetDevice(s->cfg.device);
    for (auto& kv : s->sims) {
        kv.second->dp.release();
        delete kv.second;
    }
    s->sims.clear();
    for (auto& b : s->stage) {
        if (b.h) cudaFreeHost(b.h);
        if (b.ev) cudaEventDestroy(b.ev);
    }
    // every ticket not yet released by a poll is in the map (queued or finished)
    for (auto& kv : s->tickets) delete kv.second;
    delete s;
    return UAAMG_OK;
}

}  // extern "C"
