// Host orchestration of one precision mode of the B200 UAAMG-PCG engine
// (EngineT<double> = reference-exact FP64; EngineT<float> = plain FP32 or, with
// mixed = true, FP32 CG with FP64 residual replacement).  Included by exactly one
// translation unit per T, so the kernels it launches live in the same unit.
//
// Reference structure followed:
//   hierarchy   UAAMGPreconditioner3D::buildHierarchy / apply set-up
//               (uaamg_preconditioner_3d.cpp:11-32, 205-214), once per problem
//               here instead of once per apply
//   V-cycle     vCycle (uaamg_preconditioner_3d.cpp:183-196), iterative
//   PCG         PCG3D::solve (pcg_3d.cpp:18-125), every scalar device-resident
//
// Layout: every level array uses the pitched layout (common.cuh,
// make_geom_pitched); the caller's arrays use the reference layout and are
// converted on the way in (rhs, warm-start p, preconditioner input) and out.
#pragma once
#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include "engine.h"
#include "fused.cuh"
#include "kernels.cuh"
#include "tail.cuh"
#include "tma.cuh"
#include "vec.cuh"

namespace uaamg {
namespace {

template <class T, class CS>
struct LevelBuf {
    Geom g;
    double hx, hy, hz;
    uint8_t* solid = nullptr;
    T *cx = nullptr, *cy = nullptr, *cz = nullptr, *wd = nullptr, *dg = nullptr;
    CS *hcx = nullptr, *hcy = nullptr, *hcz = nullptr;  // couplings as the marches read them
    T *x = nullptr, *b = nullptr;  // level >= 1 only (level 0 uses the CG's r and z)
    uint8_t* code = nullptr;       // cell codes (vec.cuh k_codes)
    int zc = 2;                    // planes per block of the z marches (march.cuh)
    // FP32 couplings on a level of a mixed engine whose face counts exceed 2048 (3D
    // levels 6 and down, 2D levels 12 and down): FP16 holds integers exactly only up
    // to 2048 and overflows above 65504
    bool c32 = false;
    // plane-box tensor maps of the marches: b, x, codes, couplings, diagonal, and x
    // as the parent box read by the next-finer level's prolongation
    CUtensorMap mb, mx, mcode, mcx, mcy, mcz, mdg, mxq;
    // boxes with a 2-cell ring for the fused marches (fused.cuh): b, codes, diagonal,
    // couplings
    CUtensorMap fb, fcode, fdg, fcx, fcy, fcz;
    // small 3D levels: whole-tile boxes (fused.cuh k_level_box) and this level's x as
    // their parent box
    bool box = false;
    CUtensorMap bb, bcode, bdg, bcx, bcy, bcz, bxq;
    T* trim = nullptr;  // coarse box levels: per box {d, c_x, c_y, c_z} or d = 0 (k_box_trim)
};

// 3D levels of at most this many cells run the fused steps as whole-tile boxes
// (UAAMG_BOX_MAX_CELLS overrides it, for comparisons)
constexpr double kBoxCells = 64.0 * 64.0 * 64.0;

// Kernel classes for the in-situ per-kernel timing (uaamg_profile_solve).
enum KClass : int {
    K_SWEEP = 0, K_RESTRICT, K_PROLONG, K_COARSEST, K_PMATVEC, K_UPDATE, K_ZDOT, K_FWD, K_RES,
    K_UPE, K_UPO, K_TRUE_RESIDUAL, K_RHS, K_OUTPUT, K_CAST, K_SETUP, K_TAIL, K_REPLACE, K_DOWN,
    K_UP, K_NCLASS
};
static const char* const kclass_names[K_NCLASS] = {
    "rbgs_sweep", "restrict_residual", "prolong_add", "coarsest_solve", "p_matvec_dot",
    "cg_update", "z_dot", "smooth_fwd", "residual_restrict", "prolong_smooth_even",
    "smooth_odd", "true_residual", "rhs_prepare", "output", "cast", "hierarchy_setup",
    "small_levels", "residual_replacement", "level_down", "level_up"};

struct KTag {
    int cls;
    int level;
    double bytes;  // algorithmic (compulsory) bytes of this launch (K_REPLACE: of one
                   // launch that performs the replacement; most launches return at once)
};

// Kernel launch on the engine's stream.  Outside the per-kernel profiler every
// launch on a created stream (the CUDA-graph captures always use one) carries the
// programmatic-stream-serialisation attribute (the kernels begin with pdl_entry,
// common.cuh), so a kernel's launch and block scheduling overlap the end of the one
// before it; launches on the legacy default stream are plain.
#define UAAMG_LAUNCH_SMEM(tag, kern, grid, block, smem, ...)              \
    do {                                                                  \
        const KTag tg_ = (tag);                                           \
        cudaEvent_t e0_ = nullptr, e1_ = nullptr;                         \
        if (prof_on_) prof_begin(tg_, &e0_, &e1_);                        \
        if (pdl_ && !nopdl_next_ && !prof_on_ && st_ != nullptr) {        \
            cudaLaunchConfig_t cf_ = {};                                  \
            cudaLaunchAttribute at_[1];                                   \
            at_[0].id = cudaLaunchAttributeProgrammaticStreamSerialization; \
            at_[0].val.programmaticStreamSerializationAllowed = 1;        \
            cf_.gridDim = dim3(grid);                                     \
            cf_.blockDim = dim3(block);                                   \
            cf_.dynamicSmemBytes = (smem);                                \
            cf_.stream = st_;                                             \
            cf_.attrs = at_;                                              \
            cf_.numAttrs = 1;                                             \
            cudaLaunchKernelEx(&cf_, kern, __VA_ARGS__);                  \
        } else {                                                          \
            kern<<<(grid), (block), (smem), st_>>>(__VA_ARGS__);          \
        }                                                                 \
        if (prof_on_) cudaEventRecord(e1_, st_);                          \
        nopdl_next_ = false;                                              \
        ++launches_;                                                      \
    } while (0)
#define UAAMG_LAUNCH(tag, kern, grid, block, ...) \
    UAAMG_LAUNCH_SMEM(tag, kern, grid, block, 0, __VA_ARGS__)

// CS: storage type of the coarse-level couplings the marches read (T, or __half
// in the mixed form: face counts with a per-axis scale).
template <class T, class CS = T>
class EngineT final : public Engine {
    static constexpr bool kHalf = !std::is_same<CS, T>::value;

public:
    explicit EngineT(bool mixed) : mixed_(mixed) {
        // UAAMG_NO_PDL=1 launches every kernel without the programmatic-dependent-launch
        // attribute (fully serialised on the stream), for comparisons
        const char* v = std::getenv("UAAMG_NO_PDL");
        pdl_ = !(v && v[0] == '1');
        const char* pv = std::getenv("UAAMG_PMV2D_PER_SM");
        if (pv && pv[0]) pmv2d_env_ = std::max(1, std::atoi(pv));
        const char* bc = std::getenv("UAAMG_BOX_MAX_CELLS");
        if (bc && bc[0]) box_cells_ = std::atof(bc);
        // UAAMG_NO_TRIM=1: coarse boxes always load their diagonals and couplings
        const char* nt = std::getenv("UAAMG_NO_TRIM");
        trim_ = !(nt && nt[0] == '1');
    }
    ~EngineT() override {
        release();
        if (cap_) cudaStreamDestroy(cap_);
    }

    // A new problem.  The previous problem's device buffers are kept for reuse by size
    // (a mask change on the same grid -- moving solids -- allocates nothing) and the
    // ones the new hierarchy does not take are freed afterwards.
    int set_problem(int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                    const uint8_t* d_solid, int dirichlet) override {
        release(true);
        if (dim != 2 && dim != 3) { release(); return E_ARG; }
        if (nx < 2 || ny < 2 || (dim == 3 && nz < 2)) { release(); return E_ARG; }
        dim_ = dim; dirichlet_ = dirichlet;
        dx_ = dx; dy_ = dy; dz_ = dim == 3 ? dz : 1.0;
        int e = dim == 3 ? build<3>(nx, ny, nz, d_solid) : build<2>(nx, ny, nz, d_solid);
        free_pool();
        if (e != E_OK) { release(); return e; }
        return E_OK;
    }

    int precond_apply(const double* d_r, double* d_z) override {
        if (lv_.empty()) return E_NOPROB;
        launches_ = 0;
        cudaMemsetAsync(err_, 0, sizeof(int), st_);
        if (dim_ == 3) precond_impl<3>(d_r, d_z); else precond_impl<2>(d_r, d_z);
        return sync_check();
    }

    int solve_begin(const SolveArgs& a) override {
        if (lv_.empty()) return E_NOPROB;
        launches_ = 0;
        return dim_ == 3 ? begin_impl<3>(a) : begin_impl<2>(a);
    }

    int solve_step() override {
        if (stopped_) return E_OK;
        return dim_ == 3 ? step_impl<3>() : step_impl<2>();
    }

    // The device is known to have stopped once the flag copied after some step
    // reads 1, or once every queued step has finished after max_iter was reached.
    int solve_poll(bool wait, bool* stopped) override {
        while (!stopped_ && seen_ < nstep_) {
            const int slot = seen_ & 1;
            if (wait) {
                if (cudaEventSynchronize(ev_[slot]) != cudaSuccess) return E_CUDA;
            } else {
                const cudaError_t q = cudaEventQuery(ev_[slot]);
                if (q == cudaErrorNotReady) break;
                if (q != cudaSuccess) return E_CUDA;
            }
            if (flag_host_[slot]) stopped_ = true;
            ++seen_;
        }
        if (!stopped_ && seen_ == nstep_ && it_ >= cur_.max_iter) stopped_ = true;
        *stopped = stopped_;
        return E_OK;
    }

    // Steps queued but not yet seen by solve_poll (at most two are useful).
    int solve_inflight() const override { return nstep_ - seen_; }

    int solve_end(SolveResult* res) override {
        int e = solve_end_enqueue();
        return e != E_OK ? e : solve_end_collect(res);
    }

    int solve_end_enqueue() override { return dim_ == 3 ? end_enqueue<3>() : end_enqueue<2>(); }

    int enqueue_step(cudaStream_t s, int* flag_dst) override {
        if (lv_.empty()) return E_NOPROB;
        const cudaStream_t saved = st_;
        st_ = s;
        if (dim_ == 3) {
            cg_iteration<3>(true);
            cg_iteration<3>(false);
        } else {
            cg_iteration<2>(true);
            cg_iteration<2>(false);
        }
        if (flag_dst) cudaMemcpyAsync(flag_dst, &cg_->done, sizeof(int), cudaMemcpyDeviceToHost, st_);
        st_ = saved;
        return E_OK;
    }

    int solve_end_collect(SolveResult* res) override {
        int e = sync_check();
        if (e != E_OK) return e;
        const CGState& c = *cg_host_;
        res->status = c.status;
        res->iterations = c.iter;
        res->replacements = c.replacements;
        res->rr = c.rr;
        res->rr_true = c.rr_true;
        res->bnorm = c.bnorm;
        res->r0 = c.r0;
        res->tol_abs = c.tol_abs;
        return E_OK;
    }

    // The whole solve: the host keeps two steps queued and polls one behind, so it
    // never idles the GPU waiting for a scalar.
    int solve(const SolveArgs& a, SolveResult* res) override {
        int e = solve_begin(a);
        if (e != E_OK) return e;
        bool stopped = false;
        while (!stopped) {
            if ((e = solve_step()) != E_OK) return e;
            if ((e = solve_poll(solve_inflight() >= 2 || it_ >= cur_.max_iter, &stopped)) != E_OK)
                return e;
        }
        return solve_end(res);
    }

    int nlevels() const override { return (int)lv_.size(); }

    void level_dims(int l, int* nx, int* ny, int* nz) const override {
        *nx = lv_[l].g.nx; *ny = lv_[l].g.ny; *nz = lv_[l].g.nz;
    }

    int level_trim(int l, int* boxes, int* trimmed) override {
        if (l < 0 || l >= (int)lv_.size()) return E_ARG;
        const LevelBuf<T, CS>& L = lv_[l];
        *boxes = *trimmed = 0;
        if (!L.box) return E_OK;
        const dim3 bg = box_grid(L.g);
        *boxes = (int)(bg.x * bg.y * bg.z);
        if (!L.trim || !trim_) return E_OK;
        std::vector<T> rec((size_t)4 * *boxes);
        if (cudaMemcpy(rec.data(), L.trim, rec.size() * sizeof(T), cudaMemcpyDeviceToHost) !=
            cudaSuccess)
            return E_CUDA;
        for (int b = 0; b < *boxes; ++b) *trimmed += rec[(size_t)4 * b] != T(0);
        return E_OK;
    }

    // Host copies in the reference layout of level l (row pitch nx_l + 2).
    int copy_level(int l, uint8_t* solid, double* cx, double* cy, double* cz) override {
        if (l < 0 || l >= (int)lv_.size()) return E_ARG;
        const LevelBuf<T, CS>& L = lv_[l];
        const Geom g = L.g;
        const Geom gr = make_geom(dim_, g.nx, g.ny, g.nz);
        if (cudaStreamSynchronize(st_) != cudaSuccess) return E_CUDA;
        const int nzi = dim_ == 3 ? g.nz + 2 : 1;
        auto depitch = [&](auto* dst, const auto* src) {
            for (int k = 0; k < nzi; ++k)
                for (int j = 0; j < g.ny + 2; ++j)
                    for (int i = 0; i < g.nx + 2; ++i)
                        dst[i + j * gr.sx + k * gr.sxy] = src[i + j * g.sx + k * g.sxy];
        };
        if (solid) {
            std::vector<uint8_t> tmp(g.n);
            if (cudaMemcpy(tmp.data(), L.solid, g.n, cudaMemcpyDeviceToHost) != cudaSuccess)
                return E_CUDA;
            depitch(solid, tmp.data());
        }
        std::vector<T> tmp(g.n);
        std::vector<double> tmpd(g.n);
        const T* src[3] = {L.cx, L.cy, L.cz};
        double* dst[3] = {cx, cy, cz};
        for (int q = 0; q < 3; ++q) {
            if (!dst[q]) continue;
            if (!src[q]) { for (int c = 0; c < gr.n; ++c) dst[q][c] = 0.0; continue; }
            if (cudaMemcpy(tmp.data(), src[q], g.n * sizeof(T), cudaMemcpyDeviceToHost) != cudaSuccess)
                return E_CUDA;
            for (int c = 0; c < g.n; ++c) tmpd[c] = (double)tmp[c];
            depitch(dst[q], tmpd.data());
        }
        return E_OK;
    }

    void set_stream(cudaStream_t s) override { st_ = s; }
    size_t device_bytes() const override { return bytes_; }
    long launches() const override { return launches_; }
    void set_vcycle_sweeps(bool on) override { sweeps_ = on; }
    void set_graphs(bool on) override { graphs_ = on; }
    void set_autotune(bool on) override { autotune_ = on; }
    void set_small_levels(bool on) override { tail_on_ = on; }
    void set_smoothing(int fine, int coarse) override {
        if (fine == nu_fine_ && coarse == nu_coarse_) return;
        drop_graph();
        nu_fine_ = fine;
        nu_coarse_ = coarse;
    }
    void set_fused(bool on) override {
        if (on == fused_) return;
        drop_graph();
        fused_ = on;
    }
    void set_operator(const double* d, const double* ox, const double* oy, int sx,
                      long version) override {
        vver_ = version;
        if (d == vd_ && ox == vox_ && oy == voy_ && sx == vsx_) return;
        // a captured step holds the operator's pointers: capture again
        if (gexec_) {
            cudaStreamSynchronize(st_);
            cudaGraphExecDestroy(gexec_);
            gexec_ = nullptr;
        }
        gkey_ = -1;
        vd_ = d; vox_ = ox; voy_ = oy; vsx_ = sx;
    }

    void set_profiling(bool on) override {
        prof_on_ = on;
        prof_count_ = 0;
    }

    int profile_results(std::vector<KernelTime>& out) override {
        out.clear();
        if (cudaStreamSynchronize(st_) != cudaSuccess) return E_CUDA;
        for (int q = 0; q < prof_count_; ++q) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, prof_ev_[q].first, prof_ev_[q].second) != cudaSuccess)
                return E_CUDA;
            const KTag& t = prof_tag_[q];
            KernelTime* slot = nullptr;
            for (auto& kt : out)
                if (kt.cls == t.cls && kt.level == t.level) { slot = &kt; break; }
            if (!slot) {
                KernelTime kt;
                kt.cls = t.cls;
                kt.name = kclass_names[t.cls];
                kt.level = t.level;
                kt.launches = 0;
                kt.total_ms = 0.0;
                kt.bytes = t.bytes;
                out.push_back(kt);
                slot = &out.back();
            }
            slot->launches += 1;
            slot->total_ms += ms;
        }
        // the residual replacement kernel runs every iteration but works only when a
        // replacement is due: its bytes per launch are those of the replacements
        // performed, spread over all its launches
        for (auto& kt : out)
            if (kt.cls == K_REPLACE && kt.launches > 0)
                kt.bytes = kt.bytes * (double)cg_host_->replacements / (double)kt.launches;
        return E_OK;
    }

    int timed_out() override {
        int v = 0;
        if (!err_) return 0;
        if (cudaMemcpy(&v, err_, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return 0;
        return v;
    }

private:
    bool mixed_;
    int dim_ = 0, dirichlet_ = 0;
    double dx_ = 1, dy_ = 1, dz_ = 1;
    Geom gref_;                      // the caller's (reference) layout of level 0
    std::vector<LevelBuf<T, CS>> lv_;
    T *r_ = nullptr, *z_ = nullptr, *p_ = nullptr, *p2_ = nullptr, *ap_ = nullptr, *xlo_ = nullptr;
    // variable-coefficient operator (set_operator); not owned
    const double *vd_ = nullptr, *vox_ = nullptr, *voy_ = nullptr;
    int vsx_ = 0;
    long vver_ = 0, vconv_ = -1;     // contents version set / converted into vf_
    float* vf_[3] = {nullptr, nullptr, nullptr};  // FP32 forms: s, ox, oy (level layout)
    double *b64_ = nullptr, *xd_ = nullptr, *partials_ = nullptr;
    int* err_ = nullptr;             // set by a kernel whose TMA wait gave up
    CUtensorMap map_p_, map_p2_;     // plane boxes of the two search-direction buffers
    CUtensorMap map_b64_, map_xd_, map_xlo_;  // plane boxes of b, x_hi (FP64) and x_lo (3D)
    SolveArgs cur_{};                // the solve in progress
    bool use_graph_ = false;
    int it_ = 0;                     // iterations queued
    int nstep_ = 0, seen_ = 0;       // steps queued / steps whose flag was read
    bool stopped_ = false;
    long long reduce_blocks_ = 0;    // partials_ capacity in blocks (4 doubles each)
    CGState* cg_ = nullptr;
    CGState* cg_host_ = nullptr;  // pinned
    int* flag_host_ = nullptr;    // pinned, 2 slots
    cudaEvent_t ev_[2] = {nullptr, nullptr};
    cudaStream_t st_ = 0;
    std::vector<std::pair<void*, size_t>> allocs_;  // device buffers and their bytes
    std::multimap<size_t, void*> pool_;               // kept for reuse by set_problem
    size_t bytes_ = 0;
    long launches_ = 0;
    int num_sms_ = 148;
    bool sweeps_ = false;  // V-cycle as per-colour sweeps (cross-check) instead of the marches
    bool graphs_ = true;   // replay the PCG step as a CUDA graph
    bool autotune_ = false;  // time the marches' z-chunk lengths at set-up
    bool tail_on_ = true;    // small levels in one one-block kernel (tail.cuh)
    bool fused_ = true;      // two fused marches a level (fused.cuh) instead of four
    double box_cells_ = kBoxCells;
    // blocks per SM of the 2D search direction: as many as are resident at once (one
    // wave: a second, partial wave left SMs idle at its end); UAAMG_PMV2D_PER_SM overrides
    int pmv2d_per_sm_ = 8;
    int rx_zc_ = 16;  // planes per block of the 3D replacement march (k_resid_march)
    int pmv2d_env_ = 0;
    int resid_per_sm_ = 8;  // the FP64 residual walk: resident blocks per SM (one wave)
    bool trim_ = true;       // trimmed coarse boxes (fused.cuh k_box_trim)
    bool pdl_ = true;        // programmatic dependent launch between the kernels
    bool nopdl_next_ = false;  // the next launch is plain (a kernel that usually exits at
                               // once: its blocks should not wait resident for their turn)
    int nu_fine_ = 1, nu_coarse_ = 1;  // pre- and post-smoothing sweeps: finest / coarse levels
    int tail_lt_ = 0;        // first level of the small-level kernel
    int tail_nc_ = 0;        // 1: the hierarchy has a tail (0: it does not fit the kernel)
    size_t tail_smem_ = 0;   // its dynamic shared memory (x and b of every tail level)
    cudaStream_t cap_ = nullptr;      // capture stream
    cudaGraphExec_t gexec_ = nullptr; // two PCG iterations
    long long gkey_ = -1;
    const double* ghist_ = nullptr;
    long glaunches_ = 0;              // kernels in one graph replay
    // in-situ per-launch timing (set_profiling)
    bool prof_on_ = false;
    int prof_count_ = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_ev_;
    std::vector<KTag> prof_tag_;

    int max_reduce_blocks() const { return 4 * num_sms_; }

    void drop_graph() {
        if (gexec_) {
            cudaStreamSynchronize(st_);
            cudaGraphExecDestroy(gexec_);
            gexec_ = nullptr;
        }
        gkey_ = -1;
    }

    // grid of the 2D search-direction kernel (kernels.cuh k_pmatvec_2d): 32 column
    // pairs of two rows a warp, eight warps a block, up to 8 blocks per SM (within
    // the partials' capacity)
    dim3 flat2d_grid(const Geom& g) const {
        const long long items = (long long)((g.ny + 1) / 2) * ((g.nx + 31) / 32);
        long long nb = std::min<long long>((items + 7) / 8, (long long)pmv2d_per_sm_ * num_sms_);
        nb = std::min<long long>(nb, reduce_blocks_);
        return dim3((unsigned)(nb < 1 ? 1 : nb));
    }

    // grid of the FP64 residual column walk (kernels.cuh k_resid_x64): tiles of
    // 32 x 8 columns and kResidZc planes, at most 8 blocks of 256 threads per SM
    static constexpr int kResidZc = 16;
    dim3 resid_grid(const Geom& g) const {
        const long long tiles = (long long)((g.nx + 31) / 32) * ((g.ny + 7) / 8) *
                                (g.nz ? (g.nz + kResidZc - 1) / kResidZc : 1);
        return dim3((unsigned)std::min<long long>(tiles, (long long)resid_per_sm_ * num_sms_));
    }

    // grid of the row-walk kernels (kernels.cuh for_cells): capped at 4 blocks per SM
    dim3 vec_grid(const Geom& g) const {
        const long long items = (long long)g.ny * (g.nz ? g.nz : 1) * ((g.nx + 31) / 32);
        long long nb = (items + 7) / 8;
        if (nb > max_reduce_blocks()) nb = max_reduce_blocks();
        return dim3((unsigned)(nb < 1 ? 1 : nb));
    }

    void prof_begin(const KTag& t, cudaEvent_t* e0, cudaEvent_t* e1) {
        if (prof_count_ == (int)prof_ev_.size()) {
            cudaEvent_t a = nullptr, b = nullptr;
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            prof_ev_.push_back({a, b});
            prof_tag_.push_back(t);
        }
        prof_tag_[prof_count_] = t;
        *e0 = prof_ev_[prof_count_].first;
        *e1 = prof_ev_[prof_count_].second;
        ++prof_count_;
        cudaEventRecord(*e0, st_);
    }

    static double cells(const Geom& g) {
        return (double)g.nx * g.ny * (g.nz ? g.nz : 1);
    }

    template <class P>
    int alloc(P*& p, size_t count) {
        void* q = nullptr;
        const size_t nb = count * sizeof(P);
        auto it = pool_.find(nb);
        if (it != pool_.end()) {
            q = it->second;
            pool_.erase(it);
        } else if (cudaMalloc(&q, nb) != cudaSuccess) {
            cudaGetLastError();
            return E_OOM;
        }
        allocs_.push_back({q, nb});
        bytes_ += nb;
        if (cudaMemsetAsync(q, 0, count * sizeof(P), st_) != cudaSuccess) return E_CUDA;
        p = static_cast<P*>(q);
        return E_OK;
    }

    // keep: the device buffers go to the reuse pool (set_problem) instead of being
    // freed, and the pinned host words and events stay.
    void release(bool keep = false) {
        if (!allocs_.empty() || cg_host_) cudaStreamSynchronize(st_);
        for (const auto& a : allocs_) {
            if (keep) pool_.emplace(a.second, a.first);
            else cudaFree(a.first);
        }
        allocs_.clear();
        if (!keep) free_pool();
        lv_.clear();
        bytes_ = 0;
        r_ = z_ = p_ = p2_ = ap_ = xlo_ = nullptr;
        b64_ = xd_ = partials_ = nullptr;
        vf_[0] = vf_[1] = vf_[2] = nullptr;
        vconv_ = -1;
        err_ = nullptr;
        cg_ = nullptr;
        if (!keep) {
            if (cg_host_) { cudaFreeHost(cg_host_); cg_host_ = nullptr; }
            if (flag_host_) { cudaFreeHost(flag_host_); flag_host_ = nullptr; }
            for (auto& e : ev_) if (e) { cudaEventDestroy(e); e = nullptr; }
        }
        for (auto& pr : prof_ev_) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
        prof_ev_.clear();
        if (gexec_) { cudaGraphExecDestroy(gexec_); gexec_ = nullptr; }
        gkey_ = -1;
        ghist_ = nullptr;
        prof_tag_.clear();
        prof_count_ = 0;
    }

    void free_pool() {
        for (const auto& kv : pool_) cudaFree(kv.second);
        pool_.clear();
    }

    int sync_check() {
        cudaError_t e = cudaGetLastError();
        const cudaError_t es = cudaStreamSynchronize(st_);
        if (e == cudaSuccess) e = es;
        if (e == cudaSuccess) e = cudaGetLastError();
        if (e != cudaSuccess) cuda_error = e;
        return e == cudaSuccess ? E_OK : E_CUDA;
    }

    // Blocks of a march over level g: 32 x 8 column tiles, z chunks of zc planes.
    template <int DIM>
    static dim3 march_grid(const Geom& g, int zc) {
        return dim3((unsigned)((g.nx + kMX - 1) / kMX), (unsigned)((g.ny + kMY - 1) / kMY),
                    DIM == 3 ? (unsigned)((g.nz + zc - 1) / zc) : 1u);
    }

    // Blocks of the whole-tile box kernels over level g: 8^3 tiles.
    static dim3 box_grid(const Geom& g) {
        return dim3((unsigned)((g.nx + kBT - 1) / kBT), (unsigned)((g.ny + kBT - 1) / kBT),
                    (unsigned)((g.nz + kBT - 1) / kBT));
    }

    // Largest even chunk <= 16 planes that still gives every SM several blocks.
    int pick_zc(const Geom& g) const {
        const long long tiles = (long long)((g.nx + kMX - 1) / kMX) * ((g.ny + kMY - 1) / kMY);
        int zc = 16;
        while (zc > 2 && tiles * ((g.nz + zc - 1) / zc) < 4LL * num_sms_) zc /= 2;
        return zc;
    }

    template <class K>
    static int smem_attr(K kern, size_t bytes) {
        return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) ==
                       cudaSuccess
                   ? E_OK
                   : E_CUDA;
    }

    template <int DIM, bool FINE, class CSL>
    int march_attrs() {
        int e;
        if ((e = smem_attr(k_fwd_smooth<DIM, T, FINE, CSL>, FwdCfg<DIM, T, FINE, CSL>::BYTES)) ||
            (e = smem_attr(k_restrict_res<DIM, T, FINE, CSL>, ResCfg<DIM, T, FINE, CSL>::BYTES)) ||
            (e = smem_attr(k_up_even<DIM, T, FINE, CSL>, UpeCfg<DIM, T, FINE, CSL>::BYTES)) ||
            (e = smem_attr(k_up_odd<DIM, T, FINE, false, CSL>, UpoCfg<DIM, T, FINE, CSL>::BYTES)) ||
            (e = smem_attr(k_up_odd<DIM, T, FINE, true, CSL>, UpoCfg<DIM, T, FINE, CSL>::BYTES)))
            return e;
        return E_OK;
    }

    template <bool FINE, class CSL>
    int box_attrs() {
        int e;
        if ((e = smem_attr(k_level_box<T, FINE, CSL, false, false>, BPlan<T, CSL, FINE, false>::BYTES)) ||
            (e = smem_attr(k_level_box<T, FINE, CSL, true, false>, BPlan<T, CSL, FINE, true>::BYTES)) ||
            (e = smem_attr(k_level_box<T, FINE, CSL, true, true>, BPlan<T, CSL, FINE, true>::BYTES)))
            return e;
        return E_OK;
    }

    template <int DIM, bool FINE, class CSL>
    int fused_attrs() {
        int e;
        if ((e = smem_attr(k_level_fused<DIM, T, FINE, CSL, false, false>,
                           FCfg<DIM, T, CSL, FINE, false>::BYTES)) ||
            (e = smem_attr(k_level_fused<DIM, T, FINE, CSL, true, false>,
                           FCfg<DIM, T, CSL, FINE, true>::BYTES)) ||
            (e = smem_attr(k_level_fused<DIM, T, FINE, CSL, true, true>,
                           FCfg<DIM, T, CSL, FINE, true>::BYTES)))
            return e;
        return E_OK;
    }

    template <int DIM>
    int build(int nx, int ny, int nz, const uint8_t* d_solid) {
        gref_ = make_geom(DIM, nx, ny, nz);
        {
            const Geom gp = make_geom_pitched(DIM, nx, ny, nz);
            if ((long long)gp.sx * (ny + 2) * (DIM == 3 ? nz + 2 : 1) >= (1LL << 31)) return E_ARG;
        }
        double hx = dx_, hy = dy_, hz = dz_;
        while (nx >= 2 && ny >= 2 && (DIM == 2 || nz >= 2)) {
            LevelBuf<T, CS> L;
            L.g = make_geom_pitched(DIM, nx, ny, nz);
            L.hx = hx; L.hy = hy; L.hz = hz;
            lv_.push_back(L);
            if (nx <= 4 || ny <= 4 || (DIM == 3 && nz <= 4)) break;
            nx /= 2; ny /= 2; nz /= 2;
            hx *= 2.0; hy *= 2.0; hz *= 2.0;
        }
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return E_CUDA;
        {
            int per_sm = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_resid_x64<DIM, T>, 256, 0) ==
                    cudaSuccess && per_sm > 0)
                resid_per_sm_ = std::min(per_sm, 8);
            else
                cudaGetLastError();
        }
        if (pmv2d_env_ > 0) {
            pmv2d_per_sm_ = pmv2d_env_;
        } else {
            int per_sm = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pmatvec_2d<T>, 256, 0) ==
                    cudaSuccess && per_sm > 0)
                pmv2d_per_sm_ = std::min(per_sm, 8);
            else
                cudaGetLastError();
        }
        const int nl = (int)lv_.size();
        int e;
        for (int l = 0; l < nl; ++l) {
            LevelBuf<T, CS>& L = lv_[l];
            L.zc = DIM == 3 ? pick_zc(L.g) : 2;
            // largest face count of a level-l coupling: 4^l (3D), 2^l (2D)
            L.c32 = kHalf && l > 0 && (DIM == 3 ? 2 * l : l) > 11;
            L.box = DIM == 3 && cells(L.g) <= box_cells_;
            const size_t n = (size_t)L.g.n;
            if ((e = alloc(L.solid, n))) return e;
            if ((e = alloc(L.code, n))) return e;
            if ((e = alloc(L.cx, n))) return e;
            if ((e = alloc(L.cy, n))) return e;
            if (DIM == 3 && (e = alloc(L.cz, n))) return e;
            if (dirichlet_ && (e = alloc(L.wd, n))) return e;
            if (l > 0) {
                if ((e = alloc(L.x, n))) return e;
                if ((e = alloc(L.b, n))) return e;
                if ((e = alloc(L.dg, n))) return e;
                if (L.box) {
                    const dim3 bg = box_grid(L.g);
                    if ((e = alloc(L.trim, (size_t)4 * bg.x * bg.y * bg.z))) return e;
                }
                if constexpr (kHalf) {
                    if (!L.c32) {
                        if ((e = alloc(L.hcx, n)) || (e = alloc(L.hcy, n))) return e;
                        if (DIM == 3 && (e = alloc(L.hcz, n))) return e;
                    }
                } else {
                    L.hcx = L.cx; L.hcy = L.cy; L.hcz = L.cz;
                }
            }
        }
        const Geom g0 = lv_[0].g;
        const size_t n0 = (size_t)g0.n;
        if ((e = alloc(r_, n0)) || (e = alloc(z_, n0)) || (e = alloc(p_, n0)) ||
            (e = alloc(p2_, n0)) || (e = alloc(ap_, n0)) || (e = alloc(xlo_, n0)) ||
            (e = alloc(b64_, n0)) || (e = alloc(xd_, n0)))
            return e;
        // reductions: the finest-level marches (one partial per block) and the
        // row-walk kernels (vec_grid)
        {
            const dim3 mg = march_grid<DIM>(g0, 2);  // the most blocks any chunk length gives
            reduce_blocks_ = (long long)mg.x * mg.y * mg.z;
            const dim3 rg = resid_grid(g0);
            reduce_blocks_ = std::max(reduce_blocks_, (long long)rg.x * rg.y * rg.z);
            const dim3 bg = box_grid(g0);  // a small finest level runs as boxes
            if (lv_[0].box) reduce_blocks_ = std::max(reduce_blocks_, (long long)bg.x * bg.y * bg.z);
            if (reduce_blocks_ < max_reduce_blocks()) reduce_blocks_ = max_reduce_blocks();
        }
        if ((e = alloc(partials_, (size_t)reduce_blocks_ * 4))) return e;
        if ((e = alloc(err_, 1))) return e;
        if ((e = alloc(cg_, 1))) return e;
        if (!cg_host_ && cudaMallocHost(&cg_host_, sizeof(CGState)) != cudaSuccess) return E_OOM;
        if (!flag_host_ && cudaMallocHost(&flag_host_, 2 * sizeof(int)) != cudaSuccess) return E_OOM;
        for (auto& ev : ev_)
            if (!ev && cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return E_CUDA;
        // dynamic shared memory of the marches
        if ((e = march_attrs<DIM, true, CS>()) || (e = march_attrs<DIM, false, CS>()) ||
            (e = smem_attr(k_pmatvec<DIM, T, true>, PmvCfg<DIM, T>::BYTES)) ||
            (e = smem_attr(k_pmatvec<DIM, T, false>, PmvCfg<DIM, T>::BYTES)) ||
            (e = fused_attrs<DIM, true, CS>()) || (e = fused_attrs<DIM, false, CS>()))
            return e;
        if constexpr (kHalf) {  // levels with FP32 couplings
            if ((e = march_attrs<DIM, false, T>()) || (e = fused_attrs<DIM, false, T>())) return e;
        }
        if (DIM == 3) {
            if ((e = smem_attr(k_resid_march<T, true>, RxCfg<T>::BYTES)) ||
                (e = smem_attr(k_resid_march<T, false>, RxCfg<T>::BYTES)))
                return e;
            // planes per block of the replacement march: chunks doubled until the blocks
            // fit in one wave (256^3: 64 planes, 512 blocks; 1.31 against 1.37 ms a solve
            // with 32 planes and 1024 blocks)
            int per_sm = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_resid_march<T, false>, kThreads,
                                                              RxCfg<T>::BYTES) != cudaSuccess ||
                per_sm < 1) {
                cudaGetLastError();
                per_sm = 1;
            }
            const Geom& g = lv_[0].g;
            const long long tiles = (long long)((g.nx + kMX - 1) / kMX) * ((g.ny + kMY - 1) / kMY);
            rx_zc_ = 2;
            while (rx_zc_ < g.nz && tiles * ((g.nz + rx_zc_ - 1) / rx_zc_) > (long long)per_sm * num_sms_)
                rx_zc_ *= 2;
        }
        if (DIM == 3) {
            if ((e = box_attrs<true, CS>()) || (e = box_attrs<false, CS>())) return e;
            if constexpr (kHalf) {
                if ((e = box_attrs<false, T>())) return e;
            }
        }
        // plane-box tensor maps
        constexpr int BW = PBox<T>::W, BH = PBox<T>::H;
        for (int l = 0; l < nl; ++l) {
            LevelBuf<T, CS>& L = lv_[l];
            const T* b = l == 0 ? r_ : L.b;
            const T* x = l == 0 ? z_ : L.x;
            bool ok = encode_level_map<T>(&L.mb, b, L.g, DIM, BW, BH, 1) &&
                      encode_level_map<T>(&L.mx, x, L.g, DIM, BW, BH, 1) &&
                      encode_level_map<uint8_t>(&L.mcode, L.code, L.g, DIM, PBox<uint8_t>::W,
                                                PBox<uint8_t>::H, 1);
            constexpr int CW = PBox<CS>::W;
            if (ok && l > 0 && !L.c32)
                ok = encode_level_map<CS>(&L.mcx, L.hcx, L.g, DIM, CW, BH, 1) &&
                     encode_level_map<CS>(&L.mcy, L.hcy, L.g, DIM, CW, BH, 1) &&
                     (DIM == 2 || encode_level_map<CS>(&L.mcz, L.hcz, L.g, DIM, CW, BH, 1)) &&
                     encode_level_map<CS>(&L.fcx, L.hcx, L.g, DIM, RBox<CS>::W, RBox<CS>::H, 1) &&
                     encode_level_map<CS>(&L.fcy, L.hcy, L.g, DIM, RBox<CS>::W, RBox<CS>::H, 1) &&
                     (DIM == 2 ||
                      encode_level_map<CS>(&L.fcz, L.hcz, L.g, DIM, RBox<CS>::W, RBox<CS>::H, 1));
            if (ok && l > 0 && L.c32)  // FP32 couplings read as T
                ok = encode_level_map<T>(&L.mcx, L.cx, L.g, DIM, BW, BH, 1) &&
                     encode_level_map<T>(&L.mcy, L.cy, L.g, DIM, BW, BH, 1) &&
                     (DIM == 2 || encode_level_map<T>(&L.mcz, L.cz, L.g, DIM, BW, BH, 1)) &&
                     encode_level_map<T>(&L.fcx, L.cx, L.g, DIM, RBox<T>::W, RBox<T>::H, 1) &&
                     encode_level_map<T>(&L.fcy, L.cy, L.g, DIM, RBox<T>::W, RBox<T>::H, 1) &&
                     (DIM == 2 ||
                      encode_level_map<T>(&L.fcz, L.cz, L.g, DIM, RBox<T>::W, RBox<T>::H, 1));
            if (ok && l > 0)
                ok = encode_level_map<T>(&L.mdg, L.dg, L.g, DIM, BW, BH, 1) &&
                     encode_level_map<T>(&L.fdg, L.dg, L.g, DIM, RBox<T>::W, RBox<T>::H, 1) &&
                     encode_level_map<T>(&L.mxq, L.x, L.g, DIM, QBox<T>::W, QBox<T>::H, 1);
            if (ok)
                ok = encode_level_map<T>(&L.fb, b, L.g, DIM, RBox<T>::W, RBox<T>::H, 1) &&
                     encode_level_map<uint8_t>(&L.fcode, L.code, L.g, DIM, RBox<uint8_t>::W,
                                               RBox<uint8_t>::H, 1);
            if (ok && DIM == 3) {
                // whole-tile boxes (small levels) and this level's x as the parent box of
                // the next-finer level's box kernels
                if (l > 0)
                    ok = encode_level_map<T>(&L.bxq, L.x, L.g, DIM, BQBox<T>::W, 6, 6);
                if (ok && L.box) {
                    ok = encode_level_map<T>(&L.bb, b, L.g, DIM, BBox<T>::W, kBB, kBB) &&
                         encode_level_map<uint8_t>(&L.bcode, L.code, L.g, DIM, BBox<uint8_t>::W, kBB,
                                                   kBB);
                    if (ok && l > 0) {
                        ok = encode_level_map<T>(&L.bdg, L.dg, L.g, DIM, BBox<T>::W, kBB, kBB);
                        if (ok && !L.c32)
                            ok = encode_level_map<CS>(&L.bcx, L.hcx, L.g, DIM, BBox<CS>::W, kBB, kBB) &&
                                 encode_level_map<CS>(&L.bcy, L.hcy, L.g, DIM, BBox<CS>::W, kBB, kBB) &&
                                 encode_level_map<CS>(&L.bcz, L.hcz, L.g, DIM, BBox<CS>::W, kBB, kBB);
                        if (ok && L.c32)
                            ok = encode_level_map<T>(&L.bcx, L.cx, L.g, DIM, BBox<T>::W, kBB, kBB) &&
                                 encode_level_map<T>(&L.bcy, L.cy, L.g, DIM, BBox<T>::W, kBB, kBB) &&
                                 encode_level_map<T>(&L.bcz, L.cz, L.g, DIM, BBox<T>::W, kBB, kBB);
                    }
                }
            }
            if (!ok) return E_CUDA;
        }
        if (!encode_level_map<T>(&map_p_, p_, g0, DIM, BW, BH, 1) ||
            !encode_level_map<T>(&map_p2_, p2_, g0, DIM, BW, BH, 1))
            return E_CUDA;
        if (DIM == 3 &&
            (!encode_level_map<double>(&map_b64_, b64_, g0, DIM, PBox<double>::W, PBox<double>::H, 1) ||
             !encode_level_map<double>(&map_xd_, xd_, g0, DIM, PBox<double>::W, PBox<double>::H, 1) ||
             !encode_level_map<T>(&map_xlo_, xlo_, g0, DIM, BW, BH, 1)))
            return E_CUDA;

        // hierarchy: masks, couplings, coarse diagonals
        const dim3 blk = cell_block<DIM>();
        UAAMG_LAUNCH((KTag{K_SETUP, 0, 0.0}), k_import_mask<DIM>, vec_grid(g0), dim3(32, 8), g0, gref_,
                     d_solid, lv_[0].solid);
        for (int l = 1; l < nl; ++l)
            UAAMG_LAUNCH((KTag{K_SETUP, l, 0.0}), k_restrict_solid<DIM>,
                         cell_grid<DIM>(lv_[l].g.nx, lv_[l].g.ny, lv_[l].g.nz), blk, lv_[l - 1].g,
                         lv_[l - 1].solid, lv_[l].g, lv_[l].solid);
        {
            const LevelBuf<T, CS>& L = lv_[0];
            const T idx2 = (T)(1.0 / (L.hx * L.hx)), idy2 = (T)(1.0 / (L.hy * L.hy));
            const T idz2 = DIM == 3 ? (T)(1.0 / (L.hz * L.hz)) : T(0);
            UAAMG_LAUNCH((KTag{K_SETUP, 0, 0.0}), (k_fine_coeffs<DIM, T>),
                         cell_grid<DIM>(L.g.nx, L.g.ny, L.g.nz), blk, L.g, L.solid, L.cx, L.cy, L.cz,
                         L.wd, idx2, idy2, idz2);
        }
        for (int l = 1; l < nl; ++l) {
            const LevelBuf<T, CS>& F = lv_[l - 1];
            LevelBuf<T, CS>& Cl = lv_[l];
            UAAMG_LAUNCH((KTag{K_SETUP, l, 0.0}), (k_galerkin<DIM, T>),
                         cell_grid<DIM>(Cl.g.nx, Cl.g.ny, Cl.g.nz), blk, F.g, F.cx, F.cy, F.cz, F.wd,
                         Cl.g, Cl.solid, Cl.cx, Cl.cy, Cl.cz, Cl.wd);
        }
        for (int l = 1; l < nl; ++l) {
            LevelBuf<T, CS>& Cl = lv_[l];
            if constexpr (kHalf) {  // FP16 face counts (after every level's Galerkin sums)
              if (!Cl.c32) {
                const Geom& g0 = lv_[0].g;
                const float cs[3] = {(float)(1.0 / (lv_[0].hx * lv_[0].hx)),
                                     (float)(1.0 / (lv_[0].hy * lv_[0].hy)),
                                     (float)(1.0 / (lv_[0].hz * lv_[0].hz))};
                (void)g0;
                T* src[3] = {Cl.cx, Cl.cy, Cl.cz};
                CS* dst[3] = {Cl.hcx, Cl.hcy, Cl.hcz};
                for (int a = 0; a < DIM; ++a)
                    UAAMG_LAUNCH((KTag{K_SETUP, l, 0.0}), k_coupling_half, max_reduce_blocks(), 256,
                                 (long long)Cl.g.n, src[a], dst[a], cs[a]);
              }
            }
            UAAMG_LAUNCH((KTag{K_SETUP, l, 0.0}), (k_diag<DIM, T>), vec_grid(Cl.g), dim3(32, 8), Cl.g,
                         Cl.solid, Cl.cx, Cl.cy, Cl.cz, Cl.wd, Cl.dg);
        }
        for (int l = 0; l < nl; ++l)
            UAAMG_LAUNCH((KTag{K_SETUP, l, 0.0}), k_codes<DIM>, vec_grid(lv_[l].g), dim3(32, 8),
                         lv_[l].g, lv_[l].solid, lv_[l].code, l == 0 ? 1 : 0);
        if constexpr (DIM == 3) {  // trimmed boxes of the coarse box levels
            for (int l = 1; l < nl; ++l) {
                const LevelBuf<T, CS>& Cl = lv_[l];
                if (!Cl.box) continue;
                const MLevel<T> m = mlevel(l);
                if (kHalf && !Cl.c32)
                    UAAMG_LAUNCH((KTag{K_SETUP, l, 0.0}), (k_box_trim<T, CS>), box_grid(Cl.g), 256,
                                 Cl.g, Cl.code, Cl.dg, Cl.hcx, Cl.hcy, Cl.hcz, m.csx, m.csy, m.csz,
                                 Cl.trim);
                else
                    UAAMG_LAUNCH((KTag{K_SETUP, l, 0.0}), (k_box_trim<T, T>), box_grid(Cl.g), 256,
                                 Cl.g, Cl.code, Cl.dg, Cl.cx, Cl.cy, Cl.cz, m.csx, m.csy, m.csz,
                                 Cl.trim);
            }
        }
        if ((e = sync_check()) != E_OK) return e;
        if ((e = tail_setup<DIM>()) != E_OK) return e;
        if (DIM == 3 && autotune_) return tune<DIM>();
        return E_OK;
    }

    bool use_tail() const { return tail_on_ && !sweeps_ && tail_nc_ > 0; }

    // The small levels' one-block kernel (tail.cuh): from the first level (>= 1) of at
    // most kTailCells cells down to the coarsest, while their x and b fit its shared
    // memory and the coarsest has at most two cells a thread.
    static size_t tail_cells_padded(const Geom& g) {
        return (size_t)(g.nx + 2) * (g.ny + 2) * (g.nz ? g.nz + 2 : 1);
    }

    template <int DIM>
    int tail_setup() {
        const int nl = (int)lv_.size();
        tail_nc_ = 0;
        tail_lt_ = nl;
        if (nl < 2) return E_OK;
        const Geom& gc = lv_[nl - 1].g;
        size_t elems = 2 * tail_cells_padded(gc);
        if (cells(gc) > 2.0 * tail_threads<T>() || elems * sizeof(T) > kTailSmemBytes) return E_OK;
        int lt = nl - 1;
        while (lt > 1 && cells(lv_[lt - 1].g) <= (double)kTailCells && nl - (lt - 1) <= kTailMaxLevels &&
               (elems + 2 * tail_cells_padded(lv_[lt - 1].g)) * sizeof(T) <= kTailSmemBytes) {
            --lt;
            elems += 2 * tail_cells_padded(lv_[lt].g);
        }
        // the attribute belongs to the kernel, not to this engine: always the cap
        if (cudaFuncSetAttribute(k_tail<DIM, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kTailSmemBytes) != cudaSuccess)
            return E_CUDA;
        tail_lt_ = lt;
        tail_nc_ = 1;
        tail_smem_ = elems * sizeof(T);
        return E_OK;
    }

    // Levels tail_lt_ .. nl-1 of the V-cycle (b of tail_lt_ in, its x out).
    template <int DIM>
    void tail_launch(const int* done) {
        const int nl = (int)lv_.size();
        TailArgs<T> a{};
        a.nlev = nl - tail_lt_;
        int off = 0;
        double bytes = 0.0;
        for (int q = 0; q < a.nlev; ++q) {
            const LevelBuf<T, CS>& L = lv_[tail_lt_ + q];
            TailLevel<T>& t = a.lv[q];
            t.g = L.g;
            t.csx = L.g.nx + 2;
            t.csxy = (L.g.nx + 2) * (L.g.ny + 2);
            t.xs = off;
            t.bs = off + (int)tail_cells_padded(L.g);
            off += 2 * (int)tail_cells_padded(L.g);
            t.code = L.code;
            t.cx = L.cx;
            t.cy = L.cy;
            t.cz = DIM == 3 ? L.cz : nullptr;
            t.dg = L.dg;
            t.x = L.x;
            t.b = L.b;
            t.rnx = 1.0f / (float)L.g.nx;
            t.rny = 1.0f / (float)L.g.ny;
            // codes, couplings and diagonal read once per pass, four passes
            bytes += 4.0 * cells(L.g) * ((1.0 + DIM) * sizeof(T) + 1.0);
        }
        a.smem_elems = off;
        bytes += 2.0 * cells(lv_[tail_lt_].g) * sizeof(T);  // the first level's b in, x out
        UAAMG_LAUNCH_SMEM((KTag{K_TAIL, tail_lt_, bytes}), (k_tail<DIM, T>), 1, tail_threads<T>(),
                          tail_smem_, a, done);
    }

    // Autotuner: for every level with marches, time its V-cycle marches (down and up,
    // on the level's own buffers) for each z-chunk length in {2, 4, 8, 16, 32} and
    // keep the fastest; the choice is cached per GPU, precision, level shape and
    // march kind (tune_lookup / tune_store: for the process, and in the cache file
    // when one is set).  Chunk length changes only the blocks' shape, not a per-cell
    // value; the FP64 dot products are summed per block, so their rounding (and so
    // the last bits of the iterates) may differ.
    template <int DIM>
    int tune() {
        cudaEvent_t a = nullptr, b = nullptr;
        if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return E_CUDA;
        const bool prof = prof_on_;
        prof_on_ = false;
        int e = E_OK;
        for (int l = 0; l + 1 < (int)lv_.size() && e == E_OK; ++l) {
            if (use_tail() && l >= tail_lt_) break;  // the small-level kernel runs those levels
            LevelBuf<T, CS>& L = lv_[l];
            if (L.box && fused_ && level_nu(l) == 1) continue;  // whole-tile boxes: no chunks
            const std::string key = "zc|" + tune_gpu_id() + "|" + (sizeof(T) == 8 ? "f64" : mixed_ ? "mixed" : "f32") +
                                    "|" + std::to_string(L.g.nx) + "x" + std::to_string(L.g.ny) + "x" +
                                    std::to_string(L.g.nz) + "|" + (l == 0 ? "fine" : "coarse") + "|" +
                                    (fused_ && level_nu(l) == 1 ? "fused" : "four") + (L.c32 ? "|c32" : "");
            {
                std::vector<int> v;
                if (tune_lookup(key, &v) && v.size() == 1 && v[0] >= 2 && v[0] <= 32) { L.zc = v[0]; continue; }
            }
            int best = L.zc;
            float best_ms = 1e30f;
            for (int zc = 2; zc <= 32 && e == E_OK; zc *= 2) {
                if (zc > 2 && zc / 2 >= L.g.nz) break;
                L.zc = zc;
                for (int rep = 0; rep < 3; ++rep) {  // rep 0 warms up
                    if (rep == 1) cudaEventRecord(a, st_);
                    if (l == 0) { down_level<DIM, true>(l, nullptr); up_level<DIM, true>(l, nullptr, false); }
                    else { down_level<DIM, false>(l, nullptr); up_level<DIM, false>(l, nullptr, false); }
                }
                cudaEventRecord(b, st_);
                float ms = 0.f;
                if (cudaEventSynchronize(b) != cudaSuccess || cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
                    e = sync_check();
                    if (e == E_OK) e = E_CUDA;
                    break;
                }
                if (ms < best_ms) { best_ms = ms; best = zc; }
            }
            L.zc = best;
            tune_store(key, {best});
        }
        prof_on_ = prof;
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        if (e == E_OK) e = sync_check();
        return e;
    }

    LevelView<T> view(int l, const T* r, T* z) const {
        const LevelBuf<T, CS>& L = lv_[l];
        LevelView<T> v;
        v.g = L.g;
        v.solid = L.solid;
        v.cx = L.cx; v.cy = L.cy; v.cz = L.cz; v.wd = L.wd;
        v.x = l == 0 ? z : L.x;
        v.b = l == 0 ? r : L.b;
        return v;
    }

    template <int DIM>
    void sweep(const LevelView<T>& v, int parity, const int* done, int lvl) {
        UAAMG_LAUNCH((KTag{K_SWEEP, lvl, cells(v.g) * ((2.0 + DIM) * sizeof(T) + 0.5)}), (k_sweep<DIM, T>),
                     cell_grid<DIM>((v.g.nx + 1) / 2, v.g.ny, v.g.nz), cell_block<DIM>(), v, parity,
                     done);
    }

    // z = M^{-1} r with one kernel per colour sweep, restriction and prolongation
    // (uaamg_preconditioner_3d.cpp:183-196 step by step); kept as the cross-check
    // of the fused V-cycle.
    template <int DIM>
    void vcycle_sweeps(const T* r, T* z, const int* done) {
        const int nl = (int)lv_.size();
        const dim3 blk = cell_block<DIM>();
        cudaMemsetAsync(z, 0, (size_t)lv_[0].g.n * sizeof(T), st_);
        for (int l = 0; l + 1 < nl; ++l) {
            const LevelView<T> v = view(l, r, z);
            sweep<DIM>(v, 1, done, l);
            sweep<DIM>(v, 0, done, l);
            const LevelBuf<T, CS>& Cl = lv_[l + 1];
            UAAMG_LAUNCH((KTag{K_RESTRICT, l, cells(v.g) * ((2.0 + DIM) * sizeof(T) + 1.0) + cells(Cl.g) * sizeof(T)}),
                         (k_restrict<DIM, T>), cell_grid<DIM>(Cl.g.nx, Cl.g.ny, Cl.g.nz), blk, v, Cl.g,
                         Cl.solid, Cl.b, done);
            cudaMemsetAsync(Cl.x, 0, (size_t)Cl.g.n * sizeof(T), st_);
        }
        coarsest<DIM>(r, z, done);
        for (int l = nl - 2; l >= 0; --l) {
            const LevelView<T> v = view(l, r, z);
            const LevelBuf<T, CS>& Cl = lv_[l + 1];
            UAAMG_LAUNCH((KTag{K_PROLONG, l, cells(v.g) * (2.0 * sizeof(T) + 1.0) + cells(Cl.g) * (sizeof(T) + 1.0)}),
                         (k_prolong<DIM, T>), cell_grid<DIM>(Cl.g.nx, Cl.g.ny, Cl.g.nz), blk, Cl.g,
                         Cl.solid, Cl.x, v.g, v.solid, v.x, done);
            sweep<DIM>(v, 0, done, l);
            sweep<DIM>(v, 1, done, l);
        }
    }

    // Coarsest level: 10 x (forward + reverse) sweeps from x = 0.
    template <int DIM>
    void coarsest(const T* r, T* z, const int* done) {
        const int nl = (int)lv_.size();
        const LevelBuf<T, CS>& C = lv_[nl - 1];
        T* cxp = nl == 1 ? z : C.x;
        cudaMemsetAsync(cxp, 0, (size_t)C.g.n * sizeof(T), st_);
        LevelView<T> v = view(nl - 1, r, z);
        const int ncell = v.g.nx * v.g.ny * (DIM == 3 ? v.g.nz : 1);
        if (ncell <= 65536) {
            UAAMG_LAUNCH((KTag{K_COARSEST, nl - 1, 40.0 * cells(v.g) * ((2.0 + DIM) * sizeof(T) + 0.5)}),
                         (k_coarsest<DIM, T>), 1, 1024, v, done);
        } else {
            for (int q = 0; q < 10; ++q) {
                sweep<DIM>(v, 1, done, nl - 1); sweep<DIM>(v, 0, done, nl - 1);
                sweep<DIM>(v, 0, done, nl - 1); sweep<DIM>(v, 1, done, nl - 1);
            }
        }
    }

    MLevel<T> mlevel(int l) const {
        const LevelBuf<T, CS>& L = lv_[l];
        MLevel<T> v;
        v.g = L.g;
        v.cg = l + 1 < (int)lv_.size() ? lv_[l + 1].g : L.g;
        v.idx2 = (T)(1.0 / (L.hx * L.hx));
        v.idy2 = (T)(1.0 / (L.hy * L.hy));
        v.idz2 = L.g.nz ? (T)(1.0 / (L.hz * L.hz)) : T(0);
        // FP16 couplings are face counts times the finest level's 1/h^2 per axis
        const bool half = kHalf && !L.c32;
        v.csx = half ? (T)(1.0 / (lv_[0].hx * lv_[0].hx)) : T(1);
        v.csy = half ? (T)(1.0 / (lv_[0].hy * lv_[0].hy)) : T(1);
        v.csz = half ? (T)(1.0 / (lv_[0].hz * lv_[0].hz)) : T(1);
        v.dirichlet = dirichlet_;
        v.zc = L.zc;
        return v;
    }

    // Tensor maps of a march over level l: value slots b, [x], [cx, cy, (cz), dg]
    // (coefficients on coarse levels), the codes and, for the prolongation, the
    // next-coarser level's x as parent boxes.
    template <int DIM>
    MarchMaps maps(int l, bool hasx, bool parent) const {
        const LevelBuf<T, CS>& L = lv_[l];
        MarchMaps m;
        int q = 0;
        m.v[q++] = L.mb;
        if (hasx) m.v[q++] = L.mx;
        if (l > 0) {  // slot order of MPlan: the T boxes, then the couplings
            m.v[q++] = L.mdg;
            m.v[q++] = L.mcx;
            m.v[q++] = L.mcy;
            if (DIM == 3) m.v[q++] = L.mcz;
        }
        m.code = L.mcode;
        if (parent) m.xc = lv_[l + 1].mxq;
        return m;
    }

    // Tensor maps of a fused march over level l (boxes with a 2-cell ring); up: with
    // the next-coarser level's x as parent boxes.
    FMaps fmaps(int l, bool up) const {
        const LevelBuf<T, CS>& L = lv_[l];
        FMaps m{};
        m.b = L.fb;
        m.code = L.fcode;
        if (l > 0) {
            m.dg = L.fdg;
            m.cx = L.fcx;
            m.cy = L.fcy;
            m.cz = L.fcz;
        }
        if (up) m.xc = lv_[l + 1].mxq;
        return m;
    }

    // Tensor maps of a whole-tile box kernel over level l; up: with the next-coarser
    // level's x as parent boxes.
    BMaps bmaps(int l, bool up) const {
        const LevelBuf<T, CS>& L = lv_[l];
        BMaps m{};
        m.b = L.bb;
        m.code = L.bcode;
        if (l > 0) {
            m.dg = L.bdg;
            m.cx = L.bcx;
            m.cy = L.bcy;
            m.cz = L.bcz;
            m.trim = trim_ ? L.trim : nullptr;
        }
        if (up) m.xc = lv_[l + 1].bxq;
        return m;
    }

    // The way down through level l: b (and on coarse levels the couplings) in,
    // coarse b out.  CSL: the coupling storage of this level.
    template <int DIM, bool FINE>
    void down_level(int l, const int* done) {
        if constexpr (kHalf && !FINE) {
            if (lv_[l].c32) { down_level_cs<DIM, FINE, T>(l, done); return; }
        }
        down_level_cs<DIM, FINE, CS>(l, done);
    }

    int level_nu(int l) const { return l == 0 ? nu_fine_ : nu_coarse_; }

    template <int DIM, bool FINE, class CSL>
    void down_level_cs(int l, const int* done) {
        const int nu = level_nu(l);
        const LevelBuf<T, CS>& L = lv_[l];
        const LevelBuf<T, CS>& Cl = lv_[l + 1];
        const double c = cells(L.g), cc = cells(Cl.g), t = sizeof(T);
        const double coef = FINE ? 0.0 : DIM * (double)sizeof(CSL) + t;  // couplings + diagonal
        const dim3 grid = march_grid<DIM>(L.g, L.zc), blk(kThreads);
        // a finest level with Dirichlet walls takes the four-march path (the fused
        // finest level's branch-free cell table holds no wall terms)
        if (DIM == 3 && L.box && fused_ && nu == 1 && !(FINE && dirichlet_)) {
            // whole-tile boxes: b, code (coarse levels: diagonal, couplings) in; coarse b out
            UAAMG_LAUNCH_SMEM((KTag{K_DOWN, l, c * (t + 1.0 + coef) + cc * t}),
                              (k_level_box<T, FINE, CSL, false, false>), box_grid(L.g), blk,
                              (BPlan<T, CSL, FINE, false>::BYTES), bmaps(l, false), mlevel(l), Cl.b,
                              done, err_, partials_, cg_);
            return;
        }
        if (fused_ && nu == 1 && !(FINE && dirichlet_)) {
            // b, code (coarse levels: diagonal, couplings) in; coarse b out
            UAAMG_LAUNCH_SMEM((KTag{K_DOWN, l, c * (t + 1.0 + coef) + cc * t}),
                              (k_level_fused<DIM, T, FINE, CSL, false, false>), grid, blk,
                              (FCfg<DIM, T, CSL, FINE, false>::BYTES), fmaps(l, false), mlevel(l),
                              Cl.b, done, err_, partials_, cg_);
            return;
        }
        T* x = l == 0 ? z_ : L.x;
        UAAMG_LAUNCH_SMEM((KTag{K_FWD, l, c * (2.0 * t + 1.0 + coef)}), (k_fwd_smooth<DIM, T, FINE, CSL>),
                          grid, blk, (FwdCfg<DIM, T, FINE, CSL>::BYTES), maps<DIM>(l, false, false),
                          mlevel(l), x, done, err_);
        for (int q = 1; q < nu; ++q) {  // further forward sweeps (colour 1, then 0) on the stored x
            const LevelView<T> v = view(l, r_, z_);
            sweep<DIM>(v, 1, done, l);
            sweep<DIM>(v, 0, done, l);
        }
        UAAMG_LAUNCH_SMEM((KTag{K_RES, l, c * (2.0 * t + 1.0 + coef) + cc * t}),
                          (k_restrict_res<DIM, T, FINE, CSL>), grid, blk, (ResCfg<DIM, T, FINE, CSL>::BYTES),
                          maps<DIM>(l, true, false), mlevel(l), Cl.code, Cl.b, done, err_);
    }

    // The way up through level l: coarse x in, x out (level 0 with zdot: also the
    // CG's z sums).
    template <int DIM, bool FINE>
    void up_level(int l, const int* done, bool zdot) {
        if constexpr (kHalf && !FINE) {
            if (lv_[l].c32) { up_level_cs<DIM, FINE, T>(l, done, zdot); return; }
        }
        up_level_cs<DIM, FINE, CS>(l, done, zdot);
    }

    template <int DIM, bool FINE, class CSL>
    void up_level_cs(int l, const int* done, bool zdot) {
        const int nu = level_nu(l);
        const LevelBuf<T, CS>& L = lv_[l];
        const LevelBuf<T, CS>& Cl = lv_[l + 1];
        const double c = cells(L.g), cc = cells(Cl.g), t = sizeof(T);
        const double coef = FINE ? 0.0 : DIM * (double)sizeof(CSL) + t;  // couplings + diagonal
        const dim3 grid = march_grid<DIM>(L.g, L.zc), blk(kThreads);
        T* x = l == 0 ? z_ : L.x;
        if (DIM == 3 && L.box && fused_ && nu == 1 && !(FINE && dirichlet_)) {
            // whole-tile boxes: b, code (coarse levels: diagonal, couplings), coarse x in;
            // x out
            const KTag tag{K_UP, l, c * (2.0 * t + 1.0 + coef) + cc * t};
            if (FINE && zdot)
                UAAMG_LAUNCH_SMEM(tag, (k_level_box<T, FINE, CSL, true, true>), box_grid(L.g), blk,
                                  (BPlan<T, CSL, FINE, true>::BYTES), bmaps(l, true), mlevel(l), x, done,
                                  err_, partials_, cg_);
            else
                UAAMG_LAUNCH_SMEM(tag, (k_level_box<T, FINE, CSL, true, false>), box_grid(L.g), blk,
                                  (BPlan<T, CSL, FINE, true>::BYTES), bmaps(l, true), mlevel(l), x, done,
                                  err_, partials_, cg_);
            return;
        }
        if (fused_ && nu == 1 && !(FINE && dirichlet_)) {
            // b, code (coarse levels: diagonal, couplings), coarse x in; x out
            const KTag tag{K_UP, l, c * (2.0 * t + 1.0 + coef) + cc * t};
            if (FINE && zdot)
                UAAMG_LAUNCH_SMEM(tag, (k_level_fused<DIM, T, FINE, CSL, true, true>), grid, blk,
                                  (FCfg<DIM, T, CSL, FINE, true>::BYTES), fmaps(l, true), mlevel(l), x,
                                  done, err_, partials_, cg_);
            else
                UAAMG_LAUNCH_SMEM(tag, (k_level_fused<DIM, T, FINE, CSL, true, false>), grid, blk,
                                  (FCfg<DIM, T, CSL, FINE, true>::BYTES), fmaps(l, true), mlevel(l), x,
                                  done, err_, partials_, cg_);
            return;
        }
        UAAMG_LAUNCH_SMEM((KTag{K_UPE, l, c * (2.0 * t + 1.0 + coef) + cc * t}),
                          (k_up_even<DIM, T, FINE, CSL>), grid, blk, (UpeCfg<DIM, T, FINE, CSL>::BYTES),
                          maps<DIM>(l, false, true), mlevel(l), x, done, err_);
        if (nu > 1) {  // first reverse sweep, further reverse sweeps (colour 0, then 1), z sums
            UAAMG_LAUNCH_SMEM((KTag{K_UPO, l, c * (2.5 * t + 1.0 + coef)}),
                              (k_up_odd<DIM, T, FINE, false, CSL>), grid, blk, (UpoCfg<DIM, T, FINE, CSL>::BYTES),
                              maps<DIM>(l, true, false), mlevel(l), x, done, err_, partials_, cg_);
            const LevelView<T> v = view(l, r_, z_);
            for (int q = 1; q < nu; ++q) {
                sweep<DIM>(v, 0, done, l);
                sweep<DIM>(v, 1, done, l);
            }
            if (FINE && zdot)
                UAAMG_LAUNCH((KTag{K_ZDOT, 0, c * (2.0 * t + 1.0)}), (k_zdot<DIM, T>), vec_grid(L.g),
                             dim3(32, 8), L.g, L.solid, r_, z_, partials_, cg_);
            return;
        }
        if (zdot)
            UAAMG_LAUNCH_SMEM((KTag{K_UPO, l, c * (2.5 * t + 1.0 + coef)}),
                              (k_up_odd<DIM, T, FINE, true, CSL>), grid, blk, (UpoCfg<DIM, T, FINE, CSL>::BYTES),
                              maps<DIM>(l, true, false), mlevel(l), x, done, err_, partials_, cg_);
        else
            UAAMG_LAUNCH_SMEM((KTag{K_UPO, l, c * (2.5 * t + 1.0 + coef)}),
                              (k_up_odd<DIM, T, FINE, false, CSL>), grid, blk, (UpoCfg<DIM, T, FINE, CSL>::BYTES),
                              maps<DIM>(l, true, false), mlevel(l), x, done, err_, partials_, cg_);
    }

    // z_ = M^{-1} r_ with marches on every level down to the small-level kernel (two
    // fused marches a level, fused.cuh, or four, march.cuh); the finest level's last
    // march also reduces the CG's z sums when zdot is set.
    template <int DIM>
    void vcycle_march(const int* done, bool zdot) {
        const int nl = (int)lv_.size();
        const int lt = use_tail() ? tail_lt_ : nl - 1;  // first level below the marches
        for (int l = 0; l < lt; ++l) {
            if (l == 0) down_level<DIM, true>(l, done);
            else down_level<DIM, false>(l, done);
        }
        if (use_tail()) tail_launch<DIM>(done);
        else coarsest<DIM>(r_, z_, done);
        if (nl == 1 && zdot) {
            const Geom& g = lv_[0].g;
            UAAMG_LAUNCH((KTag{K_ZDOT, 0, cells(g) * (2.0 * sizeof(T) + 1.0)}), (k_zdot<DIM, T>),
                         vec_grid(g), dim3(32, 8), g, lv_[0].solid, r_, z_, partials_, cg_);
        }
        for (int l = lt - 1; l >= 0; --l) {
            if (l == 0) up_level<DIM, true>(l, done, zdot);
            else up_level<DIM, false>(l, done, false);
        }
    }

    // z = M^{-1} r_, then (zdot) the z sums -> mean, r.z, beta.
    template <int DIM>
    void vcycle(T* z, const int* done, bool zdot) {
        if (sweeps_) {
            vcycle_sweeps<DIM>(r_, z, done);
            if (zdot) {
                const Geom& g = lv_[0].g;
                UAAMG_LAUNCH((KTag{K_ZDOT, 0, cells(g) * (2.0 * sizeof(T) + 1.0)}), (k_zdot<DIM, T>),
                             vec_grid(g), dim3(32, 8), g, lv_[0].solid, r_, z, partials_, cg_);
            }
        } else {
            vcycle_march<DIM>(done, zdot);
        }
    }

    template <int DIM>
    void precond_impl(const double* d_r, double* d_z) {
        const Geom& g = lv_[0].g;
        UAAMG_LAUNCH((KTag{K_CAST, 0, cells(g) * (8.0 + sizeof(T))}), (k_import<DIM, T>), vec_grid(g),
                     dim3(32, 8), g, gref_, d_r, r_);
        vcycle<DIM>(z_, nullptr, false);
        UAAMG_LAUNCH((KTag{K_CAST, 0, cells(g) * (8.0 + sizeof(T))}), (k_export<DIM, T>), vec_grid(g),
                     dim3(32, 8), g, gref_, z_, d_z, 0);
    }

    // ---- PCG solve, in four stages so that many engines can interleave (batch and
    // serving): begin (right-hand side, initial residual, first preconditioner
    // application, graph capture), step (queue two iterations), poll (has the
    // device stopped?), end (solution out, exit diagnostics).

    Stencil stencil() const {
        Stencil st;
        st.idx2 = 1.0 / (dx_ * dx_);
        st.idy2 = 1.0 / (dy_ * dy_);
        st.idz2 = dim_ == 3 ? 1.0 / (dz_ * dz_) : 0.0;
        st.diag = dim_ == 3 ? 2.0 * (st.idx2 + st.idy2 + st.idz2) : 2.0 * (st.idx2 + st.idy2);
        st.dirichlet = dirichlet_;
        const bool var = dim_ == 2 && vd_ && vox_ && voy_;
        st.vsx = var ? vsx_ : 0;
        st.vd = var ? vd_ : nullptr;
        st.vox = var ? vox_ : nullptr;
        st.voy = var ? voy_ : nullptr;
        st.fs = var ? vf_[0] : nullptr;
        st.fx = var ? vf_[1] : nullptr;
        st.fy = var ? vf_[2] : nullptr;
        return st;
    }

    // z = M r (or z = r), then the z sums -> mean, r.z, beta
    template <int DIM>
    void cg_precond() {
        const Geom& g = lv_[0].g;
        if (cur_.precond) {
            vcycle<DIM>(z_, &cg_->done, true);
        } else {
            cudaMemcpyAsync(z_, r_, (size_t)g.n * sizeof(T), cudaMemcpyDeviceToDevice, st_);
            UAAMG_LAUNCH((KTag{K_ZDOT, 0, cells(g) * (2.0 * sizeof(T) + 1.0)}), (k_zdot<DIM, T>),
                         vec_grid(g), dim3(32, 8), g, lv_[0].solid, r_, z_, partials_, cg_);
        }
    }

    // One PCG iteration (pcg_3d.cpp:93-124); the search direction alternates between
    // p_ and p2_ (from_p: the current one lives in p_).
    template <int DIM>
    void cg_iteration(bool from_p) {
        const Geom& g = lv_[0].g;
        const Stencil st = stencil();
        T* pnew = from_p ? p2_ : p_;
        if (DIM == 2) {
            // z, p_old, codes (and the three coefficients) in; p, Ap out
            const double nb = st.vd ? 7.0 * sizeof(T) + 1.0 : 4.0 * sizeof(T) + 1.0;
            UAAMG_LAUNCH((KTag{K_PMATVEC, 0, cells(g) * nb}), k_pmatvec_2d<T>, flat2d_grid(g),
                         dim3(32, 8), g, lv_[0].code, z_, from_p ? p_ : p2_, pnew, ap_, st,
                         partials_, cg_);
        } else {
            MarchMaps pm = maps<DIM>(0, true, false);  // z and the current search direction
            pm.v[0] = lv_[0].mx;
            pm.v[1] = from_p ? map_p_ : map_p2_;
            const KTag tag{K_PMATVEC, 0, cells(g) * (4.0 * sizeof(T) + 1.0)};
            const int zc = lv_[0].zc;
            if (dirichlet_)
                UAAMG_LAUNCH_SMEM(tag, (k_pmatvec<DIM, T, true>), march_grid<DIM>(g, zc),
                                  dim3(kThreads), (PmvCfg<DIM, T>::BYTES), pm, g, zc, pnew, ap_, st,
                                  partials_, cg_, err_);
            else
                UAAMG_LAUNCH_SMEM(tag, (k_pmatvec<DIM, T, false>), march_grid<DIM>(g, zc),
                                  dim3(kThreads), (PmvCfg<DIM, T>::BYTES), pm, g, zc, pnew, ap_, st,
                                  partials_, cg_, err_);
        }
        const long long nvec = (long long)g.n / Vec16<T>::N;
        // x_lo, r, p, Ap in; x_lo, r out (a fold after a replacement adds x_hi in and out)
        UAAMG_LAUNCH((KTag{K_UPDATE, 0, cells(g) * (6.0 * sizeof(T))}), k_update_flat<T>,
                     max_reduce_blocks(), 256, nvec, xlo_, r_, pnew, ap_, mixed_ ? xd_ : nullptr,
                     partials_, cg_, cur_.hist);
        if (mixed_) {
            // residual replacement (when due, one iteration in replace_every; the others
            // return at once): b, x_hi, x_lo, codes in; r out
            nopdl_next_ = true;
            const KTag tag{K_REPLACE, 0, cells(g) * (17.0 + 2.0 * sizeof(T))};
            if (DIM == 3) {
                MarchMaps rm;
                rm.v[0] = map_b64_;
                rm.v[1] = map_xd_;
                rm.v[2] = map_xlo_;
                rm.code = lv_[0].mcode;
                if (dirichlet_)
                    UAAMG_LAUNCH_SMEM(tag, (k_resid_march<T, true>), march_grid<DIM>(g, rx_zc_),
                                      dim3(kThreads), (RxCfg<T>::BYTES), rm, g, rx_zc_, r_, st, partials_,
                                      cg_, 5, cur_.tol, cur_.tol_mode, err_);
                else
                    UAAMG_LAUNCH_SMEM(tag, (k_resid_march<T, false>), march_grid<DIM>(g, rx_zc_),
                                      dim3(kThreads), (RxCfg<T>::BYTES), rm, g, rx_zc_, r_, st, partials_,
                                      cg_, 5, cur_.tol, cur_.tol_mode, err_);
            } else {
                UAAMG_LAUNCH(tag, (k_resid_x64<DIM, T>), resid_grid(g), dim3(32, 8), g, lv_[0].code, b64_,
                             xd_, xlo_, r_, st, kResidZc, partials_, cg_, 5, 1, cur_.tol, cur_.tol_mode);
            }
        }
        cg_precond<DIM>();
    }

    template <int DIM>
    int begin_impl(const SolveArgs& a) {
        cur_ = a;
        const Geom g = lv_[0].g;
        const uint8_t* s = lv_[0].solid;
        const dim3 vb(32, 8);
        const dim3 vg = vec_grid(g);
        const int n = g.n;
        if (DIM == 2 && sizeof(T) == 4 && vd_ && vox_ && voy_ && vconv_ != vver_) {
            // FP32 copies of the variable-coefficient operator (once per contents)
            if (!vf_[0]) {
                for (int q = 0; q < 3; ++q)
                    if (int e = alloc(vf_[q], (size_t)n)) return e;
                if (gexec_) {  // a captured step holds the copies' (null) pointers
                    cudaStreamSynchronize(st_);
                    cudaGraphExecDestroy(gexec_);
                    gexec_ = nullptr;
                }
                gkey_ = -1;
            }
            UAAMG_LAUNCH((KTag{K_SETUP, 0, cells(g) * 36.0}), k_var_coeffs, vg, vb, g, stencil(),
                         vf_[0], vf_[1], vf_[2]);
            vconv_ = vver_;
        }
        const Stencil st = stencil();

        CGState init = {};
        init.max_iter = a.max_iter;
        init.replace_every = mixed_ ? (a.replace_every > 0 ? a.replace_every : 10) : 0;
        init.breakdown = a.tol_mode == 0 ? 1e-15 : 1e-300;
        init.dirichlet = dirichlet_;
        init.init = 1;
        *cg_host_ = init;
        if (cudaMemcpyAsync(cg_, cg_host_, sizeof(CGState), cudaMemcpyHostToDevice, st_) != cudaSuccess)
            return E_CUDA;
        cudaMemsetAsync(err_, 0, sizeof(int), st_);

        // b = -(rhs - mean), re-projected; ||b|| (pcg_3d.cpp:22-36, 80-81)
        UAAMG_LAUNCH((KTag{K_RHS, 0, cells(g) * 16.0}), (k_import<DIM, double>), vg, vb, g, gref_, a.rhs, b64_);
        UAAMG_LAUNCH((KTag{K_RHS, 0, cells(g) * 9.0}), k_sum_count<DIM>, vg, vb, g, s, b64_, partials_, cg_, 3);
        UAAMG_LAUNCH((KTag{K_RHS, 0, cells(g) * 17.0}), k_rhs_negate<DIM>, vg, vb, g, s, b64_, b64_, cg_);
        UAAMG_LAUNCH((KTag{K_RHS, 0, cells(g) * 9.0}), k_sum_count<DIM>, vg, vb, g, s, b64_, partials_, cg_, 3);
        UAAMG_LAUNCH((KTag{K_RHS, 0, cells(g) * 17.0}), k_sub_mean<DIM>, vg, vb, g, s, b64_, cg_);
        UAAMG_LAUNCH((KTag{K_RHS, 0, cells(g) * 9.0}), k_norm<DIM>, vg, vb, g, s, b64_, partials_, cg_, 4);
        if (a.warm) {  // b <- b - A x_in: the solve then finds the correction to x_in
            if (a.x_ready) cudaStreamWaitEvent(st_, a.x_ready, 0);
            UAAMG_LAUNCH((KTag{K_RHS, 0, cells(g) * 16.0}), (k_import<DIM, double>), vg, vb, g, gref_, a.x, xd_);
            UAAMG_LAUNCH((KTag{K_TRUE_RESIDUAL, 0, cells(g) * 25.0}), (k_true_residual<DIM, double>), vg, vb,
                         g, s, b64_, xd_, b64_, st, partials_, cg_, 5, 3, a.tol, a.tol_mode);
        }
        UAAMG_LAUNCH((KTag{K_RHS, 0, cells(g) * (9.0 + sizeof(T))}), (k_true_residual<DIM, T>), vg, vb, g, s,
                     b64_, (const double*)nullptr, r_, st, partials_, cg_, 5, 0, a.tol, a.tol_mode);
        cudaMemsetAsync(xlo_, 0, (size_t)n * sizeof(T), st_);
        cudaMemsetAsync(p_, 0, (size_t)n * sizeof(T), st_);
        cudaMemsetAsync(xd_, 0, (size_t)n * sizeof(double), st_);
        cg_precond<DIM>();

        // Two iterations form one step (the search direction is back in p_ after
        // it); outside profiling the step is a CUDA graph captured once per problem
        // and options.
        use_graph_ = graphs_ && !prof_on_;
        if (use_graph_) {
            const long long key = ((long long)a.precond << 2) | (use_tail() ? 2 : 0) | (sweeps_ ? 1 : 0);
            if (!gexec_ || key != gkey_ || a.hist != ghist_) {
                if (gexec_) { cudaGraphExecDestroy(gexec_); gexec_ = nullptr; }
                if (!cap_ && cudaStreamCreateWithFlags(&cap_, cudaStreamNonBlocking) != cudaSuccess)
                    return E_CUDA;
                cudaStream_t saved = st_;
                const long before = launches_;
                st_ = cap_;
                cudaGraph_t graph = nullptr;
                cudaError_t ce = cudaStreamBeginCapture(cap_, cudaStreamCaptureModeThreadLocal);
                if (ce == cudaSuccess) {
                    cg_iteration<DIM>(true);
                    cg_iteration<DIM>(false);
                    ce = cudaStreamEndCapture(cap_, &graph);
                }
                st_ = saved;
                if (ce != cudaSuccess || !graph) { cuda_error = ce != cudaSuccess ? ce : cudaErrorUnknown; return E_CUDA; }
                ce = cudaGraphInstantiate(&gexec_, graph, 0);
                cudaGraphDestroy(graph);
                if (ce != cudaSuccess) { gexec_ = nullptr; cuda_error = ce; return E_CUDA; }
                glaunches_ = launches_ - before;
                launches_ = before;
                gkey_ = key;
                ghist_ = a.hist;
            }
        }
        it_ = 0;
        nstep_ = 0;
        seen_ = 0;
        stopped_ = false;
        return E_OK;
    }

    // Queues one step (two iterations) unless max_iter is reached, then the copy of
    // the device 'done' flag into slot step % 2 and that slot's event.  Kernels
    // queued after the solve stopped return at once.
    template <int DIM>
    int step_impl() {
        // two flag slots: a third step waits until the oldest one has been polled
        if (it_ >= cur_.max_iter || nstep_ - seen_ >= 2) return E_OK;
        if (use_graph_) {
            if (cudaGraphLaunch(gexec_, st_) != cudaSuccess) return E_CUDA;
            launches_ += glaunches_;
        } else {
            cg_iteration<DIM>(true);
            if (it_ + 1 < cur_.max_iter) cg_iteration<DIM>(false);
        }
        it_ += 2;
        const int slot = nstep_ & 1;
        cudaMemcpyAsync(&flag_host_[slot], &cg_->done, sizeof(int), cudaMemcpyDeviceToHost, st_);
        cudaEventRecord(ev_[slot], st_);
        ++nstep_;
        return E_OK;
    }

    template <int DIM>
    int end_enqueue() {
        const Geom g = lv_[0].g;
        const dim3 vb(32, 8);
        const dim3 vg = vec_grid(g);
        const Stencil st = stencil();
        const SolveArgs& a = cur_;
        // the solution: x_hi + x_lo in mixed mode, else the working x alone
        const double* xhi = mixed_ ? xd_ : nullptr;
        const double xb = (mixed_ ? 8.0 : 0.0) + sizeof(T);
        // exit diagnostics: FP64 true residual of the accumulated solution
        UAAMG_LAUNCH((KTag{K_TRUE_RESIDUAL, 0, cells(g) * (9.0 + xb)}), (k_resid_x64<DIM, T>),
                     resid_grid(g), dim3(32, 8), g, lv_[0].code, b64_, xhi, xlo_, (T*)nullptr, st,
                     kResidZc, partials_, cg_, 5, 2, a.tol, a.tol_mode);
        if (a.x_ready) cudaStreamWaitEvent(st_, a.x_ready, 0);  // the caller's x, accumulated into
        UAAMG_LAUNCH((KTag{K_OUTPUT, 0, cells(g) * (16.0 + xb)}), (k_export_x<DIM, T>), vg, vb, g, gref_,
                     xhi, xlo_, a.x, 1);
        if (a.project_mean && a.ref_solid) {
            const dim3 rg = vec_grid(gref_);
            UAAMG_LAUNCH((KTag{K_OUTPUT, 0, cells(g) * 9.0}), k_sum_count<DIM>, rg, vb, gref_, a.ref_solid,
                         a.x, partials_, cg_, 3);
            UAAMG_LAUNCH((KTag{K_OUTPUT, 0, cells(g) * 17.0}), k_sub_mean<DIM>, rg, vb, gref_, a.ref_solid,
                         a.x, cg_);
        }
        if (cudaMemcpyAsync(cg_host_, cg_, sizeof(CGState), cudaMemcpyDeviceToHost, st_) != cudaSuccess)
            return E_CUDA;
        return E_OK;
    }
};

#undef UAAMG_LAUNCH
#undef UAAMG_LAUNCH_SMEM

}  // namespace
}  // namespace uaamg
