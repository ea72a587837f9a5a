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
#pragma once
#include <vector>

#include "engine.h"
#include "fused.cuh"
#include "kernels.cuh"

namespace uaamg {
namespace {

template <class T>
struct LevelBuf {
    Geom g;
    double hx, hy, hz;
    uint8_t* solid = nullptr;
    T *cx = nullptr, *cy = nullptr, *cz = nullptr, *wd = nullptr;
    T *x = nullptr, *b = nullptr;  // level >= 1 only (level 0 uses the CG's r and z)
};

// Kernel classes for the in-situ per-kernel timing (uaamg_profile_solve).
enum KClass : int {
    K_SWEEP = 0, K_RESTRICT, K_PROLONG, K_COARSEST, K_PMATVEC, K_UPDATE, K_ZDOT, K_VDOWN,
    K_VUP, K_TRUE_RESIDUAL, K_FOLD, K_RHS, K_OUTPUT, K_CAST, K_SETUP, K_SCALAR, K_NCLASS
};
static const char* const kclass_names[K_NCLASS] = {
    "rbgs_sweep", "restrict_residual", "prolong_add", "coarsest_solve", "p_matvec_dot",
    "cg_update", "z_dot", "vcycle_down", "vcycle_up", "true_residual", "fold", "rhs_prepare",
    "output", "cast", "hierarchy_setup", "scalar"};

struct KTag {
    int cls;
    int level;
    double bytes;  // algorithmic (compulsory) bytes of this launch
};

#define UAAMG_LAUNCH(tag, kern, grid, block, ...)                         \
    do {                                                                  \
        const KTag tg_ = (tag);                                           \
        cudaEvent_t e0_ = nullptr, e1_ = nullptr;                         \
        if (prof_on_) prof_begin(tg_, &e0_, &e1_);                        \
        kern<<<(grid), (block), 0, st_>>>(__VA_ARGS__);                   \
        if (prof_on_) cudaEventRecord(e1_, st_);                          \
        ++launches_;                                                      \
    } while (0)

#define UAAMG_LAUNCH_SMEM(tag, kern, grid, block, smem, ...)              \
    do {                                                                  \
        const KTag tg_ = (tag);                                           \
        cudaEvent_t e0_ = nullptr, e1_ = nullptr;                         \
        if (prof_on_) prof_begin(tg_, &e0_, &e1_);                        \
        kern<<<(grid), (block), (smem), st_>>>(__VA_ARGS__);              \
        if (prof_on_) cudaEventRecord(e1_, st_);                          \
        ++launches_;                                                      \
    } while (0)

// Fused V-cycle tile shapes (cells per block tile; 256 threads per block).
template <int DIM> struct VTile;
template <> struct VTile<3> { static constexpr int X = 32, Y = 8, Z = 8; };
template <> struct VTile<2> { static constexpr int X = 64, Y = 32, Z = 1; };

template <class T>
class EngineT final : public Engine {
public:
    explicit EngineT(bool mixed) : mixed_(mixed) {}
    ~EngineT() override { release(); }

    int set_problem(int dim, int nx, int ny, int nz, double dx, double dy, double dz,
                    const uint8_t* d_solid, int dirichlet) override {
        release();
        if (dim != 2 && dim != 3) return E_ARG;
        if (nx < 2 || ny < 2 || (dim == 3 && nz < 2)) return E_ARG;
        dim_ = dim; dirichlet_ = dirichlet;
        dx_ = dx; dy_ = dy; dz_ = dim == 3 ? dz : 1.0;
        int e = dim == 3 ? build<3>(nx, ny, nz, d_solid) : build<2>(nx, ny, nz, d_solid);
        if (e != E_OK) { release(); return e; }
        return E_OK;
    }

    int precond_apply(const double* d_r, double* d_z) override {
        if (lv_.empty()) return E_NOPROB;
        launches_ = 0;
        const int n = lv_[0].g.n;
        const int tb = 256, nb = (n + tb - 1) / tb;
        const T* r = nullptr;
        T* z = nullptr;
        if (sizeof(T) == sizeof(double)) {
            r = reinterpret_cast<const T*>(d_r);
            z = reinterpret_cast<T*>(d_z);
        } else {
            UAAMG_LAUNCH((KTag{K_CAST, 0, 12.0 * n}), k_cast_from_f64<T>, nb, tb, d_r, r_, n);
            r = r_;
            z = z_;
        }
        if (dim_ == 3) vcycle<3>(r, z, nullptr, false); else vcycle<2>(r, z, nullptr, false);
        if (sizeof(T) != sizeof(double)) UAAMG_LAUNCH((KTag{K_CAST, 0, 12.0 * n}), k_cast_to_f64<T>, nb, tb, z_, d_z, n);
        return sync_check();
    }

    int solve(const SolveArgs& a, SolveResult* res) override {
        if (lv_.empty()) return E_NOPROB;
        launches_ = 0;
        int e = dim_ == 3 ? solve_impl<3>(a) : solve_impl<2>(a);
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

    int nlevels() const override { return (int)lv_.size(); }

    void level_dims(int l, int* nx, int* ny, int* nz) const override {
        *nx = lv_[l].g.nx; *ny = lv_[l].g.ny; *nz = lv_[l].g.nz;
    }

    int copy_level(int l, uint8_t* solid, double* cx, double* cy, double* cz) override {
        if (l < 0 || l >= (int)lv_.size()) return E_ARG;
        const LevelBuf<T>& L = lv_[l];
        const size_t n = (size_t)L.g.n;
        if (cudaStreamSynchronize(st_) != cudaSuccess) return E_CUDA;
        if (solid && cudaMemcpy(solid, L.solid, n, cudaMemcpyDeviceToHost) != cudaSuccess)
            return E_CUDA;
        std::vector<T> tmp(n);
        const T* src[3] = {L.cx, L.cy, L.cz};
        double* dst[3] = {cx, cy, cz};
        for (int q = 0; q < 3; ++q) {
            if (!dst[q]) continue;
            if (!src[q]) { for (size_t c = 0; c < n; ++c) dst[q][c] = 0.0; continue; }
            if (cudaMemcpy(tmp.data(), src[q], n * sizeof(T), cudaMemcpyDeviceToHost) != cudaSuccess)
                return E_CUDA;
            for (size_t c = 0; c < n; ++c) dst[q][c] = (double)tmp[c];
        }
        return E_OK;
    }

    void set_stream(cudaStream_t s) override { st_ = s; }
    size_t device_bytes() const override { return bytes_; }
    long launches() const override { return launches_; }

    void set_vcycle_sweeps(bool on) override { sweeps_ = on; }

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
        return E_OK;
    }

private:
    bool mixed_;
    int dim_ = 0, dirichlet_ = 0;
    double dx_ = 1, dy_ = 1, dz_ = 1;
    std::vector<LevelBuf<T>> lv_;
    T *r_ = nullptr, *z_ = nullptr, *p_ = nullptr, *p2_ = nullptr, *ap_ = nullptr, *xlo_ = nullptr;
    int num_sms_ = 148;
    bool sweeps_ = false;  // V-cycle as per-colour sweeps (cross-check) instead of fused
    int max_reduce_blocks() const { return 4 * num_sms_; }
    // grid of the row-walk kernels (kernels.cuh for_cells): capped at 4 blocks per SM
    dim3 vec_grid(const Geom& g) const {
        const long long items = (long long)g.ny * (g.nz ? g.nz : 1) * ((g.nx + 31) / 32);
        long long nb = (items + 7) / 8;
        if (nb > max_reduce_blocks()) nb = max_reduce_blocks();
        return dim3((unsigned)(nb < 1 ? 1 : nb));
    }
    double *b64_ = nullptr, *xd_ = nullptr, *partials_ = nullptr;
    CGState* cg_ = nullptr;
    CGState* cg_host_ = nullptr;  // pinned
    int* flag_host_ = nullptr;    // pinned, 2 slots
    cudaEvent_t ev_[2] = {nullptr, nullptr};
    cudaStream_t st_ = 0;
    std::vector<void*> allocs_;
    size_t bytes_ = 0;
    long launches_ = 0;
    // in-situ per-launch timing (set_profiling)
    bool prof_on_ = false;
    int prof_count_ = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_ev_;
    std::vector<KTag> prof_tag_;

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
        if (cudaMalloc(&q, count * sizeof(P)) != cudaSuccess) {
            cudaGetLastError();
            return E_OOM;
        }
        allocs_.push_back(q);
        bytes_ += count * sizeof(P);
        if (cudaMemsetAsync(q, 0, count * sizeof(P), st_) != cudaSuccess) return E_CUDA;
        p = static_cast<P*>(q);
        return E_OK;
    }

    void release() {
        if (!allocs_.empty() || cg_host_) cudaStreamSynchronize(st_);
        for (void* q : allocs_) cudaFree(q);
        allocs_.clear();
        lv_.clear();
        bytes_ = 0;
        r_ = z_ = p_ = p2_ = ap_ = xlo_ = nullptr;
        b64_ = xd_ = partials_ = nullptr;
        cg_ = nullptr;
        if (cg_host_) { cudaFreeHost(cg_host_); cg_host_ = nullptr; }
        if (flag_host_) { cudaFreeHost(flag_host_); flag_host_ = nullptr; }
        for (auto& e : ev_) if (e) { cudaEventDestroy(e); e = nullptr; }
        for (auto& pr : prof_ev_) { cudaEventDestroy(pr.first); cudaEventDestroy(pr.second); }
        prof_ev_.clear();
        prof_tag_.clear();
        prof_count_ = 0;
    }

    int sync_check() {
        cudaError_t e = cudaStreamSynchronize(st_);
        if (e == cudaSuccess) e = cudaGetLastError();
        return e == cudaSuccess ? E_OK : E_CUDA;
    }

    template <int DIM>
    int build(int nx, int ny, int nz, const uint8_t* d_solid) {
        double hx = dx_, hy = dy_, hz = dz_;
        while (nx >= 2 && ny >= 2 && (DIM == 2 || nz >= 2)) {
            LevelBuf<T> L;
            L.g = make_geom(DIM, nx, ny, nz);
            L.hx = hx; L.hy = hy; L.hz = hz;
            lv_.push_back(L);
            if (nx <= 4 || ny <= 4 || (DIM == 3 && nz <= 4)) break;
            nx /= 2; ny /= 2; nz /= 2;
            hx *= 2.0; hy *= 2.0; hz *= 2.0;
        }
        const int nl = (int)lv_.size();
        int e;
        for (int l = 0; l < nl; ++l) {
            LevelBuf<T>& L = lv_[l];
            const size_t n = (size_t)L.g.n;
            if ((e = alloc(L.solid, n))) return e;
            if ((e = alloc(L.cx, n))) return e;
            if ((e = alloc(L.cy, n))) return e;
            if (DIM == 3 && (e = alloc(L.cz, n))) return e;
            if (dirichlet_ && (e = alloc(L.wd, n))) return e;
            if (l > 0) {
                if ((e = alloc(L.x, n))) return e;
                if ((e = alloc(L.b, n))) return e;
            }
        }
        const Geom g0 = lv_[0].g;
        const size_t n0 = (size_t)g0.n;
        if ((e = alloc(r_, n0)) || (e = alloc(z_, n0)) || (e = alloc(p_, n0)) ||
            (e = alloc(ap_, n0)) || (e = alloc(xlo_, n0)) || (e = alloc(b64_, n0)) ||
            (e = alloc(xd_, n0)))
            return e;
        const dim3 blk = cell_block<DIM>();
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
            return E_CUDA;
        if ((e = alloc(p2_, n0))) return e;
        if ((e = alloc(partials_, (size_t)max_reduce_blocks() * 4))) return e;
        {
            using TG = TileGeo<DIM, VTile<DIM>::X, VTile<DIM>::Y, VTile<DIM>::Z>;
            const int sm = (int)TG::template smem_bytes<T>();
            cudaFuncSetAttribute(k_vdown<DIM, T, VTile<DIM>::X, VTile<DIM>::Y, VTile<DIM>::Z>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
            cudaFuncSetAttribute(k_vup<DIM, T, VTile<DIM>::X, VTile<DIM>::Y, VTile<DIM>::Z, false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
            cudaFuncSetAttribute(k_vup<DIM, T, VTile<DIM>::X, VTile<DIM>::Y, VTile<DIM>::Z, true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, sm);
        }
        if ((e = alloc(cg_, 1))) return e;
        if (cudaMallocHost(&cg_host_, sizeof(CGState)) != cudaSuccess) return E_OOM;
        if (cudaMallocHost(&flag_host_, 2 * sizeof(int)) != cudaSuccess) return E_OOM;
        for (auto& ev : ev_)
            if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) return E_CUDA;

        if (cudaMemcpyAsync(lv_[0].solid, d_solid, n0, cudaMemcpyDeviceToDevice, st_) != cudaSuccess)
            return E_CUDA;
        for (int l = 1; l < nl; ++l)
            UAAMG_LAUNCH((KTag{K_SETUP, l, 0.0}), k_restrict_solid<DIM>, cell_grid<DIM>(lv_[l].g.nx, lv_[l].g.ny, lv_[l].g.nz),
                         blk, lv_[l - 1].g, lv_[l - 1].solid, lv_[l].g, lv_[l].solid);
        {
            const LevelBuf<T>& L = lv_[0];
            const T idx2 = (T)(1.0 / (L.hx * L.hx)), idy2 = (T)(1.0 / (L.hy * L.hy));
            const T idz2 = DIM == 3 ? (T)(1.0 / (L.hz * L.hz)) : T(0);
            UAAMG_LAUNCH((KTag{K_SETUP, 0, 0.0}), (k_fine_coeffs<DIM, T>), cell_grid<DIM>(L.g.nx, L.g.ny, L.g.nz), blk, L.g,
                         L.solid, L.cx, L.cy, L.cz, L.wd, idx2, idy2, idz2);
        }
        for (int l = 1; l < nl; ++l) {
            const LevelBuf<T>& F = lv_[l - 1];
            LevelBuf<T>& Cl = lv_[l];
            UAAMG_LAUNCH((KTag{K_SETUP, l, 0.0}), (k_galerkin<DIM, T>), cell_grid<DIM>(Cl.g.nx, Cl.g.ny, Cl.g.nz), blk, F.g,
                         F.cx, F.cy, F.cz, F.wd, Cl.g, Cl.solid, Cl.cx, Cl.cy, Cl.cz, Cl.wd);
        }
        return sync_check();
    }

    LevelView<T> view(int l, const T* r, T* z) const {
        const LevelBuf<T>& L = lv_[l];
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
        UAAMG_LAUNCH((KTag{K_SWEEP, lvl, cells(v.g) * ((2.0 + DIM) * sizeof(T) + 0.5)}), (k_sweep<DIM, T>), cell_grid<DIM>((v.g.nx + 1) / 2, v.g.ny, v.g.nz),
                     cell_block<DIM>(), v, parity, done);
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
            const LevelBuf<T>& Cl = lv_[l + 1];
            UAAMG_LAUNCH((KTag{K_RESTRICT, l, cells(v.g) * ((2.0 + DIM) * sizeof(T) + 1.0) + cells(Cl.g) * sizeof(T)}), (k_restrict<DIM, T>), cell_grid<DIM>(Cl.g.nx, Cl.g.ny, Cl.g.nz), blk, v, Cl.g,
                         Cl.solid, Cl.b, done);
            cudaMemsetAsync(Cl.x, 0, (size_t)Cl.g.n * sizeof(T), st_);
        }
        {
            const LevelView<T> v = view(nl - 1, r, z);
            const int ncell = v.g.nx * v.g.ny * (DIM == 3 ? v.g.nz : 1);
            if (ncell <= 65536) {
                UAAMG_LAUNCH((KTag{K_COARSEST, nl - 1, 40.0 * cells(v.g) * ((2.0 + DIM) * sizeof(T) + 0.5)}), (k_coarsest<DIM, T>), 1, 1024, v, done);
            } else {
                for (int s = 0; s < 10; ++s) {
                    sweep<DIM>(v, 1, done, nl - 1); sweep<DIM>(v, 0, done, nl - 1);
                    sweep<DIM>(v, 0, done, nl - 1); sweep<DIM>(v, 1, done, nl - 1);
                }
            }
        }
        for (int l = nl - 2; l >= 0; --l) {
            const LevelView<T> v = view(l, r, z);
            const LevelBuf<T>& Cl = lv_[l + 1];
            UAAMG_LAUNCH((KTag{K_PROLONG, l, cells(v.g) * (2.0 * sizeof(T) + 1.0) + cells(Cl.g) * (sizeof(T) + 1.0)}), (k_prolong<DIM, T>), cell_grid<DIM>(Cl.g.nx, Cl.g.ny, Cl.g.nz), blk, Cl.g,
                         Cl.solid, Cl.x, v.g, v.solid, v.x, done);
            sweep<DIM>(v, 0, done, l);
            sweep<DIM>(v, 1, done, l);
        }
    }

    VLevel<T> vlevel(int l) const {
        const LevelBuf<T>& L = lv_[l];
        VLevel<T> v;
        v.g = L.g;
        v.solid = L.solid;
        v.cx = l == 0 ? nullptr : L.cx;
        v.cy = L.cy; v.cz = L.cz;
        v.wd = L.wd;
        v.idx2 = (T)(1.0 / (L.hx * L.hx));
        v.idy2 = (T)(1.0 / (L.hy * L.hy));
        v.idz2 = L.g.nz ? (T)(1.0 / (L.hz * L.hz)) : T(0);
        v.dirichlet = dirichlet_;
        return v;
    }

    // z = M^{-1} r with one fused kernel per level down (sweep + residual +
    // restriction) and one per level up (prolongation + sweep), fused.cuh; the
    // finest up kernel also reduces the CG's z sums when zdot is set.
    template <int DIM>
    void vcycle_fused(const T* r, T* z, const int* done, bool zdot) {
        constexpr int TX = VTile<DIM>::X, TY = VTile<DIM>::Y, TZ = VTile<DIM>::Z;
        using TG = TileGeo<DIM, TX, TY, TZ>;
        const int nl = (int)lv_.size();
        const size_t sm = TG::template smem_bytes<T>();
        const int per_sm = sm > 60000 ? 2 : 4;
        auto tiles = [&](const Geom& g, int& ntx, int& nty, int& nt) {
            ntx = (g.nx + TX - 1) / TX;
            nty = (g.ny + TY - 1) / TY;
            const int ntz = DIM == 3 ? (g.nz + TZ - 1) / TZ : 1;
            nt = ntx * nty * ntz;
        };
        for (int l = 0; l + 1 < nl; ++l) {
            const LevelBuf<T>& L = lv_[l];
            const LevelBuf<T>& Cl = lv_[l + 1];
            int ntx, nty, nt;
            tiles(L.g, ntx, nty, nt);
            const int grid = nt < per_sm * num_sms_ ? nt : per_sm * num_sms_;
            const double bytes = cells(L.g) * (sizeof(T) + 1.0 + (l ? DIM * sizeof(T) : 0.0)) +
                                 cells(Cl.g) * sizeof(T);
            UAAMG_LAUNCH_SMEM((KTag{K_VDOWN, l, bytes}), (k_vdown<DIM, T, TX, TY, TZ>), grid, 256, sm,
                              vlevel(l), l == 0 ? r : (const T*)L.b, Cl.g, Cl.solid, Cl.b, ntx, nty, nt,
                              done);
        }
        {
            const LevelBuf<T>& C = lv_[nl - 1];
            T* cx_ = nl == 1 ? z : C.x;
            cudaMemsetAsync(cx_, 0, (size_t)C.g.n * sizeof(T), st_);
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
            if (nl == 1 && zdot)
                UAAMG_LAUNCH((KTag{K_ZDOT, 0, cells(C.g) * (2.0 * sizeof(T) + 1.0)}), (k_zdot<DIM, T>),
                             vec_grid(C.g), dim3(32, 8), C.g, C.solid, r, z, partials_, cg_);
        }
        for (int l = nl - 2; l >= 0; --l) {
            const LevelBuf<T>& L = lv_[l];
            const LevelBuf<T>& Cl = lv_[l + 1];
            int ntx, nty, nt;
            tiles(L.g, ntx, nty, nt);
            const int grid = nt < per_sm * num_sms_ ? nt : per_sm * num_sms_;
            const double bytes = cells(L.g) * (2.0 * sizeof(T) + 1.0 + (l ? DIM * sizeof(T) : 0.0)) +
                                 cells(Cl.g) * (sizeof(T) + 1.0);
            const T* b = l == 0 ? r : (const T*)L.b;
            T* x = l == 0 ? z : L.x;
            if (l == 0 && zdot)
                UAAMG_LAUNCH_SMEM((KTag{K_VUP, l, bytes}), (k_vup<DIM, T, TX, TY, TZ, true>), grid, 256, sm,
                                  vlevel(l), b, Cl.g, Cl.solid, Cl.x, x, ntx, nty, nt, done, partials_, cg_);
            else
                UAAMG_LAUNCH_SMEM((KTag{K_VUP, l, bytes}), (k_vup<DIM, T, TX, TY, TZ, false>), grid, 256, sm,
                                  vlevel(l), b, Cl.g, Cl.solid, Cl.x, x, ntx, nty, nt, done, partials_, cg_);
        }
    }

    template <int DIM>
    void vcycle(const T* r, T* z, const int* done, bool zdot) {
        if (sweeps_) {
            vcycle_sweeps<DIM>(r, z, done);
            if (zdot) {
                const Geom& g = lv_[0].g;
                UAAMG_LAUNCH((KTag{K_ZDOT, 0, cells(g) * (2.0 * sizeof(T) + 1.0)}), (k_zdot<DIM, T>),
                             vec_grid(g), dim3(32, 8), g, lv_[0].solid, r, z, partials_, cg_);
            }
        } else {
            vcycle_fused<DIM>(r, z, done, zdot);
        }
    }

    template <int DIM>
    int solve_impl(const SolveArgs& a) {
        const Geom g = lv_[0].g;
        const uint8_t* s = lv_[0].solid;
        const dim3 vb(32, 8);
        const dim3 vg = vec_grid(g);
        const int n = g.n;
        Stencil st;
        st.idx2 = 1.0 / (dx_ * dx_);
        st.idy2 = 1.0 / (dy_ * dy_);
        st.idz2 = DIM == 3 ? 1.0 / (dz_ * dz_) : 0.0;
        st.diag = DIM == 3 ? 2.0 * (st.idx2 + st.idy2 + st.idz2) : 2.0 * (st.idx2 + st.idy2);
        st.dirichlet = dirichlet_;

        CGState init = {};
        init.max_iter = a.max_iter;
        init.replace_every = mixed_ ? (a.replace_every > 0 ? a.replace_every : 10) : 0;
        init.breakdown = a.tol_mode == 0 ? 1e-15 : 1e-300;
        init.dirichlet = dirichlet_;
        init.init = 1;
        *cg_host_ = init;
        if (cudaMemcpyAsync(cg_, cg_host_, sizeof(CGState), cudaMemcpyHostToDevice, st_) != cudaSuccess)
            return E_CUDA;

        // b = -(rhs - mean), re-projected; ||b|| (pcg_3d.cpp:22-36, 80-81)
        UAAMG_LAUNCH((KTag{K_RHS, 0, cells(g) * 9.0}), k_sum_count<DIM>, vg, vb, g, s, a.rhs, partials_, cg_, 3);
        UAAMG_LAUNCH((KTag{K_RHS, 0, cells(g) * 17.0}), k_rhs_negate<DIM>, vg, vb, g, s, a.rhs, b64_, cg_);
        UAAMG_LAUNCH((KTag{K_RHS, 0, cells(g) * 9.0}), k_sum_count<DIM>, vg, vb, g, s, b64_, partials_, cg_, 3);
        UAAMG_LAUNCH((KTag{K_RHS, 0, cells(g) * 17.0}), k_sub_mean<DIM>, vg, vb, g, s, b64_, cg_);
        UAAMG_LAUNCH((KTag{K_RHS, 0, cells(g) * 9.0}), k_norm<DIM>, vg, vb, g, s, b64_, partials_, cg_, 4);
        if (a.warm)  // b <- b - A x_in: the solve then finds the correction to x_in
            UAAMG_LAUNCH((KTag{K_TRUE_RESIDUAL, 0, cells(g) * 25.0}), (k_true_residual<DIM, double>), vg, vb,
                         g, s, b64_, a.x, b64_, st, partials_, cg_, 5, 3, a.tol, a.tol_mode);
        UAAMG_LAUNCH((KTag{K_RHS, 0, cells(g) * (9.0 + sizeof(T))}), (k_true_residual<DIM, T>), vg, vb, g, s,
                     b64_, (const double*)nullptr, r_, st, partials_, cg_, 5, 0, a.tol, a.tol_mode);
        cudaMemsetAsync(xlo_, 0, (size_t)n * sizeof(T), st_);
        cudaMemsetAsync(p_, 0, (size_t)n * sizeof(T), st_);
        if (mixed_) cudaMemsetAsync(xd_, 0, (size_t)n * sizeof(double), st_);

        const int* done = &cg_->done;
        // z = M r (or z = r), then the z sums -> mean, r.z, beta
        auto precond = [&]() {
            if (a.precond) {
                vcycle<DIM>(r_, z_, done, true);
            } else {
                cudaMemcpyAsync(z_, r_, (size_t)n * sizeof(T), cudaMemcpyDeviceToDevice, st_);
                UAAMG_LAUNCH((KTag{K_ZDOT, 0, cells(g) * (2.0 * sizeof(T) + 1.0)}), (k_zdot<DIM, T>), vg, vb,
                             g, s, r_, z_, partials_, cg_);
            }
        };
        precond();
        T* pc = p_;   // current search direction
        T* pn = p2_;  // next
        for (int it = 0; it < a.max_iter; ++it) {
            UAAMG_LAUNCH((KTag{K_PMATVEC, 0, cells(g) * (4.0 * sizeof(T) + 1.0)}), (k_pmatvec<DIM, T>), vg, vb,
                         g, s, z_, pc, pn, ap_, st, partials_, cg_);
            T* t = pc; pc = pn; pn = t;
            UAAMG_LAUNCH((KTag{K_UPDATE, 0, cells(g) * (6.0 * sizeof(T))}), (k_update<DIM, T>), vg, vb, g,
                         xlo_, r_, pc, ap_, partials_, cg_, a.hist);
            if (mixed_) {
                UAAMG_LAUNCH((KTag{K_FOLD, 0, cells(g) * (16.0 + 2.0 * sizeof(T) + 1.0)}), (k_fold<DIM, T>), vg,
                             vb, g, s, xd_, xlo_, cg_, 0);
                UAAMG_LAUNCH((KTag{K_TRUE_RESIDUAL, 0, cells(g) * (17.0 + sizeof(T))}), (k_true_residual<DIM, T>),
                             vg, vb, g, s, b64_, xd_, r_, st, partials_, cg_, 5, 1, a.tol, a.tol_mode);
                UAAMG_LAUNCH((KTag{K_SCALAR, 0, 0.0}), k_maxiter_check, 1, 1, cg_);
            }
            precond();
            // Poll the device 'done' flag one iteration behind, so the host never
            // idles the GPU waiting for a scalar.
            const int slot = it & 1;
            cudaMemcpyAsync(&flag_host_[slot], done, sizeof(int), cudaMemcpyDeviceToHost, st_);
            cudaEventRecord(ev_[slot], st_);
            if (it > 0) {
                if (cudaEventSynchronize(ev_[slot ^ 1]) != cudaSuccess) return E_CUDA;
                if (flag_host_[slot ^ 1]) break;
            }
        }

        const int tb = 256, nb = (n + tb - 1) / tb;
        if (mixed_) {
            UAAMG_LAUNCH((KTag{K_FOLD, 0, cells(g) * (16.0 + 2.0 * sizeof(T) + 1.0)}), (k_fold<DIM, T>), vg, vb,
                         g, s, xd_, xlo_, cg_, 1);
        } else if (sizeof(T) == sizeof(double)) {
            cudaMemcpyAsync(xd_, xlo_, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st_);
        } else {
            UAAMG_LAUNCH((KTag{K_CAST, 0, 12.0 * n}), k_cast_to_f64<T>, nb, tb, xlo_, xd_, n);
        }
        // exit diagnostics: FP64 true residual of the accumulated solution
        UAAMG_LAUNCH((KTag{K_TRUE_RESIDUAL, 0, cells(g) * 17.0}), (k_true_residual<DIM, T>), vg, vb, g, s,
                     b64_, xd_, (T*)nullptr, st, partials_, cg_, 5, 2, a.tol, a.tol_mode);
        UAAMG_LAUNCH((KTag{K_OUTPUT, 0, cells(g) * 25.0}), (k_output<DIM, double>), vg, vb, g, s, xd_, a.x);
        if (a.project_mean) {
            UAAMG_LAUNCH((KTag{K_OUTPUT, 0, cells(g) * 9.0}), k_sum_count<DIM>, vg, vb, g, s, a.x, partials_,
                         cg_, 3);
            UAAMG_LAUNCH((KTag{K_OUTPUT, 0, cells(g) * 17.0}), k_sub_mean<DIM>, vg, vb, g, s, a.x, cg_);
        }
        if (cudaMemcpyAsync(cg_host_, cg_, sizeof(CGState), cudaMemcpyDeviceToHost, st_) != cudaSuccess)
            return E_CUDA;
        return sync_check();
    }
};

#undef UAAMG_LAUNCH
#undef UAAMG_LAUNCH_SMEM

}  // namespace
}  // namespace uaamg
