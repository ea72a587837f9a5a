// Allocation-free residual check: uaamg_residual_noalloc (include/uaamg.h).
//
// Some callers cannot call cudaMalloc at all: code that runs while a stream is
// being captured into a CUDA graph (allocation is not a capturable operation),
// code inside a host callback or a custom allocator hook (no CUDA API calls that
// may allocate), or a host application that hands this library a fixed memory
// budget and owns every device allocation itself.  For them this entry point
// measures how well a pressure field p solves lap(p) = rhs -- the FP64 true
// residual ||b - A p|| and ||b|| of PCG::solve's normalised right-hand side b --
// without allocating: its only scratch (per-block partial sums, the fluid mean
// and the last-block counters) lives in the file-scope device array below, which
// every GPU that loads the library holds until the process exits.
//
// Set-up: the first call on a device, with that device current, looks up the
// array's device address (cudaGetSymbolAddress) once; make that first call before
// any stream capture.  The address belongs to the device's current context: if the
// application resets the device (cudaDeviceReset) or otherwise replaces its primary
// context, the next call sees a new context id and looks the address up again
// (again a set-up call: make it before any capture).  Every call on a device shares the one array and leaves its
// contents behind; each call clears the counters it relies on before use.  Two
// calls whose kernels overlap on the GPU (different streams, no ordering between
// them) race on the array and give wrong results: order them on one stream.
#include "../../include/uaamg.h"

#include <cuda.h>

#include <mutex>

#include "kernels.cuh"

namespace {

// Reduction blocks the two kernels use at most (their grids are capped here and
// walk the grid with a stride, so any grid size fits this scratch).
constexpr int kNoAllocBlocks = 1024;
// Layout of the scratch, in doubles: partials (kNoAllocBlocks x 2), the fluid
// sum/count (2), then 2 counters stored in the bytes of one more double each.
constexpr int kPartials = 0;
constexpr int kSums = kNoAllocBlocks * 2;
constexpr int kCounters = kSums + 2;
constexpr int kScratchDoubles = kCounters + 2;

constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};  // context id the address belongs to
std::mutex g_setup_mutex;

}  // namespace

// 16.4 KiB of device memory per GPU that loads the library.
static __device__ __align__(256) double g_uaamg_noalloc_scratch[kScratchDoubles];

namespace {

using uaamg::cidx;
using uaamg::Geom;

// Pass 1: fluid sum and count of rhs (reference layout).
template <int DIM>
__global__ void k_na_sum(Geom g, const uint8_t* __restrict__ s, const double* __restrict__ rhs,
                         double* scratch) {
    double acc[2] = {0.0, 0.0};
    uaamg::for_cells<DIM>(g, [&](int, int, int, int id) {
        if (!s[id]) { acc[0] += rhs[id]; acc[1] += 1.0; }
    });
    double tot[2];
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + kCounters);
    if (uaamg::reduce_last<2>(acc, scratch + kPartials, counter, tot)) {
        scratch[kSums] = tot[0];
        scratch[kSums + 1] = tot[1];
    }
}

// Pass 2: b = -(rhs - mean) on fluid cells, r = b - A p with the PCG operator,
// out[0] = ||r||, out[1] = ||b|| (FP64, fluid interior cells).
template <int DIM>
__global__ void k_na_residual(Geom g, const uint8_t* __restrict__ s, const double* __restrict__ rhs,
                              const double* __restrict__ p, uaamg::Stencil st, double* scratch,
                              double* out) {
    const double cnt = scratch[kSums + 1];
    const double mean = cnt > 0.0 ? scratch[kSums] / cnt : 0.0;
    double acc[2] = {0.0, 0.0};
    uaamg::for_cells<DIM>(g, [&](int i, int j, int k, int id) {
        if (s[id]) return;
        const double b = -(rhs[id] - mean);
        const double r = b - uaamg::apply_A<DIM, double>(g, s, p, i, j, k, id, st.idx2, st.idy2,
                                                         st.idz2, st.diag, 0);
        acc[0] += r * r;
        acc[1] += b * b;
    });
    double tot[2];
    unsigned int* counter = reinterpret_cast<unsigned int*>(scratch + kCounters + 1);
    if (uaamg::reduce_last<2>(acc, scratch + kPartials, counter, tot)) {
        out[0] = sqrt(tot[0]);
        out[1] = sqrt(tot[1]);
    }
}

// Id of the current context (driver entry points looked up through the runtime);
// 0 when it cannot be read.
unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void* a = nullptr;
        void* b = nullptr;
        cudaDriverEntryPointQueryResult qa, qb;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault, &qa) == cudaSuccess &&
            qa == cudaDriverEntryPointSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault, &qb) == cudaSuccess &&
            qb == cudaDriverEntryPointSuccess) {
            get_current = reinterpret_cast<GetCurrent>(a);
            get_id = reinterpret_cast<GetId>(b);
        }
        cudaGetLastError();
        looked_up = true;
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != CUDA_SUCCESS || !ctx ||
        get_id(ctx, &id) != CUDA_SUCCESS)
        return 0;
    return id;
}

// Device address of the scratch array on the current device, looked up once per
// device and context.
double* scratch_for(int dev) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    const unsigned long long ctx = current_context_id();
    if (!g_scratch_addr[dev] || ctx != g_scratch_ctx[dev]) {
        void* ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, g_uaamg_noalloc_scratch) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        g_scratch_addr[dev] = static_cast<double*>(ptr);
        g_scratch_ctx[dev] = current_context_id();  // the lookup makes the context current
    }
    return g_scratch_addr[dev];
}

}  // namespace

extern "C" uaamg_status uaamg_residual_noalloc(int dim, int nx, int ny, int nz, double dx,
                                               double dy, double dz, const uint8_t* d_solid,
                                               const double* d_rhs, const double* d_p,
                                               double* d_out, void* stream) {
    if (dim != 2 && dim != 3) return UAAMG_INVALID_ARG;
    if (nx < 2 || ny < 2 || (dim == 3 && nz < 2)) return UAAMG_INVALID_ARG;
    if (!(dx > 0) || !(dy > 0) || (dim == 3 && !(dz > 0))) return UAAMG_INVALID_ARG;
    if (!d_solid || !d_rhs || !d_p || !d_out) return UAAMG_INVALID_ARG;
    // the kernels index cells with 32-bit ints: larger grids are rejected
    const long long n = (long long)(nx + 2) * (ny + 2) * (dim == 3 ? (long long)(nz + 2) : 1);
    if (n >= (1LL << 31)) return UAAMG_INVALID_ARG;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        cudaGetLastError();
        return UAAMG_CUDA_ERROR;
    }
    double* scratch = scratch_for(dev);
    if (!scratch) return UAAMG_CUDA_ERROR;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // The last-block counters must start at 0 (a call that died mid-way could
    // have left them set).
    if (cudaMemsetAsync(scratch + kCounters, 0, 2 * sizeof(double), st) != cudaSuccess) {
        cudaGetLastError();
        return UAAMG_CUDA_ERROR;
    }
    const Geom g = uaamg::make_geom(dim, nx, ny, nz);
    uaamg::Stencil sten;
    sten.idx2 = 1.0 / (dx * dx);
    sten.idy2 = 1.0 / (dy * dy);
    sten.idz2 = dim == 3 ? 1.0 / (dz * dz) : 0.0;
    sten.diag = dim == 3 ? 2.0 * (sten.idx2 + sten.idy2 + sten.idz2) : 2.0 * (sten.idx2 + sten.idy2);
    sten.dirichlet = 0;
    const long long items = (long long)ny * (dim == 3 ? nz : 1) * ((nx + 31) / 32);
    long long nb = (items + 7) / 8;
    if (nb > kNoAllocBlocks) nb = kNoAllocBlocks;
    const dim3 grid((unsigned)nb), block(32, 8);
    if (dim == 3) {
        k_na_sum<3><<<grid, block, 0, st>>>(g, d_solid, d_rhs, scratch);
        k_na_residual<3><<<grid, block, 0, st>>>(g, d_solid, d_rhs, d_p, sten, scratch, d_out);
    } else {
        k_na_sum<2><<<grid, block, 0, st>>>(g, d_solid, d_rhs, scratch);
        k_na_residual<2><<<grid, block, 0, st>>>(g, d_solid, d_rhs, d_p, sten, scratch, d_out);
    }
    if (cudaGetLastError() != cudaSuccess) return UAAMG_CUDA_ERROR;
    return UAAMG_OK;
}
