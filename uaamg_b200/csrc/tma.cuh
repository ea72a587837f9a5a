// Tensor-memory-accelerator (TMA) tile loads for the stencil kernels: host-side
// tensor-map encoding of a level array in the pitched layout, and the device-side
// mbarrier + cp.async.bulk.tensor sequence that stages a halo box in shared
// memory.  Loads only, each block fetching its own boxes from this GPU's own memory.
//
// Alignment rules honoured here (checked on the host before encoding):
//   * array base 16-byte aligned (cudaMalloc: 256), row pitch a multiple of
//     16 bytes (make_geom_pitched);
//   * box inner extent x element size a multiple of 16 bytes;
//   * the innermost start coordinate x element size a multiple of 16 bytes
//     (callers round the start down: tile_x0); other coordinates are free and
//     may be negative or past the end (those elements read as 0).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <cuda_fp16.h>

#include <cstdint>

#include "common.cuh"

namespace uaamg {

// ---------------------------------------------------------------------------
// host

// cuTensorMapEncodeTiled from the driver, looked up once through the runtime.
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

template <class T>
inline CUtensorMapDataType tma_dtype();
template <> inline CUtensorMapDataType tma_dtype<float>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT32; }
template <> inline CUtensorMapDataType tma_dtype<double>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT64; }
template <> inline CUtensorMapDataType tma_dtype<uint8_t>() { return CU_TENSOR_MAP_DATA_TYPE_UINT8; }
template <> inline CUtensorMapDataType tma_dtype<__half>() { return CU_TENSOR_MAP_DATA_TYPE_FLOAT16; }

// Encodes a rank-2 (2D level) or rank-3 tensor map over a padded level array of
// element type E with box (bx, by[, bz]).  Returns false when the driver refuses
// the description or an alignment rule is broken.
template <class E>
inline bool encode_level_map(CUtensorMap* map, const void* base, const Geom& g, int dim, int bx,
                             int by, int bz) {
    auto enc = tensor_map_encoder();
    if (!enc) return false;
    if ((reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
    if (((size_t)g.sx * sizeof(E)) % 16 != 0) return false;
    if (((size_t)bx * sizeof(E)) % 16 != 0 || bx > 256 || by > 256 || bz > 256) return false;
    cuuint64_t dims[3] = {(cuuint64_t)g.sx, (cuuint64_t)(g.ny + 2), (cuuint64_t)(g.nz + 2)};
    cuuint64_t strides[2] = {(cuuint64_t)g.sx * sizeof(E), (cuuint64_t)g.sxy * sizeof(E)};
    cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(map, tma_dtype<E>(), dim == 3 ? 3 : 2, const_cast<void*>(base), dims,
                     strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

// ---------------------------------------------------------------------------
// device

// Start of a box along x: the lowest cell `lo` rounded down to the 16-byte
// boundary of elements of E (may be negative).
template <class E>
__host__ __device__ constexpr int tile_x0(int lo) {
    constexpr int a = 16 / (int)sizeof(E);
    return lo >= 0 ? lo / a * a : -((-lo + a - 1) / a) * a;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Waits for the barrier's phase `parity` to complete, at most `limit` polls; each
// poll suspends the thread in hardware for up to kTmaPollNs (it resumes as soon as
// the phase completes), so a waiting thread issues almost nothing.  Returns false
// on timeout.
constexpr uint32_t kTmaPollNs = 20000;
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit) {
    const uint32_t a = smem_u32(bar);
    for (long long it = 0; it < limit; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred P;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2, %3;\n\t"
            "selp.u32 %0, 1, 0, P;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity), "r"(kTmaPollNs)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// Orders this thread's earlier generic-proxy shared-memory accesses before later
// async-proxy (TMA) writes to the same buffer.
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

template <int DIM>
__device__ __forceinline__ void tma_load(void* dst, const CUtensorMap* map, int x, int y, int z,
                                         uint64_t* bar) {
    if (DIM == 3) {
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
            "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
            : "memory");
    } else {
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
            "[%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
            "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
            : "memory");
    }
}

// Polls before a TMA wait is declared stuck: at most 250000 x 20 us = 5 s.
constexpr long long kTmaWaitLimit = 250000;

}  // namespace uaamg
