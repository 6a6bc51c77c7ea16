// Tile loads by the tensor memory accelerator (TMA) for the column transforms of the whole window.
//
// A column kernel transforms CW = 8 adjacent k_x columns of one plane along y: a tile of ny rows of 8 complex
// values, 128 bytes a row at a stride of H complex values. One thread issues the tile of each array as one
// cp.async.bulk.tensor.2d load into shared memory (no cluster multicast: every tensor map covers this GPU's own
// buffers), the CTA's mbarrier counts the bytes, and the other threads wait at a barrier instead of each issuing
// ny / 16 scattered loads. The tensor map views an array of complex128 as float64 [rows][2 H]: the box is 16
// doubles (x, a multiple of 16 bytes at every column tile, since x = 2 c0 doubles = 16 c0 bytes) by ny rows; columns
// beyond H are filled with zeros by the unit. The wait for the bytes is bounded: past its limit the waiting thread
// sets the kernel's error word and the CTA returns without touching the tile, and the host reports G3D_ERR_TIMEOUT.
#pragma once
#include <cuda.h>            // CUtensorMap and its enums (types only: the encoder is taken from the runtime)
#include <cudaTypedefs.h>    // PFN_cuTensorMapEncodeTiled
#include <mutex>
#include "g3d_common.cuh"

namespace g3d {

struct TileMaps {                                  // up to six tensor maps of one kernel (kernel parameter)
    CUtensorMap m[6];
};
// The bound of a kernel's tile waits: the error word, the polls of the barrier before giving up (2^24 unless
// G3D_TMA_POLLS sets it), and bytes the barrier expects beyond the tiles (0; G3D_TMA_EXTRA_BYTES > 0 makes every wait
// run out, for the test of the timeout path: the tiles land, the barrier's phase never completes).
struct TmaWait {
    int* err;
    long polls;
    unsigned extra;
};

// ---------------------------------------------------------------- host
inline PFN_cuTensorMapEncodeTiled_v12000 tma_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}
// The map of a complex128 array [rows][H] (row stride H) for tiles of 8 columns x box_rows rows; false if the
// encoder is unavailable or refuses (the caller then uses its plain loads).
inline bool tma_map_columns(CUtensorMap* m, const cpx* base, long H, long rows, int box_rows) {
    const PFN_cuTensorMapEncodeTiled_v12000 fn = tma_encoder();
    if (!fn || !base || box_rows < 1 || box_rows > 256 || (reinterpret_cast<uintptr_t>(base) & 15)) return false;
    cuuint64_t dims[2] = {cuuint64_t(2 * H), cuuint64_t(rows)};
    cuuint64_t strides[1] = {cuuint64_t(H) * sizeof(cpx)};
    cuuint32_t box[2] = {16, cuuint32_t(box_rows)};
    cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<cpx*>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// ---------------------------------------------------------------- device
__device__ __forceinline__ unsigned smem_addr(const void* p) { return static_cast<unsigned>(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// the box at (x, y) of a 2-D map into dst (128-byte aligned), its bytes counted on bar
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
            smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}
// Thread 0 loads the 8-column tiles of n maps at (2 c0, y) into dst[k] and waits for them (bounded); every thread
// returns true when the tiles have landed, after observing the barrier's completed phase itself (so the bytes the
// unit wrote are visible to it). On a timeout the error word gets bit 1 and every thread returns false.
template <int NY>
__device__ __forceinline__ bool tma_tiles(const TileMaps& maps, const int* idx, int n, cpx* const* dst, int c0, int y,
                                          uint64_t* bar, int* ok, const TmaWait& w) {
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_expect_tx(bar, unsigned(n) * NY * 8 * sizeof(cpx) + w.extra);
        for (int k = 0; k < n; ++k) tma_load_2d(dst[k], &maps.m[idx[k]], bar, 2 * c0, y);
        bool done = false;
        for (long it = 0; it < w.polls && !done; ++it) done = mbar_try_wait(bar, 0);
        *ok = done ? 1 : 0;
        if (!done) atomicOr(w.err, 1);
    }
    __syncthreads();
    if (*ok == 0) return false;
    for (int it = 0; it < 4096 && !mbar_try_wait(bar, 0); ++it) {
    }
    return true;
}
// A column of a dense row-major tile of 8 columns: position p of column c
struct TileCol {
    int c;
    __device__ __forceinline__ int operator()(int p) const { return p * 8 + c; }
};

}  // namespace g3d
