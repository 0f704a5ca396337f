// umma.cuh -- a small tcgen05 (5th-generation tensor core) GEMM engine for the learned
// range-kernel surrogate: C[M x N] (fp32) = sum_k A[m][k] * B[n][k], bf16 operands, fp32
// accumulation in tensor memory (TMEM).
//
// One CTA computes a 128 x BN tile.  Per K-tile of kKT = 64, all 128 threads gather the A and
// B tiles into shared memory through caller-supplied loader functors (implicit GEMM: the
// im2col of a convolution happens in the loader) in the K-major, no-swizzle canonical layout
// (8 rows x 16 bytes "core matrices"); one elected thread issues four tcgen05.mma (M=128,
// N=BN, K=16) and a tcgen05.commit onto an mbarrier; every thread waits for it (bounded) before
// the tile is overwritten.  The epilogue reads the accumulator with tcgen05.ld (warp w owns
// rows 32w..32w+31, one row per thread) and hands (row, col, value) to a store functor.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace prc {
namespace umma {

constexpr int kM = 128;         // rows per CTA tile (TMEM lanes)
constexpr int kKT = 64;         // K per shared-memory tile (4 MMAs of K = 16)
constexpr int kThreads = 128;   // 4 warps
constexpr int kWaitRounds = 1 << 22;

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: K-major, no swizzle.  lbo = byte distance between the two
// 8-element K chunks of one MMA, sbo = byte distance between consecutive 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(const void* base, unsigned lbo, unsigned sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr(base) >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version for this architecture
    return d;                // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// Instruction descriptor of kind::f16: bf16 A and B (K-major), fp32 D, M = 128, N = n.
__host__ __device__ constexpr uint32_t instr_desc(int n) {
    return (1u << 4)                   // D format: f32
           | (1u << 7)                 // A format: bf16
           | (1u << 10)                // B format: bf16
           | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(kM >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    for (int i = 0; i < kWaitRounds; ++i) {
        unsigned done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Core-matrix layout of an R x kKT bf16 tile: chunk c (8 K-elements), row group g, row r:
// byte offset ((c * (R / 8) + g) * 8 + r) * 16.  Hence sbo = 128 and lbo = (R / 8) * 128.
__device__ __forceinline__ int tile_offset(int R, int row, int k) {
    return (((k >> 3) * (R >> 3) + (row >> 3)) * 8 + (row & 7)) * 16 + (k & 7) * 2;
}

// No vector loader for the A operand (the element loader fills the tile).
struct NoVecA {
    __device__ uint4 operator()(int, int) const { return make_uint4(0u, 0u, 0u, 0u); }
};

// C tile (128 x BN) at (m0, n0), summed over k in [k_lo, k_hi) (a split-K slice when the
// caller splits; K bounds the problem).  LoadA(m, k) and LoadB(n, k) return the operand values
// (bf16) for m < M, n < N, k < K; Store(m, n, v) receives the result for m < M, n < N.
// With vec_a, LoadA8(m, k) returns the 8 A values k .. k + 7 (k a multiple of 8) as one 16-byte
// vector -- exactly one row of a core matrix -- and the A tile is filled with 16-byte copies;
// K and the slice bounds must then be multiples of 8.
// Returns false (and stores nothing) if an MMA completion wait timed out.
// ROWS_A / ROWS_B: the element loader walks rows fastest (consecutive threads read consecutive
// m or n at one k), for operands stored contiguously along M or N rather than along K.
template <int BN, bool ROWS_A = false, bool ROWS_B = false, class LoadA, class LoadA8, class LoadB, class Store>
__device__ bool gemm_tile(int M, int N, int K, int m0, int n0, int k_lo, int k_hi, LoadA&& load_a, bool vec_a,
                          LoadA8&& load_a8, LoadB&& load_b, Store&& store, unsigned char* smem, uint64_t* bar,
                          uint32_t* tmem_slot) {
    static_assert(BN >= 32 && BN <= 256 && (BN & (BN - 1)) == 0, "BN: power of two in [32, 256]");
    __nv_bfloat16* sa = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* sb = reinterpret_cast<__nv_bfloat16*>(smem + kM * kKT * 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) mbar_init(bar);
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;
    const uint32_t idesc = instr_desc(BN);
    bool ok = true;
    if (k_hi > K) k_hi = K;
    const int k_tiles = k_hi > k_lo ? (k_hi - k_lo + kKT - 1) / kKT : 0;
    for (int kt = 0; kt < k_tiles && ok; ++kt) {
        const int k0 = k_lo + kt * kKT;
        if (vec_a) {
            // rows fastest: consecutive threads store consecutive 16-byte rows of a core matrix
            for (int i = tid; i < kM * (kKT / 8); i += kThreads) {
                const int r = i % kM, c = i / kM, k = k0 + c * 8;
                const uint4 v = (m0 + r < M && k < k_hi) ? load_a8(m0 + r, k) : make_uint4(0u, 0u, 0u, 0u);
                *reinterpret_cast<uint4*>(reinterpret_cast<unsigned char*>(sa) + tile_offset(kM, r, c * 8)) = v;
            }
        } else {
            for (int i = tid; i < kM * kKT; i += kThreads) {
                const int r = ROWS_A ? i % kM : i / kKT, k = ROWS_A ? i / kM : i % kKT;
                const __nv_bfloat16 v = (m0 + r < M && k0 + k < k_hi) ? load_a(m0 + r, k0 + k) : __float2bfloat16(0.0f);
                *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<unsigned char*>(sa) + tile_offset(kM, r, k)) = v;
            }
        }
        for (int i = tid; i < BN * kKT; i += kThreads) {
            const int r = ROWS_B ? i % BN : i / kKT, k = ROWS_B ? i / BN : i % kKT;
            const __nv_bfloat16 v = (n0 + r < N && k0 + k < k_hi) ? load_b(n0 + r, k0 + k) : __float2bfloat16(0.0f);
            *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<unsigned char*>(sb) + tile_offset(BN, r, k)) = v;
        }
        // generic-proxy shared-memory writes become visible to the tensor core (async proxy)
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int kk = 0; kk < kKT / 16; ++kk) {
                // K-step kk covers chunks 2kk and 2kk+1
                const uint64_t da = smem_desc(reinterpret_cast<unsigned char*>(sa) + 2 * kk * (kM / 8) * 128,
                                              (kM / 8) * 128, 128);
                const uint64_t db = smem_desc(reinterpret_cast<unsigned char*>(sb) + 2 * kk * (BN / 8) * 128,
                                              (BN / 8) * 128, 128);
                const unsigned accumulate = (kt > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(bar))
                         : "memory");
        }
        // the tile may be overwritten only after the MMAs that read it completed
        ok = mbar_wait(bar, kt & 1);
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        __syncthreads();
    }
    if (ok && k_tiles > 0) {
        const int row = warp * 32 + lane;
        const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
        for (int c0 = 0; c0 < BN; c0 += 8) {
            uint32_t v[8];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                : "r"(lane_base + c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m0 + row < M)
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    if (n0 + c0 + j < N) store(m0 + row, n0 + c0 + j, __uint_as_float(v[j]));
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
    return ok;
}

// The element-loader form.
template <int BN, class LoadA, class LoadB, class Store>
__device__ bool gemm_tile(int M, int N, int K, int m0, int n0, int k_lo, int k_hi, LoadA&& load_a, LoadB&& load_b,
                          Store&& store, unsigned char* smem, uint64_t* bar, uint32_t* tmem_slot) {
    return gemm_tile<BN, false, false>(M, N, K, m0, n0, k_lo, k_hi, load_a, false, NoVecA{}, load_b, store, smem, bar,
                                       tmem_slot);
}

// Dynamic shared memory of a gemm_tile CTA.  Padded so that at most 512 / BN CTAs fit on an SM
// (232 448 bytes of shared memory per SM): together they never ask for more than the 512 TMEM
// columns an SM has, so no tcgen05.alloc has to wait for another CTA to finish.
template <int BN>
constexpr size_t smem_bytes() {
    const size_t need = (size_t)(kM + BN) * kKT * 2;
    const size_t cap = 232448 / (512 / BN + 1) + 128;
    return need > cap ? need : cap;
}

}  // namespace umma
}  // namespace prc
