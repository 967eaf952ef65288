// umma.cuh — the 5th-generation tensor-core primitives (sm_100a) used by the
// batched kernel's moment x current contraction, as inline PTX:
//   * tensor-memory allocation (tcgen05.alloc / dealloc / relinquish),
//   * shared-memory matrix descriptors for K-major operands without swizzle,
//   * the instruction descriptor of kind::tf32 with FP32 accumulation,
//   * tcgen05.mma issue, tcgen05.commit to an mbarrier, bounded mbarrier waits,
//   * tcgen05.ld of 32 accumulator columns per thread.
//
// Operand layout (K-major, no swizzle). A matrix of R rows (M or N) and K
// 32-bit elements is stored as "core matrices" of 8 rows x 16 bytes (8 x 4
// elements), each 128 contiguous bytes with rows 16 bytes apart. The K chunks
// (4 elements) of one 8-row group follow each other (leading-dimension byte
// offset LBO = 128), and 8-row groups are K/4 x 128 bytes apart (stride byte
// offset SBO). Element (r, k) therefore sits at byte
//     (r / 8) * (K / 4) * 128 + (k / 4) * 128 + (r % 8) * 16 + (k % 4) * 4.
// One MMA consumes K = 8 (32 bytes, two chunks); the descriptor of K step t
// starts 2 t chunks (256 bytes) further.
#pragma once
#include <cstdint>

namespace bielcc_gpu {
namespace umma {

// Byte offset of element (r, k) in the layout above, K elements per row.
__host__ __device__ __forceinline__ uint32_t kmajor_offset(int r, int k, int K) {
    return (uint32_t)((r >> 3) * (K >> 2) * 128 + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

// Shared-memory descriptor (sm_100 format): start address >> 4 in bits 0-13,
// LBO >> 4 in 16-29, SBO >> 4 in 32-45, version 1 in bits 46-47, base offset
// 0, layout type 0 (no swizzle) in bits 61-63.
__device__ __forceinline__ uint64_t smem_desc(uint32_t smem_addr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::tf32: D F32 (bits 4-5 = 1), A and B TF32
// (bits 7-9 and 10-12 = 2), both K-major (bits 15, 16 = 0), N >> 3 in bits
// 17-22, M >> 4 in bits 24-28.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// ---- tensor memory (one warp executes these, all 32 lanes)
__device__ __forceinline__ void tmem_alloc(uint32_t* smem_dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(smem_dst)),
                 "r"(ncols));
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// ---- ordering between the generic proxy, thread syncs and the tensor core
// Shared-memory operands written with ordinary stores become visible to the
// tensor core (async proxy) after this fence.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ---- MMA: D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         bool accumulate) {
    const uint32_t acc = accumulate ? 1u : 0u;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(acc)
        : "memory");
}

// Arrives on the mbarrier once every MMA this thread issued before has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// ---- mbarrier
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Waits for the phase with the given parity to complete, for at most
// `limit_ns` nanoseconds of the global timer (each try_wait itself suspends
// for a bounded, implementation-defined time). Returns false when the limit
// ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
    const uint64_t t0 = global_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}

// ---- accumulator read-back: 32 consecutive 32-bit columns of this thread's
// lane (warp w reads lanes 32 (w % 4) .. + 31; taddr carries the lane base in
// bits 16-31 and the column in bits 0-15)
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// TF32 split of an FP32 value: hi = x rounded to TF32 (10 explicit mantissa
// bits, low 13 bits zero), lo = x - hi (exact in FP32) rounded to TF32. The
// three products hi*hi + hi*lo + lo*hi recover an FP32-accurate product.
__device__ __forceinline__ void tf32_split(float x, float& hi, float& lo) {
    uint32_t h, l;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
    hi = __uint_as_float(h);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(x - hi));
    lo = __uint_as_float(l);
}

}  // namespace umma
}  // namespace bielcc_gpu
