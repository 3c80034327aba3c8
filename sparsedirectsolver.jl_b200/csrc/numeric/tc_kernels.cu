// FP32 Schur updates on the fifth-generation tensor cores (tcgen05, accumulator in tensor memory).
//
// The FP32 form's grouped GEMM C -= A B^T over the plan's tiles of the contribution-block updates
// (128 x 64; tiles of 64 rows run with the other 64 operand rows zero), as 3xTF32: each operand is
// split into a TF32 high part and a TF32 low part (x = hi + lo, both rounded to nearest by
// cvt.rna.tf32.f32), and
//     A B^T ~ A_lo B_hi^T + A_hi B_lo^T + A_hi B_hi^T,
// accumulated in FP32 in tensor memory. The dropped A_lo B_lo^T term is below FP32 rounding, so the
// result has FP32 accuracy at tensor-core rates.
//
// One CTA (4 warps) per tile:
// * thread 0 issues tcgen05.mma (M = 128, N = 64, K = 8 per instruction) into 64 TMEM columns;
// * all threads stage the operands, 32 columns of the inner dimension at a time, through registers
//   into shared memory in the K-major, no-swizzle canonical layout (16-byte core-matrix rows, 8-row
//   groups 128 bytes apart (SBO), K chunks of 4 elements ROWS * 16 bytes apart (LBO)), splitting
//   them into hi and lo on the way. Two buffers: the next stage's global loads are in flight while
//   the tensor cores run the current one. The operands are the reference's column-major panels and
//   contribution blocks (leading dimension f or m, any value), whose columns need not start on the
//   16-byte boundary that a TMA tensor map requires, and the split needs a register pass anyway;
// * tcgen05.commit signals one mbarrier per buffer when the MMAs that read it are done (every wait is
//   bounded: on time-out the CTA records a status and returns after releasing its tensor memory);
// * the four warps read the accumulator back with tcgen05.ld (32 lanes x 32 bit, 16 columns per
//   instruction) and apply the epilogue of the tile.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "kernels.cuh"

namespace sds {

namespace {

constexpr int TC_BK = 32;                       // K per stage: 4 MMAs of K = 8
constexpr int TC_MROWS = 128, TC_NROWS = 64;    // MMA shape M x N
constexpr int TC_CHUNKS = TC_BK / 4;            // 16-byte K chunks per row and stage
constexpr int TC_A_BYTES = TC_CHUNKS * TC_MROWS * 16;   // 16 KB per A part
constexpr int TC_B_LBO = TC_NROWS * 16;                // B chunks 1 KB apart
constexpr int TC_B_BYTES = TC_CHUNKS * TC_B_LBO;        // 8 KB per B part
constexpr int TC_STAGE = 2 * TC_A_BYTES + 2 * TC_B_BYTES;   // one buffer: A and B, hi and lo parts
constexpr int TC_NBUF = 2;                      // operand buffers (the pipeline depth)
constexpr int TC_TMEM_COLS = 64;
constexpr int TC_HEADER = 64;                   // mbarriers (2 x 8 B) + TMEM address (4 B), padded

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

// K-major, no-swizzle shared-memory matrix descriptor (start, LBO, SBO in 16-byte units)
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t)((addr >> 4) & 0x3FFF);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFF) << 32;
    d |= (uint64_t)1 << 46;                     // descriptor version of sm_100
    return d;                                   // base offset 0, legacy LBO mode, layout type 0 (no swizzle)
}

// instruction descriptor of kind::tf32: D F32, A and B TF32, both K-major, N = 64, M = 128
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_NROWS >> 3) << 17) |
                              ((uint32_t)(TC_MROWS >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(tmem), "l"(adesc), "l"(bdesc), "r"(TC_IDESC), "r"(acc));
}

}  // namespace

// The MMA main loop: D (TMEM, 128 x 64 FP32) = A B^T over K, as 3xTF32. A is M x K column-major
// (A[r + k lda], M <= 128); B is N x K column-major (B[c + k ldb]), N <= 64. Register-staged operand pipeline with two
// shared-memory buffers: stage s + 1's global loads are in flight while the tensor cores run stage s,
// and a buffer is refilled only after the MMAs that read it have committed (one mbarrier per buffer,
// phase = the buffer's use count). Returns false (the same in every thread) when a bounded wait gave
// up; `last` = the last stage whose MMAs were committed (-1: none).
__device__ __forceinline__ bool tc32_mainloop(uint8_t* tsm, uint64_t* mbar, uint32_t tmem, const float* Ab,
                                              int64_t lda, const float* Bb, int64_t ldb, int M, int N, int K,
                                              int& last) {
    const int tid = threadIdx.x;
    // staging registers: A row `tid`, the stage's 32 columns of the inner dimension; B row tid % 64, 16
    // of them (the half tid / 64). Each load instruction of a warp reads 32 consecutive rows.
    float ra[TC_BK], rb[TC_BK / 2];
    const int rB = tid & (TC_NROWS - 1), kB = (tid / TC_NROWS) * (TC_BK / 2);
    auto load = [&](int k0) {
#pragma unroll
        for (int j = 0; j < TC_BK; ++j) {
            const int k = k0 + j;
            ra[j] = (tid < M && k < K) ? Ab[tid + (int64_t)k * lda] : 0.0f;
        }
#pragma unroll
        for (int j = 0; j < TC_BK / 2; ++j) {
            const int k = k0 + kB + j;
            rb[j] = (rB < N && k < K) ? Bb[rB + (int64_t)k * ldb] : 0.0f;
        }
    };
    // split into TF32 hi and lo parts, in the K-major no-swizzle canonical layout (16-byte chunk c of
    // row r at c LBO + 16 r)
    auto put4 = [&](const float* v, uint8_t* hi, uint8_t* lo, int off) {
        uint4 h, l;
        uint32_t* hp = &h.x;
        uint32_t* lp = &l.x;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t hb = to_tf32(v[j]);
            hp[j] = hb;
            lp[j] = to_tf32(v[j] - __uint_as_float(hb));
        }
        *reinterpret_cast<uint4*>(hi + off) = h;
        *reinterpret_cast<uint4*>(lo + off) = l;
    };
    auto store = [&](int buf) {
        uint8_t* a_hi = tsm + buf * TC_STAGE;
        uint8_t* a_lo = a_hi + TC_A_BYTES;
        uint8_t* b_hi = a_lo + TC_A_BYTES;
        uint8_t* b_lo = b_hi + TC_B_BYTES;
#pragma unroll
        for (int c = 0; c < TC_CHUNKS; ++c) put4(ra + 4 * c, a_hi, a_lo, (c * TC_MROWS + tid) * 16);
#pragma unroll
        for (int c = 0; c < TC_CHUNKS / 2; ++c) put4(rb + 4 * c, b_hi, b_lo, (kB / 4 + c) * TC_B_LBO + rB * 16);
    };
    // bounded wait (about two seconds of polls) for the commit of a buffer's use `use`
    auto wait_buf = [&](int buf, int use) -> bool {
        uint32_t done = 0;
        for (long spins = 0; !done && spins < (1L << 24); ++spins)
            asm volatile(
                "{\n\t.reg .pred p;\n\t"
                "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                "selp.b32 %0, 1, 0, p;\n\t}\n"
                : "=r"(done)
                : "r"(smem_u32(mbar + buf)), "r"((uint32_t)(use & 1))
                : "memory");
        return done != 0;
    };

    bool ok = true;
    last = -1;
    const int nst = (K + TC_BK - 1) / TC_BK;
    if (nst > 0) load(0);
    for (int st = 0; st < nst; ++st) {
        const int buf = st & 1;
        bool mine = true;
        if (st >= TC_NBUF) mine = wait_buf(buf, (st - TC_NBUF) >> 1);   // the MMAs that read this buffer
        if (mine) store(buf);
        // the generic-proxy stores must be visible to the tensor cores (async proxy)
        asm volatile("fence.proxy.async.shared::cta;");
        ok = __syncthreads_and(mine) != 0;   // one verdict for the whole CTA
        if (!ok) break;
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t ah = smem_u32(tsm + buf * TC_STAGE), al = ah + TC_A_BYTES, bh = al + TC_A_BYTES,
                           bl = bh + TC_B_BYTES;
#pragma unroll
            for (int s = 0; s < TC_BK / 8; ++s) {
                const uint32_t ao = 2 * s * TC_MROWS * 16, bo = 2 * s * TC_B_LBO;
                const uint64_t dah = smem_desc(ah + ao, TC_MROWS * 16, 128);
                const uint64_t dal = smem_desc(al + ao, TC_MROWS * 16, 128);
                const uint64_t dbh = smem_desc(bh + bo, TC_B_LBO, 128);
                const uint64_t dbl = smem_desc(bl + bo, TC_B_LBO, 128);
                mma_tf32(tmem, dal, dbh, (st > 0 || s > 0) ? 1u : 0u);
                mma_tf32(tmem, dah, dbl, 1u);
                mma_tf32(tmem, dah, dbh, 1u);
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(mbar + buf))
                         : "memory");
        }
        last = st;
        if (st + 1 < nst) load((st + 1) * TC_BK);   // in flight while the tensor cores run this stage
    }
    // the last commit covers every MMA issued before it
    if (ok && last >= 0) ok = __syncthreads_and(wait_buf(last & 1, last >> 1)) != 0;
    if (!ok && tid == 0 && last >= 0) {
        // MMAs may still be running: they read this CTA's shared memory and write the tensor memory that
        // the caller frees. Give the last commit a second bounded wait.
        wait_buf(last & 1, last >> 1);
    }
    return ok;
}

// TMEM allocation (64 columns) and the two mbarriers; every thread gets the TMEM address
__device__ __forceinline__ uint32_t tc32_setup(uint64_t* mbar, uint32_t* tmem_slot) {
    if ((threadIdx.x >> 5) == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TC_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar + 1)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    return *tmem_slot;
}

__device__ __forceinline__ void tc32_teardown(uint32_t tmem) {
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
}

// 16 accumulator columns [cb, cb + 16) of this warp's 32 TMEM lanes (row warp * 32 + lane)
__device__ __forceinline__ void tc32_ld16(uint32_t tmem, int cb, float* out) {
    uint32_t v[16];
    const uint32_t taddr = tmem + ((uint32_t)((threadIdx.x >> 5) * 32) << 16) + (uint32_t)cb;
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
    for (int j = 0; j < 16; ++j) out[j] = __uint_as_float(v[j]);
}

// The contribution-block updates: C -= A B^T over the tile's lower part (r + diag >= c).
__global__ void __launch_bounds__(128) gemm_nt_tc32_kernel(GemmArgs<float> A) {
    extern __shared__ __align__(1024) uint8_t tsm[];
    uint64_t* mbar = reinterpret_cast<uint64_t*>(tsm + TC_NBUF * TC_STAGE);   // one per buffer
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tsm + TC_NBUF * TC_STAGE + 16);

    const GemmTile t = A.tiles[blockIdx.x];
    const int member = A.members ? A.members[blockIdx.y] : blockIdx.y;
    if (A.finfo && t.front >= 0 && A.finfo[(int64_t)member * A.ns + t.front] != 0) return;
    if (t.mode == 2) {   // deferred diagonal-block write
        const float* src = A.copy_src + (int64_t)member * A.copy_stride + t.a;
        float* dst = A.cbuf + (int64_t)member * A.cstride + t.c;
        for (int q = threadIdx.x; q < t.m * t.n; q += blockDim.x) dst[q % t.m + (int64_t)(q / t.m) * t.ldc] = src[q % t.m + (int64_t)(q / t.m) * t.lda];
        return;
    }
    const float* Ab = A.abuf + (int64_t)member * A.astride + t.a;
    const float* Bb = A.bbuf + (int64_t)member * A.bstride + t.b;
    float* Cb = A.cbuf + (int64_t)member * A.cstride + t.c;
    const int M = t.m, N = t.n;
    const uint32_t tmem = tc32_setup(mbar, tmem_slot);
    int last;
    const bool ok = tc32_mainloop(tsm, mbar, tmem, Ab, t.lda, Bb, t.ldb, M, N, t.k, last);
    if (!ok && threadIdx.x == 0 && A.status) atomicExch(A.status, 2);   // the factorization fails
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (ok && last >= 0) {   // (K = 0: nothing to apply)
        const int r = threadIdx.x;
#pragma unroll
        for (int cb = 0; cb < TC_NROWS; cb += 16) {
            float v[16];
            tc32_ld16(tmem, cb, v);
            float cur[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int c = cb + j;
                cur[j] = (!t.mode && r < M && c < N && r + t.diag >= c) ? Cb[r + (int64_t)c * t.ldc] : 0.0f;
            }
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int c = cb + j;
                if (r < M && c < N && r + t.diag >= c) Cb[r + (int64_t)c * t.ldc] = t.mode ? v[j] : cur[j] - v[j];
            }
        }
    }
    tc32_teardown(tmem);
}

size_t gemm_tc32_smem() { return (size_t)TC_NBUF * TC_STAGE + TC_HEADER; }

cudaError_t launch_gemm_tc32(const GemmArgs<float>& a, int nmembers, cudaStream_t st) {
    if (a.count == 0) return cudaSuccess;
    dim3 grid(a.count, nmembers);
    gemm_nt_tc32_kernel<<<grid, 128, gemm_tc32_smem(), st>>>(a);
    return cudaGetLastError();
}

cudaError_t prepare_tc_kernels() {
    return cudaFuncSetAttribute(gemm_nt_tc32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)gemm_tc32_smem());
}

}  // namespace sds
