// FP32 Schur updates on the fifth-generation tensor cores (tcgen05, accumulator in tensor memory).
//
// The FP32 form's grouped GEMM C -= A B^T (or C = A B^T in place, the trsm by an inverse) over the
// plan's 64 x 64 tiles, as 3xTF32: each operand is split into a TF32 high part and a TF32 low part
// (x = hi + lo, both rounded to nearest by cvt.rna.tf32.f32), and
//     A B^T ~ A_lo B_hi^T + A_hi B_lo^T + A_hi B_hi^T,
// accumulated in FP32 in tensor memory. The dropped A_lo B_lo^T term is below FP32 rounding, so the
// result has FP32 accuracy at tensor-core rates.
//
// One CTA (4 warps) per tile:
// * thread 0 issues tcgen05.mma (M = 128, N = 64, K = 8 per instruction; rows 64..127 of the A
//   operand are zero, so the tile's 64 rows land in TMEM lanes 0..63);
// * the operands are staged by all threads into shared memory in the K-major, no-swizzle
//   canonical layout: 16-byte core-matrix rows, 8-row groups 128 bytes apart (SBO), K chunks of 4
//   elements ROWS * 16 bytes apart (LBO);
// * tcgen05.commit signals an mbarrier when the MMAs of a stage are done (the wait is bounded: on
//   time-out the CTA records a status and returns after releasing its tensor memory);
// * warps 0 and 1 read the accumulator back with tcgen05.ld (32 lanes x 32 bit, 16 columns per
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
constexpr int TC_B_BYTES = TC_CHUNKS * TC_NROWS * 16;   // 8 KB per B part
constexpr int TC_TMEM_COLS = 64;
constexpr int TC_HEADER = 64;                   // mbarrier (8 B) + TMEM address (4 B), padded

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

// stage one operand tile: rows r < rows_valid of X (column-major, ld ldx), columns k0 .. k0 + TC_BK
// of the inner dimension (< K), split into TF32 hi and lo parts in the canonical layout
template <int ROWS>
__device__ __forceinline__ void stage(const float* X, int64_t ldx, int rows_valid, int k0, int K, uint8_t* hi,
                                      uint8_t* lo) {
    for (int q = threadIdx.x; q < 64 * TC_CHUNKS; q += blockDim.x) {
        const int r = q % 64, c = q / 64;
        float v[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int k = k0 + 4 * c + j;
            v[j] = (r < rows_valid && k < K) ? X[r + (int64_t)k * ldx] : 0.0f;
        }
        uint4 h, l;
        uint32_t* hp = &h.x;
        uint32_t* lp = &l.x;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const uint32_t hb = to_tf32(v[j]);
            hp[j] = hb;
            lp[j] = to_tf32(v[j] - __uint_as_float(hb));
        }
        const int off = (c * ROWS + r) * 16;
        *reinterpret_cast<uint4*>(hi + off) = h;
        *reinterpret_cast<uint4*>(lo + off) = l;
    }
}

}  // namespace

__global__ void __launch_bounds__(128) gemm_nt_tc32_kernel(GemmArgs<float> A) {
    extern __shared__ __align__(1024) uint8_t tsm[];
    uint8_t* a_hi = tsm;
    uint8_t* a_lo = a_hi + TC_A_BYTES;
    uint8_t* b_hi = a_lo + TC_A_BYTES;
    uint8_t* b_lo = b_hi + TC_B_BYTES;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(b_lo + TC_B_BYTES);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(b_lo + TC_B_BYTES + 8);

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
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int M = t.m, N = t.n, K = t.k;

    // rows 64..127 of the A operand stay zero
    for (int q = tid; q < TC_CHUNKS * 64; q += blockDim.x) {
        const int r = 64 + q % 64, c = q / 64;
        *reinterpret_cast<uint4*>(a_hi + (c * TC_MROWS + r) * 16) = make_uint4(0, 0, 0, 0);
        *reinterpret_cast<uint4*>(a_lo + (c * TC_MROWS + r) * 16) = make_uint4(0, 0, 0, 0);
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TC_TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tmem_slot;

    bool ok = true;
    uint32_t phase = 0;
    const int nst = (K + TC_BK - 1) / TC_BK;
    for (int st = 0; st < nst && ok; ++st) {
        const int k0 = st * TC_BK;
        stage<TC_MROWS>(Ab, t.lda, M, k0, K, a_hi, a_lo);
        stage<TC_NROWS>(Bb, t.ldb, N, k0, K, b_hi, b_lo);
        // the generic-proxy stores must be visible to the tensor cores (async proxy)
        asm volatile("fence.proxy.async.shared::cta;");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo), bh = smem_u32(b_hi), bl = smem_u32(b_lo);
            for (int s = 0; s < TC_BK / 8; ++s) {
                const uint32_t ao = 2 * s * TC_MROWS * 16, bo = 2 * s * TC_NROWS * 16;
                const uint64_t dah = smem_desc(ah + ao, TC_MROWS * 16, 128);
                const uint64_t dal = smem_desc(al + ao, TC_MROWS * 16, 128);
                const uint64_t dbh = smem_desc(bh + bo, TC_NROWS * 16, 128);
                const uint64_t dbl = smem_desc(bl + bo, TC_NROWS * 16, 128);
                mma_tf32(tmem, dal, dbh, (st > 0 || s > 0) ? 1u : 0u);
                mma_tf32(tmem, dah, dbl, 1u);
                mma_tf32(tmem, dah, dbh, 1u);
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_u32(mbar))
                         : "memory");
        }
        // wait for the stage's MMAs (bounded: about two seconds)
        {
            uint32_t done = 0;
            long spins = 0;
            while (!done) {
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                    "selp.b32 %0, 1, 0, p;\n\t}\n"
                    : "=r"(done)
                    : "r"(smem_u32(mbar)), "r"(phase)
                    : "memory");
                if (!done && ++spins > (1L << 24)) break;
            }
            // one verdict for the whole CTA: tcgen05.ld below is warp-collective
            ok = __syncthreads_and(done != 0) != 0;
            if (!ok && tid == 0) {
                if (A.status) atomicExch(A.status, 2);
                // The stage's MMAs may still be running: they read this CTA's shared memory and write the
                // tensor memory that the exit path frees. Give their commit a second bounded wait before
                // the dealloc below. The status word already fails the factorization, so the C tile that
                // this CTA leaves unwritten is never used.
                uint32_t drained = 0;
                for (long s = 0; !drained && s < (1L << 24); ++s)
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                        "selp.b32 %0, 1, 0, p;\n\t}\n"
                        : "=r"(drained)
                        : "r"(smem_u32(mbar)), "r"(phase)
                        : "memory");
            }
        }
        phase ^= 1u;
    }
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (ok && warp < 2) {
        const int r = warp * 32 + lane;
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
        for (int cb = 0; cb < TC_NROWS; cb += 16) {
            uint32_t v[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
                "%14, %15}, [%16];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                : "r"(taddr + (uint32_t)cb));
            asm volatile("tcgen05.wait::ld.sync.aligned;");
            float cur[16];
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int c = cb + j;
                cur[j] = (!t.mode && r < M && c < N && r + t.diag >= c) ? Cb[r + (int64_t)c * t.ldc] : 0.0f;
            }
#pragma unroll
            for (int j = 0; j < 16; ++j) {
                const int c = cb + j;
                if (r < M && c < N && r + t.diag >= c) {
                    const float acc = __uint_as_float(v[j]);
                    Cb[r + (int64_t)c * t.ldc] = t.mode ? acc : cur[j] - acc;
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TC_TMEM_COLS));
}

size_t gemm_tc32_smem() { return 2 * (size_t)TC_A_BYTES + 2 * (size_t)TC_B_BYTES + TC_HEADER; }

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
