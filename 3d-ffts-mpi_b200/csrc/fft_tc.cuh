// Split-precision tensor-core form of the axis pass: every radix-16 stage is
// a dense GEMM on the 5th-generation tensor cores (tcgen05.mma, kind::f16,
// FP32 accumulators in tensor memory), the other stage (radix 2/4/8) and the
// twiddles stay on the CUDA cores in FP32.
//
// One radix-16 butterfly is y = F16 x with F16 the 16-point DFT matrix.  As a
// real GEMM row: [y_re | y_im] = [x_re | x_im] R with the 32 x 32 matrix
//   R = [[C, S], [-S, C]],  C = cos(2 pi r k / 16),  S = -+ sin(2 pi r k / 16).
// Both operands are split into 16-bit parts (fp16 rows first scaled by a power
// of two into [-1, 1), which bf16's 8-bit exponent does not need); R is split
// on the host from FP64 values.
//   fp16 (11-bit significands): x = xh + xl, R = Rh + Rl, and the product
//     keeps xh Rh + xh Rl + xl Rh (xl Rl is below FP32 rounding): 22 bits.
//   bf16 (8-bit significands): two parts carry only 16 bits, which leaves a
//     relative error near 7e-6 on a 512^3 transform, so bf16 uses three parts
//     x = xh + xm + xl, R = Rh + Rm + Rl and keeps every product down to
//     2^-16 of the main term -- xh Rh, xh Rm + xm Rh, xh Rl + xm Rm + xl Rh
//     (the dropped xm Rl, xl Rm, xl Rl are at or below FP32 rounding): 24 bits.
// The A operand of a 128-row block (16 columns per part: the row's 16 real
// then 16 imaginary values, two 16-bit values per 32-bit column) lives in
// tensor memory: each thread writes its row into its own lane with
// tcgen05.st, so A never passes through shared memory; B = [Rh | (Rm) | Rl]
// is in shared memory (K-major, no swizzle).  The K = 16 MMAs (2 per kept
// term: real and imaginary halves of K) accumulate into one block of 32 FP32
// columns, smallest terms first; each warp reads its 32 rows back with
// tcgen05.ld.  A row is one butterfly: the thread that built row m reads row
// m back, undoes its scale and stores the 16 outputs.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "fft_tile.cuh"
#include "fft_tmat.cuh"

namespace a2a {

enum TcFormat : int { TC_FP16 = 0, TC_BF16 = 1 };

// 16-bit parts each operand is split into.
__host__ __device__ constexpr int tc_parts(int fmt) { return fmt == TC_BF16 ? 3 : 2; }

// Shared-memory layout of the B operand (UMMA canonical K-major,
// SWIZZLE_NONE): an 8-row x 16-byte core matrix is 128 contiguous bytes; core
// matrices step by SBO = 128 bytes along N and by LBO bytes along K.
constexpr int kTcRows = 128;                     // M of one MMA block
constexpr int kTcChunkB = 32 / 8 * 128;          // bytes of one K chunk of B (N = 32): 512
constexpr int kTcMatB = 4 * kTcChunkB;           // one 32 x 32 matrix: 2 KB
__host__ __device__ constexpr int tc_b_bytes(int fmt) { return tc_parts(fmt) * kTcMatB; }
constexpr int kTcBBytesMax = 3 * kTcMatB;        // room for the largest split

__host__ __device__ constexpr uint64_t umma_smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);  // version 1, no swizzle
}
// kind::f16 instruction descriptor: FP32 accumulator, A/B format, both
// K-major, N = 32, M = 128.
__host__ __device__ constexpr uint32_t umma_idesc_f16(int fmt) {
    return (1u << 4) | ((uint32_t)fmt << 7) | ((uint32_t)fmt << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);
}

// (a, b) = w[0] + w[1] (+ w[2]) in 16-bit parts, a in the low and b in the
// high half of each 32-bit word (the A operand's layout: two consecutive K
// values per tensor-memory column); each part is the rounding of what the
// previous parts leave, converted two at a time.
template <int FMT> __device__ __forceinline__ void split_pair(float a, float b, uint32_t (&w)[tc_parts(FMT)]) {
#pragma unroll
    for (int i = 0; i < tc_parts(FMT); ++i) {
        if constexpr (FMT == TC_FP16) {
            const __half2 h = __floats2half2_rn(a, b);
            w[i] = *reinterpret_cast<const uint32_t*>(&h);
            const float2 f = __half22float2(h);
            a -= f.x;
            b -= f.y;
        } else {
            const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
            w[i] = *reinterpret_cast<const uint32_t*>(&h);
            const float2 f = __bfloat1622float2(h);
            a -= f.x;
            b -= f.y;
        }
    }
}

struct TcCtx {
    uint32_t b_addr;           // shared address of [Rh | (Rm) | Rl]
    uint32_t tmem;             // tensor-memory base (lane 0, column 0)
    unsigned long long* bar;   // MMA completion
    uint32_t phase;
    bool drained;              // after an abandoned stage: its MMAs did finish
};

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

__device__ __forceinline__ void tc_commit(unsigned long long* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// A operand rows written into tensor memory: 32 columns of this warp's 32
// lanes from 32 registers each.
__device__ __forceinline__ void tc_st32(uint32_t taddr, const uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};\n" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]), "r"(r[16]), "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]), "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
        : "memory");
}
__device__ __forceinline__ void tc_st16(uint32_t taddr, const uint32_t* r) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};\n" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}
__device__ __forceinline__ void tc_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }
// D = A B (+ D) with A in tensor memory (K-major, 16-bit values two to a
// 32-bit column) and B in shared memory; no output lanes disabled.
__device__ __forceinline__ void tc_mma_ts(uint32_t dtmem, uint32_t atmem, uint64_t bdesc, uint32_t idesc,
                                          uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, {%5, %6, %7, %8}, p;\n}\n" ::"r"(dtmem),
        "r"(atmem), "l"(bdesc), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

// Tensor-memory columns of one 128-row block: the A operand (16 columns per
// part: real values in 0-7, imaginary in 8-15), then the 32-column
// accumulator.  fp16: 64 columns; bf16: 80.
__host__ __device__ constexpr int tc_acc_col(int fmt) { return 16 * tc_parts(fmt); }
__host__ __device__ constexpr int tc_block_cols(int fmt) { return tc_acc_col(fmt) + 32; }

// Row swizzle of a batch-mode tile (the pass kernels' rule): the first
// stage's stride-R0 row writes of 8-line rows would otherwise meet 2-4-way
// bank conflicts.
template <class PLAN, int B, int MODE> __host__ __device__ constexpr int tc_tile_swizzle() {
    return MODE == MODE_BATCH ? tile_swizzle_shift<PLAN, B, (int)sizeof(float2)>() : -1;
}

// One radix-16 stage on the tensor cores.  THREADS == butterflies per stage;
// thread q owns butterfly q, i.e. A row q % 128 of block q / 128.  Returns
// false when the MMA completion wait gave up (the device error flag is then
// set, the rest of the pass is skipped, and ctx.drained says whether the
// stage's MMAs were seen to finish by a second bounded wait, i.e. whether the
// tensor memory may be freed).
template <class PLAN, int B, int THREADS, int MODE, bool INV, int FMT, int s, bool SRC_GLOBAL>
__device__ __forceinline__ bool tc_stage(const PassArgs<float>& a, float2* tile, const float2* tw,
                                         const uint32_t* offA_s, const size_t* base_s, TcCtx& ctx, int tid,
                                         size_t ubase, int v0) {
    using G = TileGeom<MODE, B, PLAN::N, sizeof(float2), tc_tile_swizzle<PLAN, B, MODE>()>;
    constexpr int N = PLAN::N;
    constexpr int R = PLAN::r[s];
    static_assert(R == 16, "tensor-core stages are radix 16");
    constexpr int NS = PLAN::ns(s);
    constexpr int NBL = N / R;
    static_assert(B * NBL == THREADS, "one butterfly per thread in a tensor-core stage");
    constexpr int NBLK = THREADS / kTcRows;
    static_assert(THREADS % kTcRows == 0, "whole 128-row MMA blocks");
    constexpr bool LAST = (s == PLAN::S - 1);
    constexpr bool BFAST = (MODE == MODE_BATCH) || !(LAST || SRC_GLOBAL);
    constexpr int TWO = PLAN::twoff(s);
    constexpr int NP = tc_parts(FMT);
    constexpr int BCOLS = tc_block_cols(FMT);
    constexpr int ACC = tc_acc_col(FMT);

    int b, j;
    bf_map<BFAST, B, NBL>(tid, b, j);
    float2 x[16];
    if constexpr (SRC_GLOBAL) {
        const float2* line = a.src + ubase + __ldg(a.offV + v0 + b);
#pragma unroll
        for (int r = 0; r < 16; ++r) x[r] = ld_stream(line + __ldg(a.offA + j + r * NBL));
    } else {
#pragma unroll
        for (int r = 0; r < 16; ++r) x[r] = tile[G::idx(b, j + r * NBL)];
    }
    const int m = j % NS;
    if constexpr (s > 0) {
#pragma unroll
        for (int r = 1; r < 16; ++r) x[r] = cmulw<INV>(x[r], tw[TWO + (r - 1) * NS + m]);
    }
    // fp16 (5-bit exponent): scale the row into [-1, 1) by a power of two,
    // e = exponent of the largest component (as frexp would give it), scale
    // factors built from exponent bits.  bf16 has FP32's exponent range and
    // needs no scaling.
    float down = 1.f, up = 1.f;
    if constexpr (FMT == TC_FP16) {
        float mx = 0.f;
#pragma unroll
        for (int r = 0; r < 16; ++r) mx = fmaxf(mx, fmaxf(fabsf(x[r].x), fabsf(x[r].y)));
        int e = ((__float_as_int(mx) >> 23) & 0xFF) - 126;
        e = mx > 0.f ? min(max(e, -125), 126) : 0;
        down = __int_as_float((127 - e) << 23);  // 2^-e
        up = __int_as_float((127 + e) << 23);    // 2^e
    }
    const int warp = tid / 32;
    const uint32_t lane_row = ((uint32_t)((warp % 4) * 32) << 16) + (uint32_t)((warp / 4) * BCOLS);
    {
        // the row into this warp's lanes of its block's A columns: part q at
        // columns 16q..16q+15 (real values k, k+1 in the low and high half of
        // column 16q + k/2, imaginary ones in 16q + 8 + k/2)
        uint32_t w[16 * NP];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            uint32_t pr[NP], pi[NP];
            split_pair<FMT>(x[2 * i].x * down, x[2 * i + 1].x * down, pr);
            split_pair<FMT>(x[2 * i].y * down, x[2 * i + 1].y * down, pi);
#pragma unroll
            for (int q = 0; q < NP; ++q) {
                w[16 * q + i] = pr[q];
                w[16 * q + 8 + i] = pi[q];
            }
        }
        if constexpr (NP == 2) {
            tc_st32(ctx.tmem + lane_row, reinterpret_cast<const uint32_t(&)[32]>(w));
        } else {
            tc_st32(ctx.tmem + lane_row, reinterpret_cast<const uint32_t(&)[32]>(w));
            tc_st16(ctx.tmem + lane_row + 32, w + 32);
        }
        tc_wait_st();
        tc_fence_before();
        __syncthreads();  // all A rows stored; all tile reads of this stage done
    }
    if (tid == 0) {
        tc_fence_after();
        const uint32_t idesc = umma_idesc_f16(FMT);
        // B parts: R part q at b_addr + q kTcMatB; the real half of K first
        auto bre = [&](int q) { return umma_smem_desc(ctx.b_addr + q * kTcMatB, kTcChunkB, 128); };
        auto bim = [&](int q) { return umma_smem_desc(ctx.b_addr + q * kTcMatB + 2 * kTcChunkB, kTcChunkB, 128); };
#pragma unroll
        for (int blk = 0; blk < NBLK; ++blk) {
            const uint32_t ab = ctx.tmem + blk * BCOLS;  // lane 0 of the block's A columns
            const uint32_t dacc = ab + ACC;
            // one term x_p R_q: the real and the imaginary half of K
            auto term = [&](int pa, int qb, uint32_t acc) {
                tc_mma_ts(dacc, ab + 16 * pa, bre(qb), idesc, acc);
                tc_mma_ts(dacc, ab + 16 * pa + 8, bim(qb), idesc, 1);
            };
            if constexpr (NP == 2) {
                // corrections xh Rl + xl Rh (2^-11 smaller), then xh Rh
                term(0, 1, 0);
                term(1, 0, 1);
                term(0, 0, 1);
            } else {
                // 2^-16 terms, 2^-8 terms, then xh Rh
                term(0, 2, 0);
                term(1, 1, 1);
                term(2, 0, 1);
                term(0, 1, 1);
                term(1, 0, 1);
                term(0, 0, 1);
            }
        }
        tc_commit(ctx.bar);
    }
    const bool ok = mbar_wait_bounded(ctx.bar, ctx.phase);
    if (__syncthreads_or(!ok)) {
        // the MMAs did not complete in time: flag it, skip the rest of the
        // pass, and look once more (bounded) for their completion before the
        // caller may free the tensor memory they write
        if ((tid % 32) == 0) atomicExch(a.err, 1);
        ctx.drained = __syncthreads_and(mbar_wait_bounded(ctx.bar, ctx.phase)) != 0;
        return false;
    }
    ctx.phase ^= 1u;
    tc_fence_after();
    float y[32];
    tc_ld32(ctx.tmem + lane_row + ACC, y);
#pragma unroll
    for (int k = 0; k < 16; ++k) x[k] = make_float2(y[k] * up, y[16 + k] * up);
    if constexpr (LAST) {
        float2* line = a.dst + base_s[b];
#pragma unroll
        for (int r = 0; r < 16; ++r) st_stream(line + offA_s[j + r * NBL], scl(x[r], a.scale));
    } else {
        const int jd = (j / NS) * NS * R + m;
#pragma unroll
        for (int r = 0; r < 16; ++r) tile[G::idx(b, jd + r * NS)] = x[r];
    }
    tc_fence_before();
    __syncthreads();  // tile written; accumulators read before the next stage's MMAs
    if constexpr (!LAST)
        return tc_stage<PLAN, B, THREADS, MODE, INV, FMT, s + 1, false>(a, tile, tw, offA_s, base_s, ctx, tid, ubase,
                                                                        v0);
    return true;
}

template <class PLAN, int B, int MODE, int FMT>
__host__ __device__ constexpr size_t tc_smem_bytes() {
    constexpr int N = PLAN::N;
    size_t bytes = sizeof(float2) * (size_t)TileGeom<MODE, B, N, sizeof(float2)>::elems;
    bytes = (bytes + 127) & ~size_t(127);
    bytes += tc_b_bytes(FMT);
    bytes += sizeof(float2) * (size_t)PLAN::twtotal();
    bytes += sizeof(uint32_t) * (size_t)N;
    bytes = (bytes + 15) & ~size_t(15);
    bytes += sizeof(size_t) * (size_t)B + 16;  // line bases, mbarrier, tensor-memory address
    return bytes;
}

// One CTA = one tile of B lines, THREADS = B N / 16.  Tensor memory:
// tc_block_cols(FMT) columns per 128-row block (the total rounded up to a
// power of two), allocated and freed by warp 0.
// Tensor-memory columns one CTA allocates (a power of two >= 32), and the
// CTAs per SM that many columns allow (at most 4).
template <class PLAN, int B, int FMT> __host__ __device__ constexpr int tc_tcols() {
    constexpr int NEED = (B * PLAN::N / 16 / kTcRows) * tc_block_cols(FMT);
    return NEED <= 32 ? 32 : NEED <= 64 ? 64 : NEED <= 128 ? 128 : NEED <= 256 ? 256 : 512;
}
template <class PLAN, int B, int FMT> __host__ __device__ constexpr int tc_min_blocks() {
    return 512 / tc_tcols<PLAN, B, FMT>() < 4 ? 512 / tc_tcols<PLAN, B, FMT>() : 4;
}

template <class PLAN, int B, int MODE, bool INV, int FMT>
__global__ void __launch_bounds__(B * PLAN::N / 16, (tc_min_blocks<PLAN, B, FMT>())) fft_tc_kernel(const PassArgs<float> a) {
    constexpr int N = PLAN::N;
    constexpr int THREADS = B * N / 16;
    constexpr int NBLK = THREADS / kTcRows;
    static_assert(NBLK * tc_block_cols(FMT) <= 512, "tensor memory holds 512 columns");
    constexpr uint32_t TCOLS = tc_tcols<PLAN, B, FMT>();
    using G = TileGeom<MODE, B, N, sizeof(float2), tc_tile_swizzle<PLAN, B, MODE>()>;
    constexpr int TWN = PLAN::twtotal();
    constexpr int R0 = PLAN::r[0];

    extern __shared__ __align__(128) unsigned char smem_raw[];
    float2* tile = reinterpret_cast<float2*>(smem_raw);
    size_t off = (sizeof(float2) * (size_t)G::elems + 127) & ~size_t(127);
    unsigned char* bmat = smem_raw + off;
    off += tc_b_bytes(FMT);
    float2* tw = reinterpret_cast<float2*>(smem_raw + off);
    off += sizeof(float2) * (size_t)TWN;
    uint32_t* offA_s = reinterpret_cast<uint32_t*>(smem_raw + off);
    off = (off + sizeof(uint32_t) * N + 15) & ~size_t(15);
    size_t* base_s = reinterpret_cast<size_t*>(smem_raw + off);
    off += sizeof(size_t) * B;
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smem_raw + off);
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem_raw + off + 8);

    const int tid = threadIdx.x;
    const int tilesV = a.NV / B;
    const int u = blockIdx.x / tilesV;
    const int v0 = (blockIdx.x - u * tilesV) * B;
    const size_t ubase = a.offU[u];

    if (tid < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                     "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    {
        const uint4* src = reinterpret_cast<const uint4*>(a.tcb);
        uint4* dst = reinterpret_cast<uint4*>(bmat);
        for (int i = tid; i < tc_b_bytes(FMT) / 16; i += THREADS) dst[i] = src[i];
    }
    for (int i = tid; i < TWN; i += THREADS) tw[i] = a.tw[i];
    for (int i = tid; i < N; i += THREADS) offA_s[i] = a.offA[i];
    for (int i = tid; i < B; i += THREADS) base_s[i] = ubase + a.offV[v0 + i];
    fence_proxy_async_smem();  // B operand visible to the tensor cores
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    TcCtx ctx;
    ctx.b_addr = smem_u32(bmat);
    ctx.tmem = *tmem_slot;
    ctx.bar = bar;
    ctx.phase = 0;
    ctx.drained = true;

    bool ok;
    if constexpr (R0 == 16) {
        ok = tc_stage<PLAN, B, THREADS, MODE, INV, FMT, 0, true>(a, tile, tw, offA_s, base_s, ctx, tid, ubase, v0);
    } else {
        // stage 0 on the CUDA cores: global -> registers -> shared
        constexpr int NBL = N / R0;
        constexpr int NBT = B * NBL;
        constexpr int K = (NBT + THREADS - 1) / THREADS;
        constexpr bool EXACT = (NBT % THREADS) == 0;
        constexpr bool BFAST0 = (MODE == MODE_BATCH);
        float2 x[K][R0];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int q = tid + k * THREADS;
            if (EXACT || q < NBT) {
                int b, j;
                bf_map<BFAST0, B, NBL>(q, b, j);
                const float2* line = a.src + ubase + __ldg(a.offV + v0 + b);
#pragma unroll
                for (int r = 0; r < R0; ++r) x[k][r] = ld_stream(line + __ldg(a.offA + j + r * NBL));
            }
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int q = tid + k * THREADS;
            if (EXACT || q < NBT) {
                int b, j;
                bf_map<BFAST0, B, NBL>(q, b, j);
                Dft<R0, INV, float2>::run(x[k]);
#pragma unroll
                for (int r = 0; r < R0; ++r) tile[G::idx(b, j * R0 + r)] = x[k][r];
            }
        }
        __syncthreads();
        ok = tc_stage<PLAN, B, THREADS, MODE, INV, FMT, 1, false>(a, tile, tw, offA_s, base_s, ctx, tid, ubase, v0);
    }
    // every stage ends with tcgen05.wait::ld and a block barrier.  After an
    // abandoned stage whose MMAs were never seen to finish, the columns stay
    // allocated (freeing them under running MMAs would hand them to another
    // CTA while they are written); the error flag is already set.
    if (!ok && !ctx.drained) return;
    tc_fence_after();
    if (tid < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(ctx.tmem), "r"(TCOLS)
                     : "memory");
}

// Persistent form fed by the TMA ring: each CTA allocates its tensor memory,
// loads the split operand, twiddles and offsets once, then works through
// tiles blockIdx.x, blockIdx.x + gridDim.x, ...  Every tile arrives as whole
// tensor-map copies (the single-GPU ring of fft_tmat.cuh, no multicast) in a
// 2-slot shared-memory ring; each slot is also its tile's Stockham tile
// (transformed in place), and is refilled with the tile two ahead as soon as
// its tile's last stage has read it, so one tile's copy is in flight while
// the other is transformed.  Plans whose first stage is not radix 16 (the
// CUDA-core stage 0 reads the slot into registers before rewriting it).
template <class PLAN, int B, int MODE, int FMT> __host__ __device__ constexpr uint32_t tc_ring_slot_bytes() {
    return tmat_slot_bytes_for<float, PLAN, B, MODE, 1, true>();
}
template <class PLAN, int B, int MODE, int FMT> __host__ __device__ constexpr size_t tc_ring_smem_bytes() {
    size_t bytes = kTmatAlign;  // room to align the ring
    bytes += 2 * (size_t)tc_ring_slot_bytes<PLAN, B, MODE, FMT>();
    bytes += tc_b_bytes(FMT);
    bytes += sizeof(float2) * (size_t)PLAN::twtotal();
    bytes += sizeof(uint32_t) * (size_t)PLAN::N;
    bytes = (bytes + 15) & ~size_t(15);
    bytes += sizeof(size_t) * (size_t)B;
    bytes += sizeof(unsigned long long) * 3 + 16;  // two ring barriers, the MMA barrier, tensor-memory address
    return bytes;
}

template <class PLAN, int B, int MODE, bool INV, int FMT>
__global__ void __launch_bounds__(B * PLAN::N / 16, (tc_min_blocks<PLAN, B, FMT>()))
    fft_tc_ring_kernel(const PassArgs<float> a, const __grid_constant__ TmatMaps m) {
    constexpr int N = PLAN::N;
    constexpr int THREADS = B * N / 16;
    constexpr uint32_t TCOLS = tc_tcols<PLAN, B, FMT>();
    using G = TileGeom<MODE, B, N, sizeof(float2), tc_tile_swizzle<PLAN, B, MODE>()>;
    constexpr int TWN = PLAN::twtotal();
    constexpr int R0 = PLAN::r[0];
    static_assert(R0 != 16, "the ring form starts with a CUDA-core stage");
    constexpr int NBL = N / R0;
    constexpr int NBT = B * NBL;
    constexpr int K = (NBT + THREADS - 1) / THREADS;
    constexpr bool EXACT = (NBT % THREADS) == 0;
    constexpr bool BFAST0 = (MODE == MODE_BATCH);
    constexpr int NSTG = 2;
    constexpr uint32_t SLOT = tc_ring_slot_bytes<PLAN, B, MODE, FMT>();

    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t s0 = smem_u32(smem_raw);
    unsigned char* ring = smem_raw + (((s0 + kTmatAlign - 1) & ~(kTmatAlign - 1)) - s0);
    unsigned char* bmat = ring + NSTG * SLOT;
    float2* tw = reinterpret_cast<float2*>(bmat + tc_b_bytes(FMT));
    uint32_t* offA_s = reinterpret_cast<uint32_t*>(tw + TWN);
    size_t* base_s = reinterpret_cast<size_t*>(
        reinterpret_cast<unsigned char*>(tw) + ((sizeof(float2) * TWN + sizeof(uint32_t) * N + 15) & ~size_t(15)));
    unsigned long long* rbar = reinterpret_cast<unsigned long long*>(base_s + B);  // ring slots
    unsigned long long* mbar = rbar + NSTG;                                        // MMA completion
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 1);

    const int tid = threadIdx.x;
    const int tilesV = a.NV / B;
    const int ntiles = a.NU * tilesV;
    const int mine = (int)blockIdx.x < ntiles ? (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;

    if (tid < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                     "r"(TCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 0) {
        for (int i = 0; i < NSTG; ++i) mbar_init(rbar + i, 1);
        mbar_init(mbar, 1);
        fence_mbar_init();
    }
    {
        const uint4* src = reinterpret_cast<const uint4*>(a.tcb);
        uint4* dst = reinterpret_cast<uint4*>(bmat);
        for (int i = tid; i < tc_b_bytes(FMT) / 16; i += THREADS) dst[i] = src[i];
    }
    for (int i = tid; i < TWN; i += THREADS) tw[i] = a.tw[i];
    for (int i = tid; i < N; i += THREADS) offA_s[i] = a.offA[i];
    fence_proxy_async_smem();  // B operand visible to the tensor cores
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    TcCtx ctx;
    ctx.b_addr = smem_u32(bmat);
    ctx.tmem = *tmem_slot;
    ctx.bar = mbar;
    ctx.phase = 0;
    ctx.drained = true;

    int issued = 0;  // thread 0: tiles of this CTA whose copies were issued
    if (tid == 0)
        for (; issued < NSTG && issued < mine; ++issued)
            tmat_issue<float, B, N>(m, blockIdx.x + issued * gridDim.x, tilesV, ring + issued * SLOT, rbar + issued);

    bool ok = true;
    int i = 0;
    for (; i < mine; ++i) {
        const int t = blockIdx.x + i * gridDim.x;
        const int s = i % NSTG;
        const int u = t / tilesV;
        const int v0 = (t - u * tilesV) * B;
        const size_t ubase = __ldg(a.offU + u);
        for (int b = tid; b < B; b += THREADS) base_s[b] = ubase + __ldg(a.offV + v0 + b);
        if (__syncthreads_or(!mbar_wait_bounded(rbar + s, (uint32_t)((i / NSTG) & 1)))) {
            if (tid == 0) atomicExch(a.err, 1);
            ok = false;
            break;
        }
        // stage 0 on the CUDA cores: the slot into registers, then the
        // Stockham tile written over it
        const float2* src = reinterpret_cast<const float2*>(ring + s * SLOT);
        float2* tile = reinterpret_cast<float2*>(ring + s * SLOT);
        float2 x[K][R0];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int q = tid + k * THREADS;
            if (EXACT || q < NBT) {
                int b, j;
                bf_map<BFAST0, B, NBL>(q, b, j);
#pragma unroll
                for (int r = 0; r < R0; ++r) {
                    const int n = j + r * NBL;
                    if constexpr (MODE == MODE_BATCH) {
                        x[k][r] = src[n * B + b];
                    } else {  // [z chunk][b][z within the chunk]
                        int q2, zl;
                        if (m.chunk_shift >= 0) {
                            q2 = n >> m.chunk_shift;
                            zl = n & (m.chunk - 1);
                        } else {
                            q2 = n / m.chunk;
                            zl = n - q2 * m.chunk;
                        }
                        x[k][r] = src[(q2 * B + b) * m.chunk + zl];
                    }
                }
            }
        }
        __syncthreads();  // every read of the slot before it is rewritten
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int q = tid + k * THREADS;
            if (EXACT || q < NBT) {
                int b, j;
                bf_map<BFAST0, B, NBL>(q, b, j);
                Dft<R0, INV, float2>::run(x[k]);
#pragma unroll
                for (int r = 0; r < R0; ++r) tile[G::idx(b, j * R0 + r)] = x[k][r];
            }
        }
        __syncthreads();
        if (!tc_stage<PLAN, B, THREADS, MODE, INV, FMT, 1, false>(a, tile, tw, offA_s, base_s, ctx, tid, ubase, v0)) {
            ok = false;
            ++i;  // tile i's copy has landed
            break;
        }
        // the last stage read the slot (tc_stage ends with a block barrier):
        // refill it with the tile NSTG ahead
        if (tid == 0 && issued < mine) {
            fence_proxy_async_smem();  // the generic accesses of the slot come before the async writes
            tmat_issue<float, B, N>(m, blockIdx.x + issued * gridDim.x, tilesV, ring + s * SLOT, rbar + s);
            ++issued;
        }
    }
    if (!ok && tid == 0)  // wait (bounded) for this CTA's copies still in flight before leaving
        for (int j = i; j < issued; ++j) mbar_wait_bounded(rbar + j % NSTG, (uint32_t)((j / NSTG) & 1));
    __syncthreads();
    // after an abandoned stage whose MMAs were never seen to finish, the
    // columns stay allocated (see fft_tc_kernel)
    if (!ctx.drained) return;
    tc_fence_after();
    if (tid < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(ctx.tmem), "r"(TCOLS)
                     : "memory");
}

}  // namespace a2a
