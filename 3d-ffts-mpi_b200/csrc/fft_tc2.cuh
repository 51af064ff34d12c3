// Two-stage split-precision tensor-core pass for N = 512 = 16 x 32.
//
// With n = 32 a + b and k = k1 + 16 k2 (a, k1 < 16; b, k2 < 32):
//   X[k1 + 16 k2] = sum_b W32^(b k2) W512^(b k1) sum_a x[32 a + b] W16^(a k1)
// Stage 0: for each b, the radix-16 DFT over a of the stride-32 subsequence
// (no twiddles): one 32 x 32 real GEMM row per (line, b), as the radix-16
// stage of fft_tc.cuh.  Its outputs go to tile position 16 b + k1.
// Stage 1: for each k1, the inputs tile[k1 + 16 b] times W512^(b k1), then
// the radix-32 DFT over b: one 64 x 64 real GEMM row per (line, k1), with
// K = [re b<16 | im b<16 | re b>=16 | im b>=16] and the outputs in the same
// order over k2.  A 128-row stage-1 block has two threads per row (warps w
// and w + 4 reach the same tensor-memory lanes): thread half h writes the
// inputs b in [16h, 16h + 16) (its 16 columns of each part) and reads the
// outputs k2 in [16h, 16h + 16).
//
// So a pass has two GEMM stages, one twiddle multiply and one shared-memory
// exchange per element (the three-stage 2 x 16 x 16 form has two of each
// plus a CUDA-core radix-2 stage).  Operands are split as in fft_tc.cuh
// (fp16: two parts, rows scaled by a power of two; bf16: three parts); a
// stage-1 row's scale is agreed between its two threads through shared
// memory.  Tiles of 8 lines arrive by the single-GPU TMA ring of fft_tmat.cuh
// (2 slots, transformed in place, no multicast); the slot of a tile is
// refilled as soon as its stage-1 operands are in tensor memory.
#pragma once

#include "fft_tc.cuh"

namespace a2a {

constexpr int kTc2N = 512;
constexpr int kTc2Lines = 8;
constexpr int kTc2Threads = 256;
// the radix-32 operand: K-major N x K, N = K = 64 (16-bit values): a K chunk
// of 8 values over all 64 rows is 1 KB, one part 8 KB
constexpr int kTc2ChunkB1 = 64 / 8 * 128;
constexpr int kTc2MatB1 = 8 * kTc2ChunkB1;
// both operands of one direction: the radix-16 parts, then the radix-32 parts
__host__ __device__ constexpr int tc2_b_bytes(int fmt) { return tc_parts(fmt) * (kTcMatB + kTc2MatB1); }
// tensor-memory columns: stage 0 two blocks of (16 per part + 32), stage 1
// one block of (32 per part + 64) -- the same count, reused
__host__ __device__ constexpr int tc2_cols(int fmt) { return 32 * tc_parts(fmt) + 64; }
__host__ __device__ constexpr uint32_t tc2_tcols(int fmt) { return tc2_cols(fmt) <= 128 ? 128u : 256u; }
// twiddles W512^(b k1) (forward sign), [b][k1]
constexpr int kTc2Tw = 32 * 16;

__host__ __device__ constexpr uint32_t umma_idesc_f16_n(int fmt, int n) {
    return (1u << 4) | ((uint32_t)fmt << 7) | ((uint32_t)fmt << 10) | (((uint32_t)n >> 3) << 17) | ((128u >> 4) << 24);
}

__host__ __device__ constexpr size_t tc2_smem_bytes(int fmt) {
    size_t bytes = kTmatAlign;                                        // room to align the ring
    bytes += 2 * (size_t)tmat_slot_bytes<float, kTc2Lines, kTc2N>();  // two slots
    bytes += (size_t)tc2_b_bytes(fmt);
    bytes += sizeof(float2) * (size_t)kTc2Tw;
    bytes += sizeof(uint32_t) * (size_t)kTc2N;
    bytes += sizeof(size_t) * (size_t)kTc2Lines;
    bytes += sizeof(float) * (size_t)kTc2Threads;                     // stage-1 row maxima (fp16)
    bytes += sizeof(unsigned long long) * 3 + 16;                     // ring barriers, MMA barrier, tmem address, wait flag
    return bytes;
}

// Tile positions (in place in the ring slot) of the stage-0 outputs: batch
// mode rows of 8 lines, row n stored at n ^ ((n >> 4) & 1) (the two rows a
// half-warp writes, 16 apart, land in different bank halves); line mode
// [b][n] with n's low four bits XOR-ed with bits 4-7 (a half-warp writes
// positions 16 apart).  Stage 1's reads stay conflict-free under both.
template <int MODE> __device__ __forceinline__ int tc2_pos(int b, int n) {
    if constexpr (MODE == MODE_BATCH) return (n ^ ((n >> 4) & 1)) * kTc2Lines + b;
    else return b * kTc2N + (n ^ ((n >> 4) & 15));
}

// fp16 row scale: 2^-e and 2^e with e the exponent of mx (as frexp gives it).
__device__ __forceinline__ void tc2_scale(float mx, float& down, float& up) {
    int e = ((__float_as_int(mx) >> 23) & 0xFF) - 126;
    e = mx > 0.f ? min(max(e, -125), 126) : 0;
    down = __int_as_float((127 - e) << 23);
    up = __int_as_float((127 + e) << 23);
}

// Split 16 complex values (times `down`) into NP parts, laid out as one
// radix-16 A row of fft_tc.cuh: part q in w[16q .. 16q+15], real pairs then
// imaginary pairs.
template <int FMT> __device__ __forceinline__ void tc2_split16(const float2 (&x)[16], float down,
                                                              uint32_t (&w)[16 * tc_parts(FMT)]) {
    constexpr int NP = tc_parts(FMT);
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
}

// Thread 0: the MMAs of one stage, then the commit.  Stage 0: two 128-row
// blocks (columns 0 and BC0), K = 32, N = 32, operand b0; stage 1: one block,
// K = 64 (four K = 16 steps per term), N = 64, operand b1.  Terms smallest
// first, as in fft_tc.cuh.
template <int FMT, int STAGE>
__device__ __forceinline__ void tc2_issue(uint32_t tmem, uint32_t b_addr, unsigned long long* bar) {
    constexpr int NP = tc_parts(FMT);
    tc_fence_after();
    if constexpr (STAGE == 0) {
        constexpr int BC0 = 16 * NP + 32;
        const uint32_t idesc = umma_idesc_f16_n(FMT, 32);
        auto bre = [&](int q) { return umma_smem_desc(b_addr + q * kTcMatB, kTcChunkB, 128); };
        auto bim = [&](int q) { return umma_smem_desc(b_addr + q * kTcMatB + 2 * kTcChunkB, kTcChunkB, 128); };
#pragma unroll
        for (int blk = 0; blk < 2; ++blk) {
            const uint32_t ab = tmem + blk * BC0;
            const uint32_t dacc = ab + 16 * NP;
            auto term = [&](int pa, int qb, uint32_t acc) {
                tc_mma_ts(dacc, ab + 16 * pa, bre(qb), idesc, acc);
                tc_mma_ts(dacc, ab + 16 * pa + 8, bim(qb), idesc, 1);
            };
            if constexpr (NP == 2) {
                term(0, 1, 0);
                term(1, 0, 1);
                term(0, 0, 1);
            } else {
                term(0, 2, 0);
                term(1, 1, 1);
                term(2, 0, 1);
                term(0, 1, 1);
                term(1, 0, 1);
                term(0, 0, 1);
            }
        }
    } else {
        const uint32_t idesc = umma_idesc_f16_n(FMT, 64);
        const uint32_t b1 = b_addr + NP * kTcMatB;
        const uint32_t dacc = tmem + 32 * NP;
        auto term = [&](int pa, int qb, uint32_t acc) {
#pragma unroll
            for (int c = 0; c < 4; ++c)
                tc_mma_ts(dacc, tmem + 32 * pa + 8 * c,
                          umma_smem_desc(b1 + qb * kTc2MatB1 + c * 2 * kTc2ChunkB1, kTc2ChunkB1, 128), idesc,
                          c == 0 ? acc : 1u);
        };
        if constexpr (NP == 2) {
            term(0, 1, 0);
            term(1, 0, 1);
            term(0, 0, 1);
        } else {
            term(0, 2, 0);
            term(1, 1, 1);
            term(2, 0, 1);
            term(0, 1, 1);
            term(1, 0, 1);
            term(0, 0, 1);
        }
    }
    tc_commit(bar);
}

// The persistent kernel: each CTA allocates its tensor memory and loads both
// split operands, the twiddles and the offsets once, then works through tiles
// blockIdx.x, blockIdx.x + gridDim.x, ... of 8 lines, each arriving as whole
// tensor-map copies in a 2-slot ring.  Every wait is bounded; on expiry the
// device error flag is raised, the rest of the pass is skipped, the CTA waits
// (bounded) for its copies in flight and frees its tensor memory only if the
// MMAs it committed were seen to finish.
template <int MODE, bool INV, int FMT>
__global__ void __launch_bounds__(kTc2Threads, 2)
    fft_tc2_ring_kernel(const PassArgs<float> a, const __grid_constant__ TmatMaps m) {
    constexpr int N = kTc2N;
    constexpr int B = kTc2Lines;
    constexpr int THREADS = kTc2Threads;
    constexpr int NP = tc_parts(FMT);
    constexpr int BC0 = 16 * NP + 32;  // stage-0 block columns (A parts, then the accumulator)
    constexpr int ACC0 = 16 * NP;
    constexpr int ACC1 = 32 * NP;      // stage-1 accumulator (64 columns)
    constexpr uint32_t TCOLS = tc2_tcols(FMT);
    constexpr uint32_t SLOT = tmat_slot_bytes<float, B, N>();
    constexpr int NSTG = 2;
    static_assert(B * N * sizeof(float2) <= SLOT, "a tile fits its slot");
    static_assert(2 * BC0 <= (int)TCOLS && ACC1 + 64 <= (int)TCOLS, "tensor-memory columns");

    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t s0 = smem_u32(smem_raw);
    unsigned char* ring = smem_raw + (((s0 + kTmatAlign - 1) & ~(kTmatAlign - 1)) - s0);
    unsigned char* bmat = ring + NSTG * SLOT;
    float2* tw = reinterpret_cast<float2*>(bmat + tc2_b_bytes(FMT));
    uint32_t* offA_s = reinterpret_cast<uint32_t*>(tw + kTc2Tw);
    size_t* base_s = reinterpret_cast<size_t*>(offA_s + N);
    float* pmax = reinterpret_cast<float*>(base_s + B);
    unsigned long long* rbar = reinterpret_cast<unsigned long long*>(pmax + THREADS);
    unsigned long long* mbar = rbar + NSTG;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 1);
    int* wflag = reinterpret_cast<int*>(tmem_slot + 1);

    const int tid = threadIdx.x;
    const int warp = tid / 32;
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
        for (int i = tid; i < tc2_b_bytes(FMT) / 16; i += THREADS) dst[i] = src[i];
    }
    for (int i = tid; i < kTc2Tw; i += THREADS) tw[i] = a.tw[i];
    for (int i = tid; i < N; i += THREADS) offA_s[i] = a.offA[i];
    fence_proxy_async_smem();  // operands visible to the tensor cores
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t b_addr = smem_u32(bmat);
    uint32_t phase = 0;
    bool drained = true;

    // stage 0: one radix-16 row per thread (block warp / 4, lane tid % 128)
    int b0, j0;
    if constexpr (MODE == MODE_BATCH) { b0 = tid % B; j0 = tid / B; }
    else { j0 = tid % 32; b0 = tid / 32; }
    const uint32_t row0 = ((uint32_t)((warp % 4) * 32) << 16) + (uint32_t)((warp / 4) * BC0);
    // stage 1: row tid % 128 of the one block, half h = tid / 128
    const int h = tid / 128;
    const int rr = tid % 128;
    int b1, j1;
    if constexpr (MODE == MODE_BATCH) { b1 = rr % B; j1 = rr / B; }
    else { j1 = rr % 16; b1 = rr / 16; }
    const uint32_t row1 = (uint32_t)((warp % 4) * 32) << 16;

    int issued = 0;  // thread 0: tiles of this CTA whose copies were issued
    if (tid == 0)
        for (; issued < NSTG && issued < mine; ++issued)
            tmat_issue<float, B, N>(m, blockIdx.x + issued * gridDim.x, tilesV, ring + issued * SLOT, rbar + issued);

    bool ok = true;
    int i = 0;
    // the MMA completion: thread 0 waits (bounded) and tells the CTA through
    // shared memory (0: done; 1: done after the first wait gave up; 2: never
    // seen done -- the tensor memory must then stay allocated); a failed wait
    // raises the error flag and ends the pass
    auto mma_wait = [&]() -> bool {
        if (tid == 0) *wflag = mbar_wait_bounded(mbar, phase) ? 0 : mbar_wait_bounded(mbar, phase) ? 1 : 2;
        __syncthreads();
        const int f = *wflag;
        if (f) {
            if (tid == 0) atomicExch(a.err, 1);
            drained = f == 1;
            return false;
        }
        phase ^= 1u;
        tc_fence_after();
        return true;
    };
    // line bases of this CTA's next tile (threads 0..B-1), loaded one tile ahead
    auto line_base = [&](int t) -> size_t {
        const int u = t / tilesV;
        const int v0 = (t - u * tilesV) * B;
        return (size_t)__ldg(a.offU + u) + __ldg(a.offV + v0 + tid);
    };
    size_t nbase = 0;
    if (tid < B && mine > 0) nbase = line_base(blockIdx.x);
    for (; i < mine; ++i) {
        const int t = blockIdx.x + i * gridDim.x;
        const int s = i % NSTG;
        if (tid < B) {
            base_s[tid] = nbase;
            if (i + 1 < mine) nbase = line_base(t + gridDim.x);
        }
        if (__syncthreads_or(!mbar_wait_bounded(rbar + s, (uint32_t)((i / NSTG) & 1)))) {
            if (tid == 0) atomicExch(a.err, 1);
            ok = false;
            break;
        }
        float2* slot = reinterpret_cast<float2*>(ring + s * SLOT);

        // ---- stage 0: radix-16 DFTs of x[j0 + 32 r] ----
        float2 x[16];
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const int n = j0 + 32 * r;
            if constexpr (MODE == MODE_BATCH) {
                x[r] = slot[n * B + b0];
            } else {  // [z chunk][b][z within the chunk]
                int q2, zl;
                if (m.chunk_shift >= 0) {
                    q2 = n >> m.chunk_shift;
                    zl = n & (m.chunk - 1);
                } else {
                    q2 = n / m.chunk;
                    zl = n - q2 * m.chunk;
                }
                x[r] = slot[(q2 * B + b0) * m.chunk + zl];
            }
        }
        float down = 1.f, up = 1.f;
        if constexpr (FMT == TC_FP16) {
            float mx = 0.f;
#pragma unroll
            for (int r = 0; r < 16; ++r) mx = fmaxf(mx, fmaxf(fabsf(x[r].x), fabsf(x[r].y)));
            tc2_scale(mx, down, up);
        }
        {
            uint32_t w[16 * NP];
            tc2_split16<FMT>(x, down, w);
            tc_st32(tmem + row0, reinterpret_cast<const uint32_t(&)[32]>(w));
            if constexpr (NP == 3) tc_st16(tmem + row0 + 32, w + 32);
            tc_wait_st();
        }
        tc_fence_before();
        __syncthreads();  // all A rows stored; every read of the slot done
        if (tid == 0) tc2_issue<FMT, 0>(tmem, b_addr, mbar);
        if (!mma_wait()) {
            ok = false;
            ++i;  // tile i's copy has landed
            break;
        }
        {
            float y[32];
            tc_ld32(tmem + row0 + ACC0, y);
#pragma unroll
            for (int k = 0; k < 16; ++k) slot[tc2_pos<MODE>(b0, 16 * j0 + k)] = make_float2(y[k] * up, y[16 + k] * up);
        }
        tc_fence_before();
        __syncthreads();  // stage-0 outputs in the tile; accumulators read

        // ---- stage 1: twiddles, then radix-32 DFTs over b of tile[j1 + 16 b] ----
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const int bb = 16 * h + q;
            x[q] = cmulw<INV>(slot[tc2_pos<MODE>(b1, j1 + 16 * bb)], tw[bb * 16 + j1]);  // W^0 = 1 exactly
        }
        if constexpr (FMT == TC_FP16) {
            float mx = 0.f;
#pragma unroll
            for (int q = 0; q < 16; ++q) mx = fmaxf(mx, fmaxf(fabsf(x[q].x), fabsf(x[q].y)));
            pmax[tid] = mx;
            __syncthreads();
            tc2_scale(fmaxf(mx, pmax[tid ^ 128]), down, up);
        }
        {
            uint32_t w[16 * NP];
            tc2_split16<FMT>(x, down, w);
#pragma unroll
            for (int q = 0; q < NP; ++q) tc_st16(tmem + row1 + 32 * q + 16 * h, w + 16 * q);
            tc_wait_st();
        }
        tc_fence_before();
        __syncthreads();  // all A rows stored; every read of the tile done
        if (tid == 0) {
            tc2_issue<FMT, 1>(tmem, b_addr, mbar);
            if (issued < mine) {  // the slot is free: refill it with the tile NSTG ahead
                fence_proxy_async_smem();
                tmat_issue<float, B, N>(m, blockIdx.x + issued * gridDim.x, tilesV, ring + s * SLOT, rbar + s);
                ++issued;
            }
        }
        if (!mma_wait()) {
            ok = false;
            ++i;
            break;
        }
        {
            float y[32];
            tc_ld32(tmem + row1 + ACC1 + 32 * h, y);
            float2* line = a.dst + base_s[b1];
#pragma unroll
            for (int q = 0; q < 16; ++q)
                st_stream(line + offA_s[j1 + 16 * (16 * h + q)],
                          scl(make_float2(y[q] * up, y[16 + q] * up), a.scale));
        }
        tc_fence_before();
        __syncthreads();  // accumulators read before the next tile's MMAs; line bases free
    }
    if (!ok && tid == 0)  // wait (bounded) for this CTA's copies still in flight before leaving
        for (int j = i; j < issued; ++j) mbar_wait_bounded(rbar + j % NSTG, (uint32_t)((j / NSTG) & 1));
    __syncthreads();
    if (!drained) return;  // MMAs never seen to finish: the columns stay allocated
    tc_fence_after();
    if (tid < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS) : "memory");
}

}  // namespace a2a
