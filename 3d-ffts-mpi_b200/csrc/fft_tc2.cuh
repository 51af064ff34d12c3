// Two-stage split-precision tensor-core pass, N = R0 x 32: 512 = 16 x 32 and
// 1024 = 32 x 32.
//
// With n = 32 a + b and k = k1 + R0 k2 (a, k1 < R0; b, k2 < 32):
//   X[k1 + R0 k2] = sum_b W32^(b k2) W_N^(b k1) sum_a x[32 a + b] W_R0^(a k1)
// Stage 0: for each b, the radix-R0 DFT over a of the stride-32 subsequence
// (no twiddles), one real GEMM row per (line, b); its outputs go to tile
// position R0 b + k1.  Stage 1: for each k1, the inputs tile[k1 + R0 b] times
// W_N^(b k1), then the radix-32 DFT over b, one 64 x 64 real GEMM row per
// (line, k1), with K = [re b<16 | im b<16 | re b>=16 | im b>=16] and the
// outputs in the same order over k2.  A radix-16 row (32 x 32, as in
// fft_tc.cuh) has one thread; a radix-32 row has two: warps w and w + 4 reach
// the same tensor-memory lanes, so thread half h writes the inputs of its half
// of K (its 16 columns of each part) and reads its half of N.  Every thread
// thus splits 16 complex values per stage.  Rows of a stage fill 128-row
// blocks of tensor memory (columns side by side): with one thread per row,
// block k belongs to warps 4k .. 4k+3; with two, to warps 8k .. 8k+7, warp w
// reaching lanes 32 (w mod 4) .. 32 (w mod 4) + 31.
//
// A pass has two GEMM stages, one twiddle multiply and one shared-memory
// exchange per element.  Operands are split as in fft_tc.cuh (fp16: two parts,
// rows scaled by a power of two; bf16: three parts); a radix-32 row's scale is
// agreed between its two threads through shared memory.  Tiles (8 lines at
// 512; 4 or 8 lines at 1024: 32 or 64 KB) arrive by the single-GPU TMA ring
// of fft_tmat.cuh (2 slots, transformed in place, no multicast); a tile's slot
// is refilled as soon as its stage-1 operands are in tensor memory.
#pragma once

#include "fft_tc.cuh"

namespace a2a {

// the radix-32 operand: K-major N x K, N = K = 64 (16-bit values): a K chunk
// of 8 values over all 64 rows is 1 KB, one part 8 KB
constexpr int kTc2ChunkB1 = 64 / 8 * 128;
constexpr int kTc2MatB1 = 8 * kTc2ChunkB1;

// Geometry of one instance: N = 512 with 8-line tiles, N = 1024 with 4- or
// 8-line tiles.  A radix-16 row has one thread, a radix-32 row two; rows are
// grouped in 128-row blocks of tensor memory.
template <int N, int BL> struct Tc2Geom {
    static_assert((N == 512 && BL == 8) || (N == 1024 && (BL == 4 || BL == 8)),
                  "two-stage instances: 512 = 16 x 32 (8 lines), 1024 = 32 x 32 (4 or 8 lines)");
    static constexpr int R0 = N / 32;                  // first radix (16 or 32); the second is 32
    static constexpr int NB1 = N / 32;                 // stage-1 rows per line (= R0)
    static constexpr int B = BL;                       // lines per tile
    static constexpr int ROWS0 = B * 32;               // stage-0 rows
    static constexpr int ROWS1 = B * NB1;              // stage-1 rows
    static constexpr int TPR0 = R0 == 16 ? 1 : 2;      // threads per stage-0 row
    static constexpr int THREADS = ROWS1 * 2;          // two threads per radix-32 row
    static constexpr int NBLK0 = ROWS0 / 128;          // 128-row blocks per stage
    static constexpr int NBLK1 = ROWS1 / 128;
    static constexpr int SH = R0 == 16 ? 4 : 5;        // log2 R0
    static constexpr int RMASK = 128 / (B * 8) - 1;    // batch-mode tile rows per 128 bytes, minus 1
    static constexpr int TW = 32 * NB1;                // twiddles W_N^(b k1), [b][k1]
    static_assert(ROWS0 * TPR0 == THREADS, "every thread has one stage-0 row (part)");
};

// both operands of one direction: the radix-16 parts (512 only), then the
// radix-32 parts (1024: one operand serves both stages)
template <int N> __host__ __device__ constexpr int tc2_b_bytes(int fmt) {
    return tc_parts(fmt) * ((N == 512 ? kTcMatB : 0) + kTc2MatB1);
}
// tensor-memory columns: stage 0 (two blocks of 16 per part + 32, or one of 32
// per part + 64) and stage 1 (one block of 32 per part + 64) take the same
// count, reused
// (per 128-row block of a stage)
__host__ __device__ constexpr int tc2_cols(int fmt) { return 32 * tc_parts(fmt) + 64; }
template <int NBLK> __host__ __device__ constexpr uint32_t tc2_tcols(int fmt) {
    return NBLK * tc2_cols(fmt) <= 128 ? 128u : NBLK * tc2_cols(fmt) <= 256 ? 256u : 512u;
}

__host__ __device__ constexpr uint32_t umma_idesc_f16_n(int fmt, int n) {
    return (1u << 4) | ((uint32_t)fmt << 7) | ((uint32_t)fmt << 10) | (((uint32_t)n >> 3) << 17) | ((128u >> 4) << 24);
}

template <int N, int BL> __host__ __device__ constexpr size_t tc2_smem_bytes(int fmt) {
    using G = Tc2Geom<N, BL>;
    size_t bytes = kTmatAlign;                                   // room to align the ring
    bytes += 2 * (size_t)tmat_slot_bytes<float, G::B, N>();      // two slots
    bytes += (size_t)tc2_b_bytes<N>(fmt);
    bytes += sizeof(float2) * (size_t)G::TW;
    bytes += sizeof(uint32_t) * (size_t)N;
    bytes += sizeof(size_t) * (size_t)G::B;
    bytes += sizeof(float) * (size_t)G::THREADS;                 // radix-32 row maxima (fp16)
    bytes += sizeof(unsigned long long) * 3 + 16;                // ring barriers, MMA barrier, tmem address, wait flag
    return bytes;
}

// Tile positions (in place in the ring slot) of the stage-0 outputs.  Batch
// mode: rows of B lines, row n stored at n ^ ((n >> log2 R0) & RMASK), so the
// rows R0 apart that a half-warp writes land in different bank groups; line
// mode: [b][n] with n's low four bits XOR-ed with (n >> log2 R0), so the
// positions R0 apart that a half-warp writes fall in distinct banks.  Stage 1's
// reads stay conflict-free under both.
template <int N, int BL, int MODE> __device__ __forceinline__ int tc2_pos(int b, int n) {
    using G = Tc2Geom<N, BL>;
    if constexpr (MODE == MODE_BATCH) return (n ^ ((n >> G::SH) & G::RMASK)) * G::B + b;
    else return b * N + (n ^ ((n >> G::SH) & 15));
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

// Thread 0: the MMAs of one GEMM stage over its NBLK 128-row blocks, then the
// commit.  Radix 16: blocks of 16 NP + 32 columns, K = 32 (two K = 16 steps
// per term), N = 32; radix 32: blocks of 32 NP + 64 columns, K = 64 (four
// steps per term), N = 64.
// `op` is the stage's split operand in shared memory.  Terms smallest first,
// as in fft_tc.cuh.
template <int FMT, int R, int NBLK>
__device__ __forceinline__ void tc2_issue(uint32_t tmem, uint32_t op, unsigned long long* bar) {
    constexpr int NP = tc_parts(FMT);
    constexpr int AC = R;                // A columns per part: 2R values, two per column
    constexpr int BC = NP * AC + 2 * R;  // block columns (A parts, then the accumulator)
    constexpr int KSTEPS = R / 8;        // K = 16 steps per term
    constexpr int CHUNK = R == 16 ? kTcChunkB : kTc2ChunkB1;  // bytes of one 8-value K chunk of the operand
    constexpr int PART = R == 16 ? kTcMatB : kTc2MatB1;
    const uint32_t idesc = umma_idesc_f16_n(FMT, 2 * R);
    tc_fence_after();
#pragma unroll
    for (int blk = 0; blk < NBLK; ++blk) {
        const uint32_t ab = tmem + blk * BC;
        const uint32_t dacc = ab + NP * AC;
        auto term = [&](int pa, int qb, uint32_t acc) {
#pragma unroll
            for (int c = 0; c < KSTEPS; ++c)
                tc_mma_ts(dacc, ab + AC * pa + 8 * c, umma_smem_desc(op + qb * PART + c * 2 * CHUNK, CHUNK, 128), idesc,
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

// ---- the stage steps of one thread (shared by the kernels below) ----

// Stage-0 inputs x[j0 + 32 a] of line b0 from the TMA slot, for this thread's
// 16 values of a (a = 16 h0 + q).
template <int N, int BL, int MODE>
__device__ __forceinline__ void tc2_s0_load(const float2* slot, const TmatMaps& m, int b0, int j0, int h0,
                                            float2 (&x)[16]) {
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int n = j0 + 32 * (16 * h0 + q);
        if constexpr (MODE == MODE_BATCH) {
            x[q] = slot[n * BL + b0];
        } else {  // [z chunk][b][z within the chunk]
            int q2, zl;
            if (m.chunk_shift >= 0) {
                q2 = n >> m.chunk_shift;
                zl = n & (m.chunk - 1);
            } else {
                q2 = n / m.chunk;
                zl = n - q2 * m.chunk;
            }
            x[q] = slot[(q2 * BL + b0) * m.chunk + zl];
        }
    }
}

// fp16 row scale of x (bf16: 1).  PAIR: the row's other half is thread tid ^
// 128; the two agree through pmax (a CTA barrier, so every thread calls this).
template <int FMT, bool PAIR>
__device__ __forceinline__ void tc2_row_scale(const float2 (&x)[16], float* pmax, int tid, float& down, float& up) {
    down = up = 1.f;
    if constexpr (FMT == TC_FP16) {
        float mx = 0.f;
#pragma unroll
        for (int q = 0; q < 16; ++q) mx = fmaxf(mx, fmaxf(fabsf(x[q].x), fabsf(x[q].y)));
        if constexpr (PAIR) {
            pmax[tid] = mx;
            __syncthreads();
            mx = fmaxf(mx, pmax[tid ^ 128]);
        }
        tc2_scale(mx, down, up);
    }
}

// The split A operand of this thread's row (part) into tensor memory at
// `row` (lane and block column): radix 16 -- the whole row, parts 16 columns
// apart; radix 32 -- half h of the row, parts 32 columns apart.
template <int FMT, int R>
__device__ __forceinline__ void tc2_store_a(uint32_t row, int h, const float2 (&x)[16], float down) {
    constexpr int NP = tc_parts(FMT);
    uint32_t w[16 * NP];
    tc2_split16<FMT>(x, down, w);
    if constexpr (R == 16) {
        tc_st32(row, reinterpret_cast<const uint32_t(&)[32]>(w));
        if constexpr (NP == 3) tc_st16(row + 32, w + 32);
    } else {
#pragma unroll
        for (int q = 0; q < NP; ++q) tc_st16(row + 32 * q + 16 * h, w + 16 * q);
    }
    tc_wait_st();
}

// Stage-0 outputs of this thread (accumulator columns at `acc`) into the
// tile: position R0 j0 + 16 h0 + q.
template <int N, int BL, int MODE>
__device__ __forceinline__ void tc2_s0_out(uint32_t acc, float2* slot, int b0, int j0, int h0, float up) {
    constexpr int R0 = Tc2Geom<N, BL>::R0;
    float y[32];
    tc_ld32(acc, y);
#pragma unroll
    for (int q = 0; q < 16; ++q) slot[tc2_pos<N, BL, MODE>(b0, R0 * j0 + 16 * h0 + q)] = make_float2(y[q] * up, y[16 + q] * up);
}

// Stage-1 inputs tile[j1 + NB1 b] times W_N^(b j1), for b = 16 h + q.
template <int N, int BL, int MODE, bool INV>
__device__ __forceinline__ void tc2_s1_load(const float2* slot, const float2* tw, int b1, int j1, int h,
                                            float2 (&x)[16]) {
    constexpr int NB1 = Tc2Geom<N, BL>::NB1;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
        const int bb = 16 * h + q;
        x[q] = cmulw<INV>(slot[tc2_pos<N, BL, MODE>(b1, j1 + NB1 * bb)], tw[bb * NB1 + j1]);  // W^0 = 1 exactly
    }
}

// Stage-1 outputs X[j1 + NB1 k2], k2 = 16 h + q, to the line in global memory.
// The row's unscale and the pass scale are one factor: `up` is a power of two,
// so up * scale is exact and every output is rounded once, as before.
template <int N, int BL>
__device__ __forceinline__ void tc2_s1_out(uint32_t acc, float2* line, const uint32_t* offA_s, int j1, int h, float up,
                                           float scale) {
    constexpr int NB1 = Tc2Geom<N, BL>::NB1;
    const float f = up * scale;
    float y[32];
    tc_ld32(acc, y);
#pragma unroll
    for (int q = 0; q < 16; ++q) st_stream(line + offA_s[j1 + NB1 * (16 * h + q)], make_float2(y[q] * f, y[16 + q] * f));
}

// The persistent kernel: each CTA allocates its tensor memory and loads the
// split operands, the twiddles and the offsets once, then works through tiles
// blockIdx.x, blockIdx.x + gridDim.x, ... of B lines, each arriving as whole
// tensor-map copies in a 2-slot ring.  Every wait is bounded; on expiry the
// device error flag is raised, the rest of the pass is skipped, the CTA waits
// (bounded) for its copies in flight and frees its tensor memory only if the
// MMAs it committed were seen to finish.
template <int N, int BL, int MODE, bool INV, int FMT>
__global__ void __launch_bounds__(Tc2Geom<N, BL>::THREADS, Tc2Geom<N, BL>::THREADS == 512 ? 1 : 2)
    fft_tc2_ring_kernel(const PassArgs<float> a, const __grid_constant__ TmatMaps m) {
    using G = Tc2Geom<N, BL>;
    constexpr int R0 = G::R0;
    constexpr int NB1 = G::NB1;
    constexpr int B = G::B;
    constexpr int TPR0 = G::TPR0;
    constexpr int THREADS = G::THREADS;
    constexpr int NP = tc_parts(FMT);
    constexpr int BC0 = NP * R0 + 2 * R0;  // stage-0 block columns (A parts, then the accumulator)
    constexpr int ACC0 = NP * R0;          // stage-0 accumulator, within its block
    constexpr int BC1 = 32 * NP + 64;      // stage-1 block columns
    constexpr int ACC1 = 32 * NP;          // stage-1 accumulator (64 columns), within its block
    constexpr uint32_t TCOLS = tc2_tcols<G::NBLK1>(FMT);
    constexpr uint32_t SLOT = tmat_slot_bytes<float, B, N>();  // B lines x N complex
    constexpr int NSTG = 2;
    static_assert(B * N * sizeof(float2) <= SLOT, "a tile fits its slot");
    static_assert(G::NBLK0 * BC0 <= (int)TCOLS && G::NBLK1 * BC1 <= (int)TCOLS, "tensor-memory columns");

    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t s0 = smem_u32(smem_raw);
    unsigned char* ring = smem_raw + (((s0 + kTmatAlign - 1) & ~(kTmatAlign - 1)) - s0);
    unsigned char* bmat = ring + NSTG * SLOT;
    float2* tw = reinterpret_cast<float2*>(bmat + tc2_b_bytes<N>(FMT));  // (operands of N, any tile height)
    uint32_t* offA_s = reinterpret_cast<uint32_t*>(tw + G::TW);
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
        for (int i = tid; i < tc2_b_bytes<N>(FMT) / 16; i += THREADS) dst[i] = src[i];
    }
    for (int i = tid; i < G::TW; i += THREADS) tw[i] = a.tw[i];
    for (int i = tid; i < N; i += THREADS) offA_s[i] = a.offA[i];
    fence_proxy_async_smem();  // operands visible to the tensor cores
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t op0 = smem_u32(bmat);                                // stage-0 operand (radix R0)
    const uint32_t op1 = op0 + (N == 512 ? NP * kTcMatB : 0);          // stage-1 operand (radix 32)
    uint32_t phase = 0;
    bool drained = true;

    // stage 0: radix 16 -- row tid (block tid / 128), one thread per row;
    // radix 32 -- row (tid / 256) * 128 + tid % 128, half h0 = (tid / 128) % 2.
    // The lane of a row is tid % 128, which warp tid / 32 reaches.
    int b0, j0, h0;
    uint32_t row0;
    {
        const int blk = TPR0 == 1 ? tid / 128 : tid / 256;
        const int r = blk * 128 + tid % 128;
        h0 = TPR0 == 1 ? 0 : (tid / 128) % 2;
        if constexpr (MODE == MODE_BATCH) { b0 = r % B; j0 = r / B; }
        else { j0 = r % 32; b0 = r / 32; }
        row0 = ((uint32_t)((warp % 4) * 32) << 16) + (uint32_t)(blk * BC0);
    }
    // stage 1: row (tid / 256) * 128 + tid % 128, half h = (tid / 128) % 2
    const int h = (tid / 128) % 2;
    const int rr = (tid / 256) * 128 + tid % 128;
    int b1, j1;
    if constexpr (MODE == MODE_BATCH) { b1 = rr % B; j1 = rr / B; }
    else { j1 = rr % NB1; b1 = rr / NB1; }
    const uint32_t row1 = ((uint32_t)((warp % 4) * 32) << 16) + (uint32_t)((tid / 256) * BC1);

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

        // ---- stage 0: radix-R0 DFTs of x[j0 + 32 a] (this thread's 16 a) ----
        float2 x[16];
        float down, up;
        tc2_s0_load<N, BL, MODE>(slot, m, b0, j0, h0, x);
        tc2_row_scale<FMT, TPR0 == 2>(x, pmax, tid, down, up);
        tc2_store_a<FMT, R0>(tmem + row0, h0, x, down);
        tc_fence_before();
        __syncthreads();  // all A rows stored; every read of the slot done
        if (tid == 0) tc2_issue<FMT, R0, G::NBLK0>(tmem, op0, mbar);
        if (!mma_wait()) {
            ok = false;
            ++i;  // tile i's copy has landed
            break;
        }
        tc2_s0_out<N, BL, MODE>(tmem + row0 + ACC0 + 32 * h0, slot, b0, j0, h0, up);
        tc_fence_before();
        __syncthreads();  // stage-0 outputs in the tile; accumulators read

        // ---- stage 1: twiddles, then radix-32 DFTs over b of tile[j1 + NB1 b] ----
        tc2_s1_load<N, BL, MODE, INV>(slot, tw, b1, j1, h, x);
        tc2_row_scale<FMT, true>(x, pmax, tid, down, up);
        tc2_store_a<FMT, 32>(tmem + row1, h, x, down);
        tc_fence_before();
        __syncthreads();  // all A rows stored; every read of the tile done
        if (tid == 0) {
            tc2_issue<FMT, 32, G::NBLK1>(tmem, op1, mbar);
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
        tc2_s1_out<N, BL>(tmem + row1 + ACC1 + 32 * h, a.dst + base_s[b1], offA_s, j1, h, up, a.scale);
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

// Software-pipelined form (fp16; the 256-thread instances: 512 with 8-line and
// 1024 with 4-line tiles).  Two tensor-memory regions of 128 columns, tile i
// in region i % 2; stage 0 and stage 1 commit to their own mbarriers.  While
// tile i's stage-1 MMAs run, the CTA prepares and issues tile i + 1's stage 0
// (its slot has landed); tile i's stage-1 results are then read back and
// stored while tile i + 1's stage-0 MMAs run.  Line bases are double-buffered.
// Thread 0 keeps the most recent commit not yet waited for: a CTA that gives up
// a wait frees its tensor memory only after that commit is seen complete.
template <int N, int BL> __host__ __device__ constexpr size_t tc2p_smem_bytes() {
    return tc2_smem_bytes<N, BL>(TC_FP16) + sizeof(size_t) * BL + sizeof(unsigned long long);
}

template <int N, int BL, int MODE, bool INV>
__global__ void __launch_bounds__(256, 2)
    fft_tc2p_ring_kernel(const PassArgs<float> a, const __grid_constant__ TmatMaps m) {
    using G = Tc2Geom<N, BL>;
    constexpr int FMT = TC_FP16;
    constexpr int R0 = G::R0;
    constexpr int B = G::B;
    constexpr int TPR0 = G::TPR0;
    constexpr int THREADS = 256;
    static_assert(G::THREADS == THREADS, "the pipelined form has the 256-thread geometries");
    constexpr int NP = tc_parts(FMT);
    constexpr int BC0 = NP * R0 + 2 * R0;
    constexpr int ACC0 = NP * R0;
    constexpr int ACC1 = 32 * NP;
    constexpr uint32_t REG = 128;  // columns per region
    constexpr uint32_t TCOLS = 2 * REG;
    static_assert(G::NBLK0 * BC0 <= (int)REG && G::NBLK1 * (32 * NP + 64) <= (int)REG, "a tile fits its region");
    constexpr uint32_t SLOT = tmat_slot_bytes<float, B, N>();
    constexpr int NSTG = 2;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t s0 = smem_u32(smem_raw);
    unsigned char* ring = smem_raw + (((s0 + kTmatAlign - 1) & ~(kTmatAlign - 1)) - s0);
    unsigned char* bmat = ring + NSTG * SLOT;
    float2* tw = reinterpret_cast<float2*>(bmat + tc2_b_bytes<N>(FMT));
    uint32_t* offA_s = reinterpret_cast<uint32_t*>(tw + G::TW);
    size_t* base_s = reinterpret_cast<size_t*>(offA_s + N);  // [2][B]
    float* pmax = reinterpret_cast<float*>(base_s + 2 * B);
    unsigned long long* rbar = reinterpret_cast<unsigned long long*>(pmax + THREADS);
    unsigned long long* mb0 = rbar + NSTG;  // stage-0 commits
    unsigned long long* mb1 = mb0 + 1;      // stage-1 commits
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mb1 + 1);
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
        mbar_init(mb0, 1);
        mbar_init(mb1, 1);
        fence_mbar_init();
    }
    {
        const uint4* src = reinterpret_cast<const uint4*>(a.tcb);
        uint4* dst = reinterpret_cast<uint4*>(bmat);
        for (int i = tid; i < tc2_b_bytes<N>(FMT) / 16; i += THREADS) dst[i] = src[i];
    }
    for (int i = tid; i < G::TW; i += THREADS) tw[i] = a.tw[i];
    for (int i = tid; i < N; i += THREADS) offA_s[i] = a.offA[i];
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t op0 = smem_u32(bmat);
    const uint32_t op1 = op0 + (N == 512 ? NP * kTcMatB : 0);

    // rows as in fft_tc2_ring_kernel (256 threads: one stage-1 block)
    int b0, j0, h0;
    uint32_t row0;
    {
        const int blk = TPR0 == 1 ? tid / 128 : 0;
        const int r = blk * 128 + tid % 128;
        h0 = TPR0 == 1 ? 0 : tid / 128;
        if constexpr (MODE == MODE_BATCH) { b0 = r % B; j0 = r / B; }
        else { j0 = r % 32; b0 = r / 32; }
        row0 = ((uint32_t)((warp % 4) * 32) << 16) + (uint32_t)(blk * BC0);
    }
    const int h = tid / 128;
    const int rr = tid % 128;
    int b1, j1;
    if constexpr (MODE == MODE_BATCH) { b1 = rr % B; j1 = rr / B; }
    else { j1 = rr % G::NB1; b1 = rr / G::NB1; }
    const uint32_t row1 = (uint32_t)((warp % 4) * 32) << 16;

    uint32_t ph0 = 0, ph1 = 0;
    unsigned long long* pend = nullptr;  // thread 0: the latest commit not yet waited for
    uint32_t pend_ph = 0;
    bool drained = true;
    // an MMA completion: thread 0 waits (bounded) and tells the CTA; on expiry
    // the error flag is raised and `drained` says whether the latest commit
    // was then seen complete
    auto mma_wait = [&](unsigned long long* bar, uint32_t& ph) -> bool {
        if (tid == 0) {
            int f = 0;
            if (!mbar_wait_bounded(bar, ph)) f = (pend && !mbar_wait_bounded(pend, pend_ph)) ? 2 : 1;
            else if (pend == bar && pend_ph == ph) pend = nullptr;
            *wflag = f;
        }
        __syncthreads();
        const int f = *wflag;
        if (f) {
            if (tid == 0) atomicExch(a.err, 1);
            drained = f == 1;
            return false;
        }
        ph ^= 1u;
        tc_fence_after();
        return true;
    };
    auto line_base = [&](int t) -> size_t {
        const int u = t / tilesV;
        const int v0 = (t - u * tilesV) * B;
        return (size_t)__ldg(a.offU + u) + __ldg(a.offV + v0 + tid);
    };

    int issued = 0;  // thread 0: tiles of this CTA whose copies were issued
    if (tid == 0)
        for (; issued < NSTG && issued < mine; ++issued)
            tmat_issue<float, B, N>(m, blockIdx.x + issued * gridDim.x, tilesV, ring + issued * SLOT, rbar + issued);
    size_t nbase = 0;
    if (tid < B && mine > 0) nbase = line_base(blockIdx.x);
    int consumed = 0;  // tiles whose copies were waited for
    float up0 = 1.f;   // stage-0 unscale of the tile whose stage 0 is in flight
    float2 x[16];
    float down;
    // stage 0 of this CTA's tile k into region k % 2: line bases, slot, operands, MMAs
    auto stage0 = [&](int k) -> bool {
        if (tid < B) {
            base_s[(k & 1) * B + tid] = nbase;
            if (k + 1 < mine) nbase = line_base(blockIdx.x + (k + 1) * gridDim.x);
        }
        if (__syncthreads_or(!mbar_wait_bounded(rbar + k % NSTG, (uint32_t)((k / NSTG) & 1)))) {
            if (tid == 0) atomicExch(a.err, 1);
            return false;
        }
        ++consumed;
        const float2* slot = reinterpret_cast<const float2*>(ring + (k % NSTG) * SLOT);
        tc2_s0_load<N, B, MODE>(slot, m, b0, j0, h0, x);
        tc2_row_scale<FMT, TPR0 == 2>(x, pmax, tid, down, up0);
        tc2_store_a<FMT, R0>(tmem + (uint32_t)(k & 1) * REG + row0, h0, x, down);
        tc_fence_before();
        __syncthreads();  // all A rows stored; every read of the slot done
        if (tid == 0) {
            tc2_issue<FMT, R0, G::NBLK0>(tmem + (uint32_t)(k & 1) * REG, op0, mb0);
            pend = mb0;
            pend_ph = ph0;
        }
        return true;
    };

    bool ok = mine > 0 ? stage0(0) : true;
    for (int i = 0; ok && i < mine; ++i) {
        const uint32_t reg = (uint32_t)(i & 1) * REG;
        float2* slot = reinterpret_cast<float2*>(ring + (i % NSTG) * SLOT);
        if (!mma_wait(mb0, ph0)) {  // tile i's stage 0
            ok = false;
            break;
        }
        tc2_s0_out<N, B, MODE>(tmem + reg + row0 + ACC0 + 32 * h0, slot, b0, j0, h0, up0);
        tc_fence_before();
        __syncthreads();  // stage-0 outputs in the tile; accumulators read
        float up1;
        tc2_s1_load<N, B, MODE, INV>(slot, tw, b1, j1, h, x);
        tc2_row_scale<FMT, true>(x, pmax, tid, down, up1);
        tc2_store_a<FMT, 32>(tmem + reg + row1, h, x, down);
        tc_fence_before();
        __syncthreads();  // all A rows stored; every read of the tile done
        if (tid == 0) {
            tc2_issue<FMT, 32, G::NBLK1>(tmem + reg, op1, mb1);
            pend = mb1;
            pend_ph = ph1;
            if (issued < mine) {  // the slot is free: refill it with the tile NSTG ahead
                fence_proxy_async_smem();
                tmat_issue<float, B, N>(m, blockIdx.x + issued * gridDim.x, tilesV, ring + (i % NSTG) * SLOT,
                                        rbar + (i % NSTG));
                ++issued;
            }
        }
        if (i + 1 < mine && !stage0(i + 1)) {  // under tile i's stage-1 MMAs
            ok = false;
            break;
        }
        if (!mma_wait(mb1, ph1)) {  // tile i's stage 1
            ok = false;
            break;
        }
        tc2_s1_out<N, B>(tmem + reg + row1 + ACC1 + 32 * h, a.dst + base_s[(i & 1) * B + b1], offA_s, j1, h, up1,
                         a.scale);
        tc_fence_before();
        __syncthreads();  // accumulators read before the region is reused; line bases free
    }
    if (!ok) {  // copies and MMAs still in flight, each waited for (bounded)
        if (tid == 0) {
            for (int j = consumed; j < issued; ++j) mbar_wait_bounded(rbar + j % NSTG, (uint32_t)((j / NSTG) & 1));
            *wflag = (pend && !mbar_wait_bounded(pend, pend_ph)) ? 2 : 0;
        }
        __syncthreads();
        if (*wflag == 2) drained = false;
    }
    __syncthreads();
    if (!drained) return;  // MMAs never seen to finish: the columns stay allocated
    tc_fence_after();
    if (tid < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(TCOLS) : "memory");
}

}  // namespace a2a
