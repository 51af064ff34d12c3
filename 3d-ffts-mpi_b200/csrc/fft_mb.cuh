// Axis pass over a virtual rank-major buffer split into G blocks that may live
// in other GPUs' memory: the fused form of one a2afft axis step across
// devices.  Block g holds the contiguous virtual ranks [g L, (g+1) L) (L =
// P / G), so element o of the virtual buffer is element o mod (L nlocal) of
// block o div (L nlocal).  A CTA gathers its tile's lines straight from the
// owners' bricks (peer loads over NVLink where a block is remote), transforms
// them and scatters the results back to the owners: the alltoall, the pencil
// remaps and the 1D FFTs of a reference step in one kernel, each element
// crossing the link once each way.  Processes split a pass's tiles between
// them (`tile0`, the launch's grid); no kernel waits on another GPU -- the
// caller orders the passes (every process's pass p completes before any
// process starts pass p + 1).
#pragma once

#include "fft_tile.cuh"
#include "fft_tmat.cuh"

namespace a2a {

// One tile per CTA (tile t = tile0 + blockIdx.x), the one-tile pass body with
// every global address translated to its block.
template <typename T, class PLAN, int B, int THREADS, int MODE, bool INV, int MINB>
__global__ void __launch_bounds__(THREADS, MINB) fft_mb_kernel(const PassArgs<T> a, const __grid_constant__ MbArgs<T> mb) {
    using E = cx<T>;
    using G = TileGeom<MODE, B, PLAN::N, sizeof(E)>;
    constexpr int N = PLAN::N;
    constexpr int R0 = PLAN::r[0];
    constexpr int NBL = N / R0;
    constexpr int NBT = B * NBL;
    constexpr int K = (NBT + THREADS - 1) / THREADS;
    constexpr bool EXACT = (NBT % THREADS) == 0;
    constexpr int TWN = PLAN::twtotal();
    constexpr bool BFAST0 = (MODE == MODE_BATCH);
    static_assert(PLAN::S >= 2, "the multi-block pass needs at least two stages");
    static_assert(MODE != MODE_BATCH || THREADS % B == 0, "batch mode needs THREADS % B == 0");

    extern __shared__ __align__(16) unsigned char smem_raw[];
    E* tile = reinterpret_cast<E*>(smem_raw);
    cx<T>* tw = reinterpret_cast<cx<T>*>(tile + G::elems);
    uint32_t* offA_s = reinterpret_cast<uint32_t*>(tw + TWN);
    size_t* base_s = reinterpret_cast<size_t*>(
        smem_raw + ((sizeof(E) * (size_t)G::elems + sizeof(cx<T>) * TWN + sizeof(uint32_t) * N + 15) & ~size_t(15)));

    const int tid = threadIdx.x;
    const int t = mb.tile0 + (int)blockIdx.x;
    const int tilesV = a.NV / B;
    const int u = t / tilesV;
    const int v0 = (t - u * tilesV) * B;
    const uint32_t ubase = __ldg(a.offU + u);

    E x[K][R0];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int q = tid + k * THREADS;
        if (EXACT || q < NBT) {
            int b, j;
            bf_map<BFAST0, B, NBL>(q, b, j);
            const uint32_t line = ubase + __ldg(a.offV + v0 + b);
#pragma unroll
            for (int r = 0; r < R0; ++r) x[k][r] = ld_stream(mb_addr(mb, line + __ldg(a.offA + j + r * NBL)));
        }
    }
    for (int i = tid; i < TWN; i += THREADS) tw[i] = a.tw[i];
    for (int i = tid; i < N; i += THREADS) offA_s[i] = a.offA[i];
    for (int i = tid; i < B; i += THREADS) base_s[i] = ubase + a.offV[v0 + i];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int q = tid + k * THREADS;
        if (EXACT || q < NBT) {
            int b, j;
            bf_map<BFAST0, B, NBL>(q, b, j);
            Dft<R0, INV, E>::run(x[k]);
#pragma unroll
            for (int r = 0; r < R0; ++r) tile[G::idx(b, j * R0 + r)] = x[k][r];
        }
    }
    __syncthreads();
    run_stage<T, PLAN, B, THREADS, MODE, INV, 1, 1, -1, true>(a, tile, tw, offA_s, base_s, tid, &mb);
}

// Persistent form: CTA c runs tiles tile0 + c, tile0 + c + gridDim.x, ...
// below tile1 with the register-pipelined body of the single-buffer pass
// (fft_rpipe_kernel): stage 0 of tile t leaves its results in shared memory,
// then the same registers receive tile t + gridDim.x's gathers (peer loads
// where its lines live in another GPU's block), which stay in flight while
// stages 1..S-1 of tile t run and scatter it back.  LPT = 2 (BATCH, complex
// float): a thread moves the same element of two adjacent lines as one
// 16-byte access.
template <typename T, class PLAN, int B, int THREADS, int MODE, bool INV, int MINB, int LPT>
__global__ void __launch_bounds__(THREADS, MINB)
    fft_mb_rpipe_kernel(const PassArgs<T> a, const __grid_constant__ MbArgs<T> mb) {
    using E = typename ElemOf<T, LPT>::type;
    constexpr int BV = B / LPT;
    using G = TileGeom<MODE, BV, PLAN::N, sizeof(E)>;
    constexpr int N = PLAN::N;
    constexpr int R0 = PLAN::r[0];
    constexpr int NBL = N / R0;
    constexpr int NBT = BV * NBL;
    constexpr int K = (NBT + THREADS - 1) / THREADS;
    constexpr bool EXACT = (NBT % THREADS) == 0;
    constexpr int TWN = PLAN::twtotal();
    constexpr bool BFAST0 = (MODE == MODE_BATCH);
    static_assert(PLAN::S >= 2, "the pipelined kernel needs at least two stages");
    static_assert(MODE != MODE_BATCH || THREADS % BV == 0, "batch mode needs THREADS % (B/LPT) == 0");
    static_assert(LPT == 1 || MODE == MODE_BATCH, "line pairs only in batch mode");

    extern __shared__ __align__(16) unsigned char smem_raw[];
    E* tile = reinterpret_cast<E*>(smem_raw);
    cx<T>* tw = reinterpret_cast<cx<T>*>(tile + G::elems);
    uint32_t* offA_s = reinterpret_cast<uint32_t*>(tw + TWN);
    size_t* base_s = reinterpret_cast<size_t*>(
        smem_raw + ((sizeof(E) * (size_t)G::elems + sizeof(cx<T>) * TWN + sizeof(uint32_t) * N + 15) & ~size_t(15)));

    const int tid = threadIdx.x;
    const int tilesV = a.NV / B;
    auto load_tile = [&](int t, E (&x)[K][R0]) {
        const int u = t / tilesV;
        const int v0 = (t - u * tilesV) * B;
        const uint32_t ubase = __ldg(a.offU + u);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int q = tid + k * THREADS;
            if (EXACT || q < NBT) {
                int b, j;
                bf_map<BFAST0, BV, NBL>(q, b, j);
                const uint32_t line = ubase + __ldg(a.offV + v0 + b * LPT);
#pragma unroll
                for (int r = 0; r < R0; ++r)
                    x[k][r] = ld_stream(reinterpret_cast<const E*>(mb_addr(mb, line + __ldg(a.offA + j + r * NBL))));
            }
        }
    };
    int t = mb.tile0 + (int)blockIdx.x;
    E x[K][R0];
    if (t < mb.tile1) load_tile(t, x);
    for (int i = tid; i < TWN; i += THREADS) tw[i] = a.tw[i];
    for (int i = tid; i < N; i += THREADS) offA_s[i] = a.offA[i];
    for (; t < mb.tile1; t += gridDim.x) {
        {
            const int u = t / tilesV;
            const int v0 = (t - u * tilesV) * B;
            const uint32_t ubase = __ldg(a.offU + u);
            for (int i = tid; i < BV; i += THREADS) base_s[i] = ubase + __ldg(a.offV + v0 + i * LPT);
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int q = tid + k * THREADS;
            if (EXACT || q < NBT) {
                int b, j;
                bf_map<BFAST0, BV, NBL>(q, b, j);
                Dft<R0, INV, E>::run(x[k]);
#pragma unroll
                for (int r = 0; r < R0; ++r) tile[G::idx(b, j * R0 + r)] = x[k][r];
            }
        }
        const int tn = t + gridDim.x;
        if (tn < mb.tile1) load_tile(tn, x);  // in flight through the remaining stages
        __syncthreads();
        run_stage<T, PLAN, B, THREADS, MODE, INV, LPT, 1, -1, true>(a, tile, tw, offA_s, base_s, tid, &mb);
        __syncthreads();  // tile and line bases free for the next tile
    }
}

// Batch-mode (X and Y) passes fed by TMA: a tile's lines cross the d0 (X)
// or d1 (Y) bricks along the transform axis, each brick another virtual rank
// that may live in another GPU's block.  One 3-D tensor map per virtual rank
// (in global memory, built on the host from the block addresses: the rank's
// brick [x_l][y_l][z_l] at its block's base) describes its brick; a tile is
// one box per brick along the line -- [B, 1, lx] (X) or [B, ly, 1] (Y) words
// of the lines' z range -- landing at that brick's rows of the shared tile,
// which then has the single-buffer ring kernel's [n][b] layout.  The copies
// are plain tensor-map loads (peer memory is allowed as a source; no
// multicast anywhere), completed on the slot's mbarrier with bounded waits.
// Persistent CTAs run tiles tile0 + c, tile0 + c + gridDim.x, ... below
// tile1 through a 2-slot ring; the last stage scatters to the owners' blocks
// (peer stores) with the per-element block translation.
struct MbTmaMaps {
    const CUtensorMap* map;  // one per virtual rank, 64-byte aligned, global memory
    int pass;                // 1 = X, 2 = Y
    int lx, ly, lz;          // brick extents (elements)
    int words;               // 8-byte words per complex element
    int d1, d2;              // brick grid (d0 along X is the box count of an X tile)
    int nbox;                // bricks along the transform axis (d0 for X, d1 for Y)
};

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

// Thread 0: arm the slot's barrier for tile t and issue one box per brick.
template <typename T, int B, int N>
__device__ __forceinline__ void mb_tma_issue(const MbTmaMaps& m, int t, int tilesV, unsigned char* dst,
                                             unsigned long long* bar) {
    mbar_arrive_expect_tx(bar, (uint32_t)(B * N * sizeof(cx<T>)));
    const int u = t / tilesV;
    const int v0 = (t - u * tilesV) * B;
    const int zr = v0 / m.lz, zl = v0 - zr * m.lz;
    if (m.pass == 1) {  // lines (y = u, z = v0 ..): bricks c0 = 0 .. d0-1
        const int c1 = u / m.ly, yl = u - c1 * m.ly;
        const uint32_t box = (uint32_t)(B * m.lx * sizeof(cx<T>));
        for (int c0 = 0; c0 < m.nbox; ++c0)
            tma_load_3d(dst + c0 * box, m.map + (c0 * m.d1 + c1) * m.d2 + zr, m.words * zl, yl, 0, bar);
    } else {  // lines (x = u, z = v0 ..): bricks c1 = 0 .. d1-1
        const int c0 = u / m.lx, xl = u - c0 * m.lx;
        const uint32_t box = (uint32_t)(B * m.ly * sizeof(cx<T>));
        for (int c1 = 0; c1 < m.nbox; ++c1)
            tma_load_3d(dst + c1 * box, m.map + (c0 * m.d1 + c1) * m.d2 + zr, m.words * zl, 0, xl, bar);
    }
}

template <typename T, class PLAN, int B, int THREADS, bool INV, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
    fft_mb_tmat_kernel(const PassArgs<T> a, const __grid_constant__ MbArgs<T> mb,
                       const __grid_constant__ MbTmaMaps m) {
    using E = cx<T>;
    constexpr int SWSH = tile_swizzle_shift<PLAN, B, (int)sizeof(E)>();
    using G = TileGeom<MODE_BATCH, B, PLAN::N, sizeof(E), SWSH>;
    constexpr int N = PLAN::N;
    constexpr int R0 = PLAN::r[0];
    constexpr int NBL = N / R0;
    constexpr int NBT = B * NBL;
    constexpr int K = (NBT + THREADS - 1) / THREADS;
    constexpr bool EXACT = (NBT % THREADS) == 0;
    constexpr int TWN = PLAN::twtotal();
    constexpr int NSTG = 2;
    constexpr uint32_t SLOT = tmat_slot_bytes<T, B, N>();
    static_assert(PLAN::S >= 2, "the ring kernel needs at least two stages");
    static_assert(THREADS % B == 0, "batch mode needs THREADS % B == 0");

    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t s0 = smem_u32(smem_raw);
    unsigned char* ring = smem_raw + (((s0 + kTmatAlign - 1) & ~(kTmatAlign - 1)) - s0);
    E* const tile = reinterpret_cast<E*>(ring + NSTG * SLOT);
    cx<T>* tw = reinterpret_cast<cx<T>*>(tile + G::elems);
    uint32_t* offA_s = reinterpret_cast<uint32_t*>(tw + TWN);
    size_t* base_s = reinterpret_cast<size_t*>(
        reinterpret_cast<unsigned char*>(tw) + ((sizeof(cx<T>) * TWN + sizeof(uint32_t) * N + 15) & ~size_t(15)));
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(base_s + B);

    const int tid = threadIdx.x;
    const int tilesV = a.NV / B;
    const int ntiles = mb.tile1 - mb.tile0;
    const int mine = (int)blockIdx.x < ntiles ? (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;
    if (tid == 0) {
        for (int i = 0; i < NSTG; ++i) mbar_init(bar + i, 1);
        fence_mbar_init();
    }
    for (int i = tid; i < TWN; i += THREADS) tw[i] = a.tw[i];
    for (int i = tid; i < N; i += THREADS) offA_s[i] = a.offA[i];
    __syncthreads();
    int issued = 0;  // thread 0: tiles of this CTA whose copies were issued
    if (tid == 0)
        for (; issued < NSTG && issued < mine; ++issued)
            mb_tma_issue<T, B, N>(m, mb.tile0 + blockIdx.x + issued * gridDim.x, tilesV, ring + issued * SLOT,
                                  bar + issued);

    for (int i = 0; i < mine; ++i) {
        const int t = mb.tile0 + blockIdx.x + i * gridDim.x;
        const int s = i % NSTG;
        {
            const int u = t / tilesV;
            const int v0 = (t - u * tilesV) * B;
            const uint32_t ubase = __ldg(a.offU + u);
            for (int b = tid; b < B; b += THREADS) base_s[b] = ubase + __ldg(a.offV + v0 + b);
        }
        const bool ok = mbar_wait_bounded(bar + s, (uint32_t)((i / NSTG) & 1));
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicExch(a.err, 1);
                // wait (bounded) for this CTA's copies still in flight before leaving
                for (int j = i; j < issued; ++j) mbar_wait_bounded(bar + j % NSTG, (uint32_t)((j / NSTG) & 1));
            }
            return;
        }
        const E* src = reinterpret_cast<const E*>(ring + s * SLOT);
        E x[K][R0];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int q = tid + k * THREADS;
            if (EXACT || q < NBT) {
                int b, j;
                bf_map<true, B, NBL>(q, b, j);
#pragma unroll
                for (int r = 0; r < R0; ++r) x[k][r] = src[(j + r * NBL) * B + b];
            }
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int q = tid + k * THREADS;
            if (EXACT || q < NBT) {
                int b, j;
                bf_map<true, B, NBL>(q, b, j);
                Dft<R0, INV, E>::run(x[k]);
#pragma unroll
                for (int r = 0; r < R0; ++r) tile[G::idx(b, j * R0 + r)] = x[k][r];
            }
        }
        __syncthreads();  // slot s read out; the tile and its line bases are ready
        if (tid == 0 && issued < mine) {
            fence_proxy_async_smem();  // the generic reads of slot s come before the async writes
            mb_tma_issue<T, B, N>(m, mb.tile0 + blockIdx.x + issued * gridDim.x, tilesV, ring + s * SLOT, bar + s);
            ++issued;
        }
        run_stage<T, PLAN, B, THREADS, MODE_BATCH, INV, 1, 1, SWSH, true>(a, tile, tw, offA_s, base_s, tid, &mb);
        __syncthreads();  // tile and line bases free for the next tile
    }
}

template <typename T, class PLAN, int B>
__host__ __device__ constexpr size_t mb_tmat_smem_bytes() {
    return tmat_smem_bytes<T, PLAN, B, MODE_BATCH, 1, 2, false>();
}

template <typename T, class PLAN, int B, int MODE>
__host__ __device__ constexpr size_t mb_smem_bytes() {
    return pass_smem_bytes<T, PLAN, B, MODE, KIND_DIRECT, 1>();
}

}  // namespace a2a
