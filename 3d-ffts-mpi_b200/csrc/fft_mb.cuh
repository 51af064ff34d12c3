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

template <typename T, class PLAN, int B, int MODE>
__host__ __device__ constexpr size_t mb_smem_bytes() {
    return pass_smem_bytes<T, PLAN, B, MODE, KIND_DIRECT, 1>();
}

}  // namespace a2a
