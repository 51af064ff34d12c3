// Batched form: many independent boxes (each on its own virtual-rank brick
// grid) transformed by ONE persistent launch per direction.
//
// Work items are (pass, box, tile) triples ordered pass-major: every Z tile of
// every box, then every X tile, then every Y tile.  CTAs take items in that
// order from a device work counter; an X (Y) item first waits until all Z (X)
// tiles of its box are done (a per-box, per-pass completion counter).  A CTA
// only ever waits on items with lower indices, which running CTAs already
// hold, so the waits always end; they are still bounded (about one second),
// after which the kernel raises the error flag and every CTA stops taking
// work.  The tile code is the one-tile-per-CTA pass body (direct_tile) with a
// compiled configuration per transform length, two tile heights each (the
// plan's autotuner chooses per length).
#pragma once

#include "fft_registry.cuh"

namespace a2a {

constexpr int kBatchThreads = 256;
constexpr int kBatchMaxBoxes = 65536;

// Tile height per (element type, length, variant) for kBatchThreads threads:
// three choices per length for the plan's tuner -- 0 and 1 two heights, 2 the
// height of 0 with each thread moving two adjacent lines as one 16-byte access
// (complex float, batch mode, lines in aligned pairs; elsewhere it is 0);
// complex double uses half the lines of complex float (same registers per
// thread).
constexpr int kBatchVariants = 3;
__host__ __device__ constexpr int batch_lines_f32(int n, int v) {
    return (n == 48 || n == 256 || n == 512) ? (v == 1 ? 8 : 16) : (v == 1 ? 16 : 32);
}
template <typename T> __host__ __device__ constexpr int batch_lpt(int v, int mode) {
    return (v == 2 && sizeof(T) == 4 && mode == MODE_BATCH) ? 2 : 1;
}
template <typename T> __host__ __device__ constexpr int batch_lines(int n, int v) {
    return sizeof(T) == 4 ? batch_lines_f32(n, v) : batch_lines_f32(n, v) / 2;
}
#define A2A_BATCH_FOR_EACH_N(X) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(512)
constexpr int kBatchLengths[] = {32, 48, 64, 96, 128, 192, 256, 512};
constexpr int kBatchNumLengths = 8;

// One box of the batch (device copy in the plan).
struct BatchBox {
    void* data;              // the box's rank-major bricks (set per call)
    const uint32_t* off[3];  // brick offsets per axis
    const void* tw[3];       // stage twiddles per axis (forward sign)
    int n[3];                // edges
    int var[3];              // tile variant per pass (Z, X, Y)
    int lines[3];            // tile height per pass
    int tiles[3];            // tiles per pass
    // off[a][x] = (x / lext[a]) * rstride[a] + (x % lext[a]) * lstride[a]
    // (brick extent, rank stride, in-brick stride): prefetch addresses
    // without table loads
    uint32_t lext[3], rstride[3], lstride[3];
    int split[3];            // split addressing usable per pass
    double inv_scale;        // 1 / (nx ny nz)
};

// Arguments of one launch: work items [item_lo, item_hi) of the plan's item
// list, which holds (box * 4 + pass, tile) per item, pass-major.  The three
// counters live in the plan's queue scratch and are zero at launch.
struct BatchArgs {
    const BatchBox* boxes;
    const int2* items;
    int item_lo, item_hi;
    int claim;               // most items a CTA takes per queue access
    int fused;               // 1: later passes wait for the earlier pass of their box
    int wait_extra;          // 0; > 0 makes every wait unsatisfiable (tests of the timeout path)
    int prefetch;            // 1: prefetch the CTA's next tile into L2 while running the current one
    int* taken;              // items taken so far
    int* abort;              // raised when a wait gave up: every CTA stops
    int* done;               // tiles finished per (box, pass), 3 ints per box
    int* err;                // set to 1 when a wait gave up (not cleared by launches)
};

// A run of m consecutive tiles t0 .. t0+m-1 of one pass of one box, with the
// register double-buffering of the persistent pass kernel: stage 0 of tile t
// leaves its results in shared memory, then its registers receive the global
// loads of tile t+1, which stay in flight through stages 1..S-1 of tile t.
// Loads read through L2 only (__ldcg): other CTAs of this launch wrote the
// data (earlier passes).
template <typename T, class PLAN, int B, int THREADS, int MODE, bool INV, int LPT = 1>
__device__ __forceinline__ void rpipe_run(const PassArgs<T>& a, int t0, int m, unsigned char* smem_raw, int tid) {
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
    static_assert(PLAN::S >= 2, "the pipelined run needs at least two stages");
    static_assert(MODE != MODE_BATCH || THREADS % BV == 0, "batch mode needs THREADS % (B/LPT) == 0");
    static_assert(LPT == 1 || MODE == MODE_BATCH, "line pairs only in batch mode");

    E* tile = reinterpret_cast<E*>(smem_raw);
    cx<T>* tw = reinterpret_cast<cx<T>*>(tile + G::elems);
    uint32_t* offA_s = reinterpret_cast<uint32_t*>(tw + TWN);
    size_t* base_s = reinterpret_cast<size_t*>(
        smem_raw + ((sizeof(E) * (size_t)G::elems + sizeof(cx<T>) * TWN + sizeof(uint32_t) * N + 15) & ~size_t(15)));

    const int tilesV = a.NV / B;
    uint32_t d0[R0];
    if (a.split) {
#pragma unroll
        for (int r = 0; r < R0; ++r) d0[r] = __ldg(a.offA + r * NBL);
    }
    auto load_tile = [&](int t, E (&x)[K][R0]) {
        const int u = t / tilesV;
        const int v0 = (t - u * tilesV) * B;
        const size_t ubase = __ldg(a.offU + u);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int q = tid + k * THREADS;
            if (EXACT || q < NBT) {
                int b, j;
                bf_map<BFAST0, BV, NBL>(q, b, j);
                const cx<T>* line = a.src + ubase + __ldg(a.offV + v0 + b * LPT);
                if (a.split) {
                    const cx<T>* p = line + __ldg(a.offA + j);
#pragma unroll
                    for (int r = 0; r < R0; ++r) x[k][r] = __ldcg(reinterpret_cast<const E*>(p + d0[r]));
                } else {
#pragma unroll
                    for (int r = 0; r < R0; ++r)
                        x[k][r] = __ldcg(reinterpret_cast<const E*>(line + __ldg(a.offA + j + r * NBL)));
                }
            }
        }
    };
    E x[K][R0];
    load_tile(t0, x);
    for (int i = tid; i < TWN; i += THREADS) tw[i] = a.tw[i];
    for (int i = tid; i < N; i += THREADS) offA_s[i] = a.offA[i];
    for (int t = t0; t < t0 + m; ++t) {
        {
            const int u = t / tilesV;
            const int v0 = (t - u * tilesV) * B;
            const size_t ubase = __ldg(a.offU + u);
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
        if (t + 1 < t0 + m) load_tile(t + 1, x);  // in flight through the remaining stages
        __syncthreads();
        run_stage<T, PLAN, B, THREADS, MODE, INV, LPT, 1>(a, tile, tw, offA_s, base_s, tid);
        __syncthreads();  // tile and line bases free for the next tile
    }
}

// A run of one configuration, compiled as its own function so that each
// configuration gets its own register allocation (inlined into one body they
// would share the worst case and spill).
template <typename T, bool INV, int N, int V, int MODE>
__device__ __noinline__ void batch_tile(cx<T>* data, const uint32_t* offA, const uint32_t* offU, const uint32_t* offV,
                                        const cx<T>* tw, int NU, int NV, T scale, int split, int tile, int count,
                                        unsigned char* smem, int tid) {
    using P = typename PassPlan<T, N>::Plan;
    PassArgs<T> pa;
    pa.src = data;
    pa.dst = data;
    pa.offA = offA;
    pa.offU = offU;
    pa.offV = offV;
    pa.tw = tw;
    pa.NU = NU;
    pa.NV = NV;
    pa.scale = scale;
    pa.split = split;
    pa.err = nullptr;
    pa.tcb = nullptr;
    rpipe_run<T, P, batch_lines<T>(N, V), kBatchThreads, MODE, INV, batch_lpt<T>(V, MODE)>(pa, tile, count, smem,
                                                                                           tid);
}

template <typename T, bool INV, int N>
__device__ __forceinline__ void batch_len(cx<T>* data, const uint32_t* offA, const uint32_t* offU,
                                          const uint32_t* offV, const cx<T>* tw, int NU, int NV, T scale, int split,
                                          int mode, int var, int tile, int count, unsigned char* smem, int tid) {
#define A2A_BT(V_, M_) \
    batch_tile<T, INV, N, V_, M_>(data, offA, offU, offV, tw, NU, NV, scale, split, tile, count, smem, tid)
    if (mode == MODE_LINE) {
        if (var == 1) A2A_BT(1, MODE_LINE); else A2A_BT(0, MODE_LINE);
    } else {
        if (var == 0) A2A_BT(0, MODE_BATCH); else if (var == 1) A2A_BT(1, MODE_BATCH); else A2A_BT(2, MODE_BATCH);
    }
#undef A2A_BT
}

// Polls a completion counter until it reaches `target`; false after about a
// second (or 2^24 polls), or as soon as another CTA has raised `abort`.
__device__ __forceinline__ bool wait_count(const int* ctr, int target, const int* abort) {
    const uint64_t t0 = global_ns();
    for (int i = 0; i < (1 << 24); ++i) {
        if (*reinterpret_cast<const volatile int*>(ctr) >= target) return true;
        if ((i & 255) == 255) {
            if (*reinterpret_cast<const volatile int*>(abort)) return false;
            if (global_ns() - t0 > 1000000000ull) return false;
            __nanosleep(200);
        }
    }
    return false;
}

__device__ __forceinline__ uint32_t box_off(const BatchBox& bx, int a, uint32_t x) {
    const uint32_t q = x / bx.lext[a];
    return q * bx.rstride[a] + (x - q * bx.lext[a]) * bx.lstride[a];
}

__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
}

// Asks L2 for the 128-byte lines of one tile (every address is an element of
// the tile, so nothing outside the box is touched).
template <typename T>
__device__ __forceinline__ void prefetch_tile(const BatchBox& bx, int pass, int tile, int tid) {
    constexpr int EPL = 128 / (int)sizeof(cx<T>);  // elements per 128-byte line
    const int ax = pass == 0 ? 2 : pass == 1 ? 0 : 1;
    const int au = pass == 1 ? 1 : 0;
    const int av = pass == 0 ? 1 : 2;
    const int N = bx.n[ax], B = bx.lines[pass];
    const int tilesV = bx.n[av] / B;
    const int u = tile / tilesV, v0 = (tile - u * tilesV) * B;
    const cx<T>* base = static_cast<const cx<T>*>(bx.data) + box_off(bx, au, u);
    if (pass == 0) {  // B lines, contiguous along the transform axis
        const int cpl = (N + EPL - 1) / EPL;
        for (int q = tid; q < B * cpl; q += kBatchThreads) {
            const int b = q / cpl, c = q - b * cpl;
            prefetch_l2(base + box_off(bx, av, v0 + b) + box_off(bx, ax, c * EPL));
        }
    } else {  // N rows of B adjacent lines
        const int cpr = (B + EPL - 1) / EPL;
        for (int q = tid; q < N * cpr; q += kBatchThreads) {
            const int j = q / cpr, c = q - j * cpr;
            prefetch_l2(base + box_off(bx, ax, j) + box_off(bx, av, v0 + c * EPL));
        }
    }
}

// The persistent kernel.  Thread 0 takes up to `claim` consecutive items per
// queue access (fewer as the queue drains); the CTA runs them as runs of consecutive tiles of one (box, pass).
// In the fused schedule thread 0 checks a run's dependency (every tile of the
// previous pass of its box done) once per (box, pass) change, with an acquire
// fence after the wait, and publishes finished tiles per (box, pass) with a
// release (fence, then one counter increment).  It
// publishes before it waits, so a CTA never waits while holding unpublished
// tiles.  Thread 0 takes its claims one ahead (the next claim is taken when
// the current one starts), so a CTA's claims are consecutive in the queue
// order and it runs them in that order: an item waits only on items taken
// before it, and the lowest unfinished taken item is always the current run
// of the CTA holding it, so it always runs and the waits end.
template <typename T, bool INV>
__global__ void __launch_bounds__(kBatchThreads, 2) fft_batch_kernel(const BatchArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_box, s_pass, s_tile, s_count, s_nbox, s_npass, s_ntile;
    const int tid = threadIdx.x;
    int next = 0, end = 0;           // thread 0: taken items not yet run
    // thread 0: the claim after [next, end), taken one claim ahead so that
    // its queue round trip overlaps the current run (-1: none yet)
    int pre_lo = -1, pre_n = 0;
    int ok_box = -1, ok_pass = -1;   // thread 0: last dependency seen complete
    int pend_box = 0, pend_pass = 0, pend = 0;  // thread 0: finished, unpublished tiles
    auto publish = [&]() {
        if (pend) {
            __threadfence();
            atomicAdd(a.done + 3 * pend_box + pend_pass, pend);
            pend = 0;
        }
    };
    for (;;) {
        if (tid == 0) {
            int count = -1, box = 0, pass = 0, tile = 0, nbox = -1, npass = 0, ntile = 0;
            // guided claims: up to `claim` items, fewer as the queue drains,
            // so the last runs end close together; the items left are
            // estimated from the queue position this CTA last saw (no read
            // of the counter, whose round trip would not overlap anything)
            auto claim = [&](int seen, int& lo, int& n) {
                const int left = a.item_hi - seen;
                n = max(1, min(a.claim, left / (2 * (int)gridDim.x)));
                lo = a.item_lo + atomicAdd(a.taken, n);
            };
            if (next >= end) {
                if (a.fused) publish();
                if (pre_lo < 0) claim(a.item_lo, pre_lo, pre_n);  // first claim of this CTA
                next = pre_lo;
                end = pre_lo + pre_n;
                // the following claim: its result is not read before this
                // claim's items have run
                if (next < a.item_hi) claim(end, pre_lo, pre_n);
                else pre_lo = a.item_hi;
            }
            const int i = next;
            if (i < a.item_hi && !*reinterpret_cast<volatile int*>(a.abort)) {
                const int2 it = a.items[i];
                box = it.x >> 2;
                pass = it.x & 3;
                tile = it.y;
                // the run: taken items of the same (box, pass), whose tiles
                // are consecutive in the item list
                const int stop = min(min(end, a.item_hi), i - tile + a.boxes[box].tiles[pass]);
                count = stop - i;
                next = stop;
                if (a.prefetch && next < end && next < a.item_hi) {
                    const int2 nt = a.items[next];
                    nbox = nt.x >> 2;
                    npass = nt.x & 3;
                    ntile = nt.y;
                }
                if (a.fused && pass > 0 && (box != ok_box || pass != ok_pass)) {
                    publish();
                    if (wait_count(a.done + 3 * box + pass - 1, a.boxes[box].tiles[pass - 1] + a.wait_extra,
                                   a.abort)) {
                        __threadfence();
                        ok_box = box;
                        ok_pass = pass;
                    } else {
                        atomicExch(a.err, 1);
                        atomicExch(a.abort, 1);
                        count = -1;
                    }
                }
            }
            if (count < 0 && a.fused) publish();
            s_count = count;
            s_box = box;
            s_pass = pass;
            s_tile = tile;
            s_nbox = nbox;
            s_npass = npass;
            s_ntile = ntile;
        }
        __syncthreads();
        const int count = s_count;
        if (count < 0) break;
        const int box = s_box, pass = s_pass, tile = s_tile;
        if (s_nbox >= 0) prefetch_tile<T>(a.boxes[s_nbox], s_npass, s_ntile, tid);
        {
            const BatchBox& bx = a.boxes[box];
            // pass 0 = Z (lines (x, y)), 1 = X (lines (y, z)), 2 = Y (lines (x, z))
            const int ax = pass == 0 ? 2 : pass == 1 ? 0 : 1;
            const int au = pass == 1 ? 1 : 0;
            const int av = pass == 0 ? 1 : 2;
            cx<T>* data = static_cast<cx<T>*>(bx.data);
            const T scale = (INV && pass == 2) ? T(bx.inv_scale) : T(1);
            const int mode = pass == 0 ? MODE_LINE : MODE_BATCH;
            const int var = bx.var[pass];
            const cx<T>* tw = static_cast<const cx<T>*>(bx.tw[ax]);
            switch (bx.n[ax]) {
#define A2A_BATCH_CASE(N_)                                                                                         \
    case N_:                                                                                                       \
        batch_len<T, INV, N_>(data, bx.off[ax], bx.off[au], bx.off[av], tw, bx.n[au], bx.n[av], scale,             \
                              bx.split[pass], mode, var, tile, count, smem, tid);                                  \
        break;
                A2A_BATCH_FOR_EACH_N(A2A_BATCH_CASE)
#undef A2A_BATCH_CASE
                default:
                    break;
            }
        }
        __syncthreads();
        if (tid == 0 && a.fused) {
            if (pend && (box != pend_box || pass != pend_pass)) publish();
            pend_box = box;
            pend_pass = pass;
            pend += count;
        }
    }
}

// Largest dynamic shared memory any tile of the batched kernel uses.
template <typename T> __host__ __device__ constexpr size_t batch_smem_bytes() {
    size_t m = 0;
#define A2A_BATCH_SMEM(N_)                                                                                    \
    {                                                                                                         \
        using P = typename PassPlan<T, N_>::Plan;                                                             \
        const size_t v[5] = {                                                                                 \
            pass_smem_bytes<T, P, batch_lines<T>(N_, 0), MODE_LINE, KIND_DIRECT, 1>(),                        \
            pass_smem_bytes<T, P, batch_lines<T>(N_, 0), MODE_BATCH, KIND_DIRECT, 1>(),                       \
            pass_smem_bytes<T, P, batch_lines<T>(N_, 1), MODE_LINE, KIND_DIRECT, 1>(),                        \
            pass_smem_bytes<T, P, batch_lines<T>(N_, 1), MODE_BATCH, KIND_DIRECT, 1>(),                       \
            pass_smem_bytes<T, P, batch_lines<T>(N_, 2), MODE_BATCH, KIND_DIRECT, batch_lpt<T>(2, MODE_BATCH)>()}; \
        for (size_t x : v) m = x > m ? x : m;                                                                 \
    }
    A2A_BATCH_FOR_EACH_N(A2A_BATCH_SMEM)
#undef A2A_BATCH_SMEM
    return m;
}

}  // namespace a2a
