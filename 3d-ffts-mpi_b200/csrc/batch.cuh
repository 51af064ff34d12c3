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
// two choices per length for the plan's tuner; complex double uses half the
// lines of complex float (same registers per thread).
__host__ __device__ constexpr int batch_lines_f32(int n, int v) {
    return (n == 48 || n == 256 || n == 512) ? (v ? 8 : 16) : (v ? 16 : 32);
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
    int tiles[3];            // tiles per pass
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
    int claim;               // items a CTA takes per queue access
    int fused;               // 1: later passes wait for the earlier pass of their box
    int wait_extra;          // 0; > 0 makes every wait unsatisfiable (tests of the timeout path)
    int* taken;              // items taken so far
    int* abort;              // raised when a wait gave up: every CTA stops
    int* done;               // tiles finished per (box, pass), 3 ints per box
    int* err;                // set to 1 when a wait gave up (not cleared by launches)
};

// One tile of one configuration, compiled as its own function so that each
// configuration gets its own register allocation (inlined into one body they
// would share the worst case and spill).
template <typename T, bool INV, int N, int V, int MODE>
__device__ __noinline__ void batch_tile(cx<T>* data, const uint32_t* offA, const uint32_t* offU, const uint32_t* offV,
                                        const cx<T>* tw, int NU, int NV, T scale, int split, int tile,
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
    direct_tile<T, P, batch_lines<T>(N, V), kBatchThreads, MODE, INV, 1, true>(pa, tile, smem, tid);
}

template <typename T, bool INV, int N>
__device__ __forceinline__ void batch_len(cx<T>* data, const uint32_t* offA, const uint32_t* offU,
                                          const uint32_t* offV, const cx<T>* tw, int NU, int NV, T scale, int split,
                                          int mode, int var, int tile, unsigned char* smem, int tid) {
#define A2A_BT(V_, M_) batch_tile<T, INV, N, V_, M_>(data, offA, offU, offV, tw, NU, NV, scale, split, tile, smem, tid)
    if (mode == MODE_LINE) {
        if (var == 0) A2A_BT(0, MODE_LINE); else A2A_BT(1, MODE_LINE);
    } else {
        if (var == 0) A2A_BT(0, MODE_BATCH); else A2A_BT(1, MODE_BATCH);
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

// The persistent kernel.  Thread 0 takes `claim` consecutive items per queue
// access and, in the fused schedule, checks an item's dependency (every tile
// of the previous pass of its box done) once per (box, pass) change, with an
// acquire fence after the wait; a finished tile is published by a release
// (fence, then the counter increment) after the CTA barrier.  An item waits
// only on items taken before it, so the lowest unfinished taken item always
// runs and the waits end.
template <typename T, bool INV>
__global__ void __launch_bounds__(kBatchThreads, 2) fft_batch_kernel(const BatchArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_box, s_pass, s_tile, s_go;
    const int tid = threadIdx.x;
    int next = 0, held = 0;          // thread 0: taken items not yet run
    int ok_box = -1, ok_pass = -1;   // thread 0: last dependency seen complete
    for (;;) {
        if (tid == 0) {
            int go = -1, box = 0, pass = 0, tile = 0;
            if (held == 0) {
                next = a.item_lo + atomicAdd(a.taken, a.claim);
                held = a.claim;
            }
            const int i = next++;
            --held;
            if (i < a.item_hi && !*reinterpret_cast<volatile int*>(a.abort)) {
                const int2 it = a.items[i];
                box = it.x >> 2;
                pass = it.x & 3;
                tile = it.y;
                go = 1;
                if (a.fused && pass > 0 && (box != ok_box || pass != ok_pass)) {
                    if (wait_count(a.done + 3 * box + pass - 1, a.boxes[box].tiles[pass - 1] + a.wait_extra,
                                   a.abort)) {
                        __threadfence();
                        ok_box = box;
                        ok_pass = pass;
                    } else {
                        atomicExch(a.err, 1);
                        atomicExch(a.abort, 1);
                        go = -1;
                    }
                }
            }
            s_go = go;
            s_box = box;
            s_pass = pass;
            s_tile = tile;
        }
        __syncthreads();
        if (s_go < 0) break;
        const int box = s_box, pass = s_pass, tile = s_tile;
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
                              bx.split[pass], mode, var, tile, smem, tid);                                         \
        break;
                A2A_BATCH_FOR_EACH_N(A2A_BATCH_CASE)
#undef A2A_BATCH_CASE
                default:
                    break;
            }
        }
        __syncthreads();
        if (tid == 0 && a.fused) {
            __threadfence();
            atomicAdd(a.done + 3 * box + pass, 1);
        }
    }
}

// Largest dynamic shared memory any tile of the batched kernel uses.
template <typename T> __host__ __device__ constexpr size_t batch_smem_bytes() {
    size_t m = 0;
#define A2A_BATCH_SMEM(N_)                                                                                    \
    {                                                                                                         \
        using P = typename PassPlan<T, N_>::Plan;                                                             \
        const size_t v[4] = {pass_smem_bytes<T, P, batch_lines<T>(N_, 0), MODE_LINE, KIND_DIRECT, 1>(),       \
                             pass_smem_bytes<T, P, batch_lines<T>(N_, 0), MODE_BATCH, KIND_DIRECT, 1>(),      \
                             pass_smem_bytes<T, P, batch_lines<T>(N_, 1), MODE_LINE, KIND_DIRECT, 1>(),       \
                             pass_smem_bytes<T, P, batch_lines<T>(N_, 1), MODE_BATCH, KIND_DIRECT, 1>()};     \
        for (size_t x : v) m = x > m ? x : m;                                                                 \
    }
    A2A_BATCH_FOR_EACH_N(A2A_BATCH_SMEM)
#undef A2A_BATCH_SMEM
    return m;
}

}  // namespace a2a
