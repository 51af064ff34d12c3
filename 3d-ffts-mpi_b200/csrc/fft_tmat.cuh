// Axis pass with whole tiles fetched by TMA tensor copies (KIND_TMAT2/3).
//
// The rank-major brick buffer is, seen from one z brick index zr, a 5-D
// array of 8-byte words  [x_r][y_r][x_l][y_l][z_l]  (dims d0, d1, lx, ly,
// w*lz; w = 1 word per complex float, 2 per complex double) with strides
// (d1 d2 nl, d2 nl, ly lz, lz, 1) elements, starting at zr * nl.  One tensor
// map per zr describes it; a tile of B lines is then one box (X and Y
// passes) or one box per z brick (Z pass):
//
//   Z pass, lines (x, y = v0..v0+B-1): per zr a box [lz, B, 1, 1, 1] at
//           (0, y_l, x_l, y_r, x_r)  -> shared [zr][b][z_l]
//   X pass, lines (y, z = v0..v0+B-1): box [B, 1, lx, 1, d0] at
//           (z_l, y_l, 0, y_r, 0) of map z_r -> shared [x][b]
//   Y pass, lines (x, z = v0..v0+B-1): box [B, ly, 1, d1, 1] at
//           (z_l, 0, x_l, 0, x_r) of map z_r -> shared [y][b]
//
// (a box edge above 256 words is cut into chunks along that axis).  A
// persistent CTA keeps NSTG tiles in flight in a ring of shared-memory slots,
// each completing on its own mbarrier; stage 0 reads its slot into
// registers and writes the Stockham tile (BATCH rows narrower than a bank
// row are swizzled, see TileGeom), which frees the slot for the tile NSTG
// ahead while stages 1..S-1 run.  Every copy is a plain single-CTA tensor copy.
#pragma once

#include <cuda.h>

#include "fft_tile.cuh"

namespace a2a {

constexpr int kTmatMaxMaps = 8;
constexpr uint32_t kTmatAlign = 1024;

// Kernel parameter: the tensor maps of one pass and the tile geometry.
struct TmatMaps {
    CUtensorMap map[kTmatMaxMaps];  // one per z brick index
    int pass;                       // 0 = Z, 1 = X, 2 = Y
    int lx, ly, lz;                 // brick extents (elements)
    int words;                      // 8-byte words per complex element
    int chunk;                      // box edge (elements) along the cut axis
    int chunk_shift;                // log2(chunk) when chunk is a power of two, else -1
    int nchunk;                     // boxes per z brick (Z) or per tile (X, Y)
    int nmaps;                      // d2
};

template <typename T, int B, int N> __host__ __device__ constexpr uint32_t tmat_slot_bytes() {
    return (uint32_t)((B * N * sizeof(cx<T>) + kTmatAlign - 1) / kTmatAlign * kTmatAlign);
}

// In-place rings (INPLACE): each slot also serves as its tile's Stockham tile,
// so a slot holds the larger of the copy and the (padded) tile.
template <typename T, class PLAN, int B, int MODE, int LPT, bool INPLACE>
__host__ __device__ constexpr uint32_t tmat_slot_bytes_for() {
    using E = typename ElemOf<T, LPT>::type;
    constexpr size_t tile = sizeof(E) * (size_t)TileGeom<MODE, B / LPT, PLAN::N, sizeof(E)>::elems;
    constexpr uint32_t copy = tmat_slot_bytes<T, B, PLAN::N>();
    constexpr uint32_t t = (uint32_t)((tile + kTmatAlign - 1) / kTmatAlign * kTmatAlign);
    return INPLACE && t > copy ? t : copy;
}

template <typename T, class PLAN, int B, int MODE, int LPT, int NSTG, bool INPLACE = false>
__host__ __device__ constexpr size_t tmat_smem_bytes() {
    using E = typename ElemOf<T, LPT>::type;
    constexpr int N = PLAN::N;
    constexpr int BV = B / LPT;
    size_t bytes = kTmatAlign;  // room to align the ring
    bytes += (size_t)NSTG * tmat_slot_bytes_for<T, PLAN, B, MODE, LPT, INPLACE>();
    if (!INPLACE) bytes += sizeof(E) * (size_t)TileGeom<MODE, BV, N, sizeof(E)>::elems;
    bytes += sizeof(cx<T>) * (size_t)PLAN::twtotal();
    bytes += sizeof(uint32_t) * (size_t)N;
    bytes = (bytes + 15) & ~size_t(15);
    bytes += sizeof(size_t) * (size_t)BV;
    bytes += sizeof(unsigned long long) * NSTG;
    return bytes;
}

__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                            unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}

// Thread 0: arm the slot's mbarrier for one tile and issue its boxes.
template <typename T, int B, int N>
__device__ __forceinline__ void tmat_issue(const TmatMaps& m, int t, int tilesV, unsigned char* dst,
                                           unsigned long long* bar) {
    constexpr uint32_t bytes = (uint32_t)(B * N * sizeof(cx<T>));
    const int u = t / tilesV;
    const int v0 = (t - u * tilesV) * B;
    const uint32_t cbytes = (uint32_t)(B * m.chunk * sizeof(cx<T>));
    mbar_arrive_expect_tx(bar, bytes);
    if (m.pass == 0) {  // lines (x = u, y = v0 ..)
        const int xl = u % m.lx, xr = u / m.lx, yl = v0 % m.ly, yr = v0 / m.ly;
        unsigned char* p = dst;
        for (int zr = 0; zr < m.nmaps; ++zr)
            for (int c = 0; c < m.nchunk; ++c, p += cbytes)
                tma_load_5d(p, &m.map[zr], m.words * c * m.chunk, yl, xl, yr, xr, bar);
    } else if (m.pass == 1) {  // lines (y = u, z = v0 ..)
        const int zl = v0 % m.lz, zr = v0 / m.lz, yl = u % m.ly, yr = u / m.ly;
        for (int c = 0; c < m.nchunk; ++c)
            tma_load_5d(dst + c * cbytes, &m.map[zr], m.words * zl, yl, c * m.chunk, yr, 0, bar);
    } else {  // lines (x = u, z = v0 ..)
        const int zl = v0 % m.lz, zr = v0 / m.lz, xl = u % m.lx, xr = u / m.lx;
        for (int c = 0; c < m.nchunk; ++c)
            tma_load_5d(dst + c * cbytes, &m.map[zr], m.words * zl, c * m.chunk, xl, 0, xr, bar);
    }
}

// INPLACE: every slot is its tile's Stockham tile; a slot is refilled (with
// the tile NSTG ahead) once its tile is done -- less shared memory per CTA
// (more CTAs per SM) for a shorter prefetch distance.
template <typename T, class PLAN, int B, int THREADS, int MODE, bool INV, int MINB, int LPT, int NSTG,
          bool INPLACE = false>
__global__ void __launch_bounds__(THREADS, MINB) fft_tmat_kernel(const PassArgs<T> a, const __grid_constant__ TmatMaps m) {
    using E = typename ElemOf<T, LPT>::type;
    constexpr int BV = B / LPT;
    constexpr int SWSH = MODE == MODE_BATCH ? tile_swizzle_shift<PLAN, BV, (int)sizeof(E)>() : -1;
    using G = TileGeom<MODE, BV, PLAN::N, sizeof(E), SWSH>;
    constexpr int N = PLAN::N;
    constexpr int R0 = PLAN::r[0];
    constexpr int NBL = N / R0;
    constexpr int NBT = BV * NBL;
    constexpr int K = (NBT + THREADS - 1) / THREADS;
    constexpr bool EXACT = (NBT % THREADS) == 0;
    constexpr int TWN = PLAN::twtotal();
    constexpr bool BFAST0 = (MODE == MODE_BATCH);
    constexpr uint32_t SLOT = tmat_slot_bytes_for<T, PLAN, B, MODE, LPT, INPLACE>();
    static_assert(PLAN::S >= 2, "the ring kernel needs at least two stages");
    static_assert(MODE != MODE_BATCH || THREADS % BV == 0, "batch mode needs THREADS % (B/LPT) == 0");
    static_assert(LPT == 1 || MODE == MODE_BATCH, "line pairs only in batch mode");
    static_assert(NSTG >= 2, "the ring needs at least two slots");

    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t s0 = smem_u32(smem_raw);
    unsigned char* ring = smem_raw + (((s0 + kTmatAlign - 1) & ~(kTmatAlign - 1)) - s0);
    E* const xtile = reinterpret_cast<E*>(ring + NSTG * SLOT);  // separate tile (not INPLACE)
    cx<T>* tw = reinterpret_cast<cx<T>*>(INPLACE ? ring + NSTG * SLOT : reinterpret_cast<unsigned char*>(xtile + G::elems));
    uint32_t* offA_s = reinterpret_cast<uint32_t*>(tw + TWN);
    size_t* base_s = reinterpret_cast<size_t*>(
        reinterpret_cast<unsigned char*>(tw) + ((sizeof(cx<T>) * TWN + sizeof(uint32_t) * N + 15) & ~size_t(15)));
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(base_s + BV);

    const int tid = threadIdx.x;
    const int tilesV = a.NV / B;
    const int ntiles = a.NU * tilesV;
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
            tmat_issue<T, B, N>(m, blockIdx.x + issued * gridDim.x, tilesV, ring + issued * SLOT, bar + issued);

    for (int i = 0; i < mine; ++i) {
        const int t = blockIdx.x + i * gridDim.x;
        const int s = i % NSTG;
        {
            const int u = t / tilesV;
            const int v0 = (t - u * tilesV) * B;
            const size_t ubase = __ldg(a.offU + u);
            for (int b = tid; b < BV; b += THREADS) base_s[b] = ubase + __ldg(a.offV + v0 + b * LPT);
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
        // stage 0 from the ring slot
        const E* src = reinterpret_cast<const E*>(ring + s * SLOT);
        E* tile = INPLACE ? reinterpret_cast<E*>(ring + s * SLOT) : xtile;
        E x[K][R0];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int q = tid + k * THREADS;
            if (EXACT || q < NBT) {
                int b, j;
                bf_map<BFAST0, BV, NBL>(q, b, j);
#pragma unroll
                for (int r = 0; r < R0; ++r) {
                    const int n = j + r * NBL;
                    if constexpr (MODE == MODE_BATCH) {
                        x[k][r] = src[n * BV + b];
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
        if constexpr (INPLACE) __syncthreads();  // every read of the slot before it is rewritten
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
        __syncthreads();  // slot s read out; the tile and its line bases are ready
        if (!INPLACE && tid == 0 && issued < mine) {
            fence_proxy_async_smem();  // the generic reads of slot s come before the async writes
            tmat_issue<T, B, N>(m, blockIdx.x + issued * gridDim.x, tilesV, ring + s * SLOT, bar + s);
            ++issued;
        }
        run_stage<T, PLAN, B, THREADS, MODE, INV, LPT, 1, SWSH>(a, tile, tw, offA_s, base_s, tid);
        __syncthreads();  // tile and line bases free for the next tile
        if (INPLACE && tid == 0 && issued < mine) {  // the slot's tile is done: refill it
            fence_proxy_async_smem();
            tmat_issue<T, B, N>(m, blockIdx.x + issued * gridDim.x, tilesV, ring + s * SLOT, bar + s);
            ++issued;
        }
    }
}

// KIND_TMAT2S: the 2-slot ring for batch-mode tiles of complex float (128
// threads) whose first two stages exchange through warp shuffles instead of
// shared memory.  Plans R0 x R1 x R2 with R0 R1 = 64; registered for 512 =
// 8 x 8 x 8 (8-line tiles).  (1024 = 4 x 16 x 16 would take 4-line tiles,
// 32-byte rows; measured at 1024^3 it ran the X pass in 9.0 ms against 3.4 ms
// for the wide-radix ring, so it is not registered.)
//
// Stage 0's radix-R0 butterfly j writes positions R0 j + r, and stage 1's
// radix-R1 butterfly j' reads j' + (N / R1) r'': so with NG = N / 64 the R1
// stage-0 butterflies {a + NG r''} of a line feed exactly the R0 stage-1
// butterflies {R0 a + r} (a = 0 .. NG-1), a closed 64-element exchange.  Each
// such group of a line belongs to one pair of lanes (lane = b + B (a mod
// 16/B) + 16 h, partner lane ^ 16): lane h runs stage-0 butterflies
// a + NG (R1/2 h + t) and stage-1 butterflies R0 a + R0/2 h + u
// (t < R1/2, u < R0/2), keeps the half of its outputs its own stage-1
// butterflies need and trades the other half with its partner (16 complex
// values each way).  So that every register has the same role in both lanes
// (no per-lane selects), lane h = 1 runs its stage-0 DFTs on inputs times
// (-1)^n, which rotates the outputs by R0/2 (X[k ^ R0/2]), and its stage-1
// DFTs on inputs held in the order rotated by R1/2, which multiplies output k
// by (-1)^k.  Stage 1 then writes the Stockham tile and the last stage is the
// shared-memory stage of the other ring kernels.  The tile's row swizzle
// uses row bits 6 and up (rows 64 apart, which stage 1's half-warps write
// together, land in different bank slots).  Shared-memory traffic per
// element: the slot read, one tile write and one tile read, against five
// accesses in the three-exchange schedule.
constexpr int kShflSwsh = 6;

template <class PLAN> struct ShflGeom {
    static constexpr int N = PLAN::N;
    static constexpr int R0 = PLAN::r[0];
    static constexpr int R1 = PLAN::r[1];
    static_assert(PLAN::S == 3 && R0 * R1 == 64, "the shuffle exchange pairs 64-element groups");
    static constexpr int NG = N / 64;      // groups per line
    static constexpr int B = 64 / NG;      // lines per tile (128 threads = 64 lane pairs)
    static_assert(B >= 2 && B <= 16 && 16 % B == 0, "a half-warp spans whole groups of lines");
    static constexpr int H0 = R1 / 2;      // stage-0 butterflies per lane
    static constexpr int H1 = R0 / 2;      // stage-1 butterflies per lane
};

template <class PLAN, bool INV, int MINB>
__global__ void __launch_bounds__(128, MINB) fft_tmat_shfl_kernel(const PassArgs<float> a,
                                                                   const __grid_constant__ TmatMaps m) {
    using SG = ShflGeom<PLAN>;
    constexpr int N = SG::N, R0 = SG::R0, R1 = SG::R1, B = SG::B, H0 = SG::H0, H1 = SG::H1;
    constexpr int THREADS = 128, NSTG = 2;
    using G = TileGeom<MODE_BATCH, B, N, sizeof(float2), kShflSwsh>;
    constexpr int TWN = PLAN::twtotal();
    constexpr int TWO1 = PLAN::twoff(1);
    constexpr int NS1 = PLAN::ns(1);  // = R0
    constexpr uint32_t SLOT = tmat_slot_bytes_for<float, PLAN, B, MODE_BATCH, 1, false>();

    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t s0 = smem_u32(smem_raw);
    unsigned char* ring = smem_raw + (((s0 + kTmatAlign - 1) & ~(kTmatAlign - 1)) - s0);
    float2* const tile = reinterpret_cast<float2*>(ring + NSTG * SLOT);
    float2* tw = reinterpret_cast<float2*>(tile + G::elems);
    uint32_t* offA_s = reinterpret_cast<uint32_t*>(tw + TWN);
    size_t* base_s = reinterpret_cast<size_t*>(
        reinterpret_cast<unsigned char*>(tw) + ((sizeof(float2) * TWN + sizeof(uint32_t) * N + 15) & ~size_t(15)));
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(base_s + B);

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int b = lane % B;                                        // line of the tile
    const int ga = (tid >> 5) * (16 / B) + (lane / B) % (16 / B);  // group a = 0 .. NG-1
    const int h = lane >> 4;                                       // half of the pair
    const float sgn = h ? -1.f : 1.f;
    const int tilesV = a.NV / B;
    const int ntiles = a.NU * tilesV;
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
            tmat_issue<float, B, N>(m, blockIdx.x + issued * gridDim.x, tilesV, ring + issued * SLOT, bar + issued);

    for (int i = 0; i < mine; ++i) {
        const int t = blockIdx.x + i * gridDim.x;
        const int s = i % NSTG;
        {
            const int u = t / tilesV;
            const int v0 = (t - u * tilesV) * B;
            const size_t ubase = __ldg(a.offU + u);
            for (int bb = tid; bb < B; bb += THREADS) base_s[bb] = ubase + __ldg(a.offV + v0 + bb);
        }
        const bool ok = mbar_wait_bounded(bar + s, (uint32_t)((i / NSTG) & 1));
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicExch(a.err, 1);
                for (int j = i; j < issued; ++j) mbar_wait_bounded(bar + j % NSTG, (uint32_t)((j / NSTG) & 1));
            }
            return;
        }
        const float2* src = reinterpret_cast<const float2*>(ring + s * SLOT);
        // stage 0: butterflies j = a + NG (H0 h + tt), inputs n = j + (N/R0) r
        float2 y[H0][R0];
#pragma unroll
        for (int tt = 0; tt < H0; ++tt) {
            const int j = ga + SG::NG * (H0 * h + tt);
#pragma unroll
            for (int r = 0; r < R0; ++r) {
                const float2 v = src[(j + (N / R0) * r) * B + b];
                y[tt][r] = (r & 1) ? make_float2(v.x * sgn, v.y * sgn) : v;
            }
            Dft<R0, INV, float2>::run(y[tt]);  // register k holds output k ^ (R0/2) h
        }
        // exchange: keep registers 0 .. H1-1 (outputs H1 h + u), trade the
        // others (outputs H1 (1-h) + u, the partner's stage-1 butterflies)
        float2 x[H1][R1];
#pragma unroll
        for (int u = 0; u < H1; ++u)
#pragma unroll
            for (int tt = 0; tt < H0; ++tt) {
                x[u][tt] = y[tt][u];
                x[u][H0 + tt].x = __shfl_xor_sync(0xffffffffu, y[tt][H1 + u].x, 16);
                x[u][H0 + tt].y = __shfl_xor_sync(0xffffffffu, y[tt][H1 + u].y, 16);
            }
        __syncthreads();  // slot s read out
        if (tid == 0 && issued < mine) {
            fence_proxy_async_smem();  // the generic reads of slot s come before the async writes
            tmat_issue<float, B, N>(m, blockIdx.x + issued * gridDim.x, tilesV, ring + s * SLOT, bar + s);
            ++issued;
        }
        // stage 1: butterfly j' = R0 a + H1 h + u; register rho holds input
        // r'' = rho ^ H0 h; twiddle index j' mod R0 = H1 h + u
#pragma unroll
        for (int u = 0; u < H1; ++u) {
            const int mm = H1 * h + u;
#pragma unroll
            for (int rho = 0; rho < R1; ++rho) {
                const int rr = rho ^ (H0 * h);
                if (rho == 0 || rho == H0) {
                    if (rr != 0) x[u][rho] = cmulw<INV>(x[u][rho], tw[TWO1 + (rr - 1) * NS1 + mm]);
                } else {
                    x[u][rho] = cmulw<INV>(x[u][rho], tw[TWO1 + (rr - 1) * NS1 + mm]);
                }
            }
            Dft<R1, INV, float2>::run(x[u]);  // output k times (-1)^k for h = 1
            const int jd = 64 * ga + mm;
#pragma unroll
            for (int k = 0; k < R1; ++k) {
                const float2 v = (k & 1) ? make_float2(x[u][k].x * sgn, x[u][k].y * sgn) : x[u][k];
                tile[G::idx(b, jd + NS1 * k)] = v;
            }
        }
        __syncthreads();  // the tile is written
        run_stage<float, PLAN, B, THREADS, MODE_BATCH, INV, 1, 2, kShflSwsh>(a, tile, tw, offA_s, base_s, tid);
        __syncthreads();  // tile and line bases free for the next tile
    }
}

// KIND_RPIPES: the same shuffle exchange for line-mode tiles (the Z pass),
// fed by the register-pipelined persistent loop of fft_rpipe_kernel instead
// of the ring: stage 0's inputs come straight from global memory into the
// lanes' registers (lane = a mod 8 + 8 (line mod 2) + 16 h, so a half-warp
// reads 8 consecutive elements of each of two lines), and once stage 1 has
// written the tile the same registers receive the next tile's loads, which
// stay in flight through the last stage.
template <class PLAN, bool INV, int MINB>
__global__ void __launch_bounds__(128, MINB) fft_rpipe_shfl_kernel(const PassArgs<float> a) {
    using SG = ShflGeom<PLAN>;
    constexpr int N = SG::N, R0 = SG::R0, R1 = SG::R1, B = SG::B, H0 = SG::H0, H1 = SG::H1, NG = SG::NG;
    static_assert(NG == 8 && B == 8, "line-mode pairing laid out for 8 groups of 8 lines");
    constexpr int THREADS = 128;
    using G = TileGeom<MODE_LINE, B, N, sizeof(float2)>;
    constexpr int TWN = PLAN::twtotal();
    constexpr int TWO1 = PLAN::twoff(1);
    constexpr int NS1 = PLAN::ns(1);

    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* tile = reinterpret_cast<float2*>(smem_raw);
    float2* tw = reinterpret_cast<float2*>(tile + G::elems);
    uint32_t* offA_s = reinterpret_cast<uint32_t*>(tw + TWN);
    size_t* base_s = reinterpret_cast<size_t*>(
        smem_raw + ((sizeof(float2) * (size_t)G::elems + sizeof(float2) * TWN + sizeof(uint32_t) * N + 15) & ~size_t(15)));

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int ga = lane & 7;                            // group a
    const int b = 2 * (tid >> 5) + ((lane >> 3) & 1);   // line of the tile
    const int h = lane >> 4;                            // half of the pair
    const float sgn = h ? -1.f : 1.f;
    const int tilesV = a.NV / B;
    const int ntiles = a.NU * tilesV;
    uint32_t d0[R0];
    if (a.split) {
#pragma unroll
        for (int r = 0; r < R0; ++r) d0[r] = __ldg(a.offA + r * (N / R0));
    }
    // stage 0's inputs of tile t: butterflies j = a + NG (H0 h + tt), inputs
    // n = j + (N/R0) r of this lane's line
    auto load_tile = [&](int t, float2 (&y)[H0][R0]) {
        const int u = t / tilesV;
        const int v0 = (t - u * tilesV) * B;
        const float2* line = a.src + (size_t)__ldg(a.offU + u) + __ldg(a.offV + v0 + b);
#pragma unroll
        for (int tt = 0; tt < H0; ++tt) {
            const int j = ga + NG * (H0 * h + tt);
            if (a.split) {
                const float2* q = line + __ldg(a.offA + j);
#pragma unroll
                for (int r = 0; r < R0; ++r) y[tt][r] = ld_stream(q + d0[r]);
            } else {
#pragma unroll
                for (int r = 0; r < R0; ++r) y[tt][r] = ld_stream(line + __ldg(a.offA + j + (N / R0) * r));
            }
        }
    };
    int t = blockIdx.x;
    float2 y[H0][R0];
    if (t < ntiles) load_tile(t, y);
    for (int i = tid; i < TWN; i += THREADS) tw[i] = a.tw[i];
    for (int i = tid; i < N; i += THREADS) offA_s[i] = a.offA[i];
    for (; t < ntiles; t += gridDim.x) {
        {
            const int u = t / tilesV;
            const int v0 = (t - u * tilesV) * B;
            const size_t ubase = __ldg(a.offU + u);
            for (int bb = tid; bb < B; bb += THREADS) base_s[bb] = ubase + __ldg(a.offV + v0 + bb);
        }
        // stage 0 (register k of lane h = 1 holds output k ^ R0/2)
#pragma unroll
        for (int tt = 0; tt < H0; ++tt) {
#pragma unroll
            for (int r = 1; r < R0; r += 2) y[tt][r] = make_float2(y[tt][r].x * sgn, y[tt][r].y * sgn);
            Dft<R0, INV, float2>::run(y[tt]);
        }
        float2 x[H1][R1];
#pragma unroll
        for (int u = 0; u < H1; ++u)
#pragma unroll
            for (int tt = 0; tt < H0; ++tt) {
                x[u][tt] = y[tt][u];
                x[u][H0 + tt].x = __shfl_xor_sync(0xffffffffu, y[tt][H1 + u].x, 16);
                x[u][H0 + tt].y = __shfl_xor_sync(0xffffffffu, y[tt][H1 + u].y, 16);
            }
        // stage 1 (register rho holds input rho ^ H0 h; output k times (-1)^k for h = 1)
#pragma unroll
        for (int u = 0; u < H1; ++u) {
            const int mm = H1 * h + u;
#pragma unroll
            for (int rho = 0; rho < R1; ++rho) {
                const int rr = rho ^ (H0 * h);
                if (rho == 0 || rho == H0) {
                    if (rr != 0) x[u][rho] = cmulw<INV>(x[u][rho], tw[TWO1 + (rr - 1) * NS1 + mm]);
                } else {
                    x[u][rho] = cmulw<INV>(x[u][rho], tw[TWO1 + (rr - 1) * NS1 + mm]);
                }
            }
            Dft<R1, INV, float2>::run(x[u]);
            const int jd = 64 * ga + mm;
#pragma unroll
            for (int k = 0; k < R1; ++k) {
                const float2 v = (k & 1) ? make_float2(x[u][k].x * sgn, x[u][k].y * sgn) : x[u][k];
                tile[G::idx(b, jd + NS1 * k)] = v;
            }
        }
        const int tn = t + gridDim.x;
        if (tn < ntiles) load_tile(tn, y);  // in flight through the last stage
        __syncthreads();
        run_stage<float, PLAN, B, THREADS, MODE_LINE, INV, 1, 2>(a, tile, tw, offA_s, base_s, tid);
        __syncthreads();  // tile and line bases free for the next tile
    }
}

}  // namespace a2a
