// Batched 1D FFT tile engine for sm_100a: Stockham auto-sort, mixed radix
// 2/3/4/8/16, one tile of B lines of length N per CTA, staged through shared
// memory, global traffic fused with the pencil gather/scatter.
//
// This replaces the batched cuFFT calls of the reference
// (src/a2afft/dfft/kernels/a2affts.cu:7-76, cufftPlan1d + cufftExecZ2Z/C2C on
// nlocal/Ng contiguous pencils) AND the pack/unpack remaps around them
// (src/a2afft/distribution/kernels/a2apencils.cu): a line's element n lives at
// `base[line] + offA[n]`, where the tables encode the alltoall + unpack
// composite for the virtual-rank brick layout, so the gather happens inside
// the first stage's loads and the scatter inside the last stage's stores.
//
// Stockham stage s (radix R, Ns = product of the radices before s):
//   butterfly j in [0, N/R):  x_r = in[j + r N/R] * W_{Ns R}^{r (j mod Ns)}
//                             y   = DFT_R(x)
//                             out[(j/Ns) Ns R + (j mod Ns) + r Ns] = y_r
// Stage 0 has no twiddles and reads global memory straight into registers;
// the last stage (Ns R = N) writes global memory straight from registers.
// Shared memory holds one tile, updated in place (every thread reads its
// butterfly inputs, the block synchronises, then writes).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "remap.cuh"

namespace a2a {

// --------------------------------------------------------------------------
// complex helpers
// --------------------------------------------------------------------------
template <typename T> struct CxOf;
template <> struct CxOf<float> { using type = float2; };
template <> struct CxOf<double> { using type = double2; };
template <typename T> using cx = typename CxOf<T>::type;

template <typename V> struct RealOf;
template <> struct RealOf<float2> { using type = float; };
template <> struct RealOf<double2> { using type = double; };
// float4 = the same element of two adjacent lines (complex float each); the
// batch passes move line pairs with 16-byte accesses
template <> struct RealOf<float4> { using type = float; };

template <typename V>
__host__ __device__ __forceinline__ V mk(typename RealOf<V>::type re, typename RealOf<V>::type im) {
    static_assert(sizeof(V) == 2 * sizeof(typename RealOf<V>::type), "mk builds one complex value");
    V v;
    v.x = re;
    v.y = im;
    return v;
}
template <typename V> __device__ __forceinline__ V add(V a, V b) { return mk<V>(a.x + b.x, a.y + b.y); }
template <typename V> __device__ __forceinline__ V sub(V a, V b) { return mk<V>(a.x - b.x, a.y - b.y); }
template <typename V> __device__ __forceinline__ V neg(V a) { return mk<V>(-a.x, -a.y); }
// a * (+i) and a * (-i)
template <typename V> __device__ __forceinline__ V mul_pi(V a) { return mk<V>(-a.y, a.x); }
template <typename V> __device__ __forceinline__ V mul_mi(V a) { return mk<V>(a.y, -a.x); }
template <typename V> __device__ __forceinline__ V scl(V a, typename RealOf<V>::type s) {
    return mk<V>(a.x * s, a.y * s);
}
// a * (c + i s)
template <typename V>
__device__ __forceinline__ V cmul(V a, typename RealOf<V>::type c, typename RealOf<V>::type s) {
    return mk<V>(a.x * c - a.y * s, a.x * s + a.y * c);
}
// line-pair (float4) versions of the complex operations
__device__ __forceinline__ float4 add(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float4 sub(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
__device__ __forceinline__ float4 neg(float4 a) { return make_float4(-a.x, -a.y, -a.z, -a.w); }
__device__ __forceinline__ float4 mul_pi(float4 a) { return make_float4(-a.y, a.x, -a.w, a.z); }
__device__ __forceinline__ float4 mul_mi(float4 a) { return make_float4(a.y, -a.x, a.w, -a.z); }
__device__ __forceinline__ float4 scl(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
__device__ __forceinline__ float4 cmul(float4 a, float c, float s) {
    return make_float4(a.x * c - a.y * s, a.x * s + a.y * c, a.z * c - a.w * s, a.z * s + a.w * c);
}

// a * w, or a * conj(w)
template <bool CONJ, typename V, typename W> __device__ __forceinline__ V cmulw(V a, W w) {
    return CONJ ? cmul(a, w.x, -w.y) : cmul(a, w.x, w.y);
}

// element a thread moves per (tile line, n): one complex, or for LPT = 2 the
// same index of two adjacent lines
template <typename T, int LPT> struct ElemOf { using type = cx<T>; };
template <> struct ElemOf<float, 2> { using type = float4; };

// cos(2 pi m / 16) and sin(2 pi m / 16), m = 0..15: the sixteenth roots of
// unity, to 21 significant digits.
__host__ __device__ constexpr double root16_cos(int m) {
    switch (m & 15) {
        case 0: return 1.0;
        case 1: case 15: return 0.923879532511286756128;
        case 2: case 14: return 0.707106781186547524401;
        case 3: case 13: return 0.382683432365089771728;
        case 4: case 12: return 0.0;
        case 5: case 11: return -0.382683432365089771728;
        case 6: case 10: return -0.707106781186547524401;
        case 7: case 9: return -0.923879532511286756128;
        default: return -1.0;
    }
}
__host__ __device__ constexpr double root16_sin(int m) { return root16_cos((m + 12) & 15); }
// cos(2 pi m / 32) and sin(2 pi m / 32), m = 0..31: the 32nd roots of unity,
// to 21 significant digits (the even ones equal the sixteenth roots above).
__host__ __device__ constexpr double root32_cos(int m) {
    constexpr double c[9] = {1.0,
                             0.980785280403230449126,
                             0.923879532511286756128,
                             0.831469612302545237079,
                             0.707106781186547524401,
                             0.555570233019602224743,
                             0.382683432365089771728,
                             0.195090322016128267848,
                             0.0};
    const int q = m & 31;  // cos is even about 0 and odd about 8: fold to 0..8
    return q <= 8 ? c[q] : q <= 16 ? -c[16 - q] : q <= 24 ? -c[q - 16] : c[32 - q];
}
__host__ __device__ constexpr double root32_sin(int m) { return root32_cos((m + 24) & 31); }
// sin(2 pi / 3)
constexpr double kSin60 = 0.866025403784438646763723170753;

// v * W_R^k with W_R = exp(-2 pi i / R) (forward) or its conjugate (INV).
// R divides 32; k is a compile-time constant once the caller's loops unroll,
// so the switch folds to one case.
template <int R, bool INV, typename V> __device__ __forceinline__ V twc(V v, int k) {
    static_assert(32 % R == 0, "in-register twiddles are 32nd roots of unity");
    using T = typename RealOf<V>::type;
    const int m = ((k % R) + R) % R * (32 / R);
    switch (m) {
        case 0: return v;
        case 8: return INV ? mul_pi(v) : mul_mi(v);
        case 16: return neg(v);
        case 24: return INV ? mul_mi(v) : mul_pi(v);
        default: {
            const T c = (T)root32_cos(m);
            const T s = (T)root32_sin(m);
            return cmul(v, c, INV ? s : -s);
        }
    }
}

// --------------------------------------------------------------------------
// small DFTs in registers, natural order in and out:
//   y_k = sum_n x_n exp(-+ 2 pi i n k / R)
// --------------------------------------------------------------------------
template <int R, bool INV, typename V> struct Dft;

template <bool INV, typename V> struct Dft<1, INV, V> {
    static __device__ __forceinline__ void run(V*) {}
};

template <bool INV, typename V> struct Dft<2, INV, V> {
    static __device__ __forceinline__ void run(V* v) {
        const V a = v[0];
        v[0] = add(a, v[1]);
        v[1] = sub(a, v[1]);
    }
};

template <bool INV, typename V> struct Dft<3, INV, V> {
    static __device__ __forceinline__ void run(V* v) {
        using T = typename RealOf<V>::type;
        const V t = add(v[1], v[2]);
        const V d = scl(sub(v[1], v[2]), (T)kSin60);
        const V m = sub(v[0], scl(t, (T)0.5));
        const V rot = INV ? mul_pi(d) : mul_mi(d);  // -+ i sin60 (x1 - x2)
        v[0] = add(v[0], t);
        v[1] = add(m, rot);
        v[2] = sub(m, rot);
    }
};

template <bool INV, typename V> struct Dft<4, INV, V> {
    static __device__ __forceinline__ void run(V* v) {
        const V a = add(v[0], v[2]);
        const V b = sub(v[0], v[2]);
        const V c = add(v[1], v[3]);
        V d = sub(v[1], v[3]);
        d = INV ? mul_pi(d) : mul_mi(d);
        v[0] = add(a, c);
        v[2] = sub(a, c);
        v[1] = add(b, d);
        v[3] = sub(b, d);
    }
};

// R = R1 * R2 split: n = R2 m + p, k = k1 + R1 k2,
// y[k1 + R1 k2] = sum_p W_R2^{p k2} ( W_R^{p k1} sum_m x[R2 m + p] W_R1^{m k1} )
template <int R1, int R2, bool INV, typename V> __device__ __forceinline__ void dft_split(V* v) {
    constexpr int R = R1 * R2;
    V a[R];
#pragma unroll
    for (int p = 0; p < R2; ++p) {
        V col[R1];
#pragma unroll
        for (int m = 0; m < R1; ++m) col[m] = v[R2 * m + p];
        Dft<R1, INV, V>::run(col);
#pragma unroll
        for (int k1 = 0; k1 < R1; ++k1) a[p * R1 + k1] = twc<R, INV>(col[k1], p * k1);
    }
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
        V row[R2];
#pragma unroll
        for (int p = 0; p < R2; ++p) row[p] = a[p * R1 + k1];
        Dft<R2, INV, V>::run(row);
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = row[k2];
    }
}

template <bool INV, typename V> struct Dft<8, INV, V> {
    static __device__ __forceinline__ void run(V* v) { dft_split<4, 2, INV>(v); }
};
template <bool INV, typename V> struct Dft<16, INV, V> {
    static __device__ __forceinline__ void run(V* v) { dft_split<4, 4, INV>(v); }
};
template <bool INV, typename V> struct Dft<32, INV, V> {
    static __device__ __forceinline__ void run(V* v) { dft_split<8, 4, INV>(v); }
};

// --------------------------------------------------------------------------
// radix plans
// --------------------------------------------------------------------------
template <int... Rs> struct RadixPlan {
    static constexpr int S = sizeof...(Rs);
    static constexpr int r[S] = {Rs...};
    static constexpr int N = (Rs * ...);
    // Ns before stage s
    __host__ __device__ static constexpr int ns(int s) {
        int x = 1;
        for (int i = 0; i < s; ++i) x *= r[i];
        return x;
    }
    // offset of stage s's twiddle table (stages >= 1; (R-1)*Ns entries each,
    // laid out [r-1][j mod Ns])
    __host__ __device__ static constexpr int twoff(int s) {
        int o = 0;
        for (int i = 1; i < s; ++i) o += (r[i] - 1) * ns(i);
        return o;
    }
    __host__ __device__ static constexpr int twtotal() { return twoff(S); }
};

enum PassMode : int {
    // line elements are contiguous in memory (runs of the brick's l_axis):
    // threads walk along a line (the reference's Z pencils, and every 1D
    // call on pencil buffers)
    MODE_LINE = 0,
    // consecutive lines are contiguous in memory: threads walk across lines
    // (X and Y passes over z-fastest bricks)
    MODE_BATCH = 1
};

template <typename T> struct PassArgs {
    const cx<T>* src;      // may alias dst (in-place pass)
    cx<T>* dst;
    const uint32_t* offA;  // element offset of index n along the transform axis (N entries)
    const uint32_t* offU;  // line offset, outer batch coordinate (NU entries)
    const uint32_t* offV;  // line offset, inner batch coordinate (NV entries)
    const cx<T>* tw;       // stage twiddles, forward sign, RadixPlan::twoff layout
    int NU;
    int NV;                // multiple of B
    T scale;               // multiplies every stored element
    // offA[j + r N/R] == offA[j] + offA[r N/R] for the first and last stage
    // (the brick extent along the axis and N/R divide one another): addresses
    // are then one table value per butterfly plus CTA-uniform deltas
    int split;
    int* err;              // set to 1 by a kernel whose bounded wait gave up
    const void* tcb;       // tensor-core kernels: the split radix-16 operand [Rh | Rl]
};

// Butterfly q of a stage -> (tile line b, butterfly j), NBL butterflies per
// line.  BFAST: consecutive q walk across lines (b fastest), conflict-free in
// shared memory for both layouts; otherwise q walks along a line (j fastest),
// which coalesces global accesses when a line's elements are contiguous.
template <bool BFAST, int B, int NBL> __device__ __forceinline__ void bf_map(int q, int& b, int& j) {
    if constexpr (BFAST) {
        b = q % B;
        j = q / B;
    } else {
        j = q % NBL;
        b = q / NBL;
    }
}

// Shared-memory layout of one tile of BV vector lines of ESZ-byte elements.
// A shared access of SLOTS = 128/ESZ lanes (a half warp for 8-byte, a quarter
// warp for 16-byte elements) is one wavefront when its lanes hit distinct
// 128-byte bank rows' slots.  BATCH: [n][bv] (lines fastest).  LINE: line b at
// b*LS, element n at n + n/SLOTS: the pad slot per SLOTS elements makes the
// stride-R butterfly writes of radix 2..SLOTS land in distinct slots, and
// LS == SLOTS/BV (mod SLOTS) makes a wavefront that walks across the BV lines
// (SLOTS/BV consecutive elements each) distinct as well.
//
// SWSH >= 0 (BATCH tiles whose rows are narrower than a 128-byte bank row,
// RPL = 128 / (BV ESZ) rows per bank row): row n is stored at n ^ ((n >>
// SWSH) & (RPL - 1)).  With SWSH = log2 of the first radix, the first stage's
// writes to rows R j + r (R apart for neighbouring threads) and the other
// stages' accesses to adjacent rows land in distinct bank-row slots.
template <int MODE, int BV, int N, int ESZ, int SWSH = -1> struct TileGeom {
    static constexpr int SLOTS = 128 / ESZ;
    static constexpr int LS0 = N + N / SLOTS;
    static constexpr int WANT = (SLOTS / (BV < SLOTS ? BV : SLOTS)) % SLOTS;
    static constexpr int LS = LS0 + ((WANT - LS0 % SLOTS) % SLOTS + SLOTS) % SLOTS;
    static constexpr int elems = (MODE == MODE_BATCH) ? N * BV : BV * LS;
    static constexpr int RPL = (BV * ESZ < 128) ? 128 / (BV * ESZ) : 1;
    static constexpr bool SWZ = MODE == MODE_BATCH && SWSH >= 0 && RPL >= 2;
    static __device__ __forceinline__ int idx(int b, int n) {
        if constexpr (MODE == MODE_BATCH) {
            if constexpr (SWZ)
                return (n ^ ((n >> SWSH) & (RPL - 1))) * BV + b;
            else
                return n * BV + b;
        } else {
            return b * LS + n + n / SLOTS;
        }
    }
};

// The row swizzle shift for a BATCH tile of plan PLAN with BV vectors of ESZ
// bytes per row: log2 of the first radix when it is a power of two at least
// the rows per bank row (the XOR then stays a permutation of the rows), else
// -1 (no swizzle).
template <class PLAN, int BV, int ESZ> __host__ __device__ constexpr int tile_swizzle_shift() {
    constexpr int R0 = PLAN::r[0];
    constexpr int RPL = (BV * ESZ < 128) ? 128 / (BV * ESZ) : 1;
    if ((R0 & (R0 - 1)) != 0 || RPL < 2 || RPL > R0 || (128 % (BV * ESZ)) != 0) return -1;
    int sh = 0;
    while ((1 << sh) < R0) ++sh;
    return sh;
}

// streaming loads/stores: each element is touched once per pass
template <typename V> __device__ __forceinline__ V ld_stream(const V* p) { return __ldcs(p); }
template <typename V> __device__ __forceinline__ void st_stream(V* p, V v) { __stcs(p, v); }

// asynchronous global -> shared copies (sm_80+ LDGSTS), one group per tile
template <int BYTES> __device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
    const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Stages s >= 1 (and stage 0 of the pipelined kernel): shared -> registers,
// twiddle, DFT_R, then shared (Stockham position) or, for the last stage,
// global memory at base_s[b] + offA_s[n].  A thread moves LPT lines at once.
// A virtual rank-major buffer split into blocks of equal size that may live
// in other GPUs' memory (the multi-block pass, fft_mb.cuh): element o is
// element o mod L of block o div L.
constexpr int kMbMaxBlocks = 8;
template <typename T> struct MbArgs {
    cx<T>* blk[kMbMaxBlocks];  // block base pointers (device or peer addresses)
    FastDiv fbe;               // elements per block
    int nblk;
    int tile0;                 // first tile of this launch
    int tile1;                 // one past its last tile (persistent kernels)
};
template <typename T> __device__ __forceinline__ cx<T>* mb_addr(const MbArgs<T>& m, uint32_t o) {
    uint32_t b, r;
    m.fbe.divmod(o, b, r);
    return m.blk[b] + r;
}

template <typename T, class PLAN, int B, int THREADS, int MODE, bool INV, int LPT, int s, int SWSH = -1,
          bool MB = false>
__device__ __forceinline__ void run_stage(const PassArgs<T>& a, typename ElemOf<T, LPT>::type* tile,
                                          const cx<T>* tw, const uint32_t* offA_s, const size_t* base_s, int tid,
                                          const MbArgs<T>* mb = nullptr) {
    using E = typename ElemOf<T, LPT>::type;
    constexpr int BV = B / LPT;
    using G = TileGeom<MODE, BV, PLAN::N, sizeof(E), SWSH>;
    constexpr int N = PLAN::N;
    constexpr int R = PLAN::r[s];
    constexpr int NS = PLAN::ns(s);
    constexpr int NBL = N / R;             // butterflies per line
    constexpr int NBT = BV * NBL;          // butterflies per tile
    constexpr int K = (NBT + THREADS - 1) / THREADS;
    constexpr bool EXACT = (NBT % THREADS) == 0;
    constexpr bool LAST = (s == PLAN::S - 1);
    constexpr bool BFAST = (MODE == MODE_BATCH) || !LAST;
    constexpr int TWO = PLAN::twoff(s);

    E x[K][R];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int q = tid + k * THREADS;
        if (EXACT || q < NBT) {
            int b, j;
            bf_map<BFAST, BV, NBL>(q, b, j);
#pragma unroll
            for (int r = 0; r < R; ++r) x[k][r] = tile[G::idx(b, j + r * NBL)];
        }
    }
    __syncthreads();  // the tile is updated in place
    uint32_t dl[R];
    if constexpr (LAST) {
#pragma unroll
        for (int r = 0; r < R; ++r) dl[r] = offA_s[r * NBL];
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
        const int q = tid + k * THREADS;
        if (EXACT || q < NBT) {
            int b, j;
            bf_map<BFAST, BV, NBL>(q, b, j);
            const int m = j % NS;
            if constexpr (s > 0) {
#pragma unroll
                for (int r = 1; r < R; ++r) x[k][r] = cmulw<INV>(x[k][r], tw[TWO + (r - 1) * NS + m]);
            }
            Dft<R, INV, E>::run(x[k]);
            if constexpr (LAST && MB) {
                // a line pair (LPT = 2) never straddles two blocks: both lines
                // lie in one brick, blocks hold whole bricks
                const uint32_t line = (uint32_t)base_s[b];
#pragma unroll
                for (int r = 0; r < R; ++r)
                    st_stream(reinterpret_cast<E*>(mb_addr(*mb, line + offA_s[j + r * NBL])), scl(x[k][r], a.scale));
            } else if constexpr (LAST) {
                cx<T>* line = a.dst + base_s[b];
                if (a.split) {
                    cx<T>* p = line + offA_s[j];
#pragma unroll
                    for (int r = 0; r < R; ++r)
                        st_stream(reinterpret_cast<E*>(p + dl[r]), scl(x[k][r], a.scale));
                } else {
#pragma unroll
                    for (int r = 0; r < R; ++r)
                        st_stream(reinterpret_cast<E*>(line + offA_s[j + r * NBL]), scl(x[k][r], a.scale));
                }
            } else {
                const int jd = (j / NS) * NS * R + m;
#pragma unroll
                for (int r = 0; r < R; ++r) tile[G::idx(b, jd + r * NS)] = x[k][r];
            }
        }
    }
    if constexpr (!LAST) {
        __syncthreads();
        run_stage<T, PLAN, B, THREADS, MODE, INV, LPT, s + 1, SWSH, MB>(a, tile, tw, offA_s, base_s, tid, mb);
    }
}

enum PassKind : int {
    KIND_DIRECT = 0,  // one tile per CTA, stage 0 loads global memory into registers
    KIND_PIPE = 1,    // persistent CTAs, next tile prefetched into shared memory (LDGSTS)
    KIND_TMA = 2,     // persistent CTAs, tile rows fetched by TMA bulk copies, mbarrier completion
    KIND_TC = 3,      // radix-16 stages as split-precision tcgen05 GEMMs
    KIND_RPIPE = 4,   // persistent CTAs, next tile's stage-0 loads in flight in registers
    KIND_TMAT2 = 5,   // persistent CTAs, whole tiles fetched by TMA tensor copies into a 2-slot ring
    KIND_TMAT3 = 6,   // the same with a 3-slot ring
    KIND_TMAT2W = 7,  // the 2-slot ring with the length's two-stage wide-radix plan (radix 16/32)
    KIND_TMATI = 8,   // the 2-slot ring with each slot transformed in place (no separate tile)
    KIND_TCR = 9,     // tensor-core stages, persistent CTAs fed by the in-place 2-slot TMA ring
    KIND_TMAT2S = 10, // the 2-slot ring, batch tiles, first exchange by warp shuffles (R0 R1 = 64 plans)
    KIND_RPIPES = 11, // register-pipelined line-mode tiles, first exchange by warp shuffles (512)
    KIND_TC2 = 12     // two tensor-core stages (512 = 16 x 32, 1024 = 32 x 32: GEMM, twiddle, radix-32 GEMM), TMA ring
};

constexpr int kTmaBuffers = 2;

template <typename T, class PLAN, int B, int MODE, int KIND, int LPT>
__host__ __device__ constexpr size_t pass_smem_bytes() {
    using E = typename ElemOf<T, LPT>::type;
    constexpr int N = PLAN::N;
    constexpr int BV = B / LPT;
    constexpr int NBUF = KIND == KIND_PIPE ? 2 : KIND == KIND_TMA ? kTmaBuffers : 1;
    size_t bytes = sizeof(E) * (size_t)(NBUF * TileGeom<MODE, BV, N, sizeof(E)>::elems);
    bytes += sizeof(cx<T>) * (size_t)PLAN::twtotal();
    bytes += sizeof(uint32_t) * (size_t)N;
    bytes = (bytes + 15) & ~size_t(15);
    bytes += sizeof(size_t) * (size_t)(NBUF * BV);
    if (KIND == KIND_TMA) bytes += sizeof(unsigned long long) * NBUF;  // mbarriers
    return bytes;
}

// One tile of B lines (u, v0 .. v0+B-1), tile index t = u * (NV/B) + v0/B,
// in the CTA's dynamic shared memory.  Stage 0 reads global memory straight
// into registers (j fastest in LINE mode, so the loads coalesce along the
// line).  With LPT = 2 (BATCH, complex float) a thread moves the same
// element of two adjacent lines as one 16-byte access.  CG: read through L2
// only (for data another CTA of the same launch has just written).
template <typename T, class PLAN, int B, int THREADS, int MODE, bool INV, int LPT, bool CG = false>
__device__ __forceinline__ void direct_tile(const PassArgs<T>& a, int t, unsigned char* smem_raw, int tid) {
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
    static_assert(MODE != MODE_BATCH || THREADS % BV == 0, "batch mode needs THREADS % (B/LPT) == 0");
    static_assert(LPT == 1 || MODE == MODE_BATCH, "line pairs only in batch mode");

    E* tile = reinterpret_cast<E*>(smem_raw);
    cx<T>* tw = reinterpret_cast<cx<T>*>(tile + G::elems);
    uint32_t* offA_s = reinterpret_cast<uint32_t*>(tw + TWN);
    size_t* base_s = reinterpret_cast<size_t*>(
        smem_raw + ((sizeof(E) * (size_t)G::elems + sizeof(cx<T>) * TWN + sizeof(uint32_t) * N + 15) & ~size_t(15)));

    const int tilesV = a.NV / B;
    const int u = t / tilesV;
    const int v0 = (t - u * tilesV) * B;
    const size_t ubase = a.offU[u];

    uint32_t d0[R0];
    if (a.split) {
#pragma unroll
        for (int r = 0; r < R0; ++r) d0[r] = __ldg(a.offA + r * NBL);
    }
    E x[K][R0];
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
                for (int r = 0; r < R0; ++r) {
                    const E* ptr = reinterpret_cast<const E*>(p + d0[r]);
                    x[k][r] = CG ? __ldcg(ptr) : ld_stream(ptr);
                }
            } else {
#pragma unroll
                for (int r = 0; r < R0; ++r) {
                    const E* ptr = reinterpret_cast<const E*>(line + __ldg(a.offA + j + r * NBL));
                    x[k][r] = CG ? __ldcg(ptr) : ld_stream(ptr);
                }
            }
        }
    }
    // tables for the later stages (overlaps the loads in flight)
    for (int i = tid; i < TWN; i += THREADS) tw[i] = a.tw[i];
    for (int i = tid; i < N; i += THREADS) offA_s[i] = a.offA[i];
    for (int i = tid; i < BV; i += THREADS) base_s[i] = ubase + a.offV[v0 + i * LPT];

    if constexpr (PLAN::S == 1) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int q = tid + k * THREADS;
            if (EXACT || q < NBT) {
                int b, j;
                bf_map<BFAST0, BV, NBL>(q, b, j);
                Dft<R0, INV, E>::run(x[k]);
                cx<T>* line = a.dst + ubase + __ldg(a.offV + v0 + b * LPT);
#pragma unroll
                for (int r = 0; r < R0; ++r)
                    st_stream(reinterpret_cast<E*>(line + __ldg(a.offA + j + r * NBL)), scl(x[k][r], a.scale));
            }
        }
    } else {
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
        __syncthreads();
        run_stage<T, PLAN, B, THREADS, MODE, INV, LPT, 1>(a, tile, tw, offA_s, base_s, tid);
    }
}

// KIND_DIRECT: one CTA = one tile.
template <typename T, class PLAN, int B, int THREADS, int MODE, bool INV, int MINB, int LPT>
__global__ void __launch_bounds__(THREADS, MINB) fft_pass_kernel(const PassArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    direct_tile<T, PLAN, B, THREADS, MODE, INV, LPT>(a, blockIdx.x, smem_raw, threadIdx.x);
}

// KIND_RPIPE: persistent CTAs double-buffer through registers.  Stage 0 of
// tile t leaves its results in shared memory; its registers then receive the
// global loads of tile t + gridDim.x, which stay in flight while stages
// 1..S-1 of tile t run, so each SM keeps HBM reads going through its
// butterfly phase without a second shared-memory tile.
template <typename T, class PLAN, int B, int THREADS, int MODE, bool INV, int MINB, int LPT>
__global__ void __launch_bounds__(THREADS, MINB) fft_rpipe_kernel(const PassArgs<T> a) {
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
    const int ntiles = a.NU * tilesV;
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
                    for (int r = 0; r < R0; ++r) x[k][r] = ld_stream(reinterpret_cast<const E*>(p + d0[r]));
                } else {
#pragma unroll
                    for (int r = 0; r < R0; ++r)
                        x[k][r] = ld_stream(reinterpret_cast<const E*>(line + __ldg(a.offA + j + r * NBL)));
                }
            }
        }
    };
    int t = blockIdx.x;
    E x[K][R0];
    if (t < ntiles) load_tile(t, x);
    for (int i = tid; i < TWN; i += THREADS) tw[i] = a.tw[i];
    for (int i = tid; i < N; i += THREADS) offA_s[i] = a.offA[i];
    for (; t < ntiles; t += gridDim.x) {
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
        const int tn = t + gridDim.x;
        if (tn < ntiles) load_tile(tn, x);  // in flight through the remaining stages
        __syncthreads();
        run_stage<T, PLAN, B, THREADS, MODE, INV, LPT, 1>(a, tile, tw, offA_s, base_s, tid);
        __syncthreads();  // tile and line bases free for the next tile
    }
}

// Issue the asynchronous copies of tile t into `buf` and record its line
// bases.  BATCH tiles move as rows of B contiguous elements (16-byte units;
// the host only selects this kernel when every tile's lines are contiguous and
// 16-byte aligned); LINE tiles move element by element into the padded layout.
template <typename T, class PLAN, int B, int THREADS, int MODE>
__device__ __forceinline__ void pipe_issue(const PassArgs<T>& a, int t, int tilesV, cx<T>* buf, size_t* base_s,
                                           int tid) {
    using V = cx<T>;
    using G = TileGeom<MODE, B, PLAN::N, sizeof(V)>;
    constexpr int N = PLAN::N;
    const int u = t / tilesV;
    const int v0 = (t - u * tilesV) * B;
    const size_t ubase = __ldg(a.offU + u);
    for (int b = tid; b < B; b += THREADS) base_s[b] = ubase + __ldg(a.offV + v0 + b);
    if constexpr (MODE == MODE_BATCH) {
        constexpr int EPU = 16 / sizeof(V);  // elements per 16-byte unit
        constexpr int UPR = B / EPU;         // units per tile row
        static_assert(B % EPU == 0, "tile rows must be whole 16-byte units");
        const V* row0 = a.src + ubase + __ldg(a.offV + v0);
#pragma unroll 4
        for (int w = tid; w < N * UPR; w += THREADS) {
            const int n = w / UPR;
            const int c = w - n * UPR;
            cp_async<16>(buf + n * B + c * EPU, row0 + __ldg(a.offA + n) + c * EPU);
        }
    } else {
#pragma unroll 4
        for (int e = tid; e < B * N; e += THREADS) {
            const int b = e / N;
            const int n = e - b * N;
            cp_async<sizeof(V)>(buf + G::idx(b, n), a.src + ubase + __ldg(a.offV + v0 + b) + __ldg(a.offA + n));
        }
    }
}

// KIND_PIPE: persistent CTAs walk the tiles with a stride of gridDim.x; while
// tile t is transformed in one shared buffer, tile t + gridDim.x streams into
// the other, so every SM keeps HBM reads in flight through its compute phase.
template <typename T, class PLAN, int B, int THREADS, int MODE, bool INV, int MINB, int LPT>
__global__ void __launch_bounds__(THREADS, MINB) fft_pipe_kernel(const PassArgs<T> a) {
    using V = cx<T>;
    using G = TileGeom<MODE, B, PLAN::N, sizeof(V)>;
    constexpr int N = PLAN::N;
    constexpr int TWN = PLAN::twtotal();
    static_assert(PLAN::S >= 2, "the pipelined kernel needs at least two stages");
    static_assert(MODE != MODE_BATCH || THREADS % B == 0, "batch mode needs THREADS % B == 0");
    static_assert(LPT == 1, "the pipelined kernel moves one line per thread");

    extern __shared__ __align__(16) unsigned char smem_raw[];
    V* buf0 = reinterpret_cast<V*>(smem_raw);
    V* buf1 = buf0 + G::elems;
    V* tw = buf1 + G::elems;
    uint32_t* offA_s = reinterpret_cast<uint32_t*>(tw + TWN);
    size_t* base0 = reinterpret_cast<size_t*>(
        smem_raw + ((sizeof(V) * (size_t)(2 * G::elems + TWN) + sizeof(uint32_t) * N + 15) & ~size_t(15)));
    size_t* base1 = base0 + B;

    const int tid = threadIdx.x;
    const int tilesV = a.NV / B;
    const int ntiles = a.NU * tilesV;
    int t = blockIdx.x;
    if (t < ntiles) pipe_issue<T, PLAN, B, THREADS, MODE>(a, t, tilesV, buf0, base0, tid);
    cp_async_commit();
    for (int i = tid; i < TWN; i += THREADS) tw[i] = a.tw[i];
    for (int i = tid; i < N; i += THREADS) offA_s[i] = a.offA[i];
    bool odd = false;
    for (; t < ntiles; t += gridDim.x, odd = !odd) {
        V* cur = odd ? buf1 : buf0;
        size_t* cbase = odd ? base1 : base0;
        const int tn = t + gridDim.x;
        if (tn < ntiles) pipe_issue<T, PLAN, B, THREADS, MODE>(a, tn, tilesV, odd ? buf0 : buf1, odd ? base0 : base1,
                                                              tid);
        cp_async_commit();
        cp_async_wait<1>();  // this thread's copies of tile t have landed
        __syncthreads();     // ... and every other thread's
        run_stage<T, PLAN, B, THREADS, MODE, INV, 1, 0>(a, cur, tw, offA_s, cbase, tid);
        __syncthreads();     // `cur` and `cbase` are free for the copies issued next iteration
    }
    cp_async_wait<0>();
}

// ---------------------------------------------------------------------------
// TMA bulk-copy pipeline (BATCH mode).  Every tile row -- B contiguous lines
// at one index n, B * sizeof(complex) bytes -- is one cp.async.bulk from
// global into shared memory, completing on the tile buffer's mbarrier; one
// warp issues all of a tile's rows.  Persistent CTAs keep kTmaBuffers tiles in
// flight, so the fetch of later tiles overlaps the butterflies of the current
// one without occupying L1 miss slots or the load/store queue.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, uint32_t bytes) {
    asm volatile(
        "{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(smem_u32(bar)),
        "r"(bytes)
        : "memory");
}
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}
// Wait for the given phase parity of an mbarrier, giving up after about half
// a second (or 2^22 polls): returns false then.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, uint32_t parity) {
    const uint64_t t0 = global_ns();
    for (int i = 0; i < (1 << 22); ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
        if ((i & 1023) == 1023 && global_ns() - t0 > 500000000ull) return false;
    }
    return false;
}

template <typename T, class PLAN, int B, int THREADS, int LPT>
__device__ __forceinline__ void tma_issue(const PassArgs<T>& a, int t, int tilesV, typename ElemOf<T, LPT>::type* buf,
                                          size_t* base_s, unsigned long long* bar, int tid) {
    using E = typename ElemOf<T, LPT>::type;
    constexpr int BV = B / LPT;
    constexpr int N = PLAN::N;
    constexpr uint32_t ROW = B * sizeof(cx<T>);
    const int u = t / tilesV;
    const int v0 = (t - u * tilesV) * B;
    const size_t ubase = __ldg(a.offU + u);
    for (int b = tid; b < BV; b += THREADS) base_s[b] = ubase + __ldg(a.offV + v0 + b * LPT);
    if (tid < 32) {
        if (tid == 0) {
            fence_proxy_async_smem();  // earlier generic reads of buf are ordered before the async writes
            mbar_arrive_expect_tx(bar, ROW * N);
        }
        __syncwarp();
        const cx<T>* row0 = a.src + ubase + __ldg(a.offV + v0);
        for (int n = tid; n < N; n += 32) bulk_g2s(buf + n * BV, row0 + __ldg(a.offA + n), ROW, bar);
    }
}

template <typename T, class PLAN, int B, int THREADS, int MODE, bool INV, int MINB, int LPT>
__global__ void __launch_bounds__(THREADS, MINB) fft_tma_kernel(const PassArgs<T> a) {
    using E = typename ElemOf<T, LPT>::type;
    constexpr int BV = B / LPT;
    using G = TileGeom<MODE_BATCH, BV, PLAN::N, sizeof(E)>;
    constexpr int N = PLAN::N;
    constexpr int TWN = PLAN::twtotal();
    constexpr int NBUF = kTmaBuffers;
    static_assert(MODE == MODE_BATCH, "TMA tiles move whole rows of contiguous lines");
    static_assert(PLAN::S >= 2, "the pipelined kernel needs at least two stages");
    static_assert(THREADS % BV == 0, "batch mode needs THREADS % (B/LPT) == 0");
    static_assert((B * sizeof(cx<T>)) % 16 == 0, "bulk copies move multiples of 16 bytes");

    extern __shared__ __align__(16) unsigned char smem_raw[];
    E* buf = reinterpret_cast<E*>(smem_raw);
    cx<T>* tw = reinterpret_cast<cx<T>*>(buf + NBUF * G::elems);
    uint32_t* offA_s = reinterpret_cast<uint32_t*>(tw + TWN);
    size_t* base_s = reinterpret_cast<size_t*>(
        smem_raw +
        ((sizeof(E) * (size_t)(NBUF * G::elems) + sizeof(cx<T>) * TWN + sizeof(uint32_t) * N + 15) & ~size_t(15)));
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(base_s + NBUF * BV);

    const int tid = threadIdx.x;
    const int tilesV = a.NV / B;
    const int ntiles = a.NU * tilesV;
    if (tid == 0) {
        for (int i = 0; i < NBUF; ++i) mbar_init(bar + i, 1);
        fence_mbar_init();
    }
    for (int i = tid; i < TWN; i += THREADS) tw[i] = a.tw[i];
    for (int i = tid; i < N; i += THREADS) offA_s[i] = a.offA[i];
    __syncthreads();
    for (int i = 0; i < NBUF; ++i) {
        const int ti = blockIdx.x + i * gridDim.x;
        if (ti < ntiles)
            tma_issue<T, PLAN, B, THREADS, LPT>(a, ti, tilesV, buf + i * G::elems, base_s + i * BV, bar + i, tid);
    }
    __syncthreads();  // line bases visible to every thread
    int it = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
        const int slot = it % NBUF;
        const bool ok = mbar_wait_bounded(bar + slot, (uint32_t)((it / NBUF) & 1));
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicExch(a.err, 1);
                // wait (bounded) for this CTA's copies still in flight before leaving
                for (int j = it; j < it + NBUF; ++j)
                    if (blockIdx.x + j * gridDim.x < (unsigned)ntiles)
                        mbar_wait_bounded(bar + j % NBUF, (uint32_t)((j / NBUF) & 1));
            }
            return;
        }
        run_stage<T, PLAN, B, THREADS, MODE_BATCH, INV, LPT, 0>(a, buf + slot * G::elems, tw, offA_s,
                                                               base_s + slot * BV, tid);
        __syncthreads();  // buffer `slot` and its line bases are free again
        const int tn = t + NBUF * gridDim.x;
        if (tn < ntiles)
            tma_issue<T, PLAN, B, THREADS, LPT>(a, tn, tilesV, buf + slot * G::elems, base_s + slot * BV, bar + slot,
                                                tid);
        __syncthreads();  // the new line bases are visible before they are read
    }
}

}  // namespace a2a
