// Compiled transform lengths, their radix plans and launch variants, and the
// host-side lookup of the pass kernels for (precision, N, mode, direction).
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

#include "fft_tile.cuh"
#include "fft_tmat.cuh"

namespace a2a {

// Host view of one compiled pass kernel.
struct PassKernel {
    const void* fn = nullptr;
    int kind = KIND_DIRECT;
    int n = 0;          // transform length
    int threads = 0;
    int lines = 0;      // B: lines per tile (a pass needs NV % lines == 0)
    int min_blocks = 1; // __launch_bounds__ minimum blocks per SM
    int lpt = 1;        // lines a thread moves per access (2: 16-byte line pairs)
    size_t smem = 0;    // dynamic shared memory bytes
    int nstages = 0;
    int radix[4] = {0, 0, 0, 0};
    int twtotal = 0;    // complex entries of the twiddle table
};

// Radix plan per (element type, N): radix 8/16 stages where they divide,
// one radix-2/3/4 stage for the rest.
template <typename T, int N> struct PassPlan;
#define A2A_PLAN(T_, N_, ...)                                               \
    template <> struct PassPlan<T_, N_> {                                   \
        using Plan = RadixPlan<__VA_ARGS__>;                                \
        static_assert(Plan::N == N_, "radix plan does not multiply to N");  \
    };

// clang-format off
#define A2A_PLANS(T_)                 \
    A2A_PLAN(T_,    4, 4)             \
    A2A_PLAN(T_,    8, 8)             \
    A2A_PLAN(T_,   12, 3, 4)          \
    A2A_PLAN(T_,   16, 16)            \
    A2A_PLAN(T_,   24, 3, 8)          \
    A2A_PLAN(T_,   32, 4, 8)          \
    A2A_PLAN(T_,   48, 3, 16)         \
    A2A_PLAN(T_,   64, 8, 8)          \
    A2A_PLAN(T_,   96, 3, 4, 8)       \
    A2A_PLAN(T_,  128, 8, 16)         \
    A2A_PLAN(T_,  192, 3, 4, 16)      \
    A2A_PLAN(T_,  256, 16, 16)        \
    A2A_PLAN(T_,  384, 3, 8, 16)      \
    A2A_PLAN(T_,  512, 8, 8, 8)       \
    A2A_PLAN(T_,  768, 3, 16, 16)     \
    A2A_PLAN(T_, 1024, 4, 16, 16)
A2A_PLANS(float)
A2A_PLANS(double)

// Two-stage plans with a radix-32 stage, for the lengths where they replace
// three stages (one shared-memory exchange fewer per tile): kernels of kind
// KIND_TMAT2W use these, every other kind the plans above.
template <typename T, int N> struct PassPlan2;
#define A2A_PLAN2(T_, N_, ...)                                              \
    template <> struct PassPlan2<T_, N_> {                                  \
        using Plan = RadixPlan<__VA_ARGS__>;                                \
        static_assert(Plan::N == N_, "radix plan does not multiply to N");  \
    };
A2A_PLAN2(float, 512, 16, 32)
A2A_PLAN2(float, 1024, 32, 32)
A2A_PLAN2(double, 512, 16, 32)
A2A_PLAN2(double, 1024, 32, 32)

template <typename T, int N, int KIND> struct PlanOf { using Plan = typename PassPlan<T, N>::Plan; };
template <typename T, int N> struct PlanOf<T, N, KIND_TMAT2W> { using Plan = typename PassPlan2<T, N>::Plan; };

// Launch variants X(T, N, KIND, B lines per tile, THREADS, MINB, LPT).  The first
// entry per N is the default; make_plans can time the others on the scratch
// buffer and keep the fastest (a2a_dfft_make_plans).  DIRECT tiles are about
// 32-64 KB so two or three CTAs share an SM; PIPE CTAs hold two tiles.  LPT =
// 2 (complex float, batch mode): a thread moves two adjacent lines as one
// 16-byte access, which halves the shared-memory instructions of a tile.  The
// first entry of each length is its default in both access modes (entries a
// mode cannot use are skipped): at 512 the shuffle ring kernel for batch-mode
// passes, the register-pipelined kernel for line mode.
#define A2A_VARIANTS_F32(X)                            \
    X(float,    4, KIND_DIRECT,  4,  32, 1, 1)      \
    X(float,    8, KIND_DIRECT,  8,  32, 1, 1)      \
    X(float,    8, KIND_DIRECT,  4,  32, 1, 1)      \
    X(float,   12, KIND_DIRECT,  4,  32, 1, 1)      \
    X(float,   16, KIND_DIRECT, 16,  32, 1, 1)      \
    X(float,   16, KIND_DIRECT,  4,  32, 1, 1)      \
    X(float,   24, KIND_DIRECT,  8,  32, 1, 1)      \
    X(float,   24, KIND_DIRECT,  4,  32, 1, 1)      \
    X(float,   32, KIND_DIRECT, 32,  64, 1, 2)      \
    X(float,   32, KIND_DIRECT, 32, 128, 1, 1)      \
    X(float,   32, KIND_DIRECT,  4,  32, 1, 1)      \
    X(float,   48, KIND_DIRECT, 16,  32, 1, 2)      \
    X(float,   48, KIND_DIRECT, 16,  64, 1, 1)      \
    X(float,   48, KIND_DIRECT,  4,  32, 1, 1)      \
    X(float,   64, KIND_DIRECT, 32, 128, 1, 2)      \
    X(float,   64, KIND_DIRECT, 32, 128, 1, 1)      \
    X(float,   64, KIND_PIPE,   32, 128, 4, 1)      \
    X(float,   64, KIND_DIRECT,  4,  32, 1, 1)      \
    X(float,   96, KIND_DIRECT, 32, 128, 1, 2)      \
    X(float,   96, KIND_DIRECT, 32, 128, 1, 1)      \
    X(float,   96, KIND_PIPE,   32, 128, 2, 1)      \
    X(float,   96, KIND_DIRECT,  4,  32, 1, 1)      \
    X(float,  128, KIND_DIRECT, 32, 128, 1, 2)      \
    X(float,  128, KIND_DIRECT, 16, 128, 4, 1)      \
    X(float,  128, KIND_DIRECT, 32, 256, 1, 1)      \
    X(float,  128, KIND_PIPE,   32, 256, 2, 1)      \
    X(float,  128, KIND_DIRECT,  4,  32, 1, 1)      \
    X(float,  192, KIND_DIRECT, 32, 256, 1, 2)      \
    X(float,  192, KIND_DIRECT, 32, 256, 1, 1)      \
    X(float,  192, KIND_PIPE,   16, 256, 2, 1)      \
    X(float,  192, KIND_DIRECT,  4,  64, 1, 1)      \
    X(float,  256, KIND_DIRECT, 16, 256, 2, 1)      \
    X(float,  256, KIND_RPIPE,  16, 256, 2, 1)      \
    X(float,  256, KIND_DIRECT, 32, 256, 1, 2)      \
    X(float,  256, KIND_TMA,    16, 256, 2, 1)      \
    X(float,  256, KIND_TMA,    32, 512, 1, 1)      \
    X(float,  256, KIND_DIRECT, 16, 128, 4, 2)      \
    X(float,  256, KIND_DIRECT, 32, 256, 1, 1)      \
    X(float,  256, KIND_PIPE,   16, 256, 2, 1)      \
    X(float,  256, KIND_DIRECT,  4,  64, 1, 1)      \
    X(float,  384, KIND_DIRECT, 16, 256, 1, 2)      \
    X(float,  384, KIND_DIRECT, 16, 256, 1, 1)      \
    X(float,  384, KIND_PIPE,    8, 256, 2, 1)      \
    X(float,  384, KIND_DIRECT,  4,  64, 1, 1)      \
    X(float,  512, KIND_TMAT2S,  8, 128, 2, 1)      \
    X(float,  512, KIND_RPIPE,  16, 512, 1, 2)      \
    X(float,  512, KIND_RPIPE,   8, 256, 2, 1)      \
    X(float,  512, KIND_RPIPES,  8, 128, 2, 1)      \
    X(float,  512, KIND_RPIPE,   8, 256, 3, 1)      \
    X(float,  512, KIND_DIRECT, 16, 512, 1, 2)      \
    X(float,  512, KIND_DIRECT,  8, 128, 4, 1)      \
    X(float,  512, KIND_RPIPE,  16, 512, 1, 1)      \
    X(float,  512, KIND_RPIPE,  16, 256, 1, 2)      \
    X(float,  512, KIND_DIRECT, 16, 256, 2, 2)      \
    X(float,  512, KIND_DIRECT, 16, 256, 2, 1)      \
    X(float,  512, KIND_DIRECT,  8, 128, 4, 2)      \
    X(float,  512, KIND_PIPE,    8, 256, 2, 1)      \
    X(float,  512, KIND_DIRECT,  4,  64, 1, 1)      \
    X(float,  768, KIND_DIRECT,  8, 256, 1, 2)      \
    X(float,  768, KIND_DIRECT,  8, 256, 1, 1)      \
    X(float,  768, KIND_DIRECT, 16, 384, 1, 2)      \
    X(float,  768, KIND_PIPE,    8, 384, 1, 1)      \
    X(float,  768, KIND_DIRECT,  4, 128, 1, 1)      \
    X(float, 1024, KIND_DIRECT,  8, 512, 1, 1)      \
    X(float, 1024, KIND_DIRECT, 16, 512, 1, 2)      \
    X(float, 1024, KIND_RPIPE,   8, 512, 1, 1)      \
    X(float, 1024, KIND_TMA,     8, 512, 1, 1)      \
    X(float, 1024, KIND_DIRECT,  8, 256, 1, 1)      \
    X(float, 1024, KIND_DIRECT,  8, 256, 1, 2)      \
    X(float, 1024, KIND_PIPE,    8, 512, 1, 1)      \
    X(float, 1024, KIND_DIRECT,  4, 128, 1, 1)      \
    X(float,  128, KIND_TMAT2,  32, 256, 2, 1)      \
    X(float,  256, KIND_TMAT2,  16, 256, 2, 1)      \
    X(float,  256, KIND_TMAT3,  16, 256, 1, 1)      \
    X(float,  256, KIND_TMATI,  16, 256, 2, 1)      \
    X(float,  512, KIND_TMAT2,   8, 256, 2, 1)      \
    X(float,  512, KIND_TMAT3,   8, 256, 1, 1)      \
    X(float,  512, KIND_TMAT2,  16, 512, 1, 2)      \
    X(float,  512, KIND_TMAT2,   4, 128, 4, 1)      \
    X(float,  512, KIND_TMAT3,   4, 128, 3, 1)      \
    X(float,  512, KIND_TMAT2,   8, 128, 3, 1)      \
    X(float,  512, KIND_RPIPE,   8, 128, 4, 1)      \
    X(float,  512, KIND_TMATI,   8, 128, 3, 1)      \
    X(float,  512, KIND_TMATI,   8, 256, 2, 1)      \
    X(float,  512, KIND_TMAT2W,  8, 128, 2, 1)      \
    X(float,  512, KIND_TMAT2W,  8, 256, 2, 1)      \
    X(float,  512, KIND_TMAT2W, 16, 256, 1, 2)      \
    X(float,  768, KIND_TMAT2,   8, 256, 1, 1)      \
    X(float, 1024, KIND_TMAT2,   4, 256, 2, 1)      \
    X(float, 1024, KIND_TMAT3,   4, 256, 1, 1)      \
    X(float, 1024, KIND_TMAT2,   8, 512, 1, 1)      \
    X(float, 1024, KIND_TMAT2,   2, 128, 4, 1)      \
    X(float, 1024, KIND_TMAT3,   4, 256, 1, 2)      \
    X(float, 1024, KIND_RPIPE,   4, 256, 2, 1)      \
    X(float, 1024, KIND_TMATI,   8, 256, 1, 1)      \
    X(float, 1024, KIND_TMATI,   8, 512, 1, 1)      \
    X(float, 1024, KIND_TMAT2W,  8, 256, 1, 1)      \
    X(float, 1024, KIND_TMAT2W,  4, 128, 2, 1)      \
    X(float,  768, KIND_TMAT2,   4, 128, 3, 1)      \
    X(float,  768, KIND_TMATI,   8, 256, 2, 1)      \
    X(float,  256, KIND_TMAT2,  16, 128, 3, 2)      \
    X(float,  512, KIND_TMAT2,   8, 128, 3, 2)      \
    X(float,  512, KIND_TMAT2,   8, 256, 2, 2)      \
    X(float,  512, KIND_TMATI,   8, 128, 3, 2)      \
    X(float,  512, KIND_TMAT3,   8, 128, 2, 2)      \
    X(float, 1024, KIND_TMAT2,   4, 128, 2, 2)      \
    X(float, 1024, KIND_TMATI,   4, 128, 3, 2)      \
    X(float,   96, KIND_RPIPE,  32, 128, 3, 1)      \
    X(float,   96, KIND_RPIPE,  16, 128, 4, 1)      \
    X(float,  128, KIND_RPIPE,  16, 128, 4, 1)      \
    X(float,  128, KIND_RPIPE,  32, 256, 2, 1)      \
    X(float,  192, KIND_RPIPE,  16, 256, 2, 1)      \
    X(float,  192, KIND_RPIPE,   8, 128, 4, 1)

#define A2A_VARIANTS_F64(X)                         \
    X(double,    4, KIND_DIRECT,  4,  32, 1, 1)     \
    X(double,    8, KIND_DIRECT,  8,  32, 1, 1)     \
    X(double,    8, KIND_DIRECT,  4,  32, 1, 1)     \
    X(double,   12, KIND_DIRECT,  4,  32, 1, 1)     \
    X(double,   16, KIND_DIRECT, 16,  32, 1, 1)     \
    X(double,   16, KIND_DIRECT,  4,  32, 1, 1)     \
    X(double,   24, KIND_DIRECT,  8,  32, 1, 1)     \
    X(double,   24, KIND_DIRECT,  4,  32, 1, 1)     \
    X(double,   32, KIND_DIRECT, 16, 128, 1, 1)     \
    X(double,   32, KIND_DIRECT,  4,  32, 1, 1)     \
    X(double,   48, KIND_DIRECT,  8,  64, 1, 1)     \
    X(double,   48, KIND_DIRECT,  4,  32, 1, 1)     \
    X(double,   64, KIND_DIRECT, 32, 128, 1, 1)     \
    X(double,   64, KIND_DIRECT, 16, 128, 2, 1)     \
    X(double,   64, KIND_PIPE,   16, 128, 2, 1)     \
    X(double,   64, KIND_DIRECT,  4,  32, 1, 1)     \
    X(double,   96, KIND_DIRECT, 16, 128, 1, 1)     \
    X(double,   96, KIND_PIPE,   16, 128, 2, 1)     \
    X(double,   96, KIND_DIRECT,  4,  32, 1, 1)     \
    X(double,  128, KIND_DIRECT, 16, 128, 1, 1)     \
    X(double,  128, KIND_PIPE,   16, 256, 2, 1)     \
    X(double,  128, KIND_DIRECT,  4,  32, 1, 1)     \
    X(double,  192, KIND_DIRECT, 16, 256, 1, 1)     \
    X(double,  192, KIND_PIPE,    8, 256, 1, 1)     \
    X(double,  192, KIND_DIRECT,  4,  64, 1, 1)     \
    X(double,  256, KIND_DIRECT, 16, 256, 1, 1)     \
    X(double,  256, KIND_DIRECT,  8, 128, 2, 1)     \
    X(double,  256, KIND_PIPE,    8, 256, 1, 1)     \
    X(double,  256, KIND_DIRECT,  4,  64, 1, 1)     \
    X(double,  384, KIND_DIRECT,  8, 256, 1, 1)     \
    X(double,  384, KIND_DIRECT,  4, 128, 1, 1)     \
    X(double,  512, KIND_RPIPE,   8, 512, 1, 1)     \
    X(double,  512, KIND_DIRECT,  8, 256, 1, 1)     \
    X(double,  512, KIND_TMA,     8, 256, 1, 1)     \
    X(double,  512, KIND_DIRECT,  8, 512, 1, 1)     \
    X(double,  512, KIND_PIPE,    8, 512, 1, 1)     \
    X(double,  512, KIND_DIRECT,  4, 128, 1, 1)     \
    X(double,  768, KIND_DIRECT,  4, 192, 1, 1)     \
    X(double,  768, KIND_DIRECT,  8, 384, 1, 1)     \
    X(double, 1024, KIND_DIRECT,  8, 512, 1, 1)     \
    X(double, 1024, KIND_DIRECT,  4, 256, 1, 1)     \
    X(double,  256, KIND_TMAT2,   8, 256, 2, 1)     \
    X(double,  512, KIND_TMAT2,   4, 256, 2, 1)     \
    X(double,  512, KIND_TMATI,   4, 128, 3, 1)     \
    X(double,  512, KIND_TMAT2,   8, 512, 1, 1)     \
    X(double,  768, KIND_TMAT2,   4, 192, 1, 1)     \
    X(double,  768, KIND_TMATI,   4, 192, 2, 1)     \
    X(double,  768, KIND_TMAT2,   2, 128, 3, 1)     \
    X(double,  768, KIND_TMAT3,   2, 128, 2, 1)     \
    X(double,  512, KIND_TMAT2,   2, 128, 4, 1)     \
    X(double,  512, KIND_TMAT2W,  4, 128, 2, 1)     \
    X(double, 1024, KIND_TMAT2W,  4, 128, 1, 1)     \
    X(double, 1024, KIND_TMAT2,   4, 256, 1, 1)     \
// clang-format on                                 

template <typename T, int N, int KIND, int B, int TH, int MB, int LPT, int MODE, bool INV>
PassKernel make_pass_kernel() {
    using P = typename PlanOf<T, N, KIND>::Plan;
    PassKernel k;
    if constexpr (KIND == KIND_RPIPES) {
        static_assert(sizeof(T) == 4 && B == 8 && TH == 128 && LPT == 1 && MODE == MODE_LINE,
                      "the line-mode shuffle kernel moves 8-line complex float tiles with 128 threads");
        k.fn = reinterpret_cast<const void*>(&fft_rpipe_shfl_kernel<P, INV, MB>);
    } else if constexpr (KIND == KIND_TMAT2S) {
        static_assert(sizeof(T) == 4 && B == ShflGeom<P>::B && TH == 128 && LPT == 1 && MODE == MODE_BATCH,
                      "the shuffle ring kernel moves complex float batch tiles with 128 threads");
        k.fn = reinterpret_cast<const void*>(&fft_tmat_shfl_kernel<P, INV, MB>);
    } else if constexpr (KIND == KIND_TMAT2 || KIND == KIND_TMAT3 || KIND == KIND_TMAT2W || KIND == KIND_TMATI)
        k.fn = reinterpret_cast<const void*>(
            &fft_tmat_kernel<T, P, B, TH, MODE, INV, MB, LPT, (KIND == KIND_TMAT3 ? 3 : 2), KIND == KIND_TMATI>);
    else if constexpr (KIND == KIND_PIPE)
        k.fn = reinterpret_cast<const void*>(&fft_pipe_kernel<T, P, B, TH, MODE, INV, MB, LPT>);
    else if constexpr (KIND == KIND_TMA)
        k.fn = reinterpret_cast<const void*>(&fft_tma_kernel<T, P, B, TH, MODE, INV, MB, LPT>);
    else if constexpr (KIND == KIND_RPIPE)
        k.fn = reinterpret_cast<const void*>(&fft_rpipe_kernel<T, P, B, TH, MODE, INV, MB, LPT>);
    else
        k.fn = reinterpret_cast<const void*>(&fft_pass_kernel<T, P, B, TH, MODE, INV, MB, LPT>);
    k.kind = KIND;
    k.n = N;
    k.threads = TH;
    k.lines = B;
    k.min_blocks = MB;
    k.lpt = LPT;
    if constexpr (KIND == KIND_TMAT2 || KIND == KIND_TMAT3 || KIND == KIND_TMAT2W || KIND == KIND_TMATI ||
                  KIND == KIND_TMAT2S)
        k.smem = tmat_smem_bytes<T, P, B, MODE, LPT, (KIND == KIND_TMAT3 ? 3 : 2), KIND == KIND_TMATI>();
    else
        k.smem = pass_smem_bytes<T, P, B, MODE, KIND, LPT>();
    k.nstages = P::S;
    for (int s = 0; s < P::S; ++s) k.radix[s] = P::r[s];
    k.twtotal = P::twtotal();
    return k;
}

// Line pairs (LPT = 2) and TMA row copies exist only for the batch mode; in
// line mode the lookup skips those variants.
template <typename T, int N, int KIND, int B, int TH, int MB, int LPT>
bool make_variant(int mode, bool inv, PassKernel* out) {
    if constexpr (KIND == KIND_RPIPES) {  // line mode only
        if (mode != MODE_LINE) return false;
        *out = inv ? make_pass_kernel<T, N, KIND, B, TH, MB, 1, MODE_LINE, true>()
                   : make_pass_kernel<T, N, KIND, B, TH, MB, 1, MODE_LINE, false>();
        return true;
    } else {
        if (mode == MODE_LINE) {
            if constexpr (LPT != 1 || KIND == KIND_TMA || KIND == KIND_TMAT2S) {
                return false;
            } else {
                *out = inv ? make_pass_kernel<T, N, KIND, B, TH, MB, 1, MODE_LINE, true>()
                           : make_pass_kernel<T, N, KIND, B, TH, MB, 1, MODE_LINE, false>();
                return true;
            }
        }
        *out = inv ? make_pass_kernel<T, N, KIND, B, TH, MB, LPT, MODE_BATCH, true>()
                   : make_pass_kernel<T, N, KIND, B, TH, MB, LPT, MODE_BATCH, false>();
        return true;
    }
}

// Defined in fft_pass_f32.cu / fft_pass_f64.cu: fills up to `max` variants of
// length n (default first) and returns how many exist (0: n not compiled).
int find_pass_kernels_f32(int n, int mode, bool inverse, PassKernel* out, int max);
int find_pass_kernels_f64(int n, int mode, bool inverse, PassKernel* out, int max);

constexpr int kMaxVariants = 32;

// fft_tc.cu: the split-precision tensor-core kernel of length n (fmt 0 =
// fp16, 1 = bf16); false when n has none.
bool find_tc_kernel(int n, int mode, bool inverse, int fmt, PassKernel* out);
// the persistent TMA-ring form of it, where the plan has one (not 256)
bool find_tc_ring_kernel(int n, int mode, bool inverse, int fmt, PassKernel* out);
// the two-stage tensor-core form (512 = 16 x 32, 1024 = 32 x 32: radix-R0
// GEMM, twiddle, radix-32 GEMM), fed by the TMA ring; its operand is
// tc2_b_bytes<n>(fmt) bytes per direction and its twiddle table W_n^(b k1)
// laid out [b < 32][k1 < n / 32].  wide: the 8-line, 512-thread tiles of
// 1024 (else 8 lines at 512, 4 at 1024)
bool find_tc2_kernel(int n, int mode, bool inverse, int fmt, bool wide, PassKernel* out);
// its software-pipelined form (fp16; 512 with 8-line, 1024 with 4-line tiles):
// the same tables
bool find_tc2p_kernel(int n, int mode, bool inverse, int fmt, PassKernel* out);

}  // namespace a2a
