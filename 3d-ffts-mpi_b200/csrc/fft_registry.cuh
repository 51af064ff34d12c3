// Compiled transform lengths and their launch shapes, and the host-side
// lookup of a pass kernel for (precision, N, mode, direction).
#pragma once

#include <cstddef>
#include <cuda_runtime.h>

#include "fft_tile.cuh"

namespace a2a {

// Host view of one compiled pass kernel.
struct PassKernel {
    const void* fn = nullptr;
    int n = 0;          // transform length
    int threads = 0;
    int lines = 0;      // B: lines per tile (a pass needs NV % lines == 0)
    size_t smem = 0;    // dynamic shared memory bytes
    int nstages = 0;
    int radix[4] = {0, 0, 0, 0};
    int twtotal = 0;    // complex entries of the twiddle table
};

// Launch shape per (element type, N): radix plan, lines per tile, threads.
// Tiles are ~64 KB so two or three CTAs share an SM; FP64 holds half the
// elements per thread of FP32 to stay within registers.
template <typename T, int N> struct PassCfg;

#define A2A_PASS_CFG(T_, N_, B_, TH_, ...)                                  \
    template <> struct PassCfg<T_, N_> {                                    \
        using Plan = RadixPlan<__VA_ARGS__>;                                \
        static constexpr int B = B_;                                        \
        static constexpr int THREADS = TH_;                                 \
        static_assert(Plan::N == N_, "radix plan does not multiply to N");  \
    };

// clang-format off
A2A_PASS_CFG(float,    4,  4,  32, 4)
A2A_PASS_CFG(float,    8,  8,  32, 8)
A2A_PASS_CFG(float,   12,  4,  32, 3, 4)
A2A_PASS_CFG(float,   16, 16,  32, 16)
A2A_PASS_CFG(float,   24,  8,  32, 3, 8)
A2A_PASS_CFG(float,   32, 32, 128, 4, 8)
A2A_PASS_CFG(float,   48, 16,  64, 3, 16)
A2A_PASS_CFG(float,   64, 32, 128, 8, 8)
A2A_PASS_CFG(float,   96, 32, 128, 3, 4, 8)
A2A_PASS_CFG(float,  128, 32, 256, 8, 16)
A2A_PASS_CFG(float,  192, 32, 256, 3, 4, 16)
A2A_PASS_CFG(float,  256, 32, 256, 16, 16)
A2A_PASS_CFG(float,  384, 16, 256, 3, 8, 16)
A2A_PASS_CFG(float,  512, 16, 256, 8, 8, 8)
A2A_PASS_CFG(float,  768,  8, 256, 3, 16, 16)
A2A_PASS_CFG(float, 1024,  8, 256, 4, 16, 16)

A2A_PASS_CFG(double,    4,  4,  32, 4)
A2A_PASS_CFG(double,    8,  8,  32, 8)
A2A_PASS_CFG(double,   12,  4,  32, 3, 4)
A2A_PASS_CFG(double,   16, 16,  32, 16)
A2A_PASS_CFG(double,   24,  8,  32, 3, 8)
A2A_PASS_CFG(double,   32, 16, 128, 4, 8)
A2A_PASS_CFG(double,   48,  8,  64, 3, 16)
A2A_PASS_CFG(double,   64, 32, 128, 8, 8)
A2A_PASS_CFG(double,   96, 16, 128, 3, 4, 8)
A2A_PASS_CFG(double,  128, 16, 128, 8, 16)
A2A_PASS_CFG(double,  192, 16, 256, 3, 4, 16)
A2A_PASS_CFG(double,  256, 16, 256, 16, 16)
A2A_PASS_CFG(double,  384,  8, 256, 3, 8, 16)
A2A_PASS_CFG(double,  512,  8, 256, 8, 8, 8)
A2A_PASS_CFG(double,  768,  8, 384, 3, 16, 16)
A2A_PASS_CFG(double, 1024,  8, 512, 4, 16, 16)
// clang-format on

#define A2A_FOR_EACH_N(X) \
    X(4) X(8) X(12) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) X(512) X(768) X(1024)

template <typename T, int N, int MODE, bool INV> PassKernel make_pass_kernel() {
    using C = PassCfg<T, N>;
    using P = typename C::Plan;
    PassKernel k;
    k.fn = reinterpret_cast<const void*>(&fft_pass_kernel<T, P, C::B, C::THREADS, MODE, INV>);
    k.n = N;
    k.threads = C::THREADS;
    k.lines = C::B;
    k.smem = pass_smem_bytes<T, P, C::B, MODE>();
    k.nstages = P::S;
    for (int s = 0; s < P::S; ++s) k.radix[s] = P::r[s];
    k.twtotal = P::twtotal();
    return k;
}

// Defined in fft_pass_f32.cu / fft_pass_f64.cu.  Returns false when N has no
// compiled kernel.
bool find_pass_kernel_f32(int n, int mode, bool inverse, PassKernel* out);
bool find_pass_kernel_f64(int n, int mode, bool inverse, PassKernel* out);

}  // namespace a2a
