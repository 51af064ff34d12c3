// Instantiations of the split-precision tensor-core pass kernels and their
// lookup.  Lengths whose plan ends in radix-16 stages: every stage after the
// first is a tensor-core GEMM.
#include "fft_tc.cuh"
#include "fft_tc2.cuh"
#include "internal.h"

namespace a2a {

template <int N> struct TcPlan;
template <> struct TcPlan<64> { using Plan = RadixPlan<4, 16>; static constexpr int B = 32; };
template <> struct TcPlan<128> { using Plan = RadixPlan<8, 16>; static constexpr int B = 16; };
template <> struct TcPlan<256> { using Plan = RadixPlan<16, 16>; static constexpr int B = 16; };
template <> struct TcPlan<512> { using Plan = RadixPlan<2, 16, 16>; static constexpr int B = 8; };
template <> struct TcPlan<1024> { using Plan = RadixPlan<4, 16, 16>; static constexpr int B = 4; };

// Tile height: bf16 rows take 80 tensor-memory columns per 128-row block (three
// A parts), so its 256-thread tiles are halved to one block (128 columns per
// CTA, four CTAs per SM instead of two) where that still leaves whole blocks.
template <int N, int FMT> constexpr int tc_lines() {
    constexpr int B = TcPlan<N>::B;
    return (FMT == TC_BF16 && B * N / 16 >= 2 * kTcRows) ? B / 2 : B;
}

template <int N, int MODE, bool INV, int FMT, bool RING> PassKernel make_tc_kernel() {
    using P = typename TcPlan<N>::Plan;
    constexpr int B = tc_lines<N, FMT>();
    PassKernel k;
    if constexpr (RING) {
        k.fn = reinterpret_cast<const void*>(&fft_tc_ring_kernel<P, B, MODE, INV, FMT>);
        k.kind = KIND_TCR;
        k.smem = tc_ring_smem_bytes<P, B, MODE, FMT>();
    } else {
        k.fn = reinterpret_cast<const void*>(&fft_tc_kernel<P, B, MODE, INV, FMT>);
        k.kind = KIND_TC;
        k.smem = tc_smem_bytes<P, B, MODE, FMT>();
    }
    k.n = N;
    k.threads = B * N / 16;
    k.lines = B;
    k.min_blocks = 1;
    k.lpt = 1;
    k.nstages = P::S;
    for (int s = 0; s < P::S; ++s) k.radix[s] = P::r[s];
    k.twtotal = P::twtotal();
    return k;
}

template <int N, bool RING> PassKernel tc_pick(int mode, bool inv, int fmt) {
    if (mode == MODE_LINE) {
        if (fmt == TC_FP16)
            return inv ? make_tc_kernel<N, MODE_LINE, true, TC_FP16, RING>() : make_tc_kernel<N, MODE_LINE, false, TC_FP16, RING>();
        return inv ? make_tc_kernel<N, MODE_LINE, true, TC_BF16, RING>() : make_tc_kernel<N, MODE_LINE, false, TC_BF16, RING>();
    }
    if (fmt == TC_FP16)
        return inv ? make_tc_kernel<N, MODE_BATCH, true, TC_FP16, RING>() : make_tc_kernel<N, MODE_BATCH, false, TC_FP16, RING>();
    return inv ? make_tc_kernel<N, MODE_BATCH, true, TC_BF16, RING>() : make_tc_kernel<N, MODE_BATCH, false, TC_BF16, RING>();
}

bool find_tc_kernel(int n, int mode, bool inverse, int fmt, PassKernel* out) {
    switch (n) {
        case 64: *out = tc_pick<64, false>(mode, inverse, fmt); return true;
        case 128: *out = tc_pick<128, false>(mode, inverse, fmt); return true;
        case 256: *out = tc_pick<256, false>(mode, inverse, fmt); return true;
        case 512: *out = tc_pick<512, false>(mode, inverse, fmt); return true;
        case 1024: *out = tc_pick<1024, false>(mode, inverse, fmt); return true;
        default: return false;
    }
}

// Lengths whose tensor-core plan starts with a CUDA-core stage have a ring
// form (256 = 16 x 16 has none).
bool find_tc_ring_kernel(int n, int mode, bool inverse, int fmt, PassKernel* out) {
    switch (n) {
        case 64: *out = tc_pick<64, true>(mode, inverse, fmt); return true;
        case 128: *out = tc_pick<128, true>(mode, inverse, fmt); return true;
        case 512: *out = tc_pick<512, true>(mode, inverse, fmt); return true;
        case 1024: *out = tc_pick<1024, true>(mode, inverse, fmt); return true;
        default: return false;
    }
}

template <int N, int BL, int MODE, bool INV, int FMT> PassKernel make_tc2_kernel() {
    using G = Tc2Geom<N, BL>;
    PassKernel k;
    k.fn = reinterpret_cast<const void*>(&fft_tc2_ring_kernel<N, BL, MODE, INV, FMT>);
    k.kind = KIND_TC2;
    k.smem = tc2_smem_bytes<N, BL>(FMT);
    k.n = N;
    k.threads = G::THREADS;
    k.lines = G::B;
    k.min_blocks = G::THREADS == 512 ? 1 : 2;
    k.lpt = 1;
    k.nstages = 2;
    k.radix[0] = G::R0;
    k.radix[1] = 32;
    k.twtotal = G::TW;
    return k;
}

template <int N, int BL> PassKernel tc2_pick(int mode, bool inverse, int fmt) {
#define A2A_TC2(M_, F_) \
    return inverse ? make_tc2_kernel<N, BL, M_, true, F_>() : make_tc2_kernel<N, BL, M_, false, F_>()
    if (mode == MODE_LINE) {
        if (fmt == TC_FP16) A2A_TC2(MODE_LINE, TC_FP16); else A2A_TC2(MODE_LINE, TC_BF16);
    } else {
        if (fmt == TC_FP16) A2A_TC2(MODE_BATCH, TC_FP16); else A2A_TC2(MODE_BATCH, TC_BF16);
    }
#undef A2A_TC2
}

template <int N, int BL> PassKernel tc2p_pick(int mode, bool inverse) {
    using G = Tc2Geom<N, BL>;
    PassKernel k;
    if (mode == MODE_LINE)
        k.fn = inverse ? reinterpret_cast<const void*>(&fft_tc2p_ring_kernel<N, BL, MODE_LINE, true>)
                       : reinterpret_cast<const void*>(&fft_tc2p_ring_kernel<N, BL, MODE_LINE, false>);
    else
        k.fn = inverse ? reinterpret_cast<const void*>(&fft_tc2p_ring_kernel<N, BL, MODE_BATCH, true>)
                       : reinterpret_cast<const void*>(&fft_tc2p_ring_kernel<N, BL, MODE_BATCH, false>);
    k.kind = KIND_TC2;
    k.smem = tc2p_smem_bytes<N, BL>();
    k.n = N;
    k.threads = G::THREADS;
    k.lines = G::B;
    k.min_blocks = 2;
    k.lpt = 1;
    k.nstages = 2;
    k.radix[0] = G::R0;
    k.radix[1] = 32;
    k.twtotal = G::TW;
    return k;
}

bool find_tc2p_kernel(int n, int mode, bool inverse, int fmt, PassKernel* out) {
    if (fmt != TC_FP16) return false;
    if (n == 512) { *out = tc2p_pick<512, 8>(mode, inverse); return true; }
    if (n == 1024) { *out = tc2p_pick<1024, 4>(mode, inverse); return true; }
    return false;
}

bool find_tc2_kernel(int n, int mode, bool inverse, int fmt, bool wide, PassKernel* out) {
    if (n == 512 && !wide) { *out = tc2_pick<512, 8>(mode, inverse, fmt); return true; }
    if (n == 1024) { *out = wide ? tc2_pick<1024, 8>(mode, inverse, fmt) : tc2_pick<1024, 4>(mode, inverse, fmt); return true; }
    return false;
}

}  // namespace a2a
