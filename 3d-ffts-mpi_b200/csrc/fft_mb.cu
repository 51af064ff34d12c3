// Instantiations of the multi-block pass kernel (one tile configuration per
// length and precision, both access modes and directions) and their lookup.
#include "fft_mb.cuh"
#include "internal.h"

namespace a2a {

template <typename T, int N, int B, int TH, int MB, int MODE, bool INV> PassKernel make_mb_kernel() {
    using P = typename PassPlan<T, N>::Plan;
    PassKernel k;
    k.fn = reinterpret_cast<const void*>(&fft_mb_kernel<T, P, B, TH, MODE, INV, MB>);
    k.kind = KIND_DIRECT;
    k.n = N;
    k.threads = TH;
    k.lines = B;
    k.min_blocks = MB;
    k.lpt = 1;
    k.smem = mb_smem_bytes<T, P, B, MODE>();
    k.nstages = P::S;
    for (int s = 0; s < P::S; ++s) k.radix[s] = P::r[s];
    k.twtotal = P::twtotal();
    return k;
}

template <typename T, int N, int B, int TH, int MB, int LPT, int MODE, bool INV> PassKernel make_mb_rpipe_kernel() {
    using P = typename PassPlan<T, N>::Plan;
    PassKernel k;
    k.fn = reinterpret_cast<const void*>(&fft_mb_rpipe_kernel<T, P, B, TH, MODE, INV, MB, LPT>);
    k.kind = KIND_RPIPE;
    k.n = N;
    k.threads = TH;
    k.lines = B;
    k.min_blocks = MB;
    k.lpt = LPT;
    k.smem = pass_smem_bytes<T, P, B, MODE, KIND_RPIPE, LPT>();
    k.nstages = P::S;
    for (int s = 0; s < P::S; ++s) k.radix[s] = P::r[s];
    k.twtotal = P::twtotal();
    return k;
}

template <typename T, int N, int B, int TH, int MB> PassKernel mb_pick(int mode, bool inv) {
    if (mode == MODE_LINE)
        return inv ? make_mb_kernel<T, N, B, TH, MB, MODE_LINE, true>() : make_mb_kernel<T, N, B, TH, MB, MODE_LINE, false>();
    return inv ? make_mb_kernel<T, N, B, TH, MB, MODE_BATCH, true>() : make_mb_kernel<T, N, B, TH, MB, MODE_BATCH, false>();
}

// (N, lines, threads, min blocks) per precision: the one-tile configurations
// of the single-buffer registry (multi-stage plans only)
#define A2A_MB_F32(X)                                                                                              \
    X(12, 4, 32, 1) X(24, 8, 32, 1) X(32, 32, 128, 1) X(48, 16, 64, 1) X(64, 32, 128, 1) X(96, 32, 128, 1)       \
    X(128, 32, 256, 1) X(192, 32, 256, 1) X(256, 16, 256, 2) X(384, 16, 256, 1) X(512, 8, 128, 4)                \
    X(768, 8, 256, 1) X(1024, 8, 512, 1)
#define A2A_MB_F64(X)                                                                                              \
    X(12, 4, 32, 1) X(24, 8, 32, 1) X(32, 16, 128, 1) X(48, 8, 64, 1) X(64, 32, 128, 1) X(96, 16, 128, 1)        \
    X(128, 16, 128, 1) X(192, 16, 256, 1) X(256, 16, 256, 1) X(384, 8, 256, 1) X(512, 8, 256, 1)                 \
    X(768, 4, 192, 1) X(1024, 8, 512, 1)

// 4-line tiles for passes whose line counts the configurations above do not divide
#define A2A_MB_SMALL(X)                                                                                            \
    X(12, 4, 64, 1) X(24, 4, 64, 1) X(32, 4, 64, 1) X(48, 4, 64, 1) X(64, 4, 64, 1) X(96, 4, 64, 1)              \
    X(128, 4, 64, 1) X(192, 4, 64, 1) X(256, 4, 128, 1) X(384, 4, 128, 1) X(512, 4, 128, 1)                      \
    X(768, 4, 128, 1) X(1024, 4, 128, 1)

// Persistent register-pipelined configurations (N, lines, threads, min
// blocks, lines per thread in batch mode): the single-buffer registry's
// register-pipelined tiles for the long lengths.
// Line mode (the Z pass) only: at 512^3 on one GPU the persistent body took
// the Z pass from 0.50 to 0.46 ms but was slower than one tile per CTA in
// batch mode (X, Y: 0.60-0.65 vs 0.57 ms), so batch-mode passes keep the
// one-tile body.
#define A2A_MB_RPIPE_F32(X) \
    X(256, 16, 256, 2, 1) X(512, 8, 256, 2, 1) X(1024, 4, 256, 2, 1)
#define A2A_MB_RPIPE_F64(X) \
    X(512, 8, 512, 1, 1) X(1024, 4, 256, 1, 1)

bool find_mb_rpipe_kernel(a2a_precision prec, int n, int mode, bool inverse, PassKernel* out) {
#define A2A_MB_CASE(T_, N_, B_, TH_, MB_, LPT_)                                                              \
    if (n == N_) {                                                                                          \
        if (mode == MODE_LINE)                                                                              \
            *out = inverse ? make_mb_rpipe_kernel<T_, N_, B_, TH_, MB_, 1, MODE_LINE, true>()               \
                           : make_mb_rpipe_kernel<T_, N_, B_, TH_, MB_, 1, MODE_LINE, false>();             \
        else                                                                                                \
            *out = inverse ? make_mb_rpipe_kernel<T_, N_, B_, TH_, MB_, LPT_, MODE_BATCH, true>()           \
                           : make_mb_rpipe_kernel<T_, N_, B_, TH_, MB_, LPT_, MODE_BATCH, false>();         \
        return true;                                                                                        \
    }
#define A2A_MB_F32_CASE(N_, B_, TH_, MB_, LPT_) A2A_MB_CASE(float, N_, B_, TH_, MB_, LPT_)
#define A2A_MB_F64_CASE(N_, B_, TH_, MB_, LPT_) A2A_MB_CASE(double, N_, B_, TH_, MB_, LPT_)
    if (mode != MODE_LINE) return false;
    if (prec == A2A_C128) {
        A2A_MB_RPIPE_F64(A2A_MB_F64_CASE)
    } else {
        A2A_MB_RPIPE_F32(A2A_MB_F32_CASE)
    }
#undef A2A_MB_F32_CASE
#undef A2A_MB_F64_CASE
#undef A2A_MB_CASE
    return false;
}

// Batch-mode passes fed by TMA from per-rank tensor maps (N, lines, threads,
// min blocks): the single-buffer ring kernel's tiles.
template <typename T, int N, int B, int TH, int MB, bool INV> PassKernel make_mb_tmat_kernel() {
    using P = typename PassPlan<T, N>::Plan;
    PassKernel k;
    k.fn = reinterpret_cast<const void*>(&fft_mb_tmat_kernel<T, P, B, TH, INV, MB>);
    k.kind = KIND_TMAT2;
    k.n = N;
    k.threads = TH;
    k.lines = B;
    k.min_blocks = MB;
    k.lpt = 1;
    k.smem = mb_tmat_smem_bytes<T, P, B>();
    k.nstages = P::S;
    for (int s = 0; s < P::S; ++s) k.radix[s] = P::r[s];
    k.twtotal = P::twtotal();
    return k;
}
#define A2A_MB_TMAT_F32(X) X(256, 16, 256, 2) X(512, 8, 128, 2) X(1024, 4, 256, 2)
#define A2A_MB_TMAT_F64(X) X(512, 4, 256, 2) X(1024, 4, 256, 1)

bool find_mb_tmat_kernel(a2a_precision prec, int n, bool inverse, PassKernel* out) {
#define A2A_MB_CASE(T_, N_, B_, TH_, MB_)                                                                   \
    if (n == N_) {                                                                                          \
        *out = inverse ? make_mb_tmat_kernel<T_, N_, B_, TH_, MB_, true>()                                  \
                       : make_mb_tmat_kernel<T_, N_, B_, TH_, MB_, false>();                                \
        return true;                                                                                        \
    }
#define A2A_MB_F32_CASE(N_, B_, TH_, MB_) A2A_MB_CASE(float, N_, B_, TH_, MB_)
#define A2A_MB_F64_CASE(N_, B_, TH_, MB_) A2A_MB_CASE(double, N_, B_, TH_, MB_)
    if (prec == A2A_C128) {
        A2A_MB_TMAT_F64(A2A_MB_F64_CASE)
    } else {
        A2A_MB_TMAT_F32(A2A_MB_F32_CASE)
    }
#undef A2A_MB_F32_CASE
#undef A2A_MB_F64_CASE
#undef A2A_MB_CASE
    return false;
}

bool find_mb_kernel_small(a2a_precision prec, int n, int mode, bool inverse, PassKernel* out) {
#define A2A_MB_CASE(N_, B_, TH_, MB_)                                                                       \
    if (n == N_) {                                                                                          \
        *out = prec == A2A_C128 ? mb_pick<double, N_, B_, TH_, MB_>(mode, inverse)                           \
                                : mb_pick<float, N_, B_, TH_, MB_>(mode, inverse);                           \
        return true;                                                                                        \
    }
    A2A_MB_SMALL(A2A_MB_CASE)
#undef A2A_MB_CASE
    return false;
}

bool find_mb_kernel(a2a_precision prec, int n, int mode, bool inverse, PassKernel* out) {
    if (prec == A2A_C128) {
#define A2A_MB_CASE(N_, B_, TH_, MB_) \
    if (n == N_) {                    \
        *out = mb_pick<double, N_, B_, TH_, MB_>(mode, inverse); \
        return true;                  \
    }
        A2A_MB_F64(A2A_MB_CASE)
#undef A2A_MB_CASE
        return false;
    }
#define A2A_MB_CASE(N_, B_, TH_, MB_) \
    if (n == N_) {                    \
        *out = mb_pick<float, N_, B_, TH_, MB_>(mode, inverse); \
        return true;                  \
    }
    A2A_MB_F32(A2A_MB_CASE)
#undef A2A_MB_CASE
    return false;
}

}  // namespace a2a
