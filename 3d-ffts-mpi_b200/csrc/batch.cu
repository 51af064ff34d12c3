// Instantiations of the batched persistent kernel (both precisions, both
// directions) and their host lookup.
#include "batch.cuh"
#include "internal.h"

namespace a2a {

const void* batch_kernel(a2a_precision prec, bool inverse) {
    if (prec == A2A_C128)
        return inverse ? reinterpret_cast<const void*>(&fft_batch_kernel<double, true>)
                       : reinterpret_cast<const void*>(&fft_batch_kernel<double, false>);
    return inverse ? reinterpret_cast<const void*>(&fft_batch_kernel<float, true>)
                   : reinterpret_cast<const void*>(&fft_batch_kernel<float, false>);
}

size_t batch_smem(a2a_precision prec) {
    return prec == A2A_C128 ? batch_smem_bytes<double>() : batch_smem_bytes<float>();
}

int batch_tile_lines(a2a_precision prec, int n, int variant) {
    if (variant < 0 || variant >= kBatchVariants) return 0;
    for (int i = 0; i < kBatchNumLengths; ++i)
        if (kBatchLengths[i] == n) return prec == A2A_C128 ? batch_lines<double>(n, variant) : batch_lines<float>(n, variant);
    return 0;
}

template <typename T> static size_t tile_smem(int n, int v, int mode) {
#define A2A_TS(N_)                                                                                         \
    if (n == N_) {                                                                                         \
        using P = typename PassPlan<T, N_>::Plan;                                                          \
        if (mode == MODE_LINE)                                                                             \
            return v == 1 ? pass_smem_bytes<T, P, batch_lines<T>(N_, 1), MODE_LINE, KIND_DIRECT, 1>()      \
                          : pass_smem_bytes<T, P, batch_lines<T>(N_, 0), MODE_LINE, KIND_DIRECT, 1>();     \
        if (v == 2)                                                                                        \
            return pass_smem_bytes<T, P, batch_lines<T>(N_, 2), MODE_BATCH, KIND_DIRECT,                   \
                                   batch_lpt<T>(2, MODE_BATCH)>();                                         \
        return v == 1 ? pass_smem_bytes<T, P, batch_lines<T>(N_, 1), MODE_BATCH, KIND_DIRECT, 1>()         \
                      : pass_smem_bytes<T, P, batch_lines<T>(N_, 0), MODE_BATCH, KIND_DIRECT, 1>();        \
    }
    A2A_BATCH_FOR_EACH_N(A2A_TS)
#undef A2A_TS
    return 0;
}

size_t batch_tile_smem(a2a_precision prec, int n, int variant, int mode) {
    return prec == A2A_C128 ? tile_smem<double>(n, variant, mode) : tile_smem<float>(n, variant, mode);
}

}  // namespace a2a
