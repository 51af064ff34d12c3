// Pass-kernel instantiations for complex float: every launch variant of every
// compiled N, both access modes, both directions, and their lookup.
#include "fft_registry.cuh"

namespace a2a {

int find_pass_kernels_f32(int n, int mode, bool inverse, PassKernel* out, int max) {
    int cnt = 0;
#define A2A_ADD(T_, N_, KIND_, B_, TH_, MB_, LPT_)                                     \
    if (n == N_) {                                                                     \
        PassKernel k_;                                                                 \
        if (make_variant<T_, N_, KIND_, B_, TH_, MB_, LPT_>(mode, inverse, &k_)) {      \
            if (cnt < max) out[cnt] = k_;                                              \
            ++cnt;                                                                     \
        }                                                                              \
    }
    A2A_VARIANTS_F32(A2A_ADD)
#undef A2A_ADD
    return cnt;
}

}  // namespace a2a
