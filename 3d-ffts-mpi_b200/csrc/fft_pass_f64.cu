// Pass-kernel instantiations for complex double (every compiled N, both access
// modes, both directions) and their lookup.
#include "fft_registry.cuh"

namespace a2a {

bool find_pass_kernel_f64(int n, int mode, bool inverse, PassKernel* out) {
#define A2A_CASE(N_)                                                                    \
    case N_:                                                                            \
        if (mode == MODE_LINE)                                                          \
            *out = inverse ? make_pass_kernel<double, N_, MODE_LINE, true>()              \
                           : make_pass_kernel<double, N_, MODE_LINE, false>();            \
        else                                                                            \
            *out = inverse ? make_pass_kernel<double, N_, MODE_BATCH, true>()             \
                           : make_pass_kernel<double, N_, MODE_BATCH, false>();           \
        return true;
    switch (n) {
        A2A_FOR_EACH_N(A2A_CASE)
        default:
            return false;
    }
#undef A2A_CASE
}

}  // namespace a2a
