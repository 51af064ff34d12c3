// Kernels of the a2aDistribution steps over virtual ranks: the alltoall as a
// rank-major chunk permutation, the pack/unpack pencil remaps and the
// fast-axis changes.  They reproduce, element for element, what the reference
// leaves in both buffers after each of its six steps
// (src/a2afft/distribution/a2adistribution.cpp:115-215).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace a2a {

// Division of 32-bit unsigned integers by a run-time invariant divisor with
// one multiply-high, one add and one shift (Granlund & Montgomery, "Division
// by invariant integers using multiplication", PLDI 1994, section 4):
// l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1, q = (mulhi(m, n) + n) >> l,
// with the add done in 64 bits so no n overflows.
struct FastDiv {
    uint32_t d = 1, m = 1, l = 0;
    FastDiv() = default;
    explicit FastDiv(uint32_t dv) : d(dv) {
        l = 0;
        while ((uint64_t(1) << l) < dv) ++l;
        m = uint32_t(((uint64_t(1) << 32) * ((uint64_t(1) << l) - dv)) / dv + 1);
    }
    __host__ __device__ __forceinline__ uint32_t div(uint32_t n) const {
#ifdef __CUDA_ARCH__
        const uint32_t hi = __umulhi(m, n);
#else
        const uint32_t hi = uint32_t((uint64_t(m) * n) >> 32);
#endif
        return uint32_t((uint64_t(hi) + n) >> l);
    }
    __host__ __device__ __forceinline__ void divmod(uint32_t n, uint32_t& q, uint32_t& r) const {
        q = div(n);
        r = n - q * d;
    }
};

// Geometry of one axis's pencil exchange.  Rank q's received buffer holds, for
// every sender r, `m` mini-pencils of `la` elements (chunk = m * la); the
// unpack joins the senders of one group into full pencils of `ng` elements.
struct PencilGeom {
    int axis;          // 0 = x, 1 = y, 2 = z
    int d0, d1, d2;    // brick grid
    uint32_t nlocal;   // elements per rank
    uint32_t chunk;    // nlocal / P
    uint32_t la;       // brick extent along the axis
    uint32_t ng;       // global extent along the axis
    uint32_t m;        // mini-pencils per chunk
    FastDiv f_nlocal, f_ng, f_m, f_la, f_d2;
};

// Sender rank of pencil group s and axis coordinate ca (the inverse of the
// grouping the reference's unpack kernels use: z groups ranks by (c0, c1),
// x by (c1, c2), y by (c0, c2)).
__device__ __forceinline__ uint32_t pencil_sender(const PencilGeom& g, uint32_t s, uint32_t ca) {
    if (g.axis == 2) return s * g.d2 + ca;                               // s = c0 d1 + c1, ca = c2
    if (g.axis == 0) return ca * uint32_t(g.d1 * g.d2) + s;              // s = c1 d2 + c2, ca = c0
    uint32_t c0, c2;                                                     // y: s = c0 d2 + c2, ca = c1
    g.f_d2.divmod(s, c0, c2);
    return (c0 * g.d1 + ca) * g.d2 + c2;
}

}  // namespace a2a
