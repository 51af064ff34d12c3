// Host-side state shared by the translation units of liba2afft_b200.
#pragma once

#include <cstdint>
#include <vector>
#include <cuda_runtime.h>

#include "../../include/a2afft_b200.h"
#include "fft_registry.cuh"

namespace a2a {

// The kernel choice for one use of a pass (one axis, one direction): every
// compiled variant of its length, which of them fit the pass geometry, and the
// one in use.
struct PassSlot {
    PassKernel cand[kMaxVariants];
    int occ[kMaxVariants] = {0};       // resident CTAs per SM
    bool fits[kMaxVariants] = {false};
    float tuned_ms[kMaxVariants] = {0};  // make_plans timings (0 = not timed)
    const void* tw[kMaxVariants] = {nullptr};  // own twiddle table (a candidate with another radix plan)
    int ncand = 0;
    int chosen = 0;
    const PassKernel& k() const { return cand[chosen]; }
};

enum SlotId { SLOT_Z = 0, SLOT_X = 1, SLOT_Y = 2, SLOT_LINES = 3, NSLOTS = 4 };

// Tensor maps of one axis pass for the buffer they were last built for.
struct TmatEntry {
    const void* ptr = nullptr;
    int lines = 0;
    TmatMaps maps;
};

// Everything an a2aDistribution carries, for all virtual ranks at once.
struct Dist {
    int ng[3] = {0, 0, 0};
    int P = 0;
    // virtual ranks held in the caller's buffers: [first_rank, first_rank +
    // local_ranks); all P unless a2a_distribution_set_rank_range narrowed it
    int first_rank = 0;
    int local_ranks = 0;
    int dims[3] = {0, 0, 0};
    int local[3] = {0, 0, 0};
    uint64_t nlocal = 0;
    uint64_t chunk = 0;  // nsends = nlocal / P
    int block_size = 0;
    a2a_precision prec = A2A_C128;
    size_t elem_bytes = 16;
    bool cube = true;
    cudaStream_t stream = nullptr;
    int device = 0;
    int sms = 148;

    // device tables (one allocation): brick offsets per axis, identity
    // offsets and the pencil-buffer line bases (cubes only)
    uint32_t* d_tables = nullptr;
    const uint32_t* off[3] = {nullptr, nullptr, nullptr};
    const uint32_t* iota = nullptr;
    const uint32_t* pen_u = nullptr;
    const uint32_t* pen_v = nullptr;
    int* d_err = nullptr;  // set by a kernel whose bounded wait gave up
    // FP64-generated stage twiddles per axis (forward sign), in the
    // precision of the plan
    void* d_tw = nullptr;
    const void* tw[3] = {nullptr, nullptr, nullptr};
    void* d_tw2 = nullptr;  // twiddle tables of candidates with another radix plan
    // host copies of the offset tables (geometry checks)
    std::vector<uint32_t> h_off[3];
    // pass kernels: [slot][inverse]
    PassSlot slot[NSLOTS][2];
    // tensor maps of the TMA-ring pass kernels, per axis pass (Z, X, Y)
    mutable TmatEntry tmat[3];
};

// remap.cu
cudaError_t launch_alltoall(const Dist& d, const void* src, void* dst, cudaStream_t st);
cudaError_t launch_pencil_remap(const Dist& d, int axis, bool unpack, const void* src, void* dst, cudaStream_t st);
cudaError_t launch_fast_axis(const Dist& d, int which, const void* src, void* dst, cudaStream_t st);
cudaError_t launch_scale(const Dist& d, const void* src, void* dst, double divisor, cudaStream_t st);

// api.cu: records "<what>: <detail>" for a2a_last_error and returns s
a2a_status record_error(a2a_status s, const char* what, const char* detail);

// fft_mb.cu: the multi-block pass kernel of length n (one configuration);
// false for lengths with a single-stage plan (4 8 16) or none
bool find_mb_kernel(a2a_precision prec, int n, int mode, bool inverse, PassKernel* out);
bool find_mb_kernel_small(a2a_precision prec, int n, int mode, bool inverse, PassKernel* out);  // 4-line tiles
// the persistent register-pipelined multi-block kernel of length n, where compiled
bool find_mb_rpipe_kernel(a2a_precision prec, int n, int mode, bool inverse, PassKernel* out);
// the batch-mode multi-block kernel fed by TMA from per-rank tensor maps
bool find_mb_tmat_kernel(a2a_precision prec, int n, bool inverse, PassKernel* out);

// batch.cu: the batched persistent kernel per (precision, direction), its
// dynamic shared memory, and the tile height of a length's variant (0: the
// length has no batched tile code)
const void* batch_kernel(a2a_precision prec, bool inverse);
size_t batch_smem(a2a_precision prec);
int batch_tile_lines(a2a_precision prec, int n, int variant);
size_t batch_tile_smem(a2a_precision prec, int n, int variant, int mode);

}  // namespace a2a
