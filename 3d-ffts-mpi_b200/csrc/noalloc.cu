// a2a_lines_fft_noalloc: batched 1D transforms of contiguous lines that
// allocate no device memory.
//
// Who needs this: callers that cannot call cudaMalloc.  A host application
// whose own memory manager reserved the device's memory up front cannot let
// a library allocate behind its back (the allocation fails, or fragments the
// pool it manages), and code on a latency-bound path cannot afford
// cudaMalloc's implicit device-wide synchronisation.  Every other transform
// here needs a distribution object, whose creation allocates offset and
// twiddle tables.  This entry point instead keeps its tables in one
// file-scope device array of fixed size, which every GPU that loads the
// library holds until the process exits.
//
// The tables are rebuilt in that array by a small kernel on the caller's
// stream at every call, followed by the same pass kernel that
// a2a_forward_1d_fft / a2a_inverse_1d_fft launch.  All calls share the
// array, so calls whose work overlaps on the GPU (different streams, or
// different host threads) race; calls ordered on one stream do not.
#include <mutex>

#include "internal.h"

using namespace a2a;

namespace {

constexpr size_t kScratchBytes = size_t(256) << 10;  // A2A_LINES_NOALLOC_SCRATCH_BYTES
static_assert(kScratchBytes == A2A_LINES_NOALLOC_SCRATCH_BYTES, "header and library disagree on the scratch size");
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_lines_scratch[kScratchBytes];

// Device address of g_lines_scratch per device, resolved once per device
// (with that device current) by the first call made on it.
std::mutex g_mutex;
void* g_scratch_ptr[kMaxDevices] = {};
// kernels whose dynamic shared-memory limit is already raised, per device
// (a host round trip saved on every later call)
constexpr int kMaxAttrFns = 64;
const void* g_attr_fn[kMaxDevices][kMaxAttrFns] = {};

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct Layout {
    size_t tw, offA, offU, offV, end;
};

Layout layout(int n, int twtotal, int NU, int NV, size_t elem_bytes) {
    Layout l;
    l.tw = 0;
    l.offA = align256(l.tw + (size_t)twtotal * elem_bytes);
    l.offU = align256(l.offA + sizeof(uint32_t) * (size_t)n);
    l.offV = align256(l.offU + sizeof(uint32_t) * (size_t)NU);
    l.end = align256(l.offV + sizeof(uint32_t) * (size_t)NV);
    return l;
}

struct StagePlan {
    int nstages;
    int radix[4];
};

// Stage twiddles W_{Ns R}^{r m} (forward sign) in the RadixPlan::twoff
// layout, with the exponent reduced exactly before sincospi; line tables for
// contiguous lines of length n: offA[j] = j, offU[u] = u NV n, offV[v] = v n.
template <typename T>
__global__ void __launch_bounds__(256) lines_tables_kernel(unsigned char* scratch, Layout l, StagePlan p, int n,
                                                           int NU, int NV) {
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int stride = gridDim.x * blockDim.x;
    cx<T>* tw = reinterpret_cast<cx<T>*>(scratch + l.tw);
    int base = 0, ns = p.radix[0];
    for (int s = 1; s < p.nstages; ++s) {
        const int R = p.radix[s];
        const long long M = (long long)ns * R;
        const int cnt = (R - 1) * ns;
        for (int i = tid; i < cnt; i += stride) {
            const int r = 1 + i / ns, m = i % ns;
            const long long e = ((long long)r * m) % M;
            double sn, cs;
            sincospi(2.0 * (double)e / (double)M, &sn, &cs);
            tw[base + i] = mk<cx<T>>(T(cs), T(-sn));
        }
        base += cnt;
        ns *= R;
    }
    uint32_t* offA = reinterpret_cast<uint32_t*>(scratch + l.offA);
    uint32_t* offU = reinterpret_cast<uint32_t*>(scratch + l.offU);
    uint32_t* offV = reinterpret_cast<uint32_t*>(scratch + l.offV);
    for (int i = tid; i < n; i += stride) offA[i] = uint32_t(i);
    for (int i = tid; i < NU; i += stride) offU[i] = uint32_t((uint64_t)i * NV * n);
    for (int i = tid; i < NV; i += stride) offV[i] = uint32_t((uint64_t)i * n);
}

a2a_status fail(a2a_status s, const char* msg) { return a2a::record_error(s, "a2a_lines_fft_noalloc", msg); }

a2a_status cuda_fail(cudaError_t e, const char* what) {
    return a2a::record_error(A2A_ERROR_CUDA, what, cudaGetErrorName(e));
}

}  // namespace

extern "C" a2a_status a2a_lines_fft_noalloc(void* data, int n, int64_t nlines, a2a_precision precision, int inverse,
                                            void* stream) {
    if (!data) return fail(A2A_ERROR_INVALID_VALUE, "data is NULL");
    if (reinterpret_cast<uintptr_t>(data) % 16) return fail(A2A_ERROR_MISALIGNED, "data is not 16-byte aligned");
    if (precision != A2A_C128 && precision != A2A_C64) return fail(A2A_ERROR_INVALID_VALUE, "unknown precision");
    if (nlines < 1) return fail(A2A_ERROR_INVALID_VALUE, "nlines must be >= 1");
    if ((uint64_t)nlines * (uint64_t)(n > 0 ? n : 1) >= (uint64_t(1) << 32))
        return fail(A2A_ERROR_UNSUPPORTED, "nlines * n must stay below 2^32 elements");

    // the one-tile-per-CTA kernel of length n whose tile height divides nlines
    PassKernel cand[kMaxVariants];
    const int cnt = precision == A2A_C128 ? find_pass_kernels_f64(n, MODE_LINE, inverse != 0, cand, kMaxVariants)
                                          : find_pass_kernels_f32(n, MODE_LINE, inverse != 0, cand, kMaxVariants);
    if (cnt == 0)
        return fail(A2A_ERROR_UNSUPPORTED,
                    "no compiled transform of this length (4 8 12 16 24 32 48 64 96 128 192 256 384 512 768 1024)");
    int pick = -1;
    for (int c = 0; c < std::min(cnt, kMaxVariants) && pick < 0; ++c)
        if (cand[c].kind == KIND_DIRECT && nlines % cand[c].lines == 0) pick = c;
    if (pick < 0) return fail(A2A_ERROR_UNSUPPORTED, "nlines is not a multiple of 4");
    const PassKernel& k = cand[pick];

    // NV: the largest tile multiple up to 1024 that divides nlines
    int NV = k.lines;
    while (NV * 2 <= 1024 && nlines % (NV * 2) == 0) NV *= 2;
    const int64_t NU = nlines / NV;
    const size_t eb = precision == A2A_C128 ? 16 : 8;
    if (NU > (int64_t)(kScratchBytes / sizeof(uint32_t)))
        return fail(A2A_ERROR_UNSUPPORTED, "too many lines for the fixed scratch array");
    const Layout l = layout(n, k.twtotal, (int)NU, NV, eb);
    if (l.end > kScratchBytes)
        return fail(A2A_ERROR_UNSUPPORTED, "the line tables do not fit the fixed scratch array (256 KiB)");

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) return fail(A2A_ERROR_UNSUPPORTED, "device index beyond 63");
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        if (!g_scratch_ptr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_lines_scratch);
            if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(scratch)");
            g_scratch_ptr[dev] = p;
        }
        scratch = g_scratch_ptr[dev];
    }

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned char* s = static_cast<unsigned char*>(scratch);
    StagePlan sp;
    sp.nstages = k.nstages;
    for (int i = 0; i < 4; ++i) sp.radix[i] = k.radix[i];
    if (precision == A2A_C128)
        lines_tables_kernel<double><<<8, 256, 0, st>>>(s, l, sp, n, (int)NU, NV);
    else
        lines_tables_kernel<float><<<8, 256, 0, st>>>(s, l, sp, n, (int)NU, NV);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "table kernel launch");

    {
        std::lock_guard<std::mutex> lock(g_mutex);
        int slot = 0;
        while (slot < kMaxAttrFns && g_attr_fn[dev][slot] && g_attr_fn[dev][slot] != k.fn) ++slot;
        if (slot == kMaxAttrFns || g_attr_fn[dev][slot] != k.fn) {
            e = cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem);
            if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute");
            if (slot < kMaxAttrFns) g_attr_fn[dev][slot] = k.fn;
        }
    }
    const unsigned grid = unsigned(NU * (NV / k.lines));
    const uint32_t* offA = reinterpret_cast<const uint32_t*>(s + l.offA);
    const uint32_t* offU = reinterpret_cast<const uint32_t*>(s + l.offU);
    const uint32_t* offV = reinterpret_cast<const uint32_t*>(s + l.offV);
    if (precision == A2A_C128) {
        PassArgs<double> a;
        a.src = static_cast<const double2*>(data);
        a.dst = static_cast<double2*>(data);
        a.offA = offA;
        a.offU = offU;
        a.offV = offV;
        a.tw = reinterpret_cast<const double2*>(s + l.tw);
        a.NU = (int)NU;
        a.NV = NV;
        a.scale = 1.0;
        a.split = 1;  // offA is the identity, so offA[j + r N/R] = offA[j] + offA[r N/R]
        a.err = nullptr;
        a.tcb = nullptr;
        void* args[] = {&a};
        e = cudaLaunchKernel(k.fn, dim3(grid), dim3(k.threads), args, k.smem, st);
    } else {
        PassArgs<float> a;
        a.src = static_cast<const float2*>(data);
        a.dst = static_cast<float2*>(data);
        a.offA = offA;
        a.offU = offU;
        a.offV = offV;
        a.tw = reinterpret_cast<const float2*>(s + l.tw);
        a.NU = (int)NU;
        a.NV = NV;
        a.scale = 1.0f;
        a.split = 1;
        a.err = nullptr;
        a.tcb = nullptr;
        void* args[] = {&a};
        e = cudaLaunchKernel(k.fn, dim3(grid), dim3(k.threads), args, k.smem, st);
    }
    if (e != cudaSuccess) return cuda_fail(e, "pass kernel launch");
    return A2A_SUCCESS;
}
