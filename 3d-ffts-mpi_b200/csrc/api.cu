// C ABI of liba2afft_b200: a2aDistribution / a2adfft over virtual ranks.
//
// Reference interfaces replaced (paths inside humz2k/3D-FFTs-MPI):
//   src/a2afft/distribution/a2adistribution.{h,cpp}  -> a2a_distribution_*, a2a_get/return_*_pencils
//   src/a2afft/dfft/a2adfft.{h,cpp}                  -> a2a_dfft_*
//   src/a2afft/dfft/kernels/a2affts.cu               -> a2a_forward/inverse_1d_fft, a2a_scale_fft, a2a_fast_copy_fft
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "batch.cuh"
#include "fft_mb.cuh"
#include "fft_tc.cuh"
#include "fft_tc2.cuh"
#include "internal.h"

using a2a::Dist;
using a2a::PassKernel;

struct a2a_distribution {
    Dist d;
};

struct a2a_dfft {
    a2a_distribution* dist = nullptr;
    void* scratch = nullptr;
    bool plans_made = false;
    bool autotune = true;
    a2a_method method = A2A_METHOD_PLAIN;
    // split tensor-core method: kernels per pass [Z, X, Y][inverse], twiddles
    // of their radix plans per axis, split radix-16 operands per direction
    PassKernel tc[3][2];  // the kernel in use per pass and direction
    // candidates per pass, direction: 0 = one tile per CTA, 1 = persistent
    // CTAs fed by the TMA ring (where the plan and geometry allow it), 2 =
    // the two-stage form (512 = 16 x 32, 1024 = 32 x 32), also fed by the TMA
    // ring, 3 = the two-stage form with 8-line tiles of 1024, 4 = the
    // software-pipelined two-stage form (fp16)
    PassKernel tcv[3][2][5];
    bool tcv_fits[3][5] = {};
    int tcv_occ[3][5] = {};
    float tcv_ms[3][5] = {};
    int tc_chosen[3] = {0, 0, 0};
    void* d_tc = nullptr;
    const void* tc_tw[3] = {nullptr, nullptr, nullptr};
    const void* tc_b[2] = {nullptr, nullptr};
    // two-stage form per pass: twiddles W_n^(b k1) ([b][k1]) and operands per direction
    const void* tc2_tw[3] = {nullptr, nullptr, nullptr};
    const void* tc2_b[3][2] = {};
    // multi-block pass body: persistent register-pipelined where compiled
    bool mb_persistent = true;
    // batch-mode multi-block passes: per-rank tensor maps (device memory),
    // [pass 1, 2][rank], and what they were built for
    void* d_mbmaps = nullptr;
    std::vector<const void*> mbmaps_key[3];
    int mbmaps_lines[3] = {0, 0, 0};
};

namespace {

thread_local std::string g_last_error;

a2a_status fail(a2a_status s, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return s;
}

a2a_status cuda_fail(cudaError_t e, const char* what) {
    return fail(A2A_ERROR_CUDA, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

#define A2A_CUDA(call, what)                              \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

// MPI_Dims_create(n, 3) for all-zero input dims: prime factors, largest
// first, each to the dimension with the smallest running product, then sorted
// non-increasing (the balanced factorisation the MPI standard asks for).
void dims_create(int n, int dims[3]) {
    std::vector<int> f;
    int m = n;
    for (int p = 2; (long)p * p <= m; ++p)
        while (m % p == 0) {
            f.push_back(p);
            m /= p;
        }
    if (m > 1) f.push_back(m);
    std::sort(f.rbegin(), f.rend());
    int d[3] = {1, 1, 1};
    for (int p : f) {
        int i = 0;
        for (int k = 1; k < 3; ++k)
            if (d[k] < d[i]) i = k;
        d[i] *= p;
    }
    std::sort(d, d + 3, [](int a, int b) { return a > b; });
    for (int k = 0; k < 3; ++k) dims[k] = d[k];
}

int find_kernels(a2a_precision prec, int n, int mode, bool inv, PassKernel* k, int max) {
    return prec == A2A_C128 ? a2a::find_pass_kernels_f64(n, mode, inv, k, max)
                            : a2a::find_pass_kernels_f32(n, mode, inv, k, max);
}

// Geometry of one slot: transform axis table, outer/inner batch tables.
struct SlotGeom {
    const uint32_t* offA;
    const uint32_t* offU;
    const uint32_t* offV;
    const void* tw;
    int n, NU, NV, mode;
    const std::vector<uint32_t>* hA;
    const std::vector<uint32_t>* hU;
    const std::vector<uint32_t>* hV;
};

SlotGeom slot_geom(const Dist& d, int slot) {
    switch (slot) {
        case a2a::SLOT_Z:  // lines (x, y), element z
            return {d.off[2], d.off[0], d.off[1], d.tw[2], d.ng[2], d.ng[0], d.ng[1], a2a::MODE_LINE,
                    &d.h_off[2], &d.h_off[0], &d.h_off[1]};
        case a2a::SLOT_X:  // lines (y, z), element x
            return {d.off[0], d.off[1], d.off[2], d.tw[0], d.ng[0], d.ng[1], d.ng[2], a2a::MODE_BATCH,
                    &d.h_off[0], &d.h_off[1], &d.h_off[2]};
        case a2a::SLOT_Y:  // lines (x, z), element y
            return {d.off[1], d.off[0], d.off[2], d.tw[1], d.ng[1], d.ng[0], d.ng[2], a2a::MODE_BATCH,
                    &d.h_off[1], &d.h_off[0], &d.h_off[2]};
        default:  // contiguous length-Ng lines of the held ranks' pencil buffers (cubes)
            return {d.iota, d.pen_u, d.pen_v, d.tw[0], d.ng[0],
                    int((uint64_t)d.local_ranks * d.nlocal / ((uint64_t)d.ng[0] * d.ng[0])), d.ng[0],
                    a2a::MODE_LINE, nullptr, nullptr, nullptr};
    }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library does not link the driver library itself).
using TmapEncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

TmapEncodeFn tmap_encoder() {
    static TmapEncodeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<TmapEncodeFn>(p);
    });
    return fn;
}

// Largest divisor of `ext` whose box edge (w words per element) is at most 256
// words and a whole number of 16-byte units when `inner`.
int tmat_chunk(int ext, int w, bool inner) {
    for (int c = std::min(ext, 256 / w); c >= 1; --c)
        if (ext % c == 0 && (!inner || (c * w * 8) % 16 == 0)) return c;
    return 0;
}

// The tensor maps of axis pass `slot` (Z, X, Y) for tiles of B lines on
// buffer `data` (one map per z brick index; the layout is described in
// fft_tmat.cuh).  False when the geometry has no such description: more than
// kTmatMaxMaps z bricks, a tile crossing a brick, a box edge that cannot be
// cut into boxes of at most 256 words, strides or offsets off 16 bytes, or an
// encoder refusal.
bool build_tmat(const Dist& d, int slot, int B, const void* data, a2a::TmatMaps* m) {
    if (slot != a2a::SLOT_Z && slot != a2a::SLOT_X && slot != a2a::SLOT_Y) return false;
    const TmapEncodeFn enc = tmap_encoder();
    if (!enc) return false;
    const int w = d.prec == A2A_C128 ? 2 : 1;
    const int lx = d.local[0], ly = d.local[1], lz = d.local[2];
    const int d0 = d.dims[0], d1 = d.dims[1], d2 = d.dims[2];
    const uint64_t nl = d.nlocal;
    const uint64_t esz = d.elem_bytes;
    if (d2 > a2a::kTmatMaxMaps || (w * lz * 8) % 16 || (nl * esz) % 16) return false;
    if (reinterpret_cast<uintptr_t>(data) % 16) return false;
    std::memset(m, 0, sizeof(*m));
    m->pass = slot;
    m->lx = lx;
    m->ly = ly;
    m->lz = lz;
    m->words = w;
    m->nmaps = d2;
    cuuint32_t box[5] = {1, 1, 1, 1, 1};
    if (slot == a2a::SLOT_Z) {
        if (B > 256 || ly % B) return false;
        const int c = tmat_chunk(lz, w, true);
        if (!c) return false;
        m->chunk = c;
        m->nchunk = lz / c;
        box[0] = (cuuint32_t)(w * c);
        box[1] = (cuuint32_t)B;
    } else {
        if (lz % B || w * B > 256 || (w * B * 8) % 16) return false;
        const int l = slot == a2a::SLOT_X ? lx : ly;
        const int dd = slot == a2a::SLOT_X ? d0 : d1;
        box[0] = (cuuint32_t)(w * B);
        int c = l;
        if (l > 256 || dd > 256) {
            if (dd != 1) return false;
            c = tmat_chunk(l, 1, false);
            if (!c) return false;
        }
        m->chunk = c;
        m->nchunk = l / c;
        if (slot == a2a::SLOT_X) {
            box[2] = (cuuint32_t)c;
            box[4] = (cuuint32_t)(m->nchunk == 1 ? d0 : 1);
        } else {
            box[1] = (cuuint32_t)c;
            box[3] = (cuuint32_t)(m->nchunk == 1 ? d1 : 1);
        }
    }
    m->chunk_shift = -1;
    for (int sh = 0; sh < 31; ++sh)
        if ((1 << sh) == m->chunk) m->chunk_shift = sh;
    // every box lands at a 128-byte aligned shared-memory offset
    if (((size_t)B * m->chunk * esz) % 128) return false;
    const cuuint64_t dims[5] = {(cuuint64_t)w * lz, (cuuint64_t)ly, (cuuint64_t)lx, (cuuint64_t)d1, (cuuint64_t)d0};
    const cuuint64_t strides[4] = {(cuuint64_t)lz * esz, (cuuint64_t)ly * lz * esz, (cuuint64_t)d2 * nl * esz,
                                   (cuuint64_t)d1 * d2 * nl * esz};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    for (int zr = 0; zr < d2; ++zr) {
        void* base = const_cast<char*>(static_cast<const char*>(data)) + (size_t)zr * nl * esz;
        if (enc(&m->map[zr], CU_TENSOR_MAP_DATA_TYPE_INT64, 5, base, dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return false;
    }
    return true;
}

bool is_tmat(const PassKernel& k) {
    return k.kind == a2a::KIND_TMAT2 || k.kind == a2a::KIND_TMAT3 || k.kind == a2a::KIND_TMAT2W ||
           k.kind == a2a::KIND_TMATI || k.kind == a2a::KIND_TMAT2S;
}

// Does variant k fit the slot's geometry?  Every kernel needs whole tiles.
// Kernels that move several lines per 16-byte access (the pipelined BATCH
// kernel: whole tile rows; LPT = 2: line pairs) need those lines contiguous
// and 16-byte aligned in every tile.
bool variant_fits(const Dist& d, int slot, const SlotGeom& g, const PassKernel& k) {
    if (g.NV % k.lines) return false;
    if (is_tmat(k)) {
        if (k.lpt > 1 && g.mode != a2a::MODE_BATCH) return false;
        a2a::TmatMaps probe;  // encoded against a stand-in 256-byte aligned address
        return build_tmat(d, slot, k.lines, reinterpret_cast<const void*>(uintptr_t(1) << 20), &probe);
    }
    int vec = 1;  // lines per 16-byte access
    if ((k.kind == a2a::KIND_PIPE || k.kind == a2a::KIND_TMA) && g.mode == a2a::MODE_BATCH) vec = k.lines;
    if (k.kind == a2a::KIND_TMA && g.mode != a2a::MODE_BATCH) return false;
    if (k.lpt > 1) vec = k.lpt;
    if (k.lpt > 1 && g.mode != a2a::MODE_BATCH) return false;
    if (vec == 1) return true;
    if (!g.hA) return false;
    const size_t epu = 16 / d.elem_bytes;
    if ((vec * d.elem_bytes) % 16) return false;
    for (int v0 = 0; v0 < g.NV; v0 += vec) {
        for (int b = 1; b < vec; ++b)
            if ((*g.hV)[v0 + b] != (*g.hV)[v0] + (uint32_t)b) return false;
        if ((*g.hV)[v0] % epu) return false;
    }
    for (uint32_t o : *g.hA)
        if (o % epu) return false;
    for (uint32_t o : *g.hU)
        if (o % epu) return false;
    return true;
}

// Whether offA[j + r N/R] == offA[j] + offA[r N/R] holds for the first and
// last stage of kernel k on a slot whose axis has brick extent l: true when
// l and N/R divide one another (no carry from the in-brick position into the
// rank part of the offset).
int split_ok(int l, const PassKernel& k) {
    const int nb0 = k.n / k.radix[0];
    const int nbl = k.n / k.radix[k.nstages - 1];
    auto ok = [l](int nb) { return (l % nb == 0) || (nb % l == 0); };
    return ok(nb0) && ok(nbl) ? 1 : 0;
}

// Stage twiddles W_{Ns R}^{r m} (forward sign), laid out as RadixPlan::twoff,
// generated in long double with the exponent reduced exactly.
void gen_twiddles(const PassKernel& k, std::vector<long double>& re, std::vector<long double>& im) {
    const long double pi = acosl(-1.0L);
    re.clear();
    im.clear();
    int ns = k.radix[0];
    for (int s = 1; s < k.nstages; ++s) {
        const int R = k.radix[s];
        const long long M = (long long)ns * R;
        for (int r = 1; r < R; ++r)
            for (int m = 0; m < ns; ++m) {
                const long long e = ((long long)r * m) % M;
                const long double ang = 2.0L * pi * (long double)e / (long double)M;
                re.push_back(cosl(ang));
                im.push_back(-sinl(ang));
            }
        ns *= R;
    }
}

a2a_status check_buf(void** p, const char* name) {
    if (!p || !p[0]) return fail(A2A_ERROR_INVALID_VALUE, "%s is NULL", name);
    if (reinterpret_cast<uintptr_t>(p[0]) % 16)
        return fail(A2A_ERROR_MISALIGNED, "%s[0] is not 16-byte aligned", name);
    return A2A_SUCCESS;
}

a2a_status finish(const Dist& d, cudaStream_t st, bool sync) {
    A2A_CUDA(cudaGetLastError(), "kernel launch");
    if (sync) A2A_CUDA(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    return A2A_SUCCESS;
}

template <typename T>
cudaError_t launch_pass_t(const PassKernel& k, unsigned grid, const void* src, void* dst, const uint32_t* offA,
                          const uint32_t* offU, const uint32_t* offV, const void* tw, int NU, int NV, double scale,
                          int split, int* err, cudaStream_t st, const void* maps = nullptr) {
    a2a::PassArgs<T> a;
    a.src = static_cast<const a2a::cx<T>*>(src);
    a.dst = static_cast<a2a::cx<T>*>(dst);
    a.offA = offA;
    a.offU = offU;
    a.offV = offV;
    a.tw = static_cast<const a2a::cx<T>*>(tw);
    a.NU = NU;
    a.NV = NV;
    a.scale = T(scale);
    a.split = split;
    a.err = err;
    void* args[] = {&a, const_cast<void*>(maps)};
    return cudaLaunchKernel(k.fn, dim3(grid), dim3(k.threads), args, k.smem, st);
}

// Kernels whose CTAs stay resident and stride over the tiles (grid: one wave).
bool persistent_kind(const PassKernel& k) {
    return k.kind == a2a::KIND_PIPE || k.kind == a2a::KIND_TMA || k.kind == a2a::KIND_RPIPE ||
           k.kind == a2a::KIND_RPIPES || is_tmat(k);
}

// Launch candidate `c` of a slot on buffer p (in place).
cudaError_t launch_slot(const Dist& d, int slot, bool inv, int c, void* p, double scale, cudaStream_t st) {
    const a2a::PassSlot& ps = d.slot[slot][inv ? 1 : 0];
    const PassKernel& k = ps.cand[c];
    const SlotGeom g = slot_geom(d, slot);
    const uint64_t tiles = (uint64_t)g.NU * (g.NV / k.lines);
    uint64_t grid = tiles;
    if (persistent_kind(k)) {
        const uint64_t resident = (uint64_t)std::max(ps.occ[c], 1) * d.sms;
        grid = std::min(tiles, resident);
    }
    const void* maps = nullptr;
    if (is_tmat(k)) {  // tensor maps of this pass for buffer p (rebuilt when p or the tile height changes)
        a2a::TmatEntry& ce = d.tmat[slot];
        if (ce.ptr != p || ce.lines != k.lines) {
            ce.ptr = nullptr;
            if (!build_tmat(d, slot, k.lines, p, &ce.maps)) return cudaErrorInvalidValue;
            ce.ptr = p;
            ce.lines = k.lines;
        }
        maps = &ce.maps;
    }
    const int l = slot == a2a::SLOT_Z ? d.local[2] : slot == a2a::SLOT_X ? d.local[0]
                : slot == a2a::SLOT_Y ? d.local[1] : d.ng[0];
    const int split = split_ok(l, k);
    const void* tw = ps.tw[c] ? ps.tw[c] : g.tw;  // a candidate with its own radix plan has its own table
    if (d.prec == A2A_C128)
        return launch_pass_t<double>(k, unsigned(grid), p, p, g.offA, g.offU, g.offV, tw, g.NU, g.NV, scale, split,
                                     d.d_err, st, maps);
    return launch_pass_t<float>(k, unsigned(grid), p, p, g.offA, g.offU, g.offV, tw, g.NU, g.NV, scale, split,
                                d.d_err, st, maps);
}

a2a_status setup_distribution(Dist& d, int nx, int ny, int nz, int P, int block_size, a2a_precision prec) {
    if (nx < 1 || ny < 1 || nz < 1 || P < 1)
        return fail(A2A_ERROR_INVALID_VALUE, "grid sizes and world_size must be >= 1");
    if (block_size < 1 || block_size > 1024) return fail(A2A_ERROR_INVALID_VALUE, "block_size must be in [1, 1024]");
    if (prec != A2A_C128 && prec != A2A_C64) return fail(A2A_ERROR_INVALID_VALUE, "unknown precision %d", (int)prec);
    d.ng[0] = nx;
    d.ng[1] = ny;
    d.ng[2] = nz;
    d.P = P;
    d.first_rank = 0;
    d.local_ranks = P;
    d.block_size = block_size;
    d.prec = prec;
    d.elem_bytes = prec == A2A_C128 ? 16 : 8;
    d.cube = (nx == ny && ny == nz);
    dims_create(P, d.dims);
    for (int a = 0; a < 3; ++a)  // a2adistribution.cpp:61-63
        if (d.ng[a] % d.dims[a])
            return fail(A2A_ERROR_DECOMPOSITION, "N[%d]=%d is not divisible by dims[%d]=%d", a, d.ng[a], a, d.dims[a]);
    for (int a = 0; a < 3; ++a) d.local[a] = d.ng[a] / d.dims[a];
    for (int a = 0; a < 3; ++a)  // :115-117
        if (P % d.dims[a])
            return fail(A2A_ERROR_DECOMPOSITION, "world_size=%d is not divisible by dims[%d]=%d", P, a, d.dims[a]);
    const long long lx = d.local[0], ly = d.local[1], lz = d.local[2];
    if ((lx * ly) % P || (lx * lz) % P || (ly * lz) % P)  // :119-121
        return fail(A2A_ERROR_DECOMPOSITION, "a face of the %lldx%lldx%lld brick is not divisible by world_size=%d",
                    lx, ly, lz, P);
    d.nlocal = (uint64_t)lx * ly * lz;
    d.chunk = d.nlocal / P;
    const uint64_t total = d.nlocal * (uint64_t)P;
    if (total >= (uint64_t(1) << 32))
        return fail(A2A_ERROR_UNSUPPORTED, "grids of 2^32 or more elements are not supported");

    A2A_CUDA(cudaGetDevice(&d.device), "cudaGetDevice");
    A2A_CUDA(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, d.device), "cudaDeviceGetAttribute");

    // offset tables: brick offsets per axis (global (x,y,z) lives at
    // off[0][x] + off[1][y] + off[2][z]), identity, pencil-buffer line bases
    const int maxn = std::max(nx, std::max(ny, nz));
    std::vector<uint32_t> h;
    size_t pos[6];
    const uint64_t nl = d.nlocal;
    const uint64_t d1 = d.dims[1], d2 = d.dims[2];
    pos[0] = h.size();
    for (int x = 0; x < nx; ++x) h.push_back(uint32_t((x / lx) * d1 * d2 * nl + (x % lx) * ly * lz));
    pos[1] = h.size();
    for (int y = 0; y < ny; ++y) h.push_back(uint32_t((y / ly) * d2 * nl + (y % ly) * lz));
    pos[2] = h.size();
    for (int z = 0; z < nz; ++z) h.push_back(uint32_t((z / lz) * nl + (z % lz)));
    pos[3] = h.size();
    for (int i = 0; i < maxn; ++i) h.push_back(uint32_t(i));
    pos[4] = h.size();
    for (int u = 0; u < nx; ++u) h.push_back(uint32_t((uint64_t)u * nx * nx));
    pos[5] = h.size();
    for (int v = 0; v < nx; ++v) h.push_back(uint32_t((uint64_t)v * nx));
    const size_t err_pos = h.size();
    h.push_back(0u);  // device error flag (bounded waits that gave up)
    A2A_CUDA(cudaMalloc(&d.d_tables, h.size() * sizeof(uint32_t)), "cudaMalloc(tables)");
    A2A_CUDA(cudaMemcpy(d.d_tables, h.data(), h.size() * sizeof(uint32_t), cudaMemcpyHostToDevice), "cudaMemcpy");
    for (int a = 0; a < 3; ++a) d.off[a] = d.d_tables + pos[a];
    d.iota = d.d_tables + pos[3];
    d.pen_u = d.d_tables + pos[4];
    d.pen_v = d.d_tables + pos[5];
    d.d_err = reinterpret_cast<int*>(d.d_tables + err_pos);

    for (int a = 0; a < 3; ++a) d.h_off[a].assign(h.begin() + pos[a], h.begin() + pos[a + 1]);

    // pass kernels: every compiled variant per slot, which fit, occupancy
    for (int sl = 0; sl < a2a::NSLOTS; ++sl) {
        if (sl == a2a::SLOT_LINES && !d.cube) continue;
        const int axis = sl == a2a::SLOT_Z ? 2 : sl == a2a::SLOT_X ? 0 : sl == a2a::SLOT_Y ? 1 : 0;
        const int mode = sl == a2a::SLOT_X || sl == a2a::SLOT_Y ? a2a::MODE_BATCH : a2a::MODE_LINE;
        for (int inv = 0; inv < 2; ++inv) {
            a2a::PassSlot& ps = d.slot[sl][inv];
            const int cnt = find_kernels(prec, d.ng[axis], mode, inv, ps.cand, a2a::kMaxVariants);
            if (cnt == 0)
                return fail(A2A_ERROR_UNSUPPORTED,
                            "no compiled transform of length %d (supported: 4 8 12 16 24 32 48 64 96 128 192 256 "
                            "384 512 768 1024)",
                            d.ng[axis]);
            ps.ncand = std::min(cnt, a2a::kMaxVariants);
            ps.chosen = -1;
            for (int c = 0; c < ps.ncand; ++c) {
                const PassKernel& k = ps.cand[c];
                A2A_CUDA(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem),
                         "cudaFuncSetAttribute");
                A2A_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&ps.occ[c], k.fn, k.threads, k.smem),
                         "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
            }
        }
    }

    std::vector<long double> re, im;
    size_t twpos[3], twtotal = 0;
    for (int a = 0; a < 3; ++a) {
        twpos[a] = twtotal;
        const int sl = a == 2 ? a2a::SLOT_Z : a == 0 ? a2a::SLOT_X : a2a::SLOT_Y;
        twtotal += (size_t)d.slot[sl][0].cand[0].twtotal;
    }
    if (twtotal == 0) twtotal = 1;
    A2A_CUDA(cudaMalloc(&d.d_tw, twtotal * d.elem_bytes), "cudaMalloc(twiddles)");
    std::vector<double> hd;
    std::vector<float> hf;
    for (int a = 0; a < 3; ++a) {
        const int sl = a == 2 ? a2a::SLOT_Z : a == 0 ? a2a::SLOT_X : a2a::SLOT_Y;
        gen_twiddles(d.slot[sl][0].cand[0], re, im);
        for (size_t i = 0; i < re.size(); ++i) {
            hd.push_back((double)re[i]);
            hd.push_back((double)im[i]);
            hf.push_back((float)re[i]);
            hf.push_back((float)im[i]);
        }
    }
    if (!hd.empty()) {
        if (prec == A2A_C128)
            A2A_CUDA(cudaMemcpy(d.d_tw, hd.data(), hd.size() * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
        else
            A2A_CUDA(cudaMemcpy(d.d_tw, hf.data(), hf.size() * sizeof(float), cudaMemcpyHostToDevice), "cudaMemcpy");
    }
    for (int a = 0; a < 3; ++a) d.tw[a] = static_cast<const char*>(d.d_tw) + twpos[a] * d.elem_bytes;

    // candidates whose radix plan differs from the slot's first (the wide
    // two-stage plans) get their own twiddle tables
    {
        auto same_plan = [](const PassKernel& x, const PassKernel& y) {
            if (x.nstages != y.nstages) return false;
            for (int i = 0; i < x.nstages; ++i)
                if (x.radix[i] != y.radix[i]) return false;
            return true;
        };
        std::vector<double> ed;
        std::vector<float> ef;
        std::vector<size_t> epos;  // per (slot, inv, candidate): offset + 1, or 0
        for (int sl = 0; sl < a2a::NSLOTS; ++sl)
            for (int inv = 0; inv < 2; ++inv) {
                a2a::PassSlot& ps = d.slot[sl][inv];
                for (int c = 0; c < ps.ncand; ++c) {
                    ps.tw[c] = nullptr;
                    if (same_plan(ps.cand[c], ps.cand[0])) {
                        epos.push_back(0);
                        continue;
                    }
                    epos.push_back(ed.size() / 2 + 1);
                    gen_twiddles(ps.cand[c], re, im);
                    for (size_t i = 0; i < re.size(); ++i) {
                        ed.push_back((double)re[i]);
                        ed.push_back((double)im[i]);
                        ef.push_back((float)re[i]);
                        ef.push_back((float)im[i]);
                    }
                }
            }
        if (!ed.empty()) {
            A2A_CUDA(cudaMalloc(&d.d_tw2, (ed.size() / 2) * d.elem_bytes), "cudaMalloc(twiddles)");
            if (prec == A2A_C128)
                A2A_CUDA(cudaMemcpy(d.d_tw2, ed.data(), ed.size() * sizeof(double), cudaMemcpyHostToDevice),
                         "cudaMemcpy");
            else
                A2A_CUDA(cudaMemcpy(d.d_tw2, ef.data(), ef.size() * sizeof(float), cudaMemcpyHostToDevice),
                         "cudaMemcpy");
            size_t k = 0;
            for (int sl = 0; sl < a2a::NSLOTS; ++sl)
                for (int inv = 0; inv < 2; ++inv) {
                    a2a::PassSlot& ps = d.slot[sl][inv];
                    for (int c = 0; c < ps.ncand; ++c, ++k)
                        if (epos[k]) ps.tw[c] = static_cast<const char*>(d.d_tw2) + (epos[k] - 1) * d.elem_bytes;
                }
        }
    }

    // default choice: the first variant that fits each slot's geometry
    for (int sl = 0; sl < a2a::NSLOTS; ++sl) {
        if (sl == a2a::SLOT_LINES && !d.cube) continue;
        const SlotGeom g = slot_geom(d, sl);
        for (int inv = 0; inv < 2; ++inv) {
            a2a::PassSlot& ps = d.slot[sl][inv];
            for (int c = 0; c < ps.ncand; ++c) {
                ps.fits[c] = ps.occ[c] > 0 && variant_fits(d, sl, g, ps.cand[c]);
                if (ps.fits[c] && ps.chosen < 0) ps.chosen = c;
            }
            if (ps.chosen < 0) ps.chosen = 0;  // reported by make_plans / the 1D calls
        }
    }
    return A2A_SUCCESS;
}

void release(Dist& d) {
    if (d.d_tables) cudaFree(d.d_tables);
    if (d.d_tw) cudaFree(d.d_tw);
    if (d.d_tw2) cudaFree(d.d_tw2);
    d.d_tables = nullptr;
    d.d_tw = nullptr;
    d.d_tw2 = nullptr;
}

a2a_status create_common(int nx, int ny, int nz, int P, int bs, a2a_precision prec, a2a_distribution** out) {
    if (!out) return fail(A2A_ERROR_INVALID_VALUE, "out is NULL");
    *out = nullptr;
    auto* h = new (std::nothrow) a2a_distribution();
    if (!h) return fail(A2A_ERROR_OUT_OF_MEMORY, "host allocation failed");
    const a2a_status s = setup_distribution(h->d, nx, ny, nz, P, bs, prec);
    if (s != A2A_SUCCESS) {
        release(h->d);
        delete h;
        return s;
    }
    *out = h;
    return A2A_SUCCESS;
}

a2a_status need_cube(const Dist& d, const char* what) {
    if (!d.cube) return fail(A2A_ERROR_NOT_IMPLEMENTED, "%s needs a cube (the reference API takes one Ng)", what);
    return A2A_SUCCESS;
}

// 1D transforms of the contiguous length-Ng lines of a pencil buffer.
a2a_status lines_1d(a2a_distribution* h, void** data, bool inv) {
    if (!h) return fail(A2A_ERROR_INVALID_VALUE, "distribution is NULL");
    Dist& d = h->d;
    a2a_status s;
    if ((s = need_cube(d, "1D pencil transforms")) != A2A_SUCCESS) return s;
    if ((s = check_buf(data, "d_data")) != A2A_SUCCESS) return s;
    const a2a::PassSlot& ps = d.slot[a2a::SLOT_LINES][inv ? 1 : 0];
    if (!ps.fits[ps.chosen])
        return fail(A2A_ERROR_UNSUPPORTED, "no compiled 1D kernel fits %d lines of length %d", d.ng[0], d.ng[0]);
    A2A_CUDA(launch_slot(d, a2a::SLOT_LINES, inv, ps.chosen, data[0], 1.0, d.stream), "1D pass launch");
    return finish(d, d.stream, true);
}

// One of the three in-place axis passes over the rank-major bricks.  Each
// pass's gather/scatter addresses come from the brick offset tables, i.e. the
// alltoall + unpack (and pack + alltoall) composites of the reference steps.
cudaError_t run_pass(const Dist& d, int pass, bool inv, void* p, cudaStream_t st) {
    // pass 0 = Z (lines (x, y)), 1 = X (lines (y, z)), 2 = Y (lines (x, z));
    // the Y pass carries the inverse's 1/(nx ny nz)
    const double scale = (inv && pass == 2) ? 1.0 / ((double)d.ng[0] * d.ng[1] * d.ng[2]) : 1.0;
    return launch_slot(d, pass, inv, d.slot[pass][inv ? 1 : 0].chosen, p, scale, st);
}

// One pass of the split tensor-core method.
cudaError_t run_tc_pass(const a2a_dfft* f, int pass, bool inv, void* p, cudaStream_t st) {
    const Dist& d = f->dist->d;
    const SlotGeom g = slot_geom(d, pass);
    const int axis = pass == 0 ? 2 : pass == 1 ? 0 : 1;
    const PassKernel& k = f->tc[pass][inv ? 1 : 0];
    const double scale = (inv && pass == 2) ? 1.0 / ((double)d.ng[0] * d.ng[1] * d.ng[2]) : 1.0;
    const void* maps = nullptr;
    unsigned grid = unsigned((uint64_t)g.NU * (g.NV / k.lines));
    const bool two = k.kind == a2a::KIND_TC2;
    if (k.kind == a2a::KIND_TCR || two) {  // tensor maps of this pass for buffer p, one wave of persistent CTAs
        a2a::TmatEntry& ce = d.tmat[pass];
        if (ce.ptr != p || ce.lines != k.lines) {
            ce.ptr = nullptr;
            if (!build_tmat(d, pass, k.lines, p, &ce.maps)) return cudaErrorInvalidValue;
            ce.ptr = p;
            ce.lines = k.lines;
        }
        maps = &ce.maps;
        int occ = 1;  // resident CTAs per SM of this candidate
        for (int c = 1; c < 5; ++c)
            if (f->tcv_fits[pass][c] && f->tcv[pass][inv ? 1 : 0][c].fn == k.fn) occ = f->tcv_occ[pass][c];
        grid = (unsigned)std::min<uint64_t>(grid, (uint64_t)std::max(occ, 1) * d.sms);
    }
    a2a::PassArgs<float> a;
    a.src = static_cast<const float2*>(p);
    a.dst = static_cast<float2*>(p);
    a.offA = g.offA;
    a.offU = g.offU;
    a.offV = g.offV;
    a.tw = static_cast<const float2*>(two ? f->tc2_tw[pass] : f->tc_tw[axis]);
    a.NU = g.NU;
    a.NV = g.NV;
    a.scale = float(scale);
    a.split = 0;
    a.err = d.d_err;
    a.tcb = two ? f->tc2_b[pass][inv ? 1 : 0] : f->tc_b[inv ? 1 : 0];
    void* args[] = {&a, const_cast<void*>(maps)};
    return cudaLaunchKernel(k.fn, dim3(grid), dim3(k.threads), args, k.smem, st);
}

a2a_status need_all_ranks(const Dist& d, const char* what) {
    if (d.local_ranks != d.P)
        return fail(A2A_ERROR_NOT_IMPLEMENTED,
                    "%s needs every virtual rank in one buffer; this distribution holds %d of %d (the exchange "
                    "between processes is the distributed layer's)",
                    what, d.local_ranks, d.P);
    return A2A_SUCCESS;
}

a2a_status check_dfft(a2a_dfft* f, void** data) {
    if (!f) return fail(A2A_ERROR_INVALID_VALUE, "dfft is NULL");
    if (!f->plans_made) return fail(A2A_ERROR_NO_PLANS, "make_plans has not been called");
    a2a_status s;
    if ((s = need_all_ranks(f->dist->d, "the fused transform")) != A2A_SUCCESS) return s;
    return check_buf(data, "d_data");
}

// Reads and clears the device error flag (a bounded wait in a kernel gave up).
a2a_status check_device_flag(const Dist& d) {
    int flag = 0;
    A2A_CUDA(cudaMemcpy(&flag, d.d_err, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy(error flag)");
    if (flag) {
        A2A_CUDA(cudaMemset(d.d_err, 0, sizeof(int)), "cudaMemset(error flag)");
        return fail(A2A_ERROR_TIMEOUT, "a pass kernel's bounded wait for its tile copies gave up");
    }
    return A2A_SUCCESS;
}

// The fused transform: Z, X then Y pass.
a2a_status fused(a2a_dfft* f, void** data, bool inv, cudaStream_t st, bool sync) {
    a2a_status s;
    if ((s = check_dfft(f, data)) != A2A_SUCCESS) return s;
    const Dist& d = f->dist->d;
    for (int pass = 0; pass < 3; ++pass) {
        if (f->method == A2A_METHOD_PLAIN)
            A2A_CUDA(run_pass(d, pass, inv, data[0], st), "axis pass launch");
        else
            A2A_CUDA(run_tc_pass(f, pass, inv, data[0], st), "tensor-core pass launch");
    }
    if ((s = finish(d, st, sync)) != A2A_SUCCESS) return s;
    return sync ? check_device_flag(d) : A2A_SUCCESS;
}

template <typename F> a2a_status step(a2a_distribution* h, void** b1, void** b2, F&& body) {
    if (!h) return fail(A2A_ERROR_INVALID_VALUE, "distribution is NULL");
    Dist& d = h->d;
    a2a_status s;
    if ((s = need_all_ranks(d, "the pencil steps")) != A2A_SUCCESS) return s;
    if ((s = need_cube(d, "the pencil steps")) != A2A_SUCCESS) return s;
    if ((s = check_buf(b1, "d_buff1")) != A2A_SUCCESS) return s;
    if ((s = check_buf(b2, "d_buff2")) != A2A_SUCCESS) return s;
    if (b1[0] == b2[0]) return fail(A2A_ERROR_INVALID_VALUE, "d_buff1 and d_buff2 must be distinct buffers");
    cudaError_t e = body(d, b1[0], b2[0]);
    if (e != cudaSuccess) return cuda_fail(e, "pencil step launch");
    return finish(d, d.stream, true);
}

}  // namespace

namespace {

// Byte image of the split radix-16 operand for one direction: the real
// 32 x 32 DFT matrix R (K x N: rows 0-15 take x_re, 16-31 x_im; columns 0-15
// give y_re, 16-31 y_im), split from its FP64 values as R = Rh + Rl (fp16) or
// Rh + Rm + Rl (bf16), each part the rounding of what the previous ones
// leave, stored as the K-major N x K operand of the UMMA canonical
// no-swizzle layout: element (n, k) at (k/8)*512 + (n/8)*128 + (n%8)*16 +
// (k%8)*2; the parts one after the other.
void tc_operand_image(bool inverse, int fmt, std::vector<uint16_t>& img) {
    const long double pi = acosl(-1.0L);
    const int parts = a2a::tc_parts(fmt);
    img.assign(a2a::tc_b_bytes(fmt) / 2, 0);
    for (int k = 0; k < 32; ++k)
        for (int n = 0; n < 32; ++n) {
            const int r = k % 16, c = n % 16;
            const long double ang = 2.0L * pi * (long double)((r * c) % 16) / 16.0L;
            const double C = (double)cosl(ang);
            const double S = (inverse ? 1.0 : -1.0) * (double)sinl(ang);
            double v;
            if (k < 16) v = n < 16 ? C : S;
            else v = n < 16 ? -S : C;
            const size_t off = (size_t)(k / 8) * a2a::kTcChunkB + (n / 8) * 128 + (n % 8) * 16 + (k % 8) * 2;
            for (int q = 0; q < parts; ++q) {
                uint16_t h;
                if (fmt == a2a::TC_FP16) {
                    const __half hh = __float2half_rn((float)v);
                    h = __half_as_ushort(hh);
                    v -= (double)__half2float(hh);
                } else {
                    const __nv_bfloat16 hh = __float2bfloat16_rn((float)v);
                    h = __bfloat16_as_ushort(hh);
                    v -= (double)__bfloat162float(hh);
                }
                img[(q * a2a::kTcMatB + off) / 2] = h;
            }
        }
}

size_t tc2_b_bytes_n(int n, int fmt) {
    return n == 512 ? (size_t)a2a::tc2_b_bytes<512>(fmt) : (size_t)a2a::tc2_b_bytes<1024>(fmt);
}

// The two-stage form's operand of one direction for length n: at 512 the
// radix-16 image above, then the radix-32 real DFT matrix; at 1024 the
// radix-32 matrix alone (both stages use it).  The radix-32 matrix: K x N =
// 64 x 64, K = [re b<16 | im b<16 | re b>=16 | im b>=16], N the same over the
// outputs k2, split like the radix-16 one, K-major without swizzle: element
// (n, k) at (k/8)*1024 + (n/8)*128 + (n%8)*16 + (k%8)*2 of its part.
void tc2_operand_image(int len, bool inverse, int fmt, std::vector<uint16_t>& img) {
    const int parts = a2a::tc_parts(fmt);
    img.assign(tc2_b_bytes_n(len, fmt) / 2, 0);
    size_t base = 0;  // bytes
    if (len == 512) {
        std::vector<uint16_t> b16;
        tc_operand_image(inverse, fmt, b16);
        std::copy(b16.begin(), b16.end(), img.begin());
        base = (size_t)parts * a2a::kTcMatB;
    }
    const long double pi = acosl(-1.0L);
    for (int k = 0; k < 64; ++k)
        for (int n = 0; n < 64; ++n) {
            const int kb = k / 16, nb = n / 16;
            const int r = k % 16 + 16 * (kb / 2), c = n % 16 + 16 * (nb / 2);
            const long double ang = 2.0L * pi * (long double)((r * c) % 32) / 32.0L;
            const double C = (double)cosl(ang);
            const double S = (inverse ? 1.0 : -1.0) * (double)sinl(ang);
            double v;
            if (kb % 2 == 0) v = nb % 2 == 0 ? C : S;
            else v = nb % 2 == 0 ? -S : C;
            const size_t off = (size_t)(k / 8) * a2a::kTc2ChunkB1 + (n / 8) * 128 + (n % 8) * 16 + (k % 8) * 2;
            for (int q = 0; q < parts; ++q) {
                uint16_t h;
                if (fmt == a2a::TC_FP16) {
                    const __half hh = __float2half_rn((float)v);
                    h = __half_as_ushort(hh);
                    v -= (double)__half2float(hh);
                } else {
                    const __nv_bfloat16 hh = __float2bfloat16_rn((float)v);
                    h = __bfloat16_as_ushort(hh);
                    v -= (double)__bfloat162float(hh);
                }
                img[(base + q * a2a::kTc2MatB1 + off) / 2] = h;
            }
        }
}

a2a_status setup_tc(a2a_dfft* f, a2a_method m) {
    const Dist& d = f->dist->d;
    if (d.prec != A2A_C64) return fail(A2A_ERROR_NOT_IMPLEMENTED, "the split tensor-core methods take A2A_C64 data");
    const int fmt = m == A2A_METHOD_SPLIT_FP16 ? a2a::TC_FP16 : a2a::TC_BF16;
    const char* names[3] = {"Z", "X", "Y"};
    for (int p = 0; p < 3; ++p) {
        const SlotGeom g = slot_geom(d, p);
        for (int inv = 0; inv < 2; ++inv)
            if (!a2a::find_tc_kernel(g.n, g.mode, inv, fmt, &f->tcv[p][inv][0]))
                return fail(A2A_ERROR_NOT_IMPLEMENTED,
                            "%s pass: no tensor-core kernel of length %d (available: 64 128 256 512 1024)", names[p],
                            g.n);
        if (g.NV % f->tcv[p][0][0].lines)
            return fail(A2A_ERROR_UNSUPPORTED, "%s pass: %d lines are not a multiple of the %d-line tile", names[p],
                        g.NV, f->tcv[p][0][0].lines);
        // the ring form where its plan exists and every tile is whole
        // tensor-map boxes (probed against a stand-in aligned address)
        bool ring = true;
        for (int inv = 0; inv < 2; ++inv)
            ring = ring && a2a::find_tc_ring_kernel(g.n, g.mode, inv, fmt, &f->tcv[p][inv][1]);
        if (ring) {
            a2a::TmatMaps probe;
            ring = g.NV % f->tcv[p][0][1].lines == 0 &&
                   build_tmat(d, p, f->tcv[p][0][1].lines, reinterpret_cast<const void*>(uintptr_t(1) << 20), &probe);
        }
        // the two-stage form (512, 1024; and 1024 with 8-line tiles), on the
        // same ring geometry
        bool two[2] = {true, true};
        for (int w = 0; w < 2; ++w) {
            for (int inv = 0; inv < 2; ++inv)
                two[w] = two[w] && a2a::find_tc2_kernel(g.n, g.mode, inv, fmt, w == 1, &f->tcv[p][inv][2 + w]);
            if (two[w]) {
                a2a::TmatMaps probe;
                two[w] = g.NV % f->tcv[p][0][2 + w].lines == 0 &&
                         build_tmat(d, p, f->tcv[p][0][2 + w].lines, reinterpret_cast<const void*>(uintptr_t(1) << 20),
                                    &probe);
            }
        }
        f->tcv_fits[p][0] = true;
        f->tcv_fits[p][1] = ring;
        f->tcv_fits[p][2] = two[0];
        f->tcv_fits[p][3] = two[1];
        // the pipelined two-stage form (fp16)
        bool pipe = true;
        for (int inv = 0; inv < 2; ++inv) pipe = pipe && a2a::find_tc2p_kernel(g.n, g.mode, inv, fmt, &f->tcv[p][inv][4]);
        if (pipe) {
            a2a::TmatMaps probe;
            pipe = g.NV % f->tcv[p][0][4].lines == 0 &&
                   build_tmat(d, p, f->tcv[p][0][4].lines, reinterpret_cast<const void*>(uintptr_t(1) << 20), &probe);
        }
        f->tcv_fits[p][4] = pipe;
        for (int c = 0; c < 5; ++c) {
            f->tcv_ms[p][c] = 0.f;
            if (!f->tcv_fits[p][c]) continue;
            for (int inv = 0; inv < 2; ++inv) {
                A2A_CUDA(cudaFuncSetAttribute(f->tcv[p][inv][c].fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)f->tcv[p][inv][c].smem),
                         "cudaFuncSetAttribute");
                // the ring form's tiles arrive by TMA, not through L1: give
                // the SM's unified memory to shared memory, so that two rings
                // fit per SM
                if (c >= 1)
                    A2A_CUDA(cudaFuncSetAttribute(f->tcv[p][inv][c].fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                                  100),
                             "cudaFuncSetAttribute");
            }
            // resident CTAs per SM, counted from the kernel's registers and
            // shared memory and the SM's limits (the runtime's occupancy
            // query answers 1 for these tensor-memory kernels although four
            // one-tile CTAs are resident per SM), and from tensor memory: an
            // SM has 512 columns, and a persistent CTA that waited for
            // columns would only start once another one finished
            const PassKernel& kk = f->tcv[p][0][c];
            cudaFuncAttributes fa;
            A2A_CUDA(cudaFuncGetAttributes(&fa, kk.fn), "cudaFuncGetAttributes");
            int dev = 0, smem_sm = 0, smem_rsv = 0, regs_sm = 0, thr_sm = 0;
            A2A_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
            A2A_CUDA(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev), "attr");
            A2A_CUDA(cudaDeviceGetAttribute(&smem_rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev), "attr");
            A2A_CUDA(cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev), "attr");
            A2A_CUDA(cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev), "attr");
            const size_t smem_cta = kk.smem + fa.sharedSizeBytes + (size_t)smem_rsv;
            const int regs_warp = (fa.numRegs * 32 + 255) / 256 * 256;  // allocated per warp, 256 at a time
            const int by_smem = (int)((size_t)smem_sm / smem_cta);
            const int by_regs = regs_sm / (regs_warp * (kk.threads / 32));
            const int by_thr = thr_sm / kk.threads;
            const int need = c == 4   ? 2 * a2a::tc2_cols(fmt)  // two regions
                             : c >= 2 ? (kk.threads / 256) * a2a::tc2_cols(fmt)
                                      : (kk.threads / a2a::kTcRows) * a2a::tc_block_cols(fmt);
            int cols = 32;
            while (cols < need) cols *= 2;
            f->tcv_occ[p][c] = std::min(std::min(by_smem, by_regs), std::min(by_thr, 512 / cols));
            if (f->tcv_occ[p][c] < 1) f->tcv_fits[p][c] = false;
        }
        if (!f->tcv_fits[p][0] && !f->tcv_fits[p][1])
            return fail(A2A_ERROR_UNSUPPORTED, "%s pass: no tensor-core kernel fits an SM", names[p]);
        f->tc_chosen[p] = f->tcv_fits[p][1] ? 1 : 0;  // the ring form by default
        for (int inv = 0; inv < 2; ++inv) f->tc[p][inv] = f->tcv[p][inv][f->tc_chosen[p]];
    }
    // twiddles of the tensor-core radix plans (per axis) and the operands
    std::vector<float> tw;
    size_t twpos[3];
    std::vector<long double> re, im;
    for (int axis = 0; axis < 3; ++axis) {
        const int p = axis == 2 ? 0 : axis == 0 ? 1 : 2;
        twpos[axis] = tw.size() / 2;
        gen_twiddles(f->tc[p][0], re, im);
        for (size_t i = 0; i < re.size(); ++i) {
            tw.push_back((float)re[i]);
            tw.push_back((float)im[i]);
        }
    }
    const size_t tw_bytes = ((tw.size() * sizeof(float)) + 255) & ~size_t(255);
    std::vector<uint16_t> b0, b1;
    tc_operand_image(false, fmt, b0);
    tc_operand_image(true, fmt, b1);
    // the two-stage form, per pass where it fits: W_n^(b k1) (forward sign,
    // [b < 32][k1 < n / 32]) and its operands per direction
    auto g_len = [&](int p) { return slot_geom(d, p).n; };
    std::vector<char> img2;  // host image of the segments, each 256-byte aligned
    size_t seg[3][3] = {};  // per pass: twiddle, forward and inverse operand offsets
    for (int p = 0; p < 3; ++p) {
        if (!f->tcv_fits[p][2] && !f->tcv_fits[p][3] && !f->tcv_fits[p][4]) continue;
        const int n = g_len(p);
        std::vector<float> t;
        const long double pi = acosl(-1.0L);
        for (int b = 0; b < 32; ++b)
            for (int k1 = 0; k1 < n / 32; ++k1) {
                const long double ang = 2.0L * pi * (long double)((b * k1) % n) / (long double)n;
                t.push_back((float)cosl(ang));
                t.push_back((float)-sinl(ang));
            }
        auto append = [&](const void* src, size_t bytes) {
            const size_t at = (img2.size() + 255) & ~size_t(255);
            img2.resize(at + bytes);
            std::memcpy(img2.data() + at, src, bytes);
            return at;
        };
        seg[p][0] = append(t.data(), t.size() * sizeof(float));
        for (int inv = 0; inv < 2; ++inv) {
            std::vector<uint16_t> img;
            tc2_operand_image(n, inv != 0, fmt, img);
            seg[p][1 + inv] = append(img.data(), img.size() * sizeof(uint16_t));
        }
    }
    const size_t img2_bytes = (img2.size() + 255) & ~size_t(255);
    if (f->d_tc) cudaFree(f->d_tc);
    f->d_tc = nullptr;
    const size_t bb = (size_t)a2a::tc_b_bytes(fmt);
    A2A_CUDA(cudaMalloc(&f->d_tc, tw_bytes + 2 * bb + img2_bytes), "cudaMalloc(tensor-core tables)");
    char* base = static_cast<char*>(f->d_tc);
    if (!tw.empty())
        A2A_CUDA(cudaMemcpy(base, tw.data(), tw.size() * sizeof(float), cudaMemcpyHostToDevice), "cudaMemcpy");
    A2A_CUDA(cudaMemcpy(base + tw_bytes, b0.data(), bb, cudaMemcpyHostToDevice), "cudaMemcpy");
    A2A_CUDA(cudaMemcpy(base + tw_bytes + bb, b1.data(), bb, cudaMemcpyHostToDevice), "cudaMemcpy");
    for (int axis = 0; axis < 3; ++axis) f->tc_tw[axis] = base + twpos[axis] * sizeof(float2);
    f->tc_b[0] = base + tw_bytes;
    f->tc_b[1] = base + tw_bytes + bb;
    char* base2 = base + tw_bytes + 2 * bb;  // 256-byte aligned (tw_bytes a 256-byte, bb a 2 KB multiple)
    if (!img2.empty())
        A2A_CUDA(cudaMemcpy(base2, img2.data(), img2.size(), cudaMemcpyHostToDevice), "cudaMemcpy");
    for (int p = 0; p < 3; ++p) {
        const bool any = f->tcv_fits[p][2] || f->tcv_fits[p][3] || f->tcv_fits[p][4];
        f->tc2_tw[p] = any ? base2 + seg[p][0] : nullptr;
        for (int inv = 0; inv < 2; ++inv) f->tc2_b[p][inv] = any ? base2 + seg[p][1 + inv] : nullptr;
    }
    return A2A_SUCCESS;
}

}  // namespace

namespace a2a {
a2a_status record_error(a2a_status s, const char* what, const char* detail) {
    return fail(s, "%s: %s", what, detail);
}
}  // namespace a2a

extern "C" {

a2a_status a2a_distribution_create(int ng, int world_size, int block_size, a2a_precision precision,
                                   a2a_distribution** out) {
    return create_common(ng, ng, ng, world_size, block_size, precision, out);
}

a2a_status a2a_distribution_create_box(int nx, int ny, int nz, int world_size, int block_size,
                                       a2a_precision precision, a2a_distribution** out) {
    return create_common(nx, ny, nz, world_size, block_size, precision, out);
}

a2a_status a2a_distribution_describe(const a2a_distribution* h, a2a_distribution_desc* o) {
    if (!h || !o) return fail(A2A_ERROR_INVALID_VALUE, "NULL argument");
    const Dist& d = h->d;
    o->ndims = 3;
    for (int a = 0; a < 3; ++a) {
        o->ng[a] = d.ng[a];
        o->dims[a] = d.dims[a];
        o->local_grid_size[a] = d.local[a];
    }
    o->world_size = d.P;
    o->nlocal = (int64_t)d.nlocal;
    o->nsends = (int64_t)d.chunk;
    o->block_size = d.block_size;
    o->precision = (int)d.prec;
    o->element_bytes = d.elem_bytes;
    o->buffer_bytes = (size_t)d.local_ranks * d.nlocal * d.elem_bytes;
    o->first_rank = d.first_rank;
    o->local_ranks = d.local_ranks;
    return A2A_SUCCESS;
}

a2a_status a2a_rank_coords(const a2a_distribution* h, int rank, int coords[3], int local_start[3]) {
    if (!h || !coords) return fail(A2A_ERROR_INVALID_VALUE, "NULL argument");
    const Dist& d = h->d;
    if (rank < 0 || rank >= d.P) return fail(A2A_ERROR_INVALID_VALUE, "rank %d outside [0, %d)", rank, d.P);
    coords[0] = rank / (d.dims[1] * d.dims[2]);
    coords[1] = (rank / d.dims[2]) % d.dims[1];
    coords[2] = rank % d.dims[2];
    if (local_start)
        for (int a = 0; a < 3; ++a) local_start[a] = d.local[a] * coords[a];
    return A2A_SUCCESS;
}

a2a_status a2a_distribution_set_stream(a2a_distribution* h, void* stream) {
    if (!h) return fail(A2A_ERROR_INVALID_VALUE, "distribution is NULL");
    h->d.stream = static_cast<cudaStream_t>(stream);
    return A2A_SUCCESS;
}

a2a_status a2a_get_z_pencils(a2a_distribution* h, void** b1, void** b2) {
    return step(h, b1, b2, [](Dist& d, void* p1, void* p2) {
        cudaError_t e = a2a::launch_alltoall(d, p1, p2, d.stream);
        if (e == cudaSuccess) e = a2a::launch_pencil_remap(d, 2, true, p2, p1, d.stream);
        return e;
    });
}

a2a_status a2a_return_z_pencils(a2a_distribution* h, void** b1, void** b2) {
    return step(h, b1, b2, [](Dist& d, void* p1, void* p2) {
        cudaError_t e = a2a::launch_pencil_remap(d, 2, false, p1, p2, d.stream);
        if (e == cudaSuccess) e = a2a::launch_alltoall(d, p2, p1, d.stream);
        return e;
    });
}

a2a_status a2a_get_x_pencils(a2a_distribution* h, void** b1, void** b2) {
    return step(h, b1, b2, [](Dist& d, void* p1, void* p2) {
        cudaError_t e = a2a::launch_fast_axis(d, 0, p1, p2, d.stream);
        if (e == cudaSuccess) e = a2a::launch_alltoall(d, p2, p1, d.stream);
        if (e == cudaSuccess) e = a2a::launch_pencil_remap(d, 0, true, p1, p2, d.stream);
        return e;
    });
}

a2a_status a2a_return_x_pencils(a2a_distribution* h, void** b1, void** b2) {
    return step(h, b1, b2, [](Dist& d, void* p1, void* p2) {
        cudaError_t e = a2a::launch_pencil_remap(d, 0, false, p2, p1, d.stream);
        if (e == cudaSuccess) e = a2a::launch_alltoall(d, p1, p2, d.stream);
        return e;
    });
}

a2a_status a2a_get_y_pencils(a2a_distribution* h, void** b1, void** b2) {
    return step(h, b1, b2, [](Dist& d, void* p1, void* p2) {
        cudaError_t e = a2a::launch_fast_axis(d, 1, p2, p1, d.stream);
        if (e == cudaSuccess) e = a2a::launch_alltoall(d, p1, p2, d.stream);
        if (e == cudaSuccess) e = a2a::launch_pencil_remap(d, 1, true, p2, p1, d.stream);
        return e;
    });
}

a2a_status a2a_return_y_pencils(a2a_distribution* h, void** b1, void** b2) {
    return step(h, b1, b2, [](Dist& d, void* p1, void* p2) {
        cudaError_t e = a2a::launch_pencil_remap(d, 1, false, p2, p1, d.stream);
        if (e == cudaSuccess) e = a2a::launch_alltoall(d, p1, p2, d.stream);
        if (e == cudaSuccess) e = a2a::launch_fast_axis(d, 2, p2, p1, d.stream);
        return e;
    });
}

// ---- the individual launchers of distribution/kernels/kernels.h:3-17 ----

static a2a_status one_kernel(a2a_distribution* h, void** src, void** dst, cudaError_t (*body)(Dist&, void*, void*)) {
    if (!h) return fail(A2A_ERROR_INVALID_VALUE, "distribution is NULL");
    Dist& d = h->d;
    a2a_status s;
    if ((s = need_cube(d, "the remap kernels")) != A2A_SUCCESS) return s;
    if ((s = check_buf(src, "source")) != A2A_SUCCESS) return s;
    if ((s = check_buf(dst, "dest")) != A2A_SUCCESS) return s;
    if (src[0] == dst[0]) return fail(A2A_ERROR_INVALID_VALUE, "source and dest must be distinct buffers");
    const cudaError_t e = body(d, src[0], dst[0]);
    if (e != cudaSuccess) return cuda_fail(e, "remap launch");
    return finish(d, d.stream, true);
}

a2a_status a2a_alltoall(a2a_distribution* h, void** src, void** dst) {
    if (h) {
        const a2a_status s = need_all_ranks(h->d, "the alltoall");
        if (s != A2A_SUCCESS) return s;
    }
    return one_kernel(h, src, dst, [](Dist& d, void* a, void* b) { return a2a::launch_alltoall(d, a, b, d.stream); });
}

a2a_status a2a_distribution_set_rank_range(a2a_distribution* h, int first, int count) {
    if (!h) return fail(A2A_ERROR_INVALID_VALUE, "distribution is NULL");
    Dist& d = h->d;
    if (first < 0 || count < 1 || first + count > d.P)
        return fail(A2A_ERROR_INVALID_VALUE, "rank range [%d, %d) outside [0, %d)", first, first + count, d.P);
    if (d.cube && ((uint64_t)count * d.nlocal) % ((uint64_t)d.ng[0] * d.ng[0]))
        return fail(A2A_ERROR_UNSUPPORTED, "%d ranks do not hold whole sets of Ng pencils of length Ng", count);
    d.first_rank = first;
    d.local_ranks = count;
    return A2A_SUCCESS;
}
a2a_status a2a_d_z_a2a_to_z_pencils(a2a_distribution* h, void** src, void** dst) {
    return one_kernel(h, src, dst,
                      [](Dist& d, void* a, void* b) { return a2a::launch_pencil_remap(d, 2, true, a, b, d.stream); });
}
a2a_status a2a_d_z_pencils_to_z_a2a(a2a_distribution* h, void** src, void** dst) {
    return one_kernel(h, src, dst,
                      [](Dist& d, void* a, void* b) { return a2a::launch_pencil_remap(d, 2, false, a, b, d.stream); });
}
a2a_status a2a_d_x_a2a_to_x_pencils(a2a_distribution* h, void** src, void** dst) {
    return one_kernel(h, src, dst,
                      [](Dist& d, void* a, void* b) { return a2a::launch_pencil_remap(d, 0, true, a, b, d.stream); });
}
a2a_status a2a_d_x_pencils_to_x_a2a(a2a_distribution* h, void** src, void** dst) {
    return one_kernel(h, src, dst,
                      [](Dist& d, void* a, void* b) { return a2a::launch_pencil_remap(d, 0, false, a, b, d.stream); });
}
a2a_status a2a_d_y_a2a_to_y_pencils(a2a_distribution* h, void** src, void** dst) {
    return one_kernel(h, src, dst,
                      [](Dist& d, void* a, void* b) { return a2a::launch_pencil_remap(d, 1, true, a, b, d.stream); });
}
a2a_status a2a_d_y_pencils_to_y_a2a(a2a_distribution* h, void** src, void** dst) {
    return one_kernel(h, src, dst,
                      [](Dist& d, void* a, void* b) { return a2a::launch_pencil_remap(d, 1, false, a, b, d.stream); });
}
a2a_status a2a_d_fast_z_to_x(a2a_distribution* h, void** src, void** dst) {
    return one_kernel(h, src, dst, [](Dist& d, void* a, void* b) { return a2a::launch_fast_axis(d, 0, a, b, d.stream); });
}
a2a_status a2a_d_fast_x_to_y(a2a_distribution* h, void** src, void** dst) {
    return one_kernel(h, src, dst, [](Dist& d, void* a, void* b) { return a2a::launch_fast_axis(d, 1, a, b, d.stream); });
}
a2a_status a2a_d_fast_y_to_z(a2a_distribution* h, void** src, void** dst) {
    return one_kernel(h, src, dst, [](Dist& d, void* a, void* b) { return a2a::launch_fast_axis(d, 2, a, b, d.stream); });
}

a2a_status a2a_distribution_finalize(a2a_distribution* h) {
    if (!h) return A2A_SUCCESS;
    release(h->d);
    delete h;
    return A2A_SUCCESS;
}

a2a_status a2a_forward_1d_fft(a2a_distribution* h, void** d_data) { return lines_1d(h, d_data, false); }
a2a_status a2a_inverse_1d_fft(a2a_distribution* h, void** d_data) { return lines_1d(h, d_data, true); }

a2a_status a2a_scale_fft(a2a_distribution* h, void** d_out, void** d_data) {
    if (!h) return fail(A2A_ERROR_INVALID_VALUE, "distribution is NULL");
    Dist& d = h->d;
    a2a_status s;
    if ((s = need_cube(d, "scale_fft")) != A2A_SUCCESS) return s;
    if ((s = check_buf(d_out, "d_out")) != A2A_SUCCESS) return s;
    if ((s = check_buf(d_data, "d_data")) != A2A_SUCCESS) return s;
    const double ng = d.ng[0];
    A2A_CUDA(a2a::launch_scale(d, d_data[0], d_out[0], ng * ng * ng, d.stream), "scale launch");
    return finish(d, d.stream, true);
}

a2a_status a2a_fast_copy_fft(a2a_distribution* h, void** d_out, void** d_data) {
    if (!h) return fail(A2A_ERROR_INVALID_VALUE, "distribution is NULL");
    Dist& d = h->d;
    a2a_status s;
    if ((s = check_buf(d_out, "d_out")) != A2A_SUCCESS) return s;
    if ((s = check_buf(d_data, "d_data")) != A2A_SUCCESS) return s;
    A2A_CUDA(cudaMemcpyAsync(d_out[0], d_data[0], (size_t)d.local_ranks * d.nlocal * d.elem_bytes, cudaMemcpyDeviceToDevice,
                             d.stream),
             "cudaMemcpyAsync");
    return finish(d, d.stream, true);
}

a2a_status a2a_dfft_create(a2a_distribution* dist, a2a_dfft** out) {
    if (!dist || !out) return fail(A2A_ERROR_INVALID_VALUE, "NULL argument");
    auto* f = new (std::nothrow) a2a_dfft();
    if (!f) return fail(A2A_ERROR_OUT_OF_MEMORY, "host allocation failed");
    f->dist = dist;
    *out = f;
    return A2A_SUCCESS;
}

a2a_status a2a_dfft_set_method(a2a_dfft* f, a2a_method m) {
    if (!f) return fail(A2A_ERROR_INVALID_VALUE, "dfft is NULL");
    if (m != A2A_METHOD_PLAIN && m != A2A_METHOD_SPLIT_BF16 && m != A2A_METHOD_SPLIT_FP16)
        return fail(A2A_ERROR_INVALID_VALUE, "unknown method %d", (int)m);
    if (m != A2A_METHOD_PLAIN) {
        const a2a_status s = setup_tc(f, m);
        if (s != A2A_SUCCESS) return s;
    }
    f->method = m;
    f->plans_made = false;
    return A2A_SUCCESS;
}

a2a_status a2a_dfft_make_plans(a2a_dfft* f, void** d_scratch) {
    if (!f) return fail(A2A_ERROR_INVALID_VALUE, "dfft is NULL");
    Dist& d = f->dist->d;
    f->scratch = d_scratch ? d_scratch[0] : nullptr;
    const char* names[3] = {"Z", "X", "Y"};
    for (int p = 0; p < 3; ++p)
        for (int inv = 0; inv < 2; ++inv) {
            const a2a::PassSlot& ps = d.slot[p][inv];
            if (!ps.fits[ps.chosen])
                return fail(A2A_ERROR_UNSUPPORTED, "%s pass: no compiled tile of length %d fits %d lines", names[p],
                            ps.cand[0].n, slot_geom(d, p).NV);
        }
    if (f->scratch && f->autotune && f->method == A2A_METHOD_PLAIN) {
        if (reinterpret_cast<uintptr_t>(f->scratch) % 16)
            return fail(A2A_ERROR_MISALIGNED, "d_scratch[0] is not 16-byte aligned");
        // time every fitting variant of each pass on the scratch buffer (its
        // contents are clobbered, as the reference allows) and keep the
        // fastest: one sweep over the passes, each candidate timed inside a
        // whole forward + inverse with the other passes' current choices (a
        // pass alone runs with a different cache and clock state than in the
        // transform)
        cudaStream_t st = d.stream;
        cudaEvent_t e0, e1;
        A2A_CUDA(cudaEventCreate(&e0), "cudaEventCreate");
        A2A_CUDA(cudaEventCreate(&e1), "cudaEventCreate");
        a2a_status status = A2A_SUCCESS;
        auto transform = [&]() {
            cudaError_t e = cudaSuccess;
            for (int inv = 0; inv < 2 && e == cudaSuccess; ++inv)
                for (int p = 0; p < 3 && e == cudaSuccess; ++p) e = run_pass(d, p, inv != 0, f->scratch, st);
            return e;
        };
        for (int p = 0; p < 3 && status == A2A_SUCCESS; ++p) {
            a2a::PassSlot& ps = d.slot[p][0];
            int best = ps.chosen;
            float best_ms = 1e30f;
            for (int c = 0; c < ps.ncand && status == A2A_SUCCESS; ++c) {
                ps.tuned_ms[c] = 0.f;
                if (!ps.fits[c]) continue;
                ps.chosen = c;
                d.slot[p][1].chosen = c;  // the inverse kernels share the variant list
                cudaError_t e = transform();  // warm-up
                float ms = 1e30f;
                for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
                    e = cudaEventRecord(e0, st);
                    if (e == cudaSuccess) e = transform();
                    if (e == cudaSuccess) e = cudaEventRecord(e1, st);
                    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                    float t = 0.f;
                    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
                    if (e == cudaSuccess) ms = std::min(ms, t);
                }
                if (e != cudaSuccess) {
                    status = cuda_fail(e, "autotune launch");
                    break;
                }
                ps.tuned_ms[c] = ms;
                if (ms < best_ms) {
                    best_ms = ms;
                    best = c;
                }
            }
            ps.chosen = best;
            d.slot[p][1].chosen = best;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (status != A2A_SUCCESS) return status;
    }
    if (f->scratch && f->autotune && f->method != A2A_METHOD_PLAIN) {
        if (reinterpret_cast<uintptr_t>(f->scratch) % 16)
            return fail(A2A_ERROR_MISALIGNED, "d_scratch[0] is not 16-byte aligned");
        // the same sweep over the tensor-core kernels: one tile per CTA or
        // the persistent ring form, per pass, timed inside a whole forward +
        // inverse on the scratch buffer
        cudaStream_t st = d.stream;
        cudaEvent_t e0, e1;
        A2A_CUDA(cudaEventCreate(&e0), "cudaEventCreate");
        A2A_CUDA(cudaEventCreate(&e1), "cudaEventCreate");
        cudaError_t e = cudaSuccess;
        auto transform = [&]() {
            cudaError_t r = cudaSuccess;
            for (int inv = 0; inv < 2 && r == cudaSuccess; ++inv)
                for (int p = 0; p < 3 && r == cudaSuccess; ++p) r = run_tc_pass(f, p, inv != 0, f->scratch, st);
            return r;
        };
        for (int p = 0; p < 3 && e == cudaSuccess; ++p) {
            int best = f->tc_chosen[p];
            float best_ms = 1e30f;
            for (int c = 0; c < 5 && e == cudaSuccess; ++c) {
                if (!f->tcv_fits[p][c]) continue;
                for (int inv = 0; inv < 2; ++inv) f->tc[p][inv] = f->tcv[p][inv][c];
                e = transform();  // warm-up
                float ms = 1e30f;
                for (int rep = 0; rep < 3 && e == cudaSuccess; ++rep) {
                    e = cudaEventRecord(e0, st);
                    if (e == cudaSuccess) e = transform();
                    if (e == cudaSuccess) e = cudaEventRecord(e1, st);
                    if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                    float t = 0.f;
                    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
                    if (e == cudaSuccess) ms = std::min(ms, t);
                }
                f->tcv_ms[p][c] = ms;
                if (e == cudaSuccess && ms < best_ms) {
                    best_ms = ms;
                    best = c;
                }
            }
            f->tc_chosen[p] = best;
            for (int inv = 0; inv < 2; ++inv) f->tc[p][inv] = f->tcv[p][inv][best];
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (e != cudaSuccess) return cuda_fail(e, "autotune launch");
        a2a_status s2 = check_device_flag(d);
        if (s2 != A2A_SUCCESS) return s2;
    }
    f->plans_made = true;
    return A2A_SUCCESS;
}

a2a_status a2a_dfft_check_device(const a2a_dfft* f) {
    if (!f) return fail(A2A_ERROR_INVALID_VALUE, "dfft is NULL");
    return check_device_flag(f->dist->d);
}

a2a_status a2a_dfft_variant_count(const a2a_dfft* f, int pass, int* count) {
    if (!f || !count) return fail(A2A_ERROR_INVALID_VALUE, "NULL argument");
    if (pass < 0 || pass > 2) return fail(A2A_ERROR_INVALID_VALUE, "pass must be 0 (Z), 1 (X) or 2 (Y)");
    *count = f->method == A2A_METHOD_PLAIN ? f->dist->d.slot[pass][0].ncand : 5;
    return A2A_SUCCESS;
}

a2a_status a2a_dfft_select_variant(a2a_dfft* f, int pass, int variant) {
    if (!f) return fail(A2A_ERROR_INVALID_VALUE, "dfft is NULL");
    if (pass < 0 || pass > 2) return fail(A2A_ERROR_INVALID_VALUE, "pass must be 0 (Z), 1 (X) or 2 (Y)");
    Dist& d = f->dist->d;
    if (f->method != A2A_METHOD_PLAIN) {  // 0: tile, 1: ring, 2: two-stage, 3: two-stage 8-line, 4: pipelined
        if (!f->tcv[pass][0][0].fn) return fail(A2A_ERROR_NO_PLANS, "the tensor-core kernels are not set up");
        if (variant < 0 || variant > 4) return fail(A2A_ERROR_INVALID_VALUE, "variant %d outside [0, 5)", variant);
        if (!f->tcv_fits[pass][variant])
            return fail(A2A_ERROR_UNSUPPORTED, "tensor-core variant %d does not fit this pass", variant);
        f->tc_chosen[pass] = variant;
        for (int inv = 0; inv < 2; ++inv) f->tc[pass][inv] = f->tcv[pass][inv][variant];
        return A2A_SUCCESS;
    }
    if (variant < 0 || variant >= d.slot[pass][0].ncand)
        return fail(A2A_ERROR_INVALID_VALUE, "variant %d outside [0, %d)", variant, d.slot[pass][0].ncand);
    if (!d.slot[pass][0].fits[variant] || !d.slot[pass][1].fits[variant])
        return fail(A2A_ERROR_UNSUPPORTED, "variant %d does not fit this pass's geometry", variant);
    d.slot[pass][0].chosen = variant;
    d.slot[pass][1].chosen = variant;
    return A2A_SUCCESS;
}

a2a_status a2a_dfft_set_autotune(a2a_dfft* f, int enable) {
    if (!f) return fail(A2A_ERROR_INVALID_VALUE, "dfft is NULL");
    f->autotune = enable != 0;
    return A2A_SUCCESS;
}

a2a_status a2a_dfft_plan_report(const a2a_dfft* f, char* buf, size_t len) {
    if (!f || !buf || len == 0) return fail(A2A_ERROR_INVALID_VALUE, "NULL argument");
    const Dist& d = f->dist->d;
    std::string out;
    const char* names[3] = {"Z", "X", "Y"};
    for (int p = 0; p < 3; ++p) {
        const a2a::PassSlot& ps = d.slot[p][0];
        for (int c = 0; c < ps.ncand; ++c) {
            const PassKernel& k = ps.cand[c];
            char line[256];
            snprintf(line, sizeof line,
                     "%s pass n=%d %s lines=%d lpt=%d threads=%d smem=%zu occ=%d radix=%d,%d,%d,%d fits=%d "
                     "tuned_ms=%.4f%s\n",
                     names[p], k.n,
                     k.kind == a2a::KIND_PIPE ? "pipe" : k.kind == a2a::KIND_TMA ? "tma"
                     : k.kind == a2a::KIND_RPIPE ? "rpipe" : k.kind == a2a::KIND_RPIPES ? "rpipes"
                     : k.kind == a2a::KIND_TMAT2 ? "tmat2"
                     : k.kind == a2a::KIND_TMAT3 ? "tmat3" : k.kind == a2a::KIND_TMAT2W ? "tmat2w"
                     : k.kind == a2a::KIND_TMATI ? "tmati" : k.kind == a2a::KIND_TMAT2S ? "tmat2s" : "direct",
                     k.lines, k.lpt, k.threads, k.smem,
                     ps.occ[c], k.radix[0], k.radix[1], k.radix[2], k.radix[3], (int)ps.fits[c], ps.tuned_ms[c],
                     c == ps.chosen ? " <- chosen" : "");
            out += line;
        }
    }
    if (f->method != A2A_METHOD_PLAIN)
        for (int p = 0; p < 3; ++p)
            for (int c = 0; c < 5; ++c) {
                if (!f->tcv_fits[p][c]) continue;
                const PassKernel& k = f->tcv[p][0][c];
                char line[256];
                snprintf(line, sizeof line,
                         "%s pass n=%d tensor-core %s %s lines=%d threads=%d smem=%zu occ=%d radix=%d,%d,%d "
                         "tuned_ms=%.4f%s\n",
                         names[p], k.n, f->method == A2A_METHOD_SPLIT_FP16 ? "split-fp16" : "split-bf16",
                         c == 4 ? "two-stage-pipelined" : c >= 2 ? "two-stage" : c ? "ring" : "tile", k.lines, k.threads, k.smem, f->tcv_occ[p][c], k.radix[0], k.radix[1],
                         k.radix[2], f->tcv_ms[p][c], c == f->tc_chosen[p] ? " <- in use" : "");
                out += line;
            }
    snprintf(buf, len, "%s", out.c_str());
    return out.size() < len ? A2A_SUCCESS : fail(A2A_ERROR_INVALID_VALUE, "report truncated (%zu bytes)", out.size());
}

a2a_status a2a_dfft_forward(a2a_dfft* f, void** d_data) {
    return fused(f, d_data, false, f ? f->dist->d.stream : nullptr, true);
}
a2a_status a2a_dfft_inverse(a2a_dfft* f, void** d_data) {
    return fused(f, d_data, true, f ? f->dist->d.stream : nullptr, true);
}
a2a_status a2a_dfft_backward(a2a_dfft* f, void** d_data) { return a2a_dfft_inverse(f, d_data); }
a2a_status a2a_dfft_forward_async(a2a_dfft* f, void** d_data, void* stream) {
    return fused(f, d_data, false, static_cast<cudaStream_t>(stream), false);
}
a2a_status a2a_dfft_inverse_async(a2a_dfft* f, void** d_data, void* stream) {
    return fused(f, d_data, true, static_cast<cudaStream_t>(stream), false);
}

a2a_status a2a_dfft_execute_pass_async(a2a_dfft* f, void** d_data, int pass, int inverse, void* stream) {
    a2a_status s;
    if ((s = check_dfft(f, d_data)) != A2A_SUCCESS) return s;
    if (pass < 0 || pass > 2) return fail(A2A_ERROR_INVALID_VALUE, "pass must be 0 (Z), 1 (X) or 2 (Y)");
    if (f->method == A2A_METHOD_PLAIN)
        A2A_CUDA(run_pass(f->dist->d, pass, inverse != 0, d_data[0], static_cast<cudaStream_t>(stream)),
                 "axis pass launch");
    else
        A2A_CUDA(run_tc_pass(f, pass, inverse != 0, d_data[0], static_cast<cudaStream_t>(stream)),
                 "tensor-core pass launch");
    return A2A_SUCCESS;
}

a2a_status a2a_dfft_execute_pass_blocks(a2a_dfft* f, void** blocks, int nblocks, int pass, int inverse, int part,
                                        int nparts, void* stream) {
    if (!f) return fail(A2A_ERROR_INVALID_VALUE, "dfft is NULL");
    const Dist& d = f->dist->d;
    a2a_status s;
    if ((s = need_all_ranks(d, "the multi-block pass (its tables are global)")) != A2A_SUCCESS) return s;
    if (pass < 0 || pass > 2) return fail(A2A_ERROR_INVALID_VALUE, "pass must be 0 (Z), 1 (X) or 2 (Y)");
    if (nblocks < 1 || nblocks > a2a::kMbMaxBlocks || d.P % nblocks)
        return fail(A2A_ERROR_INVALID_VALUE, "nblocks must divide world_size=%d and be in [1, %d]", d.P,
                    a2a::kMbMaxBlocks);
    if (nparts < 1 || part < 0 || part >= nparts) return fail(A2A_ERROR_INVALID_VALUE, "part must be in [0, nparts)");
    if (!blocks) return fail(A2A_ERROR_INVALID_VALUE, "blocks is NULL");
    for (int i = 0; i < nblocks; ++i) {
        if (!blocks[i]) return fail(A2A_ERROR_INVALID_VALUE, "blocks[%d] is NULL", i);
        if (reinterpret_cast<uintptr_t>(blocks[i]) % 16)
            return fail(A2A_ERROR_MISALIGNED, "blocks[%d] is not 16-byte aligned", i);
    }
    const SlotGeom g = slot_geom(d, pass);
    PassKernel k;
    // batch-mode passes: the TMA-fed kernel where its boxes fit the bricks
    bool tma = false;
    if (f->mb_persistent && g.mode == a2a::MODE_BATCH && a2a::find_mb_tmat_kernel(d.prec, g.n, inverse != 0, &k)) {
        const int w = d.prec == A2A_C128 ? 2 : 1;
        const int l = pass == 1 ? d.local[0] : d.local[1];
        tma = g.NV % k.lines == 0 && d.local[2] % k.lines == 0 && l <= 256 && w * k.lines <= 256 &&
              ((size_t)k.lines * l * d.elem_bytes) % 128 == 0 && (d.nlocal * d.elem_bytes) % 16 == 0 &&
              d.P <= 4096 && tmap_encoder() != nullptr;
    }
    const bool persistent = tma || (f->mb_persistent &&
                                    a2a::find_mb_rpipe_kernel(d.prec, g.n, g.mode, inverse != 0, &k) &&
                                    g.NV % k.lines == 0);
    if (!persistent) {
        if (!a2a::find_mb_kernel(d.prec, g.n, g.mode, inverse != 0, &k))
            return fail(A2A_ERROR_UNSUPPORTED, "no multi-block pass kernel of length %d (lengths 4, 8, 16 have none)",
                        g.n);
        if (g.NV % k.lines &&
            !(a2a::find_mb_kernel_small(d.prec, g.n, g.mode, inverse != 0, &k) && g.NV % k.lines == 0))
            return fail(A2A_ERROR_UNSUPPORTED, "%d lines are not a multiple of a 4-line tile", g.NV);
    }
    A2A_CUDA(cudaFuncSetAttribute(k.fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem),
             "cudaFuncSetAttribute");
    const int64_t tiles = (int64_t)g.NU * (g.NV / k.lines);
    const int64_t t0 = tiles * part / nparts, t1 = tiles * (part + 1) / nparts;
    if (t1 <= t0) return A2A_SUCCESS;
    int64_t grid = t1 - t0;
    if (persistent) {  // one wave of resident CTAs works through the part's tiles
        int occ = 0;
        A2A_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k.fn, k.threads, k.smem),
                 "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        grid = std::min<int64_t>(grid, (int64_t)std::max(occ, 1) * d.sms);
    }
    const double scale = (inverse && pass == 2) ? 1.0 / ((double)d.ng[0] * d.ng[1] * d.ng[2]) : 1.0;
    const uint32_t block_elems = (uint32_t)((uint64_t)(d.P / nblocks) * d.nlocal);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    a2a::MbTmaMaps mm;
    std::memset(&mm, 0, sizeof(mm));
    if (tma) {
        // one 3-D tensor map per virtual rank over its brick [x_l][y_l][z_l]
        // at its block's address, box [B, 1, lx] (X) or [B, ly, 1] (Y) words;
        // rebuilt when the blocks or the tile height change
        const int w = d.prec == A2A_C128 ? 2 : 1;
        const int lx = d.local[0], ly = d.local[1], lz = d.local[2];
        std::vector<const void*> key(blocks, blocks + nblocks);
        const size_t per = sizeof(CUtensorMap) * (size_t)d.P;
        if (!f->d_mbmaps) A2A_CUDA(cudaMalloc(&f->d_mbmaps, 3 * per), "cudaMalloc(multi-block tensor maps)");
        CUtensorMap* dmaps = reinterpret_cast<CUtensorMap*>(static_cast<char*>(f->d_mbmaps) + pass * per);
        if (f->mbmaps_key[pass] != key || f->mbmaps_lines[pass] != k.lines) {
            std::vector<CUtensorMap> hmaps((size_t)d.P);
            const TmapEncodeFn enc = tmap_encoder();
            const cuuint64_t dims[3] = {(cuuint64_t)w * lz, (cuuint64_t)ly, (cuuint64_t)lx};
            const cuuint64_t strides[2] = {(cuuint64_t)lz * d.elem_bytes, (cuuint64_t)ly * lz * d.elem_bytes};
            const cuuint32_t box[3] = {(cuuint32_t)(w * k.lines), (cuuint32_t)(pass == 1 ? 1 : ly),
                                       (cuuint32_t)(pass == 1 ? lx : 1)};
            const cuuint32_t estr[3] = {1, 1, 1};
            const int L = d.P / nblocks;
            for (int r = 0; r < d.P; ++r) {
                void* base = static_cast<char*>(blocks[r / L]) + (size_t)(r % L) * d.nlocal * d.elem_bytes;
                if (enc(&hmaps[r], CU_TENSOR_MAP_DATA_TYPE_INT64, 3, base, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
                    return fail(A2A_ERROR_CUDA, "cuTensorMapEncodeTiled refused a brick of the multi-block pass");
            }
            A2A_CUDA(cudaStreamSynchronize(st), "cudaStreamSynchronize");  // earlier passes may read the old maps
            A2A_CUDA(cudaMemcpy(dmaps, hmaps.data(), per, cudaMemcpyHostToDevice), "cudaMemcpy(tensor maps)");
            f->mbmaps_key[pass] = key;
            f->mbmaps_lines[pass] = k.lines;
        }
        mm.map = dmaps;
        mm.pass = pass;
        mm.lx = lx;
        mm.ly = ly;
        mm.lz = lz;
        mm.words = w;
        mm.d1 = d.dims[1];
        mm.d2 = d.dims[2];
        mm.nbox = pass == 1 ? d.dims[0] : d.dims[1];
    }
    cudaError_t e;
    auto launch = [&](auto tag) {
        using T = decltype(tag);
        a2a::PassArgs<T> a;
        a.src = nullptr;
        a.dst = nullptr;
        a.offA = g.offA;
        a.offU = g.offU;
        a.offV = g.offV;
        a.tw = static_cast<const a2a::cx<T>*>(g.tw);
        a.NU = g.NU;
        a.NV = g.NV;
        a.scale = T(scale);
        a.split = 0;
        a.err = d.d_err;
        a.tcb = nullptr;
        a2a::MbArgs<T> mb;
        for (int i = 0; i < a2a::kMbMaxBlocks; ++i) mb.blk[i] = static_cast<a2a::cx<T>*>(blocks[i < nblocks ? i : 0]);
        mb.fbe = a2a::FastDiv(block_elems);
        mb.nblk = nblocks;
        mb.tile0 = (int)t0;
        mb.tile1 = (int)t1;
        void* args[] = {&a, &mb, &mm};
        return cudaLaunchKernel(k.fn, dim3((unsigned)grid), dim3(k.threads), args, k.smem, st);
    };
    e = d.prec == A2A_C128 ? launch(double()) : launch(float());
    A2A_CUDA(e, "multi-block pass launch");
    return A2A_SUCCESS;
}

a2a_status a2a_dfft_set_blocks_kernel(a2a_dfft* f, int persistent) {
    if (!f) return fail(A2A_ERROR_INVALID_VALUE, "dfft is NULL");
    f->mb_persistent = persistent != 0;
    return A2A_SUCCESS;
}

a2a_status a2a_dfft_launches_per_transform(const a2a_dfft* f, int* out) {
    if (!f || !out) return fail(A2A_ERROR_INVALID_VALUE, "NULL argument");
    *out = 3;
    return A2A_SUCCESS;
}

a2a_status a2a_dfft_destroy(a2a_dfft* f) {
    if (f && f->d_tc) cudaFree(f->d_tc);
    if (f && f->d_mbmaps) cudaFree(f->d_mbmaps);
    delete f;
    return A2A_SUCCESS;
}

// ---- dump files (a2adistribution.cpp:101-111, tests/test.cpp:69-125) ----

static a2a_status host_decomp(int ng, int P, int dims[3], int local[3], long long* nlocal) {
    if (ng < 1 || P < 1) return fail(A2A_ERROR_INVALID_VALUE, "ng and world_size must be >= 1");
    dims_create(P, dims);
    for (int a = 0; a < 3; ++a)
        if (ng % dims[a] || P % dims[a])
            return fail(A2A_ERROR_DECOMPOSITION, "Ng=%d / world_size=%d do not divide by dims[%d]=%d", ng, P, a,
                        dims[a]);
    for (int a = 0; a < 3; ++a) local[a] = ng / dims[a];
    const long long lx = local[0], ly = local[1], lz = local[2];
    if ((lx * ly) % P || (lx * lz) % P || (ly * lz) % P)
        return fail(A2A_ERROR_DECOMPOSITION, "a face of the brick is not divisible by world_size=%d", P);
    *nlocal = lx * ly * lz;
    return A2A_SUCCESS;
}

a2a_status a2a_decompose(int ng, int world_size, int dims[3], int local_grid_size[3], int64_t* nlocal) {
    if (!dims || !local_grid_size || !nlocal) return fail(A2A_ERROR_INVALID_VALUE, "NULL argument");
    long long n = 0;
    const a2a_status s = host_decomp(ng, world_size, dims, local_grid_size, &n);
    *nlocal = (int64_t)n;
    return s;
}

a2a_status a2a_write_dims(int ng, int world_size, const char* path) {
    int dims[3], local[3];
    long long nlocal;
    a2a_status s;
    if (!path) return fail(A2A_ERROR_INVALID_VALUE, "path is NULL");
    if ((s = host_decomp(ng, world_size, dims, local, &nlocal)) != A2A_SUCCESS) return s;
    if (nlocal > 2147483647LL) return fail(A2A_ERROR_UNSUPPORTED, "nlocal does not fit the 32-bit field");
    FILE* fh = fopen(path, "wb");
    if (!fh) return fail(A2A_ERROR_INVALID_VALUE, "cannot open %s", path);
    const int head[3] = {world_size, ng, (int)nlocal};
    size_t w = fwrite(head, sizeof(int), 3, fh);
    w += fwrite(dims, sizeof(int), 3, fh);
    w += fwrite(local, sizeof(int), 3, fh);
    fclose(fh);
    if (w != 9) return fail(A2A_ERROR_INVALID_VALUE, "short write to %s", path);
    return A2A_SUCCESS;
}

a2a_status a2a_write_rank_dumps(int ng, int world_size, a2a_precision precision, const char* folder,
                                const void* host_input, const void* host_forward, const void* host_inverse) {
    int dims[3], local[3];
    long long nlocal;
    a2a_status s;
    if (!folder || !host_input || !host_forward || !host_inverse)
        return fail(A2A_ERROR_INVALID_VALUE, "NULL argument");
    if (precision != A2A_C128 && precision != A2A_C64)
        return fail(A2A_ERROR_INVALID_VALUE, "unknown precision %d", (int)precision);
    if ((s = host_decomp(ng, world_size, dims, local, &nlocal)) != A2A_SUCCESS) return s;
    const size_t eb = precision == A2A_C128 ? 16 : 8;
    const size_t rank_bytes = (size_t)nlocal * eb;
    const void* parts[3] = {host_input, host_forward, host_inverse};
    for (int r = 0; r < world_size; ++r) {
        char path[4096];
        snprintf(path, sizeof path, "%s/proc%d", folder, r);
        FILE* fh = fopen(path, "wb");
        if (!fh) return fail(A2A_ERROR_INVALID_VALUE, "cannot open %s", path);
        for (const void* part : parts) {
            if (fwrite(static_cast<const char*>(part) + (size_t)r * rank_bytes, 1, rank_bytes, fh) != rank_bytes) {
                fclose(fh);
                return fail(A2A_ERROR_INVALID_VALUE, "short write to %s", path);
            }
        }
        fclose(fh);
    }
    return A2A_SUCCESS;
}

// ---- host-staged transforms (fft_demo/fft_3d/fft_3d.c:6-189) ----

static a2a_status host_staged(a2a_dfft* f, void* host, void** d_buf, bool inv) {
    if (!f || !host) return fail(A2A_ERROR_INVALID_VALUE, "NULL argument");
    a2a_status s;
    if ((s = check_dfft(f, d_buf)) != A2A_SUCCESS) return s;
    const Dist& d = f->dist->d;
    const size_t bytes = (size_t)d.P * d.nlocal * d.elem_bytes;
    A2A_CUDA(cudaMemcpyAsync(d_buf[0], host, bytes, cudaMemcpyHostToDevice, d.stream), "cudaMemcpyAsync(H2D)");
    if ((s = fused(f, d_buf, inv, d.stream, false)) != A2A_SUCCESS) return s;
    A2A_CUDA(cudaMemcpyAsync(host, d_buf[0], bytes, cudaMemcpyDeviceToHost, d.stream), "cudaMemcpyAsync(D2H)");
    A2A_CUDA(cudaStreamSynchronize(d.stream), "cudaStreamSynchronize");
    return check_device_flag(d);
}

a2a_status a2a_dfft_forward_host(a2a_dfft* f, void* host_data, void** d_buffer) {
    return host_staged(f, host_data, d_buffer, false);
}
a2a_status a2a_dfft_inverse_host(a2a_dfft* f, void* host_data, void** d_buffer) {
    return host_staged(f, host_data, d_buffer, true);
}

// ---- CUDA IPC for the multi-block pass ----

// Imported allocations, one entry per (device, handle): opened once and
// closed when the last import of it is released, so two objects of one
// process that import the same peer buffer share one mapping.
struct IpcMapping {
    int device;
    unsigned char handle[sizeof(cudaIpcMemHandle_t)];
    void* base;
    int refs;
};
static std::mutex g_ipc_mutex;
static std::vector<IpcMapping> g_ipc_open;
static std::vector<std::pair<void*, size_t>> g_ipc_maps;  // (imported address, index into g_ipc_open)

using MemRangeFn = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);

static MemRangeFn mem_range_fn() {
    static MemRangeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<MemRangeFn>(p);
    });
    return fn;
}

a2a_status a2a_ipc_export(const void* dev_ptr, void* handle, uint64_t* offset) {
    if (!dev_ptr || !handle || !offset) return fail(A2A_ERROR_INVALID_VALUE, "NULL argument");
    static_assert(sizeof(cudaIpcMemHandle_t) <= A2A_IPC_HANDLE_BYTES, "IPC handle size");
    const MemRangeFn range = mem_range_fn();
    if (!range) return fail(A2A_ERROR_CUDA, "cuMemGetAddressRange is not available");
    CUdeviceptr base = 0;
    size_t size = 0;
    if (range(&base, &size, reinterpret_cast<CUdeviceptr>(dev_ptr)) != CUDA_SUCCESS)
        return fail(A2A_ERROR_INVALID_VALUE, "dev_ptr is not device memory of this process");
    cudaIpcMemHandle_t h;
    A2A_CUDA(cudaIpcGetMemHandle(&h, reinterpret_cast<void*>(base)), "cudaIpcGetMemHandle");
    std::memset(handle, 0, A2A_IPC_HANDLE_BYTES);
    std::memcpy(handle, &h, sizeof(h));
    *offset = (uint64_t)(reinterpret_cast<CUdeviceptr>(dev_ptr) - base);
    return A2A_SUCCESS;
}

a2a_status a2a_ipc_import(const void* handle, uint64_t offset, void** dev_ptr) {
    if (!handle || !dev_ptr) return fail(A2A_ERROR_INVALID_VALUE, "NULL argument");
    int dev = 0;
    A2A_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(g_ipc_mutex);
    size_t idx = g_ipc_open.size();
    for (size_t i = 0; i < g_ipc_open.size(); ++i)
        if (g_ipc_open[i].refs > 0 && g_ipc_open[i].device == dev &&
            std::memcmp(g_ipc_open[i].handle, handle, sizeof(cudaIpcMemHandle_t)) == 0)
            idx = i;
    if (idx == g_ipc_open.size()) {
        cudaIpcMemHandle_t h;
        std::memcpy(&h, handle, sizeof(h));
        void* base = nullptr;
        A2A_CUDA(cudaIpcOpenMemHandle(&base, h, cudaIpcMemLazyEnablePeerAccess), "cudaIpcOpenMemHandle");
        IpcMapping m;
        m.device = dev;
        std::memcpy(m.handle, handle, sizeof(m.handle));
        m.base = base;
        m.refs = 0;
        idx = g_ipc_open.size();
        for (size_t i = 0; i < g_ipc_open.size(); ++i)  // reuse a closed slot
            if (g_ipc_open[i].refs == 0) {
                idx = i;
                break;
            }
        if (idx == g_ipc_open.size()) g_ipc_open.push_back(m);
        else g_ipc_open[idx] = m;
    }
    ++g_ipc_open[idx].refs;
    *dev_ptr = static_cast<char*>(g_ipc_open[idx].base) + offset;
    g_ipc_maps.emplace_back(*dev_ptr, idx);
    return A2A_SUCCESS;
}

a2a_status a2a_ipc_release(void* dev_ptr) {
    void* close = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_ipc_mutex);
        auto it = g_ipc_maps.begin();
        while (it != g_ipc_maps.end() && it->first != dev_ptr) ++it;
        if (it == g_ipc_maps.end())
            return fail(A2A_ERROR_INVALID_VALUE, "dev_ptr was not imported with a2a_ipc_import");
        IpcMapping& m = g_ipc_open[it->second];
        g_ipc_maps.erase(it);
        if (--m.refs == 0) close = m.base;
    }
    if (close) A2A_CUDA(cudaIpcCloseMemHandle(close), "cudaIpcCloseMemHandle");
    return A2A_SUCCESS;
}

const char* a2a_status_string(a2a_status s) {
    switch (s) {
        case A2A_SUCCESS: return "success";
        case A2A_ERROR_INVALID_VALUE: return "invalid value";
        case A2A_ERROR_DECOMPOSITION: return "decomposition rejected";
        case A2A_ERROR_UNSUPPORTED: return "unsupported size";
        case A2A_ERROR_NO_PLANS: return "make_plans not called";
        case A2A_ERROR_MISALIGNED: return "misaligned buffer";
        case A2A_ERROR_CUDA: return "CUDA error";
        case A2A_ERROR_OUT_OF_MEMORY: return "out of memory";
        case A2A_ERROR_TIMEOUT: return "device wait timed out";
        case A2A_ERROR_NOT_IMPLEMENTED: return "not implemented";
    }
    return "unknown status";
}

const char* a2a_last_error(void) { return g_last_error.c_str(); }

int a2a_version(void) { return A2AFFT_B200_VERSION; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched form: many independent boxes (each decomposed over its own virtual
// ranks, as a2a_distribution_create_box lays them out) transformed by one
// persistent kernel launch per direction, replayed from a CUDA graph.  No
// counterpart in the reference, which transforms one grid per plan.
// ---------------------------------------------------------------------------

struct a2a_batch {
    a2a_precision prec = A2A_C64;
    int P = 0;
    int nboxes = 0;
    int sms = 148;
    std::vector<a2a_distribution*> dists;  // one per distinct box shape (offset tables, twiddles)
    std::vector<int> box_dist;             // box -> index into dists
    std::vector<a2a::BatchBox> hbox;
    std::vector<int2> items;               // (box * 4 + pass, tile), pass-major
    int pass_start[4] = {0, 0, 0, 0};
    a2a::BatchBox* d_boxes = nullptr;
    int2* d_items = nullptr;
    size_t items_cap = 0;
    // queue scratch: [0] abort, [1..3] items taken per launch, [4..] tiles
    // done per (box, pass); then the error flag (outside the cleared range)
    int* d_queue = nullptr;
    size_t queue_ints = 0;
    int var[2][a2a::kBatchNumLengths] = {};  // tile variant per (mode, length)
    bool used[2][a2a::kBatchNumLengths] = {};
    float tuned_ms[2][a2a::kBatchNumLengths][a2a::kBatchVariants] = {};
    bool pairs_ok[a2a::kBatchNumLengths] = {};  // batch-mode line pairs usable for every box of the length
    int fused = 1;   // 1: one launch per direction; 0: one launch per pass
    int claim = 16;
    int wait_extra = 0;
    int prefetch = 1;
    bool use_graph = true;
    size_t smem = 0;
    int grid = 0;
    cudaStream_t cap = nullptr;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    std::vector<void*> bound;  // data pointers held in d_boxes

    // Grouped schedule (fused == 2): the boxes of one shape form one tall
    // grid per pass (line bases = box offset + the shape's own outer-line
    // offsets, from the group's lowest box pointer), transformed by the
    // single-grid pass kernels, one launch per (shape, pass); the shapes run
    // on parallel branches (forked streams, a graph with one branch per shape
    // when captured).
    struct Group {
        int dist = 0;                  // index into dists
        std::vector<int> boxes;        // its boxes, in box order
        int64_t elems = 0;             // elements of all its boxes
        size_t tab[3] = {0, 0, 0};     // start of its per-pass line-base tables in d_gtab
        int chosen[3] = {-1, -1, -1};  // candidate per pass in the distribution's slot lists
        float tuned_ms[3][a2a::kMaxVariants] = {};
        void* base = nullptr;          // lowest box pointer of the bound buffers
    };
    std::vector<Group> groups;         // largest first
    bool grouped_possible = false;     // every (shape, pass) has a kernel the grouped schedule can run
    bool grouped_ok = false;           // the bound buffers' offsets fit the 32-bit line-base tables
    uint32_t* d_gtab = nullptr;
    size_t gtab_entries = 0;
    std::vector<cudaStream_t> gstreams;
    cudaEvent_t gfork = nullptr;
    std::vector<cudaEvent_t> gjoin;
};

namespace {

int batch_len_index(int n) {
    for (int i = 0; i < a2a::kBatchNumLengths; ++i)
        if (a2a::kBatchLengths[i] == n) return i;
    return -1;
}

void batch_drop_graphs(a2a_batch* b) {
    for (auto& e : b->exec)
        if (e) {
            cudaGraphExecDestroy(e);
            e = nullptr;
        }
}

// Per-pass geometry of box i: transform length, lines NU x NV (as slot_geom).
void batch_pass_geom(const a2a_batch* b, int i, int pass, int& n, int& NU, int& NV) {
    const Dist& d = b->dists[b->box_dist[i]]->d;
    if (pass == 0) { n = d.ng[2]; NU = d.ng[0]; NV = d.ng[1]; }
    else if (pass == 1) { n = d.ng[0]; NU = d.ng[1]; NV = d.ng[2]; }
    else { n = d.ng[1]; NU = d.ng[0]; NV = d.ng[2]; }
}

// Can the grouped schedule run candidate c of pass `pass` of shape d?  Both
// directions must have it fitting the shape's geometry, and it must address
// its lines through the offset tables (the tensor-map ring kernels describe
// one buffer per map, so a tall grid of boxes is not one tensor).  The
// geometry checks carry over from one box to the group: line bases only gain
// box offsets, which are multiples of 16 bytes.
bool group_eligible(const Dist& d, int pass, int c) {
    for (int inv = 0; inv < 2; ++inv) {
        const a2a::PassSlot& ps = d.slot[pass][inv];
        if (c < 0 || c >= ps.ncand || !ps.fits[c] || is_tmat(ps.cand[c])) return false;
    }
    return true;
}

// One pass of one group: the chosen single-grid kernel over the group's tall
// grid (K boxes x NU outer lines), in place from the group's base pointer.
cudaError_t group_pass(const a2a_batch* b, const a2a_batch::Group& g, int pass, bool inv, cudaStream_t st) {
    const Dist& d = b->dists[g.dist]->d;
    const int c = g.chosen[pass];
    const a2a::PassSlot& ps = d.slot[pass][inv ? 1 : 0];
    const PassKernel& k = ps.cand[c];
    const SlotGeom geo = slot_geom(d, pass);
    const uint64_t NU = (uint64_t)geo.NU * g.boxes.size();
    const uint64_t tiles = NU * (uint64_t)(geo.NV / k.lines);
    uint64_t grid = tiles;
    if (persistent_kind(k)) grid = std::min(tiles, (uint64_t)std::max(ps.occ[c], 1) * d.sms);
    const int l = pass == 0 ? d.local[2] : pass == 1 ? d.local[0] : d.local[1];
    const int split = split_ok(l, k);
    const void* tw = ps.tw[c] ? ps.tw[c] : geo.tw;
    const double scale = (inv && pass == 2) ? 1.0 / ((double)d.ng[0] * d.ng[1] * d.ng[2]) : 1.0;
    const uint32_t* offU = b->d_gtab + g.tab[pass];
    int* err = b->d_queue + b->queue_ints;
    if (b->prec == A2A_C128)
        return launch_pass_t<double>(k, unsigned(grid), g.base, g.base, geo.offA, offU, geo.offV, tw, (int)NU,
                                     geo.NV, scale, split, err, st);
    return launch_pass_t<float>(k, unsigned(grid), g.base, g.base, geo.offA, offU, geo.offV, tw, (int)NU, geo.NV,
                                scale, split, err, st);
}

// One direction of the grouped schedule: fork the caller's stream into the
// group streams, Z, X, Y of each group on its stream, join back.
cudaError_t batch_group_launches(a2a_batch* b, bool inv, cudaStream_t st) {
    cudaError_t e = cudaEventRecord(b->gfork, st);
    for (size_t gi = 0; gi < b->groups.size() && e == cudaSuccess; ++gi) {
        cudaStream_t s = b->gstreams[gi % b->gstreams.size()];
        e = cudaStreamWaitEvent(s, b->gfork, 0);
        for (int p = 0; p < 3 && e == cudaSuccess; ++p) e = group_pass(b, b->groups[gi], p, inv, s);
        if (e == cudaSuccess) e = cudaEventRecord(b->gjoin[gi], s);
    }
    for (size_t gi = 0; gi < b->groups.size() && e == cudaSuccess; ++gi) e = cudaStreamWaitEvent(st, b->gjoin[gi], 0);
    return e;
}

// Line-base tables of every group for the bound buffers: entry (k, u) of
// pass p = (box k's pointer - group base) / element size + the shape's outer
// offset u.  Sets grouped_ok (false when some group's boxes lie too far apart
// for 32-bit element offsets; the grouped schedule then runs as the one-launch
// schedule).  Returns whether any group's base pointer changed.
bool batch_group_tables(a2a_batch* b, cudaStream_t st, cudaError_t* err) {
    *err = cudaSuccess;
    b->grouped_ok = false;
    if (!b->grouped_possible) return false;
    bool moved = false;
    std::vector<uint32_t> h(b->gtab_entries);
    const size_t eb = b->prec == A2A_C128 ? 16 : 8;
    for (a2a_batch::Group& g : b->groups) {
        const Dist& d = b->dists[g.dist]->d;
        uintptr_t lo = UINTPTR_MAX;
        for (int i : g.boxes) lo = std::min(lo, reinterpret_cast<uintptr_t>(b->bound[i]));
        std::vector<uint64_t> boff;
        for (int i : g.boxes) {
            const uint64_t o = (reinterpret_cast<uintptr_t>(b->bound[i]) - lo) / eb;  // pointers are 16-byte aligned
            if (o + d.nlocal * (uint64_t)d.P > (uint64_t(1) << 32)) return moved;
            boff.push_back(o);
        }
        if (g.base != reinterpret_cast<void*>(lo)) moved = true;
        g.base = reinterpret_cast<void*>(lo);
        for (int p = 0; p < 3; ++p) {
            const std::vector<uint32_t>& hU = *slot_geom(d, p).hU;
            size_t pos = g.tab[p];
            for (uint64_t o : boff)
                for (uint32_t u : hU) h[pos++] = (uint32_t)(o + u);
        }
    }
    // pageable source: staged before the call returns, ordered before the
    // launches that follow on `st`
    *err = cudaMemcpyAsync(b->d_gtab, h.data(), h.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, st);
    b->grouped_ok = *err == cudaSuccess;
    return moved;
}

// Tiles per pass, the item list, launch shared memory and grid from the
// current variants; uploads the box table and the items.
a2a_status batch_layout(a2a_batch* b) {
    batch_drop_graphs(b);
    b->items.clear();
    size_t smem = 0;
    for (int p = 0; p < 3; ++p) {
        b->pass_start[p] = (int)b->items.size();
        for (int i = 0; i < b->nboxes; ++i) {
            int n, NU, NV;
            batch_pass_geom(b, i, p, n, NU, NV);
            const int mode = p == 0 ? a2a::MODE_LINE : a2a::MODE_BATCH;
            const int li = batch_len_index(n);
            const int v = b->var[mode][li];
            const int lines = a2a::batch_tile_lines(b->prec, n, v);
            if (lines <= 0 || NV % lines)
                return fail(A2A_ERROR_UNSUPPORTED, "box %d: %d lines per tile do not divide %d", i, lines, NV);
            a2a::BatchBox& bx = b->hbox[i];
            bx.var[p] = v;
            bx.lines[p] = lines;
            bx.tiles[p] = NU * (NV / lines);
            smem = std::max(smem, a2a::batch_tile_smem(b->prec, n, v, mode));
            if ((int64_t)b->items.size() + bx.tiles[p] >= (int64_t(1) << 30))
                return fail(A2A_ERROR_UNSUPPORTED, "the batch has too many tiles");
            for (int t = 0; t < bx.tiles[p]; ++t) b->items.push_back(make_int2(i * 4 + p, t));
        }
    }
    b->pass_start[3] = (int)b->items.size();
    b->smem = smem;
    const void* fn = a2a::batch_kernel(b->prec, false);
    int occ = 0;
    A2A_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, a2a::kBatchThreads, smem),
             "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    if (occ < 1) return fail(A2A_ERROR_UNSUPPORTED, "the batched kernel does not fit an SM with %zu bytes", smem);
    b->grid = std::max(1, std::min(b->pass_start[3], occ * b->sms));
    if (b->items.size() > b->items_cap) {
        if (b->d_items) cudaFree(b->d_items);
        b->d_items = nullptr;
        b->items_cap = 0;
        A2A_CUDA(cudaMalloc(&b->d_items, b->items.size() * sizeof(int2)), "cudaMalloc(batch items)");
        b->items_cap = b->items.size();
    }
    if (!b->items.empty())
        A2A_CUDA(cudaMemcpy(b->d_items, b->items.data(), b->items.size() * sizeof(int2), cudaMemcpyHostToDevice),
                 "cudaMemcpy(batch items)");
    A2A_CUDA(cudaMemcpy(b->d_boxes, b->hbox.data(), b->hbox.size() * sizeof(a2a::BatchBox), cudaMemcpyHostToDevice),
             "cudaMemcpy(batch boxes)");
    return A2A_SUCCESS;
}

// Enqueues one direction: clear the queue counters, then the persistent
// launch (or one launch per pass).
cudaError_t batch_launches(a2a_batch* b, bool inv, cudaStream_t st) {
    if (b->fused == 2 && b->grouped_ok) return batch_group_launches(b, inv, st);
    cudaError_t e = cudaMemsetAsync(b->d_queue, 0, b->queue_ints * sizeof(int), st);
    if (e != cudaSuccess) return e;
    const void* fn = a2a::batch_kernel(b->prec, inv);
    const int fused = b->fused == 0 ? 0 : 1;  // the grouped schedule without usable tables: one launch
    a2a::BatchArgs a;
    a.boxes = b->d_boxes;
    a.items = b->d_items;
    a.claim = b->claim;
    a.fused = fused;
    a.wait_extra = b->wait_extra;
    a.prefetch = b->prefetch;
    a.abort = b->d_queue;
    a.done = b->d_queue + 4;
    a.err = b->d_queue + b->queue_ints;
    const int launches = fused ? 1 : 3;
    for (int k = 0; k < launches && e == cudaSuccess; ++k) {
        a.item_lo = fused ? 0 : b->pass_start[k];
        a.item_hi = fused ? b->pass_start[3] : b->pass_start[k + 1];
        a.taken = b->d_queue + 1 + k;
        const int grid = std::max(1, std::min(a.item_hi - a.item_lo, b->grid));
        void* args[] = {&a};
        e = cudaLaunchKernel(fn, dim3(grid), dim3(a2a::kBatchThreads), args, b->smem, st);
    }
    return e;
}

a2a_status batch_capture(a2a_batch* b) {
    batch_drop_graphs(b);
    if (!b->use_graph) return A2A_SUCCESS;
    for (int inv = 0; inv < 2; ++inv) {
        cudaGraph_t g = nullptr;
        A2A_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
        const cudaError_t e = batch_launches(b, inv != 0, b->cap);
        const cudaError_t e2 = cudaStreamEndCapture(b->cap, &g);
        if (e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return cuda_fail(e, "batched launch (capture)");
        }
        A2A_CUDA(e2, "cudaStreamEndCapture");
        const cudaError_t e3 = cudaGraphInstantiate(&b->exec[inv], g, 0);
        cudaGraphDestroy(g);
        A2A_CUDA(e3, "cudaGraphInstantiate");
    }
    return A2A_SUCCESS;
}

// Points the device box table at the caller's buffers (only when they changed).
a2a_status batch_bind(a2a_batch* b, void** data, cudaStream_t st) {
    if (!data) return fail(A2A_ERROR_INVALID_VALUE, "d_data is NULL");
    bool changed = false;
    for (int i = 0; i < b->nboxes; ++i) {
        if (!data[i]) return fail(A2A_ERROR_INVALID_VALUE, "d_data[%d] is NULL", i);
        if (reinterpret_cast<uintptr_t>(data[i]) % 16)
            return fail(A2A_ERROR_MISALIGNED, "d_data[%d] is not 16-byte aligned", i);
        if (b->bound[i] != data[i]) changed = true;
    }
    if (!changed) return A2A_SUCCESS;
    for (int i = 0; i < b->nboxes; ++i) {
        b->bound[i] = data[i];
        b->hbox[i].data = data[i];
    }
    // pageable source: the call returns once the table is staged, and the
    // copy is ordered before the launches that follow on `st`
    A2A_CUDA(cudaMemcpyAsync(b->d_boxes, b->hbox.data(), b->hbox.size() * sizeof(a2a::BatchBox),
                             cudaMemcpyHostToDevice, st),
             "cudaMemcpyAsync(batch boxes)");
    // the grouped schedule's launches carry the group base pointers: a
    // captured graph of them is stale once a base moves
    const bool was_ok = b->grouped_ok;
    cudaError_t e = cudaSuccess;
    const bool moved = batch_group_tables(b, st, &e);
    A2A_CUDA(e, "cudaMemcpyAsync(batch group tables)");
    if (b->fused == 2 && (moved || was_ok != b->grouped_ok)) batch_drop_graphs(b);
    return A2A_SUCCESS;
}

a2a_status batch_check_flag(a2a_batch* b) {
    int flag = 0;
    int* err = b->d_queue + b->queue_ints;
    A2A_CUDA(cudaMemcpy(&flag, err, sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy(error flag)");
    if (flag) {
        A2A_CUDA(cudaMemset(err, 0, sizeof(int)), "cudaMemset(error flag)");
        return fail(A2A_ERROR_TIMEOUT, "a batched work item's bounded wait for the previous pass of its box gave up");
    }
    return A2A_SUCCESS;
}

a2a_status batch_run(a2a_batch* b, void** data, bool inv, cudaStream_t st, bool sync) {
    if (!b) return fail(A2A_ERROR_INVALID_VALUE, "batch is NULL");
    a2a_status s;
    if ((s = batch_bind(b, data, st)) != A2A_SUCCESS) return s;
    if (b->use_graph) {
        if (!b->exec[0] && (s = batch_capture(b)) != A2A_SUCCESS) return s;
        A2A_CUDA(cudaGraphLaunch(b->exec[inv ? 1 : 0], st), "cudaGraphLaunch");
    } else {
        A2A_CUDA(batch_launches(b, inv, st), "batched launch");
    }
    if (!sync) return A2A_SUCCESS;
    A2A_CUDA(cudaStreamSynchronize(st), "cudaStreamSynchronize");
    return batch_check_flag(b);
}

void batch_free(a2a_batch* b) {
    if (!b) return;
    batch_drop_graphs(b);
    if (b->cap) cudaStreamDestroy(b->cap);
    if (b->d_boxes) cudaFree(b->d_boxes);
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_queue) cudaFree(b->d_queue);
    if (b->d_gtab) cudaFree(b->d_gtab);
    for (cudaStream_t s : b->gstreams) cudaStreamDestroy(s);
    if (b->gfork) cudaEventDestroy(b->gfork);
    for (cudaEvent_t ev : b->gjoin) cudaEventDestroy(ev);
    for (a2a_distribution* h : b->dists) {
        release(h->d);
        delete h;
    }
    delete b;
}

// The grouped schedule's groups (one per box shape, largest first), their
// table space, streams and events, and default kernels (each pass's
// single-grid default where the grouped schedule can run it, else the first
// candidate it can).
a2a_status batch_groups_setup(a2a_batch* b) {
    b->groups.clear();
    for (int k = 0; k < (int)b->dists.size(); ++k) {
        a2a_batch::Group g;
        g.dist = k;
        const Dist& d = b->dists[k]->d;
        for (int i = 0; i < b->nboxes; ++i)
            if (b->box_dist[i] == k) g.boxes.push_back(i);
        g.elems = (int64_t)g.boxes.size() * (int64_t)(d.nlocal * d.P);
        b->groups.push_back(g);
    }
    std::stable_sort(b->groups.begin(), b->groups.end(),
                     [](const a2a_batch::Group& x, const a2a_batch::Group& y) { return x.elems > y.elems; });
    b->grouped_possible = true;
    size_t pos = 0;
    for (a2a_batch::Group& g : b->groups) {
        const Dist& d = b->dists[g.dist]->d;
        for (int p = 0; p < 3; ++p) {
            const SlotGeom geo = slot_geom(d, p);
            g.tab[p] = pos;
            pos += (size_t)geo.NU * g.boxes.size();
            // a tall grid's tile count stays an int in the kernels
            if ((uint64_t)geo.NU * g.boxes.size() * geo.NV >= (uint64_t(1) << 31)) b->grouped_possible = false;
            const int def = d.slot[p][0].chosen;
            int pick = group_eligible(d, p, def) ? def : -1;
            for (int c = 0; c < d.slot[p][0].ncand && pick < 0; ++c)
                if (group_eligible(d, p, c)) pick = c;
            if (pick < 0) b->grouped_possible = false;
            g.chosen[p] = pick;
        }
    }
    b->gtab_entries = pos;
    if (!b->grouped_possible) return A2A_SUCCESS;
    A2A_CUDA(cudaMalloc(&b->d_gtab, std::max<size_t>(pos, 1) * sizeof(uint32_t)), "cudaMalloc(batch group tables)");
    const size_t ns = std::min<size_t>(b->groups.size(), 8);
    for (size_t i = 0; i < ns; ++i) {
        cudaStream_t s = nullptr;
        A2A_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate(batch group)");
        b->gstreams.push_back(s);
    }
    A2A_CUDA(cudaEventCreateWithFlags(&b->gfork, cudaEventDisableTiming), "cudaEventCreate");
    for (size_t i = 0; i < b->groups.size(); ++i) {
        cudaEvent_t ev = nullptr;
        A2A_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
        b->gjoin.push_back(ev);
    }
    return A2A_SUCCESS;
}

}  // namespace

extern "C" {

a2a_status a2a_batch_create(int nboxes, const int* shapes, int world_size, a2a_precision precision,
                            a2a_batch** out) {
    if (!out) return fail(A2A_ERROR_INVALID_VALUE, "out is NULL");
    *out = nullptr;
    if (!shapes) return fail(A2A_ERROR_INVALID_VALUE, "shapes is NULL");
    if (nboxes < 1 || nboxes > a2a::kBatchMaxBoxes)
        return fail(A2A_ERROR_INVALID_VALUE, "nboxes must be in [1, %d]", a2a::kBatchMaxBoxes);
    if (precision != A2A_C128 && precision != A2A_C64)
        return fail(A2A_ERROR_INVALID_VALUE, "unknown precision %d", (int)precision);
    for (int i = 0; i < 3 * nboxes; ++i)
        if (batch_len_index(shapes[i]) < 0)
            return fail(A2A_ERROR_UNSUPPORTED,
                        "box %d: edge %d has no batched tile code (supported: 32 48 64 96 128 192 256 512)", i / 3,
                        shapes[i]);
    auto* b = new (std::nothrow) a2a_batch();
    if (!b) return fail(A2A_ERROR_OUT_OF_MEMORY, "host allocation failed");
    b->prec = precision;
    b->P = world_size;
    b->nboxes = nboxes;
    a2a_status s = A2A_SUCCESS;
    for (int i = 0; i < nboxes && s == A2A_SUCCESS; ++i) {
        int k = 0;
        for (; k < (int)b->dists.size(); ++k) {
            const Dist& d = b->dists[k]->d;
            if (d.ng[0] == shapes[3 * i] && d.ng[1] == shapes[3 * i + 1] && d.ng[2] == shapes[3 * i + 2]) break;
        }
        if (k == (int)b->dists.size()) {
            a2a_distribution* h = nullptr;
            s = create_common(shapes[3 * i], shapes[3 * i + 1], shapes[3 * i + 2], world_size, 64, precision, &h);
            if (s != A2A_SUCCESS) {
                const std::string why = g_last_error;
                s = fail(s, "box %d (%dx%dx%d): %s", i, shapes[3 * i], shapes[3 * i + 1], shapes[3 * i + 2],
                         why.c_str());
                break;
            }
            b->dists.push_back(h);
        }
        b->box_dist.push_back(k);
    }
    if (s != A2A_SUCCESS) {
        batch_free(b);
        return s;
    }
    b->sms = b->dists[0]->d.sms;
    b->hbox.resize(nboxes);
    b->bound.assign(nboxes, nullptr);
    for (int i = 0; i < nboxes; ++i) {
        const Dist& d = b->dists[b->box_dist[i]]->d;
        a2a::BatchBox& bx = b->hbox[i];
        bx.data = nullptr;
        for (int a = 0; a < 3; ++a) {
            bx.off[a] = d.off[a];
            bx.tw[a] = d.tw[a];
            bx.n[a] = d.ng[a];
        }
        for (int p = 0; p < 3; ++p) {
            const int sl = p;  // SLOT_Z, SLOT_X, SLOT_Y
            const int axis = p == 0 ? 2 : p == 1 ? 0 : 1;
            bx.split[p] = split_ok(d.local[axis], d.slot[sl][0].cand[0]);
            int n, NU, NV;
            batch_pass_geom(b, i, p, n, NU, NV);
            b->used[p == 0 ? a2a::MODE_LINE : a2a::MODE_BATCH][batch_len_index(n)] = true;
        }
        bx.inv_scale = 1.0 / ((double)d.ng[0] * d.ng[1] * d.ng[2]);
        // the offset tables' closed form (setup_distribution)
        const uint32_t nl = (uint32_t)d.nlocal;
        bx.lext[0] = d.local[0];
        bx.rstride[0] = (uint32_t)(d.dims[1] * d.dims[2]) * nl;
        bx.lstride[0] = (uint32_t)(d.local[1] * d.local[2]);
        bx.lext[1] = d.local[1];
        bx.rstride[1] = (uint32_t)d.dims[2] * nl;
        bx.lstride[1] = (uint32_t)d.local[2];
        bx.lext[2] = d.local[2];
        bx.rstride[2] = nl;
        bx.lstride[2] = 1;
    }
    // default variants: the first tile height that divides every pass using it
    for (int m = 0; m < 2; ++m)
        for (int li = 0; li < a2a::kBatchNumLengths; ++li) {
            if (!b->used[m][li]) continue;
            const int n = a2a::kBatchLengths[li];
            int pick = -1;
            for (int v = 0; v < 2 && pick < 0; ++v) {
                const int lines = a2a::batch_tile_lines(precision, n, v);
                bool ok = true;
                for (int i = 0; i < nboxes && ok; ++i)
                    for (int p = 0; p < 3; ++p) {
                        int pn, NU, NV;
                        batch_pass_geom(b, i, p, pn, NU, NV);
                        const int pm = p == 0 ? a2a::MODE_LINE : a2a::MODE_BATCH;
                        if (pn == n && pm == m && NV % lines) ok = false;
                    }
                if (ok) pick = v;
            }
            if (pick < 0) {
                batch_free(b);
                return fail(A2A_ERROR_UNSUPPORTED, "no batched tile of length %d divides the boxes' line counts", n);
            }
            b->var[m][li] = pick;
        }
    // batch-mode line pairs (16-byte accesses of two adjacent lines): complex
    // float, and in every box using the length each tile's lines in aligned,
    // contiguous pairs (checked on the offset tables, as for the single grid)
    for (int li = 0; li < a2a::kBatchNumLengths; ++li) {
        const int n = a2a::kBatchLengths[li];
        bool ok = precision == A2A_C64 && b->used[a2a::MODE_BATCH][li];
        for (int i = 0; i < nboxes && ok; ++i)
            for (int p = 1; p < 3 && ok; ++p) {
                int pn, NU, NV;
                batch_pass_geom(b, i, p, pn, NU, NV);
                if (pn != n) continue;
                const Dist& d = b->dists[b->box_dist[i]]->d;
                const std::vector<uint32_t>& hA = d.h_off[p == 1 ? 0 : 1];
                const std::vector<uint32_t>& hU = d.h_off[p == 1 ? 1 : 0];
                const std::vector<uint32_t>& hV = d.h_off[2];
                for (int v = 0; v + 1 < NV && ok; v += 2) ok = hV[v + 1] == hV[v] + 1 && hV[v] % 2 == 0;
                for (uint32_t o : hA) ok = ok && o % 2 == 0;
                for (uint32_t o : hU) ok = ok && o % 2 == 0;
                ok = ok && NV % 2 == 0;
            }
        b->pairs_ok[li] = ok;
    }
    const size_t max_smem = a2a::batch_smem(precision);
    cudaError_t e = cudaSuccess;
    for (int inv = 0; inv < 2 && e == cudaSuccess; ++inv)
        e = cudaFuncSetAttribute(a2a::batch_kernel(precision, inv != 0), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)max_smem);
    b->queue_ints = 4 + 3 * (size_t)nboxes;
    if (e == cudaSuccess) e = cudaMalloc(&b->d_boxes, sizeof(a2a::BatchBox) * nboxes);
    if (e == cudaSuccess) e = cudaMalloc(&b->d_queue, (b->queue_ints + 1) * sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(b->d_queue, 0, (b->queue_ints + 1) * sizeof(int));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        batch_free(b);
        return cuda_fail(e, "batch set-up");
    }
    if ((s = batch_groups_setup(b)) != A2A_SUCCESS || (s = batch_layout(b)) != A2A_SUCCESS) {
        batch_free(b);
        return s;
    }
    *out = b;
    return A2A_SUCCESS;
}

a2a_status a2a_batch_box_elements(const a2a_batch* b, int box, int64_t* elements) {
    if (!b || !elements) return fail(A2A_ERROR_INVALID_VALUE, "NULL argument");
    if (box < 0 || box >= b->nboxes) return fail(A2A_ERROR_INVALID_VALUE, "box %d outside [0, %d)", box, b->nboxes);
    const Dist& d = b->dists[b->box_dist[box]]->d;
    *elements = (int64_t)d.nlocal * d.P;
    return A2A_SUCCESS;
}

a2a_status a2a_batch_set_schedule(a2a_batch* b, int fused, int claim, int prefetch) {
    if (!b) return fail(A2A_ERROR_INVALID_VALUE, "batch is NULL");
    if (fused < 0 || fused > 2) return fail(A2A_ERROR_INVALID_VALUE, "fused must be 0, 1 or 2");
    if (fused == 2 && !b->grouped_possible)
        return fail(A2A_ERROR_UNSUPPORTED,
                    "the grouped schedule needs, for every box shape and pass, a single-grid kernel that addresses "
                    "its lines through the offset tables");
    if (claim < 1 || claim > 64) return fail(A2A_ERROR_INVALID_VALUE, "claim must be in [1, 64]");
    if (prefetch != 0 && prefetch != 1) return fail(A2A_ERROR_INVALID_VALUE, "prefetch must be 0 or 1");
    b->fused = fused;
    b->claim = claim;
    b->prefetch = prefetch;
    batch_drop_graphs(b);
    return A2A_SUCCESS;
}

a2a_status a2a_batch_select_variant(a2a_batch* b, int length, int batch_mode, int variant) {
    if (!b) return fail(A2A_ERROR_INVALID_VALUE, "batch is NULL");
    const int li = batch_len_index(length);
    if (li < 0 || (batch_mode != 0 && batch_mode != 1) || variant < 0 || variant >= a2a::kBatchVariants)
        return fail(A2A_ERROR_INVALID_VALUE, "length %d / mode %d / variant %d out of range", length, batch_mode,
                    variant);
    if (variant == 2 && !(batch_mode && b->pairs_ok[li]))
        return fail(A2A_ERROR_UNSUPPORTED, "length %d: line pairs need batch mode, complex float and aligned pairs",
                    length);
    const int m = batch_mode ? a2a::MODE_BATCH : a2a::MODE_LINE;
    const int old = b->var[m][li];
    b->var[m][li] = variant;
    const a2a_status s = batch_layout(b);
    if (s != A2A_SUCCESS) {
        b->var[m][li] = old;
        batch_layout(b);
    }
    return s;
}

a2a_status a2a_batch_set_graph(a2a_batch* b, int enable) {
    if (!b) return fail(A2A_ERROR_INVALID_VALUE, "batch is NULL");
    b->use_graph = enable != 0;
    batch_drop_graphs(b);
    return A2A_SUCCESS;
}

a2a_status a2a_batch_inject_stall(a2a_batch* b, int enable) {
    if (!b) return fail(A2A_ERROR_INVALID_VALUE, "batch is NULL");
    b->wait_extra = enable ? 1 : 0;
    batch_drop_graphs(b);
    return A2A_SUCCESS;
}

a2a_status a2a_batch_make_plans(a2a_batch* b, void** d_scratch) {
    if (!b) return fail(A2A_ERROR_INVALID_VALUE, "batch is NULL");
    if (!d_scratch) return A2A_SUCCESS;  // defaults
    a2a_status s;
    cudaStream_t st = b->cap;
    if ((s = batch_bind(b, d_scratch, st)) != A2A_SUCCESS) return s;
    cudaEvent_t e0, e1;
    A2A_CUDA(cudaEventCreate(&e0), "cudaEventCreate");
    A2A_CUDA(cudaEventCreate(&e1), "cudaEventCreate");
    const bool graph = b->use_graph;
    b->use_graph = false;
    b->fused = b->fused == 0 ? 0 : 1;  // the tile sweep times the persistent kernel
    // forward + inverse per trial (the inverse keeps the scratch values bounded)
    auto timed = [&](float* out) -> a2a_status {
        cudaError_t e = cudaSuccess;
        float best = 1e30f;
        for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
            e = cudaEventRecord(e0, st);
            if (e == cudaSuccess) e = batch_launches(b, false, st);
            if (e == cudaSuccess) e = batch_launches(b, true, st);
            if (e == cudaSuccess) e = cudaEventRecord(e1, st);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float t = 0.f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
            if (e == cudaSuccess && rep > 0) best = std::min(best, t);
        }
        if (e != cudaSuccess) return cuda_fail(e, "batched autotune launch");
        *out = best;
        return batch_check_flag(b);
    };
    float cur = 0.f;
    s = timed(&cur);
    // one sweep over the knobs in use: each length's tile height per mode,
    // then the schedule (one launch, or one per pass)
    for (int m = 0; m < 2 && s == A2A_SUCCESS; ++m)
        for (int li = 0; li < a2a::kBatchNumLengths && s == A2A_SUCCESS; ++li) {
            if (!b->used[m][li]) continue;
            const int old = b->var[m][li];
            b->tuned_ms[m][li][old] = cur;
            int best = old;
            for (int v = 0; v < a2a::kBatchVariants && s == A2A_SUCCESS; ++v) {
                if (v == old || (v == 2 && !(m == a2a::MODE_BATCH && b->pairs_ok[li]))) continue;
                b->var[m][li] = v;
                if (batch_layout(b) != A2A_SUCCESS) {  // this tile does not divide every box
                    b->var[m][li] = best;
                    s = batch_layout(b);
                    continue;
                }
                float t = 0.f;
                if ((s = timed(&t)) != A2A_SUCCESS) break;
                b->tuned_ms[m][li][v] = t;
                if (t < cur) {
                    cur = t;
                    best = v;
                }
                b->var[m][li] = best;
                if (s == A2A_SUCCESS) s = batch_layout(b);
            }
        }
    // the schedule: one launch or one per pass, items per queue access, L2
    // prefetch of the next tile
    auto try_knob = [&](int* knob, int value) {
        if (s != A2A_SUCCESS || *knob == value) return;
        const int old = *knob;
        *knob = value;
        float t = 0.f;
        s = timed(&t);
        if (s == A2A_SUCCESS && t < cur)
            cur = t;
        else
            *knob = old;
    };
    try_knob(&b->fused, 1 - b->fused);
    for (int c : {4, 8, 16, 32, 64}) try_knob(&b->claim, c);
    try_knob(&b->prefetch, 1 - b->prefetch);
    // the grouped schedule: per (shape, pass) the fastest single-grid kernel
    // it can run (forward + inverse pass on the group alone), then the
    // whole grouped transform against the persistent schedule
    if (s == A2A_SUCCESS && b->grouped_possible && b->grouped_ok) {
        for (a2a_batch::Group& g : b->groups) {
            const Dist& d = b->dists[g.dist]->d;
            for (int p = 0; p < 3 && s == A2A_SUCCESS; ++p) {
                int best = g.chosen[p];
                float bt = 1e30f;
                for (int c = 0; c < d.slot[p][0].ncand && s == A2A_SUCCESS; ++c) {
                    if (!group_eligible(d, p, c)) continue;
                    g.chosen[p] = c;
                    cudaError_t e = cudaSuccess;
                    float t = 1e30f;
                    for (int rep = 0; rep < 4 && e == cudaSuccess; ++rep) {
                        e = cudaEventRecord(e0, st);
                        if (e == cudaSuccess) e = group_pass(b, g, p, false, st);
                        if (e == cudaSuccess) e = group_pass(b, g, p, true, st);
                        if (e == cudaSuccess) e = cudaEventRecord(e1, st);
                        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
                        float x = 0.f;
                        if (e == cudaSuccess) e = cudaEventElapsedTime(&x, e0, e1);
                        if (e == cudaSuccess && rep > 0) t = std::min(t, x);
                    }
                    if (e != cudaSuccess) {
                        s = cuda_fail(e, "grouped autotune launch");
                        break;
                    }
                    if ((s = batch_check_flag(b)) != A2A_SUCCESS) break;
                    g.tuned_ms[p][c] = t;
                    if (t < bt) {
                        bt = t;
                        best = c;
                    }
                }
                g.chosen[p] = best;
            }
        }
        try_knob(&b->fused, 2);
    }
    b->use_graph = graph;
    batch_drop_graphs(b);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return s;
}

a2a_status a2a_batch_plan_report(const a2a_batch* b, char* buf, size_t len) {
    if (!b || !buf || len == 0) return fail(A2A_ERROR_INVALID_VALUE, "NULL argument");
    std::string r;
    char line[256];
    snprintf(line, sizeof line,
             "boxes=%d world_size=%d precision=%s schedule=%s claim=%d prefetch=%d grid=%d smem=%zu items=%d\n",
             b->nboxes, b->P, b->prec == A2A_C128 ? "c128" : "c64",
             b->fused == 2 ? (b->grouped_ok ? "grouped" : "grouped(unusable offsets: one-launch)")
             : b->fused ? "one-launch" : "per-pass",
             b->claim, b->prefetch, b->grid, b->smem, b->pass_start[3]);
    r += line;
    if (b->grouped_possible)
        for (const a2a_batch::Group& g : b->groups) {
            const Dist& d = b->dists[g.dist]->d;
            snprintf(line, sizeof line, "  group %dx%dx%d boxes=%zu:", d.ng[0], d.ng[1], d.ng[2], g.boxes.size());
            r += line;
            const char* names[3] = {"Z", "X", "Y"};
            for (int p = 0; p < 3; ++p) {
                const int c = g.chosen[p];
                const PassKernel& k = d.slot[p][0].cand[c];
                snprintf(line, sizeof line, " %s %s lines=%d lpt=%d threads=%d (tuned ms %.4f)", names[p],
                         k.kind == a2a::KIND_PIPE ? "pipe" : k.kind == a2a::KIND_TMA ? "tma"
                         : k.kind == a2a::KIND_RPIPE ? "rpipe" : k.kind == a2a::KIND_RPIPES ? "rpipes" : "direct",
                         k.lines, k.lpt, k.threads, g.tuned_ms[p][c]);
                r += line;
            }
            r += "\n";
        }
    for (int m = 0; m < 2; ++m)
        for (int li = 0; li < a2a::kBatchNumLengths; ++li) {
            if (!b->used[m][li]) continue;
            const int n = a2a::kBatchLengths[li];
            snprintf(line, sizeof line, "  N=%d %s lines=%d%s (tuned ms: %.4f / %.4f / %.4f)\n", n,
                     m ? "batch" : "line", a2a::batch_tile_lines(b->prec, n, b->var[m][li]),
                     b->var[m][li] == 2 ? " as pairs" : "", b->tuned_ms[m][li][0], b->tuned_ms[m][li][1],
                     b->tuned_ms[m][li][2]);
            r += line;
        }
    snprintf(buf, len, "%s", r.c_str());
    return A2A_SUCCESS;
}

a2a_status a2a_batch_forward(a2a_batch* b, void** d_data) { return batch_run(b, d_data, false, nullptr, true); }
a2a_status a2a_batch_inverse(a2a_batch* b, void** d_data) { return batch_run(b, d_data, true, nullptr, true); }
a2a_status a2a_batch_forward_async(a2a_batch* b, void** d_data, void* stream) {
    return batch_run(b, d_data, false, static_cast<cudaStream_t>(stream), false);
}
a2a_status a2a_batch_inverse_async(a2a_batch* b, void** d_data, void* stream) {
    return batch_run(b, d_data, true, static_cast<cudaStream_t>(stream), false);
}

a2a_status a2a_batch_check_device(a2a_batch* b) {
    if (!b) return fail(A2A_ERROR_INVALID_VALUE, "batch is NULL");
    return batch_check_flag(b);
}

a2a_status a2a_batch_launches_per_transform(const a2a_batch* b, int* out) {
    if (!b || !out) return fail(A2A_ERROR_INVALID_VALUE, "NULL argument");
    *out = (b->fused == 2 && b->grouped_ok) ? 3 * (int)b->groups.size() : b->fused ? 1 : 3;
    return A2A_SUCCESS;
}

a2a_status a2a_batch_destroy(a2a_batch* b) {
    batch_free(b);
    return A2A_SUCCESS;
}

}  // extern "C"
