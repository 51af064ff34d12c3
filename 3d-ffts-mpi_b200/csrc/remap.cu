// Distribution-step kernels (see remap.cuh) and their launchers.
#include "internal.h"
#include "remap.cuh"

namespace a2a {

// ---------------------------------------------------------------------------
// alltoall over virtual ranks: dst[q][r][i] = src[r][q][i], i < chunk
// (MPI_Alltoall with nsends = nlocal / P, a2adistribution.cpp:117-125).
// U is the copy unit (16-byte vectors whenever the chunk allows).
// ---------------------------------------------------------------------------
template <typename U>
__global__ void __launch_bounds__(256) alltoall_kernel(const U* __restrict__ src, U* __restrict__ dst, int P,
                                                       uint64_t chunk_units) {
    const uint64_t per_chunk_blocks = (chunk_units + blockDim.x - 1) / blockDim.x;
    const uint64_t total = per_chunk_blocks * uint64_t(P) * P;
    for (uint64_t blk = blockIdx.x; blk < total; blk += gridDim.x) {
        const uint64_t pair = blk / per_chunk_blocks;  // destination chunk q*P + r
        const uint64_t i = (blk - pair * per_chunk_blocks) * blockDim.x + threadIdx.x;
        if (i >= chunk_units) continue;
        const uint64_t q = pair / P, r = pair - q * P;
        dst[pair * chunk_units + i] = src[(r * P + q) * chunk_units + i];
    }
}

// ---------------------------------------------------------------------------
// unpack (UNPACK = true): dst (pencils) <- src (received order);
// pack   (UNPACK = false): dst (send order) <- src (pencils).
// g walks the pencil order of every rank, so pencil-side accesses are
// contiguous and the other side moves in runs of `la`.
// ---------------------------------------------------------------------------
template <typename V, bool UNPACK>
__global__ void __launch_bounds__(256) pencil_remap_kernel(const V* __restrict__ src, V* __restrict__ dst,
                                                           const PencilGeom geo, uint64_t total) {
    for (uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; g < total;
         g += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t q = g / geo.nlocal;
        const uint32_t rem = uint32_t(g - q * geo.nlocal);
        uint32_t p, n, s, j, ca, e;
        geo.f_ng.divmod(rem, p, n);   // pencil p, element n along the axis
        geo.f_m.divmod(p, s, j);      // pencil group s, line j inside the chunk
        geo.f_la.divmod(n, ca, e);    // sender's axis coordinate, offset in its run
        const uint32_t r = pencil_sender(geo, s, ca);
        const uint64_t other = q * geo.nlocal + uint64_t(r) * geo.chunk + uint64_t(j) * geo.la + e;
        if (UNPACK)
            dst[g] = src[other];
        else
            dst[other] = src[g];
    }
}

// ---------------------------------------------------------------------------
// Fast-axis change: per rank r and batch index m, a 2D transpose
//   dst[r nl + m smD + a saD + c] = src[r nl + m smS + c scS + a]
// through a 32 x 33 shared tile (a is contiguous in src, c in dst).
// ---------------------------------------------------------------------------
struct TransposeGeom {
    int A, C, M;
    uint64_t nl, smS, scS, smD, saD;
};

template <typename V>
__global__ void __launch_bounds__(256) transpose_kernel(const V* __restrict__ src, V* __restrict__ dst,
                                                        const TransposeGeom t) {
    __shared__ V tile[32][33];
    const int tilesA = (t.A + 31) / 32;
    const int ta = blockIdx.x % tilesA, tc = blockIdx.x / tilesA;
    const uint64_t m = blockIdx.y;
    const uint64_t r = blockIdx.z;
    const V* s = src + r * t.nl + m * t.smS;
    V* d = dst + r * t.nl + m * t.smD;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        const int a = ta * 32 + tx, c = tc * 32 + ty + k;
        if (a < t.A && c < t.C) tile[ty + k][tx] = s[uint64_t(c) * t.scS + a];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 32; k += 8) {
        const int a = ta * 32 + ty + k, c = tc * 32 + tx;
        if (a < t.A && c < t.C) d[uint64_t(a) * t.saD + c] = tile[tx][ty + k];
    }
}

// out = data / s (launch_scale_fft, dfft/kernels/a2affts.cu:78-92: a division,
// kept as one so results match the reference bit for bit)
template <typename V, typename T>
__global__ void __launch_bounds__(256) scale_kernel(const V* __restrict__ in, V* __restrict__ out, T s,
                                                    uint64_t n) {
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        V v = in[i];
        v.x = v.x / s;
        v.y = v.y / s;
        out[i] = v;
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static int grid_for(uint64_t work, int block, int sms) {
    const uint64_t want = (work + block - 1) / block;
    const uint64_t cap = uint64_t(sms) * 16;
    return int(want < cap ? (want > 0 ? want : 1) : cap);
}

cudaError_t launch_alltoall(const Dist& d, const void* src, void* dst, cudaStream_t st) {
    const uint64_t bytes = uint64_t(d.chunk) * d.elem_bytes;
    const int P = d.P;
    if (bytes % 16 == 0) {
        const uint64_t units = bytes / 16;
        const uint64_t blocks = ((units + 255) / 256) * uint64_t(P) * P;
        alltoall_kernel<uint4><<<grid_for(blocks * 256, 256, d.sms), 256, 0, st>>>(
            static_cast<const uint4*>(src), static_cast<uint4*>(dst), P, units);
    } else {
        const uint64_t units = bytes / 8;  // complex float, odd chunk
        const uint64_t blocks = ((units + 255) / 256) * uint64_t(P) * P;
        alltoall_kernel<uint2><<<grid_for(blocks * 256, 256, d.sms), 256, 0, st>>>(
            static_cast<const uint2*>(src), static_cast<uint2*>(dst), P, units);
    }
    return cudaGetLastError();
}

static PencilGeom pencil_geom(const Dist& d, int axis) {
    PencilGeom g;
    g.axis = axis;
    g.d0 = d.dims[0];
    g.d1 = d.dims[1];
    g.d2 = d.dims[2];
    g.nlocal = uint32_t(d.nlocal);
    g.chunk = uint32_t(d.chunk);
    g.la = uint32_t(d.local[axis]);
    g.ng = uint32_t(d.ng[axis]);
    g.m = g.chunk / g.la;
    g.f_nlocal = FastDiv(g.nlocal);
    g.f_ng = FastDiv(g.ng);
    g.f_m = FastDiv(g.m);
    g.f_la = FastDiv(g.la);
    g.f_d2 = FastDiv(uint32_t(d.dims[2]));
    return g;
}

template <typename V>
static cudaError_t remap_t(const Dist& d, int axis, bool unpack, const void* src, void* dst, cudaStream_t st) {
    const PencilGeom g = pencil_geom(d, axis);
    const uint64_t total = uint64_t(d.local_ranks) * d.nlocal;
    const int grid = grid_for(total, 256, d.sms);
    if (unpack)
        pencil_remap_kernel<V, true><<<grid, 256, 0, st>>>(static_cast<const V*>(src), static_cast<V*>(dst), g, total);
    else
        pencil_remap_kernel<V, false><<<grid, 256, 0, st>>>(static_cast<const V*>(src), static_cast<V*>(dst), g,
                                                            total);
    return cudaGetLastError();
}

cudaError_t launch_pencil_remap(const Dist& d, int axis, bool unpack, const void* src, void* dst, cudaStream_t st) {
    return d.prec == A2A_C128 ? remap_t<double2>(d, axis, unpack, src, dst, st)
                              : remap_t<float2>(d, axis, unpack, src, dst, st);
}

template <typename V>
static cudaError_t transpose_t(const Dist& d, const TransposeGeom& t, const void* src, void* dst, cudaStream_t st) {
    dim3 grid(unsigned(((t.A + 31) / 32) * ((t.C + 31) / 32)), unsigned(t.M), unsigned(d.local_ranks));
    transpose_kernel<V><<<grid, 256, 0, st>>>(static_cast<const V*>(src), static_cast<V*>(dst), t);
    return cudaGetLastError();
}

// which: 0 = fast_z_to_x ([x][y][z] -> [z][y][x], a2achangefastaxis.cu:4-22),
//        1 = fast_x_to_y ([z][y][x] -> [x][z][y], :35-53),
//        2 = fast_y_to_z ([x][z][y] -> [x][y][z], :66-84).
cudaError_t launch_fast_axis(const Dist& d, int which, const void* src, void* dst, cudaStream_t st) {
    const uint64_t lx = d.local[0], ly = d.local[1], lz = d.local[2];
    TransposeGeom t;
    t.nl = d.nlocal;
    if (which == 0) {  // a = z, c = x, m = y
        t.A = int(lz); t.C = int(lx); t.M = int(ly);
        t.smS = lz; t.scS = ly * lz; t.smD = lx; t.saD = ly * lx;
    } else if (which == 1) {  // a = x, c = y, m = z
        t.A = int(lx); t.C = int(ly); t.M = int(lz);
        t.smS = ly * lx; t.scS = lx; t.smD = ly; t.saD = lz * ly;
    } else {  // a = y, c = z, m = x
        t.A = int(ly); t.C = int(lz); t.M = int(lx);
        t.smS = lz * ly; t.scS = ly; t.smD = ly * lz; t.saD = lz;
    }
    return d.prec == A2A_C128 ? transpose_t<double2>(d, t, src, dst, st) : transpose_t<float2>(d, t, src, dst, st);
}

cudaError_t launch_scale(const Dist& d, const void* src, void* dst, double divisor, cudaStream_t st) {
    const uint64_t n = uint64_t(d.local_ranks) * d.nlocal;
    const int grid = grid_for(n, 256, d.sms);
    if (d.prec == A2A_C128)
        scale_kernel<double2, double><<<grid, 256, 0, st>>>(static_cast<const double2*>(src),
                                                            static_cast<double2*>(dst), divisor, n);
    else
        scale_kernel<float2, float><<<grid, 256, 0, st>>>(static_cast<const float2*>(src), static_cast<float2*>(dst),
                                                          float(divisor), n);
    return cudaGetLastError();
}

}  // namespace a2a
