/*
 * a2afft_b200 -- C ABI of a B200 (sm_100a) pencil-decomposed 3D FFT that is a
 * drop-in for the a2afft library of humz2k/3D-FFTs-MPI (src/a2afft).
 *
 * The reference runs one MPI rank per GPU: rank r owns a brick of the global
 * Ng^3 grid (brick grid dims = MPI_Dims_create(P, 3)) stored [x][y][z]
 * row-major, and a 3D transform is three rounds of
 * alltoall + pack/unpack + batched 1D cuFFT.  Here the P ranks are VIRTUAL:
 * every rank's brick lives in one device buffer, rank-major -- rank r's brick
 * starts at element r * nlocal and has exactly the reference's per-rank
 * layout.  A "buffer" below is therefore world_size * nlocal complex elements
 * (interleaved re/im; double for A2A_C128, float for A2A_C64).
 *
 * Buffers are passed as `void**` exactly like the reference passes
 * `fftPrecision**` (the library reads buf[0]; it never writes the pointer).
 * Every entry point returns an a2a_status; nothing aborts or prints.
 * Calls without a stream argument run on the object's stream (default: the
 * legacy default stream) and synchronise it before returning, which is the
 * reference's behaviour (every step there ends in cudaDeviceSynchronize).
 * `_async` variants only enqueue work.
 */
#ifndef A2AFFT_B200_H
#define A2AFFT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define A2AFFT_B200_VERSION 100 /* 1.0.0 */

typedef enum a2a_status {
    A2A_SUCCESS = 0,
    A2A_ERROR_INVALID_VALUE = 1,   /* null pointer, bad enum, non-positive size */
    A2A_ERROR_DECOMPOSITION = 2,   /* a grid the reference asserts on
                                      (distribution/a2adistribution.cpp:61-80) */
    A2A_ERROR_UNSUPPORTED = 3,     /* a transform length with no compiled kernel */
    A2A_ERROR_NO_PLANS = 4,        /* forward/inverse before make_plans */
    A2A_ERROR_MISALIGNED = 5,      /* a device buffer not 16-byte aligned */
    A2A_ERROR_CUDA = 6,            /* a CUDA runtime call failed */
    A2A_ERROR_OUT_OF_MEMORY = 7,   /* the plan's own tables could not be allocated */
    A2A_ERROR_TIMEOUT = 8,         /* a bounded device-side wait gave up */
    A2A_ERROR_NOT_IMPLEMENTED = 9  /* a method not available for this plan */
} a2a_status;

/* Element type.  The reference compiles `#define fftPrecision double`
 * (dfft/a2adfft.h:1) with an FP32 variant (dfft/kernels/a2affts.cu:25-35,
 * src/fft_demo). */
typedef enum a2a_precision {
    A2A_C128 = 0, /* complex double, 16 bytes (reference default) */
    A2A_C64 = 1   /* complex float, 8 bytes */
} a2a_precision;

/* How the 1D butterflies are computed (no reference counterpart: the
 * reference always calls cuFFT). */
typedef enum a2a_method {
    A2A_METHOD_PLAIN = 0,      /* CUDA-core Stockham mixed radix 2/3/4/8/16 */
    A2A_METHOD_SPLIT_BF16 = 1, /* radix-16 stages on tensor cores, split bf16 */
    A2A_METHOD_SPLIT_FP16 = 2  /* radix-16 stages on tensor cores, split fp16 */
} a2a_method;

/* Public fields of a2aDistribution (distribution/a2adistribution.h:8-17). */
typedef struct a2a_distribution_desc {
    int ndims;              /* always 3 */
    int ng[3];              /* global grid; ng[0]==ng[1]==ng[2]==Ng for cubes */
    int world_size;         /* number of (virtual) ranks P */
    int dims[3];            /* MPI_Dims_create(P, 3) */
    int local_grid_size[3]; /* ng[a] / dims[a] */
    int64_t nlocal;         /* complexes per rank */
    int64_t nsends;         /* nlocal / P: complexes per peer per alltoall */
    int block_size;         /* the reference's CUDA block size argument */
    int precision;          /* a2a_precision */
    size_t element_bytes;   /* 16 (C128) or 8 (C64) */
    size_t buffer_bytes;    /* local_ranks * nlocal * element_bytes */
    int first_rank;         /* virtual ranks held in the caller's buffers: */
    int local_ranks;        /* [first_rank, first_rank + local_ranks), all by default */
} a2a_distribution_desc;

typedef struct a2a_distribution a2a_distribution; /* a2aDistribution */
typedef struct a2a_dfft a2a_dfft;                 /* a2adfft */

/* ---- a2aDistribution ---------------------------------------------------- */

/* a2aDistribution(MPI_Comm, int Ng, int blockSize)
 * (distribution/a2adistribution.cpp:44-113).  The communicator is replaced by
 * the number of virtual ranks.  Returns A2A_ERROR_DECOMPOSITION where the
 * reference asserts.  Allocates only small device tables on the current
 * device. */
a2a_status a2a_distribution_create(int ng, int world_size, int block_size,
                                   a2a_precision precision, a2a_distribution** out);

/* Extension with no reference counterpart: an nx x ny x nz box with the same
 * brick rules applied per axis.  Only the fused transform (a2a_dfft_*)
 * accepts boxes; the pencil steps and 1D calls need a cube. */
a2a_status a2a_distribution_create_box(int nx, int ny, int nz, int world_size, int block_size,
                                       a2a_precision precision, a2a_distribution** out);

a2a_status a2a_distribution_describe(const a2a_distribution* dist, a2a_distribution_desc* out);

/* rank2coords + get_local_grid_start (a2adistribution.cpp:14-42). */
a2a_status a2a_rank_coords(const a2a_distribution* dist, int rank, int coords[3], int local_start[3]);

/* Narrows the buffers this process passes to the per-rank kernels (the
 * remaps, fast-axis changes, 1D transforms, scale, copy) to virtual ranks
 * [first, first + count): the layout when the P ranks are spread over
 * several processes/GPUs, each holding a contiguous block (the per-rank
 * kernels are identical for every rank).  The alltoall, the six steps and the
 * fused transform need all P ranks in one buffer and then return
 * A2A_ERROR_NOT_IMPLEMENTED; the exchange between processes is done by the
 * caller (see 3d-ffts-mpi_b200/distributed.py).  No reference counterpart:
 * there every process is one rank. */
a2a_status a2a_distribution_set_rank_range(a2a_distribution* dist, int first, int count);

/* Stream used by the calls below that take no stream (NULL = default). */
a2a_status a2a_distribution_set_stream(a2a_distribution* dist, void* cuda_stream);

/* The six transpose steps of a2aDistribution (a2adistribution.cpp:115-215),
 * over all virtual ranks at once.  On return BOTH buffers hold what the
 * reference leaves in them (the alltoall becomes a rank-major chunk
 * permutation in device memory).  One deliberate difference: the Y return
 * packs with the true inverse of the Y unpack; the reference's
 * d_y_pencils_to_y_a2a (distribution/kernels/a2apencils.cu:189-208) is not a
 * permutation unless dims[1]==2 or dims[0]==1, and the two agree wherever it
 * is. */
a2a_status a2a_get_z_pencils(a2a_distribution* dist, void** d_buff1, void** d_buff2);    /* :115-129 */
a2a_status a2a_return_z_pencils(a2a_distribution* dist, void** d_buff1, void** d_buff2); /* :131-145 */
a2a_status a2a_get_x_pencils(a2a_distribution* dist, void** d_buff1, void** d_buff2);    /* :147-163 */
a2a_status a2a_return_x_pencils(a2a_distribution* dist, void** d_buff1, void** d_buff2); /* :165-179 */
a2a_status a2a_get_y_pencils(a2a_distribution* dist, void** d_buff1, void** d_buff2);    /* :181-197 */
a2a_status a2a_return_y_pencils(a2a_distribution* dist, void** d_buff1, void** d_buff2); /* :199-215 */

/* The individual kernels the steps are made of, as the reference exposes
 * them in distribution/kernels/kernels.h:3-17 (each synchronous; source and
 * dest are distinct buffers of world_size * nlocal elements):
 * MPI_Alltoall with nsends = nlocal / world_size over the virtual ranks
 * (a2adistribution.cpp:117-125); the pack/unpack remaps
 * (distribution/kernels/a2apencils.cu:5-226; the Y pack is the true inverse
 * of the Y unpack, see above); the fast-axis changes
 * (distribution/kernels/a2achangefastaxis.cu:4-93). */
a2a_status a2a_alltoall(a2a_distribution* dist, void** source, void** dest);
a2a_status a2a_d_z_a2a_to_z_pencils(a2a_distribution* dist, void** source, void** dest);
a2a_status a2a_d_z_pencils_to_z_a2a(a2a_distribution* dist, void** source, void** dest);
a2a_status a2a_d_x_a2a_to_x_pencils(a2a_distribution* dist, void** source, void** dest);
a2a_status a2a_d_x_pencils_to_x_a2a(a2a_distribution* dist, void** source, void** dest);
a2a_status a2a_d_y_a2a_to_y_pencils(a2a_distribution* dist, void** source, void** dest);
a2a_status a2a_d_y_pencils_to_y_a2a(a2a_distribution* dist, void** source, void** dest);
a2a_status a2a_d_fast_z_to_x(a2a_distribution* dist, void** source, void** dest);
a2a_status a2a_d_fast_x_to_y(a2a_distribution* dist, void** source, void** dest);
a2a_status a2a_d_fast_y_to_z(a2a_distribution* dist, void** source, void** dest);

/* a2aDistribution::finalize (a2adistribution.cpp:217-224); also frees the
 * object.  NULL is accepted. */
a2a_status a2a_distribution_finalize(a2a_distribution* dist);

/* ---- 1D kernels (dfft/kernels/kernels.h:5-11) --------------------------- */

/* forward_1d_fft / inverse_1d_fft (dfft/kernels/a2affts.cu:7-76): in place,
 * unnormalised, every contiguous length-Ng line of the buffer (the pencils a
 * get_*_pencils step produced). */
a2a_status a2a_forward_1d_fft(a2a_distribution* dist, void** d_data);
a2a_status a2a_inverse_1d_fft(a2a_distribution* dist, void** d_data);

/* No counterpart in the reference.  The same in-place, unnormalised
 * transform of `nlines` contiguous lines of length n (n one of 4 8 12 16 24
 * 32 48 64 96 128 192 256 384 512 768 1024; nlines a multiple of 4) without
 * any distribution object, for callers that cannot allocate device memory:
 * an application whose memory manager reserved the device's memory up front,
 * or a latency-bound path that cannot take cudaMalloc's implicit
 * synchronisation.  It allocates nothing: its offset and twiddle tables live
 * in a fixed file-scope device array of A2A_LINES_NOALLOC_SCRATCH_BYTES,
 * which every GPU that loads the library holds until the process exits.
 * The first call on a device resolves that array's address (with the device
 * current) and keeps it for the life of the process; make that first call
 * before any stream capture, and do not use this entry point on a device
 * after cudaDeviceReset (the module may then reload elsewhere).  Each call
 * rebuilds the tables on `stream` and then transforms; calls share the array,
 * so calls that overlap on the GPU race.  Sizes whose tables exceed the
 * array (more than about 64K groups of up to 1024 lines) return
 * A2A_ERROR_UNSUPPORTED.  Enqueue only: the caller synchronises. */
#define A2A_LINES_NOALLOC_SCRATCH_BYTES (256u * 1024u)
a2a_status a2a_lines_fft_noalloc(void* data, int n, int64_t nlines, a2a_precision precision, int inverse,
                                 void* stream);

/* launch_scale_fft (a2affts.cu:78-92, 108-116): out = data / Ng^3. */
a2a_status a2a_scale_fft(a2a_distribution* dist, void** d_out, void** d_data);
/* launch_fast_copy_fft (a2affts.cu:94-106, 118-125): out = data. */
a2a_status a2a_fast_copy_fft(a2a_distribution* dist, void** d_out, void** d_data);

/* ---- a2adfft ------------------------------------------------------------ */

/* a2adfft(a2aDistribution&) (dfft/a2adfft.cpp:7-16).  The distribution must
 * outlive the dfft object. */
a2a_status a2a_dfft_create(a2a_distribution* dist, a2a_dfft** out);

/* Selects the butterfly method (default A2A_METHOD_PLAIN); call before
 * make_plans.  The split tensor-core methods need A2A_C64. */
a2a_status a2a_dfft_set_method(a2a_dfft* dfft, a2a_method method);

/* a2adfft::make_plans(fftPrecision** d_scratch) (dfft/a2adfft.cpp:18-24).
 * The scratch buffer is borrowed as in the reference (same size as a data
 * buffer).  The fused transform runs in place and never touches it; when it
 * is given (and autotuning is on, the default), make_plans times every
 * compiled launch variant of each axis pass on it -- clobbering its contents,
 * as the reference's transforms do -- inside a whole forward + inverse with
 * the other passes' current choices (one sweep Z, X, Y), and keeps the
 * fastest; the report's tuned_ms is that forward + inverse time.  With NULL the
 * default variant of each pass is used.  The choice is stored in the
 * distribution and shared by every dfft built on it. */
a2a_status a2a_dfft_make_plans(a2a_dfft* dfft, void** d_scratch);

/* Turns the make_plans timing run on (default) or off.  No reference
 * counterpart. */
a2a_status a2a_dfft_set_autotune(a2a_dfft* dfft, int enable);

/* Reads and clears the distribution's device error flag: A2A_ERROR_TIMEOUT
 * when a pass kernel gave up a bounded wait for its tile copies since the
 * last check (the synchronous transforms check it themselves; after
 * _async calls, synchronise the stream first).  No reference counterpart. */
a2a_status a2a_dfft_check_device(const a2a_dfft* dfft);

/* Launch variants compiled for a pass (0 = Z, 1 = X, 2 = Y), and a manual
 * choice among them (overrides the default or the make_plans timing; fails
 * with A2A_ERROR_UNSUPPORTED for a variant that does not fit the pass).  With
 * a split tensor-core method there are five: 0 = one tile per CTA, 1 =
 * persistent CTAs fed by a TMA ring (the default where it fits), 2 = the
 * two-stage form (lengths 512 and 1024: a radix-16 or radix-32 GEMM, one
 * twiddle, a radix-32 GEMM; TMA ring), 3 = the two-stage form with 8-line
 * tiles (1024), 4 = the two-stage form software-pipelined over two
 * tensor-memory regions (fp16).  No reference counterpart. */
a2a_status a2a_dfft_variant_count(const a2a_dfft* dfft, int pass, int* count);
a2a_status a2a_dfft_select_variant(a2a_dfft* dfft, int pass, int variant);

/* Text report of every pass variant (length, tile, threads, occupancy,
 * make_plans timing, the chosen one) into buf.  No reference counterpart. */
a2a_status a2a_dfft_plan_report(const a2a_dfft* dfft, char* buf, size_t len);

/* a2adfft::forward / inverse (dfft/a2adfft.cpp:26-158): in place on
 * d_data[0], rank-major bricks in, rank-major bricks out, natural frequency
 * order, forward unnormalised, inverse scaled by 1/(nx*ny*nz).  Implemented
 * as three fused axis passes (each gathers its pencils straight from the
 * bricks, transforms them and scatters them back) instead of the reference's
 * 19 array passes; the scratch buffer is not touched. */
a2a_status a2a_dfft_forward(a2a_dfft* dfft, void** d_data);
a2a_status a2a_dfft_inverse(a2a_dfft* dfft, void** d_data);
a2a_status a2a_dfft_backward(a2a_dfft* dfft, void** d_data); /* alias of inverse */
a2a_status a2a_dfft_forward_async(a2a_dfft* dfft, void** d_data, void* cuda_stream);
a2a_status a2a_dfft_inverse_async(a2a_dfft* dfft, void** d_data, void* cuda_stream);

/* One of the three fused passes of a transform, enqueued on `cuda_stream`
 * (for profiling and for overlapping work between passes): pass 0 = Z,
 * 1 = X, 2 = Y; forward then is passes 0,1,2 with inverse=0, and the inverse
 * is passes 0,1,2 with inverse=1 (pass 2 applies the 1/(nx*ny*nz) scale).
 * No reference counterpart: the reference's forward is not divisible. */
a2a_status a2a_dfft_execute_pass_async(a2a_dfft* dfft, void** d_data, int pass, int inverse, void* cuda_stream);

/* Number of kernel launches one forward (or inverse) enqueues. */
a2a_status a2a_dfft_launches_per_transform(const a2a_dfft* dfft, int* out);

/* ---- several GPUs: the fused pass over peer memory ----------------------- */

/* The reference exchanges each axis step between ranks with MPI_Alltoall plus
 * pack/unpack kernels (distribution/a2adistribution.cpp:115-215).  Here one
 * pass kernel does the whole step across devices: the virtual rank-major
 * buffer is split into `nblocks` blocks of equal size (block g holds the
 * contiguous virtual ranks [g L, (g+1) L), L = world_size / nblocks,
 * world_size / nblocks * nlocal elements), blocks[g] its address on this
 * device (this process's own block, or another GPU's block mapped with
 * a2a_ipc_import); the kernel gathers each tile's lines from the owners,
 * transforms them and scatters them back (peer loads and stores over
 * NVLink).  A pass's tiles are split evenly into `nparts` parts and this
 * call enqueues part `part` on `cuda_stream`.  The caller orders the passes:
 * every part of pass p must be complete before any part of pass p + 1 starts
 * (e.g. synchronise the stream, then a process-group barrier).  The inverse's
 * pass 2 applies 1/(nx*ny*nz).  No kernel waits on another device. */
a2a_status a2a_dfft_execute_pass_blocks(a2a_dfft* dfft, void** blocks, int nblocks, int pass, int inverse, int part,
                                        int nparts, void* cuda_stream);

/* The kernel bodies a2a_dfft_execute_pass_blocks uses: 1 (default) one wave
 * of persistent CTAs per call, each working through its share of the part's
 * tiles -- the X and Y passes fed by TMA tensor-map copies of each brick
 * (one map per virtual rank, built from `blocks` and kept until they change,
 * so calls of one dfft with different `blocks` must not overlap on the GPU;
 * plain loads, also from peer memory), the Z pass with the next tile's
 * gathers in flight in registers -- at lengths 256, 512, 1024 complex float
 * and 512, 1024 complex double where the tiles fit; elsewhere, or with 0, one
 * tile per CTA.  All give the same result.  No reference counterpart. */
a2a_status a2a_dfft_set_blocks_kernel(a2a_dfft* dfft, int persistent);

/* Sharing a device buffer with another process (CUDA IPC): export writes an
 * opaque handle of A2A_IPC_HANDLE_BYTES bytes and the buffer's offset inside
 * its allocation; import maps it in this process (on its current device)
 * and returns the buffer's address there; release undoes one import.  A
 * handle imported more than once on one device shares one mapping, which is
 * unmapped when its last import is released.  No reference counterpart. */
#define A2A_IPC_HANDLE_BYTES 64
a2a_status a2a_ipc_export(const void* dev_ptr, void* handle, uint64_t* offset);
a2a_status a2a_ipc_import(const void* handle, uint64_t offset, void** dev_ptr);
a2a_status a2a_ipc_release(void* dev_ptr);

a2a_status a2a_dfft_destroy(a2a_dfft* dfft);

/* ---- host-staged transforms -------------------------------------------- */

/* The FP32 demo driver's pattern (src/fft_demo/fft_3d/fft_3d.c:6-189): the
 * data lives in host memory; it is copied to d_buffer[0] (a device buffer
 * of the plan's size), transformed there and copied back, synchronously. */
a2a_status a2a_dfft_forward_host(a2a_dfft* dfft, void* host_data, void** d_buffer);
a2a_status a2a_dfft_inverse_host(a2a_dfft* dfft, void* host_data, void** d_buffer);

/* ---- host-only decomposition -------------------------------------------- */

/* The decomposition a2a_distribution_create would make (dims =
 * MPI_Dims_create(world_size, 3), local brick, nlocal) and its validation,
 * on the host only: for processes that have no device or have not created
 * one yet.  No reference counterpart as a separate call. */
a2a_status a2a_decompose(int ng, int world_size, int dims[3], int local_grid_size[3], int64_t* nlocal);

/* ---- dump files ---------------------------------------------------------- */

/* The reference's `dims` file (distribution/a2adistribution.cpp:101-111):
 * nine int32 -- world_size, Ng, nlocal, dims[3], local_grid_size[3].  Host
 * only; needs no device. */
a2a_status a2a_write_dims(int ng, int world_size, const char* path);

/* The reference test's per-rank dumps (tests/test.cpp:69-125): for every
 * rank r, file `<folder>/proc<r>` holding that rank's brick of the input,
 * the forward result and the inverse result, one after the other (complex
 * double for A2A_C128 as in src/a2afft, complex float for A2A_C64 as in
 * src/fft_demo).  The three host buffers are rank-major (world_size *
 * nlocal elements each).  The reference names files `proc<digit>` and so
 * stops at 10 ranks; here r is written in full.  Host only. */
a2a_status a2a_write_rank_dumps(int ng, int world_size, a2a_precision precision, const char* folder,
                                const void* host_input, const void* host_forward, const void* host_inverse);

/* ---- batched form --------------------------------------------------------- */

/* Many independent boxes transformed together: one persistent kernel launch
 * per direction (replayed from a CUDA graph) works through every tile of
 * every box, the X and Y tiles of a box starting once the box's previous
 * pass is done.  No counterpart in the reference, which plans one grid at a
 * time; each box has exactly the layout a2a_distribution_create_box(nx, ny,
 * nz, world_size, ...) gives it (world_size virtual ranks, rank-major
 * bricks), and its transform equals that distribution's a2a_dfft_forward /
 * a2a_dfft_inverse (the inverse scaled by 1/(nx ny nz)). */
typedef struct a2a_batch a2a_batch;

/* shapes: nboxes triples (nx, ny, nz); every edge one of 32 48 64 96 128 192
 * 256 512.  Boxes of one shape share their offset tables. */
a2a_status a2a_batch_create(int nboxes, const int* shapes, int world_size, a2a_precision precision,
                            a2a_batch** out);
/* Complex elements of box `box`'s buffer (world_size * nlocal). */
a2a_status a2a_batch_box_elements(const a2a_batch* batch, int box, int64_t* elements);
/* Optional tuning on caller buffers d_scratch[0..nboxes) (clobbered): for
 * each transform length in use, the tile height per access mode, then the
 * schedule (one launch or one per pass, claim 4..64, prefetch).  NULL keeps
 * the defaults. */
a2a_status a2a_batch_make_plans(a2a_batch* batch, void** d_scratch);
/* fused = 1: one launch per direction (later passes wait, device-side, for
 * the earlier pass of their box); 0: one launch per pass.  claim: most work
 * items a CTA takes per queue access (1..64; fewer as the queue drains).  prefetch = 1: each CTA asks L2 for
 * its next tile while it transforms the current one.
 * fused = 2 (grouped): the boxes of each shape form one tall grid per pass
 * (line bases: box offset from the shape's lowest box pointer + the shape's
 * own line offsets) transformed by the single-grid pass kernels, one launch
 * per (shape, pass), each shape's three passes on its own stream branch
 * forked from and joined back to the caller's stream (parallel branches of
 * the captured graph).  claim and prefetch do not apply.  Needs, per shape
 * and pass, a kernel that addresses lines through the offset tables
 * (A2A_ERROR_UNSUPPORTED otherwise), and every shape's boxes within 2^32
 * elements of one another in the bound buffers; where they are not, calls
 * run the fused = 1 schedule.  make_plans picks per (shape, pass) the kernel
 * and then times this schedule against the others. */
a2a_status a2a_batch_set_schedule(a2a_batch* batch, int fused, int claim, int prefetch);
/* Tile choice for one length in line (batch_mode = 0, the Z pass) or batch
 * mode (the X and Y passes): 0 and 1 are two tile heights; 2 (batch mode,
 * A2A_C64, boxes whose lines pair into aligned 16-byte accesses) is height 0
 * with each thread moving two adjacent lines at once. */
a2a_status a2a_batch_select_variant(a2a_batch* batch, int length, int batch_mode, int variant);
/* 1 (default): replay a captured CUDA graph; 0: plain launches. */
a2a_status a2a_batch_set_graph(a2a_batch* batch, int enable);
/* Test hook for the timeout path: every device-side wait asks for one tile
 * more than its pass has, so it gives up (after about a second) and the next
 * synchronising call returns A2A_ERROR_TIMEOUT.  0 restores normal runs. */
a2a_status a2a_batch_inject_stall(a2a_batch* batch, int enable);
a2a_status a2a_batch_plan_report(const a2a_batch* batch, char* buf, size_t len);
/* d_data[b]: box b's device buffer (16-byte aligned).  Synchronous forms
 * check the device error flag; the _async forms only enqueue on `stream`.
 * Calls of one batch object share its queue scratch: calls that overlap on
 * the GPU race. */
a2a_status a2a_batch_forward(a2a_batch* batch, void** d_data);
a2a_status a2a_batch_inverse(a2a_batch* batch, void** d_data);
a2a_status a2a_batch_forward_async(a2a_batch* batch, void** d_data, void* stream);
a2a_status a2a_batch_inverse_async(a2a_batch* batch, void** d_data, void* stream);
/* Reads and clears the batch's device error flag (A2A_ERROR_TIMEOUT if set). */
a2a_status a2a_batch_check_device(a2a_batch* batch);
a2a_status a2a_batch_launches_per_transform(const a2a_batch* batch, int* out);
a2a_status a2a_batch_destroy(a2a_batch* batch);

/* ---- misc --------------------------------------------------------------- */

const char* a2a_status_string(a2a_status status);
/* Detail of the last error raised on the calling thread ("" if none). */
const char* a2a_last_error(void);
int a2a_version(void);

#ifdef __cplusplus
}
#endif
#endif /* A2AFFT_B200_H */
