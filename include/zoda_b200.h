/*
 * zoda_b200.h -- C ABI of libzoda_b200.so, the sm_100a replacement for
 * zoda-cu's column-wise Reed-Solomon extension over BabyBear
 * (p = 2^31 - 2^27 + 1).
 *
 * Part 1 is the reference's own FFI, symbol for symbol: a Rust crate that
 * declares the block in src/ntt/cuda.rs:15-22 links against this library
 * unchanged (as libntt_cuda.a or this .so).
 *
 * Part 2 adds device-resident calls behind a context: the fused extension
 * (one HBM pass, row-major in and out), its host-buffer variant, the batched
 * multi-square launch and the serving loop.
 *
 * All element buffers hold canonical u32 BabyBear values in [0, p).
 * No call aborts the process; every failure comes back as a status code.
 */
#ifndef ZODA_B200_H
#define ZODA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ======================================================================
 * Part 1: the reference FFI (cuda/ntt_kernel.cu:184-208)
 * ====================================================================== */

/* Replaces cuda/ntt_kernel.cu:190-193 (bound at src/ntt/cuda.rs:17).
 * Forward NTT, in place, of `polys` polynomials laid `stride` u32 apart in
 * host memory (pinned from cuda_host_alloc is fastest, pageable works).
 * Only values[c*stride .. c*stride + n) are transformed; the rest of each
 * polynomial is left untouched. roots = [w^0 .. w^(n-1)] for a primitive
 * n-th root w (src/ntt/cuda.rs:111-114 passes roots_of_unity(n)). Natural
 * order in and out. Returns 0 on success, else a nonzero cudaError_t value
 * (cudaErrorInvalidValue = 1 for bad arguments, including a roots table
 * that is not the powers of a primitive n-th root). Synchronous. */
int cuda_ntt(uint32_t* values, const uint32_t* roots, uint32_t n, uint32_t polys, uint32_t stride);

/* Replaces cuda/ntt_kernel.cu:196-208 (bound at src/ntt/cuda.rs:18).
 * Inverse NTT with the same layout: the transform with inverse roots
 * [roots[0], roots[n-1], ..., roots[1]], then every value times n^-1. */
int cuda_intt(uint32_t* values, const uint32_t* roots, uint32_t n, uint32_t polys, uint32_t stride);

/* Replaces cuda/ntt_kernel.cu:184-187 (bound at src/ntt/cuda.rs:19):
 * pinned host allocation of `count` u32, NULL on failure. */
uint32_t* cuda_host_alloc(size_t count);

/* Replaces cuda/ntt_kernel.cu:188 (bound at src/ntt/cuda.rs:20). */
void cuda_host_free(uint32_t* p);

/* src/ntt/cuda.rs:21 also binds cudaGetDeviceCount; it resolves from the
 * CUDA runtime this library links. */

/* ======================================================================
 * Part 2: device-resident API
 * ====================================================================== */

typedef enum zoda_status {
    ZODA_OK = 0,
    ZODA_ERR_ARG = 1,         /* bad argument (size, alignment, null)        */
    ZODA_ERR_CUDA = 2,        /* a CUDA call failed; see zoda_last_error     */
    ZODA_ERR_NOMEM = 3,       /* device or host allocation failed            */
    ZODA_ERR_UNSUPPORTED = 4, /* shape this build does not handle            */
    ZODA_ERR_BUDGET = 5,      /* request exceeds the admission budget        */
    ZODA_ERR_TIMEOUT = 6,     /* a bounded wait ran out                      */
    ZODA_ERR_CANCELLED = 7,   /* request cancelled before it ran             */
    ZODA_ERR_STATE = 8        /* call not valid in the object's state        */
} zoda_status;

typedef struct zoda_ctx zoda_ctx;

/* Human-readable name of a status. */
const char* zoda_status_string(zoda_status s);
/* Text of the last CUDA error seen on this thread ("" if none). */
const char* zoda_last_error(void);

/* Creates a context on `device`: uploads the twiddle tables (omega_8192^j
 * and, per side S, g^i / S with g = omega_2S) and sets kernel attributes.
 * Replaces the per-call root generation and upload of src/ntt/cuda.rs:112
 * and cuda/ntt_kernel.cu:111-114. */
zoda_status zoda_ctx_create(int device, zoda_ctx** out);
void zoda_ctx_destroy(zoda_ctx* ctx);

/* Largest k the extension accepts (2^26): one fused pass up to 4096, three
 * four-step passes above (no column of more than 4096 rows fits on chip). */
uint32_t zoda_max_side(void);

/* Kernel variant of the fused extension on a context. AUTO runs the side's
 * plan (below); the others force one kernel with default knobs (for tests;
 * TMA supports k in [32, 4096], FOURSTEP k in [1024, 4096]). */
typedef enum zoda_extend_impl {
    ZODA_IMPL_AUTO = 0,
    ZODA_IMPL_DIRECT = 1,
    ZODA_IMPL_TMA = 2,
    ZODA_IMPL_FOURSTEP = 3 /* three passes of sqrt(k)-point transforms, as above 4096 */
} zoda_extend_impl;
zoda_status zoda_ctx_set_impl(zoda_ctx* ctx, int impl);

/* Per-side launch plan of the fused extension. No counterpart in the
 * reference, whose kernel shape is fixed (cuda/ntt_kernel.cu:130-160). With
 * ZODA_IMPL_AUTO a side that has a plan (from zoda_autotune or
 * zoda_plan_set) runs that plan; a side without one runs the default plan
 * (TMA for 128 <= k <= 2048, else direct; sched 0, l2_promo 3, blocked 0,
 * stagger 1, radix 16). Every plan computes the same bits; only the speed
 * differs. */
typedef struct zoda_plan {
    int32_t impl;     /* ZODA_IMPL_DIRECT, ZODA_IMPL_TMA (k >= 32) or ZODA_IMPL_FOURSTEP
                         (1024 <= k <= 4096)                                          */
    int32_t sched;    /* direct kernel: the leftover radix at the INTT's last level (0)
                         or its first level (1). FOURSTEP with ctas 2 or 4: 1 = tiles
                         are copied into shared memory by cp.async while the previous
                         one computes (each pass's next tile; in the chunked launch,
                         the next pass-A tile)                                        */
    int32_t l2_promo; /* TMA kernel: L2 promotion of tile loads, 0 none, 1 64 B,
                         2 128 B, 3 256 B                                              */
    int32_t blocked;  /* 0 = CTA i takes tiles i, i + grid, ...; 1 = one contiguous run.
                         FOURSTEP: 0 = three launches over the whole square; 1 = one
                         persistent launch that runs the three passes column chunk by
                         column chunk, so each chunk's intermediate stays in L2      */
    int32_t stagger;  /* TMA kernel: 0 = the two warp-groups run in step; 1, 2, 3 = the
                         second starts once the first begins its last INTT level, its
                         second INTT level, or its first (less apart, more shared code) */
    int32_t radix;    /* level radix 16 (512 threads, 16 positions per thread) or 8
                         (1024 threads, 8 positions: twice the warps; direct kernel
                         from k = 64)                                              */
    float ms;         /* the tuner's time for this plan (0 when set by hand)            */
    int32_t ctas;     /* FOURSTEP: CTAs resident per SM in its passes, 1 (512 threads),
                         2 (256 threads at radix 16, 512 at radix 8), 4 (256 threads,
                         radix 8) or 5 (256 threads, radix 4: the one plan that takes
                         radix 4); 0 counts as 1. Ignored by the other kernels.     */
} zoda_plan;

/* Times every candidate plan for each power-of-two side in [side_min,
 * side_max] (sides 1..4096) on a synthetic [side][cols] square
 * (cols = 0: about 256 MiB of input, rounded to the side's tile width), with
 * `reps` timed runs after one warm-up. A candidate whose output differs in
 * any bit from the default plan's is rejected. The fastest is installed on
 * the context (the default plan instead when it is within 1% of the fastest)
 * and written to plans[log2(side)] when `plans` is not NULL (an array of 13).
 * Allocates and frees its own buffers; synchronous. */
zoda_status zoda_autotune(zoda_ctx* ctx, uint32_t side_min, uint32_t side_max, uint64_t cols, uint32_t reps,
                          zoda_plan* plans);
/* Reads (ZODA_ERR_STATE when the side has no plan) or installs the plan of
 * one side, e.g. from a saved tuning file; zoda_plan_clear drops them all. */
zoda_status zoda_plan_get(const zoda_ctx* ctx, uint32_t side, zoda_plan* plan);
zoda_status zoda_plan_set(zoda_ctx* ctx, uint32_t side, const zoda_plan* plan);
void zoda_plan_clear(zoda_ctx* ctx);

/* Returns ZODA_ERR_TIMEOUT (and clears the flag) if a kernel on this context
 * gave up a bounded wait since the last call, else ZODA_OK. Synchronizes the
 * device first. */
zoda_status zoda_ctx_check(zoda_ctx* ctx);

/* Self-test of the bounded-wait path every staged kernel uses: one small
 * kernel waits on a shared-memory barrier that nothing completes. When the
 * bound runs out (the same 2^18 polls, about a second) it sets the context's
 * flag and returns, so the next zoda_ctx_check returns ZODA_ERR_TIMEOUT and
 * clears it; the context stays usable. No counterpart in the reference.
 * Asynchronous on `stream`. */
zoda_status zoda_selftest_bounded_wait(zoda_ctx* ctx, void* stream);

/* Fused extension, device memory. d_in is row-major [k][cols], d_out is
 * row-major [2k][cols]; row j of d_out is every column's degree-<k
 * interpolant evaluated at omega_2k^j, i.e. the rows the reference gathers
 * from its column-major square (src/benchmarks/utils.rs:167-168,
 * src/zoda/babybear.rs:155): even rows equal the input rows. k must be a
 * power of two in [1, zoda_max_side()], cols a multiple of 4, both pointers
 * 16-byte aligned and non-overlapping. Asynchronous on `stream`, a
 * cudaStream_t (NULL is the legacy default stream, as in every CUDA API). */
zoda_status zoda_extend_device(zoda_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t k, uint64_t cols,
                               void* stream);

/* Timing of a host-buffer call, in milliseconds. The copies and kernels of
 * different column chunks overlap, so the three busy times (CUDA events) can
 * add up to more than total_ms. */
typedef struct zoda_timing {
    float h2d_ms;       /* host -> device copies of the input, summed              */
    float kernel_ms;    /* fused extension kernels, summed                         */
    float d2h_ms;       /* device -> host copies of output rows, summed            */
    float total_ms;     /* the whole call, host wall clock                         */
    uint64_t h2d_bytes; /* bytes the call copied host -> device                    */
    uint64_t d2h_bytes; /* bytes the call copied device -> host (odd rows, plus the
                           even rows of the chunks that return over PCIe)           */
} zoda_timing;

/* Fused extension from host memory to host memory: the reference's
 * `encode_gpu` window (src/benchmarks/utils.rs:100-146) without the host
 * transpose and padding, which the kernel makes unnecessary. h_in row-major
 * [k][cols], h_out row-major [2k][cols]; pinned buffers give full PCIe speed.
 * The square moves in column chunks over three streams, so uploads,
 * kernels and downloads overlap; device buffers are the context's cached
 * chunk buffers. The odd output rows cross PCIe; the even rows equal the
 * input rows, and host threads copy most of them meanwhile (those of the last
 * eighth of the column chunks come back over PCIe instead). Synchronous,
 * also on failure: an error return happens only after every copy the call
 * queued has finished, so the caller may free its buffers at once. `timing`
 * may be NULL. */
zoda_status zoda_extend_host(zoda_ctx* ctx, const uint32_t* h_in, uint32_t* h_out, uint32_t k, uint64_t cols,
                             zoda_timing* timing);

/* Fault injection for tests of the error paths; no counterpart in the
 * reference. Arms `site`: the call passes through it `after` more times, then
 * the next pass fails and the site disarms. site 0 disarms everything. Sites:
 *   ZODA_FAULT_HOST_CHUNK  the launch of one column chunk in zoda_extend_host,
 *                          after earlier chunks' copies have been queued: the
 *                          call fails with ZODA_ERR_CUDA (zoda_last_error says
 *                          "injected fault");
 *   ZODA_FAULT_PIPE_WAIT   one pipelined four-step launch (plan impl 3,
 *                          blocked 1) waits for one finished tile more than a
 *                          chunk has: its bounded dependency waits run out
 *                          (about a second), every CTA flags the error and
 *                          leaves, and zoda_ctx_check reports ZODA_ERR_TIMEOUT
 *                          (the output is then incomplete). */
#define ZODA_FAULT_HOST_CHUNK 1u
#define ZODA_FAULT_PIPE_WAIT 2u
zoda_status zoda_ctx_inject_fault(zoda_ctx* ctx, uint32_t site, uint32_t after);

/* ----------------------------------------------------------------------
 * Batched extension: many squares of mixed sides in one persistent launch.
 * No reference counterpart; the reference encodes one square per call
 * (src/benchmarks/utils.rs:100-146).
 * ---------------------------------------------------------------------- */

/* One square of a batch: d_in row-major [k][cols], d_out row-major [2k][cols],
 * device memory, 16-byte aligned; k a power of two in [32, 2048], cols a
 * multiple of 4. */
typedef struct zoda_square {
    const uint32_t* d_in;
    uint32_t* d_out;
    uint32_t k;
    uint32_t reserved; /* 0 */
    uint64_t cols;
} zoda_square;

typedef struct zoda_batch zoda_batch;

/* Plans a batch on `ctx`: sorts the squares by decreasing side, builds their
 * TMA descriptors and the (square, column tile) work queue in device memory.
 * The buffers are not touched until zoda_batch_run. */
zoda_status zoda_batch_create(zoda_ctx* ctx, const zoda_square* squares, uint32_t n, zoda_batch** out);

/* Encodes every square of the batch with one persistent kernel whose CTAs
 * (one per SM) take (square, column tile) items from a device counter, big
 * squares first. The first call captures the counter reset and the launch
 * into a CUDA graph; every call replays that graph on `stream` (a
 * cudaStream_t, NULL = legacy default stream). Asynchronous. Runs of one
 * batch must not overlap on the GPU (they share the counter). */
zoda_status zoda_batch_run(zoda_batch* batch, void* stream);

/* Total input elements (sum of k * cols) of the batch. */
uint64_t zoda_batch_elements(const zoda_batch* batch);

void zoda_batch_destroy(zoda_batch* batch);

/* ----------------------------------------------------------------------
 * Serving loop: squares arrive one by one and are encoded with continuous
 * batching. No reference counterpart (the reference has no server).
 *
 * A native thread owns the GPU side. Every pass it retires finished
 * launches, then admits waiting requests in arrival order while their
 * outputs fit in the HBM budget (an output arena allocated once at
 * creation) and launches them together as one batched kernel on a free
 * stream. Requests that arrive while others run join the next launch, and
 * up to `max_inflight` launches overlap on the device.
 * ---------------------------------------------------------------------- */

typedef struct zoda_server zoda_server;

typedef struct zoda_server_config {
    uint64_t hbm_budget_bytes; /* output arena size = admission budget; 0 = 64 GiB   */
    uint32_t max_inflight;     /* launches in flight (streams); 0 = 4                */
    uint32_t max_batch;        /* squares per launch; 0 = 128                        */
} zoda_server_config;

typedef struct zoda_request_info {
    uint32_t* d_out;   /* output [2k][cols], row-major, in the server's arena       */
    double queue_ms;   /* submit -> launch                                          */
    double latency_ms; /* submit -> completion observed by the server thread       */
    int32_t status;    /* zoda_status of the request                                */
    int32_t reserved;
} zoda_request_info;

typedef struct zoda_server_stats {
    uint64_t submitted, completed, cancelled, launches;
    uint64_t elements;   /* input elements of completed requests */
    double p50_ms, p99_ms, mean_ms, max_ms; /* latency of completed requests */
    double first_submit_to_last_done_ms;
} zoda_server_stats;

/* Creates the server on ctx's device: allocates the output arena and the
 * per-stream descriptor buffers, starts the thread. ZODA_ERR_NOMEM when the
 * arena does not fit. */
zoda_status zoda_server_create(zoda_ctx* ctx, const zoda_server_config* cfg, zoda_server** out);

/* Queues one square: d_in row-major [k][cols] in device memory, k a power of
 * two in [32, 2048], cols a multiple of 4. d_in must stay valid and unchanged
 * until the request completes. ZODA_ERR_BUDGET if its output (8*k*cols bytes)
 * exceeds the whole budget. Returns at once with a ticket. */
zoda_status zoda_server_submit(zoda_server* srv, const uint32_t* d_in, uint32_t k, uint64_t cols,
                               uint64_t* ticket);

/* Waits up to timeout_ms (0 = do not wait) for the request; ZODA_ERR_TIMEOUT
 * if it has not finished. On success info describes it; the output stays in
 * the arena until zoda_server_release. */
zoda_status zoda_server_wait(zoda_server* srv, uint64_t ticket, uint32_t timeout_ms, zoda_request_info* info);

/* Returns a finished request's output region to the arena. */
zoda_status zoda_server_release(zoda_server* srv, uint64_t ticket);

/* Drops a request that has not been launched yet (ZODA_ERR_STATE otherwise);
 * a later wait reports ZODA_ERR_CANCELLED. */
zoda_status zoda_server_cancel(zoda_server* srv, uint64_t ticket);

zoda_status zoda_server_get_stats(zoda_server* srv, zoda_server_stats* stats);

/* Stops the thread after in-flight launches finish; queued requests are
 * cancelled. */
void zoda_server_destroy(zoda_server* srv);

/* ----------------------------------------------------------------------
 * Any shape, and recovery from erasures
 * ---------------------------------------------------------------------- */

/* Encode of k data rows with n parity rows, as src/benchmarks/utils.rs:100-146
 * and src/zoda/babybear.rs:137-152 define it: n_k = next_pow2(k) and
 * n_kn = next_pow2(k + n) (utils.rs:42-48); the k rows, zero-padded to n_k,
 * are interpolated over n_k points and evaluated at the n_kn points
 * omega_{n_kn}^j; d_out receives rows j = 0 .. k+n-1 (the encoded_rows of
 * utils.rs:167-168), row-major [k+n][cols]. d_in is row-major [k][cols].
 * Limits: next_pow2(k) <= 4096, k + n <= 2^27, cols % 4 == 0, 16-byte aligned
 * buffers that do not overlap. When n_kn = 2 n_k (n <= 2 n_k - k, e.g. any
 * k = n) the fused extension kernels run it in one pass, as zoda_extend_device
 * does for power-of-two squares; other shapes run one interpolation and one
 * evaluation per coset on the general column transform, in column chunks
 * whose scratch (<= 256 MiB) the context keeps. Asynchronous on `stream`. */
zoda_status zoda_encode_device(zoda_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t k, uint32_t n,
                               uint64_t cols, void* stream);

/* k-of-2k erasure decoder. No counterpart in the reference, whose tests only
 * re-encode and RLC-check (utils.rs:186-272); this is the recovery a sampling
 * light node or a repairing full node runs.
 * d_code is the [2k][cols] extension (rows in natural order, as
 * zoda_extend_device writes them); only the rows listed in known_rows[0 ..
 * nknown) are read, the others may hold anything. At least k distinct rows
 * must be known. d_data receives the original [k][cols] data. k is a power of
 * two <= 4096. When every even row is known the data is copied out; otherwise
 * the call runs two fused passes, each an INTT and an NTT over 2k points (see
 * general.cu), with the context's scratch (<= 256 MiB). If `mismatch` is not NULL the call also
 * checks that the known rows are one codeword, stores the number of
 * inconsistent coefficients there (0 = consistent) and synchronizes `stream`;
 * otherwise it is asynchronous on `stream`. */
zoda_status zoda_recover_device(zoda_ctx* ctx, const uint32_t* d_code, const uint32_t* known_rows, uint32_t nknown,
                                uint32_t k, uint64_t cols, uint32_t* d_data, uint64_t* mismatch, void* stream);

/* ----------------------------------------------------------------------
 * Row-side consumers: data root and random linear combinations
 * ---------------------------------------------------------------------- */

/* compute_data_root (src/benchmarks/utils.rs:51-59): SHA-256 over the
 * little-endian bytes of rows[0 .. nrows*cols) (row-major, host memory),
 * written as 64 lowercase hex digits plus a NUL. Host only, no GPU needed. */
zoda_status zoda_data_root_host(const uint32_t* rows, uint64_t nrows, uint64_t cols, char out_hex[65]);

/* generate_deterministic_coefficients (src/zoda/rlc.rs:48-65) on the device:
 * for column i < ncols, digest = SHA-256(root[0 .. root_len) || u64_le(i)) and
 * d_coeff[4*i + l] = u64_be(digest[8l .. 8l+8)) mod p, l < 4 (RLC_LIMBS,
 * rlc.rs:18). `root` is the hex string of the data root. Asynchronous. */
zoda_status zoda_rlc_coefficients_device(zoda_ctx* ctx, const char* root, size_t root_len, uint64_t ncols,
                                         uint32_t* d_coeff, void* stream);

/* rlc_row (src/zoda/rlc.rs:32-40) for every row: d_out[4*r + l] =
 * sum_c d_rows[r*cols + c] * d_coeff[4*c + l] mod p, rows <= 262140.
 * One HBM read of the matrix. Asynchronous. */
zoda_status zoda_rlc_rows_device(zoda_ctx* ctx, const uint32_t* d_rows, uint32_t rows, uint64_t cols,
                                 const uint32_t* d_coeff, uint32_t* d_out, void* stream);

/* The RLC soundness check of src/benchmarks/utils.rs:225-272 over EVERY
 * encoded row instead of 64 samples: the RLC of the k data rows d_data
 * [k][cols], extended like the data (zoda_encode_device with cols = 4), must
 * equal the RLC of each of the k + n encoded rows d_code [k+n][cols], limb
 * for limb. Stores the number of (row, limb) pairs that differ in
 * *mismatches (0 = the encoding passes) and synchronizes `stream`. */
zoda_status zoda_rlc_check_device(zoda_ctx* ctx, const uint32_t* d_data, const uint32_t* d_code, uint32_t k,
                                  uint32_t n, uint64_t cols, const uint32_t* d_coeff, uint64_t* mismatches,
                                  void* stream);

/* ======================================================================
 * Part 3: a transform for callers that cannot allocate device memory
 * ====================================================================== */

/* No counterpart in the reference: the reference allocates device memory on
 * every call (cuda/ntt_kernel.cu:111-121).
 *
 * For callers that may not allocate device memory while they run: device
 * memory owned by a pool allocator that forbids raw cudaMalloc, or a
 * latency-bound path where cudaMalloc/cudaFree would synchronise the device
 * and stall other streams. The call performs no cudaMalloc, no cudaFree and
 * no allocating library call; the caller passes the input and the output.
 *
 * What it computes: for each of `polys` polynomials of n canonical u32,
 * laid end to end in device memory (polynomial c at d_in[c*n .. c*n + n)),
 *   d_out[c*n + k] = scale * sum_{i<n} d_in[c*n + i] * w^(s*i*k)  mod p,
 * with w = 31^((p-1)/n), s = +1 and scale = 1 when inverse = 0, and
 * s = -1 and scale = n^-1 mod p when inverse = 1 (natural order in and
 * out, canonical results). d_out may equal d_in. n must be a power of two
 * <= 4096. Asynchronous on `stream` (NULL = the legacy default stream).
 *
 * Limits: the working copy lives in a fixed 16 MiB device array inside the
 * library, so n * round_up(polys, 4) must be <= 4194304 u32; larger requests
 * return ZODA_ERR_UNSUPPORTED with the reason in zoda_last_error(). Every GPU
 * that loads the library holds that array (and a 64 KiB twiddle table) until
 * the process exits.
 *
 * Set-up: the first call on each device (with that device current) looks up
 * the arrays' device addresses and uploads the twiddle table, synchronously;
 * make that first call before capturing any stream into a CUDA graph.
 *
 * Concurrency: all calls on a device share the one array and it keeps the
 * last call's contents. Calls whose work can overlap on the GPU (different
 * streams, or different host threads, without ordering between them) race and
 * corrupt each other's results; order them on one stream or with events. */
zoda_status zoda_ntt_device_noalloc(const uint32_t* d_in, uint32_t* d_out, uint32_t n, uint32_t polys, int inverse,
                                    void* stream);

#ifdef __cplusplus
}
#endif
#endif /* ZODA_B200_H */
