/*
 * posit_gpu.h -- C ABI of the B200 posit32 BLAS (libposit_gpu_b200.so).
 *
 * A posit32 is passed as its raw 32-bit pattern (uint32_t): the SoftPosit posit32
 * class of the reference is one 32-bit word (member `value`), so a posit32* is a
 * uint32_t* and a posit32 argument is its `.value`.  Matrices are column-major with
 * leading dimensions, exactly as in the reference.
 *
 * Return codes: 0 on success; 1..13 is the BLAS "info" of the first bad argument (the
 * number the reference hands to Mxerbla, which exits -- here it is returned);
 * negative values are POSIT_E_* below.
 */
#ifndef POSIT_GPU_H
#define POSIT_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define POSIT_E_CUDA (-1)         /* a CUDA runtime call failed (see posit_last_cuda_error) */
#define POSIT_E_NO_DEVICE (-2)    /* no usable CUDA device */
#define POSIT_E_NO_MEMORY (-3)    /* device or pinned-host allocation failed */
#define POSIT_E_DEVICE_FAULT (-4) /* a kernel raised its error flag (bounded wait expired) */
#define POSIT_E_WORKSPACE (-5)    /* caller-provided workspace too small */
#define POSIT_E_NOALLOC_LIMIT (-6) /* shape needs more scratch than posit_rgemm_dev_noalloc has */
#define POSIT_E_UNSUPPORTED (-7)   /* reserved: a variant this library does not implement on the device */

/* Replaces initOpenCL (libRpack/def.h:63, libRpack/Rgemm_opencl.cpp:59-70): selects
 * the current CUDA device, creates its context and warms the kernels.  Optional: every
 * entry point initialises lazily.  Returns 0 or a POSIT_E_* code. */
int posit_init(void);

/* C <- alpha*op(A)*op(B) + beta*C on HOST buffers, synchronous.
 * Replaces RgemmG (libRpack/mpblas_posit.h:49-55, libRpack/Rgemm_opencl.cpp:199-250)
 * and has the semantics of the CPU Rgemm (libRpack/Rgemm.cpp:62-251): transa/transb
 * are 'N', 'T' or 'C' in either case ('C' means transposed; RgemmG treated it as 'N'),
 * argument checks return the Rgemm info code, quick returns as in Rgemm.cpp:134-157,
 * and per-element operation order as in Rgemm.cpp:163-247, so results are bit-identical
 * to the CPU Rgemm for every transpose case.  Unlike RgemmG there is no CPU path for
 * small m or n (Rgemm_opencl.cpp:232-235), and only the m x n submatrix of C is read
 * and written (RgemmG copies whole ldc*n spans). */
int posit_rgemm(char transa, char transb, int m, int n, int k, uint32_t alpha, const uint32_t *A,
                int lda, const uint32_t *B, int ldb, uint32_t beta, uint32_t *C, int ldc);

/* Device-memory form of posit_rgemm: A, B, C are device pointers; the call is
 * asynchronous on `stream` (a cudaStream_t; NULL = the calling thread's default
 * stream).  `workspace` may be NULL, in which case a stream-ordered allocation of
 * posit_rgemm_workspace_size() bytes is made and freed on `stream`; otherwise it must be
 * a device buffer of at least that many bytes, 16-byte aligned, not in use by another
 * call in flight.  No reference counterpart: the reference ships host buffers on every
 * call (Rgemm_opencl.cpp:165-173); this is what keeps factorizations device-resident. */
int posit_rgemm_dev(char transa, char transb, int m, int n, int k, uint32_t alpha, const uint32_t *A,
                    int lda, const uint32_t *B, int ldb, uint32_t beta, uint32_t *C, int ldc,
                    void *workspace, size_t workspace_bytes, void *stream);

/* posit_rgemm_dev for callers that cannot allocate device memory (a host whose memory
 * manager has reserved the GPU's memory, or a loop that must not let cudaMalloc/cudaFree
 * synchronise the device).  No counterpart in the reference.  It allocates nothing: its
 * scratch is a static device array of POSIT_NOALLOC_SCRATCH_BYTES compiled into the
 * library, held by every GPU that loads the library until the process exits.  Shapes
 * whose posit_rgemm_workspace_size exceeds that size return POSIT_E_NOALLOC_LIMIT (e.g.
 * 2048 x 2048 x 2032 fits, 2048^3 does not; an 8192 x 8192 x 256 trailing update needs
 * 34 MB and fits).
 * Argument errors return the Rgemm info code first; calls that form no product (alpha
 * == 0, k == 0, the quick returns) use no scratch and are never refused.
 * The first call on a device looks up the array's address; make it before any stream
 * capture, and do not call it again after a cudaDeviceReset (the cached address is then
 * stale).  All calls share the array: calls that overlap on the GPU race. */
#define POSIT_NOALLOC_SCRATCH_BYTES (64u << 20)
int posit_rgemm_dev_noalloc(char transa, char transb, int m, int n, int k, uint32_t alpha,
                            const uint32_t *A, int lda, const uint32_t *B, int ldb, uint32_t beta,
                            uint32_t *C, int ldc, void *stream);

/* Bytes of device workspace posit_rgemm_dev needs for this shape (0 when none). */
size_t posit_rgemm_workspace_size(char transa, char transb, int m, int n, int k);

/* ---- Device-resident factorizations and solves ------------------------------------
 * Bit-identical to the reference's CPU Rgetrf / Rgetrs / Rpotrf / Rpotrs (at any block
 * size: LU and lower Cholesky in the reference's operation order do not depend on it,
 * for inputs without NaR).  Return value: 0, the number of an illegal argument (as the
 * reference passes to Mxerbla: 1, 2, 4, ... ), or a negative POSIT_E_* code.  The
 * numerical result goes to *info exactly as in the reference (first zero pivot / first
 * non-positive leading minor, 1-based; 0 on success).  LU continues past a zero pivot as
 * the reference does, and its factors stay bit-identical; a Cholesky factorization that
 * stops (info > 0) leaves the not-yet-factored part of A in an unspecified state (the
 * reference's left-looking blocking and this right-looking one differ there).
 * nb <= 0 selects the panel width measured fastest on B200 for that n (the autotuner's
 * table, built in).  Upper Cholesky is the exception: in the reference's order
 * (left-looking, each entry's update a dot product over the rows above it, Rpotrf.cpp:96-118)
 * its bits depend on nb, which is therefore the caller's -- the reference CPU routine's
 * own block size comes from iMlaenv, 64 (iMlaenv.cpp:223-228), and nb <= 0 selects that.
 *
 * _dev forms: device pointers (ipiv and info included: *info is written on the device,
 * asynchronously on `stream`); workspace is stream-ordered.  Host forms: host pointers,
 * synchronous.  Every variant runs on the device: Rgetrs with trans 'N', 'T' or 'C'
 * (Rgetrs.cpp:84-113), Rpotrf and Rpotrs with uplo 'L' or 'U' (Rpotrf.cpp:96-143,
 * Rpotrs.cpp:84-106). */
#define POSIT_RPOTRF_UPPER_DEFAULT_NB 64
/* The panel width nb <= 0 selects for an n x n LU (lu = 1) or lower Cholesky (lu = 0);
 * host-only, no device needed. */
int posit_tuned_panel_width(int lu, int n);

/* Rgetrf (libRpack/Rgetrf.cpp:32-137; mplapack_posit.h:48), Rgetrf_opencl (mplapack_posit.h:49) */
int posit_rgetrf_dev(int m, int n, uint32_t *A, int lda, int *ipiv, int nb, int *info, void *stream);
int posit_rgetrf(int m, int n, uint32_t *A, int lda, int *ipiv, int nb, int *info);
/* Rgetrs (libRpack/Rgetrs.cpp:32-118; mplapack_posit.h:46) */
int posit_rgetrs_dev(char trans, int n, int nrhs, const uint32_t *A, int lda, const int *ipiv, uint32_t *B,
                     int ldb, void *stream);
int posit_rgetrs(char trans, int n, int nrhs, const uint32_t *A, int lda, const int *ipiv, uint32_t *B, int ldb);
/* Rpotrf (libRpack/Rpotrf.cpp:32-154; mplapack_posit.h:38), Rpotrf_opencl (mplapack_posit.h:43) */
int posit_rpotrf_dev(char uplo, int n, uint32_t *A, int lda, int nb, int *info, void *stream);
int posit_rpotrf(char uplo, int n, uint32_t *A, int lda, int nb, int *info);
/* Rpotrs (libRpack/Rpotrs.cpp:32-110; mplapack_posit.h:41) */
int posit_rpotrs_dev(char uplo, int n, int nrhs, const uint32_t *A, int lda, uint32_t *B, int ldb, void *stream);
int posit_rpotrs(char uplo, int n, int nrhs, const uint32_t *A, int lda, uint32_t *B, int ldb);

/* ---- Batched factor-and-solve (no reference counterpart) ---------------------------
 * Many independent LU or Cholesky problems, each factored in place and solved for its
 * right-hand sides, in ONE persistent kernel fed by a device work queue (largest
 * problems first), captured once in a CUDA graph.  Results are bit-identical to the
 * per-call path (posit_rgetrf_dev + posit_rgetrs_dev, posit_rpotrf_dev('L') +
 * posit_rpotrs_dev('L')) and hence to the CPU routines.  Each problem runs on one thread
 * block, so this is for many small-to-medium problems (n <= POSIT_BATCH_MAX_N). */
#define POSIT_BATCH_LU 0
#define POSIT_BATCH_CHOLESKY 1
#define POSIT_BATCH_MAX_N 4096
typedef struct {
    int kind;           /* POSIT_BATCH_LU or POSIT_BATCH_CHOLESKY (lower) */
    int n, lda, nrhs, ldb;
    uint32_t *A;        /* device, n x n, factored in place */
    uint32_t *B;        /* device, n x nrhs, overwritten by the solution */
    int *ipiv;          /* device, n 1-based pivots (LU only) */
    int *info;          /* device, the reference's info */
} posit_batch_problem;
typedef struct posit_batch_plan posit_batch_plan;
/* Uploads the descriptors (host array) and captures the launch; returns 0, 1/2 for bad
 * arguments / a bad descriptor, or POSIT_E_*. */
int posit_batch_plan_create(const posit_batch_problem *probs, int nprob, posit_batch_plan **plan);
/* Many independent GEMMs (device pointers), each with the semantics and bits of
 * posit_rgemm_dev, in ONE persistent kernel fed by a device queue of output tiles
 * (longest k first), captured in a CUDA graph.  tile_table (9 ints, or NULL for the
 * built-in default) maps the (m, n) size bucket -- row: m <= 32, <= 64, > 64; column: the
 * same for n -- to a tile shape: 0 = 64x32, 1 = 32x32, 2 = 32x64 outputs per block; the
 * autotuner (posit_gpu_b200/autotune.py) measures it.  A bad argument returns its Rgemm
 * info code and its problem index in *bad_index. */
typedef struct {
    char transa, transb;
    int m, n, k;
    uint32_t alpha, beta;
    const uint32_t *A;
    int lda;
    const uint32_t *B;
    int ldb;
    uint32_t *C;
    int ldc;
} posit_batch_gemm;
int posit_batch_gemm_plan_create(const posit_batch_gemm *probs, int nprob, const int *tile_table,
                                 posit_batch_plan **plan, int *bad_index);

/* Replays a plan's captured launch on `stream` (asynchronous). */
int posit_batch_plan_launch(posit_batch_plan *plan, void *stream);
void posit_batch_plan_destroy(posit_batch_plan *plan);

/* ---- Served solves (no reference counterpart) ---------------------------------------
 * A request loop for Ax = b solves of mixed kind, n and nrhs that arrive over time.  A
 * loop thread admits queued requests in arrival order (with order_window_ms > 0: windows of
 * that many ms in arrival order, the largest work first within a window) while
 * admitted-but-unfinished
 * requests stay under max_inflight and their device bytes (matrix/factor, right-hand
 * sides, workspace) under the memory budget, evicting idle cached factors (least
 * recently used first) when it is short; a request that finds no free lane of its kind
 * waits, and so do later ones of that kind, while the other kind moves on.  Requests with n <= batch_max_n admitted
 * together run as one launch of the batched kernel above; larger ones run the blocked
 * device path (posit_rgetrf_dev + posit_rgetrs_dev, posit_rpotrf_dev('L') +
 * posit_rpotrs_dev('L')), each on a stream of its own, so units overlap on the GPU and
 * requests that arrive meanwhile are admitted as lanes, slots and memory free up.  A
 * request with matrix_id >= 0 leaves its factor on the device; a later request with the
 * same id runs the solve only (its A may then be NULL).
 *
 * Results are bit-identical to the per-call path -- and so to the CPU Rgetrf/Rgetrs,
 * Rpotrf/Rpotrs -- whether served alone, in any mix, or from the cache.  When info != 0
 * the contents of X are unspecified.  Host buffers must stay valid until the request is
 * finished; page-locked buffers are copied asynchronously, pageable ones cost a host copy
 * on the serving threads.  Multiple client threads may submit and wait concurrently.
 * The lanes are CUDA streams; CUDA maps streams onto CUDA_DEVICE_MAX_CONNECTIONS hardware
 * queues (default 8, at most 32), read when the process creates its CUDA context: set it
 * to 32 in the environment for units on different lanes to overlap fully. */
#define POSIT_E_QUEUE_FULL (-8)      /* the server's queue holds max_queue requests */
#define POSIT_E_CANCELLED (-9)       /* cancelled before admission, or the server shut down */
#define POSIT_E_NOT_CACHED (-10)     /* A == NULL and no factor is cached under matrix_id */
#define POSIT_E_MISMATCH (-11)       /* matrix_id cached with another kind or n */
#define POSIT_E_UNKNOWN_TICKET (-12) /* no such ticket (or its result was already taken) */
#define POSIT_SERVER_DEFAULT_BUDGET ((size_t)150000000000ull) /* 150 GB */
#define POSIT_SERVER_PRIORITY_N 2048
typedef struct posit_server posit_server;
typedef struct {
    size_t memory_budget; /* device bytes; 0 = 150 GB (capped at free memory - 2 GiB) */
    int max_inflight;     /* admitted, unfinished requests; 0 = 4096 */
    int max_queue;        /* submitted, not yet admitted requests; 0 = 2^20 */
    int lanes;            /* CUDA streams work units run on; 0 = 64 */
    int launch_threads;   /* threads issuing the units' CUDA work; 0 = 8 */
    int batch_max_n;      /* n <= this goes to the batched kernel; 0 = 256 (max POSIT_BATCH_MAX_N) */
    int nb;               /* panel width of the blocked path; 0 = the tuned width for each n, at
                             least 32 (wider panels serve more requests per second when many
                             share the GPU; the bits do not depend on nb) */
    int cache_off;        /* 1: never keep factors */
    int batch_lanes;      /* lanes reserved for batched units; 0 = 4 */
    int order_window_ms;  /* > 0: requests submitted within one window of this many ms are
                             admitted largest work first, windows in arrival order; 0 = arrival order */
    int priority_n;       /* blocked requests with n >= this run on lanes of the device's greatest
                             stream priority (a quarter of the blocked lanes), so the longest
                             requests get SMs first; 0 = POSIT_SERVER_PRIORITY_N, < 0 = none */
} posit_server_config;
typedef struct {
    int kind;             /* POSIT_BATCH_LU or POSIT_BATCH_CHOLESKY (lower) */
    int n, nrhs;
    long long matrix_id;  /* >= 0: cache the factor under this id (or use the cached one) */
    const uint32_t *A;    /* host n x n, column-major, lda = n; NULL = use the cached factor */
    const uint32_t *B;    /* host n x nrhs, ldb = n */
    uint32_t *X;          /* host n x nrhs, receives the solution (may be B) */
} posit_solve_request;
typedef struct {
    int status;           /* 0 or POSIT_E_* (the request did not run, or failed) */
    int info;             /* the factorization's info (Rgetrf / Rpotrf) */
    int cache_hit;        /* 1: solved on a cached factor */
    int path;             /* 0: batched kernel, 1: blocked path */
    double queue_ms;      /* submit -> admission */
    double latency_ms;    /* submit -> solution in X */
} posit_solve_result;
typedef struct {
    long long submitted, completed, failed, cancelled;
    long long cache_hits, cache_misses, evictions;
    long long batched_units, blocked_units, inflight_peak;
    size_t budget_bytes, bytes_in_use, bytes_peak, cached_bytes;
} posit_server_stats;
/* 0 or POSIT_E_*; with cfg == NULL every field takes its default. */
int posit_server_create(const posit_server_config *cfg, posit_server **server);
/* Queues a request: 0 and a ticket, 1..6 for a bad argument (kind, n, nrhs, A, B, X), or
 * POSIT_E_NO_MEMORY (can never fit the budget) / POSIT_E_QUEUE_FULL / POSIT_E_CANCELLED. */
int posit_server_submit(posit_server *s, const posit_solve_request *req, long long *ticket);
/* Blocks until the request is finished and takes its result (the ticket is then gone). */
int posit_server_wait(posit_server *s, long long ticket, posit_solve_result *res);
/* 1 and the result if finished (the ticket is then gone), 0 if not yet. */
int posit_server_poll(posit_server *s, long long ticket, posit_solve_result *res);
/* 0: cancelled (it had not been admitted); 1: admitted or finished already. */
int posit_server_cancel(posit_server *s, long long ticket);
int posit_server_get_stats(posit_server *s, posit_server_stats *st);
/* Cancels queued requests, waits for admitted ones, frees everything. */
void posit_server_destroy(posit_server *s);

/* Element-wise conversions on device buffers, asynchronous on `stream`.
 * Replace the SoftPosit class conversions the reference drivers use to build their
 * inputs and error norms (posit32 = double, main_gemm.cpp:99-104; .toDouble(),
 * main_gemm.cpp:162-163).  double -> posit32 is correctly rounded (nearest, ties to the
 * even pattern, never to zero or NaR; NaN/inf -> NaR); posit32 -> double is exact. */
int posit_from_double_dev(const double *x, uint32_t *out, size_t n, void *stream);
int posit_to_double_dev(const uint32_t *x, double *out, size_t n, void *stream);

/* Reads (and with clear != 0 resets) the device-side error flags raised by kernels. */
int posit_device_error(int clear);

/* Instrumentation (no reference counterpart).  When enabled, CUDA events are recorded
 * around every GEMM main-kernel launch on its own stream; posit_profile_read waits for
 * them and returns the summed main-kernel time, the number of main-kernel launches and
 * the number of all kernels this library launched since the last reset. */
void posit_profile_enable(int on);
int posit_profile_read(double *main_kernel_ms, long long *main_launches, long long *all_launches, int reset);

/* The last CUDA error code seen by the library (cudaError_t value). */
int posit_last_cuda_error(void);

/* Human-readable text for a return code. */
const char *posit_strerror(int code);

#ifdef __cplusplus
}
#endif
#endif /* POSIT_GPU_H */
