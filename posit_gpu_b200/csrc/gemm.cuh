// gemm.cuh -- posit32 GEMM kernels for sm_100a (declarations shared by the C ABI).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace pg {

// Output tile of one CTA and the k-depth of one staged tile.  A thread owns TM x TN
// outputs; 16 x 16 threads; rows and columns are owned in pairs 32 apart (own_off).
constexpr int TM = 4; // rows per thread
constexpr int TN = 2; // columns per thread
constexpr int BM = 16 * TM;
constexpr int BN = 16 * TN;
constexpr int BK = 16;
constexpr int NTHREADS = 256;
constexpr int STAGES = 3;
constexpr int MIN_CTAS_PER_SM = 3;
static_assert(TM % 2 == 0 && TN % 2 == 0, "operands are loaded in pairs");

// Which entries of C a launch writes (gemm_launch_tri).
constexpr int TRI_FULL = 0;
constexpr int TRI_LOWER = 1; // row >= column
constexpr int TRI_UPPER = 2; // row <= column

// Error flags a kernel can raise (read back with posit_get_device_error).
constexpr int DEV_ERR_WAIT_TIMEOUT = 1;

struct GemmPlan {
    int m, n, k;
    int mt, nt, kt; // tile counts
    size_t a_bytes, b_bytes, flag_bytes;
};

GemmPlan gemm_plan(int m, int n, int k);

// The Rgemm argument checks (Rgemm.cpp:90-128) in the reference's order: 0, or the info
// code of the first bad argument.  Sets nota/notb ('N' or 'n').
int rgemm_check_args(char ta, char tb, int m, int n, int k, int lda, int ldb, int ldc, bool &nota, bool &notb);
size_t gemm_workspace_bytes(int m, int n, int k);

// Decode op(A) and alpha*op(B) (or op(B) for the dot-then-combine order) into the
// workspace, then run the main kernel.  Device pointers; stream-ordered.
cudaError_t gemm_launch(bool nota, bool notb, int m, int n, int k, uint32_t alpha,
                        const uint32_t *A, int lda, const uint32_t *B, int ldb, uint32_t beta,
                        uint32_t *C, int ldc, void *workspace, cudaStream_t stream);

// Same, writing only the entries on or below the diagonal of C (row >= column), and
// doing nothing when *stop != 0 (stop may be null).
cudaError_t gemm_launch_lower(bool nota, bool notb, int m, int n, int k, uint32_t alpha,
                              const uint32_t *A, int lda, const uint32_t *B, int ldb, uint32_t beta,
                              uint32_t *C, int ldc, void *workspace, cudaStream_t stream, const int *stop);

// Any of the three: all of C, its lower or its upper triangle (TRI_*), doing nothing when
// *stop != 0 (stop may be null).
cudaError_t gemm_launch_tri(int tri, bool nota, bool notb, int m, int n, int k, uint32_t alpha,
                            const uint32_t *A, int lda, const uint32_t *B, int ldb, uint32_t beta,
                            uint32_t *C, int ldc, void *workspace, cudaStream_t stream, const int *stop);

// The calls that form no product (alpha == 0, or k == 0), on the m x n submatrix:
// C <- 0 or beta*C; with `dot` (TN/TT and k == 0, alpha != 0) C <- alpha*0 or
// alpha*0 + beta*C, which is NaR everywhere when alpha is NaR.
cudaError_t scale_launch(int m, int n, bool dot, uint32_t alpha, uint32_t beta, uint32_t *C, int ldc,
                         cudaStream_t stream);

// Element-wise IEEE double <-> posit32 conversion on device buffers.
cudaError_t convert_launch(bool to_posit, const void *in, void *out, size_t n, cudaStream_t stream);

int read_device_error(bool clear);
// Device address of the kernels' error flag (for stream-ordered copies of it).
cudaError_t device_error_address(int **p);

// Optional instrumentation: CUDA events around each main-kernel launch, recorded on
// the launch stream, plus a count of this library's kernel launches.
void profile_enable(bool on);
int profile_read(double *main_ms, long long *main_launches, long long *all_launches, bool reset);

} // namespace pg
