// batch_gemm.cuh -- batched posit32 GEMMs (batch_gemm.cu).
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace pg {

// One GEMM of a batch (device pointers), arguments already checked.
struct BatchGemmDesc {
    int nota, notb;
    int m, n, k;
    uint32_t alpha, beta;
    const uint32_t *A;
    int lda;
    const uint32_t *B;
    int ldb;
    uint32_t *C;
    int ldc;
};

// One queue item: an output tile of problem `prob` with tile shape `cfg`.
struct BatchTile {
    int prob, mt, nt, cfg;
};

// Tile shapes: 0 = 64x32, 1 = 32x32, 2 = 32x64 (rows x columns of C per CTA).
constexpr int BATCH_TILE_CONFIGS = 3;
__host__ __device__ inline int batch_tile_rows(int cfg) { return cfg == 0 ? 64 : 32; }
__host__ __device__ inline int batch_tile_cols(int cfg) { return cfg == 2 ? 64 : 32; }

size_t batch_gemm_smem_bytes();
cudaError_t batch_gemm_launch(const BatchGemmDesc *probs, const BatchTile *tiles, int ntiles, int *next, int ctas,
                              cudaStream_t st);

} // namespace pg
