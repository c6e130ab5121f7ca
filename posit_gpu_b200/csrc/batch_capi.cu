// batch_capi.cu -- C ABI for batched factor-and-solve plans (include/posit_gpu.h).
#include "../../include/posit_gpu.h"
#include "batch.cuh"
#include "batch_gemm.cuh"

#include <ctype.h>

#include <algorithm>
#include <new>
#include <numeric>
#include <vector>

struct posit_batch_plan {
    int nprob = 0;
    int ctas = 0;
    void *d_probs = nullptr; // pg::BatchProblem[] or pg::BatchGemmDesc[]
    void *d_order = nullptr; // int[] (factor plans) or pg::BatchTile[] (GEMM plans)
    int *d_next = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

static_assert(sizeof(posit_batch_problem) == sizeof(pg::BatchProblem), "descriptor layouts agree");

static void plan_free(posit_batch_plan *p)
{
    if (!p)
        return;
    if (p->exec)
        cudaGraphExecDestroy(p->exec);
    if (p->graph)
        cudaGraphDestroy(p->graph);
    cudaFree(p->d_probs);
    cudaFree(p->d_order);
    cudaFree(p->d_next);
    delete p;
}

extern "C" int posit_batch_plan_create(const posit_batch_problem *probs, int nprob, posit_batch_plan **out)
{
    if (!probs || nprob < 0 || !out)
        return 1;
    for (int i = 0; i < nprob; ++i) {
        const posit_batch_problem &q = probs[i];
        if ((q.kind != POSIT_BATCH_LU && q.kind != POSIT_BATCH_CHOLESKY) || q.n < 0 || q.n > POSIT_BATCH_MAX_N ||
            q.lda < (q.n > 1 ? q.n : 1) || q.nrhs < 0 || q.ldb < (q.n > 1 ? q.n : 1) || !q.info)
            return 2;
    }
    posit_batch_plan *p = new (std::nothrow) posit_batch_plan();
    if (!p)
        return POSIT_E_NO_MEMORY;
    p->nprob = nprob;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    p->ctas = sms * 8;
    // largest problems first (work grows like n^3)
    std::vector<int> order(nprob);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return probs[a].n > probs[b].n; });
    cudaError_t e = cudaMalloc((void **)&p->d_probs, sizeof(pg::BatchProblem) * (nprob > 0 ? nprob : 1));
    if (e == cudaSuccess)
        e = cudaMalloc(&p->d_order, sizeof(int) * (nprob > 0 ? nprob : 1));
    if (e == cudaSuccess)
        e = cudaMalloc(&p->d_next, sizeof(int));
    if (e == cudaSuccess && nprob > 0)
        e = cudaMemcpy(p->d_probs, probs, sizeof(pg::BatchProblem) * nprob, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nprob > 0)
        e = cudaMemcpy(p->d_order, order.data(), sizeof(int) * nprob, cudaMemcpyHostToDevice);
    // capture: reset the queue counter, run the persistent kernel
    cudaStream_t cs = nullptr;
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t le = pg::batch_factor_launch(reinterpret_cast<pg::BatchProblem *>(p->d_probs), nprob,
                                                     reinterpret_cast<int *>(p->d_order), p->d_next, p->ctas, cs);
            e = cudaStreamEndCapture(cs, &p->graph);
            if (e == cudaSuccess)
                e = le;
        }
        cudaStreamDestroy(cs);
    }
    if (e == cudaSuccess)
        e = cudaGraphInstantiate(&p->exec, p->graph, 0);
    if (e != cudaSuccess) {
        plan_free(p);
        return e == cudaErrorMemoryAllocation ? POSIT_E_NO_MEMORY : POSIT_E_CUDA;
    }
    *out = p;
    return 0;
}

// ---- batched GEMM -------------------------------------------------------------
static bool same_c(char a, char b) { return toupper((unsigned char)a) == toupper((unsigned char)b); }

// Rgemm.cpp:90-128 checks for one problem.
static int gemm_args(const posit_batch_gemm &q)
{
    bool nota = same_c(q.transa, 'N'), notb = same_c(q.transb, 'N');
    int nrowa = nota ? q.m : q.k, nrowb = notb ? q.k : q.n;
    if (!nota && !same_c(q.transa, 'C') && !same_c(q.transa, 'T'))
        return 1;
    if (!notb && !same_c(q.transb, 'C') && !same_c(q.transb, 'T'))
        return 2;
    if (q.m < 0)
        return 3;
    if (q.n < 0)
        return 4;
    if (q.k < 0)
        return 5;
    if (q.lda < (nrowa > 1 ? nrowa : 1))
        return 8;
    if (q.ldb < (nrowb > 1 ? nrowb : 1))
        return 10;
    if (q.ldc < (q.m > 1 ? q.m : 1))
        return 13;
    return 0;
}

static int size_bucket(int x) { return x <= 32 ? 0 : (x <= 64 ? 1 : 2); }

// Default tile-shape table (rows: m bucket <=32, <=64, >64; columns: n bucket), used
// when the caller passes none, as the autotuner measured it on B200: 32x32 outputs per
// block, except 64x32 for m in 33..64 with n > 64 and 32x64 when both exceed 64.
static const int kDefaultTileTable[9] = {1, 1, 1, 1, 1, 0, 1, 1, 2}; // tuning_b200.json

extern "C" int posit_batch_gemm_plan_create(const posit_batch_gemm *probs, int nprob, const int *tile_table,
                                            posit_batch_plan **out, int *bad_index)
{
    if (!probs || nprob < 0 || !out)
        return POSIT_E_WORKSPACE;
    const int *table = tile_table ? tile_table : kDefaultTileTable;
    for (int c = 0; c < 9; ++c)
        if (table[c] < 0 || table[c] >= pg::BATCH_TILE_CONFIGS)
            return POSIT_E_WORKSPACE;
    std::vector<pg::BatchGemmDesc> desc(nprob > 0 ? nprob : 1);
    std::vector<pg::BatchTile> tiles;
    for (int i = 0; i < nprob; ++i) {
        const posit_batch_gemm &q = probs[i];
        int info = gemm_args(q);
        if (info) {
            if (bad_index)
                *bad_index = i;
            return info;
        }
        pg::BatchGemmDesc &d = desc[i];
        d.nota = same_c(q.transa, 'N');
        d.notb = same_c(q.transb, 'N');
        d.m = q.m;
        d.n = q.n;
        d.k = q.k;
        d.alpha = q.alpha;
        d.beta = q.beta;
        d.A = q.A;
        d.lda = q.lda;
        d.B = q.B;
        d.ldb = q.ldb;
        d.C = q.C;
        d.ldc = q.ldc;
        // quick return (Rgemm.cpp:134-136): no work at all
        if (q.m == 0 || q.n == 0 || ((q.alpha == 0 || q.k == 0) && q.beta == 0x40000000u))
            continue;
        const int cfg = table[size_bucket(q.m) * 3 + size_bucket(q.n)];
        const int bm = pg::batch_tile_rows(cfg), bn = pg::batch_tile_cols(cfg);
        for (int nt = 0; nt < (q.n + bn - 1) / bn; ++nt)
            for (int mt = 0; mt < (q.m + bm - 1) / bm; ++mt)
                tiles.push_back(pg::BatchTile{i, mt, nt, cfg});
    }
    // longest k first
    std::stable_sort(tiles.begin(), tiles.end(),
                     [&](const pg::BatchTile &a, const pg::BatchTile &b) { return desc[a.prob].k > desc[b.prob].k; });
    posit_batch_plan *p = new (std::nothrow) posit_batch_plan();
    if (!p)
        return POSIT_E_NO_MEMORY;
    p->nprob = (int)tiles.size();
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    p->ctas = sms * 2;
    const size_t nt = tiles.size() > 0 ? tiles.size() : 1;
    cudaError_t e = cudaMalloc(&p->d_probs, sizeof(pg::BatchGemmDesc) * desc.size());
    if (e == cudaSuccess)
        e = cudaMalloc(&p->d_order, sizeof(pg::BatchTile) * nt);
    if (e == cudaSuccess)
        e = cudaMalloc((void **)&p->d_next, sizeof(int));
    if (e == cudaSuccess)
        e = cudaMemcpy(p->d_probs, desc.data(), sizeof(pg::BatchGemmDesc) * desc.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !tiles.empty())
        e = cudaMemcpy(p->d_order, tiles.data(), sizeof(pg::BatchTile) * tiles.size(), cudaMemcpyHostToDevice);
    cudaStream_t cs = nullptr;
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            cudaError_t le = pg::batch_gemm_launch(reinterpret_cast<pg::BatchGemmDesc *>(p->d_probs),
                                                   reinterpret_cast<pg::BatchTile *>(p->d_order), p->nprob,
                                                   p->d_next, p->ctas, cs);
            e = cudaStreamEndCapture(cs, &p->graph);
            if (e == cudaSuccess)
                e = le;
        }
        cudaStreamDestroy(cs);
    }
    if (e == cudaSuccess)
        e = cudaGraphInstantiate(&p->exec, p->graph, 0);
    if (e != cudaSuccess) {
        plan_free(p);
        return e == cudaErrorMemoryAllocation ? POSIT_E_NO_MEMORY : POSIT_E_CUDA;
    }
    *out = p;
    return 0;
}

extern "C" int posit_batch_plan_launch(posit_batch_plan *plan, void *stream)
{
    if (!plan)
        return 1;
    cudaError_t e = cudaGraphLaunch(plan->exec, stream ? (cudaStream_t)stream : cudaStreamPerThread);
    return e == cudaSuccess ? 0 : POSIT_E_CUDA;
}

extern "C" void posit_batch_plan_destroy(posit_batch_plan *plan) { plan_free(plan); }
