// batch_capi.cu -- C ABI for batched factor-and-solve plans (include/posit_gpu.h).
#include "../../include/posit_gpu.h"
#include "batch.cuh"

#include <algorithm>
#include <new>
#include <numeric>
#include <vector>

struct posit_batch_plan {
    int nprob = 0;
    int ctas = 0;
    pg::BatchProblem *d_probs = nullptr;
    int *d_order = nullptr;
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
    cudaError_t e = cudaMalloc(&p->d_probs, sizeof(pg::BatchProblem) * (nprob > 0 ? nprob : 1));
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
            cudaError_t le = pg::batch_factor_launch(p->d_probs, nprob, p->d_order, p->d_next, p->ctas, cs);
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
