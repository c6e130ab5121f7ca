// serve.cu -- the request loop for served Ax = b solves (include/posit_gpu.h).
//
// One loop thread admits queued requests in arrival order (optionally largest work first
// within windows of order_window_ms) while the admitted but
// unfinished requests stay under `max_inflight` and their device bytes (matrix or
// factor, right-hand sides, workspace) under the memory budget; when the budget is
// short it first evicts idle cached factors, least recently used first.  Admitted
// requests become work units on lanes (a CUDA stream with its page-locked staging
// buffers; one unit per lane at a time; a few lanes are reserved for batched units):
//   * the requests with n <= batch_max_n admitted in one pass form one unit: one launch
//     of the batched factor-and-solve kernel (batch.cu), one problem per thread block,
//     largest first;
//   * each larger request is a unit of its own: the blocked device factorization and
//     solve of lapack.cu, the path of posit_rgetrf_dev + posit_rgetrs_dev.
// Units on different lanes run concurrently on the GPU.  A pass runs whenever a request
// arrives or a unit finishes, so requests that arrive while others are on the GPU are
// admitted as soon as a lane, a slot and memory are free (continuous batching).  The CUDA
// work of a unit is issued by launcher threads, so a long launch sequence never holds up
// admission, and a unit reports its end through a host function on its stream.
//
// A factor whose request carries matrix_id >= 0 stays on the device after its unit has
// finished; a later request with that id runs only the solve on it (batched:
// BATCH_SOLVE_ONLY; blocked: Rgetrs / Rpotrs).  Every kernel is one the per-call entry
// points run, with the same per-element operation order, so a request's solution and
// info are the same bits served alone, in any mix, from the cache, or through
// posit_rgetrf + posit_rgetrs (posit_rpotrf + posit_rpotrs).
#include "../../include/posit_gpu.h"
#include "batch.cuh"
#include "gemm.cuh"
#include "lapack.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <new>
#include <string.h>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;
constexpr int ST_PENDING = 0, ST_ADMITTED = 1, ST_DONE = 2;

size_t round_up(size_t x) { return (x + 255) & ~(size_t)255; }
size_t factor_bytes(int n) { return round_up((size_t)n * n * 4) + round_up((size_t)n * 4) + 256; }
size_t rhs_bytes(int n, int nrhs) { return round_up((size_t)n * nrhs * 4); }
double ms_between(Clock::time_point a, Clock::time_point b)
{
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// A matrix on the device: its factor once the factoring unit has finished.
struct Factor {
    long long id = -1;
    int kind = 0, n = 0;
    void *block = nullptr; // [A: n*n posit32][ipiv: n ints][info]
    uint32_t *dA = nullptr;
    int *dipiv = nullptr;
    int *dinfo = nullptr;
    size_t bytes = 0;
    int refs = 0;        // admitted requests using it
    bool ready = false;  // factored, info known on the host
    bool cached = false; // registered under id
    int info = 0;
    uint64_t lru = 0;
};

struct Request {
    long long ticket = 0;
    posit_solve_request q{};
    std::atomic<int> state{ST_PENDING};
    Clock::time_point t_submit, t_admit;
    posit_solve_result res{};
    Factor *f = nullptr;
    bool hit = false;
    uint32_t *dB = nullptr;
    size_t b_bytes = 0;
    bool x_staged = false; // X is pageable: the solution goes through the lane's buffer
    size_t x_off = 0;
};
using Req = std::shared_ptr<Request>;

struct Lane {
    cudaStream_t st = nullptr;
    pg::BatchProblem *h_desc = nullptr; // page-locked descriptors of a batched unit
    size_t desc_cap = 0;
    int *h_info = nullptr; // page-locked: info per request, then the error flag
    size_t info_cap = 0;
    unsigned char *h_x = nullptr; // page-locked staging for pageable X
    size_t x_cap = 0;
    std::vector<void *> retired; // outgrown page-locked buffers (freed at shutdown)
    bool busy = false;           // loop thread only
    bool for_batches = false;    // reserved for batched units
    bool high = false;           // created with the device's greatest stream priority
};

struct Unit {
    struct ::posit_server *srv = nullptr;
    Lane *lane = nullptr;
    bool batched = false;
    std::vector<Req> reqs;
    size_t extra_bytes = 0; // workspace counted in the budget
    int status = 0;         // POSIT_E_* raised while launching
};

} // namespace

struct posit_server {
    // configuration
    size_t budget = 0;
    int max_inflight = 0, max_queue = 0, batch_max_n = 0, nb = 0, priority_n = 0;
    double order_window_ms = 0.0; // 0: arrival order
    bool cache_on = true;
    int device = 0, sms = 148;
    cudaMemPool_t pool = nullptr;
    cudaStream_t free_st = nullptr;
    int *d_err = nullptr;
    std::vector<Lane> lanes;

    // shared with clients, launchers and host callbacks (under mu)
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_launch;
    std::deque<Req> incoming;
    std::vector<Unit *> finished;
    std::deque<Unit *> launch_q;
    std::unordered_map<long long, Req> tickets;
    long long next_ticket = 1;
    bool stop = false, launch_stop = false;
    std::atomic<long long> queued{0};

    // loop thread only
    Clock::time_point t_created = Clock::now(); // origin of the admission-order windows
    std::deque<Req> pending;
    std::unordered_map<long long, Factor *> cache;
    size_t used = 0;
    int inflight = 0, units_inflight = 0;
    uint64_t tick = 0;

    // statistics
    std::atomic<long long> n_submitted{0}, n_completed{0}, n_failed{0}, n_cancelled{0}, n_hits{0}, n_misses{0},
        n_evict{0}, n_batched{0}, n_blocked{0}, inflight_peak{0};
    std::atomic<size_t> a_used{0}, a_peak{0}, a_cached{0};

    std::thread loop_thread;
    std::vector<std::thread> launchers;
};

namespace {

// Panel width of a blocked unit: the configured one, or the tuned width for its n but at
// least SERVE_MIN_NB.  The tuned widths minimise one factorization's time alone; with many
// units sharing the GPU the panels' latency hides behind other units and the trailing
// GEMMs' efficiency counts (k = 16 runs at 64 % of k = 256's rate), so wider panels serve
// more requests per second (the serving burst: 656 solves/s at nb = 32 against 567 at 16,
// then the tuned width up to n = 4096, 523 at 64, 457 at 128).  The bits do not depend on nb.
constexpr int SERVE_MIN_NB = 32;
// Largest thread-block cluster of a served unit's panels (0: the library's 8).
constexpr int SERVE_PANEL_CTAS = 0;
int serve_nb(const posit_server *s, int kind, int n)
{
    return s->nb > 0 ? s->nb : std::max(SERVE_MIN_NB, pg::tuned_panel_width(kind == POSIT_BATCH_LU, n));
}

size_t ws_bytes(const posit_server *s, int kind, int n)
{
    const int nb = serve_nb(s, kind, n);
    return kind == POSIT_BATCH_LU ? pg::rgetrf_workspace_bytes(n, n, nb) : pg::rpotrf_workspace_bytes(n, nb);
}

// Largest device footprint a request can have.
size_t request_bytes(const posit_server *s, const posit_solve_request &q)
{
    size_t b = factor_bytes(q.n) + rhs_bytes(q.n, q.nrhs);
    if (q.n > s->batch_max_n)
        b += ws_bytes(s, q.kind, q.n);
    return b;
}

int fail_code(cudaError_t e) { return e == cudaErrorMemoryAllocation ? POSIT_E_NO_MEMORY : POSIT_E_CUDA; }

void dev_free(posit_server *s, void *p)
{
    if (p)
        cudaFreeAsync(p, s->free_st);
}

void account(posit_server *s)
{
    s->a_used.store(s->used);
    if (s->used > s->a_peak.load())
        s->a_peak.store(s->used);
}

void drop_factor(posit_server *s, Factor *f)
{
    if (f->cached) {
        s->cache.erase(f->id);
        s->a_cached.fetch_sub(f->bytes);
    }
    dev_free(s, f->block);
    s->used -= f->bytes;
    account(s);
    delete f;
}

// Takes `need` bytes of the budget, evicting idle cached factors (least recently used
// first) while it is short.  False when it stays short.
bool reserve(posit_server *s, size_t need)
{
    while (s->used + need > s->budget) {
        Factor *victim = nullptr;
        for (auto &kv : s->cache) {
            Factor *f = kv.second;
            if (f->refs == 0 && f->ready && (!victim || f->lru < victim->lru))
                victim = f;
        }
        if (!victim)
            return false;
        drop_factor(s, victim);
        s->n_evict++;
    }
    s->used += need;
    account(s);
    return true;
}

void release(posit_server *s, size_t bytes)
{
    s->used -= bytes;
    account(s);
}

template <class T> bool grow_pinned(Lane &L, T *&buf, size_t &cap, size_t need)
{
    if (need <= cap)
        return true;
    size_t nc = std::max(need, 2 * cap);
    void *p = nullptr;
    if (cudaMallocHost(&p, nc * sizeof(T)) != cudaSuccess)
        return false;
    if (buf)
        L.retired.push_back(buf); // freeing page-locked memory would wait for the device
    buf = static_cast<T *>(p);
    cap = nc;
    return true;
}

bool is_pinned(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// Allocates the factor block (first use of the matrix) and uploads A.
cudaError_t upload_matrix(posit_server *s, Factor *f, const uint32_t *A, cudaStream_t st)
{
    const int n = f->n;
    cudaError_t e = cudaMallocFromPoolAsync(&f->block, f->bytes, s->pool, st);
    if (e != cudaSuccess)
        return e;
    unsigned char *b = static_cast<unsigned char *>(f->block);
    f->dA = reinterpret_cast<uint32_t *>(b);
    f->dipiv = reinterpret_cast<int *>(b + round_up((size_t)n * n * 4));
    f->dinfo = reinterpret_cast<int *>(b + round_up((size_t)n * n * 4) + round_up((size_t)n * 4));
    e = cudaMemcpyAsync(f->dA, A, (size_t)n * n * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(f->dinfo, 0, sizeof(int), st);
    return e;
}

cudaError_t upload_rhs(posit_server *s, Request &r, cudaStream_t st)
{
    if (r.b_bytes == 0)
        return cudaSuccess;
    cudaError_t e = cudaMallocFromPoolAsync((void **)&r.dB, r.b_bytes, s->pool, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(r.dB, r.q.B, (size_t)r.q.n * r.q.nrhs * 4, cudaMemcpyHostToDevice, st);
    return e;
}

// Solution, info and the kernels' error flag back to the host, for request i of the unit.
cudaError_t download(posit_server *s, Lane &L, Request &r, int i, cudaStream_t st)
{
    cudaError_t e = cudaSuccess;
    const size_t xb = (size_t)r.q.n * r.q.nrhs * 4;
    if (xb) {
        void *dst = r.x_staged ? (void *)(L.h_x + r.x_off) : (void *)r.q.X;
        e = cudaMemcpyAsync(dst, r.dB, xb, cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(&L.h_info[i], r.f->dinfo, sizeof(int), cudaMemcpyDeviceToHost, st);
    return e;
}

// Page-locked room for the unit's infos and for its pageable solutions.
int prepare_lane(Unit *u)
{
    Lane &L = *u->lane;
    if (!grow_pinned(L, L.h_info, L.info_cap, u->reqs.size() + 1))
        return POSIT_E_NO_MEMORY;
    if (u->batched && !grow_pinned(L, L.h_desc, L.desc_cap, u->reqs.size()))
        return POSIT_E_NO_MEMORY;
    size_t xbytes = 0;
    for (auto &r : u->reqs) {
        r->x_staged = r->q.n > 0 && r->q.nrhs > 0 && !is_pinned(r->q.X);
        if (r->x_staged) {
            r->x_off = xbytes;
            xbytes += round_up((size_t)r->q.n * r->q.nrhs * 4);
        }
    }
    if (xbytes && !grow_pinned(L, L.h_x, L.x_cap, xbytes))
        return POSIT_E_NO_MEMORY;
    return 0;
}

#define SV_TRY(expr)                                                                                       \
    do {                                                                                                   \
        cudaError_t e_ = (expr);                                                                           \
        if (e_ != cudaSuccess)                                                                             \
            return fail_code(e_);                                                                          \
    } while (0)

int launch_batched(posit_server *s, Unit *u)
{
    Lane &L = *u->lane;
    cudaStream_t st = L.st;
    const int np = (int)u->reqs.size();
    for (int i = 0; i < np; ++i) {
        Request &r = *u->reqs[i];
        Factor *f = r.f;
        if (!r.hit)
            SV_TRY(upload_matrix(s, f, r.q.A, st));
        SV_TRY(upload_rhs(s, r, st));
        pg::BatchProblem &d = L.h_desc[i];
        d.kind = r.q.kind | (r.hit ? pg::BATCH_SOLVE_ONLY : 0);
        d.n = r.q.n;
        d.lda = std::max(1, r.q.n);
        d.nrhs = r.q.nrhs;
        d.ldb = std::max(1, r.q.n);
        d.A = f->dA;
        d.B = r.dB;
        d.ipiv = f->dipiv;
        d.info = f->dinfo;
    }
    void *dd = nullptr;
    const size_t desc_bytes = round_up(sizeof(pg::BatchProblem) * np);
    SV_TRY(cudaMallocFromPoolAsync(&dd, desc_bytes + 256, s->pool, st));
    int *d_next = reinterpret_cast<int *>(static_cast<unsigned char *>(dd) + desc_bytes);
    cudaError_t e = cudaMemcpyAsync(dd, L.h_desc, sizeof(pg::BatchProblem) * np, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = pg::batch_factor_launch(static_cast<pg::BatchProblem *>(dd), np, nullptr, d_next,
                                    std::min(np, s->sms * 8), st);
    cudaFreeAsync(dd, st);
    if (e != cudaSuccess)
        return fail_code(e);
    for (int i = 0; i < np; ++i)
        SV_TRY(download(s, L, *u->reqs[i], i, st));
    SV_TRY(cudaMemcpyAsync(&L.h_info[np], s->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    return 0;
}

int launch_blocked(posit_server *s, Unit *u)
{
    Lane &L = *u->lane;
    cudaStream_t st = L.st;
    Request &r = *u->reqs[0];
    Factor *f = r.f;
    const int n = r.q.n;
    if (!r.hit) {
        SV_TRY(upload_matrix(s, f, r.q.A, st));
        void *ws = nullptr;
        SV_TRY(cudaMallocFromPoolAsync(&ws, ws_bytes(s, r.q.kind, n), s->pool, st));
        cudaError_t e = r.q.kind == POSIT_BATCH_LU
                            ? pg::rgetrf_launch(n, n, f->dA, n, f->dipiv, serve_nb(s, r.q.kind, n), f->dinfo, ws, st,
                                                SERVE_PANEL_CTAS)
                            : pg::rpotrf_lower_launch(n, f->dA, n, serve_nb(s, r.q.kind, n), f->dinfo, ws, st,
                                                      SERVE_PANEL_CTAS);
        cudaFreeAsync(ws, st);
        if (e != cudaSuccess)
            return fail_code(e);
    }
    SV_TRY(upload_rhs(s, r, st));
    if (r.q.nrhs > 0) {
        if (r.q.kind == POSIT_BATCH_LU)
            SV_TRY(pg::rgetrs_launch(n, r.q.nrhs, f->dA, n, f->dipiv, r.dB, n, st));
        else
            SV_TRY(pg::rpotrs_lower_launch(n, r.q.nrhs, f->dA, n, r.dB, n, st));
    }
    SV_TRY(download(s, L, r, 0, st));
    SV_TRY(cudaMemcpyAsync(&L.h_info[1], s->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
    return 0;
}

void CUDART_CB unit_done(void *p)
{
    Unit *u = static_cast<Unit *>(p);
    posit_server *s = u->srv;
    std::lock_guard<std::mutex> g(s->mu);
    s->finished.push_back(u);
    s->cv_work.notify_one();
}

void launcher_main(posit_server *s)
{
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        s->cv_launch.wait(lk, [&] { return s->launch_stop || !s->launch_q.empty(); });
        if (s->launch_q.empty())
            return;
        Unit *u = s->launch_q.front();
        s->launch_q.pop_front();
        lk.unlock();
        int rc = prepare_lane(u);
        if (rc == 0)
            rc = u->batched ? launch_batched(s, u) : launch_blocked(s, u);
        if (rc == 0) {
            cudaError_t e = cudaLaunchHostFunc(u->lane->st, unit_done, u);
            if (e != cudaSuccess)
                rc = fail_code(e);
        }
        lk.lock();
        if (rc != 0) {
            // let what was queued drain before the loop releases the unit's memory
            u->status = rc;
            lk.unlock();
            cudaStreamSynchronize(u->lane->st);
            cudaGetLastError();
            lk.lock();
            s->finished.push_back(u);
            s->cv_work.notify_one();
        }
    }
}

void finish_request(posit_server *s, const Req &r, int status, int info, std::vector<Req> &done)
{
    r->res.status = status;
    r->res.info = info;
    r->res.cache_hit = r->hit ? 1 : 0;
    r->res.path = r->q.n > s->batch_max_n ? 1 : 0;
    const auto now = Clock::now();
    r->res.queue_ms = ms_between(r->t_submit, r->t_admit);
    r->res.latency_ms = ms_between(r->t_submit, now);
    (status == 0 ? s->n_completed : s->n_failed)++;
    done.push_back(r);
}

// A unit's end (loop thread): results, cache state, memory.
void finish_unit(posit_server *s, Unit *u, std::vector<Req> &done)
{
    Lane &L = *u->lane;
    const int np = (int)u->reqs.size();
    const int dev_err = u->status == 0 ? L.h_info[np] : 0;
    for (int i = 0; i < np; ++i) {
        const Req &r = u->reqs[i];
        Factor *f = r->f;
        const int status = u->status ? u->status : (dev_err ? POSIT_E_DEVICE_FAULT : 0);
        const int info = status == 0 ? L.h_info[i] : 0;
        if (!r->hit && status == 0) {
            f->ready = true;
            f->info = info;
        }
        if (status == 0 && r->x_staged)
            memcpy(r->q.X, L.h_x + r->x_off, (size_t)r->q.n * r->q.nrhs * 4);
        dev_free(s, r->dB);
        r->dB = nullptr;
        release(s, r->b_bytes);
        f->refs--;
        if (status != 0 && !f->ready && f->cached) { // a failed factorization is no factor
            s->cache.erase(f->id);
            s->a_cached.fetch_sub(f->bytes);
            f->cached = false;
        }
        if (!f->cached && f->refs == 0)
            drop_factor(s, f);
        r->f = nullptr;
        s->inflight--;
        finish_request(s, r, status, info, done);
    }
    release(s, u->extra_bytes);
    L.busy = false;
    s->units_inflight--;
    delete u;
}

// Admission order: arrival order by default.  With order_window_ms > 0, requests submitted
// within one such window are taken largest estimated work first (factorization n^3, solve
// n^2 * nrhs), the windows themselves first come, first served: a makespan-oriented order
// for batch jobs.  (Measured on the serving burst it starts the long solves at once but
// gains no throughput -- the burst is bound by the GPU's work, not by the order -- and
// raises the median latency, so it is not the default.)
double est_work(const Req &r)
{
    const double n = r->q.n;
    const double fact = r->q.kind == POSIT_BATCH_LU ? 2.0 / 3.0 : 1.0 / 3.0;
    return fact * n * n * n + 2.0 * n * n * r->q.nrhs;
}

void order_pending(posit_server *s)
{
    if (s->order_window_ms <= 0.0 || s->pending.size() < 2)
        return;
    const Clock::time_point t0 = s->t_created;
    std::stable_sort(s->pending.begin(), s->pending.end(), [&](const Req &a, const Req &b) {
        const long wa = (long)(ms_between(t0, a->t_submit) / s->order_window_ms);
        const long wb = (long)(ms_between(t0, b->t_submit) / s->order_window_ms);
        if (wa != wb)
            return wa < wb;
        return est_work(a) > est_work(b);
    });
}

// One admission pass over the queue, in admission order (loop thread).
void admit(posit_server *s, std::vector<Req> &done, std::vector<Unit *> &units)
{
    order_pending(s);
    // Lanes reserved for batched units keep small requests from waiting behind long
    // blocked ones; a batched unit may also take a free blocked lane.
    // Blocked lanes: those of the greatest priority take the requests of n >= priority_n
    // first; either kind takes the other's lanes when its own are busy.
    std::vector<Lane *> idle_batch, idle_hi, idle_lo;
    for (auto &L : s->lanes)
        if (!L.busy)
            (L.for_batches ? idle_batch : (L.high ? idle_hi : idle_lo)).push_back(&L);
    Unit *group = nullptr;
    bool small_waits = false, large_waits = false; // no lane: later ones of that kind wait too
    auto drop = [&](std::deque<Req>::iterator it) {
        s->queued--;
        return s->pending.erase(it);
    };
    for (auto it = s->pending.begin(); it != s->pending.end();) {
        Req r = *it;
        if (r->state.load() != ST_PENDING) { // cancelled by the client
            it = drop(it);
            continue;
        }
        const posit_solve_request &q = r->q;
        Factor *f = nullptr;
        if (s->cache_on && q.matrix_id >= 0) {
            auto c = s->cache.find(q.matrix_id);
            if (c != s->cache.end())
                f = c->second;
        }
        int early = 0; // a request that finishes without the GPU
        if (f && (f->kind != q.kind || f->n != q.n))
            early = POSIT_E_MISMATCH;
        else if (!f && !q.A && q.n > 0)
            early = POSIT_E_NOT_CACHED;
        if (early || q.n == 0) {
            int exp = ST_PENDING;
            if (r->state.compare_exchange_strong(exp, ST_ADMITTED)) {
                r->t_admit = Clock::now();
                finish_request(s, r, early, 0, done);
            }
            it = drop(it);
            continue;
        }
        if (f && !f->ready) { // its factorization is on the GPU: wait for it
            ++it;
            continue;
        }
        if (s->inflight >= s->max_inflight)
            break;
        const bool hit = f != nullptr;
        const bool small = q.n <= s->batch_max_n;
        const bool none_blocked = idle_hi.empty() && idle_lo.empty();
        if (small) {
            small_waits |= !group && idle_batch.empty() && none_blocked;
        } else {
            large_waits |= none_blocked;
        }
        if (small ? small_waits : large_waits) {
            ++it;
            continue;
        }
        const size_t ws = (!small && !hit) ? ws_bytes(s, q.kind, q.n) : 0;
        const size_t need = rhs_bytes(q.n, q.nrhs) + (hit ? 0 : factor_bytes(q.n)) + ws;
        if (!reserve(s, need))
            break;
        int exp = ST_PENDING;
        if (!r->state.compare_exchange_strong(exp, ST_ADMITTED)) {
            release(s, need);
            it = drop(it);
            continue;
        }
        r->t_admit = Clock::now();
        if (hit) {
            f->refs++;
            r->hit = true;
            s->n_hits++;
        } else {
            f = new Factor();
            f->id = q.matrix_id;
            f->kind = q.kind;
            f->n = q.n;
            f->bytes = factor_bytes(q.n);
            f->refs = 1;
            f->cached = s->cache_on && q.matrix_id >= 0;
            if (f->cached) {
                s->cache[q.matrix_id] = f;
                s->a_cached.fetch_add(f->bytes);
                s->n_misses++;
            }
        }
        f->lru = ++s->tick;
        r->f = f;
        r->b_bytes = rhs_bytes(q.n, q.nrhs);
        s->inflight++;
        if (s->inflight > s->inflight_peak.load())
            s->inflight_peak.store(s->inflight);
        if (small) {
            if (!group) {
                group = new Unit();
                group->srv = s;
                group->batched = true;
                auto &from = !idle_batch.empty() ? idle_batch : (!idle_lo.empty() ? idle_lo : idle_hi);
                group->lane = from.back();
                from.pop_back();
            }
            group->reqs.push_back(r);
        } else {
            Unit *u = new Unit();
            u->srv = s;
            const bool prio = s->priority_n > 0 && q.n >= s->priority_n;
            auto &from = prio ? (!idle_hi.empty() ? idle_hi : idle_lo) : (!idle_lo.empty() ? idle_lo : idle_hi);
            u->lane = from.back();
            from.pop_back();
            u->reqs.push_back(r);
            u->extra_bytes = ws;
            units.push_back(u);
            s->n_blocked++;
        }
        it = drop(it);
    }
    if (group) {
        std::stable_sort(group->reqs.begin(), group->reqs.end(),
                         [](const Req &a, const Req &b) { return a->q.n > b->q.n; });
        units.push_back(group);
        s->n_batched++;
    }
    for (Unit *u : units) {
        u->lane->busy = true;
        s->units_inflight++;
    }
}

void loop_main(posit_server *s)
{
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    bool stop_seen = false;
    for (;;) {
        s->cv_work.wait(lk, [&] { return (s->stop && !stop_seen) || !s->incoming.empty() || !s->finished.empty(); });
        std::vector<Unit *> fin;
        fin.swap(s->finished);
        std::deque<Req> inc;
        inc.swap(s->incoming);
        const bool stopping = s->stop;
        stop_seen = stopping;
        lk.unlock();
        std::vector<Req> done;
        std::vector<Unit *> units;
        for (Unit *u : fin)
            finish_unit(s, u, done);
        for (auto &r : inc)
            s->pending.push_back(r);
        if (stopping) {
            for (auto &r : s->pending) {
                int exp = ST_PENDING;
                if (r->state.compare_exchange_strong(exp, ST_ADMITTED)) {
                    r->t_admit = Clock::now();
                    r->res.status = POSIT_E_CANCELLED;
                    r->res.latency_ms = ms_between(r->t_submit, r->t_admit);
                    s->n_cancelled++;
                    done.push_back(r);
                }
                s->queued--;
            }
            s->pending.clear();
        } else {
            admit(s, done, units);
        }
        lk.lock();
        for (auto &r : done)
            r->state.store(ST_DONE);
        for (Unit *u : units)
            s->launch_q.push_back(u);
        if (!units.empty())
            s->cv_launch.notify_all();
        if (!done.empty())
            s->cv_done.notify_all();
        if (stopping && s->units_inflight == 0 && s->incoming.empty() && s->finished.empty())
            return;
    }
}

void shutdown_resources(posit_server *s)
{
    for (auto &kv : s->cache) {
        dev_free(s, kv.second->block);
        delete kv.second;
    }
    s->cache.clear();
    for (auto &L : s->lanes) {
        if (L.st) {
            cudaStreamSynchronize(L.st);
            cudaStreamDestroy(L.st);
        }
        cudaFreeHost(L.h_desc);
        cudaFreeHost(L.h_info);
        cudaFreeHost(L.h_x);
        for (void *p : L.retired)
            cudaFreeHost(p);
    }
    s->lanes.clear();
    if (s->free_st) {
        cudaStreamSynchronize(s->free_st);
        cudaStreamDestroy(s->free_st);
    }
    if (s->pool)
        cudaMemPoolDestroy(s->pool);
}

} // namespace

extern "C" {

int posit_server_create(const posit_server_config *cfg, posit_server **out)
{
    if (!out)
        return POSIT_E_WORKSPACE;
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return POSIT_E_NO_DEVICE;
    }
    posit_server_config c{};
    if (cfg)
        c = *cfg;
    posit_server *s = new (std::nothrow) posit_server();
    if (!s)
        return POSIT_E_NO_MEMORY;
    cudaGetDevice(&s->device);
    cudaDeviceGetAttribute(&s->sms, cudaDevAttrMultiProcessorCount, s->device);
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const size_t margin = (size_t)2 << 30;
    s->budget = c.memory_budget ? c.memory_budget : POSIT_SERVER_DEFAULT_BUDGET;
    if (free_b > margin)
        s->budget = std::min(s->budget, free_b - margin);
    s->max_inflight = c.max_inflight > 0 ? c.max_inflight : 4096;
    s->max_queue = c.max_queue > 0 ? c.max_queue : (1 << 20);
    s->batch_max_n = c.batch_max_n > 0 ? std::min(c.batch_max_n, POSIT_BATCH_MAX_N) : 256;
    s->nb = c.nb > 0 ? c.nb : 0; // 0: the server's width for each request's n (serve_nb)
    s->priority_n = c.priority_n < 0 ? 0 : (c.priority_n > 0 ? c.priority_n : POSIT_SERVER_PRIORITY_N);
    s->order_window_ms = c.order_window_ms > 0 ? (double)c.order_window_ms : 0.0;
    s->cache_on = c.cache_off == 0;
    const int nlanes = std::max(2, c.lanes > 0 ? c.lanes : 64);
    const int nbatch = std::min(nlanes - 1, c.batch_lanes > 0 ? c.batch_lanes : 4);
    const int nlaunch = c.launch_threads > 0 ? c.launch_threads : 8;

    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = s->device;
    e = cudaMemPoolCreate(&s->pool, &props);
    if (e == cudaSuccess) {
        uint64_t keep = UINT64_MAX; // keep freed memory in the pool for the next request
        e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e == cudaSuccess)
        e = cudaStreamCreateWithFlags(&s->free_st, cudaStreamNonBlocking);
    if (e == cudaSuccess)
        e = pg::device_error_address(&s->d_err);
    int prio_least = 0, prio_greatest = 0;
    if (e == cudaSuccess)
        e = cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
    const int nhigh = s->priority_n > 0 ? std::max(1, (nlanes - nbatch) / 4) : 0;
    s->lanes.resize(nlanes);
    for (int i = 0; i < nlanes && e == cudaSuccess; ++i) {
        Lane &L = s->lanes[i];
        L.for_batches = i < nbatch;
        L.high = !L.for_batches && i >= nlanes - nhigh;
        e = cudaStreamCreateWithPriority(&L.st, cudaStreamNonBlocking, L.high ? prio_greatest : prio_least);
    }
    if (e != cudaSuccess) {
        shutdown_resources(s);
        delete s;
        return fail_code(e);
    }
    s->loop_thread = std::thread(loop_main, s);
    for (int i = 0; i < nlaunch; ++i)
        s->launchers.emplace_back(launcher_main, s);
    *out = s;
    return 0;
}

int posit_server_submit(posit_server *s, const posit_solve_request *q, long long *ticket)
{
    if (!s || !q || !ticket)
        return POSIT_E_WORKSPACE;
    if (q->kind != POSIT_BATCH_LU && q->kind != POSIT_BATCH_CHOLESKY)
        return 1;
    if (q->n < 0)
        return 2;
    if (q->nrhs < 0)
        return 3;
    if (!q->A && q->n > 0 && (q->matrix_id < 0 || !s->cache_on))
        return 4;
    if ((!q->B || !q->X) && (size_t)q->n * q->nrhs > 0)
        return !q->B ? 5 : 6;
    if (request_bytes(s, *q) > s->budget)
        return POSIT_E_NO_MEMORY;
    Req r = std::make_shared<Request>();
    r->q = *q;
    r->t_submit = Clock::now();
    std::lock_guard<std::mutex> g(s->mu);
    if (s->stop)
        return POSIT_E_CANCELLED;
    if (s->queued.load() >= s->max_queue)
        return POSIT_E_QUEUE_FULL;
    r->ticket = s->next_ticket++;
    s->tickets[r->ticket] = r;
    s->incoming.push_back(r);
    s->queued++;
    s->n_submitted++;
    s->cv_work.notify_one();
    *ticket = r->ticket;
    return 0;
}

int posit_server_wait(posit_server *s, long long ticket, posit_solve_result *res)
{
    if (!s)
        return POSIT_E_WORKSPACE;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end())
        return POSIT_E_UNKNOWN_TICKET;
    Req r = it->second;
    s->cv_done.wait(lk, [&] { return r->state.load() == ST_DONE; });
    if (res)
        *res = r->res;
    s->tickets.erase(ticket);
    return 0;
}

int posit_server_poll(posit_server *s, long long ticket, posit_solve_result *res)
{
    if (!s)
        return POSIT_E_WORKSPACE;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end())
        return POSIT_E_UNKNOWN_TICKET;
    if (it->second->state.load() != ST_DONE)
        return 0;
    if (res)
        *res = it->second->res;
    s->tickets.erase(it);
    return 1;
}

int posit_server_cancel(posit_server *s, long long ticket)
{
    if (!s)
        return POSIT_E_WORKSPACE;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end())
        return POSIT_E_UNKNOWN_TICKET;
    Req r = it->second;
    int exp = ST_PENDING;
    if (!r->state.compare_exchange_strong(exp, ST_DONE))
        return 1; // admitted or finished already
    r->res.status = POSIT_E_CANCELLED;
    r->res.latency_ms = ms_between(r->t_submit, Clock::now());
    s->n_cancelled++;
    s->cv_done.notify_all();
    return 0;
}

int posit_server_get_stats(posit_server *s, posit_server_stats *st)
{
    if (!s || !st)
        return POSIT_E_WORKSPACE;
    st->submitted = s->n_submitted.load();
    st->completed = s->n_completed.load();
    st->failed = s->n_failed.load();
    st->cancelled = s->n_cancelled.load();
    st->cache_hits = s->n_hits.load();
    st->cache_misses = s->n_misses.load();
    st->evictions = s->n_evict.load();
    st->batched_units = s->n_batched.load();
    st->blocked_units = s->n_blocked.load();
    st->inflight_peak = s->inflight_peak.load();
    st->budget_bytes = s->budget;
    st->bytes_in_use = s->a_used.load();
    st->bytes_peak = s->a_peak.load();
    st->cached_bytes = s->a_cached.load();
    return 0;
}

void posit_server_destroy(posit_server *s)
{
    if (!s)
        return;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
        s->cv_work.notify_all();
    }
    s->loop_thread.join();
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->launch_stop = true;
        s->cv_launch.notify_all();
    }
    for (auto &t : s->launchers)
        t.join();
    shutdown_resources(s);
    delete s;
}

} // extern "C"
