// Batched, continuously-admitting reconstruction engine (the served form of
// the path) and its C ABI.
//
// The reference runs one cudaShrinkWrap per request on one of three CUDA
// streams, from a std::thread per task (src/imresh/io/taskQueue.cu:91-193);
// every cycle synchronises the host twice and allocates and frees device
// memory.  Here all admitted reconstructions live on the device at once and
// advance together: one step runs one shrink-wrap cycle of every active
// reconstruction, with every pass of the cycle launched once per image-side
// class (rows grouped by width, columns by height) over a device-resident
// work list that covers all reconstructions of that class.  Reconstructions
// of different sizes therefore share every launch of their class; new
// requests are admitted between steps as device memory frees up, finished
// ones (stop test met or cycles exhausted, decided on the device) retire and
// their results are copied out.  Between steps a reconstruction can be saved
// to host memory and suspended, and resumed later in this or another engine.
//
// A step is one CUDA graph: the launches of one cycle of every active
// reconstruction are captured once and replayed step after step; the graph
// is rebuilt (re-captured and updated in place where its shape allows) only
// when the active set changes.  Every kernel skips the items of stopped
// reconstructions, so a graph stays valid while its reconstructions finish
// on the device.  The host learns of finished reconstructions from an
// asynchronous copy of all job states made after every step and read two
// steps later, so the host never waits for the step it just launched: the
// GPU always has the next step queued while the host admits, retires and
// rebuilds.  Results leave through pinned staging and reach the caller's
// buffer once their copy is known to be complete.  The staging is pinned by
// a helper thread while the GPU runs (pinning 168 MB of results at the end of
// a batch cost 70-79 ms on the caller's thread), and the last copy into the
// callers' (pageable, often never touched) buffers runs on several threads.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include <stdio.h>

#include "imresh_b200.h"
#include "kernels.cuh"
#include "engine_host.hpp"

namespace imr {

static double now_ms()
{
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// Pinned host staging for retired results: chunks of kStageChunk bytes (or
// one result's size if larger), filled front to back and reused once every
// result in them has been handed over.
struct Staging {
    char *p = nullptr;
    size_t cap = 0;
    size_t used = 0;   // bytes handed out since the chunk was last empty
    int busy = 0;      // results in it not yet handed over
};
constexpr size_t kStageChunk = (size_t)16 << 20;
constexpr size_t kStageMax = (size_t)1 << 30;   // pinned staging the helper grows to at most

// Helper thread that pins staging chunks ahead of need: the engine asks for
// room for the results of every resident request, the helper allocates it
// (cudaMallocHost, with the engine's device current) while the caller's
// thread drives the GPU, and the engine adopts the chunks between steps.
// One chunk per step: pinning holds driver locks that the caller's next CUDA
// calls wait for (all 168 MB at once stalled a step by 74 ms; one 16 MB chunk
// takes ~7 ms, less than the queued GPU work).
struct StageGrower {
    std::thread th;
    std::mutex mu;
    std::condition_variable cv;
    size_t want = 0, have = 0;   // bytes requested in total / allocated so far
    size_t min_chunk = kStageChunk;
    int credit = 0;              // chunks the helper may allocate now
    std::vector<Staging> ready;  // allocated, not adopted yet
    bool stop = false, failed = false;
};

struct EJob {
    int slot = -1;
    unsigned W = 0, H = 0;
    imr_params p{};
    const float *h_in = nullptr;
    float *h_out = nullptr;
    long long tag = 0;
    double t_submit = 0, t_done = 0;
    char *arena = nullptr;
    JobDev J{};
    JobShape S;
    int cycles_done = 0;
    float last_error = 0.f;
    int status = IMR_SUCCESS;
    long admit_step = -1;       // its state was set before this step's state copy: older copies are stale
    long cycles_launched = 0;   // cycles queued for it so far (a request ends after n_cycles + 1)
    bool intensity = false;     // h_in is a measured intensity: the modulus is its square root
    long copy_step = -1;        // retiring: its result copy precedes this step's status copy
    int staging = -1;           // retiring: index of its pinned staging chunk (-1: direct copy)
    size_t staging_off = 0;     // its place in that chunk
    std::vector<char> resume;   // snapshot to continue from (empty: a new request)
};

// Snapshot of one reconstruction between engine steps: the header, then
// X, g_prev (complex64), the modulus (float32), the support mask (bytes)
// and the per-cycle errors (float32), each W*H (errors: n_err) long.
struct SnapHeader {
    char magic[8];
    uint32_t W, H;
    imr_params p;
    long long tag;
    JobState st;
    uint32_t n_err;
    uint32_t pad;
    uint64_t bytes;
};
constexpr char kSnapMagic[8] = {'I', 'M', 'R', 'S', 'N', 'A', 'P', '1'};

static size_t snap_bytes(unsigned W, unsigned H, unsigned n_err)
{
    const size_t N = (size_t)W * H;
    return sizeof(SnapHeader) + N * 8 * 2 + N * 4 + N + (size_t)n_err * 4;
}

// kernels + list slice of one launch group
struct Group {
    int key_n = 0;            // image side of the class
    bool pipelined = false;
    RowKernels rk{};
    ColKernels ck{};
    size_t smem = 0, smem_fin = 0;
    std::vector<WorkItem> items;   // sorted by job n_hio, descending
    std::vector<int> hio_count;    // items whose job runs iteration i
    int list_base = 0;             // index of this group's first WorkList header
};

// The jobs of one (row kernel, column kernel) class: their whole cycle --
// finish, vertical blur, every row and column pass -- depends on nothing
// outside the class, so in the chained schedule each class is one branch of
// the step graph and the classes run concurrently.
struct Chain {
    Group row, col;
    std::vector<WorkItem> vb;
    int vb_base = 0;
};
constexpr int kBranchStreams = 16;

// Step configurations the tuner compares on real steps (all give the same
// bits): the schedule, and the persistent grids at 100 % or 50 % of the
// occupancy limit (fewer, longer-running CTAs overlap more copy with compute
// when a class has few items per CTA).
struct TuneCfg {
    int schedule, grid_pct;
};
constexpr TuneCfg kTuneCands[] = {{0, 100}, {1, 100}, {0, 50}, {1, 50}};
constexpr int kTuneN = 4;

}  // namespace imr

using namespace imr;

struct imr_engine {
    int dev = 0;
    cudaStream_t s = nullptr;       // the caller's stream: every engine operation is ordered on it
    cudaStream_t cs = nullptr;      // private stream the step graph is captured on
    cudaMemPool_t pool = nullptr;   // the engine's own pool: freed arenas stay cached for new admissions
    size_t budget = 0, used = 0, peak = 0;
    int max_slots = 0;
    JobDev *dj = nullptr;           // [max_slots]
    JobState *dst = nullptr;        // [max_slots]
    JobState *hst[2] = {nullptr, nullptr};   // pinned copies of dst after steps of each parity
    cudaEvent_t ev_st[2] = {nullptr, nullptr};
    long st_step[2] = {-1, -1};     // the step whose state copy each of them receives
    long synced_step = -1;          // last step whose state copy the host has acted on
    std::vector<int> free_slots;
    std::deque<EJob *> pending;
    std::vector<EJob *> active;
    std::vector<EJob *> retiring;   // finished on the device, result copy in flight
    std::deque<EJob *> done;
    std::vector<Staging> staging;
    StageGrower grower;
    // work lists: device buffers and two pinned staging copies (alternating per rebuild)
    WorkItem *d_items = nullptr;
    size_t items_cap = 0;
    WorkList *d_lists = nullptr;
    size_t lists_cap = 0;
    WorkItem *h_items[2] = {nullptr, nullptr};
    WorkList *h_lists[2] = {nullptr, nullptr};
    size_t h_items_cap[2] = {0, 0}, h_lists_cap[2] = {0, 0};
    cudaEvent_t ev_lists[2] = {nullptr, nullptr};
    int lists_parity = 0;
    // the step graph over the active set
    bool dirty = true;
    std::vector<EJob *> fresh;      // admitted since the last step: column init before the next graph
    std::vector<Group> init_groups;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    long kernels_per_step = 0;
    long launches = 0;              // kernels run (graph kernels count once per step)
    long host_launches = 0;         // launch calls issued by the host (a graph launch counts once)
    long graph_builds = 0, graph_updates = 0;
    long steps = 0;
    int sms = 148;
    int schedule = 0;                 // IMR_SCHEDULE_GROUPED / IMR_SCHEDULE_CHAINED
    int grid_pct = 100;               // persistent grids at this % of the occupancy limit
    int cycles_per_step = 1;          // shrink-wrap cycles captured into one step's graph
    // online tuner: per admitted-set signature, run each candidate for one
    // step, time it on the device, keep the fastest (ms per resident pixel)
    bool tune = false;
    std::string tune_path;            // cache file ("": memory only)
    std::map<std::string, TuneCfg> tune_cache;
    std::string tune_sig;             // signature of the set being run
    int tune_next = -1;               // next candidate to launch (-1: settled)
    long tune_step[kTuneN] = {};      // the step each candidate ran at
    double tune_ms[kTuneN] = {};      // its measured ms per pixel (0: not yet)
    long tune_explored = 0, tune_hits = 0;
    cudaStream_t bs[kBranchStreams] = {};
    cudaEvent_t ev_fork = nullptr, ev_join[kBranchStreams] = {};
    int inject_alloc_fail = 0;      // the next admissions whose allocation is made to fail
    long alloc_failures = 0;
    size_t reserved = 0;            // bytes the engine's pool has been grown to
    size_t max_active_px = 0;       // bound on the pixels of the resident requests (0: none)
    size_t active_px = 0;
    // admission by measured step time: every step's graph is timed on the
    // device; ms_per_px follows step ms / resident pixels (EWMA), and with a
    // target step time the resident pixels are held to target / ms_per_px
    double target_step_ms = 0.0;
    double ms_per_px = 0.0;
    cudaEvent_t ev_t0[2] = {nullptr, nullptr}, ev_t1[2] = {nullptr, nullptr};
    size_t step_px[2] = {0, 0};
    double step_launch_ms[2] = {0.0, 0.0};   // host time of the step's graph launch call
    double last_step_ms = 0.0;
    double device_ms = 0.0;           // device time of all observed steps
};

#define CKE(call)                      \
    do {                               \
        cudaError_t e_ = (call);       \
        if (e_ != cudaSuccess) {       \
            set_error(#call, e_);      \
            return IMR_ERR_CUDA;       \
        }                              \
    } while (0)

static int grow(imr_engine *E, size_t n_items, size_t n_lists)
{
    if (n_items > E->items_cap || n_lists > E->lists_cap) {
        // queued steps may still read the old lists
        CKE(cudaStreamSynchronize(E->s));
    }
    if (n_items > E->items_cap) {
        size_t cap = std::max(n_items, E->items_cap * 2 + 1024);
        if (E->d_items) cudaFree(E->d_items);
        E->d_items = nullptr;
        CKE(cudaMalloc(&E->d_items, cap * sizeof(WorkItem)));
        E->items_cap = cap;
    }
    if (n_lists > E->lists_cap) {
        size_t cap = std::max(n_lists, E->lists_cap * 2 + 256);
        if (E->d_lists) cudaFree(E->d_lists);
        E->d_lists = nullptr;
        CKE(cudaMalloc(&E->d_lists, cap * sizeof(WorkList)));
        E->lists_cap = cap;
    }
    const int q = E->lists_parity;
    // the staging copy of this parity was last uploaded two rebuilds ago
    CKE(cudaEventSynchronize(E->ev_lists[q]));
    if (n_items > E->h_items_cap[q]) {
        if (E->h_items[q]) cudaFreeHost(E->h_items[q]);
        E->h_items[q] = nullptr;
        const size_t cap = std::max(n_items, E->h_items_cap[q] * 2 + 1024);
        CKE(cudaMallocHost(&E->h_items[q], cap * sizeof(WorkItem)));
        E->h_items_cap[q] = cap;
    }
    if (n_lists > E->h_lists_cap[q]) {
        if (E->h_lists[q]) cudaFreeHost(E->h_lists[q]);
        E->h_lists[q] = nullptr;
        const size_t cap = std::max(n_lists, E->h_lists_cap[q] * 2 + 256);
        CKE(cudaMallocHost(&E->h_lists[q], cap * sizeof(WorkList)));
        E->h_lists_cap[q] = cap;
    }
    return IMR_SUCCESS;
}

// Loop-kernel grid: enough CTAs to fill the GPU, never more than the items.
static int loop_grid(const imr_engine *E, int items) { return std::max(1, std::min(items, E->sms * 16)); }

static void finish_now(imr_engine *E, EJob *j, int status)
{
    j->status = status;
    j->t_done = now_ms();
    E->done.push_back(j);
}

// Grow the pool's reserve in one piece before a batch of admissions: the
// pool keeps what it is given (release threshold: never), so the arenas of
// the batch are then carved from memory it already holds instead of each
// admission growing the pool on its own (one driver mapping per arena cost
// 0.2-0.7 s for 512 admissions).
static void reserve_for(imr_engine *E)
{
    size_t want = 0, px = E->active_px;
    int slots = (int)E->free_slots.size();
    bool idle = E->active.empty() && E->fresh.empty();
    for (EJob *j : E->pending) {   // the requests admit() is about to take, by the same tests
        if (slots == 0) break;
        const size_t jp = (size_t)j->W * j->H;
        if (E->used + want + j->S.bytes > E->budget && !idle) break;
        if (E->max_active_px && px + jp > E->max_active_px && !idle) break;
        if (E->target_step_ms > 0 && E->ms_per_px > 0 && (double)(px + jp) * E->ms_per_px > E->target_step_ms &&
            !idle)
            break;
        want += (j->S.bytes + 511) / 512 * 512;
        px += jp;
        --slots;
        idle = false;
    }
    if (want == 0 || E->used + want <= E->reserved) return;
    const size_t grow = E->used + want - E->reserved;
    if (E->inject_alloc_fail > 0) return;   // the injected failures are the admissions' own
    void *tmp = nullptr;
    if (cudaMallocFromPoolAsync(&tmp, grow, E->pool, E->s) == cudaSuccess) {
        cudaFreeAsync(tmp, E->s);
        E->reserved += grow;
    } else {
        cudaGetLastError();   // not fatal: each admission then allocates (and may fail) on its own
    }
}

// The modulus of a request submitted as a measured intensity: M = sqrt(I),
// correctly rounded (sqrtf), in place.
static __global__ void k_sqrt_inplace(float *v, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        v[i] = sqrtf(v[i]);
}

static int admit(imr_engine *E)
{
    reserve_for(E);
    while (!E->pending.empty() && !E->free_slots.empty()) {
        EJob *j = E->pending.front();
        const bool idle = E->active.empty() && E->fresh.empty();
        if (E->used + j->S.bytes > E->budget && !idle) break;
        const size_t px = (size_t)j->W * j->H;
        if (E->max_active_px && E->active_px + px > E->max_active_px && !idle) break;
        if (E->target_step_ms > 0 && E->ms_per_px > 0 &&
            (double)(E->active_px + px) * E->ms_per_px > E->target_step_ms && !idle)
            break;
        E->pending.pop_front();
        j->slot = E->free_slots.back();
        E->free_slots.pop_back();
        cudaError_t e;
        if (E->inject_alloc_fail > 0) {   // host-side fault injection: this allocation fails
            --E->inject_alloc_fail;
            e = cudaErrorMemoryAllocation;
        } else {
            e = cudaMallocFromPoolAsync((void **)&j->arena, j->S.bytes, E->pool, E->s);
        }
        if (e != cudaSuccess) {
            ++E->alloc_failures;
            cudaGetLastError();
            E->free_slots.push_back(j->slot);
            j->slot = -1;
            j->arena = nullptr;
            if (idle && E->retiring.empty()) {
                // nothing running will free memory: the request cannot be served
                snprintf(g_last_error, sizeof(g_last_error), "engine: %zu device bytes for a %ux%u request not available",
                         j->S.bytes, j->W, j->H);
                finish_now(E, j, IMR_ERR_OUT_OF_MEMORY);
                continue;
            }
            E->pending.push_front(j);   // retry once a running reconstruction has retired
            break;
        }
        E->used += j->S.bytes;
        E->peak = std::max(E->peak, E->used);
        E->active_px += px;
        job_bind(j->J, j->S, j->arena, E->dst + j->slot);
        int rc = job_upload(j->J, j->S, j->arena, E->dj + j->slot, E->s);
        if (rc) return rc;
        if (j->resume.empty()) {
            CKE(cudaMemsetAsync(E->dst + j->slot, 0, sizeof(JobState), E->s));
            CKE(cudaMemcpyAsync((void *)j->J.M, j->h_in, (size_t)j->W * j->H * 4, cudaMemcpyHostToDevice, E->s));
            if (j->intensity) {
                const size_t n = (size_t)j->W * j->H;
                k_sqrt_inplace<<<(unsigned)std::min<size_t>((n + 255) / 256, (size_t)E->sms * 8), 256, 0, E->s>>>(
                    const_cast<float *>(j->J.M), n);
                CKE(cudaGetLastError());
                ++E->launches;
                ++E->host_launches;
            }
            if ((rc = job_modulus_tiles(j->J, E->s))) return rc;
            if (j->J.Mt) {
                ++E->launches;
                ++E->host_launches;
            }
            E->fresh.push_back(j);
        } else {   // continue a suspended reconstruction where it stopped
            const SnapHeader *h = (const SnapHeader *)j->resume.data();
            const size_t N = (size_t)j->W * j->H;
            const char *d = j->resume.data() + sizeof(SnapHeader);
            // on the engine's stream, after job_upload's clearing of the mask and
            // errors; synchronised below before the snapshot buffer is released
            CKE(cudaMemcpyAsync(E->dst + j->slot, &h->st, sizeof(JobState), cudaMemcpyHostToDevice, E->s));
            CKE(cudaMemcpyAsync(j->J.X, d, N * 8, cudaMemcpyHostToDevice, E->s));
            CKE(cudaMemcpyAsync(j->J.G, d + N * 8, N * 8, cudaMemcpyHostToDevice, E->s));
            CKE(cudaMemcpyAsync((void *)j->J.M, d + N * 16, N * 4, cudaMemcpyHostToDevice, E->s));
            if ((rc = job_modulus_tiles(j->J, E->s))) return rc;
            if (j->J.Mt) {
                ++E->launches;
                ++E->host_launches;
            }
            CKE(cudaMemcpyAsync(j->J.mask, d + N * 20, N, cudaMemcpyHostToDevice, E->s));
            CKE(cudaMemcpyAsync(j->J.errors, d + N * 21, (size_t)h->n_err * 4, cudaMemcpyHostToDevice, E->s));
            CKE(cudaStreamSynchronize(E->s));
            j->cycles_launched = h->st.cycle;   // the cycle it continues with
            std::vector<char>().swap(j->resume);
        }
        j->admit_step = E->steps;   // the slot's previous state is in every older state copy
        E->active.push_back(j);
        E->dirty = true;
    }
    return IMR_SUCCESS;
}

// Group jobs by the kernels they run (rows: by width class, columns: by
// height class and pipelining), so all jobs that share a kernel share its
// launches -- e.g. every Bluestein width with the same work length.  Items
// are sorted by the job's HIO count so iteration i runs a prefix of the list.
static void build_groups(const std::vector<EJob *> &jobs, bool rows, std::vector<Group> &out)
{
    std::map<std::pair<const void *, int>, std::vector<EJob *>> by;
    for (EJob *j : jobs) {
        const void *key = rows ? (const void *)j->S.rk.hio : (j->S.p_cols ? (const void *)j->S.ck.p_col
                                                                           : (const void *)j->S.ck.col);
        const int pl = rows ? (j->S.p_rows ? 1 : 0) : (j->S.p_cols ? 1 : 0);
        by[{key, pl}].push_back(j);
    }
    out.clear();
    for (auto &kv : by) {
        Group g;
        auto &v = kv.second;
        std::stable_sort(v.begin(), v.end(), [](EJob *a, EJob *b) { return a->J.n_hio > b->J.n_hio; });
        const EJob *j0 = v.front();
        g.key_n = rows ? (int)j0->W : (int)j0->H;
        g.pipelined = kv.first.second != 0;
        g.rk = j0->S.rk;
        g.ck = j0->S.ck;
        int max_hio = 0;
        for (EJob *j : v) {
            g.smem = std::max(g.smem, rows ? j->S.smem_row : j->S.smem_col);
            g.smem_fin = std::max(g.smem_fin, j->S.smem_fin);
            const int nt = rows ? j->J.n_row_tiles : j->J.n_col_tiles;
            for (int t = 0; t < nt; ++t) g.items.push_back(WorkItem{j->slot, t});
            max_hio = std::max(max_hio, j->J.n_hio);
        }
        g.hio_count.assign(max_hio, 0);
        for (EJob *j : v) {
            const int nt = rows ? j->J.n_row_tiles : j->J.n_col_tiles;
            for (int i = 0; i < j->J.n_hio; ++i) g.hio_count[i] += nt;
        }
        out.push_back(std::move(g));
    }
}

// The launches of one cycle of every job in the groups, on stream s (a
// capturing stream when the step graph is built).  Returns the kernel count.
static int launch_cycle(imr_engine *E, cudaStream_t s, const WorkList *L, std::vector<Group> &rowg,
                        std::vector<Group> &colg, int vb_base, size_t n_vb, long *kernels)
{
    long k = 0;
    int rc;
    for (auto &g : rowg) {
        if (g.pipelined) {
            if ((rc = launch_finish(g.rk, (int)g.items.size(), g.smem_fin, s, E->dj, L + g.list_base, nullptr,
                                    E->grid_pct)))
                return rc;
        } else {
            g.rk.finish<<<loop_grid(E, (int)g.items.size()), g.rk.threads, g.smem_fin, s>>>(E->dj, L + g.list_base,
                                                                                         nullptr);
        }
        ++k;
    }
    if (n_vb) {
        k_vblur<<<loop_grid(E, (int)n_vb), kVbThreads, 0, s>>>(E->dj, L + vb_base);
        ++k;
    }
    int max_hio = 0;
    for (auto &g : rowg) max_hio = std::max(max_hio, (int)g.hio_count.size());
    for (int i = 0; i < max_hio; ++i) {
        for (auto &g : rowg) {
            if (i >= (int)g.hio_count.size()) continue;
            const WorkList *Li = L + g.list_base + 1 + i;
            const int n = g.hio_count[i];
            if (g.pipelined) {
                auto kf = i == 0 ? g.rk.p_hio_first : g.rk.p_hio;
                const int sm = i == 0 ? g.rk.p_smem_first : g.rk.p_smem;
                kf<<<scaled_grid((const void *)kf, g.rk.threads, sm, n, E->grid_pct), g.rk.threads, sm, s>>>(E->dj,
                                                                                                          Li);
            } else {
                (i == 0 ? g.rk.hio_first : g.rk.hio)<<<loop_grid(E, n), g.rk.threads, g.smem, s>>>(E->dj, Li);
            }
            ++k;
        }
        for (auto &g : colg) {
            if (i >= (int)g.hio_count.size()) continue;
            const WorkList *Li = L + g.list_base + 1 + i;
            const int n = g.hio_count[i];
            if (g.pipelined)
                g.ck.p_col<<<scaled_grid((const void *)g.ck.p_col, g.ck.p_threads, g.ck.p_smem, n, E->grid_pct),
                             g.ck.p_threads, g.ck.p_smem, s>>>(E->dj, Li);
            else
                g.ck.col<<<loop_grid(E, n), g.ck.threads, g.smem, s>>>(E->dj, Li);
            ++k;
        }
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("engine kernel launch", e);
        return IMR_ERR_CUDA;
    }
    *kernels = k;
    return IMR_SUCCESS;
}

static void build_chains(const std::vector<EJob *> &jobs, std::vector<Chain> &out)
{
    std::map<std::tuple<const void *, int, const void *, int>, std::vector<EJob *>> by;
    for (EJob *j : jobs) {
        const void *ck = j->S.p_cols ? (const void *)j->S.ck.p_col : (const void *)j->S.ck.col;
        by[std::make_tuple((const void *)j->S.rk.hio, j->S.p_rows ? 1 : 0, ck, j->S.p_cols ? 1 : 0)].push_back(j);
    }
    out.clear();
    for (auto &kv : by) {
        Chain c;
        std::vector<Group> g;
        build_groups(kv.second, true, g);
        c.row = std::move(g[0]);
        build_groups(kv.second, false, g);
        c.col = std::move(g[0]);
        for (EJob *j : kv.second)
            for (int t = 0; t < j->J.n_vb_tiles; ++t) c.vb.push_back(WorkItem{j->slot, t});
        out.push_back(std::move(c));
    }
}

// One cycle of the jobs of one chain, on stream s.
static int launch_chain(imr_engine *E, cudaStream_t s, const WorkList *L, Chain &c, long *kernels)
{
    std::vector<Group> rg(1), cg(1);
    rg[0] = c.row;
    cg[0] = c.col;
    long k = 0;
    const int rc = launch_cycle(E, s, L, rg, cg, c.vb_base, c.vb.size(), &k);
    *kernels += k;
    return rc;
}

// ---- online tuner ----------------------------------------------------------
// Signature of the admitted set: its kernel classes (row length, column
// length, pipelined or not) with their job counts.
static std::string set_signature(const std::vector<EJob *> &jobs)
{
    std::map<std::tuple<int, int, int, int>, int> n;
    for (EJob *j : jobs) ++n[std::make_tuple((int)j->W, (int)j->H, j->S.p_rows ? 1 : 0, j->S.p_cols ? 1 : 0)];
    std::string sig;
    char buf[64];
    for (auto &kv : n) {
        snprintf(buf, sizeof(buf), "%dx%d%c%c*%d;", std::get<0>(kv.first), std::get<1>(kv.first),
                 std::get<2>(kv.first) ? 'p' : 't', std::get<3>(kv.first) ? 'p' : 't', kv.second);
        sig += buf;
    }
    return sig;
}

static void tune_load(imr_engine *E)
{
    E->tune_cache.clear();
    if (E->tune_path.empty()) return;
    FILE *f = fopen(E->tune_path.c_str(), "r");
    if (!f) return;
    char line[8192];
    while (fgets(line, sizeof(line), f)) {
        char *tab = strchr(line, '\t');
        if (!tab) continue;
        *tab = 0;
        int sched = 0, pct = 100;
        if (sscanf(tab + 1, "%d %d", &sched, &pct) == 2 && (sched == 0 || sched == 1) && pct > 0 && pct <= 100)
            E->tune_cache[line] = TuneCfg{sched, pct};
    }
    fclose(f);
}

static void tune_store(imr_engine *E, const std::string &sig, const TuneCfg &c, double ms_per_mpx)
{
    E->tune_cache[sig] = c;
    if (E->tune_path.empty()) return;
    FILE *f = fopen(E->tune_path.c_str(), "a");
    if (!f) return;
    fprintf(f, "%s\t%d %d %.6f\n", sig.c_str(), c.schedule, c.grid_pct, ms_per_mpx);
    fclose(f);
}

// Before a rebuild: a new set starts its exploration (or takes its cached
// configuration); during exploration each candidate runs for kTuneRuns steps
// and the last of them is timed (the first launch of a new graph carries
// one-time costs).
constexpr int kTuneRuns = 2;

static void tune_before_step(imr_engine *E)
{
    if (!E->tune || E->active.empty()) return;
    const std::string sig = set_signature(E->active);
    if (sig != E->tune_sig) {
        E->tune_sig = sig;
        auto it = E->tune_cache.find(sig);
        if (it != E->tune_cache.end()) {
            E->tune_next = -1;
            ++E->tune_hits;
            if (E->schedule != it->second.schedule || E->grid_pct != it->second.grid_pct) E->dirty = true;
            E->schedule = it->second.schedule;
            E->grid_pct = it->second.grid_pct;
            return;
        }
        E->tune_next = 0;
        for (int c = 0; c < kTuneN; ++c) {
            E->tune_step[c] = -1;
            E->tune_ms[c] = 0.0;
        }
    }
    if (E->tune_next >= 0 && E->tune_next < kTuneN * kTuneRuns) {
        const TuneCfg &c = kTuneCands[E->tune_next / kTuneRuns];
        if (E->schedule != c.schedule || E->grid_pct != c.grid_pct) E->dirty = true;
        E->schedule = c.schedule;
        E->grid_pct = c.grid_pct;
    }
}

// After the launch of step n: note which candidate it ran.
static void tune_after_launch(imr_engine *E, long n)
{
    if (!E->tune || E->tune_next < 0 || E->tune_next >= kTuneN * kTuneRuns) return;
    if (E->tune_next % kTuneRuns == kTuneRuns - 1) E->tune_step[E->tune_next / kTuneRuns] = n;
    ++E->tune_next;
    ++E->tune_explored;
}

// When the device time of step m is known: record it; once every candidate
// is timed, keep the fastest.
static void tune_observe(imr_engine *E, long m, double ms_per_px)
{
    if (!E->tune || E->tune_next < 0) return;
    for (int c = 0; c < kTuneN; ++c)
        if (E->tune_step[c] == m) E->tune_ms[c] = ms_per_px;
    for (int c = 0; c < kTuneN; ++c)
        if (!(E->tune_ms[c] > 0)) return;
    int best = 0;
    for (int c = 1; c < kTuneN; ++c)
        if (E->tune_ms[c] < E->tune_ms[best]) best = c;
    E->tune_next = -1;
    tune_store(E, E->tune_sig, kTuneCands[best], E->tune_ms[best] * 1e6);
    if (E->schedule != kTuneCands[best].schedule || E->grid_pct != kTuneCands[best].grid_pct) E->dirty = true;
    E->schedule = kTuneCands[best].schedule;
    E->grid_pct = kTuneCands[best].grid_pct;
}

// Rebuild the work lists of the active set and the newly admitted jobs'
// column init, upload them (stream-ordered after the queued steps, which
// still read the previous lists), and re-capture the step graph.
static int rebuild(imr_engine *E)
{
    std::vector<Group> rowg, colg;
    std::vector<Chain> chains;
    std::vector<WorkItem> vb;
    build_groups(E->fresh, false, E->init_groups);
    const bool chained = E->schedule == IMR_SCHEDULE_CHAINED;
    if (chained) {
        build_chains(E->active, chains);
    } else {
        build_groups(E->active, true, rowg);
        build_groups(E->active, false, colg);
        for (EJob *j : E->active)
            for (int t = 0; t < j->J.n_vb_tiles; ++t) vb.push_back(WorkItem{j->slot, t});
    }
    size_t n_items = vb.size(), n_lists = 1;
    for (auto *G : {&E->init_groups, &rowg, &colg})
        for (auto &g : *G) {
            n_items += g.items.size();
            n_lists += 1 + g.hio_count.size();
        }
    for (auto &c : chains) {
        n_items += c.vb.size() + c.row.items.size() + c.col.items.size();
        n_lists += 3 + c.row.hio_count.size() + c.col.hio_count.size();
    }
    int rc = grow(E, n_items, n_lists);
    if (rc) return rc;
    const int q = E->lists_parity;
    WorkItem *hi = E->h_items[q];
    WorkList *hl = E->h_lists[q];
    size_t ip = 0, lp = 0;
    auto put = [&](const std::vector<WorkItem> &items, const std::vector<int> &counts, int &base) {
        const WorkItem *dptr = E->d_items + ip;
        if (!items.empty()) memcpy(hi + ip, items.data(), items.size() * sizeof(WorkItem));
        base = (int)lp;
        hl[lp++] = WorkList{dptr, (int)items.size()};
        for (int c : counts) hl[lp++] = WorkList{dptr, c};
        ip += items.size();
    };
    int vb_base = 0;
    put(vb, {}, vb_base);
    for (auto *G : {&E->init_groups, &rowg, &colg})
        for (auto &g : *G) put(g.items, g.hio_count, g.list_base);
    for (auto &c : chains) {
        put(c.vb, {}, c.vb_base);
        put(c.row.items, c.row.hio_count, c.row.list_base);
        put(c.col.items, c.col.hio_count, c.col.list_base);
    }
    if (ip) CKE(cudaMemcpyAsync(E->d_items, hi, ip * sizeof(WorkItem), cudaMemcpyHostToDevice, E->s));
    CKE(cudaMemcpyAsync(E->d_lists, hl, lp * sizeof(WorkList), cudaMemcpyHostToDevice, E->s));
    CKE(cudaEventRecord(E->ev_lists[q], E->s));
    E->lists_parity ^= 1;

    // capture one cycle of every active job
    cudaGraph_t g = nullptr;
    long kernels = 0;
    CKE(cudaStreamBeginCapture(E->cs, cudaStreamCaptureModeThreadLocal));
    if (!chained) {
        for (int c = 0; c < E->cycles_per_step && rc == IMR_SUCCESS; ++c)
            rc = launch_cycle(E, E->cs, E->d_lists, rowg, colg, vb_base, vb.size(), &kernels);
    } else {
        // one branch per chain (chains beyond the branch streams share them in turn)
        cudaError_t e = cudaEventRecord(E->ev_fork, E->cs);
        const int nb = std::min((int)chains.size(), kBranchStreams);
        for (int b = 0; b < nb && e == cudaSuccess; ++b) e = cudaStreamWaitEvent(E->bs[b], E->ev_fork, 0);
        for (size_t c = 0; c < chains.size() && e == cudaSuccess && rc == IMR_SUCCESS; ++c)
            for (int k = 0; k < E->cycles_per_step && rc == IMR_SUCCESS; ++k)
                rc = launch_chain(E, E->bs[c % kBranchStreams], E->d_lists, chains[c], &kernels);
        for (int b = 0; b < nb && e == cudaSuccess; ++b) {
            e = cudaEventRecord(E->ev_join[b], E->bs[b]);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(E->cs, E->ev_join[b], 0);
        }
        if (e != cudaSuccess && rc == IMR_SUCCESS) {
            set_error("engine step graph branches", e);
            rc = IMR_ERR_CUDA;
        }
    }
    const cudaError_t ec = cudaStreamEndCapture(E->cs, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    CKE(ec);
    bool updated = false;
    if (E->gexec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(E->gexec, g, &info) == cudaSuccess) {
            updated = true;
        } else {
            cudaGetLastError();
            cudaGraphExecDestroy(E->gexec);
            E->gexec = nullptr;
        }
    }
    if (!updated) {
        const cudaError_t e = cudaGraphInstantiate(&E->gexec, g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            set_error("engine step graph", e);
            return IMR_ERR_CUDA;
        }
    }
    // upload now, so the first launch of the new graph does not carry it
    CKE(cudaGraphUpload(E->gexec, E->s));
    if (E->graph) cudaGraphDestroy(E->graph);
    E->graph = g;
    E->kernels_per_step = kernels;
    ++(updated ? E->graph_updates : E->graph_builds);
    E->dirty = false;
    return IMR_SUCCESS;
}

static void grower_main(imr_engine *E);

// Ask the helper for staging room for the results of every resident request
// (at most kStageMax), starting it on first use.
static void stage_request(imr_engine *E)
{
    size_t want = 0, big = kStageChunk;
    for (EJob *j : E->active) {
        const size_t b = ((size_t)j->W * j->H * 4 + 255) / 256 * 256;
        want += b;
        big = std::max(big, b);
    }
    want = std::min(want, kStageMax);
    StageGrower &g = E->grower;
    {
        std::lock_guard<std::mutex> lk(g.mu);
        if (g.failed) return;
        g.want = std::max(g.want, want);
        g.min_chunk = std::max(g.min_chunk, big);
        if (g.have >= g.want) return;
        g.credit = 1;
    }
    if (!g.th.joinable()) {
        try {
            g.th = std::thread(grower_main, E);
        } catch (...) {   // no thread: staging is allocated on demand, as without the helper
            std::lock_guard<std::mutex> lk(g.mu);
            g.failed = true;
            return;
        }
    }
    g.cv.notify_one();
}

static void grower_main(imr_engine *E)
{
    StageGrower &g = E->grower;
    cudaSetDevice(E->dev);
    std::unique_lock<std::mutex> lk(g.mu);
    for (;;) {
        g.cv.wait(lk, [&] { return g.stop || (g.credit > 0 && g.have < g.want); });
        if (g.stop) return;
        --g.credit;
        const size_t cap = g.min_chunk;
        lk.unlock();
        Staging st;
        const bool ok = cudaMallocHost(&st.p, cap) == cudaSuccess;
        if (!ok) cudaGetLastError();
        lk.lock();
        if (!ok) {   // pinned memory exhausted: the engine allocates on demand from now on
            g.failed = true;
            g.want = g.have;
            continue;
        }
        st.cap = cap;
        g.ready.push_back(st);
        g.have += cap;
    }
}

// Take over the chunks the helper has pinned.
static void stage_adopt(imr_engine *E)
{
    StageGrower &g = E->grower;
    std::lock_guard<std::mutex> lk(g.mu);
    for (Staging &st : g.ready) E->staging.push_back(st);
    g.ready.clear();
}

// A place for one result of `bytes` in the staging: after the results
// already in a chunk, in an empty chunk, or in a new chunk allocated here
// when the helper has not caught up.  Returns the chunk (-2: no pinned memory).
static int stage_place(imr_engine *E, size_t bytes, size_t *off)
{
    for (size_t i = 0; i < E->staging.size(); ++i) {
        Staging &st = E->staging[i];
        if (st.busy == 0) st.used = 0;
        if (st.cap - st.used >= bytes) {
            *off = st.used;
            st.used += bytes;
            return (int)i;
        }
    }
    Staging st;
    const size_t cap = std::max(bytes, kStageChunk);
    if (cudaMallocHost(&st.p, cap) != cudaSuccess) {
        cudaGetLastError();
        return -2;
    }
    st.cap = cap;
    st.used = bytes;
    *off = 0;
    E->staging.push_back(st);
    return (int)E->staging.size() - 1;
}

// Copy finished results from the staging into the callers' buffers; a large
// hand-over runs on several threads (first writes to fresh pageable buffers
// fault their pages in, which one thread does at a few GB/s).
struct HandOver {
    void *dst;
    const void *src;
    size_t bytes;
};
static void hand_over(std::vector<HandOver> &h)
{
    size_t total = 0;
    for (const HandOver &x : h) total += x.bytes;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t nt = std::min<size_t>({(size_t)8, (size_t)hw, h.size(), total / ((size_t)4 << 20) + 1});
    if (nt <= 1) {
        for (const HandOver &x : h) memcpy(x.dst, x.src, x.bytes);
        return;
    }
    // thread t copies results t, t + nt, ...; results of threads that could not
    // be started are copied here
    std::vector<std::thread> th;
    size_t started = 0;
    for (size_t t = 0; t < nt; ++t) {
        try {
            th.emplace_back([&h, t, nt] {
                for (size_t i = t; i < h.size(); i += nt) memcpy(h[i].dst, h[i].src, h[i].bytes);
            });
            ++started;
        } catch (...) {
            break;
        }
    }
    for (size_t t = started; t < nt; ++t)
        for (size_t i = t; i < h.size(); i += nt) memcpy(h[i].dst, h[i].src, h[i].bytes);
    for (auto &x : th) x.join();
}

// Retire the jobs that had stopped (or failed) by the end of step m, whose
// states are in hst: copy their results out (stream-ordered, before the next
// step), release their device memory and slots.
static int observe(imr_engine *E, const JobState *hs, long m)
{
    E->synced_step = m;
    if (hs && m >= 0) {   // the device time of step m (its events completed before its state copy)
        const int q = (int)(m & 1);
        float ms = 0.f;
        if (E->step_px[q] && cudaEventElapsedTime(&ms, E->ev_t0[q], E->ev_t1[q]) == cudaSuccess) {
            E->last_step_ms = ms;
            E->device_ms += ms;
            const double r = ms / (double)E->step_px[q];
            E->ms_per_px = E->ms_per_px > 0 ? 0.8 * E->ms_per_px + 0.2 * r : r;
            // the tuner weighs a configuration by the device time plus the host
            // time its graph launch takes (a larger graph costs the host more)
            tune_observe(E, m, (ms + E->step_launch_ms[q]) / (double)E->step_px[q]);
        }
        cudaGetLastError();
    }
    // result copies issued before step m's state copy are complete
    std::vector<HandOver> ho;
    std::vector<EJob *> handed, still;
    for (EJob *j : E->retiring) {
        if (j->copy_step >= 0 && j->copy_step <= m) {
            if (j->staging >= 0)
                ho.push_back(HandOver{j->h_out, E->staging[j->staging].p + j->staging_off, (size_t)j->W * j->H * 4});
            handed.push_back(j);
        } else {
            still.push_back(j);
        }
    }
    if (!ho.empty()) hand_over(ho);
    for (EJob *j : handed) {
        if (j->staging >= 0) --E->staging[j->staging].busy;
        finish_now(E, j, j->status);
    }
    E->retiring.swap(still);
    if (!hs) return IMR_SUCCESS;
    std::vector<EJob *> keep, out;
    for (EJob *j : E->active) {
        const JobState &st = hs[j->slot];
        if (m < j->admit_step || !(st.stop || st.err)) {
            keep.push_back(j);
            continue;
        }
        j->cycles_done = st.cycles_done;
        j->last_error = st.last_error;
        j->status = st.err ? IMR_ERR_DEVICE_TIMEOUT : IMR_SUCCESS;
        cudaPointerAttributes pa;
        const bool pinned = cudaPointerGetAttributes(&pa, j->h_out) == cudaSuccess &&
                            (pa.type == cudaMemoryTypeHost || pa.type == cudaMemoryTypeManaged);
        cudaGetLastError();
        j->staging = pinned ? -1 : 0;
        out.push_back(j);
    }
    if (out.empty()) return IMR_SUCCESS;
    stage_adopt(E);
    // places first (a chunk holding a result is busy, so the next result goes
    // after it), all or none
    for (size_t k = 0; k < out.size(); ++k) {
        EJob *j = out[k];
        if (j->staging < 0) continue;
        const size_t b = ((size_t)j->W * j->H * 4 + 255) / 256 * 256;
        const int chunk = stage_place(E, b, &j->staging_off);
        if (chunk == -2) {
            for (size_t u = 0; u < k; ++u)
                if (out[u]->staging >= 0) --E->staging[out[u]->staging].busy;
            set_error("engine result staging", cudaErrorMemoryAllocation);
            return IMR_ERR_OUT_OF_MEMORY;
        }
        j->staging = chunk;
        ++E->staging[chunk].busy;
    }
    for (EJob *j : out) {
        const size_t b = (size_t)j->W * j->H * 4;
        void *dst = j->h_out;
        if (j->staging >= 0) dst = E->staging[j->staging].p + j->staging_off;
        CKE(cudaMemcpyAsync(dst, j->J.out, b, cudaMemcpyDeviceToHost, E->s));
        CKE(cudaFreeAsync(j->arena, E->s));
        j->arena = nullptr;
        j->copy_step = E->steps;   // the copy precedes the state copy of the next step launched
        E->used -= j->S.bytes;
        E->active_px -= (size_t)j->W * j->H;
        E->free_slots.push_back(j->slot);
        E->retiring.push_back(j);
        E->dirty = true;
    }
    E->active.swap(keep);
    return IMR_SUCCESS;
}

// Act on the newest state copy that has already landed, without waiting
// (imr_engine_poll between steps).
static int reap(imr_engine *E)
{
    for (int pass = 0; pass < 2; ++pass) {
        int q = E->st_step[0] < E->st_step[1] ? 0 : 1;   // older first
        if (pass == 1) q ^= 1;
        const long m = E->st_step[q];
        if (m <= E->synced_step) continue;
        const cudaError_t e = cudaEventQuery(E->ev_st[q]);
        if (e == cudaErrorNotReady) break;
        CKE(e);
        if (int rc = observe(E, E->hst[q], m)) return rc;
    }
    return IMR_SUCCESS;
}

// Wait for everything queued and hand every retiring result to the caller.
static int drain(imr_engine *E)
{
    CKE(cudaStreamSynchronize(E->s));
    return observe(E, nullptr, E->steps);
}

static EJob *find_active(imr_engine *E, long long tag)
{
    for (EJob *j : E->active)
        if (j->tag == tag) return j;
    return nullptr;
}

extern "C" {

int imr_engine_create(imr_engine **out, size_t device_bytes, int max_jobs, void *stream)
{
    if (!out || max_jobs < 1) return IMR_ERR_INVALID_VALUE;
    *out = nullptr;
    int rc = ensure_kernel_attributes();
    if (rc) return rc;
    imr_engine *E = new imr_engine();
    cudaGetDevice(&E->dev);
    cudaDeviceGetAttribute(&E->sms, cudaDevAttrMultiProcessorCount, E->dev);
    E->s = (cudaStream_t)stream;
    {   // a pool of its own that keeps freed memory (release threshold: never), so
        // admitting a request after another retired does not go back to the driver
        cudaMemPoolProps pp;
        memset(&pp, 0, sizeof(pp));
        pp.allocType = cudaMemAllocationTypePinned;
        pp.handleTypes = cudaMemHandleTypeNone;
        pp.location.type = cudaMemLocationTypeDevice;
        pp.location.id = E->dev;
        cudaError_t pe = cudaMemPoolCreate(&E->pool, &pp);
        uint64_t keep = UINT64_MAX;
        if (pe == cudaSuccess) pe = cudaMemPoolSetAttribute(E->pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (pe != cudaSuccess) {
            set_error("engine memory pool", pe);
            if (E->pool) cudaMemPoolDestroy(E->pool);
            delete E;
            return IMR_ERR_CUDA;
        }
    }
    if (device_bytes == 0) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        device_bytes = fr / 10 * 8;
    }
    E->budget = device_bytes;
    E->max_slots = max_jobs;
    cudaError_t e = cudaMalloc(&E->dj, sizeof(JobDev) * max_jobs);
    if (e == cudaSuccess) e = cudaMalloc(&E->dst, sizeof(JobState) * max_jobs);
    for (int q = 0; q < 2 && e == cudaSuccess; ++q) {
        e = cudaMallocHost(&E->hst[q], sizeof(JobState) * max_jobs);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&E->ev_st[q], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&E->ev_lists[q], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreate(&E->ev_t0[q]);
        if (e == cudaSuccess) e = cudaEventCreate(&E->ev_t1[q]);
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&E->cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&E->ev_fork, cudaEventDisableTiming);
    for (int b = 0; b < kBranchStreams && e == cudaSuccess; ++b) {
        e = cudaStreamCreateWithFlags(&E->bs[b], cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&E->ev_join[b], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaMemset(E->dst, 0, sizeof(JobState) * max_jobs);
    if (e != cudaSuccess) {
        set_error("engine create", e);
        imr_engine_destroy(E);
        return IMR_ERR_OUT_OF_MEMORY;
    }
    for (int i = max_jobs - 1; i >= 0; --i) E->free_slots.push_back(i);
    *out = E;
    return IMR_SUCCESS;
}

static int submit(imr_engine *E, const float *h_in, bool intensity, float *h_out, unsigned W, unsigned H,
                  const imr_params *params, long long tag)
{
    if (!E || !h_in || !h_out || W == 0 || H == 0) return IMR_ERR_INVALID_VALUE;
    EJob *j = new EJob();
    j->W = W;
    j->H = H;
    resolve_params(params, j->p);
    int rc = job_prepare(W, H, j->p, j->J, j->S);
    if (rc) {
        delete j;
        return rc;
    }
    j->h_in = h_in;
    j->intensity = intensity;
    j->h_out = h_out;
    j->tag = tag;
    j->t_submit = now_ms();
    E->pending.push_back(j);
    return IMR_SUCCESS;
}

int imr_engine_submit(imr_engine *E, const float *h_modulus, float *h_out, unsigned W, unsigned H,
                      const imr_params *params, long long tag)
{
    return submit(E, h_modulus, false, h_out, W, H, params, tag);
}

int imr_engine_submit_intensity(imr_engine *E, const float *h_intensity, float *h_out, unsigned W, unsigned H,
                                const imr_params *params, long long tag)
{
    return submit(E, h_intensity, true, h_out, W, H, params, tag);
}

int imr_engine_step(imr_engine *E)
{
    if (!E) return IMR_ERR_INVALID_VALUE;
    int rc;
    const long n = E->steps;
    if (n >= 2 && n - 2 > E->synced_step) {   // the state after step n - 2 (copied into hst[n & 1])
        const int q = (int)(n & 1);
        CKE(cudaEventSynchronize(E->ev_st[q]));
        if ((rc = observe(E, E->hst[q], n - 2))) return rc;
    }
    if (n > 0 && E->pending.empty() && !E->active.empty()) {
        // every cycle of every running request is queued and nothing waits:
        // read the last step's state instead of queueing steps that would only
        // find them stopped
        bool all = true;
        for (EJob *j : E->active) all = all && j->cycles_launched >= (long)j->J.n_cycles + 1;
        if (all) {
            const int q = (int)((n - 1) & 1);
            CKE(cudaEventSynchronize(E->ev_st[q]));
            if (n - 1 > E->synced_step && (rc = observe(E, E->hst[q], n - 1))) return rc;
            if (E->active.empty()) return drain(E);
        }
    }
    if ((rc = admit(E))) return rc;
    if (E->active.empty()) {   // nothing to run: hand over what is still in flight
        E->fresh.clear();
        return E->retiring.empty() ? IMR_SUCCESS : drain(E);
    }
    tune_before_step(E);
    if (E->dirty && (rc = rebuild(E))) return rc;
    // column init of the newly admitted jobs, then one cycle of every active job
    const WorkList *L = E->d_lists;
    for (auto &g : E->init_groups) {
        g.ck.init<<<loop_grid(E, (int)g.items.size()), g.ck.threads, g.ck.smem ? g.ck.smem : g.smem, E->s>>>(
            E->dj, L + g.list_base);
        ++E->launches;
        ++E->host_launches;
    }
    CKE(cudaGetLastError());
    E->init_groups.clear();
    E->fresh.clear();
    const int q = (int)(n & 1);
    CKE(cudaEventRecord(E->ev_t0[q], E->s));
    const double tl = now_ms();
    CKE(cudaGraphLaunch(E->gexec, E->s));
    E->step_launch_ms[q] = now_ms() - tl;
    CKE(cudaEventRecord(E->ev_t1[q], E->s));
    E->step_px[q] = E->active_px;
    tune_after_launch(E, n);
    for (EJob *j : E->active) j->cycles_launched += E->cycles_per_step;
    stage_request(E);   // staging for these requests' results, pinned while the GPU runs
    ++E->host_launches;
    E->launches += E->kernels_per_step;
    CKE(cudaMemcpyAsync(E->hst[q], E->dst, sizeof(JobState) * E->max_slots, cudaMemcpyDeviceToHost, E->s));
    CKE(cudaEventRecord(E->ev_st[q], E->s));
    E->st_step[q] = n;
    ++E->steps;
    return IMR_SUCCESS;
}

int imr_engine_poll(imr_engine *E, imr_result *results, int max_results, int *n_results)
{
    if (!E || !n_results || (max_results > 0 && !results)) return IMR_ERR_INVALID_VALUE;
    if (int rc = reap(E)) return rc;
    int n = 0;
    while (n < max_results && !E->done.empty()) {
        EJob *j = E->done.front();
        E->done.pop_front();
        imr_result &r = results[n++];
        r.tag = j->tag;
        r.width = j->W;
        r.height = j->H;
        r.cycles_done = j->cycles_done;
        r.last_error = j->last_error;
        r.latency_ms = j->t_done - j->t_submit;
        r.status = j->status;
        delete j;
    }
    *n_results = n;
    return IMR_SUCCESS;
}

int imr_engine_run(imr_engine *E)
{
    if (!E) return IMR_ERR_INVALID_VALUE;
    while (!E->pending.empty() || !E->active.empty() || !E->retiring.empty()) {
        int rc = imr_engine_step(E);
        if (rc) return rc;
    }
    return IMR_SUCCESS;
}

int imr_engine_cancel(imr_engine *E, long long tag)
{
    if (!E) return IMR_ERR_INVALID_VALUE;
    for (auto it = E->pending.begin(); it != E->pending.end(); ++it)
        if ((*it)->tag == tag) {
            EJob *j = *it;
            E->pending.erase(it);
            finish_now(E, j, IMR_ERR_CANCELLED);
            return IMR_SUCCESS;
        }
    EJob *j = find_active(E, tag);
    if (!j) {
        snprintf(g_last_error, sizeof(g_last_error), "engine: no pending or running request with tag %lld", tag);
        return IMR_ERR_INVALID_VALUE;
    }
    // steps already queued may still run it: its memory is released after them
    E->active.erase(std::find(E->active.begin(), E->active.end(), j));
    E->fresh.erase(std::remove(E->fresh.begin(), E->fresh.end(), j), E->fresh.end());
    CKE(cudaFreeAsync(j->arena, E->s));
    j->arena = nullptr;
    E->used -= j->S.bytes;
    E->active_px -= (size_t)j->W * j->H;
    E->free_slots.push_back(j->slot);
    E->dirty = true;
    finish_now(E, j, IMR_ERR_CANCELLED);
    return IMR_SUCCESS;
}

int imr_engine_set_admission(imr_engine *E, size_t max_active_pixels)
{
    if (!E) return IMR_ERR_INVALID_VALUE;
    E->max_active_px = max_active_pixels;
    return IMR_SUCCESS;
}

int imr_engine_set_schedule(imr_engine *E, int schedule)
{
    if (!E || (schedule != IMR_SCHEDULE_GROUPED && schedule != IMR_SCHEDULE_CHAINED)) return IMR_ERR_INVALID_VALUE;
    if (schedule != E->schedule) {
        E->schedule = schedule;
        E->dirty = true;
    }
    return IMR_SUCCESS;
}

int imr_engine_set_cycles_per_step(imr_engine *E, int cycles)
{
    if (!E || cycles < 1 || cycles > 256) return IMR_ERR_INVALID_VALUE;
    if (cycles != E->cycles_per_step) {
        E->cycles_per_step = cycles;
        E->ms_per_px = 0;   // the running step cost per pixel was for the old step length
        E->dirty = true;
    }
    return IMR_SUCCESS;
}

int imr_engine_set_autotune(imr_engine *E, int enable, const char *cache_path)
{
    if (!E) return IMR_ERR_INVALID_VALUE;
    E->tune = enable != 0;
    E->tune_path = cache_path ? cache_path : "";
    E->tune_sig.clear();
    E->tune_next = -1;
    tune_load(E);
    return IMR_SUCCESS;
}

int imr_engine_set_step_target(imr_engine *E, double target_step_ms)
{
    if (!E || target_step_ms < 0) return IMR_ERR_INVALID_VALUE;
    E->target_step_ms = target_step_ms;
    return IMR_SUCCESS;
}

int imr_engine_inject_alloc_failures(imr_engine *E, int count)
{
    if (!E || count < 0) return IMR_ERR_INVALID_VALUE;
    E->inject_alloc_fail = count;
    return IMR_SUCCESS;
}

int imr_engine_snapshot_size(imr_engine *E, long long tag, size_t *bytes)
{
    if (!E || !bytes) return IMR_ERR_INVALID_VALUE;
    EJob *j = find_active(E, tag);
    if (!j) return IMR_ERR_INVALID_VALUE;
    *bytes = snap_bytes(j->W, j->H, (unsigned)j->J.n_cycles + 1);
    return IMR_SUCCESS;
}

int imr_engine_checkpoint(imr_engine *E, long long tag, void *h_buf, size_t cap)
{
    if (!E || !h_buf) return IMR_ERR_INVALID_VALUE;
    EJob *j = find_active(E, tag);
    if (!j) return IMR_ERR_INVALID_VALUE;
    const unsigned n_err = (unsigned)j->J.n_cycles + 1;
    const size_t bytes = snap_bytes(j->W, j->H, n_err), N = (size_t)j->W * j->H;
    if (cap < bytes) return IMR_ERR_INVALID_VALUE;
    CKE(cudaStreamSynchronize(E->s));   // the device state at rest after the queued steps
    SnapHeader h;
    memset(&h, 0, sizeof(h));
    memcpy(h.magic, kSnapMagic, 8);
    h.W = j->W;
    h.H = j->H;
    h.p = j->p;
    h.tag = j->tag;
    h.n_err = n_err;
    h.bytes = bytes;
    CKE(cudaMemcpy(&h.st, E->dst + j->slot, sizeof(JobState), cudaMemcpyDeviceToHost));
    if (h.st.stop || h.st.err) {   // finished on the device: its result is on the way, nothing to save
        snprintf(g_last_error, sizeof(g_last_error), "engine: request %lld has already finished", tag);
        return IMR_ERR_INVALID_VALUE;
    }
    char *d = (char *)h_buf;
    memcpy(d, &h, sizeof(h));
    d += sizeof(h);
    CKE(cudaMemcpy(d, j->J.X, N * 8, cudaMemcpyDeviceToHost));
    CKE(cudaMemcpy(d + N * 8, j->J.G, N * 8, cudaMemcpyDeviceToHost));
    CKE(cudaMemcpy(d + N * 16, j->J.M, N * 4, cudaMemcpyDeviceToHost));
    CKE(cudaMemcpy(d + N * 20, j->J.mask, N, cudaMemcpyDeviceToHost));
    CKE(cudaMemcpy(d + N * 21, j->J.errors, (size_t)n_err * 4, cudaMemcpyDeviceToHost));
    return IMR_SUCCESS;
}

int imr_engine_suspend(imr_engine *E, long long tag, void *h_buf, size_t cap)
{
    int rc = imr_engine_checkpoint(E, tag, h_buf, cap);
    if (rc) return rc;
    EJob *j = find_active(E, tag);
    E->active.erase(std::find(E->active.begin(), E->active.end(), j));
    E->fresh.erase(std::remove(E->fresh.begin(), E->fresh.end(), j), E->fresh.end());
    CKE(cudaFreeAsync(j->arena, E->s));
    CKE(cudaStreamSynchronize(E->s));
    E->used -= j->S.bytes;
    E->active_px -= (size_t)j->W * j->H;
    E->free_slots.push_back(j->slot);
    E->dirty = true;
    delete j;
    return IMR_SUCCESS;
}

int imr_engine_resume(imr_engine *E, const void *h_buf, size_t bytes, float *h_out)
{
    if (!E || !h_buf || !h_out || bytes < sizeof(SnapHeader)) return IMR_ERR_INVALID_VALUE;
    SnapHeader h;
    memcpy(&h, h_buf, sizeof(h));
    if (memcmp(h.magic, kSnapMagic, 8) != 0 || h.W == 0 || h.H == 0 || h.bytes != bytes ||
        bytes != snap_bytes(h.W, h.H, h.n_err) || h.n_err != h.p.nCycles + 1)
        return IMR_ERR_INVALID_VALUE;
    EJob *j = new EJob();
    j->W = h.W;
    j->H = h.H;
    j->p = h.p;
    int rc = job_prepare(h.W, h.H, j->p, j->J, j->S);
    if (rc) {
        delete j;
        return rc;
    }
    j->resume.assign((const char *)h_buf, (const char *)h_buf + bytes);
    j->h_out = h_out;
    j->tag = h.tag;
    j->t_submit = now_ms();
    E->pending.push_back(j);
    return IMR_SUCCESS;
}

int imr_engine_stats(imr_engine *E, imr_engine_info *st)
{
    if (!E || !st) return IMR_ERR_INVALID_VALUE;
    st->pending = (int)E->pending.size();
    st->active = (int)(E->active.size() + E->retiring.size());
    st->done = (int)E->done.size();
    st->device_bytes_used = E->used;
    st->device_bytes_peak = E->peak;
    st->device_bytes_budget = E->budget;
    st->launches = E->launches;
    st->steps = E->steps;
    st->host_launches = E->host_launches;
    st->kernels_per_step = E->kernels_per_step;
    st->graph_builds = E->graph_builds;
    st->graph_updates = E->graph_updates;
    st->alloc_failures = E->alloc_failures;
    st->resident = (int)E->active.size();
    st->resident_px = E->active_px;
    st->last_step_ms = E->last_step_ms;
    st->ms_per_mpx = E->ms_per_px * 1e6;
    st->device_ms = E->device_ms;
    st->schedule = E->schedule;
    st->grid_pct = E->grid_pct;
    st->tune_explored = E->tune_explored;
    st->tune_cache_hits = E->tune_hits;
    st->cycles_per_step = E->cycles_per_step;
    return IMR_SUCCESS;
}

int imr_engine_destroy(imr_engine *E)
{
    if (!E) return IMR_SUCCESS;
    cudaStreamSynchronize(E->s);
    for (EJob *j : E->active) {
        if (j->arena) cudaFreeAsync(j->arena, E->s);
        delete j;
    }
    for (EJob *j : E->retiring) delete j;
    for (EJob *j : E->pending) delete j;
    for (EJob *j : E->done) delete j;
    cudaStreamSynchronize(E->s);
    if (E->gexec) cudaGraphExecDestroy(E->gexec);
    if (E->graph) cudaGraphDestroy(E->graph);
    if (E->dj) cudaFree(E->dj);
    if (E->dst) cudaFree(E->dst);
    for (int q = 0; q < 2; ++q) {
        if (E->hst[q]) cudaFreeHost(E->hst[q]);
        if (E->h_items[q]) cudaFreeHost(E->h_items[q]);
        if (E->h_lists[q]) cudaFreeHost(E->h_lists[q]);
        if (E->ev_st[q]) cudaEventDestroy(E->ev_st[q]);
        if (E->ev_lists[q]) cudaEventDestroy(E->ev_lists[q]);
        if (E->ev_t0[q]) cudaEventDestroy(E->ev_t0[q]);
        if (E->ev_t1[q]) cudaEventDestroy(E->ev_t1[q]);
    }
    {
        std::lock_guard<std::mutex> lk(E->grower.mu);
        E->grower.stop = true;
    }
    E->grower.cv.notify_one();
    if (E->grower.th.joinable()) E->grower.th.join();
    stage_adopt(E);
    for (auto &st : E->staging)
        if (st.p) cudaFreeHost(st.p);
    if (E->d_items) cudaFree(E->d_items);
    if (E->d_lists) cudaFree(E->d_lists);
    if (E->cs) cudaStreamDestroy(E->cs);
    if (E->ev_fork) cudaEventDestroy(E->ev_fork);
    for (int b = 0; b < kBranchStreams; ++b) {
        if (E->bs[b]) cudaStreamDestroy(E->bs[b]);
        if (E->ev_join[b]) cudaEventDestroy(E->ev_join[b]);
    }
    if (E->pool) cudaMemPoolDestroy(E->pool);
    delete E;
    return IMR_SUCCESS;
}

}  // extern "C"
