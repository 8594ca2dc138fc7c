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
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <deque>
#include <map>
#include <vector>

#include "imresh_b200.h"
#include "kernels.cuh"
#include "engine_host.hpp"

namespace imr {

static double now_ms()
{
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

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

}  // namespace imr

using namespace imr;

struct imr_engine {
    int dev = 0;
    cudaStream_t s = nullptr;
    cudaMemPool_t pool = nullptr;   // the engine's own pool: freed arenas stay cached for new admissions
    size_t budget = 0, used = 0, peak = 0;
    int max_slots = 0;
    JobDev *dj = nullptr;           // [max_slots]
    JobState *dst = nullptr;        // [max_slots]
    JobState *hst = nullptr;        // pinned mirror
    std::vector<int> free_slots;
    std::deque<EJob *> pending;
    std::vector<EJob *> active;
    std::vector<EJob *> done;
    WorkItem *d_items = nullptr;
    size_t items_cap = 0;
    WorkList *d_lists = nullptr;
    size_t lists_cap = 0;
    WorkItem *h_items = nullptr;   // pinned staging
    WorkList *h_lists = nullptr;
    long launches = 0;
    long steps = 0;
    int sms = 148;
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
    if (n_items > E->items_cap) {
        size_t cap = std::max(n_items, E->items_cap * 2 + 1024);
        if (E->d_items) cudaFree(E->d_items);
        if (E->h_items) cudaFreeHost(E->h_items);
        CKE(cudaMalloc(&E->d_items, cap * sizeof(WorkItem)));
        CKE(cudaMallocHost(&E->h_items, cap * sizeof(WorkItem)));
        E->items_cap = cap;
    }
    if (n_lists > E->lists_cap) {
        size_t cap = std::max(n_lists, E->lists_cap * 2 + 256);
        if (E->d_lists) cudaFree(E->d_lists);
        if (E->h_lists) cudaFreeHost(E->h_lists);
        CKE(cudaMalloc(&E->d_lists, cap * sizeof(WorkList)));
        CKE(cudaMallocHost(&E->h_lists, cap * sizeof(WorkList)));
        E->lists_cap = cap;
    }
    return IMR_SUCCESS;
}

// Loop-kernel grid: enough CTAs to fill the GPU, never more than the items.
static int loop_grid(const imr_engine *E, int items) { return std::max(1, std::min(items, E->sms * 16)); }

static int admit(imr_engine *E, std::vector<EJob *> &fresh)
{
    while (!E->pending.empty() && !E->free_slots.empty()) {
        EJob *j = E->pending.front();
        if (E->used + j->S.bytes > E->budget && !(E->active.empty() && fresh.empty())) break;
        E->pending.pop_front();
        j->slot = E->free_slots.back();
        E->free_slots.pop_back();
        cudaError_t e = cudaMallocFromPoolAsync((void **)&j->arena, j->S.bytes, E->pool, E->s);
        if (e != cudaSuccess) {   // allocation failed: back to the queue, retry later
            E->free_slots.push_back(j->slot);
            j->slot = -1;
            E->pending.push_front(j);
            cudaGetLastError();
            break;
        }
        E->used += j->S.bytes;
        E->peak = std::max(E->peak, E->used);
        job_bind(j->J, j->S, j->arena, E->dst + j->slot);
        int rc = job_upload(j->J, j->S, j->arena, E->dj + j->slot, E->s);
        if (rc) return rc;
        if (j->resume.empty()) {
            CKE(cudaMemsetAsync(E->dst + j->slot, 0, sizeof(JobState), E->s));
            CKE(cudaMemcpyAsync((void *)j->J.M, j->h_in, (size_t)j->W * j->H * 4, cudaMemcpyHostToDevice, E->s));
            if ((rc = job_modulus_tiles(j->J, E->s))) return rc;
            if (j->J.Mt) ++E->launches;
            fresh.push_back(j);
        } else {   // continue a suspended reconstruction where it stopped
            const SnapHeader *h = (const SnapHeader *)j->resume.data();
            const size_t N = (size_t)j->W * j->H;
            const char *d = j->resume.data() + sizeof(SnapHeader);
            // on the engine's stream, after job_upload's clearing of the mask and
            // errors; a copy from pageable memory has staged its source on return
            CKE(cudaMemcpyAsync(E->dst + j->slot, &h->st, sizeof(JobState), cudaMemcpyHostToDevice, E->s));
            CKE(cudaMemcpyAsync(j->J.X, d, N * 8, cudaMemcpyHostToDevice, E->s));
            CKE(cudaMemcpyAsync(j->J.G, d + N * 8, N * 8, cudaMemcpyHostToDevice, E->s));
            CKE(cudaMemcpyAsync((void *)j->J.M, d + N * 16, N * 4, cudaMemcpyHostToDevice, E->s));
            if ((rc = job_modulus_tiles(j->J, E->s))) return rc;
            if (j->J.Mt) ++E->launches;
            CKE(cudaMemcpyAsync(j->J.mask, d + N * 20, N, cudaMemcpyHostToDevice, E->s));
            CKE(cudaMemcpyAsync(j->J.errors, d + N * 21, (size_t)h->n_err * 4, cudaMemcpyHostToDevice, E->s));
            CKE(cudaStreamSynchronize(E->s));
            std::vector<char>().swap(j->resume);
        }
        E->active.push_back(j);
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

static int launch_step(imr_engine *E, const std::vector<EJob *> &fresh)
{
    cudaStream_t s = E->s;
    // --- column init of newly admitted jobs
    std::vector<Group> init_groups, rowg, colg;
    build_groups(fresh, false, init_groups);
    std::vector<EJob *> live;
    for (EJob *j : E->active) live.push_back(j);
    build_groups(live, true, rowg);
    build_groups(live, false, colg);
    // vertical-blur items: every live job
    std::vector<WorkItem> vb;
    for (EJob *j : live)
        for (int t = 0; t < j->J.n_vb_tiles; ++t) vb.push_back(WorkItem{j->slot, t});

    size_t n_items = vb.size(), n_lists = 1;
    for (auto *G : {&init_groups, &rowg, &colg})
        for (auto &g : *G) {
            n_items += g.items.size();
            n_lists += 1 + g.hio_count.size();
        }
    int rc = grow(E, n_items, n_lists);
    if (rc) return rc;
    size_t ip = 0, lp = 0;
    auto put = [&](const std::vector<WorkItem> &items, const std::vector<int> &counts, int &base) {
        const WorkItem *dptr = E->d_items + ip;
        memcpy(E->h_items + ip, items.data(), items.size() * sizeof(WorkItem));
        base = (int)lp;
        E->h_lists[lp++] = WorkList{dptr, (int)items.size()};
        for (int c : counts) E->h_lists[lp++] = WorkList{dptr, c};
        ip += items.size();
    };
    int vb_base = 0;
    put(vb, {}, vb_base);
    for (auto *G : {&init_groups, &rowg, &colg})
        for (auto &g : *G) put(g.items, g.hio_count, g.list_base);
    CKE(cudaMemcpyAsync(E->d_items, E->h_items, ip * sizeof(WorkItem), cudaMemcpyHostToDevice, s));
    CKE(cudaMemcpyAsync(E->d_lists, E->h_lists, lp * sizeof(WorkList), cudaMemcpyHostToDevice, s));
    const WorkList *L = E->d_lists;

    for (auto &g : init_groups) {
        g.ck.init<<<loop_grid(E, (int)g.items.size()), g.ck.threads, g.ck.smem ? g.ck.smem : g.smem, s>>>(
            E->dj, L + g.list_base);
        ++E->launches;
    }
    // --- one shrink-wrap cycle of every live job
    for (auto &g : rowg) {
        if (g.pipelined) {
            if ((rc = launch_finish(g.rk, (int)g.items.size(), g.smem_fin, s, E->dj, L + g.list_base, nullptr)))
                return rc;
        } else {
            g.rk.finish<<<loop_grid(E, (int)g.items.size()), g.rk.threads, g.smem_fin, s>>>(E->dj, L + g.list_base,
                                                                                         nullptr);
        }
        ++E->launches;
    }
    if (!vb.empty()) {
        k_vblur<<<loop_grid(E, (int)vb.size()), kVbThreads, 0, s>>>(E->dj, L + vb_base);
        ++E->launches;
    }
    int max_hio = 0;
    for (auto &g : rowg) max_hio = std::max(max_hio, (int)g.hio_count.size());
    for (int i = 0; i < max_hio; ++i) {
        for (auto &g : rowg) {
            if (i >= (int)g.hio_count.size()) continue;
            const WorkList *Li = L + g.list_base + 1 + i;
            const int n = g.hio_count[i];
            if (g.pipelined) {
                auto k = i == 0 ? g.rk.p_hio_first : g.rk.p_hio;
                const int sm = i == 0 ? g.rk.p_smem_first : g.rk.p_smem;
                k<<<persistent_grid((const void *)k, g.rk.threads, sm, n), g.rk.threads, sm, s>>>(E->dj, Li);
            } else {
                (i == 0 ? g.rk.hio_first : g.rk.hio)<<<loop_grid(E, n), g.rk.threads, g.smem, s>>>(E->dj, Li);
            }
            ++E->launches;
        }
        for (auto &g : colg) {
            if (i >= (int)g.hio_count.size()) continue;
            const WorkList *Li = L + g.list_base + 1 + i;
            const int n = g.hio_count[i];
            if (g.pipelined)
                g.ck.p_col<<<persistent_grid((const void *)g.ck.p_col, g.ck.p_threads, g.ck.p_smem, n),
                             g.ck.p_threads, g.ck.p_smem, s>>>(E->dj, Li);
            else
                g.ck.col<<<loop_grid(E, n), g.ck.threads, g.smem, s>>>(E->dj, Li);
            ++E->launches;
        }
    }
    CKE(cudaGetLastError());
    return IMR_SUCCESS;
}

static int retire(imr_engine *E)
{
    CKE(cudaMemcpyAsync(E->hst, E->dst, sizeof(JobState) * E->max_slots, cudaMemcpyDeviceToHost, E->s));
    CKE(cudaStreamSynchronize(E->s));
    std::vector<EJob *> keep, out;
    for (EJob *j : E->active) {
        const JobState &st = E->hst[j->slot];
        if (st.stop || st.err) {
            j->cycles_done = st.cycles_done;
            j->last_error = st.last_error;
            j->status = st.err ? IMR_ERR_DEVICE_TIMEOUT : IMR_SUCCESS;
            CKE(cudaMemcpyAsync(j->h_out, j->J.out, (size_t)j->W * j->H * 4, cudaMemcpyDeviceToHost, E->s));
            CKE(cudaFreeAsync(j->arena, E->s));
            out.push_back(j);
        } else {
            keep.push_back(j);
        }
    }
    E->active.swap(keep);
    if (!out.empty()) {
        CKE(cudaStreamSynchronize(E->s));
        const double t = now_ms();
        for (EJob *j : out) {
            j->t_done = t;
            E->used -= j->S.bytes;
            E->free_slots.push_back(j->slot);
            j->arena = nullptr;
            E->done.push_back(j);
        }
    }
    return IMR_SUCCESS;
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
    if (e == cudaSuccess) e = cudaMallocHost(&E->hst, sizeof(JobState) * max_jobs);
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

int imr_engine_submit(imr_engine *E, const float *h_modulus, float *h_out, unsigned W, unsigned H,
                      const imr_params *params, long long tag)
{
    if (!E || !h_modulus || !h_out || W == 0 || H == 0) return IMR_ERR_INVALID_VALUE;
    EJob *j = new EJob();
    j->W = W;
    j->H = H;
    resolve_params(params, j->p);
    int rc = job_prepare(W, H, j->p, j->J, j->S);
    if (rc) {
        delete j;
        return rc;
    }
    j->h_in = h_modulus;
    j->h_out = h_out;
    j->tag = tag;
    j->t_submit = now_ms();
    E->pending.push_back(j);
    return IMR_SUCCESS;
}

int imr_engine_step(imr_engine *E)
{
    if (!E) return IMR_ERR_INVALID_VALUE;
    std::vector<EJob *> fresh;
    int rc = admit(E, fresh);
    if (rc) return rc;
    if (E->active.empty()) return IMR_SUCCESS;
    if ((rc = launch_step(E, fresh))) return rc;
    ++E->steps;
    return retire(E);
}

int imr_engine_poll(imr_engine *E, imr_result *results, int max_results, int *n_results)
{
    if (!E || !n_results || (max_results > 0 && !results)) return IMR_ERR_INVALID_VALUE;
    int n = 0;
    while (n < max_results && !E->done.empty()) {
        EJob *j = E->done.front();
        E->done.erase(E->done.begin());
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
    while (!E->pending.empty() || !E->active.empty()) {
        int rc = imr_engine_step(E);
        if (rc) return rc;
    }
    return IMR_SUCCESS;
}

static EJob *find_active(imr_engine *E, long long tag)
{
    for (EJob *j : E->active)
        if (j->tag == tag) return j;
    return nullptr;
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
    CKE(cudaStreamSynchronize(E->s));   // between steps the device state is at rest
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
    CKE(cudaFreeAsync(j->arena, E->s));
    CKE(cudaStreamSynchronize(E->s));
    E->used -= j->S.bytes;
    E->free_slots.push_back(j->slot);
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
    st->active = (int)E->active.size();
    st->done = (int)E->done.size();
    st->device_bytes_used = E->used;
    st->device_bytes_peak = E->peak;
    st->device_bytes_budget = E->budget;
    st->launches = E->launches;
    st->steps = E->steps;
    return IMR_SUCCESS;
}

int imr_engine_destroy(imr_engine *E)
{
    if (!E) return IMR_SUCCESS;
    cudaStreamSynchronize(E->s);
    for (EJob *j : E->active) {
        if (j->arena) cudaFree(j->arena);
        delete j;
    }
    for (EJob *j : E->pending) delete j;
    for (EJob *j : E->done) delete j;
    if (E->dj) cudaFree(E->dj);
    if (E->dst) cudaFree(E->dst);
    if (E->hst) cudaFreeHost(E->hst);
    if (E->d_items) cudaFree(E->d_items);
    if (E->h_items) cudaFreeHost(E->h_items);
    if (E->d_lists) cudaFree(E->d_lists);
    if (E->h_lists) cudaFreeHost(E->h_lists);
    if (E->pool) {
        cudaStreamSynchronize(E->s);
        cudaMemPoolDestroy(E->pool);
    }
    delete E;
    return IMR_SUCCESS;
}

}  // extern "C"
