// Proof server: continuous batching of proving jobs on one GPU.
//
// Jobs (a circuit in the vg_session_load layout plus a seed) enter a FIFO
// queue.  `slots` worker threads each own a session, i.e. a CUDA stream with
// its device tables, commitment buffers and GKR state.  A worker takes the
// job at the head of the queue as soon as it is free and the job's device
// footprint fits the HBM budget next to what the other workers hold, so jobs
// that arrive while others are proving are admitted as slots and memory free
// up, and their kernels overlap on the device.  Session buffers only grow
// (loading a circuit reuses them), so a worker's held memory is the largest
// footprint it has served; an idle worker gives its memory back when the head
// job cannot be admitted otherwise.  Each job's result equals the result of
// proving it alone: sessions share no state, and the proof is a function of
// (circuit, seed) only.
#include <cuda_runtime.h>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include "virgo_b200.h"

int vg_fail(int code, const char *fmt, ...);

namespace
{
using clk = std::chrono::steady_clock;

struct Job {
    long long id = 0;
    int d = 0;
    std::vector<long> n;
    std::vector<const uint8_t *> ty;
    std::vector<const void *> u, v;
    int index_bytes = 8;
    unsigned seed = 0;
    bool want_transcript = true;
    size_t footprint = 0;
    clk::time_point t_submit, t_start, t_end;
    // result
    bool done = false;
    int rc = VG_OK;
    std::string err;
    vg_proof_stats st{};
    std::vector<uint8_t> transcript;
};

size_t ceil_pow2_log(long x)
{
    size_t k = 0;
    while ((1L << k) < x) ++k;
    return k;
}
}  // namespace

// Device bytes a session needs for a circuit of file layers n[0..d): layer
// values and gate records, the edge sets of both phases, the GKR tables, and
// the commitment (4 codeword sets of 65 slices plus the FRI levels and trees).
extern "C" size_t vg_job_footprint(int d, const long *n)
{
    if (d < 1 || !n) return 0;
    const long pad = 1L << (d > 3 ? 17 : 15);
    const long n0 = std::max(n[0], pad);
    long maxw = 1L << ceil_pow2_log(n0);
    size_t gates = 0, vals = 2 * (size_t)maxw;   // input + relay layer
    for (int i = 1; i < d; ++i) {
        const long w = 1L << ceil_pow2_log(std::max(n[i], 2L));
        maxw = std::max(maxw, w);
        vals += w;
        gates += w;
    }
    const int L = (int)ceil_pow2_log(n0);
    const size_t S = (size_t)1 << (L - 1);
    size_t b = 0;
    b += vals * 16;                         // layer values
    b += (gates + (size_t)maxw) * 9;        // gate records (type, u, v)
    b += 2 * (gates + (size_t)maxw) * 14;   // edge sets of both phases (gate, wire, type) + offsets
    b += (size_t)maxw * 16 * 9 / 2 * 2;     // sumcheck tables, ping-pong
    b += (size_t)maxw * 16;                 // beta_g by gate
    b += 4 * 65 * S * 16;                   // l, h, q and virtual-oracle codewords
    b += 65 * S * 16 + 4 * S * 32;          // FRI levels, Merkle trees
    b += (size_t)64 << 20;                  // staging, scratch, twiddles
    b += vg_fft_gkr_footprint(L - 6);       // the fft_gkr side proof
    return b + b / 8;
}

struct vg_server {
    int device = 0;
    size_t budget = 0, held_total = 0;
    std::vector<std::thread> workers;
    std::vector<size_t> held;      // per worker: bytes its session holds
    std::vector<int> busy;
    std::deque<Job *> queue;
    std::map<long long, std::unique_ptr<Job> > jobs;
    long long next_id = 1;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    void worker(int w);
};

void vg_server::worker(int w)
{
    cudaSetDevice(device);
    vg_session *s = nullptr;
    for (;;) {
        Job *job = nullptr;
        {
            std::unique_lock<std::mutex> lk(mu);
            for (;;) {
                if (stop) {
                    lk.unlock();
                    if (s) vg_session_destroy(s);
                    return;
                }
                if (!queue.empty()) {
                    Job *head = queue.front();
                    const size_t need = std::max(held[w], head->footprint);
                    if (held_total - held[w] + need <= budget || held_total == held[w]) {
                        // admitted (a job alone on the device is always admitted)
                        held_total += need - held[w];
                        held[w] = need;
                        queue.pop_front();
                        job = head;
                        busy[w] = 1;
                        break;
                    }
                    if (s && head->footprint > held[w]) {
                        // give this idle worker's memory back, then let the others retry
                        lk.unlock();
                        vg_session_destroy(s);
                        s = nullptr;
                        lk.lock();
                        held_total -= held[w];
                        held[w] = 0;
                        cv_work.notify_all();
                        continue;
                    }
                }
                cv_work.wait(lk);
            }
        }
        job->t_start = clk::now();
        int rc = VG_OK;
        if (!s) rc = vg_session_new(&s);
        if (rc == VG_OK)
            rc = vg_session_load(s, job->d, job->n.data(), job->ty.data(), job->u.data(), job->v.data(), job->index_bytes);
        uint8_t *tr = nullptr;
        size_t len = 0;
        if (rc == VG_OK) rc = vg_session_prove(s, job->seed, job->want_transcript ? 1 : 0, &job->st, &tr, &len);
        if (rc != VG_OK) job->err = vg_last_error();
        if (tr) {
            job->transcript.assign(tr, tr + len);
            vg_free(tr);
        }
        job->t_end = clk::now();
        {
            std::lock_guard<std::mutex> lk(mu);
            job->rc = rc;
            job->done = true;
            busy[w] = 0;
        }
        cv_done.notify_all();
        cv_work.notify_all();
    }
}

extern "C" int vg_server_create(int device, int slots, size_t hbm_budget, vg_server **out)
{
    if (!out || slots < 1 || slots > 256) return vg_fail(VG_ERR_ARG, "vg_server_create: bad argument (slots %d)", slots);
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return vg_fail(VG_ERR_NO_DEVICE, "vg_server_create: no device %d", device);
    }
    vg_server *s = new vg_server();
    s->device = device;
    if (!hbm_budget) {   // default: 90% of what is free now, counting the pool's idle reserve as free
        size_t fr = 0, tot = 0;
        cudaSetDevice(device);
        cudaMemGetInfo(&fr, &tot);
        cudaMemPool_t pool;
        uint64_t reserved = 0, used = 0;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
            cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
        }
        cudaGetLastError();
        hbm_budget = (fr + (reserved > used ? reserved - used : 0)) / 10 * 9;
    }
    s->budget = hbm_budget;
    {   // stream-ordered allocations keep their freed blocks (see vg_alloc); the
        // budget is reserved in the pool up front, so sessions growing their
        // buffers for a larger circuit draw reserved memory instead of mapping
        // new memory through the driver while the other slots prove
        cudaSetDevice(device);
        cudaMemPool_t pool;
        uint64_t thr = ~0ull, reserved = 0;
        cudaStream_t st;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess &&
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr) == cudaSuccess &&
            cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
            reserved < hbm_budget && cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) == cudaSuccess) {
            void *p = nullptr;
            if (cudaMallocAsync(&p, hbm_budget - reserved, st) == cudaSuccess) cudaFreeAsync(p, st);
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        cudaGetLastError();
    }
    s->held.assign(slots, 0);
    s->busy.assign(slots, 0);
    for (int w = 0; w < slots; ++w) s->workers.emplace_back([s, w]() { s->worker(w); });
    *out = s;
    return VG_OK;
}

extern "C" int vg_server_submit(vg_server *s, int d, const long *n, const uint8_t *const *ty, const void *const *u,
                                const void *const *v, int index_bytes, unsigned seed, int want_transcript,
                                long long *job_id)
{
    if (!s || d < 1 || !n || !ty || !u || !v || !job_id || (index_bytes != 4 && index_bytes != 8))
        return vg_fail(VG_ERR_ARG, "vg_server_submit: bad argument");
    std::unique_ptr<Job> j(new Job());
    j->d = d;
    j->n.assign(n, n + d);
    j->ty.assign(ty, ty + d);
    j->u.assign(u, u + d);
    j->v.assign(v, v + d);
    j->index_bytes = index_bytes;
    j->seed = seed;
    j->want_transcript = want_transcript != 0;
    j->footprint = vg_job_footprint(d, n);
    j->t_submit = clk::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        j->id = s->next_id++;
        *job_id = j->id;
        s->queue.push_back(j.get());
        s->jobs[j->id] = std::move(j);
    }
    s->cv_work.notify_all();
    return VG_OK;
}

extern "C" int vg_server_wait(vg_server *s, long long job_id, vg_job_info *info, uint8_t **transcript,
                              size_t *transcript_len)
{
    if (!s) return vg_fail(VG_ERR_ARG, "vg_server_wait: null server");
    std::unique_ptr<Job> j;
    {
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->jobs.find(job_id);
        if (it == s->jobs.end()) return vg_fail(VG_ERR_ARG, "vg_server_wait: unknown job %lld", job_id);
        Job *p = it->second.get();
        s->cv_done.wait(lk, [&]() { return p->done; });
        j = std::move(it->second);
        s->jobs.erase(it);
    }
    auto sec = [](clk::time_point a, clk::time_point b) { return std::chrono::duration<double>(b - a).count(); };
    if (info) {
        memset(info, 0, sizeof *info);
        info->status = j->rc;
        info->queued_s = sec(j->t_submit, j->t_start);
        info->run_s = sec(j->t_start, j->t_end);
        info->latency_s = sec(j->t_submit, j->t_end);
        info->footprint = j->footprint;
        info->stats = j->st;
    }
    if (transcript && transcript_len) {
        *transcript_len = j->transcript.size();
        *transcript = (uint8_t *)malloc(j->transcript.size() ? j->transcript.size() : 1);
        if (!j->transcript.empty()) memcpy(*transcript, j->transcript.data(), j->transcript.size());
    }
    if (j->rc != VG_OK) return vg_fail(j->rc, "job %lld: %s", job_id, j->err.c_str());
    return VG_OK;
}

extern "C" int vg_server_destroy(vg_server *s)
{
    if (!s) return VG_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->queue.clear();
    }
    s->cv_work.notify_all();
    for (auto &t : s->workers) t.join();
    // give the pool's unused reserve back to the device
    cudaMemPool_t pool;
    cudaSetDevice(s->device);
    cudaDeviceSynchronize();
    if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    cudaGetLastError();
    delete s;
    return VG_OK;
}
