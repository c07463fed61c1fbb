// be_server.cu -- serving loop: continuous batching of 2D / 3D labeling requests.
//
// The reference labels files one after another from a host loop (ProcessImages,
// main.cpp:309-340; Process3DImages, :495-514).  The server instead accepts requests from any
// thread at any time:
//   * admission: a request is admitted when its device memory (input, labels, its share of the
//     pipeline workspace) fits both the byte budget -- by default 80% of the device's free memory
//     at creation -- and the memory free on the device right now (cudaMemGetInfo plus what the
//     server's own pool holds unused, read each time a batch is formed, so memory another tenant
//     of the GPU took after creation is seen), and a lane (CUDA stream) is free; otherwise it waits
//     in the queue, and a request that could never fit the budget is refused with BE_ERR_BUSY;
//   * batching: every time a lane is free, all admitted waiting requests (up to max_batch) are
//     copied in and labeled together by the persistent-kernel pipeline of be_batch (2D and 3D in one
//     go), so requests that arrive while others run join the next batch;
//   * overlap: `lanes` batches can be in flight at once on separate streams;
//   * residency: device buffers come from a stream-ordered memory pool that keeps its memory, so a
//     steady stream of requests does not go back to the driver.
// Each request's result is the same as labeling it alone: the batch kernels give every image its
// own tiles, segments and label space.
#include "be.h"
#include "be_api_internal.h"
#include "be_kernels.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

using namespace be;
using Clock = std::chrono::steady_clock;

namespace {

enum ReqState { QUEUED = 0, RUNNING = 1, DONE = 2 };

struct Req {
    uint64_t id;
    be_request r;
    Clock::time_point t_submit;
    int state = QUEUED;
    int status = BE_OK;
    bool cancelled = false;
    int64_t ncomp = 0;
    double latency_us = 0;
    size_t bytes = 0;
    uint8_t *d_in = nullptr;
    int32_t *d_out = nullptr;
};

struct Lane {
    cudaStream_t s = nullptr;
    cudaEvent_t done = nullptr;
    bool busy = false;
    std::vector<Req *> reqs;
    void *d_work = nullptr;          // descriptors + workspaces + counts of the running batch
    int64_t *h_counts = nullptr;     // pinned
    size_t h_counts_cap = 0;
    std::vector<Img2D> d2;
    std::vector<Img3D> d3;
    void *h_desc = nullptr;          // pinned staging of the descriptors
    size_t h_desc_cap = 0;
};

size_t al256(size_t v) { return (v + 255) / 256 * 256; }

int64_t voxels(const be_request &r) { return int64_t(r.dims[0]) * r.dims[1] * (r.dims[2] > 0 ? r.dims[2] : 1); }

// Device bytes of one request: input, labels and an upper bound of its workspace share.
size_t request_bytes(const be_request &r)
{
    const int64_t n = voxels(r);
    const bool dev = (r.flags & BE_REQ_DEVICE_BUFFERS) != 0;
    return (dev ? 0 : size_t(n) * 5) + size_t(n) * 2 + (size_t(1) << 20);
}

}  // namespace

struct be_server {
    be_server_config cfg{};
    int sms = 148;
    size_t budget = 0, used = 0;
    cudaMemPool_t pool = nullptr;
    std::vector<Lane> lanes;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Req *> pending;
    std::unordered_map<uint64_t, Req *> reqs;
    uint64_t next_id = 1;
    bool stop = false;
    std::thread worker;
    // statistics
    std::vector<double> lat_us;
    int64_t completed = 0, rejected = 0, failed = 0, batches = 0, pixels = 0;
    Clock::time_point t_first{}, t_last{};
    bool any = false;
    int64_t alloc_count = 0;

    // Live free memory, read at most every kLiveRefresh (the query can stall the device queue);
    // in between, the estimate follows the server's own admissions and releases.
    size_t live_q = 0, used_q = 0;
    Clock::time_point live_t{};
    bool live_valid = false;
    void run();
    size_t live_headroom();
    size_t live_estimate(bool refresh);
    bool launch(Lane &ln, std::vector<Req *> &batch);
    void finish(Lane &ln, int status);
    void *alloc(size_t bytes, cudaStream_t s, int *status);
};

void *be_server::alloc(size_t bytes, cudaStream_t s, int *status)
{
    ++alloc_count;
    if (cfg.inject_alloc_failure_every > 0 && alloc_count % cfg.inject_alloc_failure_every == 0) {
        *status = BE_ERR_OOM;   // host-side fault injection (tests)
        return nullptr;
    }
    void *p = nullptr;
    if (cudaMallocFromPoolAsync(&p, bytes, pool, s) != cudaSuccess) {
        cudaGetLastError();
        *status = BE_ERR_OOM;
        return nullptr;
    }
    return p;
}

// Device memory a new batch can take now: free memory plus what the pool holds but does not use.
size_t be_server::live_headroom()
{
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    unsigned long long reserved = 0, in_use = 0;   // the pool attributes are 64-bit
    if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess ||
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &in_use) != cudaSuccess) {
        cudaGetLastError();
        reserved = in_use = 0;
    }
    return fr + size_t(reserved > in_use ? reserved - in_use : 0);
}

size_t be_server::live_estimate(bool refresh)
{
    constexpr auto kLiveRefresh = std::chrono::milliseconds(20);
    const Clock::time_point now = Clock::now();
    if (refresh || !live_valid || now - live_t > kLiveRefresh) {
        live_q = live_headroom();
        used_q = used;
        live_t = now;
        live_valid = true;
    }
    // Memory the server admitted since the query is gone from the headroom; memory it released
    // since is back (in its pool).
    const size_t est = live_q + used_q;
    return est > used ? est - used : 0;
}

// Copies in, labels and copies out one batch on lane `ln`; false when nothing could be started.
bool be_server::launch(Lane &ln, std::vector<Req *> &batch)
{
    cudaStream_t s = ln.s;
    ln.reqs.clear();
    ln.d2.clear();
    ln.d3.clear();
    std::vector<Req *> ok;
    for (Req *q : batch) {
        int st = BE_OK;
        if (q->r.flags & BE_REQ_DEVICE_BUFFERS) {
            q->d_in = const_cast<uint8_t *>(q->r.in);
            q->d_out = q->r.out;
        } else {
            const size_t n = size_t(voxels(q->r));
            q->d_in = static_cast<uint8_t *>(alloc(n, s, &st));
            if (st == BE_OK) q->d_out = static_cast<int32_t *>(alloc(n * 4, s, &st));
            if (st != BE_OK) {
                if (q->d_in) cudaFreeAsync(q->d_in, s);
                q->d_in = nullptr;
                q->d_out = nullptr;
                q->status = st;
                continue;
            }
            // Requests' host buffers: pinned memory makes these copies asynchronous.
            cudaMemcpyAsync(q->d_in, q->r.in, n, cudaMemcpyHostToDevice, s);
        }
        ok.push_back(q);
    }
    // Failed admissions finish immediately.
    for (Req *q : batch)
        if (q->status != BE_OK) ln.reqs.push_back(q);
    if (ok.empty()) return false;
    int64_t t2 = 0, s2 = 0, t3 = 0, s3 = 0;
    for (size_t i = 0; i < ok.size(); ++i) {
        const be_request &r = ok[i]->r;
        const int index = int(i);
        if (r.dims[2] > 0) {
            Img3D im;
            fill_img3d(im, ok[i]->d_in, r.dims[0], r.dims[1], r.dims[2], r.threshold, ok[i]->d_out, t3, s3, index);
            t3 += int64_t(im.t0) * im.t1 * im.t2;
            s3 += int64_t(r.dims[0]) * r.dims[1] * im.t2;
            ln.d3.push_back(im);
        } else {
            Img2D im;
            fill_img2d(im, ok[i]->d_in, r.dims[1], r.dims[0], r.dims[1], r.threshold, ok[i]->d_out, r.dims[1],
                       t2, s2, index, 0);
            t2 += int64_t(im.tiles_x) * im.tiles_y;
            s2 += int64_t(r.dims[0]) * im.tiles_x;
            ln.d2.push_back(im);
        }
    }
    const int nimg = int(ok.size());
    const Geometry g2 = geometry_2d(), g3 = geometry_3d();
    const size_t w2 = ln.d2.empty() ? 0 : layout_work(g2, t2, s2, nimg, nullptr, nullptr);
    const size_t w3 = ln.d3.empty() ? 0 : layout_work(g3, t3, s3, nimg, nullptr, nullptr);
    const size_t o_d3 = al256(ln.d2.size() * sizeof(Img2D));
    const size_t o_cnt = o_d3 + al256(ln.d3.size() * sizeof(Img3D));
    const size_t o_w2 = o_cnt + al256(size_t(nimg) * sizeof(int64_t));
    const size_t o_w3 = o_w2 + al256(w2);
    const size_t total = o_w3 + al256(w3);
    int st = BE_OK;
    ln.d_work = alloc(total, s, &st);
    auto fail_all = [&](int code) {
        for (Req *q : ok) {
            q->status = code;
            if (!(q->r.flags & BE_REQ_DEVICE_BUFFERS)) {
                cudaFreeAsync(q->d_in, s);
                cudaFreeAsync(q->d_out, s);
            }
            q->d_in = nullptr;
            q->d_out = nullptr;
        }
        ln.reqs.insert(ln.reqs.end(), ok.begin(), ok.end());
        return false;
    };
    if (!ln.d_work) return fail_all(st);
    // Descriptors through pinned staging (the lane owns it until the batch completes).
    const size_t desc_bytes = o_cnt;
    if (desc_bytes > ln.h_desc_cap) {
        if (ln.h_desc) cudaFreeHost(ln.h_desc);
        ln.h_desc = nullptr;
        ln.h_desc_cap = 0;
        if (cudaMallocHost(&ln.h_desc, desc_bytes * 2) == cudaSuccess) ln.h_desc_cap = desc_bytes * 2;
    }
    if (size_t(nimg) > ln.h_counts_cap) {
        if (ln.h_counts) cudaFreeHost(ln.h_counts);
        ln.h_counts = nullptr;
        ln.h_counts_cap = 0;
        if (cudaMallocHost(&ln.h_counts, size_t(nimg) * 2 * sizeof(int64_t)) == cudaSuccess)
            ln.h_counts_cap = size_t(nimg) * 2;
    }
    if (!ln.h_desc || !ln.h_counts) {
        cudaFreeAsync(ln.d_work, s);
        ln.d_work = nullptr;
        return fail_all(BE_ERR_OOM);
    }
    char *hb = static_cast<char *>(ln.h_desc);
    if (!ln.d2.empty()) std::memcpy(hb, ln.d2.data(), ln.d2.size() * sizeof(Img2D));
    if (!ln.d3.empty()) std::memcpy(hb + o_d3, ln.d3.data(), ln.d3.size() * sizeof(Img3D));
    char *base = static_cast<char *>(ln.d_work);
    cudaMemcpyAsync(base, hb, desc_bytes, cudaMemcpyHostToDevice, s);
    int64_t *counts = reinterpret_cast<int64_t *>(base + o_cnt);
    cudaError_t le = cudaSuccess;
    if (!ln.d2.empty()) {
        Work W;
        layout_work(g2, t2, s2, nimg, base + o_w2, &W);
        W.ncomp = counts;
        cudaMemsetAsync(W.queue, 0, kQueueWords * sizeof(uint32_t), s);
        reset_scan_state(W, s);   // the pool's memory is not zeroed
        ImgList2D L{reinterpret_cast<const Img2D *>(base), int(ln.d2.size()), ln.d2[0]};
        le = uf2d_launch(0, L, W, sms, true, s);
    }
    if (!ln.d3.empty() && le == cudaSuccess) {
        Work W;
        layout_work(g3, t3, s3, nimg, base + o_w3, &W);
        W.ncomp = counts;
        cudaMemsetAsync(W.queue, 0, kQueueWords * sizeof(uint32_t), s);
        reset_scan_state(W, s);
        ImgList3D L{reinterpret_cast<const Img3D *>(base + o_d3), int(ln.d3.size()), ln.d3[0]};
        le = launch_uf3d(L, W, sms, true, s);
    }
    cudaMemcpyAsync(ln.h_counts, counts, size_t(nimg) * sizeof(int64_t), cudaMemcpyDeviceToHost, s);
    for (Req *q : ok) {
        if (!(q->r.flags & BE_REQ_DEVICE_BUFFERS)) {
            cudaMemcpyAsync(q->r.out, q->d_out, size_t(voxels(q->r)) * 4, cudaMemcpyDeviceToHost, s);
            cudaFreeAsync(q->d_in, s);
            cudaFreeAsync(q->d_out, s);
        }
        q->d_in = nullptr;
        q->d_out = nullptr;
    }
    cudaFreeAsync(ln.d_work, s);
    ln.d_work = nullptr;
    cudaEventRecord(ln.done, s);
    ln.reqs.insert(ln.reqs.end(), ok.begin(), ok.end());
    if (le != cudaSuccess)
        for (Req *q : ok) q->status = BE_ERR_CUDA;
    return true;
}

// Completes every request of a lane (called with `mu` held).
void be_server::finish(Lane &ln, int)
{
    const Clock::time_point now = Clock::now();
    int i = 0;
    for (Req *q : ln.reqs) {
        if (q->status == BE_OK) {
            q->ncomp = ln.h_counts ? ln.h_counts[i++] : 0;
            ++completed;
            pixels += voxels(q->r);
            q->latency_us = std::chrono::duration<double, std::micro>(now - q->t_submit).count();
            lat_us.push_back(q->latency_us);
            if (!any) {
                t_first = q->t_submit;
                any = true;
            }
            t_last = now;
        } else {
            ++failed;
        }
        if (q->cancelled) q->status = BE_ERR_CANCELLED;
        q->state = DONE;
        used -= std::min(used, q->bytes);
    }
    ln.reqs.clear();
    ln.busy = false;
    cv_done.notify_all();
}

void be_server::run()
{
    cudaSetDevice(cfg.device);
    std::unique_lock<std::mutex> lock(mu);
    for (;;) {
        // Retire finished batches.
        for (Lane &ln : lanes)
            if (ln.busy && cudaEventQuery(ln.done) == cudaSuccess) finish(ln, BE_OK);
        bool inflight = false;
        for (Lane &ln : lanes) inflight |= ln.busy;
        if (stop && pending.empty() && !inflight) break;
        // Start a batch on a free lane with every admissible waiting request.
        Lane *free_lane = nullptr;
        for (Lane &ln : lanes)
            if (!ln.busy) {
                free_lane = &ln;
                break;
            }
        bool started = false;
        if (free_lane && !pending.empty()) {
            std::vector<Req *> batch;
            size_t live = live_estimate(false);
            bool refreshed = false;
            size_t take = 0;
            while (!pending.empty() && int(batch.size()) < cfg.max_batch) {
                Req *q = pending.front();
                if (q->cancelled) {
                    pending.pop_front();
                    q->status = BE_ERR_CANCELLED;
                    q->state = DONE;
                    cv_done.notify_all();
                    continue;
                }
                const size_t need = request_bytes(q->r);
                if (need > budget) {          // can never fit
                    pending.pop_front();
                    q->status = BE_ERR_BUSY;
                    q->state = DONE;
                    ++rejected;
                    cv_done.notify_all();
                    continue;
                }
                if (used + need > budget) break;   // wait for memory to free up
                if (take + need > live && !refreshed) {   // the estimate says no: read it again
                    live = live_estimate(true);
                    refreshed = true;
                }
                if (take + need > live) break;     // the device is fuller than the budget says
                take += need;
                pending.pop_front();
                q->bytes = need;
                used += need;
                q->state = RUNNING;
                batch.push_back(q);
            }
            if (!batch.empty()) {
                free_lane->busy = true;   // reserved while the lock is dropped
                lock.unlock();
                started = launch(*free_lane, batch);
                lock.lock();
                if (!started) finish(*free_lane, BE_OK);
                else ++batches;
            }
        }
        if (!started) {
            if (inflight) {
                lock.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(20));
                lock.lock();
            } else {
                cv_work.wait_for(lock, std::chrono::milliseconds(5));
            }
        }
    }
}

extern "C" {

void be_server_default_config(be_server_config *cfg)
{
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->device = 0;
    cfg->max_device_bytes = 0;
    cfg->lanes = 2;
    cfg->max_batch = 256;
    cfg->inject_alloc_failure_every = 0;
}

int be_server_create(const be_server_config *cfg, be_server **out)
{
    if (!cfg || !out || cfg->lanes <= 0 || cfg->max_batch <= 0) return BE_ERR_INVALID;
    *out = nullptr;
    if (cudaSetDevice(cfg->device) != cudaSuccess) return BE_ERR_CUDA;
    be_server *sv = new be_server();
    sv->cfg = *cfg;
    cudaDeviceGetAttribute(&sv->sms, cudaDevAttrMultiProcessorCount, cfg->device);
    size_t fr = 0, tot = 0;
    cudaMemGetInfo(&fr, &tot);
    sv->budget = cfg->max_device_bytes > 0 ? size_t(cfg->max_device_bytes) : fr / 10 * 8;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = cfg->device;
    if (cudaMemPoolCreate(&sv->pool, &props) != cudaSuccess) {
        delete sv;
        return BE_ERR_CUDA;
    }
    uint64_t keep = ~0ull;   // keep freed memory in the pool (resident buffers)
    cudaMemPoolSetAttribute(sv->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    sv->lanes.resize(size_t(cfg->lanes));
    for (Lane &ln : sv->lanes) {
        if (cudaStreamCreateWithFlags(&ln.s, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&ln.done, cudaEventDisableTiming) != cudaSuccess) {
            be_server_destroy(sv);
            return BE_ERR_CUDA;
        }
    }
    sv->worker = std::thread([sv] { sv->run(); });
    *out = sv;
    return BE_OK;
}

int be_server_submit(be_server *sv, const be_request *req, uint64_t *id)
{
    if (!sv || !req || !id || !req->in || !req->out || req->dims[0] <= 0 || req->dims[1] <= 0 ||
        voxels(*req) >= (int64_t(1) << 31) || req->threshold < 0 || req->threshold > 255)
        return BE_ERR_INVALID;
    Req *q = new Req();
    q->r = *req;
    q->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        if (sv->stop) {
            delete q;
            return BE_ERR_INVALID;
        }
        q->id = sv->next_id++;
        sv->reqs[q->id] = q;
        sv->pending.push_back(q);
    }
    sv->cv_work.notify_one();
    *id = q->id;
    return BE_OK;
}

int be_server_wait(be_server *sv, uint64_t id, int64_t timeout_us, be_result *res)
{
    if (!sv) return BE_ERR_INVALID;
    std::unique_lock<std::mutex> lock(sv->mu);
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end()) return BE_ERR_INVALID;
    Req *q = it->second;
    const auto pred = [q] { return q->state == DONE; };
    if (timeout_us < 0) sv->cv_done.wait(lock, pred);
    else if (!sv->cv_done.wait_for(lock, std::chrono::microseconds(timeout_us), pred)) return BE_ERR_TIMEOUT;
    if (res) {
        res->status = q->status;
        res->n_components = q->ncomp;
        res->latency_us = q->latency_us;
    }
    const int st = q->status;
    sv->reqs.erase(it);
    delete q;
    return st;
}

int be_server_cancel(be_server *sv, uint64_t id)
{
    if (!sv) return BE_ERR_INVALID;
    std::lock_guard<std::mutex> lock(sv->mu);
    auto it = sv->reqs.find(id);
    if (it == sv->reqs.end()) return BE_ERR_INVALID;
    it->second->cancelled = true;   // queued: dropped; running: completes, reported cancelled
    return BE_OK;
}

int be_server_stats(be_server *sv, be_serve_stats *st)
{
    if (!sv || !st) return BE_ERR_INVALID;
    std::lock_guard<std::mutex> lock(sv->mu);
    std::memset(st, 0, sizeof(*st));
    st->completed = sv->completed;
    st->rejected = sv->rejected;
    st->failed = sv->failed;
    st->batches = sv->batches;
    st->pixels = sv->pixels;
    std::vector<double> v = sv->lat_us;
    if (!v.empty()) {
        std::sort(v.begin(), v.end());
        auto pct = [&](double p) { return v[std::min(v.size() - 1, size_t(p * (v.size() - 1) + 0.5))]; };
        st->p50_us = pct(0.50);
        st->p99_us = pct(0.99);
        double sum = 0;
        for (double x : v) sum += x;
        st->mean_us = sum / v.size();
        st->wall_s = std::chrono::duration<double>(sv->t_last - sv->t_first).count();
    }
    st->device_bytes_in_use = int64_t(sv->used);
    st->device_bytes_budget = int64_t(sv->budget);
    return BE_OK;
}

int be_server_reset_stats(be_server *sv)
{
    if (!sv) return BE_ERR_INVALID;
    std::lock_guard<std::mutex> lock(sv->mu);
    sv->lat_us.clear();
    sv->completed = sv->rejected = sv->failed = sv->batches = sv->pixels = 0;
    sv->any = false;
    return BE_OK;
}

int be_server_destroy(be_server *sv)
{
    if (!sv) return BE_OK;
    {
        std::lock_guard<std::mutex> lock(sv->mu);
        sv->stop = true;
    }
    sv->cv_work.notify_all();
    if (sv->worker.joinable()) sv->worker.join();
    cudaSetDevice(sv->cfg.device);
    for (Lane &ln : sv->lanes) {
        if (ln.s) cudaStreamSynchronize(ln.s);
        if (ln.done) cudaEventDestroy(ln.done);
        if (ln.s) cudaStreamDestroy(ln.s);
        if (ln.h_counts) cudaFreeHost(ln.h_counts);
        if (ln.h_desc) cudaFreeHost(ln.h_desc);
    }
    for (auto &kv : sv->reqs) delete kv.second;
    if (sv->pool) cudaMemPoolDestroy(sv->pool);
    delete sv;
    return BE_OK;
}

}  // extern "C"
