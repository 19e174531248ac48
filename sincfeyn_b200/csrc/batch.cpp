/* batch.cpp -- many integrals at once: sqb_hsum_batch() and its tuner.
 *
 * A batch is a list of integrals (graph, h, N, eps, top), e.g. every graph of a class at several h.
 * Each integral is one sqb_hsum() (the reference's hsum(), driver/sum.c:556-814), unchanged; the batch
 * runs them concurrently from a pool of host worker threads.  Every worker owns a CUDA stream, its
 * buffers and its share of device memory (the runtime's state is per thread), and pulls the next
 * integral from a shared queue, largest estimated cost first (longest-processing-time order), so that
 * the latency-bound parts of one integral (the top-level grow, which waits for every frontier's sums
 * on the host) overlap the FP64-bound level passes of others and small integrals fill the gaps
 * that a single integral's launches leave on the device.
 *
 * Device time: the caller's stream records a start event that every worker stream waits on before its
 * first launch; every worker records an end event after its last; the caller's stream waits on all of
 * them and records the stop event.  The elapsed time between start and stop is the batch's device time.
 *
 * An integral that runs out of device memory beside the others (the grow's tables of a large four-loop
 * integral at small h reach tens of GB) is not an error of the batch: it is run again after the queue
 * is drained, alone on the device, by the calling thread.
 *
 * With opts.group the units of work are the integrals of one graph (up to SQB_GROUP_MAX, e.g. the graph at
 * several h), each run by sqb_hsum_group: its refinement levels are shared launches over all of them.
 *
 * The tuner runs a calibration list (normally a few integrals of the batch) twice per candidate worker
 * count, the candidates in turn, and returns the count with the highest evaluated points per second of
 * device time, each count rated by its better run: a count's first run also pays its workers' first
 * allocations, and with one run per count the tuner picked 2 workers for the three-loop set in one process
 * (8.12 s a step) and 4 in another (7.99 s), its rates for the same count differing by up to 1.8x. */
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include <algorithm>
#include <stdio.h>
#include <string.h>
#include <cuda_runtime.h>
#include "sincfeyn_b200.h"
#include "sqb_rt.h"

extern "C" void sqb_set_error_msg(const char *msg);
extern "C" void sqb_set_mem_share(double f);

namespace {

struct Batch {
    const sqb_job_t *jobs = nullptr; int n = 0, nw = 0;
    std::vector<std::vector<int>> units;     /* opts.group: the jobs of one graph, run by one sqb_hsum_group */
    sqb_opts_t o;
    sqb_result_t *res = nullptr; int *rcs = nullptr;
    std::vector<int> order;
    std::atomic<int> next{0};
    cudaEvent_t start = nullptr;
    std::vector<cudaEvent_t> ends;
    std::vector<int> ended;          /* worker recorded its end event */
    std::mutex m; std::condition_variable cv; int left = 0, failures = 0; std::string err;
    std::vector<int> retry;          /* jobs that ran out of device memory: run again alone */
};

bool out_of_memory(const char *msg){
    return strstr(msg, "out of memory") || strstr(msg, "allocation");
}

/* the pool: workers wait for a new generation.  Its mutex and condition variable are never destroyed:
 * the workers are detached and still wait on them when the process exits, and destroying a condition
 * variable that has waiters blocks (glibc), which would hang the exit. */
std::mutex &PM = *new std::mutex;
std::condition_variable &PCV = *new std::condition_variable;
Batch *CUR = nullptr;
unsigned long GEN = 0;
int NSTARTED = 0;
const int MAXW = 32;

void serve(Batch *b, int id){
    sqb_set_mem_share(1.0/b->nw);
    std::string err;
    int ok = sqb_dev_init(b->o.device) == 0;
    cudaStream_t s = ok ? (cudaStream_t)sqb_dev_stream() : nullptr;
    if(ok && cudaStreamWaitEvent(s, b->start, 0) != cudaSuccess) ok = 0;
    if(!ok) err = std::string("worker ") + std::to_string(id) + ": " + sqb_last_error();
    while(ok){
        const int k = b->next.fetch_add(1);
        if(k >= (int)b->order.size()) break;
        std::vector<int> js;
        if(b->units.empty()) js.push_back(b->order[k]); else js = b->units[b->order[k]];
        if(js.size() == 1){
            const sqb_job_t &J = b->jobs[js[0]];
            b->rcs[js[0]] = sqb_hsum(J.graph, J.h, J.N, J.eps, J.top, &b->o, &b->res[js[0]]);
        } else {
            std::vector<sqb_job_t> uj; std::vector<sqb_result_t> ur(js.size()); std::vector<int> uc(js.size());
            for(int j : js) uj.push_back(b->jobs[j]);
            sqb_hsum_group(uj.data(), (int)js.size(), &b->o, ur.data(), uc.data());
            for(size_t q = 0; q < js.size(); q++){ b->res[js[q]] = ur[q]; b->rcs[js[q]] = uc[q]; }
        }
        for(int j : js){
            if(!b->rcs[j]) continue;
            std::lock_guard<std::mutex> lk(b->m);
            if(out_of_memory(sqb_error())) b->retry.push_back(j);
            else {
                b->failures++;
                if(b->err.empty()) b->err = std::string(b->jobs[j].graph) + ": " + sqb_error();
            }
        }
    }
    int rec = ok && cudaEventRecord(b->ends[id], s) == cudaSuccess;
    std::lock_guard<std::mutex> lk(b->m);
    b->ended[id] = rec;
    if(!err.empty()){ b->failures++; if(b->err.empty()) b->err = err; }
    if(--b->left == 0) b->cv.notify_all();
}

void worker(int id){
    unsigned long seen = 0;
    for(;;){
        Batch *b; int nw;
        {
            std::unique_lock<std::mutex> lk(PM);
            PCV.wait(lk, [&]{ return GEN != seen; });
            seen = GEN; b = CUR; nw = b ? b->nw : 0;     /* read under the lock: b outlives only its workers */
        }
        if(id < nw) serve(b, id);
    }
}

}  // namespace

extern "C" int sqb_hsum_batch(const sqb_job_t *jobs, int n, const sqb_opts_t *o_in, int workers,
                              sqb_result_t *res, int *rcs, double *device_ms){
    static std::mutex one;            /* one batch at a time */
    std::lock_guard<std::mutex> guard(one);
    if(device_ms) *device_ms = 0;
    if(n <= 0) return 0;
    sqb_opts_t o; if(o_in) o = *o_in; else sqb_default_opts(&o);
    if(workers < 1) workers = 1;
    if(workers > MAXW) workers = MAXW;
    if(workers > n) workers = n;
    if(sqb_dev_init(o.device)){ sqb_set_error_msg(sqb_last_error()); return -1; }
    for(int j = 0; j < n; j++){
        if(!sqb_find_graph(jobs[j].graph)){
            char m[256]; snprintf(m, sizeof m, "unknown graph %s", jobs[j].graph); sqb_set_error_msg(m); return -1;
        }
        rcs[j] = 0; memset(&res[j], 0, sizeof res[j]);
    }
    Batch b;
    b.jobs = jobs; b.n = n; b.nw = workers; b.o = o; b.res = res; b.rcs = rcs;
    std::vector<double> cost;
    if(o.group){
        /* the jobs of each graph in list order, SQB_GROUP_MAX at a time; a unit costs its jobs' sum */
        std::vector<std::string> names;
        for(int j = 0; j < n; j++){
            size_t u = 0;
            while(u < names.size() && (names[u] != jobs[j].graph || b.units[u].size() >= SQB_GROUP_MAX)) u++;
            if(u == names.size()){ names.push_back(jobs[j].graph); b.units.push_back({}); cost.push_back(0); }
            b.units[u].push_back(j); cost[u] += jobs[j].cost;
        }
    } else for(int j = 0; j < n; j++) cost.push_back(jobs[j].cost);
    const int nu = (int)cost.size();
    if(workers > nu) workers = nu;
    b.nw = workers; b.left = workers;
    b.order.resize(nu);
    for(int u = 0; u < nu; u++) b.order[u] = u;
    std::stable_sort(b.order.begin(), b.order.end(), [&](int x, int y){ return cost[x] > cost[y]; });
    b.ends.assign(workers, nullptr); b.ended.assign(workers, 0);
    cudaStream_t s = (cudaStream_t)sqb_dev_stream();
    int rc = 0;
    if(cudaEventCreate(&b.start) != cudaSuccess) rc = -1;
    for(int i = 0; i < workers && !rc; i++) if(cudaEventCreate(&b.ends[i]) != cudaSuccess) rc = -1;
    if(!rc && cudaEventRecord(b.start, s) != cudaSuccess) rc = -1;
    if(rc){
        sqb_set_error_msg("sqb_hsum_batch: event setup failed");
        if(b.start) cudaEventDestroy(b.start);
        for(cudaEvent_t e : b.ends) if(e) cudaEventDestroy(e);
        return -1;
    }
    {
        std::lock_guard<std::mutex> lk(PM);
        while(NSTARTED < workers){ std::thread(worker, NSTARTED).detach(); NSTARTED++; }
        CUR = &b; GEN++;
    }
    PCV.notify_all();
    {
        std::unique_lock<std::mutex> lk(b.m);
        b.cv.wait(lk, [&]{ return b.left == 0; });
    }
    { std::lock_guard<std::mutex> lk(PM); CUR = nullptr; }
    for(int i = 0; i < workers; i++) if(b.ended[i]) cudaStreamWaitEvent(s, b.ends[i], 0);
    if(!b.retry.empty()){
        /* alone on the device now: every worker has finished, and its memory is back in the pool */
        std::sort(b.retry.begin(), b.retry.end());
        cudaStreamSynchronize(s);
        for(int j : b.retry){
            const sqb_job_t &J = jobs[j];
            sqb_set_mem_share(1.0);
            rcs[j] = sqb_hsum(J.graph, J.h, J.N, J.eps, J.top, &o, &res[j]);
            if(rcs[j]){ b.failures++; if(b.err.empty()) b.err = std::string(J.graph) + ": " + sqb_error(); }
        }
    }
    cudaEvent_t stop = nullptr;
    if(cudaEventCreate(&stop) == cudaSuccess && cudaEventRecord(stop, s) == cudaSuccess && cudaEventSynchronize(stop) == cudaSuccess){
        float t = 0; cudaEventElapsedTime(&t, b.start, stop);
        if(device_ms) *device_ms = t;
    }
    if(stop) cudaEventDestroy(stop);
    cudaEventDestroy(b.start);
    for(cudaEvent_t e : b.ends) cudaEventDestroy(e);
    if(b.failures){ sqb_set_error_msg(b.err.c_str()); return b.failures; }
    return 0;
}

extern "C" int sqb_batch_tune(const sqb_job_t *jobs, int n, const sqb_opts_t *o, const int *cand, int ncand,
                              double *rate, int *best){
    *best = 0;
    std::vector<sqb_result_t> res(n > 0 ? n : 1);
    std::vector<int> rcs(n > 0 ? n : 1);
    for(int c = 0; c < ncand; c++) rate[c] = 0;
    for(int round = 0; round < 2; round++)
        for(int c = 0; c < ncand; c++){
            double ms = 0;
            int rc = sqb_hsum_batch(jobs, n, o, cand[c], res.data(), rcs.data(), &ms);
            if(rc) return rc;
            double ev = 0; for(int j = 0; j < n; j++) ev += (double)res[j].nev;
            const double r = ms > 0 ? ev/(ms*1e-3) : 0;
            if(r > rate[c]) rate[c] = r;
        }
    double top = -1;
    for(int c = 0; c < ncand; c++) if(rate[c] > top){ top = rate[c]; *best = cand[c]; }
    return 0;
}
